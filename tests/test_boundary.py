"""Boundary entries that need no GPU: route planning (plan_cuda_route,
crates/jxr-cuda/src/route.rs:23-49, and its tests), output surface layouts
(SurfaceLayout, crates/jxr-core/src/surface.rs) and the dense batch layout."""
import numpy as np
import pytest

import jxr_b200 as J
from jxr_b200 import api

C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA
B = api.BACKEND


def route(*args):
    try:
        return api.plan_cuda_route(*args)
    except J.CudaError as e:
        return e.kind


def test_explicit_cuda_is_strict_and_auto_needs_the_threshold():
    assert route(B["CUDA"], 0, True, False) == "Cuda"
    assert route(B["CUDA"], 1 << 30, False, False) == "Unavailable"
    assert route(B["AUTO"], 16383, True, False) == "Cpu"
    assert route(B["AUTO"], 16384, True, False) == "Cuda"
    assert route(B["AUTO"], 1 << 30, False, False) == "Cpu"
    assert route(B["CPU"], 1 << 30, True, False) == "Cpu"
    assert route(B["METAL"], 1 << 30, True, False) == "UnsupportedBackend"


def test_resident_output_needs_cuda():
    assert route(B["CPU"], 0, True, True) == "ResidentOutputRequiresCuda"
    assert route(B["AUTO"], 0, True, True) == "Cuda"
    assert route(B["AUTO"], 0, False, True) == "Unavailable"
    assert route(B["CUDA"], 0, True, True) == "Cuda"
    assert route(B["METAL"], 0, True, True) == "UnsupportedBackend"


def test_reconstructed_coefficients_count_every_plane_sample():
    img = J.synth(64, 48, color_format=C_["YUV420"], quality=75, overlap=1, seed=2, threads=1)
    p = J.CudaDecodePlan(img.arena, img.geometry, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 64, 48))
    assert p.reconstructed_coefficients() == 64 * 48 + 2 * 32 * 24


@pytest.mark.parametrize("case", ["rgb8", "nchw_f32", "yuv420_planar", "bits", "rgba_u16"])
def test_output_layouts(case):
    if case == "yuv420_planar":
        img = J.synth(48, 32, color_format=C_["YUV420"], quality=75, overlap=1, seed=3, threads=1)
        out = J.OutputFormat(C_["YUV420"], D["U8"], S["U8"], L["YUV"], 46, 30)
    elif case == "bits":
        img = J.synth(40, 24, color_format=C_["LUMA"], quality=40, overlap=1, seed=4, threads=1)
        out = J.OutputFormat(C_["LUMA"], D["BIT1_BLACK"], S["BITS"], L["LUMA"], 37, 21)
    elif case == "rgba_u16":
        img = J.synth(32, 32, alpha_mode=A["INTEGRATED"], alpha_qp=(8, 8, 8), quality=80, overlap=1, seed=5,
                      threads=1)
        out = J.OutputFormat(C_["RGB"], D["U16"], S["U16"], L["RGBA"], 32, 32, alpha_bit_depth=D["U16"])
    else:
        img = J.synth(32, 32, quality=80, overlap=1, seed=6, threads=1)
        out = (J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 30, 29) if case == "rgb8" else
               J.OutputFormat(C_["RGB"], D["F32"], S["F32"], L["RGB"], 32, 32, nchw=1))
    p = J.CudaDecodePlan(img.arena, img.geometry, out)
    lay = p.output_layout()
    assert lay["byte_len"] == p.output_bytes()
    assert (lay["width"], lay["height"]) == (out.crop_width, out.crop_height)
    planes = lay["planes"]
    # every plane inside the surface, the last one ending at its end
    end = max(q["byte_offset"] + q["row_stride_bytes"] * q["height"] for q in planes)
    assert end == lay["byte_len"]
    if case == "rgb8":
        assert planes == [dict(byte_offset=0, row_stride_bytes=90, width=30, height=29, channels=3)]
    if case == "nchw_f32":
        assert [q["byte_offset"] for q in planes] == [0, 32 * 32 * 4, 2 * 32 * 32 * 4]
    if case == "yuv420_planar":
        assert [(q["width"], q["height"]) for q in planes] == [(46, 30), (23, 15), (23, 15)]
    if case == "bits":
        assert planes[0]["row_stride_bytes"] == 5
    if case == "rgba_u16":
        assert planes[0]["channels"] == 4 and lay["element_bytes"] == 2


def test_dense_batch_layout_aligns_each_image():
    imgs = [J.synth(w, h, quality=80, overlap=1, seed=w, threads=1) for w, h in [(16, 16), (48, 32), (32, 16)]]
    plans = [J.CudaDecodePlan(i.arena, i.geometry, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 16 * i.geometry.macroblocks_x,
                                                                   16 * i.geometry.macroblocks_y)) for i in imgs]
    offs, total = api.batch_layout(plans)
    assert offs[0] == 0 and all(o % 256 == 0 for o in offs)
    for a, b, p in zip(offs, offs[1:], plans):
        assert b >= a + p.output_bytes()
    assert total == offs[-1] + plans[-1].output_bytes()
