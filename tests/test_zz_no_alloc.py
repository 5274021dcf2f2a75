"""jxrb_decode_static, the entry point that allocates nothing, against the
oracle and against jxrb_decode_to_host on the same plans.

The descriptors live in the library's fixed device scratch; the coefficients
and the output are device buffers the test owns.  Outputs are integer bytes,
so the tolerance is zero: every byte must match.  Two calls run back to back
to show that the scratch (status word and scheduling counters included) is
reset between calls."""
import ctypes as C
import os

import numpy as np
import pytest

import jxr_b200 as J
from tests._bridge import decode_synth

pytestmark = pytest.mark.gpu

C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA


@pytest.fixture(scope="module")
def session():
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    s = J.CudaDecoderSession(0)
    yield s
    s.close()


def device_copy(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def decode_static(plan, coeff, alpha=None, fill=0xA5):
    """One call through the C ABI into a device buffer pre-filled with `fill`."""
    import torch
    n = plan.output_bytes()
    n4 = (n + 3) // 4 * 4
    out = torch.full((n4,), fill, dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()
    st = J.lib().jxrb_decode_static(0, plan.handle, C.c_void_p(coeff.data_ptr()),
                                    C.c_void_p(alpha.data_ptr()) if alpha is not None else None,
                                    C.c_void_p(out.data_ptr()), n4, None)
    J.api._check(st)
    return out[:n].cpu().numpy()


def cases():
    rgb = J.synth(400, 336, quality=85, overlap=2, tile_width=8, tile_height=8, seed=71)
    yield "rgb8_interior", rgb, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 400, 336)
    sub = J.synth(160, 96, color_format=C_["YUV420"], quality=75, overlap=1, tile_width=2, tile_height=3,
                  hard_tiles=1, seed=72)
    yield "yuv420_hard", sub, J.OutputFormat(C_["RGB"], D["U16"], S["U16"], L["BGR"], 150, 90, crop_x=3,
                                             crop_y=2)
    hdr = J.synth(208, 176, content=J.CONTENT["HDR_HALF"], alpha_mode=A["SEPARATE"], scaled=0, quality=0,
                  qp=(4, 8, 16), overlap=2, alpha_overlap=0, tile_width=5, tile_height=4, seed=73)
    yield "half_alpha_f32_nchw", hdr, J.OutputFormat(C_["RGB"], D["F16"], S["F16"], L["RGBA"], 208, 176,
                                                     alpha_bit_depth=D["F16"], nchw=1, widen_f16=1)
    bits = J.synth(88, 40, color_format=C_["LUMA"], quality=40, overlap=1, seed=74)
    yield "bilevel", bits, J.OutputFormat(C_["LUMA"], D["BIT1_BLACK"], S["BITS"], L["LUMA"], 85, 37)
    wide = J.synth(352, 288, color_format=C_["YUV420"], quality=80, overlap=2, tile_width=6, tile_height=5,
                   hard_tiles=1, seed=75)
    yield "yuv420_interior", wide, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 352, 288)


@pytest.mark.parametrize("name", ["rgb8_interior", "yuv420_hard", "half_alpha_f32_nchw", "bilevel",
                                  "yuv420_interior"])
def test_matches_decode_to_host_twice(session, name):
    img, out = next((i, o) for n, i, o in cases() if n == name)
    plan = J.CudaDecodePlan(img.arena, img.geometry, out, img.alpha_arena)
    rc, want = decode_synth(img, out, threads=os.cpu_count() or 1)
    assert rc == 0
    coeff = device_copy(img.arena.coefficients)
    alpha = device_copy(img.alpha_arena.coefficients) if img.alpha_arena is not None else None
    first = decode_static(plan, coeff, alpha, fill=0xA5)
    second = decode_static(plan, coeff, alpha, fill=0x5A)
    assert np.array_equal(first, want)
    assert np.array_equal(second, want)
    assert np.array_equal(session.decode_to_host(plan), want)


def test_two_plans_in_a_row(session):
    imgs = [(i, o) for _, i, o in cases()][:2]
    plans = [J.CudaDecodePlan(i.arena, i.geometry, o, i.alpha_arena) for i, o in imgs]
    wants = [session.decode_to_host(p) for p in plans]
    coeffs = [device_copy(i.arena.coefficients) for i, _ in imgs]
    for _ in range(2):
        for p, c, w in zip(plans, coeffs, wants):
            assert np.array_equal(decode_static(p, c), w)


def test_overflow_status_like_decode_to_host(session):
    img = J.synth(64, 64, quality=75, overlap=2, seed=17)
    img.arena.coefficients[100:140] = 2**30
    plan = J.CudaDecodePlan(img.arena, img.geometry, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 64, 64))
    with pytest.raises(J.CudaError) as ref:
        session.decode_to_host(plan)
    with pytest.raises(J.CudaError) as got:
        decode_static(plan, device_copy(img.arena.coefficients))
    assert (got.value.status, got.value.stage) == (ref.value.status, ref.value.stage)
    # the next call starts from a clean status word
    ok = J.synth(64, 64, quality=75, overlap=2, seed=18)
    p2 = J.CudaDecodePlan(ok.arena, ok.geometry, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 64, 64))
    assert np.array_equal(decode_static(p2, device_copy(ok.arena.coefficients)), session.decode_to_host(p2))


def dc_only_plan(mx, my, seed=0):
    """A three-plane DC-only plan of mx x my macroblocks (one coefficient a
    macroblock a plane), random DC values, unit quantizers, no overlap."""
    n = mx * my
    y, x = np.divmod(np.arange(n, dtype=np.uint32), mx)
    rng = np.random.default_rng(seed)
    arena = J.Arena(coefficients=rng.integers(-2000, 2000, 3 * n, dtype=np.int32),
                    coefficient_offsets=np.arange(3 * n, dtype=np.uint32),
                    quantizers=np.ones((3 * n, 3), np.uint32), bands=np.zeros(3 * n, np.uint8),
                    hp_predictions=np.zeros(3 * n, np.uint8), coded_x=np.tile(x, 3), coded_y=np.tile(y, 3),
                    planes=np.array([[k * n, n, k * n, n, 4, 4] for k in range(3)], np.uint64))
    geom = J.Geometry(mx, my, color_format=C_["YUV444"], overlap=0)
    out = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 16 * mx, 16 * my)
    return arena, geom, out


def test_4096_square_three_planes_fits_the_scratch(session):
    # the documented size: 256 x 256 macroblocks, three planes
    arena, geom, out = dc_only_plan(256, 256, seed=5)
    plan = J.CudaDecodePlan(arena, geom, out)
    coeff = device_copy(arena.coefficients)
    want = session.decode_to_host(plan)
    assert np.array_equal(decode_static(plan, coeff, fill=0x11), want)
    assert np.array_equal(decode_static(plan, coeff, fill=0xEE), want)


def test_plan_above_scratch_limit_is_refused(session):
    # 300 x 300 macroblocks, three DC-only planes: 16 bytes a macroblock a
    # plane is 4,320,000 bytes of tables, above the 4 MiB scratch
    arena, geom, out = dc_only_plan(300, 300)
    plan = J.CudaDecodePlan(arena, geom, out)
    coeff = device_copy(arena.coefficients)
    with pytest.raises(J.CudaError) as err:
        decode_static(plan, coeff)
    assert err.value.status == 10                       # JXRB_RESOURCE_LIMIT
    assert "4194304" in str(err.value)
