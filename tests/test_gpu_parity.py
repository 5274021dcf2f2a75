"""CUDA engine vs the CPU oracle, bit-exact, through the C ABI.

Each case codes a seeded synthetic image with the forward analysis, then
reconstructs it on the GPU (jxrb_decode_to_host / submissions) and in the
oracle, and compares every output byte and the error status."""
import numpy as np
import pytest

import jxr_b200 as J
from tests._bridge import decode_synth, oracle_decode

pytestmark = pytest.mark.gpu

C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA


@pytest.fixture(scope="module")
def session():
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    s = J.CudaDecoderSession(0)
    yield s
    s.close()


def rgb8(w, h, **kw):
    return J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], w, h, **kw)


def check(session, img, out, expect_ok=True):
    rc, ref = decode_synth(img, out)
    plan = J.CudaDecodePlan(img.arena, img.geometry, out, img.alpha_arena)
    if rc != 0:
        with pytest.raises(J.CudaError):
            session.decode_to_host(plan)
        assert not expect_ok, f"oracle failed with {rc}"
        return
    got = session.decode_to_host(plan)
    assert got.size == ref.size
    if not np.array_equal(got, ref):
        bad = np.nonzero(got != ref)[0]
        raise AssertionError(f"{bad.size} of {ref.size} bytes differ; first at {bad[:8]}: "
                             f"gpu {got[bad[:8]]} oracle {ref[bad[:8]]}")


@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("tiles", [(0, 0, 0), (4, 4, 1), (3, 2, 1), (5, 3, 0), (1, 1, 1)])
def test_rgb444(session, overlap, tiles):
    tw, th, hard = tiles
    img = J.synth(208, 176, quality=80, overlap=overlap, tile_width=tw, tile_height=th, hard_tiles=hard,
                  seed=11 + overlap)
    check(session, img, rgb8(208, 176))


@pytest.mark.parametrize("color", ["YUV420", "YUV422"])
@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("tiles", [(0, 0, 0), (2, 3, 1), (1, 1, 1), (3, 2, 0)])
def test_subsampled_chroma(session, color, overlap, tiles):
    tw, th, hard = tiles
    img = J.synth(160, 96, color_format=C_[color], quality=75, overlap=overlap, tile_width=tw, tile_height=th,
                  hard_tiles=hard, seed=5)
    check(session, img, rgb8(160, 96))


@pytest.mark.parametrize("centering", [(0, 0), (2, 2), (4, 1), (3, 4)])
def test_chroma_centering(session, centering):
    img = J.synth(96, 80, color_format=C_["YUV420"], quality=70, overlap=1, seed=2)
    img.geometry.chroma_centering_x, img.geometry.chroma_centering_y = centering
    check(session, img, rgb8(96, 80))


def test_planar_yuv420_native_output(session):
    img = J.synth(128, 96, color_format=C_["YUV420"], quality=75, overlap=2, tile_width=3, tile_height=2,
                  hard_tiles=1, seed=9)
    out = J.OutputFormat(C_["YUV420"], D["U8"], S["U8"], L["YUV"], 128, 96)
    check(session, img, out)


@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_gray16_lossless(session, overlap):
    img = J.synth(224, 192, content=J.CONTENT["GRAY16"], color_format=C_["LUMA"], quality=100, scaled=0,
                  overlap=overlap, tile_width=6, tile_height=5, hard_tiles=1, seed=4)
    out = J.OutputFormat(C_["LUMA"], D["U16"], S["U16"], L["LUMA"], 224, 192)
    check(session, img, out)


@pytest.mark.parametrize("layout", ["RGBA", "BGRA"])
@pytest.mark.parametrize("premultiply", [0, 1])
def test_rgba_integrated_alpha(session, layout, premultiply):
    img = J.synth(240, 208, alpha_mode=A["INTEGRATED"], quality=85, overlap=2, alpha_overlap=2, alpha_qp=(8, 8, 8),
                  tile_width=7, tile_height=6, hard_tiles=1, seed=6)
    out = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L[layout], 240, 208, alpha_bit_depth=D["U8"],
                         premultiply_alpha=premultiply)
    check(session, img, out)


def test_hdr_half_separate_alpha_f32_nchw(session):
    img = J.synth(208, 176, content=J.CONTENT["HDR_HALF"], alpha_mode=A["SEPARATE"], scaled=0, quality=0,
                  qp=(4, 8, 16), overlap=2, alpha_overlap=0, tile_width=5, tile_height=4, hard_tiles=0, seed=8)
    out = J.OutputFormat(C_["RGB"], D["F16"], S["F16"], L["RGBA"], 208, 176, alpha_bit_depth=D["F16"], nchw=1,
                         widen_f16=1)
    check(session, img, out)


@pytest.mark.parametrize("name,depth,storage,layout,extra", [
    ("u16", "U16", "U16", "RGB", dict(shift_bits=0)),
    ("u16s", "U16", "U16", "RGB", dict(shift_bits=3)),
    ("u10", "U10", "U16", "RGB", {}),
    ("i16", "I16", "I16", "BGR", dict(shift_bits=2)),
    ("i32", "I32", "I32", "RGBX", dict(shift_bits=4)),
    ("f16", "F16", "F16", "RGB", {}),
    ("f32", "F32", "F32", "RGB", dict(mantissa_length=13, exponent_bias=4)),
    ("rgb555", "RGB555", "RGB555", "RGB", {}),
    ("rgb565", "RGB565", "RGB565", "RGB", {}),
    ("rgb101010", "RGB101010", "RGB101010", "RGB", {}),
    ("bgrx", "U8", "U8", "BGRX", {}),
])
def test_output_formats(session, name, depth, storage, layout, extra):
    img = J.synth(160, 160, quality=60, overlap=1, seed=12)
    out = J.OutputFormat(C_["RGB"], D[depth], S[storage], L[layout], 160, 160, **extra)
    check(session, img, out)


def test_rgbe(session):
    img = J.synth(64, 48, quality=75, overlap=1, seed=13)
    out = J.OutputFormat(C_["RGBE"], D["U8"], S["RGBE"], L["RGB"], 64, 48)
    check(session, img, out)


@pytest.mark.parametrize("depth", ["BIT1_WHITE", "BIT1_BLACK"])
def test_bilevel(session, depth):
    img = J.synth(88, 40, color_format=C_["LUMA"], quality=40, overlap=1, seed=14)
    out = J.OutputFormat(C_["LUMA"], D[depth], S["BITS"], L["LUMA"], 85, 37, crop_x=3, crop_y=2)
    check(session, img, out)


@pytest.mark.parametrize("crop", [(0, 0, 100, 70), (5, 3, 90, 60), (17, 33, 31, 29), (63, 47, 1, 1),
                                  (70, 67, 130, 101), (1, 2, 191, 158)])
def test_crops(session, crop):
    x, y, w, h = crop
    img = J.synth(208, 176, quality=70, overlap=2, tile_width=20, tile_height=20, hard_tiles=0, seed=15)
    check(session, img, rgb8(w, h, crop_x=x, crop_y=y))


def test_window_of_macroblocks(session):
    # a region decode: reconstruct a window of whole tiles treated as a plane
    img = J.synth(160, 128, quality=75, overlap=2, tile_width=3, tile_height=2, hard_tiles=1, seed=16)
    g = img.geometry
    g.macroblock_origin_x, g.macroblock_origin_y, g.macroblocks_x, g.macroblocks_y = 3, 2, 6, 4
    check(session, img, rgb8(96, 64))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_bands_and_prediction(session, seed):
    # every macroblock draws its bands and high-pass direction
    img = J.synth(224, 208, content=J.CONTENT["RANDOM"], overlap=2, tile_width=5, tile_height=6, hard_tiles=1,
                  seed=seed)
    check(session, img, J.OutputFormat(C_["RGB"], D["I32"], S["I32"], L["RGB"], 224, 208))
    soft = J.synth(208, 176, content=J.CONTENT["RANDOM"], overlap=seed % 3, seed=seed + 3)
    check(session, soft, J.OutputFormat(C_["RGB"], D["I32"], S["I32"], L["RGB"], 208, 176))
    gray = J.synth(176, 160, content=J.CONTENT["RANDOM"], color_format=C_["LUMA"], overlap=2, seed=seed + 5)
    check(session, gray, J.OutputFormat(C_["LUMA"], D["I32"], S["I32"], L["LUMA"], 176, 160))
    img420 = J.synth(96, 80, content=J.CONTENT["RANDOM"], color_format=C_["YUV420"], overlap=2, seed=seed + 7)
    check(session, img420, J.OutputFormat(C_["RGB"], D["I32"], S["I32"], L["RGB"], 96, 80))


def test_overflow_is_reported_like_the_oracle(session):
    img = J.synth(64, 64, quality=75, overlap=2, seed=17)
    img.arena.coefficients[100:140] = 2**30
    check(session, img, rgb8(64, 64), expect_ok=False)


def test_odd_size_c1_shape(session):
    img = J.synth(512, 512, quality=75, overlap=1, seed=1)
    check(session, img, rgb8(512, 512))


def test_batch_matches_single(session):
    imgs = [J.synth(16 * (3 + i), 16 * (2 + 2 * i), quality=75, overlap=i % 3, seed=20 + i,
                    color_format=C_["YUV420"] if i % 2 else C_["YUV444"]) for i in range(5)]
    plans = [J.CudaDecodePlan(im.arena, im.geometry, rgb8(im.geometry.macroblocks_x * 16,
                                                          im.geometry.macroblocks_y * 16)) for im in imgs]
    sub = session.submit_batch(plans)
    sub.wait()
    for i, (im, p) in enumerate(zip(imgs, plans)):
        rc, ref = decode_synth(im, p.output)
        assert rc == 0
        assert np.array_equal(sub.readback(i), ref)


@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("color", ["YUV444", "YUV420"])
def test_large_interior_tiles(session, overlap, color):
    # images wide enough that most tiles take the interior path
    img = J.synth(400, 336, color_format=C_[color], quality=85, overlap=overlap, tile_width=8, tile_height=8,
                  hard_tiles=int(overlap == 1), seed=30 + overlap)
    check(session, img, rgb8(400, 336))
    check(session, img, J.OutputFormat(C_["RGB"], D["U16"], S["U16"], L["BGR"], 400, 336))


def test_interior_rgb8_unaligned_crop(session):
    img = J.synth(320, 320, quality=75, overlap=2, seed=41)
    check(session, img, rgb8(301, 297, crop_x=7, crop_y=5))


# 4:2:0 images wide enough for the 4:2:0 interior kernel (luma and both
# chroma planes of a tile in one CTA), against the oracle in every variant
# the kernel branches on: centering, overlap, hard tiles, output paths.
@pytest.mark.parametrize("centering", [(0, 0), (4, 1), (3, 4), (2, 0)])
@pytest.mark.parametrize("overlap", [1, 2])
def test_yuv420_interior_centering(session, centering, overlap):
    img = J.synth(336, 272, color_format=C_["YUV420"], quality=80, overlap=overlap, seed=50 + overlap)
    img.geometry.chroma_centering_x, img.geometry.chroma_centering_y = centering
    check(session, img, rgb8(336, 272))


@pytest.mark.parametrize("tiles", [(5, 4, 1), (6, 5, 0), (9, 7, 1), (1, 1, 1)])
def test_yuv420_interior_tiles(session, tiles):
    tw, th, hard = tiles
    img = J.synth(352, 304, color_format=C_["YUV420"], quality=70, overlap=2, tile_width=tw, tile_height=th,
                  hard_tiles=hard, seed=60 + tw)
    check(session, img, rgb8(352, 304))


@pytest.mark.parametrize("name,depth,storage,layout,extra", [
    ("bgr", "U8", "U8", "BGR", {}),
    ("rgbx", "U8", "U8", "RGBX", {}),
    ("bgrx", "U8", "U8", "BGRX", {}),
    ("i32", "I32", "I32", "RGB", dict(shift_bits=3)),
    ("f16_nchw", "F16", "F16", "RGB", dict(nchw=1, widen_f16=1)),
    ("f32", "F32", "F32", "RGB", dict(mantissa_length=13, exponent_bias=4)),
    ("rgb565", "RGB565", "RGB565", "RGB", {}),
    ("u16_nchw", "U16", "U16", "RGB", dict(nchw=1)),
])
def test_yuv420_interior_outputs(session, name, depth, storage, layout, extra):
    img = J.synth(320, 288, color_format=C_["YUV420"], quality=75, overlap=2, seed=70)
    check(session, img, J.OutputFormat(C_["RGB"], D[depth], S[storage], L[layout], 320, 288, **extra))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_yuv420_interior_random(session, seed):
    # every macroblock draws its bands and high-pass direction; values large
    # enough that some images overflow, reported with the oracle's stage
    img = J.synth(320, 272, content=J.CONTENT["RANDOM"], color_format=C_["YUV420"], overlap=seed % 3,
                  tile_width=6, tile_height=5, hard_tiles=seed % 2, seed=80 + seed)
    check(session, img, J.OutputFormat(C_["RGB"], D["I32"], S["I32"], L["RGB"], 320, 272), expect_ok=False)
    check(session, img, rgb8(320, 272), expect_ok=False)


def test_yuv420_interior_lossless_and_crop(session):
    img = J.synth(304, 288, color_format=C_["YUV420"], quality=100, scaled=0, overlap=1, seed=90)
    check(session, img, rgb8(304, 288))
    img = J.synth(336, 320, color_format=C_["YUV420"], quality=75, overlap=2, seed=91)
    check(session, img, rgb8(301, 283, crop_x=13, crop_y=9))
    check(session, img, rgb8(64, 64, crop_x=130, crop_y=150))


def test_yuv420_interior_overflow(session):
    img = J.synth(320, 288, color_format=C_["YUV420"], quality=75, overlap=2, seed=92)
    n = img.arena.coefficients.size
    img.arena.coefficients[n // 2:n // 2 + 64] = 2**30
    check(session, img, rgb8(320, 288), expect_ok=False)


# Tiles that touch the plane's edge (and no hard tile boundary) take the edge
# kernels: sizes with partial tiles, one-macroblock planes, crops along the
# edges, every output path and plane count.
@pytest.mark.parametrize("size", [(16, 16), (16, 80), (80, 16), (48, 112), (272, 208), (304, 176), (96, 96)])
@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_edge_tiles_sizes(session, size, overlap):
    w, h = size
    img = J.synth(w, h, quality=80, overlap=overlap, seed=100 + w + h + overlap)
    check(session, img, rgb8(w, h))


@pytest.mark.parametrize("crop", [(0, 0, 7, 5), (1, 1, 270, 206), (265, 0, 7, 208), (0, 203, 272, 5), (2, 3, 9, 9)])
def test_edge_tiles_crops(session, crop):
    x, y, w, h = crop
    img = J.synth(272, 208, quality=75, overlap=2, seed=110)
    check(session, img, rgb8(w, h, crop_x=x, crop_y=y))


@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_edge_tiles_planes(session, overlap):
    gray = J.synth(208, 144, content=J.CONTENT["GRAY16"], color_format=C_["LUMA"], quality=100, scaled=0,
                   overlap=overlap, seed=120 + overlap)
    check(session, gray, J.OutputFormat(C_["LUMA"], D["U16"], S["U16"], L["LUMA"], 208, 144))
    rgba = J.synth(176, 240, alpha_mode=A["INTEGRATED"], quality=85, overlap=overlap, alpha_overlap=2 - overlap,
                   alpha_qp=(8, 8, 8), seed=121 + overlap)
    check(session, rgba, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGBA"], 176, 240, alpha_bit_depth=D["U8"]))
    check(session, rgba, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["BGRA"], 176, 240, alpha_bit_depth=D["U8"],
                                        premultiply_alpha=1))
    hdr = J.synth(144, 208, content=J.CONTENT["HDR_HALF"], alpha_mode=A["SEPARATE"], scaled=0, quality=0,
                  qp=(4, 8, 16), overlap=overlap, alpha_overlap=overlap, seed=122 + overlap)
    check(session, hdr, J.OutputFormat(C_["RGB"], D["F16"], S["F16"], L["RGBA"], 144, 208, alpha_bit_depth=D["F16"],
                                       nchw=1, widen_f16=1))
    two = J.synth(160, 112, content=J.CONTENT["RANDOM"], overlap=overlap, seed=123 + overlap)
    check(session, two, J.OutputFormat(C_["RGB"], D["I32"], S["I32"], L["RGB"], 160, 112), expect_ok=False)


@pytest.mark.parametrize("tiles", [(2, 2, 1), (5, 3, 1), (7, 6, 1), (3, 9, 1)])
def test_edge_tiles_with_hard_tiles(session, tiles):
    # edge tiles beside hard tile boundaries take the general kernel, the rest
    # the edge kernel
    tw, th, hard = tiles
    img = J.synth(336, 304, quality=80, overlap=2, tile_width=tw, tile_height=th, hard_tiles=hard, seed=130 + tw)
    check(session, img, rgb8(336, 304))


def test_edge_tiles_overflow(session):
    img = J.synth(208, 176, quality=75, overlap=2, seed=140)
    img.arena.coefficients[:64] = 2**30
    check(session, img, rgb8(208, 176), expect_ok=False)


# 4:2:0 tiles at the plane's edge take the 4:2:0 edge kernel (planes of at
# least 2 x 2 macroblocks): first-level chroma pairs and corner residuals,
# cut chroma and luma cells, chroma reads clamped at the plane's edge.
@pytest.mark.parametrize("size", [(32, 32), (48, 32), (32, 80), (96, 64), (208, 144), (16, 48)])
@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_yuv420_edge_sizes(session, size, overlap):
    w, h = size
    img = J.synth(w, h, color_format=C_["YUV420"], quality=80, overlap=overlap, seed=150 + w + h + overlap)
    check(session, img, rgb8(w, h))


@pytest.mark.parametrize("centering", [(0, 0), (4, 4), (1, 3), (2, 1)])
def test_yuv420_edge_centering_and_crops(session, centering):
    img = J.synth(176, 112, color_format=C_["YUV420"], quality=75, overlap=2, seed=160)
    img.geometry.chroma_centering_x, img.geometry.chroma_centering_y = centering
    check(session, img, rgb8(176, 112))
    check(session, img, rgb8(5, 111, crop_x=171, crop_y=1))
    check(session, img, rgb8(175, 3, crop_x=0, crop_y=109))


@pytest.mark.parametrize("seed", [1, 2])
def test_yuv420_edge_random_and_outputs(session, seed):
    img = J.synth(144, 96, content=J.CONTENT["RANDOM"], color_format=C_["YUV420"], overlap=2, seed=170 + seed)
    check(session, img, J.OutputFormat(C_["RGB"], D["I32"], S["I32"], L["RGB"], 144, 96), expect_ok=False)
    img = J.synth(112, 80, color_format=C_["YUV420"], quality=70, overlap=seed, seed=172 + seed)
    check(session, img, J.OutputFormat(C_["RGB"], D["F16"], S["F16"], L["RGB"], 112, 80, nchw=1, widen_f16=1))
    check(session, img, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["BGRX"], 112, 80))


# YUVK images (four colour planes) to CMYK: the interior and edge kernels of
# four full-resolution planes without alpha, the colour conversion to CMYK
# and its direct form, interleaved and NCHW; with alpha (five planes) and
# hard tiles, the general kernel.
@pytest.mark.parametrize("name,output,depth,extra", [
    ("cmyk_u8", "CMYK", "U8", {}),
    ("cmyk_direct", "CMYK_DIRECT", "U8", {}),
    ("cmyk_u16", "CMYK", "U16", {}),
    ("cmyk_nchw", "CMYK", "U8", dict(nchw=1)),
])
def test_yuvk_to_cmyk(session, name, output, depth, extra):
    img = J.synth(336, 272, color_format=C_["YUVK"], quality=80, overlap=2, seed=5)
    check(session, img, J.OutputFormat(C_[output], D[depth], S[depth], L["CMYK"], 336, 272, **extra))


def test_yuvk_with_alpha_and_hard_tiles(session):
    img = J.synth(176, 144, color_format=C_["YUVK"], alpha_mode=A["INTEGRATED"], quality=80, overlap=1,
                  alpha_overlap=1, alpha_qp=(8, 8, 8), seed=6)
    check(session, img, J.OutputFormat(C_["CMYK"], D["U8"], S["U8"], L["CMYKA"], 176, 144, alpha_bit_depth=D["U8"]))
    img = J.synth(208, 176, color_format=C_["YUVK"], quality=70, overlap=1, tile_width=5, tile_height=4,
                  hard_tiles=1, seed=7)
    check(session, img, J.OutputFormat(C_["CMYK"], D["U8"], S["U8"], L["CMYK"], 208, 176))


# Grayscale with alpha (two planes: the two-plane interior and edge kernels),
# integrated and separate, premultiplied; N-component images stored directly.
@pytest.mark.parametrize("depth,premultiply", [("U8", 0), ("U16", 0), ("U8", 1)])
def test_luma_alpha(session, depth, premultiply):
    img = J.synth(336, 272, color_format=C_["LUMA"], alpha_mode=A["INTEGRATED"], quality=80, overlap=2,
                  alpha_overlap=1, alpha_qp=(8, 8, 8), seed=8)
    check(session, img, J.OutputFormat(C_["LUMA"], D[depth], S[depth], L["LUMA_ALPHA"], 336, 272,
                                       alpha_bit_depth=D[depth], premultiply_alpha=premultiply))


def test_luma_separate_alpha(session):
    img = J.synth(208, 176, color_format=C_["LUMA"], alpha_mode=A["SEPARATE"], quality=80, overlap=1,
                  alpha_overlap=2, alpha_qp=(4, 4, 4), seed=9)
    check(session, img, J.OutputFormat(C_["LUMA"], D["U8"], S["U8"], L["LUMA_ALPHA"], 208, 176,
                                       alpha_bit_depth=D["U8"]))


@pytest.mark.parametrize("depth", ["U8", "U16"])
def test_ncomponent(session, depth):
    img = J.synth(336, 272, color_format=C_["NCOMPONENT"], quality=80, overlap=2, seed=10)
    check(session, img, J.OutputFormat(C_["NCOMPONENT"], D[depth], S[depth], L["NCOMPONENT"], 336, 272))


# Planar 4:2:2 / 4:2:0 native outputs (crop included) and premultiplied
# alpha in 16-bit integers and half floats.
def test_planar_native_outputs(session):
    img = J.synth(176, 112, color_format=C_["YUV422"], quality=75, overlap=2, tile_width=3, tile_height=2,
                  hard_tiles=1, seed=11)
    check(session, img, J.OutputFormat(C_["YUV422"], D["U8"], S["U8"], L["YUV"], 176, 112))
    check(session, img, J.OutputFormat(C_["YUV422"], D["U8"], S["U8"], L["YUV"], 170, 100, crop_x=2, crop_y=5))
    img = J.synth(128, 96, color_format=C_["YUV420"], quality=75, overlap=1, seed=12)
    check(session, img, J.OutputFormat(C_["YUV420"], D["U16"], S["U16"], L["YUV"], 128, 96))


def test_premultiplied_u16_and_half(session):
    img = J.synth(240, 208, alpha_mode=A["INTEGRATED"], quality=85, overlap=2, alpha_overlap=2, alpha_qp=(8, 8, 8),
                  seed=13)
    check(session, img, J.OutputFormat(C_["RGB"], D["U16"], S["U16"], L["RGBA"], 240, 208, alpha_bit_depth=D["U16"],
                                       premultiply_alpha=1))
    img = J.synth(208, 176, content=J.CONTENT["HDR_HALF"], alpha_mode=A["SEPARATE"], scaled=0, quality=0,
                  qp=(4, 8, 16), overlap=2, alpha_overlap=0, seed=14)
    check(session, img, J.OutputFormat(C_["RGB"], D["F16"], S["F16"], L["RGBA"], 208, 176, alpha_bit_depth=D["F16"],
                                       premultiply_alpha=1))


def test_readback_all_matches_per_image_readback(session):
    imgs = [J.synth(16 * (3 + i), 16 * (2 + i), quality=75, overlap=i % 3, seed=40 + i,
                    color_format=C_["YUV420"] if i % 2 else C_["YUV444"]) for i in range(5)]
    plans = [J.CudaDecodePlan(im.arena, im.geometry, rgb8(im.geometry.macroblocks_x * 16 - 3,
                                                          im.geometry.macroblocks_y * 16 - 1)) for im in imgs]
    sub = session.submit_batch(plans)
    sub.wait()
    offs = sub.output_offsets()
    total = offs[-1] + plans[-1].output_bytes()
    host = np.full(total, 0xA5, np.uint8)
    sub.readback_all(host.ctypes.data, total)
    for i, p in enumerate(plans):
        assert np.array_equal(host[offs[i]:offs[i] + p.output_bytes()], sub.readback(i))
    with pytest.raises(J.CudaError):
        sub.readback_all(host.ctypes.data, total + (1 << 20))
    sub.close()
