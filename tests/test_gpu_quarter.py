"""Reduced-resolution requests (a quarter and a sixteenth) on resident
images against the oracle's reduced reconstruction, byte for byte: whole
images and regions, every overlap mode, subsampled chroma, hard tiles and
alpha."""
import dataclasses

import numpy as np
import pytest

import jxr_b200 as J
from tests._bridge import oracle_decode
from tests.test_gpu_requests import expected_window

pytestmark = pytest.mark.gpu

C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA


@pytest.fixture(scope="module")
def session():
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    s = J.CudaDecoderSession(0)
    yield s
    s.close()


IMAGES = {
    "rgb444_o0": dict(width=208, height=176, quality=80, overlap=0, seed=61),
    "rgb444_o1_hard": dict(width=240, height=208, quality=80, overlap=1, tile_width=5, tile_height=4, hard_tiles=1,
                           seed=62),
    "rgb444_o2_soft": dict(width=400, height=336, quality=85, overlap=2, tile_width=8, tile_height=7, seed=63),
    "rgb444_o2_hard": dict(width=272, height=224, quality=70, overlap=2, tile_width=3, tile_height=6, hard_tiles=1,
                           seed=64),
    "rgb420_o1": dict(width=320, height=256, color_format=C_["YUV420"], quality=75, overlap=1, seed=65),
    "rgb420_o2_hard": dict(width=288, height=224, color_format=C_["YUV420"], quality=75, overlap=2, tile_width=4,
                           tile_height=5, hard_tiles=1, seed=66),
    "rgb422_o2": dict(width=256, height=192, color_format=C_["YUV422"], quality=70, overlap=2, tile_width=6,
                      tile_height=4, seed=67),
    "rgba_o2": dict(width=240, height=208, alpha_mode=A["INTEGRATED"], quality=85, overlap=2, alpha_overlap=2,
                    alpha_qp=(8, 8, 8), tile_width=7, tile_height=6, hard_tiles=1, seed=68),
}


@pytest.fixture(scope="module")
def images():
    return {k: J.synth(**v) for k, v in IMAGES.items()}


def fmt(name, w, h, x=0, y=0):
    if name.startswith("rgba"):
        return J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGBA"], w, h, crop_x=x, crop_y=y,
                              alpha_bit_depth=D["U8"])
    return J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], w, h, crop_x=x, crop_y=y)


def oracle_quarter(img, out, d=4):
    ox, oy, wx, wy = expected_window(img.geometry, out, d)
    g = dataclasses.replace(img.geometry, macroblock_origin_x=ox, macroblock_origin_y=oy, macroblocks_x=wx,
                            macroblocks_y=wy)
    x0, y0 = out.crop_x // d, out.crop_y // d
    x1, y1 = -(-(out.crop_x + out.crop_width) // d), -(-(out.crop_y + out.crop_height) // d)
    o = dataclasses.replace(out, crop_x=x0 - 16 // d * ox, crop_y=y0 - 16 // d * oy, crop_width=x1 - x0,
                            crop_height=y1 - y0)
    return oracle_decode(img.arena, g, o, img.alpha_arena, threads=8, denominator=d)


def run(session, reqs):
    sub = session.submit_requests(reqs)
    sub.wait()
    outs = [sub.readback(i) for i in range(len(reqs))]
    sub.close()
    return outs


@pytest.mark.parametrize("d", [4, 16])
@pytest.mark.parametrize("name", list(IMAGES))
def test_reduced_whole_image_and_regions(session, images, name, d):
    img = images[name]
    W, H = IMAGES[name]["width"], IMAGES[name]["height"]
    rimg = session.upload(img.arena, img.geometry, img.alpha_arena)
    rng = np.random.default_rng(sum(name.encode()) + d)
    regions = [(0, 0, W, H), (5, 3, 37, 29), (W - 41, H - 19, 41, 19)]
    for _ in range(4):
        w, h = int(rng.integers(4, W // 2)), int(rng.integers(4, H // 2))
        regions.append((int(rng.integers(0, W - w + 1)), int(rng.integers(0, H - h + 1)), w, h))
    outs = [fmt(name, w, h, x, y) for x, y, w, h in regions]
    reqs = [rimg.request(o, d) for o in outs]
    got = run(session, reqs)
    for region, o, g in zip(regions, outs, got):
        rc, ref = oracle_quarter(img, o, d)
        assert rc == 0, region
        assert g.size == ref.size and np.array_equal(g, ref), region


def test_reduced_and_full_requests_in_one_launch(session, images):
    residents = {k: session.upload(v.arena, v.geometry, v.alpha_arena) for k, v in images.items()}
    reqs, refs = [], []
    for k, name in enumerate(IMAGES):
        W, H = IMAGES[name]["width"], IMAGES[name]["height"]
        o = fmt(name, W, H)
        d = (4, 1, 16)[k % 3]
        reqs.append(residents[name].request(o, d))
        refs.append(oracle_quarter(images[name], o, d) if d > 1 else
                    oracle_decode(images[name].arena, images[name].geometry, o, images[name].alpha_arena, 8))
    for g, (rc, ref) in zip(run(session, reqs), refs):
        assert rc == 0 and np.array_equal(g, ref)


def test_quarter_needs_the_low_pass_band(session):
    img = J.synth(96, 80, content=J.CONTENT["RANDOM"], overlap=1, seed=5)
    assert (img.arena.bands == 0).any()
    rimg = session.upload(img.arena, img.geometry)
    with pytest.raises(J.CudaError) as err:
        rimg.request(fmt("rgb", 96, 80), 4)
    assert err.value.status == 6


def test_sixteenth_needs_no_low_pass_band(session):
    img = J.synth(96, 80, content=J.CONTENT["RANDOM"], overlap=2, seed=5)
    assert (img.arena.bands == 0).any()
    rimg = session.upload(img.arena, img.geometry)
    o = fmt("rgb", 96, 80)
    got = run(session, [rimg.request(o, 16)])[0]
    rc, ref = oracle_quarter(img, o, 16)
    assert rc == 0 and np.array_equal(got, ref)


def test_sixteenth_refuses_subsampled_planar_output(session):
    img = J.synth(64, 48, color_format=C_["YUV420"], quality=75, overlap=1, seed=6)
    rimg = session.upload(img.arena, img.geometry)
    with pytest.raises(J.CudaError) as err:
        rimg.request(J.OutputFormat(C_["YUV420"], D["U8"], S["U8"], L["YUV"], 64, 48), 16)
    assert err.value.status == 6 and "sixteenth" in str(err.value)
