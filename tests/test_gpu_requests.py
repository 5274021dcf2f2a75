"""Resident images and requests: full and region decodes through
jxrb_submit_requests against the oracle, and the region rule's property that
a region decode stores exactly the pixels of the full decode inside it."""
import dataclasses

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


def expected_window(geom, out, denominator=1):
    """reconstruction_bounds (crates/jxr-native/src/prepare.rs:321-352) and the
    window of the required tiles (decode/reconstruction.rs:509-546), restated;
    a sixteenth interpolates no chroma (metadata.rs:255-263)."""
    subsampled = geom.color_format in (C_["YUV420"], C_["YUV422"])
    interp = subsampled and out.output_color not in (C_["YUV420"], C_["YUV422"]) and denominator != 16
    halo = 1 if (geom.overlap or interp) else 0
    x, y, w, h = out.crop_x, out.crop_y, out.crop_width, out.crop_height
    b = [max(0, x // 16 - halo), max(0, y // 16 - halo), min(-(-(x + w) // 16) + halo, geom.macroblocks_x),
         min(-(-(y + h) // 16) + halo, geom.macroblocks_y)]

    def span(sizes, lo, hi):
        pos, s, e = 0, None, 0
        for size in sizes:
            if pos < hi and pos + size > lo:
                s = pos if s is None else min(s, pos)
                e = max(e, pos + size)
            pos += size
        return s, e - s

    ox, wx = span(geom.tile_column_widths or [geom.macroblocks_x], b[0], b[2])
    oy, wy = span(geom.tile_row_heights or [geom.macroblocks_y], b[1], b[3])
    return ox, oy, wx, wy


def oracle_region(img, out):
    ox, oy, wx, wy = expected_window(img.geometry, out)
    g = dataclasses.replace(img.geometry, macroblock_origin_x=ox, macroblock_origin_y=oy, macroblocks_x=wx,
                            macroblocks_y=wy)
    o = dataclasses.replace(out, crop_x=out.crop_x - 16 * ox, crop_y=out.crop_y - 16 * oy)
    return oracle_decode(img.arena, g, o, img.alpha_arena, threads=8)


def run(session, reqs):
    sub = session.submit_requests(reqs)
    sub.wait()
    outs = [sub.readback(i) for i in range(len(reqs))]
    sub.close()
    return outs


IMAGES = {
    "rgb444_soft_o2": dict(width=400, height=336, quality=85, overlap=2, tile_width=8, tile_height=7, seed=51),
    "rgb420_hard_o1": dict(width=352, height=288, color_format=C_["YUV420"], quality=75, overlap=1, tile_width=5,
                           tile_height=6, hard_tiles=1, seed=52),
    "rgb422_soft_o2": dict(width=288, height=224, color_format=C_["YUV422"], quality=70, overlap=2, tile_width=6,
                           tile_height=4, seed=53),
    "gray16_o0": dict(width=320, height=272, content=J.CONTENT["GRAY16"], color_format=C_["LUMA"], quality=100,
                      scaled=0, overlap=0, tile_width=7, tile_height=5, seed=54),
}


@pytest.fixture(scope="module")
def images():
    return {k: J.synth(**v) for k, v in IMAGES.items()}


def fmt(name, w, h, x=0, y=0):
    if name.startswith("gray"):
        return J.OutputFormat(C_["LUMA"], D["U16"], S["U16"], L["LUMA"], w, h, crop_x=x, crop_y=y)
    return J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], w, h, crop_x=x, crop_y=y)


@pytest.mark.parametrize("name", list(IMAGES))
def test_full_request_matches_plan(session, images, name):
    img = images[name]
    W, H = IMAGES[name]["width"], IMAGES[name]["height"]
    out = fmt(name, W, H)
    rimg = session.upload(img.arena, img.geometry, img.alpha_arena)
    req = rimg.request(out)
    assert req.window() == (0, 0, img.geometry.macroblocks_x, img.geometry.macroblocks_y)
    got, = run(session, [req])
    rc, ref = decode_synth(img, out, threads=8)
    assert rc == 0 and np.array_equal(got, ref)


@pytest.mark.parametrize("name", list(IMAGES))
def test_regions_match_oracle_and_full_decode(session, images, name):
    img = images[name]
    W, H = IMAGES[name]["width"], IMAGES[name]["height"]
    full_out = fmt(name, W, H)
    rc, full = decode_synth(img, full_out, threads=8)
    assert rc == 0
    ch, eb = (1, 2) if name.startswith("gray") else (3, 1)
    full = full.reshape(H, W, ch * eb)
    rng = np.random.default_rng(sum(name.encode()))
    rimg = session.upload(img.arena, img.geometry, img.alpha_arena)
    regions = [(0, 0, W, H), (0, 0, 17, 9), (W - 31, H - 23, 31, 23), (100, 64, 1, 1)]
    for _ in range(6):
        w, h = int(rng.integers(1, W // 2)), int(rng.integers(1, H // 2))
        regions.append((int(rng.integers(0, W - w + 1)), int(rng.integers(0, H - h + 1)), w, h))
    reqs, outs = [], []
    for x, y, w, h in regions:
        o = fmt(name, w, h, x, y)
        r = rimg.request(o)
        assert r.window() == expected_window(img.geometry, o)
        reqs.append(r)
        outs.append(o)
    got = run(session, reqs)
    for (x, y, w, h), o, g in zip(regions, outs, got):
        rc, ref = oracle_region(img, o)
        assert rc == 0 and np.array_equal(g, ref), (x, y, w, h)
        assert np.array_equal(g.reshape(h, w, ch * eb), full[y:y + h, x:x + w]), (x, y, w, h)


def test_requests_alone_and_in_a_mix(session, images):
    rng = np.random.default_rng(9)
    residents = {k: session.upload(v.arena, v.geometry, v.alpha_arena) for k, v in images.items()}
    reqs = []
    for k in range(24):
        name = list(IMAGES)[k % len(IMAGES)]
        W, H = IMAGES[name]["width"], IMAGES[name]["height"]
        if k % 3 == 0:
            reqs.append(residents[name].request(fmt(name, W, H)))
        else:
            w, h = int(rng.integers(16, W)), int(rng.integers(16, H))
            reqs.append(residents[name].request(fmt(name, w, h, int(rng.integers(0, W - w + 1)),
                                                    int(rng.integers(0, H - h + 1)))))
    mixed = run(session, reqs)
    for r, m in zip(reqs, mixed):
        alone, = run(session, [r])
        assert np.array_equal(alone, m)
