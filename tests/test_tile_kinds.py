"""Which tile kernel takes each 4 x 4-macroblock tile (jxrb_plan_tile_kinds),
against a restatement of the rule on the CPU: interior tiles need macroblocks
mx0-1 .. mx0+4 inside the plane and no hard tile starting at macroblocks
mx0 .. mx0+4; edge tiles only the latter, the plane's own edges aside; 4:2:0
edge tiles also need a plane of at least 2 x 2 macroblocks; 1-bit, planar and
4:2:2 outputs always take the general kernel."""
import pytest

import jxr_b200 as J

C_, D, S, L = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT
T = 4


def restated(mbs_x, mbs_y, kind, tile_w=0, tile_h=0, hard=0):
    def starts(n, size):
        return {k for k in range(1, n) if hard and size and k % size == 0}
    sx, sy = starts(mbs_x, tile_w), starts(mbs_y, tile_h)
    out = dict(interior=0, interior_420=0, edge=0, edge_420=0, general=0)
    for ty in range(-(-mbs_y // T)):
        for tx in range(-(-mbs_x // T)):
            mx0, my0 = tx * T, ty * T
            clear_x = not any(k in sx for k in range(max(mx0, 1), min(mx0 + T, mbs_x - 1) + 1))
            clear_y = not any(k in sy for k in range(max(my0, 1), min(my0 + T, mbs_y - 1) + 1))
            inside = mx0 >= 1 and my0 >= 1 and mx0 + T < mbs_x and my0 + T < mbs_y
            if kind is None or not (clear_x and clear_y):
                out["general"] += 1
            elif inside:
                out["interior_420" if kind == "420" else "interior"] += 1
            elif kind == "420":
                out["edge_420" if mbs_x >= 2 and mbs_y >= 2 else "general"] += 1
            else:
                out["edge"] += 1
    return out


def kinds(w, h, out=None, **kw):
    img = J.synth(w, h, quality=60, threads=4, **kw)
    out = out or J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], w, h)
    return J.CudaDecodePlan(img.arena, img.geometry, out, img.alpha_arena).tile_kinds()


def test_c2_shape_splits_interior_and_edge():
    # a 1024 x 1024 plane: 16 x 16 tiles, the outer ring on the plane's edge
    assert kinds(1024, 1024, overlap=2, tile_width=16, tile_height=16) == \
        dict(interior=196, interior_420=0, edge=60, edge_420=0, general=0)


@pytest.mark.parametrize("size", [(16, 16), (48, 80), (160, 96), (208, 176), (336, 272), (400, 336)])
@pytest.mark.parametrize("fmt", ["YUV444", "YUV420", "LUMA"])
def test_soft_tiles(size, fmt):
    w, h = size
    got = kinds(w, h, color_format=C_[fmt], overlap=1)
    assert got == restated(w // 16, h // 16, "420" if fmt == "YUV420" else "full")


@pytest.mark.parametrize("tiles", [(5, 3), (8, 8), (2, 7), (13, 11)])
@pytest.mark.parametrize("fmt", ["YUV444", "YUV420"])
def test_hard_tiles(tiles, fmt):
    tw, th = tiles
    got = kinds(400, 336, color_format=C_[fmt], overlap=2, tile_width=tw, tile_height=th, hard_tiles=1)
    assert got == restated(25, 21, "420" if fmt == "YUV420" else "full", tw, th, 1)


def test_outputs_that_take_the_general_kernel():
    assert kinds(160, 96, color_format=C_["YUV422"])["general"] == 6
    planar = J.OutputFormat(C_["YUV420"], D["U8"], S["U8"], L["YUV"], 336, 272)
    assert kinds(336, 272, color_format=C_["YUV420"], out=planar) == restated(21, 17, None)
    bits = J.OutputFormat(C_["LUMA"], D["BIT1_BLACK"], S["BITS"], L["LUMA"], 208, 176)
    assert kinds(208, 176, color_format=C_["LUMA"], out=bits) == restated(13, 11, None)


def test_yuvk_takes_the_four_plane_kernels():
    assert kinds(336, 272, color_format=C_["YUVK"], overlap=2,
                 out=J.OutputFormat(C_["CMYK"], D["U8"], S["U8"], L["CMYK"], 336, 272)) == restated(21, 17, "full")
