"""Device-free validation of jxrb_plan_create: every rejection of the
planner, reached by corrupting one field of a valid arena, geometry or output
request, and a seeded fuzz of the planner.

The reference validates its plans before any CUDA resource exists
(crates/jxr-cuda/src/plan.rs:91-148, 255-355, 405-610) and pins four of its
rejections in crates/jxr-cuda/src/plan/tests.rs:39-96; those four come first
here.  Nothing in this file needs a GPU: plan creation reads host metadata
only."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import jxr_b200 as J
from jxr_b200 import api

C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA
INVALID_PLAN, UNSUPPORTED_OUTPUT, RESOURCE_LIMIT = 4, 6, 10


def luma_arena(coords, bands=0, step=1):
    """A luma arena of DC-only macroblocks at `coords` (one coefficient each),
    like the reference's luma_arena test helper."""
    n = len(coords)
    per = {0: 1, 1: 16, 2: 256, 3: 256}[bands]
    return J.Arena(coefficients=np.zeros(n * per, np.int32),
                   coefficient_offsets=np.arange(n, dtype=np.uint32) * per,
                   quantizers=np.full((n, 3), step, np.uint32), bands=np.full(n, bands, np.uint8),
                   hp_predictions=np.zeros(n, np.uint8), coded_x=np.array([c[0] for c in coords], np.uint32),
                   coded_y=np.array([c[1] for c in coords], np.uint32),
                   planes=np.array([[0, n * per, 0, n, 4, 4]], np.uint64))


def grid(mx, my):
    return [(x, y) for y in range(my) for x in range(mx)]


def luma_geometry(mx, my, **kw):
    return J.Geometry(mx, my, color_format=C_["LUMA"], components=1, overlap=0, **kw)


def luma_output(mx, my, **kw):
    return J.OutputFormat(C_["LUMA"], D["U8"], S["U8"], L["LUMA"], 16 * mx, 16 * my, **kw)


def rejected(arena, geom, out, alpha=None):
    with pytest.raises(J.CudaError) as e:
        J.CudaDecodePlan(arena, geom, out, alpha)
    return e.value.status, str(e.value)


def test_valid_plans_are_accepted():
    p = J.CudaDecodePlan(luma_arena(grid(2, 2)), luma_geometry(2, 2), luma_output(2, 2))
    assert p.output_bytes() == 32 * 32


# ---- the reference's four pinned rejections (plan/tests.rs:39-96) ----------

def test_rejects_top_left_prediction():
    a = luma_arena([(0, 0)], bands=3)
    a.hp_predictions[0] = 3
    st, msg = rejected(a, luma_geometry(1, 1), luma_output(1, 1))
    assert st == INVALID_PLAN and "top-left high-pass prediction" in msg


def test_rejects_duplicate_macroblock_coordinates():
    st, msg = rejected(luma_arena([(0, 0), (0, 0), (0, 1), (1, 1)]), luma_geometry(2, 2), luma_output(2, 2))
    assert st == INVALID_PLAN and "duplicate macroblock coordinates" in msg


def test_rejects_a_window_the_arena_does_not_cover():
    # the reference's arena at (1, 0) for a 1 x 1 plane: the window's one
    # position has no macroblock
    st, msg = rejected(luma_arena([(1, 0)]), luma_geometry(1, 1), luma_output(1, 1))
    assert st == INVALID_PLAN and "no coefficients" in msg


def test_rejects_a_coefficient_span_outside_the_upload():
    a = luma_arena([(0, 0)])
    a.coefficient_offsets[0] = 1
    st, msg = rejected(a, luma_geometry(1, 1), luma_output(1, 1))
    assert st == INVALID_PLAN and "coefficient span outside its plane" in msg


# ---- the rest of the planner's rejections -------------------------------

def corrupt_arena(field, value, bands=0):
    a = luma_arena(grid(2, 2), bands=bands)
    getattr(a, field)[1] = value
    return a


@pytest.mark.parametrize("field,value,bands,needle", [
    ("hp_predictions", 4, 3, "high-pass prediction direction"),
    ("bands", 4, 0, "band presence"),
    ("quantizers", 0, 0, "zero quantizer"),
    ("coefficient_offsets", 1000, 0, "coefficient span outside its plane"),
])
def test_rejects_macroblock_metadata(field, value, bands, needle):
    st, msg = rejected(corrupt_arena(field, value, bands), luma_geometry(2, 2), luma_output(2, 2))
    assert st == INVALID_PLAN and needle in msg


@pytest.mark.parametrize("row,needle", [
    ([0, 4, 0, 4, 2, 4], "block geometry differs"),        # 4:2:2 block shape for a luma plane
    ([0, 99, 0, 4, 4, 4], "coefficient plane range"),
    ([0, 4, 1, 4, 4, 4], "macroblock plane range"),
])
def test_rejects_plane_descriptors(row, needle):
    a = luma_arena(grid(2, 2))
    a.planes = np.array([row], np.uint64)
    st, msg = rejected(a, luma_geometry(2, 2), luma_output(2, 2))
    assert st == INVALID_PLAN and needle in msg


def test_rejects_a_plane_count_unlike_the_colour_format():
    a = luma_arena(grid(2, 2))
    g = dataclasses.replace(luma_geometry(2, 2), color_format=C_["YUV444"], components=3)
    st, msg = rejected(a, g, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 32, 32))
    assert st == INVALID_PLAN and "plane count" in msg


@pytest.mark.parametrize("change,status,needle", [
    (dict(macroblocks_x=0), INVALID_PLAN, "empty reconstruction window"),
    (dict(macroblocks_x=65535 * 4 + 1), RESOURCE_LIMIT, "window too large"),
    (dict(overlap=3), INVALID_PLAN, "overlap mode"),
    (dict(alpha_overlap=-1), INVALID_PLAN, "overlap mode"),
    (dict(color_format=C_["RGBE"]), INVALID_PLAN, "coded colour format"),
    (dict(color_format=C_["NCOMPONENT"], components=5), UNSUPPORTED_OUTPUT, "N-component"),
    (dict(tile_column_widths=[1]), INVALID_PLAN, "tile partition does not cover"),
    (dict(tile_row_heights=[1]), INVALID_PLAN, "tile partition does not cover"),
])
def test_rejects_geometry(change, status, needle):
    g = dataclasses.replace(luma_geometry(2, 2), **change)
    st, msg = rejected(luma_arena(grid(2, 2)), g, luma_output(2, 2))
    assert st == status and needle in msg


def test_rejects_a_missing_or_empty_separate_alpha_arena():
    g = dataclasses.replace(luma_geometry(2, 2), alpha_mode=A["SEPARATE"])
    out = J.OutputFormat(C_["LUMA"], D["U8"], S["U8"], L["LUMA_ALPHA"], 32, 32, alpha_bit_depth=D["U8"])
    st, msg = rejected(luma_arena(grid(2, 2)), g, out)
    assert st == INVALID_PLAN and "separate alpha arena missing" in msg
    empty = luma_arena(grid(2, 2))
    empty.planes = np.zeros((0, 6), np.uint64)
    st, msg = rejected(luma_arena(grid(2, 2)), g, out, alpha=empty)
    assert st == INVALID_PLAN and "has no plane" in msg


def yuv420_arena(mx, my):
    """DC-only 4:2:0 planes: 4x4 blocks for luma, 2x2 for chroma."""
    n = mx * my
    xy = grid(mx, my)
    return J.Arena(coefficients=np.zeros(3 * n, np.int32), coefficient_offsets=np.arange(3 * n, dtype=np.uint32),
                   quantizers=np.ones((3 * n, 3), np.uint32), bands=np.zeros(3 * n, np.uint8),
                   hp_predictions=np.zeros(3 * n, np.uint8),
                   coded_x=np.array([c[0] for c in xy] * 3, np.uint32),
                   coded_y=np.array([c[1] for c in xy] * 3, np.uint32),
                   planes=np.array([[0, n, 0, n, 4, 4], [n, n, n, n, 2, 2], [2 * n, n, 2 * n, n, 2, 2]], np.uint64))


def test_rejects_an_unknown_chroma_centering_for_interpolated_output():
    g = J.Geometry(2, 2, color_format=C_["YUV420"], overlap=0, chroma_centering_x=7)
    st, msg = rejected(yuv420_arena(2, 2), g, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 32, 32))
    assert st == UNSUPPORTED_OUTPUT and "chroma centering" in msg
    # native planar output needs no filter: accepted
    J.CudaDecodePlan(yuv420_arena(2, 2), g, J.OutputFormat(C_["YUV420"], D["U8"], S["U8"], L["YUV"], 32, 32))


@pytest.mark.parametrize("change,status,needle", [
    (dict(crop_width=0), INVALID_PLAN, "empty crop"),
    (dict(crop_x=1), INVALID_PLAN, "crop window lies outside"),
    (dict(crop_height=33), INVALID_PLAN, "crop window lies outside"),
])
def test_rejects_crops(change, status, needle):
    st, msg = rejected(luma_arena(grid(2, 2)), luma_geometry(2, 2), dataclasses.replace(luma_output(2, 2), **change))
    assert st == status and needle in msg


@pytest.mark.parametrize("crop,needle", [((1, 0), "even column"), ((0, 1), "even row")])
def test_rejects_odd_planar_chroma_crops(crop, needle):
    g = J.Geometry(2, 2, color_format=C_["YUV420"], overlap=0)
    out = J.OutputFormat(C_["YUV420"], D["U8"], S["U8"], L["YUV"], 30, 30, crop_x=crop[0], crop_y=crop[1])
    st, msg = rejected(yuv420_arena(2, 2), g, out)
    assert st == UNSUPPORTED_OUTPUT and needle in msg


def rgb_plan_parts(alpha=False):
    img = J.synth(32, 32, quality=80, overlap=1, seed=3, alpha_mode=A["INTEGRATED"] if alpha else 0,
                  alpha_qp=(8, 8, 8) if alpha else (0, 0, 0), threads=1)
    return img.arena, img.geometry


@pytest.mark.parametrize("alpha,out,status,needle", [
    (False, dict(layout=L["RGBA"]), INVALID_PLAN, "alpha layout and prepared alpha plane differ"),
    (False, dict(premultiply_alpha=1), INVALID_PLAN, "premultiplied output without alpha"),
    (False, dict(storage=S["U16"]), UNSUPPORTED_OUTPUT, "bit depth and typed storage"),
    (False, dict(layout=L["LUMA"]), UNSUPPORTED_OUTPUT, "output colour and channel layout"),
    (False, dict(output_color=C_["CMYK"], layout=L["CMYK"]), UNSUPPORTED_OUTPUT, "internal and output colour"),
    (False, dict(output_color=C_["YUV444"], layout=L["YUV"], bit_depth=D["F16"], storage=S["F16"]),
     UNSUPPORTED_OUTPUT, "T.832"),
    (False, dict(bit_depth=D["F32"], storage=S["F32"], mantissa_length=24), UNSUPPORTED_OUTPUT, "mantissa"),
    (False, dict(widen_f16=1), UNSUPPORTED_OUTPUT, "widening applies to F16"),
    (False, dict(bit_depth=D["RGB565"], storage=S["RGB565"], nchw=1), UNSUPPORTED_OUTPUT, "NCHW"),
    (False, dict(bit_depth=D["I16"], storage=S["I16"], shift_bits=32), UNSUPPORTED_OUTPUT, "SHIFT_BITS"),
    (True, dict(layout=L["RGBA"], premultiply_alpha=1, nchw=1, alpha_bit_depth=D["U8"]), UNSUPPORTED_OUTPUT,
     "premultiplied output is interleaved"),
    (True, dict(layout=L["RGBA"], bit_depth=D["F32"], storage=S["F32"], alpha_bit_depth=D["U8"]),
     UNSUPPORTED_OUTPUT, "alpha and primary floating-point depth"),
    (True, dict(output_color=C_["YUV444"], layout=L["YUVA"], premultiply_alpha=1, alpha_bit_depth=D["U8"]),
     UNSUPPORTED_OUTPUT, "premultiplied YUV output"),
])
def test_rejects_output_requests(alpha, out, status, needle):
    arena, geom = rgb_plan_parts(alpha)
    base = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 32, 32)
    st, msg = rejected(arena, geom, dataclasses.replace(base, **out))
    assert st == status and needle in msg, msg


def test_rejects_a_plane_beyond_the_table_offset_range():
    # a macroblock 2^28 coefficients into its plane does not fit the 28-bit
    # offset of a table entry; the planner reads metadata only, so the count
    # can be claimed without the memory behind it
    a = luma_arena([(0, 0)])
    a.coefficient_offsets[0] = 1 << 28
    count = (1 << 28) + 1
    a.planes = np.array([[0, count, 0, 1, 4, 4]], np.uint64)
    c, keep = a.to_c()
    c.coefficient_count = count
    g, gkeep = luma_geometry(1, 1).to_c()
    o = luma_output(1, 1).to_c()
    h = C.c_void_p()
    st = J.lib().jxrb_plan_create(C.byref(c), None, C.byref(g), C.byref(o), C.byref(h))
    assert st == RESOURCE_LIMIT and b"2^28" in J.lib().jxrb_last_error()


def test_rejects_null_arguments():
    h = C.c_void_p()
    assert J.lib().jxrb_plan_create(None, None, None, None, C.byref(h)) == INVALID_PLAN


# ---- fuzz: crates/jxr/fuzz/fuzz_targets/cuda_plan.rs, seeded ---------------

FIELDS_U32 = ["coefficient_offsets", "coded_x", "coded_y"]
FIELDS_U8 = ["bands", "hp_predictions"]


def mutate(rng, arena, geom, out):
    """One random corruption of the plan's inputs."""
    a = dataclasses.replace(arena, **{f: getattr(arena, f).copy() for f in
                                      FIELDS_U32 + FIELDS_U8 + ["quantizers", "planes"]})
    g, o = geom, out
    for _ in range(int(rng.integers(1, 4))):
        k = int(rng.integers(0, 7))
        if k == 0:
            f = FIELDS_U32[int(rng.integers(0, 3))]
            arr = getattr(a, f)
            arr[int(rng.integers(0, arr.size))] = int(rng.integers(0, 1 << 32, dtype=np.uint64))
        elif k == 1:
            f = FIELDS_U8[int(rng.integers(0, 2))]
            arr = getattr(a, f)
            arr[int(rng.integers(0, arr.size))] = int(rng.integers(0, 256))
        elif k == 2:
            a.quantizers.reshape(-1)[int(rng.integers(0, a.quantizers.size))] = int(rng.integers(0, 3))
        elif k == 3:
            a.planes.reshape(-1)[int(rng.integers(0, a.planes.size))] = int(rng.integers(0, 1 << 20))
        elif k == 4:
            g = dataclasses.replace(g, **{["macroblocks_x", "macroblocks_y", "macroblock_origin_x",
                                            "macroblock_origin_y", "overlap", "color_format"][int(rng.integers(0, 6))]:
                                          int(rng.integers(0, 12))})
        elif k == 5:
            o = dataclasses.replace(o, **{["crop_x", "crop_y", "crop_width", "crop_height"][int(rng.integers(0, 4))]:
                                          int(rng.integers(0, 600))})
        else:
            o = dataclasses.replace(o, **{["bit_depth", "storage", "layout", "output_color"][int(rng.integers(0, 4))]:
                                          int(rng.integers(0, 14))})
    return a, g, o


def test_fuzz_plan_builder():
    """Random corruptions of valid inputs: the planner returns a status for
    each (never crashes), and every plan it accepts keeps its invariants."""
    rng = np.random.default_rng(1234)
    img = J.synth(160, 128, quality=80, overlap=2, tile_width=3, tile_height=2, hard_tiles=1, seed=9, threads=1)
    base = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 160, 128)
    accepted = 0
    statuses = set()
    for _ in range(1500):
        a, g, o = mutate(rng, img.arena, img.geometry, base)
        try:
            p = J.CudaDecodePlan(a, g, o)
        except J.CudaError as e:
            statuses.add(e.status)
            assert e.status in (INVALID_PLAN, UNSUPPORTED_OUTPUT, RESOURCE_LIMIT)
            assert str(e).split(": ", 1)[1]           # a reason is given
            continue
        accepted += 1
        assert p.output_bytes() > 0
        k = p.tile_kinds()
        mx, my = g.macroblocks_x, g.macroblocks_y
        assert sum(k.values()) == ((mx + 3) // 4) * ((my + 3) // 4)
        assert p.traffic_bytes() >= p.output_bytes()
        p.close()
    assert accepted > 0 and {INVALID_PLAN, UNSUPPORTED_OUTPUT} <= statuses
