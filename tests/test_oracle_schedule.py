"""The oracle's overlap schedules and high-pass placement on bare sample
planes, pinned to the reference's own known answers (each test cites the
reference test it transcribes), plus consistency checks of the schedule
forms against each other and against the forward filters."""
import ctypes as C

import numpy as np
import pytest

import jxr_b200 as J
from tests import _oracle as O


def sign_extend(v):
    return v - (1 << 32) if v >= 1 << 31 else v


# crates/jxr-native/src/reconstruct/overlap.rs:497-501
def test_four_point_operator_has_stable_exact_result():
    assert O.block_op("jo_inverse_overlap_4", [1, 2, 3, 4]) == (0, [2, 1, 4, 5])


# crates/jxr-native/src/reconstruct/overlap.rs:488-495
def test_overlap_operators_preserve_zero():
    assert O.block_op("jo_inverse_overlap_4", [0] * 4) == (0, [0] * 4)
    assert O.block_op("jo_inverse_overlap_4x4", [0] * 16) == (0, [0] * 16)


# crates/jxr-native/src/reconstruct/overlap.rs:503-531
def test_hard_boundary_uses_independent_edge_operators():
    source = [1, 1, 1, 1, 9, 9, 9, 9] * 4
    rc, soft = O.apply_overlap(source, 8, 4, [0, 4, 8], [0, 4], False)
    assert rc == 0
    assert soft.tolist() == [1, 1, 3, 6, 8, 11, 11, 12, 1, 1, 3, 6, 8, 11, 13, 14,
                             1, 1, 3, 6, 8, 11, 11, 12, 1, 1, 3, 6, 8, 11, 13, 14]
    rc, hard = O.apply_overlap(source, 8, 4, [0, 4, 8], [0, 4], True)
    assert rc == 0
    assert hard.tolist() == [1, 1, 1, 1, 11, 12, 11, 12, 1, 1, 1, 1, 13, 14, 13, 14,
                             1, 1, 1, 1, 11, 12, 11, 12, 1, 1, 1, 1, 13, 14, 13, 14]


# crates/jxr-native/src/reconstruct/overlap.rs:533-565
def test_full_plane_operators_cover_the_two_sample_image_edges():
    rows = [
        [-88, -88, -88, -88, -87, -87, -88, -88, -87, -87, -88, -88, -87, -87, -88, -88],
        [-87, -87, -88, -88, -87, -87, -88, -88, -87, -87, -88, -88, -87, -87, -87, -87],
        [-88, -88, -87, -87, -88, -88, -87, -87, -88, -88, -87, -87, -88, -88, -88, -88],
        [-87, -87, -88, -88, -88, -88, -88, -88, -88, -88, -88, -88, -88, -88, -87, -87],
    ]
    order = [0, 1, 2, 2, 3, 3, 2, 2, 3, 3, 2, 2, 3, 3, 0, 1]
    samples = [v for r in order for v in rows[r]]
    rc, out = O.apply_overlap(samples, 16, 16, [0, 16], [0, 16], False)
    assert rc == 0
    assert out.tolist() == [-128] * 256


# crates/jxr-native/src/reconstruct/subsampled_overlap.rs:312-324
def test_zero_plane_is_stable_for_both_subsampled_geometries():
    rc, a = O.apply_overlap([0] * 16, 4, 4, [0, 4], [0, 4], False, subsampled=True)
    assert rc == 0 and a.tolist() == [0] * 16
    rc, b = O.apply_overlap([0] * 32, 4, 8, [0, 4], [0, 8], False, subsampled=True)
    assert rc == 0 and b.tolist() == [0] * 32


# crates/jxr-native/src/reconstruct/subsampled_overlap.rs:326-365
def test_subsampled_postfilter_has_stable_exact_results():
    source = [i * 37 % 101 - 50 for i in range(48)]

    def filtered(w, h, cols, rows, hard):
        rc, out = O.apply_overlap(source[:w * h], w, h, cols, rows, hard, subsampled=True)
        assert rc == 0
        return out.tolist()

    assert filtered(4, 4, [0, 4], [0, 4], False) == [-39, -2, 21, -43, 20, 23, -20, -19, 48, -10, 6, -50, -28, 9,
                                                       -28, 9]
    assert filtered(6, 8, [0, 6], [0, 8], False) == [
        -39, -2, 21, -49, -25, 12, -41, 24, 41, -14, 23, -70, -27, 24, -20, 5, 42, -56, 28,
        35, -7, 17, -46, -1, 40, -24, -8, 39, -26, 11, 38, -4, 33, -50, -12, 9, -8, 15, 52,
        -30, 7, -38, -29, 8, -29, 18, 41, -23]
    assert filtered(6, 8, [0, 2, 6], [0, 4, 8], True) == [
        -13, 11, 15, -49, -25, 12, -41, 22, 28, -14, 23, -70, -27, 35, -19, 5, 42, -56, 47,
        131, -40, -3, -40, -3, -34, -132, -7, 30, -6, 31, 38, -12, 49, -50, -12, 9, -8, 0,
        61, -30, 7, -38, 26, 89, -19, 18, 41, -23]
    # one 4:2:0 macroblock: each top corner is the other's neighbour
    assert filtered(2, 2, [0, 2], [0, 2], False) == [-13, 11, -40, -144]


# crates/jxr-core/src/device_plan/overlap.rs:284-299
def test_full_schedule_centres_interior_work_inside_two_sample_edges():
    off, steps, kinds = O.full_schedule(16, 16, [0, 16], [0, 16], False)
    assert off[0] == 2 + 2 * 16
    assert off[1] == 6 + 2 * 16
    assert off[3] == 2 + 6 * 16
    assert kinds[0] == kinds[1] == kinds[3] == 0 and steps[0] == 16


def apply_schedule(samples, width, offsets, steps, kinds):
    """Run a flat operator list (the device plan's form) with the oracle's
    block operators."""
    s = np.asarray(samples, dtype=np.int64).copy()
    for o, st, k in zip(offsets.tolist(), steps.tolist(), kinds.tolist()):
        if k == 0:
            idx = [o + r * width + c for r in range(4) for c in range(4)]
            rc, v = O.block_op("jo_inverse_overlap_4x4", s[idx].tolist())
        elif k == 1:
            idx = [o + i * st for i in range(4)]
            rc, v = O.block_op("jo_inverse_overlap_4", s[idx].tolist())
        else:
            idx = [o, o + 1, o + width, o + width + 1]
            rc, v = O.block_op("jo_inverse_overlap_4", s[idx].tolist())
        assert rc == 0
        s[idx] = v
    return s.astype(np.int32)


LAYOUTS = [([0, 24], [0, 16], False), ([0, 8, 24], [0, 4, 16], True), ([0, 4, 12, 24], [0, 8, 12, 16], True),
           ([0, 8, 16, 24], [0, 16], False)]


@pytest.mark.parametrize("cols,rows,hard", LAYOUTS)
def test_flat_schedule_equals_the_plane_schedule(cols, rows, hard):
    rng = np.random.default_rng(7)
    src = rng.integers(-3000, 3000, 24 * 16).astype(np.int32)
    rc, want = O.apply_overlap(src, 24, 16, cols, rows, hard)
    assert rc == 0
    off, steps, kinds = O.full_schedule(24, 16, cols, rows, hard)
    assert np.array_equal(apply_schedule(src, 24, off, steps, kinds), want)


def forward_plane(samples, width, height, cols, rows, hard):
    """The prefilter of the plane schedule, built from the generator's forward
    operators in the reverse order of the postfilter (the schedule's
    operators are disjoint, so any order of them inverts)."""
    s = np.asarray(samples, dtype=np.int32).copy()
    off, steps, kinds = O.full_schedule(width, height, cols, rows, hard)
    lib = J.api.synth_lib()
    for o, st, k in zip(off.tolist(), steps.tolist(), kinds.tolist()):
        if k == 0:
            idx = [o + r * width + c for r in range(4) for c in range(4)]
            buf = (C.c_int32 * 16)(*s[idx].tolist())
            lib.jxrb_forward_overlap_4x4(buf)
        else:
            idx = [o + i * st for i in range(4)] if k == 1 else [o, o + 1, o + width, o + width + 1]
            buf = (C.c_int32 * 4)(*s[idx].tolist())
            lib.jxrb_forward_overlap_4(buf)
        s[idx] = list(buf)
    return s


@pytest.mark.parametrize("cols,rows,hard", LAYOUTS)
def test_forward_then_postfilter_is_identity(cols, rows, hard):
    rng = np.random.default_rng(11)
    src = rng.integers(-4000, 4000, 24 * 16).astype(np.int32)
    pre = forward_plane(src, 24, 16, cols, rows, hard)
    rc, back = O.apply_overlap(pre, 24, 16, cols, rows, hard)
    assert rc == 0 and np.array_equal(back, src)


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:659-700 (place_high_pass,
# assert_placed): the second of two macroblocks of a row whose samples start
# at -7.
def place(high, step, bc, br, bands=3):
    width = 2 * bc * 4
    return O.place_high_pass(high, step, bands, bc, br, np.full(width * br * 4, -7, np.int32), width, bc)


def expected_placed(high, step, bc, br, coded=True):
    width = 2 * bc * 4
    out = []
    for index in range(width * br * 4):
        x, y = index % width, index // width
        if x < bc * 4:
            out.append(-7)
            continue
        block = y // 4 * bc + (x - bc * 4) // 4
        position = y % 4 * 4 + x % 4
        out.append(0 if position == 0 or not coded else sign_extend((high[block * 16 + position] * step) & 0xFFFFFFFF))
    return out


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:718-731
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
@pytest.mark.parametrize("step", [1, 2, 3, 37, 113, 65536])
def test_high_pass_blocks_are_placed_as_their_checked_products(bc, br, step):
    high = [i * 37 % 255 - 127 for i in range(256)]
    rc, rows = place(high, step, bc, br)
    assert rc == 0
    assert rows.tolist() == expected_placed(high, step, bc, br)


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:733-783
@pytest.mark.parametrize("step", [1, 2, 3, 37, 113, 65536, 2**31 - 1, 2**31, 2**32 - 1])
def test_high_pass_dequantization_fails_exactly_where_the_checked_product_does(step):
    lo, hi = -2**31, 2**31 - 1
    lower, upper = int(lo / step), int(hi / step)          # truncating division, as i64 / i64
    candidates = [lo, max(lo, lower - 1), lower, -1, 0, 1, upper, min(hi, upper + 1), hi]
    for candidate in candidates:
        for position in (5, 250, 32):
            high = [0] * 256
            high[position] = candidate
            rc, rows = place(high, step, 4, 4)
            product = candidate * step
            fits = position % 16 == 0 or lo <= product <= hi
            if fits:
                assert rc == 0, (step, candidate, position)
                assert rows.tolist() == expected_placed(high, step, 4, 4)
            else:
                assert rc == O.JO_ERR_OVERFLOW, (step, candidate, position)


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:785-808
def test_a_macroblock_without_a_high_pass_band_places_zero_blocks():
    for bands in (0, 1):                 # DcOnly, NoHighPass
        rc, rows = place([2**31 - 1] * 256, 3, 2, 4, bands=bands)
        assert rc == 0
        assert rows.tolist() == expected_placed([0] * 256, 3, 2, 4)
    # a zero step fails whether or not the band is coded
    rc, _ = place([0] * 256, 0, 4, 4, bands=0)
    assert rc == O.JO_ERR_INVALID
