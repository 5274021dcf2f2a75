"""Pins the CPU oracle to the reference's own golden vectors and known-answer
tests.  Each case cites the reference test it is taken from; the values are
the reference's, transcribed."""
import numpy as np
import pytest

from tests import _oracle as O

I32_MAX, I32_MIN = 2**31 - 1, -(2**31)


# crates/jxr-math/src/transform.rs:497-509
def test_inverse_core_transform_t835_signed_rounding_case():
    rc, out = O.block_op("jo_inverse_core_transform",
                         [50, -42, 9, 21, 126, 33, -6, -18, -24, 21, -3, -9, -6, -33, 6, 15])
    assert rc == 0
    assert out == [50, 50, 47, 49, 39, 38, 41, 41, -30, -44, 27, 36, -47, -55, -23, -20]


# crates/jxr-math/src/transform.rs:489-495
def test_dc_only_block_is_uniform():
    rc, out = O.block_op("jo_inverse_core_transform", [16] + [0] * 15)
    assert rc == 0 and out == [4] * 16


# crates/jxr-math/src/transform.rs:511-516
def test_inverse_chroma_422_golden():
    rc, out = O.block_op("jo_inverse_chroma_422", [1, 2, 3, 4, 5, 6, 7, 8])
    assert rc == 0 and out == [4, -3, -4, -2, 12, -2, -3, -1]


# crates/jxr-math/src/transform.rs:461-472: forward 4:2:0 of a flat [6;4] is
# [12,0,0,0], so the inverse of [12,0,0,0] is the flat block.
def test_inverse_chroma_420_of_flat_dc():
    rc, out = O.block_op("jo_inverse_chroma_420", [12, 0, 0, 0])
    assert rc == 0 and out == [6, 6, 6, 6]


# crates/jxr-math/src/overlap.rs:538-547
def test_subsampled_filters_have_exact_results():
    assert O.block_op("jo_inverse_overlap_2", [1, 2]) == (0, [2, 3])
    assert O.block_op("jo_inverse_overlap_2x2", [1, 2, 3, 4]) == (0, [3, 4, 4, 5])


# crates/jxr-math/src/overlap.rs:528-536
def test_inverse_filters_preserve_zero():
    assert O.block_op("jo_inverse_overlap_4", [0] * 4) == (0, [0] * 4)
    assert O.block_op("jo_inverse_overlap_4x4", [0] * 16) == (0, [0] * 16)


def test_checked_operators_report_overflow():
    # crates/jxr-math/src/arithmetic.rs:86-98 (checked operations reject overflow)
    assert O.block_op("jo_inverse_overlap_4", [I32_MAX] * 4)[0] == O.JO_ERR_OVERFLOW
    assert O.block_op("jo_inverse_core_transform", [I32_MAX] * 16)[0] == O.JO_ERR_OVERFLOW
    assert O.block_op("jo_inverse_overlap_2x2", [I32_MAX] * 4)[0] == O.JO_ERR_OVERFLOW


# crates/jxr-math/tests/math_contract.rs:4-10
def test_dequantize_and_overflow():
    assert O.dequantize(-7, 4) == (0, -28)
    assert O.dequantize(I32_MAX, 4)[0] == O.JO_ERR_OVERFLOW


# crates/jxr-math/src/prediction.rs:160-172
def test_subsampled_420_prediction_uses_two_by_two_block_geometry():
    c = [0] * 256
    c[12], c[16 + 12], c[2 * 16 + 12], c[3 * 16 + 12] = 5, 7, 11, 13
    rc, out = O.predict_high_pass(c, 1, 2, 2)
    assert rc == 0
    assert out[16 + 12] == 12 and out[3 * 16 + 12] == 24


def test_top_left_prediction_is_rejected():
    # crates/jxr-native/src/decode/reconstruction.rs:475-481
    assert O.predict_high_pass([0] * 256, 3, 4, 4)[0] == O.JO_ERR_INVALID


# crates/jxr-math/src/sampling.rs:121-145, 252-282
def test_chroma_interpolation_golden():
    assert O.upsample_pair(0, 8, 16, 0) == (0, [8, 12])
    assert O.upsample_pair(0, 8, 16, 4) == (0, [4, 8])
    assert O.upsample_pair(-9, -4, 3, 2) == (0, [-5, -2])
    for centering in range(5):
        for s in (I32_MAX, I32_MIN):
            assert O.upsample_pair(s, s, s, centering) == (0, [s, s])
    assert O.upsample_pair(I32_MIN, I32_MAX, I32_MIN, 0) == (0, [I32_MAX, 0])
    assert O.upsample_pair(0, 0, 0, 7)[0] != 0


# crates/jxr-math/src/sampling.rs:147-187: the interpolation equals the
# Table 180 sum computed in 64 bits over samples near multiples of eight.
def test_chroma_interpolation_equals_64_bit_sum():
    weights = [[4, 4, 0, 8], [5, 3, 1, 7], [6, 2, 2, 6], [7, 1, 3, 5], [8, 0, 4, 4]]
    samples = []
    for index in range(49):
        offset = index % 7 - 3
        base = [I32_MIN + 3, I32_MAX - 3, 0, 8, -8, 0x12345678, -0x12345678][index // 7]
        samples.append(base + offset)
    exact = lambda a, wa, b, wb: (a * wa + b * wb + 4) >> 3
    for centering in range(5):
        h0, h1, h2, h3 = weights[centering]
        for prev in samples[::3]:
            for cur in samples[::2]:
                for nxt in (prev, cur, samples[centering * 9]):
                    assert O.upsample_pair(prev, cur, nxt, centering) == (
                        0, [exact(prev, h2, cur, h3), exact(cur, h0, nxt, h1)])


# crates/jxr-math/src/rgbe.rs:132-146
def test_rgbe_postscale_golden():
    assert O.postscale_rgbe([128, 256, 64]) == [64, 128, 32, 2]
    assert O.postscale_rgbe([-1, 0, 127]) == [0, 0, 127, 1]
    assert O.postscale_rgbe([I32_MAX, 0, 0])[3] == 255


def _prescale_rgbe(b):
    # crates/jxr-math/src/rgbe.rs:34-55 (the encoder's inverse), restated to
    # run the reference's round-trip property test.
    rgb = [0, 0, 0]
    for ch in range(3):
        m, e = b[ch], b[3]
        if m != 0 and e != 0:
            while m < 128 and e > 1:
                m <<= 1
                e -= 1
            rgb[ch] = (e << 7) | (m & 0x7F) if e > 1 else m
    return rgb


# crates/jxr-math/src/rgbe.rs:107-128
def test_rgbe_prescale_postscale_round_trip():
    mantissas = [0, 1, 2, 63, 64, 127, 128, 129, 200, 255]
    for e in [1, 2, 3, 100, 128, 254, 255]:
        for r in mantissas:
            for g in mantissas:
                for b in mantissas:
                    brightest = max(r, g, b)
                    if not (brightest >= 128 or (e == 1 and brightest != 0)):
                        continue
                    assert O.postscale_rgbe(_prescale_rgbe([r, g, b, e])) == [r, g, b, e]
    assert O.postscale_rgbe(_prescale_rgbe([0, 0, 0, 0])) == [0, 0, 0, 0]


# crates/jxr-math/src/alpha.rs:62-89
def test_premultiply_golden():
    assert O.premultiply_unsigned(255, 128, 255) == (0, 128)
    assert O.premultiply_unsigned(7, 0, 255) == (0, 0)
    assert O.premultiply_signed(-20000, 16384, 32767) == (0, -10000)
    assert O.premultiply_signed(20000, -1, 32767) == (0, 0)
    assert O.premultiply_sign_magnitude_15(0x8000 | 0x4E20, 16384) == (0, 0x8000 | 0x2710)
    L = O.lib()
    assert L.jo_premultiply_f32(-4.0, 0.25) == -1.0
    assert L.jo_premultiply_f32(4.0, 2.0) == 4.0


def test_half_widening_is_exact_for_every_bit_pattern():
    h = np.arange(65536, dtype=np.uint16)
    got = np.array([O.lib().jo_widen_f16(int(v)) for v in h], dtype=np.uint32)
    f = h.view(np.float16).astype(np.float32).view(np.uint32)
    finite = (h & 0x7C00) != 0x7C00
    assert np.array_equal(got[finite], f[finite])
    nan_or_inf = ~finite
    # Infinity and NaN keep their payload bits shifted into binary32.
    expect = ((h[nan_or_inf].astype(np.uint32) & 0x8000) << 16) | 0x7F800000 | (
        (h[nan_or_inf].astype(np.uint32) & 0x3FF) << 13)
    assert np.array_equal(got[nan_or_inf], expect)


def _dc_plane(value, step, bands, overlap, bc=4, br=4):
    count = bc * br
    coeffs = np.zeros(count * 16 if bands >= 2 else max(count, 1), np.int32)
    coeffs[0] = value
    return dict(coefficients=coeffs, offsets=[0], quantizers=[step, 1, 1], bands=[bands],
                hp_prediction=[0], macroblocks_x=1, macroblocks_y=1, block_columns=bc,
                block_rows=br, overlap=overlap)


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:29-46
def test_dc_only_macroblock_reconstructs_constant_plane():
    rc, plane = O.reconstruct_plane(_dc_plane(256, 1, 0, 0))
    assert rc == 0 and plane.shape == (16, 16) and (plane == 16).all()


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:48-79: with both
# overlap levels the samples of a DC of 256 lie between 32 and 36 and every
# 4x4 block averages 33.
def test_two_level_overlap_of_a_dc_macroblock():
    rc, plane = O.reconstruct_plane(_dc_plane(256, 1, 1, 2))
    assert rc == 0
    assert plane.min() == 32 and plane.max() == 36
    means = plane.reshape(4, 4, 4, 4).transpose(0, 2, 1, 3).reshape(16, 16).mean(axis=1)
    assert (np.floor(means) == 33).all()


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:84-126
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
def test_subsampled_dc_macroblock_is_flat(bc, br):
    dc = 256 if bc == 4 else 128
    rc, plane = O.reconstruct_plane(_dc_plane(dc, 1, 1, 0, bc, br))
    assert rc == 0 and (plane == 16).all()


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:128-146: both levels of
# overlap raise a DC-only macroblock of 256 to a mean of 33.
def test_sixteenth_mean_of_two_level_dc_macroblock():
    rc, plane = O.reconstruct_plane(_dc_plane(256, 1, 0, 2))
    assert rc == 0 and int(plane.mean()) == 33


# crates/jxr-native/src/output_format/color.rs:235-270
def test_colour_conversion_golden():
    def rgb(yuv, packed=False, storage=1, depth=2, layout=4):
        planes = [dict(_dc_plane(0, 1, 0, 0)) for _ in range(3)]
        out = O.make_output(internal_color=3, output_color=4, depth=depth, storage=storage,
                            layout=layout, crop_width=1, crop_height=1, ncomponents=3)
        # format one pixel directly
        import ctypes as C
        arrs = [np.array([[v]], np.int32) for v in yuv]
        ptrs = (C.POINTER(C.c_int32) * 3)(*[a.ctypes.data_as(C.POINTER(C.c_int32)) for a in arrs])
        n = O.output_bytes(out)
        buf = np.zeros(n, np.uint8)
        rc = O.lib().jo_format_output(ptrs, 3, None, 1, 1, C.byref(out), buf.ctypes.data, n)
        return rc, buf
    # I32 output with no bias shows the converted values themselves.
    rc, buf = rgb([10, 3, 5], storage=4, depth=7)
    assert rc == 0 and list(buf.view(np.int32)) == [6, 12, 11]


# crates/jxr-native/src/output_format/scaling.rs:433-456, 480-531
def test_scaling_golden():
    import ctypes as C

    def one(sample, **kw):
        out = O.make_output(internal_color=0, output_color=0, layout=0, crop_width=1,
                            crop_height=1, ncomponents=1, **kw)
        a = np.array([[sample]], np.int32)
        ptrs = (C.POINTER(C.c_int32) * 1)(a.ctypes.data_as(C.POINTER(C.c_int32)))
        n = O.output_bytes(out)
        buf = np.zeros(n, np.uint8)
        rc = O.lib().jo_format_output(ptrs, 1, None, 1, 1, C.byref(out), buf.ctypes.data, n)
        return rc, buf
    # scaled U8 adds the bias then rounds down
    assert one(-1, depth=2, storage=1, scaled=1) == (0, np.array([128], np.uint8))
    assert list(one(-5, depth=2, storage=1, scaled=1)[1]) == [127]
    # integer post-shift follows scaling
    assert list(one(7, depth=5, storage=3, scaled=1, shift_bits=3)[1].view(np.int16)) == [8]
    # a post-scaled sample past the 32-bit limit is clipped to it
    for s, e in [((1 << 21) - 1, I32_MAX & ~0x3FF), (1 << 21, I32_MAX), (I32_MAX, I32_MAX),
                 (-(1 << 21), I32_MIN), (-(1 << 21) - 1, I32_MIN)]:
        assert list(one(s, depth=7, storage=4, shift_bits=10)[1].view(np.int32)) == [e]
    # an F32 exponent past the format clips to the largest finite value
    f32 = lambda s: int(one(s, depth=8, storage=6, mantissa_length=4, exponent_bias=1)[1].view(np.uint32)[0])
    assert f32(129 << 4) == 0x7F800000
    assert f32(130 << 4) == 0x7F7FFFFF
    assert f32(-(130 << 4)) == 0xFF7FFFFF
    assert f32(I32_MAX) == 0x7F7FFFFF
    assert f32(1 << 4) == 0x3F800000 and f32(-(1 << 4)) == 0xBF800000
    # F16 is sign and clamped magnitude
    f16 = lambda s: int(one(s, depth=6, storage=5)[1].view(np.uint16)[0])
    assert f16(-40000) == 0xFFFF and f16(17) == 17
