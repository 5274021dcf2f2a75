/*
 * jxr_oracle.c -- CPU restatement of the frames-sg/jxr reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  Nothing in the
 * product links or loads this file.
 *
 * Each function names the reference function and file:line it restates.
 * Arithmetic is the reference's checked form: an intermediate outside int32
 * makes the whole operation fail, as `checked_add` / `checked_sub` /
 * `checked_mul` / `checked_i64_to_i32` do in crates/jxr-math/src/arithmetic.rs:58-84.
 */
#include "jxr_oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* checked arithmetic: crates/jxr-math/src/arithmetic.rs:58-84               */
/* ------------------------------------------------------------------------ */
#define CK(expr) do { if (expr) return JO_ERR_OVERFLOW; } while (0)

static inline int add(int32_t a, int32_t b, int32_t *r) { return __builtin_add_overflow(a, b, r); }
static inline int sub(int32_t a, int32_t b, int32_t *r) { return __builtin_sub_overflow(a, b, r); }
static inline int mul(int32_t a, int32_t b, int32_t *r) { return __builtin_mul_overflow(a, b, r); }
static inline int neg(int32_t a, int32_t *r) { if (a == INT32_MIN) return 1; *r = -a; return 0; }
/* (a*3 + k) >> s, each step checked */
static inline int mul3_add_shr(int32_t a, int32_t k, int s, int32_t *r)
{
    int32_t t;
    if (mul(a, 3, &t)) return 1;
    if (add(t, k, &t)) return 1;
    *r = t >> s;
    return 0;
}
/* (a + k) >> s, checked */
static inline int add_shr(int32_t a, int32_t k, int s, int32_t *r)
{
    int32_t t;
    if (add(a, k, &t)) return 1;
    *r = t >> s;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* core transform: crates/jxr-math/src/transform.rs                          */
/* ------------------------------------------------------------------------ */

/* crates/jxr-math/data/reconstruction.abi:2 */
static const int INVERSE_PERMUTATION[16] = {0, 8, 4, 13, 2, 15, 3, 14, 1, 12, 5, 9, 7, 11, 6, 10};

/* t2x2h, transform.rs:226-237 */
static int t2x2h(int32_t v[4], int32_t rounding)
{
    int32_t d, first, second;
    CK(add(v[0], v[3], &v[0]));
    CK(sub(v[1], v[2], &v[1]));
    CK(sub(v[0], v[1], &d));
    CK(add_shr(d, rounding, 1, &first));
    second = v[2];
    CK(sub(first, v[3], &v[2]));
    CK(sub(first, second, &v[3]));
    CK(sub(v[0], v[3], &v[0]));
    CK(add(v[1], v[2], &v[1]));
    return JO_OK;
}

/* inverse_todd, transform.rs:240-275 */
static int inverse_todd(int32_t v[4])
{
    int32_t t;
    CK(add(v[1], v[3], &v[1]));
    CK(sub(v[0], v[2], &v[0]));
    CK(sub(v[3], v[1] >> 1, &v[3]));
    CK(add_shr(v[0], 1, 1, &t)); CK(add(v[2], t, &v[2]));
    CK(mul3_add_shr(v[1], 4, 3, &t)); CK(sub(v[0], t, &v[0]));
    CK(mul3_add_shr(v[0], 4, 3, &t)); CK(add(v[1], t, &v[1]));
    CK(mul3_add_shr(v[3], 4, 3, &t)); CK(sub(v[2], t, &v[2]));
    CK(mul3_add_shr(v[2], 4, 3, &t)); CK(add(v[3], t, &v[3]));
    CK(add_shr(v[1], 1, 1, &t)); CK(sub(v[2], t, &v[2]));
    CK(add_shr(v[0], 1, 1, &t)); CK(sub(t, v[3], &v[3]));
    CK(add(v[1], v[2], &v[1]));
    CK(sub(v[0], v[3], &v[0]));
    return JO_OK;
}

/* inverse_todd_odd, transform.rs:278-312 */
static int inverse_todd_odd(int32_t v[4])
{
    int32_t t, first, second;
    CK(add(v[3], v[0], &v[3]));
    CK(sub(v[2], v[1], &v[2]));
    first = v[3] >> 1;
    second = v[2] >> 1;
    CK(sub(v[0], first, &v[0]));
    CK(add(v[1], second, &v[1]));
    CK(mul3_add_shr(v[1], 3, 3, &t)); CK(sub(v[0], t, &v[0]));
    CK(mul3_add_shr(v[0], 3, 2, &t)); CK(add(v[1], t, &v[1]));
    CK(mul3_add_shr(v[1], 4, 3, &t)); CK(sub(v[0], t, &v[0]));
    CK(sub(v[1], second, &v[1]));
    CK(add(v[0], first, &v[0]));
    CK(add(v[2], v[1], &v[2]));
    CK(sub(v[3], v[0], &v[3]));
    CK(neg(v[1], &v[1]));
    CK(neg(v[2], &v[2]));
    return JO_OK;
}

typedef int (*op4)(int32_t v[4]);
static int t2x2h_round(int32_t v[4]) { return t2x2h(v, 1); }
static int t2x2h_zero(int32_t v[4]) { return t2x2h(v, 0); }

/* transform_group, transform.rs:152-169 */
static int group4(int32_t *c, int a, int b, int d, int e, op4 op)
{
    int32_t v[4] = {c[a], c[b], c[d], c[e]};
    int rc = op(v);
    if (rc) return rc;
    c[a] = v[0]; c[b] = v[1]; c[d] = v[2]; c[e] = v[3];
    return JO_OK;
}

/* inverse_core_transform, transform.rs:8-22 (permutation 171-192) */
int jo_inverse_core_transform(int32_t c[16])
{
    int32_t in[16];
    memcpy(in, c, sizeof in);
    for (int i = 0; i < 16; i++) c[INVERSE_PERMUTATION[i]] = in[i];
    CK(group4(c, 0, 1, 4, 5, t2x2h_round));
    CK(group4(c, 2, 3, 6, 7, inverse_todd));
    CK(group4(c, 8, 12, 9, 13, inverse_todd));
    CK(group4(c, 10, 11, 14, 15, inverse_todd_odd));
    CK(group4(c, 0, 3, 12, 15, t2x2h_zero));
    CK(group4(c, 5, 6, 9, 10, t2x2h_zero));
    CK(group4(c, 1, 2, 13, 14, t2x2h_zero));
    CK(group4(c, 4, 7, 8, 11, t2x2h_zero));
    return JO_OK;
}

/* inverse_chroma_420, transform.rs:52-56 */
int jo_inverse_chroma_420(int32_t c[4])
{
    int32_t t;
    CK(t2x2h(c, 0));
    t = c[1]; c[1] = c[2]; c[2] = t;
    return JO_OK;
}

/* inverse_t2pt, transform.rs:128-135 */
static int inverse_t2pt(int32_t v[2])
{
    int32_t t;
    CK(add_shr(v[1], 1, 1, &t));
    CK(sub(v[0], t, &v[0]));
    CK(add(v[1], v[0], &v[1]));
    return JO_OK;
}

/* inverse_chroma_422, transform.rs:60-89 */
int jo_inverse_chroma_422(int32_t c[8])
{
    int32_t pair[2] = {c[0], c[4]}, t;
    CK(inverse_t2pt(pair));
    c[0] = pair[0]; c[4] = pair[1];
    int32_t first[4] = {c[0], c[1], c[2], c[3]};
    CK(t2x2h(first, 0));
    memcpy(c, first, sizeof first);
    t = c[1]; c[1] = c[2]; c[2] = t;
    int32_t second[4] = {c[4], c[6], c[5], c[7]};
    CK(t2x2h(second, 0));
    c[4] = second[0]; c[6] = second[1]; c[5] = second[2]; c[7] = second[3];
    t = c[5]; c[5] = c[6]; c[6] = t;
    return JO_OK;
}

/* ------------------------------------------------------------------------ */
/* overlap operators: crates/jxr-math/src/overlap.rs                         */
/* ------------------------------------------------------------------------ */

/* inverse_rotate, overlap.rs:285-295 */
static int inverse_rotate(int32_t v[2])
{
    int32_t t;
    CK(add_shr(v[1], 1, 1, &t)); CK(sub(v[0], t, &v[0]));
    CK(add_shr(v[0], 1, 1, &t)); CK(add(v[1], t, &v[1]));
    return JO_OK;
}

/* inverse_scale, overlap.rs:377-391 */
static int inverse_scale(int32_t v[2])
{
    int32_t t;
    CK(add(v[0], v[1], &v[0]));
    CK(sub(v[0] >> 1, v[1], &v[1]));
    CK(mul(v[1], 3, &t)); CK(add(v[0], t >> 3, &v[0]));
    CK(mul(v[0], 3, &t)); CK(add(v[1], t >> 4, &v[1]));
    CK(add(v[1], v[0] >> 7, &v[1]));
    CK(sub(v[1], v[0] >> 10, &v[1]));
    return JO_OK;
}

/* inverse_overlap_filter_4, overlap.rs:10-55 */
int jo_inverse_overlap_4(int32_t v[4])
{
    int32_t t, pair[2];
    CK(add(v[0], v[3], &v[0]));
    CK(add(v[1], v[2], &v[1]));
    CK(add_shr(v[0], 1, 1, &t)); CK(sub(v[3], t, &v[3]));
    CK(add_shr(v[1], 1, 1, &t)); CK(sub(v[2], t, &v[2]));
    pair[0] = v[0]; pair[1] = v[3]; CK(inverse_scale(pair)); v[0] = pair[0]; v[3] = pair[1];
    pair[0] = v[1]; pair[1] = v[2]; CK(inverse_scale(pair)); v[1] = pair[0]; v[2] = pair[1];
    CK(mul3_add_shr(v[3], 4, 3, &t)); CK(add(v[0], t, &v[0]));
    CK(mul3_add_shr(v[2], 4, 3, &t)); CK(add(v[1], t, &v[1]));
    CK(sub(v[3], v[0] >> 1, &v[3]));
    CK(sub(v[2], v[1] >> 1, &v[2]));
    CK(add(v[0], v[3], &v[0]));
    CK(add(v[1], v[2], &v[1]));
    CK(neg(v[3], &v[3]));
    CK(neg(v[2], &v[2]));
    pair[0] = v[2]; pair[1] = v[3]; CK(inverse_rotate(pair)); v[2] = pair[0]; v[3] = pair[1];
    CK(add_shr(v[0], 1, 1, &t)); CK(add(v[3], t, &v[3]));
    CK(add_shr(v[1], 1, 1, &t)); CK(add(v[2], t, &v[2]));
    CK(sub(v[0], v[3], &v[0]));
    CK(sub(v[1], v[2], &v[1]));
    return JO_OK;
}

/* inverse_hadamard_post, overlap.rs:394-409 */
static int inverse_hadamard_post(int32_t v[4])
{
    int32_t t;
    CK(sub(v[1], v[2], &v[1]));
    CK(mul3_add_shr(v[3], 4, 3, &t)); CK(add(v[0], t, &v[0]));
    CK(sub(v[3], v[1] >> 1, &v[3]));
    CK(sub(v[0], v[1], &t)); CK(sub(t >> 1, v[2], &v[2]));
    t = v[2]; v[2] = v[3]; v[3] = t;
    CK(sub(v[0], v[3], &v[0]));
    CK(add(v[1], v[2], &v[1]));
    return JO_OK;
}

/* inverse_todd_odd_post, overlap.rs:412-436 */
static int inverse_todd_odd_post(int32_t v[4])
{
    int32_t t, first, second;
    CK(add(v[3], v[0], &v[3]));
    CK(sub(v[2], v[1], &v[2]));
    first = v[3] >> 1;
    second = v[2] >> 1;
    CK(sub(v[0], first, &v[0]));
    CK(add(v[1], second, &v[1]));
    CK(mul3_add_shr(v[1], 6, 3, &t)); CK(sub(v[0], t, &v[0]));
    CK(mul3_add_shr(v[0], 2, 2, &t)); CK(add(v[1], t, &v[1]));
    CK(mul3_add_shr(v[1], 4, 3, &t)); CK(sub(v[0], t, &v[0]));
    CK(sub(v[1], second, &v[1]));
    CK(add(v[0], first, &v[0]));
    CK(add(v[2], v[1], &v[2]));
    CK(sub(v[3], v[0], &v[3]));
    return JO_OK;
}

static int pair2(int32_t *c, int a, int b, int (*op)(int32_t v[2]))
{
    int32_t v[2] = {c[a], c[b]};
    int rc = op(v);
    if (rc) return rc;
    c[a] = v[0]; c[b] = v[1];
    return JO_OK;
}

/* inverse_overlap_filter_4x4, overlap.rs:139-161 */
int jo_inverse_overlap_4x4(int32_t c[16])
{
    static const int groups[4][4] = {{0, 3, 12, 15}, {1, 2, 13, 14}, {4, 7, 8, 11}, {5, 6, 9, 10}};
    static const int rotations[4][2] = {{13, 12}, {9, 8}, {7, 3}, {6, 2}};
    static const int scales[4][2] = {{0, 15}, {1, 14}, {4, 11}, {5, 10}};
    for (int i = 0; i < 4; i++) CK(group4(c, groups[i][0], groups[i][1], groups[i][2], groups[i][3], t2x2h_zero));
    for (int i = 0; i < 4; i++) CK(pair2(c, rotations[i][0], rotations[i][1], inverse_rotate));
    CK(group4(c, 10, 11, 14, 15, inverse_todd_odd_post));
    for (int i = 0; i < 4; i++) CK(pair2(c, scales[i][0], scales[i][1], inverse_scale));
    for (int i = 0; i < 4; i++) CK(group4(c, groups[i][0], groups[i][1], groups[i][2], groups[i][3], inverse_hadamard_post));
    return JO_OK;
}

/* inverse_overlap_filter_2x2, overlap.rs:167-204 */
int jo_inverse_overlap_2x2(int32_t v[4])
{
    int32_t t;
    CK(add(v[0], v[3], &v[0]));
    CK(add(v[1], v[2], &v[1]));
    CK(add_shr(v[0], 1, 1, &t)); CK(sub(v[3], t, &v[3]));
    CK(add_shr(v[1], 1, 1, &t)); CK(sub(v[2], t, &v[2]));
    CK(add_shr(v[0], 2, 2, &t)); CK(add(v[1], t, &v[1]));
    CK(add_shr(v[1], 1, 1, &t)); CK(add(v[0], t, &v[0]));
    CK(add(v[0], v[1] >> 5, &v[0]));
    CK(add(v[0], v[1] >> 9, &v[0]));
    CK(add(v[0], v[1] >> 13, &v[0]));
    CK(add_shr(v[0], 2, 2, &t)); CK(add(v[1], t, &v[1]));
    CK(add_shr(v[0], 1, 1, &t)); CK(add(v[3], t, &v[3]));
    CK(add_shr(v[1], 1, 1, &t)); CK(add(v[2], t, &v[2]));
    CK(sub(v[0], v[3], &v[0]));
    CK(sub(v[1], v[2], &v[1]));
    return JO_OK;
}

/* inverse_overlap_filter_2, overlap.rs:210-227 */
int jo_inverse_overlap_2(int32_t v[2])
{
    int32_t t;
    CK(add_shr(v[0], 2, 2, &t)); CK(add(v[1], t, &v[1]));
    CK(add_shr(v[1], 1, 1, &t)); CK(add(v[0], t, &v[0]));
    CK(add(v[0], v[1] >> 5, &v[0]));
    CK(add(v[0], v[1] >> 9, &v[0]));
    CK(add(v[0], v[1] >> 13, &v[0]));
    CK(add_shr(v[0], 2, 2, &t)); CK(add(v[1], t, &v[1]));
    return JO_OK;
}

/* ------------------------------------------------------------------------ */
/* quantization and prediction                                               */
/* ------------------------------------------------------------------------ */

/* Quantizer::dequantize, crates/jxr-math/src/quantization.rs:53-56 */
int jo_dequantize(int32_t coefficient, uint32_t step, int32_t *out)
{
    int64_t w = (int64_t)coefficient * (int64_t)step;
    if (w < INT32_MIN || w > INT32_MAX) return JO_ERR_OVERFLOW;
    *out = (int32_t)w;
    return JO_OK;
}

/* predict_geometry / predict_block, crates/jxr-math/src/prediction.rs:110-154;
 * the top-left direction is rejected as crates/jxr-native/src/decode/reconstruction.rs:464-496 does. */
int jo_predict_high_pass(int32_t c[256], int direction, int columns, int rows)
{
    if (direction == 0) return JO_OK;
    if (direction == 1) {
        for (int row = 0; row < rows; row++)
            for (int column = 1; column < columns; column++) {
                int block = row * columns + column;
                for (int p = 4; p <= 12; p += 4)
                    CK(add(c[block * 16 + p], c[(block - 1) * 16 + p], &c[block * 16 + p]));
            }
        return JO_OK;
    }
    if (direction == 2) {
        for (int row = 1; row < rows; row++)
            for (int column = 0; column < columns; column++) {
                int block = row * columns + column;
                for (int p = 1; p <= 3; p++)
                    CK(add(c[block * 16 + p], c[(block - columns) * 16 + p], &c[block * 16 + p]));
            }
        return JO_OK;
    }
    return JO_ERR_INVALID;
}

/* ------------------------------------------------------------------------ */
/* chroma interpolation: crates/jxr-math/src/sampling.rs:26-58, 105-115      */
/* ------------------------------------------------------------------------ */
static const int32_t CENTERING_WEIGHTS[5][4] = {
    {4, 4, 0, 8}, {5, 3, 1, 7}, {6, 2, 2, 6}, {7, 1, 3, 5}, {8, 0, 4, 4}};

/* (first*w1 + second*w2 + 4) >> 3 computed in 64 bits; the result always lies
 * between the two samples, which is what weighted_pair (sampling.rs:105-115)
 * computes with split 32-bit arithmetic. */
static int32_t weighted_pair(int32_t first, int32_t w1, int32_t second, int32_t w2)
{
    int64_t s = (int64_t)first * w1 + (int64_t)second * w2 + 4;
    return (int32_t)(s >> 3);
}

int jo_upsample_pair(int32_t previous, int32_t current, int32_t next, int centering, int32_t out[2])
{
    if (centering < 0 || centering > 4) return JO_ERR_UNSUPPORTED;
    const int32_t *h = CENTERING_WEIGHTS[centering];
    out[0] = weighted_pair(previous, h[2], current, h[3]);
    out[1] = weighted_pair(current, h[0], next, h[1]);
    return JO_OK;
}

/* ------------------------------------------------------------------------ */
/* RGBE and alpha: crates/jxr-math/src/rgbe.rs:7-101, alpha.rs:6-54          */
/* ------------------------------------------------------------------------ */
void jo_postscale_rgbe(const int32_t rgb[3], uint8_t out[4])
{
    int32_t mant[3], expo[3], e = 0;
    for (int i = 0; i < 3; i++) {
        int32_t v = rgb[i];
        if (v <= 0) { mant[i] = 0; expo[i] = 0; }
        else if ((v >> 7) > 1) { mant[i] = (v & 0x7f) + 128; expo[i] = v >> 7; }
        else { mant[i] = v; expo[i] = 1; }
        if (expo[i] > e) e = expo[i];
    }
    for (int i = 0; i < 3; i++) {
        int32_t v = mant[i];
        if (e > expo[i]) {
            int32_t d = e - expo[i];
            v = d >= 31 ? 0 : (int32_t)(((int64_t)2 * v + 1) >> (d + 1));
        }
        out[i] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
    }
    out[3] = (uint8_t)(e > 255 ? 255 : e);
}

int jo_premultiply_unsigned(uint32_t value, uint32_t alpha, uint32_t maximum, uint32_t *out)
{
    if (maximum == 0) return JO_ERR_OVERFLOW;
    if (value > maximum) value = maximum;
    if (alpha > maximum) alpha = maximum;
    uint64_t r = ((uint64_t)value * alpha + maximum / 2) / maximum;
    if (r > UINT32_MAX) return JO_ERR_OVERFLOW;
    *out = (uint32_t)r;
    return JO_OK;
}

int jo_premultiply_signed(int32_t value, int32_t alpha, int32_t maximum, int32_t *out)
{
    if (maximum <= 0) return JO_ERR_OVERFLOW;
    if (alpha < 0) alpha = 0;
    if (alpha > maximum) alpha = maximum;
    uint64_t magnitude = value < 0 ? (uint64_t)(-(int64_t)value) : (uint64_t)value;
    uint64_t r = (magnitude * (uint64_t)alpha + (uint64_t)maximum / 2) / (uint64_t)maximum;
    if (r > (uint64_t)INT64_MAX) return JO_ERR_OVERFLOW;
    int64_t s = value < 0 ? -(int64_t)r : (int64_t)r;
    if (s < INT32_MIN || s > INT32_MAX) return JO_ERR_OVERFLOW;
    *out = (int32_t)s;
    return JO_OK;
}

int jo_premultiply_sign_magnitude_15(uint16_t value, uint16_t alpha, uint16_t *out)
{
    uint32_t a = (alpha & 0x8000) ? 0 : (alpha & 0x7fff), m;
    int rc = jo_premultiply_unsigned(value & 0x7fff, a, 0x7fff, &m);
    if (rc) return rc;
    *out = (uint16_t)((value & 0x8000) | m);
    return JO_OK;
}

float jo_premultiply_f32(float value, float alpha)
{
    /* f32::clamp(0.0, 1.0): NaN stays NaN */
    float a = alpha;
    if (a < 0.0f) a = 0.0f;
    if (a > 1.0f) a = 1.0f;
    return value * a;
}

/* Exact binary16 -> binary32 widening of a half bit pattern, NaN payloads and
 * subnormals preserved (IEEE 754 format conversion, done on the bits). */
uint32_t jo_widen_f16(uint16_t h)
{
    uint32_t sign = (uint32_t)(h & 0x8000) << 16;
    uint32_t exponent = (h >> 10) & 0x1f;
    uint32_t mantissa = h & 0x3ff;
    if (exponent == 0x1f) return sign | 0x7f800000u | (mantissa << 13);
    if (exponent != 0) return sign | ((exponent + 112) << 23) | (mantissa << 13);
    if (mantissa == 0) return sign;
    int e = 113;
    while (!(mantissa & 0x400)) { mantissa <<= 1; e--; }
    return sign | ((uint32_t)e << 23) | ((mantissa & 0x3ff) << 13);
}

/* ------------------------------------------------------------------------ */
/* plane reconstruction                                                      */
/* ------------------------------------------------------------------------ */

void jo_plane_extent(const jo_plane *p, uint32_t *w, uint32_t *h)
{
    *w = p->macroblocks_x * p->block_columns * 4;
    *h = p->macroblocks_y * p->block_rows * 4;
}

typedef struct { uint32_t left, right, top, bottom; } region_t;

/* The regions an overlap schedule filters on its own: each tile when the
 * boundaries are hard, the whole plane otherwise
 * (crates/jxr-native/src/reconstruct/overlap.rs:52-62,
 *  crates/jxr-core/src/device_plan/overlap.rs:65-100). */
static int build_regions(const jo_plane *p, uint32_t hscale, uint32_t vscale, region_t **out, int *count)
{
    if (!p->hard_tiles) {
        region_t *r = malloc(sizeof *r);
        if (!r) return JO_ERR_INVALID;
        r->left = 0; r->right = p->macroblocks_x * hscale;
        r->top = 0; r->bottom = p->macroblocks_y * vscale;
        *out = r; *count = 1;
        return JO_OK;
    }
    int nc = (int)p->column_boundary_count - 1, nr = (int)p->row_boundary_count - 1;
    if (nc < 1 || nr < 1) return JO_ERR_INVALID;
    region_t *r = malloc(sizeof *r * (size_t)nc * (size_t)nr);
    if (!r) return JO_ERR_INVALID;
    int n = 0;
    for (int j = 0; j < nr; j++)
        for (int i = 0; i < nc; i++) {
            r[n].left = p->column_boundaries[i] * hscale;
            r[n].right = p->column_boundaries[i + 1] * hscale;
            r[n].top = p->row_boundaries[j] * vscale;
            r[n].bottom = p->row_boundaries[j + 1] * vscale;
            n++;
        }
    *out = r; *count = n;
    return JO_OK;
}

static int filter4_at(int32_t *s, size_t i0, size_t i1, size_t i2, size_t i3)
{
    int32_t v[4] = {s[i0], s[i1], s[i2], s[i3]};
    int rc = jo_inverse_overlap_4(v);
    if (rc) return rc;
    s[i0] = v[0]; s[i1] = v[1]; s[i2] = v[2]; s[i3] = v[3];
    return JO_OK;
}

/* Full-resolution overlap schedule of one region: interior 4x4 windows at
 * (left+2+4i, top+2+4j), four-sample edge strips in the columns
 * left, left+1, right-2, right-1 and the rows top, top+1, bottom-2, bottom-1,
 * and 2x2 corners through the four-sample operator.
 * crates/jxr-native/src/reconstruct/overlap.rs:124-323 (whole-plane strip);
 * crates/jxr-core/src/device_plan/overlap.rs:125-178 (the same window list).
 * The windows are disjoint, so the order they run in does not matter. */
static int full_region(int32_t *s, size_t stride, region_t g, int threads)
{
    int err = 0;
    long rows = 0;
    for (uint32_t y = g.top + 2; y + 2 < g.bottom; y += 4) rows++;
    (void)threads;
#pragma omp parallel for schedule(static) num_threads(threads) reduction(|:err) if (threads > 1)
    for (long j = 0; j < rows; j++) {
        uint32_t y = g.top + 2 + 4 * (uint32_t)j;
        for (uint32_t x = g.left + 2; x + 2 < g.right; x += 4) {
            int32_t v[16];
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) v[r * 4 + c] = s[(y + r) * stride + x + c];
            if (jo_inverse_overlap_4x4(v)) { err = 1; continue; }
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) s[(y + r) * stride + x + c] = v[r * 4 + c];
        }
        uint32_t xs[4] = {g.left, g.left + 1, g.right - 2, g.right - 1};
        for (int k = 0; k < 4; k++)
            err |= filter4_at(s, y * stride + xs[k], (y + 1) * stride + xs[k],
                              (y + 2) * stride + xs[k], (y + 3) * stride + xs[k]) != 0;
    }
    if (err) return JO_ERR_OVERFLOW;
    uint32_t ys[4] = {g.top, g.top + 1, g.bottom - 2, g.bottom - 1};
    for (uint32_t x = g.left + 2; x + 2 < g.right; x += 4)
        for (int k = 0; k < 4; k++) {
            size_t o = (size_t)ys[k] * stride + x;
            CK(filter4_at(s, o, o + 1, o + 2, o + 3));
        }
    uint32_t cx[4] = {g.left, g.right - 2, g.left, g.right - 2};
    uint32_t cy[4] = {g.top, g.top, g.bottom - 2, g.bottom - 2};
    for (int k = 0; k < 4; k++) {
        size_t o = (size_t)cy[k] * stride + cx[k];
        CK(filter4_at(s, o, o + 1, o + stride, o + stride + 1));
    }
    return JO_OK;
}

/* One boundary row of a subsampled region: each corner loses its row
 * neighbour, the two-sample windows along the row are filtered, and each
 * corner regains the neighbour's filtered value.
 * crates/jxr-native/src/reconstruct/subsampled_overlap.rs:257-272 */
static int subsampled_boundary_row(int32_t *s, size_t stride, region_t g, uint32_t row)
{
    size_t base = (size_t)row * stride;
    size_t c0 = base + g.left, n0 = base + g.left + 1;
    size_t c1 = base + g.right - 1, n1 = base + g.right - 2;
    CK(sub(s[c0], s[n0], &s[c0]));
    CK(sub(s[c1], s[n1], &s[c1]));
    for (uint32_t x = g.left + 2; x < g.right; x += 2) {
        int32_t v[2] = {s[base + x - 1], s[base + x]};
        CK(jo_inverse_overlap_2(v));
        s[base + x - 1] = v[0]; s[base + x] = v[1];
    }
    CK(add(s[c0], s[n0], &s[c0]));
    CK(add(s[c1], s[n1], &s[c1]));
    return JO_OK;
}

/* The decoder's subsampled first-level schedule of one region, first step to
 * last: the first row, then each pair of rows (y-1, y) for y = top+2, top+4, ...
 * with its 2x2 windows and two side pairs, then the last row.
 * crates/jxr-native/src/reconstruct/subsampled_overlap.rs:244-296 */
static int subsampled_region(int32_t *s, size_t stride, region_t g)
{
    CK(subsampled_boundary_row(s, stride, g, g.top));
    for (uint32_t y = g.top + 2; y < g.bottom; y += 2) {
        for (uint32_t x = g.left + 2; x < g.right; x += 2) {
            size_t a = (size_t)(y - 1) * stride + x - 1, b = (size_t)y * stride + x - 1;
            int32_t v[4] = {s[a], s[a + 1], s[b], s[b + 1]};
            CK(jo_inverse_overlap_2x2(v));
            s[a] = v[0]; s[a + 1] = v[1]; s[b] = v[2]; s[b + 1] = v[3];
        }
        uint32_t xs[2] = {g.left, g.right - 1};
        for (int k = 0; k < 2; k++) {
            size_t a = (size_t)(y - 1) * stride + xs[k], b = (size_t)y * stride + xs[k];
            int32_t v[2] = {s[a], s[b]};
            CK(jo_inverse_overlap_2(v));
            s[a] = v[0]; s[b] = v[1];
        }
    }
    CK(subsampled_boundary_row(s, stride, g, g.bottom - 1));
    return JO_OK;
}

/* Regions of a sample plane from its tile boundaries in samples (first 0,
 * last the extent): each tile when hard, the whole plane otherwise. */
static int sample_regions(uint32_t width, uint32_t height, const uint32_t *cols, uint32_t ncols,
                          const uint32_t *rows, uint32_t nrows, int hard, region_t **out, int *count)
{
    if (ncols < 2 || nrows < 2 || cols[0] != 0 || rows[0] != 0 || cols[ncols - 1] != width ||
        rows[nrows - 1] != height)
        return JO_ERR_INVALID;
    for (uint32_t i = 1; i < ncols; i++) if (cols[i - 1] >= cols[i]) return JO_ERR_INVALID;
    for (uint32_t i = 1; i < nrows; i++) if (rows[i - 1] >= rows[i]) return JO_ERR_INVALID;
    int n = hard ? (int)((ncols - 1) * (nrows - 1)) : 1;
    region_t *r = malloc(sizeof *r * (size_t)n);
    if (!r) return JO_ERR_INVALID;
    if (!hard) {
        r[0].left = 0; r[0].right = width; r[0].top = 0; r[0].bottom = height;
    } else {
        int k = 0;
        for (uint32_t j = 0; j + 1 < nrows; j++)
            for (uint32_t i = 0; i + 1 < ncols; i++) {
                r[k].left = cols[i]; r[k].right = cols[i + 1];
                r[k].top = rows[j]; r[k].bottom = rows[j + 1];
                k++;
            }
    }
    *out = r; *count = n;
    return JO_OK;
}

int jo_apply_overlap(int32_t *samples, uint32_t width, uint32_t height, const uint32_t *column_boundaries,
                     uint32_t column_count, const uint32_t *row_boundaries, uint32_t row_count, int hard)
{
    /* apply_overlap::<Postfilter>, crates/jxr-native/src/reconstruct/overlap.rs:72-89 */
    region_t *regions = NULL;
    int count = 0;
    int rc = sample_regions(width, height, column_boundaries, column_count, row_boundaries, row_count, hard,
                            &regions, &count);
    for (int i = 0; rc == JO_OK && i < count; i++) rc = full_region(samples, width, regions[i], 1);
    free(regions);
    return rc;
}

int jo_apply_subsampled_first_overlap(int32_t *samples, uint32_t width, uint32_t height,
                                      const uint32_t *column_boundaries, uint32_t column_count,
                                      const uint32_t *row_boundaries, uint32_t row_count, int hard)
{
    /* apply_subsampled_first_overlap::<Postfilter>,
     * crates/jxr-native/src/reconstruct/subsampled_overlap.rs:110-296 */
    region_t *regions = NULL;
    int count = 0;
    int rc = sample_regions(width, height, column_boundaries, column_count, row_boundaries, row_count, hard,
                            &regions, &count);
    for (int i = 0; rc == JO_OK && i < count; i++) rc = subsampled_region(samples, width, regions[i]);
    free(regions);
    return rc;
}

int jo_full_schedule(uint32_t width, uint32_t height, const uint32_t *column_boundaries, uint32_t column_count,
                     const uint32_t *row_boundaries, uint32_t row_count, int hard, uint32_t *offsets,
                     uint32_t *steps, uint32_t *kinds, uint32_t capacity, uint32_t *count)
{
    /* full_schedule, crates/jxr-core/src/device_plan/overlap.rs:125-178: per
     * region, the 4x4 windows (kind 0) row by row, then the column edge
     * strips at left, left+1, right-2, right-1 (kind 1, step = stride), the
     * row edge strips at top, top+1, bottom-2, bottom-1 (kind 1, step 1), and
     * the four corners (kind 2); `offsets` hold each operator's first
     * sample. */
    region_t *regions = NULL;
    int nreg = 0;
    int rc = sample_regions(width, height, column_boundaries, column_count, row_boundaries, row_count, hard,
                            &regions, &nreg);
    if (rc) return rc;
    uint32_t n = 0;
#define PUSH(x, y, st, kd) do { if (n < capacity) { offsets[n] = (y) * width + (x); steps[n] = (st); kinds[n] = (kd); } n++; } while (0)
    for (int i = 0; i < nreg; i++) {
        region_t g = regions[i];
        for (uint32_t y = g.top + 2; y + 2 < g.bottom; y += 4)
            for (uint32_t x = g.left + 2; x + 2 < g.right; x += 4) PUSH(x, y, width, 0u);
        for (uint32_t y = g.top + 2; y + 2 < g.bottom; y += 4) {
            uint32_t xs[4] = {g.left, g.left + 1, g.right - 2, g.right - 1};
            for (int k = 0; k < 4; k++) PUSH(xs[k], y, width, 1u);
        }
        for (uint32_t x = g.left + 2; x + 2 < g.right; x += 4) {
            uint32_t ys[4] = {g.top, g.top + 1, g.bottom - 2, g.bottom - 1};
            for (int k = 0; k < 4; k++) PUSH(x, ys[k], 1u, 1u);
        }
        uint32_t cx[4] = {g.left, g.right - 2, g.left, g.right - 2};
        uint32_t cy[4] = {g.top, g.top, g.bottom - 2, g.bottom - 2};
        for (int k = 0; k < 4; k++) PUSH(cx[k], cy[k], width, 2u);
    }
#undef PUSH
    free(regions);
    *count = n;
    return n <= capacity ? JO_OK : JO_ERR_INVALID;
}

static size_t coefficients_per_macroblock(int bands, uint32_t block_count)
{
    /* crates/jxr-native/src/tile_decode/output.rs (PlaneWriter::push) and
     * decode/reconstruction.rs:587-613: DC only 1, no high-pass one per block,
     * otherwise sixteen per block. */
    if (bands == JO_BANDS_DC_ONLY) return 1;
    if (bands == JO_BANDS_NO_HIGH_PASS) return block_count;
    return (size_t)block_count * 16;
}

/* One macroblock: unpack (decode/reconstruction.rs:587-613), high-pass
 * prediction (464-496), dequantize and first-level transform
 * (reconstruct/pipeline.rs:605-680), place the block DCs (593-603) and the
 * dequantized high-pass coefficients (543-586). */
static int place_macroblock(const jo_plane *p, uint32_t mx, uint32_t my, int32_t *low, size_t low_width,
                            int32_t *samples, size_t width)
{
    uint32_t bc = p->block_columns, br = p->block_rows, count = bc * br;
    size_t index = (size_t)my * p->macroblocks_x + mx;
    size_t offset = p->offsets[index];
    int bands = p->bands[index];
    if (bands < 0 || bands > 3) return JO_ERR_INVALID;
    size_t need = coefficients_per_macroblock(bands, count);
    if (offset > p->coefficient_count || need > p->coefficient_count - offset) return JO_ERR_INVALID;
    const int32_t *packed = p->coefficients + offset;
    const uint32_t *q = p->quantizers + index * 3;
    if (q[0] == 0 || q[1] == 0 || q[2] == 0) return JO_ERR_INVALID; /* ZeroQuantizer */
    int32_t lowq[16] = {0};
    int32_t high[256];
    memset(high, 0, sizeof high);
    if (bands == JO_BANDS_DC_ONLY) {
        lowq[0] = packed[0];
    } else if (bands == JO_BANDS_NO_HIGH_PASS) {
        for (uint32_t b = 0; b < count; b++) lowq[b] = packed[b];
    } else {
        for (uint32_t b = 0; b < count; b++) {
            lowq[b] = packed[b * 16];
            for (int k = 1; k < 16; k++) high[b * 16 + k] = packed[b * 16 + k];
        }
    }
    int rc = jo_predict_high_pass(high, p->hp_prediction[index], (int)bc, (int)br);
    if (rc) return rc;
    int32_t l[16] = {0};
    CK(jo_dequantize(lowq[0], q[0], &l[0]));
    if (bands != JO_BANDS_DC_ONLY)
        for (uint32_t b = 1; b < count; b++) CK(jo_dequantize(lowq[b], q[1], &l[b]));
    if (bc == 4 && br == 4) {
        CK(jo_inverse_core_transform(l));
    } else if (bc == 2 && br == 4) {
        CK(jo_inverse_chroma_422(l));
    } else if (bc == 2 && br == 2) {
        CK(jo_inverse_chroma_420(l));
    } else {
        return JO_ERR_INVALID;
    }
    if (p->scale_after_first_transform)
        for (uint32_t b = 0; b < count; b++) CK(mul(l[b], 2, &l[b]));
    for (uint32_t r = 0; r < br; r++)
        for (uint32_t c = 0; c < bc; c++)
            low[((size_t)my * br + r) * low_width + (size_t)mx * bc + c] = l[r * bc + c];
    return jo_place_high_pass(high, q[2], bands, bc, br, samples + (size_t)my * br * 4 * width, width,
                              (size_t)mx * bc);
}

int jo_place_high_pass(const int32_t high[256], uint32_t step, int bands, uint32_t block_columns,
                       uint32_t block_rows, int32_t *rows, size_t width, size_t column)
{
    /* dequantize_high_pass_into, crates/jxr-native/src/reconstruct/pipeline.rs:543-586:
     * block b's coefficient k at row (b / columns)*4 + k/4, column
     * (column + b % columns)*4 + k%4, as its checked product with the step;
     * element zero of every block (the block DC's place) and every element
     * of a macroblock without a coded high-pass band are zero. */
    if (step == 0) return JO_ERR_INVALID; /* ZeroQuantizer("high-pass") */
    uint32_t count = block_columns * block_rows;
    for (uint32_t b = 0; b < count; b++) {
        size_t oy = (size_t)(b / block_columns) * 4, ox = (column + b % block_columns) * 4;
        for (int k = 0; k < 16; k++) {
            int32_t v = 0;
            if (k != 0 && bands >= JO_BANDS_NO_FLEXBITS) CK(jo_dequantize(high[b * 16 + k], step, &v));
            rows[(oy + (size_t)(k >> 2)) * width + ox + (size_t)(k & 3)] = v;
        }
    }
    return JO_OK;
}

int jo_reconstruct_plane(const jo_plane *p, int32_t *samples, int threads)
{
    uint32_t bc = p->block_columns, br = p->block_rows;
    if (!((bc == 4 && br == 4) || (bc == 2 && br == 4) || (bc == 2 && br == 2))) return JO_ERR_INVALID;
    if (p->overlap < 0 || p->overlap > 2) return JO_ERR_INVALID;
    if (p->hard_tiles) {
        /* validate_partition, reconstruct/pipeline.rs:743-756 */
        const uint32_t *cb = p->column_boundaries, *rb = p->row_boundaries;
        uint32_t nc = p->column_boundary_count, nr = p->row_boundary_count;
        if (nc < 2 || nr < 2 || cb[0] != 0 || rb[0] != 0 || cb[nc - 1] != p->macroblocks_x ||
            rb[nr - 1] != p->macroblocks_y)
            return JO_ERR_INVALID;
        for (uint32_t i = 1; i < nc; i++) if (cb[i - 1] >= cb[i]) return JO_ERR_INVALID;
        for (uint32_t i = 1; i < nr; i++) if (rb[i - 1] >= rb[i]) return JO_ERR_INVALID;
    }
    size_t low_width = (size_t)p->macroblocks_x * bc, low_height = (size_t)p->macroblocks_y * br;
    size_t width = low_width * 4, height = low_height * 4;
    if (width == 0 || height == 0) return JO_OK;
    int32_t *low = malloc(sizeof *low * low_width * low_height);
    if (!low) return JO_ERR_INVALID;
    int err = 0;
    long mb_rows = (long)p->macroblocks_y;
#pragma omp parallel for schedule(static) num_threads(threads) reduction(|:err) if (threads > 1)
    for (long my = 0; my < mb_rows; my++)
        for (uint32_t mx = 0; mx < p->macroblocks_x; mx++) {
            int rc = place_macroblock(p, mx, (uint32_t)my, low, low_width, samples, width);
            if (rc) err |= rc;
        }
    if (err) { free(low); return (err & JO_ERR_INVALID) ? JO_ERR_INVALID : JO_ERR_OVERFLOW; }
    region_t *regions = NULL;
    int count = 0, rc = JO_OK;
    if (p->overlap == 2) {
        /* first level: StripPlan::filter_low, reconstruct/strip.rs:286-308 */
        rc = build_regions(p, bc, br, &regions, &count);
        for (int i = 0; rc == JO_OK && i < count; i++)
            rc = bc == 4 ? full_region(low, low_width, regions[i], threads)
                         : subsampled_region(low, low_width, regions[i]);
        free(regions);
        if (rc) { free(low); return rc; }
    }
    /* second-level transform: transform_macroblock_row, reconstruct/strip.rs:587-607 */
    long block_rows = (long)low_height;
#pragma omp parallel for schedule(static) num_threads(threads) reduction(|:err) if (threads > 1)
    for (long by = 0; by < block_rows; by++)
        for (size_t bx = 0; bx < low_width; bx++) {
            int32_t v[16];
            size_t o = (size_t)by * 4 * width + bx * 4;
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) v[r * 4 + c] = samples[o + (size_t)r * width + (size_t)c];
            v[0] = low[(size_t)by * low_width + bx];
            if (jo_inverse_core_transform(v)) { err = 1; continue; }
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) samples[o + (size_t)r * width + (size_t)c] = v[r * 4 + c];
        }
    free(low);
    if (err) return JO_ERR_OVERFLOW;
    if (p->overlap >= 1) {
        /* second level: StripPlan::filter_samples, reconstruct/strip.rs:313-328 */
        rc = build_regions(p, bc * 4, br * 4, &regions, &count);
        for (int i = 0; rc == JO_OK && i < count; i++) rc = full_region(samples, width, regions[i], threads);
        free(regions);
    }
    return rc;
}

/* widen_row / double_row / ChromaStrip::advance,
 * crates/jxr-native/src/reconstruct/chroma.rs:174-328: vertical interpolation
 * (4:2:0) from the rows above and below, then horizontal; the end samples
 * stand in for missing neighbours. */
static int widen_row(const int32_t *row, uint32_t width, int centering, int32_t *out)
{
    for (uint32_t i = 0; i < width; i++) {
        int32_t prev = row[i == 0 ? 0 : i - 1], next = row[i + 1 < width ? i + 1 : width - 1];
        CK(jo_upsample_pair(prev, row[i], next, centering, out + 2 * i) != JO_OK);
    }
    return JO_OK;
}

int jo_upsample_chroma(const int32_t *chroma, uint32_t width, uint32_t height, int sampling,
                       int centering_x, int centering_y, int32_t *out, int threads)
{
    if (centering_x < 0 || centering_x > 4) return JO_ERR_UNSUPPORTED;
    if (width == 0 || height == 0) return JO_OK;
    size_t ow = (size_t)width * 2;
    int err = 0;
    if (sampling == 2) {
#pragma omp parallel for schedule(static) num_threads(threads) reduction(|:err) if (threads > 1)
        for (long y = 0; y < (long)height; y++)
            err |= widen_row(chroma + (size_t)y * width, width, centering_x, out + (size_t)y * ow);
        return err ? JO_ERR_OVERFLOW : JO_OK;
    }
    if (sampling != 1) return JO_ERR_INVALID;
    if (centering_y < 0 || centering_y > 4) return JO_ERR_UNSUPPORTED;
#pragma omp parallel for schedule(static) num_threads(threads) reduction(|:err) if (threads > 1)
    for (long y = 0; y < (long)height; y++) {
        int32_t *even = malloc(sizeof(int32_t) * width * 2), *odd = even + width;
        if (!even) { err = 1; continue; }
        const int32_t *above = chroma + (size_t)(y == 0 ? 0 : y - 1) * width;
        const int32_t *row = chroma + (size_t)y * width;
        const int32_t *below = chroma + (size_t)((uint32_t)y + 1 < height ? y + 1 : height - 1) * width;
        for (uint32_t x = 0; x < width; x++) {
            int32_t pair[2];
            jo_upsample_pair(above[x], row[x], below[x], centering_y, pair);
            even[x] = pair[0]; odd[x] = pair[1];
        }
        err |= widen_row(even, width, centering_x, out + (size_t)(2 * y) * ow);
        err |= widen_row(odd, width, centering_x, out + (size_t)(2 * y + 1) * ow);
        free(even);
    }
    return err ? JO_ERR_OVERFLOW : JO_OK;
}

/* ------------------------------------------------------------------------ */
/* output formatting                                                         */
/* ------------------------------------------------------------------------ */

static int is_packed_depth(int d) { return d == JO_DEPTH_RGB555 || d == JO_DEPTH_RGB565 || d == JO_DEPTH_RGB101010; }

/* ChannelLayout::channel_count / has_alpha, crates/jxr-core/src/format.rs:76-100 */
static int layout_channels(int layout, int ncomp)
{
    switch (layout) {
    case JO_LAYOUT_LUMA: return 1;
    case JO_LAYOUT_LUMA_ALPHA: return 2;
    case JO_LAYOUT_YUV: case JO_LAYOUT_RGB: case JO_LAYOUT_BGR: return 3;
    case JO_LAYOUT_YUVA: case JO_LAYOUT_RGBX: case JO_LAYOUT_RGBA: case JO_LAYOUT_BGRX:
    case JO_LAYOUT_BGRA: case JO_LAYOUT_CMYK: return 4;
    case JO_LAYOUT_CMYKA: return 5;
    case JO_LAYOUT_NCOMPONENT: return ncomp;
    case JO_LAYOUT_NCOMPONENT_ALPHA: return ncomp + 1;
    }
    return 0;
}
static int layout_has_alpha(int layout)
{
    return layout == JO_LAYOUT_LUMA_ALPHA || layout == JO_LAYOUT_YUVA || layout == JO_LAYOUT_RGBA ||
           layout == JO_LAYOUT_BGRA || layout == JO_LAYOUT_CMYKA || layout == JO_LAYOUT_NCOMPONENT_ALPHA;
}

static size_t storage_bytes(int storage)
{
    switch (storage) {
    case JO_STORE_U8: return 1;
    case JO_STORE_U16: case JO_STORE_I16: case JO_STORE_F16: case JO_STORE_RGB555: case JO_STORE_RGB565: return 2;
    default: return 4;
    }
}

static int is_planar_yuv(const jo_output *r)
{
    return r->output_color == JO_COLOR_YUV420 || r->output_color == JO_COLOR_YUV422;
}

size_t jo_output_bytes(const jo_output *r)
{
    size_t w = r->crop_width, h = r->crop_height;
    if (r->storage == JO_STORE_BITS) return (w + 7) / 8 * h;
    if (r->storage >= JO_STORE_RGB555) return w * h * storage_bytes(r->storage);
    if (is_planar_yuv(r)) {
        size_t cw = w / 2, ch = r->output_color == JO_COLOR_YUV420 ? h / 2 : h;
        size_t n = w * h + 2 * cw * ch + (layout_has_alpha(r->layout) ? w * h : 0);
        return n * storage_bytes(r->storage);
    }
    size_t bytes = r->widen_f16 ? 4 : storage_bytes(r->storage);
    return w * h * (size_t)layout_channels(r->layout, r->ncomponents) * bytes;
}

/* One resolved channel scale: ChannelScale::resolve / apply,
 * crates/jxr-native/src/output_format/scaling.rs:37-119, bias 299-318,
 * saturating_shift_left 325-328. */
typedef struct { int padding; int32_t shifted_bias; int32_t rounding; int shift; int post_shift; int invalid; } scale_t;

static int depth_bias(int depth, int shift_bits, int32_t *bias)
{
    int32_t base = 0; int shift = 0;
    switch (depth) {
    case JO_DEPTH_RGB555: base = 1 << 4; break;
    case JO_DEPTH_RGB565: base = 1 << 5; break;
    case JO_DEPTH_U8: base = 1 << 7; break;
    case JO_DEPTH_U10: case JO_DEPTH_RGB101010: base = 1 << 9; break;
    case JO_DEPTH_U16: base = 1 << 15; shift = shift_bits; break;
    case JO_DEPTH_I16: case JO_DEPTH_I32: base = 0; shift = shift_bits; break;
    default: base = 0; break;
    }
    if (shift >= 32) return JO_ERR_UNSUPPORTED;
    *bias = base >> shift;
    return JO_OK;
}

static scale_t resolve_scale(int component, int output_color, int depth, int shift_bits, int scaled)
{
    scale_t s = {0};
    int32_t bias;
    if (depth_bias(depth, shift_bits, &bias)) { s.invalid = 1; return s; }
    int32_t cb = bias;
    if (output_color == JO_COLOR_CMYK) cb = component < 3 ? bias >> 1 : -(bias >> 1);
    else if (output_color == JO_COLOR_RGBE) cb = 0;
    int sc = scaled ? 3 : 0;
    int64_t shifted = (int64_t)cb * ((int64_t)1 << sc);
    if (shifted < INT32_MIN || shifted > INT32_MAX) { s.invalid = 1; return s; }
    s.shifted_bias = (int32_t)shifted;
    s.rounding = scaled ? ((depth == JO_DEPTH_BIT1_WHITE || depth == JO_DEPTH_BIT1_BLACK || depth == JO_DEPTH_U16) ? 4 : 3) : 0;
    s.shift = (depth == JO_DEPTH_RGB565 && component != 1) ? sc + 1 : sc;
    s.post_shift = (depth == JO_DEPTH_U16 || depth == JO_DEPTH_I16 || depth == JO_DEPTH_I32) ? shift_bits : -1;
    return s;
}

static int apply_scale(const scale_t *s, int32_t sample, int32_t *out)
{
    if (s->padding) { *out = 0; return JO_OK; }
    if (s->invalid) return JO_ERR_UNSUPPORTED;
    int32_t b, r;
    CK(add(sample, s->shifted_bias, &b));
    CK(add(b, s->rounding, &r));
    r >>= s->shift;
    if (s->post_shift >= 0) {
        int bits = s->post_shift < 31 ? s->post_shift : 31;
        int64_t w = (int64_t)r * ((int64_t)1 << bits);
        r = w > INT32_MAX ? INT32_MAX : w < INT32_MIN ? INT32_MIN : (int32_t)w;
    }
    *out = r;
    return JO_OK;
}

static int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : v > hi ? hi : v; }

/* float16_bits, scaling.rs:235-241 */
static int f16_bits(int32_t sample, int scaled, uint16_t *out)
{
    scale_t s = resolve_scale(0, JO_COLOR_LUMA, JO_DEPTH_F16, 0, scaled);
    int32_t v;
    int rc = apply_scale(&s, sample, &v);
    if (rc) return rc;
    uint32_t m = v < 0 ? (uint32_t)(-(int64_t)v) : (uint32_t)v;
    if (m > 32767) m = 32767;
    *out = (uint16_t)((v < 0 ? 0x8000 : 0) | m);
    return JO_OK;
}

/* float32_bits, scaling.rs:243-297: exponent overflow clips to the largest
 * finite value of the sign. */
static int f32_bits(int32_t sample, int scaled, int mantissa_length, int exponent_bias, uint32_t *out)
{
    if (mantissa_length > 23) return JO_ERR_UNSUPPORTED;
    scale_t s = resolve_scale(0, JO_COLOR_LUMA, JO_DEPTH_F32, 0, scaled);
    int32_t v;
    int rc = apply_scale(&s, sample, &v);
    if (rc) return rc;
    uint32_t sign = v < 0 ? 0x80000000u : 0;
    uint64_t magnitude = v < 0 ? (uint64_t)(-(int64_t)v) : (uint64_t)v;
    int length = mantissa_length;
    uint64_t implicit = (uint64_t)1 << length;
    int64_t exponent = (int64_t)(magnitude >> length);
    uint64_t mantissa = (magnitude & (implicit - 1)) | implicit;
    if (exponent == 0) { mantissa ^= implicit; exponent = 1; }
    exponent = exponent - exponent_bias + 127;
    while (mantissa < implicit && exponent > 1 && mantissa > 0) { exponent--; mantissa <<= 1; }
    if (mantissa < implicit) exponent = 0;
    else mantissa ^= implicit;
    mantissa <<= 23 - length;
    if (exponent < 0 || exponent > 255) { *out = sign | 0x7f7fffffu; return JO_OK; }
    if (mantissa > 0x7fffff) return JO_ERR_OVERFLOW;
    *out = sign | ((uint32_t)exponent << 23) | (uint32_t)mantissa;
    return JO_OK;
}

/* convert / inverse_yuv / inverse_yuvk, output_format/color.rs:9-125 */
static int convert_color(int internal, int output, const int32_t in[4], int packed_rgb, int rbns, int32_t out[4])
{
    int32_t t, g, r, b;
    if (internal == JO_COLOR_LUMA && output == JO_COLOR_LUMA) { out[0] = in[0]; out[1] = out[2] = out[3] = 0; return JO_OK; }
    if (internal == JO_COLOR_LUMA && output == JO_COLOR_RGB) { out[0] = out[1] = out[2] = in[0]; out[3] = 0; return JO_OK; }
    if (internal == JO_COLOR_YUV444 && (output == JO_COLOR_RGB || output == JO_COLOR_RGBE)) {
        CK(sub(0, in[1], &t));
        CK(sub(in[0], t >> 1, &g));
        CK(add(t, g, &r)); CK(sub(r, (in[2] >> 1) + (in[2] & 1), &r));
        CK(add(in[2], r, &b));
        if (packed_rgb && !rbns) { out[0] = b; out[2] = r; } else { out[0] = r; out[2] = b; }
        out[1] = g; out[3] = 0;
        return JO_OK;
    }
    if (internal == JO_COLOR_YUVK && output == JO_COLOR_CMYK) {
        int32_t k, m, c, y;
        CK(add(in[3], in[0] >> 1, &k));
        CK(sub(k, in[0], &m)); CK(sub(m, in[1] >> 1, &m));
        CK(add(in[1], m, &c)); CK(add(c, in[2] >> 1, &c));
        CK(sub(c, in[2], &y));
        out[0] = c; out[1] = m; out[2] = y; out[3] = k;
        return JO_OK;
    }
    if (internal == JO_COLOR_YUVK && output == JO_COLOR_CMYK_DIRECT) {
        out[0] = in[1]; out[1] = in[2]; out[2] = in[3]; out[3] = in[0];
        return JO_OK;
    }
    return JO_ERR_UNSUPPORTED;
}

static int is_direct(int internal, int output)
{
    /* packing.rs:696-701 */
    return (internal == JO_COLOR_LUMA && output == JO_COLOR_LUMA) ||
           (internal == output && (internal == JO_COLOR_YUV420 || internal == JO_COLOR_YUV422 || internal == JO_COLOR_YUV444)) ||
           (internal == JO_COLOR_NCOMPONENT && output == JO_COLOR_NCOMPONENT);
}

/* Primaries of each ordered pixel (packing.rs:560-585 PixelShape::primary_count). */
static int primary_count(const jo_output *r)
{
    switch (r->layout) {
    case JO_LAYOUT_LUMA: return 1;
    case JO_LAYOUT_YUV: case JO_LAYOUT_RGB: case JO_LAYOUT_BGR: return 3;
    case JO_LAYOUT_RGBX: case JO_LAYOUT_BGRX: case JO_LAYOUT_CMYK: case JO_LAYOUT_CMYKA: return 4;
    case JO_LAYOUT_NCOMPONENT: case JO_LAYOUT_NCOMPONENT_ALPHA: return r->ncomponents;
    default: return layout_channels(r->layout, r->ncomponents) - 1;
    }
}

/* validate_matrix, output_format/validate.rs:108-250 (the policy part). */
static int validate_request(const jo_output *r, int has_alpha)
{
    int layout = r->layout;
    if (r->storage >= JO_STORE_RGB555) layout = JO_LAYOUT_RGB;
    if (layout_has_alpha(layout) != has_alpha) return JO_ERR_INVALID;
    if (r->premultiply && !has_alpha) return JO_ERR_INVALID;
    if (r->premultiply && (r->output_color == JO_COLOR_YUV420 || r->output_color == JO_COLOR_YUV422 || r->output_color == JO_COLOR_YUV444))
        return JO_ERR_UNSUPPORTED;
    int d = r->depth, s = r->storage;
    int ok = ((d == JO_DEPTH_BIT1_WHITE || d == JO_DEPTH_BIT1_BLACK) && s == JO_STORE_BITS && r->layout == JO_LAYOUT_LUMA) ||
             (d == JO_DEPTH_U8 && (s == JO_STORE_U8 || s == JO_STORE_RGBE)) ||
             ((d == JO_DEPTH_U10 || d == JO_DEPTH_U16) && s == JO_STORE_U16) ||
             (d == JO_DEPTH_I16 && s == JO_STORE_I16) || (d == JO_DEPTH_I32 && s == JO_STORE_I32) ||
             (d == JO_DEPTH_F16 && s == JO_STORE_F16) || (d == JO_DEPTH_F32 && s == JO_STORE_F32) ||
             (d == JO_DEPTH_RGB555 && s == JO_STORE_RGB555) || (d == JO_DEPTH_RGB565 && s == JO_STORE_RGB565) ||
             (d == JO_DEPTH_RGB101010 && s == JO_STORE_RGB101010);
    if (!ok) return JO_ERR_UNSUPPORTED;
    int oc = r->output_color;
    switch (oc) {
    case JO_COLOR_LUMA: ok = layout == JO_LAYOUT_LUMA || layout == JO_LAYOUT_LUMA_ALPHA; break;
    case JO_COLOR_RGB:
        ok = layout == JO_LAYOUT_RGB || layout == JO_LAYOUT_RGBX || layout == JO_LAYOUT_RGBA || layout == JO_LAYOUT_BGR ||
             layout == JO_LAYOUT_BGRX || layout == JO_LAYOUT_BGRA;
        break;
    case JO_COLOR_YUV420: case JO_COLOR_YUV422: case JO_COLOR_YUV444: ok = layout == JO_LAYOUT_YUV || layout == JO_LAYOUT_YUVA; break;
    case JO_COLOR_CMYK: case JO_COLOR_CMYK_DIRECT: ok = layout == JO_LAYOUT_CMYK || layout == JO_LAYOUT_CMYKA; break;
    case JO_COLOR_RGBE: ok = s == JO_STORE_RGBE; break;
    case JO_COLOR_NCOMPONENT: ok = layout == JO_LAYOUT_NCOMPONENT || layout == JO_LAYOUT_NCOMPONENT_ALPHA; break;
    default: ok = 0;
    }
    if (!ok) return JO_ERR_UNSUPPORTED;
    int ic = r->internal_color;
    int integer_rgb = !(d == JO_DEPTH_F16 || d == JO_DEPTH_F32);
    if (ic == JO_COLOR_LUMA && oc == JO_COLOR_RGB) ok = integer_rgb;
    else if ((ic == JO_COLOR_LUMA && oc == JO_COLOR_LUMA) || (ic == JO_COLOR_YUV444 && (oc == JO_COLOR_RGB || oc == JO_COLOR_RGBE)) ||
             (ic == JO_COLOR_YUVK && (oc == JO_COLOR_CMYK || oc == JO_COLOR_CMYK_DIRECT)))
        ok = 1;
    else if ((ic == JO_COLOR_YUV420 || ic == JO_COLOR_YUV422 || ic == JO_COLOR_YUV444) && ic == oc) ok = 1;
    else if (ic == JO_COLOR_NCOMPONENT && oc == JO_COLOR_NCOMPONENT) ok = 1;
    else ok = 0;
    if (!ok) return JO_ERR_UNSUPPORTED;
    switch (oc) {
    case JO_COLOR_LUMA: ok = !is_packed_depth(d); break;
    case JO_COLOR_RGB: ok = 1; break;
    case JO_COLOR_YUV420: case JO_COLOR_YUV422: case JO_COLOR_YUV444:
        ok = d == JO_DEPTH_U8 || d == JO_DEPTH_U10 || d == JO_DEPTH_U16 || d == JO_DEPTH_I16; break;
    case JO_COLOR_RGBE: ok = d == JO_DEPTH_U8; break;
    default: ok = d == JO_DEPTH_U8 || d == JO_DEPTH_U16;
    }
    if (!ok) return JO_ERR_UNSUPPORTED;
    if ((d == JO_DEPTH_F32 && r->mantissa_length > 23) || (has_alpha && r->alpha_depth == JO_DEPTH_F32 && r->alpha_mantissa_length > 23))
        return JO_ERR_UNSUPPORTED;
    if (r->widen_f16 && s != JO_STORE_F16) return JO_ERR_UNSUPPORTED;
    return JO_OK;
}

static void store_word(uint8_t *out, size_t index, uint32_t value, size_t bytes)
{
    for (size_t b = 0; b < bytes; b++) out[index + b] = (uint8_t)(value >> (8 * b));
}

/* Premultiply one stored pixel in place (output_format/premultiply.rs:10-105). */
static int premultiply_pixel(uint8_t *px, int storage, int channels)
{
    size_t bytes = storage_bytes(storage);
    uint32_t words[8];
    for (int c = 0; c < channels; c++) {
        uint32_t w = 0;
        for (size_t b = 0; b < bytes; b++) w |= (uint32_t)px[c * bytes + b] << (8 * b);
        words[c] = w;
    }
    uint32_t a = words[channels - 1];
    for (int c = 0; c < channels - 1; c++) {
        uint32_t v = words[c], u;
        int32_t sv;
        uint16_t h;
        switch (storage) {
        case JO_STORE_U8: CK(jo_premultiply_unsigned(v, a, 255, &u) != JO_OK); words[c] = u; break;
        case JO_STORE_U16: CK(jo_premultiply_unsigned(v, a, 65535, &u) != JO_OK); words[c] = u; break;
        case JO_STORE_I16: CK(jo_premultiply_signed((int16_t)v, (int16_t)a, 32767, &sv) != JO_OK); words[c] = (uint16_t)(int16_t)sv; break;
        case JO_STORE_I32: CK(jo_premultiply_signed((int32_t)v, (int32_t)a, INT32_MAX, &sv) != JO_OK); words[c] = (uint32_t)sv; break;
        case JO_STORE_F16: CK(jo_premultiply_sign_magnitude_15((uint16_t)v, (uint16_t)a, &h) != JO_OK); words[c] = h; break;
        case JO_STORE_F32: {
            float fv, fa, fr;
            memcpy(&fv, &v, 4); memcpy(&fa, &a, 4);
            fr = jo_premultiply_f32(fv, fa);
            memcpy(&words[c], &fr, 4);
            break;
        }
        default: return JO_ERR_UNSUPPORTED;
        }
    }
    for (int c = 0; c < channels; c++) store_word(px, (size_t)c * bytes, words[c], bytes);
    return JO_OK;
}

typedef struct {
    const int32_t *const *planes; int plane_count; const int32_t *alpha;
    uint32_t width; const jo_output *r;
} ctx_t;

/* Stored value of one channel of a pixel in storage words: fill_ordered and
 * the typed stores of output_format/packing.rs:248-358. */
static int channel_word(const ctx_t *cx, int32_t sample, int component, int alpha, uint32_t *word)
{
    const jo_output *r = cx->r;
    int padding = !alpha && (r->layout == JO_LAYOUT_RGBX || r->layout == JO_LAYOUT_BGRX) && component == 3;
    if (padding) { *word = 0; return JO_OK; }
    int depth = alpha ? r->alpha_depth : r->depth;
    int shift_bits = alpha ? r->alpha_shift_bits : r->shift_bits;
    int scaled = alpha ? r->alpha_scaled : r->scaled;
    int color = alpha ? JO_COLOR_LUMA : r->output_color;
    int comp = alpha ? 0 : component;
    int32_t v;
    switch (r->storage) {
    case JO_STORE_F16: {
        uint16_t h;
        int rc = f16_bits(sample, scaled, &h);
        if (rc) return rc;
        *word = r->widen_f16 ? jo_widen_f16(h) : h;
        return JO_OK;
    }
    case JO_STORE_F32: {
        int ml = alpha ? r->alpha_mantissa_length : r->mantissa_length;
        int eb = alpha ? r->alpha_exponent_bias : r->exponent_bias;
        if (depth != JO_DEPTH_F32) return JO_ERR_UNSUPPORTED;
        return f32_bits(sample, scaled, ml, eb, word);
    }
    default: break;
    }
    scale_t s = resolve_scale(comp, color, depth, shift_bits, scaled);
    int rc = apply_scale(&s, sample, &v);
    if (rc) return rc;
    switch (r->storage) {
    case JO_STORE_U8: *word = (uint32_t)clampi(v, 0, 255); break;
    case JO_STORE_U16: *word = (uint32_t)clampi(v, 0, depth == JO_DEPTH_U10 ? 1023 : 65535); break;
    case JO_STORE_I16: *word = (uint16_t)(int16_t)clampi(v, -32768, 32767); break;
    case JO_STORE_I32: *word = (uint32_t)v; break;
    default: return JO_ERR_UNSUPPORTED;
    }
    return JO_OK;
}

static int32_t plane_at(const int32_t *p, uint32_t width, uint32_t x, uint32_t y) { return p[(size_t)y * width + x]; }

static int format_pixel(const ctx_t *cx, uint32_t sx, uint32_t sy, uint8_t *dst, size_t channel_stride)
{
    const jo_output *r = cx->r;
    int32_t in[4] = {0, 0, 0, 0}, conv[4];
    int n = cx->plane_count < 4 ? cx->plane_count : 4;
    size_t bytes = r->widen_f16 ? 4 : storage_bytes(r->storage);
    if (r->output_color == JO_COLOR_NCOMPONENT) {
        int ch = 0;
        for (int c = 0; c < cx->plane_count; c++, ch++) {
            uint32_t w;
            CK(channel_word(cx, plane_at(cx->planes[c], cx->width, sx, sy), c, 0, &w) != JO_OK);
            store_word(dst, (size_t)ch * channel_stride * bytes, w, bytes);
        }
        if (cx->alpha) {
            uint32_t w;
            CK(channel_word(cx, plane_at(cx->alpha, cx->width, sx, sy), ch, 1, &w) != JO_OK);
            store_word(dst, (size_t)ch * channel_stride * bytes, w, bytes);
        }
        return JO_OK;
    }
    for (int c = 0; c < n; c++) in[c] = plane_at(cx->planes[c], cx->width, sx, sy);
    if (is_direct(r->internal_color, r->output_color)) memcpy(conv, in, sizeof conv);
    else {
        int rc = convert_color(r->internal_color, r->output_color, in, is_packed_depth(r->depth), r->red_blue_not_swapped, conv);
        if (rc) return rc;
    }
    int32_t prim[4];
    if (r->layout == JO_LAYOUT_BGR || r->layout == JO_LAYOUT_BGRX || r->layout == JO_LAYOUT_BGRA) {
        prim[0] = conv[2]; prim[1] = conv[1]; prim[2] = conv[0]; prim[3] = 0;
    } else memcpy(prim, conv, sizeof prim);
    int pc = primary_count(r);
    for (int c = 0; c < pc; c++) {
        uint32_t w;
        int rc = channel_word(cx, prim[c], c, 0, &w);
        if (rc) return rc;
        store_word(dst, (size_t)c * channel_stride * bytes, w, bytes);
    }
    if (cx->alpha) {
        uint32_t w;
        int rc = channel_word(cx, plane_at(cx->alpha, cx->width, sx, sy), pc, 1, &w);
        if (rc) return rc;
        store_word(dst, (size_t)pc * channel_stride * bytes, w, bytes);
    }
    return JO_OK;
}

/* pack_rgb555_into .. pack_rgbe_into, output_format/packed_color.rs:47-150 */
static int packed_pixel(const ctx_t *cx, uint32_t sx, uint32_t sy, uint32_t *word)
{
    const jo_output *r = cx->r;
    int32_t in[4] = {0, 0, 0, 0}, conv[4];
    int n = cx->plane_count < 4 ? cx->plane_count : 4;
    for (int c = 0; c < n; c++) in[c] = plane_at(cx->planes[c], cx->width, sx, sy);
    if (is_direct(r->internal_color, r->output_color)) memcpy(conv, in, sizeof conv);
    else {
        int rc = convert_color(r->internal_color, r->output_color, in, is_packed_depth(r->depth), r->red_blue_not_swapped, conv);
        if (rc) return rc;
    }
    int32_t v[3];
    if (r->storage == JO_STORE_RGBE) {
        for (int c = 0; c < 3; c++) {
            scale_t s = resolve_scale(c, JO_COLOR_RGBE, JO_DEPTH_U8, 0, r->scaled);
            CK(apply_scale(&s, conv[c], &v[c]) != JO_OK);
        }
        uint8_t b[4];
        jo_postscale_rgbe(v, b);
        *word = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
        return JO_OK;
    }
    uint32_t f[3];
    for (int c = 0; c < 3; c++) {
        scale_t s = resolve_scale(c, JO_COLOR_RGB, r->depth, 0, r->scaled);
        CK(apply_scale(&s, conv[c], &v[c]) != JO_OK);
        uint32_t maximum = r->depth == JO_DEPTH_RGB555 ? 31 : r->depth == JO_DEPTH_RGB101010 ? 1023 : (c == 1 ? 63 : 31);
        f[c] = v[c] < 0 ? 0 : ((uint32_t)v[c] > maximum ? maximum : (uint32_t)v[c]);
    }
    if (r->depth == JO_DEPTH_RGB555) *word = f[2] | (f[1] << 5) | (f[0] << 10);
    else if (r->depth == JO_DEPTH_RGB565) *word = f[2] | (f[1] << 5) | (f[0] << 11);
    else *word = f[2] | (f[1] << 10) | (f[0] << 20);
    return JO_OK;
}

/* Native planar YUV 4:2:0 / 4:2:2 output: output_format/planar.rs:76-222. */
static int format_planar(const int32_t *const *planes, const int32_t *alpha, uint32_t width, uint32_t height,
                         const jo_output *r, uint8_t *out)
{
    int c420 = r->output_color == JO_COLOR_YUV420;
    uint32_t cw = width / 2, chh = c420 ? height / 2 : height;
    struct { const int32_t *p; uint32_t pw; uint32_t x, y, w, h; int alpha; int comp; } win[4];
    int n = 0;
    win[n].p = planes[0]; win[n].pw = width; win[n].x = r->crop_x; win[n].y = r->crop_y;
    win[n].w = r->crop_width; win[n].h = r->crop_height; win[n].alpha = 0; win[n].comp = 0; n++;
    for (int c = 1; c < 3; c++) {
        win[n].p = planes[c]; win[n].pw = cw; win[n].x = r->crop_x / 2; win[n].y = c420 ? r->crop_y / 2 : r->crop_y;
        win[n].w = r->crop_width / 2; win[n].h = c420 ? r->crop_height / 2 : r->crop_height; win[n].alpha = 0; win[n].comp = c; n++;
    }
    if (alpha) {
        win[n].p = alpha; win[n].pw = width; win[n].x = r->crop_x; win[n].y = r->crop_y;
        win[n].w = r->crop_width; win[n].h = r->crop_height; win[n].alpha = 1; win[n].comp = 0; n++;
    }
    (void)chh;
    size_t bytes = storage_bytes(r->storage), pos = 0;
    for (int i = 0; i < n; i++) {
        int scaled = win[i].alpha ? r->alpha_scaled : r->scaled;
        for (uint32_t y = 0; y < win[i].h; y++)
            for (uint32_t x = 0; x < win[i].w; x++) {
                int32_t v;
                scale_t s = resolve_scale(win[i].comp, r->output_color, r->depth, r->shift_bits, scaled);
                CK(apply_scale(&s, win[i].p[(size_t)(win[i].y + y) * win[i].pw + win[i].x + x], &v) != JO_OK);
                uint32_t w;
                if (r->storage == JO_STORE_U8) w = (uint32_t)clampi(v, 0, 255);
                else if (r->storage == JO_STORE_U16) w = (uint32_t)clampi(v, 0, r->depth == JO_DEPTH_U10 ? 1023 : 65535);
                else if (r->storage == JO_STORE_I16) w = (uint16_t)(int16_t)clampi(v, -32768, 32767);
                else return JO_ERR_UNSUPPORTED;
                store_word(out, pos, w, bytes);
                pos += bytes;
            }
    }
    return JO_OK;
}

int jo_format_output(const int32_t *const *planes, int plane_count, const int32_t *alpha, uint32_t width,
                     uint32_t height, const jo_output *r, void *outv, size_t out_len)
{
    uint8_t *out = outv;
    int rc = validate_request(r, alpha != NULL);
    if (rc) return rc;
    if (out_len < jo_output_bytes(r)) return JO_ERR_INVALID;
    if (r->crop_width == 0 || r->crop_height == 0) return JO_OK;
    if (is_planar_yuv(r)) {
        if (plane_count != 3) return JO_ERR_INVALID;
        return format_planar(planes, alpha, width, height, r, out);
    }
    if ((uint64_t)r->crop_x + r->crop_width > width || (uint64_t)r->crop_y + r->crop_height > height) return JO_ERR_INVALID;
    ctx_t cx = {planes, plane_count, alpha, width, r};
    if (r->storage == JO_STORE_BITS) {
        size_t row_bytes = (r->crop_width + 7) / 8;
        memset(out, 0, row_bytes * r->crop_height);
        scale_t s = resolve_scale(0, JO_COLOR_LUMA, r->depth, 0, r->scaled);
        for (uint32_t y = 0; y < r->crop_height; y++)
            for (uint32_t x = 0; x < r->crop_width; x++) {
                int32_t v;
                CK(apply_scale(&s, plane_at(planes[0], width, r->crop_x + x, r->crop_y + y), &v) != JO_OK);
                int32_t bit = clampi(v, 0, 1);
                if (r->depth == JO_DEPTH_BIT1_BLACK) bit = 1 - bit;
                out[y * row_bytes + x / 8] |= (uint8_t)(bit << (7 - x % 8));
            }
        return JO_OK;
    }
    if (r->storage >= JO_STORE_RGB555) {
        size_t bytes = storage_bytes(r->storage);
        for (uint32_t y = 0; y < r->crop_height; y++)
            for (uint32_t x = 0; x < r->crop_width; x++) {
                uint32_t w;
                rc = packed_pixel(&cx, r->crop_x + x, r->crop_y + y, &w);
                if (rc) return rc;
                store_word(out, ((size_t)y * r->crop_width + x) * bytes, w, bytes);
            }
        return JO_OK;
    }
    int channels = r->output_color == JO_COLOR_NCOMPONENT ? plane_count + (alpha ? 1 : 0) : layout_channels(r->layout, r->ncomponents);
    size_t bytes = r->widen_f16 ? 4 : storage_bytes(r->storage);
    size_t npx = (size_t)r->crop_width * r->crop_height;
    for (uint32_t y = 0; y < r->crop_height; y++)
        for (uint32_t x = 0; x < r->crop_width; x++) {
            size_t p = (size_t)y * r->crop_width + x;
            uint8_t *dst = r->nchw ? out + p * bytes : out + p * (size_t)channels * bytes;
            rc = format_pixel(&cx, r->crop_x + x, r->crop_y + y, dst, r->nchw ? npx : 1);
            if (rc) return rc;
        }
    if (r->premultiply) {
        if (r->nchw || r->widen_f16) return JO_ERR_UNSUPPORTED;
        for (size_t p = 0; p < npx; p++) {
            rc = premultiply_pixel(out + p * (size_t)channels * bytes, r->storage, channels);
            if (rc) return rc;
        }
    }
    return JO_OK;
}

int jo_decode_image(const jo_image *im, const jo_output *r, void *out, size_t out_len, int threads)
{
    if (im->plane_count < 1 || im->plane_count > 16) return JO_ERR_INVALID;
    int32_t *planes[17] = {0};
    uint32_t pw[17], ph[17];
    int n = im->plane_count + (im->alpha ? 1 : 0), rc = JO_OK;
    for (int i = 0; i < n; i++) {
        const jo_plane *p = i < im->plane_count ? &im->planes[i] : im->alpha;
        jo_plane_extent(p, &pw[i], &ph[i]);
        planes[i] = malloc(sizeof(int32_t) * ((size_t)pw[i] * ph[i] + 1));
        if (!planes[i]) { rc = JO_ERR_INVALID; goto done; }
        rc = jo_reconstruct_plane(p, planes[i], threads);
        if (rc) goto done;
    }
    const int32_t *alpha = im->alpha ? planes[im->plane_count] : NULL;
    int subsampled = im->coded_color == JO_COLOR_YUV420 || im->coded_color == JO_COLOR_YUV422;
    if (subsampled && !is_planar_yuv(r)) {
        if (im->plane_count != 3) { rc = JO_ERR_INVALID; goto done; }
        for (int c = 1; c < 3; c++) {
            uint32_t ow = pw[c] * 2, oh = im->coded_color == JO_COLOR_YUV420 ? ph[c] * 2 : ph[c];
            if (ow != pw[0] || oh != ph[0]) { rc = JO_ERR_INVALID; goto done; }
            int32_t *up = malloc(sizeof(int32_t) * (size_t)ow * oh);
            if (!up) { rc = JO_ERR_INVALID; goto done; }
            rc = jo_upsample_chroma(planes[c], pw[c], ph[c], im->coded_color == JO_COLOR_YUV420 ? 1 : 2,
                                    im->centering_x, im->centering_y, up, threads);
            free(planes[c]);
            planes[c] = up;
            if (rc) goto done;
        }
    }
    for (int i = 1; i < im->plane_count && !is_planar_yuv(r); i++)
        if (pw[i] != pw[0] && !subsampled) { rc = JO_ERR_INVALID; goto done; }
    rc = jo_format_output((const int32_t *const *)planes, im->plane_count, alpha, pw[0], ph[0], r, out, out_len);
done:
    for (int i = 0; i < n; i++) free(planes[i]);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* forward operators (crates/jxr-math/src/transform.rs:30-146,316-400,        */
/* overlap.rs:61-374): the analysis side, exact inverses of the operators    */
/* above.  The inputs they see here (flat probe planes) stay far inside      */
/* int32, so they are written unchecked.                                     */
/* ------------------------------------------------------------------------ */
static void f_t2x2h(int32_t *a, int32_t *b, int32_t *c, int32_t *d, int32_t rounding)
{
    *a += *d;
    *b -= *c;
    int32_t first = (*a - *b + rounding) >> 1, second = *c;
    *c = first - *d;
    *d = first - second;
    *a -= *d;
    *b += *c;
}

static void f_todd(int32_t *a, int32_t *b, int32_t *c, int32_t *d)
{
    *a += *d;
    *b -= *c;
    *d = ((*a + 1) >> 1) - *d;
    *c += (*b + 1) >> 1;
    *d -= (3 * *c + 4) >> 3;
    *c += (3 * *d + 4) >> 3;
    *b -= (3 * *a + 4) >> 3;
    *a += (3 * *b + 4) >> 3;
    *c -= (*a + 1) >> 1;
    *d += *b >> 1;
    *a += *c;
    *b -= *d;
}

static void f_todd_odd(int32_t *a, int32_t *b, int32_t *c, int32_t *d)
{
    *b = -*b;
    *c = -*c;
    *d += *a;
    *c -= *b;
    int32_t first = *d >> 1, second = *c >> 1;
    *a -= first;
    *b += second;
    *a += (3 * *b + 4) >> 3;
    *b -= (3 * *a + 3) >> 2;
    *a += (3 * *b + 3) >> 3;
    *b -= second;
    *a += first;
    *c += *b;
    *d -= *a;
}

/* forward_core_transform, transform.rs:30-93 (with forward_permute, 195-205) */
static void f_core(int32_t s[16])
{
    f_t2x2h(&s[4], &s[7], &s[8], &s[11], 0);
    f_t2x2h(&s[1], &s[2], &s[13], &s[14], 0);
    f_t2x2h(&s[5], &s[6], &s[9], &s[10], 0);
    f_t2x2h(&s[0], &s[3], &s[12], &s[15], 0);
    f_todd_odd(&s[10], &s[11], &s[14], &s[15]);
    f_todd(&s[8], &s[12], &s[9], &s[13]);
    f_todd(&s[2], &s[3], &s[6], &s[7]);
    f_t2x2h(&s[0], &s[1], &s[4], &s[5], 1);
    int32_t in[16];
    memcpy(in, s, sizeof in);
    for (int i = 0; i < 16; i++) s[i] = in[INVERSE_PERMUTATION[i]];
}

/* forward_chroma_420, transform.rs:95-104 */
static void f_chroma_420(int32_t s[4])
{
    int32_t t = s[1]; s[1] = s[2]; s[2] = t;
    f_t2x2h(&s[0], &s[1], &s[2], &s[3], 0);
}

/* forward_chroma_422, transform.rs:106-146 */
static void f_chroma_422(int32_t s[8])
{
    int32_t t = s[5]; s[5] = s[6]; s[6] = t;
    f_t2x2h(&s[4], &s[6], &s[5], &s[7], 0);
    t = s[1]; s[1] = s[2]; s[2] = t;
    f_t2x2h(&s[0], &s[1], &s[2], &s[3], 0);
    s[4] -= s[0];
    s[0] += (s[4] + 1) >> 1;
}

static void f_rotate(int32_t *a, int32_t *b) { *b -= (*a + 1) >> 1; *a += (*b + 1) >> 1; }

static void f_scale(int32_t *a, int32_t *b)
{
    *b += *a >> 10;
    *b -= *a >> 7;
    *b -= (3 * *a) >> 4;
    *a -= (3 * *b) >> 3;
    *b = (*a >> 1) - *b;
    *a -= *b;
}

static void f_hadamard_pre(int32_t *a, int32_t *b, int32_t *c, int32_t *d)
{
    *b -= *c;
    *a += *d;
    int32_t t = *c; *c = *d; *d = t;
    *c = ((*a - *b) >> 1) - *c;
    *d += *b >> 1;
    *a -= (3 * *d + 4) >> 3;
    *b += *c;
}

static void f_todd_odd_pre(int32_t *a, int32_t *b, int32_t *c, int32_t *d)
{
    *d += *a;
    *c -= *b;
    int32_t first = *d >> 1, second = *c >> 1;
    *a -= first;
    *b += second;
    *a += (3 * *b + 4) >> 3;
    *b -= (3 * *a + 2) >> 2;
    *a += (3 * *b + 6) >> 3;
    *b -= second;
    *a += first;
    *c += *b;
    *d -= *a;
}

/* forward_overlap_filter_4x4, overlap.rs:112-160 */
static void f_overlap_4x4(int32_t v[16])
{
    f_hadamard_pre(&v[0], &v[3], &v[12], &v[15]);
    f_hadamard_pre(&v[1], &v[2], &v[13], &v[14]);
    f_hadamard_pre(&v[4], &v[7], &v[8], &v[11]);
    f_hadamard_pre(&v[5], &v[6], &v[9], &v[10]);
    f_scale(&v[0], &v[15]);
    f_scale(&v[1], &v[14]);
    f_scale(&v[4], &v[11]);
    f_scale(&v[5], &v[10]);
    f_todd_odd_pre(&v[10], &v[11], &v[14], &v[15]);
    f_rotate(&v[13], &v[12]);
    f_rotate(&v[9], &v[8]);
    f_rotate(&v[7], &v[3]);
    f_rotate(&v[6], &v[2]);
    f_t2x2h(&v[0], &v[3], &v[12], &v[15], 0);
    f_t2x2h(&v[1], &v[2], &v[13], &v[14], 0);
    f_t2x2h(&v[4], &v[7], &v[8], &v[11], 0);
    f_t2x2h(&v[5], &v[6], &v[9], &v[10], 0);
}

/* forward_overlap_filter_4, overlap.rs:61-110 */
static void f_overlap_4(int32_t *a, int32_t *b, int32_t *c, int32_t *d)
{
    *b += *c;
    *a += *d;
    *c -= (*b + 1) >> 1;
    *d -= (*a + 1) >> 1;
    f_rotate(c, d);
    *c = -*c;
    *d = -*d;
    *b -= *c;
    *a -= *d;
    *c += *b >> 1;
    *d += *a >> 1;
    *b -= (3 * *c + 4) >> 3;
    *a -= (3 * *d + 4) >> 3;
    f_scale(b, c);
    f_scale(a, d);
    *c += (*b + 1) >> 1;
    *d += (*a + 1) >> 1;
    *b -= *c;
    *a -= *d;
}

/* forward_overlap_filter_2, overlap.rs:265-297 */
static void f_overlap_2(int32_t *a, int32_t *b)
{
    *b -= (*a + 2) >> 2;
    *a -= *b >> 13;
    *a -= *b >> 9;
    *a -= *b >> 5;
    *a -= (*b + 1) >> 1;
    *b -= (*a + 2) >> 2;
}

/* forward_overlap_filter_2x2, overlap.rs:234-263 */
static void f_overlap_2x2(int32_t *a, int32_t *b, int32_t *c, int32_t *d)
{
    *b += *c;
    *a += *d;
    *c -= (*b + 1) >> 1;
    *d -= (*a + 1) >> 1;
    f_overlap_2(a, b);
    *c += (*b + 1) >> 1;
    *d += (*a + 1) >> 1;
    *b -= *c;
    *a -= *d;
}

/* The full-resolution schedule of full_region with the forward operators:
 * its windows are disjoint, so each is simply replaced by its inverse. */
static void forward_full_region(int32_t *s, size_t stride, region_t g)
{
    for (uint32_t y = g.top + 2; y + 2 < g.bottom; y += 4)
        for (uint32_t x = g.left + 2; x + 2 < g.right; x += 4) {
            int32_t v[16];
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) v[r * 4 + c] = s[(y + r) * stride + x + c];
            f_overlap_4x4(v);
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) s[(y + r) * stride + x + c] = v[r * 4 + c];
        }
    for (uint32_t y = g.top + 2; y + 2 < g.bottom; y += 4) {
        uint32_t xs[4] = {g.left, g.left + 1, g.right - 2, g.right - 1};
        for (int k = 0; k < 4; k++)
            f_overlap_4(&s[y * stride + xs[k]], &s[(y + 1) * stride + xs[k]], &s[(y + 2) * stride + xs[k]],
                        &s[(y + 3) * stride + xs[k]]);
    }
    uint32_t ys[4] = {g.top, g.top + 1, g.bottom - 2, g.bottom - 1};
    for (uint32_t x = g.left + 2; x + 2 < g.right; x += 4)
        for (int k = 0; k < 4; k++) {
            size_t o = (size_t)ys[k] * stride + x;
            f_overlap_4(&s[o], &s[o + 1], &s[o + 2], &s[o + 3]);
        }
    uint32_t cx[4] = {g.left, g.right - 2, g.left, g.right - 2};
    uint32_t cy[4] = {g.top, g.top, g.bottom - 2, g.bottom - 2};
    for (int k = 0; k < 4; k++) {
        size_t o = (size_t)cy[k] * stride + cx[k];
        f_overlap_4(&s[o], &s[o + 1], &s[o + stride], &s[o + stride + 1]);
    }
}

/* subsampled_boundary_row run backwards with the forward operator */
static void forward_subsampled_boundary_row(int32_t *s, size_t stride, region_t g, uint32_t row)
{
    size_t base = (size_t)row * stride;
    size_t c0 = base + g.left, n0 = base + g.left + 1;
    size_t c1 = base + g.right - 1, n1 = base + g.right - 2;
    s[c1] -= s[n1];
    s[c0] -= s[n0];
    for (uint32_t x = g.left + 2; x < g.right; x += 2) f_overlap_2(&s[base + x - 1], &s[base + x]);
    s[c1] += s[n1];
    s[c0] += s[n0];
}

/* subsampled_region run last step first with the forward operators */
static void forward_subsampled_region(int32_t *s, size_t stride, region_t g)
{
    forward_subsampled_boundary_row(s, stride, g, g.bottom - 1);
    uint32_t rows = 0;
    for (uint32_t y = g.top + 2; y < g.bottom; y += 2) rows++;
    for (uint32_t k = rows; k-- > 0;) {
        uint32_t y = g.top + 2 + 2 * k;
        uint32_t xs[2] = {g.left, g.right - 1};
        for (int i = 1; i >= 0; i--)
            f_overlap_2(&s[(size_t)(y - 1) * stride + xs[i]], &s[(size_t)y * stride + xs[i]]);
        for (uint32_t x = g.left + 2; x < g.right; x += 2) {
            size_t a = (size_t)(y - 1) * stride + x - 1, b = (size_t)y * stride + x - 1;
            f_overlap_2x2(&s[a], &s[a + 1], &s[b], &s[b + 1]);
        }
    }
    forward_subsampled_boundary_row(s, stride, g, g.top);
}

/* Quantizer::quantize, crates/jxr-math/src/quantization.rs:28-50 */
static int32_t quantize_step(int32_t c, uint32_t step, uint32_t offset)
{
    if (offset >= step) offset = step - 1;
    uint32_t m = c < 0 ? (uint32_t)(-(int64_t)c) : (uint32_t)c;
    uint32_t carry = (m % step) >= step - offset ? 1u : 0u;
    uint32_t q = m / step + carry;
    return c < 0 ? -(int32_t)q : (int32_t)q;
}

int jo_analyze_plane(const jo_plane *p, const int32_t *samples, int32_t *coefficients)
{
    uint32_t bc = p->block_columns, br = p->block_rows, count = bc * br;
    if (!((bc == 4 && br == 4) || (bc == 2 && br == 4) || (bc == 2 && br == 2))) return JO_ERR_INVALID;
    size_t lw = (size_t)p->macroblocks_x * bc, lh = (size_t)p->macroblocks_y * br;
    size_t width = lw * 4, height = lh * 4;
    int32_t *s = malloc(sizeof *s * width * height + 1);
    int32_t *low = malloc(sizeof *low * lw * lh + 1);
    int32_t *high = malloc(sizeof *high * width * height + 1);
    if (!s || !low || !high) { free(s); free(low); free(high); return JO_ERR_INVALID; }
    memcpy(s, samples, sizeof *s * width * height);
    region_t *regions = NULL;
    int n = 0, rc = JO_OK;
    if (p->overlap >= 1) {
        rc = build_regions(p, bc * 4, br * 4, &regions, &n);
        for (int i = 0; rc == JO_OK && i < n; i++) forward_full_region(s, width, regions[i]);
        free(regions);
    }
    for (size_t by = 0; rc == JO_OK && by < lh; by++)
        for (size_t bx = 0; bx < lw; bx++) {
            int32_t v[16];
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) v[r * 4 + c] = s[(by * 4 + r) * width + bx * 4 + c];
            f_core(v);
            low[by * lw + bx] = v[0];
            memcpy(&high[(by * lw + bx) * 16], v, sizeof v);
        }
    if (rc == JO_OK && p->overlap == 2) {
        rc = build_regions(p, bc, br, &regions, &n);
        for (int i = 0; rc == JO_OK && i < n; i++) {
            if (bc == 4) forward_full_region(low, lw, regions[i]);
            else forward_subsampled_region(low, lw, regions[i]);
        }
        free(regions);
    }
    /* DC and low-pass bands at a unit step, divided by two (to nearest)
     * where reconstruction doubles them (Steps::new, analyze.rs:505-535) */
    uint32_t divisor = p->scale_after_first_transform ? 2u : 1u;
    for (uint32_t my = 0; rc == JO_OK && my < p->macroblocks_y; my++)
        for (uint32_t mx = 0; mx < p->macroblocks_x; mx++) {
            int32_t l[16] = {0};
            for (uint32_t r = 0; r < br; r++)
                for (uint32_t c = 0; c < bc; c++) l[r * bc + c] = low[((size_t)my * br + r) * lw + mx * bc + c];
            if (count == 16) f_core(l);
            else if (count == 4) f_chroma_420(l);
            else f_chroma_422(l);
            int32_t *out = coefficients + ((size_t)my * p->macroblocks_x + mx) * count * 16;
            for (uint32_t b = 0; b < count; b++) {
                size_t bx = (size_t)mx * bc + b % bc, by = (size_t)my * br + b / bc;
                memcpy(out + b * 16, &high[(by * lw + bx) * 16], 16 * sizeof(int32_t));
                out[b * 16] = quantize_step(l[b], divisor, divisor / 2);
            }
        }
    free(s); free(low); free(high);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* reduced-resolution (quarter) reconstruction                               */
/* ------------------------------------------------------------------------ */

/* block_dc_plane (crates/jxr-native/src/reconstruct/pipeline.rs:459-541) with
 * the DC and low-pass bands: each macroblock's dequantized DC/LP values
 * through the first-level inverse transform (doubled where the plane is
 * scaled), placed one per block, then the first-level overlap filter when
 * the plane has two levels.  `out` is (macroblocks_x*bc) x (macroblocks_y*br). */
static int block_dc_plane_bands(const jo_plane *p, int dc_only, int32_t *out);

static int block_dc_plane(const jo_plane *p, int32_t *out) { return block_dc_plane_bands(p, 0, out); }

/* `dc_only`: LowBands::Dc (the low-pass coefficients left out, as the
 * sixteenth-resolution picture of a two-level plane wants them). */
static int block_dc_plane_bands(const jo_plane *p, int dc_only, int32_t *out)
{
    uint32_t bc = p->block_columns, br = p->block_rows, count = bc * br;
    if (!((bc == 4 && br == 4) || (bc == 2 && br == 4) || (bc == 2 && br == 2))) return JO_ERR_INVALID;
    size_t lw = (size_t)p->macroblocks_x * bc;
    for (uint32_t my = 0; my < p->macroblocks_y; my++)
        for (uint32_t mx = 0; mx < p->macroblocks_x; mx++) {
            size_t index = (size_t)my * p->macroblocks_x + mx;
            size_t offset = p->offsets[index];
            int bands = p->bands[index];
            if (bands < 0 || bands > 3) return JO_ERR_INVALID;
            size_t need = coefficients_per_macroblock(bands, count);
            if (offset > p->coefficient_count || need > p->coefficient_count - offset) return JO_ERR_INVALID;
            const int32_t *packed = p->coefficients + offset;
            const uint32_t *q = p->quantizers + index * 3;
            if (q[0] == 0 || q[1] == 0 || q[2] == 0) return JO_ERR_INVALID;
            int32_t l[16] = {0};
            CK(jo_dequantize(packed[0], q[0], &l[0]));
            if (bands != JO_BANDS_DC_ONLY && !dc_only)
                for (uint32_t b = 1; b < count; b++) {
                    int32_t v = bands == JO_BANDS_NO_HIGH_PASS ? packed[b] : packed[b * 16];
                    CK(jo_dequantize(v, q[1], &l[b]));
                }
            if (count == 16) CK(jo_inverse_core_transform(l));
            else if (count == 8) CK(jo_inverse_chroma_422(l));
            else CK(jo_inverse_chroma_420(l));
            if (p->scale_after_first_transform)
                for (uint32_t b = 0; b < count; b++) CK(mul(l[b], 2, &l[b]));
            for (uint32_t r = 0; r < br; r++)
                for (uint32_t c = 0; c < bc; c++) out[((size_t)my * br + r) * lw + (size_t)mx * bc + c] = l[r * bc + c];
        }
    if (p->overlap == 2) {
        region_t *regions = NULL;
        int n = 0, rc = build_regions(p, bc, br, &regions, &n);
        for (int i = 0; rc == JO_OK && i < n; i++)
            rc = bc == 4 ? full_region(out, lw, regions[i], 1) : subsampled_region(out, lw, regions[i]);
        free(regions);
        if (rc) return rc;
    }
    return JO_OK;
}

/* macroblock_dc_plane (crates/jxr-native/src/reconstruct/pipeline.rs:387-457):
 * one value a macroblock.  Without two-level overlap, its dequantized DC
 * (doubled where the plane is scaled); with it, the first-level picture of
 * the DC band alone (block_dc_plane with LowBands::Dc, overlap filter
 * included) summed over each macroblock's blocks, row by row, checked.
 * `out` is macroblocks_x x macroblocks_y. */
static int macroblock_dc_plane(const jo_plane *p, int32_t *out)
{
    uint32_t bc = p->block_columns, br = p->block_rows;
    if (!((bc == 4 && br == 4) || (bc == 2 && br == 4) || (bc == 2 && br == 2))) return JO_ERR_INVALID;
    size_t mbs = (size_t)p->macroblocks_x * p->macroblocks_y;
    if (p->overlap != 2) {
        for (size_t m = 0; m < mbs; m++) {
            int bands = p->bands[m];
            if (bands < 0 || bands > 3) return JO_ERR_INVALID;
            size_t offset = p->offsets[m], need = coefficients_per_macroblock(bands, bc * br);
            if (offset > p->coefficient_count || need > p->coefficient_count - offset) return JO_ERR_INVALID;
            const uint32_t *q = p->quantizers + m * 3;
            if (q[0] == 0 || q[1] == 0 || q[2] == 0) return JO_ERR_INVALID;
            int32_t dc;
            CK(jo_dequantize(p->coefficients[offset], q[0], &dc));
            if (p->scale_after_first_transform) CK(mul(dc, 2, &dc));
            out[m] = dc;
        }
        return JO_OK;
    }
    size_t lw = (size_t)p->macroblocks_x * bc;
    int32_t *low = malloc(sizeof(int32_t) * lw * p->macroblocks_y * br + 1);
    if (!low) return JO_ERR_INVALID;
    int rc = block_dc_plane_bands(p, 1, low);
    for (uint32_t my = 0; rc == JO_OK && my < p->macroblocks_y; my++)
        for (uint32_t mx = 0; rc == JO_OK && mx < p->macroblocks_x; mx++) {
            int32_t sum = 0;
            for (uint32_t r = 0; rc == JO_OK && r < br; r++)
                for (uint32_t c = 0; c < bc; c++)
                    if (add(sum, low[((size_t)my * br + r) * lw + (size_t)mx * bc + c], &sum)) { rc = JO_ERR_OVERFLOW; break; }
            out[(size_t)my * p->macroblocks_x + mx] = sum;
        }
    free(low);
    return rc;
}

/* ProbeAxis (crates/jxr-native/src/reconstruct/sample_scale.rs:352-430): one
 * probe region for each extent (up to 5 macroblocks) the component's regions
 * have along the axis, and for each macroblock of the component the probe
 * macroblock placed like it (probe_offset, 432-443). */
#define PROBE_EXTENT 5
typedef struct {
    uint32_t boundaries[PROBE_EXTENT + 2];
    int boundary_count;
    uint32_t macroblocks;
    uint32_t *positions;   /* one per component macroblock */
} probe_axis;

static uint32_t probe_offset(uint32_t offset, uint32_t extent)
{
    const uint32_t ends = PROBE_EXTENT / 2;
    if (extent <= PROBE_EXTENT || offset < ends) return offset;
    if (extent - offset <= ends) return PROBE_EXTENT - (extent - offset);
    return ends;
}

static int probe_axis_new(const uint32_t *regions, uint32_t count, probe_axis *a)
{
    int starts[PROBE_EXTENT + 1];
    for (int i = 0; i <= PROBE_EXTENT; i++) starts[i] = -1;
    a->boundaries[0] = 0;
    a->boundary_count = 1;
    a->macroblocks = 0;
    a->positions = NULL;
    if (count < 2) return JO_ERR_INVALID;
    a->positions = malloc(sizeof(uint32_t) * (regions[count - 1] + 1));
    if (!a->positions) return JO_ERR_INVALID;
    uint32_t n = 0;
    for (uint32_t i = 0; i + 1 < count; i++) {
        if (regions[i + 1] <= regions[i]) { free(a->positions); a->positions = NULL; return JO_ERR_INVALID; }
        uint32_t extent = regions[i + 1] - regions[i];
        uint32_t pe = extent < PROBE_EXTENT ? extent : PROBE_EXTENT;
        if (starts[pe] < 0) {
            starts[pe] = (int)a->macroblocks;
            a->macroblocks += pe;
            a->boundaries[a->boundary_count++] = a->macroblocks;
        }
        for (uint32_t o = 0; o < extent; o++) a->positions[n++] = (uint32_t)starts[pe] + probe_offset(o, extent);
    }
    return JO_OK;
}

typedef struct { int64_t divisor, bias; } flat_terms;

/* SampleScale::new / apply / FlatTerms::level, sample_scale.rs:155-350, and
 * scale_reduced_samples (pipeline.rs:81-117): scale the unscaled reduced
 * picture `pic` of plane `p` in place.  Quarter resolution (denominator 4):
 * one sample a block, transform gain 2^2 (BLOCK_DC_GAIN_BITS), pictures by
 * block_dc_plane.  Sixteenth (16): one sample a macroblock, gain 2^(2 + 2)
 * for 4x4 blocks and 2^(1 + 2) for subsampled chroma (macroblock_dc_gain_bits),
 * pictures by macroblock_dc_plane. */
static int apply_sample_scale(const jo_plane *p, int denominator, int32_t *pic)
{
    uint32_t bc = p->block_columns, br = p->block_rows;
    const int sixteenth = denominator == 16;
    const uint32_t ux = sixteenth ? 1 : bc, uy = sixteenth ? 1 : br;
    const int gain_bits = sixteenth ? ((bc == 4 && br == 4) ? 2 : 1) + 2 : 2;
    size_t w = (size_t)p->macroblocks_x * ux, h = (size_t)p->macroblocks_y * uy;
    if (p->overlap == 0) {
        for (size_t i = 0; i < w * h; i++) pic[i] >>= gain_bits;
        return JO_OK;
    }
    /* the regions the filters see: tiles when hard, else the plane */
    uint32_t plane_x[2] = {0, p->macroblocks_x}, plane_y[2] = {0, p->macroblocks_y};
    const uint32_t *cr = p->hard_tiles ? p->column_boundaries : plane_x;
    const uint32_t *rr = p->hard_tiles ? p->row_boundaries : plane_y;
    uint32_t ncr = p->hard_tiles ? p->column_boundary_count : 2, nrr = p->hard_tiles ? p->row_boundary_count : 2;
    probe_axis ax, ay;
    int rc = probe_axis_new(cr, ncr, &ax);
    if (rc) return rc;
    rc = probe_axis_new(rr, nrr, &ay);
    if (rc) { free(ax.positions); return rc; }
    /* the probe image: flat planes of each level through the analysis and
     * the reduced decode, as hard tiles of the probe extents */
    uint32_t pmx = ax.macroblocks, pmy = ay.macroblocks, count = bc * br;
    size_t samples_n = (size_t)pmx * bc * 4 * pmy * br * 4;
    size_t mbs = (size_t)pmx * pmy, stride = (size_t)pmx * ux, length = stride * pmy * uy;
    size_t picture_n = (size_t)pmx * bc * pmy * br;   /* the larger of the two picture sizes */
    int32_t *flat = malloc(sizeof(int32_t) * samples_n);
    int32_t *coeff = malloc(sizeof(int32_t) * mbs * count * 16);
    uint32_t *offsets = malloc(sizeof(uint32_t) * mbs), *quant = malloc(sizeof(uint32_t) * mbs * 3);
    uint8_t *bands = malloc(mbs), *hp = calloc(mbs, 1);
    int32_t *picture = malloc(sizeof(int32_t) * picture_n);
    int64_t *rise = calloc(length, sizeof(int64_t)), *offset = calloc(length, sizeof(int64_t));
    flat_terms *terms = malloc(sizeof(flat_terms) * length);
    if (!flat || !coeff || !offsets || !quant || !bands || !hp || !picture || !rise || !offset || !terms) {
        rc = JO_ERR_INVALID;
        goto out;
    }
    for (size_t m = 0; m < mbs; m++) {
        offsets[m] = (uint32_t)(m * count * 16);
        quant[m * 3] = quant[m * 3 + 1] = quant[m * 3 + 2] = 1;
        bands[m] = JO_BANDS_ALL;
    }
    jo_plane probe = *p;
    probe.coefficients = coeff;
    probe.coefficient_count = mbs * count * 16;
    probe.offsets = offsets;
    probe.quantizers = quant;
    probe.bands = bands;
    probe.hp_prediction = hp;
    probe.macroblocks_x = pmx;
    probe.macroblocks_y = pmy;
    probe.hard_tiles = 1;
    probe.column_boundaries = ax.boundaries;
    probe.column_boundary_count = (uint32_t)ax.boundary_count;
    probe.row_boundaries = ay.boundaries;
    probe.row_boundary_count = (uint32_t)ay.boundary_count;
    /* PROBE_LEVELS, sample_scale.rs:42 */
    static const int32_t levels[4] = {0x10001, 0x10002, 0x10003, 0x10004};
    int64_t span = 0, cnt = 0;
    for (int li = 0; li < 4 && rc == JO_OK; li++) {
        for (int sign = 1; sign >= -1 && rc == JO_OK; sign -= 2) {
            int32_t level = sign * levels[li];
            for (size_t i = 0; i < samples_n; i++) flat[i] = level;
            rc = jo_analyze_plane(&probe, flat, coeff);
            if (rc == JO_OK) rc = sixteenth ? macroblock_dc_plane(&probe, picture) : block_dc_plane(&probe, picture);
            for (size_t i = 0; rc == JO_OK && i < length; i++) {
                if (sign > 0) { rise[i] += picture[i]; offset[i] += picture[i]; }
                else { rise[i] -= picture[i]; offset[i] += picture[i]; }
            }
        }
        span += 2 * (int64_t)levels[li];
        cnt += 2;
    }
    for (size_t i = 0; rc == JO_OK && i < length; i++) {
        int64_t divisor = cnt * rise[i];
        if (divisor <= 0) { rc = JO_ERR_OVERFLOW; break; }
        terms[i].divisor = divisor;
        terms[i].bias = offset[i] * span - divisor / 2;
    }
    int64_t gain = cnt * span;
    for (size_t y = 0; rc == JO_OK && y < h; y++) {
        size_t prow = (size_t)ay.positions[y / uy] * uy + y % uy;
        for (size_t x = 0; x < w; x++) {
            size_t pcol = (size_t)ax.positions[x / ux] * ux + x % ux;
            const flat_terms t = terms[prow * stride + pcol];
            int32_t c = pic[y * w + x];
            if (c == 0) continue;
            int64_t num = (int64_t)c * gain - t.bias;
            int64_t q = num / t.divisor, r = num % t.divisor;
            if (r < 0) q -= 1;   /* div_euclid with a positive divisor */
            if (q < INT32_MIN || q > INT32_MAX) { rc = JO_ERR_OVERFLOW; break; }
            pic[y * w + x] = (int32_t)q;
        }
    }
out:
    free(flat); free(coeff); free(offsets); free(quant); free(bands); free(hp); free(picture);
    free(rise); free(offset); free(terms); free(ax.positions); free(ay.positions);
    return rc;
}

void jo_plane_extent_scaled(const jo_plane *p, int denominator, uint32_t *w, uint32_t *h)
{
    if (denominator == 16) {
        /* one sample a macroblock, subsampled chroma included */
        *w = p->macroblocks_x;
        *h = p->macroblocks_y;
        return;
    }
    jo_plane_extent(p, w, h);
    *w /= (uint32_t)denominator;
    *h /= (uint32_t)denominator;
}

static int check_hard_partition(const jo_plane *p)
{
    if (!p->hard_tiles) return JO_OK;
    const uint32_t *cb = p->column_boundaries, *rb = p->row_boundaries;
    uint32_t nc = p->column_boundary_count, nr = p->row_boundary_count;
    if (nc < 2 || nr < 2 || cb[0] != 0 || rb[0] != 0 || cb[nc - 1] != p->macroblocks_x ||
        rb[nr - 1] != p->macroblocks_y)
        return JO_ERR_INVALID;
    return JO_OK;
}

int jo_reconstruct_plane_quarter(const jo_plane *p, int32_t *samples)
{
    int rc = check_hard_partition(p);
    if (rc) return rc;
    rc = block_dc_plane(p, samples);
    if (rc) return rc;
    return apply_sample_scale(p, 4, samples);
}

int jo_reconstruct_plane_sixteenth(const jo_plane *p, int32_t *samples)
{
    /* reconstruct_sixteenth, crates/jxr-native/src/reconstruct/pipeline.rs:223-260 */
    int rc = check_hard_partition(p);
    if (rc) return rc;
    rc = macroblock_dc_plane(p, samples);
    if (rc) return rc;
    return apply_sample_scale(p, 16, samples);
}

int jo_decode_image_scaled(const jo_image *im, int denominator, const jo_output *r, void *out, size_t out_len,
                           int threads)
{
    if (denominator == 1) return jo_decode_image(im, r, out, out_len, threads);
    if (denominator != 4 && denominator != 16) return JO_ERR_UNSUPPORTED;
    /* a sixteenth has a chroma sample for each macroblock as luma does: no
     * interpolation, and subsampled planar output is refused
     * (crates/jxr-native/src/prepare.rs:185-192, metadata.rs:255-263) */
    if (denominator == 16 && is_planar_yuv(r)) return JO_ERR_UNSUPPORTED;
    if (im->plane_count < 1 || im->plane_count > 16) return JO_ERR_INVALID;
    int32_t *planes[17] = {0};
    uint32_t pw[17], ph[17];
    int n = im->plane_count + (im->alpha ? 1 : 0), rc = JO_OK;
    for (int i = 0; i < n; i++) {
        const jo_plane *p = i < im->plane_count ? &im->planes[i] : im->alpha;
        jo_plane_extent_scaled(p, denominator, &pw[i], &ph[i]);
        planes[i] = malloc(sizeof(int32_t) * ((size_t)pw[i] * ph[i] + 1));
        if (!planes[i]) { rc = JO_ERR_INVALID; goto done; }
        rc = denominator == 4 ? jo_reconstruct_plane_quarter(p, planes[i]) : jo_reconstruct_plane_sixteenth(p, planes[i]);
        if (rc) goto done;
    }
    const int32_t *alpha = im->alpha ? planes[im->plane_count] : NULL;
    int subsampled = denominator == 4 && (im->coded_color == JO_COLOR_YUV420 || im->coded_color == JO_COLOR_YUV422);
    if (subsampled && !is_planar_yuv(r)) {
        if (im->plane_count != 3) { rc = JO_ERR_INVALID; goto done; }
        for (int c = 1; c < 3; c++) {
            uint32_t ow = pw[c] * 2, oh = im->coded_color == JO_COLOR_YUV420 ? ph[c] * 2 : ph[c];
            if (ow != pw[0] || oh != ph[0]) { rc = JO_ERR_INVALID; goto done; }
            int32_t *up = malloc(sizeof(int32_t) * (size_t)ow * oh);
            if (!up) { rc = JO_ERR_INVALID; goto done; }
            rc = jo_upsample_chroma(planes[c], pw[c], ph[c], im->coded_color == JO_COLOR_YUV420 ? 1 : 2,
                                    im->centering_x, im->centering_y, up, threads);
            free(planes[c]);
            planes[c] = up;
            if (rc) goto done;
        }
    }
    rc = jo_format_output((const int32_t *const *)planes, im->plane_count, alpha, pw[0], ph[0], r, out, out_len);
done:
    for (int i = 0; i < n; i++) free(planes[i]);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* presentation orientation (crates/jxr/src/decoder/orientation.rs:5-211)    */
/* ------------------------------------------------------------------------ */

static int swaps_axes(int o) { return o >= JO_ORIENT_TRANSPOSE; }

/* source_coordinates, orientation.rs:193-211 */
static void source_coordinates(int o, size_t w, size_t h, size_t dx, size_t dy, size_t *sx, size_t *sy)
{
    switch (o) {
    case JO_ORIENT_MIRROR_HORIZONTAL: *sx = w - 1 - dx; *sy = dy; break;
    case JO_ORIENT_ROTATE180: *sx = w - 1 - dx; *sy = h - 1 - dy; break;
    case JO_ORIENT_MIRROR_VERTICAL: *sx = dx; *sy = h - 1 - dy; break;
    case JO_ORIENT_TRANSPOSE: *sx = dy; *sy = dx; break;
    case JO_ORIENT_ROTATE90: *sx = dy; *sy = h - 1 - dx; break;
    case JO_ORIENT_TRANSVERSE: *sx = w - 1 - dy; *sy = h - 1 - dx; break;
    case JO_ORIENT_ROTATE270: *sx = w - 1 - dy; *sy = dx; break;
    default: *sx = dx; *sy = dy;
    }
}

int jo_orient(const uint8_t *src, uint8_t *dst, uint32_t width, uint32_t height, uint32_t pixel_bytes,
              int orientation)
{
    /* orient_values, orientation.rs:164-189: whole pixels moved, channels in
     * their order; pixel_bytes 0 is one-bit luma packed most significant bit
     * first, each row padded to a byte (orient_bitpacked, 93-162) */
    if (orientation < 0 || orientation > JO_ORIENT_ROTATE270) return JO_ERR_INVALID;
    size_t w = width, h = height;
    size_t ow = swaps_axes(orientation) ? h : w, oh = swaps_axes(orientation) ? w : h;
    if (pixel_bytes == 0) {
        size_t in_stride = (w + 7) / 8, out_stride = (ow + 7) / 8;
        memset(dst, 0, out_stride * oh);
        for (size_t y = 0; y < oh; y++)
            for (size_t x = 0; x < ow; x++) {
                size_t sx, sy;
                source_coordinates(orientation, w, h, x, y, &sx, &sy);
                if (src[sy * in_stride + sx / 8] & (0x80 >> (sx % 8))) dst[y * out_stride + x / 8] |= (uint8_t)(0x80 >> (x % 8));
            }
        return JO_OK;
    }
    for (size_t y = 0; y < oh; y++)
        for (size_t x = 0; x < ow; x++) {
            size_t sx, sy;
            source_coordinates(orientation, w, h, x, y, &sx, &sy);
            memcpy(dst + (y * ow + x) * pixel_bytes, src + (sy * w + sx) * pixel_bytes, pixel_bytes);
        }
    return JO_OK;
}
