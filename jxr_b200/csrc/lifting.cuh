// lifting.cuh -- exact JPEG XR lifting operators for the B200 engine.
//
// Every operator exists in two forms sharing one operation order:
//   * a wrapping form (CK = false) for inputs whose magnitudes are below the
//     operator's bound, where no intermediate can leave int32, and
//   * a checked form (CK = true) that reports the first intermediate that
//     leaves int32, as the reference's checked arithmetic does
//     (crates/jxr-math/src/arithmetic.rs:58-84).
// A caller tests the bound and picks the form, so values and errors are the
// reference's in both cases.  Bounds: 2^25 for the core transform and 2^23 for
// the 4x4 overlap operator -- the bounds under which the reference runs its own
// wrapping lane kernels of the same operation order
// (crates/jxr-native/src/reconstruct/lanes.rs:34-37); the unit tests check the
// two forms against each other over inputs at those bounds.
//
// Operation orders follow crates/jxr-math/src/transform.rs and overlap.rs.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define JXR_HD __host__ __device__ __forceinline__
#else
#define JXR_HD inline
#endif

namespace jxr {

constexpr int32_t kTransformBound = 1 << 25;
constexpr int32_t kOverlapBound = 1 << 23;

// Overflow-tracking integer steps.  `bad` accumulates overflow in checked form.
template <bool CK> struct Ar;

template <> struct Ar<false> {
    JXR_HD static int32_t add(int32_t a, int32_t b, bool &) { return a + b; }
    JXR_HD static int32_t sub(int32_t a, int32_t b, bool &) { return a - b; }
    JXR_HD static int32_t mul3(int32_t a, bool &) { return a * 3; }
    JXR_HD static int32_t neg(int32_t a, bool &) { return -a; }
};

template <> struct Ar<true> {
    JXR_HD static int32_t add(int32_t a, int32_t b, bool &bad) {
        int32_t r = (int32_t)((uint32_t)a + (uint32_t)b);
        bad |= ((a ^ r) & (b ^ r)) < 0;
        return r;
    }
    JXR_HD static int32_t sub(int32_t a, int32_t b, bool &bad) {
        int32_t r = (int32_t)((uint32_t)a - (uint32_t)b);
        bad |= ((a ^ b) & (a ^ r)) < 0;
        return r;
    }
    JXR_HD static int32_t mul3(int32_t a, bool &bad) {
        int64_t w = (int64_t)a * 3;
        bad |= w != (int64_t)(int32_t)w;
        return (int32_t)w;
    }
    JXR_HD static int32_t neg(int32_t a, bool &bad) {
        bad |= a == INT32_MIN;
        return (int32_t)(0u - (uint32_t)a);
    }
};

// |v| as the reference's magnitude test: v ^ (v >> 31) is |v| for v >= 0 and
// |v| - 1 otherwise; the OR of these bounds every magnitude below a power of
// two (crates/jxr-native/src/reconstruct/pipeline.rs:557-577).
JXR_HD uint32_t mag(int32_t v) { return (uint32_t)(v ^ (v >> 31)); }

// ---- core transform: crates/jxr-math/src/transform.rs -------------------

template <bool CK>
JXR_HD void t2x2h(int32_t &a, int32_t &b, int32_t &c, int32_t &d, int32_t rounding, bool &bad) {
    using A = Ar<CK>;
    a = A::add(a, d, bad);
    b = A::sub(b, c, bad);
    int32_t first = A::add(A::sub(a, b, bad), rounding, bad) >> 1;
    int32_t second = c;
    c = A::sub(first, d, bad);
    d = A::sub(first, second, bad);
    a = A::sub(a, d, bad);
    b = A::add(b, c, bad);
}

template <bool CK>
JXR_HD void inverse_todd(int32_t &a, int32_t &b, int32_t &c, int32_t &d, bool &bad) {
    using A = Ar<CK>;
    b = A::add(b, d, bad);
    a = A::sub(a, c, bad);
    d = A::sub(d, b >> 1, bad);
    c = A::add(c, A::add(a, 1, bad) >> 1, bad);
    a = A::sub(a, A::add(A::mul3(b, bad), 4, bad) >> 3, bad);
    b = A::add(b, A::add(A::mul3(a, bad), 4, bad) >> 3, bad);
    c = A::sub(c, A::add(A::mul3(d, bad), 4, bad) >> 3, bad);
    d = A::add(d, A::add(A::mul3(c, bad), 4, bad) >> 3, bad);
    c = A::sub(c, A::add(b, 1, bad) >> 1, bad);
    d = A::sub(A::add(a, 1, bad) >> 1, d, bad);
    b = A::add(b, c, bad);
    a = A::sub(a, d, bad);
}

template <bool CK>
JXR_HD void inverse_todd_odd(int32_t &a, int32_t &b, int32_t &c, int32_t &d, bool &bad) {
    using A = Ar<CK>;
    d = A::add(d, a, bad);
    c = A::sub(c, b, bad);
    int32_t first = d >> 1, second = c >> 1;
    a = A::sub(a, first, bad);
    b = A::add(b, second, bad);
    a = A::sub(a, A::add(A::mul3(b, bad), 3, bad) >> 3, bad);
    b = A::add(b, A::add(A::mul3(a, bad), 3, bad) >> 2, bad);
    a = A::sub(a, A::add(A::mul3(b, bad), 4, bad) >> 3, bad);
    b = A::sub(b, second, bad);
    a = A::add(a, first, bad);
    c = A::add(c, b, bad);
    d = A::sub(d, a, bad);
    b = A::neg(b, bad);
    c = A::neg(c, bad);
}

// Inverse 4x4 core transform of a block held in coefficient order (index k
// of the coded block; transform.rs:8-22).  Output is in raster sample order.
template <bool CK>
JXR_HD bool inverse_pct(int32_t (&v)[16]) {
    bool bad = false;
    // inverse permutation 0,8,4,13,2,15,3,14,1,12,5,9,7,11,6,10
    // (crates/jxr-math/data/reconstruction.abi:2): c[P[i]] = v[i].
    int32_t c0 = v[0], c8 = v[1], c4 = v[2], c13 = v[3], c2 = v[4], c15 = v[5], c3 = v[6], c14 = v[7];
    int32_t c1 = v[8], c12 = v[9], c5 = v[10], c9 = v[11], c7 = v[12], c11 = v[13], c6 = v[14], c10 = v[15];
    t2x2h<CK>(c0, c1, c4, c5, 1, bad);
    inverse_todd<CK>(c2, c3, c6, c7, bad);
    inverse_todd<CK>(c8, c12, c9, c13, bad);
    inverse_todd_odd<CK>(c10, c11, c14, c15, bad);
    t2x2h<CK>(c0, c3, c12, c15, 0, bad);
    t2x2h<CK>(c5, c6, c9, c10, 0, bad);
    t2x2h<CK>(c1, c2, c13, c14, 0, bad);
    t2x2h<CK>(c4, c7, c8, c11, 0, bad);
    v[0] = c0; v[1] = c1; v[2] = c2; v[3] = c3; v[4] = c4; v[5] = c5; v[6] = c6; v[7] = c7;
    v[8] = c8; v[9] = c9; v[10] = c10; v[11] = c11; v[12] = c12; v[13] = c13; v[14] = c14; v[15] = c15;
    return bad;
}

// First-level transforms of subsampled chroma (transform.rs:52-89).
template <bool CK>
JXR_HD bool inverse_chroma_420(int32_t (&v)[4]) {
    bool bad = false;
    t2x2h<CK>(v[0], v[1], v[2], v[3], 0, bad);
    int32_t t = v[1]; v[1] = v[2]; v[2] = t;
    return bad;
}

template <bool CK>
JXR_HD bool inverse_chroma_422(int32_t (&v)[8]) {
    using A = Ar<CK>;
    bool bad = false;
    v[0] = A::sub(v[0], A::add(v[4], 1, bad) >> 1, bad);
    v[4] = A::add(v[4], v[0], bad);
    t2x2h<CK>(v[0], v[1], v[2], v[3], 0, bad);
    int32_t t = v[1]; v[1] = v[2]; v[2] = t;
    t2x2h<CK>(v[4], v[6], v[5], v[7], 0, bad);
    t = v[5]; v[5] = v[6]; v[6] = t;
    return bad;
}

// ---- overlap operators: crates/jxr-math/src/overlap.rs -----------------

template <bool CK>
JXR_HD void inverse_scale(int32_t &a, int32_t &b, bool &bad) {
    using A = Ar<CK>;
    a = A::add(a, b, bad);
    b = A::sub(a >> 1, b, bad);
    a = A::add(a, A::mul3(b, bad) >> 3, bad);
    b = A::add(b, A::mul3(a, bad) >> 4, bad);
    b = A::add(b, a >> 7, bad);
    b = A::sub(b, a >> 10, bad);
}

template <bool CK>
JXR_HD void inverse_rotate(int32_t &a, int32_t &b, bool &bad) {
    using A = Ar<CK>;
    a = A::sub(a, A::add(b, 1, bad) >> 1, bad);
    b = A::add(b, A::add(a, 1, bad) >> 1, bad);
}

template <bool CK>
JXR_HD void inverse_hadamard_post(int32_t &a, int32_t &b, int32_t &c, int32_t &d, bool &bad) {
    using A = Ar<CK>;
    b = A::sub(b, c, bad);
    a = A::add(a, A::add(A::mul3(d, bad), 4, bad) >> 3, bad);
    d = A::sub(d, b >> 1, bad);
    c = A::sub(A::sub(a, b, bad) >> 1, c, bad);
    int32_t t = c; c = d; d = t;
    a = A::sub(a, d, bad);
    b = A::add(b, c, bad);
}

template <bool CK>
JXR_HD void inverse_todd_odd_post(int32_t &a, int32_t &b, int32_t &c, int32_t &d, bool &bad) {
    using A = Ar<CK>;
    d = A::add(d, a, bad);
    c = A::sub(c, b, bad);
    int32_t first = d >> 1, second = c >> 1;
    a = A::sub(a, first, bad);
    b = A::add(b, second, bad);
    a = A::sub(a, A::add(A::mul3(b, bad), 6, bad) >> 3, bad);
    b = A::add(b, A::add(A::mul3(a, bad), 2, bad) >> 2, bad);
    a = A::sub(a, A::add(A::mul3(b, bad), 4, bad) >> 3, bad);
    b = A::sub(b, second, bad);
    a = A::add(a, first, bad);
    c = A::add(c, b, bad);
    d = A::sub(d, a, bad);
}

// Inverse 4x4 overlap window in raster order (overlap.rs:139-161).
template <bool CK>
JXR_HD bool inverse_pot4x4(int32_t (&v)[16]) {
    bool bad = false;
    t2x2h<CK>(v[0], v[3], v[12], v[15], 0, bad);
    t2x2h<CK>(v[1], v[2], v[13], v[14], 0, bad);
    t2x2h<CK>(v[4], v[7], v[8], v[11], 0, bad);
    t2x2h<CK>(v[5], v[6], v[9], v[10], 0, bad);
    inverse_rotate<CK>(v[13], v[12], bad);
    inverse_rotate<CK>(v[9], v[8], bad);
    inverse_rotate<CK>(v[7], v[3], bad);
    inverse_rotate<CK>(v[6], v[2], bad);
    inverse_todd_odd_post<CK>(v[10], v[11], v[14], v[15], bad);
    inverse_scale<CK>(v[0], v[15], bad);
    inverse_scale<CK>(v[1], v[14], bad);
    inverse_scale<CK>(v[4], v[11], bad);
    inverse_scale<CK>(v[5], v[10], bad);
    inverse_hadamard_post<CK>(v[0], v[3], v[12], v[15], bad);
    inverse_hadamard_post<CK>(v[1], v[2], v[13], v[14], bad);
    inverse_hadamard_post<CK>(v[4], v[7], v[8], v[11], bad);
    inverse_hadamard_post<CK>(v[5], v[6], v[9], v[10], bad);
    return bad;
}

// Four-sample edge / corner operator (overlap.rs:10-55); always checked:
// edges are a small share of the work.
JXR_HD bool inverse_pot4(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    using A = Ar<true>;
    bool bad = false;
    a = A::add(a, d, bad);
    b = A::add(b, c, bad);
    d = A::sub(d, A::add(a, 1, bad) >> 1, bad);
    c = A::sub(c, A::add(b, 1, bad) >> 1, bad);
    inverse_scale<true>(a, d, bad);
    inverse_scale<true>(b, c, bad);
    a = A::add(a, A::add(A::mul3(d, bad), 4, bad) >> 3, bad);
    b = A::add(b, A::add(A::mul3(c, bad), 4, bad) >> 3, bad);
    d = A::sub(d, a >> 1, bad);
    c = A::sub(c, b >> 1, bad);
    a = A::add(a, d, bad);
    b = A::add(b, c, bad);
    d = A::neg(d, bad);
    c = A::neg(c, bad);
    inverse_rotate<true>(c, d, bad);
    d = A::add(d, A::add(a, 1, bad) >> 1, bad);
    c = A::add(c, A::add(b, 1, bad) >> 1, bad);
    a = A::sub(a, d, bad);
    b = A::sub(b, c, bad);
    return bad;
}

// Subsampled first-level operators (overlap.rs:167-227); always checked.
JXR_HD bool inverse_pot2(int32_t &a, int32_t &b) {
    using A = Ar<true>;
    bool bad = false;
    b = A::add(b, A::add(a, 2, bad) >> 2, bad);
    a = A::add(a, A::add(b, 1, bad) >> 1, bad);
    a = A::add(a, b >> 5, bad);
    a = A::add(a, b >> 9, bad);
    a = A::add(a, b >> 13, bad);
    b = A::add(b, A::add(a, 2, bad) >> 2, bad);
    return bad;
}

JXR_HD bool inverse_pot2x2(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    using A = Ar<true>;
    bool bad = false;
    a = A::add(a, d, bad);
    b = A::add(b, c, bad);
    d = A::sub(d, A::add(a, 1, bad) >> 1, bad);
    c = A::sub(c, A::add(b, 1, bad) >> 1, bad);
    bad |= inverse_pot2(a, b);
    d = A::add(d, A::add(a, 1, bad) >> 1, bad);
    c = A::add(c, A::add(b, 1, bad) >> 1, bad);
    a = A::sub(a, d, bad);
    b = A::sub(b, c, bad);
    return bad;
}

// Bound dispatch: the wrapping form where every input is below the bound,
// the checked form otherwise.
JXR_HD bool pct16(int32_t (&v)[16]) {
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) m |= mag(v[i]);
    if (m < (uint32_t)kTransformBound) return inverse_pct<false>(v);
    return inverse_pct<true>(v);
}

JXR_HD bool pot16(int32_t (&v)[16]) {
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) m |= mag(v[i]);
    if (m < (uint32_t)kOverlapBound) return inverse_pot4x4<false>(v);
    return inverse_pot4x4<true>(v);
}

// Checked dequantization (quantization.rs:53-56).
JXR_HD int32_t dequant(int32_t c, uint32_t step, bool &bad) {
    int64_t w = (int64_t)c * (int64_t)step;
    bad |= w != (int64_t)(int32_t)w;
    return (int32_t)w;
}

}  // namespace jxr
