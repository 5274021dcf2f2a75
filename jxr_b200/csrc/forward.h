// forward.h -- the analysis side of the codec: forward lifting operators and
// the forward overlap schedules over a plane, exact inverses of the
// reconstruction operators of lifting.cuh.  Used by the synthetic input
// generator (synth.cpp) and by the calibration of quarter-resolution sample
// scales (sample_scale.cpp).
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "lifting.cuh"   // JXR_HD: the operators below run on the host and the device

namespace jxr {
namespace fwd {

// ---------------------------------------------------------------------------
// forward lifting (crates/jxr-math/src/transform.rs:30-146, overlap.rs:57-374),
// wrapping int32: inputs here never approach the range where it would wrap
// ---------------------------------------------------------------------------
JXR_HD void t2x2h(int32_t &a, int32_t &b, int32_t &c, int32_t &d, int32_t rounding) {
    a += d;
    b -= c;
    const int32_t first = (a - b + rounding) >> 1, second = c;
    c = first - d;
    d = first - second;
    a -= d;
    b += c;
}

JXR_HD void forward_todd(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    a += d;
    b -= c;
    d = ((a + 1) >> 1) - d;
    c += (b + 1) >> 1;
    d -= (3 * c + 4) >> 3;
    c += (3 * d + 4) >> 3;
    b -= (3 * a + 4) >> 3;
    a += (3 * b + 4) >> 3;
    c -= (a + 1) >> 1;
    d += b >> 1;
    a += c;
    b -= d;
}

JXR_HD void forward_todd_odd(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    b = -b;
    c = -c;
    d += a;
    c -= b;
    const int32_t first = d >> 1, second = c >> 1;
    a -= first;
    b += second;
    a += (3 * b + 4) >> 3;
    b -= (3 * a + 3) >> 2;
    a += (3 * b + 3) >> 3;
    b -= second;
    a += first;
    c += b;
    d -= a;
}

JXR_HD void forward_pct(int32_t (&s)[16]) {
    t2x2h(s[4], s[7], s[8], s[11], 0);
    t2x2h(s[1], s[2], s[13], s[14], 0);
    t2x2h(s[5], s[6], s[9], s[10], 0);
    t2x2h(s[0], s[3], s[12], s[15], 0);
    forward_todd_odd(s[10], s[11], s[14], s[15]);
    forward_todd(s[8], s[12], s[9], s[13]);
    forward_todd(s[2], s[3], s[6], s[7]);
    t2x2h(s[0], s[1], s[4], s[5], 1);
    int32_t in[16];
#pragma unroll
    for (int i = 0; i < 16; i++) in[i] = s[i];
    // the coefficient order: index k holds transform output P[k], P = 0, 8,
    // 4, 13, 2, 15, 3, 14, 1, 12, 5, 9, 7, 11, 6, 10 (reconstruction.abi:2)
    s[0] = in[0]; s[1] = in[8]; s[2] = in[4]; s[3] = in[13]; s[4] = in[2]; s[5] = in[15]; s[6] = in[3]; s[7] = in[14];
    s[8] = in[1]; s[9] = in[12]; s[10] = in[5]; s[11] = in[9]; s[12] = in[7]; s[13] = in[11]; s[14] = in[6]; s[15] = in[10];
}

JXR_HD void forward_420(int32_t (&s)[4]) {
    const int32_t t = s[1]; s[1] = s[2]; s[2] = t;
    t2x2h(s[0], s[1], s[2], s[3], 0);
}

JXR_HD void forward_422(int32_t (&s)[8]) {
    int32_t t = s[5]; s[5] = s[6]; s[6] = t;
    t2x2h(s[4], s[6], s[5], s[7], 0);
    t = s[1]; s[1] = s[2]; s[2] = t;
    t2x2h(s[0], s[1], s[2], s[3], 0);
    s[4] -= s[0];
    s[0] += (s[4] + 1) >> 1;
}

JXR_HD void forward_rotate(int32_t &a, int32_t &b) {
    b -= (a + 1) >> 1;
    a += (b + 1) >> 1;
}

JXR_HD void forward_scale(int32_t &a, int32_t &b) {
    b += a >> 10;
    b -= a >> 7;
    b -= (3 * a) >> 4;
    a -= (3 * b) >> 3;
    b = (a >> 1) - b;
    a -= b;
}

JXR_HD void forward_hadamard_pre(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    b -= c;
    a += d;
    const int32_t t = c; c = d; d = t;
    c = ((a - b) >> 1) - c;
    d += b >> 1;
    a -= (3 * d + 4) >> 3;
    b += c;
}

JXR_HD void forward_todd_odd_pre(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    d += a;
    c -= b;
    const int32_t first = d >> 1, second = c >> 1;
    a -= first;
    b += second;
    a += (3 * b + 4) >> 3;
    b -= (3 * a + 2) >> 2;
    a += (3 * b + 6) >> 3;
    b -= second;
    a += first;
    c += b;
    d -= a;
}

JXR_HD void forward_pot4x4(int32_t (&v)[16]) {
    forward_hadamard_pre(v[0], v[3], v[12], v[15]);
    forward_hadamard_pre(v[1], v[2], v[13], v[14]);
    forward_hadamard_pre(v[4], v[7], v[8], v[11]);
    forward_hadamard_pre(v[5], v[6], v[9], v[10]);
    forward_scale(v[0], v[15]);
    forward_scale(v[1], v[14]);
    forward_scale(v[4], v[11]);
    forward_scale(v[5], v[10]);
    forward_todd_odd_pre(v[10], v[11], v[14], v[15]);
    forward_rotate(v[13], v[12]);
    forward_rotate(v[9], v[8]);
    forward_rotate(v[7], v[3]);
    forward_rotate(v[6], v[2]);
    t2x2h(v[0], v[3], v[12], v[15], 0);
    t2x2h(v[1], v[2], v[13], v[14], 0);
    t2x2h(v[4], v[7], v[8], v[11], 0);
    t2x2h(v[5], v[6], v[9], v[10], 0);
}

JXR_HD void forward_pot4(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    b += c;
    a += d;
    c -= (b + 1) >> 1;
    d -= (a + 1) >> 1;
    forward_rotate(c, d);
    c = -c;
    d = -d;
    b -= c;
    a -= d;
    c += b >> 1;
    d += a >> 1;
    b -= (3 * c + 4) >> 3;
    a -= (3 * d + 4) >> 3;
    forward_scale(b, c);
    forward_scale(a, d);
    c += (b + 1) >> 1;
    d += (a + 1) >> 1;
    b -= c;
    a -= d;
}

JXR_HD void forward_pot2(int32_t &a, int32_t &b) {
    b -= (a + 2) >> 2;
    a -= b >> 13;
    a -= b >> 9;
    a -= b >> 5;
    a -= (b + 1) >> 1;
    b -= (a + 2) >> 2;
}

JXR_HD void forward_pot2x2(int32_t &a, int32_t &b, int32_t &c, int32_t &d) {
    b += c;
    a += d;
    c -= (b + 1) >> 1;
    d -= (a + 1) >> 1;
    forward_pot2(a, b);
    c += (b + 1) >> 1;
    d += (a + 1) >> 1;
    b -= c;
    a -= d;
}

// ---------------------------------------------------------------------------
// forward overlap schedules over a plane (the decoder's window lists, run with
// the forward operators; the subsampled one last step first)
// ---------------------------------------------------------------------------
struct Region { uint32_t l, r, t, b; };

inline std::vector<Region> regions(uint32_t w, uint32_t h, const std::vector<uint32_t> &cols, const std::vector<uint32_t> &rows,
                            bool hard, uint32_t sx, uint32_t sy) {
    std::vector<Region> out;
    if (!hard) {
        out.push_back({0, w, 0, h});
        return out;
    }
    for (size_t j = 0; j + 1 < rows.size(); j++)
        for (size_t i = 0; i + 1 < cols.size(); i++)
            out.push_back({cols[i] * sx, cols[i + 1] * sx, rows[j] * sy, rows[j + 1] * sy});
    return out;
}

inline void prefilter_full(std::vector<int32_t> &s, size_t stride, const std::vector<Region> &regs) {
    for (const Region &g : regs) {
        for (uint32_t y = g.t + 2; y + 2 < g.b; y += 4)
            for (uint32_t x = g.l + 2; x + 2 < g.r; x += 4) {
                int32_t v[16];
                for (int r = 0; r < 4; r++)
                    for (int c = 0; c < 4; c++) v[r * 4 + c] = s[(y + r) * stride + x + c];
                forward_pot4x4(v);
                for (int r = 0; r < 4; r++)
                    for (int c = 0; c < 4; c++) s[(y + r) * stride + x + c] = v[r * 4 + c];
            }
        auto f4 = [&](size_t a, size_t b, size_t c, size_t d) { forward_pot4(s[a], s[b], s[c], s[d]); };
        for (uint32_t y = g.t + 2; y + 2 < g.b; y += 4)
            for (uint32_t x : {g.l, g.l + 1, g.r - 2, g.r - 1})
                f4(y * stride + x, (y + 1) * stride + x, (y + 2) * stride + x, (y + 3) * stride + x);
        for (uint32_t x = g.l + 2; x + 2 < g.r; x += 4)
            for (uint32_t y : {g.t, g.t + 1, g.b - 2, g.b - 1}) {
                size_t o = y * stride + x;
                f4(o, o + 1, o + 2, o + 3);
            }
        const uint32_t cx[4] = {g.l, g.r - 2, g.l, g.r - 2}, cy[4] = {g.t, g.t, g.b - 2, g.b - 2};
        for (int k = 0; k < 4; k++) {
            size_t o = cy[k] * stride + cx[k];
            f4(o, o + 1, o + stride, o + stride + 1);
        }
    }
}

// The subsampled decoder steps of a region, inverted and run last to first.
inline void prefilter_subsampled(std::vector<int32_t> &s, size_t stride, const std::vector<Region> &regs) {
    for (const Region &g : regs) {
        auto boundary_row = [&](uint32_t row) {  // inverse of the decoder's boundary row
            size_t base = (size_t)row * stride;
            size_t c0 = base + g.l, n0 = base + g.l + 1, c1 = base + g.r - 1, n1 = base + g.r - 2;
            s[c1] -= s[n1];
            s[c0] -= s[n0];
            std::vector<uint32_t> xs;
            for (uint32_t x = g.l + 2; x < g.r; x += 2) xs.push_back(x);
            for (size_t m = xs.size(); m-- > 0;) forward_pot2(s[base + xs[m] - 1], s[base + xs[m]]);
            s[c1] += s[n1];
            s[c0] += s[n0];
        };
        boundary_row(g.b - 1);
        std::vector<uint32_t> ys;
        for (uint32_t y = g.t + 2; y < g.b; y += 2) ys.push_back(y);
        for (size_t k = ys.size(); k-- > 0;) {
            const uint32_t y = ys[k];
            for (uint32_t x : {g.r - 1, g.l})
                forward_pot2(s[(size_t)(y - 1) * stride + x], s[(size_t)y * stride + x]);
            std::vector<uint32_t> xs;
            for (uint32_t x = g.l + 2; x < g.r; x += 2) xs.push_back(x);
            for (size_t m = xs.size(); m-- > 0;) {
                const uint32_t x = xs[m];
                size_t a = (size_t)(y - 1) * stride + x - 1, b = (size_t)y * stride + x - 1;
                forward_pot2x2(s[a], s[a + 1], s[b], s[b + 1]);
            }
        }
        boundary_row(g.t);
    }
}

// Quantizer::quantize (crates/jxr-math/src/quantization.rs:28-50)
JXR_HD int quantize(int32_t c, uint32_t step, uint32_t offset) {
    if (offset >= step) offset = step - 1;
    const uint32_t m = c < 0 ? (uint32_t)(-(int64_t)c) : (uint32_t)c;
    const uint32_t carry = (m % step) >= step - offset ? 1 : 0;
    const uint32_t q = m / step + carry;
    return c < 0 ? -(int32_t)q : (int32_t)q;
}

}  // namespace fwd
}  // namespace jxr
