// synth.cpp -- seeded synthetic arenas (see synth.h).
#include "synth.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/jxr_b200.h"
#include "forward.h"

namespace {

using namespace jxr::fwd;

// ---------------------------------------------------------------------------
// seeded generation
// ---------------------------------------------------------------------------
inline uint64_t splitmix(uint64_t &state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double uniform(uint64_t &state) { return (splitmix(state) >> 11) * (1.0 / 9007199254740992.0); }
inline uint64_t hash64(uint64_t x) {
    uint64_t s = x;
    return splitmix(s);
}
inline double gauss_at(uint64_t seed, uint64_t index) {
    const uint64_t h1 = hash64(seed ^ (index * 2 + 1)), h2 = hash64(seed ^ (index * 2 + 2) ^ 0xABCDEFull);
    const double u1 = ((h1 >> 11) + 1) * (1.0 / 9007199254740993.0), u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// RGB8 photo content: 6 sinusoids (periods log-uniform 8..128 px, random
// phase and orientation) + N(0, 8^2) + 20 random flat rectangles, clipped.
std::vector<uint16_t> photo(uint32_t w, uint32_t h, int channels, uint64_t seed, int threads, int range) {
    uint64_t st = seed * 0x100000001B3ull + 17;
    struct Wave { double kx, ky, phase, amp[3]; };
    Wave waves[6];
    for (auto &wv : waves) {
        const double period = std::exp(std::log(8.0) + uniform(st) * (std::log(128.0) - std::log(8.0)));
        const double theta = uniform(st) * 3.141592653589793;
        wv.kx = 6.283185307179586 / period * std::cos(theta);
        wv.ky = 6.283185307179586 / period * std::sin(theta);
        wv.phase = uniform(st) * 6.283185307179586;
        for (double &a : wv.amp) a = 8.0 + uniform(st) * 24.0;
    }
    struct Rect { uint32_t x0, y0, x1, y1; double c[3]; };
    Rect rects[20];
    for (auto &r : rects) {
        const uint32_t rw = 1 + (uint32_t)(uniform(st) * std::max(1u, w / 4)), rh = 1 + (uint32_t)(uniform(st) * std::max(1u, h / 4));
        r.x0 = (uint32_t)(uniform(st) * w);
        r.y0 = (uint32_t)(uniform(st) * h);
        r.x1 = std::min(w, r.x0 + rw);
        r.y1 = std::min(h, r.y0 + rh);
        for (double &c : r.c) c = uniform(st) * 255.0;
    }
    const double base[3] = {96.0 + uniform(st) * 64, 96.0 + uniform(st) * 64, 96.0 + uniform(st) * 64};
    std::vector<uint16_t> out((size_t)w * h * channels);
    const double scale = range / 255.0;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long y = 0; y < (long)h; y++)
        for (uint32_t x = 0; x < w; x++) {
            double v[3];
            for (int c = 0; c < 3; c++) {
                double s = base[c];
                for (auto &wv : waves) s += wv.amp[c] * std::sin(wv.kx * x + wv.ky * y + wv.phase);
                s += 8.0 * gauss_at(seed * 3 + c, (uint64_t)y * w + x);
                v[c] = s;
            }
            for (auto &r : rects)
                if (x >= r.x0 && x < r.x1 && (uint32_t)y >= r.y0 && (uint32_t)y < r.y1)
                    for (int c = 0; c < 3; c++) v[c] = r.c[c];
            for (int c = 0; c < channels; c++) {
                const double q = std::min(255.0, std::max(0.0, v[c % 3])) * scale;
                out[((size_t)y * w + x) * channels + c] = (uint16_t)std::lround(q);
            }
        }
    return out;
}

// Soft-edged random ellipses, 8-bit alpha.
std::vector<uint16_t> ellipses(uint32_t w, uint32_t h, uint64_t seed, int threads) {
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 91;
    struct E { double cx, cy, rx, ry, soft; };
    E es[12];
    for (auto &e : es) {
        e.cx = uniform(st) * w;
        e.cy = uniform(st) * h;
        e.rx = 4 + uniform(st) * w / 3.0;
        e.ry = 4 + uniform(st) * h / 3.0;
        e.soft = 0.05 + uniform(st) * 0.3;
    }
    std::vector<uint16_t> a((size_t)w * h);
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long y = 0; y < (long)h; y++)
        for (uint32_t x = 0; x < w; x++) {
            double v = 0.1;
            for (auto &e : es) {
                const double dx = (x - e.cx) / e.rx, dy = (y - e.cy) / e.ry, d = std::sqrt(dx * dx + dy * dy);
                const double t = std::min(1.0, std::max(0.0, (1.0 - d) / e.soft));
                v = std::max(v, t);
            }
            a[(size_t)y * w + x] = (uint16_t)std::lround(v * 255.0);
        }
    return a;
}

// binary16 bits of a positive finite double, round to nearest even
uint16_t half_bits(double v) {
    if (v <= 0) return 0;
    int e;
    double m = std::frexp(v, &e);  // v = m * 2^e, m in [0.5, 1)
    int exp16 = e - 1 + 15;
    if (exp16 >= 31) return 0x7bff;
    if (exp16 <= 0) {
        const double sub = std::ldexp(v, 24);
        return (uint16_t)std::nearbyint(sub);
    }
    double frac = (m * 2.0 - 1.0) * 1024.0;
    uint32_t f = (uint32_t)std::nearbyint(frac);
    if (f == 1024) { f = 0; exp16++; }
    if (exp16 >= 31) return 0x7bff;
    return (uint16_t)((exp16 << 10) | f);
}

// exp of seeded smooth noise in [1e-3, 64] as half bits, 3 channels
std::vector<uint16_t> hdr(uint32_t w, uint32_t h, uint64_t seed, int threads) {
    uint64_t st = seed * 0xD1B54A32D192ED03ull + 5;
    struct Wave { double kx, ky, phase, amp; };
    std::vector<Wave> waves(8);
    for (auto &wv : waves) {
        const double period = std::exp(std::log(64.0) + uniform(st) * (std::log(2048.0) - std::log(64.0)));
        const double theta = uniform(st) * 6.283185307179586;
        wv.kx = 6.283185307179586 / period * std::cos(theta);
        wv.ky = 6.283185307179586 / period * std::sin(theta);
        wv.phase = uniform(st) * 6.283185307179586;
        wv.amp = 0.5 + uniform(st);
    }
    double total = 0;
    for (auto &wv : waves) total += wv.amp;
    const double lo = std::log(1e-3), hi = std::log(64.0);
    std::vector<uint16_t> out((size_t)w * h * 3);
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long y = 0; y < (long)h; y++)
        for (uint32_t x = 0; x < w; x++)
            for (int c = 0; c < 3; c++) {
                double s = 0;
                for (size_t k = 0; k < waves.size(); k++) {
                    const Wave &wv = waves[k];
                    s += wv.amp * std::sin(wv.kx * x + wv.ky * y + wv.phase + 0.7 * c * (k + 1));
                }
                const double t = 0.5 + 0.5 * s / total;  // [0, 1]
                out[((size_t)y * w + x) * 3 + c] = half_bits(std::exp(lo + t * (hi - lo)));
            }
    return out;
}

// ---------------------------------------------------------------------------
// quantization parameters
// ---------------------------------------------------------------------------
// QP -> step, crates/jxr-native/src/tile_decode/quantizer.rs:309-331
uint32_t quant_map(int qp, bool scaled, uint32_t shift) {
    if (qp <= 0) return 1;
    uint32_t mant, expo;
    if (scaled) {
        if (qp < 16) { mant = qp; expo = shift; }
        else { mant = 16 + qp % 16; expo = (qp >> 4) - 1 + shift; }
    } else if (qp < 32) { mant = (qp + 3) >> 2; expo = 0; }
    else if (qp < 48) { mant = (17 + qp % 16) / 2; expo = (qp >> 4) - 2; }
    else { mant = 16 + qp % 16; expo = (qp >> 4) - 3; }
    return mant << expo;
}

// quality -> (DC, LP, HP) QPs of 8-bit colour, encode/quality.rs:295-500:
// primary components (role Primary) and colour differences (Difference).
void quality_qps(int quality, int sampling_offset, int primary[3], int difference[3]) {
    if (quality >= 100) {
        for (int i = 0; i < 3; i++) primary[i] = difference[i] = 0;
        return;
    }
    int level;
    if (quality >= 99) level = 10;
    else if (quality >= 93) level = 16 + 8 * (98 - quality);
    else if (quality >= 91) level = 64 + 3 * (92 - quality);
    else if (quality >= 76) level = 70 + 2 * (90 - quality);
    else if (quality >= 11) level = 100 + (75 - quality);
    else level = 165 + 6 * (10 - quality);
    const int p = (level + 1) / 2, dlev = level / 2;
    const int excess = std::max(0, level - 64) / 2, relief = std::min(excess, 16);
    int off = dlev < 16 ? dlev * sampling_offset / 16 : sampling_offset;
    const int dparam = std::min(255, dlev + off);
    primary[0] = p - relief; primary[1] = p; primary[2] = p;
    difference[0] = dparam - relief; difference[1] = dparam; difference[2] = dparam;
}


struct PlaneSpec {
    std::vector<int32_t> samples;   // sample domain, row-major (W x H)
    uint32_t W, H;
    int bc, br;
    bool scale2;
    int overlap;
    uint32_t q[3];
};

}  // namespace

struct jxrb_synth {
    // arenas: index 0 primary, 1 separate alpha
    struct Arena {
        std::vector<int32_t> coefficients;
        std::vector<uint32_t> offsets, quantizers, coded_x, coded_y;
        std::vector<uint8_t> bands, hp;
        std::vector<uint64_t> plane_words;
    } arena[2];
    bool has_separate = false;
    uint32_t mbs_x = 0, mbs_y = 0;
    std::vector<uint32_t> tile_w, tile_h;
    std::vector<uint16_t> source;
    uint32_t source_channels = 0, source_bytes = 1;
};

namespace {

// Forward analysis of one plane into quantized macroblocks (raster):
// dc_lp[mb][16] and hp[mb][256] (coefficient order per block), crates/jxr-native/src/analyze.rs:56-131.
void analyze_plane(PlaneSpec &p, const std::vector<uint32_t> &cols, const std::vector<uint32_t> &rows, bool hard,
                   std::vector<int32_t> &low_q, std::vector<int32_t> &high_q, int threads) {
    const uint32_t mbx = p.W / (p.bc * 4), mby = p.H / (p.br * 4);
    const size_t stride = p.W;
    if (p.overlap >= 1) prefilter_full(p.samples, stride, regions(p.W, p.H, cols, rows, hard, p.bc * 4, p.br * 4));
    const uint32_t lw = mbx * p.bc, lh = mby * p.br;
    std::vector<int32_t> low((size_t)lw * lh);
    std::vector<int32_t> coeffs((size_t)lw * lh * 16);
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long by = 0; by < (long)lh; by++)
        for (uint32_t bx = 0; bx < lw; bx++) {
            int32_t v[16];
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) v[r * 4 + c] = p.samples[((size_t)by * 4 + r) * stride + bx * 4 + c];
            forward_pct(v);
            low[(size_t)by * lw + bx] = v[0];
            std::memcpy(&coeffs[((size_t)by * lw + bx) * 16], v, sizeof v);
        }
    if (p.overlap == 2) {
        if (p.bc == 4) prefilter_full(low, lw, regions(lw, lh, cols, rows, hard, p.bc, p.br));
        else prefilter_subsampled(low, lw, regions(lw, lh, cols, rows, hard, p.bc, p.br));
    }
    const int count = p.bc * p.br;
    low_q.assign((size_t)mbx * mby * 16, 0);
    high_q.assign((size_t)mbx * mby * 256, 0);
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long my = 0; my < (long)mby; my++)
        for (uint32_t mx = 0; mx < mbx; mx++) {
            const size_t m = (size_t)my * mbx + mx;
            int32_t l[16] = {0};
            for (int r = 0; r < p.br; r++)
                for (int c = 0; c < p.bc; c++) l[r * p.bc + c] = low[((size_t)my * p.br + r) * lw + mx * p.bc + c];
            if (p.scale2)
                for (int k = 0; k < count; k++) l[k] >>= 1;
            if (count == 16) forward_pct(l);
            else if (count == 4) { int32_t w[4] = {l[0], l[1], l[2], l[3]}; forward_420(w); std::memcpy(l, w, sizeof w); }
            else { int32_t w[8]; std::memcpy(w, l, sizeof w); forward_422(w); std::memcpy(l, w, sizeof w); }
            low_q[m * 16] = quantize(l[0], p.q[0], p.q[0] / 2);
            for (int k = 1; k < count; k++) low_q[m * 16 + k] = quantize(l[k], p.q[1], p.q[1] / 2);
            for (int b = 0; b < count; b++) {
                const int bx = mx * p.bc + b % p.bc, by = my * p.br + b / p.bc;
                const int32_t *src = &coeffs[((size_t)by * lw + bx) * 16];
                for (int k = 1; k < 16; k++) high_q[m * 256 + b * 16 + k] = quantize(src[k], p.q[2], p.q[2] / 3);
            }
        }
}

// high_pass_mode, crates/jxr-native/src/tile_decode/syntax.rs:203-231
int hp_direction(const int32_t *const *lows, int ncomp, int chroma) {
    auto energy = [](const int32_t *l, std::initializer_list<int> pos) {
        uint64_t s = 0;
        for (int p : pos) s += (uint64_t)std::abs((int64_t)l[p]);
        return s;
    };
    uint64_t horizontal = energy(lows[0], {1, 2, 3}), vertical = energy(lows[0], {4, 8, 12});
    if (ncomp >= 3) {
        for (int c = 1; c < 3; c++) {
            if (chroma == 1) { horizontal += energy(lows[c], {1}); vertical += energy(lows[c], {2}); }
            else if (chroma == 2) { horizontal += energy(lows[c], {1, 5}); vertical += energy(lows[c], {2, 6}); }
            else { horizontal += energy(lows[c], {1}); vertical += energy(lows[c], {4}); }
        }
    }
    if (horizontal * 4 < vertical) return 1;
    if (vertical * 4 < horizontal) return 2;
    return 0;
}

// Residuals of in-macroblock prediction: the inverse of
// crates/jxr-math/src/prediction.rs:110-154 (last block first).
void predict_forward(int32_t *hp, int dir, int bc, int br) {
    if (dir == 1) {
        for (int r = 0; r < br; r++)
            for (int c = bc - 1; c >= 1; c--)
                for (int k : {4, 8, 12}) hp[(r * bc + c) * 16 + k] -= hp[(r * bc + c - 1) * 16 + k];
    } else if (dir == 2) {
        for (int r = br - 1; r >= 1; r--)
            for (int c = 0; c < bc; c++)
                for (int k : {1, 2, 3}) hp[(r * bc + c) * 16 + k] -= hp[((r - 1) * bc + c) * 16 + k];
    }
}

void write_arena(jxrb_synth::Arena &a, std::vector<std::vector<int32_t>> &lows, std::vector<std::vector<int32_t>> &highs,
                 const std::vector<PlaneSpec> &specs, const std::vector<std::vector<uint8_t>> &dirs, uint32_t mbx, uint32_t mby,
                 const std::vector<uint32_t> &tw, const std::vector<uint32_t> &th, int bands, uint64_t seed,
                 bool random_meta) {
    uint64_t st = seed ^ 0x5151;
    for (size_t pi = 0; pi < specs.size(); pi++) {
        const PlaneSpec &p = specs[pi];
        const int count = p.bc * p.br;
        const uint64_t coeff0 = a.coefficients.size(), mb0 = a.offsets.size();
        // tile-major macroblock order, raster within a tile (the order the
        // tile decoder pushes them in)
        uint32_t ty0 = 0;
        for (uint32_t tr : th) {
            uint32_t tx0 = 0;
            for (uint32_t tc : tw) {
                for (uint32_t y = ty0; y < ty0 + tr; y++)
                    for (uint32_t x = tx0; x < tx0 + tc; x++) {
                        const size_t m = (size_t)y * mbx + x;
                        int b = bands;
                        int dir = dirs[pi][m];
                        if (random_meta) {
                            b = (int)(splitmix(st) % 4);
                            dir = (int)(splitmix(st) % 3);
                        }
                        if (b < 2) dir = 0;
                        a.offsets.push_back((uint32_t)(a.coefficients.size()));
                        a.quantizers.push_back(p.q[0]);
                        a.quantizers.push_back(p.q[1]);
                        a.quantizers.push_back(p.q[2]);
                        a.bands.push_back((uint8_t)b);
                        a.hp.push_back((uint8_t)dir);
                        a.coded_x.push_back(x);
                        a.coded_y.push_back(y);
                        int32_t *low = &lows[pi][m * 16];
                        int32_t *hp = &highs[pi][m * 256];
                        if (b >= 2) predict_forward(hp, dir, p.bc, p.br);
                        if (b == 0) a.coefficients.push_back(low[0]);
                        else if (b == 1) for (int k = 0; k < count; k++) a.coefficients.push_back(low[k]);
                        else
                            for (int k = 0; k < count; k++) {
                                a.coefficients.push_back(low[k]);
                                for (int j = 1; j < 16; j++) a.coefficients.push_back(hp[k * 16 + j]);
                            }
                    }
                tx0 += tc;
            }
            ty0 += tr;
        }
        const uint64_t words[6] = {coeff0, a.coefficients.size() - coeff0, mb0, a.offsets.size() - mb0,
                                   (uint64_t)p.bc, (uint64_t)p.br};
        a.plane_words.insert(a.plane_words.end(), words, words + 6);
    }
}

std::vector<uint32_t> tile_sizes(uint32_t total, uint32_t size) {
    std::vector<uint32_t> out;
    if (size == 0 || size >= total) {
        out.push_back(total);
        return out;
    }
    for (uint32_t at = 0; at < total; at += size) out.push_back(std::min(size, total - at));
    return out;
}

std::vector<uint32_t> boundaries(const std::vector<uint32_t> &sizes) {
    std::vector<uint32_t> b{0};
    for (uint32_t s : sizes) b.push_back(b.back() + s);
    return b;
}

}  // namespace

extern "C" {

int jxrb_synth_create(const jxrb_synth_request *r, int threads, jxrb_synth **out) {
    if (!r || !out || r->width == 0 || r->height == 0) return JXRB_INVALID_PLAN;
    if (threads <= 0) threads = 1;
    std::unique_ptr<jxrb_synth> s(new jxrb_synth);
    const uint32_t mbx = (r->width + 15) / 16, mby = (r->height + 15) / 16;
    const uint32_t W = mbx * 16, H = mby * 16;
    s->mbs_x = mbx;
    s->mbs_y = mby;
    s->tile_w = tile_sizes(mbx, r->tile_width);
    s->tile_h = tile_sizes(mby, r->tile_height);
    const auto cols = boundaries(s->tile_w), rows = boundaries(s->tile_h);
    const int color = r->color_format;
    const int ncomp = color == JXRB_COLOR_LUMA ? 1 : color == JXRB_COLOR_YUVK ? 4 : 3;
    const int chroma = color == JXRB_COLOR_YUV420 ? 1 : color == JXRB_COLOR_YUV422 ? 2 : 0;
    const bool scaled = r->scaled != 0;
    const bool random = r->content == JXRB_CONTENT_RANDOM;
    // source pixels
    std::vector<uint16_t> src;
    int channels = ncomp == 1 ? 1 : 3;
    int range = 255;
    if (r->content == JXRB_CONTENT_HDR_HALF) {
        src = hdr(r->width, r->height, r->seed, threads);
        channels = 3;
        s->source_bytes = 2;
    } else if (r->content == JXRB_CONTENT_GRAY16) {
        range = 65535;
        src = photo(r->width, r->height, channels, r->seed, threads, range);
        s->source_bytes = 2;
    } else {
        src = photo(r->width, r->height, channels, r->seed, threads, 255);
        s->source_bytes = 1;
    }
    s->source_channels = channels;
    // sample planes (extended to whole macroblocks by edge replication)
    auto pixel = [&](uint32_t x, uint32_t y, int c) {
        x = std::min(x, r->width - 1);
        y = std::min(y, r->height - 1);
        return (int32_t)src[((size_t)y * r->width + x) * channels + c];
    };
    // output unscaling (scaling.rs:121-147): sample = (value << shift) - shifted bias
    const int sh = scaled ? 3 : 0;
    int32_t bias = r->content == JXRB_CONTENT_HDR_HALF ? 0 : (range == 65535 ? 32768 : 128);
    std::vector<PlaneSpec> specs(ncomp);
    for (int c = 0; c < ncomp; c++) {
        specs[c].bc = (chroma && c > 0) ? 2 : 4;
        specs[c].br = (chroma == 1 && c > 0) ? 2 : 4;
        specs[c].W = W / (4 / specs[c].bc);
        specs[c].H = H / (4 / specs[c].br);
        specs[c].scale2 = scaled && c != 0;
        specs[c].overlap = r->overlap;
    }
    {
        std::vector<int32_t> Y((size_t)W * H), U, V, K;
        if (ncomp >= 3) { U.resize((size_t)W * H); V.resize((size_t)W * H); }
        if (ncomp == 4) K.resize((size_t)W * H);
#pragma omp parallel for schedule(static) num_threads(threads)
        for (long y = 0; y < (long)H; y++)
            for (uint32_t x = 0; x < W; x++) {
                const size_t i = (size_t)y * W + x;
                if (ncomp == 1) {
                    Y[i] = (pixel(x, y, 0) << sh) - (bias << sh);
                    continue;
                }
                const int32_t rr = (pixel(x, y, 0) << sh) - (bias << sh);
                const int32_t gg = (pixel(x, y, 1) << sh) - (bias << sh);
                const int32_t bb = (pixel(x, y, 2) << sh) - (bias << sh);
                // forward_yuv, output_format/color.rs:76-84
                const int32_t v = bb - rr;
                const int32_t t = rr - gg + ((v >> 1) + (v & 1));
                Y[i] = gg + (t >> 1);
                U[i] = -t;
                V[i] = v;
                // YUVK: a fourth plane of its own content (the mean of two
                // source channels), coded like the colour differences
                if (ncomp == 4) K[i] = (((pixel(x, y, 0) + pixel(x, y, 2)) >> 1) << sh) - (bias << sh);
            }
        specs[0].samples = std::move(Y);
        if (ncomp == 4) specs[3].samples = std::move(K);
        if (ncomp >= 3) {
            for (int c = 1; c < 3; c++) {
                std::vector<int32_t> &full = c == 1 ? U : V;
                if (!chroma) { specs[c].samples = std::move(full); continue; }
                // decimation: 1-4-6-4-1 / 16 mirrored (sampling.rs:78-100)
                const uint32_t cw = specs[c].W, ch = specs[c].H;
                std::vector<int32_t> half((size_t)cw * H);
                auto mirror = [](long p, long last) { if (p < 0) p = -p; if (p > last) p = std::max(0L, 2 * last - p); return std::min(p, last); };
                const int64_t wts[5] = {1, 4, 6, 4, 1};
#pragma omp parallel for schedule(static) num_threads(threads)
                for (long y = 0; y < (long)H; y++)
                    for (uint32_t x = 0; x < cw; x++) {
                        int64_t sum = 8;
                        for (int k = 0; k < 5; k++) sum += wts[k] * full[(size_t)y * W + mirror(2 * (long)x + k - 2, W - 1)];
                        half[(size_t)y * cw + x] = (int32_t)(sum >> 4);
                    }
                if (chroma == 2) { specs[c].samples = std::move(half); continue; }
                std::vector<int32_t> q((size_t)cw * ch);
#pragma omp parallel for schedule(static) num_threads(threads)
                for (long y = 0; y < (long)ch; y++)
                    for (uint32_t x = 0; x < cw; x++) {
                        int64_t sum = 8;
                        for (int k = 0; k < 5; k++) sum += wts[k] * half[(size_t)mirror(2 * y + k - 2, H - 1) * cw + x];
                        q[(size_t)y * cw + x] = (int32_t)(sum >> 4);
                    }
                specs[c].samples = std::move(q);
            }
        }
    }
    // quantizers
    int prim[3], diff[3];
    if (r->quality > 0) {
        quality_qps(r->quality, chroma == 1 ? 4 : chroma == 2 ? 8 : 16, prim, diff);
    } else {
        for (int i = 0; i < 3; i++) prim[i] = diff[i] = r->qp[i];
    }
    for (int c = 0; c < ncomp; c++) {
        const int *qp = c == 0 ? prim : diff;
        for (int b = 0; b < 3; b++) specs[c].q[b] = jxrb_quant_step(qp[b], scaled, c, b);
    }
    // analysis
    std::vector<std::vector<int32_t>> lows(ncomp), highs(ncomp);
    for (int c = 0; c < ncomp; c++) {
        if (random) {
            uint64_t st = r->seed * 7919 + c;
            lows[c].assign((size_t)mbx * mby * 16, 0);
            highs[c].assign((size_t)mbx * mby * 256, 0);
            for (auto &v : lows[c]) v = (int32_t)(splitmix(st) % 2001) - 1000;
            for (auto &v : highs[c]) v = (int32_t)(splitmix(st) % 401) - 200;
            for (int b = 0; b < 3; b++) specs[c].q[b] = 1 + (uint32_t)(splitmix(st) % 6);
        } else {
            analyze_plane(specs[c], cols, rows, r->hard_tiles != 0, lows[c], highs[c], threads);
        }
    }
    std::vector<uint8_t> dirs((size_t)mbx * mby, 0);
    for (size_t m = 0; m < dirs.size(); m++) {
        const int32_t *l[3] = {&lows[0][m * 16], ncomp >= 3 ? &lows[1][m * 16] : nullptr,
                               ncomp >= 3 ? &lows[2][m * 16] : nullptr};
        dirs[m] = (uint8_t)hp_direction(l, ncomp, chroma);
    }
    // alpha
    std::vector<PlaneSpec> alpha_spec;
    std::vector<std::vector<int32_t>> alow, ahigh;
    if (r->alpha_mode != JXRB_ALPHA_NONE) {
        std::vector<uint16_t> a = ellipses(r->width, r->height, r->seed + 1, threads);
        PlaneSpec p;
        p.bc = p.br = 4;
        p.W = W;
        p.H = H;
        p.scale2 = false;
        p.overlap = r->alpha_overlap;
        p.samples.resize((size_t)W * H);
        const bool half = r->content == JXRB_CONTENT_HDR_HALF;
        const int ash = (!half && scaled && r->alpha_qp[0] > 0) ? 3 : 0;
        for (uint32_t y = 0; y < H; y++)
            for (uint32_t x = 0; x < W; x++) {
                const int32_t v = a[(size_t)std::min(y, r->height - 1) * r->width + std::min(x, r->width - 1)];
                p.samples[(size_t)y * W + x] = half ? (int32_t)half_bits(v / 255.0) : ((v << ash) - (128 << ash));
            }
        for (int b = 0; b < 3; b++) p.q[b] = jxrb_quant_step(r->alpha_qp[b], ash != 0, 0, b);
        alpha_spec.push_back(std::move(p));
        alow.resize(1);
        ahigh.resize(1);
        analyze_plane(alpha_spec[0], cols, rows, r->hard_tiles != 0, alow[0], ahigh[0], threads);
    }
    if (r->alpha_mode == JXRB_ALPHA_INTEGRATED) {
        specs.push_back(alpha_spec[0]);
        lows.push_back(std::move(alow[0]));
        highs.push_back(std::move(ahigh[0]));
    }
    std::vector<std::vector<uint8_t>> plane_dirs(ncomp, dirs);
    if (r->alpha_mode == JXRB_ALPHA_INTEGRATED) {
        std::vector<uint8_t> adirs((size_t)mbx * mby, 0);
        for (size_t m = 0; m < adirs.size(); m++) {
            const int32_t *l[1] = {&lows.back()[m * 16]};
            adirs[m] = (uint8_t)hp_direction(l, 1, 0);
        }
        plane_dirs.push_back(std::move(adirs));
    }
    write_arena(s->arena[0], lows, highs, specs, plane_dirs, mbx, mby, s->tile_w, s->tile_h, r->bands, r->seed, random);
    if (r->alpha_mode == JXRB_ALPHA_SEPARATE) {
        std::vector<uint8_t> adirs((size_t)mbx * mby, 0);
        for (size_t m = 0; m < adirs.size(); m++) {
            const int32_t *l[1] = {&alow[0][m * 16]};
            adirs[m] = (uint8_t)hp_direction(l, 1, 0);
        }
        std::vector<std::vector<uint8_t>> alpha_dirs{adirs};
        write_arena(s->arena[1], alow, ahigh, alpha_spec, alpha_dirs, mbx, mby, s->tile_w, s->tile_h, r->bands,
                    r->seed + 3, random);
        s->has_separate = true;
    }
    s->source = std::move(src);
    *out = s.release();
    return 0;
}

void jxrb_synth_destroy(jxrb_synth *s) { delete s; }

int jxrb_synth_arena(const jxrb_synth *s, int which, jxrb_synth_arena_view *v) {
    if (!s || !v || which < 0 || which > 1) return JXRB_INVALID_PLAN;
    std::memset(v, 0, sizeof *v);
    if (which == 1 && !s->has_separate) return 0;
    const auto &a = s->arena[which];
    v->coefficients = a.coefficients.data();
    v->coefficient_count = a.coefficients.size();
    v->coefficient_offsets = a.offsets.data();
    v->quantizers = a.quantizers.data();
    v->coded_x = a.coded_x.data();
    v->coded_y = a.coded_y.data();
    v->bands = a.bands.data();
    v->hp_predictions = a.hp.data();
    v->macroblock_count = a.offsets.size();
    v->plane_words = a.plane_words.data();
    v->plane_count = (uint32_t)(a.plane_words.size() / 6);
    return 0;
}

int jxrb_synth_geometry(const jxrb_synth *s, uint32_t *mbs_x, uint32_t *mbs_y, const uint32_t **tile_widths,
                        uint32_t *tile_columns, const uint32_t **tile_heights, uint32_t *tile_rows) {
    if (!s) return JXRB_INVALID_PLAN;
    *mbs_x = s->mbs_x;
    *mbs_y = s->mbs_y;
    *tile_widths = s->tile_w.data();
    *tile_columns = (uint32_t)s->tile_w.size();
    *tile_heights = s->tile_h.data();
    *tile_rows = (uint32_t)s->tile_h.size();
    return 0;
}

const void *jxrb_synth_source(const jxrb_synth *s, uint32_t *channels, uint32_t *bytes) {
    if (!s) return nullptr;
    *channels = s->source_channels;
    *bytes = s->source_bytes;
    if (s->source_bytes == 1) {
        // narrow copy kept beside the 16-bit one
        static thread_local std::vector<uint8_t> narrow;
        narrow.assign(s->source.begin(), s->source.end());
        return narrow.data();
    }
    return s->source.data();
}

int jxrb_forward_core_transform(int32_t v[16]) { forward_pct(*reinterpret_cast<int32_t(*)[16]>(v)); return 0; }
int jxrb_forward_overlap_4x4(int32_t v[16]) { forward_pot4x4(*reinterpret_cast<int32_t(*)[16]>(v)); return 0; }
int jxrb_forward_overlap_4(int32_t v[4]) { forward_pot4(v[0], v[1], v[2], v[3]); return 0; }
int jxrb_forward_overlap_2x2(int32_t v[4]) { forward_pot2x2(v[0], v[1], v[2], v[3]); return 0; }
int jxrb_forward_overlap_2(int32_t v[2]) { forward_pot2(v[0], v[1]); return 0; }
int jxrb_forward_chroma_420(int32_t v[4]) { forward_420(*reinterpret_cast<int32_t(*)[4]>(v)); return 0; }
int jxrb_forward_chroma_422(int32_t v[8]) { forward_422(*reinterpret_cast<int32_t(*)[8]>(v)); return 0; }

// component_steps, crates/jxr-native/src/tile_decode/quantizer.rs:147-158:
// DC and low-pass of the first component take one more bit of scaled shift.
int jxrb_analyze_plane_cpu(const int32_t *samples, uint32_t width, uint32_t height, uint32_t block_columns,
                           uint32_t block_rows, int32_t scaled, int32_t overlap, const uint32_t steps[3],
                           const uint32_t *column_boundaries, uint32_t column_count, const uint32_t *row_boundaries,
                           uint32_t row_count, int32_t hard_tiles, int32_t *low_q, int32_t *high_q) {
    if (!samples || !steps || !column_boundaries || !row_boundaries || !low_q || !high_q) return JXRB_INVALID_PLAN;
    PlaneSpec p;
    p.samples.assign(samples, samples + (size_t)width * height);
    p.W = width;
    p.H = height;
    p.bc = (int)block_columns;
    p.br = (int)block_rows;
    p.scale2 = scaled != 0;
    p.overlap = overlap;
    for (int b = 0; b < 3; b++) p.q[b] = steps[b];
    const std::vector<uint32_t> cols(column_boundaries, column_boundaries + column_count);
    const std::vector<uint32_t> rows(row_boundaries, row_boundaries + row_count);
    std::vector<int32_t> lq, hq;
    analyze_plane(p, cols, rows, hard_tiles != 0, lq, hq, 1);
    std::copy(lq.begin(), lq.end(), low_q);
    std::copy(hq.begin(), hq.end(), high_q);
    return JXRB_OK;
}

uint32_t jxrb_quant_step(int32_t qp, int32_t scaled, int32_t component, int32_t band) {
    const uint32_t shift = band == 2 ? 1u : (component == 0 ? 1u : 0u);
    return quant_map(qp, scaled != 0, shift);
}

}  // extern "C"
