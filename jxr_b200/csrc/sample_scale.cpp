// sample_scale.cpp -- calibration of reduced-resolution sample scales (see
// sample_scale.h).  Host code: the probe is a few macroblocks along each axis.
#include "sample_scale.h"

#include <algorithm>
#include <cstdint>
#include <vector>

#include "forward.h"
#include "lifting.cuh"

namespace jxr {
namespace {

constexpr uint32_t kProbeExtent = 5;                                   // sample_scale.rs:52
constexpr int32_t kProbeLevels[4] = {0x10001, 0x10002, 0x10003, 0x10004};  // sample_scale.rs:42

// ProbeAxis (sample_scale.rs:352-430): one probe region for each region
// extent the component has along the axis (extents of five or more share
// one), and for each component macroblock the probe macroblock placed like it.
struct ProbeAxis {
    std::vector<uint32_t> boundaries{0};
    uint32_t macroblocks = 0;
    std::vector<uint32_t> positions;
};

uint32_t probe_offset(uint32_t offset, uint32_t extent) {   // sample_scale.rs:432-443
    const uint32_t ends = kProbeExtent / 2;
    if (extent <= kProbeExtent || offset < ends) return offset;
    if (extent - offset <= ends) return kProbeExtent - (extent - offset);
    return ends;
}

bool probe_axis(const std::vector<uint32_t> &regions, ProbeAxis &a) {
    int starts[kProbeExtent + 1];
    std::fill(starts, starts + kProbeExtent + 1, -1);
    if (regions.size() < 2) return false;
    for (size_t i = 0; i + 1 < regions.size(); i++) {
        if (regions[i + 1] <= regions[i]) return false;
        const uint32_t extent = regions[i + 1] - regions[i];
        const uint32_t pe = std::min(extent, kProbeExtent);
        if (starts[pe] < 0) {
            starts[pe] = (int)a.macroblocks;
            a.macroblocks += pe;
            a.boundaries.push_back(a.macroblocks);
        }
        for (uint32_t o = 0; o < extent; o++) a.positions.push_back((uint32_t)starts[pe] + probe_offset(o, extent));
    }
    return true;
}

struct Geo {
    int bc, br;
    bool scale2;
    int overlap;
    bool sixteenth;                     // one sample a macroblock
    uint32_t mbs_x, mbs_y;
    std::vector<uint32_t> cols, rows;   // hard region boundaries of the probe
};

// The decoder's first-level overlap schedule over the block-DC plane of the
// probe (every region a hard tile), full resolution: disjoint windows.
bool inverse_low_full(std::vector<int32_t> &s, size_t stride, const fwd::Region &g) {
    bool bad = false;
    for (uint32_t y = g.t + 2; y + 2 < g.b; y += 4)
        for (uint32_t x = g.l + 2; x + 2 < g.r; x += 4) {
            int32_t v[16];
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) v[r * 4 + c] = s[(y + r) * stride + x + c];
            bad |= inverse_pot4x4<true>(v);
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) s[(y + r) * stride + x + c] = v[r * 4 + c];
        }
    auto f4 = [&](size_t a, size_t b, size_t c, size_t d) { bad |= inverse_pot4(s[a], s[b], s[c], s[d]); };
    for (uint32_t y = g.t + 2; y + 2 < g.b; y += 4)
        for (uint32_t x : {g.l, g.l + 1, g.r - 2, g.r - 1})
            f4(y * stride + x, (y + 1) * stride + x, (y + 2) * stride + x, (y + 3) * stride + x);
    for (uint32_t x = g.l + 2; x + 2 < g.r; x += 4)
        for (uint32_t y : {g.t, g.t + 1, g.b - 2, g.b - 1}) {
            const size_t o = y * stride + x;
            f4(o, o + 1, o + 2, o + 3);
        }
    const uint32_t cx[4] = {g.l, g.r - 2, g.l, g.r - 2}, cy[4] = {g.t, g.t, g.b - 2, g.b - 2};
    for (int k = 0; k < 4; k++) {
        const size_t o = cy[k] * stride + cx[k];
        f4(o, o + 1, o + stride, o + stride + 1);
    }
    return bad;
}

// The subsampled first-level schedule of one region, first step to last
// (crates/jxr-native/src/reconstruct/subsampled_overlap.rs:244-296).
bool inverse_low_subsampled(std::vector<int32_t> &s, size_t stride, const fwd::Region &g) {
    using A = Ar<true>;
    bool bad = false;
    auto boundary_row = [&](uint32_t row) {
        const size_t base = (size_t)row * stride;
        const size_t c0 = base + g.l, n0 = base + g.l + 1, c1 = base + g.r - 1, n1 = base + g.r - 2;
        s[c0] = A::sub(s[c0], s[n0], bad);
        s[c1] = A::sub(s[c1], s[n1], bad);
        for (uint32_t x = g.l + 2; x < g.r; x += 2) bad |= inverse_pot2(s[base + x - 1], s[base + x]);
        s[c0] = A::add(s[c0], s[n0], bad);
        s[c1] = A::add(s[c1], s[n1], bad);
    };
    boundary_row(g.t);
    for (uint32_t y = g.t + 2; y < g.b; y += 2) {
        for (uint32_t x = g.l + 2; x < g.r; x += 2) {
            const size_t a = (size_t)(y - 1) * stride + x - 1, b = (size_t)y * stride + x - 1;
            bad |= inverse_pot2x2(s[a], s[a + 1], s[b], s[b + 1]);
        }
        for (uint32_t x : {g.l, g.r - 1}) bad |= inverse_pot2(s[(size_t)(y - 1) * stride + x], s[(size_t)y * stride + x]);
    }
    boundary_row(g.b - 1);
    return bad;
}

// The unscaled reduced picture of a flat probe image at `level`: the
// unit-step analysis (analyze_component, crates/jxr-native/src/analyze.rs:56-86,
// with Steps::new 505-535) and then the reduced decode: block_dc_plane
// (pipeline.rs:459-541) for a quarter, macroblock_dc_plane (387-457) for a
// sixteenth.
bool flat_picture(const Geo &g, int32_t level, std::vector<int32_t> &picture) {
    const uint32_t lw = g.mbs_x * g.bc, lh = g.mbs_y * g.br, W = lw * 4, H = lh * 4;
    std::vector<int32_t> s((size_t)W * H, level);
    if (g.overlap >= 1) fwd::prefilter_full(s, W, fwd::regions(W, H, g.cols, g.rows, true, g.bc * 4, g.br * 4));
    std::vector<int32_t> low((size_t)lw * lh);
    for (uint32_t by = 0; by < lh; by++)
        for (uint32_t bx = 0; bx < lw; bx++) {
            int32_t v[16];
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) v[r * 4 + c] = s[((size_t)by * 4 + r) * W + bx * 4 + c];
            fwd::forward_pct(v);
            low[(size_t)by * lw + bx] = v[0];
        }
    const auto low_regions = fwd::regions(lw, lh, g.cols, g.rows, true, g.bc, g.br);
    if (g.overlap == 2) {
        if (g.bc == 4) fwd::prefilter_full(low, lw, low_regions);
        else fwd::prefilter_subsampled(low, lw, low_regions);
    }
    const uint32_t divisor = g.scale2 ? 2 : 1;
    const int count = g.bc * g.br;
    picture.assign((size_t)lw * lh, 0);
    bool bad = false;
    for (uint32_t my = 0; my < g.mbs_y; my++)
        for (uint32_t mx = 0; mx < g.mbs_x; mx++) {
            int32_t l[16] = {0};
            for (int r = 0; r < g.br; r++)
                for (int c = 0; c < g.bc; c++) l[r * g.bc + c] = low[((size_t)my * g.br + r) * lw + mx * g.bc + c];
            if (count == 16) {
                fwd::forward_pct(*reinterpret_cast<int32_t(*)[16]>(l));
            } else if (count == 4) {
                int32_t w[4] = {l[0], l[1], l[2], l[3]};
                fwd::forward_420(w);
                std::copy(w, w + 4, l);
            } else {
                int32_t w[8];
                std::copy(l, l + 8, w);
                fwd::forward_422(w);
                std::copy(w, w + 8, l);
            }
            for (int k = 0; k < count; k++) l[k] = fwd::quantize(l[k], divisor, divisor / 2);
            // the reduced decode of the quantized macroblock (unit steps)
            if (g.sixteenth && g.overlap != 2) {
                // the macroblock's DC, doubled where the plane is scaled
                picture[(size_t)my * g.mbs_x + mx] = g.scale2 ? dequant(l[0], 2, bad) : l[0];
                continue;
            }
            if (g.sixteenth) std::fill(l + 1, l + count, 0);   // LowBands::Dc
            if (count == 16) {
                bad |= inverse_pct<true>(*reinterpret_cast<int32_t(*)[16]>(l));
            } else if (count == 4) {
                int32_t w[4] = {l[0], l[1], l[2], l[3]};
                bad |= inverse_chroma_420<true>(w);
                std::copy(w, w + 4, l);
            } else {
                int32_t w[8];
                std::copy(l, l + 8, w);
                bad |= inverse_chroma_422<true>(w);
                std::copy(w, w + 8, l);
            }
            for (int k = 0; k < count; k++)
                if (g.scale2) l[k] = dequant(l[k], 2, bad);
            for (int r = 0; r < g.br; r++)
                for (int c = 0; c < g.bc; c++) picture[((size_t)my * g.br + r) * lw + mx * g.bc + c] = l[r * g.bc + c];
        }
    if (g.sixteenth && g.overlap != 2) {
        picture.resize((size_t)g.mbs_x * g.mbs_y);   // one sample a macroblock
        return !bad;
    }
    if (g.overlap == 2)
        for (const fwd::Region &rg : low_regions)
            bad |= g.bc == 4 ? inverse_low_full(picture, lw, rg) : inverse_low_subsampled(picture, lw, rg);
    if (g.sixteenth) {
        // each macroblock's blocks summed, row by row (sum_macroblocks,
        // pipeline.rs:421-457); a macroblock's place precedes its blocks'
        for (uint32_t my = 0; my < g.mbs_y; my++)
            for (uint32_t mx = 0; mx < g.mbs_x; mx++) {
                int32_t sum = 0;
                for (int r = 0; r < g.br; r++)
                    for (int c = 0; c < g.bc; c++)
                        sum = Ar<true>::add(sum, picture[((size_t)my * g.br + r) * lw + mx * g.bc + c], bad);
                picture[(size_t)my * g.mbs_x + mx] = sum;
            }
        picture.resize((size_t)g.mbs_x * g.mbs_y);
    }
    return !bad;
}

}  // namespace

bool reduced_scale(int denominator, int bc, int br, bool scale2, int overlap, uint32_t mbs_x, uint32_t mbs_y,
                   const std::vector<uint32_t> &cols, const std::vector<uint32_t> &rows, QuarterScale &out,
                   std::string &why) {
    out = QuarterScale{};
    const bool sixteenth = denominator == 16;
    // samples a macroblock across and down the reduced picture
    const uint32_t ux = sixteenth ? 1u : (uint32_t)bc, uy = sixteenth ? 1u : (uint32_t)br;
    if (overlap == 0) {
        // the transform gains alone (scale_reduced_samples, pipeline.rs:81-102):
        // BLOCK_DC_GAIN_BITS (sample_scale.rs:16), and for a sixteenth the
        // macroblock transform's too (macroblock_dc_gain_bits, 22-30)
        out.shift = sixteenth ? ((bc == 4 && br == 4) ? 2 : 1) + 2 : 2;
        return true;
    }
    ProbeAxis ax, ay;
    if (!probe_axis(cols, ax) || !probe_axis(rows, ay) || ax.positions.size() != mbs_x ||
        ay.positions.size() != mbs_y) {
        why = "reduced-resolution sample scale: invalid tile partition";
        return false;
    }
    Geo g{bc, br, scale2, overlap, sixteenth, ax.macroblocks, ay.macroblocks, ax.boundaries, ay.boundaries};
    const size_t stride = (size_t)ax.macroblocks * ux, length = stride * ay.macroblocks * uy;
    std::vector<int64_t> rise(length, 0), offset(length, 0);
    int64_t span = 0, count = 0;
    std::vector<int32_t> up, down;
    for (int32_t level : kProbeLevels) {
        if (!flat_picture(g, level, up) || !flat_picture(g, -level, down) || up.size() != length ||
            down.size() != length) {
            why = "reduced-resolution sample scale: probe arithmetic overflow";
            return false;
        }
        for (size_t i = 0; i < length; i++) {
            rise[i] += (int64_t)up[i] - down[i];
            offset[i] += (int64_t)up[i] + down[i];
        }
        span += 2 * (int64_t)level;
        count += 2;
    }
    out.divisor.resize(length);
    out.bias.resize(length);
    for (size_t i = 0; i < length; i++) {
        const int64_t divisor = count * rise[i];
        if (divisor <= 0) {
            why = "reduced-resolution sample scale";
            return false;
        }
        out.divisor[i] = divisor;
        out.bias[i] = offset[i] * span - divisor / 2;
    }
    out.gain = count * span;
    out.probe_stride = (uint32_t)stride;
    out.columns.resize((size_t)mbs_x * ux);
    out.rows.resize((size_t)mbs_y * uy);
    for (size_t x = 0; x < out.columns.size(); x++) out.columns[x] = ax.positions[x / ux] * ux + (uint32_t)(x % ux);
    for (size_t y = 0; y < out.rows.size(); y++) out.rows[y] = ay.positions[y / uy] * uy + (uint32_t)(y % uy);
    return true;
}

}  // namespace jxr
