// recon_kernel.cu -- fused JPEG XR reconstruction for sm_100a.
//
// One CTA reconstructs one output tile of an image, every plane, in a single
// pass: dequantization and the first-level inverse transform of each
// macroblock, the first-level overlap filter on the block-DC plane, high-pass
// prediction, dequantization and the second-level inverse transform of each
// block, the second-level overlap filter on the samples, and finally chroma
// upsampling, colour conversion, scaling and packing into the output surface.
// Intermediates live in shared memory only: HBM sees the arena once and the
// output once; the halo a tile shares with its neighbours is served from L2.
//
// Geometry.  Every overlap operator of the reference's schedules
// (crates/jxr-core/src/device_plan/overlap.rs:125-253,
// crates/jxr-native/src/reconstruct/overlap.rs:124-323) lies inside one 4x4
// "cell" whose origin is 2 (mod 4) in plane coordinates: an interior window,
// four edge strips, or four 2x2 corners, depending on whether a region
// boundary (plane edge or hard tile edge) passes through the middle of the
// cell horizontally, vertically, or both.  The subsampled chroma schedule
// (crates/jxr-native/src/reconstruct/subsampled_overlap.rs:244-296) is the
// same with 2x2 cells at odd origins, plus ordered corner residuals.  A CTA
// therefore owns the output columns [16*mx0 + 2, 16*mx1 + 2) of its
// macroblock range (0 and the plane width at the edges), whole cells, and
// reconstructs the blocks those cells read.
//
// Shared memory.  Each plane's blocks are held block-major: block b of the
// tile occupies 16 consecutive ints, its row r (4 samples, one 16-byte chunk)
// stored at chunk r ^ ((b >> 1) & 3), which keeps 128-bit accesses of
// consecutive blocks free of bank conflicts.  The coded high-pass coefficients
// of a block land in their slot straight from HBM (cp.async, 16 bytes at a
// time) while the first level runs; prediction, dequantization and the
// second-level transform then work in place.
//
// Stages run plane-major within each barrier phase (all planes' first levels,
// then all planes' first-level overlap, ...), so every phase has the work of
// every plane to spread over the CTA's threads.
#include <cuda_runtime.h>
#include <stdint.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <mutex>

#include "engine.h"
#include "lifting.cuh"

namespace jxr {

constexpr int kThreads = 256;
constexpr int kTileMbs = 4;                    // macroblocks across / down a CTA tile
constexpr int kTileBlocks = kTileMbs * 4 + 1;  // 17 blocks across / down (full resolution)
constexpr int kPlaneInts = kTileBlocks * kTileBlocks * 16;
constexpr int kDcInts = 24 * 24;

enum OutKind : int32_t { kOutGeneric = 0, kOutRgb8 = 1, kOutDirect = 2, kOutF16Wide = 3 };

// failure flags of one tile, reported as the reference's stage codes
enum TileFlag : int {
    kFlagFirst = 1, kFlagOverlap = 2, kFlagPrediction = 4, kFlagSecond = 8, kFlagOutput = 16, kFlagInvalid = 32
};

struct PlaneGeom {
    int W, H;                    // sample plane
    int Wdc, Hdc;                // block-DC plane
    int bx0, bx1, by0, by1;      // blocks reconstructed (inclusive)
    int cx0, cx1, cy0, cy1;      // overlap cells (inclusive, step 4); empty if cx1 < cx0
    int mx0, mx1, my0, my1;      // macroblocks whose first level runs (inclusive)
    int nbx;                     // blocks across the tile
    int dw;                      // DC tile stride
    int ox0, ox1, oy0, oy1;      // subsampled first-level cells (odd origins, inclusive)
    int sx0, sx1, sy0, sy1;      // samples the output reads (exclusive ends)
    uint32_t vmask, hmask;       // sample cells split by a region boundary (bit i: cell cx0 + 4i)
    uint32_t dvmask, dhmask;     // first-level cells (full resolution) split likewise
};

__device__ __forceinline__ int cell_of(int p) { return ((p + 2) & ~3) - 2; }
__device__ __forceinline__ int odd_cell_of(int p) { return p - 1 + (p & 1); }

// Whether a region boundary lies at plane position p.  `lg` is log2 of the
// plane's macroblock extent along the axis (2, 3 or 4: every extent is a
// power of two), `starts` marks the macroblocks where a hard tile begins.
__device__ __forceinline__ bool boundary_at(int p, int extent, int lg, int hard, const uint8_t *starts) {
    if (p <= 0 || p >= extent) return true;
    if (!hard || (p & ((1 << lg) - 1)) != 0) return false;
    return starts[p >> lg] != 0;
}

__device__ __forceinline__ int log2_of(int v) { return 31 - __clz(v); }

__device__ __forceinline__ int swz(int b) { return (b >> 1) & 3; }

// element (r, c) of block slot b
__device__ __forceinline__ int elem(int b, int r, int c) { return b * 16 + ((r ^ swz(b)) << 2) + c; }

// ---------------------------------------------------------------------------
// geometry of one plane for the CTA's output region [X0, X1) x [Y0, Y1)
// (full-resolution sample coordinates)
// ---------------------------------------------------------------------------
__device__ void plane_geometry(const PlaneDev &p, bool chroma_plane, int chroma, int X0, int X1, int Y0, int Y1,
                               PlaneGeom &g) {
    g.Wdc = (int)p.mbs_x * p.bc;
    g.Hdc = (int)p.mbs_y * p.br;
    g.W = g.Wdc * 4;
    g.H = g.Hdc * 4;
    int s0, s1, t0, t1;
    if (chroma_plane && chroma != 0) {
        // samples the T.832 example upsampler reads: one beyond either side
        s0 = max(0, (X0 >> 1) - 1);
        s1 = min(g.W, ((X1 - 1) >> 1) + 2);
        if (chroma == 1) {
            t0 = max(0, (Y0 >> 1) - 1);
            t1 = min(g.H, ((Y1 - 1) >> 1) + 2);
        } else {
            t0 = Y0;
            t1 = Y1;
        }
    } else {
        s0 = X0; s1 = X1; t0 = Y0; t1 = Y1;
    }
    g.sx0 = s0; g.sx1 = s1; g.sy0 = t0; g.sy1 = t1;
    if (p.overlap >= 1) {
        g.cx0 = cell_of(s0); g.cx1 = cell_of(s1 - 1);
        g.cy0 = cell_of(t0); g.cy1 = cell_of(t1 - 1);
        g.bx0 = max(0, g.cx0) >> 2; g.bx1 = (min(g.W, g.cx1 + 4) - 1) >> 2;
        g.by0 = max(0, g.cy0) >> 2; g.by1 = (min(g.H, g.cy1 + 4) - 1) >> 2;
    } else {
        g.cx0 = 0; g.cx1 = -1; g.cy0 = 0; g.cy1 = -1;
        g.bx0 = s0 >> 2; g.bx1 = (s1 - 1) >> 2;
        g.by0 = t0 >> 2; g.by1 = (t1 - 1) >> 2;
    }
    // High-pass prediction runs from the first block of a macroblock row or
    // column, so reconstruction starts at a macroblock boundary.
    g.bx0 = (g.bx0 / p.bc) * p.bc;
    g.by0 = (g.by0 / p.br) * p.br;
    int d0x, d1x, d0y, d1y;  // DC cover, exclusive end
    g.ox0 = 0; g.ox1 = -1; g.oy0 = 0; g.oy1 = -1;
    if (p.overlap == 2) {
        if (p.bc == 4) {
            d0x = max(0, cell_of(g.bx0)); d1x = min(g.Wdc, cell_of(g.bx1) + 4);
            d0y = max(0, cell_of(g.by0)); d1y = min(g.Hdc, cell_of(g.by1) + 4);
        } else {
            // odd 2x2 cells, one more on each side for the corner residuals
            g.ox0 = odd_cell_of(g.bx0) - 2; g.ox1 = odd_cell_of(g.bx1) + 2;
            g.oy0 = odd_cell_of(g.by0) - 2; g.oy1 = odd_cell_of(g.by1) + 2;
            d0x = max(0, g.ox0); d1x = min(g.Wdc, g.ox1 + 2);
            d0y = max(0, g.oy0); d1y = min(g.Hdc, g.oy1 + 2);
        }
    } else {
        d0x = g.bx0; d1x = g.bx1 + 1; d0y = g.by0; d1y = g.by1 + 1;
    }
    g.mx0 = d0x / p.bc; g.mx1 = (d1x - 1) / p.bc;
    g.my0 = d0y / p.br; g.my1 = (d1y - 1) / p.br;
    g.nbx = g.bx1 - g.bx0 + 1;
    g.dw = (g.mx1 - g.mx0 + 1) * p.bc;
}

// Region-boundary flags of the cells of one plane, one cell a lane
// (a tile has at most 18 cells along an axis).
__device__ void plane_masks(const PlaneDev &p, PlaneGeom &g, int lane) {
    const int lx = log2_of(p.bc * 4), ly = log2_of(p.br * 4);
    const int ncx = g.cx1 >= g.cx0 ? (g.cx1 - g.cx0) / 4 + 1 : 0;
    const int ncy = g.cy1 >= g.cy0 ? (g.cy1 - g.cy0) / 4 + 1 : 0;
    const bool v = lane < ncx && boundary_at(g.cx0 + 4 * lane + 2, g.W, lx, p.hard, p.col_start);
    const bool h = lane < ncy && boundary_at(g.cy0 + 4 * lane + 2, g.H, ly, p.hard, p.row_start);
    g.vmask = __ballot_sync(0xffffffffu, v);
    g.hmask = __ballot_sync(0xffffffffu, h);
    bool dv = false, dh = false;
    if (p.overlap == 2 && p.bc == 4) {
        const int c0 = cell_of(g.bx0), r0 = cell_of(g.by0);
        const int ndx = (cell_of(g.bx1) - c0) / 4 + 1, ndy = (cell_of(g.by1) - r0) / 4 + 1;
        dv = lane < ndx && boundary_at(c0 + 4 * lane + 2, g.Wdc, 2, p.hard, p.col_start);
        dh = lane < ndy && boundary_at(r0 + 4 * lane + 2, g.Hdc, 2, p.hard, p.row_start);
    }
    g.dvmask = __ballot_sync(0xffffffffu, dv);
    g.dhmask = __ballot_sync(0xffffffffu, dh);
}

// ---------------------------------------------------------------------------
// stage 0: coded high-pass coefficients of every block into its slot
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_group1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ void stage_load_blocks(const PlaneDev &p, const PlaneGeom &g, int32_t *t, int item) {
    const int bx = g.bx0 + item % g.nbx, by = g.by0 + item / g.nbx;
    const int mx = bx / p.bc, my = by / p.br;
    const uint4 e = __ldg(&p.mbs[(size_t)my * p.mbs_stride + mx]);
    const int bands = (e.x >> 28) & 3;
    const int blk = (by - my * p.br) * p.bc + (bx - mx * p.bc);
    const int s = swz(item);
    int32_t *dst = t + item * 16;
    if (bands >= 2) {
        const int32_t *src = p.coeff + (e.x & 0x0fffffffu) + blk * 16;
        if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
#pragma unroll
            for (int r = 0; r < 4; r++) cp_async16(dst + ((r ^ s) << 2), src + r * 4);
        } else {
#pragma unroll
            for (int r = 0; r < 4; r++)
                *reinterpret_cast<int4 *>(dst + ((r ^ s) << 2)) =
                    make_int4(__ldg(src + r * 4), __ldg(src + r * 4 + 1), __ldg(src + r * 4 + 2), __ldg(src + r * 4 + 3));
        }
    } else {
#pragma unroll
        for (int r = 0; r < 4; r++) *reinterpret_cast<int4 *>(dst + r * 4) = make_int4(0, 0, 0, 0);
    }
}

// ---------------------------------------------------------------------------
// stage A: dequantize + first-level inverse transform of one macroblock
// (crates/jxr-native/src/reconstruct/pipeline.rs:605-680)
// ---------------------------------------------------------------------------
__device__ bool stage_first_level(const PlaneDev &p, const PlaneGeom &g, int32_t *dc, int item) {
    const int nmx = g.mx1 - g.mx0 + 1;
    const int mx = g.mx0 + item % nmx, my = g.my0 + item / nmx;
    const uint4 e = __ldg(&p.mbs[(size_t)my * p.mbs_stride + mx]);
    const int bands = (e.x >> 28) & 3;
    const int32_t *c = p.coeff + (e.x & 0x0fffffffu);
    const int count = p.bc * p.br;
    const int stride = bands >= 2 ? 16 : 1;
    int32_t v[16];
    bool bad = false;
    v[0] = dequant(__ldg(c), e.y, bad);
#pragma unroll
    for (int k = 1; k < 16; k++) v[k] = (k < count && bands != 0) ? dequant(__ldg(c + k * stride), e.z, bad) : 0;
    const int lx = (mx - g.mx0) * p.bc, ly = (my - g.my0) * p.br;
    int32_t *out = dc + ly * g.dw + lx;
    if (count == 16) {
        bad |= pct16(v);
        if (p.scale2) {
#pragma unroll
            for (int k = 0; k < 16; k++) v[k] = dequant(v[k], 2, bad);
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int cc = 0; cc < 4; cc++) out[r * g.dw + cc] = v[r * 4 + cc];
    } else if (count == 4) {
        int32_t w[4] = {v[0], v[1], v[2], v[3]};
        bad |= inverse_chroma_420<true>(w);
#pragma unroll
        for (int k = 0; k < 4; k++) w[k] = p.scale2 ? dequant(w[k], 2, bad) : w[k];
        out[0] = w[0]; out[1] = w[1]; out[g.dw] = w[2]; out[g.dw + 1] = w[3];
    } else {
        int32_t w[8] = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
        bad |= inverse_chroma_422<true>(w);
#pragma unroll
        for (int k = 0; k < 8; k++) w[k] = p.scale2 ? dequant(w[k], 2, bad) : w[k];
#pragma unroll
        for (int r = 0; r < 4; r++) { out[r * g.dw] = w[2 * r]; out[r * g.dw + 1] = w[2 * r + 1]; }
    }
    return bad;
}

// ---------------------------------------------------------------------------
// stage B: first-level overlap on the DC tile, full resolution (raster DC tile)
// ---------------------------------------------------------------------------
__device__ bool dc_cell(const PlaneGeom &g, int32_t *dc, int item) {
    const int c0 = cell_of(g.bx0), r0 = cell_of(g.by0);
    const int ncx = (cell_of(g.bx1) - c0) / 4 + 1;
    const int i = item % ncx, j = item / ncx;
    const int cx = c0 + 4 * i, cy = r0 + 4 * j;
    const bool vs = (g.dvmask >> i) & 1, hs = (g.dhmask >> j) & 1;
    const int ox = g.mx0 * 4, oy = g.my0 * 4, st = g.dw;
    bool bad = false;
    if (!vs && !hs) {
        int32_t *base = dc + (cy - oy) * st + (cx - ox);
        int32_t v[16];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) v[r * 4 + c] = base[r * st + c];
        bad |= pot16(v);
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) base[r * st + c] = v[r * 4 + c];
        return bad;
    }
    auto at = [&](int x, int y) -> int32_t & { return dc[(y - oy) * st + (x - ox)]; };
    if (vs && !hs) {
        for (int c = 0; c < 4; c++) {
            const int x = cx + c;
            if (x < 0 || x >= g.Wdc) continue;
            bad |= inverse_pot4(at(x, cy), at(x, cy + 1), at(x, cy + 2), at(x, cy + 3));
        }
    } else if (!vs && hs) {
        for (int r = 0; r < 4; r++) {
            const int y = cy + r;
            if (y < 0 || y >= g.Hdc) continue;
            bad |= inverse_pot4(at(cx, y), at(cx + 1, y), at(cx + 2, y), at(cx + 3, y));
        }
    } else {
        for (int k = 0; k < 4; k++) {
            const int x = cx + (k & 1) * 2, y = cy + (k >> 1) * 2;
            if (x < 0 || x >= g.Wdc || y < 0 || y >= g.Hdc) continue;
            bad |= inverse_pot4(at(x, y), at(x + 1, y), at(x, y + 1), at(x + 1, y + 1));
        }
    }
    return bad;
}

// ---------------------------------------------------------------------------
// stage B for subsampled chroma: odd 2x2 cells, ordered corner residuals
// (crates/jxr-native/src/reconstruct/subsampled_overlap.rs:244-296).
// phase 0: corners lose their neighbour (regions two wide run whole here),
// phase 1: squares and pairs, phase 2: corners regain the neighbour.
// ---------------------------------------------------------------------------
__device__ bool subsampled_cell(const PlaneDev &p, const PlaneGeom &g, int32_t *dc, int item, int phase) {
    const int ncx = (g.ox1 - g.ox0) / 2 + 1;
    const int cx = g.ox0 + 2 * (item % ncx), cy = g.oy0 + 2 * (item / ncx);
    const int ox = g.mx0 * p.bc, oy = g.my0 * p.br;
    const int cov_x0 = max(0, g.ox0), cov_x1 = min(g.Wdc, g.ox1 + 2);
    const int cov_y0 = max(0, g.oy0), cov_y1 = min(g.Hdc, g.oy1 + 2);
    auto at = [&](int x, int y) -> int32_t & { return dc[(y - oy) * g.dw + (x - ox)]; };
    auto inside = [&](int x, int y) { return x >= cov_x0 && x < cov_x1 && y >= cov_y0 && y < cov_y1; };
    const int lx = log2_of(p.bc), ly = log2_of(p.br);
    auto vb = [&](int x) { return boundary_at(x, g.Wdc, lx, p.hard, p.col_start); };
    auto hb = [&](int y) { return boundary_at(y, g.Hdc, ly, p.hard, p.row_start); };
    using A = Ar<true>;
    bool bad = false;
    if (phase == 1) {
        const bool vs = vb(cx + 1), hs = hb(cy + 1);
        if (!vs && !hs) {
            if (inside(cx, cy) && inside(cx + 1, cy + 1))
                bad |= inverse_pot2x2(at(cx, cy), at(cx + 1, cy), at(cx, cy + 1), at(cx + 1, cy + 1));
        } else if (vs && !hs) {
            for (int c = 0; c < 2; c++) {
                const int x = cx + c;
                if (inside(x, cy) && inside(x, cy + 1)) bad |= inverse_pot2(at(x, cy), at(x, cy + 1));
            }
        } else if (!vs && hs) {
            for (int r = 0; r < 2; r++) {
                const int y = cy + r;
                if (inside(cx, y) && inside(cx + 1, y)) bad |= inverse_pot2(at(cx, y), at(cx + 1, y));
            }
        }
        return bad;
    }
    if (!hb(cy + 1)) return false;  // no boundary row in this cell
    for (int k = 0; k < 4; k++) {
        const int x = cx + (k & 1), y = cy + (k >> 1);
        if (!inside(x, y)) continue;
        const bool left_corner = vb(x), right_corner = vb(x + 1);
        if (left_corner == right_corner) continue;  // not a corner (or a one-wide region)
        if (right_corner && vb(x - 1)) continue;    // right corner of a two-wide region: with its partner
        if (left_corner && vb(x + 2)) {             // two-wide region: every step of the row here
            if (phase != 0 || !inside(x + 1, y)) continue;
            int32_t &c0 = at(x, y), &c1 = at(x + 1, y);
            c0 = A::sub(c0, c1, bad);
            c1 = A::sub(c1, c0, bad);
            c0 = A::add(c0, c1, bad);
            c1 = A::add(c1, c0, bad);
            continue;
        }
        const int n = left_corner ? x + 1 : x - 1;
        if (!inside(n, y)) continue;
        at(x, y) = phase == 0 ? A::sub(at(x, y), at(n, y), bad) : A::add(at(x, y), at(n, y), bad);
    }
    return bad;
}

// ---------------------------------------------------------------------------
// stage C1: in-macroblock prediction (crates/jxr-math/src/prediction.rs:110-154),
// one thread per block row (from left) or block column (from top)
// ---------------------------------------------------------------------------
__device__ bool stage_prediction(const PlaneDev &p, const PlaneGeom &g, int32_t *t, int item, bool &invalid) {
    const int mbx0 = g.bx0 / p.bc, mbx1 = g.bx1 / p.bc, mby0 = g.by0 / p.br;
    const int nmx = mbx1 - mbx0 + 1;
    const int lines = 4;
    const int line = item % lines, m = item / lines;
    const int mx = mbx0 + m % nmx, my = mby0 + m / nmx;
    const uint4 e = __ldg(&p.mbs[(size_t)my * p.mbs_stride + mx]);
    const int hp = (e.x >> 30) & 3;
    const int bands = (e.x >> 28) & 3;
    if (hp == 0 || bands < 2) return false;
    if (hp == 3) { invalid = true; return false; }
    using A = Ar<true>;
    bool bad = false;
    if (hp == 1) {  // from left: along block row `line`
        if (line >= p.br) return false;
        const int by = my * p.br + line;
        if (by < g.by0 || by > g.by1) return false;
        for (int c = 1; c < p.bc; c++) {
            const int bx = mx * p.bc + c;
            if (bx > g.bx1) break;
            const int b = (by - g.by0) * g.nbx + (bx - g.bx0);
            // coefficients 4, 8, 12: element (r, 0) for r = 1..3
#pragma unroll
            for (int r = 1; r < 4; r++) t[elem(b, r, 0)] = A::add(t[elem(b, r, 0)], t[elem(b - 1, r, 0)], bad);
        }
    } else {        // from top: along block column `line`
        if (line >= p.bc) return false;
        const int bx = mx * p.bc + line;
        if (bx < g.bx0 || bx > g.bx1) return false;
        for (int r = 1; r < p.br; r++) {
            const int by = my * p.br + r;
            if (by > g.by1) break;
            const int b = (by - g.by0) * g.nbx + (bx - g.bx0);
            // coefficients 1, 2, 3: element (0, c) for c = 1..3
#pragma unroll
            for (int c = 1; c < 4; c++) t[elem(b, 0, c)] = A::add(t[elem(b, 0, c)], t[elem(b - g.nbx, 0, c)], bad);
        }
    }
    return bad;
}

// ---------------------------------------------------------------------------
// stage C2: dequantize, take the block DC, inverse core transform (in place)
// ---------------------------------------------------------------------------
__device__ bool stage_block_transform(const PlaneDev &p, const PlaneGeom &g, int32_t *t, const int32_t *dc, int item) {
    const int bx = g.bx0 + item % g.nbx, by = g.by0 + item / g.nbx;
    const int mx = bx / p.bc, my = by / p.br;
    const uint32_t step = __ldg(&p.mbs[(size_t)my * p.mbs_stride + mx].w);
    int32_t *blk = t + item * 16;
    const int s = swz(item);
    int32_t v[16];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int4 q = *reinterpret_cast<const int4 *>(blk + ((r ^ s) << 2));
        v[r * 4 + 0] = q.x; v[r * 4 + 1] = q.y; v[r * 4 + 2] = q.z; v[r * 4 + 3] = q.w;
    }
    bool bad = false;
    uint32_t m = 0;
#pragma unroll
    for (int k = 1; k < 16; k++) m |= mag(v[k]);
    v[0] = dc[(by - g.my0 * p.br) * g.dw + (bx - g.mx0 * p.bc)];
    // |v| <= m + 1 for every coded coefficient, so (m + 1) * step bounds the
    // dequantized ones; below the transform bound with the DC, the wrapping
    // transform is the checked one
    const uint64_t bound = (uint64_t)(m + 1) * step;
    if (bound < (uint64_t)kTransformBound && mag(v[0]) < (uint32_t)kTransformBound) {
#pragma unroll
        for (int k = 1; k < 16; k++) v[k] = v[k] * (int32_t)step;
        inverse_pct<false>(v);
    } else {
#pragma unroll
        for (int k = 1; k < 16; k++) v[k] = dequant(v[k], step, bad);
        bad |= pct16(v);
    }
#pragma unroll
    for (int r = 0; r < 4; r++)
        *reinterpret_cast<int4 *>(blk + ((r ^ s) << 2)) = make_int4(v[r * 4], v[r * 4 + 1], v[r * 4 + 2], v[r * 4 + 3]);
    return bad;
}

// ---------------------------------------------------------------------------
// stage D: second-level overlap cells on the block-major sample tile
// ---------------------------------------------------------------------------
struct TileView {
    int32_t *t;
    int bx0, by0, nbx;
    __device__ __forceinline__ int32_t &at(int x, int y) const {
        const int b = ((y >> 2) - by0) * nbx + ((x >> 2) - bx0);
        return t[elem(b, y & 3, x & 3)];
    }
};

__device__ bool sample_cell(const PlaneGeom &g, const TileView &v, int item) {
    const int ncx = (g.cx1 - g.cx0) / 4 + 1;
    const int i = item % ncx, j = item / ncx;
    const int cx = g.cx0 + 4 * i, cy = g.cy0 + 4 * j;
    const bool vs = (g.vmask >> i) & 1, hs = (g.hmask >> j) & 1;
    bool bad = false;
    if (!vs && !hs) {
        // the cell takes the lower-right quarter of block (bx, by), and the
        // neighbouring quarters of the three blocks right of and below it
        const int bx = (cx >> 2) - v.bx0, by = (cy >> 2) - v.by0;
        const int b00 = by * v.nbx + bx, b01 = b00 + 1, b10 = b00 + v.nbx, b11 = b10 + 1;
        int32_t w[16];
        const int2 a0 = *reinterpret_cast<const int2 *>(&v.t[elem(b00, 2, 2)]);
        const int2 a1 = *reinterpret_cast<const int2 *>(&v.t[elem(b01, 2, 0)]);
        const int2 a2 = *reinterpret_cast<const int2 *>(&v.t[elem(b00, 3, 2)]);
        const int2 a3 = *reinterpret_cast<const int2 *>(&v.t[elem(b01, 3, 0)]);
        const int2 a4 = *reinterpret_cast<const int2 *>(&v.t[elem(b10, 0, 2)]);
        const int2 a5 = *reinterpret_cast<const int2 *>(&v.t[elem(b11, 0, 0)]);
        const int2 a6 = *reinterpret_cast<const int2 *>(&v.t[elem(b10, 1, 2)]);
        const int2 a7 = *reinterpret_cast<const int2 *>(&v.t[elem(b11, 1, 0)]);
        w[0] = a0.x; w[1] = a0.y; w[2] = a1.x; w[3] = a1.y;
        w[4] = a2.x; w[5] = a2.y; w[6] = a3.x; w[7] = a3.y;
        w[8] = a4.x; w[9] = a4.y; w[10] = a5.x; w[11] = a5.y;
        w[12] = a6.x; w[13] = a6.y; w[14] = a7.x; w[15] = a7.y;
        bad |= pot16(w);
        *reinterpret_cast<int2 *>(&v.t[elem(b00, 2, 2)]) = make_int2(w[0], w[1]);
        *reinterpret_cast<int2 *>(&v.t[elem(b01, 2, 0)]) = make_int2(w[2], w[3]);
        *reinterpret_cast<int2 *>(&v.t[elem(b00, 3, 2)]) = make_int2(w[4], w[5]);
        *reinterpret_cast<int2 *>(&v.t[elem(b01, 3, 0)]) = make_int2(w[6], w[7]);
        *reinterpret_cast<int2 *>(&v.t[elem(b10, 0, 2)]) = make_int2(w[8], w[9]);
        *reinterpret_cast<int2 *>(&v.t[elem(b11, 0, 0)]) = make_int2(w[10], w[11]);
        *reinterpret_cast<int2 *>(&v.t[elem(b10, 1, 2)]) = make_int2(w[12], w[13]);
        *reinterpret_cast<int2 *>(&v.t[elem(b11, 1, 0)]) = make_int2(w[14], w[15]);
        return bad;
    }
    if (vs && !hs) {
        for (int c = 0; c < 4; c++) {
            const int x = cx + c;
            if (x < 0 || x >= g.W) continue;
            bad |= inverse_pot4(v.at(x, cy), v.at(x, cy + 1), v.at(x, cy + 2), v.at(x, cy + 3));
        }
    } else if (!vs && hs) {
        for (int r = 0; r < 4; r++) {
            const int y = cy + r;
            if (y < 0 || y >= g.H) continue;
            bad |= inverse_pot4(v.at(cx, y), v.at(cx + 1, y), v.at(cx + 2, y), v.at(cx + 3, y));
        }
    } else {
        for (int k = 0; k < 4; k++) {
            const int x = cx + (k & 1) * 2, y = cy + (k >> 1) * 2;
            if (x < 0 || x >= g.W || y < 0 || y >= g.H) continue;
            bad |= inverse_pot4(v.at(x, y), v.at(x + 1, y), v.at(x, y + 1), v.at(x + 1, y + 1));
        }
    }
    return bad;
}

// ---------------------------------------------------------------------------
// stage E helpers
// ---------------------------------------------------------------------------
struct PlaneView {
    TileView tv;
    int x0, x1, y0, y1;  // samples the tile holds for the output: the plane
                         // clamped to them reads what clamping to the plane
                         // reads for every output pixel
    __device__ __forceinline__ int32_t at(int x, int y) const { return tv.at(x, y); }
    __device__ __forceinline__ int32_t clamped(int x, int y) const {
        return tv.at(min(max(x, x0), x1 - 1), min(max(y, y0), y1 - 1));
    }
};

// T.832 Table 180 pair (crates/jxr-math/src/sampling.rs:47-58,105-115):
// weights (h2, h3) for the even output, (h0, h1) for the odd one.
__device__ __forceinline__ int32_t weighted(int32_t a, int wa, int32_t b, int wb) {
    return (a >> 3) * wa + (b >> 3) * wb + (((a & 7) * wa + (b & 7) * wb + 4) >> 3);
}
__device__ __forceinline__ int32_t up_even(int32_t prev, int32_t cur, int c) { return weighted(prev, c, cur, 8 - c); }
__device__ __forceinline__ int32_t up_odd(int32_t cur, int32_t next, int c) { return weighted(cur, 4 + c, next, 4 - c); }

// The same for samples below 2^28 in magnitude: the weights sum to 8, so the
// weighted sum stays below 2^31 and one floor division by 8 gives the value
// the split form gives.
__device__ __forceinline__ int32_t up_even_small(int32_t prev, int32_t cur, int c) {
    return (prev * c + cur * (8 - c) + 4) >> 3;
}
__device__ __forceinline__ int32_t up_odd_small(int32_t cur, int32_t next, int c) {
    return (cur * (4 + c) + next * (4 - c) + 4) >> 3;
}

__device__ __forceinline__ int32_t apply_scale(const ChannelScale &s, int32_t sample, bool &bad) {
    using A = Ar<true>;
    int32_t v = A::add(A::add(sample, s.shifted_bias, bad), s.rounding, bad) >> s.shift;
    if (s.post_shift >= 0) {
        const int64_t w = (int64_t)v << s.post_shift;
        v = w > INT32_MAX ? INT32_MAX : (w < INT32_MIN ? INT32_MIN : (int32_t)w);
    }
    return v;
}

// float32_bits, crates/jxr-native/src/output_format/scaling.rs:243-297
__device__ uint32_t f32_bits(int32_t v, int length, int bias, bool &bad) {
    const uint32_t sign = v < 0 ? 0x80000000u : 0u;
    const uint64_t magnitude = v < 0 ? (uint64_t)(-(int64_t)v) : (uint64_t)v;
    const uint64_t implicit = 1ull << length;
    int64_t exponent = (int64_t)(magnitude >> length);
    uint64_t mantissa = (magnitude & (implicit - 1)) | implicit;
    if (exponent == 0) { mantissa ^= implicit; exponent = 1; }
    exponent = exponent - bias + 127;
    while (mantissa < implicit && exponent > 1 && mantissa > 0) { exponent--; mantissa <<= 1; }
    if (mantissa < implicit) exponent = 0;
    else mantissa ^= implicit;
    mantissa <<= 23 - length;
    if (exponent < 0 || exponent > 255) return sign | 0x7f7fffffu;
    if (mantissa > 0x7fffff) { bad = true; return 0; }
    return sign | ((uint32_t)exponent << 23) | (uint32_t)mantissa;
}

// Exact binary16 -> binary32 widening of a half bit pattern: the hardware
// conversion for finite halves (every half is exactly a float, so any exact
// conversion gives these bits); infinities and NaNs keep their payload bits,
// spelled out.  A branchy bit-level form of the finite case cost the F16
// output path a fifth of its time.
__device__ __forceinline__ uint32_t widen_f16(uint32_t h) {
    if (((h >> 10) & 0x1f) == 0x1f) return ((h & 0x8000u) << 16) | 0x7f800000u | ((h & 0x3ffu) << 13);
    return __float_as_uint(__half2float(__ushort_as_half((unsigned short)h)));
}

// A scaled sample stored as F16 bits -- sign | min(|v|, 32767), the
// reference's float16_bits (crates/jxr-native/src/output_format/scaling.rs:235-241)
// -- then widened to binary32.
__device__ __forceinline__ uint32_t f16_widened(int32_t v) {
    const uint32_t mm = min((uint32_t)(v < 0 ? -(int64_t)v : v), 32767u);
    return widen_f16((v < 0 ? 0x8000u : 0u) | mm);
}

__device__ __forceinline__ uint32_t premultiply_u(uint32_t v, uint32_t a, uint32_t maximum) {
    v = min(v, maximum); a = min(a, maximum);
    return (uint32_t)(((uint64_t)v * a + maximum / 2) / maximum);
}

__device__ __forceinline__ int32_t premultiply_s(int32_t v, int32_t a, int32_t maximum, bool &bad) {
    a = min(max(a, 0), maximum);
    const uint64_t m = v < 0 ? (uint64_t)(-(int64_t)v) : (uint64_t)v;
    const int64_t r = (int64_t)((m * (uint64_t)a + (uint64_t)(maximum / 2)) / (uint64_t)maximum);
    const int64_t s = v < 0 ? -r : r;
    bad |= s != (int64_t)(int32_t)s;
    return (int32_t)s;
}

__device__ __forceinline__ void store_elem(uint8_t *dst, uint32_t w, int bytes) {
    if (bytes == 1) *dst = (uint8_t)w;
    else if (bytes == 2) *reinterpret_cast<uint16_t *>(dst) = (uint16_t)w;
    else *reinterpret_cast<uint32_t *>(dst) = w;
}

// Converted components (crates/jxr-native/src/output_format/color.rs:9-52)
__device__ __forceinline__ void convert(const OutputDev &o, const int32_t in[4], int32_t out[4], bool &bad) {
    using A = Ar<true>;
    switch (o.conv) {
    case kConvLumaToRgb: out[0] = out[1] = out[2] = in[0]; out[3] = 0; break;
    case kConvYuvToRgb: {
        const int32_t t = A::sub(0, in[1], bad);
        const int32_t g = A::sub(in[0], t >> 1, bad);
        const int32_t r = A::sub(A::add(t, g, bad), (in[2] >> 1) + (in[2] & 1), bad);
        const int32_t b = A::add(in[2], r, bad);
        if (o.packed_swap) { out[0] = b; out[2] = r; } else { out[0] = r; out[2] = b; }
        out[1] = g; out[3] = 0;
        break;
    }
    case kConvYuvkToCmyk: {
        const int32_t k = A::add(in[3], in[0] >> 1, bad);
        const int32_t m = A::sub(A::sub(k, in[0], bad), in[1] >> 1, bad);
        const int32_t c = A::add(A::add(in[1], m, bad), in[2] >> 1, bad);
        out[0] = c; out[1] = m; out[2] = A::sub(c, in[2], bad); out[3] = k;
        break;
    }
    case kConvYuvkToCmykDirect: out[0] = in[1]; out[1] = in[2]; out[2] = in[3]; out[3] = in[0]; break;
    default: out[0] = in[0]; out[1] = in[1]; out[2] = in[2]; out[3] = in[3]; break;
    }
}

// Inverse RCT without checks for components whose magnitudes are below 2^28
// (every intermediate then stays below 2^30).
__device__ __forceinline__ void yuv_to_rgb_fast(int32_t y, int32_t u, int32_t v, int32_t &r, int32_t &g, int32_t &b) {
    const int32_t t = -u;
    g = y - (t >> 1);
    r = t + g - ((v >> 1) + (v & 1));
    b = v + r;
}

// v clamped to 0 .. 255 (one min-then-relu instruction)
__device__ __forceinline__ uint32_t clamp_u8(int32_t v) { return (uint32_t)__vimin_s32_relu(v, 255); }

// Three bytes r, g, b (each below 256) packed into bytes 0..2 of a word in the
// byte order `order` selects (0x7410: r g b; 0x7014: b g r); byte 3 is zero.
__device__ __forceinline__ uint32_t pack_rgb8(uint32_t r, uint32_t g, uint32_t b, uint32_t order) {
    return __byte_perm(__byte_perm(r, g, 0x7740u), b, order);
}

// The general output of one pixel: every colour conversion, store kind,
// channel order, alpha and premultiplication of the output stage
// (crates/jxr-native/src/output_format/packing.rs, packed_color.rs,
// premultiply.rs, scaling.rs).
__device__ void format_pixel(const OutputDev &o, const int32_t comp[4], int32_t alpha_sample, uint8_t *dst,
                             uint64_t channel_stride, bool &bad) {
    int32_t conv[4];
    convert(o, comp, conv, bad);
    if (o.store >= kStoreRgb555) {
        int32_t v[3];
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = apply_scale(o.ch[c], conv[c], bad);
        uint32_t w;
        if (o.store == kStoreRgbe) {
            // crates/jxr-math/src/rgbe.rs:7-101
            int32_t mant[3], ex[3], e = 0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int32_t x = v[c];
                if (x <= 0) { mant[c] = 0; ex[c] = 0; }
                else if ((x >> 7) > 1) { mant[c] = (x & 0x7f) + 128; ex[c] = x >> 7; }
                else { mant[c] = x; ex[c] = 1; }
                e = max(e, ex[c]);
            }
            w = (uint32_t)min(e, 255) << 24;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                int32_t m = mant[c];
                if (e > ex[c]) {
                    const int d = e - ex[c];
                    m = d >= 31 ? 0 : (int32_t)((2 * (int64_t)m + 1) >> (d + 1));
                }
                w |= (uint32_t)min(max(m, 0), 255) << (8 * c);
            }
        } else {
            uint32_t f[3];
#pragma unroll
            for (int c = 0; c < 3; c++) f[c] = v[c] < 0 ? 0u : min((uint32_t)v[c], (uint32_t)o.ch[c].hi);
            if (o.store == kStoreRgb555) w = f[2] | (f[1] << 5) | (f[0] << 10);
            else if (o.store == kStoreRgb565) w = f[2] | (f[1] << 5) | (f[0] << 11);
            else w = f[2] | (f[1] << 10) | (f[0] << 20);
        }
        store_elem(dst, w, o.elem_bytes);
        return;
    }
    uint32_t words[JXRB_MAX_CHANNELS];
#pragma unroll
    for (int c = 0; c < JXRB_MAX_CHANNELS; c++) {
        if (c >= o.channels) break;
        const ChannelScale &s = o.ch[c];
        const int src = s.source;
        const int32_t sample = s.alpha ? alpha_sample : (src == 0 ? conv[0] : src == 1 ? conv[1] : src == 2 ? conv[2] : conv[3]);
        uint32_t w = 0;
        if (s.padding) {
            w = 0;
        } else if (o.store == kStoreF16) {
            const int32_t x = apply_scale(s, sample, bad);
            const uint32_t m = min((uint32_t)(x < 0 ? -(int64_t)x : x), 32767u);
            w = (x < 0 ? 0x8000u : 0u) | m;
        } else if (o.store == kStoreF32) {
            w = f32_bits(apply_scale(s, sample, bad), s.f_mantissa, s.f_bias, bad);
        } else {
            const int32_t x = apply_scale(s, sample, bad);
            w = (uint32_t)min(max(x, s.lo), s.hi);
        }
        words[c] = w;
    }
    if (o.premultiply) {
        // crates/jxr-native/src/output_format/premultiply.rs:10-105, on the stored values
        const int n = o.channels;
        const uint32_t a = words[n - 1];
#pragma unroll
        for (int c = 0; c < JXRB_MAX_CHANNELS - 1; c++) {
            if (c >= n - 1) break;
            switch (o.store) {
            case kStoreU8: words[c] = premultiply_u(words[c], a, 255); break;
            case kStoreU16: words[c] = premultiply_u(words[c], a, 65535); break;
            case kStoreI16: words[c] = (uint16_t)(int16_t)premultiply_s((int16_t)words[c], (int16_t)a, 32767, bad); break;
            case kStoreI32: words[c] = (uint32_t)premultiply_s((int32_t)words[c], (int32_t)a, INT32_MAX, bad); break;
            case kStoreF16: {
                const uint32_t av = (a & 0x8000u) ? 0u : (a & 0x7fffu);
                words[c] = (words[c] & 0x8000u) | premultiply_u(words[c] & 0x7fffu, av, 0x7fff);
                break;
            }
            case kStoreF32: {
                float fa = __uint_as_float(a);
                fa = fa < 0.f ? 0.f : (fa > 1.f ? 1.f : fa);
                words[c] = __float_as_uint(__fmul_rn(__uint_as_float(words[c]), fa));
                break;
            }
            default: break;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < JXRB_MAX_CHANNELS; c++) {
        if (c >= o.channels) break;
        uint32_t w = words[c];
        if (o.widen_f16) w = widen_f16(w);
        store_elem(dst + (uint64_t)c * channel_stride, w, o.elem_bytes);
    }
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
struct WorkItem {
    uint32_t image;
    uint16_t tx, ty;
};

struct TileShared {
    PlaneGeom geo[JXRB_MAX_PLANES];
    int bad;
    uint32_t next;   // interior kernels: the work item claimed to follow the current one
};

// Colour components of full-resolution pixel (x, y): luma and full-resolution
// planes read directly, subsampled chroma interpolated.
template <class View>
__device__ __forceinline__ void components(const ImageDev &im, const View *views, int x, int y, int32_t comp[4]) {
    const int ncol = min(im.nplanes, 4);
#pragma unroll
    for (int c = 0; c < 4; c++) {
        comp[c] = 0;
        if (c >= ncol) break;
        const View &v = views[c];
        if (im.chroma != 0 && (c == 1 || c == 2)) {
            const int cx = x >> 1;
            if (im.chroma == 2) {
                comp[c] = (x & 1) ? up_odd(v.clamped(cx, y), v.clamped(cx + 1, y), im.centering_x)
                                  : up_even(v.clamped(cx - 1, y), v.clamped(cx, y), im.centering_x);
            } else {
                const int cy = y >> 1;
                int32_t col[3];
#pragma unroll
                for (int d = -1; d <= 1; d++)
                    col[d + 1] = (y & 1) ? up_odd(v.clamped(cx + d, cy), v.clamped(cx + d, cy + 1), im.centering_y)
                                         : up_even(v.clamped(cx + d, cy - 1), v.clamped(cx + d, cy), im.centering_y);
                comp[c] = (x & 1) ? up_odd(col[1], col[2], im.centering_x) : up_even(col[0], col[1], im.centering_x);
            }
        } else {
            comp[c] = v.at(x, y);
        }
    }
}

template <class View>
__device__ void output_generic(const ImageDev &im, const View *views, int X0, int X1, int Y0, int Y1, bool &bad) {
    const OutputDev &o = im.out;
    const int ax0 = max(X0, (int)o.crop_x), ax1 = min(X1, (int)(o.crop_x + o.crop_w));
    const int ay0 = max(Y0, (int)o.crop_y), ay1 = min(Y1, (int)(o.crop_y + o.crop_h));
    if (ax0 >= ax1 || ay0 >= ay1) return;
    const int nx = ax1 - ax0, ny = ay1 - ay0;
    if (o.planar_yuv) {
        // native planar YUV: each plane at its own resolution, the chroma
        // crop halved (crates/jxr-native/src/output_format/planar.rs:76-123)
        const int cw = o.crop_w / 2, chh = o.planar_yuv == 1 ? o.crop_h / 2 : o.crop_h;
        const int ccx = o.crop_x / 2, ccy = o.planar_yuv == 1 ? o.crop_y / 2 : o.crop_y;
        const uint64_t luma_bytes = (uint64_t)o.crop_w * o.crop_h * o.elem_bytes;
        const uint64_t chroma_bytes = (uint64_t)cw * chh * o.elem_bytes;
        for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) {
            const int x = ax0 + i % nx, y = ay0 + i / nx;
            const uint64_t at = ((uint64_t)(y - o.crop_y) * o.crop_w + (x - o.crop_x)) * o.elem_bytes;
            int32_t v = apply_scale(o.ch[0], views[0].at(x, y), bad);
            store_elem(o.base + at, (uint32_t)min(max(v, o.ch[0].lo), o.ch[0].hi), o.elem_bytes);
            if (im.alpha >= 0) {
                v = apply_scale(o.ch[3], views[im.alpha].at(x, y), bad);
                store_elem(o.base + luma_bytes + 2 * chroma_bytes + at, (uint32_t)min(max(v, o.ch[3].lo), o.ch[3].hi),
                           o.elem_bytes);
            }
        }
        // chroma samples whose luma position 2x (and 2y for 4:2:0) this tile owns
        const int sx0 = max((X0 + 1) >> 1, ccx), sx1 = min((X1 + 1) >> 1, ccx + cw);
        const int sy0 = o.planar_yuv == 1 ? max((Y0 + 1) >> 1, ccy) : max(Y0, ccy);
        const int sy1 = o.planar_yuv == 1 ? min((Y1 + 1) >> 1, ccy + chh) : min(Y1, ccy + chh);
        if (sx0 < sx1 && sy0 < sy1) {
            const int ncx = sx1 - sx0, ncy = sy1 - sy0;
            for (int i = threadIdx.x; i < ncx * ncy; i += blockDim.x) {
                const int cx = sx0 + i % ncx, cy = sy0 + i / ncx;
                const uint64_t at = ((uint64_t)(cy - ccy) * cw + (cx - ccx)) * o.elem_bytes;
                for (int c = 1; c < 3; c++) {
                    const int32_t w = apply_scale(o.ch[c], views[c].at(cx, cy), bad);
                    store_elem(o.base + luma_bytes + (uint64_t)(c - 1) * chroma_bytes + at,
                               (uint32_t)min(max(w, o.ch[c].lo), o.ch[c].hi), o.elem_bytes);
                }
            }
        }
        return;
    }
    if (o.store == kStoreBits) {
        // one byte of eight pixels per thread; bytes shared with a
        // neighbouring tile set their bits atomically (the surface is zeroed)
        const int bx0 = (ax0 - (int)o.crop_x) >> 3, bx1 = (ax1 - (int)o.crop_x + 7) >> 3;
        const int nbx = bx1 - bx0;
        for (int i = threadIdx.x; i < nbx * ny; i += blockDim.x) {
            const int by = ay0 + i / nbx, bx = bx0 + i % nbx;
            uint32_t byte = 0;
            bool whole = true;
            for (int k = 0; k < 8; k++) {
                const int x = (int)o.crop_x + bx * 8 + k;
                if (x >= (int)(o.crop_x + o.crop_w)) break;
                if (x < X0 || x >= X1) { whole = false; continue; }
                const int32_t v = apply_scale(o.ch[0], views[0].at(x, by), bad);
                int32_t bit = min(max(v, 0), 1);
                if (o.bit_black) bit = 1 - bit;
                byte |= (uint32_t)bit << (7 - k);
            }
            uint8_t *dst = o.base + (uint64_t)(by - o.crop_y) * o.row_stride + bx;
            if (whole) {
                *dst = (uint8_t)byte;
            } else if (byte) {
                uint32_t *word = reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(dst) & ~(uintptr_t)3);
                const int sh = (int)(reinterpret_cast<uintptr_t>(dst) & 3) * 8;
                atomicOr(word, byte << sh);
            }
        }
        return;
    }
    const uint64_t pixel_bytes = o.nchw ? (uint64_t)o.elem_bytes : (uint64_t)o.elem_bytes * o.channels;
    const uint64_t chs = o.nchw ? o.plane_stride : (uint64_t)o.elem_bytes;
    for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) {
        const int x = ax0 + i % nx, y = ay0 + i / nx;
        int32_t comp[4];
        components(im, views, x, y, comp);
        const int32_t a = im.alpha >= 0 ? views[im.alpha].at(x, y) : 0;
        uint8_t *dst = o.base + (uint64_t)(y - o.crop_y) * o.row_stride + (uint64_t)(x - o.crop_x) * pixel_bytes;
        format_pixel(o, comp, a, dst, chs, bad);
    }
}

// Output work is spread over row chunks: four horizontally adjacent pixels
// of one block row (x = 4k .. 4k+3).  A chunk wholly inside the tile's output
// region reads each full-resolution plane with one 128-bit shared load and
// writes with wide stores; a partial chunk (at the tile's two-sample offset
// and crop edges) goes pixel by pixel.
struct ChunkRange {
    int ax0, ax1, ay0, ay1;  // output pixels of the tile (inclusive-exclusive)
    int kb0, nkb, ny;        // block columns and rows of chunks
};

__device__ __forceinline__ bool chunk_range(const OutputDev &o, int X0, int X1, int Y0, int Y1, ChunkRange &r) {
    r.ax0 = max(X0, (int)o.crop_x); r.ax1 = min(X1, (int)(o.crop_x + o.crop_w));
    r.ay0 = max(Y0, (int)o.crop_y); r.ay1 = min(Y1, (int)(o.crop_y + o.crop_h));
    if (r.ax0 >= r.ax1 || r.ay0 >= r.ay1) return false;
    r.kb0 = r.ax0 >> 2;
    r.nkb = ((r.ax1 - 1) >> 2) - r.kb0 + 1;
    r.ny = r.ay1 - r.ay0;
    return true;
}

// one 4-sample row chunk of a full-resolution plane
__device__ __forceinline__ int4 row_chunk(const PlaneView &v, int kb, int y) {
    const TileView &t = v.tv;
    const int b = ((y >> 2) - t.by0) * t.nbx + (kb - t.bx0);
    return *reinterpret_cast<const int4 *>(&t.t[elem(b, y & 3, 0)]);
}

__device__ __forceinline__ void chunk_components(const ImageDev &im, const PlaneView *views, int kb, int y,
                                                 int32_t comp[3][4]) {
    const int4 yv = row_chunk(views[0], kb, y);
    comp[0][0] = yv.x; comp[0][1] = yv.y; comp[0][2] = yv.z; comp[0][3] = yv.w;
    if (im.chroma == 0) {
        const int4 u = row_chunk(views[1], kb, y), w = row_chunk(views[2], kb, y);
        comp[1][0] = u.x; comp[1][1] = u.y; comp[1][2] = u.z; comp[1][3] = u.w;
        comp[2][0] = w.x; comp[2][1] = w.y; comp[2][2] = w.z; comp[2][3] = w.w;
        return;
    }
    // subsampled chroma: the chunk's four pixels take chroma columns
    // 2k-1 .. 2k+2 (clamped), interpolated vertically first for 4:2:0
    const int cx0 = 2 * kb;
#pragma unroll
    for (int c = 1; c <= 2; c++) {
        const PlaneView &v = views[c];
        int32_t col[4];
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const int cx = cx0 - 1 + d;
            if (im.chroma == 2) {
                col[d] = v.clamped(cx, y);
            } else {
                const int cy = y >> 1;
                col[d] = (y & 1) ? up_odd(v.clamped(cx, cy), v.clamped(cx, cy + 1), im.centering_y)
                                 : up_even(v.clamped(cx, cy - 1), v.clamped(cx, cy), im.centering_y);
            }
        }
        comp[c][0] = up_even(col[0], col[1], im.centering_x);
        comp[c][1] = up_odd(col[1], col[2], im.centering_x);
        comp[c][2] = up_even(col[1], col[2], im.centering_x);
        comp[c][3] = up_odd(col[2], col[3], im.centering_x);
    }
}

// 8-bit RGB / BGR (+ alpha) from YUV: the common photographic output.
__device__ void output_rgb8(const ImageDev &im, const PlaneView *views, int X0, int X1, int Y0, int Y1, bool &bad) {
    const OutputDev &o = im.out;
    ChunkRange cr;
    if (!chunk_range(o, X0, X1, Y0, Y1, cr)) return;
    const ChannelScale &sc = o.ch[0];
    const int32_t add = sc.shifted_bias + sc.rounding;
    const int shift = sc.shift;
    const bool alpha = im.alpha >= 0;
    const int32_t aadd = alpha ? o.ch[3].shifted_bias + o.ch[3].rounding : 0;
    const int ashift = alpha ? o.ch[3].shift : 0;
    const bool reverse = o.ch[0].source == 2;
    const int pb = o.channels;  // 3 or 4 bytes a pixel
    for (int i = threadIdx.x; i < cr.nkb * cr.ny; i += blockDim.x) {
        const int kb = cr.kb0 + i % cr.nkb, y = cr.ay0 + i / cr.nkb;
        const int x0 = max(4 * kb, cr.ax0), x1 = min(4 * kb + 4, cr.ax1);
        int32_t comp[3][4];
        chunk_components(im, views, kb, y, comp);
        int4 av = make_int4(0, 0, 0, 0);
        if (alpha) av = row_chunk(views[im.alpha], kb, y);
        const int32_t a[4] = {av.x, av.y, av.z, av.w};
        uint8_t *row = o.base + (uint64_t)(y - o.crop_y) * o.row_stride;
        uint32_t m = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) m |= mag(comp[0][k]) | mag(comp[1][k]) | mag(comp[2][k]) | mag(a[k]);
        if (m >= (1u << 28) || o.premultiply) {
            for (int x = x0; x < x1; x++) {
                const int k = x - 4 * kb;
                const int32_t cc[4] = {comp[0][k], comp[1][k], comp[2][k], 0};
                format_pixel(o, cc, a[k], row + (uint64_t)(x - o.crop_x) * pb, 1, bad);
            }
            continue;
        }
        uint32_t px[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            int32_t r, g, b;
            yuv_to_rgb_fast(comp[0][k], comp[1][k], comp[2][k], r, g, b);
            const uint32_t R = (uint32_t)min(max((r + add) >> shift, 0), 255);
            const uint32_t G = (uint32_t)min(max((g + add) >> shift, 0), 255);
            const uint32_t B = (uint32_t)min(max((b + add) >> shift, 0), 255);
            const uint32_t A8 = alpha ? (uint32_t)min(max((a[k] + aadd) >> ashift, 0), 255) : 0u;
            px[k] = (reverse ? B : R) | (G << 8) | ((reverse ? R : B) << 16) | (A8 << 24);
        }
        uint8_t *dst = row + (uint64_t)(x0 - o.crop_x) * pb;
        const bool whole = x0 == 4 * kb && x1 == 4 * kb + 4;
        if (whole && pb == 4 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
            *reinterpret_cast<uint4 *>(dst) = make_uint4(px[0], px[1], px[2], px[3]);
        } else if (whole && pb == 3 && (reinterpret_cast<uintptr_t>(dst) & 3) == 0) {
            // 12 bytes: R0 G0 B0 R1 | G1 B1 R2 G2 | B2 R3 G3 B3
            uint32_t *d = reinterpret_cast<uint32_t *>(dst);
            d[0] = (px[0] & 0xffffffu) | (px[1] << 24);
            d[1] = ((px[1] >> 8) & 0xffffu) | (px[2] << 16);
            d[2] = ((px[2] >> 16) & 0xffu) | ((px[3] & 0xffffffu) << 8);
        } else {
            for (int x = x0; x < x1; x++) {
                const uint32_t w = px[x - 4 * kb];
                uint8_t *d = row + (uint64_t)(x - o.crop_x) * pb;
                d[0] = (uint8_t)w; d[1] = (uint8_t)(w >> 8); d[2] = (uint8_t)(w >> 16);
                if (pb == 4) d[3] = (uint8_t)(w >> 24);
            }
        }
    }
}

// One channel straight from one plane (luma to U8 / U16 / I16 / I32).
__device__ void output_direct(const ImageDev &im, const PlaneView *views, int X0, int X1, int Y0, int Y1, bool &bad) {
    const OutputDev &o = im.out;
    ChunkRange cr;
    if (!chunk_range(o, X0, X1, Y0, Y1, cr)) return;
    const ChannelScale &s = o.ch[0];
    const int eb = o.elem_bytes;
    for (int i = threadIdx.x; i < cr.nkb * cr.ny; i += blockDim.x) {
        const int kb = cr.kb0 + i % cr.nkb, y = cr.ay0 + i / cr.nkb;
        const int x0 = max(4 * kb, cr.ax0), x1 = min(4 * kb + 4, cr.ax1);
        const int4 v4 = row_chunk(views[0], kb, y);
        const int32_t v[4] = {v4.x, v4.y, v4.z, v4.w};
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; k++) w[k] = (uint32_t)min(max(apply_scale(s, v[k], bad), s.lo), s.hi);
        uint8_t *row = o.base + (uint64_t)(y - o.crop_y) * o.row_stride;
        uint8_t *dst = row + (uint64_t)(x0 - o.crop_x) * eb;
        const bool whole = x0 == 4 * kb && x1 == 4 * kb + 4;
        if (whole && eb == 2 && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
            *reinterpret_cast<uint2 *>(dst) = make_uint2((w[0] & 0xffffu) | (w[1] << 16), (w[2] & 0xffffu) | (w[3] << 16));
        } else if (whole && eb == 1 && (reinterpret_cast<uintptr_t>(dst) & 3) == 0) {
            *reinterpret_cast<uint32_t *>(dst) = (w[0] & 0xffu) | ((w[1] & 0xffu) << 8) | ((w[2] & 0xffu) << 16) | (w[3] << 24);
        } else if (whole && eb == 4 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
            *reinterpret_cast<uint4 *>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
        } else {
            for (int x = x0; x < x1; x++) store_elem(row + (uint64_t)(x - o.crop_x) * eb, w[x - 4 * kb], eb);
        }
    }
}

// F16 output bits widened to binary32 (+ alpha), interleaved or NCHW.
__device__ void output_f16wide(const ImageDev &im, const PlaneView *views, int X0, int X1, int Y0, int Y1, bool &bad) {
    const OutputDev &o = im.out;
    ChunkRange cr;
    if (!chunk_range(o, X0, X1, Y0, Y1, cr)) return;
    const uint64_t pixel_bytes = o.nchw ? 4ull : 4ull * o.channels;
    const uint64_t chs = o.nchw ? o.plane_stride : 4ull;
    const bool alpha = im.alpha >= 0;
    for (int i = threadIdx.x; i < cr.nkb * cr.ny; i += blockDim.x) {
        const int kb = cr.kb0 + i % cr.nkb, y = cr.ay0 + i / cr.nkb;
        const int x0 = max(4 * kb, cr.ax0), x1 = min(4 * kb + 4, cr.ax1);
        int32_t comp[3][4] = {};
        if (im.nplanes >= 3) {
            chunk_components(im, views, kb, y, comp);
        } else {
            const int4 yv = row_chunk(views[0], kb, y);
            comp[0][0] = yv.x; comp[0][1] = yv.y; comp[0][2] = yv.z; comp[0][3] = yv.w;
        }
        int4 av = make_int4(0, 0, 0, 0);
        if (alpha) av = row_chunk(views[im.alpha], kb, y);
        const int32_t a[4] = {av.x, av.y, av.z, av.w};
        uint32_t words[4][4];  // [channel][pixel]
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int32_t in[4] = {comp[0][k], comp[1][k], comp[2][k], 0};
            int32_t conv[4];
            convert(o, in, conv, bad);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                if (c >= o.channels) break;
                const ChannelScale &s = o.ch[c];
                const int src = s.source;
                const int32_t sample = s.alpha ? a[k] : (src == 0 ? conv[0] : src == 1 ? conv[1] : conv[2]);
                const int32_t v = apply_scale(s, sample, bad);
                const uint32_t m = min((uint32_t)(v < 0 ? -(int64_t)v : v), 32767u);
                words[c][k] = widen_f16(s.padding ? 0u : ((v < 0 ? 0x8000u : 0u) | m));
            }
        }
        uint8_t *row = o.base + (uint64_t)(y - o.crop_y) * o.row_stride;
        const bool whole = x0 == 4 * kb && x1 == 4 * kb + 4;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (c >= o.channels) break;
            uint8_t *dst = row + (uint64_t)(x0 - o.crop_x) * pixel_bytes + c * chs;
            if (whole && o.nchw && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
                *reinterpret_cast<uint4 *>(dst) = make_uint4(words[c][0], words[c][1], words[c][2], words[c][3]);
            } else {
                for (int x = x0; x < x1; x++)
                    *reinterpret_cast<uint32_t *>(row + (uint64_t)(x - o.crop_x) * pixel_bytes + c * chs) = words[c][x - 4 * kb];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Interior tiles of images whose planes are all at full resolution (luma,
// YUV 4:4:4, YUVK, with or without alpha).  The host marks a tile interior
// when its macroblocks [mx0-1, mx0+4] x [my0-1, my0+4] exist and no hard tile
// begins inside them: every overlap cell of the tile is then a plain 4x4
// window and the geometry is fixed -- 17 x 17 blocks, 16 x 16 sample cells,
// a 24 x 24 block-DC tile -- so each of the 256 threads owns one sample cell
// and, holding its 16 final samples of every plane in registers, converts
// and stores those pixels itself.
// ---------------------------------------------------------------------------
constexpr int kIB = 17;             // blocks across / down
constexpr int kIDC = 24;            // DC tile side (macroblocks mx0-1 .. mx0+4)
constexpr int kIBlocks = kIB * kIB;
constexpr int kLpInts = 36 * 16;    // DC / low-pass coefficients of 6 x 6 macroblocks
// The three-plane interior kernel keeps each macroblock's 16 low-pass values
// 80 bytes apart: eight consecutive macroblocks' 16-byte reads then fall in
// eight distinct bank groups (at 64 bytes, in two).  The others keep 64: the
// four-plane kernel measured slower with the padding (C3 1.138 -> 1.18 ms a
// step; its first level reads its own macroblocks' values from the blocks).
template <int NP> __host__ __device__ constexpr int lp_stride() { return NP == 3 ? 20 : 16; }
template <int NP> __host__ __device__ constexpr int lp_ints() { return 36 * lp_stride<NP>(); }
constexpr int kMbcInts = 36 * 4;    // their 16-byte entries

__device__ __forceinline__ void store12(uint8_t *d, const uint32_t px[4]) {
    // R0 G0 B0 R1 | G1 B1 R2 G2 | B2 R3 G3 B3
    const uint32_t w0 = (px[0] & 0xffffffu) | (px[1] << 24);
    const uint32_t w1 = ((px[1] >> 8) & 0xffffu) | (px[2] << 16);
    const uint32_t w2 = ((px[2] >> 16) & 0xffu) | ((px[3] & 0xffffffu) << 8);
    const uintptr_t a = reinterpret_cast<uintptr_t>(d);
    if ((a & 3) == 0) {
        uint32_t *q = reinterpret_cast<uint32_t *>(d);
        q[0] = w0; q[1] = w1; q[2] = w2;
    } else if ((a & 1) == 0) {
        *reinterpret_cast<uint16_t *>(d) = (uint16_t)w0;
        *reinterpret_cast<uint32_t *>(d + 2) = (w0 >> 16) | (w1 << 16);
        *reinterpret_cast<uint32_t *>(d + 6) = (w1 >> 16) | (w2 << 16);
        *reinterpret_cast<uint16_t *>(d + 10) = (uint16_t)(w2 >> 16);
    } else {
        const uint32_t w[3] = {w0, w1, w2};
#pragma unroll
        for (int k = 0; k < 12; k++) d[k] = (uint8_t)(w[k >> 2] >> (8 * (k & 3)));
    }
}

__device__ __forceinline__ void store16(uint8_t *d, uint32_t a, uint32_t b, uint32_t c, uint32_t e) {
    const uintptr_t p = reinterpret_cast<uintptr_t>(d);
    if ((p & 15) == 0) {
        *reinterpret_cast<uint4 *>(d) = make_uint4(a, b, c, e);
    } else if ((p & 7) == 0) {
        *reinterpret_cast<uint2 *>(d) = make_uint2(a, b);
        *reinterpret_cast<uint2 *>(d + 8) = make_uint2(c, e);
    } else if ((p & 3) == 0) {
        uint32_t *q = reinterpret_cast<uint32_t *>(d);
        q[0] = a; q[1] = b; q[2] = c; q[3] = e;
    } else {
        const uint32_t w[4] = {a, b, c, e};
#pragma unroll
        for (int k = 0; k < 16; k++) d[k] = (uint8_t)(w[k >> 2] >> (8 * (k & 3)));
    }
}

__device__ __forceinline__ void store8(uint8_t *d, uint32_t a, uint32_t b) {
    const uintptr_t p = reinterpret_cast<uintptr_t>(d);
    if ((p & 7) == 0) {
        *reinterpret_cast<uint2 *>(d) = make_uint2(a, b);
    } else if ((p & 3) == 0) {
        reinterpret_cast<uint32_t *>(d)[0] = a;
        reinterpret_cast<uint32_t *>(d)[1] = b;
    } else {
        const uint32_t w[2] = {a, b};
#pragma unroll
        for (int k = 0; k < 8; k++) d[k] = (uint8_t)(w[k >> 2] >> (8 * (k & 3)));
    }
}

// The 16 samples of sample cell b00 (lower-right quarter of block b00 and the
// neighbouring quarters of the blocks right of and below it), second-level
// overlap applied when the plane has it.  `small`: every block transform of
// the tile had inputs below 2^16 in magnitude, so the cell's values are below
// 35.3 * 2^16 and the wrapping operator needs no magnitude test (interval
// bounds of the inverse transform and overlap steps: outputs below 2^27.8,
// intermediates below 2^28.2).  Returns the overflow flag.
__device__ __forceinline__ bool cell_samples(const int32_t *t, int b00, int overlap, int32_t (&w)[16],
                                             bool small = false) {
    const int b01 = b00 + 1, b10 = b00 + kIB, b11 = b10 + 1;
    const int2 a0 = *reinterpret_cast<const int2 *>(&t[elem(b00, 2, 2)]);
    const int2 a1 = *reinterpret_cast<const int2 *>(&t[elem(b01, 2, 0)]);
    const int2 a2 = *reinterpret_cast<const int2 *>(&t[elem(b00, 3, 2)]);
    const int2 a3 = *reinterpret_cast<const int2 *>(&t[elem(b01, 3, 0)]);
    const int2 a4 = *reinterpret_cast<const int2 *>(&t[elem(b10, 0, 2)]);
    const int2 a5 = *reinterpret_cast<const int2 *>(&t[elem(b11, 0, 0)]);
    const int2 a6 = *reinterpret_cast<const int2 *>(&t[elem(b10, 1, 2)]);
    const int2 a7 = *reinterpret_cast<const int2 *>(&t[elem(b11, 1, 0)]);
    w[0] = a0.x; w[1] = a0.y; w[2] = a1.x; w[3] = a1.y;
    w[4] = a2.x; w[5] = a2.y; w[6] = a3.x; w[7] = a3.y;
    w[8] = a4.x; w[9] = a4.y; w[10] = a5.x; w[11] = a5.y;
    w[12] = a6.x; w[13] = a6.y; w[14] = a7.x; w[15] = a7.y;
    if (overlap < 1) return false;
    return small ? inverse_pot4x4<false>(w) : pot16(w);
}

// Whether macroblock m of a tile's 6 x 6 ring-and-tile grid is one of the
// tile's own 4 x 4.
__device__ __forceinline__ bool inner_mb(int m) {
    const int a = m % 6, b = m / 6;
    return a >= 1 && a <= 4 && b >= 1 && b <= 4;
}

// Ring macroblock r (0..19) of the 6 x 6 grid: the top row, then the left
// and right macroblocks of rows 1..4 in turn, then the bottom row.
__device__ __forceinline__ int ring_mb(int r) {
    return r < 6 ? r : r < 14 ? 6 + ((r - 6) >> 1) * 6 + ((r - 6) & 1) * 5 : r + 16;
}

// The DC / low-pass values of a tile's own macroblock that codes no
// high-pass band: its coefficient run holds them alone (one DC, or all 16).
__device__ __forceinline__ void low_pass_run(const int32_t *coeff, uint4 e, int32_t (&v)[16]) {
    const int32_t *src = coeff + (e.x & 0x0fffffffu);
    const bool lp = ((e.x >> 28) & 3) != 0;
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = k == 0 || lp ? __ldg(src + k) : 0;
}

// The DC / low-pass values of a tile's own 4 x 4 macroblocks into their
// low-pass slots (`stride` apart), one value a thread, for `planes` planes
// of `plane_ints` tile ints each.  A macroblock that codes high-pass bands
// has them as coefficient 0 of its 16 blocks, staged with the blocks; one
// that codes none holds them alone in its coefficient run (one DC, or all
// 16), read here directly.
__device__ __forceinline__ void inner_low_pass(const ImageDev &im, const int32_t *tiles, int plane_ints,
                                               const uint4 *mbc, int32_t *lps, int lp_ints, int stride, int planes) {
    for (int k = threadIdx.x; k < planes * 256; k += kThreads) {
        const int pi = k >> 8, q = k & 255, mi = q >> 4, kk = q & 15;
        const int m = (1 + (mi >> 2)) * 6 + 1 + (mi & 3);
        const uint4 e = mbc[pi * 36 + m];
        const int bands = (e.x >> 28) & 3;
        int32_t v;
        if (bands >= 2) {
            const int s = (4 * (mi >> 2) + (kk >> 2)) * kIB + 4 * (mi & 3) + (kk & 3);
            v = tiles[pi * plane_ints + elem(s, 0, 0)];
        } else {
            v = kk == 0 || bands != 0 ? __ldg(im.plane[pi].coeff + (e.x & 0x0fffffffu) + kk) : 0;
        }
        lps[pi * lp_ints + m * stride + kk] = v;
    }
}

// One 16-byte piece of a coded block into its slot: copied asynchronously
// when the macroblock codes high-pass coefficients (and the piece is
// aligned), zero when it codes none.
__device__ __forceinline__ void copy_chunk(int32_t *dst, const int32_t *coeff, uint4 e, int offset) {
    const int bands = (e.x >> 28) & 3;
    if (bands >= 2) {
        const int32_t *src = coeff + (e.x & 0x0fffffffu) + offset;
        if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) cp_async16(dst, src);
        else *reinterpret_cast<int4 *>(dst) = make_int4(__ldg(src), __ldg(src + 1), __ldg(src + 2), __ldg(src + 3));
    } else {
        *reinterpret_cast<int4 *>(dst) = make_int4(0, 0, 0, 0);
    }
}

// The table entries of macroblocks mx0-1 .. mx0+4 x my0-1 .. my0+4 of every
// plane of an interior tile, copied asynchronously into `mbc` (one group).
// With EDGE (tiles that may touch the plane's edge) each of those macroblocks
// outside the plane gets a zero entry: no bands, no prediction, zero steps.
template <int NP, bool EDGE>
__device__ __forceinline__ void load_entries(const ImageDev &im, int tx, int ty, uint4 *mbc) {
    const int tid = threadIdx.x;
    if (tid < NP * 36) {
        const int pi = tid / 36, m = tid - pi * 36;
        const PlaneDev &p = im.plane[pi];
        const int mx = tx * kTileMbs - 1 + m % 6, my = ty * kTileMbs - 1 + m / 6;
        if (!EDGE || (mx >= 0 && my >= 0 && mx < (int)p.mbs_x && my < (int)p.mbs_y))
            cp_async16(&mbc[tid], &p.mbs[(size_t)my * p.mbs_stride + mx]);
        else
            mbc[tid] = make_uint4(0u, 0u, 0u, 0u);
    }
    cp_async_commit();
}

// A first-level overlap window of an edge tile whose centre lies on the
// plane's edge: the four-sample edge operator down each column (vs) or along
// each row (hs) of the window, or on each 2 x 2 quarter at a corner, wherever
// those lie in the plane (first_level_overlap, crates/jxr-native/src/
// reconstruct/overlap.rs).  (wx, wy): the window in DC tile coordinates,
// (ox, oy): the plane position of the DC tile's origin.
__device__ __noinline__ bool dc_edge_window(int32_t *dc, int wx, int wy, int ox, int oy, int Wdc, int Hdc, bool vs,
                                            bool hs) {
    auto at = [&](int x, int y) -> int32_t & { return dc[y * kIDC + x]; };
    auto in = [&](int x, int y) { return ox + x >= 0 && ox + x < Wdc && oy + y >= 0 && oy + y < Hdc; };
    bool bad = false;
    if (vs && !hs) {
        for (int c = 0; c < 4; c++)
            if (in(wx + c, wy)) bad |= inverse_pot4(at(wx + c, wy), at(wx + c, wy + 1), at(wx + c, wy + 2), at(wx + c, wy + 3));
    } else if (!vs && hs) {
        for (int r = 0; r < 4; r++)
            if (in(wx, wy + r)) bad |= inverse_pot4(at(wx, wy + r), at(wx + 1, wy + r), at(wx + 2, wy + r), at(wx + 3, wy + r));
    } else {
        for (int k = 0; k < 4; k++) {
            const int x = wx + (k & 1) * 2, y = wy + (k >> 1) * 2;
            if (in(x, y)) bad |= inverse_pot4(at(x, y), at(x + 1, y), at(x, y + 1), at(x + 1, y + 1));
        }
    }
    return bad;
}

// The sample cells of an edge tile that the plane's edge cuts, in four
// lines: the plane's column -2 beside the tile's rows (left), its row -2
// above the tile's columns (top), column W-2 (right) and row H-2 (bottom,
// without the cell the right line holds).  Cell origins (X, Y) are plane
// positions; the tile's 16 x 16 cell grid starts at (16 mx0 + 2, 16 my0 + 2).
struct EdgeCells {
    int W, H;
    int n[4];          // cells in each line
    int x[4], y[4];    // first cell of each line
    int dx[4], dy[4];  // step along the line
};

__device__ __forceinline__ EdgeCells edge_cells(const ImageDev &im, int mx0, int my0) {
    EdgeCells e;
    e.W = 16 * (int)im.plane[0].mbs_x;
    e.H = 16 * (int)im.plane[0].mbs_y;
    const int gx0 = 16 * mx0 + 2, gy0 = 16 * my0 + 2;            // grid origin
    const int gx1 = min(gx0 + 60, e.W - 2), gy1 = min(gy0 + 60, e.H - 2);   // last grid cell in the plane
    const int ly0 = my0 == 0 ? -2 : gy0;
    e.x[0] = -2; e.y[0] = ly0; e.dx[0] = 0; e.dy[0] = 4;
    e.n[0] = mx0 == 0 ? (gy1 - ly0) / 4 + 1 : 0;
    e.x[1] = gx0; e.y[1] = -2; e.dx[1] = 4; e.dy[1] = 0;
    e.n[1] = my0 == 0 ? (gx1 - gx0) / 4 + 1 : 0;
    const bool right = e.W - 2 <= gx0 + 60, bottom = e.H - 2 <= gy0 + 60;
    e.x[2] = e.W - 2; e.y[2] = gy0; e.dx[2] = 0; e.dy[2] = 4;
    e.n[2] = right ? (gy1 - gy0) / 4 + 1 : 0;
    e.x[3] = gx0; e.y[3] = e.H - 2; e.dx[3] = 4; e.dy[3] = 0;
    e.n[3] = bottom ? ((right ? e.W - 6 : gx1) - gx0) / 4 + 1 : 0;
    return e;
}

// Cell k of the lines: its origin and the part of it inside the plane
// ([c0, c1) x [r0, r1)).  False past the last cell.
__device__ __forceinline__ bool edge_cell_at(const EdgeCells &e, int k, int &X, int &Y, int &c0, int &c1, int &r0,
                                             int &r1) {
    int line = 0;
    while (line < 4 && k >= e.n[line]) k -= e.n[line++];
    if (line == 4) return false;
    X = e.x[line] + k * e.dx[line];
    Y = e.y[line] + k * e.dy[line];
    c0 = max(X, 0); c1 = min(X + 4, e.W);
    r0 = max(Y, 0); r1 = min(Y + 4, e.H);
    return true;
}

// The grid cells of an edge tile that lie wholly inside the plane (x0 + 2 < W,
// y0 + 2 < H): ncx x ncy of them, thread t taking cell (t % ncx, t / ncx)
// (the division as a multiply by ceil(2^16 / ncx), exact for t < 256).
__device__ __forceinline__ void edge_grid(const EdgeCells &ec, int mx0, int my0, int &cx, int &cy, bool &in) {
    const int ncx = min(16, (ec.W - 16 * mx0) / 4 - 1), ncy = min(16, (ec.H - 16 * my0) / 4 - 1);
    const int t = threadIdx.x;
    cy = (t * ((65536 + ncx - 1) / ncx)) >> 16;
    cx = t - cy * ncx;
    in = t < ncx * ncy;
}

// Stage D at the plane's edge, in place: in each cell the edge cuts, the
// four-sample operator down each of its two columns in the plane, along each
// of its two rows, or on its corner quarter (second_level_overlap,
// crates/jxr-native/src/reconstruct/overlap.rs).  Returns the overflow flag.
template <int NP>
__device__ __forceinline__ bool edge_overlap(const ImageDev &im, int32_t *tiles, int mx0, int my0, const EdgeCells &ec) {
    const int cells = ec.n[0] + ec.n[1] + ec.n[2] + ec.n[3];
    bool bad = false;
    for (int item = threadIdx.x; item < cells * 2 * NP; item += kThreads) {
        const int pi = item / (cells * 2), q = item - pi * cells * 2, k = q >> 1, o = q & 1;
        if (im.plane[pi].overlap < 1) continue;
        int X, Y, c0, c1, r0, r1;
        edge_cell_at(ec, k, X, Y, c0, c1, r0, r1);
        int32_t *t = tiles + pi * kPlaneInts;
        auto at = [&](int x, int y) -> int32_t & {
            const int sx = x - 16 * mx0, sy = y - 16 * my0;
            return t[elem((sy >> 2) * kIB + (sx >> 2), sy & 3, sx & 3)];
        };
        const bool vs = c1 - c0 < 4, hs = r1 - r0 < 4;
        if (vs && !hs) {
            const int x = c0 + o;
            bad |= inverse_pot4(at(x, Y), at(x, Y + 1), at(x, Y + 2), at(x, Y + 3));
        } else if (!vs && hs) {
            const int y = r0 + o;
            bad |= inverse_pot4(at(X, y), at(X + 1, y), at(X + 2, y), at(X + 3, y));
        } else if (o == 0) {
            bad |= inverse_pot4(at(c0, r0), at(c0 + 1, r0), at(c0, r0 + 1), at(c0 + 1, r0 + 1));
        }
    }
    return bad;
}

// One pixel through the specialised stores of the tile kernels' grid -- RGB8
// from YUV (alpha or padding in a fourth byte) and one channel stored as it
// is -- where they apply; the same bytes as the general store.  False where
// the pixel needs the general store.
template <int NP>
__device__ __forceinline__ bool fast_pixel(const ImageDev &im, const int32_t comp[4], int32_t a, uint8_t *dst,
                                           bool &bad) {
    const OutputDev &o = im.out;
    if (NP >= 3 && o.kind == kOutRgb8 && !o.premultiply) {
        const bool alpha = NP == 4 && im.alpha >= 0;
        if (o.channels == 4 && !alpha && !o.ch[3].padding) return false;
        if ((mag(comp[0]) | mag(comp[1]) | mag(comp[2]) | (alpha ? mag(a) : 0u)) >= (1u << 28)) return false;
        const ChannelScale &sc = o.ch[0];
        const int32_t add = sc.shifted_bias + sc.rounding;
        int32_t R, G, B;
        yuv_to_rgb_fast(comp[0], comp[1], comp[2], R, G, B);
        const uint32_t r8 = (uint32_t)min(max((R + add) >> sc.shift, 0), 255);
        const uint32_t g8 = (uint32_t)min(max((G + add) >> sc.shift, 0), 255);
        const uint32_t b8 = (uint32_t)min(max((B + add) >> sc.shift, 0), 255);
        const bool reverse = sc.source == 2;
        dst[0] = (uint8_t)(reverse ? b8 : r8);
        dst[1] = (uint8_t)g8;
        dst[2] = (uint8_t)(reverse ? r8 : b8);
        if (o.channels == 4) {
            const ChannelScale &sa = o.ch[3];
            dst[3] = alpha ? (uint8_t)min(max((a + sa.shifted_bias + sa.rounding) >> sa.shift, 0), 255) : 0;
        }
        return true;
    }
    if (NP == 1 && o.kind == kOutDirect) {
        const ChannelScale &s = o.ch[0];
        store_elem(dst, (uint32_t)min(max(apply_scale(s, comp[0], bad), s.lo), s.hi), o.elem_bytes);
        return true;
    }
    return false;
}

// Stage E at the plane's edge: the pixels of the cut cells (at most eight a
// cell), one a thread, through the general store.  Returns the output flag.
template <int NP>
__device__ __forceinline__ bool edge_pixels(const ImageDev &im, const int32_t *tiles, int mx0, int my0,
                                         const EdgeCells &ec) {
    const OutputDev &o = im.out;
    const bool has_alpha = im.alpha >= 0;
    const uint64_t pixel_bytes = o.nchw ? (uint64_t)o.elem_bytes : (uint64_t)o.elem_bytes * o.channels;
    const uint64_t chs = o.nchw ? o.plane_stride : (uint64_t)o.elem_bytes;
    const int cells = ec.n[0] + ec.n[1] + ec.n[2] + ec.n[3];
    bool bad = false;
    for (int item = threadIdx.x; item < cells * 8; item += kThreads) {
        int X, Y, c0, c1, r0, r1;
        edge_cell_at(ec, item >> 3, X, Y, c0, c1, r0, r1);
        const int w = c1 - c0, slot = item & 7;
        if (slot >= w * (r1 - r0)) continue;
        const int x = c0 + slot % w, y = r0 + slot / w;
        if (x < (int)o.crop_x || x >= (int)(o.crop_x + o.crop_w) || y < (int)o.crop_y ||
            y >= (int)(o.crop_y + o.crop_h))
            continue;
        const int sx = x - 16 * mx0, sy = y - 16 * my0;
        const int e = elem((sy >> 2) * kIB + (sx >> 2), sy & 3, sx & 3);
        int32_t comp[4] = {0, 0, 0, 0};
#pragma unroll
        for (int pi = 0; pi < NP; pi++)
            if (pi < im.nplanes && pi < 4) comp[pi] = tiles[pi * kPlaneInts + e];
        const int32_t a = has_alpha ? tiles[(NP - 1) * kPlaneInts + e] : 0;
        uint8_t *dst = o.base + (uint64_t)(y - o.crop_y) * o.row_stride + (uint64_t)(x - o.crop_x) * pixel_bytes;
        if (!fast_pixel<NP>(im, comp, a, dst, bad)) format_pixel(o, comp, a, dst, chs, bad);
    }
    return bad;
}

// One interior tile.  Its macroblock entries are already in `mbc` (copied
// while the previous tile ran); while it runs, the entries of the next work
// item go into `mbc_next`.  `claimed` is thread 0's claim of that next item.
//
// Tiles that touch the plane's edge (and no hard tile boundary) run here
// too.  Macroblocks outside the plane carry zero entries, so every stage runs
// unchanged over them and leaves zeros; the overlap windows and cells whose
// centre lies on the plane's edge take the reference's edge and corner
// operators, cells outside the plane are skipped, and the cells the edge cuts
// -- the plane's first and last two sample columns and rows -- are done after
// the grid, their pixels one a thread.
template <int NP, int MODE>
__device__ void interior_tile(const ImageDev &im, int tx, int ty, int32_t *smem, const uint4 *mbc, uint4 *mbc_next,
                              uint32_t claimed, const ImageDev *__restrict__ images, const WorkItem *__restrict__ items,
                              uint32_t item_count, TileShared &sh, uint32_t *status) {
    const int mx0 = tx * kTileMbs, my0 = ty * kTileMbs;
    const int tid = threadIdx.x;
    // MODE 0: interior tiles only; 1: edge tiles only; 2: either, by position
    const bool edge = MODE == 1 || (MODE == 2 && (mx0 == 0 || my0 == 0 || mx0 + kTileMbs >= (int)im.plane[0].mbs_x ||
                                                  my0 + kTileMbs >= (int)im.plane[0].mbs_y));
    int32_t *tiles = smem;                       // NP planes of kIBlocks slots
    int32_t *dcs = smem + NP * kPlaneInts;       // NP DC tiles of kIDC x kIDC
    int32_t *lps = dcs + NP * kDcInts;           // NP x 36 macroblocks x 16 DC / low-pass coefficients (lp_stride<NP>() apart)
    if (tid == 0) sh.bad = 0;
    int bad = 0;
    // phase 1: every coefficient the tile reads, in flight at once.  The DC /
    // low-pass coefficients of the ring of 20 macroblocks around the tile, 4
    // bytes each; then the coded blocks, 16 bytes a thread.  Each of the
    // tile's 4 x 4 macroblocks is 1 KB of the arena: 64 threads copy one, in
    // order, and its low-pass coefficients -- coefficient 0 of each of its
    // blocks -- arrive with it, so they are not gathered as 16 scattered
    // words.  The halo follows: the first block column of the macroblocks
    // right of the tile, the first block row of those below it, and the
    // corner block.
    for (int k = tid; k < NP * 320; k += kThreads) {
        const int pi = k / 320, q = k - pi * 320, m = ring_mb(q >> 4), kk = q & 15;
        const uint4 e = mbc[pi * 36 + m];
        const int bands = (e.x >> 28) & 3;
        int32_t *dst = lps + pi * lp_ints<NP>() + m * lp_stride<NP>() + kk;
        if (kk == 0 || bands != 0)
            cp_async4(dst, im.plane[pi].coeff + (e.x & 0x0fffffffu) + (bands >= 2 ? kk * 16 : kk));
        else
            *dst = 0;
    }
    // the planes one after another in the four-plane kernel, whose code size
    // stalls instruction fetch (C3 1.004 -> 0.990 ms a step), unrolled in the
    // others
    constexpr int kCopyUnroll = NP == 4 ? 1 : NP;
#pragma unroll kCopyUnroll
    for (int pi = 0; pi < NP; pi++) {
        const int32_t *coeff = im.plane[pi].coeff;
        int32_t *tile = tiles + pi * kPlaneInts;
        const uint4 *ent = mbc + pi * 36;
#pragma unroll
        for (int pass = 0; pass < 4; pass++) {
            const int mb = pass * 4 + (tid >> 6), c = tid & 63;
            const int a = mb & 3, b = mb >> 2, blk = c >> 2, r = c & 3;
            const int sidx = (4 * b + (blk >> 2)) * kIB + 4 * a + (blk & 3);
            copy_chunk(tile + sidx * 16 + ((r ^ swz(sidx)) << 2), coeff, ent[(b + 1) * 6 + a + 1], c * 4);
        }
        if (tid < 33 * 4) {
            const int hb = tid >> 2, r = tid & 3;
            const int i = hb < 16 ? 16 : hb < 32 ? hb - 16 : 16;
            const int j = hb < 16 ? hb : 16;
            const int sidx = j * kIB + i;
            copy_chunk(tile + sidx * 16 + ((r ^ swz(sidx)) << 2), coeff, ent[((j >> 2) + 1) * 6 + (i >> 2) + 1],
                       (((j & 3) << 2) + (i & 3)) * 16 + r * 4);
        }
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    // The tile's own low-pass values: with three planes copied into the
    // padded slots first, one value a thread, so that stage A reads every
    // macroblock's 16 values as four conflict-free 16-byte loads (C2
    // 0.1694 -> 0.1668 ms a step); with four planes the extra pass and
    // barrier cost more than the conflicts of reading them in stage A straight
    // from the blocks (C3 1.131 -> 1.165 ms), so those read them there.
    constexpr bool kCopyInner = NP == 3;
    if (kCopyInner) {
        inner_low_pass(im, tiles, kPlaneInts, mbc, lps, lp_ints<NP>(), lp_stride<NP>(), NP);
        __syncthreads();
    }
    // stage A: first level of macroblocks mx0-1 .. mx0+4 (every one exists)
    for (int item = tid; item < NP * 36; item += kThreads) {
        const int pi = item / 36, m = item - pi * 36;
        const PlaneDev &p = im.plane[pi];
        const uint4 e = mbc[item];
        int32_t v[16];
        bool b = false;
        if (!kCopyInner && inner_mb(m)) {
            if (((e.x >> 28) & 3) >= 2) {
                const int32_t *t = tiles + pi * kPlaneInts;
                const int s0 = (4 * (m / 6) - 4) * kIB + 4 * (m % 6) - 4;
#pragma unroll
                for (int k = 0; k < 16; k++) v[k] = t[elem(s0 + (k >> 2) * kIB + (k & 3), 0, 0)];
            } else {
                low_pass_run(p.coeff, e, v);
            }
        } else {
            const int32_t *l = lps + pi * lp_ints<NP>() + m * lp_stride<NP>();
#pragma unroll
            for (int k = 0; k < 16; k += 4) {
                const int4 q = *reinterpret_cast<const int4 *>(l + k);
                v[k] = q.x; v[k + 1] = q.y; v[k + 2] = q.z; v[k + 3] = q.w;
            }
        }
        // one magnitude test of the coded values: below the transform's bound
        // after dequantization, every product fits and the wrapping
        // transform is exact; otherwise the checked steps
        uint32_t lm = 0;
#pragma unroll
        for (int k = 1; k < 16; k++) lm |= mag(v[k]);
        if ((uint64_t)(lm + 1) * e.z < (uint64_t)kTransformBound &&
            (uint64_t)(mag(v[0]) + 1) * e.y < (uint64_t)kTransformBound) {
            v[0] *= (int32_t)e.y;
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] *= (int32_t)e.z;
            inverse_pct<false>(v);
        } else {
            v[0] = dequant(v[0], e.y, b);
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] = dequant(v[k], e.z, b);
            b |= pct16(v);
        }
        if (p.scale2) {
#pragma unroll
            for (int k = 0; k < 16; k++) v[k] = dequant(v[k], 2, b);
        }
        int32_t *out = dcs + pi * kDcInts + (m / 6) * 4 * kIDC + (m % 6) * 4;
#pragma unroll
        for (int r = 0; r < 4; r++)
            *reinterpret_cast<int4 *>(out + r * kIDC) = make_int4(v[r * 4], v[r * 4 + 1], v[r * 4 + 2], v[r * 4 + 3]);
        if (b) bad |= kFlagFirst;
    }
    if (tid == 0) sh.next = claimed;
    __syncthreads();
    // the next work item's macroblock entries, in flight through stage B
    const uint32_t next = sh.next;
    const WorkItem wnext = next < item_count ? items[next] : WorkItem{0, 0, 0};
    const ImageDev &imn = images[wnext.image & kImageMask];
    if (next < item_count) load_entries<NP, MODE != 0>(imn, wnext.tx, wnext.ty, mbc_next);
    // stages B and C1 in one pass: they touch disjoint data (the DC tile; the
    // first row and column of the high-pass blocks), so one barrier follows
    // both.  The overlap windows, the heavier items, go to threads that get no
    // second item; the prediction lines fill the rest.
    constexpr int kItemsB = NP * 25, kItemsC1 = NP * 100;
    constexpr int kFirstB = (kItemsB + kItemsC1 < kThreads ? kItemsB + kItemsC1 : kThreads) - kItemsB;
    for (int k = tid; k < kItemsB + kItemsC1; k += kThreads) {
        if (k >= kFirstB && k < kFirstB + kItemsB) {
            // stage B: first-level overlap, 5 x 5 interior windows at DC (2 + 4a, 2 + 4b)
            const int item = k - kFirstB;
            const int pi = item / 25, c = item - pi * 25;
            if (im.plane[pi].overlap != 2) continue;
            if (edge) {
                // the window's centre lies on macroblock boundary (mx0 + a, my0 + b)
                const PlaneDev &p = im.plane[pi];
                const int ca = mx0 + c % 5, cb = my0 + c / 5;
                if (ca > (int)p.mbs_x || cb > (int)p.mbs_y) continue;   // beyond the plane
                const bool vs = ca == 0 || ca == (int)p.mbs_x, hs = cb == 0 || cb == (int)p.mbs_y;
                if (vs || hs) {
                    if (dc_edge_window(dcs + pi * kDcInts, 2 + 4 * (c % 5), 2 + 4 * (c / 5), 4 * (mx0 - 1),
                                       4 * (my0 - 1), 4 * (int)p.mbs_x, 4 * (int)p.mbs_y, vs, hs))
                        bad |= kFlagOverlap;
                    continue;
                }
            }
            int32_t *base = dcs + pi * kDcInts + (2 + 4 * (c / 5)) * kIDC + 2 + 4 * (c % 5);
            int32_t v[16];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int2 a = *reinterpret_cast<const int2 *>(base + r * kIDC);
                const int2 b = *reinterpret_cast<const int2 *>(base + r * kIDC + 2);
                v[r * 4] = a.x; v[r * 4 + 1] = a.y; v[r * 4 + 2] = b.x; v[r * 4 + 3] = b.y;
            }
            if (pot16(v)) bad |= kFlagOverlap;
#pragma unroll
            for (int r = 0; r < 4; r++) {
                *reinterpret_cast<int2 *>(base + r * kIDC) = make_int2(v[r * 4], v[r * 4 + 1]);
                *reinterpret_cast<int2 *>(base + r * kIDC + 2) = make_int2(v[r * 4 + 2], v[r * 4 + 3]);
            }
        } else {
            // stage C1: prediction within macroblocks mx0 .. mx0+4; of the fifth
            // column and row of macroblocks only their first block column / row
            // lies in the tile, along which the other direction of prediction
            // still runs
            const int item = k < kFirstB ? k : k - kItemsB;
            const int pi = item / 100, q = item - pi * 100;
            const int line = q & 3, m = q >> 2;
            const int a = m % 5, b = m / 5;
            const uint4 e = mbc[pi * 36 + (b + 1) * 6 + a + 1];
            const int hp = (e.x >> 30) & 3, bands = (e.x >> 28) & 3;
            if (hp == 0 || bands < 2) continue;
            if (hp == 3) { bad |= kFlagInvalid; continue; }
            int32_t *t = tiles + pi * kPlaneInts;
            using A = Ar<true>;
            bool ov = false;
            if (hp == 1) {
                // from left along block row `line`: needs columns 1..3 (a < 4)
                if (a == 4 || (b == 4 && line != 0)) continue;
                const int j = 4 * b + line;
#pragma unroll
                for (int c = 1; c < 4; c++) {
                    const int sidx = j * kIB + 4 * a + c;
#pragma unroll
                    for (int r = 1; r < 4; r++) t[elem(sidx, r, 0)] = A::add(t[elem(sidx, r, 0)], t[elem(sidx - 1, r, 0)], ov);
                }
            } else {
                // from top along block column `line`: needs rows 1..3 (b < 4)
                if (b == 4 || (a == 4 && line != 0)) continue;
                const int i = 4 * a + line;
#pragma unroll
                for (int r = 1; r < 4; r++) {
                    const int sidx = (4 * b + r) * kIB + i;
#pragma unroll
                    for (int c = 1; c < 4; c++) t[elem(sidx, 0, c)] = A::add(t[elem(sidx, 0, c)], t[elem(sidx - kIB, 0, c)], ov);
                }
            }
            if (ov) bad |= kFlagPrediction;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // stage C2: block transforms of the 17 x 17 blocks; an edge tile's items
    // are only its blocks inside the plane (q / bcols as a multiply by
    // ceil(2^16 / bcols), exact for q < 2^16 / 17)
    int bcols = kIB, brows = kIB, bmagic = 0;
    if (edge) {
        bcols = min(kIB, 4 * ((int)im.plane[0].mbs_x - mx0));
        brows = min(kIB, 4 * ((int)im.plane[0].mbs_y - my0));
        bmagic = (65536 + bcols - 1) / bcols;
    }
    const int bcount = bcols * brows;
    bool small = true;   // every transform input of this thread's blocks below 2^16
    for (int item = tid; item < NP * bcount; item += kThreads) {
        int pi, s, i, j;
        if (edge) {
            int q = item;
            for (pi = 0; q >= bcount; pi++) q -= bcount;
            j = (q * bmagic) >> 16;
            i = q - j * bcols;
            s = j * kIB + i;
        } else {
            pi = item / kIBlocks;
            s = item - pi * kIBlocks;
            i = s % kIB;
            j = s / kIB;
        }
        const uint32_t step = mbc[pi * 36 + ((j >> 2) + 1) * 6 + (i >> 2) + 1].w;
        int32_t *blk = tiles + pi * kPlaneInts + s * 16;
        const int sw = swz(s);
        int32_t v[16];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int4 q = *reinterpret_cast<const int4 *>(blk + ((r ^ sw) << 2));
            v[r * 4 + 0] = q.x; v[r * 4 + 1] = q.y; v[r * 4 + 2] = q.z; v[r * 4 + 3] = q.w;
        }
        uint32_t m = 0;
#pragma unroll
        for (int k = 1; k < 16; k++) m |= mag(v[k]);
        v[0] = dcs[pi * kDcInts + (j + 4) * kIDC + i + 4];
        bool b = false;
        small &= (uint64_t)(m + 1) * step <= (1u << 16) && mag(v[0]) < (1u << 16);
        if ((uint64_t)(m + 1) * step < (uint64_t)kTransformBound && mag(v[0]) < (uint32_t)kTransformBound) {
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] = v[k] * (int32_t)step;
            inverse_pct<false>(v);
        } else {
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] = dequant(v[k], step, b);
            b |= pct16(v);
        }
        if (b) bad |= kFlagSecond;
#pragma unroll
        for (int r = 0; r < 4; r++)
            *reinterpret_cast<int4 *>(blk + ((r ^ sw) << 2)) = make_int4(v[r * 4], v[r * 4 + 1], v[r * 4 + 2], v[r * 4 + 3]);
    }
    const bool tile_small = __syncthreads_and(small) != 0;
    bool grid_cell = true;
    int gcx = tid & 15, gcy = tid >> 4;   // the thread's cell of the 16 x 16 grid
    EdgeCells ec;
    if (edge) {
        ec = edge_cells(im, mx0, my0);
        if (edge_overlap<NP>(im, tiles, mx0, my0, ec)) bad |= kFlagOverlap;
        __syncthreads();
        // cells past the plane's edge, or cut by it, leave the grid; the
        // rest are packed onto the first threads, so that whole warps idle
        edge_grid(ec, mx0, my0, gcx, gcy, grid_cell);
    }
    // stage D + E: the thread's sample cell, every plane, then its 16 pixels
    if (grid_cell) {
        const int cx = gcx, cy = gcy;
        const int b00 = cy * kIB + cx;
        const OutputDev &o = im.out;
        const int x0 = 16 * mx0 + 2 + 4 * cx, y0 = 16 * my0 + 2 + 4 * cy;
        const bool inside = x0 >= (int)o.crop_x && x0 + 4 <= (int)(o.crop_x + o.crop_w) && y0 >= (int)o.crop_y &&
                            y0 + 4 <= (int)(o.crop_y + o.crop_h);
        const int kind = o.kind;
        const bool has_alpha = im.alpha >= 0;
        bool obad = false, done = false;
        if (inside && kind == kOutRgb8 && NP >= 3 && !o.premultiply) {
            int32_t y[16], u[16], v[16];
            bool ov = cell_samples(tiles, b00, im.plane[0].overlap, y, tile_small);
            ov |= cell_samples(tiles + kPlaneInts, b00, im.plane[1].overlap, u, tile_small);
            ov |= cell_samples(tiles + 2 * kPlaneInts, b00, im.plane[2].overlap, v, tile_small);
            if (ov) bad |= kFlagOverlap;
            uint32_t m = 0;
            if (!tile_small) {
#pragma unroll
                for (int k = 0; k < 16; k++) m |= mag(y[k]) | mag(u[k]) | mag(v[k]);
            }
            if (m < (1u << 28)) {
                const ChannelScale &sc = o.ch[0];
                const int32_t add = sc.shifted_bias + sc.rounding;
                const int shift = sc.shift;
                // byte order of the packed pixel: R G B, or B G R
                const uint32_t order = sc.source == 2 ? 0x7014u : 0x7410u;
                uint32_t px[16];
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    // each colour is luma plus terms in u and v, so adding the
                    // output bias to luma adds it to all three (no
                    // intermediate nears int32 below 2^28)
                    int32_t R, G, B;
                    yuv_to_rgb_fast(y[k] + add, u[k], v[k], R, G, B);
                    px[k] = pack_rgb8(clamp_u8(R >> shift), clamp_u8(G >> shift), clamp_u8(B >> shift), order);
                }
                bool alpha_ok = true;
                if (NP == 4 && has_alpha) {
                    int32_t a[16];
                    if (cell_samples(tiles + 3 * kPlaneInts, b00, im.plane[3].overlap, a, tile_small))
                        bad |= kFlagOverlap;
                    const ChannelScale &sa = o.ch[3];
                    const int32_t aadd = sa.shifted_bias + sa.rounding;
                    uint32_t am = 0;
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        am |= mag(a[k]);
                        px[k] |= clamp_u8((a[k] + aadd) >> sa.shift) << 24;
                    }
                    alpha_ok = tile_small || am < (1u << 28);
                }
                if (alpha_ok) {
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        uint8_t *dst = o.base + (uint64_t)(y0 + r - o.crop_y) * o.row_stride +
                                       (uint64_t)(x0 - o.crop_x) * o.channels;
                        if (o.channels == 4) store16(dst, px[4 * r], px[4 * r + 1], px[4 * r + 2], px[4 * r + 3]);
                        else store12(dst, &px[4 * r]);
                    }
                    done = true;
                }
            }
        } else if (inside && kind == kOutDirect && NP == 1) {
            int32_t y[16];
            if (cell_samples(tiles, b00, im.plane[0].overlap, y, tile_small)) bad |= kFlagOverlap;
            const ChannelScale &s = o.ch[0];
            const int eb = o.elem_bytes;
#pragma unroll
            for (int r = 0; r < 4; r++) {
                uint32_t q[4];
#pragma unroll
                for (int c = 0; c < 4; c++) q[c] = (uint32_t)min(max(apply_scale(s, y[r * 4 + c], obad), s.lo), s.hi);
                uint8_t *dst = o.base + (uint64_t)(y0 + r - o.crop_y) * o.row_stride + (uint64_t)(x0 - o.crop_x) * eb;
                if (eb == 2) store8(dst, (q[0] & 0xffffu) | (q[1] << 16), (q[2] & 0xffffu) | (q[3] << 16));
                else if (eb == 4) store16(dst, q[0], q[1], q[2], q[3]);
                else for (int c = 0; c < 4; c++) dst[c] = (uint8_t)q[c];
            }
            done = true;
        } else if (inside && kind == kOutF16Wide && o.nchw && NP == 4 && o.channels <= NP) {
            // colour channel planes first, then alpha
            int32_t y[16], u[16], v[16];
            bool ov = cell_samples(tiles, b00, im.plane[0].overlap, y, tile_small);
            ov |= cell_samples(tiles + kPlaneInts, b00, im.plane[1].overlap, u, tile_small);
            ov |= cell_samples(tiles + 2 * kPlaneInts, b00, im.plane[2].overlap, v, tile_small);
            if (ov) bad |= kFlagOverlap;
            uint8_t *base = o.base + (uint64_t)(y0 - o.crop_y) * o.row_stride + (uint64_t)(x0 - o.crop_x) * 4;
            const int primaries = has_alpha ? o.channels - 1 : o.channels;
            const uint64_t rs = o.row_stride, ps = o.plane_stride;
            // The channels' terms in registers (the stores may alias the
            // descriptor).  YUV below 2^28 keeps the inverse RCT below 2^30,
            // and terms below 2^28 keep every scaling step below 2^31: no
            // checked step can overflow, so the unchecked forms give the same
            // values.  A tile whose transform inputs were all below 2^16 has
            // its overlap outputs below 2^27.8, so its cells skip that test.
            // The lean form takes R, G and B to channels 0, 1, 2 with no
            // padding channel; other orders take the general form.
            // Four-plane kernels only: in the three-plane one the extra code
            // costs the RGB8 path more than it saves here.
            int32_t cadd[3], cshift[3];
            bool lean = o.conv == kConvYuvToRgb && !o.packed_swap;
#pragma unroll
            for (int ch = 0; ch < 3; ch++) {
                const ChannelScale &s = o.ch[ch];
                cadd[ch] = s.shifted_bias + s.rounding;
                cshift[ch] = s.shift;
                lean &= s.source == ch && !s.padding && s.post_shift < 0 && mag(s.shifted_bias) < (1u << 28) &&
                        mag(s.rounding) < (1u << 28);
            }
            if (lean && !tile_small) {
                uint32_t m = 0;
#pragma unroll
                for (int k = 0; k < 16; k++) m |= mag(y[k]) | mag(u[k]) | mag(v[k]);
                lean = m < (1u << 28);
            }
#pragma unroll
            for (int r = 0; r < 4; r++) {
                uint32_t q[3][4];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int k = r * 4 + c;
                    if (lean) {
                        int32_t R, G, B;
                        yuv_to_rgb_fast(y[k], u[k], v[k], R, G, B);
                        q[0][c] = f16_widened((R + cadd[0]) >> cshift[0]);
                        q[1][c] = f16_widened((G + cadd[1]) >> cshift[1]);
                        q[2][c] = f16_widened((B + cadd[2]) >> cshift[2]);
                    } else {
                        const int32_t in[4] = {y[k], u[k], v[k], 0};
                        int32_t conv[4];
                        convert(o, in, conv, obad);
#pragma unroll
                        for (int ch = 0; ch < 3; ch++) {
                            const ChannelScale &s = o.ch[ch];
                            const int src = s.source;
                            const int32_t val = apply_scale(s, src == 0 ? conv[0] : src == 1 ? conv[1] : conv[2], obad);
                            const uint32_t mm = min((uint32_t)(val < 0 ? -(int64_t)val : val), 32767u);
                            q[ch][c] = widen_f16(s.padding ? 0u : ((val < 0 ? 0x8000u : 0u) | mm));
                        }
                    }
                }
#pragma unroll
                for (int ch = 0; ch < 3; ch++)
                    if (ch < primaries) store16(base + r * rs + ch * ps, q[ch][0], q[ch][1], q[ch][2], q[ch][3]);
            }
            if (has_alpha && NP == 4) {
                int32_t a[16];
                if (cell_samples(tiles + 3 * kPlaneInts, b00, im.plane[3].overlap, a, tile_small)) bad |= kFlagOverlap;
                const ChannelScale &s = o.ch[o.channels - 1];
                bool alean = s.post_shift < 0 && mag(s.shifted_bias) < (1u << 28) && mag(s.rounding) < (1u << 28);
                if (alean && !tile_small) {
                    uint32_t am = 0;
#pragma unroll
                    for (int k = 0; k < 16; k++) am |= mag(a[k]);
                    alean = am < (1u << 29);
                }
                const int32_t aadd = s.shifted_bias + s.rounding, ashift = s.shift;
                uint8_t *abase = base + (uint64_t)(o.channels - 1) * ps;
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    uint32_t q[4];
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        q[c] = f16_widened(alean ? (a[r * 4 + c] + aadd) >> ashift : apply_scale(s, a[r * 4 + c], obad));
                    store16(abase + r * rs, q[0], q[1], q[2], q[3]);
                }
            }
            done = true;
        } else if (inside && kind == kOutF16Wide && o.nchw && NP == 3 && o.channels <= NP) {
            // colour channel planes first, then alpha
            int32_t y[16], u[16], v[16];
            bool ov = cell_samples(tiles, b00, im.plane[0].overlap, y, tile_small);
            ov |= cell_samples(tiles + kPlaneInts, b00, im.plane[1].overlap, u, tile_small);
            ov |= cell_samples(tiles + 2 * kPlaneInts, b00, im.plane[2].overlap, v, tile_small);
            if (ov) bad |= kFlagOverlap;
            uint8_t *base = o.base + (uint64_t)(y0 - o.crop_y) * o.row_stride + (uint64_t)(x0 - o.crop_x) * 4;
            const int primaries = has_alpha ? o.channels - 1 : o.channels;
#pragma unroll
            for (int r = 0; r < 4; r++) {
                uint32_t q[3][4];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int k = r * 4 + c;
                    const int32_t in[4] = {y[k], u[k], v[k], 0};
                    int32_t conv[4];
                    convert(o, in, conv, obad);
#pragma unroll
                    for (int ch = 0; ch < 3; ch++) {
                        const ChannelScale &s = o.ch[ch];
                        const int src = s.source;
                        const int32_t val = apply_scale(s, src == 0 ? conv[0] : src == 1 ? conv[1] : conv[2], obad);
                        const uint32_t mm = min((uint32_t)(val < 0 ? -(int64_t)val : val), 32767u);
                        q[ch][c] = widen_f16(s.padding ? 0u : ((val < 0 ? 0x8000u : 0u) | mm));
                    }
                }
#pragma unroll
                for (int ch = 0; ch < 3; ch++)
                    if (ch < primaries)
                        store16(base + r * o.row_stride + ch * o.plane_stride, q[ch][0], q[ch][1], q[ch][2], q[ch][3]);
            }
            if (has_alpha && NP == 4) {
                int32_t a[16];
                if (cell_samples(tiles + 3 * kPlaneInts, b00, im.plane[3].overlap, a, tile_small)) bad |= kFlagOverlap;
                const ChannelScale &s = o.ch[o.channels - 1];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    uint32_t q[4];
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int32_t val = apply_scale(s, a[r * 4 + c], obad);
                        const uint32_t mm = min((uint32_t)(val < 0 ? -(int64_t)val : val), 32767u);
                        q[c] = widen_f16((val < 0 ? 0x8000u : 0u) | mm);
                    }
                    store16(base + r * o.row_stride + (o.channels - 1) * o.plane_stride, q[0], q[1], q[2], q[3]);
                }
            }
            done = true;
        }
        if (!done) {
            // any other output, or pixels at the crop edge: the general store,
            // pixel by pixel, from every plane's cell samples
            int32_t w[NP][16];
#pragma unroll
            for (int pi = 0; pi < NP; pi++)
                if (cell_samples(tiles + pi * kPlaneInts, b00, im.plane[pi].overlap, w[pi], tile_small))
                    bad |= kFlagOverlap;
            const uint64_t pixel_bytes = o.nchw ? (uint64_t)o.elem_bytes : (uint64_t)o.elem_bytes * o.channels;
            const uint64_t chs = o.nchw ? o.plane_stride : (uint64_t)o.elem_bytes;
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) {
                    const int x = x0 + c, yy = y0 + r;
                    if (x < (int)o.crop_x || x >= (int)(o.crop_x + o.crop_w) || yy < (int)o.crop_y ||
                        yy >= (int)(o.crop_y + o.crop_h))
                        continue;
                    const int k = r * 4 + c;
                    int32_t comp[4] = {0, 0, 0, 0};
#pragma unroll
                    for (int pi = 0; pi < NP; pi++)
                        if (pi < im.nplanes && pi < 4) comp[pi] = w[pi][k];
                    const int32_t a = has_alpha ? w[NP - 1][k] : 0;
                    uint8_t *dst = o.base + (uint64_t)(yy - o.crop_y) * o.row_stride + (uint64_t)(x - o.crop_x) * pixel_bytes;
                    format_pixel(o, comp, a, dst, chs, obad);
                }
        }
        if (obad) bad |= kFlagOutput;
    }
    if (edge && edge_pixels<NP>(im, tiles, mx0, my0, ec)) bad |= kFlagOutput;
    if (bad) atomicOr(&sh.bad, bad);
    __syncthreads();
    if (tid == 0 && sh.bad) {
        const int b = sh.bad;
        const uint32_t code = (b & kFlagInvalid) ? kStatusInvalid
                            : (b & kFlagFirst) ? kStatusFirstTransform
                            : (b & kFlagOverlap) ? kStatusOverlap
                            : (b & kFlagPrediction) ? kStatusPrediction
                            : (b & kFlagSecond) ? kStatusSecondTransform
                            : kStatusOutput;
        atomicCAS(status, 0u, code);
    }
    __syncthreads();
}

__device__ void reconstruct_tile(const ImageDev &im, int tx, int ty, int32_t *smem, TileShared &sh, uint32_t *status) {
    const int mx0 = tx * kTileMbs, mx1 = min(mx0 + kTileMbs, (int)im.mbs_x);
    const int my0 = ty * kTileMbs, my1 = min(my0 + kTileMbs, (int)im.mbs_y);
    const int LW = (int)im.mbs_x * 16, LH = (int)im.mbs_y * 16;
    const int X0 = mx0 == 0 ? 0 : 16 * mx0 + 2, X1 = mx1 == (int)im.mbs_x ? LW : 16 * mx1 + 2;
    const int Y0 = my0 == 0 ? 0 : 16 * my0 + 2, Y1 = my1 == (int)im.mbs_y ? LH : 16 * my1 + 2;
    const int np = im.nplanes + (im.alpha >= 0 ? 1 : 0);
    int32_t *tiles = smem;
    int32_t *dcs = smem + np * kPlaneInts;
    {
        const int pi = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (pi < np) {
            PlaneGeom g;
            plane_geometry(im.plane[pi], pi >= 1 && pi <= 2 && pi < im.nplanes, im.chroma, X0, X1, Y0, Y1, g);
            plane_masks(im.plane[pi], g, lane);
            if (lane == 0) sh.geo[pi] = g;
        }
    }
    if (threadIdx.x == 0) sh.bad = 0;
    __syncthreads();
    int bad = 0;
    // stage 0: every block's coefficients on their way; stage A meanwhile
    {
        int item = threadIdx.x;
        for (int pi = 0; pi < np; pi++) {
            const PlaneGeom &g = sh.geo[pi];
            const int n = g.nbx * (g.by1 - g.by0 + 1);
            for (; item < n; item += blockDim.x) stage_load_blocks(im.plane[pi], g, tiles + pi * kPlaneInts, item);
            item -= n;
        }
        cp_async_commit();
    }
    {
        int item = threadIdx.x;
        for (int pi = 0; pi < np; pi++) {
            const PlaneGeom &g = sh.geo[pi];
            const int n = (g.mx1 - g.mx0 + 1) * (g.my1 - g.my0 + 1);
            for (; item < n; item += blockDim.x)
                if (stage_first_level(im.plane[pi], g, dcs + pi * kDcInts, item)) bad |= kFlagFirst;
            item -= n;
        }
    }
    __syncthreads();
    // stage B: first-level overlap (overlap mode 2 only)
    {
        int item = threadIdx.x;
        for (int pi = 0; pi < np; pi++) {
            const PlaneDev &p = im.plane[pi];
            const PlaneGeom &g = sh.geo[pi];
            if (p.overlap != 2 || p.bc != 4) continue;
            const int n = ((cell_of(g.bx1) - cell_of(g.bx0)) / 4 + 1) * ((cell_of(g.by1) - cell_of(g.by0)) / 4 + 1);
            for (; item < n; item += blockDim.x)
                if (dc_cell(g, dcs + pi * kDcInts, item)) bad |= kFlagOverlap;
            item -= n;
        }
    }
    bool any_subsampled = false;
    for (int pi = 0; pi < np; pi++) any_subsampled |= im.plane[pi].overlap == 2 && im.plane[pi].bc != 4;
    if (any_subsampled) {
        for (int phase = 0; phase < 3; phase++) {
            int item = threadIdx.x;
            for (int pi = 0; pi < np; pi++) {
                const PlaneDev &p = im.plane[pi];
                const PlaneGeom &g = sh.geo[pi];
                if (p.overlap != 2 || p.bc == 4) continue;
                const int n = ((g.ox1 - g.ox0) / 2 + 1) * ((g.oy1 - g.oy0) / 2 + 1);
                for (; item < n; item += blockDim.x)
                    if (subsampled_cell(p, g, dcs + pi * kDcInts, item, phase)) bad |= kFlagOverlap;
                item -= n;
            }
            __syncthreads();
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // stage C1: prediction
    {
        int item = threadIdx.x;
        bool invalid = false;
        for (int pi = 0; pi < np; pi++) {
            const PlaneDev &p = im.plane[pi];
            const PlaneGeom &g = sh.geo[pi];
            const int n = (g.bx1 / p.bc - g.bx0 / p.bc + 1) * (g.by1 / p.br - g.by0 / p.br + 1) * 4;
            for (; item < n; item += blockDim.x)
                if (stage_prediction(p, g, tiles + pi * kPlaneInts, item, invalid)) bad |= kFlagPrediction;
            item -= n;
        }
        if (invalid) bad |= kFlagInvalid;
    }
    __syncthreads();
    // stage C2: block transforms
    {
        int item = threadIdx.x;
        for (int pi = 0; pi < np; pi++) {
            const PlaneGeom &g = sh.geo[pi];
            const int n = g.nbx * (g.by1 - g.by0 + 1);
            for (; item < n; item += blockDim.x)
                if (stage_block_transform(im.plane[pi], g, tiles + pi * kPlaneInts, dcs + pi * kDcInts, item))
                    bad |= kFlagSecond;
            item -= n;
        }
    }
    __syncthreads();
    // stage D: second-level overlap
    {
        int item = threadIdx.x;
        for (int pi = 0; pi < np; pi++) {
            const PlaneDev &p = im.plane[pi];
            const PlaneGeom &g = sh.geo[pi];
            if (p.overlap < 1) continue;
            const TileView tv{tiles + pi * kPlaneInts, g.bx0, g.by0, g.nbx};
            const int n = ((g.cx1 - g.cx0) / 4 + 1) * ((g.cy1 - g.cy0) / 4 + 1);
            for (; item < n; item += blockDim.x)
                if (sample_cell(g, tv, item)) bad |= kFlagOverlap;
            item -= n;
        }
    }
    __syncthreads();
    // stage E: output
    PlaneView views[JXRB_MAX_PLANES];
#pragma unroll
    for (int pi = 0; pi < JXRB_MAX_PLANES; pi++) {
        if (pi >= np) break;
        const PlaneGeom &g = sh.geo[pi];
        views[pi].tv = TileView{tiles + pi * kPlaneInts, g.bx0, g.by0, g.nbx};
        views[pi].x0 = g.sx0;
        views[pi].x1 = g.sx1;
        views[pi].y0 = g.sy0;
        views[pi].y1 = g.sy1;
    }
    bool obad = false;
    switch (im.out.kind) {
    case kOutRgb8: output_rgb8(im, views, X0, X1, Y0, Y1, obad); break;
    case kOutDirect: output_direct(im, views, X0, X1, Y0, Y1, obad); break;
    case kOutF16Wide: output_f16wide(im, views, X0, X1, Y0, Y1, obad); break;
    default: output_generic(im, views, X0, X1, Y0, Y1, obad); break;
    }
    if (obad) bad |= kFlagOutput;
    if (bad) atomicOr(&sh.bad, bad);
    __syncthreads();
    if (threadIdx.x == 0 && sh.bad) {
        const int b = sh.bad;
        const uint32_t code = (b & kFlagInvalid) ? kStatusInvalid
                            : (b & kFlagFirst) ? kStatusFirstTransform
                            : (b & kFlagOverlap) ? kStatusOverlap
                            : (b & kFlagPrediction) ? kStatusPrediction
                            : (b & kFlagSecond) ? kStatusSecondTransform
                            : kStatusOutput;
        atomicCAS(status, 0u, code);
    }
    __syncthreads();
}

// Dynamic tile scheduling: CTAs claim work items from counters[0]; the last
// CTA to leave resets both counters for the next launch on the stream.
__device__ __forceinline__ bool claim(uint32_t *counters, uint32_t count, uint32_t &item) {
    __shared__ uint32_t s_item;
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[0], 1u);
    __syncthreads();
    item = s_item;
    __syncthreads();
    return item < count;
}

__device__ __forceinline__ void retire(uint32_t *counters) {
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&counters[1], 1u) == gridDim.x - 1) {
            counters[0] = 0;
            counters[1] = 0;
            __threadfence();
        }
    }
}

// Border tiles and every image the interior path does not take.
extern "C" __global__ void __launch_bounds__(kThreads, 2)
jxrb_reconstruct_tiles(const ImageDev *__restrict__ images, const WorkItem *__restrict__ items, uint32_t item_count,
                       uint32_t *status, uint32_t *counters) {
    extern __shared__ __align__(16) int32_t smem[];
    __shared__ TileShared sh;
    uint32_t i;
    while (claim(counters, item_count, i)) {
        const WorkItem w = items[i];
        reconstruct_tile(images[w.image & kImageMask], w.tx, w.ty, smem, sh, status);
    }
    retire(counters);
}

// ---------------------------------------------------------------------------
// Interior tiles of YUV 4:2:0 images (three planes, chroma 2 x 2 blocks a
// macroblock).  Luma is the full-resolution interior tile above.  Each
// chroma plane holds the 11 x 11 blocks of macroblocks mx0-1 .. mx0+4 (the
// last one's first block column / row only): block column 2*mx0-2 is there
// for high-pass prediction alone; columns 2*mx0-1 .. 2*mx0+8 are
// reconstructed, and their samples, after the second-level overlap cells at
// chroma origins 8*mx0-2 + 4k (k = 0..8), are the ones the luma pixels of the
// tile interpolate from (4 chroma columns and rows around each luma cell).
// In the interior every first-level chroma window is a plain 2 x 2 square
// at odd DC origins and every overlap cell a plain 4 x 4 window.
// ---------------------------------------------------------------------------
constexpr int kCB = 11;                          // chroma blocks across / down
constexpr int kCBlocks = kCB * kCB;
constexpr int kCPlaneInts = kCBlocks * 16;
constexpr int kCDC = 12;                         // chroma DC tile side
constexpr int kCLpInts = 36 * 4;                 // DC / low-pass of 6 x 6 macroblocks
constexpr int kSmem420Ints = kPlaneInts + kDcInts + kLpInts + 2 * (kCPlaneInts + kCDC * kCDC + kCLpInts) + 2 * 3 * kMbcInts;

// The 16 samples of the 4 x 4 cell whose upper-left quarter is the lower-right
// quarter of block b00 of a tile `stride` blocks wide; second-level overlap
// applied when the plane has it, and written back when `store` is set.
__device__ __forceinline__ bool cell_rw(int32_t *t, int b00, int stride, int overlap, int32_t (&w)[16], bool store,
                                        bool small = false) {
    const int b01 = b00 + 1, b10 = b00 + stride, b11 = b10 + 1;
    int2 *q[8] = {reinterpret_cast<int2 *>(&t[elem(b00, 2, 2)]), reinterpret_cast<int2 *>(&t[elem(b01, 2, 0)]),
                  reinterpret_cast<int2 *>(&t[elem(b00, 3, 2)]), reinterpret_cast<int2 *>(&t[elem(b01, 3, 0)]),
                  reinterpret_cast<int2 *>(&t[elem(b10, 0, 2)]), reinterpret_cast<int2 *>(&t[elem(b11, 0, 0)]),
                  reinterpret_cast<int2 *>(&t[elem(b10, 1, 2)]), reinterpret_cast<int2 *>(&t[elem(b11, 1, 0)])};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int2 a = *q[k];
        w[2 * k] = a.x;
        w[2 * k + 1] = a.y;
    }
    const bool bad = overlap < 1 ? false : small ? inverse_pot4x4<false>(w) : pot16(w);
    if (store) {
#pragma unroll
        for (int k = 0; k < 8; k++) *q[k] = make_int2(w[2 * k], w[2 * k + 1]);
    }
    return bad;
}

// A first-level chroma square of a 4:2:0 edge tile whose centre lies on the
// plane's edge (subsampled_overlap.rs:244-296): the two-sample operator on
// its column (vs) or row (hs) inside the plane; none on a plane corner.  On
// the top and bottom rows the plane's corner samples take their residual
// around the pair that holds their neighbour: corner minus neighbour before
// the pair's operator, plus after.  (wx, wy): the square in DC tile
// coordinates, ox: the plane column of the DC tile's origin.
__device__ bool chroma_edge_square(int32_t *cd, int wx, int wy, bool vs, bool hs, bool left, bool top, int ox,
                                   int Wdc) {
    using A = Ar<true>;
    auto at = [&](int x, int y) -> int32_t & { return cd[y * kCDC + x]; };
    bool bad = false;
    if (vs && !hs) {
        const int x = left ? wx + 1 : wx;
        bad |= inverse_pot2(at(x, wy), at(x, wy + 1));
    } else if (!vs && hs) {
        const int y = top ? wy + 1 : wy;
        const bool lc = ox + wx == 1, rc = ox + wx + 1 == Wdc - 2;
        if (lc) at(wx - 1, y) = A::sub(at(wx - 1, y), at(wx, y), bad);
        if (rc) at(wx + 2, y) = A::sub(at(wx + 2, y), at(wx + 1, y), bad);
        bad |= inverse_pot2(at(wx, y), at(wx + 1, y));
        if (lc) at(wx - 1, y) = A::add(at(wx - 1, y), at(wx, y), bad);
        if (rc) at(wx + 2, y) = A::add(at(wx + 2, y), at(wx + 1, y), bad);
    }
    return bad;
}

// A second-level chroma cell of a 4:2:0 edge tile that the plane's edge cuts,
// at chroma position (X, Y), in place: the four-sample operator down each
// column inside the plane, along each row, or on the corner quarter.  (ox, oy):
// the chroma position of the tile's sample origin; (Wc, Hc): the chroma plane.
__device__ bool chroma_cut_cell(int32_t *t, int X, int Y, int ox, int oy, int Wc, int Hc) {
    auto at = [&](int x, int y) -> int32_t & {
        const int sx = x - ox, sy = y - oy;
        return t[elem((sy >> 2) * kCB + (sx >> 2), sy & 3, sx & 3)];
    };
    const int c0 = max(X, 0), c1 = min(X + 4, Wc), r0 = max(Y, 0), r1 = min(Y + 4, Hc);
    const bool vs = c1 - c0 < 4, hs = r1 - r0 < 4;
    bool bad = false;
    if (vs && !hs) {
        for (int x = c0; x < c1; x++) bad |= inverse_pot4(at(x, Y), at(x, Y + 1), at(x, Y + 2), at(x, Y + 3));
    } else if (!vs && hs) {
        for (int y = r0; y < r1; y++) bad |= inverse_pot4(at(X, y), at(X + 1, y), at(X + 2, y), at(X + 3, y));
    } else {
        bad |= inverse_pot4(at(c0, r0), at(c0 + 1, r0), at(c0, r0 + 1), at(c0 + 1, r0 + 1));
    }
    return bad;
}

// Stage E at the plane's edge of a 4:2:0 tile: the pixels of the cut luma
// cells, one a thread; chroma interpolated with its reads clamped to the
// plane, as the general path does.  Returns the output flag.
__device__ bool edge_pixels_420(const ImageDev &im, const int32_t *ytile, const int32_t *ctile, int mx0, int my0,
                                const EdgeCells &ec) {
    const OutputDev &o = im.out;
    const uint64_t pixel_bytes = o.nchw ? (uint64_t)o.elem_bytes : (uint64_t)o.elem_bytes * o.channels;
    const uint64_t chs = o.nchw ? o.plane_stride : (uint64_t)o.elem_bytes;
    const int Wc = ec.W >> 1, Hc = ec.H >> 1, ox = 8 * mx0 - 8, oy = 8 * my0 - 8;
    const int cells = ec.n[0] + ec.n[1] + ec.n[2] + ec.n[3];
    bool bad = false;
    for (int item = threadIdx.x; item < cells * 8; item += kThreads) {
        int X, Y, c0, c1, r0, r1;
        edge_cell_at(ec, item >> 3, X, Y, c0, c1, r0, r1);
        const int w = c1 - c0, slot = item & 7;
        if (slot >= w * (r1 - r0)) continue;
        const int x = c0 + slot % w, y = r0 + slot / w;
        if (x < (int)o.crop_x || x >= (int)(o.crop_x + o.crop_w) || y < (int)o.crop_y ||
            y >= (int)(o.crop_y + o.crop_h))
            continue;
        const int sx = x - 16 * mx0, sy = y - 16 * my0;
        int32_t comp[4] = {ytile[elem((sy >> 2) * kIB + (sx >> 2), sy & 3, sx & 3)], 0, 0, 0};
        const int cx = x >> 1, cy = y >> 1;
#pragma unroll
        for (int pc = 0; pc < 2; pc++) {
            const int32_t *t = ctile + pc * kCPlaneInts;
            auto C = [&](int a, int b) {
                const int ta = min(max(a, 0), Wc - 1) - ox, tb = min(max(b, 0), Hc - 1) - oy;
                return t[elem((tb >> 2) * kCB + (ta >> 2), tb & 3, ta & 3)];
            };
            int32_t col[3];
#pragma unroll
            for (int d = -1; d <= 1; d++)
                col[d + 1] = (y & 1) ? up_odd(C(cx + d, cy), C(cx + d, cy + 1), im.centering_y)
                                     : up_even(C(cx + d, cy - 1), C(cx + d, cy), im.centering_y);
            comp[1 + pc] = (x & 1) ? up_odd(col[1], col[2], im.centering_x) : up_even(col[0], col[1], im.centering_x);
        }
        uint8_t *dst = o.base + (uint64_t)(y - o.crop_y) * o.row_stride + (uint64_t)(x - o.crop_x) * pixel_bytes;
        if (!fast_pixel<3>(im, comp, 0, dst, bad)) format_pixel(o, comp, 0, dst, chs, bad);
    }
    return bad;
}

// Edge tiles (MODE 1, or MODE 2 by position): tiles of a 4:2:0 image (at
// least 2 x 2 macroblocks) that touch the plane's edge and no hard tile
// boundary, as the full-resolution edge tiles, with the chroma planes'
// first-level squares and second-level cells on the plane's edge taking the
// edge operators (and corner residuals).
template <int MODE>
__device__ void interior_tile_420(const ImageDev &im, int tx, int ty, int32_t *smem, const uint4 *mbc, uint4 *mbc_next,
                                  uint32_t claimed, const ImageDev *__restrict__ images,
                                  const WorkItem *__restrict__ items, uint32_t item_count, TileShared &sh,
                                  uint32_t *status) {
    const int mx0 = tx * kTileMbs, my0 = ty * kTileMbs;
    const int tid = threadIdx.x;
    const bool edge = MODE == 1 || (MODE == 2 && (mx0 == 0 || my0 == 0 || mx0 + kTileMbs >= (int)im.plane[0].mbs_x ||
                                                  my0 + kTileMbs >= (int)im.plane[0].mbs_y));
    int32_t *ytile = smem;                              // luma: 17 x 17 blocks
    int32_t *ydc = ytile + kPlaneInts;                  // 24 x 24
    int32_t *ylp = ydc + kDcInts;                       // 36 x 16
    int32_t *ctile = ylp + kLpInts;                     // chroma: 2 x 11 x 11 blocks
    int32_t *cdc = ctile + 2 * kCPlaneInts;             // 2 x 12 x 12
    int32_t *clp = cdc + 2 * kCDC * kCDC;               // 2 x 36 x 4
    if (tid == 0) sh.bad = 0;
    int bad = 0;
    // phase 1: the DC / low-pass values (luma 16, chroma 4 a macroblock) of
    // the ring of luma macroblocks and of the 6 x 6 chroma macroblocks, then
    // the blocks.  Those of the tile's own luma macroblocks arrive with their
    // blocks (coefficient 0 of each) and are read from the slots.
    for (int k = tid; k < 320 + 2 * kCLpInts; k += kThreads) {
        int pi, m, kk;
        int32_t *dst;
        if (k < 320) { pi = 0; m = ring_mb(k >> 4); kk = k & 15; dst = ylp + m * 16 + kk; }
        else { const int q = k - 320; pi = 1 + q / kCLpInts; const int r = q - (pi - 1) * kCLpInts; m = r >> 2; kk = r & 3; dst = clp + q; }
        const uint4 e = mbc[pi * 36 + m];
        const int bands = (e.x >> 28) & 3;
        if (kk == 0 || bands != 0)
            cp_async4(dst, im.plane[pi].coeff + (e.x & 0x0fffffffu) + (bands >= 2 ? kk * 16 : kk));
        else
            *dst = 0;
    }
    {
        const int32_t *coeff = im.plane[0].coeff;
#pragma unroll
        for (int pass = 0; pass < 4; pass++) {
            const int mb = pass * 4 + (tid >> 6), c = tid & 63;
            const int a = mb & 3, b = mb >> 2, blk = c >> 2, r = c & 3;
            const int sidx = (4 * b + (blk >> 2)) * kIB + 4 * a + (blk & 3);
            copy_chunk(ytile + sidx * 16 + ((r ^ swz(sidx)) << 2), coeff, mbc[(b + 1) * 6 + a + 1], c * 4);
        }
        if (tid < 33 * 4) {
            const int hb = tid >> 2, r = tid & 3;
            const int i = hb < 16 ? 16 : hb < 32 ? hb - 16 : 16;
            const int j = hb < 16 ? hb : 16;
            const int sidx = j * kIB + i;
            copy_chunk(ytile + sidx * 16 + ((r ^ swz(sidx)) << 2), coeff, mbc[((j >> 2) + 1) * 6 + (i >> 2) + 1],
                       (((j & 3) << 2) + (i & 3)) * 16 + r * 4);
        }
    }
    for (int k = tid; k < 2 * kCBlocks * 4; k += kThreads) {
        const int pc = k / (kCBlocks * 4), q = k - pc * (kCBlocks * 4), sidx = q >> 2, r = q & 3;
        const int i = sidx % kCB, j = sidx / kCB;
        copy_chunk(ctile + pc * kCPlaneInts + sidx * 16 + ((r ^ swz(sidx)) << 2), im.plane[1 + pc].coeff,
                   mbc[(1 + pc) * 36 + (j >> 1) * 6 + (i >> 1)], (((j & 1) << 1) + (i & 1)) * 16 + r * 4);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    // stage A: first level of the 6 x 6 macroblocks of every plane
    for (int item = tid; item < 3 * 36; item += kThreads) {
        const int pi = item / 36, m = item - pi * 36;
        const PlaneDev &p = im.plane[pi];
        const uint4 e = mbc[item];
        bool b = false;
        if (pi == 0) {
            int32_t v[16];
            if (inner_mb(m)) {
                if (((e.x >> 28) & 3) >= 2) {
                    const int s0 = (4 * (m / 6) - 4) * kIB + 4 * (m % 6) - 4;
#pragma unroll
                    for (int k = 0; k < 16; k++) v[k] = ytile[elem(s0 + (k >> 2) * kIB + (k & 3), 0, 0)];
                } else {
                    low_pass_run(p.coeff, e, v);
                }
            } else {
                const int32_t *l = ylp + m * 16;
#pragma unroll
                for (int k = 0; k < 16; k += 4) {
                    const int4 q = *reinterpret_cast<const int4 *>(l + k);
                    v[k] = q.x; v[k + 1] = q.y; v[k + 2] = q.z; v[k + 3] = q.w;
                }
            }
            uint32_t lm = 0;   // one magnitude test, as in the full-resolution tile
#pragma unroll
            for (int k = 1; k < 16; k++) lm |= mag(v[k]);
            if ((uint64_t)(lm + 1) * e.z < (uint64_t)kTransformBound &&
                (uint64_t)(mag(v[0]) + 1) * e.y < (uint64_t)kTransformBound) {
                v[0] *= (int32_t)e.y;
#pragma unroll
                for (int k = 1; k < 16; k++) v[k] *= (int32_t)e.z;
                inverse_pct<false>(v);
            } else {
                v[0] = dequant(v[0], e.y, b);
#pragma unroll
                for (int k = 1; k < 16; k++) v[k] = dequant(v[k], e.z, b);
                b |= pct16(v);
            }
            if (p.scale2) {
#pragma unroll
                for (int k = 0; k < 16; k++) v[k] = dequant(v[k], 2, b);
            }
            int32_t *out = ydc + (m / 6) * 4 * kIDC + (m % 6) * 4;
#pragma unroll
            for (int r = 0; r < 4; r++)
                *reinterpret_cast<int4 *>(out + r * kIDC) = make_int4(v[r * 4], v[r * 4 + 1], v[r * 4 + 2], v[r * 4 + 3]);
        } else {
            const int4 q = *reinterpret_cast<const int4 *>(clp + (pi - 1) * kCLpInts + m * 4);
            int32_t w[4] = {dequant(q.x, e.y, b), dequant(q.y, e.z, b), dequant(q.z, e.z, b), dequant(q.w, e.z, b)};
            b |= inverse_chroma_420<true>(w);
#pragma unroll
            for (int k = 0; k < 4; k++) w[k] = p.scale2 ? dequant(w[k], 2, b) : w[k];
            int32_t *out = cdc + (pi - 1) * kCDC * kCDC + (m / 6) * 2 * kCDC + (m % 6) * 2;
            out[0] = w[0]; out[1] = w[1]; out[kCDC] = w[2]; out[kCDC + 1] = w[3];
        }
        if (b) bad |= kFlagFirst;
    }
    if (tid == 0) sh.next = claimed;
    __syncthreads();
    const uint32_t next = sh.next;
    if (next < item_count) {
        const WorkItem wn = items[next];
        load_entries<3, MODE != 0>(images[wn.image & kImageMask], wn.tx, wn.ty, mbc_next);
    }
    // stages B and C1 in one pass (disjoint data: the DC tiles; the first
    // rows and columns of the high-pass blocks); the overlap items go to
    // threads that get no second item.
    //   B: first-level overlap -- luma 5 x 5 windows at DC (2 + 4a, 2 + 4b),
    //      chroma 5 x 5 squares at DC (1 + 2a, 1 + 2b);
    //   C1: high-pass prediction.  Luma as in the full-resolution tile;
    //      chroma within each 2 x 2-block macroblock: from left, block column
    //      1 from column 0 of a block row; from top, block row 1 from row 0.
    constexpr int kItemsB = 3 * 25, kItemsC1 = 100 + 2 * 72;
    constexpr int kFirstB = (kItemsB + kItemsC1 < kThreads ? kItemsB + kItemsC1 : kThreads) - kItemsB;
    for (int k = tid; k < kItemsB + kItemsC1; k += kThreads) {
        if (k >= kFirstB && k < kFirstB + kItemsB) {
            const int item = k - kFirstB;
            const int pi = item / 25, c = item - pi * 25;
            if (im.plane[pi].overlap != 2) continue;
            bool b;
            if (edge) {
                // the window's or square's centre lies on macroblock boundary (mx0 + a, my0 + b)
                const PlaneDev &p = im.plane[pi];
                const int ca = mx0 + c % 5, cb = my0 + c / 5;
                if (ca > (int)p.mbs_x || cb > (int)p.mbs_y) continue;   // beyond the plane
                const bool vs = ca == 0 || ca == (int)p.mbs_x, hs = cb == 0 || cb == (int)p.mbs_y;
                if (vs || hs) {
                    if (pi == 0)
                        b = dc_edge_window(ydc, 2 + 4 * (c % 5), 2 + 4 * (c / 5), 4 * (mx0 - 1), 4 * (my0 - 1),
                                           4 * (int)p.mbs_x, 4 * (int)p.mbs_y, vs, hs);
                    else
                        b = chroma_edge_square(cdc + (pi - 1) * kCDC * kCDC, 1 + 2 * (c % 5), 1 + 2 * (c / 5), vs, hs,
                                               ca == 0, cb == 0, 2 * (mx0 - 1), 2 * (int)p.mbs_x);
                    if (b) bad |= kFlagOverlap;
                    continue;
                }
            }
            if (pi == 0) {
                int32_t *base = ydc + (2 + 4 * (c / 5)) * kIDC + 2 + 4 * (c % 5);
                int32_t v[16];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const int2 a = *reinterpret_cast<const int2 *>(base + r * kIDC);
                    const int2 d = *reinterpret_cast<const int2 *>(base + r * kIDC + 2);
                    v[r * 4] = a.x; v[r * 4 + 1] = a.y; v[r * 4 + 2] = d.x; v[r * 4 + 3] = d.y;
                }
                b = pot16(v);
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    *reinterpret_cast<int2 *>(base + r * kIDC) = make_int2(v[r * 4], v[r * 4 + 1]);
                    *reinterpret_cast<int2 *>(base + r * kIDC + 2) = make_int2(v[r * 4 + 2], v[r * 4 + 3]);
                }
            } else {
                int32_t *base = cdc + (pi - 1) * kCDC * kCDC + (1 + 2 * (c / 5)) * kCDC + 1 + 2 * (c % 5);
                b = inverse_pot2x2(base[0], base[1], base[kCDC], base[kCDC + 1]);
            }
            if (b) bad |= kFlagOverlap;
        } else {
            const int item = k < kFirstB ? k : k - kItemsB;
            using A = Ar<true>;
            bool ov = false;
            if (item < 100) {
                const int line = item & 3, m = item >> 2;
                const int a = m % 5, b = m / 5;
                const uint4 e = mbc[(b + 1) * 6 + a + 1];
                const int hp = (e.x >> 30) & 3, bands = (e.x >> 28) & 3;
                if (hp == 0 || bands < 2) continue;
                if (hp == 3) { bad |= kFlagInvalid; continue; }
                if (hp == 1) {
                    if (a == 4 || (b == 4 && line != 0)) continue;
                    const int j = 4 * b + line;
#pragma unroll
                    for (int c = 1; c < 4; c++) {
                        const int sidx = j * kIB + 4 * a + c;
#pragma unroll
                        for (int r = 1; r < 4; r++)
                            ytile[elem(sidx, r, 0)] = A::add(ytile[elem(sidx, r, 0)], ytile[elem(sidx - 1, r, 0)], ov);
                    }
                } else {
                    if (b == 4 || (a == 4 && line != 0)) continue;
                    const int i = 4 * a + line;
#pragma unroll
                    for (int r = 1; r < 4; r++) {
                        const int sidx = (4 * b + r) * kIB + i;
#pragma unroll
                        for (int c = 1; c < 4; c++)
                            ytile[elem(sidx, 0, c)] = A::add(ytile[elem(sidx, 0, c)], ytile[elem(sidx - kIB, 0, c)], ov);
                    }
                }
            } else {
                const int q = item - 100, pc = q / 72, rem = q - pc * 72, line = rem & 1, m = rem >> 1;
                const int a = m % 6, b = m / 6;
                const uint4 e = mbc[(1 + pc) * 36 + m];
                const int hp = (e.x >> 30) & 3, bands = (e.x >> 28) & 3;
                if (hp == 0 || bands < 2) continue;
                if (hp == 3) { bad |= kFlagInvalid; continue; }
                int32_t *t = ctile + pc * kCPlaneInts;
                if (hp == 1) {
                    // block row 2b + line: column 2a + 1 from column 2a
                    if (a == 5 || (b == 5 && line != 0)) continue;
                    const int sidx = (2 * b + line) * kCB + 2 * a + 1;
#pragma unroll
                    for (int r = 1; r < 4; r++) t[elem(sidx, r, 0)] = A::add(t[elem(sidx, r, 0)], t[elem(sidx - 1, r, 0)], ov);
                } else {
                    // block column 2a + line: row 2b + 1 from row 2b
                    if (b == 5 || (a == 5 && line != 0)) continue;
                    const int sidx = (2 * b + 1) * kCB + 2 * a + line;
#pragma unroll
                    for (int c = 1; c < 4; c++) t[elem(sidx, 0, c)] = A::add(t[elem(sidx, 0, c)], t[elem(sidx - kCB, 0, c)], ov);
                }
            }
            if (ov) bad |= kFlagPrediction;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // stage C2: block transforms -- luma 17 x 17, chroma blocks 1..10 x 1..10;
    // an edge tile's items are only its blocks inside the plane (divisions
    // as multiplies by ceil(2^16 / n), exact for these small quotients)
    int lcols = kIB, lrows = kIB, lmagic = 0, ccols = 10, crows = 10, cmagic = 0;
    if (edge) {
        const int rx = (int)im.plane[0].mbs_x - mx0, ry = (int)im.plane[0].mbs_y - my0;
        lcols = min(kIB, 4 * rx);
        lrows = min(kIB, 4 * ry);
        ccols = min(10, 2 * rx + 1);
        crows = min(10, 2 * ry + 1);
        lmagic = (65536 + lcols - 1) / lcols;
        cmagic = (65536 + ccols - 1) / ccols;
    }
    const int lcount = lcols * lrows, ccount = ccols * crows;
    bool small = true;   // every transform input of this thread's blocks below 2^16 (as in interior_tile)
    for (int item = tid; item < lcount + 2 * ccount; item += kThreads) {
        int32_t *blk;
        uint32_t step;
        int32_t dcv;
        int sw;
        if (item < lcount) {
            int i, j;
            if (edge) {
                j = (item * lmagic) >> 16;
                i = item - j * lcols;
            } else {
                i = item % kIB;
                j = item / kIB;
            }
            const int s = j * kIB + i;
            step = mbc[((j >> 2) + 1) * 6 + (i >> 2) + 1].w;
            blk = ytile + s * 16;
            sw = swz(s);
            dcv = ydc[(j + 4) * kIDC + i + 4];
        } else {
            const int q = item - lcount;
            int pc, i, j;
            if (edge) {
                pc = q >= ccount ? 1 : 0;
                const int rem = q - pc * ccount, r = (rem * cmagic) >> 16;
                i = 1 + rem - r * ccols;
                j = 1 + r;
            } else {
                pc = q / 100;
                const int rem = q - pc * 100;
                i = 1 + rem % 10;
                j = 1 + rem / 10;
            }
            const int sidx = j * kCB + i;
            step = mbc[(1 + pc) * 36 + (j >> 1) * 6 + (i >> 1)].w;
            blk = ctile + pc * kCPlaneInts + sidx * 16;
            sw = swz(sidx);
            dcv = cdc[pc * kCDC * kCDC + j * kCDC + i];
        }
        int32_t v[16];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int4 q = *reinterpret_cast<const int4 *>(blk + ((r ^ sw) << 2));
            v[r * 4 + 0] = q.x; v[r * 4 + 1] = q.y; v[r * 4 + 2] = q.z; v[r * 4 + 3] = q.w;
        }
        uint32_t m = 0;
#pragma unroll
        for (int k = 1; k < 16; k++) m |= mag(v[k]);
        v[0] = dcv;
        bool b = false;
        small &= (uint64_t)(m + 1) * step <= (1u << 16) && mag(v[0]) < (1u << 16);
        if ((uint64_t)(m + 1) * step < (uint64_t)kTransformBound && mag(v[0]) < (uint32_t)kTransformBound) {
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] = v[k] * (int32_t)step;
            inverse_pct<false>(v);
        } else {
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] = dequant(v[k], step, b);
            b |= pct16(v);
        }
        if (b) bad |= kFlagSecond;
#pragma unroll
        for (int r = 0; r < 4; r++)
            *reinterpret_cast<int4 *>(blk + ((r ^ sw) << 2)) = make_int4(v[r * 4], v[r * 4 + 1], v[r * 4 + 2], v[r * 4 + 3]);
    }
    // a small tile's overlap outputs stay below 2^27.8, and the chroma
    // interpolated from them below 2^28: no magnitude tests below
    const bool tile_small = __syncthreads_and(small) != 0;
    // stage D (chroma): the 9 x 9 second-level cells of each chroma plane, in place
    for (int item = tid; item < 2 * 81; item += kThreads) {
        const int pc = item / 81, c = item - pc * 81;
        int32_t *t = ctile + pc * kCPlaneInts;
        if (edge) {
            // cells past the chroma plane's edge, or cut by it
            const int Wc = 8 * (int)im.plane[1].mbs_x, Hc = 8 * (int)im.plane[1].mbs_y;
            const int X = 8 * mx0 - 2 + 4 * (c % 9), Y = 8 * my0 - 2 + 4 * (c / 9);
            if (X >= Wc || Y >= Hc) continue;
            if (X + 2 == 0 || X + 2 == Wc || Y + 2 == 0 || Y + 2 == Hc) {
                if (im.plane[1 + pc].overlap >= 1 && chroma_cut_cell(t, X, Y, 8 * mx0 - 8, 8 * my0 - 8, Wc, Hc))
                    bad |= kFlagOverlap;
                continue;
            }
        }
        int32_t w[16];
        if (cell_rw(t, (1 + c / 9) * kCB + 1 + c % 9, kCB, im.plane[1 + pc].overlap, w, true, tile_small))
            bad |= kFlagOverlap;
    }
    EdgeCells ec;
    bool grid_cell = true;
    int gcx = tid & 15, gcy = tid >> 4;   // the thread's cell of the 16 x 16 grid
    if (edge) {
        // stage D for the luma cells the plane's edge cuts, in place
        ec = edge_cells(im, mx0, my0);
        if (edge_overlap<1>(im, ytile, mx0, my0, ec)) bad |= kFlagOverlap;
        edge_grid(ec, mx0, my0, gcx, gcy, grid_cell);
    }
    __syncthreads();
    // stage E: each thread's luma cell, the chroma around it interpolated
    // (T.832 Table 180, vertical then horizontal), converted and stored
    if (grid_cell) {
        const int cx = gcx, cy = gcy;
        const OutputDev &o = im.out;
        const int x0 = 16 * mx0 + 2 + 4 * cx, y0 = 16 * my0 + 2 + 4 * cy;
        const bool inside = x0 >= (int)o.crop_x && x0 + 4 <= (int)(o.crop_x + o.crop_w) && y0 >= (int)o.crop_y &&
                            y0 + 4 <= (int)(o.crop_y + o.crop_h);
        bool obad = false, done = false;
        int32_t y[16];
        if (cell_rw(ytile, cy * kIB + cx, kIB, im.plane[0].overlap, y, false, tile_small)) bad |= kFlagOverlap;
        // chroma samples (tile coordinates) 8 + 2cx .. 11 + 2cx, 8 + 2cy .. 11 + 2cy
        if (tile_small && !edge && inside && o.kind == kOutRgb8 && !o.premultiply &&
            (o.channels == 3 || o.ch[3].padding)) {
            // RGB8 of an interior small tile, row by row: each luma row's
            // chroma from the two chroma rows it lies between, read afresh,
            // so that no cell holds both chroma planes' 4 x 4 neighbourhoods
            // (every sample is below 2^28: no tests, the one-division form)
            const ChannelScale &sc = o.ch[0];
            const int32_t add = sc.shifted_bias + sc.rounding;
            const int shift = sc.shift;
            const uint32_t order = sc.source == 2 ? 0x7014u : 0x7410u;
            const int cyc = im.centering_y, cxc = im.centering_x;
#pragma unroll
            for (int r = 0; r < 4; r++) {
                // luma row y0 + r takes chroma rows a and a + 1 of the
                // neighbourhood, as the 4 x 4 form below does
                const int a = (r + 1) >> 1;
                int32_t ch[2][4];
#pragma unroll
                for (int pc = 0; pc < 2; pc++) {
                    const int32_t *t = ctile + pc * kCPlaneInts;
                    int32_t sa[4], sb[4];
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int sx = 8 + 2 * cx + 2 * h, ya = 8 + 2 * cy + a, yb = ya + 1;
                        const int2 pa = *reinterpret_cast<const int2 *>(&t[elem((ya >> 2) * kCB + (sx >> 2), ya & 3, sx & 3)]);
                        const int2 pb = *reinterpret_cast<const int2 *>(&t[elem((yb >> 2) * kCB + (sx >> 2), yb & 3, sx & 3)]);
                        sa[2 * h] = pa.x; sa[2 * h + 1] = pa.y;
                        sb[2 * h] = pb.x; sb[2 * h + 1] = pb.y;
                    }
                    int32_t col[4];
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        col[k] = (r & 1) ? up_odd_small(sa[k], sb[k], cyc) : up_even_small(sa[k], sb[k], cyc);
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        ch[pc][c] = (c & 1) ? up_odd_small(col[1 + (c >> 1)], col[2 + (c >> 1)], cxc)
                                            : up_even_small(col[(c >> 1)], col[1 + (c >> 1)], cxc);
                }
                uint32_t px[4];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    int32_t R, G, B;
                    yuv_to_rgb_fast(y[r * 4 + c] + add, ch[0][c], ch[1][c], R, G, B);
                    px[c] = pack_rgb8(clamp_u8(R >> shift), clamp_u8(G >> shift), clamp_u8(B >> shift), order);
                }
                uint8_t *dst = o.base + (uint64_t)(y0 + r - o.crop_y) * o.row_stride + (uint64_t)(x0 - o.crop_x) * o.channels;
                if (o.channels == 4) store16(dst, px[0], px[1], px[2], px[3]);
                else store12(dst, px);
            }
            done = true;
        }
        int32_t u[16], v[16];
#pragma unroll
        for (int pc = 0; pc < 2 && !done; pc++) {
            const int32_t *t = ctile + pc * kCPlaneInts;
            int32_t s[4][4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int sy = 8 + 2 * cy + r;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int sx = 8 + 2 * cx + 2 * h;
                    const int2 a = *reinterpret_cast<const int2 *>(&t[elem((sy >> 2) * kCB + (sx >> 2), sy & 3, sx & 3)]);
                    s[r][2 * h] = a.x;
                    s[r][2 * h + 1] = a.y;
                }
            }
            int32_t *dst = pc == 0 ? u : v;
            // chroma samples below 2^28 take the one-division form: in an
            // interior small tile they all are (overlap outputs below
            // 2^27.8); elsewhere the 16 read are tested
            bool fast = tile_small && !edge;
            if (!fast) {
                uint32_t cm = 0;
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int k = 0; k < 4; k++) cm |= mag(s[r][k]);
                fast = cm < (1u << 28);
            }
            if (fast) {
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    int32_t col[4];
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        col[k] = (r & 1) ? up_odd_small(s[1 + (r >> 1)][k], s[2 + (r >> 1)][k], im.centering_y)
                                         : up_even_small(s[(r >> 1)][k], s[1 + (r >> 1)][k], im.centering_y);
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        dst[r * 4 + c] = (c & 1) ? up_odd_small(col[1 + (c >> 1)], col[2 + (c >> 1)], im.centering_x)
                                                 : up_even_small(col[(c >> 1)], col[1 + (c >> 1)], im.centering_x);
                }
            } else {
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    // luma row y0 + r: chroma row (y0 + r) >> 1 = tile row 9 + 2cy + (r >> 1)
                    int32_t col[4];
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        col[k] = (r & 1) ? up_odd(s[1 + (r >> 1)][k], s[2 + (r >> 1)][k], im.centering_y)
                                         : up_even(s[(r >> 1)][k], s[1 + (r >> 1)][k], im.centering_y);
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        dst[r * 4 + c] = (c & 1) ? up_odd(col[1 + (c >> 1)], col[2 + (c >> 1)], im.centering_x)
                                                 : up_even(col[(c >> 1)], col[1 + (c >> 1)], im.centering_x);
                }
            }
        }
        // RGB8 from YUV; a fourth byte can only be padding (no alpha plane)
        if (!done && inside && o.kind == kOutRgb8 && !o.premultiply && (o.channels == 3 || o.ch[3].padding)) {
            uint32_t m = 0;
            if (!tile_small) {
#pragma unroll
                for (int k = 0; k < 16; k++) m |= mag(y[k]) | mag(u[k]) | mag(v[k]);
            }
            if (m < (1u << 28)) {
                const ChannelScale &sc = o.ch[0];
                const int32_t add = sc.shifted_bias + sc.rounding;
                const int shift = sc.shift;
                // byte order of the packed pixel: R G B, or B G R
                const uint32_t order = sc.source == 2 ? 0x7014u : 0x7410u;
                uint32_t px[16];
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    // each colour is luma plus terms in u and v, so adding the
                    // output bias to luma adds it to all three (no
                    // intermediate nears int32 below 2^28)
                    int32_t R, G, B;
                    yuv_to_rgb_fast(y[k] + add, u[k], v[k], R, G, B);
                    px[k] = pack_rgb8(clamp_u8(R >> shift), clamp_u8(G >> shift), clamp_u8(B >> shift), order);
                }
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    uint8_t *dst = o.base + (uint64_t)(y0 + r - o.crop_y) * o.row_stride + (uint64_t)(x0 - o.crop_x) * o.channels;
                    if (o.channels == 4) store16(dst, px[4 * r], px[4 * r + 1], px[4 * r + 2], px[4 * r + 3]);
                    else store12(dst, &px[4 * r]);
                }
                done = true;
            }
        }
        if (!done) {
            const uint64_t pixel_bytes = o.nchw ? (uint64_t)o.elem_bytes : (uint64_t)o.elem_bytes * o.channels;
            const uint64_t chs = o.nchw ? o.plane_stride : (uint64_t)o.elem_bytes;
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) {
                    const int x = x0 + c, yy = y0 + r;
                    if (x < (int)o.crop_x || x >= (int)(o.crop_x + o.crop_w) || yy < (int)o.crop_y ||
                        yy >= (int)(o.crop_y + o.crop_h))
                        continue;
                    const int k = r * 4 + c;
                    const int32_t comp[4] = {y[k], u[k], v[k], 0};
                    uint8_t *dst = o.base + (uint64_t)(yy - o.crop_y) * o.row_stride + (uint64_t)(x - o.crop_x) * pixel_bytes;
                    format_pixel(o, comp, 0, dst, chs, obad);
                }
        }
        if (obad) bad |= kFlagOutput;
    }
    if (edge && edge_pixels_420(im, ytile, ctile, mx0, my0, ec)) bad |= kFlagOutput;
    if (bad) atomicOr(&sh.bad, bad);
    __syncthreads();
    if (tid == 0 && sh.bad) {
        const int b = sh.bad;
        const uint32_t code = (b & kFlagInvalid) ? kStatusInvalid
                            : (b & kFlagFirst) ? kStatusFirstTransform
                            : (b & kFlagOverlap) ? kStatusOverlap
                            : (b & kFlagPrediction) ? kStatusPrediction
                            : (b & kFlagSecond) ? kStatusSecondTransform
                            : kStatusOutput;
        atomicCAS(status, 0u, code);
    }
    __syncthreads();
}

// The descriptor of image `index` into shared memory, when the CTA's
// previous tile was of another image (`held`): the tile's stages read its
// fields from there rather than through L1.  Every thread takes the same
// branch (the work item is the CTA's); the tile before ended on a barrier.
__device__ __forceinline__ void hold_image(const ImageDev *__restrict__ images, uint32_t index, ImageDev &simg,
                                           uint32_t &held) {
    if (index == held) return;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(images + index);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&simg);
    for (int k = threadIdx.x; k < (int)(sizeof(ImageDev) / 4); k += kThreads) dst[k] = __ldg(src + k);
    held = index;
    __syncthreads();
}

// Tiles of YUV 4:2:0 images: interior (MODE 0), edge (MODE 1) or both (MODE 2).
template <int MODE>
__global__ void __launch_bounds__(kThreads, 3)
jxrb_interior420_tiles(const ImageDev *__restrict__ images, const WorkItem *__restrict__ items, uint32_t item_count,
                       uint32_t *status, uint32_t *counters) {
    extern __shared__ __align__(16) int32_t smem_420[];
    __shared__ TileShared sh;
    uint4 *mbc[2];
    mbc[0] = reinterpret_cast<uint4 *>(smem_420 + kSmem420Ints - 2 * 3 * kMbcInts);
    mbc[1] = mbc[0] + 3 * 36;
    uint32_t i;
    if (claim(counters, item_count, i)) {
        {
            const WorkItem w = items[i];
            load_entries<3, MODE != 0>(images[w.image & kImageMask], w.tx, w.ty, mbc[0]);
            cp_async_wait_all();
            __syncthreads();
        }
        __shared__ ImageDev simg;
        uint32_t held = 0xffffffffu;
        for (int buf = 0;; buf ^= 1) {
            const uint32_t claimed = threadIdx.x == 0 ? atomicAdd(&counters[0], 1u) : 0u;
            const WorkItem cur = items[i];
            hold_image(images, cur.image & kImageMask, simg, held);
            interior_tile_420<MODE>(simg, cur.tx, cur.ty, smem_420, mbc[buf], mbc[buf ^ 1],
                                    claimed, images, items, item_count, sh, status);
            i = sh.next;
            __syncthreads();
            if (i >= item_count) break;
        }
    }
    retire(counters);
}

// CTAs an SM the NP-plane interior kernel is compiled for.  Shared memory
// (about 24 KB a plane) admits two four-plane tiles, so their kernel takes the
// registers of two (no spills); fewer planes run three (at 64 registers, for
// four, the one- and two-plane kernels spill).
template <int NP> constexpr int interior_ctas() { return NP == 4 ? 2 : 3; }

// Tiles of images with NP full-resolution planes: interior tiles (MODE 0),
// edge tiles (MODE 1) or both, each by its position (MODE 2).
template <int NP, int MODE>
__global__ void __launch_bounds__(kThreads, interior_ctas<NP>())
jxrb_interior_tiles(const ImageDev *__restrict__ images, const WorkItem *__restrict__ items, uint32_t item_count,
                    uint32_t *status, uint32_t *counters) {
    extern __shared__ __align__(16) int32_t smem_interior[];
    __shared__ TileShared sh;
    uint4 *mbc[2];
    mbc[0] = reinterpret_cast<uint4 *>(smem_interior + NP * (kPlaneInts + kDcInts + lp_ints<NP>()));
    mbc[1] = mbc[0] + NP * 36;
    uint32_t i;
    if (claim(counters, item_count, i)) {
        const WorkItem w = items[i];
        load_entries<NP, MODE != 0>(images[w.image & kImageMask], w.tx, w.ty, mbc[0]);
        cp_async_wait_all();
        __syncthreads();
        __shared__ ImageDev simg;
        uint32_t held = 0xffffffffu;
        for (int buf = 0;; buf ^= 1) {
            // the item after this one, claimed now and used halfway through the tile
            const uint32_t claimed = threadIdx.x == 0 ? atomicAdd(&counters[0], 1u) : 0u;
            const WorkItem cur = items[i];
            hold_image(images, cur.image & kImageMask, simg, held);
            interior_tile<NP, MODE>(simg, cur.tx, cur.ty, smem_interior, mbc[buf],
                                    mbc[buf ^ 1], claimed, images, items, item_count, sh, status);
            i = sh.next;
            __syncthreads();
            if (i >= item_count) break;
        }
    }
    retire(counters);
}

}  // namespace jxr

// ---------------------------------------------------------------------------
// host launch helpers
// ---------------------------------------------------------------------------
namespace jxr {

size_t tile_smem_bytes(int planes) {
    return (size_t)planes * (kPlaneInts + kDcInts + kLpInts + kMbcInts) * sizeof(int32_t);
}

// Interior tiles keep padded low-pass slots and a second set of macroblock
// entries (the next tile's).
static size_t interior_smem_bytes(int planes) {
    const int lp = planes == 3 ? lp_ints<3>() : lp_ints<1>();
    return (size_t)planes * (kPlaneInts + kDcInts + lp + 2 * kMbcInts) * sizeof(int32_t);
}

typedef void (*TileKernel)(const ImageDev *, const WorkItem *, uint32_t, uint32_t *, uint32_t *);

// The interior segment's kernel of NP-plane images: with their edge tiles
// folded in (kFoldEdges) or interior tiles only.
template <int NP>
static TileKernel interior_kernel() {
    if constexpr (kFoldEdges[NP - 1]) return jxrb_interior_tiles<NP, 2>;
    else return jxrb_interior_tiles<NP, 0>;
}

static TileKernel segment_kernel(int segment) {
    switch (segment) {
    case 0: return interior_kernel<1>();
    case 1: return interior_kernel<2>();
    case 2: return interior_kernel<3>();
    case 3: return interior_kernel<4>();
    case 4: return kFoldEdges[4] ? jxrb_interior420_tiles<2> : jxrb_interior420_tiles<0>;
    case 5: return jxrb_interior_tiles<1, 1>;
    case 6: return jxrb_interior_tiles<2, 1>;
    case 7: return jxrb_interior_tiles<3, 1>;
    case 8: return jxrb_interior_tiles<4, 1>;
    case 9: return jxrb_interior420_tiles<1>;
    default: return jxrb_reconstruct_tiles;
    }
}

// Planes of a segment's tiles (the general kernel: the set's most).
static int segment_planes(int segment, int max_planes) {
    if (segment < 4) return segment + 1;
    if (segment == 4 || segment == 9) return 3;
    if (segment < kSegmentOther) return segment - 4;
    return max_planes;
}

static size_t segment_smem_bytes(int segment, int max_planes) {
    if (segment == 4 || segment == 9) return (size_t)kSmem420Ints * sizeof(int32_t);
    if (segment < kSegmentOther) return interior_smem_bytes(segment_planes(segment, max_planes));
    return tile_smem_bytes(max_planes);
}

// Launch the work list's segments (interior tiles with one to four
// full-resolution planes, interior tiles of 4:2:0 images, every other tile).
// `bounds` holds the kSegments + 1 segment boundaries; `counters` two words a
// segment.
// What the launcher learns about a device once: its SM count, which segment
// kernels have their dynamic shared-memory limit raised on it (a function
// attribute holds per device), and how many CTAs of each segment kernel fit
// an SM at each plane count.  Guarded by a lock: sessions on several threads
// and devices launch concurrently.
struct DeviceLaunchState {
    int sms = 0;
    bool configured[kSegments] = {};
    int fit[kSegments][JXRB_MAX_PLANES + 1] = {};
};
constexpr int kMaxLaunchDevices = 64;
static DeviceLaunchState g_launch_state[kMaxLaunchDevices];
static std::mutex g_launch_lock;

// SM count and CTAs per SM of segment `seg` at `planes` planes on the current
// device, raising the kernel's shared-memory limit there first.
static cudaError_t segment_fit(int seg, int planes, size_t smem, int &sms, int &fit) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxLaunchDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> guard(g_launch_lock);
    DeviceLaunchState &d = g_launch_state[dev];
    if (d.sms == 0) {
        e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    TileKernel k = segment_kernel(seg);
    if (!d.configured[seg]) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem_bytes(JXRB_MAX_PLANES));
        if (e != cudaSuccess) return e;
        d.configured[seg] = true;
    }
    int &f = d.fit[seg][planes];
    if (f == 0 && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&f, k, kThreads, smem) != cudaSuccess || f < 1)) {
        cudaGetLastError();
        f = 1;
    }
    sms = d.sms;
    fit = f;
    return cudaSuccess;
}

cudaError_t launch_tiles(const ImageDev *images, const void *items, const uint32_t *bounds, int max_planes,
                         uint32_t *status, uint32_t *counters, cudaStream_t stream, cudaStream_t side,
                         cudaEvent_t fork, cudaEvent_t join, const LaunchTuning *tune) {
    const WorkItem *list = static_cast<const WorkItem *>(items);
    // The edge and other tiles (segments kSideSegment0 ..) run beside the
    // interior kernels on `side`, forked from and joined back to `stream`, so
    // their short, latency-bound launches hide under the long ones.
    const bool both = bounds[kSegments] > bounds[kSideSegment0] && bounds[kSideSegment0] > bounds[0] &&
                      side != nullptr && (tune == nullptr || tune->side_stream);
    if (both) {
        cudaError_t e = cudaEventRecord(fork, stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(side, fork, 0);
        if (e != cudaSuccess) return e;
    }
    for (int seg0 = 0; seg0 < kSegments; seg0++) {
        // the side stream's kernels first, so that they start with the others
        const int seg = seg0 == 0 ? kSegmentOther : seg0 <= kSegmentOther - kSideSegment0 ? kSideSegment0 + seg0 - 1
                                                                                          : seg0 - (kSegmentOther - kSideSegment0) - 1;
        cudaStream_t st = (both && seg >= kSideSegment0) ? side : stream;
        const uint32_t count = bounds[seg + 1] - bounds[seg];
        if (count == 0) continue;
        TileKernel k = segment_kernel(seg);
        const int planes = segment_planes(seg, max_planes);
        const size_t smem = segment_smem_bytes(seg, max_planes);
        int sms = 0, fit = 0;
        cudaError_t fe = segment_fit(seg, planes, smem, sms, fit);
        if (fe != cudaSuccess) return fe;
        int per_sm = fit;
        const int slot = seg == kSegmentOther ? 4 : planes - 1;   // entry of the launch tuning
        if (tune && tune->blocks_per_sm[slot] > 0 && (int)tune->blocks_per_sm[slot] < fit)
            per_sm = (int)tune->blocks_per_sm[slot];
        const long full = (long)sms * per_sm;
        const int blocks = (int)((long)count < full ? (long)count : full);
        k<<<blocks, kThreads, smem, st>>>(images, list + bounds[seg], count, status, counters + 2 * seg);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (both) {
        cudaError_t e = cudaEventRecord(join, side);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, join, 0);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int tile_mbs() { return kTileMbs; }

// ---------------------------------------------------------------------------
// reduced resolution: one sample a block (a quarter, reconstruct_quarter,
// crates/jxr-native/src/reconstruct/pipeline.rs:175-222) or a macroblock (a
// sixteenth, reconstruct_sixteenth, 223-260).  The pictures are at most a
// sixteenth of the full-resolution sample count, so each stage is its own
// small kernel over pictures in global memory; blockIdx.y selects the plane
// (or the request, for the output).
// ---------------------------------------------------------------------------

// The first level of every macroblock of the plane: dequantized DC and
// low-pass values through the first-level inverse transform, doubled where
// the plane is scaled, one value a block (block_dc_plane, pipeline.rs:459-541).
// A sixteenth leaves the low-pass values out (LowBands::Dc); without
// two-level overlap it stops at the macroblock's DC, doubled where scaled,
// written straight into the macroblock picture (macroblock_dc_plane, 387-409).
__global__ void __launch_bounds__(256) jxrb_quarter_first_level(const QuarterPlane *__restrict__ planes,
                                                                uint32_t *status) {
    const QuarterPlane &p = planes[blockIdx.y];
    const uint32_t n = p.mbs_x * p.mbs_y;
    const int count = p.bc * p.br;
    const size_t pw = (size_t)p.mbs_x * p.bc;
    const bool dc_only = p.sixteenth != 0;
    bool bad = false;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        const uint32_t mx = m % p.mbs_x, my = m / p.mbs_x;
        const uint4 e = __ldg(&p.mbs[(size_t)my * p.mbs_stride + mx]);
        const int bands = (e.x >> 28) & 3;
        const int32_t *c = p.coeff + (e.x & 0x0fffffffu);
        const int stride = bands >= 2 ? 16 : 1;
        int32_t v[16];
        v[0] = dequant(__ldg(c), e.y, bad);
        if (dc_only && p.overlap != 2) {
            p.out[m] = p.scale2 ? dequant(v[0], 2, bad) : v[0];
            continue;
        }
#pragma unroll
        for (int k = 1; k < 16; k++)
            v[k] = (k < count && bands != 0 && !dc_only) ? dequant(__ldg(c + k * stride), e.z, bad) : 0;
        int32_t *out = p.pic + (size_t)my * p.br * pw + (size_t)mx * p.bc;
        if (count == 16) {
            bad |= pct16(v);
#pragma unroll
            for (int k = 0; k < 16; k++) v[k] = p.scale2 ? dequant(v[k], 2, bad) : v[k];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int cc = 0; cc < 4; cc++) out[r * pw + cc] = v[r * 4 + cc];
        } else if (count == 4) {
            int32_t w[4] = {v[0], v[1], v[2], v[3]};
            bad |= inverse_chroma_420<true>(w);
#pragma unroll
            for (int k = 0; k < 4; k++) w[k] = p.scale2 ? dequant(w[k], 2, bad) : w[k];
            out[0] = w[0]; out[1] = w[1]; out[pw] = w[2]; out[pw + 1] = w[3];
        } else {
            int32_t w[8] = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
            bad |= inverse_chroma_422<true>(w);
#pragma unroll
            for (int k = 0; k < 8; k++) w[k] = p.scale2 ? dequant(w[k], 2, bad) : w[k];
#pragma unroll
            for (int r = 0; r < 4; r++) { out[r * pw] = w[2 * r]; out[r * pw + 1] = w[2 * r + 1]; }
        }
    }
    if (bad) atomicCAS(status, 0u, (uint32_t)kStatusFirstTransform);
}

// The first-level overlap filter over a two-level plane's picture, one cell a
// thread.  Full resolution: 4x4 cells at origins 2 (mod 4), disjoint, one
// pass (phase 0).  Subsampled chroma: 2x2 cells at odd origins in three
// ordered phases (corners lose their neighbour, squares and pairs, corners
// regain it), the schedule of crates/jxr-native/src/reconstruct/subsampled_overlap.rs:244-296.
__global__ void __launch_bounds__(256) jxrb_quarter_overlap(const QuarterPlane *__restrict__ planes, int phase,
                                                            uint32_t *status) {
    const QuarterPlane &p = planes[blockIdx.y];
    if (p.overlap != 2) return;
    const int W = (int)p.mbs_x * p.bc, H = (int)p.mbs_y * p.br;
    const int lx = log2_of(p.bc), ly = log2_of(p.br);
    int32_t *pic = p.pic;
    auto at = [&](int x, int y) -> int32_t & { return pic[(size_t)y * W + x]; };
    auto inside = [&](int x, int y) { return x >= 0 && x < W && y >= 0 && y < H; };
    auto vb = [&](int x) { return boundary_at(x, W, lx, p.hard, p.col_start); };
    auto hb = [&](int y) { return boundary_at(y, H, ly, p.hard, p.row_start); };
    bool bad = false;
    if (p.bc == 4) {
        if (phase != 0) return;
        const int ncx = W / 4 + 1, ncy = H / 4 + 1;
        for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < ncx * ncy; item += gridDim.x * blockDim.x) {
            const int cx = -2 + 4 * (item % ncx), cy = -2 + 4 * (item / ncx);
            const bool vs = vb(cx + 2), hs = hb(cy + 2);
            if (!vs && !hs) {
                int32_t v[16];
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) v[r * 4 + c] = at(cx + c, cy + r);
                bad |= pot16(v);
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) at(cx + c, cy + r) = v[r * 4 + c];
            } else if (vs && !hs) {
                for (int c = 0; c < 4; c++)
                    if (cx + c >= 0 && cx + c < W)
                        bad |= inverse_pot4(at(cx + c, cy), at(cx + c, cy + 1), at(cx + c, cy + 2), at(cx + c, cy + 3));
            } else if (!vs && hs) {
                for (int r = 0; r < 4; r++)
                    if (cy + r >= 0 && cy + r < H)
                        bad |= inverse_pot4(at(cx, cy + r), at(cx + 1, cy + r), at(cx + 2, cy + r), at(cx + 3, cy + r));
            } else {
                for (int k = 0; k < 4; k++) {
                    const int x = cx + (k & 1) * 2, y = cy + (k >> 1) * 2;
                    if (inside(x, y)) bad |= inverse_pot4(at(x, y), at(x + 1, y), at(x, y + 1), at(x + 1, y + 1));
                }
            }
        }
    } else {
        using A = Ar<true>;
        const int ncx = W / 2 + 1, ncy = H / 2 + 1;
        for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < ncx * ncy; item += gridDim.x * blockDim.x) {
            const int cx = -1 + 2 * (item % ncx), cy = -1 + 2 * (item / ncx);
            if (phase == 1) {
                const bool vs = vb(cx + 1), hs = hb(cy + 1);
                if (!vs && !hs) {
                    if (inside(cx, cy) && inside(cx + 1, cy + 1))
                        bad |= inverse_pot2x2(at(cx, cy), at(cx + 1, cy), at(cx, cy + 1), at(cx + 1, cy + 1));
                } else if (vs && !hs) {
                    for (int c = 0; c < 2; c++)
                        if (inside(cx + c, cy) && inside(cx + c, cy + 1)) bad |= inverse_pot2(at(cx + c, cy), at(cx + c, cy + 1));
                } else if (!vs && hs) {
                    for (int r = 0; r < 2; r++)
                        if (inside(cx, cy + r) && inside(cx + 1, cy + r)) bad |= inverse_pot2(at(cx, cy + r), at(cx + 1, cy + r));
                }
                continue;
            }
            if (!hb(cy + 1)) continue;   // no boundary row in this cell
            for (int k = 0; k < 4; k++) {
                const int x = cx + (k & 1), y = cy + (k >> 1);
                if (!inside(x, y)) continue;
                const bool left_corner = vb(x), right_corner = vb(x + 1);
                if (left_corner == right_corner) continue;   // not a corner
                if (right_corner && vb(x - 1)) continue;     // right corner of a two-wide region: with its partner
                if (left_corner && vb(x + 2)) {              // two-wide region: every step of the row here
                    if (phase != 0 || !inside(x + 1, y)) continue;
                    int32_t &c0 = at(x, y), &c1 = at(x + 1, y);
                    c0 = A::sub(c0, c1, bad);
                    c1 = A::sub(c1, c0, bad);
                    c0 = A::add(c0, c1, bad);
                    c1 = A::add(c1, c0, bad);
                    continue;
                }
                const int n = left_corner ? x + 1 : x - 1;
                if (!inside(n, y)) continue;
                at(x, y) = phase == 0 ? A::sub(at(x, y), at(n, y), bad) : A::add(at(x, y), at(n, y), bad);
            }
        }
    }
    if (bad) atomicCAS(status, 0u, (uint32_t)kStatusOverlap);
}

// A sixteenth of a two-level plane: each macroblock's filtered block values
// summed, row by row, checked, into the macroblock picture (sum_macroblocks,
// pipeline.rs:421-457).
__global__ void __launch_bounds__(256) jxrb_sixteenth_sum(const QuarterPlane *__restrict__ planes, uint32_t *status) {
    const QuarterPlane &p = planes[blockIdx.y];
    if (!p.sixteenth || p.overlap != 2) return;
    const uint32_t n = p.mbs_x * p.mbs_y;
    const size_t pw = (size_t)p.mbs_x * p.bc;
    bool bad = false;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        const uint32_t mx = m % p.mbs_x, my = m / p.mbs_x;
        const int32_t *b = p.pic + (size_t)my * p.br * pw + (size_t)mx * p.bc;
        int32_t sum = 0;
        for (int r = 0; r < p.br; r++)
            for (int c = 0; c < p.bc; c++) sum = Ar<true>::add(sum, b[r * pw + c], bad);
        p.out[m] = sum;
    }
    if (bad) atomicCAS(status, 0u, (uint32_t)kStatusSecondTransform);
}

// Each sample scaled to the level it stands for: a shift without overlap
// filtering, else the flat terms of the probe sample placed like it
// (SampleScale::apply and FlatTerms::level, sample_scale.rs:250-350).
__global__ void __launch_bounds__(256) jxrb_quarter_scale(const QuarterPlane *__restrict__ planes, uint32_t *status) {
    const QuarterPlane &p = planes[blockIdx.y];
    const uint32_t W = p.sixteenth ? p.mbs_x : p.mbs_x * p.bc;
    const uint32_t n = W * (p.sixteenth ? p.mbs_y : p.mbs_y * p.br);
    bool bad = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t v = p.out[i];
        if (p.shift >= 0) {
            p.out[i] = v >> p.shift;
            continue;
        }
        if (v == 0) continue;
        const uint32_t t = __ldg(&p.rows[i / W]) * p.probe_stride + __ldg(&p.cols[i % W]);
        const int64_t d = __ldg(&p.divisor[t]);
        const int64_t num = (int64_t)v * p.gain - __ldg(&p.bias[t]);
        int64_t q = num / d;
        if (num % d < 0) q -= 1;   // Euclidean division by a positive divisor
        bad |= q < INT32_MIN || q > INT32_MAX;
        p.out[i] = (int32_t)q;
    }
    if (bad) atomicCAS(status, 0u, (uint32_t)kStatusSecondTransform);
}

// A picture in global memory, read like a tile's plane view.
struct GlobalView {
    const int32_t *p;
    int w, h;
    __device__ __forceinline__ int32_t at(int x, int y) const { return p[(size_t)y * w + x]; }
    __device__ __forceinline__ int32_t clamped(int x, int y) const {
        return at(min(max(x, 0), w - 1), min(max(y, 0), h - 1));
    }
};

// Chroma upsampling, colour conversion, scaling and packing of the scaled
// pictures: the full-resolution output path over bands of eight rows.
__global__ void __launch_bounds__(256) jxrb_quarter_output(const ImageDev *__restrict__ images,
                                                           const QuarterImage *__restrict__ quarters,
                                                           const QuarterPlane *__restrict__ planes, uint32_t *status) {
    const QuarterImage q = quarters[blockIdx.y];
    const ImageDev &im = images[q.image];
    GlobalView views[JXRB_MAX_PLANES];
    for (uint32_t k = 0; k < q.planes && k < JXRB_MAX_PLANES; k++) {
        const QuarterPlane &p = planes[q.first_plane + k];
        views[k] = p.sixteenth ? GlobalView{p.out, (int)p.mbs_x, (int)p.mbs_y}
                               : GlobalView{p.out, (int)(p.mbs_x * p.bc), (int)(p.mbs_y * p.br)};
    }
    bool bad = false;
    const int bands = ((int)q.height + 7) / 8;
    for (int b = blockIdx.x; b < bands; b += gridDim.x)
        output_generic(im, views, 0, (int)q.width, b * 8, min((int)q.height, b * 8 + 8), bad);
    if (bad) atomicCAS(status, 0u, (uint32_t)kStatusOutput);
}

// The reduced-resolution stages of a set: `planes` planes of `count`
// requests, the largest plane holding `max_mbs` macroblocks and `max_samples`
// picture samples, the tallest request `max_rows` rows; `sixteenth_sums`: a
// sixteenth of a two-level plane is among them.
cudaError_t launch_quarter(const ImageDev *images, const QuarterImage *quarters, uint32_t count,
                           const QuarterPlane *planes, uint32_t plane_count, bool two_level, bool sixteenth_sums,
                           uint32_t max_mbs, uint32_t max_samples, uint32_t max_rows, uint32_t *status,
                           cudaStream_t stream) {
    if (count == 0 || plane_count == 0) return cudaSuccess;
    auto blocks = [](uint64_t work) { return (unsigned)std::min<uint64_t>(std::max<uint64_t>((work + 255) / 256, 1), 1024); };
    // blockIdx.y selects a plane or request: at most 65535 of them a launch
    for (uint32_t base = 0; base < plane_count; base += 65535) {
        const unsigned n = (unsigned)std::min<uint32_t>(plane_count - base, 65535);
        jxrb_quarter_first_level<<<dim3(blocks(max_mbs), n), 256, 0, stream>>>(planes + base, status);
        if (two_level)
            for (int phase = 0; phase < 3; phase++)
                jxrb_quarter_overlap<<<dim3(blocks(max_samples / 4 + 64), n), 256, 0, stream>>>(planes + base, phase,
                                                                                                status);
        if (sixteenth_sums) jxrb_sixteenth_sum<<<dim3(blocks(max_mbs), n), 256, 0, stream>>>(planes + base, status);
        jxrb_quarter_scale<<<dim3(blocks(max_samples), n), 256, 0, stream>>>(planes + base, status);
    }
    for (uint32_t base = 0; base < count; base += 65535) {
        const unsigned n = (unsigned)std::min<uint32_t>(count - base, 65535);
        jxrb_quarter_output<<<dim3(std::max(1u, std::min((max_rows + 7) / 8, 256u)), n), 256, 0, stream>>>(
            images, quarters + base, planes, status);
    }
    return cudaGetLastError();
}

}  // namespace jxr
