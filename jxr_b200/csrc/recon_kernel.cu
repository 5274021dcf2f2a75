// recon_kernel.cu -- fused JPEG XR reconstruction for sm_100a.
//
// One CTA reconstructs one output tile of an image, every plane, in a single
// pass: dequantization and the first-level inverse transform of each
// macroblock, the first-level overlap filter on the block-DC plane, high-pass
// prediction, dequantization and the second-level inverse transform of each
// block, the second-level overlap filter on the samples, and finally chroma
// upsampling, colour conversion, scaling and packing into the output surface.
// Intermediates live in shared memory only: HBM sees the arena once and the
// output once, plus the halo the tile shares with its neighbours (served from
// L2).
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
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine.h"
#include "lifting.cuh"

namespace jxr {

constexpr int kThreads = 256;
constexpr int kTileMbs = 4;                       // macroblocks across / down a CTA tile
constexpr int kTileSamples = (kTileMbs * 4 + 4) * 4;  // 68: sample tile side (full resolution)
constexpr int kTileInts = kTileSamples * kTileSamples;
constexpr int kDcInts = 32 * 32;

struct PlaneGeom {
    int W, H;            // sample plane
    int Wdc, Hdc;        // block-DC plane
    int bx0, bx1, by0, by1;      // blocks reconstructed (inclusive)
    int cx0, cx1, cy0, cy1;      // overlap cells (inclusive, step 4); empty if cx1 < cx0
    int mx0, mx1, my0, my1;      // macroblocks whose first level runs (inclusive)
    int sw;                      // sample tile stride
    int dw;                      // DC tile stride
    int ox0, ox1, oy0, oy1;      // subsampled first-level cells (odd origins, inclusive)
};

__device__ __forceinline__ int cell_of(int p) { return ((p + 2) & ~3) - 2; }
__device__ __forceinline__ int odd_cell_of(int p) { return p - 1 + (p & 1); }

// Whether a region boundary lies at plane position p (a multiple of the
// plane's macroblock extent `scale` along the axis).
__device__ __forceinline__ bool boundary_at(int p, int extent, int scale, int hard, const uint8_t *starts) {
    if (p <= 0 || p >= extent) return true;
    if (!hard || (p % scale) != 0) return false;
    return starts[p / scale] != 0;
}

__device__ __forceinline__ void fail(uint32_t *status, uint32_t code) { atomicCAS(status, 0u, code); }

// ---------------------------------------------------------------------------
// geometry of one plane for the CTA's output region [X0, X1) x [Y0, Y1)
// (full-resolution sample coordinates)
// ---------------------------------------------------------------------------
__device__ PlaneGeom plane_geometry(const PlaneDev &p, int chroma_plane, int chroma, int X0, int X1, int Y0, int Y1) {
    PlaneGeom g;
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
    g.sw = (g.bx1 - g.bx0 + 1) * 4;
    g.dw = (g.mx1 - g.mx0 + 1) * p.bc;
    return g;
}

// ---------------------------------------------------------------------------
// stage A: dequantize + first-level inverse transform of each macroblock
// (crates/jxr-native/src/reconstruct/pipeline.rs:605-680)
// ---------------------------------------------------------------------------
__device__ void stage_first_level(const PlaneDev &p, const PlaneGeom &g, int32_t *dc, bool &bad) {
    const int nmx = g.mx1 - g.mx0 + 1, nmy = g.my1 - g.my0 + 1;
    const int count = p.bc * p.br;
    for (int i = threadIdx.x; i < nmx * nmy; i += blockDim.x) {
        const int mx = g.mx0 + i % nmx, my = g.my0 + i / nmx;
        const uint4 e = p.mbs[(size_t)my * p.mbs_x + mx];
        const uint32_t off = e.x & 0x0fffffffu;
        const int bands = (e.x >> 28) & 3;
        const int32_t *c = p.coeff + off;
        int32_t v[16];
        bool b = false;
        v[0] = dequant(__ldg(c), e.y, b);
#pragma unroll
        for (int k = 1; k < 16; k++) {
            int32_t q = 0;
            if (k < count && bands != 0) q = __ldg(c + (bands >= 2 ? k * 16 : k));
            v[k] = k < count ? dequant(q, e.z, b) : 0;
        }
        if (count == 16) {
            b |= pct16(v);
        } else if (count == 4) {
            int32_t w[4] = {v[0], v[1], v[2], v[3]};
            b |= inverse_chroma_420<true>(w);
            v[0] = w[0]; v[1] = w[1]; v[2] = w[2]; v[3] = w[3];
        } else {
            int32_t w[8] = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
            b |= inverse_chroma_422<true>(w);
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] = w[k];
        }
        if (p.scale2) {
#pragma unroll
            for (int k = 0; k < 16; k++) {
                if (k < count) {
                    int64_t w = (int64_t)v[k] * 2;
                    b |= w != (int64_t)(int32_t)w;
                    v[k] = (int32_t)w;
                }
            }
        }
        const int lx = (mx - g.mx0) * p.bc, ly = (my - g.my0) * p.br;
        for (int r = 0; r < p.br; r++)
            for (int cc = 0; cc < p.bc; cc++) dc[(ly + r) * g.dw + lx + cc] = v[r * p.bc + cc];
        bad |= b;
    }
}

// ---------------------------------------------------------------------------
// stage B / D: full-resolution overlap cells over a tile whose element (0,0)
// is plane position (ox, oy).  `scale_x` / `scale_y` are the plane's
// macroblock extents in this plane's units.
// ---------------------------------------------------------------------------
__device__ void overlap_cells(int32_t *t, int stride, int ox, int oy, int W, int H, int cx0, int cx1, int cy0, int cy1,
                              int scale_x, int scale_y, const PlaneDev &p, bool &bad) {
    if (cx1 < cx0 || cy1 < cy0) return;
    const int ncx = (cx1 - cx0) / 4 + 1, ncy = (cy1 - cy0) / 4 + 1;
    for (int i = threadIdx.x; i < ncx * ncy; i += blockDim.x) {
        const int cx = cx0 + 4 * (i % ncx), cy = cy0 + 4 * (i / ncx);
        const bool vs = boundary_at(cx + 2, W, scale_x, p.hard, p.col_start);
        const bool hs = boundary_at(cy + 2, H, scale_y, p.hard, p.row_start);
        int32_t *base = t + (cy - oy) * stride + (cx - ox);
        if (!vs && !hs) {
            int32_t v[16];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) v[r * 4 + c] = base[r * stride + c];
            bad |= pot16(v);
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) base[r * stride + c] = v[r * 4 + c];
        } else if (vs && !hs) {
            for (int c = 0; c < 4; c++) {
                const int x = cx + c;
                if (x < 0 || x >= W) continue;
                bad |= inverse_pot4(base[c], base[stride + c], base[2 * stride + c], base[3 * stride + c]);
            }
        } else if (!vs && hs) {
            for (int r = 0; r < 4; r++) {
                const int y = cy + r;
                if (y < 0 || y >= H) continue;
                int32_t *q = base + r * stride;
                bad |= inverse_pot4(q[0], q[1], q[2], q[3]);
            }
        } else {
            for (int k = 0; k < 4; k++) {
                const int x = cx + (k & 1) * 2, y = cy + (k >> 1) * 2;
                if (x < 0 || x >= W || y < 0 || y >= H) continue;
                int32_t *q = base + (k >> 1) * 2 * stride + (k & 1) * 2;
                bad |= inverse_pot4(q[0], q[1], q[stride], q[stride + 1]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// stage B for subsampled chroma: odd 2x2 cells, ordered corner residuals
// (crates/jxr-native/src/reconstruct/subsampled_overlap.rs:244-296)
// ---------------------------------------------------------------------------
__device__ void subsampled_cells(int32_t *dc, const PlaneDev &p, const PlaneGeom &g, bool &bad) {
    const int ncx = (g.ox1 - g.ox0) / 2 + 1, ncy = (g.oy1 - g.oy0) / 2 + 1;
    const int ox = g.mx0 * p.bc, oy = g.my0 * p.br;            // DC tile origin
    const int cov_x0 = max(0, g.ox0), cov_x1 = min(g.Wdc, g.ox1 + 2);
    const int cov_y0 = max(0, g.oy0), cov_y1 = min(g.Hdc, g.oy1 + 2);
    auto at = [&](int x, int y) -> int32_t & { return dc[(y - oy) * g.dw + (x - ox)]; };
    auto inside = [&](int x, int y) { return x >= cov_x0 && x < cov_x1 && y >= cov_y0 && y < cov_y1; };
    auto vb = [&](int x) { return boundary_at(x, g.Wdc, p.bc, p.hard, p.col_start); };
    auto hb = [&](int y) { return boundary_at(y, g.Hdc, p.br, p.hard, p.row_start); };
    // A corner of a region in a boundary row: sample (x, y) with a vertical
    // boundary on one side.  Its neighbour is the next sample inward.
    // phase 1: corners lose their neighbour (regions two wide run whole here)
    for (int pass = 0; pass < 2; pass++) {
        for (int i = threadIdx.x; i < ncx * ncy; i += blockDim.x) {
            const int cx = g.ox0 + 2 * (i % ncx), cy = g.oy0 + 2 * (i / ncx);
            if (!hb(cy + 1)) continue;  // no boundary row in this cell
            for (int k = 0; k < 4; k++) {
                const int x = cx + (k & 1), y = cy + (k >> 1);
                if (!inside(x, y) || x >= g.Wdc || y >= g.Hdc) continue;
                const bool left_corner = vb(x), right_corner = vb(x + 1);
                if (!left_corner && !right_corner) continue;
                const bool two_wide = left_corner && vb(x + 2) && !right_corner;
                const bool two_wide_right = right_corner && vb(x - 1) && !left_corner;
                if (two_wide_right) continue;   // handled with its left partner
                if (two_wide) {
                    if (pass == 1 || !inside(x + 1, y)) continue;
                    int32_t &c0 = at(x, y), &c1 = at(x + 1, y);
                    using A = Ar<true>;
                    c0 = A::sub(c0, c1, bad);
                    c1 = A::sub(c1, c0, bad);
                    c0 = A::add(c0, c1, bad);
                    c1 = A::add(c1, c0, bad);
                    continue;
                }
                const int n = left_corner ? x + 1 : x - 1;
                if (left_corner && right_corner) continue;  // one-wide: not a valid region
                if (!inside(n, y)) continue;
                using A = Ar<true>;
                if (pass == 0) at(x, y) = A::sub(at(x, y), at(n, y), bad);
                else at(x, y) = A::add(at(x, y), at(n, y), bad);
            }
        }
        if (pass == 1) break;
        __syncthreads();
        // phase 2: squares and pairs
        for (int i = threadIdx.x; i < ncx * ncy; i += blockDim.x) {
            const int cx = g.ox0 + 2 * (i % ncx), cy = g.oy0 + 2 * (i / ncx);
            const bool vs = vb(cx + 1), hs = hb(cy + 1);
            if (!vs && !hs) {
                if (!inside(cx, cy) || !inside(cx + 1, cy + 1)) continue;
                bad |= inverse_pot2x2(at(cx, cy), at(cx + 1, cy), at(cx, cy + 1), at(cx + 1, cy + 1));
            } else if (vs && !hs) {
                for (int c = 0; c < 2; c++) {
                    const int x = cx + c;
                    if (!inside(x, cy) || !inside(x, cy + 1)) continue;
                    bad |= inverse_pot2(at(x, cy), at(x, cy + 1));
                }
            } else if (!vs && hs) {
                for (int r = 0; r < 2; r++) {
                    const int y = cy + r;
                    if (!inside(cx, y) || !inside(cx + 1, y)) continue;
                    bad |= inverse_pot2(at(cx, y), at(cx + 1, y));
                }
            }
        }
        __syncthreads();
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// stage C: high-pass load, prediction, dequantization, second-level transform
// ---------------------------------------------------------------------------
__device__ void stage_high_pass(const PlaneDev &p, const PlaneGeom &g, int32_t *t, const int32_t *dc, bool &bad,
                                bool &bad_prediction) {
    const int nbx = g.bx1 - g.bx0 + 1, nby = g.by1 - g.by0 + 1;
    // C0: place the coded coefficients of each block in its 4x4 footprint
    for (int i = threadIdx.x; i < nbx * nby; i += blockDim.x) {
        const int bx = g.bx0 + i % nbx, by = g.by0 + i / nbx;
        const int mx = bx / p.bc, my = by / p.br;
        const uint4 e = p.mbs[(size_t)my * p.mbs_x + mx];
        const int bands = (e.x >> 28) & 3;
        const int blk = (by - my * p.br) * p.bc + (bx - mx * p.bc);
        int32_t *dst = t + (by - g.by0) * 4 * g.sw + (bx - g.bx0) * 4;
        if (bands >= 2) {
            const int32_t *src = p.coeff + (e.x & 0x0fffffffu) + blk * 16;
            if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
                const int4 *s4 = reinterpret_cast<const int4 *>(src);
#pragma unroll
                for (int r = 0; r < 4; r++) *reinterpret_cast<int4 *>(dst + r * g.sw) = __ldg(s4 + r);
            } else {
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) dst[r * g.sw + c] = __ldg(src + r * 4 + c);
            }
        } else {
#pragma unroll
            for (int r = 0; r < 4; r++) *reinterpret_cast<int4 *>(dst + r * g.sw) = make_int4(0, 0, 0, 0);
        }
    }
    __syncthreads();
    // C1: in-macroblock prediction (crates/jxr-math/src/prediction.rs:110-154),
    // one thread per block row (from left) or block column (from top)
    {
        const int mbx0 = g.bx0 / p.bc, mbx1 = g.bx1 / p.bc, mby0 = g.by0 / p.br, mby1 = g.by1 / p.br;
        const int nmx = mbx1 - mbx0 + 1, nmy = mby1 - mby0 + 1;
        const int lines = max(p.bc, p.br);
        for (int i = threadIdx.x; i < nmx * nmy * lines; i += blockDim.x) {
            const int line = i % lines, m = i / lines;
            const int mx = mbx0 + m % nmx, my = mby0 + m / nmx;
            const uint4 e = p.mbs[(size_t)my * p.mbs_x + mx];
            const int hp = (e.x >> 30) & 3;
            if (hp == 0) continue;
            if (hp == 3) { bad_prediction = true; continue; }
            const int bands = (e.x >> 28) & 3;
            if (bands < 2) continue;
            using A = Ar<true>;
            if (hp == 1) {  // from left: along block row `line`
                if (line >= p.br) continue;
                const int by = my * p.br + line;
                if (by < g.by0 || by > g.by1) continue;
                for (int c = 1; c < p.bc; c++) {
                    const int bx = mx * p.bc + c;
                    if (bx > g.bx1) break;
                    int32_t *cur = t + (by - g.by0) * 4 * g.sw + (bx - g.bx0) * 4;
                    const int32_t *prev = cur - 4;
                    // coefficients 4, 8, 12: first column, rows 1..3
#pragma unroll
                    for (int r = 1; r < 4; r++) cur[r * g.sw] = A::add(cur[r * g.sw], prev[r * g.sw], bad);
                }
            } else {        // from top: along block column `line`
                if (line >= p.bc) continue;
                const int bx = mx * p.bc + line;
                if (bx < g.bx0 || bx > g.bx1) continue;
                for (int r = 1; r < p.br; r++) {
                    const int by = my * p.br + r;
                    if (by > g.by1) break;
                    int32_t *cur = t + (by - g.by0) * 4 * g.sw + (bx - g.bx0) * 4;
                    const int32_t *prev = cur - 4 * g.sw;
                    // coefficients 1, 2, 3: first row, columns 1..3
#pragma unroll
                    for (int c = 1; c < 4; c++) cur[c] = A::add(cur[c], prev[c], bad);
                }
            }
        }
    }
    __syncthreads();
    // C2: dequantize, take the block DC, inverse core transform
    const int dox = g.mx0 * p.bc, doy = g.my0 * p.br;
    for (int i = threadIdx.x; i < nbx * nby; i += blockDim.x) {
        const int bx = g.bx0 + i % nbx, by = g.by0 + i / nbx;
        const int mx = bx / p.bc, my = by / p.br;
        const uint4 e = p.mbs[(size_t)my * p.mbs_x + mx];
        int32_t *blk = t + (by - g.by0) * 4 * g.sw + (bx - g.bx0) * 4;
        int32_t v[16];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            int4 q = *reinterpret_cast<const int4 *>(blk + r * g.sw);
            v[r * 4 + 0] = q.x; v[r * 4 + 1] = q.y; v[r * 4 + 2] = q.z; v[r * 4 + 3] = q.w;
        }
        const uint32_t step = e.w;
        uint32_t m = 0;
#pragma unroll
        for (int k = 1; k < 16; k++) m |= mag(v[k]);
        // |v| <= m + 1 for every coefficient, so this product bounds them all
        if ((uint64_t)(m + 1) * step <= 0x7fffffffull) {
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] = v[k] * (int32_t)step;
        } else {
#pragma unroll
            for (int k = 1; k < 16; k++) v[k] = dequant(v[k], step, bad);
        }
        v[0] = dc[(by - doy) * g.dw + (bx - dox)];
        bad |= pct16(v);
#pragma unroll
        for (int r = 0; r < 4; r++)
            *reinterpret_cast<int4 *>(blk + r * g.sw) = make_int4(v[r * 4], v[r * 4 + 1], v[r * 4 + 2], v[r * 4 + 3]);
    }
}

// ---------------------------------------------------------------------------
// stage E: output
// ---------------------------------------------------------------------------
struct PlaneView {
    const int32_t *t;  // sample tile
    int sw;            // stride
    int ox, oy;        // plane position of tile element (0,0)
    int W, H;          // plane extent
};

__device__ __forceinline__ int32_t view_at(const PlaneView &v, int x, int y) {
    return v.t[(y - v.oy) * v.sw + (x - v.ox)];
}

__device__ __forceinline__ int32_t view_clamped(const PlaneView &v, int x, int y) {
    x = min(max(x, 0), v.W - 1);
    y = min(max(y, 0), v.H - 1);
    return view_at(v, x, y);
}

// T.832 Table 180 pair, crates/jxr-math/src/sampling.rs:47-58,105-115.
__device__ __forceinline__ int32_t upsample_tap(int32_t prev, int32_t cur, int32_t next, int centering, int odd) {
    const int h0 = 4 + centering, h1 = 4 - centering, h2 = centering, h3 = 8 - centering;
    const int32_t a = odd ? cur : prev, b = odd ? next : cur;
    const int wa = odd ? h0 : h2, wb = odd ? h1 : h3;
    return (a >> 3) * wa + (b >> 3) * wb + (((a & 7) * wa + (b & 7) * wb + 4) >> 3);
}

__device__ int32_t chroma_sample(const PlaneView &v, int x, int y, int chroma, int cxc, int cyc) {
    const int cx = x >> 1;
    if (chroma == 2) {
        return upsample_tap(view_clamped(v, cx - 1, y), view_clamped(v, cx, y), view_clamped(v, cx + 1, y), cxc, x & 1);
    }
    const int cy = y >> 1;
    int32_t col[3];
#pragma unroll
    for (int d = -1; d <= 1; d++) {
        col[d + 1] = upsample_tap(view_clamped(v, cx + d, cy - 1), view_clamped(v, cx + d, cy),
                                  view_clamped(v, cx + d, cy + 1), cyc, y & 1);
    }
    return upsample_tap(col[0], col[1], col[2], cxc, x & 1);
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

// Exact binary16 -> binary32 widening of a half bit pattern.
__device__ __forceinline__ uint32_t widen_f16(uint32_t h) {
    const uint32_t sign = (h & 0x8000u) << 16, e = (h >> 10) & 0x1f;
    uint32_t m = h & 0x3ff;
    if (e == 0x1f) return sign | 0x7f800000u | (m << 13);
    if (e != 0) return sign | ((e + 112) << 23) | (m << 13);
    if (m == 0) return sign;
    const int lz = __clz(m) - 21;        // shifts that bring bit 10 to the top of the field
    return sign | ((uint32_t)(113 - lz) << 23) | (((m << lz) & 0x3ffu) << 13);
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
    for (int c = 0; c < o.channels; c++) {
        const ChannelScale &s = o.ch[c];
        const int32_t sample = s.alpha ? alpha_sample : conv[s.source & 3];
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
        for (int c = 0; c < n - 1; c++) {
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
    for (int c = 0; c < o.channels; c++) {
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

__device__ void reconstruct_tile(const ImageDev &im, int tx, int ty, int32_t *smem, uint32_t *status) {
    __shared__ int s_bad;
    __shared__ int s_stage;
    if (threadIdx.x == 0) { s_bad = 0; s_stage = 0; }
    const int mx0 = tx * kTileMbs, mx1 = min(mx0 + kTileMbs, (int)im.mbs_x);
    const int my0 = ty * kTileMbs, my1 = min(my0 + kTileMbs, (int)im.mbs_y);
    const int LW = (int)im.mbs_x * 16, LH = (int)im.mbs_y * 16;
    const int X0 = mx0 == 0 ? 0 : 16 * mx0 + 2, X1 = mx1 == (int)im.mbs_x ? LW : 16 * mx1 + 2;
    const int Y0 = my0 == 0 ? 0 : 16 * my0 + 2, Y1 = my1 == (int)im.mbs_y ? LH : 16 * my1 + 2;
    const int nplanes = im.nplanes + (im.alpha >= 0 ? 1 : 0);
    int32_t *dcbuf = smem + nplanes * kTileInts;
    PlaneView views[JXRB_MAX_PLANES];
    __syncthreads();
    for (int pi = 0; pi < nplanes; pi++) {
        const PlaneDev &p = im.plane[pi];
        const bool chroma_plane = pi >= 1 && pi <= 2 && pi < im.nplanes;
        const PlaneGeom g = plane_geometry(p, chroma_plane, im.chroma, X0, X1, Y0, Y1);
        int32_t *t = smem + pi * kTileInts;
        bool bad = false, badp = false;
        stage_first_level(p, g, dcbuf, bad);
        if (bad) atomicOr(&s_bad, kStatusFirstTransform);
        bad = false;
        __syncthreads();
        if (p.overlap == 2) {
            if (p.bc == 4) {
                overlap_cells(dcbuf, g.dw, g.mx0 * 4, g.my0 * 4, g.Wdc, g.Hdc, cell_of(g.bx0), cell_of(g.bx1),
                              cell_of(g.by0), cell_of(g.by1), 4, 4, p, bad);
                __syncthreads();
            } else {
                subsampled_cells(dcbuf, p, g, bad);
            }
            if (bad) atomicOr(&s_bad, kStatusOverlap);
            bad = false;
        }
        stage_high_pass(p, g, t, dcbuf, bad, badp);
        if (bad) atomicOr(&s_bad, kStatusSecondTransform);
        if (badp) atomicOr(&s_bad, kStatusInvalid);
        bad = false;
        __syncthreads();
        if (p.overlap >= 1) {
            overlap_cells(t, g.sw, g.bx0 * 4, g.by0 * 4, g.W, g.H, g.cx0, g.cx1, g.cy0, g.cy1, p.bc * 4, p.br * 4, p,
                          bad);
            if (bad) atomicOr(&s_bad, kStatusOverlap);
            bad = false;
        }
        views[pi].t = t;
        views[pi].sw = g.sw;
        views[pi].ox = g.bx0 * 4;
        views[pi].oy = g.by0 * 4;
        views[pi].W = g.W;
        views[pi].H = g.H;
        __syncthreads();
    }
    // output
    const OutputDev &o = im.out;
    const int ax0 = max(X0, (int)o.crop_x), ax1 = min(X1, (int)(o.crop_x + o.crop_w));
    const int ay0 = max(Y0, (int)o.crop_y), ay1 = min(Y1, (int)(o.crop_y + o.crop_h));
    bool bad = false;
    if (ax0 < ax1 && ay0 < ay1) {
        const int nx = ax1 - ax0, ny = ay1 - ay0;
        const uint64_t pixel_bytes = o.nchw ? (uint64_t)o.elem_bytes : (uint64_t)o.elem_bytes * o.channels;
        const uint64_t chs = o.nchw ? o.plane_stride : (uint64_t)o.elem_bytes;
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
                int32_t v = apply_scale(o.ch[0], view_at(views[0], x, y), bad);
                store_elem(o.base + at, (uint32_t)min(max(v, o.ch[0].lo), o.ch[0].hi), o.elem_bytes);
                if (im.alpha >= 0) {
                    v = apply_scale(o.ch[3], view_at(views[im.alpha], x, y), bad);
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
                        const int32_t w = apply_scale(o.ch[c], view_at(views[c], cx, cy), bad);
                        store_elem(o.base + luma_bytes + (uint64_t)(c - 1) * chroma_bytes + at,
                                   (uint32_t)min(max(w, o.ch[c].lo), o.ch[c].hi), o.elem_bytes);
                    }
                }
            }
        } else if (o.store == kStoreBits) {
            // one byte of eight pixels per thread; byte-aligned runs only
            const int bx0 = (ax0 - (int)o.crop_x) >> 3, bx1 = (ax1 - (int)o.crop_x + 7) >> 3;
            const int nbx = bx1 - bx0;
            for (int i = threadIdx.x; i < nbx * ny; i += blockDim.x) {
                const int by = ay0 + i / nbx, bx = bx0 + i % nbx;
                uint32_t byte = 0;
                bool mine = true;
                for (int k = 0; k < 8; k++) {
                    const int x = (int)o.crop_x + bx * 8 + k;
                    if (x >= (int)(o.crop_x + o.crop_w)) break;
                    if (x < X0 || x >= X1) { mine = false; break; }
                    int32_t v = apply_scale(o.ch[0], view_at(views[0], x, by), bad);
                    int32_t bit = min(max(v, 0), 1);
                    if (o.bit_black) bit = 1 - bit;
                    byte |= (uint32_t)bit << (7 - k);
                }
                if (!mine) {
                    // a byte shared with a neighbouring tile: set bits atomically
                    byte = 0;
                    for (int k = 0; k < 8; k++) {
                        const int x = (int)o.crop_x + bx * 8 + k;
                        if (x >= (int)(o.crop_x + o.crop_w)) break;
                        if (x < X0 || x >= X1) continue;
                        int32_t v = apply_scale(o.ch[0], view_at(views[0], x, by), bad);
                        int32_t bit = min(max(v, 0), 1);
                        if (o.bit_black) bit = 1 - bit;
                        byte |= (uint32_t)bit << (7 - k);
                    }
                    uint8_t *dst = o.base + (uint64_t)(by - o.crop_y) * o.row_stride + bx;
                    uint32_t *word = reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(dst) & ~(uintptr_t)3);
                    const int sh = (int)(reinterpret_cast<uintptr_t>(dst) & 3) * 8;
                    atomicOr(word, byte << sh);
                    continue;
                }
                o.base[(uint64_t)(by - o.crop_y) * o.row_stride + bx] = (uint8_t)byte;
            }
        } else {
            for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) {
                const int x = ax0 + i % nx, y = ay0 + i / nx;
                int32_t comp[4] = {0, 0, 0, 0};
                const int ncol = min(im.nplanes, 4);
                for (int c = 0; c < ncol; c++) {
                    if (im.chroma != 0 && (c == 1 || c == 2))
                        comp[c] = chroma_sample(views[c], x, y, im.chroma, im.centering_x, im.centering_y);
                    else
                        comp[c] = view_at(views[c], x, y);
                }
                const int32_t a = im.alpha >= 0 ? view_at(views[im.alpha], x, y) : 0;
                uint8_t *dst = o.base + (uint64_t)(y - o.crop_y) * o.row_stride + (uint64_t)(x - o.crop_x) * pixel_bytes;
                format_pixel(o, comp, a, dst, chs, bad);
            }
        }
    }
    if (bad) atomicOr(&s_bad, kStatusOutput);
    __syncthreads();
    if (threadIdx.x == 0 && s_bad) {
        const int b = s_bad;
        const uint32_t code = (b & kStatusInvalid) ? kStatusInvalid
                            : (b & kStatusFirstTransform) ? kStatusFirstTransform
                            : (b & kStatusOverlap) ? kStatusOverlap
                            : (b & kStatusSecondTransform) ? kStatusSecondTransform
                            : kStatusOutput;
        fail(status, code);
    }
    __syncthreads();
}

extern "C" __global__ void __launch_bounds__(kThreads)
jxrb_reconstruct_tiles(const ImageDev *__restrict__ images, const WorkItem *__restrict__ items, uint32_t item_count,
                       uint32_t *status) {
    extern __shared__ __align__(16) int32_t smem[];
    for (uint32_t i = blockIdx.x; i < item_count; i += gridDim.x) {
        const WorkItem w = items[i];
        reconstruct_tile(images[w.image], w.tx, w.ty, smem, status);
    }
}

}  // namespace jxr

// ---------------------------------------------------------------------------
// host launch helpers
// ---------------------------------------------------------------------------
namespace jxr {

size_t tile_smem_bytes(int planes) { return (size_t)planes * kTileInts * sizeof(int32_t) + kDcInts * sizeof(int32_t); }

cudaError_t launch_tiles(const ImageDev *images, const void *items, uint32_t item_count, int max_planes,
                         uint32_t *status, int grid, cudaStream_t stream) {
    const size_t smem = tile_smem_bytes(max_planes);
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(jxrb_reconstruct_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)tile_smem_bytes(JXRB_MAX_PLANES));
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (item_count == 0) return cudaSuccess;
    const int blocks = grid > 0 ? grid : (int)item_count;
    jxrb_reconstruct_tiles<<<blocks, kThreads, smem, stream>>>(images, static_cast<const WorkItem *>(items),
                                                               item_count, status);
    return cudaGetLastError();
}

int tile_mbs() { return kTileMbs; }

}  // namespace jxr
