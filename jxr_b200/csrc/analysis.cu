// analysis.cu -- the forward half of the codec on the GPU: the mirror of the
// reconstruction path, from sample planes to quantized coefficients.
//
// The reference analyses on the CPU only (analyze_component,
// crates/jxr-native/src/analyze.rs:56-131): the second-level prefilter (the
// forward overlap operators over the sample plane, overlap modes 1 and 2),
// the forward core transform of every 4x4 block, the first-level prefilter
// over the plane of block DCs (overlap mode 2; the ordered subsampled
// schedule for 4:2:0 / 4:2:2 chroma), the forward transform of each
// macroblock's block DCs (halved first where the plane is scaled), and the
// quantization of the DC, low-pass and high-pass bands (Quantizer::quantize,
// crates/jxr-math/src/quantization.rs:28-50).  Here each stage is a kernel
// over the plane: the overlap operators of one level are disjoint (the
// subsampled corners aside, which run in three ordered phases as in the
// decoder), so every operator, block and macroblock is its own work item.
// The results equal the CPU analysis bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/jxr_b200.h"
#include "forward.h"

namespace jxr {
jxrb_status report_error(jxrb_status s, const char *why);
jxrb_status report_cuda(cudaError_t e, const char *what);
}  // namespace jxr

namespace {

using namespace jxr::fwd;

// One plane on the device.  `starts` maps mark the macroblock columns / rows
// where a hard tile begins (all zero with soft tiles).
struct APlane {
    int32_t *samples;          // W x H, prefiltered in place
    int32_t *low;              // block DCs, (W/4) x (H/4)
    int32_t *low_q;            // 16 a macroblock
    int32_t *high_q;           // 256 a macroblock
    const uint8_t *col_start, *row_start;
    const uint32_t *cols;      // column region boundaries in macroblocks (0 .. mbs_x)
    uint32_t ncols;
    uint32_t W, H, mbs_x, mbs_y;
    int32_t bc, br, scale2, overlap, hard;
    uint32_t q[3];
};

__device__ __forceinline__ bool boundary(int p, int extent, int lg, int hard, const uint8_t *starts) {
    if (p <= 0 || p >= extent) return true;
    return hard && (p & ((1 << lg) - 1)) == 0 && starts[p >> lg];
}

__device__ __forceinline__ int log2i(int v) { return 31 - __clz(v); }

// The full-resolution overlap schedule of a plane of W x H values whose
// macroblocks are 2^lx x 2^ly of them, run forward: one 4x4 cell a thread,
// cells at origins 2 (mod 4); a cell a region boundary crosses takes the
// edge strips or corner quarters (the decoder's window list, forward
// operators; crates/jxr-native/src/reconstruct/overlap.rs:124-323).
__device__ void prefilter_cells(int32_t *s, int W, int H, int lx, int ly, int hard, const uint8_t *col_start,
                                const uint8_t *row_start) {
    const int ncx = W / 4 + 1, ncy = H / 4 + 1;
    auto at = [&](int x, int y) -> int32_t & { return s[(size_t)y * W + x]; };
    auto inside = [&](int x, int y) { return x >= 0 && x < W && y >= 0 && y < H; };
    for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < ncx * ncy; item += gridDim.x * blockDim.x) {
        const int cx = -2 + 4 * (item % ncx), cy = -2 + 4 * (item / ncx);
        const bool vs = boundary(cx + 2, W, lx, hard, col_start), hs = boundary(cy + 2, H, ly, hard, row_start);
        if (!vs && !hs) {
            int32_t v[16];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) v[r * 4 + c] = at(cx + c, cy + r);
            forward_pot4x4(v);
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) at(cx + c, cy + r) = v[r * 4 + c];
        } else if (vs && !hs) {
            for (int c = 0; c < 4; c++)
                if (cx + c >= 0 && cx + c < W) forward_pot4(at(cx + c, cy), at(cx + c, cy + 1), at(cx + c, cy + 2), at(cx + c, cy + 3));
        } else if (!vs && hs) {
            for (int r = 0; r < 4; r++)
                if (cy + r >= 0 && cy + r < H) forward_pot4(at(cx, cy + r), at(cx + 1, cy + r), at(cx + 2, cy + r), at(cx + 3, cy + r));
        } else {
            for (int k = 0; k < 4; k++) {
                const int x = cx + (k & 1) * 2, y = cy + (k >> 1) * 2;
                if (inside(x, y)) forward_pot4(at(x, y), at(x + 1, y), at(x, y + 1), at(x + 1, y + 1));
            }
        }
    }
}

__global__ void __launch_bounds__(256) jxrb_analysis_prefilter(const APlane *__restrict__ planes) {
    const APlane &p = planes[blockIdx.y];
    if (p.overlap < 1) return;
    prefilter_cells(p.samples, (int)p.W, (int)p.H, log2i(p.bc * 4), log2i(p.br * 4), p.hard, p.col_start, p.row_start);
}

// Forward core transform of every block: its DC into the block-DC plane, its
// other fifteen coefficients into the block's slot of the high-pass output
// (quantized later).
__global__ void __launch_bounds__(256) jxrb_analysis_blocks(const APlane *__restrict__ planes) {
    const APlane &p = planes[blockIdx.y];
    const uint32_t lw = p.W / 4, n = lw * (p.H / 4);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t bx = i % lw, by = i / lw;
        int32_t v[16];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int4 q = *reinterpret_cast<const int4 *>(&p.samples[((size_t)by * 4 + r) * p.W + bx * 4]);
            v[r * 4] = q.x; v[r * 4 + 1] = q.y; v[r * 4 + 2] = q.z; v[r * 4 + 3] = q.w;
        }
        forward_pct(v);
        p.low[i] = v[0];
        const uint32_t m = (by / p.br) * p.mbs_x + bx / p.bc, b = (by % p.br) * p.bc + bx % p.bc;
        int32_t *h = p.high_q + (size_t)m * 256 + b * 16;
        h[0] = 0;
#pragma unroll
        for (int k = 1; k < 16; k++) h[k] = v[k];
    }
}

// First-level prefilter of full-resolution planes: the cells of the block-DC plane.
__global__ void __launch_bounds__(256) jxrb_analysis_low_full(const APlane *__restrict__ planes) {
    const APlane &p = planes[blockIdx.y];
    if (p.overlap != 2 || p.bc != 4) return;
    prefilter_cells(p.low, (int)(p.W / 4), (int)(p.H / 4), 2, 2, p.hard, p.col_start, p.row_start);
}

// First-level prefilter of subsampled chroma, the decoder's ordered schedule
// inverted (crates/jxr-native/src/reconstruct/subsampled_overlap.rs:244-296):
// phase 0, each boundary row's corners lose their neighbour (right corner
// first); phase 1, every two-sample pair and 2x2 square forward; phase 2, the
// corners regain their (now filtered) neighbour.  A region two samples wide
// runs its four corner steps in that order as well.
__global__ void __launch_bounds__(256) jxrb_analysis_low_subsampled(const APlane *__restrict__ planes, int phase) {
    const APlane &p = planes[blockIdx.y];
    if (p.overlap != 2 || p.bc != 2) return;
    const int W = (int)(p.W / 4), H = (int)(p.H / 4);
    const int lx = log2i(p.bc), ly = log2i(p.br);
    int32_t *s = p.low;
    auto at = [&](int x, int y) -> int32_t & { return s[(size_t)y * W + x]; };
    auto vb = [&](int x) { return boundary(x, W, lx, p.hard, p.col_start); };
    auto hb = [&](int y) { return boundary(y, H, ly, p.hard, p.row_start); };
    if (phase == 1) {
        auto inside = [&](int x, int y) { return x >= 0 && x < W && y >= 0 && y < H; };
        const int ncx = W / 2 + 1, ncy = H / 2 + 1;
        for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < ncx * ncy; item += gridDim.x * blockDim.x) {
            const int cx = -1 + 2 * (item % ncx), cy = -1 + 2 * (item / ncx);
            const bool vs = vb(cx + 1), hs = hb(cy + 1);
            if (!vs && !hs) {
                if (inside(cx, cy) && inside(cx + 1, cy + 1))
                    forward_pot2x2(at(cx, cy), at(cx + 1, cy), at(cx, cy + 1), at(cx + 1, cy + 1));
            } else if (vs && !hs) {
                for (int c = 0; c < 2; c++)
                    if (inside(cx + c, cy) && inside(cx + c, cy + 1)) forward_pot2(at(cx + c, cy), at(cx + c, cy + 1));
            } else if (!vs && hs) {
                for (int r = 0; r < 2; r++)
                    if (inside(cx, cy + r) && inside(cx + 1, cy + r)) forward_pot2(at(cx, cy + r), at(cx + 1, cy + r));
            }
        }
        return;
    }
    // phases 0 and 2: one (boundary row, column region) a thread
    const int nreg = (int)p.ncols - 1;
    for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < H * nreg; item += gridDim.x * blockDim.x) {
        const int y = item / nreg, k = item % nreg;
        const bool top = hb(y), bottom = hb(y + 1);
        if (!top && !bottom) continue;
        const int l = (int)p.cols[k] * p.bc, r = (int)p.cols[k + 1] * p.bc;
        int32_t &c0 = at(l, y), &n0 = at(l + 1, y), &c1 = at(r - 1, y), &n1 = at(r - 2, y);
        if (phase == 0) {
            c1 -= n1;
            c0 -= n0;
        } else {
            c1 += n1;
            c0 += n0;
        }
    }
}

// Each macroblock's block DCs (halved where the plane is scaled) through the
// forward first-level transform, and every band quantized (analyze.rs:88-131;
// rounding offsets of half the step for DC and low-pass, a third for
// high-pass).
__global__ void __launch_bounds__(256) jxrb_analysis_quantize(const APlane *__restrict__ planes) {
    const APlane &p = planes[blockIdx.y];
    const uint32_t n = p.mbs_x * p.mbs_y, lw = p.W / 4;
    const int count = p.bc * p.br;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        const uint32_t mx = m % p.mbs_x, my = m / p.mbs_x;
        int32_t l[16];
#pragma unroll
        for (int k = 0; k < 16; k++) l[k] = 0;
        for (int r = 0; r < p.br; r++)
            for (int c = 0; c < p.bc; c++) l[r * p.bc + c] = p.low[((size_t)my * p.br + r) * lw + mx * p.bc + c];
        if (p.scale2)
            for (int k = 0; k < count; k++) l[k] >>= 1;
        if (count == 16) {
            forward_pct(l);
        } else if (count == 4) {
            int32_t w[4] = {l[0], l[1], l[2], l[3]};
            forward_420(w);
            for (int k = 0; k < 4; k++) l[k] = w[k];
        } else {
            int32_t w[8] = {l[0], l[1], l[2], l[3], l[4], l[5], l[6], l[7]};
            forward_422(w);
            for (int k = 0; k < 8; k++) l[k] = w[k];
        }
        int32_t *lq = p.low_q + (size_t)m * 16;
        lq[0] = quantize(l[0], p.q[0], p.q[0] / 2);
        for (int k = 1; k < 16; k++) lq[k] = k < count ? quantize(l[k], p.q[1], p.q[1] / 2) : 0;
        int32_t *h = p.high_q + (size_t)m * 256;
        for (int b = 0; b < 16; b++) {
            // element 0 of each block is the block DC's place: zero (past the
            // block count the whole block is zero)
            h[b * 16] = 0;
            for (int k = 1; k < 16; k++) h[b * 16 + k] = b < count ? quantize(h[b * 16 + k], p.q[2], p.q[2] / 3) : 0;
        }
    }
}

unsigned grid_for(uint64_t work) {
    return (unsigned)std::min<uint64_t>(std::max<uint64_t>((work + 255) / 256, 1), 2048);
}

}  // namespace

extern "C" jxrb_status jxrb_analyze_planes(const jxrb_analysis_plane *planes, uint32_t count, void *cuda_stream) {
    if (!planes || count == 0) return jxr::report_error(JXRB_INVALID_PLAN, "no planes");
    if (count > 65535) return jxr::report_error(JXRB_RESOURCE_LIMIT, "too many planes in one call");
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    // descriptors, tile-start maps and region lists in one allocation
    std::vector<APlane> dev(count);
    std::vector<uint8_t> maps;
    std::vector<uint32_t> cols;
    std::vector<size_t> map_at(count), cols_at(count);
    uint64_t max_samples = 0, max_mbs = 0, max_rows = 0;
    bool two_level = false, subsampled = false;
    for (uint32_t i = 0; i < count; i++) {
        const jxrb_analysis_plane &a = planes[i];
        const bool full = a.block_columns == 4 && a.block_rows == 4;
        const bool c420 = a.block_columns == 2 && a.block_rows == 2, c422 = a.block_columns == 2 && a.block_rows == 4;
        if (!full && !c420 && !c422) return jxr::report_error(JXRB_INVALID_PLAN, "block shape (4x4, 2x4 or 2x2)");
        const uint32_t mw = a.block_columns * 4, mh = a.block_rows * 4;
        if (a.width == 0 || a.height == 0 || a.width % mw || a.height % mh)
            return jxr::report_error(JXRB_INVALID_PLAN, "plane extent is not a whole number of macroblocks");
        if (a.overlap < 0 || a.overlap > 2) return jxr::report_error(JXRB_INVALID_PLAN, "overlap mode");
        if (a.steps[0] == 0 || a.steps[1] == 0 || a.steps[2] == 0) return jxr::report_error(JXRB_INVALID_PLAN, "zero quantizer");
        if (!a.samples || !a.low_scratch || !a.low_q || !a.high_q)
            return jxr::report_error(JXRB_INVALID_DESTINATION, "null device buffer");
        const uint32_t mbs_x = a.width / mw, mbs_y = a.height / mh;
        // tile starts and column regions from the boundaries (0 .. extent)
        const uint32_t *cb = a.column_boundaries, *rb = a.row_boundaries;
        if (!cb || !rb || a.column_count < 2 || a.row_count < 2 || cb[0] != 0 || rb[0] != 0 ||
            cb[a.column_count - 1] != mbs_x || rb[a.row_count - 1] != mbs_y)
            return jxr::report_error(JXRB_INVALID_PLAN, "tile boundaries must run from 0 to the macroblock extent");
        for (uint32_t k = 1; k < a.column_count; k++)
            if (cb[k] <= cb[k - 1]) return jxr::report_error(JXRB_INVALID_PLAN, "tile column boundaries");
        for (uint32_t k = 1; k < a.row_count; k++)
            if (rb[k] <= rb[k - 1]) return jxr::report_error(JXRB_INVALID_PLAN, "tile row boundaries");
        map_at[i] = maps.size();
        maps.resize(maps.size() + mbs_x + mbs_y + 2, 0);
        if (a.hard_tiles) {
            for (uint32_t k = 1; k + 1 < a.column_count; k++) maps[map_at[i] + cb[k]] = 1;
            for (uint32_t k = 1; k + 1 < a.row_count; k++) maps[map_at[i] + mbs_x + 1 + rb[k]] = 1;
        }
        cols_at[i] = cols.size();
        if (a.hard_tiles) cols.insert(cols.end(), cb, cb + a.column_count);
        else { cols.push_back(0); cols.push_back(mbs_x); }
        APlane &d = dev[i];
        d.samples = a.samples;
        d.low = a.low_scratch;
        d.low_q = a.low_q;
        d.high_q = a.high_q;
        d.W = a.width;
        d.H = a.height;
        d.mbs_x = mbs_x;
        d.mbs_y = mbs_y;
        d.bc = (int)a.block_columns;
        d.br = (int)a.block_rows;
        d.scale2 = a.scaled ? 1 : 0;
        d.overlap = a.overlap;
        d.hard = a.hard_tiles ? 1 : 0;
        d.ncols = a.hard_tiles ? a.column_count : 2;
        for (int b = 0; b < 3; b++) d.q[b] = a.steps[b];
        max_samples = std::max<uint64_t>(max_samples, (uint64_t)a.width * a.height);
        max_mbs = std::max<uint64_t>(max_mbs, (uint64_t)mbs_x * mbs_y);
        max_rows = std::max<uint64_t>(max_rows, (uint64_t)(a.height / 4) * (d.ncols - 1));
        two_level |= a.overlap == 2;
        subsampled |= a.overlap == 2 && !full;
    }
    const size_t desc_bytes = sizeof(APlane) * count, maps_at = (desc_bytes + 255) / 256 * 256;
    const size_t cols_at0 = (maps_at + maps.size() + 15) / 16 * 16, total = cols_at0 + cols.size() * 4;
    void *mem = nullptr;
    cudaError_t e = cudaMallocAsync(&mem, total, stream);
    if (e != cudaSuccess) return jxr::report_cuda(e, "cudaMallocAsync (analysis descriptors)");
    uint8_t *base = static_cast<uint8_t *>(mem);
    for (uint32_t i = 0; i < count; i++) {
        dev[i].col_start = base + maps_at + map_at[i];
        dev[i].row_start = base + maps_at + map_at[i] + dev[i].mbs_x + 1;
        dev[i].cols = reinterpret_cast<const uint32_t *>(base + cols_at0) + cols_at[i];
    }
    std::vector<uint8_t> host(total, 0);
    std::copy(reinterpret_cast<const uint8_t *>(dev.data()), reinterpret_cast<const uint8_t *>(dev.data()) + desc_bytes,
              host.begin());
    std::copy(maps.begin(), maps.end(), host.begin() + maps_at);
    std::copy(reinterpret_cast<const uint8_t *>(cols.data()), reinterpret_cast<const uint8_t *>(cols.data()) + cols.size() * 4,
              host.begin() + cols_at0);
    e = cudaMemcpyAsync(mem, host.data(), total, cudaMemcpyHostToDevice, stream);
    const APlane *d = static_cast<const APlane *>(mem);
    const dim3 g_cells(grid_for(max_samples / 16 + 64), count), g_blocks(grid_for(max_samples / 16), count);
    const dim3 g_mbs(grid_for(max_mbs), count), g_rows(grid_for(max_rows), count);
    if (e == cudaSuccess) {
        jxrb_analysis_prefilter<<<g_cells, 256, 0, stream>>>(d);
        jxrb_analysis_blocks<<<g_blocks, 256, 0, stream>>>(d);
        if (two_level) jxrb_analysis_low_full<<<g_cells, 256, 0, stream>>>(d);
        if (subsampled) {
            jxrb_analysis_low_subsampled<<<g_rows, 256, 0, stream>>>(d, 0);
            jxrb_analysis_low_subsampled<<<g_cells, 256, 0, stream>>>(d, 1);
            jxrb_analysis_low_subsampled<<<g_rows, 256, 0, stream>>>(d, 2);
        }
        jxrb_analysis_quantize<<<g_mbs, 256, 0, stream>>>(d);
        e = cudaGetLastError();
    }
    // the host image of the descriptors is read by the copy: wait for it
    const cudaError_t s = cudaStreamSynchronize(stream);
    cudaFreeAsync(mem, stream);
    if (e != cudaSuccess) return jxr::report_cuda(e, "analysis launch");
    if (s != cudaSuccess) return jxr::report_cuda(s, "analysis");
    return JXRB_OK;
}
