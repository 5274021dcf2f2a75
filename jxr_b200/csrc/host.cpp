// host.cpp -- planner, sessions and submissions behind the C ABI.
//
// The planner restates the validation of CudaDecodePlan::from_prepared
// (crates/jxr-cuda/src/plan.rs:91-148, 255-355, 357-734) and the output
// dispatch of build_output_dispatch (crates/jxr-core/src/device_plan/output.rs:52-295)
// for this engine's descriptors (engine.h).
#include <cuda_runtime.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/jxr_b200.h"
#include "engine.h"
#include "sample_scale.h"

namespace jxr {
size_t tile_smem_bytes(int planes);
cudaError_t launch_tiles(const ImageDev *images, const void *items, const uint32_t *bounds, int max_planes,
                         uint32_t *status, uint32_t *counters, cudaStream_t stream, cudaStream_t side,
                         cudaEvent_t fork, cudaEvent_t join, const LaunchTuning *tune);
int tile_mbs();
cudaError_t launch_quarter(const ImageDev *images, const QuarterImage *quarters, uint32_t count,
                           const QuarterPlane *planes, uint32_t plane_count, bool two_level, bool sixteenth_sums,
                           uint32_t max_mbs, uint32_t max_samples, uint32_t max_rows, uint32_t *status,
                           cudaStream_t stream);
}  // namespace jxr

using namespace jxr;

namespace {

thread_local std::string g_error;
thread_local uint32_t g_stage = 0;

jxrb_status fail(jxrb_status s, const std::string &why) {
    g_error = why;
    return s;
}

jxrb_status cuda_fail(cudaError_t e, const char *what) {
    g_error = std::string(what) + ": " + cudaGetErrorString(e);
    return JXRB_DRIVER;
}

#define CUDA_TRY(call, what)                                   \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, what);     \
    } while (0)

#define TRY(expr)                                              \
    do {                                                       \
        jxrb_status s_ = (expr);                               \
        if (s_ != JXRB_OK) return s_;                          \
    } while (0)

struct WorkItemHost {
    uint32_t image;
    uint16_t tx, ty;
};
static_assert(sizeof(WorkItemHost) == 8, "work item layout");

struct PlaneHost {
    int arena = 0;                 // 0 primary, 1 separate alpha
    uint64_t coeff_offset = 0;     // plane base within its arena (coefficients)
    std::vector<uint4> mbs;        // raster macroblock table
    std::vector<uint8_t> col_start, row_start;
    uint32_t mbs_x = 0, mbs_y = 0;
    int bc = 4, br = 4, scale2 = 0, overlap = 0, hard = 0;
};

// The interior tag an image's interior tiles carry (engine.h): its plane
// count when every plane is at full resolution (at most four), kTag420 for a
// YUV 4:2:0 image of three planes, 0 when every tile takes the general kernel.
// 1-bit and planar outputs always take the general kernel.
template <class Planes>
uint32_t interior_tag(const Planes &planes, int chroma, const OutputDev &out) {
    const size_t np = planes.size();
    if (np < 1 || np > 4 || out.store == kStoreBits || out.planar_yuv) return 0;
    bool full = true;
    for (const auto &p : planes) full &= p.bc == 4 && p.br == 4;
    if (full) return (uint32_t)np;
    if (np == 3 && chroma == 1 && planes[0].bc == 4 && planes[0].br == 4 && planes[1].bc == 2 && planes[1].br == 2 &&
        planes[2].bc == 2 && planes[2].br == 2)
        return kTag420;
    return 0;
}

// Whether tile (tx, ty) of a window mbs_x x mbs_y macroblocks wide is an
// interior tile: macroblocks mx0-1 .. mx0+4 and my0-1 .. my0+4 inside the
// window and, with hard tiles, no tile starting at columns mx0 .. mx0+4 or
// rows my0 .. my0+4 (`starts_x` / `starts_y`: window-relative tile-start
// flags of the luma plane, or null without hard tiles).
bool interior_tile_at(uint32_t tx, uint32_t ty, uint32_t T, uint32_t mbs_x, uint32_t mbs_y, const uint8_t *starts_x,
                      const uint8_t *starts_y) {
    const uint32_t mx0 = tx * T, my0 = ty * T;
    if (mx0 < 1 || my0 < 1 || mx0 + T >= mbs_x || my0 + T >= mbs_y) return false;
    if (starts_x)
        for (uint32_t k = mx0; k <= mx0 + T; k++)
            if (starts_x[k] || starts_y[my0 + (k - mx0)]) return false;
    return true;
}

// Whether tile (tx, ty) of a full-resolution image may take the edge kernel:
// no hard tile starts at its macroblock columns mx0 .. mx0+4 or rows
// my0 .. my0+4 inside the window, the window's own edges aside.
bool edge_tile_at(uint32_t tx, uint32_t ty, uint32_t T, uint32_t mbs_x, uint32_t mbs_y, const uint8_t *starts_x,
                  const uint8_t *starts_y) {
    if (!starts_x) return true;
    const uint32_t mx0 = tx * T, my0 = ty * T;
    for (uint32_t k = std::max(mx0, 1u); k <= mx0 + T && k < mbs_x; k++)
        if (starts_x[k]) return false;
    for (uint32_t k = std::max(my0, 1u); k <= my0 + T && k < mbs_y; k++)
        if (starts_y[k]) return false;
    return true;
}

// The tag of tile (tx, ty) of an image whose interior tag is `kind`: the
// interior kernels' where the tile qualifies, the edge kernels' for the other
// tiles that qualify, else 0 (the general kernel).
uint32_t tile_tag(uint32_t kind, uint32_t tx, uint32_t ty, uint32_t T, uint32_t mbs_x, uint32_t mbs_y,
                  const uint8_t *starts_x, const uint8_t *starts_y) {
    if (!kind) return 0;
    if (interior_tile_at(tx, ty, T, mbs_x, mbs_y, starts_x, starts_y)) return kind;
    if (!edge_tile_at(tx, ty, T, mbs_x, mbs_y, starts_x, starts_y)) return 0;
    if (kind <= 4) return kTagEdge + kind;
    // 4:2:0 edge tiles need two chroma DC samples between the plane's corners
    return kind == kTag420 && mbs_x >= 2 && mbs_y >= 2 ? kTagEdge420 : 0;
}

// Work-list segment of a tag (engine.h).  Folded edge tiles (kFoldEdges) go
// to their interior kernel's segment -- one kernel, so that their latency
// hides among the interior tiles -- ahead of its interior tiles.
bool folded_edge_tag(uint32_t tag) {
    if (tag > kTagEdge && tag <= kTagEdge + 4) return kFoldEdges[tag - kTagEdge - 1];
    return tag == kTagEdge420 && kFoldEdges[4];
}
int segment_of_tag(uint32_t tag) {
    if (folded_edge_tag(tag)) return tag == kTagEdge420 ? 4 : (int)(tag - kTagEdge) - 1;
    return tag ? (int)tag - 1 : kSegmentOther;
}
int rank_of_tag(uint32_t tag) { return folded_edge_tag(tag) ? 0 : 1; }

// Stable order of a work list by segment (a counting sort: one pass to count,
// one to place); `bounds` receives the kSegments + 1 segment boundaries.
void order_by_segment(std::vector<WorkItemHost> &items, uint32_t *bounds) {
    auto key = [](const WorkItemHost &w) {
        const uint32_t tag = w.image >> kTagShift;
        return segment_of_tag(tag) * 2 + rank_of_tag(tag);
    };
    uint32_t cursor[2 * kSegments] = {};
    for (const WorkItemHost &w : items) cursor[key(w)]++;
    uint32_t at = 0;
    for (int k = 0; k < 2 * kSegments; k++) {
        if ((k & 1) == 0) bounds[k / 2] = at;
        const uint32_t n = cursor[k];
        cursor[k] = at;
        at += n;
    }
    bounds[kSegments] = at;
    std::vector<WorkItemHost> sorted(items.size());
    for (const WorkItemHost &w : items) sorted[cursor[key(w)]++] = w;
    items.swap(sorted);
}

}  // namespace

struct jxrb_plan {
    const int32_t *coefficients[2] = {nullptr, nullptr};
    uint64_t coefficient_count[2] = {0, 0};
    std::vector<PlaneHost> planes;   // colour planes, then alpha
    int nplanes = 0;
    int alpha = -1;
    int chroma = 0;
    int centering_x = 0, centering_y = 0;
    uint32_t mbs_x = 0, mbs_y = 0;
    OutputDev out{};                 // base pointer filled at submission
    uint64_t output_bytes = 0;
    uint64_t traffic_bytes = 0;
    uint64_t metadata_bytes = 0;
};

namespace {

// ---------------------------------------------------------------------------
// output policy: validate_matrix (crates/jxr-native/src/output_format/validate.rs:108-250)
// and the channel scales of scaling.rs:37-119
// ---------------------------------------------------------------------------
int layout_channels(int layout, int ncomp) {
    switch (layout) {
    case JXRB_LAYOUT_LUMA: return 1;
    case JXRB_LAYOUT_LUMA_ALPHA: return 2;
    case JXRB_LAYOUT_YUV: case JXRB_LAYOUT_RGB: case JXRB_LAYOUT_BGR: return 3;
    case JXRB_LAYOUT_YUVA: case JXRB_LAYOUT_RGBX: case JXRB_LAYOUT_RGBA: case JXRB_LAYOUT_BGRX:
    case JXRB_LAYOUT_BGRA: case JXRB_LAYOUT_CMYK: return 4;
    case JXRB_LAYOUT_CMYKA: return 5;
    case JXRB_LAYOUT_NCOMPONENT: return ncomp;
    case JXRB_LAYOUT_NCOMPONENT_ALPHA: return ncomp + 1;
    default: return 0;
    }
}

bool layout_has_alpha(int l) {
    return l == JXRB_LAYOUT_LUMA_ALPHA || l == JXRB_LAYOUT_YUVA || l == JXRB_LAYOUT_RGBA || l == JXRB_LAYOUT_BGRA ||
           l == JXRB_LAYOUT_CMYKA || l == JXRB_LAYOUT_NCOMPONENT_ALPHA;
}

int storage_bytes(int s) {
    switch (s) {
    case JXRB_STORE_U8: return 1;
    case JXRB_STORE_U16: case JXRB_STORE_I16: case JXRB_STORE_F16: case JXRB_STORE_RGB555: case JXRB_STORE_RGB565: return 2;
    default: return 4;
    }
}

bool packed_depth(int d) { return d == JXRB_DEPTH_RGB555 || d == JXRB_DEPTH_RGB565 || d == JXRB_DEPTH_RGB101010; }

bool resolve_scale(int component, int output_color, int depth, int shift_bits, int scaled, ChannelScale &s) {
    int32_t base = 0;
    int shift = 0;
    switch (depth) {
    case JXRB_DEPTH_RGB555: base = 1 << 4; break;
    case JXRB_DEPTH_RGB565: base = 1 << 5; break;
    case JXRB_DEPTH_U8: base = 1 << 7; break;
    case JXRB_DEPTH_U10: case JXRB_DEPTH_RGB101010: base = 1 << 9; break;
    case JXRB_DEPTH_U16: base = 1 << 15; shift = shift_bits; break;
    case JXRB_DEPTH_I16: case JXRB_DEPTH_I32: base = 0; shift = shift_bits; break;
    default: break;
    }
    if (shift < 0 || shift >= 32) return false;
    const int32_t bias = base >> shift;
    int32_t cb = bias;
    if (output_color == JXRB_COLOR_CMYK) cb = component < 3 ? bias >> 1 : -(bias >> 1);
    else if (output_color == JXRB_COLOR_RGBE) cb = 0;
    const int sc = scaled ? 3 : 0;
    const int64_t shifted = (int64_t)cb * ((int64_t)1 << sc);
    if (shifted < INT32_MIN || shifted > INT32_MAX) return false;
    s.shifted_bias = (int32_t)shifted;
    s.rounding = scaled ? ((depth == JXRB_DEPTH_BIT1_WHITE || depth == JXRB_DEPTH_BIT1_BLACK || depth == JXRB_DEPTH_U16) ? 4 : 3) : 0;
    s.shift = (depth == JXRB_DEPTH_RGB565 && component != 1) ? sc + 1 : sc;
    s.post_shift = (depth == JXRB_DEPTH_U16 || depth == JXRB_DEPTH_I16 || depth == JXRB_DEPTH_I32) ? std::min(shift_bits, 31) : -1;
    s.lo = INT32_MIN;
    s.hi = INT32_MAX;
    return true;
}

void clip_range(int storage, int depth, ChannelScale &s) {
    switch (storage) {
    case JXRB_STORE_U8: s.lo = 0; s.hi = 255; break;
    case JXRB_STORE_U16: s.lo = 0; s.hi = depth == JXRB_DEPTH_U10 ? 1023 : 65535; break;
    case JXRB_STORE_I16: s.lo = -32768; s.hi = 32767; break;
    default: s.lo = INT32_MIN; s.hi = INT32_MAX; break;
    }
}

jxrb_status validate_output(const jxrb_output_format &r, int internal, bool has_alpha) {
    int layout = r.layout;
    if (r.storage >= JXRB_STORE_RGB555) layout = JXRB_LAYOUT_RGB;
    if (layout_has_alpha(layout) != has_alpha) return fail(JXRB_INVALID_PLAN, "alpha layout and prepared alpha plane differ");
    if (r.premultiply_alpha && !has_alpha) return fail(JXRB_INVALID_PLAN, "premultiplied output without alpha");
    const int oc = r.output_color, d = r.bit_depth, s = r.storage;
    if (r.premultiply_alpha && (oc == JXRB_COLOR_YUV420 || oc == JXRB_COLOR_YUV422 || oc == JXRB_COLOR_YUV444))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "premultiplied YUV output");
    bool ok = ((d == JXRB_DEPTH_BIT1_WHITE || d == JXRB_DEPTH_BIT1_BLACK) && s == JXRB_STORE_BITS && r.layout == JXRB_LAYOUT_LUMA) ||
              (d == JXRB_DEPTH_U8 && (s == JXRB_STORE_U8 || s == JXRB_STORE_RGBE)) ||
              ((d == JXRB_DEPTH_U10 || d == JXRB_DEPTH_U16) && s == JXRB_STORE_U16) ||
              (d == JXRB_DEPTH_I16 && s == JXRB_STORE_I16) || (d == JXRB_DEPTH_I32 && s == JXRB_STORE_I32) ||
              (d == JXRB_DEPTH_F16 && s == JXRB_STORE_F16) || (d == JXRB_DEPTH_F32 && s == JXRB_STORE_F32) ||
              (d == JXRB_DEPTH_RGB555 && s == JXRB_STORE_RGB555) || (d == JXRB_DEPTH_RGB565 && s == JXRB_STORE_RGB565) ||
              (d == JXRB_DEPTH_RGB101010 && s == JXRB_STORE_RGB101010);
    if (!ok) return fail(JXRB_UNSUPPORTED_OUTPUT, "bit depth and typed storage");
    switch (oc) {
    case JXRB_COLOR_LUMA: ok = layout == JXRB_LAYOUT_LUMA || layout == JXRB_LAYOUT_LUMA_ALPHA; break;
    case JXRB_COLOR_RGB:
        ok = layout == JXRB_LAYOUT_RGB || layout == JXRB_LAYOUT_RGBX || layout == JXRB_LAYOUT_RGBA ||
             layout == JXRB_LAYOUT_BGR || layout == JXRB_LAYOUT_BGRX || layout == JXRB_LAYOUT_BGRA;
        break;
    case JXRB_COLOR_YUV420: case JXRB_COLOR_YUV422: case JXRB_COLOR_YUV444:
        ok = layout == JXRB_LAYOUT_YUV || layout == JXRB_LAYOUT_YUVA; break;
    case JXRB_COLOR_CMYK: case JXRB_COLOR_CMYK_DIRECT: ok = layout == JXRB_LAYOUT_CMYK || layout == JXRB_LAYOUT_CMYKA; break;
    case JXRB_COLOR_RGBE: ok = s == JXRB_STORE_RGBE; break;
    case JXRB_COLOR_NCOMPONENT: ok = layout == JXRB_LAYOUT_NCOMPONENT || layout == JXRB_LAYOUT_NCOMPONENT_ALPHA; break;
    default: ok = false;
    }
    if (!ok) return fail(JXRB_UNSUPPORTED_OUTPUT, "output colour and channel layout");
    const bool integer_rgb = !(d == JXRB_DEPTH_F16 || d == JXRB_DEPTH_F32);
    if (internal == JXRB_COLOR_LUMA && oc == JXRB_COLOR_RGB) ok = integer_rgb;
    else if ((internal == JXRB_COLOR_LUMA && oc == JXRB_COLOR_LUMA) ||
             (internal == JXRB_COLOR_YUV444 && (oc == JXRB_COLOR_RGB || oc == JXRB_COLOR_RGBE)) ||
             (internal == JXRB_COLOR_YUVK && (oc == JXRB_COLOR_CMYK || oc == JXRB_COLOR_CMYK_DIRECT)))
        ok = true;
    else if ((internal == JXRB_COLOR_YUV420 || internal == JXRB_COLOR_YUV422 || internal == JXRB_COLOR_YUV444) && internal == oc)
        ok = true;
    else ok = internal == JXRB_COLOR_NCOMPONENT && oc == JXRB_COLOR_NCOMPONENT;
    if (!ok) return fail(JXRB_UNSUPPORTED_OUTPUT, "internal and output colour formats");
    switch (oc) {
    case JXRB_COLOR_LUMA: ok = !packed_depth(d); break;
    case JXRB_COLOR_RGB: ok = true; break;
    case JXRB_COLOR_YUV420: case JXRB_COLOR_YUV422: case JXRB_COLOR_YUV444:
        ok = d == JXRB_DEPTH_U8 || d == JXRB_DEPTH_U10 || d == JXRB_DEPTH_U16 || d == JXRB_DEPTH_I16; break;
    case JXRB_COLOR_RGBE: ok = d == JXRB_DEPTH_U8; break;
    default: ok = d == JXRB_DEPTH_U8 || d == JXRB_DEPTH_U16;
    }
    if (!ok) return fail(JXRB_UNSUPPORTED_OUTPUT, "T.832 output colour and bit depth matrix");
    if ((d == JXRB_DEPTH_F32 && r.mantissa_length > 23) ||
        (has_alpha && r.alpha_bit_depth == JXRB_DEPTH_F32 && r.alpha_mantissa_length > 23))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "BD32F mantissa length exceeds 23 bits");
    if (r.widen_f16 && s != JXRB_STORE_F16) return fail(JXRB_UNSUPPORTED_OUTPUT, "widening applies to F16 output");
    if (r.nchw && (s == JXRB_STORE_BITS || s >= JXRB_STORE_RGB555 || oc == JXRB_COLOR_YUV420 || oc == JXRB_COLOR_YUV422))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "NCHW applies to per-channel storage");
    if (r.premultiply_alpha && (r.nchw || r.widen_f16))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "premultiplied output is interleaved");
    if (has_alpha && s == JXRB_STORE_F32 && r.alpha_bit_depth != JXRB_DEPTH_F32)
        return fail(JXRB_UNSUPPORTED_OUTPUT, "alpha and primary floating-point depth");
    return JXRB_OK;
}

jxrb_status build_output(const jxrb_output_format &r, int internal, int ncomp, bool has_alpha, int scaled,
                         int alpha_scaled, OutputDev &o, uint64_t &bytes) {
    TRY(validate_output(r, internal, has_alpha));
    std::memset(&o, 0, sizeof o);
    o.crop_x = r.crop_x; o.crop_y = r.crop_y; o.crop_w = r.crop_width; o.crop_h = r.crop_height;
    o.store = r.storage;
    o.widen_f16 = r.widen_f16 ? 1 : 0;
    o.nchw = r.nchw ? 1 : 0;
    o.premultiply = r.premultiply_alpha ? 1 : 0;
    o.elem_bytes = o.widen_f16 ? 4 : storage_bytes(r.storage);
    o.bit_black = r.bit_depth == JXRB_DEPTH_BIT1_BLACK;
    const int oc = r.output_color, d = r.bit_depth;
    o.packed_swap = packed_depth(d) && !r.red_blue_not_swapped;
    if (internal == JXRB_COLOR_LUMA && oc == JXRB_COLOR_RGB) o.conv = kConvLumaToRgb;
    else if (internal == JXRB_COLOR_YUV444 && (oc == JXRB_COLOR_RGB || oc == JXRB_COLOR_RGBE)) o.conv = kConvYuvToRgb;
    else if (internal == JXRB_COLOR_YUVK && oc == JXRB_COLOR_CMYK) o.conv = kConvYuvkToCmyk;
    else if (internal == JXRB_COLOR_YUVK && oc == JXRB_COLOR_CMYK_DIRECT) o.conv = kConvYuvkToCmykDirect;
    else o.conv = kConvDirect;
    const uint64_t w = r.crop_width, h = r.crop_height;
    auto bad_scale = [] { return fail(JXRB_UNSUPPORTED_OUTPUT, "integer SHIFT_BITS greater than 31"); };
    if (oc == JXRB_COLOR_YUV420 || oc == JXRB_COLOR_YUV422) {
        // native planar YUV (crates/jxr-native/src/output_format/planar.rs)
        o.planar_yuv = oc == JXRB_COLOR_YUV420 ? 1 : 2;
        for (int c = 0; c < 3; c++) {
            if (!resolve_scale(c, oc, d, r.shift_bits, scaled, o.ch[c])) return bad_scale();
            clip_range(r.storage, d, o.ch[c]);
        }
        if (has_alpha) {
            if (!resolve_scale(0, JXRB_COLOR_LUMA, r.alpha_bit_depth, r.alpha_shift_bits, alpha_scaled, o.ch[3])) return bad_scale();
            clip_range(r.storage, r.alpha_bit_depth, o.ch[3]);
        }
        const uint64_t cw = w / 2, ch = o.planar_yuv == 1 ? h / 2 : h;
        o.channels = 1;
        o.row_stride = w * o.elem_bytes;
        bytes = (w * h + 2 * cw * ch + (has_alpha ? w * h : 0)) * o.elem_bytes;
        return JXRB_OK;
    }
    if (r.storage == JXRB_STORE_BITS) {
        if (!resolve_scale(0, JXRB_COLOR_LUMA, d, 0, scaled, o.ch[0])) return bad_scale();
        o.channels = 1;
        o.row_stride = (w + 7) / 8;
        bytes = o.row_stride * h;
        return JXRB_OK;
    }
    if (r.storage >= JXRB_STORE_RGB555) {
        const int color = r.storage == JXRB_STORE_RGBE ? JXRB_COLOR_RGBE : JXRB_COLOR_RGB;
        const int depth = r.storage == JXRB_STORE_RGBE ? JXRB_DEPTH_U8 : d;
        for (int c = 0; c < 3; c++) {
            if (!resolve_scale(c, color, depth, 0, scaled, o.ch[c])) return bad_scale();
            o.ch[c].lo = 0;
            o.ch[c].hi = d == JXRB_DEPTH_RGB555 ? 31 : d == JXRB_DEPTH_RGB101010 ? 1023 : (c == 1 ? 63 : 31);
        }
        o.channels = 1;
        o.row_stride = w * o.elem_bytes;
        bytes = o.row_stride * h;
        return JXRB_OK;
    }
    // ordered channels: primaries in layout order, then alpha (packing.rs:538-585)
    int primaries;
    if (oc == JXRB_COLOR_NCOMPONENT) primaries = ncomp;
    else {
        switch (r.layout) {
        case JXRB_LAYOUT_LUMA: primaries = 1; break;
        case JXRB_LAYOUT_YUV: case JXRB_LAYOUT_RGB: case JXRB_LAYOUT_BGR: primaries = 3; break;
        case JXRB_LAYOUT_RGBX: case JXRB_LAYOUT_BGRX: case JXRB_LAYOUT_CMYK: case JXRB_LAYOUT_CMYKA: primaries = 4; break;
        default: primaries = layout_channels(r.layout, ncomp) - 1;
        }
    }
    o.channels = primaries + (has_alpha ? 1 : 0);
    if (o.channels > JXRB_MAX_CHANNELS || primaries > 4) return fail(JXRB_UNSUPPORTED_OUTPUT, "too many output channels");
    const bool reverse = r.layout == JXRB_LAYOUT_BGR || r.layout == JXRB_LAYOUT_BGRX || r.layout == JXRB_LAYOUT_BGRA;
    const bool padded = r.layout == JXRB_LAYOUT_RGBX || r.layout == JXRB_LAYOUT_BGRX;
    for (int c = 0; c < primaries; c++) {
        ChannelScale &s = o.ch[c];
        s.source = reverse && c < 3 ? 2 - c : c;
        s.padding = padded && c == 3;
        s.f_scaled = scaled;
        s.f_mantissa = r.mantissa_length;
        s.f_bias = r.exponent_bias;
        int depth = d;
        if (r.storage == JXRB_STORE_F16 || r.storage == JXRB_STORE_F32) {
            if (!resolve_scale(0, JXRB_COLOR_LUMA, depth, 0, scaled, s)) return bad_scale();
        } else {
            if (!resolve_scale(c, oc, depth, r.shift_bits, scaled, s)) return bad_scale();
            clip_range(r.storage, depth, s);
        }
        s.padding = padded && c == 3;
    }
    if (has_alpha) {
        ChannelScale &s = o.ch[primaries];
        if (!resolve_scale(0, JXRB_COLOR_LUMA, r.alpha_bit_depth, r.alpha_shift_bits, alpha_scaled, s)) return bad_scale();
        if (r.storage != JXRB_STORE_F16 && r.storage != JXRB_STORE_F32) clip_range(r.storage, r.alpha_bit_depth, s);
        s.alpha = 1;
        s.source = 4;
        s.f_scaled = alpha_scaled;
        s.f_mantissa = r.alpha_mantissa_length;
        s.f_bias = r.alpha_exponent_bias;
    }
    if (o.nchw) {
        o.row_stride = w * o.elem_bytes;
        o.plane_stride = w * h * o.elem_bytes;
    } else {
        o.row_stride = w * o.channels * o.elem_bytes;
    }
    bytes = w * h * o.channels * o.elem_bytes;
    // specialised output paths of the kernel (the generic one covers the rest)
    const bool rgb_layout = r.layout == JXRB_LAYOUT_RGB || r.layout == JXRB_LAYOUT_BGR || r.layout == JXRB_LAYOUT_RGBA ||
                            r.layout == JXRB_LAYOUT_BGRA;
    if (r.storage == JXRB_STORE_U8 && o.conv == kConvYuvToRgb && !o.nchw && rgb_layout &&
        (o.channels == 3 || o.channels == 4))
        o.kind = 1;
    else if (o.conv == kConvDirect && o.channels == 1 && !has_alpha && !o.nchw &&
             (r.storage == JXRB_STORE_U8 || r.storage == JXRB_STORE_U16 || r.storage == JXRB_STORE_I16 ||
              r.storage == JXRB_STORE_I32))
        o.kind = 2;
    else if (r.storage == JXRB_STORE_F16 && o.widen_f16 && !o.premultiply && o.channels <= 4)
        o.kind = 3;
    else
        o.kind = 0;
    return JXRB_OK;
}

// tile boundaries within the window (crates/jxr-core/src/device_plan/overlap.rs:102-123)
jxrb_status window_starts(const uint32_t *sizes, uint32_t count, uint32_t origin, uint32_t extent,
                          std::vector<uint8_t> &starts) {
    starts.assign(extent, 0);
    uint64_t end = (uint64_t)origin + extent, position = 0;
    for (uint32_t i = 0; i < count; i++) {
        position += sizes[i];
        if (position > origin && position < end) starts[position - origin] = 1;
    }
    if (position < end) return fail(JXRB_INVALID_PLAN, "tile partition does not cover reconstruction window");
    return JXRB_OK;
}

uint64_t coefficients_per_macroblock(int bands, int blocks) {
    if (bands == JXRB_BANDS_DC_ONLY) return 1;
    if (bands == JXRB_BANDS_NO_HIGH_PASS) return (uint64_t)blocks;
    return (uint64_t)blocks * 16;
}

// One plane's macroblock table: every window position exactly once, every
// coefficient span inside the plane and the arena (plan.rs:405-610).
jxrb_status build_plane(const jxrb_arena &a, uint32_t index, const jxrb_image_geometry &g, int bc, int br,
                        PlaneHost &out) {
    if (index >= a.plane_count) return fail(JXRB_INVALID_PLAN, "coefficient plane index is out of range");
    const jxrb_coefficient_plane &p = a.planes[index];
    if (p.block_columns != (uint32_t)bc || p.block_rows != (uint32_t)br)
        return fail(JXRB_INVALID_PLAN, "coefficient plane block geometry differs from the colour format");
    if (p.coefficient_offset + p.coefficient_count > a.coefficient_count || p.coefficient_offset > a.coefficient_count)
        return fail(JXRB_INVALID_PLAN, "coefficient plane range");
    if (p.macroblock_offset + p.macroblock_count > a.macroblock_count || p.macroblock_offset > a.macroblock_count)
        return fail(JXRB_INVALID_PLAN, "macroblock plane range");
    const uint64_t n = (uint64_t)g.macroblocks_x * g.macroblocks_y;
    out.mbs.assign(n, make_uint4(0, 0, 0, 0));
    std::vector<uint8_t> seen(n, 0);
    out.mbs_x = g.macroblocks_x;
    out.mbs_y = g.macroblocks_y;
    out.bc = bc;
    out.br = br;
    out.coeff_offset = p.coefficient_offset;
    uint64_t filled = 0;
    for (uint64_t m = p.macroblock_offset; m < p.macroblock_offset + p.macroblock_count; m++) {
        const uint32_t cx = a.coded_x[m], cy = a.coded_y[m];
        if (cx < g.macroblock_origin_x || cy < g.macroblock_origin_y) continue;
        const uint32_t lx = cx - g.macroblock_origin_x, ly = cy - g.macroblock_origin_y;
        if (lx >= g.macroblocks_x || ly >= g.macroblocks_y) continue;   // outside the window
        const uint64_t pos = (uint64_t)ly * g.macroblocks_x + lx;
        if (seen[pos]) return fail(JXRB_INVALID_PLAN, "duplicate macroblock coordinates");
        seen[pos] = 1;
        filled++;
        const int bands = a.bands[m];
        const int hp = a.hp_predictions[m];
        if (bands > 3) return fail(JXRB_INVALID_PLAN, "band presence");
        if (hp == 3) return fail(JXRB_INVALID_PLAN, "top-left high-pass prediction");
        if (hp > 3) return fail(JXRB_INVALID_PLAN, "high-pass prediction direction");
        const uint32_t q0 = a.quantizers[3 * m], q1 = a.quantizers[3 * m + 1], q2 = a.quantizers[3 * m + 2];
        if (q0 == 0 || q1 == 0 || q2 == 0) return fail(JXRB_INVALID_PLAN, "zero quantizer");
        const uint64_t off = a.coefficient_offsets[m];
        const uint64_t need = coefficients_per_macroblock(bands, bc * br);
        if (off < p.coefficient_offset || off + need > p.coefficient_offset + p.coefficient_count)
            return fail(JXRB_INVALID_PLAN, "macroblock coefficient span outside its plane");
        const uint64_t rel = off - p.coefficient_offset;
        if (rel >= (1ull << 28)) return fail(JXRB_RESOURCE_LIMIT, "plane exceeds 2^28 coefficients");
        out.mbs[pos] = make_uint4((uint32_t)rel | ((uint32_t)bands << 28) | ((uint32_t)hp << 30), q0, q1, q2);
    }
    if (filled != n) return fail(JXRB_INVALID_PLAN, "reconstruction window has a macroblock with no coefficients");
    out.hard = g.hard_tiles ? 1 : 0;
    TRY(window_starts(g.tile_column_widths, g.tile_columns, g.macroblock_origin_x, g.macroblocks_x, out.col_start));
    TRY(window_starts(g.tile_row_heights, g.tile_rows, g.macroblock_origin_y, g.macroblocks_y, out.row_start));
    return JXRB_OK;
}

// ---------------------------------------------------------------------------
// pinned staging of uploads from pageable host memory
// ---------------------------------------------------------------------------

// Copies into the pinned staging buffers.  With AVX2 (x86-64 hosts), 32-byte
// loads and non-temporal 32-byte stores: a staging buffer is read next by the
// copy engine, never by this core, so streaming stores skip each destination
// line's read for ownership and keep the source's lines in the cache.
#if defined(__x86_64__)
__attribute__((target("avx2"))) static void stream_copy_avx2(uint8_t *d, const uint8_t *s, size_t n) {
    size_t i = 0;
    for (; i + 128 <= n; i += 128) {
        const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i));
        const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i + 32));
        const __m256i c = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i + 64));
        const __m256i e = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i + 96));
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i), a);
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i + 32), b);
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i + 64), c);
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i + 96), e);
    }
    _mm_sfence();
    if (i < n) std::memcpy(d + i, s + i, n - i);
}

static void stage_copy(uint8_t *d, const uint8_t *s, size_t n) {
    static const bool avx2 = __builtin_cpu_supports("avx2");
    if (avx2 && (reinterpret_cast<uintptr_t>(d) & 31) == 0) stream_copy_avx2(d, s, n);
    else std::memcpy(d, s, n);
}
#else
static void stage_copy(uint8_t *d, const uint8_t *s, size_t n) { std::memcpy(d, s, n); }
#endif

// Threads of the staging copy pool: JXRB_STAGING_THREADS when set (1 .. 64),
// else three quarters of the host's hardware threads, at most 12.  On a
// 16-thread host a 4096 x 4096 RGB8 decode end to end from pageable arenas
// ran at 2.6 Gpix/s with 4 threads, 3.1 with 8, 3.3 with 12 and 3.2 with 15,
// against 4.2 from page-locked arenas.
static unsigned staging_threads() {
    if (const char *v = std::getenv("JXRB_STAGING_THREADS")) {
        const long t = std::strtol(v, nullptr, 10);
        if (t >= 1 && t <= 64) return (unsigned)t;
    }
    return std::max(1u, std::min(12u, std::thread::hardware_concurrency() * 3 / 4));
}

// A memcpy split over a few worker threads and the caller: one thread cannot
// fill a PCIe Gen5 link from pageable memory, several can.
class CopyPool {
public:
    explicit CopyPool(unsigned threads) {
        for (unsigned i = 0; i < threads; i++) workers_.emplace_back([this] { loop(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread &t : workers_) t.join();
    }
    void copy(uint8_t *dst, const uint8_t *src, size_t n) {
        const size_t parts = std::min<size_t>(workers_.size() + 1, std::max<size_t>(1, n >> 20));
        if (parts <= 1) {
            std::memcpy(dst, src, n);
            return;
        }
        std::unique_lock<std::mutex> l(m_);
        dst_ = dst;
        src_ = src;
        n_ = n;
        parts_ = parts;
        next_ = 0;
        done_ = 0;
        generation_++;
        cv_.notify_all();
        take_parts(l);
        done_cv_.wait(l, [&] { return done_ == parts_; });
    }

private:
    // parts of the current copy, taken one at a time (called with the lock)
    void take_parts(std::unique_lock<std::mutex> &l) {
        while (next_ < parts_) {
            const size_t k = next_++, parts = parts_, n = n_;
            uint8_t *d = dst_;
            const uint8_t *sp = src_;
            l.unlock();
            const size_t chunk = ((n + parts - 1) / parts + 4095) & ~size_t(4095);
            const size_t at = k * chunk;
            if (at < n) stage_copy(d + at, sp + at, std::min(chunk, n - at));
            l.lock();
            if (++done_ == parts_) done_cv_.notify_all();
        }
    }
    void loop() {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> l(m_);
        for (;;) {
            cv_.wait(l, [&] { return stop_ || generation_ != seen; });
            if (stop_) return;
            seen = generation_;
            take_parts(l);
        }
    }
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    uint8_t *dst_ = nullptr;
    const uint8_t *src_ = nullptr;
    size_t n_ = 0, parts_ = 0, next_ = 0, done_ = 0;
    uint64_t generation_ = 0;
    bool stop_ = false;
};

// The session's pinned staging ring.  An upload from page-locked (or device)
// memory is one asynchronous copy that reads the source while the
// submission runs.  An upload from pageable memory goes through kSlots pinned
// buffers of kChunk bytes in turn: each chunk is copied into the next free
// buffer by the copy pool, then sent to the device asynchronously while the
// next chunk is staged -- double buffering, so the link stays busy -- and
// when the upload call returns the source has been read in full.  The
// reference uploads arenas with a blocking copy from pageable memory
// (crates/jxr-cuda/src/upload_cache.rs:92-94).  Used under the session lock.
class Staging {
public:
    static constexpr size_t kChunk = size_t(16) << 20;
    static constexpr int kSlots = 4;

    ~Staging() {
        for (Slot &sl : slots_) {
            if (sl.done) {
                cudaEventSynchronize(sl.done);
                cudaEventDestroy(sl.done);
            }
            if (sl.host) cudaFreeHost(sl.host);
        }
    }
    // bytes from `src` to device memory at `dst` on `stream`; `pinned` (when
    // not null) tells whether the source was read asynchronously
    jxrb_status upload(uint8_t *dst, const void *src, size_t bytes, cudaStream_t stream, bool *pinned = nullptr) {
        if (bytes == 0) return JXRB_OK;
        cudaPointerAttributes a{};
        const bool registered = cudaPointerGetAttributes(&a, src) == cudaSuccess && a.type != cudaMemoryTypeUnregistered;
        cudaGetLastError();
        if (pinned) *pinned = registered;
        if (registered) {
            CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, stream), "upload (page-locked source)");
            return JXRB_OK;
        }
        if (!slots_[0].host) {
            for (Slot &sl : slots_) {
                CUDA_TRY(cudaHostAlloc(&sl.host, kChunk, cudaHostAllocDefault), "cudaHostAlloc (staging)");
                CUDA_TRY(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "cudaEventCreate (staging)");
            }
        }
        const uint8_t *sp = static_cast<const uint8_t *>(src);
        for (size_t off = 0; off < bytes; off += kChunk) {
            const size_t n = std::min(kChunk, bytes - off);
            Slot &sl = slots_[next_];
            next_ = (next_ + 1) % kSlots;
            if (sl.pending) CUDA_TRY(cudaEventSynchronize(sl.done), "staging slot wait");
            pool_.copy(static_cast<uint8_t *>(sl.host), sp + off, n);
            CUDA_TRY(cudaMemcpyAsync(dst + off, sl.host, n, cudaMemcpyHostToDevice, stream), "upload (staged)");
            CUDA_TRY(cudaEventRecord(sl.done, stream), "staging slot event");
            sl.pending = true;
        }
        staged_ += bytes;
        return JXRB_OK;
    }
    uint64_t staged_bytes() const { return staged_; }

private:
    struct Slot {
        void *host = nullptr;
        cudaEvent_t done = nullptr;
        bool pending = false;
    };
    Slot slots_[kSlots];
    int next_ = 0;
    uint64_t staged_ = 0;
    CopyPool pool_{staging_threads()};
};

// ---------------------------------------------------------------------------
// device buffers of one launch set (one or more images)
// ---------------------------------------------------------------------------
struct DeviceSet {
    void *mem = nullptr;              // one allocation
    bool stream_ordered = false;      // allocated with cudaMallocAsync
    size_t bytes = 0;
    ImageDev *images = nullptr;
    WorkItemHost *items = nullptr;
    uint32_t *status = nullptr;
    uint32_t *counters = nullptr;     // two words a kernel segment (dynamic tile scheduling)
    uint32_t item_count = 0;
    uint32_t bounds[kSegments + 1] = {};   // work-list segment boundaries (engine.h)
    cudaStream_t side = nullptr;      // second stream for the other tiles' kernel
    bool own_side = true;             // created for this set (else the session's)
    cudaEvent_t fork = nullptr, join = nullptr;
    LaunchTuning tune{{0, 0, 0, 0, 0}, 1};
    int max_planes = 1;
    // quarter-resolution requests (request sets only)
    QuarterImage *quarters = nullptr;
    QuarterPlane *qplanes = nullptr;
    uint32_t q_count = 0, q_planes = 0, q_max_mbs = 0, q_max_samples = 0, q_max_rows = 0;
    bool q_two_level = false, q_sixteenth_sums = false;
    std::vector<uint8_t> host_quarter;  // descriptors and scale terms, uploaded in one copy
    std::vector<ImageDev> host_images;
    std::vector<WorkItemHost> host_items;
    // the callers' coefficients, copied by upload_coefficients after every
    // upload from the library's own (pageable) host memory
    struct CoefficientCopy { size_t at; const void *src; size_t bytes; };
    std::vector<CoefficientCopy> coefficient_copies;
    std::vector<uint32_t> image_items;   // first item of each image, + total
    std::vector<uint64_t> output_offsets;
    uint64_t output_bytes = 0;
    uint64_t upload_bytes = 0;
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Lay out, allocate and upload every input of `plans`; output pointers are
// bound later by bind_output.  Copies run on `stream`; the host buffers are
// read before this returns (a synchronize on pageable sources).
jxrb_status build_device_set(const jxrb_plan *const *plans, uint32_t count, cudaStream_t stream, DeviceSet &set,
                             Staging *staging = nullptr) {
    set.host_images.assign(count, ImageDev{});
    set.image_items.assign(count + 1, 0);
    set.output_offsets.assign(count, 0);
    const uint32_t T = (uint32_t)tile_mbs();
    // layout: images | items | status | per plane (table, starts) | coefficients
    size_t at = 0;
    const size_t images_at = at;
    at = align_up(at + sizeof(ImageDev) * count, 256);
    uint32_t items = 0;
    bool bits = false;
    for (uint32_t i = 0; i < count; i++) {
        set.image_items[i] = items;
        items += ((plans[i]->mbs_x + T - 1) / T) * ((plans[i]->mbs_y + T - 1) / T);
        set.output_offsets[i] = align_up(set.output_bytes, 256);
        set.output_bytes = set.output_offsets[i] + plans[i]->output_bytes;
        bits |= plans[i]->out.store == kStoreBits;
    }
    // 1-bit outputs set bits of bytes shared between tiles with 32-bit
    // atomics, which may touch the three bytes after the last one
    if (bits) set.output_bytes = align_up(set.output_bytes, 4);
    set.image_items[count] = items;
    set.item_count = items;
    const size_t items_at = at;
    at = align_up(at + sizeof(WorkItemHost) * items, 256);
    const size_t status_at = at;
    at = align_up(at + sizeof(uint32_t), 64);
    const size_t counters_at = at;
    at = align_up(at + kCounterWords * sizeof(uint32_t), 256);
    // every image's tables in one region (staged on the host and copied at
    // once: one copy from pageable memory, not three a plane), then the
    // coefficients
    struct Copy { size_t at; const void *src; size_t bytes; };
    std::vector<Copy> copies;
    std::vector<std::vector<size_t>> table_at(count), col_at(count), row_at(count);
    std::vector<size_t> coeff_at(count * 2, 0);
    const size_t tables_at = at;
    for (uint32_t i = 0; i < count; i++) {
        const jxrb_plan &p = *plans[i];
        for (const PlaneHost &ph : p.planes) {
            table_at[i].push_back(at);
            copies.push_back({at, ph.mbs.data(), ph.mbs.size() * sizeof(uint4)});
            at = align_up(at + ph.mbs.size() * sizeof(uint4), 256);
            col_at[i].push_back(at);
            copies.push_back({at, ph.col_start.data(), ph.col_start.size()});
            at = align_up(at + ph.col_start.size() + 1, 16);
            row_at[i].push_back(at);
            copies.push_back({at, ph.row_start.data(), ph.row_start.size()});
            at = align_up(at + ph.row_start.size() + 1, 256);
        }
    }
    const size_t tables_end = at;
    for (uint32_t i = 0; i < count; i++) {
        const jxrb_plan &p = *plans[i];
        for (int a = 0; a < 2; a++) {
            if (!p.coefficients[a]) continue;
            coeff_at[i * 2 + a] = at;
            set.coefficient_copies.push_back({at, p.coefficients[a], p.coefficient_count[a] * sizeof(int32_t)});
            at = align_up(at + p.coefficient_count[a] * sizeof(int32_t), 256);
        }
    }
    set.bytes = at;
    // stream-ordered allocation from the device pool: submissions reuse freed
    // blocks instead of paying cudaMalloc each time
    CUDA_TRY(cudaMallocAsync(&set.mem, set.bytes, stream), "cudaMallocAsync (inputs)");
    set.stream_ordered = true;
    uint8_t *base = static_cast<uint8_t *>(set.mem);
    set.images = reinterpret_cast<ImageDev *>(base + images_at);
    set.items = reinterpret_cast<WorkItemHost *>(base + items_at);
    set.status = reinterpret_cast<uint32_t *>(base + status_at);
    set.counters = reinterpret_cast<uint32_t *>(base + counters_at);
    set.host_items.resize(items);
    set.max_planes = 1;
    for (uint32_t i = 0; i < count; i++) {
        const jxrb_plan &p = *plans[i];
        ImageDev &im = set.host_images[i];
        std::memset(&im, 0, sizeof im);
        im.nplanes = p.nplanes;
        im.alpha = p.alpha;
        im.chroma = p.chroma;
        im.centering_x = p.centering_x;
        im.centering_y = p.centering_y;
        im.mbs_x = p.mbs_x;
        im.mbs_y = p.mbs_y;
        im.tiles_x = (p.mbs_x + T - 1) / T;
        im.tiles_y = (p.mbs_y + T - 1) / T;
        im.tile_mbs = T;
        im.first_item = set.image_items[i];
        im.out = p.out;
        set.max_planes = std::max(set.max_planes, (int)p.planes.size());
        for (size_t k = 0; k < p.planes.size(); k++) {
            const PlaneHost &ph = p.planes[k];
            PlaneDev &pd = im.plane[k];
            pd.coeff = reinterpret_cast<const int32_t *>(base + coeff_at[i * 2 + ph.arena]) + ph.coeff_offset;
            pd.mbs = reinterpret_cast<const uint4 *>(base + table_at[i][k]);
            pd.col_start = base + col_at[i][k];
            pd.row_start = base + row_at[i][k];
            pd.mbs_x = ph.mbs_x;
            pd.mbs_y = ph.mbs_y;
            pd.bc = ph.bc;
            pd.br = ph.br;
            pd.scale2 = ph.scale2;
            pd.overlap = ph.overlap;
            pd.hard = ph.hard;
            pd.mbs_stride = ph.mbs_x;
        }
        // interior tiles (interior_tile / interior_tile_420 in recon_kernel.cu)
        const uint32_t kind = interior_tag(p.planes, p.chroma, p.out);
        const PlaneHost &p0 = p.planes[0];
        const uint8_t *sx = p0.hard ? p0.col_start.data() : nullptr, *sy = p0.hard ? p0.row_start.data() : nullptr;
        uint32_t it = set.image_items[i];
        for (uint32_t ty = 0; ty < im.tiles_y; ty++)
            for (uint32_t tx = 0; tx < im.tiles_x; tx++) {
                const uint32_t tag = tile_tag(kind, tx, ty, T, p.mbs_x, p.mbs_y, sx, sy);
                set.host_items[it++] = WorkItemHost{i | tag << kTagShift, (uint16_t)tx, (uint16_t)ty};
            }
    }
    {
        std::vector<uint8_t> tables(tables_end - tables_at, 0);
        for (const Copy &c : copies)
            if (c.bytes) std::memcpy(tables.data() + (c.at - tables_at), c.src, c.bytes);
        if (!tables.empty()) {
            if (staging) TRY(staging->upload(base + tables_at, tables.data(), tables.size(), stream));
            else CUDA_TRY(cudaMemcpyAsync(base + tables_at, tables.data(), tables.size(), cudaMemcpyHostToDevice, stream),
                          "upload tables");
        }
        set.upload_bytes += tables.size();
    }
    // order the work list by kernel segment
    order_by_segment(set.host_items, set.bounds);
    CUDA_TRY(cudaMemcpyAsync(set.items, set.host_items.data(), sizeof(WorkItemHost) * items, cudaMemcpyHostToDevice,
                             stream), "upload work list");
    CUDA_TRY(cudaMemsetAsync(set.counters, 0, kCounterWords * sizeof(uint32_t), stream), "counter reset");
    CUDA_TRY(cudaMemsetAsync(set.status, 0, sizeof(uint32_t), stream), "status reset");
    // the other tiles' kernel runs on a second stream beside the interior ones
    if (set.bounds[kSegments] > set.bounds[kSideSegment0] && set.bounds[kSideSegment0] > 0 && !set.side) {
        CUDA_TRY(cudaStreamCreateWithFlags(&set.side, cudaStreamNonBlocking), "cudaStreamCreate");
        CUDA_TRY(cudaEventCreateWithFlags(&set.fork, cudaEventDisableTiming), "cudaEventCreate");
        CUDA_TRY(cudaEventCreateWithFlags(&set.join, cudaEventDisableTiming), "cudaEventCreate");
    }
    return JXRB_OK;
}

// The callers' coefficients to the device, after every other upload of the
// set: a copy from pageable host memory (the library's tables, work list and
// descriptors) waits for its stream's earlier work, so behind these copies it
// would hold the caller until every coefficient had crossed; from pinned
// memory these are asynchronous.
jxrb_status upload_coefficients(DeviceSet &set, cudaStream_t stream, Staging *staging = nullptr) {
    uint8_t *base = static_cast<uint8_t *>(set.mem);
    for (const DeviceSet::CoefficientCopy &c : set.coefficient_copies) {
        if (c.bytes == 0) continue;
        if (staging) TRY(staging->upload(base + c.at, c.src, c.bytes, stream));
        else CUDA_TRY(cudaMemcpyAsync(base + c.at, c.src, c.bytes, cudaMemcpyHostToDevice, stream), "upload coefficients");
        set.upload_bytes += c.bytes;
    }
    set.coefficient_copies.clear();
    return JXRB_OK;
}

// Bind the output surfaces (dense, plan order, 256-byte aligned) and upload
// the image descriptors.
jxrb_status bind_output(DeviceSet &set, uint8_t *dst, cudaStream_t stream) {
    for (size_t i = 0; i < set.host_images.size(); i++) set.host_images[i].out.base = dst + set.output_offsets[i];
    CUDA_TRY(cudaMemcpyAsync(set.images, set.host_images.data(), sizeof(ImageDev) * set.host_images.size(),
                             cudaMemcpyHostToDevice, stream), "upload image descriptors");
    for (size_t i = 0; i < set.host_images.size(); i++) {
        if (set.host_images[i].out.store == kStoreBits) {
            const uint64_t end = i + 1 < set.host_images.size() ? set.output_offsets[i + 1] : set.output_bytes;
            const uint64_t n = end - set.output_offsets[i];
            CUDA_TRY(cudaMemsetAsync(dst + set.output_offsets[i], 0, n, stream), "clear bit output");
        }
    }
    return JXRB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// session / submission objects
// ---------------------------------------------------------------------------
struct jxrb_session {
    int device = 0;
    std::vector<cudaStream_t> streams;
    std::vector<cudaStream_t> sides;   // per stream: where requests' edge-tile kernels run beside it
    std::atomic<uint32_t> next_stream{0};
    std::mutex lock;   // serialises encoding of submissions (runtime.rs:42)
    std::atomic<uint64_t> submissions{0}, uploaded{0}, read_back{0}, held{0}, launches{0};
    std::unique_ptr<Staging> staging;  // pinned ring for pageable sources, made at the first submission (under `lock`)
    cudaStream_t upload = nullptr;     // uploads of resident images
};

namespace {

// The stream of the next submission: the first idle one (its earlier work
// done) in turn from the session's cursor, else the next in turn.  Uploads
// from pageable host memory wait for their stream's earlier work, so a busy
// stream would stall the caller until a previous submission finishes.
size_t pick_stream(jxrb_session *s) {
    const size_t n = s->streams.size();
    const size_t start = s->next_stream++ % n;
    for (size_t d = 0; d < n; d++) {
        const size_t k = (start + d) % n;
        const cudaError_t a = cudaStreamQuery(s->streams[k]);
        const cudaError_t b = a == cudaSuccess ? cudaStreamQuery(s->sides[k]) : a;
        if (a != cudaSuccess || b != cudaSuccess) cudaGetLastError();   // not-ready is no error to report later
        if (a == cudaSuccess && b == cudaSuccess) return k;
    }
    return start;
}

}  // namespace

struct jxrb_submission {
    jxrb_session *session = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    // device-timed stages of plan submissions (jxrb_submission_report):
    // recorded before the first upload and before the first launch; `done`
    // then times the end of the reconstruction
    cudaEvent_t begin = nullptr, launched = nullptr;
    double readback_ms = 0.0;     // host-timed copies back (jxrb_readback / _all)
    DeviceSet set;
    void *owned_output = nullptr;
    uint8_t *output = nullptr;
    bool waited = false;
    jxrb_status result = JXRB_OK;
    uint32_t status_word = 0;
};

struct jxrb_resident {
    jxrb_session *session = nullptr;
    DeviceSet set;
    std::vector<DeviceSet> singles;  // per-image sets sharing nothing (per-image launches)
    uint8_t *bound = nullptr;
    cudaGraphExec_t graph = nullptr; // captured launch sequence (jxrb_resident_capture)
    cudaStream_t capture = nullptr;  // stream the capture is recorded on
};

// One plane of a resident image: where its table and tile-start maps sit in
// the image's device allocation, and the host copies the planner needs.
struct ImagePlane {
    int arena = 0;
    uint64_t coeff_offset = 0;
    int bc = 4, br = 4, scale2 = 0, overlap = 0, hard = 0;
    std::vector<uint8_t> col_start, row_start;   // whole image
    std::vector<uint64_t> prefix;                // 2-D prefix sums of input bytes a macroblock
    std::vector<uint32_t> dc_only;               // 2-D prefix counts of macroblocks coding the DC band alone
    size_t table_at = 0, col_at = 0, row_at = 0;
};

// An image whose coefficients, macroblock tables and tile maps stay on the
// device (the reference's upload cache entry, upload_cache.rs:65-153), so
// that each request on it uploads only an image descriptor and a work list.
struct jxrb_image {
    jxrb_session *session = nullptr;
    uint8_t *mem = nullptr;
    size_t bytes = 0;
    size_t coeff_at[2] = {0, 0};
    std::vector<ImagePlane> planes;
    int nplanes = 0, alpha = -1, chroma = 0, ncomp = 0;
    uint32_t mbs_x = 0, mbs_y = 0;
    jxrb_image_geometry geom{};
    std::vector<uint32_t> tile_w, tile_h;
    // quarter-resolution sample scales by plane and window (calibrated once)
    mutable std::mutex scale_lock;
    mutable std::map<std::vector<uint32_t>, std::shared_ptr<const QuarterScale>> scales;
};

// A decode of (a region of) a resident image into one output format.
struct jxrb_request {
    const jxrb_image *image = nullptr;
    uint32_t ox = 0, oy = 0, wx = 0, wy = 0;    // reconstruction window, macroblocks
    OutputDev out{};
    uint64_t output_bytes = 0, traffic_bytes = 0;
    int denominator = 1;                        // 1: full resolution, 4: a quarter, 16: a sixteenth
    std::vector<std::shared_ptr<const QuarterScale>> scales;   // per plane (quarter)
};

namespace {

jxrb_status check_session(jxrb_session *s) {
    if (!s) return fail(JXRB_INVALID_SUBMISSION_STATE, "null session");
    CUDA_TRY(cudaSetDevice(s->device), "cudaSetDevice");
    return JXRB_OK;
}

void release_set(DeviceSet &set) {
    if (set.side && set.own_side) {
        cudaStreamSynchronize(set.side);
        cudaStreamDestroy(set.side);
    }
    set.side = nullptr;
    if (set.fork) cudaEventDestroy(set.fork);
    if (set.join) cudaEventDestroy(set.join);
    set.fork = set.join = nullptr;
}

jxrb_status launch_set(jxrb_session *s, DeviceSet &set, cudaStream_t stream) {
    cudaError_t e = launch_tiles(set.images, set.items, set.bounds, set.max_planes, set.status, set.counters, stream,
                                 set.side, set.fork, set.join, &set.tune);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    for (int k = 0; k < kSegments; k++) s->launches += set.bounds[k + 1] > set.bounds[k];
    if (set.q_count) {
        e = launch_quarter(set.images, set.quarters, set.q_count, set.qplanes, set.q_planes, set.q_two_level,
                           set.q_sixteenth_sums, set.q_max_mbs, set.q_max_samples, set.q_max_rows, set.status, stream);
        if (e != cudaSuccess) return cuda_fail(e, "reduced-resolution launch");
        s->launches += 3 + (set.q_two_level ? 3 : 0) + (set.q_sixteenth_sums ? 1 : 0);
    }
    return JXRB_OK;
}

jxrb_status status_to_error(uint32_t word) {
    if (word == 0) return JXRB_OK;
    g_stage = word;
    if (word == kStatusInvalid) return fail(JXRB_INVALID_PLAN, "invalid macroblock metadata met on the device");
    char buf[96];
    std::snprintf(buf, sizeof buf, "integer overflow in reconstruction stage %u", word);
    return fail(JXRB_KERNEL_ARITHMETIC, buf);
}

jxrb_status submit_common(jxrb_session *s, const jxrb_plan *const *plans, uint32_t count, void *dst, uint64_t dst_len,
                          jxrb_submission **out) {
    TRY(check_session(s));
    if (!out) return fail(JXRB_INVALID_SUBMISSION_STATE, "null submission out-pointer");
    if (count == 0) return fail(JXRB_INVALID_PLAN, "empty batch");
    if (count > kImageMask) return fail(JXRB_RESOURCE_LIMIT, "too many images in one launch");
    for (uint32_t i = 0; i < count; i++)
        if (!plans[i]) return fail(JXRB_INVALID_PLAN, "null plan");
    std::unique_ptr<jxrb_submission> sub(new jxrb_submission);
    sub->session = s;
    sub->stream = s->streams[pick_stream(s)];
    std::lock_guard<std::mutex> guard(s->lock);
    CUDA_TRY(cudaEventCreate(&sub->begin), "cudaEventCreate");
    CUDA_TRY(cudaEventCreate(&sub->launched), "cudaEventCreate");
    CUDA_TRY(cudaEventRecord(sub->begin, sub->stream), "cudaEventRecord");
    if (!s->staging) s->staging.reset(new Staging);
    TRY(build_device_set(plans, count, sub->stream, sub->set, s->staging.get()));
    if (dst) {
        if (dst_len < sub->set.output_bytes) return fail(JXRB_INVALID_DESTINATION, "destination is smaller than the output");
        sub->output = static_cast<uint8_t *>(dst);
    } else {
        CUDA_TRY(cudaMallocAsync(&sub->owned_output, std::max<uint64_t>(sub->set.output_bytes, 1), sub->stream),
                 "cudaMallocAsync (output)");
        sub->output = static_cast<uint8_t *>(sub->owned_output);
    }
    TRY(bind_output(sub->set, sub->output, sub->stream));
    TRY(upload_coefficients(sub->set, sub->stream, s->staging.get()));
    CUDA_TRY(cudaEventRecord(sub->launched, sub->stream), "cudaEventRecord");
    TRY(launch_set(s, sub->set, sub->stream));
    CUDA_TRY(cudaEventCreate(&sub->done), "cudaEventCreate");
    CUDA_TRY(cudaEventRecord(sub->done, sub->stream), "cudaEventRecord");
    s->submissions++;
    s->uploaded += sub->set.upload_bytes;
    *out = sub.release();
    return JXRB_OK;
}

// Colour planes and chroma subsampling of a coded colour format.
jxrb_status color_planes(const jxrb_image_geometry &g, int &ncomp, int &chroma) {
    ncomp = g.components;
    chroma = 0;
    switch (g.color_format) {
    case JXRB_COLOR_LUMA: ncomp = 1; break;
    case JXRB_COLOR_YUV420: ncomp = 3; chroma = 1; break;
    case JXRB_COLOR_YUV422: ncomp = 3; chroma = 2; break;
    case JXRB_COLOR_YUV444: ncomp = 3; break;
    case JXRB_COLOR_YUVK: ncomp = 4; break;
    case JXRB_COLOR_NCOMPONENT:
        if (ncomp < 1 || ncomp > 4) return fail(JXRB_UNSUPPORTED_OUTPUT, "N-component images of 1 to 4 components");
        break;
    default: return fail(JXRB_INVALID_PLAN, "coded colour format");
    }
    return JXRB_OK;
}

// The planes of a plan: every colour plane's (and the alpha plane's)
// macroblock table over the window, validated against its arena
// (CudaDecodePlan::from_prepared's build_planes, crates/jxr-cuda/src/plan.rs:405-610).
jxrb_status build_plan_planes(const jxrb_arena *primary, const jxrb_arena *alpha, const jxrb_image_geometry *g,
                              jxrb_plan &plan) {
    jxrb_plan *p = &plan;
    if (g->macroblocks_x == 0 || g->macroblocks_y == 0) return fail(JXRB_INVALID_PLAN, "empty reconstruction window");
    if (g->macroblocks_x > 65535u * 4 || g->macroblocks_y > 65535u * 4) return fail(JXRB_RESOURCE_LIMIT, "window too large");
    if (g->overlap < 0 || g->overlap > 2 || g->alpha_overlap < 0 || g->alpha_overlap > 2)
        return fail(JXRB_INVALID_PLAN, "overlap mode");
    int ncomp = 0, chroma = 0;
    TRY(color_planes(*g, ncomp, chroma));
    const bool has_alpha = g->alpha_mode != JXRB_ALPHA_NONE;
    if (g->alpha_mode == JXRB_ALPHA_SEPARATE && !alpha) return fail(JXRB_INVALID_PLAN, "separate alpha arena missing");
    p->coefficients[0] = primary->coefficients;
    p->coefficient_count[0] = primary->coefficient_count;
    p->nplanes = ncomp;
    p->chroma = chroma;
    p->centering_x = g->chroma_centering_x;
    p->centering_y = g->chroma_centering_y;
    p->mbs_x = g->macroblocks_x;
    p->mbs_y = g->macroblocks_y;
    const uint32_t expected_planes = ncomp + (g->alpha_mode == JXRB_ALPHA_INTEGRATED ? 1 : 0);
    if (primary->plane_count != expected_planes) return fail(JXRB_INVALID_PLAN, "arena plane count differs from the colour format");
    for (int c = 0; c < ncomp; c++) {
        PlaneHost ph;
        const int bc = (chroma && c > 0 && c < 3) ? 2 : 4;
        const int br = (chroma == 1 && c > 0 && c < 3) ? 2 : 4;
        TRY(build_plane(*primary, c, *g, bc, br, ph));
        ph.arena = 0;
        ph.overlap = g->overlap;
        // crates/jxr-core/src/image.rs:77-85: every component after the first
        ph.scale2 = g->scaled && c != 0;
        p->planes.push_back(std::move(ph));
    }
    if (has_alpha) {
        PlaneHost ph;
        if (g->alpha_mode == JXRB_ALPHA_INTEGRATED) {
            TRY(build_plane(*primary, ncomp, *g, 4, 4, ph));
            ph.arena = 0;
        } else {
            if (alpha->plane_count < 1) return fail(JXRB_INVALID_PLAN, "separate alpha arena has no plane");
            TRY(build_plane(*alpha, 0, *g, 4, 4, ph));
            ph.arena = 1;
            p->coefficients[1] = alpha->coefficients;
            p->coefficient_count[1] = alpha->coefficient_count;
        }
        ph.overlap = g->alpha_overlap;
        ph.scale2 = 0;  // an alpha plane's one component is the first
        p->alpha = (int)p->planes.size();
        p->planes.push_back(std::move(ph));
    }
    return JXRB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// descriptors of one plan laid out in a fixed device region, for the
// allocation-free entry point of static_scratch.cu
// ---------------------------------------------------------------------------
namespace jxr {

jxrb_status report_error(jxrb_status s, const char *why) { return fail(s, why); }
jxrb_status report_cuda(cudaError_t e, const char *what) { return cuda_fail(e, what); }
jxrb_status report_status_word(uint32_t word) { return status_to_error(word); }

// Bytes of the layout stage_plan writes for `plan`.
size_t staged_bytes(const jxrb_plan &p) {
    const uint32_t T = (uint32_t)tile_mbs();
    const size_t items = (size_t)((p.mbs_x + T - 1) / T) * ((p.mbs_y + T - 1) / T);
    size_t at = align_up(sizeof(ImageDev), 256);
    at = align_up(at + sizeof(WorkItemHost) * items, 256);
    at = align_up(at + sizeof(uint32_t), 64);
    at = align_up(at + kCounterWords * sizeof(uint32_t), 256);
    for (const PlaneHost &ph : p.planes) {
        at = align_up(at + ph.mbs.size() * sizeof(uint4), 256);
        at = align_up(at + ph.col_start.size() + 1, 16);
        at = align_up(at + ph.row_start.size() + 1, 256);
    }
    return at;
}

// Write the descriptors of `plan` into `host` (at most `capacity` bytes),
// with every pointer aimed at the device region `device` that the caller
// fills from `host` with one copy.  The status word and the counters are
// zero in the copy.  Coefficients stay where the caller put them on the
// device; `dst` is the caller's device output.  Allocates nothing.
jxrb_status stage_plan(const jxrb_plan *plan, const int32_t *coefficients, const int32_t *alpha_coefficients,
                       uint8_t *dst, uint64_t dst_bytes, uint8_t *host, uint8_t *device, size_t capacity,
                       StagedLayout &layout) {
    if (!plan) return fail(JXRB_INVALID_PLAN, "null plan");
    const jxrb_plan &p = *plan;
    const size_t need = staged_bytes(p);
    if (need > capacity) {
        char buf[160];
        std::snprintf(buf, sizeof buf,
                      "plan needs %zu bytes of descriptor scratch; the allocation-free path holds at most %zu",
                      need, capacity);
        return fail(JXRB_RESOURCE_LIMIT, buf);
    }
    const bool bits = p.out.store == kStoreBits;
    const uint64_t out_bytes = bits ? align_up(p.output_bytes, 4) : p.output_bytes;
    if (!dst || dst_bytes < out_bytes) return fail(JXRB_INVALID_DESTINATION, "destination is smaller than the output");
    for (const PlaneHost &ph : p.planes) {
        if (ph.arena == 0 && !coefficients) return fail(JXRB_INVALID_PLAN, "null device coefficients");
        if (ph.arena == 1 && !alpha_coefficients) return fail(JXRB_INVALID_PLAN, "null device alpha coefficients");
    }
    std::memset(host, 0, need);
    const uint32_t T = (uint32_t)tile_mbs();
    const uint32_t tiles_x = (p.mbs_x + T - 1) / T, tiles_y = (p.mbs_y + T - 1) / T;
    const size_t items = (size_t)tiles_x * tiles_y;
    layout.bytes = need;
    layout.items_at = align_up(sizeof(ImageDev), 256);
    layout.status_at = align_up(layout.items_at + sizeof(WorkItemHost) * items, 256);
    layout.counters_at = align_up(layout.status_at + sizeof(uint32_t), 64);
    layout.clear_bytes = bits ? out_bytes : 0;
    size_t at = align_up(layout.counters_at + kCounterWords * sizeof(uint32_t), 256);

    ImageDev &im = *reinterpret_cast<ImageDev *>(host);
    im.nplanes = p.nplanes;
    im.alpha = p.alpha;
    im.chroma = p.chroma;
    im.centering_x = p.centering_x;
    im.centering_y = p.centering_y;
    im.mbs_x = p.mbs_x;
    im.mbs_y = p.mbs_y;
    im.tiles_x = tiles_x;
    im.tiles_y = tiles_y;
    im.tile_mbs = T;
    im.first_item = 0;
    im.out = p.out;
    im.out.base = dst;
    for (size_t k = 0; k < p.planes.size(); k++) {
        const PlaneHost &ph = p.planes[k];
        PlaneDev &pd = im.plane[k];
        pd.coeff = (ph.arena ? alpha_coefficients : coefficients) + ph.coeff_offset;
        std::memcpy(host + at, ph.mbs.data(), ph.mbs.size() * sizeof(uint4));
        pd.mbs = reinterpret_cast<const uint4 *>(device + at);
        at = align_up(at + ph.mbs.size() * sizeof(uint4), 256);
        std::memcpy(host + at, ph.col_start.data(), ph.col_start.size());
        pd.col_start = device + at;
        at = align_up(at + ph.col_start.size() + 1, 16);
        std::memcpy(host + at, ph.row_start.data(), ph.row_start.size());
        pd.row_start = device + at;
        at = align_up(at + ph.row_start.size() + 1, 256);
        pd.mbs_x = ph.mbs_x;
        pd.mbs_y = ph.mbs_y;
        pd.bc = ph.bc;
        pd.br = ph.br;
        pd.scale2 = ph.scale2;
        pd.overlap = ph.overlap;
        pd.hard = ph.hard;
        pd.mbs_stride = ph.mbs_x;
    }
    // work list in kernel segments, as the submissions order it (the
    // conditions of build_device_set): the interior tiles, then the rest
    const int np = (int)p.planes.size();
    const uint32_t kind = interior_tag(p.planes, p.chroma, p.out);
    const PlaneHost &p0 = p.planes[0];
    const uint8_t *sx = p0.hard ? p0.col_start.data() : nullptr, *sy = p0.hard ? p0.row_start.data() : nullptr;
    // count the tiles of each segment, then place each at its segment's cursor
    uint32_t count[kSegments] = {};
    for (uint32_t ty = 0; ty < tiles_y; ty++)
        for (uint32_t tx = 0; tx < tiles_x; tx++)
            count[segment_of_tag(tile_tag(kind, tx, ty, T, p.mbs_x, p.mbs_y, sx, sy))]++;
    uint32_t cursor[kSegments];
    layout.bounds[0] = 0;
    for (int s = 0; s < kSegments; s++) {
        cursor[s] = layout.bounds[s];
        layout.bounds[s + 1] = layout.bounds[s] + count[s];
    }
    layout.max_planes = std::max(1, np);
    WorkItemHost *list = reinterpret_cast<WorkItemHost *>(host + layout.items_at);
    for (uint32_t ty = 0; ty < tiles_y; ty++)
        for (uint32_t tx = 0; tx < tiles_x; tx++) {
            const uint32_t tag = tile_tag(kind, tx, ty, T, p.mbs_x, p.mbs_y, sx, sy);
            list[cursor[segment_of_tag(tag)]++] = WorkItemHost{tag << kTagShift, (uint16_t)tx, (uint16_t)ty};
        }
    return JXRB_OK;
}

}  // namespace jxr

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int jxrb_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) return 0;
    return prop.major == 10 ? 1 : 0;
}

const char *jxrb_last_error(void) { return g_error.c_str(); }

uint32_t jxrb_last_stage(void) { return g_stage; }

jxrb_status jxrb_session_create(int ordinal, const jxrb_session_options *options, jxrb_session **out) {
    if (!out) return fail(JXRB_INVALID_SUBMISSION_STATE, "null session out-pointer");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(JXRB_UNAVAILABLE, "no CUDA device");
    }
    if (ordinal < 0 || ordinal >= n) return fail(JXRB_UNAVAILABLE, "device ordinal out of range");
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, ordinal), "cudaGetDeviceProperties");
    if (prop.major != 10) return fail(JXRB_UNSUPPORTED_DEVICE, "the engine is built for sm_100 (B200)");
    CUDA_TRY(cudaSetDevice(ordinal), "cudaSetDevice");
    {
        // keep freed submission memory in the device pool for the next one
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, ordinal) == cudaSuccess) {
            uint64_t keep = options && options->scratch_bytes ? options->scratch_bytes : UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    std::unique_ptr<jxrb_session> s(new jxrb_session);
    s->device = ordinal;
    const uint32_t streams = options && options->streams ? options->streams : 4;
    for (uint32_t i = 0; i < streams; i++) {
        cudaStream_t st, side;
        CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        s->streams.push_back(st);
        CUDA_TRY(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), "cudaStreamCreate");
        s->sides.push_back(side);
    }
    CUDA_TRY(cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking), "cudaStreamCreate");
    *out = s.release();
    return JXRB_OK;
}

void jxrb_session_destroy(jxrb_session *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
    for (cudaStream_t st : s->sides) cudaStreamSynchronize(st);
    if (s->upload) cudaStreamSynchronize(s->upload);
    s->staging.reset();
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    for (cudaStream_t st : s->sides) cudaStreamDestroy(st);
    if (s->upload) cudaStreamDestroy(s->upload);
    delete s;
}

jxrb_status jxrb_session_diagnostics(const jxrb_session *s, jxrb_diagnostics *out) {
    if (!s || !out) return fail(JXRB_INVALID_SUBMISSION_STATE, "null argument");
    out->submissions = s->submissions;
    out->bytes_uploaded = s->uploaded;
    out->bytes_read_back = s->read_back;
    out->device_bytes_held = s->held;
    out->kernel_launches = s->launches;
    out->bytes_staged = s->staging ? s->staging->staged_bytes() : 0;
    return JXRB_OK;
}

jxrb_status jxrb_plan_create(const jxrb_arena *primary, const jxrb_arena *alpha, const jxrb_image_geometry *g,
                             const jxrb_output_format *output, jxrb_plan **out) {
    if (!primary || !g || !output || !out) return fail(JXRB_INVALID_PLAN, "null argument");
    std::unique_ptr<jxrb_plan> p(new jxrb_plan);
    int ncomp = 0, chroma = 0;
    TRY(color_planes(*g, ncomp, chroma));
    const int color = g->color_format;
    if (chroma && (g->chroma_centering_x < 0 || g->chroma_centering_x > 4 || g->chroma_centering_y < 0 ||
                   g->chroma_centering_y > 4) && output->output_color != color)
        return fail(JXRB_UNSUPPORTED_OUTPUT, "unknown chroma centering has no exact reconstruction filter");
    const bool has_alpha = g->alpha_mode != JXRB_ALPHA_NONE;
    TRY(build_plan_planes(primary, alpha, g, *p));
    const int oc = output->output_color;
    const int internal = (chroma && !(oc == color)) ? JXRB_COLOR_YUV444 : color;
    if (output->crop_width == 0 || output->crop_height == 0) return fail(JXRB_INVALID_PLAN, "empty crop");
    if ((uint64_t)output->crop_x + output->crop_width > (uint64_t)g->macroblocks_x * 16 ||
        (uint64_t)output->crop_y + output->crop_height > (uint64_t)g->macroblocks_y * 16)
        return fail(JXRB_INVALID_PLAN, "crop window lies outside the reconstruction window");
    if ((oc == JXRB_COLOR_YUV420 || oc == JXRB_COLOR_YUV422) && (output->crop_x & 1))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "planar chroma crop must start on an even column");
    if (oc == JXRB_COLOR_YUV420 && (output->crop_y & 1))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "planar 4:2:0 crop must start on an even row");
    TRY(build_output(*output, internal, ncomp, has_alpha, g->scaled, g->alpha_scaled, p->out, p->output_bytes));
    uint64_t traffic = p->output_bytes;
    for (const PlaneHost &ph : p->planes) traffic += ph.mbs.size() * sizeof(uint4);
    p->metadata_bytes = traffic - p->output_bytes;
    for (const PlaneHost &ph : p->planes) {
        // coefficients each macroblock stores
        for (const uint4 &e : ph.mbs) traffic += 4 * coefficients_per_macroblock((e.x >> 28) & 3, ph.bc * ph.br);
    }
    p->traffic_bytes = traffic;
    *out = p.release();
    return JXRB_OK;
}

void jxrb_plan_destroy(jxrb_plan *plan) { delete plan; }

uint64_t jxrb_plan_output_bytes(const jxrb_plan *plan) { return plan ? plan->output_bytes : 0; }

uint64_t jxrb_plan_traffic_bytes(const jxrb_plan *plan) { return plan ? plan->traffic_bytes : 0; }

jxrb_status jxrb_plan_tile_kinds(const jxrb_plan *plan, jxrb_tile_kinds *out) {
    if (!plan) return fail(JXRB_INVALID_PLAN, "null plan");
    if (!out) return fail(JXRB_INVALID_DESTINATION, "null result");
    const jxrb_plan &p = *plan;
    const uint32_t T = (uint32_t)tile_mbs();
    const uint32_t kind = interior_tag(p.planes, p.chroma, p.out);
    const PlaneHost &p0 = p.planes[0];
    const uint8_t *sx = p0.hard ? p0.col_start.data() : nullptr, *sy = p0.hard ? p0.row_start.data() : nullptr;
    *out = jxrb_tile_kinds{};
    for (uint32_t ty = 0; ty < (p.mbs_y + T - 1) / T; ty++)
        for (uint32_t tx = 0; tx < (p.mbs_x + T - 1) / T; tx++) {
            const uint32_t tag = tile_tag(kind, tx, ty, T, p.mbs_x, p.mbs_y, sx, sy);
            if (tag == 0) out->general++;
            else if (tag == kTagEdge420) out->edge_420++;
            else if (tag > kTagEdge) out->edge++;
            else if (tag == kTag420) out->interior_420++;
            else out->interior++;
        }
    return JXRB_OK;
}

jxrb_status jxrb_submit(jxrb_session *s, const jxrb_plan *plan, jxrb_submission **out) {
    return submit_common(s, &plan, 1, nullptr, 0, out);
}

jxrb_status jxrb_submit_into(jxrb_session *s, const jxrb_plan *plan, void *dst, uint64_t dst_len, jxrb_submission **out) {
    if (!dst) return fail(JXRB_INVALID_DESTINATION, "null destination");
    return submit_common(s, &plan, 1, dst, dst_len, out);
}

jxrb_status jxrb_submit_batch(jxrb_session *s, const jxrb_plan *const *plans, uint32_t count, void *dst, uint64_t dst_len,
                              jxrb_submission **out) {
    if (!plans) return fail(JXRB_INVALID_PLAN, "null plan list");
    return submit_common(s, plans, count, dst, dst_len, out);
}

jxrb_status jxrb_wait(jxrb_submission *sub, int64_t timeout_ns) {
    if (!sub) return fail(JXRB_INVALID_SUBMISSION_STATE, "null submission");
    if (sub->waited) return sub->result;
    CUDA_TRY(cudaSetDevice(sub->session->device), "cudaSetDevice");
    if (timeout_ns >= 0) {
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::nanoseconds(timeout_ns);
        for (;;) {
            cudaError_t q = cudaEventQuery(sub->done);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return cuda_fail(q, "cudaEventQuery");
            if (std::chrono::steady_clock::now() >= deadline) return fail(JXRB_TIMEOUT, "submission still running");
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    } else {
        CUDA_TRY(cudaEventSynchronize(sub->done), "cudaEventSynchronize");
    }
    CUDA_TRY(cudaMemcpy(&sub->status_word, sub->set.status, sizeof(uint32_t), cudaMemcpyDeviceToHost), "status read");
    sub->waited = true;
    sub->result = status_to_error(sub->status_word);
    return sub->result;
}

jxrb_status jxrb_is_complete(jxrb_submission *sub, int *complete) {
    if (!sub || !complete) return fail(JXRB_INVALID_SUBMISSION_STATE, "null argument");
    cudaError_t q = cudaEventQuery(sub->done);
    if (q == cudaErrorNotReady) { *complete = 0; return JXRB_OK; }
    if (q != cudaSuccess) return cuda_fail(q, "cudaEventQuery");
    *complete = 1;
    return JXRB_OK;
}

jxrb_status jxrb_enqueue_consumer_wait(jxrb_submission *sub, void *stream) {
    if (!sub) return fail(JXRB_INVALID_SUBMISSION_STATE, "null submission");
    CUDA_TRY(cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), sub->done, 0), "cudaStreamWaitEvent");
    return JXRB_OK;
}

void *jxrb_submission_device_ptr(jxrb_submission *sub, uint32_t index) {
    if (!sub || index >= sub->set.output_offsets.size()) return nullptr;
    return sub->output + sub->set.output_offsets[index];
}

jxrb_status jxrb_readback(jxrb_submission *sub, uint32_t index, void *host, uint64_t bytes) {
    TRY(jxrb_wait(sub, -1));
    if (index >= sub->set.output_offsets.size()) return fail(JXRB_INVALID_DESTINATION, "image index out of range");
    const ImageDev &im = sub->set.host_images[index];
    (void)im;
    const uint64_t end = index + 1 < sub->set.output_offsets.size() ? sub->set.output_offsets[index + 1] : sub->set.output_bytes;
    const uint64_t avail = end - sub->set.output_offsets[index];
    if (bytes > avail) return fail(JXRB_INVALID_DESTINATION, "readback larger than the image output");
    const auto t0 = std::chrono::steady_clock::now();
    CUDA_TRY(cudaMemcpy(host, sub->output + sub->set.output_offsets[index], bytes, cudaMemcpyDeviceToHost), "readback");
    sub->readback_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    sub->session->read_back += bytes;
    return JXRB_OK;
}

jxrb_status jxrb_readback_all(jxrb_submission *sub, void *host, uint64_t bytes) {
    TRY(jxrb_wait(sub, -1));
    if (!host && bytes) return fail(JXRB_INVALID_DESTINATION, "null host buffer");
    if (bytes > sub->set.output_bytes) return fail(JXRB_INVALID_DESTINATION, "readback larger than the outputs");
    const auto t0 = std::chrono::steady_clock::now();
    CUDA_TRY(cudaMemcpy(host, sub->output, bytes, cudaMemcpyDeviceToHost), "readback");
    sub->readback_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    sub->session->read_back += bytes;
    return JXRB_OK;
}

void jxrb_submission_destroy(jxrb_submission *sub) {
    if (!sub) return;
    cudaSetDevice(sub->session->device);
    if (sub->done) {
        cudaEventSynchronize(sub->done);
        cudaEventDestroy(sub->done);
    }
    if (sub->begin) cudaEventDestroy(sub->begin);
    if (sub->launched) cudaEventDestroy(sub->launched);
    release_set(sub->set);
    if (sub->set.mem) cudaFreeAsync(sub->set.mem, sub->stream);
    if (sub->owned_output) cudaFreeAsync(sub->owned_output, sub->stream);
    delete sub;
}

jxrb_status jxrb_decode_to_host(jxrb_session *s, const jxrb_plan *plan, void *host, uint64_t bytes) {
    jxrb_submission *sub = nullptr;
    TRY(jxrb_submit(s, plan, &sub));
    jxrb_status st = jxrb_readback(sub, 0, host, std::min<uint64_t>(bytes, plan->output_bytes));
    jxrb_submission_destroy(sub);
    return st;
}

jxrb_status jxrb_session_create_default(jxrb_session **out) { return jxrb_session_create(0, nullptr, out); }

jxrb_status jxrb_plan_route(int request, uint64_t reconstructed_coefficients, int cuda_usable, int resident_output,
                            int *decision) {
    // plan_cuda_route, crates/jxr-cuda/src/route.rs:23-49
    if (!decision) return fail(JXRB_INVALID_PLAN, "null decision");
    if (request < JXRB_BACKEND_AUTO || request > JXRB_BACKEND_METAL) return fail(JXRB_UNSUPPORTED_BACKEND, "backend request");
    if (resident_output) {
        if (request == JXRB_BACKEND_CPU)
            return fail(JXRB_RESIDENT_OUTPUT_REQUIRES_CUDA, "CUDA-resident output requires the CUDA backend");
        if (request == JXRB_BACKEND_METAL) return fail(JXRB_UNSUPPORTED_BACKEND, "the CUDA adapter does not serve Metal");
        if (!cuda_usable) return fail(JXRB_UNAVAILABLE, "CUDA is unavailable on this host");
        *decision = JXRB_ROUTE_CUDA;
        return JXRB_OK;
    }
    switch (request) {
    case JXRB_BACKEND_METAL: return fail(JXRB_UNSUPPORTED_BACKEND, "the CUDA adapter does not serve Metal");
    case JXRB_BACKEND_CUDA:
        if (!cuda_usable) return fail(JXRB_UNAVAILABLE, "CUDA is unavailable on this host");
        *decision = JXRB_ROUTE_CUDA;
        return JXRB_OK;
    case JXRB_BACKEND_AUTO:
        *decision = cuda_usable && reconstructed_coefficients >= JXRB_CUDA_AUTO_THRESHOLD ? JXRB_ROUTE_CUDA
                                                                                         : JXRB_ROUTE_CPU;
        return JXRB_OK;
    default:
        *decision = JXRB_ROUTE_CPU;
        return JXRB_OK;
    }
}

uint64_t jxrb_plan_reconstructed_coefficients(const jxrb_plan *plan) {
    // the samples every plane reconstructs (the route's work measure)
    if (!plan) return 0;
    uint64_t n = 0;
    for (const PlaneHost &ph : plan->planes) n += (uint64_t)ph.mbs_x * ph.mbs_y * 16ull * ph.bc * ph.br;
    return n;
}

jxrb_status jxrb_plan_output_layout(const jxrb_plan *plan, jxrb_surface_layout *out) {
    // SurfaceLayout (crates/jxr-core/src/surface.rs:19-142) of the plan's output
    if (!plan || !out) return fail(JXRB_INVALID_PLAN, "null argument");
    const OutputDev &o = plan->out;
    std::memset(out, 0, sizeof *out);
    out->width = o.crop_w;
    out->height = o.crop_h;
    out->byte_len = plan->output_bytes;
    out->element_bytes = (uint32_t)o.elem_bytes;
    auto plane = [&](uint32_t k, uint64_t offset, uint64_t stride, uint32_t w, uint32_t h, uint32_t channels) {
        out->planes[k] = jxrb_surface_plane{offset, stride, w, h, channels};
        out->plane_count = k + 1;
    };
    const uint64_t w = o.crop_w, h = o.crop_h, e = (uint64_t)o.elem_bytes;
    if (o.planar_yuv) {
        const uint64_t cw = w / 2, ch = o.planar_yuv == 1 ? h / 2 : h;
        plane(0, 0, w * e, (uint32_t)w, (uint32_t)h, 1);
        plane(1, w * h * e, cw * e, (uint32_t)cw, (uint32_t)ch, 1);
        plane(2, (w * h + cw * ch) * e, cw * e, (uint32_t)cw, (uint32_t)ch, 1);
        if (plan->alpha >= 0) plane(3, (w * h + 2 * cw * ch) * e, w * e, (uint32_t)w, (uint32_t)h, 1);
    } else if (o.nchw) {
        for (int c = 0; c < o.channels && c < 6; c++) plane((uint32_t)c, c * o.plane_stride, o.row_stride, (uint32_t)w,
                                                             (uint32_t)h, 1);
    } else {
        plane(0, 0, o.row_stride, (uint32_t)w, (uint32_t)h, (uint32_t)o.channels);
    }
    return JXRB_OK;
}

jxrb_status jxrb_allocate_destination(jxrb_session *s, uint64_t bytes, void **device_destination) {
    // allocate_destination, crates/jxr-cuda/src/session.rs:85-92: zeroed device memory the caller owns
    TRY(check_session(s));
    if (!device_destination) return fail(JXRB_INVALID_DESTINATION, "null out-pointer");
    void *p = nullptr;
    CUDA_TRY(cudaMalloc(&p, std::max<uint64_t>(bytes, 1)), "cudaMalloc (destination)");
    cudaError_t e = cudaMemset(p, 0, std::max<uint64_t>(bytes, 1));
    if (e != cudaSuccess) {
        cudaFree(p);
        return cuda_fail(e, "cudaMemset (destination)");
    }
    *device_destination = p;
    return JXRB_OK;
}

jxrb_status jxrb_batch_layout(const jxrb_plan *const *plans, uint32_t count, uint64_t *offsets, uint64_t *bytes) {
    // the dense batch layout of jxrb_submit_batch: plan order, each output
    // 256-byte aligned (DenseCudaBatchLayout, crates/jxr-cuda/src/destination.rs)
    if (!plans || !bytes || count == 0) return fail(JXRB_INVALID_PLAN, "empty batch");
    uint64_t at = 0;
    bool bits = false;
    for (uint32_t i = 0; i < count; i++) {
        if (!plans[i]) return fail(JXRB_INVALID_PLAN, "null plan");
        at = align_up(at, 256);
        if (offsets) offsets[i] = at;
        at += plans[i]->output_bytes;
        bits |= plans[i]->out.store == kStoreBits;
    }
    *bytes = bits ? align_up(at, 4) : at;
    return JXRB_OK;
}

jxrb_status jxrb_allocate_batch_destination(jxrb_session *s, const jxrb_plan *const *plans, uint32_t count,
                                            void **device_destination, uint64_t *bytes) {
    // allocate_batch_destination, crates/jxr-cuda/src/session.rs:94-101
    uint64_t n = 0;
    TRY(jxrb_batch_layout(plans, count, nullptr, &n));
    TRY(jxrb_allocate_destination(s, n, device_destination));
    if (bytes) *bytes = n;
    return JXRB_OK;
}

jxrb_status jxrb_free_destination(jxrb_session *s, void *device_destination) {
    TRY(check_session(s));
    if (device_destination) CUDA_TRY(cudaFree(device_destination), "cudaFree (destination)");
    return JXRB_OK;
}

jxrb_status jxrb_decode_batch_to_host(jxrb_session *s, const jxrb_plan *const *plans, uint32_t count,
                                      void *const *hosts, const uint64_t *bytes) {
    // decode_batch_to_host, crates/jxr-cuda/src/session.rs:221-235: caller
    // order kept, one launch for the batch, each image to its own host buffer
    if (!hosts || !bytes) return fail(JXRB_INVALID_DESTINATION, "null host buffers");
    jxrb_submission *sub = nullptr;
    TRY(jxrb_submit_batch(s, plans, count, nullptr, 0, &sub));
    jxrb_status st = JXRB_OK;
    for (uint32_t i = 0; i < count && st == JXRB_OK; i++)
        st = jxrb_readback(sub, i, hosts[i], std::min<uint64_t>(bytes[i], plans[i]->output_bytes));
    jxrb_submission_destroy(sub);
    return st;
}

jxrb_status jxrb_submission_report(jxrb_submission *sub, jxrb_decode_report *out) {
    // decode_report, crates/jxr-cuda/src/plan.rs:214-253: the host stages
    // before the arena, the reconstruction stages on CUDA, the readback on
    // the host when one ran; plus device-timed upload and reconstruction
    if (!sub || !out) return fail(JXRB_INVALID_SUBMISSION_STATE, "null argument");
    TRY(jxrb_wait(sub, -1));
    std::memset(out, 0, sizeof *out);
    out->requested_backend = JXRB_BACKEND_CUDA;
    out->selected_backend = JXRB_ROUTE_CUDA;
    out->fallback = 0;
    uint32_t n = 0;
    for (int st = JXRB_STAGE_PARSE; st <= JXRB_STAGE_DC_LOW_PASS_PREDICTION; st++)
        out->stages[n++] = jxrb_stage_report{st, JXRB_EXECUTOR_CPU_SCALAR};
    for (int st = JXRB_STAGE_DEQUANTIZE_FIRST_TRANSFORM; st <= JXRB_STAGE_CROP_CLIP_PACK; st++)
        out->stages[n++] = jxrb_stage_report{st, JXRB_EXECUTOR_CUDA};
    if (sub->readback_ms > 0.0)
        out->stages[n++] = jxrb_stage_report{JXRB_STAGE_HOST_READBACK, JXRB_EXECUTOR_CPU_SCALAR};
    out->stage_count = n;
    float ms = 0.f;
    if (sub->begin && sub->launched && cudaEventElapsedTime(&ms, sub->begin, sub->launched) == cudaSuccess)
        out->upload_ms = ms;
    if (sub->launched && sub->done && cudaEventElapsedTime(&ms, sub->launched, sub->done) == cudaSuccess)
        out->reconstruct_ms = ms;
    cudaGetLastError();   // events without timing (request submissions) report zero
    out->readback_ms = (float)sub->readback_ms;
    return JXRB_OK;
}

jxrb_status jxrb_resident_create(jxrb_session *s, const jxrb_plan *const *plans, uint32_t count, jxrb_resident **out) {
    TRY(check_session(s));
    if (!plans || !out || count == 0) return fail(JXRB_INVALID_PLAN, "empty resident set");
    std::unique_ptr<jxrb_resident> r(new jxrb_resident);
    r->session = s;
    cudaStream_t st = s->streams[0];
    TRY(build_device_set(plans, count, st, r->set));
    r->singles.resize(count);
    for (uint32_t i = 0; i < count; i++) TRY(build_device_set(&plans[i], 1, st, r->singles[i]));
    TRY(upload_coefficients(r->set, st));
    for (DeviceSet &d : r->singles) TRY(upload_coefficients(d, st));
    CUDA_TRY(cudaStreamSynchronize(st), "resident upload");
    uint64_t held = r->set.bytes;
    for (auto &d : r->singles) held += d.bytes;
    s->held += held;
    *out = r.release();
    return JXRB_OK;
}

static jxrb_status resident_bind(jxrb_resident *r, void *dst, uint64_t dst_len, cudaStream_t st) {
    if (!dst || dst_len < r->set.output_bytes) return fail(JXRB_INVALID_DESTINATION, "destination is smaller than the output");
    uint8_t *d = static_cast<uint8_t *>(dst);
    if (r->bound != d) {
        TRY(bind_output(r->set, d, st));
        for (size_t i = 0; i < r->singles.size(); i++) TRY(bind_output(r->singles[i], d + r->set.output_offsets[i], st));
        r->bound = d;
    }
    return JXRB_OK;
}

jxrb_status jxrb_resident_run(jxrb_resident *r, void *dst, uint64_t dst_len, int batched, void *stream) {
    if (!r) return fail(JXRB_INVALID_SUBMISSION_STATE, "null resident set");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : r->session->streams[0];
    TRY(resident_bind(r, dst, dst_len, st));
    if (batched) {
        TRY(launch_set(r->session, r->set, st));
    } else {
        for (auto &one : r->singles) TRY(launch_set(r->session, one, st));
    }
    return JXRB_OK;
}

jxrb_status jxrb_resident_set_tuning(jxrb_resident *r, const jxrb_launch_tuning *t) {
    if (!r || !t) return fail(JXRB_INVALID_SUBMISSION_STATE, "null argument");
    LaunchTuning lt;
    for (int k = 0; k < 5; k++) lt.blocks_per_sm[k] = t->blocks_per_sm[k];
    lt.side_stream = t->side_stream ? 1 : 0;
    r->set.tune = lt;
    for (auto &one : r->singles) one.tune = lt;
    return JXRB_OK;
}

jxrb_status jxrb_resident_capture(jxrb_resident *r, void *dst, uint64_t dst_len, int batched) {
    if (!r) return fail(JXRB_INVALID_SUBMISSION_STATE, "null resident set");
    CUDA_TRY(cudaSetDevice(r->session->device), "cudaSetDevice");
    if (!r->capture) CUDA_TRY(cudaStreamCreateWithFlags(&r->capture, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaStream_t st = r->capture;
    // descriptors are bound outside the graph: it holds the launches only
    TRY(resident_bind(r, dst, dst_len, st));
    CUDA_TRY(cudaStreamSynchronize(st), "bind");
    if (r->graph) {
        cudaGraphExecDestroy(r->graph);
        r->graph = nullptr;
    }
    CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    jxrb_status launched = JXRB_OK;
    if (batched) {
        launched = launch_set(r->session, r->set, st);
    } else {
        for (auto &one : r->singles) {
            launched = launch_set(r->session, one, st);
            if (launched != JXRB_OK) break;
        }
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (launched != JXRB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return launched;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&r->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        r->graph = nullptr;
        return cuda_fail(e, "cudaGraphInstantiate");
    }
    return JXRB_OK;
}

jxrb_status jxrb_resident_replay(jxrb_resident *r, void *stream) {
    if (!r || !r->graph) return fail(JXRB_INVALID_SUBMISSION_STATE, "no captured launch sequence");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : r->session->streams[0];
    CUDA_TRY(cudaGraphLaunch(r->graph, st), "cudaGraphLaunch");
    return JXRB_OK;
}

jxrb_status jxrb_resident_status(jxrb_resident *r, uint32_t *status) {
    if (!r || !status) return fail(JXRB_INVALID_SUBMISSION_STATE, "null argument");
    uint32_t word = 0, w = 0;
    CUDA_TRY(cudaMemcpy(&w, r->set.status, sizeof w, cudaMemcpyDeviceToHost), "status read");
    word = w;
    for (auto &one : r->singles) {
        CUDA_TRY(cudaMemcpy(&w, one.status, sizeof w, cudaMemcpyDeviceToHost), "status read");
        if (!word) word = w;
    }
    *status = word;
    return status_to_error(word);
}

uint64_t jxrb_resident_output_bytes(const jxrb_resident *r) { return r ? r->set.output_bytes : 0; }

uint32_t jxrb_resident_launches(const jxrb_resident *r, int batched) {
    // kernel launches of one run: one per non-empty work-list segment
    if (!r) return 0;
    auto segments = [](const DeviceSet &d) {
        uint32_t n = 0;
        for (int s = 0; s < kSegments; s++) n += d.bounds[s + 1] > d.bounds[s];
        return n;
    };
    if (batched) return segments(r->set);
    uint32_t n = 0;
    for (const DeviceSet &d : r->singles) n += segments(d);
    return n;
}

void jxrb_resident_destroy(jxrb_resident *r) {
    if (!r) return;
    cudaSetDevice(r->session->device);
    for (cudaStream_t st : r->session->streams) cudaStreamSynchronize(st);
    cudaStream_t st = r->session->streams[0];
    if (r->graph) cudaGraphExecDestroy(r->graph);
    if (r->capture) {
        cudaStreamSynchronize(r->capture);
        cudaStreamDestroy(r->capture);
    }
    release_set(r->set);
    if (r->set.mem) cudaFreeAsync(r->set.mem, st);
    for (auto &d : r->singles) {
        release_set(d);
        if (d.mem) cudaFreeAsync(d.mem, st);
    }
    cudaStreamSynchronize(st);
    delete r;
}

}  // extern "C"

namespace {

// Input bytes of the macroblocks [x0, x1) x [y0, y1) of a resident plane.
uint64_t rect_bytes(const ImagePlane &p, uint32_t stride, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1) {
    const uint32_t w = stride + 1;
    return p.prefix[(size_t)y1 * w + x1] - p.prefix[(size_t)y0 * w + x1] - p.prefix[(size_t)y1 * w + x0] +
           p.prefix[(size_t)y0 * w + x0];
}

// The work items and descriptors of a batch of requests.
jxrb_status build_request_set(jxrb_session *s, const jxrb_request *const *reqs, uint32_t count, size_t side_index,
                              cudaStream_t stream, DeviceSet &set) {
    set.host_images.assign(count, ImageDev{});
    set.image_items.assign(count + 1, 0);
    set.output_offsets.assign(count, 0);
    const uint32_t T = (uint32_t)tile_mbs();
    uint32_t items = 0;
    bool bits = false;
    for (uint32_t i = 0; i < count; i++) {
        const jxrb_request &r = *reqs[i];
        set.image_items[i] = items;
        if (r.denominator == 1) items += ((r.wx + T - 1) / T) * ((r.wy + T - 1) / T);
        set.output_offsets[i] = align_up(set.output_bytes, 256);
        set.output_bytes = set.output_offsets[i] + r.output_bytes;
        bits |= r.out.store == kStoreBits;
    }
    if (bits) set.output_bytes = align_up(set.output_bytes, 4);
    set.image_items[count] = items;
    set.item_count = items;
    size_t at = align_up(sizeof(ImageDev) * count, 256);
    const size_t items_at = at;
    at = align_up(at + sizeof(WorkItemHost) * items, 256);
    const size_t status_at = at;
    at = align_up(at + sizeof(uint32_t), 64);
    const size_t counters_at = at;
    at = align_up(at + kCounterWords * sizeof(uint32_t), 256);
    // quarter-resolution requests: their image and plane descriptors and scale
    // terms (one host blob, one copy), then their pictures
    struct QPlaneAt { size_t divisor = 0, bias = 0, cols = 0, rows = 0, pic = 0, out = 0; };
    std::vector<QPlaneAt> qat;
    const size_t q_at = at;
    for (uint32_t i = 0; i < count; i++)
        if (reqs[i]->denominator != 1) {
            set.q_count++;
            set.q_planes += (uint32_t)reqs[i]->image->planes.size();
        }
    const size_t qimages_at = q_at;
    at = align_up(at + sizeof(QuarterImage) * set.q_count, 16);
    const size_t qplanes_at = at;
    at = align_up(at + sizeof(QuarterPlane) * set.q_planes, 256);
    for (uint32_t i = 0; i < count; i++) {
        const jxrb_request &r = *reqs[i];
        if (r.denominator == 1) continue;
        for (size_t k = 0; k < r.image->planes.size(); k++) {
            const QuarterScale &q = *r.scales[k];
            QPlaneAt a;
            if (q.shift < 0) {
                a.divisor = at; at = align_up(at + 8 * q.divisor.size(), 16);
                a.bias = at; at = align_up(at + 8 * q.bias.size(), 16);
                a.cols = at; at = align_up(at + 4 * q.columns.size(), 16);
                a.rows = at; at = align_up(at + 4 * q.rows.size(), 16);
            }
            qat.push_back(a);
        }
    }
    const size_t q_end = align_up(at, 256);
    at = q_end;
    {
        size_t n = 0;
        for (uint32_t i = 0; i < count; i++) {
            const jxrb_request &r = *reqs[i];
            if (r.denominator == 1) continue;
            for (const ImagePlane &ip : r.image->planes) {
                QPlaneAt &a = qat[n++];
                // the block picture: a quarter's own; a sixteenth's when two
                // filter levels need it; a sixteenth's macroblock picture
                const bool blocks = r.denominator == 4 || ip.overlap == 2;
                if (blocks) {
                    a.pic = at;
                    at = align_up(at + 4ull * r.wx * ip.bc * r.wy * ip.br, 256);
                }
                a.out = a.pic;
                if (r.denominator == 16) {
                    a.out = at;
                    at = align_up(at + 4ull * r.wx * r.wy, 256);
                }
            }
        }
    }
    set.bytes = at;
    CUDA_TRY(cudaMallocAsync(&set.mem, set.bytes, stream), "cudaMallocAsync (descriptors)");
    set.stream_ordered = true;
    uint8_t *base = static_cast<uint8_t *>(set.mem);
    set.images = reinterpret_cast<ImageDev *>(base);
    set.items = reinterpret_cast<WorkItemHost *>(base + items_at);
    set.status = reinterpret_cast<uint32_t *>(base + status_at);
    set.counters = reinterpret_cast<uint32_t *>(base + counters_at);
    set.quarters = reinterpret_cast<QuarterImage *>(base + qimages_at);
    set.qplanes = reinterpret_cast<QuarterPlane *>(base + qplanes_at);
    set.host_quarter.assign(q_end - q_at, 0);
    uint32_t qi = 0, qp = 0;
    set.host_items.resize(items);
    set.max_planes = 1;
    for (uint32_t i = 0; i < count; i++) {
        const jxrb_request &r = *reqs[i];
        const jxrb_image &img = *r.image;
        ImageDev &im = set.host_images[i];
        std::memset(&im, 0, sizeof im);
        im.nplanes = img.nplanes;
        im.alpha = img.alpha;
        // a sixteenth has a chroma sample for each macroblock, as luma does
        im.chroma = r.denominator == 16 ? 0 : img.chroma;
        im.centering_x = img.geom.chroma_centering_x;
        im.centering_y = img.geom.chroma_centering_y;
        im.mbs_x = r.wx;
        im.mbs_y = r.wy;
        im.tiles_x = r.denominator == 1 ? (r.wx + T - 1) / T : 0;
        im.tiles_y = r.denominator == 1 ? (r.wy + T - 1) / T : 0;
        im.tile_mbs = T;
        im.first_item = set.image_items[i];
        im.out = r.out;
        if (r.denominator != 1) {
            const bool sixteenth = r.denominator == 16;
            uint8_t *blob = set.host_quarter.data();
            QuarterImage &q = reinterpret_cast<QuarterImage *>(blob + (qimages_at - q_at))[qi++];
            q.image = i;
            q.first_plane = qp;
            q.planes = (uint32_t)img.planes.size();
            q.width = sixteenth ? r.wx : r.wx * 4;
            q.height = sixteenth ? r.wy : r.wy * 4;
            set.q_max_rows = std::max(set.q_max_rows, q.height);
            for (size_t k = 0; k < img.planes.size(); k++, qp++) {
                const ImagePlane &ip = img.planes[k];
                const QuarterScale &sc = *r.scales[k];
                const QPlaneAt &a = qat[qp];
                QuarterPlane &d = reinterpret_cast<QuarterPlane *>(blob + (qplanes_at - q_at))[qp];
                d.coeff = reinterpret_cast<const int32_t *>(img.mem + img.coeff_at[ip.arena]) + ip.coeff_offset;
                d.mbs = reinterpret_cast<const uint4 *>(img.mem + ip.table_at) + (size_t)r.oy * img.mbs_x + r.ox;
                d.col_start = img.mem + ip.col_at + r.ox;
                d.row_start = img.mem + ip.row_at + r.oy;
                d.pic = a.pic ? reinterpret_cast<int32_t *>(base + a.pic) : nullptr;
                d.out = reinterpret_cast<int32_t *>(base + a.out);
                d.sixteenth = sixteenth ? 1 : 0;
                d.mbs_x = r.wx;
                d.mbs_y = r.wy;
                d.mbs_stride = img.mbs_x;
                d.bc = ip.bc;
                d.br = ip.br;
                d.scale2 = ip.scale2;
                d.overlap = ip.overlap;
                d.hard = ip.hard;
                d.shift = sc.shift;
                d.gain = sc.gain;
                d.probe_stride = sc.probe_stride;
                if (sc.shift < 0) {
                    std::memcpy(blob + (a.divisor - q_at), sc.divisor.data(), 8 * sc.divisor.size());
                    std::memcpy(blob + (a.bias - q_at), sc.bias.data(), 8 * sc.bias.size());
                    std::memcpy(blob + (a.cols - q_at), sc.columns.data(), 4 * sc.columns.size());
                    std::memcpy(blob + (a.rows - q_at), sc.rows.data(), 4 * sc.rows.size());
                    d.divisor = reinterpret_cast<const int64_t *>(base + a.divisor);
                    d.bias = reinterpret_cast<const int64_t *>(base + a.bias);
                    d.cols = reinterpret_cast<const uint32_t *>(base + a.cols);
                    d.rows = reinterpret_cast<const uint32_t *>(base + a.rows);
                }
                set.q_two_level |= ip.overlap == 2;
                set.q_sixteenth_sums |= sixteenth && ip.overlap == 2;
                set.q_max_mbs = std::max(set.q_max_mbs, r.wx * r.wy);
                set.q_max_samples = std::max(set.q_max_samples, r.wx * ip.bc * r.wy * ip.br);
            }
        }
        set.max_planes = std::max(set.max_planes, (int)img.planes.size());
        for (size_t k = 0; k < img.planes.size(); k++) {
            const ImagePlane &ip = img.planes[k];
            PlaneDev &pd = im.plane[k];
            pd.coeff = reinterpret_cast<const int32_t *>(img.mem + img.coeff_at[ip.arena]) + ip.coeff_offset;
            pd.mbs = reinterpret_cast<const uint4 *>(img.mem + ip.table_at) + (size_t)r.oy * img.mbs_x + r.ox;
            pd.col_start = img.mem + ip.col_at + r.ox;
            pd.row_start = img.mem + ip.row_at + r.oy;
            pd.mbs_x = r.wx;
            pd.mbs_y = r.wy;
            pd.bc = ip.bc;
            pd.br = ip.br;
            pd.scale2 = ip.scale2;
            pd.overlap = ip.overlap;
            pd.hard = ip.hard;
            pd.mbs_stride = img.mbs_x;
        }
        // interior tiles: the conditions of build_device_set, on the window
        // (interior tiles never touch its first macroblock row or column)
        const uint32_t kind = interior_tag(img.planes, img.chroma, r.out);
        const ImagePlane &p0 = img.planes[0];
        const uint8_t *sx = p0.hard ? p0.col_start.data() + r.ox : nullptr;
        const uint8_t *sy = p0.hard ? p0.row_start.data() + r.oy : nullptr;
        uint32_t it = set.image_items[i];
        for (uint32_t ty = 0; ty < im.tiles_y; ty++)
            for (uint32_t tx = 0; tx < im.tiles_x; tx++) {
                const uint32_t tag = tile_tag(kind, tx, ty, T, r.wx, r.wy, sx, sy);
                set.host_items[it++] = WorkItemHost{i | tag << kTagShift, (uint16_t)tx, (uint16_t)ty};
            }
    }
    order_by_segment(set.host_items, set.bounds);
    if (items)
        CUDA_TRY(cudaMemcpyAsync(set.items, set.host_items.data(), sizeof(WorkItemHost) * items,
                                 cudaMemcpyHostToDevice, stream), "upload work list");
    if (!set.host_quarter.empty())
        CUDA_TRY(cudaMemcpyAsync(base + q_at, set.host_quarter.data(), set.host_quarter.size(), cudaMemcpyHostToDevice,
                                 stream), "upload quarter-resolution descriptors");
    CUDA_TRY(cudaMemsetAsync(set.counters, 0, kCounterWords * sizeof(uint32_t), stream), "counter reset");
    CUDA_TRY(cudaMemsetAsync(set.status, 0, sizeof(uint32_t), stream), "status reset");
    if (set.bounds[kSegments] > set.bounds[kSideSegment0] && set.bounds[kSideSegment0] > 0) {
        set.side = s->sides[side_index];
        set.own_side = false;
        CUDA_TRY(cudaEventCreateWithFlags(&set.fork, cudaEventDisableTiming), "cudaEventCreate");
        CUDA_TRY(cudaEventCreateWithFlags(&set.join, cudaEventDisableTiming), "cudaEventCreate");
    }
    return JXRB_OK;
}

}  // namespace

extern "C" {

jxrb_status jxrb_image_create(jxrb_session *s, const jxrb_arena *primary, const jxrb_arena *alpha,
                              const jxrb_image_geometry *g, jxrb_image **out) {
    TRY(check_session(s));
    if (!primary || !g || !out) return fail(JXRB_INVALID_PLAN, "null argument");
    if (g->macroblock_origin_x || g->macroblock_origin_y)
        return fail(JXRB_INVALID_PLAN, "a resident image covers the whole coded image (window origin 0)");
    uint64_t cols = 0, rows = 0;
    for (uint32_t i = 0; i < g->tile_columns; i++) cols += g->tile_column_widths[i];
    for (uint32_t i = 0; i < g->tile_rows; i++) rows += g->tile_row_heights[i];
    if (cols != g->macroblocks_x || rows != g->macroblocks_y)
        return fail(JXRB_INVALID_PLAN, "tile grid differs from the image's macroblocks");
    jxrb_plan plan;
    TRY(build_plan_planes(primary, alpha, g, plan));
    std::unique_ptr<jxrb_image> img(new jxrb_image);
    img->session = s;
    img->nplanes = plan.nplanes;
    img->alpha = plan.alpha;
    img->chroma = plan.chroma;
    img->mbs_x = plan.mbs_x;
    img->mbs_y = plan.mbs_y;
    img->geom = *g;
    img->tile_w.assign(g->tile_column_widths, g->tile_column_widths + g->tile_columns);
    img->tile_h.assign(g->tile_row_heights, g->tile_row_heights + g->tile_rows);
    img->geom.tile_column_widths = img->tile_w.data();
    img->geom.tile_row_heights = img->tile_h.data();
    int ncomp = 0, chroma = 0;
    TRY(color_planes(*g, ncomp, chroma));
    img->ncomp = ncomp;
    struct Copy { size_t at; const void *src; size_t bytes; };
    std::vector<Copy> copies;
    size_t at = 0;
    for (int a = 0; a < 2; a++) {
        if (!plan.coefficients[a]) continue;
        img->coeff_at[a] = at;
        copies.push_back({at, plan.coefficients[a], plan.coefficient_count[a] * sizeof(int32_t)});
        at = align_up(at + plan.coefficient_count[a] * sizeof(int32_t), 256);
    }
    for (const PlaneHost &ph : plan.planes) {
        ImagePlane ip;
        ip.arena = ph.arena;
        ip.coeff_offset = ph.coeff_offset;
        ip.bc = ph.bc;
        ip.br = ph.br;
        ip.scale2 = ph.scale2;
        ip.overlap = ph.overlap;
        ip.hard = ph.hard;
        ip.col_start = ph.col_start;
        ip.row_start = ph.row_start;
        ip.table_at = at;
        copies.push_back({at, ph.mbs.data(), ph.mbs.size() * sizeof(uint4)});
        at = align_up(at + ph.mbs.size() * sizeof(uint4), 256);
        ip.col_at = at;
        copies.push_back({at, ip.col_start.data(), ip.col_start.size()});
        at = align_up(at + ip.col_start.size() + 1, 16);
        ip.row_at = at;
        copies.push_back({at, ip.row_start.data(), ip.row_start.size()});
        at = align_up(at + ip.row_start.size() + 1, 256);
        const uint32_t w = plan.mbs_x + 1;
        ip.prefix.assign((size_t)(plan.mbs_y + 1) * w, 0);
        ip.dc_only.assign((size_t)(plan.mbs_y + 1) * w, 0);
        for (uint32_t y = 0; y < plan.mbs_y; y++)
            for (uint32_t x = 0; x < plan.mbs_x; x++) {
                const uint4 &e = ph.mbs[(size_t)y * plan.mbs_x + x];
                const uint64_t b = 16 + 4 * coefficients_per_macroblock((e.x >> 28) & 3, ph.bc * ph.br);
                const size_t i = (size_t)(y + 1) * w + x + 1, up = (size_t)y * w + x + 1, left = i - 1, diag = up - 1;
                ip.prefix[i] = b + ip.prefix[up] + ip.prefix[left] - ip.prefix[diag];
                ip.dc_only[i] = (((e.x >> 28) & 3) == 0) + ip.dc_only[up] + ip.dc_only[left] - ip.dc_only[diag];
            }
        img->planes.push_back(std::move(ip));
    }
    img->bytes = at;
    // on the session's upload stream, through its pinned staging ring, so
    // that an upload on admission waits for no batch in flight
    std::lock_guard<std::mutex> guard(s->lock);
    cudaStream_t st = s->upload;
    if (!s->staging) s->staging.reset(new Staging);
    void *mem = nullptr;
    CUDA_TRY(cudaMallocAsync(&mem, img->bytes, st), "cudaMallocAsync (resident image)");
    img->mem = static_cast<uint8_t *>(mem);
    for (const Copy &c : copies) {
        if (!c.bytes) continue;
        const jxrb_status e = s->staging->upload(img->mem + c.at, c.src, c.bytes, st);
        if (e != JXRB_OK) {
            cudaFreeAsync(mem, st);
            return e;
        }
    }
    CUDA_TRY(cudaStreamSynchronize(st), "resident image upload");
    s->uploaded += img->bytes;
    s->held += img->bytes;
    *out = img.release();
    return JXRB_OK;
}

uint64_t jxrb_image_device_bytes(const jxrb_image *img) { return img ? img->bytes : 0; }

void jxrb_image_destroy(jxrb_image *img) {
    if (!img) return;
    jxrb_session *s = img->session;
    cudaSetDevice(s->device);
    // Stream-ordered release, with no host wait: the memory returns to the
    // pool once every stream of the session has finished the work enqueued
    // so far (requests on this image among it).  A serving loop evicting
    // images under its budget keeps its batches in flight meanwhile.
    bool ordered = img->mem != nullptr;
    for (size_t k = 0; ordered && k < s->streams.size() + s->sides.size(); k++) {
        cudaStream_t st = k < s->streams.size() ? s->streams[k] : s->sides[k - s->streams.size()];
        if (st == s->streams[0]) continue;
        cudaEvent_t e = nullptr;
        ordered = cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventRecord(e, st) == cudaSuccess && cudaStreamWaitEvent(s->streams[0], e, 0) == cudaSuccess;
        if (e) cudaEventDestroy(e);
    }
    if (img->mem) {
        if (!ordered) {
            // the ordering could not be set up: wait for every stream instead
            cudaGetLastError();
            for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
            for (cudaStream_t st : s->sides) cudaStreamSynchronize(st);
        }
        cudaFreeAsync(img->mem, s->streams[0]);
    }
    s->held -= img->bytes;
    delete img;
}

jxrb_status jxrb_request_create(const jxrb_image *img, const jxrb_output_format *output, jxrb_request **out) {
    return jxrb_request_create_scaled(img, output, 1, out);
}

jxrb_status jxrb_request_create_scaled(const jxrb_image *img, const jxrb_output_format *output, int denominator,
                                       jxrb_request **out) {
    if (!img || !output || !out) return fail(JXRB_INVALID_PLAN, "null argument");
    if (denominator != 1 && denominator != 4 && denominator != 16)
        return fail(JXRB_UNSUPPORTED_OUTPUT, "reduced resolution: a quarter (denominator 4) or a sixteenth (16)");
    const jxrb_image_geometry &g = img->geom;
    const uint64_t W = (uint64_t)img->mbs_x * 16, H = (uint64_t)img->mbs_y * 16;
    const uint64_t x = output->crop_x, y = output->crop_y, w = output->crop_width, h = output->crop_height;
    if (w == 0 || h == 0) return fail(JXRB_INVALID_PLAN, "empty crop");
    if (x + w > W || y + h > H) return fail(JXRB_INVALID_PLAN, "region lies outside the image");
    const int oc = output->output_color;
    const bool subsampled_out = oc == JXRB_COLOR_YUV420 || oc == JXRB_COLOR_YUV422;
    if (img->chroma && (g.chroma_centering_x < 0 || g.chroma_centering_x > 4 || g.chroma_centering_y < 0 ||
                        g.chroma_centering_y > 4) && oc != g.color_format)
        return fail(JXRB_UNSUPPORTED_OUTPUT, "unknown chroma centering has no exact reconstruction filter");
    // macroblocks the region needs: those it covers and one more on each side
    // where overlap filtering or chroma interpolation reaches
    // (reconstruction_bounds, crates/jxr-native/src/prepare.rs:321-352)
    // a sixteenth has a chroma sample for each macroblock: nothing to
    // interpolate, and no subsampled planes to store (prepare.rs:185-192,
    // interpolates_chroma, crates/jxr-native/src/metadata.rs:255-263)
    if (denominator == 16 && subsampled_out)
        return fail(JXRB_UNSUPPORTED_OUTPUT, "sixteenth-resolution subsampled planar YUV output");
    const bool interpolates = img->chroma && !subsampled_out && denominator != 16;
    const uint32_t halo = (g.overlap != 0 || interpolates) ? 1u : 0u;
    const uint32_t b0 = (uint32_t)(x / 16) > halo ? (uint32_t)(x / 16) - halo : 0u;
    const uint32_t b1 = (uint32_t)(y / 16) > halo ? (uint32_t)(y / 16) - halo : 0u;
    const uint32_t b2 = (uint32_t)std::min<uint64_t>((x + w + 15) / 16 + halo, img->mbs_x);
    const uint32_t b3 = (uint32_t)std::min<uint64_t>((y + h + 15) / 16 + halo, img->mbs_y);
    // the window of the tiles those macroblocks fall in
    // (tile_plans' required_for_reconstruction, prepare.rs:265-306, and
    // Window::of_plan, crates/jxr-native/src/decode/reconstruction.rs:509-546)
    auto span = [](const std::vector<uint32_t> &sizes, uint32_t lo, uint32_t hi, uint32_t &o, uint32_t &n) {
        uint32_t start = UINT32_MAX, end = 0, pos = 0;
        for (uint32_t size : sizes) {
            if (pos < hi && pos + size > lo) {
                start = std::min(start, pos);
                end = std::max(end, pos + size);
            }
            pos += size;
        }
        o = start;
        n = end - start;
    };
    std::unique_ptr<jxrb_request> r(new jxrb_request);
    r->image = img;
    r->denominator = denominator;
    span(img->tile_w, b0, b2, r->ox, r->wx);
    span(img->tile_h, b1, b3, r->oy, r->wy);
    jxrb_output_format wo = *output;
    wo.crop_x = (uint32_t)(x - 16ull * r->ox);
    wo.crop_y = (uint32_t)(y - 16ull * r->oy);
    if (denominator != 1) {
        // the region at the reduced resolution (native_output_region,
        // crates/jxr-native/src/prepare.rs:196-216), in window coordinates
        const uint64_t d = (uint64_t)denominator, per_mb = 16 / d;
        const uint64_t qx0 = x / d, qy0 = y / d, qx1 = (x + w + d - 1) / d, qy1 = (y + h + d - 1) / d;
        wo.crop_x = (uint32_t)(qx0 - per_mb * r->ox);
        wo.crop_y = (uint32_t)(qy0 - per_mb * r->oy);
        wo.crop_width = (uint32_t)(qx1 - qx0);
        wo.crop_height = (uint32_t)(qy1 - qy0);
        // validate_native_scale (prepare.rs:155-183): a quarter's picture is
        // made of low-pass coefficients, which every macroblock must code (a
        // sixteenth's of the DC band alone)
        for (const ImagePlane &ip : img->planes) {
            if (denominator != 4) break;
            const uint32_t W1 = img->mbs_x + 1;
            const uint32_t x0 = r->ox, y0 = r->oy, x1 = r->ox + r->wx, y1 = r->oy + r->wy;
            const uint32_t n = ip.dc_only[(size_t)y1 * W1 + x1] - ip.dc_only[(size_t)y0 * W1 + x1] -
                               ip.dc_only[(size_t)y1 * W1 + x0] + ip.dc_only[(size_t)y0 * W1 + x0];
            if (n) return fail(JXRB_UNSUPPORTED_OUTPUT, "quarter-resolution decode requires an LP band");
        }
        // the sample scale of each plane over this window's regions
        for (size_t k = 0; k < img->planes.size(); k++) {
            const ImagePlane &ip = img->planes[k];
            std::vector<uint32_t> cols{0}, rows{0};
            auto inner = [](const std::vector<uint32_t> &sizes, uint32_t o, uint32_t n, std::vector<uint32_t> &b) {
                uint32_t pos = 0;
                for (uint32_t size : sizes) {
                    pos += size;
                    if (pos > o && pos < o + n) b.push_back(pos - o);
                }
                b.push_back(n);
            };
            if (ip.hard) {
                inner(img->tile_w, r->ox, r->wx, cols);
                inner(img->tile_h, r->oy, r->wy, rows);
            } else {
                cols.push_back(r->wx);
                rows.push_back(r->wy);
            }
            std::vector<uint32_t> key{(uint32_t)denominator, (uint32_t)ip.bc, (uint32_t)ip.br, (uint32_t)ip.scale2,
                                      (uint32_t)ip.overlap, 0xffffffffu};
            key.insert(key.end(), cols.begin(), cols.end());
            key.push_back(0xffffffffu);
            key.insert(key.end(), rows.begin(), rows.end());
            std::shared_ptr<const QuarterScale> scale;
            {
                std::lock_guard<std::mutex> guard(img->scale_lock);
                auto it = img->scales.find(key);
                if (it != img->scales.end()) scale = it->second;
            }
            if (!scale) {
                auto made = std::make_shared<QuarterScale>();
                std::string why;
                if (!reduced_scale(denominator, ip.bc, ip.br, ip.scale2 != 0, ip.overlap, r->wx, r->wy, cols, rows,
                                   *made, why))
                    return fail(JXRB_KERNEL_ARITHMETIC, why);
                std::lock_guard<std::mutex> guard(img->scale_lock);
                scale = img->scales.emplace(key, std::move(made)).first->second;
            }
            r->scales.push_back(scale);
        }
    }
    if (subsampled_out && (wo.crop_x & 1))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "planar chroma crop must start on an even column");
    if (oc == JXRB_COLOR_YUV420 && (wo.crop_y & 1))
        return fail(JXRB_UNSUPPORTED_OUTPUT, "planar 4:2:0 crop must start on an even row");
    const int internal = (img->chroma && (oc != g.color_format || denominator == 16)) ? JXRB_COLOR_YUV444
                                                                                       : g.color_format;
    TRY(build_output(wo, internal, img->ncomp, img->alpha >= 0, g.scaled, g.alpha_scaled, r->out, r->output_bytes));
    uint64_t traffic = r->output_bytes;
    for (const ImagePlane &ip : img->planes)
        traffic += denominator == 4    ? (uint64_t)r->wx * r->wy * (16 + 4ull * ip.bc * ip.br)   // table entry, DC/LP values
                   : denominator == 16 ? (uint64_t)r->wx * r->wy * (16 + 4)                      // table entry, DC value
                                       : rect_bytes(ip, img->mbs_x, r->ox, r->oy, r->ox + r->wx, r->oy + r->wy);
    r->traffic_bytes = traffic;
    *out = r.release();
    return JXRB_OK;
}

void jxrb_request_destroy(jxrb_request *r) { delete r; }

uint64_t jxrb_request_output_bytes(const jxrb_request *r) { return r ? r->output_bytes : 0; }

uint64_t jxrb_request_traffic_bytes(const jxrb_request *r) { return r ? r->traffic_bytes : 0; }

jxrb_status jxrb_request_window(const jxrb_request *r, uint32_t window[4]) {
    if (!r || !window) return fail(JXRB_INVALID_PLAN, "null argument");
    window[0] = r->ox;
    window[1] = r->oy;
    window[2] = r->wx;
    window[3] = r->wy;
    return JXRB_OK;
}

jxrb_status jxrb_submit_requests(jxrb_session *s, const jxrb_request *const *reqs, uint32_t count, void *dst,
                                 uint64_t dst_len, jxrb_submission **out) {
    TRY(check_session(s));
    if (!out || !reqs) return fail(JXRB_INVALID_SUBMISSION_STATE, "null argument");
    if (count == 0) return fail(JXRB_INVALID_PLAN, "empty batch");
    if (count > kImageMask) return fail(JXRB_RESOURCE_LIMIT, "too many images in one launch");
    for (uint32_t i = 0; i < count; i++) {
        if (!reqs[i]) return fail(JXRB_INVALID_PLAN, "null request");
        if (reqs[i]->image->session != s) return fail(JXRB_INVALID_PLAN, "request on another session's image");
    }
    std::unique_ptr<jxrb_submission> sub(new jxrb_submission);
    sub->session = s;
    const size_t k = pick_stream(s);
    sub->stream = s->streams[k];
    std::lock_guard<std::mutex> guard(s->lock);
    TRY(build_request_set(s, reqs, count, k, sub->stream, sub->set));
    if (dst) {
        if (dst_len < sub->set.output_bytes) return fail(JXRB_INVALID_DESTINATION, "destination is smaller than the output");
        sub->output = static_cast<uint8_t *>(dst);
    } else {
        CUDA_TRY(cudaMallocAsync(&sub->owned_output, std::max<uint64_t>(sub->set.output_bytes, 1), sub->stream),
                 "cudaMallocAsync (output)");
        sub->output = static_cast<uint8_t *>(sub->owned_output);
    }
    TRY(bind_output(sub->set, sub->output, sub->stream));
    TRY(launch_set(s, sub->set, sub->stream));
    CUDA_TRY(cudaEventCreateWithFlags(&sub->done, cudaEventDisableTiming), "cudaEventCreate");
    CUDA_TRY(cudaEventRecord(sub->done, sub->stream), "cudaEventRecord");
    s->submissions++;
    *out = sub.release();
    return JXRB_OK;
}

}  // extern "C"
