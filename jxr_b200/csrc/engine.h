// engine.h -- device descriptors shared by the host planner and the kernels.
//
// Layout in HBM (one image):
//   * coefficients: the arena's int32 coefficients exactly as the host entropy
//     decoder produced them (crates/jxr-core/src/plan.rs:136-142), uploaded
//     unchanged;
//   * one macroblock table per plane, raster order over the reconstruction
//     window, 16 bytes an entry (uint4): x = coefficient offset relative to
//     the plane base | bands << 28 | hp_prediction << 30, y/z/w = DC,
//     low-pass and high-pass quantization steps;
//   * per plane two byte maps marking the macroblock columns and rows where a
//     hard tile begins;
//   * the output surface.
#pragma once
#include <stdint.h>

#define JXRB_MAX_PLANES 5
#define JXRB_MAX_CHANNELS 6

namespace jxr {

enum StoreKind : int32_t {
    kStoreBits = 0, kStoreU8 = 1, kStoreU16 = 2, kStoreI16 = 3, kStoreI32 = 4,
    kStoreF16 = 5, kStoreF32 = 6, kStoreRgb555 = 7, kStoreRgb565 = 8,
    kStoreRgb101010 = 9, kStoreRgbe = 10
};

enum ColorConv : int32_t {
    kConvDirect = 0,      // channels are the components themselves
    kConvLumaToRgb = 1,   // replicate luma
    kConvYuvToRgb = 2,    // inverse RCT (crates/jxr-native/src/output_format/color.rs:100-108)
    kConvYuvkToCmyk = 3,  // color.rs:110-121
    kConvYuvkToCmykDirect = 4
};

// One resolved channel scale (crates/jxr-native/src/output_format/scaling.rs:37-119).
struct ChannelScale {
    int32_t shifted_bias;
    int32_t rounding;
    int32_t shift;
    int32_t post_shift;   // < 0: none
    int32_t lo, hi;       // clip range of the store
    int32_t padding;      // RGBX/BGRX padding channel: stores zero
    int32_t source;       // index into the converted components, or 4 for alpha
    int32_t alpha;        // channel is alpha
    int32_t f_mantissa;   // F32: mantissa length; F16: unused
    int32_t f_bias;       // F32: exponent bias
    int32_t f_scaled;     // F16/F32: scaled flag of the channel
};

struct OutputDev {
    uint8_t *base;            // device surface
    uint64_t row_stride;      // bytes between rows (interleaved)
    uint64_t plane_stride;    // bytes between channel planes (NCHW / planar)
    uint32_t crop_x, crop_y, crop_w, crop_h;  // full-resolution coordinates
    int32_t store;            // StoreKind
    int32_t channels;         // stored channels per pixel
    int32_t conv;             // ColorConv
    int32_t packed_swap;      // packed RGB with red/blue swapped
    int32_t nchw;             // channel planes instead of interleaved
    int32_t widen_f16;        // F16 bits widened to binary32
    int32_t premultiply;
    int32_t planar_yuv;       // 1: 4:2:0, 2: 4:2:2 native planar output
    int32_t bit_black;        // 1-bit output: one is black
    int32_t elem_bytes;       // bytes of one stored element
    int32_t depth_max;        // unused
    int32_t kind;             // output path: 0 generic, 1 RGB8 from YUV, 2 one channel direct, 3 F16 widened
    ChannelScale ch[JXRB_MAX_CHANNELS];
};

struct PlaneDev {
    const int32_t *coeff;     // plane coefficient base
    const uint4 *mbs;         // macroblock table
    const uint8_t *col_start; // 1 where a hard tile starts (macroblock columns)
    const uint8_t *row_start; // (macroblock rows)
    uint32_t mbs_x, mbs_y;
    int32_t bc, br;           // blocks across / down a macroblock
    int32_t scale2;           // doubled after the first-level transform
    int32_t overlap;          // 0, 1, 2
    int32_t hard;             // hard tile boundaries
    uint32_t mbs_stride;      // macroblock table entries between rows (a window may view a larger table)
};

struct ImageDev {
    PlaneDev plane[JXRB_MAX_PLANES];
    int32_t nplanes;          // colour planes
    int32_t alpha;            // index of the alpha plane or -1
    int32_t chroma;           // 0: full resolution, 1: 4:2:0, 2: 4:2:2 (planes 1, 2)
    int32_t centering_x, centering_y;
    uint32_t mbs_x, mbs_y;    // luma macroblock window
    uint32_t tiles_x, tiles_y;
    uint32_t tile_mbs;        // macroblocks across and down a CTA tile
    uint32_t first_item;      // index of this image's first work item
    uint32_t pad;
    OutputDev out;
};

// One plane of a reduced-resolution request (a quarter or a sixteenth of
// the resolution).  Its pictures live in the submission's scratch.  A
// quarter: the first-level kernel writes the block picture -- one sample a
// block -- the overlap kernel filters it in place, the scale kernel scales it
// and the output kernel reads it.  A sixteenth: one sample a macroblock, the
// macroblock's DC written straight into the macroblock picture, or, with
// two-level overlap, the block picture of the DC band filtered and summed
// over each macroblock into it.
struct QuarterPlane {
    const int32_t *coeff;       // plane coefficient base
    const uint4 *mbs;           // macroblock table at the window origin
    const uint8_t *col_start;   // hard tile starts (window-relative macroblocks)
    const uint8_t *row_start;
    int32_t *pic;               // block picture, (mbs_x*bc) x (mbs_y*br); unused by a one-level sixteenth
    int32_t *out;               // the reduced picture scaled and stored: pic for a quarter, mbs_x x mbs_y for a sixteenth
    const int64_t *divisor;     // flat terms of the probe picture (shift < 0)
    const int64_t *bias;
    const uint32_t *cols;       // picture column / row -> probe column / row
    const uint32_t *rows;
    int64_t gain;
    uint32_t mbs_x, mbs_y, mbs_stride;
    int32_t bc, br, scale2, overlap, hard;
    int32_t shift;              // >= 0: samples >>= shift; < 0: flat terms
    uint32_t probe_stride;
    int32_t sixteenth;          // 1: one sample a macroblock
};

// A reduced-resolution request: its image descriptor (output, colour
// planes, chroma) and its planes in the QuarterPlane list.
struct QuarterImage {
    uint32_t image;             // index into the set's image descriptors
    uint32_t first_plane;       // its planes: first_plane .. first_plane + planes
    uint32_t planes;
    uint32_t width, height;     // reduced-resolution luma picture
};

// Work-list segments, one tile kernel each: interior tiles of images with
// 1..4 full-resolution planes (segments 0..3), interior tiles of YUV 4:2:0
// images (segment 4), tiles of images with 1..4 full-resolution planes that
// touch the plane's edge but no hard tile boundary (segments 5..8), such tiles
// of 4:2:0 images (segment 9), then every other tile (segment 10).  A work
// item carries a tag in the top bits of its image index: its segment + 1, or
// 0 for the last segment (edge tiles folded into their interior kernel, see
// kFoldEdges, keep their edge tag but sit in the interior segment).
constexpr int kSegments = 11;
constexpr int kSegmentOther = kSegments - 1;
constexpr uint32_t kTag420 = 5;
constexpr uint32_t kTagEdge = 5;               // + plane count: edge tiles
constexpr uint32_t kTagEdge420 = 10;
constexpr int kTagShift = 28;
constexpr uint32_t kImageMask = (1u << kTagShift) - 1;
constexpr int kSideSegment0 = 5;               // segments run beside the interior ones
// Edge tiles that the interior kernel of the same images takes instead of an
// edge kernel (one launch, edge tiles first in it), by plane count 1..4, then
// 4:2:0; their edge segment then stays empty.
constexpr bool kFoldEdges[5] = {false, false, true, false, false};
constexpr int kCounterWords = 2 * kSegments;   // two scheduling words a segment

// Launch shape of the tile kernels, chosen by the autotuner.  Entries 0..3
// serve the full-resolution segments by plane count, entry 4 the other tiles;
// the 4:2:0 interior segment, a three-plane interior kernel, takes entry 2.
struct LaunchTuning {
    uint32_t blocks_per_sm[5];   // resident CTAs per SM; 0 = as many as fit
    int32_t side_stream;         // other tiles' kernel on a second stream beside the interior ones
};

// Where the descriptors of one plan sit inside a fixed device region (the
// allocation-free entry point of static_scratch.cu): the image descriptor at
// offset 0, then the work list, the status word, the counters and the
// per-plane macroblock tables and tile-start maps.
struct StagedLayout {
    size_t bytes;            // descriptor bytes from the region's start
    size_t items_at;         // offsets within the region
    size_t status_at;
    size_t counters_at;
    uint32_t bounds[kSegments + 1];   // work-list segment boundaries
    int max_planes;
    uint64_t clear_bytes;    // output bytes to zero before the launch (1-bit outputs), else 0
};

// Status codes written with a first-error compare-and-swap, the stage codes
// of the reference's kernels (crates/jxr-cuda/src/kernels/main.rs:52-56).
enum StatusCode : uint32_t {
    kStatusFirstTransform = 1,
    kStatusOverlap = 2,
    kStatusPrediction = 3,
    kStatusSecondTransform = 4,
    kStatusOutput = 16,
    kStatusInvalid = 32
};

}  // namespace jxr
