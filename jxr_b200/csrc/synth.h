// synth.h -- seeded synthetic coefficient arenas: the forward (analysis)
// half of the reference encoder applied to generated images.
//
// The reference's own encoder (crates/jxr-native/src/encode.rs, analyze.rs)
// cannot be built here, so inputs are produced by restating its forward
// path: output unscaling (scaling.rs:121-147), the forward colour transform
// (output_format/color.rs:54-86), 4:2:0 decimation (crates/jxr-math/src/sampling.rs:78-100),
// the overlap prefilter and forward core transform of both levels
// (crates/jxr-math/src/overlap.rs, transform.rs forward functions), quantization
// (crates/jxr-math/src/quantization.rs:35-50) with the quality-to-QP map of
// crates/jxr-native/src/encode/quality.rs:295-500 and the QP-to-step map of
// crates/jxr-native/src/tile_decode/quantizer.rs:147-158,309-331, and
// high-pass prediction residuals with the direction rule of
// crates/jxr-native/src/tile_decode/syntax.rs:203-231.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    JXRB_CONTENT_PHOTO_RGB8 = 0,   /* 6 sinusoids + N(0, 8^2) + 20 flat rectangles, [0, 255] */
    JXRB_CONTENT_HDR_HALF = 1,     /* exp(smooth noise) in [1e-3, 64] as binary16 */
    JXRB_CONTENT_GRAY16 = 2,       /* the photo content at 16 bits */
    JXRB_CONTENT_RANDOM = 3        /* uniform random coefficients (stress: every band, prediction) */
};

typedef struct jxrb_synth_request {
    uint32_t width, height;        /* pixels; padded up to whole macroblocks */
    int32_t content;               /* JXRB_CONTENT_* */
    int32_t color_format;          /* JXRB_COLOR_LUMA / YUV420 / YUV422 / YUV444 */
    int32_t alpha_mode;            /* JXRB_ALPHA_* : alpha is seeded soft-edged ellipses */
    int32_t overlap, alpha_overlap;
    int32_t scaled;                /* SCALED_FLAG of the colour planes */
    int32_t quality;               /* 1..100, or 0 to take the QPs below */
    int32_t qp[3];                 /* DC, LP, HP QP parameters of every colour component */
    int32_t alpha_qp[3];           /* alpha plane QPs (0 = lossless) */
    uint32_t tile_width, tile_height;  /* macroblocks; 0 = one tile */
    int32_t hard_tiles;
    int32_t bands;                 /* JXRB_BANDS_* coded by every macroblock (random content mixes) */
    uint64_t seed;
} jxrb_synth_request;

typedef struct jxrb_synth jxrb_synth;

/* Generate the arena(s) of one image. */
int jxrb_synth_create(const jxrb_synth_request *request, int threads, jxrb_synth **out);
void jxrb_synth_destroy(jxrb_synth *s);

/* Arena and geometry views (pointers stay valid until destroy).  `which`:
 * 0 = primary arena, 1 = separate alpha arena (NULL fields when absent). */
typedef struct jxrb_synth_arena_view {
    const int32_t *coefficients; uint64_t coefficient_count;
    const uint32_t *coefficient_offsets, *quantizers, *coded_x, *coded_y;
    const uint8_t *bands, *hp_predictions;
    uint64_t macroblock_count;
    const uint64_t *plane_words; /* 6 words a plane: coefficient offset/count, macroblock offset/count, bc, br */
    uint32_t plane_count;
} jxrb_synth_arena_view;

int jxrb_synth_arena(const jxrb_synth *s, int which, jxrb_synth_arena_view *out);
/* Geometry: macroblocks across/down, tile widths/heights (macroblocks),
 * source pixels (width, height). */
int jxrb_synth_geometry(const jxrb_synth *s, uint32_t *mbs_x, uint32_t *mbs_y, const uint32_t **tile_widths,
                        uint32_t *tile_columns, const uint32_t **tile_heights, uint32_t *tile_rows);
/* Source image: interleaved channels (uint8 / uint16), before coding. */
const void *jxrb_synth_source(const jxrb_synth *s, uint32_t *channels, uint32_t *bytes_per_sample);

/* Forward operators, exported for the exact-inverse tests of the oracle. */
int jxrb_forward_core_transform(int32_t v[16]);
int jxrb_forward_overlap_4x4(int32_t v[16]);
int jxrb_forward_overlap_4(int32_t v[4]);
int jxrb_forward_overlap_2x2(int32_t v[4]);
int jxrb_forward_overlap_2(int32_t v[2]);
int jxrb_forward_chroma_420(int32_t v[4]);
int jxrb_forward_chroma_422(int32_t v[8]);
uint32_t jxrb_quant_step(int32_t qp, int32_t scaled, int32_t component, int32_t band);

/* The generator's CPU forward analysis of one sample plane (the checker of the
 * engine's GPU analysis, jxrb_analyze_planes): `samples` (width x height) is
 * read, not changed; `low_q` receives 16 values a macroblock, `high_q` 256,
 * raster order.  Tile boundaries in macroblocks, 0 .. extent. */
int jxrb_analyze_plane_cpu(const int32_t *samples, uint32_t width, uint32_t height, uint32_t block_columns,
                           uint32_t block_rows, int32_t scaled, int32_t overlap, const uint32_t steps[3],
                           const uint32_t *column_boundaries, uint32_t column_count, const uint32_t *row_boundaries,
                           uint32_t row_count, int32_t hard_tiles, int32_t *low_q, int32_t *high_q);

#ifdef __cplusplus
}
#endif
