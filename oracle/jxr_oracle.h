/*
 * jxr_oracle.h -- CPU restatement of the JPEG XR reconstruction path of the
 * frames-sg/jxr reference (crates/jxr-math, crates/jxr-native/src/reconstruct,
 * crates/jxr-native/src/output_format).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark call it to obtain
 * the reference's results.  The product (the CUDA engine under jxr_b200/)
 * never links, loads or calls it.
 *
 * Every operation is the checked integer form of the reference: an
 * intermediate that leaves int32 is an error (JO_ERR_OVERFLOW), exactly where
 * the reference's `checked_*` arithmetic returns Err.
 */
#ifndef JXR_ORACLE_H
#define JXR_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    JO_OK = 0,
    JO_ERR_OVERFLOW = 1,   /* checked arithmetic left int32 */
    JO_ERR_INVALID = 2,    /* geometry / request the reference rejects */
    JO_ERR_UNSUPPORTED = 3 /* combination the reference rejects as unsupported */
};

/* ---- exact math (crates/jxr-math) -------------------------------------- */
int jo_inverse_core_transform(int32_t v[16]);
int jo_inverse_chroma_420(int32_t v[4]);
int jo_inverse_chroma_422(int32_t v[8]);
int jo_inverse_overlap_4(int32_t v[4]);
int jo_inverse_overlap_4x4(int32_t v[16]);
int jo_inverse_overlap_2x2(int32_t v[4]);
int jo_inverse_overlap_2(int32_t v[2]);
int jo_dequantize(int32_t coefficient, uint32_t step, int32_t *out);
/* direction: 0 none, 1 from left, 2 from top, 3 top-left (rejected) */
int jo_predict_high_pass(int32_t coefficients[256], int direction,
                         int block_columns, int block_rows);
int jo_upsample_pair(int32_t previous, int32_t current, int32_t next,
                     int centering, int32_t out[2]);
void jo_postscale_rgbe(const int32_t rgb[3], uint8_t out[4]);
int jo_premultiply_unsigned(uint32_t value, uint32_t alpha, uint32_t maximum,
                            uint32_t *out);
int jo_premultiply_signed(int32_t value, int32_t alpha, int32_t maximum,
                          int32_t *out);
int jo_premultiply_sign_magnitude_15(uint16_t value, uint16_t alpha,
                                     uint16_t *out);
float jo_premultiply_f32(float value, float alpha);
uint32_t jo_widen_f16(uint16_t bits);

/* ---- plane reconstruction (crates/jxr-native/src/reconstruct) ---------- */

/* Bands coded by a macroblock (jxr-core BandPresence). */
enum { JO_BANDS_DC_ONLY = 0, JO_BANDS_NO_HIGH_PASS = 1, JO_BANDS_NO_FLEXBITS = 2, JO_BANDS_ALL = 3 };

typedef struct jo_plane {
    const int32_t *coefficients;   /* arena coefficients */
    size_t coefficient_count;
    /* per macroblock, raster order over the plane window */
    const uint32_t *offsets;       /* first coefficient of the macroblock */
    const uint32_t *quantizers;    /* 3 per macroblock: DC, low-pass, high-pass step */
    const uint8_t *bands;          /* JO_BANDS_* */
    const uint8_t *hp_prediction;  /* 0 none, 1 left, 2 top, 3 top-left */
    uint32_t macroblocks_x, macroblocks_y;
    uint32_t block_columns, block_rows; /* (4,4), (2,4) or (2,2) */
    int scale_after_first_transform;
    int overlap;                   /* 0, 1, 2 */
    int hard_tiles;
    /* tile boundaries inside the window in macroblocks, first 0, last = extent */
    const uint32_t *column_boundaries; uint32_t column_boundary_count;
    const uint32_t *row_boundaries; uint32_t row_boundary_count;
} jo_plane;

/* ---- overlap schedules on a bare sample plane --------------------------
 * Boundaries are tile boundaries in samples, the first 0 and the last the
 * extent; with `hard` each tile is filtered on its own. */
/* Full-resolution postfilter (apply_overlap::<Postfilter>,
 * crates/jxr-native/src/reconstruct/overlap.rs:72-89). */
int jo_apply_overlap(int32_t *samples, uint32_t width, uint32_t height, const uint32_t *column_boundaries,
                     uint32_t column_count, const uint32_t *row_boundaries, uint32_t row_count, int hard);
/* Subsampled first-level postfilter (apply_subsampled_first_overlap::<Postfilter>,
 * crates/jxr-native/src/reconstruct/subsampled_overlap.rs:110-296). */
int jo_apply_subsampled_first_overlap(int32_t *samples, uint32_t width, uint32_t height,
                                      const uint32_t *column_boundaries, uint32_t column_count,
                                      const uint32_t *row_boundaries, uint32_t row_count, int hard);
/* The full-resolution schedule as the device plan's flat operator list
 * (full_schedule, crates/jxr-core/src/device_plan/overlap.rs:125-178):
 * first sample, step and kind (0 window, 1 edge strip, 2 corner) of each
 * operator in order.  `count` receives the operator count; fails when it
 * exceeds `capacity`. */
int jo_full_schedule(uint32_t width, uint32_t height, const uint32_t *column_boundaries, uint32_t column_count,
                     const uint32_t *row_boundaries, uint32_t row_count, int hard, uint32_t *offsets,
                     uint32_t *steps, uint32_t *kinds, uint32_t capacity, uint32_t *count);
/* One macroblock's high-pass band placed as dequantized samples
 * (dequantize_high_pass_into, crates/jxr-native/src/reconstruct/pipeline.rs:543-586):
 * `rows` is a band of block_rows*4 sample rows, `width` samples across; the
 * macroblock's blocks start at block column `column`. */
int jo_place_high_pass(const int32_t high[256], uint32_t step, int bands, uint32_t block_columns,
                       uint32_t block_rows, int32_t *rows, size_t width, size_t column);

/* Width and height of the sample plane a jo_plane reconstructs. */
void jo_plane_extent(const jo_plane *plane, uint32_t *width, uint32_t *height);

/* Reconstruct one component plane into `samples` (width*height int32).
 * `threads` > 1 spreads the independent work of each stage over threads. */
int jo_reconstruct_plane(const jo_plane *plane, int32_t *samples, int threads);

/* T.832 example chroma upsampling of a whole plane.  sampling: 1 = 4:2:0,
 * 2 = 4:2:2.  `out` is (2*width) x (height or 2*height). */
int jo_upsample_chroma(const int32_t *chroma, uint32_t width, uint32_t height,
                       int sampling, int centering_x, int centering_y,
                       int32_t *out, int threads);

/* ---- output formatting (crates/jxr-native/src/output_format) ----------- */

enum { /* colour formats */
    JO_COLOR_LUMA = 0, JO_COLOR_YUV420 = 1, JO_COLOR_YUV422 = 2, JO_COLOR_YUV444 = 3,
    JO_COLOR_RGB = 4, JO_COLOR_CMYK = 5, JO_COLOR_CMYK_DIRECT = 6, JO_COLOR_YUVK = 7,
    JO_COLOR_RGBE = 8, JO_COLOR_NCOMPONENT = 9
};
enum { /* output bit depths (jxr-core OutputBitDepth) */
    JO_DEPTH_BIT1_WHITE = 0, JO_DEPTH_BIT1_BLACK = 1, JO_DEPTH_U8 = 2, JO_DEPTH_U10 = 3,
    JO_DEPTH_U16 = 4, JO_DEPTH_I16 = 5, JO_DEPTH_F16 = 6, JO_DEPTH_I32 = 7,
    JO_DEPTH_F32 = 8, JO_DEPTH_RGB555 = 9, JO_DEPTH_RGB101010 = 10, JO_DEPTH_RGB565 = 11
};
enum { /* storage kinds (jxr-core PixelFormat) */
    JO_STORE_BITS = 0, JO_STORE_U8 = 1, JO_STORE_U16 = 2, JO_STORE_I16 = 3, JO_STORE_I32 = 4,
    JO_STORE_F16 = 5, JO_STORE_F32 = 6, JO_STORE_RGB555 = 7, JO_STORE_RGB565 = 8,
    JO_STORE_RGB101010 = 9, JO_STORE_RGBE = 10
};
enum { /* channel layouts (jxr-core ChannelLayout) */
    JO_LAYOUT_LUMA = 0, JO_LAYOUT_LUMA_ALPHA = 1, JO_LAYOUT_YUV = 2, JO_LAYOUT_YUVA = 3,
    JO_LAYOUT_RGB = 4, JO_LAYOUT_RGBX = 5, JO_LAYOUT_RGBA = 6, JO_LAYOUT_BGR = 7,
    JO_LAYOUT_BGRX = 8, JO_LAYOUT_BGRA = 9, JO_LAYOUT_CMYK = 10, JO_LAYOUT_CMYKA = 11,
    JO_LAYOUT_NCOMPONENT = 12, JO_LAYOUT_NCOMPONENT_ALPHA = 13
};

typedef struct jo_output {
    int internal_color;      /* colour of the planes given (after upsampling) */
    int output_color;
    int depth; int shift_bits; int mantissa_length; int exponent_bias;
    int storage; int layout; int ncomponents;
    int scaled;
    int alpha_depth; int alpha_shift_bits; int alpha_mantissa_length;
    int alpha_exponent_bias; int alpha_scaled; /* used when an alpha plane is given */
    int red_blue_not_swapped;
    int premultiply;
    uint32_t crop_x, crop_y, crop_width, crop_height;
    /* Extensions with no reference counterpart on the GPU path:
     * nchw: store each channel as its own crop_width x crop_height plane
     *       (the reference's CPU batch NCHW reorder);
     * widen_f16: store F16 output bits widened exactly to binary32. */
    int nchw;
    int widen_f16;
} jo_output;

/* Bytes the output of `request` occupies. */
size_t jo_output_bytes(const jo_output *request);

/* Format full-resolution component planes (all width x height, origin 0).
 * planes[0..ncomp), alpha may be NULL.  Native planar YUV 4:2:0/4:2:2 output
 * takes the planes at their coded (subsampled) size instead. */
int jo_format_output(const int32_t *const *planes, int plane_count,
                     const int32_t *alpha, uint32_t width, uint32_t height,
                     const jo_output *request, void *out, size_t out_len);

/* ---- whole image ---------------------------------------------------------- */
typedef struct jo_image {
    const jo_plane *planes; int plane_count;  /* primary components */
    const jo_plane *alpha;                    /* NULL when no alpha plane */
    int coded_color;                          /* JO_COLOR_* of the coded planes */
    int centering_x, centering_y;             /* chroma centering codes */
} jo_image;

/* Reconstruct every plane, upsample 4:2:0/4:2:2 chroma where the output is
 * not native planar YUV, and format. */
int jo_decode_image(const jo_image *image, const jo_output *request, void *out,
                    size_t out_len, int threads);

/* ---- analysis and reduced resolution ------------------------------------ */

/* analyze_component with unit quantizers and every band
 * (crates/jxr-native/src/analyze.rs:56-86): the exact inverse of full
 * reconstruction, the DC and low-pass bands halved to nearest where the plane
 * doubles them (Steps::new, analyze.rs:505-535).  `plane` supplies the
 * geometry only.  `coefficients` receives macroblocks * blocks * 16 values in
 * arena order (block b of a macroblock at [b*16], its DC/LP value first). */
int jo_analyze_plane(const jo_plane *plane, const int32_t *samples, int32_t *coefficients);

/* Quarter-resolution reconstruction of one plane (reconstruct_quarter,
 * crates/jxr-native/src/reconstruct/pipeline.rs:175-222): one sample a block,
 * the block DC after the first level, scaled to the level it stands for
 * (SampleScale, reconstruct/sample_scale.rs).  `samples` is
 * (macroblocks_x*block_columns) x (macroblocks_y*block_rows). */
int jo_reconstruct_plane_quarter(const jo_plane *plane, int32_t *samples);
void jo_plane_extent_scaled(const jo_plane *plane, int denominator, uint32_t *width, uint32_t *height);

/* Sixteenth-resolution reconstruction of one plane (reconstruct_sixteenth,
 * crates/jxr-native/src/reconstruct/pipeline.rs:223-260): one sample a
 * macroblock, macroblocks_x x macroblocks_y, scaled like the quarter. */
int jo_reconstruct_plane_sixteenth(const jo_plane *plane, int32_t *samples);
/* Presentation orientation of a packed surface (apply_orientation,
 * crates/jxr/src/decoder/orientation.rs:5-211): `width` x `height` pixels of
 * `pixel_bytes` each (0: one-bit luma, rows padded to bytes) into `dst`,
 * whose width and height are swapped for the transposing orientations. */
enum {
    JO_ORIENT_IDENTITY = 0, JO_ORIENT_MIRROR_HORIZONTAL = 1, JO_ORIENT_ROTATE180 = 2, JO_ORIENT_MIRROR_VERTICAL = 3,
    JO_ORIENT_TRANSPOSE = 4, JO_ORIENT_ROTATE90 = 5, JO_ORIENT_TRANSVERSE = 6, JO_ORIENT_ROTATE270 = 7
};
int jo_orient(const uint8_t *src, uint8_t *dst, uint32_t width, uint32_t height, uint32_t pixel_bytes,
              int orientation);
/* jo_decode_image at 1/denominator resolution (1, 4 or 16); the request's crop
 * is in reduced coordinates. */
int jo_decode_image_scaled(const jo_image *image, int denominator, const jo_output *request, void *out,
                           size_t out_len, int threads);

#ifdef __cplusplus
}
#endif
#endif
