/*
 * jxr_b200.h -- C ABI of the B200 JPEG XR reconstruction engine.
 *
 * This is the drop-in boundary for the GPU reconstruction path of the
 * frames-sg/jxr decoder: every entry point below replaces one public item of
 * the reference's `jxr_cuda` crate (re-exported as `jxr::cuda`,
 * crates/jxr/src/lib.rs:43-44), cited beside it.  Host code keeps the
 * reference's entropy decoder (crates/jxr-native) and hands its
 * `CoefficientArena` (crates/jxr-core/src/plan.rs:136-142) to
 * jxrb_plan_create; the engine reconstructs on the GPU and leaves the pixels
 * in device memory (or copies them back).
 *
 * Conventions: plain pointers and sizes, no CUDA types (a stream is passed
 * as `void *` holding a cudaStream_t).  Every function returns a
 * jxrb_status; jxrb_last_error() gives the reason of the calling thread's
 * last failure.  No call ever falls back to a CPU reconstruction: as in the
 * reference (docs/cuda-backend.md:134-139), a failure after submission is
 * returned, not retried.
 */
#ifndef JXR_B200_H
#define JXR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error kinds of crates/jxr-cuda/src/error.rs:8-92 (CudaError). */
typedef enum jxrb_status {
    JXRB_OK = 0,
    JXRB_UNAVAILABLE = 1,             /* CudaError::Unavailable */
    JXRB_UNSUPPORTED_DEVICE = 2,      /* CudaError::UnsupportedDevice (not sm_100) */
    JXRB_UNSUPPORTED_BACKEND = 3,     /* CudaError::UnsupportedBackend */
    JXRB_INVALID_PLAN = 4,            /* CudaError::InvalidPlan */
    JXRB_INVALID_DESTINATION = 5,     /* CudaError::InvalidDestination */
    JXRB_UNSUPPORTED_OUTPUT = 6,      /* CudaError::UnsupportedOutputFormat */
    JXRB_RUNTIME_INITIALIZATION = 7,  /* CudaError::RuntimeInitialization */
    JXRB_KERNEL_ARITHMETIC = 8,       /* CudaError::KernelArithmetic (stage in jxrb_last_stage) */
    JXRB_INVALID_SUBMISSION_STATE = 9,/* CudaError::InvalidSubmissionState */
    JXRB_RESOURCE_LIMIT = 10,         /* CudaError::ResourceLimit */
    JXRB_STATE_INVARIANT = 11,        /* CudaError::StatePoisoned / StateInvariant */
    JXRB_DRIVER = 12,                 /* CudaError::Driver */
    JXRB_TIMEOUT = 13,                /* a bounded wait elapsed (no reference counterpart) */
    JXRB_RESIDENT_OUTPUT_REQUIRES_CUDA = 14 /* CudaError::ResidentOutputRequiresCuda */
} jxrb_status;

/* ---- colour, depth, storage and layout codes ---------------------------
 * jxr-core ColorFormat (crates/jxr-core/src/format.rs), OutputBitDepth
 * (crates/jxr-core/src/output_policy.rs:20-48), PixelFormat storage and
 * ChannelLayout (format.rs:60-100). */
enum {
    JXRB_COLOR_LUMA = 0, JXRB_COLOR_YUV420 = 1, JXRB_COLOR_YUV422 = 2, JXRB_COLOR_YUV444 = 3,
    JXRB_COLOR_RGB = 4, JXRB_COLOR_CMYK = 5, JXRB_COLOR_CMYK_DIRECT = 6, JXRB_COLOR_YUVK = 7,
    JXRB_COLOR_RGBE = 8, JXRB_COLOR_NCOMPONENT = 9
};
enum {
    JXRB_DEPTH_BIT1_WHITE = 0, JXRB_DEPTH_BIT1_BLACK = 1, JXRB_DEPTH_U8 = 2, JXRB_DEPTH_U10 = 3,
    JXRB_DEPTH_U16 = 4, JXRB_DEPTH_I16 = 5, JXRB_DEPTH_F16 = 6, JXRB_DEPTH_I32 = 7,
    JXRB_DEPTH_F32 = 8, JXRB_DEPTH_RGB555 = 9, JXRB_DEPTH_RGB101010 = 10, JXRB_DEPTH_RGB565 = 11
};
enum {
    JXRB_STORE_BITS = 0, JXRB_STORE_U8 = 1, JXRB_STORE_U16 = 2, JXRB_STORE_I16 = 3, JXRB_STORE_I32 = 4,
    JXRB_STORE_F16 = 5, JXRB_STORE_F32 = 6, JXRB_STORE_RGB555 = 7, JXRB_STORE_RGB565 = 8,
    JXRB_STORE_RGB101010 = 9, JXRB_STORE_RGBE = 10
};
enum {
    JXRB_LAYOUT_LUMA = 0, JXRB_LAYOUT_LUMA_ALPHA = 1, JXRB_LAYOUT_YUV = 2, JXRB_LAYOUT_YUVA = 3,
    JXRB_LAYOUT_RGB = 4, JXRB_LAYOUT_RGBX = 5, JXRB_LAYOUT_RGBA = 6, JXRB_LAYOUT_BGR = 7,
    JXRB_LAYOUT_BGRX = 8, JXRB_LAYOUT_BGRA = 9, JXRB_LAYOUT_CMYK = 10, JXRB_LAYOUT_CMYKA = 11,
    JXRB_LAYOUT_NCOMPONENT = 12, JXRB_LAYOUT_NCOMPONENT_ALPHA = 13
};
enum { JXRB_ALPHA_NONE = 0, JXRB_ALPHA_INTEGRATED = 1, JXRB_ALPHA_SEPARATE = 2 };
enum { JXRB_BANDS_DC_ONLY = 0, JXRB_BANDS_NO_HIGH_PASS = 1, JXRB_BANDS_NO_FLEXBITS = 2, JXRB_BANDS_ALL = 3 };

/* ---- inputs --------------------------------------------------------------- */

/* CoefficientPlane, crates/jxr-core/src/plan.rs:124-134. */
typedef struct jxrb_coefficient_plane {
    uint64_t coefficient_offset;
    uint64_t coefficient_count;
    uint64_t macroblock_offset;
    uint64_t macroblock_count;
    uint32_t block_columns;   /* 4, or 2 for subsampled chroma */
    uint32_t block_rows;      /* 4, or 2 for 4:2:0 chroma */
} jxrb_coefficient_plane;

/* CoefficientArena + MacroblockMetadata (SoA), crates/jxr-core/src/plan.rs:62-142.
 * Host memory.  The metadata is read by jxrb_plan_create and not kept.  The
 * coefficients are read at submission: from pageable memory through the
 * session's pinned staging ring, in full before jxrb_submit* returns, so the
 * caller may reuse or free them then, as the reference's owned plans allow;
 * from page-locked memory (cudaHostAlloc / cudaHostRegister) by an
 * asynchronous copy that runs with the submission, so they must stay valid
 * and unchanged until jxrb_wait returns or the submission is destroyed. */
typedef struct jxrb_arena {
    const int32_t *coefficients;
    uint64_t coefficient_count;
    const uint32_t *coefficient_offsets;  /* per macroblock */
    const uint32_t *quantizers;           /* per macroblock: DC, low-pass, high-pass steps */
    const uint8_t *bands;                 /* per macroblock, JXRB_BANDS_* */
    const uint8_t *hp_predictions;        /* per macroblock: 0 none, 1 left, 2 top, 3 top-left */
    const uint32_t *coded_x;              /* macroblock column in the coded plane */
    const uint32_t *coded_y;              /* macroblock row in the coded plane */
    uint64_t macroblock_count;
    const jxrb_coefficient_plane *planes;
    uint32_t plane_count;
} jxrb_arena;

/* Image geometry: the parts of ImageInfo / PreparedPlan
 * (crates/jxr-core/src/image.rs:57-112, plan.rs:209-247) the path needs. */
typedef struct jxrb_image_geometry {
    uint32_t macroblock_origin_x, macroblock_origin_y;  /* reconstruction window, macroblocks */
    uint32_t macroblocks_x, macroblocks_y;
    const uint32_t *tile_column_widths;   /* whole-image tile grid, macroblocks (TileGrid) */
    uint32_t tile_columns;
    const uint32_t *tile_row_heights;
    uint32_t tile_rows;
    int32_t hard_tiles;
    int32_t color_format;                 /* coded colour, JXRB_COLOR_* (LUMA, YUV4xx, YUVK, NCOMPONENT) */
    int32_t components;                   /* colour components (1, 3, 4 or N) */
    int32_t overlap;                      /* 0, 1, 2 */
    int32_t scaled;                       /* SCALED_FLAG of the primary planes */
    int32_t alpha_mode;                   /* JXRB_ALPHA_* */
    int32_t alpha_overlap;
    int32_t alpha_scaled;
    int32_t chroma_centering_x, chroma_centering_y;
} jxrb_image_geometry;

/* OutputFormatRequest, crates/jxr-core/src/output_policy.rs (and the
 * extensions nchw / widen_f16 below).  Its `scaled` flags are the coded
 * planes' SCALED_FLAG, taken from jxrb_image_geometry. */
typedef struct jxrb_output_format {
    int32_t output_color;                 /* JXRB_COLOR_* */
    int32_t bit_depth;                    /* JXRB_DEPTH_* */
    int32_t shift_bits, mantissa_length, exponent_bias;
    int32_t storage;                      /* JXRB_STORE_* */
    int32_t layout;                       /* JXRB_LAYOUT_* */
    int32_t alpha_bit_depth;              /* alpha plane format (AlphaFormatRequest; its
                                             scaled flag is the geometry's alpha_scaled) */
    int32_t alpha_shift_bits, alpha_mantissa_length, alpha_exponent_bias;
    int32_t red_blue_not_swapped;
    int32_t premultiply_alpha;
    uint32_t crop_x, crop_y, crop_width, crop_height;  /* in window sample coordinates */
    /* Extensions (no reference counterpart on the GPU path):
     * nchw: channel planes of crop_width x crop_height instead of interleaved
     *       pixels (the reference's CPU BatchLayout::Nchw);
     * widen_f16: F16 output bits widened exactly to binary32. */
    int32_t nchw;
    int32_t widen_f16;
} jxrb_output_format;

typedef struct jxrb_session jxrb_session;
typedef struct jxrb_plan jxrb_plan;
typedef struct jxrb_submission jxrb_submission;
typedef struct jxrb_resident jxrb_resident;

typedef struct jxrb_session_options {
    uint32_t streams;            /* CUDA streams, round-robin (runtime.rs:17 uses 4) */
    uint64_t scratch_bytes;      /* device memory the session may hold for uploads */
} jxrb_session_options;

typedef struct jxrb_diagnostics {
    uint64_t submissions;
    uint64_t bytes_uploaded;
    uint64_t bytes_read_back;
    uint64_t device_bytes_held;
    uint64_t kernel_launches;
    uint64_t bytes_staged;        /* of bytes_uploaded: read from pageable memory through the pinned staging ring */
} jxrb_diagnostics;

/* ---- routing ------------------------------------------------------------
 * BackendRequest (crates/jxr-core/src/request.rs) and CudaRouteDecision /
 * CUDA_AUTO_THRESHOLD (crates/jxr-cuda/src/route.rs:8-20). */
enum { JXRB_BACKEND_AUTO = 0, JXRB_BACKEND_CPU = 1, JXRB_BACKEND_CUDA = 2, JXRB_BACKEND_METAL = 3 };
enum { JXRB_ROUTE_CPU = 0, JXRB_ROUTE_CUDA = 1 };
#define JXRB_CUDA_AUTO_THRESHOLD 16384u
/* plan_cuda_route, crates/jxr-cuda/src/route.rs:23-49: where a decode of
 * `reconstructed_coefficients` runs.  Explicit CUDA requests are strict
 * (JXRB_UNAVAILABLE when CUDA is not usable); Auto picks CUDA at or above the
 * threshold; resident (device) output needs CUDA
 * (JXRB_RESIDENT_OUTPUT_REQUIRES_CUDA for a CPU request); Metal is
 * JXRB_UNSUPPORTED_BACKEND.  Pure: probes and changes nothing. */
jxrb_status jxrb_plan_route(int backend_request, uint64_t reconstructed_coefficients, int cuda_usable,
                            int resident_output, int *decision);

/* ---- availability and errors ------------------------------------------- */

/* CudaDecoderSession::is_available, crates/jxr-cuda/src/session.rs:35-40. */
int jxrb_available(void);
/* Message of the calling thread's last failure (no reference counterpart:
 * the reference returns typed Rust errors). */
const char *jxrb_last_error(void);
/* Stage code of the last KernelArithmetic failure (1, 2, 3, 4, 16),
 * crates/jxr-cuda/src/kernels/main.rs:98-188. */
uint32_t jxrb_last_stage(void);

/* ---- sessions ------------------------------------------------------------ */

/* CudaDecoderSession::new(ordinal), session.rs:42-101. */
jxrb_status jxrb_session_create(int ordinal, const jxrb_session_options *options, jxrb_session **out);
/* CudaDecoderSession::system_default, session.rs:42-45: device 0, default options. */
jxrb_status jxrb_session_create_default(jxrb_session **out);
/* Drop of CudaDecoderSession: waits for pending work. */
void jxrb_session_destroy(jxrb_session *session);
/* CudaDecoderSession::buffer_pool_diagnostics / upload_cache_diagnostics, session.rs:250-268. */
jxrb_status jxrb_session_diagnostics(const jxrb_session *session, jxrb_diagnostics *out);

/* ---- plans --------------------------------------------------------------- */

/* CudaDecodePlan::from_prepared, crates/jxr-cuda/src/plan.rs:91-148: validates
 * the arena against the geometry (block shapes, one macroblock per window
 * position, coefficient ranges, no top-left high-pass prediction, non-zero
 * quantizers, tile partition) and the output policy, and builds the
 * per-plane macroblock tables.  `alpha` is the separate-alpha arena or NULL. */
jxrb_status jxrb_plan_create(const jxrb_arena *primary, const jxrb_arena *alpha,
                             const jxrb_image_geometry *geometry, const jxrb_output_format *output,
                             jxrb_plan **out);
void jxrb_plan_destroy(jxrb_plan *plan);
/* SurfaceLayout::byte_len of the plan's output, crates/jxr-core/src/surface.rs:28-142. */
uint64_t jxrb_plan_output_bytes(const jxrb_plan *plan);
/* Algorithmic device bytes of one reconstruction: coefficients + 16-byte
 * macroblock entries read, output written. */
uint64_t jxrb_plan_traffic_bytes(const jxrb_plan *plan);
/* Samples the plan's planes reconstruct: the work measure jxrb_plan_route
 * compares with JXRB_CUDA_AUTO_THRESHOLD. */
uint64_t jxrb_plan_reconstructed_coefficients(const jxrb_plan *plan);

/* SurfaceLayout / SurfacePlaneLayout, crates/jxr-core/src/surface.rs:10-27:
 * where each plane of the plan's output lies (one plane for interleaved
 * pixels, three or four for planar YUV, one a channel for NCHW). */
typedef struct jxrb_surface_plane {
    uint64_t byte_offset;
    uint64_t row_stride_bytes;
    uint32_t width, height;
    uint32_t channels;
} jxrb_surface_plane;
typedef struct jxrb_surface_layout {
    uint32_t width, height;
    uint64_t byte_len;
    uint32_t element_bytes;       /* bytes of one stored element (0 for one-bit) */
    uint32_t plane_count;
    jxrb_surface_plane planes[6];
} jxrb_surface_layout;
/* CudaSubmission::output_layout (crates/jxr-cuda/src/submission.rs:68) of a plan. */
jxrb_status jxrb_plan_output_layout(const jxrb_plan *plan, jxrb_surface_layout *out);
/* How the plan's 4 x 4-macroblock tiles split between the tile kernels:
 * interior tiles (full-resolution planes, 4:2:0), tiles on the plane's edge
 * away from hard tile boundaries (likewise) and the general kernel's tiles.
 * No counterpart in the reference: a diagnostic of this engine's launches. */
typedef struct jxrb_tile_kinds {
    uint32_t interior, interior_420, edge, edge_420, general;
} jxrb_tile_kinds;
jxrb_status jxrb_plan_tile_kinds(const jxrb_plan *plan, jxrb_tile_kinds *out);

/* ---- submissions ------------------------------------------------------- */

/* CudaDecoderSession::submit, session.rs:103-110: uploads the arena and
 * reconstructs into session-owned device memory. */
jxrb_status jxrb_submit(jxrb_session *session, const jxrb_plan *plan, jxrb_submission **out);
/* CudaDecoderSession::submit_into, session.rs:165-190: reconstructs into a
 * caller-owned device buffer of at least jxrb_plan_output_bytes bytes. */
jxrb_status jxrb_submit_into(jxrb_session *session, const jxrb_plan *plan, void *device_destination,
                             uint64_t destination_bytes, jxrb_submission **out);
/* CudaDecoderSession::submit_dense_batch / submit_batch_into, session.rs:126-212:
 * every image of `plans` in ONE launch over a shared work list (persistent
 * batch kernel); outputs packed densely in plan order into
 * `device_destination` (or session memory when NULL). */
jxrb_status jxrb_submit_batch(jxrb_session *session, const jxrb_plan *const *plans, uint32_t count,
                              void *device_destination, uint64_t destination_bytes, jxrb_submission **out);
/* CudaSubmission::wait, submission.rs:96-155.  timeout_ns < 0 waits forever. */
jxrb_status jxrb_wait(jxrb_submission *submission, int64_t timeout_ns);
/* CudaSubmission::is_complete, submission.rs:43-60. */
jxrb_status jxrb_is_complete(jxrb_submission *submission, int *complete);
/* CudaSubmission::enqueue_consumer_wait, submission.rs:62-80. */
jxrb_status jxrb_enqueue_consumer_wait(jxrb_submission *submission, void *cuda_stream);
/* CudaSubmission::pending_device_buffer, submission.rs:82-94: image `index`'s output. */
void *jxrb_submission_device_ptr(jxrb_submission *submission, uint32_t index);
/* CudaDecoderSession::readback / readback_batch_image, session.rs:221-248. */
jxrb_status jxrb_readback(jxrb_submission *submission, uint32_t index, void *host, uint64_t bytes);
/* Every output of a submission in one copy: the first `bytes` of its output
 * region as laid out on the device (plan order, each output 256-byte
 * aligned; image i starts at jxrb_submission_device_ptr(i) minus that of
 * image 0).  No counterpart in the reference, which reads back one image at
 * a time; for a batch this spares one synchronous copy an image. */
jxrb_status jxrb_readback_all(jxrb_submission *submission, void *host, uint64_t bytes);
/* Drop of CudaSubmission: waits before releasing (docs/cuda-backend.md:124-126). */
void jxrb_submission_destroy(jxrb_submission *submission);
/* CudaDecoderSession::decode_to_host, session.rs:214-219. */
jxrb_status jxrb_decode_to_host(jxrb_session *session, const jxrb_plan *plan, void *host, uint64_t bytes);
/* CudaDecoderSession::decode_batch_to_host, session.rs:221-235: every plan in
 * one batched launch, image i copied to hosts[i] (at most bytes[i]). */
jxrb_status jxrb_decode_batch_to_host(jxrb_session *session, const jxrb_plan *const *plans, uint32_t count,
                                      void *const *hosts, const uint64_t *bytes);

/* ---- caller-owned destinations --------------------------------------------
 * CudaDecoderSession::allocate_destination / allocate_batch_destination
 * (session.rs:85-101): zeroed device memory the caller owns and passes to
 * jxrb_submit_into / jxrb_submit_batch, released with jxrb_free_destination. */
jxrb_status jxrb_allocate_destination(jxrb_session *session, uint64_t bytes, void **device_destination);
/* The dense batch layout (DenseCudaBatchLayout, crates/jxr-cuda/src/destination.rs):
 * image i at offsets[i] (plan order, each 256-byte aligned; `offsets` may be
 * NULL), `bytes` in all. */
jxrb_status jxrb_batch_layout(const jxrb_plan *const *plans, uint32_t count, uint64_t *offsets, uint64_t *bytes);
jxrb_status jxrb_allocate_batch_destination(jxrb_session *session, const jxrb_plan *const *plans, uint32_t count,
                                            void **device_destination, uint64_t *bytes);
jxrb_status jxrb_free_destination(jxrb_session *session, void *device_destination);

/* ---- decode reports ---------------------------------------------------------
 * DecodeReport / StageReport (crates/jxr-core/src/report.rs:9-90) as the CUDA
 * plan builds it (decode_report, crates/jxr-cuda/src/plan.rs:214-253): the
 * host stages before the arena, the reconstruction stages on CUDA (fused into
 * one pass here), the host readback when one ran.  Extension: device-timed
 * upload and reconstruction (CUDA events; zero for request submissions) and
 * host-timed readback, in milliseconds. */
enum {
    JXRB_STAGE_PARSE = 0, JXRB_STAGE_ENTROPY_DECODE = 1, JXRB_STAGE_INVERSE_SCAN = 2,
    JXRB_STAGE_COEFFICIENT_REMAP = 3, JXRB_STAGE_DC_LOW_PASS_PREDICTION = 4,
    JXRB_STAGE_DEQUANTIZE_FIRST_TRANSFORM = 5, JXRB_STAGE_FIRST_OVERLAP = 6, JXRB_STAGE_HIGH_PASS_PREDICTION = 7,
    JXRB_STAGE_SECOND_TRANSFORM = 8, JXRB_STAGE_SECOND_OVERLAP = 9, JXRB_STAGE_CHROMA_RECONSTRUCTION = 10,
    JXRB_STAGE_COLOR_ALPHA_CONVERSION = 11, JXRB_STAGE_CROP_CLIP_PACK = 12, JXRB_STAGE_HOST_READBACK = 13
};
enum { JXRB_EXECUTOR_CPU_SCALAR = 0, JXRB_EXECUTOR_CPU_SIMD = 1, JXRB_EXECUTOR_METAL = 2, JXRB_EXECUTOR_CUDA = 3 };
typedef struct jxrb_stage_report {
    int32_t stage;
    int32_t executor;
} jxrb_stage_report;
typedef struct jxrb_decode_report {
    int32_t requested_backend;    /* JXRB_BACKEND_* */
    int32_t selected_backend;     /* JXRB_ROUTE_* */
    int32_t fallback;             /* 0: none (a submitted decode never falls back) */
    uint32_t stage_count;
    jxrb_stage_report stages[16];
    float upload_ms, reconstruct_ms, readback_ms;
} jxrb_decode_report;
/* The report of a submission (waits for it). */
jxrb_status jxrb_submission_report(jxrb_submission *submission, jxrb_decode_report *out);

/* ---- resident inputs ------------------------------------------------------
 * The upload cache of crates/jxr-cuda/src/upload_cache.rs:65-153 made
 * explicit: arenas uploaded once and reconstructed many times (benchmarks,
 * serving loops that keep coefficient buffers on the device). */
jxrb_status jxrb_resident_create(jxrb_session *session, const jxrb_plan *const *plans, uint32_t count,
                                 jxrb_resident **out);
/* Reconstruct every resident image into `device_destination` (outputs packed
 * in plan order) on `cuda_stream` (NULL: the session's first stream).
 * batched != 0: one launch over all images; 0: one launch per image. */
jxrb_status jxrb_resident_run(jxrb_resident *resident, void *device_destination, uint64_t destination_bytes,
                              int batched, void *cuda_stream);
/* Device status word of the resident set (0 when every launch succeeded). */
jxrb_status jxrb_resident_status(jxrb_resident *resident, uint32_t *status);
uint64_t jxrb_resident_output_bytes(const jxrb_resident *resident);
uint32_t jxrb_resident_launches(const jxrb_resident *resident, int batched);
void jxrb_resident_destroy(jxrb_resident *resident);

/* Launch shape of the tile kernels for a resident set, as chosen by the
 * autotuner (jxr_b200/autotune.py).  No reference counterpart: the reference
 * fixes 128-thread CTAs per macroblock (kernels/main.rs:98-207). */
typedef struct jxrb_launch_tuning {
    uint32_t blocks_per_sm[5];   /* resident CTAs per SM, 0 = as many as fit: entries 0..3 for interior tiles with
                                    1..4 full-resolution planes (entry 2 also for 4:2:0 interior tiles), entry 4 for
                                    the other tiles */
    int32_t side_stream;         /* 1: the edge and general tile kernels run on a second stream beside the interior ones */
} jxrb_launch_tuning;
jxrb_status jxrb_resident_set_tuning(jxrb_resident *resident, const jxrb_launch_tuning *tuning);
/* Capture the launch sequence of one run (batched != 0: the persistent batch
 * launch; 0: one launch per image) into a CUDA graph bound to
 * `device_destination`; jxrb_resident_replay launches it on `cuda_stream`.
 * No reference counterpart (the reference records no graphs). */
jxrb_status jxrb_resident_capture(jxrb_resident *resident, void *device_destination, uint64_t destination_bytes,
                                  int batched);
jxrb_status jxrb_resident_replay(jxrb_resident *resident, void *cuda_stream);

/* ---- resident images and requests (the serving path) ----------------------
 * An image whose coefficients, macroblock tables and tile maps are uploaded
 * once and stay on the device, as the reference's upload cache keeps them
 * (crates/jxr-cuda/src/upload_cache.rs:65-153).  Each request on it -- the
 * whole image, or a region -- then uploads only an image descriptor and a
 * tile work list, and any number of requests, on any resident images, run as
 * one batched launch. */
typedef struct jxrb_image jxrb_image;
typedef struct jxrb_request jxrb_request;
/* Validates the arena like jxrb_plan_create (window origin 0, the tile grid
 * covering the whole image) and uploads it.  The arena may be freed after. */
jxrb_status jxrb_image_create(jxrb_session *session, const jxrb_arena *primary, const jxrb_arena *separate_alpha,
                              const jxrb_image_geometry *geometry, jxrb_image **out);
uint64_t jxrb_image_device_bytes(const jxrb_image *image);
/* Images (like resident sets) belong to their session: destroy them before
 * it, and after the requests made on them.  The call does not wait: the
 * image's device memory returns to the pool once the session's streams have
 * finished the work enqueued before the call. */
void jxrb_image_destroy(jxrb_image *image);
/* A decode of the region `output->crop_*` (image sample coordinates; the
 * whole image for a full decode) into `output`'s format.  The engine
 * reconstructs the tiles the region needs -- the macroblocks it covers plus
 * one more on each side when overlap filtering or chroma interpolation
 * reaches them (reconstruction_bounds, crates/jxr-native/src/prepare.rs:321-352),
 * widened to whole tiles (Window::of_plan,
 * crates/jxr-native/src/decode/reconstruction.rs:509-546) -- and stores the
 * region only.  The image must outlive the request. */
jxrb_status jxrb_request_create(const jxrb_image *image, const jxrb_output_format *output, jxrb_request **out);
/* jxrb_request_create at 1/denominator of the resolution: 1, 4 or 16, the
 * reference's DecodeScale::{Full, Quarter, Sixteenth}
 * (crates/jxr-native/src/reconstruct/pipeline.rs:160-260, region scaling
 * prepare.rs:196-216).  A quarter: one sample a block, the block DC after the
 * first-level transform and overlap filter, scaled to the level it stands for
 * (SampleScale, reconstruct/sample_scale.rs); every macroblock of the window
 * must code the low-pass band (JXRB_UNSUPPORTED_OUTPUT otherwise).  A
 * sixteenth: one sample a macroblock, its DC (with two-level overlap the
 * first-level picture of the DC band summed over the macroblock), scaled
 * likewise; chroma has a sample for each macroblock as luma does, so it is
 * never interpolated and subsampled planar YUV output is refused.
 * `output->crop_*` is the region at full resolution; the output covers it at
 * the reduced resolution (x/d, y/d .. ceil((x+w)/d), ceil((y+h)/d)).  The
 * reference runs these on the CPU only; here they are GPU requests like any
 * other. */
jxrb_status jxrb_request_create_scaled(const jxrb_image *image, const jxrb_output_format *output, int denominator,
                                       jxrb_request **out);
void jxrb_request_destroy(jxrb_request *request);
uint64_t jxrb_request_output_bytes(const jxrb_request *request);
/* Compulsory bytes: window coefficients and macroblock table entries, plus the output. */
uint64_t jxrb_request_traffic_bytes(const jxrb_request *request);
/* The reconstruction window: origin x, y and extent x, y in macroblocks. */
jxrb_status jxrb_request_window(const jxrb_request *request, uint32_t window[4]);
/* One batched launch over `count` requests; outputs packed in request order,
 * each 256-byte aligned, in `device_destination` (or session memory when
 * NULL).  The submission is used like jxrb_submit_batch's. */
jxrb_status jxrb_submit_requests(jxrb_session *session, const jxrb_request *const *requests, uint32_t count,
                                 void *device_destination, uint64_t destination_bytes, jxrb_submission **out);

/* ---- presentation orientation ---------------------------------------------
 * The reference's Orientation (crates/jxr-core/src/format.rs:464-474) and
 * apply_orientation (crates/jxr/src/decoder/orientation.rs:5-211), which
 * JxrDecoder::decode_oriented applies to a full-image decode
 * (crates/jxr/src/decoder.rs:327-333). */
enum {
    JXRB_ORIENT_IDENTITY = 0, JXRB_ORIENT_MIRROR_HORIZONTAL = 1, JXRB_ORIENT_ROTATE180 = 2,
    JXRB_ORIENT_MIRROR_VERTICAL = 3, JXRB_ORIENT_TRANSPOSE = 4, JXRB_ORIENT_ROTATE90 = 5,
    JXRB_ORIENT_TRANSVERSE = 6, JXRB_ORIENT_ROTATE270 = 7
};
/* Bytes of the oriented surface: width and height swap for the four
 * transposing orientations; pixel_bytes 0 is one-bit luma, each row padded
 * to a whole byte. */
uint64_t jxrb_oriented_bytes(uint32_t width, uint32_t height, uint32_t pixel_bytes, int orientation);
/* Orient a packed, interleaved surface of `width` x `height` pixels of
 * `pixel_bytes` bytes each (at most 48; 0: one-bit luma) from
 * `device_source` into `device_destination` (jxrb_oriented_bytes bytes,
 * apart from the source) on `cuda_stream` (NULL: the legacy default
 * stream); pixels move whole, their channels in order.  Asynchronous: the
 * caller orders its reads after the stream.  A region decode, or planar
 * output, has no orientation in the reference (Unsupported there): orient
 * whole single-plane surfaces, or each NCHW channel plane on its own. */
jxrb_status jxrb_orient(const void *device_source, void *device_destination, uint32_t width, uint32_t height,
                        uint32_t pixel_bytes, int orientation, void *cuda_stream);

/* ---- forward analysis (the encoder's front half) ---------------------------
 * analyze_component, crates/jxr-native/src/analyze.rs:56-131, which the
 * reference runs on the CPU only: the prefilter over the sample plane
 * (overlap 1 and 2), the forward core transform of each block, the prefilter
 * over the plane of block DCs (overlap 2), the forward first-level transform
 * of each macroblock (block DCs halved first where `scaled`) and the
 * quantization of the three bands (Quantizer::quantize,
 * crates/jxr-math/src/quantization.rs:28-50; offsets of half the step for DC
 * and low-pass, a third for high-pass).  Device buffers throughout. */
typedef struct jxrb_analysis_plane {
    int32_t *samples;             /* width x height, row-major, 16-byte aligned; prefiltered in place */
    uint32_t width, height;       /* whole macroblocks: 16 x 16 samples, 8 x 16 (4:2:2) or 8 x 8 (4:2:0) chroma */
    uint32_t block_columns, block_rows;   /* 4 x 4, 2 x 4 or 2 x 2 */
    int32_t scaled;
    int32_t overlap;              /* 0, 1, 2 */
    uint32_t steps[3];            /* DC, low-pass, high-pass quantizer steps */
    const uint32_t *column_boundaries;    /* host: tile boundaries in macroblocks, 0 .. extent */
    uint32_t column_count;
    const uint32_t *row_boundaries;
    uint32_t row_count;
    int32_t hard_tiles;
    int32_t *low_scratch;         /* (width/4) x (height/4) */
    int32_t *low_q;               /* out: 16 a macroblock, raster: DC then low-pass, zero past the block count */
    int32_t *high_q;              /* out: 256 a macroblock: block b's coefficient k at b*16+k (k = 0 unused, zero) */
} jxrb_analysis_plane;
/* Analyse `count` planes on `cuda_stream` (NULL: the legacy default stream);
 * returns once the outputs are written. */
jxrb_status jxrb_analyze_planes(const jxrb_analysis_plane *planes, uint32_t count, void *cuda_stream);

/* ---- reconstruction without allocation ---------------------------------
 * No counterpart in the reference.  For callers that must not allocate
 * device memory at the time they decode: a serving loop whose memory budget
 * is already spent, code running inside an allocator's callbacks, or a
 * process that forbids device allocation after start-up.  Every other entry
 * point allocates per-submission descriptors; this one uses a fixed 4 MiB
 * scratch array that is part of the library (one per device) and calls no
 * allocating routine.
 *
 * Reconstructs `plan` from coefficients the caller already holds on device
 * `device` (`device_coefficients`: the primary arena's coefficients in arena
 * order; `device_alpha_coefficients`: the separate alpha arena's, or NULL)
 * into `device_destination` on `cuda_stream` (NULL: the legacy default
 * stream), and returns once the reconstruction has finished, with the same
 * error codes as jxrb_decode_to_host.  The output bytes equal those of the
 * other entry points for the same plan.
 *
 * Limits: the plan's descriptors (16 bytes a macroblock a plane, plus the
 * tile work list) must fit in 4 MiB, which a 4096 x 4096 three-plane image
 * does; a larger plan returns JXRB_RESOURCE_LIMIT with the sizes in
 * jxrb_last_error() and touches no device.
 * The first call on a device looks up the scratch array's address, which is
 * set-up work of its own; make that first call before any stream capture
 * begins on that device.  The call itself synchronises `cuda_stream` and
 * reads the status word back, so it cannot be made on a capturing stream.
 * The caller's current device is the same after the call as before it.
 * The scratch is shared by every call on a device, so calls that overlapped
 * would race on it: calls take a process-wide lock and return only after
 * their kernels have finished (on error paths too), so they run one at a
 * time. */
jxrb_status jxrb_decode_static(int device, const jxrb_plan *plan, const int32_t *device_coefficients,
                               const int32_t *device_alpha_coefficients, void *device_destination,
                               uint64_t destination_bytes, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif
