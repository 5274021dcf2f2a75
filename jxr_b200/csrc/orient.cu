// orient.cu -- the presentation orientation of a decoded surface on the GPU.
//
// The reference applies an image's orientation (EXIF-like: mirrors,
// rotations, transposes) to the decoded host samples after the decode
// (apply_orientation, crates/jxr/src/decoder/orientation.rs:5-211, called by
// JxrDecoder::decode_oriented, crates/jxr/src/decoder.rs:327-333).  Here it is
// a device pass over the surface the engine left in HBM: each CTA writes one
// 32 x 32-pixel tile of the oriented surface, reading the source rectangle
// that tile comes from into shared memory first, so that both the reads and
// the writes run along rows.  Pixels move whole, their channels in order;
// one-bit luma (rows padded to bytes, most significant bit first) moves bit
// by bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/jxr_b200.h"

namespace jxr {
jxrb_status report_error(jxrb_status s, const char *why);
jxrb_status report_cuda(cudaError_t e, const char *what);
}  // namespace jxr

namespace {

constexpr int kTile = 32;
constexpr uint32_t kMaxPixelBytes = 48;   // a 32 x 32 tile of them fills 48 KB of shared memory

__device__ __forceinline__ bool swaps_axes(int o) { return o >= JXRB_ORIENT_TRANSPOSE; }

// source_coordinates (orientation.rs:193-211): the source pixel of
// destination pixel (dx, dy) of a w x h source.
__device__ __forceinline__ void source_of(int o, uint32_t w, uint32_t h, uint32_t dx, uint32_t dy, uint32_t &sx,
                                          uint32_t &sy) {
    switch (o) {
    case JXRB_ORIENT_MIRROR_HORIZONTAL: sx = w - 1 - dx; sy = dy; break;
    case JXRB_ORIENT_ROTATE180: sx = w - 1 - dx; sy = h - 1 - dy; break;
    case JXRB_ORIENT_MIRROR_VERTICAL: sx = dx; sy = h - 1 - dy; break;
    case JXRB_ORIENT_TRANSPOSE: sx = dy; sy = dx; break;
    case JXRB_ORIENT_ROTATE90: sx = dy; sy = h - 1 - dx; break;
    case JXRB_ORIENT_TRANSVERSE: sx = w - 1 - dy; sy = h - 1 - dx; break;
    case JXRB_ORIENT_ROTATE270: sx = w - 1 - dy; sy = dx; break;
    default: sx = dx; sy = dy;
    }
}

// One destination tile of 32 x 32 pixels, `words` words of type W a pixel.
// The source pixels of a tile form a rectangle of at most 32 x 32 (every
// orientation maps rows and columns to rows or columns); it is staged in
// shared memory, then written out along destination rows.
template <typename W>
__global__ void __launch_bounds__(256) jxrb_orient_tiles(const W *__restrict__ src, W *__restrict__ dst, uint32_t w,
                                                        uint32_t h, uint32_t words, int o) {
    extern __shared__ __align__(16) unsigned char orient_smem[];
    W *tile = reinterpret_cast<W *>(orient_smem);
    const bool swap = swaps_axes(o);
    const uint32_t ow = swap ? h : w, oh = swap ? w : h;
    const uint32_t dx0 = blockIdx.x * kTile, dy0 = blockIdx.y * kTile;
    const uint32_t dx1 = min(dx0 + kTile, ow), dy1 = min(dy0 + kTile, oh);
    // the source rectangle: the extremes of the tile's corners
    uint32_t ax, ay, bx, by;
    source_of(o, w, h, dx0, dy0, ax, ay);
    source_of(o, w, h, dx1 - 1, dy1 - 1, bx, by);
    const uint32_t sx0 = min(ax, bx), sy0 = min(ay, by), sx1 = max(ax, bx) + 1, sy1 = max(ay, by) + 1;
    const uint32_t sw = sx1 - sx0, sh = sy1 - sy0;
    const uint32_t row_words = sw * words;
    for (uint32_t i = threadIdx.x; i < row_words * sh; i += blockDim.x) {
        const uint32_t r = i / row_words, c = i - r * row_words;
        tile[i] = src[((size_t)(sy0 + r) * w + sx0) * words + c];
    }
    __syncthreads();
    const uint32_t dw = dx1 - dx0, out_words = dw * words;
    for (uint32_t i = threadIdx.x; i < out_words * (dy1 - dy0); i += blockDim.x) {
        const uint32_t r = i / out_words, c = i - r * out_words;
        const uint32_t px = c / words, k = c - px * words;
        uint32_t sx, sy;
        source_of(o, w, h, dx0 + px, dy0 + r, sx, sy);
        dst[((size_t)(dy0 + r) * ow + dx0) * words + c] = tile[((sy - sy0) * sw + (sx - sx0)) * words + k];
    }
}

// One-bit luma: one destination byte a thread (orient_bitpacked,
// orientation.rs:93-162).
__global__ void __launch_bounds__(256) jxrb_orient_bits(const uint8_t *__restrict__ src, uint8_t *__restrict__ dst,
                                                       uint32_t w, uint32_t h, int o) {
    const bool swap = swaps_axes(o);
    const uint32_t ow = swap ? h : w, oh = swap ? w : h;
    const uint32_t in_stride = (w + 7) / 8, out_stride = (ow + 7) / 8;
    const size_t n = (size_t)out_stride * oh;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t y = (uint32_t)(i / out_stride), xb = (uint32_t)(i % out_stride);
        uint32_t byte = 0;
        for (uint32_t b = 0; b < 8; b++) {
            const uint32_t x = xb * 8 + b;
            if (x >= ow) break;
            uint32_t sx, sy;
            source_of(o, w, h, x, y, sx, sy);
            if (src[(size_t)sy * in_stride + sx / 8] & (0x80u >> (sx % 8))) byte |= 0x80u >> b;
        }
        dst[i] = (uint8_t)byte;
    }
}

template <typename W>
cudaError_t launch_tiles(const void *src, void *dst, uint32_t w, uint32_t h, uint32_t words, int o,
                         cudaStream_t stream) {
    const bool swap = o >= JXRB_ORIENT_TRANSPOSE;
    const uint32_t ow = swap ? h : w, oh = swap ? w : h;
    const dim3 grid((ow + kTile - 1) / kTile, (oh + kTile - 1) / kTile);
    const size_t smem = (size_t)kTile * kTile * words * sizeof(W);
    jxrb_orient_tiles<W><<<grid, 256, smem, stream>>>(static_cast<const W *>(src), static_cast<W *>(dst), w, h, words,
                                                      o);
    return cudaGetLastError();
}

}  // namespace

extern "C" uint64_t jxrb_oriented_bytes(uint32_t width, uint32_t height, uint32_t pixel_bytes, int orientation) {
    const bool swap = orientation >= JXRB_ORIENT_TRANSPOSE;
    const uint64_t ow = swap ? height : width, oh = swap ? width : height;
    return pixel_bytes ? ow * oh * pixel_bytes : (ow + 7) / 8 * oh;
}

extern "C" jxrb_status jxrb_orient(const void *device_source, void *device_destination, uint32_t width,
                                   uint32_t height, uint32_t pixel_bytes, int orientation, void *cuda_stream) {
    if (orientation < JXRB_ORIENT_IDENTITY || orientation > JXRB_ORIENT_ROTATE270)
        return jxr::report_error(JXRB_INVALID_PLAN, "orientation code");
    if (!device_source || !device_destination) return jxr::report_error(JXRB_INVALID_DESTINATION, "null surface");
    if (device_source == device_destination)
        return jxr::report_error(JXRB_INVALID_DESTINATION, "orientation needs a destination apart from its source");
    if (pixel_bytes > kMaxPixelBytes)
        return jxr::report_error(JXRB_UNSUPPORTED_OUTPUT, "orientation of pixels above 48 bytes");
    if (width == 0 || height == 0) return JXRB_OK;
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e;
    if (pixel_bytes == 0) {
        const uint64_t n = jxrb_oriented_bytes(width, height, 0, orientation);
        const unsigned blocks = (unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
        jxrb_orient_bits<<<blocks, 256, 0, stream>>>(static_cast<const uint8_t *>(device_source),
                                                    static_cast<uint8_t *>(device_destination), width, height,
                                                    orientation);
        e = cudaGetLastError();
    } else {
        // the widest word that divides the pixel and both surfaces' alignment
        const uintptr_t a = reinterpret_cast<uintptr_t>(device_source) | reinterpret_cast<uintptr_t>(device_destination);
        if (pixel_bytes % 4 == 0 && a % 4 == 0)
            e = launch_tiles<uint32_t>(device_source, device_destination, width, height, pixel_bytes / 4, orientation,
                                       stream);
        else if (pixel_bytes % 2 == 0 && a % 2 == 0)
            e = launch_tiles<uint16_t>(device_source, device_destination, width, height, pixel_bytes / 2, orientation,
                                       stream);
        else
            e = launch_tiles<uint8_t>(device_source, device_destination, width, height, pixel_bytes, orientation,
                                      stream);
    }
    if (e != cudaSuccess) return jxr::report_cuda(e, "orientation launch");
    return JXRB_OK;
}
