// static_scratch.cu -- jxrb_decode_static, the entry point that allocates nothing.
//
// Every other entry point keeps the per-launch descriptors (image
// descriptor, tile work list, status word, scheduling counters, macroblock
// tables, tile-start maps) in device memory it allocates per submission.
// This one keeps them in a fixed array of device memory that is part of the
// library itself, so that callers which may not allocate -- code that runs
// while a memory budget is exhausted, inside an allocator's own callbacks, or
// under a policy that forbids device allocation after start-up -- can still
// reconstruct an image whose coefficients they already hold on the device.
//
// Limits: the descriptors of one plan must fit in kScratchBytes (4 MiB), which
// holds a 4096 x 4096 three-plane image (3 x 65,536 macroblocks of 16 bytes
// each, plus the work list); larger plans are refused with
// JXRB_RESOURCE_LIMIT before any device work.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/jxr_b200.h"
#include "engine.h"

namespace jxr {
cudaError_t launch_tiles(const ImageDev *images, const void *items, const uint32_t *bounds, int max_planes,
                         uint32_t *status, uint32_t *counters, cudaStream_t stream, cudaStream_t side,
                         cudaEvent_t fork, cudaEvent_t join, const LaunchTuning *tune);
size_t staged_bytes(const jxrb_plan &plan);
jxrb_status stage_plan(const jxrb_plan *plan, const int32_t *coefficients, const int32_t *alpha_coefficients,
                       uint8_t *dst, uint64_t dst_bytes, uint8_t *host, uint8_t *device, size_t capacity,
                       StagedLayout &layout);
jxrb_status report_error(jxrb_status s, const char *why);
jxrb_status report_cuda(cudaError_t e, const char *what);
jxrb_status report_status_word(uint32_t word);
}  // namespace jxr

namespace {

constexpr size_t kScratchBytes = size_t(4) << 20;
constexpr int kMaxDevices = 64;

// The descriptor scratch: one copy per device, created with the module.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host image of the descriptors, written by the planner and copied to the
// scratch in one transfer.
alignas(256) unsigned char g_stage[kScratchBytes];

// The scratch's device address, looked up once per device.
void *g_scratch_ptr[kMaxDevices] = {};

// One call at a time: the scratch and its host image are shared.
std::mutex g_lock;

// Set-up, once per device with that device current: the address of the
// scratch array on it.
jxrb_status scratch_address(int device, unsigned char **out) {
    if (!g_scratch_ptr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess) return jxr::report_cuda(e, "cudaGetSymbolAddress (descriptor scratch)");
        g_scratch_ptr[device] = ptr;
    }
    *out = static_cast<unsigned char *>(g_scratch_ptr[device]);
    return JXRB_OK;
}

}  // namespace

extern "C" jxrb_status jxrb_decode_static(int device, const jxrb_plan *plan, const int32_t *device_coefficients,
                                          const int32_t *device_alpha_coefficients, void *device_destination,
                                          uint64_t destination_bytes, void *cuda_stream) {
    if (!plan) return jxr::report_error(JXRB_INVALID_PLAN, "null plan");
    const size_t need = jxr::staged_bytes(*plan);
    if (need > kScratchBytes) {
        char why[160];
        std::snprintf(why, sizeof why,
                      "plan needs %zu bytes of descriptor scratch; the allocation-free path holds at most %zu",
                      need, kScratchBytes);
        return jxr::report_error(JXRB_RESOURCE_LIMIT, why);
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return jxr::report_error(JXRB_UNAVAILABLE, "no CUDA device");
    }
    if (device < 0 || device >= n || device >= kMaxDevices)
        return jxr::report_error(JXRB_UNAVAILABLE, "device ordinal out of range");
    std::lock_guard<std::mutex> guard(g_lock);
    // the caller's current device is put back on every return
    int previous = 0;
    cudaError_t e = cudaGetDevice(&previous);
    if (e != cudaSuccess) return jxr::report_cuda(e, "cudaGetDevice");
    struct RestoreDevice {
        int device;
        ~RestoreDevice() { cudaSetDevice(device); }
    } restore{previous};
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return jxr::report_cuda(e, "cudaSetDevice");
    unsigned char *scratch = nullptr;
    jxrb_status st = scratch_address(device, &scratch);
    if (st != JXRB_OK) return st;
    // descriptors (status word and counters zero) into the host image, then
    // into the scratch
    jxr::StagedLayout layout{};
    st = jxr::stage_plan(plan, device_coefficients, device_alpha_coefficients,
                         static_cast<uint8_t *>(device_destination), destination_bytes, g_stage, scratch,
                         kScratchBytes, layout);
    if (st != JXRB_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    // From the upload on, every return waits for the stream first: the lock
    // is what keeps the next call off the scratch and its host image, so it
    // must not be released while this call's copy or kernels still run.
    auto drained = [&](jxrb_status s) {
        cudaStreamSynchronize(stream);
        cudaGetLastError();
        return s;
    };
    e = cudaMemcpyAsync(scratch, g_stage, layout.bytes, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return drained(jxr::report_cuda(e, "descriptor upload"));
    // 1-bit outputs set bits with atomics and need a zeroed destination
    if (layout.clear_bytes) {
        e = cudaMemsetAsync(device_destination, 0, layout.clear_bytes, stream);
        if (e != cudaSuccess) return drained(jxr::report_cuda(e, "clear bit output"));
    }
    uint32_t *status = reinterpret_cast<uint32_t *>(scratch + layout.status_at);
    e = jxr::launch_tiles(reinterpret_cast<const jxr::ImageDev *>(scratch), scratch + layout.items_at, layout.bounds,
                          layout.max_planes, status, reinterpret_cast<uint32_t *>(scratch + layout.counters_at),
                          stream, nullptr, nullptr, nullptr, nullptr);
    if (e != cudaSuccess) return drained(jxr::report_cuda(e, "kernel launch"));
    uint32_t word = 0;
    e = cudaMemcpyAsync(&word, status, sizeof word, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return drained(jxr::report_cuda(e, "status readback"));
    return jxr::report_status_word(word);
}
