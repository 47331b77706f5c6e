// vnlb.Aggregate for one output frame without any allocation.
//
// The frame's contributing stack rows, its source rows and its output rows
// pass through one fixed device scratch, a file-scope __device__ array of
// kNoAllocScratchBytes, in bands of whole rows.  The call makes no cudaMalloc
// or cudaFree and uses no allocating library routine.  It exists for callers
// that cannot allocate device memory while they serve frames.  An example is
// a frame server that reserves its device memory budget when it starts and
// shares the GPU with other filters: there a cudaMalloc in the middle of a
// clip can fail under memory pressure, and a cudaFree waits for all work on
// the device.  The reference has no counterpart; its render_aggregate_frame
// (src/vs/plugin.cpp:966-1045) sums on the CPU.
//
// Arithmetic per sample: the numerators and weights of the contributing
// anchor stacks, summed in anchor order and rounded at each step, then
// numerator / weight, or the source sample where the weight sum is not
// positive.  These are the operations of the whole-clip aggregate kernel, so
// the two agree bit for bit.
//
// Set-up: the first call on a device, with that device current, looks up the
// scratch's device address with cudaGetSymbolAddress.  That first call can
// also be what loads this library's device code on the device.  Make the
// first call on each device before any stream capture begins.
//
// Races: there is one scratch per device.  Calls whose GPU work overlapped
// would race on it.  This file prevents that by holding a per-device host
// lock from the set-up until the call's stream work has finished, on the
// error paths too: once a copy or the kernel has been queued, an error return
// first drains the stream.
//
// Stream: every call queues its copies and kernel on the legacy default
// stream.  So a call waits for the caller's blocking streams on that device,
// and it must not run while one of them is being captured.
//
// Current device: the call makes device_id current while it runs and puts
// back the caller's current device before it returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr size_t kNoAllocScratchFloats = kNoAllocScratchBytes / sizeof(float);
constexpr int kNoAllocMaxDevices = 64;

// Band layout, for a band of `rows` rows of width W (band = rows * W):
//   [count][C][2][band]  numerators, then weights, of each contributing stack
//   [C][band]            source rows
//   [C][band]            output rows
// Every value the kernel reads is written by that band's copies first, so no
// part of the scratch has to start at zero.
__device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

std::mutex g_noalloc_lock[kNoAllocMaxDevices];  // held for a whole call
float* g_noalloc_ptr[kNoAllocMaxDevices];       // scratch address per device; null until set up

thread_local char g_noalloc_message[256];

const char* message(const char* format, long long a = 0, long long b = 0, long long c = 0, long long d = 0) {
    std::snprintf(g_noalloc_message, sizeof(g_noalloc_message), format, a, b, c, d);
    return g_noalloc_message;
}

const char* cuda_message(const char* what, cudaError_t status) {
    std::snprintf(g_noalloc_message, sizeof(g_noalloc_message), "VNLB CUDA: %s failed: %s", what,
                  cudaGetErrorString(status));
    return g_noalloc_message;
}

// Puts back the calling thread's current device on every return path.
struct DeviceRestore {
    int previous = -1;
    DeviceRestore() {
        if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
    }
    ~DeviceRestore() {
        if (previous >= 0) cudaSetDevice(previous);
    }
};

struct BandLaunch {
    int width, rows, channels, count;
    float* scratch;
};

__global__ void aggregate_band_kernel(BandLaunch L) {
    const size_t band = static_cast<size_t>(L.width) * L.rows;
    const size_t total = band * L.channels;
    const float* stage = L.scratch;
    const float* source = stage + static_cast<size_t>(L.count) * L.channels * 2 * band;
    float* out = L.scratch + static_cast<size_t>(L.count) * L.channels * 2 * band + total;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(i / band);
        const size_t p = i - static_cast<size_t>(c) * band;
        float num = 0.0f, w = 0.0f;
        for (int k = 0; k < L.count; ++k) {
            const float* s = stage + (static_cast<size_t>(k) * L.channels + c) * 2 * band;
            num = __fadd_rn(num, s[p]);
            w = __fadd_rn(w, s[band + p]);
        }
        out[i] = w > 0.0f ? __fdiv_rn(num, w) : source[i];
    }
}

}  // namespace

const char* aggregate_frame_noalloc(const float* stacks, const float* source, int width, int height, int frames,
                                    int channels, int search_bwd, int search_fwd, int patch_time, int device_id,
                                    int n, float* out) {
    // argument checks, before any CUDA call
    if (!stacks || !source || !out) return "VNLB: null argument";
    if (width <= 0 || height <= 0 || frames <= 0 || !(channels == 1 || channels == 3))
        return "VNLB: Aggregate requires matching constant GrayS or YUV444PS clips";
    if (patch_time <= 0 || search_bwd < 0 || search_fwd < 0)
        return "VNLB: patch_time must be positive and search_bwd/search_fwd must be non-negative";
    const int slots = search_bwd + search_fwd + patch_time;
    if (slots > kMaxContributors) return "VNLB: at most 32 contribution slots are supported";
    if (n < 0 || n >= frames) return message("VNLB: output frame %lld is outside the clip of %lld frames", n, frames);
    if (device_id < 0 || device_id >= kNoAllocMaxDevices)
        return message("VNLB CUDA: device %lld is outside the %lld devices this call supports", device_id,
                       kNoAllocMaxDevices);

    // contributing anchors of frame n, in anchor order (render_aggregate_frame)
    const int first = std::max(0, n - (search_fwd + patch_time - 1));
    const int last = std::min(frames - 1, n + search_bwd);
    const int count = last - first + 1;
    const size_t row_floats = (static_cast<size_t>(count) * channels * 2 + 2 * static_cast<size_t>(channels)) * width;
    if (row_floats > kNoAllocScratchFloats)
        return message("VNLB: Aggregate without allocation stages at most %lld bytes per band of rows; one row of "
                       "this frame needs %lld bytes (width %lld, %lld contributing stacks)",
                       static_cast<long long>(kNoAllocScratchBytes), static_cast<long long>(row_floats * sizeof(float)),
                       width, count);
    const int band_rows = static_cast<int>(std::min<size_t>(height, kNoAllocScratchFloats / row_floats));

    std::lock_guard<std::mutex> guard(g_noalloc_lock[device_id]);
    DeviceRestore restore;  // destroyed before the lock is released
    cudaError_t status = cudaSetDevice(device_id);
    if (status != cudaSuccess) return cuda_message("cudaSetDevice", status);
    if (!g_noalloc_ptr[device_id]) {
        float* ptr = nullptr;
        status = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch);
        if (status != cudaSuccess) return cuda_message("cudaGetSymbolAddress(aggregate scratch)", status);
        g_noalloc_ptr[device_id] = ptr;
    }
    float* scratch = g_noalloc_ptr[device_id];
    const cudaStream_t stream = nullptr;  // legacy default stream, as the whole-clip aggregate uses
    // An error after work was queued: wait for that work before the lock is
    // released, so that no later call overwrites a scratch still in use.
    auto drained = [stream](const char* what, cudaError_t error) {
        cudaStreamSynchronize(stream);
        return cuda_message(what, error);
    };

    const size_t plane = static_cast<size_t>(width) * height;
    const size_t stack_values = plane * channels * slots * 2;
    for (int y0 = 0; y0 < height; y0 += band_rows) {
        const int rows = std::min(band_rows, height - y0);
        const size_t band = static_cast<size_t>(width) * rows;
        const size_t bytes = band * sizeof(float);
        // stack rows: slot s of anchor a holds its numerator rows at s*2*H and
        // its weight rows at s*2*H + H of each plane [slots*2*H][W]
        for (int k = 0; k < count; ++k) {
            const int a = first + k;
            const int slot = n - a + search_bwd;
            for (int c = 0; c < channels; ++c) {
                const float* plane_base = stacks + stack_values * a + static_cast<size_t>(c) * slots * 2 * plane;
                const float* num_rows = plane_base + (static_cast<size_t>(slot) * 2 * height + y0) * width;
                const float* weight_rows = num_rows + plane;
                float* dst = scratch + (static_cast<size_t>(k) * channels + c) * 2 * band;
                status = cudaMemcpyAsync(dst, num_rows, bytes, cudaMemcpyHostToDevice, stream);
                if (status != cudaSuccess) return drained("cudaMemcpyAsync(stack band)", status);
                status = cudaMemcpyAsync(dst + band, weight_rows, bytes, cudaMemcpyHostToDevice, stream);
                if (status != cudaSuccess) return drained("cudaMemcpyAsync(stack band)", status);
            }
        }
        float* src_band = scratch + static_cast<size_t>(count) * channels * 2 * band;
        float* out_band = src_band + band * channels;
        for (int c = 0; c < channels; ++c) {
            const float* src = source + plane * channels * n + static_cast<size_t>(c) * plane +
                               static_cast<size_t>(y0) * width;
            status = cudaMemcpyAsync(src_band + c * band, src, bytes, cudaMemcpyHostToDevice, stream);
            if (status != cudaSuccess) return drained("cudaMemcpyAsync(source band)", status);
        }
        BandLaunch L{width, rows, channels, count, scratch};
        const size_t total = band * channels;
        const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
        aggregate_band_kernel<<<blocks, 256, 0, stream>>>(L);
        status = cudaGetLastError();
        if (status != cudaSuccess) return drained("aggregate band kernel launch", status);
        for (int c = 0; c < channels; ++c) {
            float* dst = out + static_cast<size_t>(c) * plane + static_cast<size_t>(y0) * width;
            status = cudaMemcpyAsync(dst, out_band + c * band, bytes, cudaMemcpyDeviceToHost, stream);
            if (status != cudaSuccess) return drained("cudaMemcpyAsync(output band)", status);
        }
    }
    // the output is on the host, and the scratch free for the next call, once
    // the stream has drained
    status = cudaStreamSynchronize(stream);
    if (status != cudaSuccess) return cuda_message("cudaStreamSynchronize", status);
    return nullptr;
}

}  // namespace vnlbgpu
