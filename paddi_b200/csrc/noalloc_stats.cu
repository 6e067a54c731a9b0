// noalloc_stats.cu -- window statistics that allocate no device memory.
//
// Some callers cannot let a library call cudaMalloc:
//   * hosts that hand out all device memory through their own allocator and
//     treat any other allocation as a budget violation (JVM / .NET / FFI
//     embeddings with a managed device pool, multi-tenant servers with a
//     fixed per-tenant budget);
//   * latency-critical loops, where cudaMalloc / cudaFree can synchronise the
//     device and stall unrelated streams.
// paddi_compute_statistics_noalloc serves them.  It runs the same kernels as
// paddi_compute_statistics, with the statistics kernel's scratch arrays (per
// window: float4 update terms, float mean, FP64 mean and inverse norm, flat
// flag; one flat-window counter) in the file-scope device array below.  That
// array is fixed at PADDI_NOALLOC_MAX_WINDOWS windows (about 5 MB) and stays
// on every device that loads the library until the process exits.
//
// Rules a caller must follow:
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress; make that first call before any stream capture
//     begins on the device.  Every later call that is not being captured
//     resolves it again (a host-side lookup), so the address stays right after
//     cudaDeviceReset or under another context of the same device; a call
//     under capture uses the address of the device's last uncaptured call;
//   * every call on a device uses the same array, so calls whose GPU work can
//     overlap (other streams, other host threads) race with each other: keep
//     them on one stream, one after another;
//   * larger inputs are refused with PADDI_ERR_INVALID_ARG before anything is
//     enqueued.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/paddi.h"
#include "paddi_internal.cuh"

#define PADDI_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr size_t kSlots = (size_t)PADDI_NOALLOC_MAX_WINDOWS + PADDI_PAD_WIN; // + zeroed tail
constexpr size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kOffWst = 0;
constexpr size_t kOffMu = kOffWst + up256(sizeof(float4) * kSlots);
constexpr size_t kOffMu64 = kOffMu + up256(sizeof(float) * kSlots);
constexpr size_t kOffInv64 = kOffMu64 + up256(sizeof(double) * kSlots);
constexpr size_t kOffFlat = kOffInv64 + up256(sizeof(double) * kSlots);
constexpr size_t kOffCount = kOffFlat + up256(kSlots);
constexpr size_t kBytes = kOffCount + 256;

constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char *g_base[kMaxDevices] = {}; // device address of the scratch, per device

} // namespace

// The scratch itself.  In host code this name is only a stand-in for the
// device symbol; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_stats_scratch[kBytes];

PADDI_API paddi_status paddi_compute_statistics_noalloc(const float *d_T, float *d_mean,
                                                        float *d_std, size_t n, uint32_t m,
                                                        void *stream)
{
    if (!d_T || !d_mean || !d_std || m < 3 || m > 1024 || n < 2 * (size_t)m)
        return PADDI_ERR_INVALID_ARG;
    const size_t N = n - m + 1;
    if (N > (size_t)PADDI_NOALLOC_MAX_WINDOWS) return PADDI_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return PADDI_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kMaxDevices) return PADDI_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // under stream capture the lookup is not repeated (nor is anything but the
    // two kernels and the memset enqueued); otherwise it is, so a module that
    // was loaded again (device reset, another context) is found at its new address
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        cudaGetLastError();
        cap = cudaStreamCaptureStatusActive; // unknown: treat as captured
    }
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> g(g_lock);
        if (!g_base[dev] || cap == cudaStreamCaptureStatusNone) {
            // set-up with this device current: the scratch's device address
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_stats_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return PADDI_ERR_CUDA;
            }
            g_base[dev] = static_cast<unsigned char *>(p);
        }
        base = g_base[dev];
    }
    int32_t *count = reinterpret_cast<int32_t *>(base + kOffCount);
    double *mu64 = reinterpret_cast<double *>(base + kOffMu64);
    double *inv64 = reinterpret_cast<double *>(base + kOffInv64);
    // the flat-window counter is accumulated with atomics: it must start at 0
    if (cudaMemsetAsync(count, 0, sizeof(int32_t), st) != cudaSuccess) {
        cudaGetLastError();
        return PADDI_ERR_CUDA;
    }
    cudaError_t e = paddi_launch_stats(d_T, (int64_t)n, (int32_t)m,
                                       reinterpret_cast<float4 *>(base + kOffWst),
                                       reinterpret_cast<float *>(base + kOffMu), mu64, inv64,
                                       base + kOffFlat, count, st);
    if (e == cudaSuccess)
        e = paddi_launch_export_stats(mu64, inv64, (int32_t)N, (int32_t)m, d_mean, d_std, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return PADDI_ERR_CUDA;
    }
    return PADDI_OK;
}
