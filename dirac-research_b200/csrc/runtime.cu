// Library-wide runtime pieces: version, device check, last-error record and the
// per-device scratch buffer used when callers pass no scratch.

#include <atomic>
#include <cstdio>
#include <mutex>

#include "dgpu_internal.cuh"

namespace dgpu {

namespace {
std::mutex g_err_mu;
char g_last_error[512] = "";

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch[kMaxDevices] = {};
size_t g_scratch_bytes[kMaxDevices] = {};
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
}

int library_scratch(size_t bytes, void** out) {
    int dev = 0;
    DGPU_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return DGPU_ERR_DEVICE;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch_bytes[dev] < bytes) {
        if (g_scratch[dev]) {
            // kernels queued earlier may still read the old buffer
            DGPU_CHECK_CUDA(cudaDeviceSynchronize());
            cudaFree(g_scratch[dev]);
            g_scratch[dev] = nullptr;
            g_scratch_bytes[dev] = 0;
        }
        size_t want = align_up(bytes, 1 << 20);
        if (cudaMalloc(&g_scratch[dev], want) != cudaSuccess) {
            cudaGetLastError();
            g_scratch[dev] = nullptr;
            return DGPU_ERR_NOMEM;
        }
        g_scratch_bytes[dev] = want;
    }
    *out = g_scratch[dev];
    return DGPU_OK;
}

}  // namespace dgpu

extern "C" const char* dgpu_version(void) { return "dirac-b200 0.1 (sm_100a)"; }

extern "C" const char* dgpu_last_error(void) { return dgpu::g_last_error; }

extern "C" unsigned long long dgpu_launch_count(void) { return dgpu::g_launches.load(); }

extern "C" int dgpu_device_check(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return DGPU_ERR_DEVICE;
    }
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return DGPU_ERR_DEVICE;
    if (p.major != 10) return DGPU_ERR_DEVICE;
    return p.major * 10 + p.minor;
}
