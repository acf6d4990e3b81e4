// Calibration of the integer roofline the motion-estimation kernels are measured against: the
// rate at which this GPU executes the block-difference term acc += |a - b| on register-resident
// 32-bit integers (subtract, absolute value, add: the three operations a search counts per
// pixel and candidate).  Sixty-four independent terms per loop iteration over eight
// accumulators keep every integer pipe busy; one more addition per iteration carries a
// dependency through the loop so that nothing can be hoisted.

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int CAL_THREADS = 256;
constexpr int CAL_TERMS = 64;  // |a - b| terms per iteration and thread

__global__ void __launch_bounds__(CAL_THREADS) int_rate_kernel(int iters, int seed, int* sink) {
    int x[8], acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = seed * (int)(threadIdx.x + 37 * k) + (int)blockIdx.x;
        acc[k] = 0;
    }
    int y = seed ^ (int)blockIdx.x;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += abs(x[k] - (y + 3 * j));
        y += acc[it & 7];
    }
    int s = y;
#pragma unroll
    for (int k = 0; k < 8; ++k) s ^= acc[k];
    if (s == 0x7fffffff) *sink = s;  // keeps the work observable
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_measure_int_rate(double* ops_per_second) {
    if (!ops_per_second) return DGPU_ERR_ARG;
    int dev = 0, sms = 0;
    DGPU_CHECK_CUDA(cudaGetDevice(&dev));
    DGPU_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int* sink = nullptr;
    DGPU_CHECK_CUDA(cudaMalloc(&sink, sizeof(int)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = DGPU_OK;
    const int blocks = sms * 8, iters = 2048;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = DGPU_ERR_CUDA;
    float ms = 0.0f;
    for (int rep = 0; rep < 2 && rc == DGPU_OK; ++rep) {  // the first run warms clocks and caches
        cudaEventRecord(e0);
        int_rate_kernel<<<blocks, CAL_THREADS>>>(iters, 12345 + rep, sink);
        count_launch();
        cudaEventRecord(e1);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            rc = DGPU_ERR_CUDA;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    if (rc != DGPU_OK || ms <= 0.0f) return rc != DGPU_OK ? rc : DGPU_ERR_CUDA;
    const double ops = (double)blocks * CAL_THREADS * iters * (3.0 * CAL_TERMS + 1.0);
    *ops_per_second = ops / (ms * 1e-3);
    return DGPU_OK;
}
