// Internal helpers shared by the CUDA translation units of libdiracgpu.
#pragma once

#include <cuda_runtime.h>
#include <functional>
#include <stddef.h>
#include <stdint.h>

#include "dirac_gpu.h"

namespace dgpu {

#define DGPU_CHECK_CUDA(expr)                                 \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) {                              \
            dgpu::set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
            return DGPU_ERR_CUDA;                             \
        }                                                     \
    } while (0)

// Every kernel launch of the library goes through this check, which also counts it
// (dgpu_launch_count reports the running total).
#define DGPU_CHECK_LAUNCH()                  \
    do {                                     \
        dgpu::count_launch();                \
        DGPU_CHECK_CUDA(cudaGetLastError()); \
    } while (0)

void count_launch();
// Adds n launches to the running total (kernels replayed from a captured CUDA graph).
void count_launches(unsigned long long n);

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Scratch owned by the library, one buffer per (device, stream): used when a caller passes
// scratch == NULL.  Grown with cudaMalloc on demand; an outgrown buffer is kept (not freed)
// until process exit, since another host thread may still hold it.  Calls on one stream are
// ordered by the stream; calls that pass NULL scratch on the same stream from several host
// threads at once share the buffer and race.
int library_scratch(size_t bytes, void* stream, void** out);

// Runs body(begin, end) over [0, n) split into chunks of at least `grain` items on the
// library's host worker threads (a process-wide pool) and the calling thread; returns when
// every chunk is done.  Small ranges run inline.
void parallel_for(int n, int grain, const std::function<void(int, int)>& body);

// dgpu_code_residue_batch, also giving the largest band maximum M of the call (max_coeff, may
// be NULL; INT_MAX when the call failed before reading the band maxima).  In a component
// without intra prediction M is its largest |coefficient|, and every quantised index is at
// most M; an intra component's DC band enters with the maximum of its DPCM differences, so M
// bounds none of its DC prediction residues.
int code_residue_batch(int n, const int* intra, const int* depth, int32_t* const* coeff, const int* cw, const int* ch,
                       const float* lambda, const float* band_wt, const float* band_ecf, const int* band_ncb,
                       int* band_qidx, int* band_skip, int* band_bits, uint8_t* cb_skip, int32_t* const* qout,
                       void* workspace, size_t ws_bytes, void* stream, int* max_coeff);

// Waits for the work queued on st so far (cudaStreamSynchronize; with blocking waits switched
// on, the thread sleeps on a blocking-sync event instead of polling).
cudaError_t host_wait(cudaStream_t st);

__host__ __device__ inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace dgpu
