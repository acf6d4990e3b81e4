// Half-pel upconversion and 2x decimation (the motion-estimation pyramid) for sm_100a.
//
// Upconversion replaces UpConverter::DoUpConverter (libdirac_common/upconvert.cpp:55-200):
// even output rows/columns copy the source, odd ones come from the 8-tap filter
// (21, -7, 3, -1) with +16 >> 5, accumulated in an int16 as the reference does, then clipped
// to the sample range; rows first, then columns.  Decimation replaces
// DownConverter::DoDownConvert (libdirac_motionest/downconvert.cpp:51-204): a 12-tap
// separable filter (86, 46, 4, -8, -4, 4) with +128 >> 8, vertical into an int16 row buffer,
// then horizontal.  Both reference loops clamp source indices at the picture edges (their
// three-loop edge handling is a clamp for the sizes they accept), which the kernels apply
// per sample.
//
// Layout: one CTA per 64 x 16 tile of source samples.  The upconverter stages the source
// tile plus a 4-sample halo in shared memory, computes the vertical half-pel rows there,
// then writes each source sample's 2 x 2 output quad; every output row segment is a
// contiguous 256-byte run.  The decimator stages its vertically filtered row buffer in
// shared memory and writes one output sample per thread.

#include <algorithm>
#include <cmath>

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int UTX = 64, UTY = 16, UH = 4;  // upconvert tile and halo
constexpr int UP_THREADS = 256;

struct UpJob {
    const int16_t* src;
    int16_t* dst;
    int w, h, src_stride, dst_stride;
    int lo, hi;  // clip range
    int tiles_x, tile_begin;
};
constexpr int MAX_UP_JOBS = 32;
struct UpJobs {
    int njobs;
    UpJob job[MAX_UP_JOBS];
};

__device__ __forceinline__ int16_t up_tap_sum(int a0, int b0, int a1, int b1, int a2, int b2, int a3, int b3) {
    // int16 accumulator, truncated after every addition (upconvert.cpp:90-96)
    int16_t s = 16;
    s = (int16_t)(s + (a0 + b0) * 21);
    s = (int16_t)(s + (a1 + b1) * -7);
    s = (int16_t)(s + (a2 + b2) * 3);
    s = (int16_t)(s + (a3 + b3) * -1);
    return (int16_t)(s >> 5);
}

__global__ void __launch_bounds__(UP_THREADS) upconvert_kernel(const __grid_constant__ UpJobs jobs) {
    constexpr int SWU = UTX + 2 * UH;  // staged width (72)
    __shared__ int16_t src[UTY + 2 * UH][SWU];  // source tile + halo (clamped)
    __shared__ int16_t vh[UTY][SWU];             // vertical half-pel rows

    int j = 0;
    while (j + 1 < jobs.njobs && jobs.job[j + 1].tile_begin <= (int)blockIdx.x) ++j;
    const UpJob& jb = jobs.job[j];
    const int t = blockIdx.x - jb.tile_begin;
    const int ty = t / jb.tiles_x, tx = t - ty * jb.tiles_x;
    const int x0 = tx * UTX, y0 = ty * UTY;

    // The staged tile holds the source at clamped coordinates, so the taps below index it
    // directly: a tap row / column clamped to the picture is the staged one (halo >= 4).
    for (int idx = threadIdx.x; idx < (UTY + 2 * UH) * SWU; idx += UP_THREADS) {
        const int r = idx / SWU, c = idx - r * SWU;
        const int gy = clampi(y0 - UH + r, 0, jb.h - 1);
        const int gx = clampi(x0 - UH + c, 0, jb.w - 1);
        src[r][c] = jb.src[(size_t)gy * jb.src_stride + gx];
    }
    __syncthreads();
    // vertical half-pel sample between source rows y and y+1 (rows y-3 .. y+4), every column
    for (int idx = threadIdx.x; idx < UTY * SWU; idx += UP_THREADS) {
        const int r = idx / SWU, c = idx - r * SWU;
        const int16_t s = up_tap_sum(src[r + UH][c], src[r + UH + 1][c], src[r + UH - 1][c], src[r + UH + 2][c],
                                     src[r + UH - 2][c], src[r + UH + 3][c], src[r + UH - 3][c], src[r + UH + 4][c]);
        vh[r][c] = (int16_t)clampi(s, jb.lo, jb.hi);
    }
    __syncthreads();
    // 2 x 2 output quads: a thread takes four consecutive source columns of one row and slides
    // the 8-tap windows of the source row and the vertical half-pel row along them
    constexpr int NQ = 4;
    const int r = threadIdx.x / (UTX / NQ), c0 = (threadIdx.x - r * (UTX / NQ)) * NQ;
    const int gy = y0 + r, gx0 = x0 + c0;
    if (gy >= jb.h || gx0 >= jb.w) return;
    int a[NQ + 7], b[NQ + 7];  // staged columns c0 + UH - 3 .. c0 + UH + NQ + 3
#pragma unroll
    for (int k = 0; k < NQ + 7; ++k) {
        a[k] = src[r + UH][c0 + UH - 3 + k];
        b[k] = vh[r][c0 + UH - 3 + k];
    }
    int16_t e[2 * NQ], o[2 * NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        // source column c0 + q sits at window index q + 3
        const int m = q + 3;
        e[2 * q] = (int16_t)a[m];
        o[2 * q] = (int16_t)b[m];
        e[2 * q + 1] = (int16_t)clampi(up_tap_sum(a[m], a[m + 1], a[m - 1], a[m + 2], a[m - 2], a[m + 3], a[m - 3],
                                                  a[m + 4]), jb.lo, jb.hi);
        o[2 * q + 1] = (int16_t)clampi(up_tap_sum(b[m], b[m + 1], b[m - 1], b[m + 2], b[m - 2], b[m + 3], b[m - 3],
                                                  b[m + 4]), jb.lo, jb.hi);
    }
    int16_t* d0 = jb.dst + (size_t)(2 * gy) * jb.dst_stride + 2 * gx0;
    int16_t* d1 = d0 + jb.dst_stride;
    const int nq = min(NQ, jb.w - gx0);
    if (nq == NQ && ((reinterpret_cast<uintptr_t>(d0) | reinterpret_cast<uintptr_t>(d1)) & 15) == 0) {
        int4 ve, vo;
        ve.x = (int)(uint16_t)e[0] | ((int)(uint16_t)e[1] << 16);
        ve.y = (int)(uint16_t)e[2] | ((int)(uint16_t)e[3] << 16);
        ve.z = (int)(uint16_t)e[4] | ((int)(uint16_t)e[5] << 16);
        ve.w = (int)(uint16_t)e[6] | ((int)(uint16_t)e[7] << 16);
        vo.x = (int)(uint16_t)o[0] | ((int)(uint16_t)o[1] << 16);
        vo.y = (int)(uint16_t)o[2] | ((int)(uint16_t)o[3] << 16);
        vo.z = (int)(uint16_t)o[4] | ((int)(uint16_t)o[5] << 16);
        vo.w = (int)(uint16_t)o[6] | ((int)(uint16_t)o[7] << 16);
        *reinterpret_cast<int4*>(d0) = ve;
        *reinterpret_cast<int4*>(d1) = vo;
    } else {
        // 4-byte aligned pair stores (dst_stride and the base are even-aligned)
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            if (q < nq) {
                *reinterpret_cast<short2*>(d0 + 2 * q) = make_short2(e[2 * q], e[2 * q + 1]);
                *reinterpret_cast<short2*>(d1 + 2 * q) = make_short2(o[2 * q], o[2 * q + 1]);
            }
        }
    }
}

// ---- decimation ---------------------------------------------------------------------------

constexpr int DTX = 32, DTY = 8;  // output tile
constexpr int DN_THREADS = 256;
constexpr int DBUF_W = 2 * DTX + 12;

struct DownJob {
    const int16_t* src;
    int16_t* dst;
    int ow, oh, src_stride, dst_stride;  // output size; source region is 2*ow x 2*oh
    int tiles_x, tile_begin;
};
constexpr int MAX_DOWN_JOBS = 32;
struct DownJobs {
    int njobs;
    DownJob job[MAX_DOWN_JOBS];
};

__constant__ int c_down_taps[6] = {86, 46, 4, -8, -4, 4};

__global__ void __launch_bounds__(DN_THREADS) downconvert_kernel(const __grid_constant__ DownJobs jobs) {
    __shared__ int16_t rowbuf[DTY][DBUF_W];
    int j = 0;
    while (j + 1 < jobs.njobs && jobs.job[j + 1].tile_begin <= (int)blockIdx.x) ++j;
    const DownJob& jb = jobs.job[j];
    const int t = blockIdx.x - jb.tile_begin;
    const int ty = t / jb.tiles_x, tx = t - ty * jb.tiles_x;
    const int ox0 = tx * DTX, oy0 = ty * DTY;
    const int xlen = 2 * jb.ow, ylen = 2 * jb.oh;
    const int bx0 = 2 * ox0 - 5;  // source column of rowbuf[.][0]
    for (int idx = threadIdx.x; idx < DTY * DBUF_W; idx += DN_THREADS) {
        const int r = idx / DBUF_W, c = idx - r * DBUF_W;
        const int oy = oy0 + r;
        if (oy >= jb.oh) continue;
        const int x = clampi(bx0 + c, 0, xlen - 1);
        const int y = 2 * oy;
        int sum = 128;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int ya = clampi(y - k, 0, ylen - 1), yb = clampi(y + 1 + k, 0, ylen - 1);
            sum += (jb.src[(size_t)ya * jb.src_stride + x] + jb.src[(size_t)yb * jb.src_stride + x]) * c_down_taps[k];
        }
        rowbuf[r][c] = (int16_t)(sum >> 8);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < DTY * DTX; idx += DN_THREADS) {
        const int r = idx / DTX, c = idx - r * DTX;
        const int oy = oy0 + r, ox = ox0 + c;
        if (oy >= jb.oh || ox >= jb.ow) continue;
        const int x = 2 * ox;
        int sum = 128;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int xa = clampi(x - k, 0, xlen - 1) - bx0, xb = clampi(x + 1 + k, 0, xlen - 1) - bx0;
            sum += (rowbuf[r][xa] + rowbuf[r][xb]) * c_down_taps[k];
        }
        jb.dst[(size_t)oy * jb.dst_stride + ox] = (int16_t)(sum >> 8);
    }
}

// ---- clip ---------------------------------------------------------------------------------

// Centre-weighted median prefilter (CWMFilterComponent, libdirac_encoder/prefilter.cpp:50-82,
// Median :84-125): each sample with rows 1 .. h-2 and columns 1 .. w-3 (the reference's loop
// stops two columns short of the right edge) becomes the median of its 3 x 3 neighbourhood
// with the centre counted `weight` times (weight = max(1, 10 - strength)); an even count
// takes the rounded mean of the two middle values.  Other samples are copied.  The k-th
// smallest of that multiset follows from the eight sorted neighbours and how many of them
// are below the centre.
__global__ void cwm_kernel(const int16_t* __restrict__ in, int in_stride, int16_t* __restrict__ out,
                           int out_stride, int w, int h, int weight) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const int16_t* r = in + (size_t)y * in_stride;
    const int c = r[x];
    int v = c;
    if (y >= 1 && y <= h - 2 && x >= 1 && x <= w - 3) {
        int n[8];
        int k = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if (dy || dx) n[k++] = in[(size_t)(y + dy) * in_stride + x + dx];
        for (int i = 1; i < 8; ++i) {  // insertion sort of the eight neighbours
            const int t = n[i];
            int j = i - 1;
            while (j >= 0 && n[j] > t) {
                n[j + 1] = n[j];
                --j;
            }
            n[j + 1] = t;
        }
        int below = 0;
        for (int i = 0; i < 8; ++i) below += n[i] < c;
        const int len = weight + 8;
        auto kth = [&](int q) { return q < below ? n[q] : (q < below + weight ? c : n[q - weight]); };
        v = (len & 1) ? kth((len - 1) / 2) : (kth(len / 2 - 1) + kth(len / 2) + 1) >> 1;
    }
    out[(size_t)y * out_stride + x] = (int16_t)v;
}

// RECTLP residue prefilter (LPFilter / HFilter / VFilter, libdirac_encoder/prefilter.cpp:
// 141-306): a 17-tap integer low-pass filter (taps summing to about 2^14) applied along rows,
// then along columns, each output (sum + 2^13) >> 14 clamped to [-128, 127] (the reference's
// bounds, whatever the bit depth), source indices clamped to the component.
struct LpTaps {
    int t[17];  // t[k + 8] multiplies the sample at offset -k
};

__global__ void lp_rows_kernel(const int16_t* __restrict__ in, int in_stride, int16_t* __restrict__ out,
                               int out_stride, int w, int h, const __grid_constant__ LpTaps T) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const int16_t* r = in + (size_t)y * in_stride;
    int sum = 1 << 13;
    for (int k = -8; k <= 8; ++k) sum += T.t[k + 8] * r[clampi(x - k, 0, w - 1)];
    out[(size_t)y * out_stride + x] = (int16_t)clampi(sum >> 14, -128, 127);
}

__global__ void lp_cols_kernel(const int16_t* __restrict__ in, int in_stride, int16_t* __restrict__ out,
                               int out_stride, int w, int h, const __grid_constant__ LpTaps T) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= w || y >= h) return;
    int sum = 1 << 13;
    for (int k = -8; k <= 8; ++k) sum += T.t[k + 8] * in[(size_t)clampi(y - k, 0, h - 1) * in_stride + x];
    out[(size_t)y * out_stride + x] = (int16_t)clampi(sum >> 14, -128, 127);
}

__global__ void clip_kernel(int16_t* p, int w, int h, int stride, int lo, int hi) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x < w && y < h) {
        int16_t* q = p + (size_t)y * stride + x;
        *q = (int16_t)clampi(*q, lo, hi);
    }
}

}  // namespace

int launch_upconvert(int n, const int16_t* const* src, const int* w, const int* h, const int* src_stride,
                     const int* bit_depth, int16_t* const* dst, const int* dst_stride, cudaStream_t st) {
    UpJobs jobs;
    jobs.njobs = 0;
    int tiles = 0;
    for (int i = 0; i < n; ++i) {
        if (!src[i] || !dst[i] || w[i] < 8 || h[i] < 8 || src_stride[i] < w[i] || dst_stride[i] < 2 * w[i] ||
            (dst_stride[i] & 1) || (reinterpret_cast<uintptr_t>(dst[i]) & 3) || bit_depth[i] < 2 || bit_depth[i] > 15)
            return DGPU_ERR_ARG;
        UpJob& jb = jobs.job[jobs.njobs++];
        jb.src = src[i];
        jb.dst = dst[i];
        jb.w = w[i];
        jb.h = h[i];
        jb.src_stride = src_stride[i];
        jb.dst_stride = dst_stride[i];
        jb.lo = -(1 << (bit_depth[i] - 1));
        jb.hi = (1 << (bit_depth[i] - 1)) - 1;
        jb.tiles_x = (w[i] + UTX - 1) / UTX;
        jb.tile_begin = tiles;
        tiles += jb.tiles_x * ((h[i] + UTY - 1) / UTY);
        if (jobs.njobs == MAX_UP_JOBS || i == n - 1) {
            upconvert_kernel<<<tiles, UP_THREADS, 0, st>>>(jobs);
            DGPU_CHECK_LAUNCH();
            jobs.njobs = 0;
            tiles = 0;
        }
    }
    return DGPU_OK;
}

int launch_downconvert(int n, const int16_t* const* src, const int* w, const int* h, const int* src_stride,
                       int16_t* const* dst, const int* dst_stride, cudaStream_t st) {
    DownJobs jobs;
    jobs.njobs = 0;
    int tiles = 0;
    for (int i = 0; i < n; ++i) {
        const int ow = w[i] / 2, oh = h[i] / 2;
        if (!src[i] || !dst[i] || ow < 12 || oh < 12 || src_stride[i] < w[i] || dst_stride[i] < ow)
            return DGPU_ERR_ARG;
        DownJob& jb = jobs.job[jobs.njobs++];
        jb.src = src[i];
        jb.dst = dst[i];
        jb.ow = ow;
        jb.oh = oh;
        jb.src_stride = src_stride[i];
        jb.dst_stride = dst_stride[i];
        jb.tiles_x = (ow + DTX - 1) / DTX;
        jb.tile_begin = tiles;
        tiles += jb.tiles_x * ((oh + DTY - 1) / DTY);
        if (jobs.njobs == MAX_DOWN_JOBS || i == n - 1) {
            downconvert_kernel<<<tiles, DN_THREADS, 0, st>>>(jobs);
            DGPU_CHECK_LAUNCH();
            jobs.njobs = 0;
            tiles = 0;
        }
    }
    return DGPU_OK;
}

int launch_clip(int16_t* p, int w, int h, int stride, int bit_depth, cudaStream_t st) {
    if (!p || w <= 0 || h <= 0 || stride < w || bit_depth < 2 || bit_depth > 15) return DGPU_ERR_ARG;
    dim3 grid((w + 255) / 256, h);
    clip_kernel<<<grid, 256, 0, st>>>(p, w, h, stride, -(1 << (bit_depth - 1)), (1 << (bit_depth - 1)) - 1);
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}

}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_upconvert(const int16_t* pic, int w, int h, int stride, int bit_depth, int16_t* up,
                              int up_stride, void* stream) {
    return launch_upconvert(1, &pic, &w, &h, &stride, &bit_depth, &up, &up_stride, as_stream(stream));
}

extern "C" int dgpu_upconvert_batch(int n, const int16_t* const* pic, const int* w, const int* h,
                                    const int* stride, const int* bit_depth, int16_t* const* up,
                                    const int* up_stride, void* stream) {
    if (n <= 0 || !pic || !w || !h || !stride || !bit_depth || !up || !up_stride) return DGPU_ERR_ARG;
    return launch_upconvert(n, pic, w, h, stride, bit_depth, up, up_stride, as_stream(stream));
}

extern "C" int dgpu_downconvert(const int16_t* pic, int w, int h, int stride, int16_t* out, int out_stride,
                                void* stream) {
    return launch_downconvert(1, &pic, &w, &h, &stride, &out, &out_stride, as_stream(stream));
}

extern "C" int dgpu_downconvert_batch(int n, const int16_t* const* pic, const int* w, const int* h,
                                      const int* stride, int16_t* const* out, const int* out_stride,
                                      void* stream) {
    if (n <= 0 || !pic || !w || !h || !stride || !out || !out_stride) return DGPU_ERR_ARG;
    return launch_downconvert(n, pic, w, h, stride, out, out_stride, as_stream(stream));
}

extern "C" int dgpu_clip(int16_t* pic, int w, int h, int stride, int bit_depth, void* stream) {
    return launch_clip(pic, w, h, stride, bit_depth, as_stream(stream));
}

// MakeLPRectFilter (prefilter.cpp:141-181) for LPFilter's bandwidth (:183-193): a Hanning-
// windowed sinc of 17 taps in double, scaled to a DC gain of 2^18, rounded half away from zero
// and brought to 2^14 by (t + 8) >> 4.
static void rect_lp_taps(float qf, int strength, LpTaps& T) {
    const float bw = std::min(std::max(qf + 3.0f - float(strength), 1.0f), 10.0f) / 10.0f;
    const float pi = 3.1415926535f;
    double d[17];
    for (int i = -8; i <= 8; ++i) d[i + 8] = std::cos(double((pi * i) / 18));  // float argument, double cosine
    for (int i = -8; i <= 8; ++i) {
        const double v = pi * 1.0 * bw * i;
        d[i + 8] *= v == 0.0 ? 1.0 : std::sin(v) / v;
    }
    double sum = 0.0;
    for (int i = 0; i < 17; ++i) sum += d[i];
    for (int i = 0; i < 17; ++i) {
        d[i] *= double(1 << 18);
        d[i] /= sum;
        const int r = d[i] > 0 ? int(d[i] + 0.5) : -int(-d[i] + 0.5);
        T.t[i] = (r + 8) >> 4;
    }
}

extern "C" int dgpu_rect_lp_filter(int16_t* pic, int w, int h, int stride, float qf, int strength, int16_t* scratch,
                                   void* stream) {
    if (!pic || stride < w) return DGPU_ERR_ARG;
    if (w < 17 || h < 17) return DGPU_ERR_SIZE;  // the reference's edge loops assume 17 samples
    int16_t* tmp = scratch;
    if (!tmp) {
        void* p = nullptr;
        const int rc = library_scratch((size_t)w * h * sizeof(int16_t), stream, &p);
        if (rc) return rc;
        tmp = static_cast<int16_t*>(p);
    }
    LpTaps T;
    rect_lp_taps(qf, strength, T);
    cudaStream_t st = as_stream(stream);
    dim3 grid((w + 255) / 256, h);
    lp_rows_kernel<<<grid, 256, 0, st>>>(pic, stride, tmp, w, w, h, T);
    DGPU_CHECK_LAUNCH();
    lp_cols_kernel<<<grid, 256, 0, st>>>(tmp, w, pic, stride, w, h, T);
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}

namespace dgpu {
namespace {

// DIAGLP residue prefilter (DiagFilter, libdirac_encoder/prefilter.cpp:535-588, with
// DiagFilterBchkD / DiagFilterD :307-398): a 13 x 13 two-dimensional low-pass filter given by
// one quadrant of taps f[j][i] (offsets 0..6 down and across; the other quadrants mirror it),
// each output (2^15 + sum) >> 16 cast to int16, source indices clamped to the component (the
// reference's unclamped interior loop reads the same samples).  The quadrants are the
// reference's hand-designed tables for bandwidths 0.2 .. 0.9 (GetDiagLPFilter, :401-531), mixed
// with a unit impulse by the strength and quality factor; they decide the filtered samples.
struct DiagTaps {
    int f[7][7];
};

const int kDiagLPTables[8][7][7] = {
    {  // bandwidth 0.2
        {  2855,   2540,   1775,    947,    364,     89,     10},
        {  2540,   2251,   1551,    804,    290,     59,      1},
        {  1775,   1551,   1020,    475,    130,      3,    -10},
        {   947,    804,    475,    165,      5,    -22,     -6},
        {   364,    290,    130,      5,    -28,    -10,      0},
        {    89,     59,      3,    -22,    -10,      0,      0},
        {    10,      1,    -10,     -6,      0,      0,      0},
    },
    {  // bandwidth 0.3
        {  5767,   4718,   2498,    745,     72,      5,     23},
        {  4718,   3796,   1875,    423,    -58,    -41,      7},
        {  2498,   1875,    643,   -146,   -241,    -88,     -9},
        {   745,    423,   -146,   -367,   -220,    -51,     -2},
        {    72,    -58,   -241,   -220,    -78,     -5,      0},
        {     5,    -41,    -88,    -51,     -5,      0,      0},
        {    23,      7,     -9,     -2,      0,      0,      0},
    },
    {  // bandwidth 0.4
        { 10534,   7642,   2603,    194,     56,    120,     28},
        {  7642,   5237,   1218,   -383,   -153,     40,      2},
        {  2603,   1218,   -771,   -958,   -269,     -3,     -7},
        {   194,   -383,   -958,   -541,    -18,     48,      4},
        {    56,   -153,   -269,    -18,     96,     22,      0},
        {   120,     40,     -3,     48,     22,      0,      0},
        {    28,      2,     -7,      4,      0,      0,      0},
    },
    {  // bandwidth 0.5
        { 16421,  10159,   1716,     33,    325,     57,      6},
        { 10159,   5309,   -580,   -747,     44,    -43,    -25},
        {  1716,   -580,  -2310,   -763,    100,    -19,    -12},
        {    33,   -747,   -763,    308,    326,     27,      1},
        {   325,     44,    100,    326,     84,    -14,      0},
        {    57,    -43,    -19,     27,    -14,      0,      0},
        {     6,    -25,    -12,      1,      0,      0,      0},
    },
    {  // bandwidth 0.6
        { 23511,  11883,    566,    524,    231,     18,     41},
        { 11883,   3647,  -2496,   -361,    -96,    -97,      1},
        {   566,  -2496,  -2329,    459,    152,     -7,     18},
        {   524,   -361,    459,    979,     33,    -28,      3},
        {   231,    -96,    152,     33,   -184,    -15,      0},
        {    18,    -97,     -7,    -28,    -15,      0,      0},
        {    41,      1,     18,      3,      0,      0,      0},
    },
    {  // bandwidth 0.7
        { 32188,  12652,      3,    921,      1,    128,      0},
        { 12652,    295,  -3414,     -2,   -343,     -1,    -37},
        {     3,  -3414,   -212,   1273,      1,     98,      0},
        {   921,     -2,   1273,    110,   -363,      0,     -8},
        {     1,   -343,      1,   -363,    -29,     29,      0},
        {   128,     -1,     98,      0,     29,      0,      0},
        {     0,    -37,      0,     -8,      0,      0,      0},
    },
    {  // bandwidth 0.8
        { 41902,  12084,    435,    610,    188,     34,     37},
        { 12084,  -4268,  -2715,   -286,   -144,    -84,     -2},
        {   435,  -2715,   2809,    640,    127,     10,     17},
        {   610,   -286,    640,  -1250,    -45,    -26,      2},
        {   188,   -144,    127,    -45,    259,     -8,      0},
        {    34,    -84,     10,    -26,     -8,      0,      0},
        {    37,     -2,     17,      2,      0,      0,      0},
    },
    {  // bandwidth 0.9
        { 53098,  10449,   1546,     73,    342,     38,     12},
        { 10449,  -9060,   -873,   -727,     52,    -65,    -20},
        {  1546,   -873,   4261,   -627,    137,    -27,     -7},
        {    73,   -727,   -627,   -804,    328,     14,      2},
        {   342,     52,    137,    328,    -83,    -20,      0},
        {    38,    -65,    -27,     14,    -20,      0,      0},
        {    12,    -20,     -7,      2,      0,      0,      0},
    },
};

constexpr int DIAG_TX = 32, DIAG_TY = 8, DIAG_R = 6;

__global__ void __launch_bounds__(DIAG_TX* DIAG_TY) diag_lp_kernel(const int16_t* __restrict__ in, int in_stride,
                                                                   int16_t* __restrict__ out, int out_stride, int w,
                                                                   int h, const __grid_constant__ DiagTaps T) {
    __shared__ int16_t tile[DIAG_TY + 2 * DIAG_R][DIAG_TX + 2 * DIAG_R];
    const int x0 = blockIdx.x * DIAG_TX, y0 = blockIdx.y * DIAG_TY;
    const int tid = threadIdx.y * DIAG_TX + threadIdx.x;
    // the tile and its halo, coordinates clamped to the component
    for (int k = tid; k < (DIAG_TY + 2 * DIAG_R) * (DIAG_TX + 2 * DIAG_R); k += DIAG_TX * DIAG_TY) {
        const int ty = k / (DIAG_TX + 2 * DIAG_R), tx = k - ty * (DIAG_TX + 2 * DIAG_R);
        const int sy = clampi(y0 + ty - DIAG_R, 0, h - 1), sx = clampi(x0 + tx - DIAG_R, 0, w - 1);
        tile[ty][tx] = in[(size_t)sy * in_stride + sx];
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= h) return;
    const int cx = threadIdx.x + DIAG_R, cy = threadIdx.y + DIAG_R;
    int val = 1 << 15;
    val += T.f[0][0] * tile[cy][cx];
#pragma unroll
    for (int i = 1; i <= DIAG_R; ++i) val += T.f[0][i] * (tile[cy][cx + i] + tile[cy][cx - i]);
#pragma unroll
    for (int j = 1; j <= DIAG_R; ++j) {
        val += T.f[j][0] * (tile[cy - j][cx] + tile[cy + j][cx]);
#pragma unroll
        for (int i = 1; i <= DIAG_R; ++i)
            val += T.f[j][i] * (tile[cy - j][cx + i] + tile[cy - j][cx - i] + tile[cy + j][cx + i] + tile[cy + j][cx - i]);
    }
    out[(size_t)y * out_stride + x] = (int16_t)(val >> 16);
}

// DiagFilter's taps for a quality factor and strength (prefilter.cpp:535-556, in the
// reference's float / double arithmetic); false when its bandwidth is above 0.9 and the
// reference leaves the component unchanged.
bool diag_lp_taps(float qf, int strength, DiagTaps& T) {
    const float ffactor = (8.0 + strength - 4.0 - qf) / 5.0;
    const int factor = std::max(0, std::min(256, int(ffactor * 256.0)));
    const float bw = (1.0 - ffactor) * 0.6 + 0.4;
    if (bw > 0.9) return false;
    const int qbf = std::min(std::max(int(bw * 10.0 + 0.5), 2), 10);
    for (int j = 0; j < 7; ++j)
        for (int i = 0; i < 7; ++i)
            T.f[j][i] = qbf == 10 ? (i == 0 && j == 0 ? 65536 : 0) : kDiagLPTables[qbf - 2][j][i];
    T.f[0][0] = (factor * T.f[0][0] + ((1 << 8) - factor) * (1 << 16) + (1 << 7)) >> 8;
    for (int i = 1; i < 7; ++i) T.f[0][i] = (factor * T.f[0][i] + (1 << 7)) >> 8;
    for (int j = 1; j < 7; ++j)
        for (int i = 0; i < 7; ++i) T.f[j][i] = (factor * T.f[j][i] + (1 << 7)) >> 8;
    return true;
}

}  // namespace
}  // namespace dgpu

extern "C" int dgpu_diag_lp_filter(int16_t* pic, int w, int h, int stride, float qf, int strength,
                                   int16_t* scratch, void* stream) {
    if (!pic || stride < w) return DGPU_ERR_ARG;
    if (w < 7 || h < 7) return DGPU_ERR_SIZE;  // the reference's edge loops assume 7 samples
    DiagTaps T;
    if (!diag_lp_taps(qf, strength, T)) return DGPU_OK;
    int16_t* tmp = scratch;
    if (!tmp) {
        void* p = nullptr;
        const int rc = library_scratch((size_t)w * h * sizeof(int16_t), stream, &p);
        if (rc) return rc;
        tmp = static_cast<int16_t*>(p);
    }
    cudaStream_t st = as_stream(stream);
    // the reference filters from the unfiltered component into a copy
    DGPU_CHECK_CUDA(cudaMemcpy2DAsync(tmp, (size_t)w * sizeof(int16_t), pic, (size_t)stride * sizeof(int16_t),
                                      (size_t)w * sizeof(int16_t), h, cudaMemcpyDeviceToDevice, st));
    dim3 grid((w + DIAG_TX - 1) / DIAG_TX, (h + DIAG_TY - 1) / DIAG_TY);
    diag_lp_kernel<<<grid, dim3(DIAG_TX, DIAG_TY), 0, st>>>(tmp, w, pic, stride, w, h, T);
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}

extern "C" int dgpu_cwm_filter(const int16_t* in, int in_stride, int16_t* out, int out_stride, int w, int h,
                               int strength, void* stream) {
    if (!in || !out || in == out || w < 1 || h < 1 || in_stride < w || out_stride < w) return DGPU_ERR_ARG;
    const int weight = strength >= 9 ? 1 : 10 - strength;
    dim3 grid((w + 255) / 256, h);
    cwm_kernel<<<grid, 256, 0, as_stream(stream)>>>(in, in_stride, out, out_stride, w, h, weight);
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}
