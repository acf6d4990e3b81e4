// Quantiser selection statistics and quantisation with reconstruction, for sm_100a.
//
// Replaces the data-parallel part of PictureCompressor::SelectQuantisers / QuantChooser
// (libdirac_encoder/picture_compress.cpp:603-709, quant_chooser.cpp:62-362) and the
// quantise-and-reconstruct arithmetic of the band coders (GenericBandCodec::CodeVal /
// CodeCoeffBlock / ClearBlock, band_codec_template.h:53-174, 470-557; IntraDCBandCodec,
// band_codec.cpp:81-96; CompCompressor::Compress, comp_compress.cpp:64-156).
//
// Flow for a batch of components:
//   1. (intra) the DC band's raster DPCM against the previous int16 value
//      (AddSubAverage) into a work copy; band and code-block absolute maxima.
//   2. statistics per band, per candidate quantiser q and per sampling pattern (every 2nd
//      column and row for the integral and half-step passes, every 2nd row for the
//      quarter-step pass): count0 = sum of quantised magnitudes, positive / negative counts
//      and the 4th-power error sum, the last as an exact 128-bit integer.  A sum that the
//      reference's sequential double accumulation could round (a term of 9741 or more, or a
//      total of 2^53 or more) is flagged.
//   3. host: the reference's three-pass Lagrangian search in double precision with the host
//      libm (exactly the reference's arithmetic); flagged sums are recomputed first by a
//      sequential double kernel in the reference's order.
//   4. quantise and reconstruct in place; the intra DC band (prediction from reconstructed
//      neighbours) as an anti-diagonal wavefront in one CTA.

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include <atomic>
#include <mutex>

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int QMAX = 101;          // candidate quantisers per band with statistics (covers |c| < 2^24)
constexpr int MAX_BANDS = 3 * 8 + 1;
constexpr uint64_t EXACT_TERM = 9741;  // pow4 of smaller values is exact in double
constexpr int STAT_THREADS = 256;

// QuantiserLists (libdirac_common/common.cpp:931-981)
__host__ __device__ inline int qf4(int q) {
    if (q == 0) return 4;
    if (q == 1) return 5;
    const unsigned long long base = 1ull << (q / 4);
    unsigned long long f;
    switch (q % 4) {
        case 0: f = 4 * base; break;
        case 1: f = (503829 * base + 52958) / 105917; break;
        case 2: f = (665857 * base + 58854) / 117708; break;
        default: f = (440253 * base + 32722) / 65444; break;
    }
    return (int)f;
}
__host__ __device__ inline int intra_off4(int q) { return q == 0 ? 1 : (q == 1 ? 2 : (qf4(q) + 1) >> 1); }
__host__ __device__ inline int inter_off4(int q) { return q == 0 ? 1 : (q == 1 ? 2 : (3 * qf4(q) + 4) >> 3); }

// SubbandList::Init (wavelet_utils.cpp:144-190): band b (1-based) of a cw x ch array.
__host__ __device__ inline void band_rect(int depth, int cw, int ch, int b, int& xp, int& yp, int& xl, int& yl) {
    if (b == 3 * depth + 1) {
        xp = 0;
        yp = 0;
        xl = cw >> depth;
        yl = ch >> depth;
        return;
    }
    const int level = (b - 1) / 3 + 1, kind = (b - 1) % 3;
    xl = cw >> level;
    yl = ch >> level;
    xp = (kind == 0 || kind == 2) ? xl : 0;
    yp = (kind == 0 || kind == 1) ? yl : 0;
}

struct Stat {  // statistics of one (band, pattern, q), device accumulators
    unsigned long long count0;
    unsigned long long posneg;   // positive count (low 32 bits) + negative count (high 32)
    unsigned long long err_lo, err_hi;
    unsigned int inexact;
    unsigned int pad;
};

struct Comp {
    const int32_t* coeff;     // transformed component (dense, cw x ch)
    int32_t* dcwork;          // intra: the DC band after DPCM (xl x yl of the DC band)
    int cw, ch, depth, intra;
    int nbands;
    int band_first;           // index of band 1 in the global band tables
};

struct BandTask {  // one band: where its data lives and where its statistics go
    const int32_t* data;      // top-left of the band in its array
    int stride, xl, yl;
    int comp;
    int band;                 // global band index
    int cb_first, xn, yn;     // code blocks of the band
    int chunk_first[2];       // first CTA of the band in each sampling pattern's flattened grid
    int elem_first;           // first CTA of the band in the row-chunked grid (maxima)
    int rows_per_cta;         // rows of the band per CTA of that grid
};

constexpr int MAX_COMPS = 256;
constexpr int MAX_TASKS = MAX_COMPS * MAX_BANDS;


// ---- 1. DC DPCM and maxima ----------------------------------------------------------------

__global__ void dc_dpcm_kernel(const int32_t* c, int stride, int xl, int yl, int32_t* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= xl * yl) return;
    const int j = k / xl, i = k - j * xl;
    const int prev = k == 0 ? 0 : (int)(int16_t)c[(size_t)((k - 1) / xl) * stride + (k - 1) % xl];
    out[k] = c[(size_t)j * stride + i] - prev;
}

// Per band: max |c|.  Per code block: max |c| (for QuantChooser::SetSkip).  Lanes of a warp
// that fall in the same code block combine their maxima before one atomic.
// Code block (0 .. n-1) holding position pos of a band side of length len split into n:
// block c covers [c * len / n, (c + 1) * len / n) (integer division), as the band coders
// split a band.
__device__ __forceinline__ int cb_of(int pos, int len, int n) {
    int c = (pos * n) / len;
    while (c + 1 < n && ((c + 1) * len) / n <= pos) ++c;
    while (c > 0 && (c * len) / n > pos) --c;
    return c;
}

constexpr int MAX_PER_CTA = 256 * 8;  // about the elements per CTA of the row-chunked grids
constexpr int ROW_THREADS = 256;      // eight warps: a warp per row, lanes across the row

// Rows of a band side of length xl per CTA of the row-chunked grids: at least one per warp.
__host__ __device__ inline int rows_per_cta(int xl) { return max(ROW_THREADS / 32, MAX_PER_CTA / max(xl, 1)); }

// A lane's walk along one band row at columns lane, lane + 32, ...: its code block column cx
// (blocks split the row at (c * xl) / xn, integer division) follows with one comparison per
// step instead of a division per element.
struct CbWalk {
    int cx, bnd, xl, xn;
    __device__ __forceinline__ CbWalk(int i0, int xl_, int xn_) : xl(xl_), xn(xn_) {
        cx = cb_of(i0, xl, xn);
        bnd = ((cx + 1) * xl) / xn;
    }
    // moves to column i (non-decreasing); returns whether the block changed
    __device__ __forceinline__ bool to(int i) {
        bool moved = false;
        while (cx + 1 < xn && i >= bnd) {
            ++cx;
            bnd = ((cx + 1) * xl) / xn;
            moved = true;
        }
        return moved;
    }
};

// grid: row chunks of the bands laid end to end (BandTask::elem_first, rows_per_cta).  Each
// warp takes rows; a lane keeps the maximum of its current code block and folds it into the
// CTA's shared copy when it leaves the block; the CTA then folds those into cb_max.
__global__ void __launch_bounds__(ROW_THREADS) band_max_kernel(const BandTask* tasks, int ntasks, int* band_max,
                                                               int* cb_max) {
    __shared__ int s_cb[256];
    int lo_b = 0, hi_b = ntasks - 1;
    while (lo_b < hi_b) {
        const int mid = (lo_b + hi_b + 1) >> 1;
        if (tasks[mid].elem_first <= (int)blockIdx.x) lo_b = mid;
        else hi_b = mid - 1;
    }
    const BandTask T = tasks[lo_b];
    const int r0 = ((int)blockIdx.x - T.elem_first) * T.rows_per_cta;
    const int r1 = min(T.yl, r0 + T.rows_per_cta);
    const int cy0 = cb_of(r0, T.yl, T.yn), cy1 = cb_of(r1 - 1, T.yl, T.yn);
    const int ncell = (cy1 - cy0 + 1) * T.xn;
    const bool local = ncell <= 256;
    for (int k = threadIdx.x; k < ncell && local; k += blockDim.x) s_cb[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int m = 0;
    for (int j = r0 + warp; j < r1; j += ROW_THREADS / 32) {
        const int cy = cb_of(j, T.yl, T.yn);
        const int32_t* row = T.data + (size_t)j * T.stride;
        if (lane >= T.xl) continue;
        CbWalk w(lane, T.xl, T.xn);
        int run = 0;
        for (int i = lane; i < T.xl; i += 32) {
            const int prev = w.cx;
            if (w.to(i)) {
                if (run) {
                    if (local) atomicMax(&s_cb[(cy - cy0) * T.xn + prev], run);
                    else atomicMax(&cb_max[T.cb_first + cy * T.xn + prev], run);
                }
                run = 0;
            }
            const int a = abs(row[i]);
            run = max(run, a);
            m = max(m, a);
        }
        if (run) {
            if (local) atomicMax(&s_cb[(cy - cy0) * T.xn + w.cx], run);
            else atomicMax(&cb_max[T.cb_first + cy * T.xn + w.cx], run);
        }
    }
    m = __reduce_max_sync(0xffffffffu, (unsigned)m);
    if (lane == 0 && m) atomicMax(&band_max[T.band], m);
    __syncthreads();
    for (int k = threadIdx.x; k < ncell && local; k += blockDim.x)
        if (s_cb[k]) atomicMax(&cb_max[T.cb_first + cy0 * T.xn + k], s_cb[k]);
}

// ---- 2. statistics ------------------------------------------------------------------------

// Number of quantisers whose statistics a band needs: 4 * (bit length of max) + 5 covers
// the reference's 4 * floor(log2 max) + 5 whatever its libm rounding.
__device__ __forceinline__ int stat_range(int maxv) {
    if (maxv < 1) return 0;
    const int bitlen = 32 - __clz(maxv);
    return min(4 * bitlen + 5, QMAX);
}

// grid: one CTA per chunk of STAT_THREADS * 8 sampled coefficients, the bands' chunks laid end
// to end (BandTask::chunk_first of the pattern; 0: 2x2, 1: 1x2).
// n / d: for n < 2^24 (every magnitude times 4 of 8- to 14-bit video) the float estimate
// n * RN(1/d) is within one of the quotient (relative error below 2^-23, quotient below
// 2^22), and one integer correction makes it exact.
__device__ __forceinline__ unsigned udiv_recip(unsigned n, unsigned d, float inv) {
    if (n >= (1u << 24)) return n / d;  // outside the estimate's range: plain division
    unsigned q = (unsigned)((float)n * inv);
    if (q * d > n) --q;
    else if ((q + 1) * d <= n) ++q;
    return q;
}

// Statistics of one sampling pattern (0: 2 x 2 for the first two passes, over every even
// quantiser; 1: 1 x 2 for the third pass, over the per-band range qrange[band] = (lo, hi)).
// Layout: stats[(pattern * nbands + band) * QMAX + q].
__global__ void __launch_bounds__(STAT_THREADS) stats_kernel(const BandTask* tasks, const int* band_max,
                                                             Stat* stats, int pattern, int nbands,
                                                             const int2* qrange) {
    // the band whose chunks hold this CTA: the last with chunk_first <= blockIdx.x
    int lo_b = 0, hi_b = nbands - 1;
    while (lo_b < hi_b) {
        const int mid = (lo_b + hi_b + 1) >> 1;
        if (tasks[mid].chunk_first[pattern] <= (int)blockIdx.x) lo_b = mid;
        else hi_b = mid - 1;
    }
    const BandTask T = tasks[lo_b];
    const int xr = pattern ? 1 : 2;
    const int nq = stat_range(band_max[T.band]);
    const int sx = (T.xl + xr - 1) / xr, sy = (T.yl + 1) / 2;
    const int nsamp = sx * sy;
    const int per_cta = STAT_THREADS * 8;
    const int base = ((int)blockIdx.x - T.chunk_first[pattern]) * per_cta;
    if (base >= nsamp || nq == 0) return;
    __shared__ unsigned long long s_c0[QMAX], s_pn[QMAX], s_lo[QMAX], s_hi[QMAX];
    __shared__ unsigned int s_inx[QMAX];
    // Pattern 0 tail: a sample quantises to zero for every quantiser from the first whose factor
    // exceeds 4|v| on, and then adds the same term |v|^4 (count and signs unchanged).  Its term
    // goes once to the bin of that first even quantiser; a running sum over the bins then gives
    // every quantiser its tail.
    __shared__ unsigned long long s_tlo[QMAX], s_thi[QMAX];
    __shared__ unsigned int s_tinx[QMAX];
    __shared__ int s_qf[QMAX];
    for (int q = threadIdx.x; q < QMAX; q += STAT_THREADS) {
        s_c0[q] = s_pn[q] = s_lo[q] = s_hi[q] = 0;
        s_inx[q] = 0;
        s_tlo[q] = s_thi[q] = 0;
        s_tinx[q] = 0;
        s_qf[q] = qf4(q);
    }
    __syncthreads();
    int a[8];
    bool neg[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int k = base + t * STAT_THREADS + threadIdx.x;
        a[t] = -1;
        neg[t] = false;
        if (k < nsamp) {
            const int sj = k / sx, si = k - sj * sx;
            const int v = T.data[(size_t)(2 * sj) * T.stride + xr * si];
            a[t] = abs(v);
            neg[t] = v <= 0;
        }
    }
    const int lane = threadIdx.x & 31;
    const int qlo = qrange ? qrange[T.band].x : 0;
    const int qhi = qrange ? min(qrange[T.band].y, nq - 1) : nq - 1;
    // q0[t]: the first quantiser of the loop whose factor exceeds 4 a (every later one too);
    // from it on the sample is in the tail (pattern 0 only; pattern 1 has no tail)
    int q0[8];
    int qmax_w = qlo;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        q0[t] = qhi + 2;
        if (a[t] < 0 || pattern) continue;
        const unsigned a4 = (unsigned)a[t] << 2;
        int lo_q = 0, hi_q = (qhi >> 1) + 1;  // even quantisers 2 k, k in [lo_q, hi_q)
        while (lo_q < hi_q) {
            const int mid = (lo_q + hi_q) >> 1;
            if ((unsigned)s_qf[2 * mid] > a4) hi_q = mid;
            else lo_q = mid + 1;
        }
        q0[t] = 2 * lo_q;
        qmax_w = max(qmax_w, q0[t]);
    }
    if (!pattern) {
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int key = (a[t] >= 0 && q0[t] <= qhi) ? q0[t] : -1;
            const unsigned grp = __match_any_sync(0xffffffffu, key);
            unsigned long long p = 0;
            unsigned inx = 0;
            if (key >= 0) {
                if ((unsigned)a[t] >= EXACT_TERM) {
                    inx = 1;
                } else {
                    const unsigned e2 = (unsigned)a[t] * (unsigned)a[t];
                    p = (unsigned long long)e2 * e2;
                }
            }
            // group sums in 27-bit pieces, so that 32-bit reductions cannot overflow
            const unsigned plo = (unsigned)(p & ((1ull << 27) - 1)), phi = (unsigned)(p >> 27);
            const unsigned slo = __reduce_add_sync(grp, plo), shi = __reduce_add_sync(grp, phi);
            const unsigned sinx = __reduce_or_sync(grp, inx);
            if (key >= 0 && lane == __ffs(grp) - 1) {
                const unsigned long long v = (unsigned long long)slo + ((unsigned long long)shi << 27);
                const unsigned long long old = atomicAdd(&s_tlo[key], v);
                if (old + v < old) atomicAdd(&s_thi[key], 1ull);
                if (sinx) atomicOr(&s_tinx[key], 1u);
            }
        }
    }
    // quantisers past every sample's first zero need no per-sample work in this warp
    const int qend = pattern ? qhi : min(qhi, (int)__reduce_max_sync(0xffffffffu, (unsigned)qmax_w) - 2);
    for (int q = qlo; q <= qend; q += (pattern ? 1 : 2)) {
        const unsigned qf = (unsigned)qf4(q);
        const float inv = __frcp_rn((float)qf);
        const int off = inter_off4(q);
        unsigned long long c0 = 0, lo = 0, hi = 0;
        unsigned int pos = 0, ng = 0, inx = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            if (a[t] < 0 || q >= q0[t]) continue;  // the tail holds q >= q0
            const unsigned qv = udiv_recip((unsigned)a[t] << 2, qf, inv);
            unsigned long long e;
            if (qv == 0) {
                e = (unsigned long long)a[t];
            } else {
                c0 += qv;
                const int r = (int)((qv * qf + off + 2) >> 2);
                e = (unsigned long long)llabs((long long)a[t] - r);
                if (neg[t]) ++ng; else ++pos;
            }
            if (e >= EXACT_TERM) {
                inx = 1;
            } else {
                const unsigned e2 = (unsigned)e * (unsigned)e;  // e < 9741: e^2 < 2^27
                const unsigned long long p = (unsigned long long)e2 * e2;
                lo += p;
                if (lo < p) ++hi;
            }
        }
        // warp reduction (128-bit sum with carries)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long olo = __shfl_down_sync(0xffffffffu, lo, o);
            const unsigned long long ohi = __shfl_down_sync(0xffffffffu, hi, o);
            const unsigned long long nlo = lo + olo;
            hi += ohi + (nlo < lo ? 1 : 0);
            lo = nlo;
            c0 += __shfl_down_sync(0xffffffffu, c0, o);
        }
        pos = __reduce_add_sync(0xffffffffu, pos);
        ng = __reduce_add_sync(0xffffffffu, ng);
        inx = __reduce_or_sync(0xffffffffu, inx);
        if (lane == 0) {
            atomicAdd(&s_c0[q], c0);
            atomicAdd(&s_pn[q], (unsigned long long)pos | ((unsigned long long)ng << 32));
            const unsigned long long old = atomicAdd(&s_lo[q], lo);
            atomicAdd(&s_hi[q], hi + (old + lo < old ? 1 : 0));
            if (inx) atomicOr(&s_inx[q], 1u);
        }
    }
    __syncthreads();
    if (!pattern && threadIdx.x == 0) {
        // running sum of the tail bins over the even quantisers
        unsigned long long rlo = 0, rhi = 0;
        unsigned rinx = 0;
        for (int q = qlo; q <= qhi; q += 2) {
            const unsigned long long nlo = rlo + s_tlo[q];
            rhi += s_thi[q] + (nlo < rlo ? 1 : 0);
            rlo = nlo;
            rinx |= s_tinx[q];
            const unsigned long long old = s_lo[q];
            s_lo[q] = old + rlo;
            s_hi[q] += rhi + (old + rlo < old ? 1 : 0);
            s_inx[q] |= rinx;
        }
    }
    __syncthreads();
    Stat* S = stats + ((size_t)pattern * nbands + T.band) * QMAX;
    for (int q = threadIdx.x; q < nq; q += STAT_THREADS) {
        if (s_c0[q] == 0 && s_pn[q] == 0 && s_lo[q] == 0 && s_hi[q] == 0 && s_inx[q] == 0) continue;
        atomicAdd(&S[q].count0, s_c0[q]);
        atomicAdd(&S[q].posneg, s_pn[q]);
        const unsigned long long old = atomicAdd(&S[q].err_lo, s_lo[q]);
        atomicAdd(&S[q].err_hi, s_hi[q] + (old + s_lo[q] < old ? 1 : 0));
        if (s_inx[q]) atomicOr(&S[q].inexact, 1u);
    }
}

// Fallback for the sums the exact path cannot represent (a term or the total at or above
// 2^53): the reference's sequential double accumulation of pow4(error) in its raster order
// (quant_chooser.cpp:149-264), written back into the entry (err_lo holds the double's bits,
// pad = 1).  Entries: pattern 0, stats[t * QMAX + q]; pattern 1, the compact third-pass
// array stats[t * 3 + j] for q = qrange[t].x + j.  Each warp scans 32 entries at a time and
// resolves the flagged ones together: the lanes compute the terms of 32 consecutive samples,
// lane 0 adds them one by one in order.
__device__ __forceinline__ bool stat_inexact(const Stat& S) {
    return S.inexact || S.err_hi != 0 || S.err_lo >= (1ull << 53);
}

__global__ void seq_resolve_kernel(const BandTask* tasks, Stat* stats, int n_entries, int pattern,
                                   const int2* qrange) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    const int per = pattern ? 3 : QMAX;
    for (int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n_entries; base += warps * 32) {
        const int e = base + lane;
        bool flag = false;
        if (e < n_entries) {
            const Stat& S = stats[e];
            flag = S.pad == 0 && stat_inexact(S);
            if (flag && pattern) flag = qrange[e / 3].x + e % 3 <= qrange[e / 3].y;
        }
        unsigned m = __ballot_sync(0xffffffffu, flag);
        while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const int ent = base + l;
            const int t = ent / per;
            const int q = pattern ? qrange[t].x + ent % 3 : ent % QMAX;
            const BandTask T = tasks[t];
            const int xr = pattern ? 1 : 2;
            const int sx = (T.xl + xr - 1) / xr, sy = (T.yl + 1) / 2;
            const int n = sx * sy;
            const int qf = qf4(q), off = inter_off4(q);
            double s = 0.0;
            for (int k0 = 0; k0 < n; k0 += 32) {
                double term = 0.0;
                const int i = k0 + lane;
                if (i < n) {
                    const int sj = i / sx, si = i - sj * sx;
                    const int a = abs(T.data[(size_t)(2 * sj) * T.stride + xr * si]);
                    const int qv = (a << 2) / qf;
                    const double ev = !qv ? (double)a : (double)(a - ((qv * qf + off + 2) >> 2));
                    term = __dmul_rn(__dmul_rn(__dmul_rn(ev, ev), ev), ev);
                }
                const int cnt = min(32, n - k0);
                for (int k = 0; k < cnt; ++k) s = __dadd_rn(s, __shfl_sync(0xffffffffu, term, k));
            }
            if (lane == 0) {
                stats[ent].err_lo = (unsigned long long)__double_as_longlong(s);
                stats[ent].err_hi = 0;
                stats[ent].pad = 1;
            }
        }
    }
}

// CTAs of 128 threads (four warps, 32 entries per warp per scan step) for n entries, at most
// four per SM.
inline int resolve_grid(int n) { return std::max(1, std::min(148 * 4, (n + 127) / 128)); }

// Gathers the third pass's statistics, the three quantisers qrange[band] of each band, into
// a compact [band][3] array for the host.
__global__ void gather_stats_kernel(const Stat* stats, const int2* qrange, int nbands, Stat* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nbands) return;
    const int t = i / 3, j = i - 3 * t;
    const int2 r = qrange[t];
    Stat v{};
    if (r.x + j <= r.y) v = stats[(size_t)t * QMAX + r.x + j];
    out[i] = v;
}

// ---- 4. quantise and reconstruct ------------------------------------------------------------

struct QBand {
    int32_t* data;      // band top-left in the coefficient array (reconstructed in place)
    int32_t* qout;      // band top-left in the index array, or null
    int stride;
    int xl, yl, xn, yn;
    int qf, off, skip;
    const uint8_t* cb_skip;  // code blocks of this band
    int first;          // first CTA of the band in the row-chunked grid
    int rows;           // rows per CTA
};


__device__ __forceinline__ int cb_index(int pos, int len, int n) {
    int c = (pos * n) / len;
    while (c + 1 < n && ((c + 1) * len) / n <= pos) ++c;
    while (c > 0 && (c * len) / n > pos) --c;
    return c;
}

// grid: row chunks of the bands (device table) laid end to end; a warp per row, lanes
// across it, the code block followed by CbWalk.  (|v| << 2) / qf through udiv_recip (exact).
__global__ void __launch_bounds__(ROW_THREADS) quantise_kernel(const QBand* bands, int nbands) {
    int lo_b = 0, hi_b = nbands - 1;
    while (lo_b < hi_b) {
        const int mid = (lo_b + hi_b + 1) >> 1;
        if (bands[mid].first <= (int)blockIdx.x) lo_b = mid;
        else hi_b = mid - 1;
    }
    const QBand B = bands[lo_b];
    const int r0 = ((int)blockIdx.x - B.first) * B.rows;
    const int r1 = min(B.yl, r0 + B.rows);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float inv = __frcp_rn((float)B.qf);
    for (int j = r0 + warp; j < r1; j += ROW_THREADS / 32) {
        if (lane >= B.xl) break;
        const uint8_t* skip_row = B.cb_skip + cb_index(j, B.yl, B.yn) * B.xn;
        int32_t* row = B.data + (size_t)j * B.stride;
        int32_t* qrow = B.qout ? B.qout + (size_t)j * B.stride : nullptr;
        CbWalk w(lane, B.xl, B.xn);
        for (int i = lane; i < B.xl; i += 32) {
            w.to(i);
            int r = 0, qi = 0;
            if (!B.skip && !skip_row[w.cx]) {
                const int val = row[i];
                const unsigned qv = udiv_recip((unsigned)abs(val) << 2, (unsigned)B.qf, inv);
                if (qv) {
                    r = (int)((qv * (unsigned)B.qf + B.off + 2) >> 2);
                    if (val <= 0) r = -r;
                }
                qi = val < 0 ? -(int)qv : (int)qv;
            }
            row[i] = r;
            if (qrow) qrow[i] = qi;
        }
    }
}

// Intra DC band: prediction from reconstructed left / top-left / top neighbours
// (GetPrediction, band_codec_template.h:531-557), one anti-diagonal per step.
struct DcJob {
    int32_t* c;
    int32_t* qout;
    const uint8_t* cb_skip;
    int stride, xl, yl, xn, yn, qf, off;
};

// One CTA per intra component's DC band (a device table of jobs).
__global__ void dc_intra_kernel(const DcJob* jobs) {
    const DcJob J = jobs[blockIdx.x];
    int32_t* const c = J.c;
    int32_t* const qout = J.qout;
    const uint8_t* const cb_skip = J.cb_skip;
    const int stride = J.stride, xl = J.xl, yl = J.yl, xn = J.xn, yn = J.yn, qf = J.qf, off = J.off;
    for (int t = 0; t < xl + yl - 1; ++t) {
        for (int x = threadIdx.x; x < xl; x += blockDim.x) {
            const int y = t - x;
            if (y < 0 || y >= yl) continue;
            int pred;
            if (y != 0) {
                if (x != 0) {
                    const int sum = c[(size_t)y * stride + x - 1] + c[(size_t)(y - 1) * stride + x - 1] +
                                    c[(size_t)(y - 1) * stride + x] + 3 / 2;
                    pred = sum < 0 ? (sum - 2) / 3 : sum / 3;
                } else {
                    pred = c[(size_t)(y - 1) * stride];
                }
            } else {
                pred = x != 0 ? c[x - 1] : 0;
            }
            pred = (int16_t)pred;
            int32_t* v = c + (size_t)y * stride + x;
            const bool skip = cb_skip[cb_index(y, yl, yn) * xn + cb_index(x, xl, xn)];
            if (skip) {
                *v = pred;
                if (qout) qout[(size_t)y * stride + x] = 0;
            } else {
                const int val = (int16_t)(*v - pred);
                const unsigned qv = ((unsigned)abs(val) << 2) / (unsigned)qf;
                int r = 0;
                if (qv) {
                    r = (int)((qv * (unsigned)qf + off + 2) >> 2);
                    if (val <= 0) r = -r;
                }
                if (qout) qout[(size_t)y * stride + x] = val < 0 ? -(int)qv : (int)qv;
                *v = r + pred;
            }
        }
        __syncthreads();
    }
}

// ---- 5. dequantisation (the decoder's side) -------------------------------------------------
//
// After entropy decoding, the band decoders turn each magnitude q into
// (q * qf4 + offset + 2) >> 2 with the coded sign (GenericBandCodec::DecodeVal,
// band_codec_template.h:330-356), zero a skipped code block (ClearBlock, :488-496) or a
// skipped band (CompDecompressor::SetToVal, comp_decompress.cpp:121-125, 154-163), and in an
// intra picture add to the DC band's values the prediction from their reconstructed
// neighbours (GenericIntraDCBandCodec::DecodeCoeffBlock / ClearBlock / GetPrediction,
// band_codec_template.h:500-557).  The band table travels as a kernel parameter, so a call
// needs no device table and no host synchronisation.

constexpr int DQ_MAX_BANDS = 64;

struct DqBand {
    const void* q;      // band top-left in the index array (int32 or int16 elements)
    int32_t* c;         // band top-left in the coefficient array
    const uint8_t* cb;  // the band's code-block skip flags (device)
    int stride, xl, yl, xn, yn;
    int qf, off;        // QuantFactor4 and the intra / inter offset of the band's quantiser
    int skip;           // whole band zero
    int dc;             // intra DC band: predictions added by dc_decode_kernel
    int first, rows;    // first CTA and rows per CTA in the row-chunked grid
};

struct DqArgs {
    DqBand band[DQ_MAX_BANDS];
    int nbands;
    int dc_band[DQ_MAX_BANDS];  // bands decoded by dc_decode_kernel, one CTA each
};

// The decoded value of a signed index: int32 arithmetic as DecodeVal's (CoeffType).
__device__ __forceinline__ int dequant_value(int qi, int qf, int off) {
    if (qi == 0) return 0;
    const unsigned mag = qi < 0 ? 0u - (unsigned)qi : (unsigned)qi;
    const int v = (int)(mag * (unsigned)qf + (unsigned)(off + 2)) >> 2;
    return qi < 0 ? -v : v;
}

// grid: row chunks of the bands laid end to end, a warp per row, lanes across it, the code
// block followed by CbWalk.  An intra DC band gets its decoded residues here (zero in skipped
// code blocks); dc_decode_kernel then adds the predictions.  Idx: the index element type
// (int32, or int16 where every index fits: half the bytes read).
template <typename Idx>
__global__ void __launch_bounds__(ROW_THREADS) dequantise_kernel(const __grid_constant__ DqArgs A) {
    int lo_b = 0, hi_b = A.nbands - 1;
    while (lo_b < hi_b) {
        const int mid = (lo_b + hi_b + 1) >> 1;
        if (A.band[mid].first <= (int)blockIdx.x) lo_b = mid;
        else hi_b = mid - 1;
    }
    const DqBand& B = A.band[lo_b];
    const int r0 = ((int)blockIdx.x - B.first) * B.rows;
    const int r1 = min(B.yl, r0 + B.rows);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int xl = B.xl;
    for (int j = r0 + warp; j < r1; j += ROW_THREADS / 32) {
        if (lane >= xl) break;
        const Idx* qrow = static_cast<const Idx*>(B.q) + (size_t)j * B.stride;  // int32: may alias row
        int32_t* row = B.c + (size_t)j * B.stride;
        if (B.skip) {
            for (int i = lane; i < xl; i += 32) row[i] = 0;
            continue;
        }
        const uint8_t* skip_row = B.cb + cb_of(j, B.yl, B.yn) * B.xn;
        CbWalk w(lane, xl, B.xn);
        // four loads in flight per lane before the first store (each element is read before
        // it is written, by the same lane, so in-place calls are safe)
        for (int i0 = lane; i0 < xl; i0 += 128) {
            int v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = i0 + 32 * u < xl ? qrow[i0 + 32 * u] : 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = i0 + 32 * u;
                if (i < xl) {
                    w.to(i);
                    row[i] = skip_row[w.cx] ? 0 : dequant_value(v[u], B.qf, B.off);
                }
            }
        }
    }
}

// Intra DC bands, one CTA each, after dequantise_kernel has written the decoded residues:
// value = residue + prediction from the reconstructed left / top-left / top neighbours
// (int32, as the decoder's GetPrediction computes it); in a skipped code block the residue is
// zero and the value the prediction alone.  Positions on one anti-diagonal depend only on
// earlier diagonals, so the diagonals run in order and each one in parallel; that equals the
// reference's code block by code block raster order.
__global__ void dc_decode_kernel(const __grid_constant__ DqArgs A) {
    const DqBand& B = A.band[A.dc_band[blockIdx.x]];
    int32_t* const c = B.c;
    const int stride = B.stride, xl = B.xl, yl = B.yl;
    for (int t = 0; t < xl + yl - 1; ++t) {
        for (int x = threadIdx.x; x < xl; x += blockDim.x) {
            const int y = t - x;
            if (y < 0 || y >= yl) continue;
            int pred;
            if (y != 0) {
                if (x != 0) {
                    const int sum = c[(size_t)y * stride + x - 1] + c[(size_t)(y - 1) * stride + x - 1] +
                                    c[(size_t)(y - 1) * stride + x] + 3 / 2;
                    pred = sum < 0 ? (sum - 2) / 3 : sum / 3;
                } else {
                    pred = c[(size_t)(y - 1) * stride];
                }
            } else {
                pred = x != 0 ? c[x - 1] : 0;
            }
            c[(size_t)y * stride + x] += pred;
        }
        __syncthreads();
    }
}

// ---- intra DC wavefronts in shared memory ---------------------------------------------------
//
// The same recurrences with the band staged in shared memory: one coalesced pass in, the
// anti-diagonals against shared memory (a step costs a barrier and a few shared accesses
// instead of dependent global round trips), one coalesced pass out.  Used when the band fits.

constexpr int DC_SMEM_MAX = 200 * 1024;
constexpr int DC_THREADS = 256;

__device__ __forceinline__ int dc_pred_smem(const int32_t* s, int xl, int x, int y) {
    if (y != 0) {
        if (x != 0) {
            const int sum = s[y * xl + x - 1] + s[(y - 1) * xl + x - 1] + s[(y - 1) * xl + x] + 3 / 2;
            return sum < 0 ? (sum - 2) / 3 : sum / 3;
        }
        return s[(y - 1) * xl];
    }
    return x != 0 ? s[x - 1] : 0;
}

// Loads an xl x yl band (row stride `stride`) into shared memory with several loads in flight
// per thread.
__device__ __forceinline__ void dc_stage_in(int32_t* s, const int32_t* g, int stride, int xl, int n) {
    for (int k0 = threadIdx.x; k0 < n; k0 += 8 * DC_THREADS) {
        int v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int k = k0 + u * DC_THREADS;
            const int y = k / xl;
            v[u] = k < n ? g[(size_t)y * stride + (k - y * xl)] : 0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (k0 + u * DC_THREADS < n) s[k0 + u * DC_THREADS] = v[u];
    }
}

// Encoder side (dc_intra_kernel's arithmetic).
__global__ void __launch_bounds__(DC_THREADS) dc_intra_smem_kernel(const DcJob* jobs) {
    extern __shared__ int32_t s_dc[];
    const DcJob J = jobs[blockIdx.x];
    const int xl = J.xl, yl = J.yl, n = xl * yl;
    dc_stage_in(s_dc, J.c, J.stride, xl, n);
    __syncthreads();
    for (int t = 0; t < xl + yl - 1; ++t) {
        const int x0 = max(0, t - yl + 1), x1 = min(t, xl - 1);
        for (int x = x0 + (int)threadIdx.x; x <= x1; x += DC_THREADS) {
            const int y = t - x;
            const int pred = (int16_t)dc_pred_smem(s_dc, xl, x, y);
            const bool skip = J.cb_skip[cb_index(y, yl, J.yn) * J.xn + cb_index(x, xl, J.xn)];
            int32_t& v = s_dc[y * xl + x];
            int qi = 0;
            if (skip) {
                v = pred;
            } else {
                const int val = (int16_t)(v - pred);
                const unsigned qv = ((unsigned)abs(val) << 2) / (unsigned)J.qf;
                int r = 0;
                if (qv) {
                    r = (int)((qv * (unsigned)J.qf + J.off + 2) >> 2);
                    if (val <= 0) r = -r;
                }
                qi = val < 0 ? -(int)qv : (int)qv;
                v = r + pred;
            }
            if (J.qout) J.qout[(size_t)y * J.stride + x] = qi;
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < n; k += DC_THREADS) {
        const int y = k / xl;
        J.c[(size_t)y * J.stride + (k - y * xl)] = s_dc[k];
    }
}

// Decoder side (dc_decode_kernel's arithmetic) over the residues dequantise_kernel wrote.
__global__ void __launch_bounds__(DC_THREADS) dc_decode_smem_kernel(const __grid_constant__ DqArgs A) {
    extern __shared__ int32_t s_dc[];
    const DqBand& B = A.band[A.dc_band[blockIdx.x]];
    const int xl = B.xl, yl = B.yl, n = xl * yl;
    dc_stage_in(s_dc, B.c, B.stride, xl, n);
    __syncthreads();
    for (int t = 0; t < xl + yl - 1; ++t) {
        const int x0 = max(0, t - yl + 1), x1 = min(t, xl - 1);
        for (int x = x0 + (int)threadIdx.x; x <= x1; x += DC_THREADS) {
            const int y = t - x;
            s_dc[y * xl + x] += dc_pred_smem(s_dc, xl, x, y);
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < n; k += DC_THREADS) {
        const int y = k / xl;
        B.c[(size_t)y * B.stride + (k - y * xl)] = s_dc[k];
    }
}

// Opts the shared-memory DC kernels into DC_SMEM_MAX bytes of dynamic shared memory, once
// per device (the attribute belongs to the current device; one fixed value, so concurrent
// host threads never launch against a smaller setting).
int dc_smem_setup() {
    static std::mutex mu;
    static uint64_t done = 0;  // devices 0..63 already set up
    int dev = 0;
    DGPU_CHECK_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
    std::lock_guard<std::mutex> lock(mu);
    if (bit && (done & bit)) return DGPU_OK;
    DGPU_CHECK_CUDA(
        cudaFuncSetAttribute(dc_intra_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DC_SMEM_MAX));
    DGPU_CHECK_CUDA(
        cudaFuncSetAttribute(dc_decode_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DC_SMEM_MAX));
    done |= bit;
    return DGPU_OK;
}

// ---- host: the reference's Lagrangian choice (quant_chooser.cpp:62-147, 266-318) -------------

struct HostStat {
    double error;
    int count0, pos, neg;
};

struct CostD {
    double Error, ENTROPY, TOTAL;
};

CostD lagrangian(const HostStat& s, int count1, float wt, float lambda, float ecf) {
    CostD c;
    c.Error = s.error / double(count1);
    c.Error = std::sqrt(c.Error) / (wt * wt);
    double p0 = double(s.count0) / double(s.count0 + count1);
    double p1 = 1.0 - p0;
    if (p0 != 0.0 && p1 != 0.0)
        c.ENTROPY = -(p0 * std::log(p0) + p1 * std::log(p1)) / std::log(2.0);
    else
        c.ENTROPY = 0.0;
    c.ENTROPY *= double(s.count0 + count1);
    c.ENTROPY /= double(count1);
    double se;
    if (s.pos + s.neg != 0) {
        p0 = double(s.neg) / double(s.pos + s.neg);
        p1 = 1.0 - p0;
        if (p0 != 0.0 && p1 != 0.0)
            se = -((p0 * std::log(p0) + p1 * std::log(p1)) / std::log(2.0));
        else
            se = 0.0;
    } else {
        se = 0.0;
    }
    se *= double(s.neg + s.pos);
    se /= double(count1);
    c.ENTROPY += se;
    c.ENTROPY *= ecf;
    c.TOTAL = c.Error + lambda * c.ENTROPY;
    return c;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_quant_factor4(int q) { return (q < 0 || q > 119) ? DGPU_ERR_ARG : qf4(q); }

// Page-locked host staging for the statistics read-back, one growing buffer per host thread
// (released at thread exit).
struct PinnedScratch {
    void* p = nullptr;
    size_t n = 0;
    ~PinnedScratch() {
        if (p) cudaFreeHost(p);
    }
};

static int pinned_scratch(size_t bytes, char** out) {
    thread_local PinnedScratch buf;
    if (buf.n < bytes) {
        if (buf.p) cudaFreeHost(buf.p);
        buf.p = nullptr;
        buf.n = 0;
        if (cudaMallocHost(&buf.p, bytes) != cudaSuccess) {
            cudaGetLastError();
            buf.p = nullptr;
            return DGPU_ERR_NOMEM;
        }
        buf.n = bytes;
    }
    *out = static_cast<char*>(buf.p);
    return DGPU_OK;
}

// Device workspace of one dgpu_code_residue_batch call: task table, band and code-block
// maxima, statistics, intra DC prediction residues, code-block skip flags and the
// sequential-sum fallback cases.
static size_t residue_ws_need(int nb_total, int ncb_total, size_t dcwork_elems) {
    return align_up(sizeof(BandTask) * nb_total, 256) + align_up(sizeof(int) * nb_total, 256) +
           align_up(sizeof(int2) * nb_total, 256) +
           align_up(sizeof(int) * ncb_total, 256) + align_up(sizeof(Stat) * nb_total * 2 * QMAX, 256) +
           align_up(sizeof(int32_t) * dcwork_elems, 256) + align_up(ncb_total, 256) +
           align_up(sizeof(Stat) * nb_total * 3, 256) + align_up(sizeof(QBand) * nb_total, 256) +
           align_up(sizeof(DcJob) * nb_total, 256) + 256;
}

extern "C" size_t dgpu_code_residue_workspace_bytes(int n, const int* intra, const int* depth, const int* cw,
                                                     const int* ch, const int* band_ncb) {
    if (n <= 0 || n > MAX_COMPS || !intra || !depth || !cw || !ch || !band_ncb) return 0;
    int nb_total = 0, ncb_total = 0;
    size_t dcwork_elems = 0;
    for (int c = 0; c < n; ++c) {
        const int d = depth[c];
        if (d < 1 || d > 8) return 0;
        for (int b = 0; b < 3 * d + 1; ++b)
            ncb_total += band_ncb[2 * (nb_total + b)] * band_ncb[2 * (nb_total + b) + 1];
        if (intra[c]) dcwork_elems += (size_t)(cw[c] >> d) * (ch[c] >> d);
        nb_total += 3 * d + 1;
    }
    return residue_ws_need(nb_total, ncb_total, dcwork_elems);
}

namespace dgpu {

int code_residue_batch(int n, const int* intra, const int* depth, int32_t* const* coeff, const int* cw, const int* ch,
                       const float* lambda, const float* band_wt, const float* band_ecf, const int* band_ncb,
                       int* band_qidx, int* band_skip, int* band_bits, uint8_t* cb_skip, int32_t* const* qout,
                       void* workspace, size_t ws_bytes, void* stream, int* max_coeff) {
    if (max_coeff) *max_coeff = INT_MAX;  // unknown until the band maxima are read
    if (n <= 0 || n > MAX_COMPS || !intra || !depth || !coeff || !cw || !ch || !lambda || !band_wt || !band_ecf ||
        !band_ncb || !band_qidx || !band_skip || !band_bits || !cb_skip)
        return DGPU_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    // ---- geometry and task tables ----
    std::vector<Comp> comps(n);
    std::vector<BandTask> tasks;
    int nb_total = 0, ncb_total = 0;
    std::vector<int> band_cb_first;
    size_t dcwork_elems = 0;
    for (int c = 0; c < n; ++c) {
        const int d = depth[c];
        if (!coeff[c] || d < 1 || d > 8 || cw[c] <= 0 || ch[c] <= 0 || cw[c] % (1 << d) || ch[c] % (1 << d))
            return DGPU_ERR_ARG;
        comps[c] = Comp{coeff[c], nullptr, cw[c], ch[c], d, intra[c] ? 1 : 0, 3 * d + 1, nb_total};
        for (int b = 1; b <= 3 * d + 1; ++b) {
            const int xn = band_ncb[2 * (nb_total + b - 1)], yn = band_ncb[2 * (nb_total + b - 1) + 1];
            if (xn <= 0 || yn <= 0) return DGPU_ERR_ARG;
            band_cb_first.push_back(ncb_total);
            ncb_total += xn * yn;
        }
        if (intra[c]) dcwork_elems += (size_t)(cw[c] >> d) * (ch[c] >> d);
        nb_total += 3 * d + 1;
    }
    if (nb_total > MAX_TASKS) return DGPU_ERR_ARG;
    // ---- workspace ----
    const size_t need = residue_ws_need(nb_total, ncb_total, dcwork_elems);
    if (!workspace) {
        int rc = library_scratch(need, stream, &workspace);
        if (rc) return rc;
    } else if (ws_bytes < need) {
        return DGPU_ERR_NOMEM;
    }
    char* p = static_cast<char*>(workspace);
    auto take = [&](size_t bytes) {
        char* q = p;
        p += align_up(bytes, 256);
        return q;
    };
    BandTask* d_tasks = reinterpret_cast<BandTask*>(take(sizeof(BandTask) * nb_total));
    int* d_band_max = reinterpret_cast<int*>(take(sizeof(int) * nb_total));
    int2* d_range = reinterpret_cast<int2*>(take(sizeof(int2) * nb_total));
    int* d_cb_max = reinterpret_cast<int*>(take(sizeof(int) * ncb_total));
    Stat* d_stats = reinterpret_cast<Stat*>(take(sizeof(Stat) * nb_total * 2 * QMAX));
    int32_t* d_dcwork = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * dcwork_elems));
    uint8_t* d_cbskip = reinterpret_cast<uint8_t*>(take(ncb_total));
    Stat* d_stats3 = reinterpret_cast<Stat*>(take(sizeof(Stat) * nb_total * 3));
    QBand* d_qbands = reinterpret_cast<QBand*>(take(sizeof(QBand) * nb_total));
    DcJob* d_dcjobs = reinterpret_cast<DcJob*>(take(sizeof(DcJob) * nb_total));

    size_t dcoff = 0;
    int chunks[2] = {0, 0}, echunks = 0;
    for (int c = 0; c < n; ++c) {
        Comp& C = comps[c];
        if (C.intra) {
            C.dcwork = d_dcwork + dcoff;
            dcoff += (size_t)(C.cw >> C.depth) * (C.ch >> C.depth);
        }
        for (int b = 1; b <= C.nbands; ++b) {
            int xp, yp, xl, yl;
            band_rect(C.depth, C.cw, C.ch, b, xp, yp, xl, yl);
            BandTask T;
            const bool dcw = C.intra && b == C.nbands;
            T.data = dcw ? C.dcwork : C.coeff + (size_t)yp * C.cw + xp;
            T.stride = dcw ? xl : C.cw;
            T.xl = xl;
            T.yl = yl;
            T.comp = c;
            T.band = C.band_first + b - 1;
            T.cb_first = band_cb_first[T.band];
            T.xn = band_ncb[2 * T.band];
            T.yn = band_ncb[2 * T.band + 1];
            T.elem_first = echunks;
            T.rows_per_cta = rows_per_cta(xl);
            echunks += (yl + T.rows_per_cta - 1) / T.rows_per_cta;
            for (int pat = 0; pat < 2; ++pat) {
                const int xr = pat ? 1 : 2;
                const long long ns = (long long)((xl + xr - 1) / xr) * ((yl + 1) / 2);
                T.chunk_first[pat] = chunks[pat];
                chunks[pat] += (int)((ns + STAT_THREADS * 8 - 1) / (STAT_THREADS * 8));
            }
            tasks.push_back(T);
        }
    }
    DGPU_CHECK_CUDA(cudaMemcpyAsync(d_tasks, tasks.data(), sizeof(BandTask) * nb_total, cudaMemcpyHostToDevice, st));
    DGPU_CHECK_CUDA(cudaMemsetAsync(d_band_max, 0, sizeof(int) * nb_total, st));
    DGPU_CHECK_CUDA(cudaMemsetAsync(d_cb_max, 0, sizeof(int) * ncb_total, st));
    DGPU_CHECK_CUDA(cudaMemsetAsync(d_stats, 0, sizeof(Stat) * nb_total * 2 * QMAX, st));
    // ---- 1. DC DPCM (intra) and maxima ----
    for (int c = 0; c < n; ++c) {
        const Comp& C = comps[c];
        if (!C.intra) continue;
        const int xl = C.cw >> C.depth, yl = C.ch >> C.depth;
        dc_dpcm_kernel<<<(xl * yl + 255) / 256, 256, 0, st>>>(C.coeff, C.cw, xl, yl, C.dcwork);
        DGPU_CHECK_LAUNCH();
    }
    band_max_kernel<<<echunks, ROW_THREADS, 0, st>>>(d_tasks, nb_total, d_band_max, d_cb_max);
    DGPU_CHECK_LAUNCH();
    // ---- 2. statistics and the reference's three-pass Lagrangian choice per band ----
    // Passes 1 and 2 use the 2 x 2 pattern over every even quantiser; pass 3 needs the 1 x 2
    // pattern at three quantisers only, known once pass 2 is decided: its statistics are
    // gathered in a second, much smaller launch.
    stats_kernel<<<chunks[0], STAT_THREADS, 0, st>>>(d_tasks, d_band_max, d_stats, 0, nb_total, nullptr);
    DGPU_CHECK_LAUNCH();
    seq_resolve_kernel<<<resolve_grid((int)((size_t)nb_total * QMAX)), 128, 0, st>>>(
        d_tasks, d_stats, (int)((size_t)nb_total * QMAX), 0, nullptr);
    DGPU_CHECK_LAUNCH();
    // statistics and maxima come back through page-locked memory (one buffer per host thread)
    const size_t n_pat = (size_t)nb_total * QMAX;
    char* pin = nullptr;
    {
        const int rc = pinned_scratch(sizeof(Stat) * (n_pat + 3 * (size_t)nb_total) +
                                          sizeof(int) * (nb_total + ncb_total) + sizeof(int2) * nb_total + 256, &pin);
        if (rc) return rc;
    }
    Stat* hs = reinterpret_cast<Stat*>(pin);
    Stat* hs3 = hs + n_pat;  // third pass: [band][3], the quantisers qrange[band]
    int* hmax = reinterpret_cast<int*>(pin + sizeof(Stat) * (n_pat + 3 * (size_t)nb_total));
    int* hcb = hmax + nb_total;
    int2* hrange = reinterpret_cast<int2*>(align_up(reinterpret_cast<size_t>(hcb + ncb_total), 16));
    DGPU_CHECK_CUDA(cudaMemcpyAsync(hs, d_stats, sizeof(Stat) * n_pat, cudaMemcpyDeviceToHost, st));
    DGPU_CHECK_CUDA(cudaMemcpyAsync(hmax, d_band_max, sizeof(int) * nb_total, cudaMemcpyDeviceToHost, st));
    DGPU_CHECK_CUDA(cudaMemcpyAsync(hcb, d_cb_max, sizeof(int) * ncb_total, cudaMemcpyDeviceToHost, st));
    DGPU_CHECK_CUDA(host_wait(st));
    if (max_coeff) *max_coeff = nb_total ? *std::max_element(hmax, hmax + nb_total) : 0;
    // Statistics of (band t, pattern, q): pattern 0 at hs[t * QMAX + q]; pattern 1 (only the
    // three quantisers of the band's range) at hs3[t * 3 + q - lo].  Sums the exact path could
    // not represent were replaced on the device by the reference's sequential double sums.
    std::vector<int2> hrange_v(nb_total, make_int2(0, -1));
    auto host_stat = [&](int t, int pat, int q) {
        const Stat& S = pat == 0 ? hs[(size_t)t * QMAX + q] : hs3[(size_t)t * 3 + (q - hrange_v[t].x)];
        HostStat h;
        h.count0 = (int)(uint32_t)S.count0;
        h.pos = (int)(uint32_t)(S.posneg & 0xffffffffu);
        h.neg = (int)(uint32_t)(S.posneg >> 32);
        if (S.pad) {
            double d;
            std::memcpy(&d, &S.err_lo, sizeof d);
            h.error = d;
        } else {
            h.error = (double)S.err_lo;
        }
        return h;
    };
    std::vector<std::vector<CostD>> cost(nb_total);
    std::vector<int> mn2(nb_total, 0), nqs(nb_total, 0);
    std::atomic<int> too_big{0};
    parallel_for(nb_total, 64, [&](int t0, int t1) {
    for (int t = t0; t < t1; ++t) {
        const BandTask& T = tasks[t];
        const int maxv = hmax[t];
        hrange[t] = make_int2(0, -1);
        if (maxv < 1) continue;
        const int max_bit = int(std::floor(std::log(float(maxv)) / std::log(2.0)));
        const int nq = 4 * max_bit + 5;
        if (nq > QMAX) {
            too_big = 1;
            continue;
        }
        nqs[t] = nq;
        cost[t].resize(nq);
        int lo = 0, hi = nq - 1, step = 4, mn = 0;
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) {
                lo = std::max(mn - 2, 0);
                hi = std::min(mn + 2, nq - 1);
                step = 2;
            }
            const int count1 = (T.xl / 2) * (T.yl / 2);
            for (int qq = lo; qq <= hi; qq += step)
                cost[t][qq] = lagrangian(host_stat(t, 0, qq), count1, band_wt[t], lambda[T.comp], band_ecf[t]);
            mn = lo;
            for (int qq = lo + step; qq <= hi; qq += step)
                if (cost[t][qq].TOTAL < cost[t][mn].TOTAL) mn = qq;
        }
        mn2[t] = mn;
        hrange[t] = make_int2(std::max(mn - 1, 0), std::min(mn + 1, nq - 1));
    }
    });
    if (too_big) return DGPU_ERR_SIZE;
    for (int t = 0; t < nb_total; ++t) hrange_v[t] = hrange[t];
    DGPU_CHECK_CUDA(cudaMemcpyAsync(d_range, hrange, sizeof(int2) * nb_total, cudaMemcpyHostToDevice, st));
    stats_kernel<<<chunks[1], STAT_THREADS, 0, st>>>(d_tasks, d_band_max, d_stats, 1, nb_total, d_range);
    DGPU_CHECK_LAUNCH();
    gather_stats_kernel<<<(3 * nb_total + 255) / 256, 256, 0, st>>>(d_stats + n_pat, d_range, nb_total, d_stats3);
    DGPU_CHECK_LAUNCH();
    seq_resolve_kernel<<<resolve_grid(3 * nb_total), 128, 0, st>>>(d_tasks, d_stats3, 3 * nb_total, 1, d_range);
    DGPU_CHECK_LAUNCH();
    DGPU_CHECK_CUDA(cudaMemcpyAsync(hs3, d_stats3, sizeof(Stat) * 3 * nb_total, cudaMemcpyDeviceToHost, st));
    DGPU_CHECK_CUDA(host_wait(st));
    std::vector<uint8_t> hskip(ncb_total, 0);
    parallel_for(nb_total, 64, [&](int t0, int t1) {
    for (int t = t0; t < t1; ++t) {
        const BandTask& T = tasks[t];
        int q = 0, bits = 0;
        if (hmax[t] >= 1) {
            const int lo = hrange[t].x, hi = hrange[t].y;
            const int count1 = (T.xl / 1) * (T.yl / 2);
            for (int qq = lo; qq <= hi; ++qq)
                cost[t][qq] = lagrangian(host_stat(t, 1, qq), count1, band_wt[t], lambda[T.comp], band_ecf[t]);
            int mn = lo;
            for (int qq = lo + 1; qq <= hi; ++qq)
                if (cost[t][qq].TOTAL < cost[t][mn].TOTAL) mn = qq;
            const double bit_sum = cost[t][mn].ENTROPY * T.xl * T.yl;
            bits = int(bit_sum);
            q = mn;
            const int thr = qf4(q);
            for (int k = 0; k < T.xn * T.yn; ++k) hskip[T.cb_first + k] = (hcb[T.cb_first + k] << 2) < thr;
        }
        band_qidx[t] = q;
        band_bits[t] = bits;
        band_skip[t] = bits == 0;
    }
    });
    std::memcpy(cb_skip, hskip.data(), ncb_total);
    DGPU_CHECK_CUDA(cudaMemcpyAsync(d_cbskip, hskip.data(), ncb_total, cudaMemcpyHostToDevice, st));
    // ---- 4. quantise and reconstruct, DC bands first (every intra component in one launch) ----
    {
        std::vector<DcJob> dj;
        int threads = 32;
        size_t smem = 0;
        for (int c = 0; c < n; ++c) {
            const Comp& C = comps[c];
            const int t = C.band_first + C.nbands - 1;
            if (!C.intra || band_skip[t]) continue;
            const int xl = C.cw >> C.depth, yl = C.ch >> C.depth;
            const int q = band_qidx[t];
            threads = std::max(threads, std::min(1024, ((xl + 31) / 32) * 32));
            smem = std::max(smem, (size_t)xl * yl * sizeof(int32_t));
            dj.push_back(DcJob{const_cast<int32_t*>(C.coeff), qout ? qout[c] : nullptr, d_cbskip + tasks[t].cb_first,
                               C.cw, xl, yl, tasks[t].xn, tasks[t].yn, qf4(q), intra_off4(q)});
        }
        if (!dj.empty()) {
            DGPU_CHECK_CUDA(cudaMemcpyAsync(d_dcjobs, dj.data(), sizeof(DcJob) * dj.size(), cudaMemcpyHostToDevice, st));
            if (smem <= (size_t)DC_SMEM_MAX) {
                const int rc = dc_smem_setup();
                if (rc) return rc;
                dc_intra_smem_kernel<<<(int)dj.size(), DC_THREADS, smem, st>>>(d_dcjobs);
            } else {
                dc_intra_kernel<<<(int)dj.size(), threads, 0, st>>>(d_dcjobs);
            }
            DGPU_CHECK_LAUNCH();
        }
    }
    // one launch over every band not quantised above, from a device table
    std::vector<QBand> qb;
    qb.reserve(nb_total);
    int qchunks = 0;
    for (int t = 0; t < nb_total; ++t) {
        const BandTask& T = tasks[t];
        const Comp& C = comps[T.comp];
        if (C.intra && t == C.band_first + C.nbands - 1 && !band_skip[t]) continue;  // done above
        int xp, yp, xl, yl;
        band_rect(C.depth, C.cw, C.ch, t - C.band_first + 1, xp, yp, xl, yl);
        QBand B;
        B.data = const_cast<int32_t*>(C.coeff) + (size_t)yp * C.cw + xp;
        B.qout = qout && qout[T.comp] ? qout[T.comp] + (size_t)yp * C.cw + xp : nullptr;
        B.stride = C.cw;
        B.xl = xl;
        B.yl = yl;
        B.xn = T.xn;
        B.yn = T.yn;
        B.qf = qf4(band_qidx[t]);
        B.off = C.intra ? intra_off4(band_qidx[t]) : inter_off4(band_qidx[t]);
        B.skip = band_skip[t];
        B.cb_skip = d_cbskip + T.cb_first;
        B.first = qchunks;
        B.rows = rows_per_cta(xl);
        qchunks += (yl + B.rows - 1) / B.rows;
        qb.push_back(B);
    }
    if (qb.empty()) return DGPU_OK;
    // a copy from pageable memory returns once the source has been staged, so qb may go
    DGPU_CHECK_CUDA(cudaMemcpyAsync(d_qbands, qb.data(), sizeof(QBand) * qb.size(), cudaMemcpyHostToDevice, st));
    quantise_kernel<<<qchunks, ROW_THREADS, 0, st>>>(d_qbands, (int)qb.size());
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}

}  // namespace dgpu

extern "C" int dgpu_code_residue_batch(int n, const int* intra, const int* depth, int32_t* const* coeff,
                                       const int* cw, const int* ch, const float* lambda, const float* band_wt,
                                       const float* band_ecf, const int* band_ncb, int* band_qidx, int* band_skip,
                                       int* band_bits, uint8_t* cb_skip, int32_t* const* qout, void* workspace,
                                       size_t ws_bytes, void* stream) {
    return code_residue_batch(n, intra, depth, coeff, cw, ch, lambda, band_wt, band_ecf, band_ncb, band_qidx,
                              band_skip, band_bits, cb_skip, qout, workspace, ws_bytes, stream, nullptr);
}

namespace {

// Launches the dequantisation of the bands collected in A (row-chunked grid, then the intra
// DC wavefronts) and empties A.
int launch_dequantise(DqArgs& A, int ndc, int chunks, bool idx16, cudaStream_t st) {
    if (A.nbands == 0) return DGPU_OK;
    if (chunks > 0) {
        if (idx16) dequantise_kernel<int16_t><<<chunks, ROW_THREADS, 0, st>>>(A);
        else dequantise_kernel<int32_t><<<chunks, ROW_THREADS, 0, st>>>(A);
        DGPU_CHECK_LAUNCH();
    }
    if (ndc > 0) {
        size_t smem = 0;
        for (int k = 0; k < ndc; ++k) {
            const DqBand& B = A.band[A.dc_band[k]];
            smem = std::max(smem, (size_t)B.xl * B.yl * sizeof(int32_t));
        }
        if (smem <= (size_t)DC_SMEM_MAX) {
            const int rc = dc_smem_setup();
            if (rc) return rc;
            dc_decode_smem_kernel<<<ndc, DC_THREADS, smem, st>>>(A);
        } else {
            dc_decode_kernel<<<ndc, 256, 0, st>>>(A);
        }
        DGPU_CHECK_LAUNCH();
    }
    A.nbands = 0;
    return DGPU_OK;
}

}  // namespace

namespace {

// dgpu_dequantise_batch over int32 (idx16 false) or int16 (true) index arrays.
int dequantise_batch(int n, const int* intra, const int* depth, const void* const* qindex, bool idx16,
                     int32_t* const* coeff, const int* cw, const int* ch, const int* band_ncb, const int* band_qidx,
                     const int* band_skip, const uint8_t* cb_skip, void* stream) {
    if (n <= 0 || n > MAX_COMPS || !intra || !depth || !qindex || !coeff || !cw || !ch || !band_ncb || !band_qidx ||
        !band_skip || !cb_skip)
        return DGPU_ERR_ARG;
    // validate everything before the first launch
    for (int c = 0, b0 = 0; c < n; ++c) {
        const int d = depth[c];
        if (d < 1 || d > 8 || !qindex[c] || !coeff[c] || cw[c] <= 0 || ch[c] <= 0 || (cw[c] % (1 << d)) != 0 ||
            (ch[c] % (1 << d)) != 0)
            return DGPU_ERR_ARG;
        for (int b = 0; b < 3 * d + 1; ++b) {
            const int g = b0 + b;
            if (band_ncb[2 * g] < 1 || band_ncb[2 * g + 1] < 1) return DGPU_ERR_ARG;
            // an index the decoder would refuse (band_codec_template.h:250-258)
            if (!band_skip[g] && (band_qidx[g] < 0 || band_qidx[g] > 119)) return DGPU_ERR_ARG;
        }
        b0 += 3 * d + 1;
    }
    cudaStream_t st = as_stream(stream);
    DqArgs A;
    A.nbands = 0;
    int chunks = 0, ndc = 0;
    size_t cb_off = 0;
    for (int c = 0, b0 = 0; c < n; ++c) {
        const int d = depth[c], nb = 3 * d + 1;
        if (A.nbands + nb > DQ_MAX_BANDS) {
            const int rc = launch_dequantise(A, ndc, chunks, idx16, st);
            if (rc) return rc;
            chunks = ndc = 0;
        }
        for (int b = 1; b <= nb; ++b) {
            const int g = b0 + b - 1;
            int xp, yp, xl, yl;
            band_rect(d, cw[c], ch[c], b, xp, yp, xl, yl);
            DqBand& B = A.band[A.nbands];
            const size_t at = (size_t)yp * cw[c] + xp;
            B.q = idx16 ? (const void*)(static_cast<const int16_t*>(qindex[c]) + at)
                        : (const void*)(static_cast<const int32_t*>(qindex[c]) + at);
            B.c = coeff[c] + at;
            B.cb = cb_skip + cb_off;
            B.stride = cw[c];
            B.xl = xl;
            B.yl = yl;
            B.xn = band_ncb[2 * g];
            B.yn = band_ncb[2 * g + 1];
            B.skip = band_skip[g] ? 1 : 0;
            const int q = B.skip ? 0 : band_qidx[g];
            B.qf = qf4(q);
            B.off = intra[c] ? intra_off4(q) : inter_off4(q);
            B.dc = (intra[c] && b == nb && !B.skip) ? 1 : 0;
            B.rows = rows_per_cta(xl);
            B.first = chunks;
            chunks += (yl + B.rows - 1) / B.rows;
            if (B.dc) A.dc_band[ndc++] = A.nbands;
            cb_off += (size_t)B.xn * B.yn;
            ++A.nbands;
        }
        b0 += nb;
    }
    return launch_dequantise(A, ndc, chunks, idx16, st);
}

}  // namespace

extern "C" int dgpu_dequantise_batch(int n, const int* intra, const int* depth, const int32_t* const* qindex,
                                     int32_t* const* coeff, const int* cw, const int* ch, const int* band_ncb,
                                     const int* band_qidx, const int* band_skip, const uint8_t* cb_skip,
                                     void* stream) {
    if (!qindex || n <= 0 || n > MAX_COMPS) return DGPU_ERR_ARG;
    const void* q[MAX_COMPS];
    for (int c = 0; c < n; ++c) q[c] = qindex[c];
    return dequantise_batch(n, intra, depth, q, false, coeff, cw, ch, band_ncb, band_qidx, band_skip, cb_skip,
                            stream);
}

extern "C" int dgpu_dequantise_batch16(int n, const int* intra, const int* depth, const int16_t* const* qindex,
                                       int32_t* const* coeff, const int* cw, const int* ch, const int* band_ncb,
                                       const int* band_qidx, const int* band_skip, const uint8_t* cb_skip,
                                       void* stream) {
    if (!qindex || n <= 0 || n > MAX_COMPS) return DGPU_ERR_ARG;
    const void* q[MAX_COMPS];
    for (int c = 0; c < n; ++c) q[c] = qindex[c];
    return dequantise_batch(n, intra, depth, q, true, coeff, cw, ch, band_ncb, band_qidx, band_skip, cb_skip,
                            stream);
}

// CoeffArray::SetBandWeights (libdirac_common/wavelet_utils.cpp:192-382) with
// PerceptualWeight (:384-395): perceptual weights of the 3*depth+1 bands of one component,
// then the compensation for the unscaled lifting filters.  Host-only helper (no GPU use);
// types and operation order follow the reference (float frequencies, double weights).
extern "C" int dgpu_band_weights(int filter, int depth, int cw, int ch, int comp, int cformat, float cpd,
                                 float cpd_scale, int field_coding, double* out) {
    if (!out || depth < 1 || depth > 8 || cw <= 0 || ch <= 0) return DGPU_ERR_ARG;
    const int nb = 3 * depth + 1;
    // Subband::SetWt takes a float (wavelet_utils.cpp:112): every stored weight is rounded
    auto set_wt = [](double w) -> double { return (double)(float)w; };
    const float c = cpd * cpd_scale;
    float chroma_xfac = 1.0f, chroma_yfac = 1.0f;
    if (comp != 0) {
        if (cformat == 1) {
            chroma_xfac = 2.0f;
            chroma_yfac = 1.0f;
        } else if (cformat == 2) {
            chroma_xfac = 2.0f;
            chroma_yfac = 2.0f;
        }
    }
    int xp, yp, xl, yl;
    band_rect(depth, cw, ch, 1, xp, yp, xl, yl);
    const int xlen = 2 * xl, ylen = 2 * yl;
    auto scale_of = [&](int b) { return b == nb ? (1 << depth) : (1 << ((b - 1) / 3 + 1)); };
    if (c != 0.0f) {
        for (int b = 1; b <= nb; ++b) {
            band_rect(depth, cw, ch, b, xp, yp, xl, yl);
            float xfreq = c * (float(xp) + (float(xl) / 2.0)) / float(xlen);
            float yfreq = c * (float(yp) + (float(yl) / 2.0)) / float(ylen);
            if (field_coding) yfreq /= 2.0;
            const float xf = xfreq / chroma_xfac, yf = yfreq / chroma_yfac;
            double freq_sqd(xf * xf + yf * yf);
            if (comp != 0) freq_sqd *= 1.2;
            const float w = 0.255 * std::pow(1.0 + 0.2561 * freq_sqd, 0.75);
            out[b - 1] = set_wt(w);
        }
        float min_weight = out[nb - 1];
        for (int b = 1; b <= nb - 1; ++b) min_weight = ((min_weight > out[b - 1]) ? out[b - 1] : min_weight);
        out[nb - 1] = set_wt(min_weight);
        double overall = 0.0;
        for (int b = 1; b <= nb; ++b) {
            const double frac = 1.0 / ((double)scale_of(b) * scale_of(b));
            overall += frac / (out[b - 1] * out[b - 1]);
        }
        overall = std::sqrt(overall);
        for (int b = nb; b > 0; --b) out[b - 1] = set_wt(out[b - 1] * overall);
    } else {
        for (int b = 1; b <= nb; ++b) out[b - 1] = set_wt(1.0);
    }
    double lfac, hfac;
    int filt_shift;
    switch (filter) {
        case DGPU_DD9_7: lfac = 1.218660804; hfac = 0.780720058; filt_shift = 1; break;
        case DGPU_LEGALL5_3: lfac = 1.179535649; hfac = 0.81649658; filt_shift = 1; break;
        case DGPU_DD13_7: lfac = 1.235705971; hfac = 0.780719354; filt_shift = 1; break;
        case DGPU_HAAR0: lfac = 1.414213562; hfac = 0.707106781; filt_shift = 0; break;
        case DGPU_HAAR1: lfac = 1.414213562; hfac = 0.707106781; filt_shift = 1; break;
        case DGPU_DAUB9_7: lfac = 1.149604398; hfac = 0.869864452; filt_shift = 1; break;
        default: lfac = 1.0; hfac = 1.0; filt_shift = 0; break;
    }
    double cf = (1 << (depth * filt_shift)) / std::pow(lfac, 2 * depth);
    out[nb - 1] = set_wt(out[nb - 1] * cf);
    for (int level = 1; level <= depth; ++level) {
        const int shift = (depth - level + 1) * filt_shift;
        for (int orient = 3; orient >= 1; --orient) {
            const int idx = 3 * (depth - level) + orient;
            cf = 1.0 / std::pow(lfac, 2 * (depth - level));
            band_rect(depth, cw, ch, idx, xp, yp, xl, yl);
            if (xp != 0 && yp != 0)
                cf /= (hfac * hfac);
            else
                cf /= (lfac * hfac);
            cf *= double(1 << shift);
            out[idx - 1] = set_wt(out[idx - 1] * cf);
        }
    }
    return DGPU_OK;
}

// EncoderParams::SetUsualCodeBlocks (common.cpp:488-510) as PictureCompressor::SetupCodeBlocks
// applies it (picture_compress.cpp:582-601): code blocks (x, y) per band from the luma size.
extern "C" int dgpu_code_blocks(int depth, int luma_w, int luma_h, int spatial_partition, int* ncb) {
    if (!ncb || depth < 1 || depth > 8) return DGPU_ERR_ARG;
    const int nb = 3 * depth + 1;
    const int xl_pad = (luma_w + (1 << depth) - 1) & ~((1 << depth) - 1);
    const int yl_pad = (luma_h + (1 << depth) - 1) & ~((1 << depth) - 1);
    for (int b = 1; b <= nb; ++b) {
        int xr = 1, yr = 1;
        if (spatial_partition) {
            const int level = depth - (b - 1) / 3;
            if (level == 0) {
                xr = std::max(1, (xl_pad >> depth) / 4);
                yr = std::max(1, (yl_pad >> depth) / 4);
            } else {
                const int i = depth - level + 1;
                xr = std::max(1, (xl_pad >> i) / 12);
                yr = std::max(1, (yl_pad >> i) / 12);
            }
        }
        ncb[2 * (b - 1)] = xr;
        ncb[2 * (b - 1) + 1] = yr;
    }
    return DGPU_OK;
}
