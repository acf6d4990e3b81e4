// Motion estimation for sm_100a: pel-accurate hierarchical block matching, sub-pel
// refinement and superblock mode decision, bit-exact with the reference's decisions.
//
// Replaces PictureCompressor::PixelME / SubPixelME / ModeDecisionME and the classes they
// drive (PixelMatcher, libdirac_motionest/pixel_match.cpp; MEData::SetLambdaMap,
// libdirac_common/motion.cpp:128-333; SubpelRefine and BlockMatcher::RefineMatchSubp,
// me_subpel.cpp, block_match.cpp:327-467; ModeDecider, me_mode_decn.cpp).
//
// Dependencies.  In every stage a block's predictor comes from neighbours decided before it
// in raster order (left, top, top-right; plus top-left for sub-pel; the left, top-left and
// top superblocks for mode decision), so each stage is a wavefront.  A wavefront stage is one
// persistent launch: warps claim units in raster order from an atomic ticket, wait (bounded
// spin) for the completion flags of the neighbours they read, and publish their own flag with
// release semantics.  Raster-ordered tickets make this deadlock-free whatever the grid size:
// the lowest unfinished ticket only waits on lower tickets, which are finished or running.
// Work that does not depend on the raster order runs fully parallel first: for the pel search
// these are the zero-centred and guide-centred candidate lists; only the predictor-centred
// list is evaluated inside the wavefront.
//
// Exactness.  Candidates are evaluated in the reference's list order and the first strictly
// smaller cost wins, as in the reference (a duplicate of an earlier candidate can never be
// strictly smaller, so duplicates need no removal).  Sub-pel and superblock costs are float
// sums the reference accumulates pixel by pixel in raster order from mvcost * lambda.  A float
// sum of non-negative integers can only round when it crosses a power of two, so the warp
// computes exact prefix sums with integer scans and applies one double -> float
// round-to-nearest-even at each crossing (FloatSeq below), which reproduces the sequential
// float result.  The library is compiled with --fmad=false: a*b+c is never fused.
//
// The lambda map's transition statistics are long double in the reference; that small step
// (one value per block) runs on the host between the pel and the sub-pel stages.

#include <cuda/atomic>

#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <atomic>
#include <mutex>
#include <thread>
#include <vector>

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int WARPS_PER_CTA = 4;
constexpr int ME_THREADS = 32 * WARPS_PER_CTA;
constexpr long long SPIN_LIMIT = 1LL << 21;  // about 2 s of polling at the longest back-off

// Failure-detection and ordering checks of a wavefront launch (dgpu_debug_wavefront): the
// polls after which a wait gives up, a unit whose completion flag is left unset so that its
// dependants' waits run out (pel wavefront only; -1: none), and an optional audit array that
// receives, for every unit of the launch's first job, the position at which it was decided
// ([0] is the running counter).  Normal calls carry {SPIN_LIMIT, -1, nullptr}.
// ops, when not null, accumulates the launch's algorithmic integer operations: 3 per
// pixel of every block difference the reference's search evaluates (subtract, absolute value,
// add), plus the interpolation of sub-pel predictions (interp_ops) and the bi-prediction and
// intra terms of mode decision.
struct WaveDebug {
    long long spin_limit;
    int skip_unit;
    int* audit;
    unsigned long long* ops;
};

__device__ __forceinline__ void audit_unit(const WaveDebug& d, int job, int unit) {
    if (d.audit && job == 0) d.audit[1 + unit] = atomicAdd(d.audit, 1);
}

// Interpolation operations per predicted sample at precision p (1 half-pel: a sample of the
// upconverted plane; 2 quarter-pel: a rounded mean of two or four samples; 3 eighth-pel: four
// weighted samples).
__device__ __forceinline__ int interp_ops(int p) { return p <= 1 ? 0 : p == 2 ? 4 : 8; }

// Adds n operations to the launch's count (one lane per warp).
__device__ __forceinline__ void count_ops(unsigned long long* ops, long long n) {
    if (ops && (threadIdx.x & 31) == 0 && n > 0) atomicAdd(ops, (unsigned long long)n);
}

struct Olb {
    int xblen, yblen, xbsep, ybsep, xoff, yoff;
};

inline Olb make_olb(int xblen, int yblen, int xbsep, int ybsep) {
    return Olb{xblen, yblen, xbsep, ybsep, (xblen - xbsep) / 2, (yblen - ybsep) / 2};
}

struct Blim {
    int xp, yp, xl, yl;
};

// BlockDiffParams::SetBlockLimits (me_utils.cpp:58-80); lengths may come out <= 0.
__device__ __forceinline__ Blim block_limits(const Olb& o, int pw, int ph, int bx, int by) {
    Blim b;
    const int lx = bx * o.xbsep - o.xoff, ly = by * o.ybsep - o.yoff;
    b.xp = lx > 0 ? lx : 0;
    b.yp = ly > 0 ? ly : 0;
    b.xl = o.xblen - b.xp + lx;
    b.yl = o.yblen - b.yp + ly;
    if (b.xp + b.xl - 1 > pw - 1) b.xl = pw - b.xp;
    if (b.yp + b.yl - 1 > ph - 1) b.yl = ph - b.yp;
    return b;
}

__device__ __forceinline__ int med3(int a, int b, int c) { return a + b + c - max(max(a, b), c) - min(min(a, b), c); }
__device__ __forceinline__ short2 mv_median3(short2 a, short2 b, short2 c) {
    return make_short2((short)med3(a.x, b.x, c.x), (short)med3(a.y, b.y, c.y));
}
__device__ __forceinline__ short2 mv_mean(short2 a, short2 b) {
    return make_short2((short)((a.x + b.x + 1) >> 1), (short)((a.y + b.y + 1) >> 1));
}
__device__ __forceinline__ int norm1(int x, int y) { return abs(x) + abs(y); }
// BlockMatcher::GetVarUp (block_match.cpp:213-220)
__device__ __forceinline__ int getvarup(short2 pred, int mx, int my) {
    return min(norm1(mx - pred.x, my - pred.y), norm1(mx, my));
}

// MvMedian of 0-4 vectors (motion.cpp:560-600)
__device__ short2 mv_median_list(const short2* v, int n) {
    if (n == 1) return v[0];
    if (n == 2) return mv_mean(v[0], v[1]);
    if (n == 3) return mv_median3(v[0], v[1], v[2]);
    if (n == 4) {
        int sx = 0, sy = 0, mxx = v[0].x, mnx = v[0].x, mxy = v[0].y, mny = v[0].y;
        for (int i = 0; i < 4; ++i) {
            sx += v[i].x;
            sy += v[i].y;
            mxx = max(mxx, (int)v[i].x);
            mnx = min(mnx, (int)v[i].x);
            mxy = max(mxy, (int)v[i].y);
            mny = min(mny, (int)v[i].y);
        }
        return make_short2((short)((sx - (mxx + mnx) + 1) >> 1), (short)((sy - (mxy + mny) + 1) >> 1));
    }
    return make_short2(0, 0);
}

// The k-th candidate of AddNewVlist(centre, r, r) (block_match.cpp:89-126): the centre, then
// (+i, 0), (-i, 0) for i = 1..r, then for j = 1..r and i = -r..r: (i, +j), (i, -j).
__device__ __forceinline__ short2 cand_at(short2 c, int r, int k) {
    if (k == 0) return c;
    if (k <= 2 * r) {
        const int i = (k + 1) >> 1;
        return make_short2((short)(c.x + ((k & 1) ? i : -i)), c.y);
    }
    const int u = k - (2 * r + 1), per = 2 * (2 * r + 1);
    const int j = u / per + 1, q = u - (j - 1) * per;
    const int i = (q >> 1) - r;
    return make_short2((short)(c.x + i), (short)(c.y + ((q & 1) ? -j : j)));
}

// ---- completion flags ---------------------------------------------------------------------

__device__ __forceinline__ void publish(int* flag) {
    cuda::atomic_ref<int, cuda::thread_scope_device> f(*flag);
    f.store(1, cuda::memory_order_release);
}

// Every lane waits (acquire) until *flag is set; gives up after `limit` polls and records the
// failure in *err (the host turns it into DGPU_ERR_CUDA).
// Once any wait has timed out, every later wait returns within 1024 polls, so a failed launch
// ends within about one timeout.
__device__ __forceinline__ void wait_flag(int* flag, int* err, long long limit) {
    cuda::atomic_ref<int, cuda::thread_scope_device> f(*flag);
    cuda::atomic_ref<int, cuda::thread_scope_device> e(*err);
    long long n = 0;
    unsigned ns = 32;
    while (f.load(cuda::memory_order_acquire) == 0) {
        if (++n > limit || ((n & 1023) == 0 && e.load(cuda::memory_order_relaxed) != 0)) {
            atomicOr(err, 1);
            return;
        }
        // back off (up to ~1 us) so that warps waiting far ahead of the wavefront take few
        // issue slots from the ones working on it
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

__device__ __forceinline__ int warp_ticket(int* counter) {
    int t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(counter, 1);
    return __shfl_sync(0xffffffffu, t, 0);
}

// ---- wavefront order over many jobs -------------------------------------------------------
// Units (x, y) of a W x H grid whose dependencies all lie on earlier "diagonals"
// t' = x' + slope * y' < t = x + slope * y (slope 2: left and top-right neighbours, slope 1:
// left, top-left and top).  Tickets enumerate diagonal by diagonal, and within a diagonal job
// by job, so every job of a launch advances its wavefront at the same time and a ticket only
// ever waits on smaller tickets.  prefix[t] = units of one job on diagonals before t.
struct Wave {
    const int* prefix;  // T + 1 entries
    int T, W, slope, njobs;
    int life;           // units a warp (a CTA of the mode wavefront) takes before it exits
};

__device__ __forceinline__ void wave_unit(const Wave& w, int u, int& j, int& x, int& y) {
    int lo = 0, hi = w.T - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&w.prefix[mid]) * w.njobs <= u) lo = mid;
        else hi = mid - 1;
    }
    const int p0 = __ldg(&w.prefix[lo]);
    const int c = __ldg(&w.prefix[lo + 1]) - p0;  // > 0: lo is the last diagonal starting at or before u
    const int r = u - p0 * w.njobs;
    j = r / c;
    const int ex = lo - (w.W - 1);
    y = (ex > 0 ? (ex + w.slope - 1) / w.slope : 0) + (r - j * c);
    x = lo - w.slope * y;
}

// ---- exact sequential float sums ------------------------------------------------------------

// Running value of the reference's  sum = start; sum += (float)d  loop, for d >= 0 integers.
struct FloatSeq {
    double c;      // current float value of the sum (held exactly in a double)
    double bound;  // smallest power of two above c: additions below it are exact
};

// The exponent e with v in [2^(e-1), 2^e) of a positive normal double, from its bits.
__device__ __forceinline__ int exp_above(double v) {
    return (int)((unsigned long long)__double_as_longlong(v) >> 52 & 0x7ff) - 1022;
}

// 2^e as a double, from its bits (e within the normal range).
__device__ __forceinline__ double pow2_of(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// Whether a non-negative double is a multiple of 2^k: the trailing zeros of its mantissa
// (implicit bit included) plus its binary exponent reach k.
__device__ __forceinline__ bool multiple_of_pow2(double v, int k) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    const int be = (int)(b >> 52 & 0x7ff);
    unsigned long long m = b & ((1ULL << 52) - 1);
    if (be == 0 && m == 0) return true;  // zero
    if (be) m |= 1ULL << 52;
    const int e = (be ? be : 1) - 1075;  // v = m * 2^e
    return __ffsll((long long)m) - 1 + e >= k;
}

__device__ __forceinline__ double pow2_above(double c) {
    if (c <= 0.0) return 16777216.0;  // integer partial sums from 0 are exact below 2^24
    return pow2_of(exp_above(c));     // c in [2^(e-1), 2^e)
}

__device__ __forceinline__ FloatSeq float_seq_start(float start) {
    FloatSeq f;
    f.c = (double)start;
    f.bound = pow2_above(f.c);
    return f;
}

// Adds a non-negative integer total to the running sum when no addition of its terms, in any
// order, can round: either no power of two is crossed, or the current value is a multiple of
// the float spacing at the final value (then every partial sum, a multiple of that spacing
// below 2^24, is a float).  Returns false, changing nothing, otherwise.
__device__ __forceinline__ bool float_seq_add_exact(FloatSeq& f, int total) {
    const double fin = f.c + (double)total;
    if (fin < f.bound) {
        f.c = fin;
        return true;
    }
    if (fin >= 16777216.0) return false;
    const int e = exp_above(fin);  // fin in [2^(e-1), 2^e): float spacing 2^(e-24)
    if (!multiple_of_pow2(f.c, e - 24)) return false;
    f.c = fin;
    f.bound = pow2_of(e);
    return true;
}

// Adds one term per lane (lane order = raster order; lanes without a term pass 0).
__device__ __forceinline__ void float_seq_add(FloatSeq& f, int d) {
    const int lane = threadIdx.x & 31;
    const int total = __reduce_add_sync(0xffffffffu, d);
    if (float_seq_add_exact(f, total)) return;
    int pre = d;  // inclusive prefix over lanes
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= o) pre += v;
    }
    int base = 0;  // prefix already folded into f.c
    for (;;) {
        const double need = f.bound - f.c;
        const unsigned m = __ballot_sync(0xffffffffu, (double)(pre - base) >= need);
        if (m == 0) {
            f.c += (double)(total - base);
            return;
        }
        const int pk = __shfl_sync(0xffffffffu, pre, __ffs(m) - 1);
        f.c = (double)__double2float_rn(f.c + (double)(pk - base));
        f.bound = pow2_above(f.c);
        base = pk;
    }
}

// ---- block differences ----------------------------------------------------------------------

// Block pixels are spread over the warp in raster order: pixel k of the block (row-major,
// xl per row) belongs to lane k % 32 at step k / 32, so every lane is busy whatever the block
// width, and lane order within a step is raster order.  PixWalk tracks one lane's position.
struct PixWalk {
    int row, col, drow, dcol, xl;
    __device__ __forceinline__ PixWalk(int xl_, int k0 = 0) : xl(xl_) {
        const int k = k0 + (threadIdx.x & 31);
        row = k / xl;
        col = k - row * xl;
        drow = 32 / xl;
        dcol = 32 - drow * xl;
    }
    __device__ __forceinline__ void next() {
        col += dcol;
        row += drow;
        if (col >= xl) {
            col -= xl;
            ++row;
        }
    }
};

// Prediction sample from an upconverted reference (uw x uh) at precision p (1 half,
// 2 quarter, 3 eighth), coordinates clamped to the array (me_utils.cpp:410-1170).
__device__ __forceinline__ int up_at(const int16_t* up, int uw, int uh, int yy, int xx) {
    return up[(size_t)clampi(yy, 0, uh - 1) * uw + clampi(xx, 0, uw - 1)];
}
__device__ __forceinline__ int up_pred(const int16_t* up, int uw, int uh, int p, int x, int y, int mx, int my) {
    if (p == 1) return up_at(up, uw, uh, 2 * y + my, 2 * x + mx);
    if (p == 2) {
        const int rx = mx & 1, ry = my & 1;
        const int bx = 2 * x + (mx >> 1), by = 2 * y + (my >> 1);
        return ((2 - rx) * (2 - ry) * up_at(up, uw, uh, by, bx) + rx * (2 - ry) * up_at(up, uw, uh, by, bx + 1) +
                (2 - rx) * ry * up_at(up, uw, uh, by + 1, bx) + rx * ry * up_at(up, uw, uh, by + 1, bx + 1) + 2) >> 2;
    }
    const int rx = mx & 3, ry = my & 3;
    const int bx = 2 * x + (mx >> 2), by = 2 * y + (my >> 2);
    return ((4 - rx) * (4 - ry) * up_at(up, uw, uh, by, bx) + rx * (4 - ry) * up_at(up, uw, uh, by, bx + 1) +
            (4 - rx) * ry * up_at(up, uw, uh, by + 1, bx) + rx * ry * up_at(up, uw, uh, by + 1, bx + 1) + 8) >> 4;
}

// Float sum, in raster order from start, of |pred - pic| over a block: the cost loop of
// BlockDiff{Half,Quarter,Eighth}Pel::Diff.  Returns the reference's float result.  Eight
// steps (256 pixels) are loaded at once; when their total cannot make any addition round,
// the whole chunk is added in one go, otherwise step by step in raster order.
// The per-precision bodies are templates; the entry points are kept out of line, so that
// the wavefront kernels hold one copy of each (their instruction footprint, not their
// arithmetic, limited them).
// Whether every sample up_pred reads for the block at vector (mx, my), precision P, lies in
// the uw x uh plane (then no coordinate needs clamping); and the block's prediction as the
// offset of its first sample's base position and four bilinear weights.
template <int P>
struct UpFast {
    int ox, oy, w00, w01, w10, w11;
    bool inside;
    __device__ __forceinline__ UpFast(const Blim& b, int uw, int uh, int mx, int my) {
        int span;
        if (P == 1) {
            ox = mx;
            oy = my;
            w00 = 1;
            w01 = w10 = w11 = 0;
            span = 0;
        } else {
            constexpr int M = P == 2 ? 1 : 3, SH = P == 2 ? 1 : 2, ONE = M + 1;
            const int rx = mx & M, ry = my & M;
            ox = mx >> SH;
            oy = my >> SH;
            w00 = (ONE - rx) * (ONE - ry);
            w01 = rx * (ONE - ry);
            w10 = (ONE - rx) * ry;
            w11 = rx * ry;
            span = 1;
        }
        inside = 2 * b.xp + ox >= 0 && 2 * (b.xp + b.xl - 1) + ox + span <= uw - 1 && 2 * b.yp + oy >= 0 &&
                 2 * (b.yp + b.yl - 1) + oy + span <= uh - 1;
    }
    // up_pred at sample (x, y) when inside
    __device__ __forceinline__ int at(const int16_t* up, int uw, int x, int y) const {
        const int16_t* q = up + (size_t)(2 * y + oy) * uw + 2 * x + ox;
        if (P == 1) return q[0];
        constexpr int RND = P == 2 ? 2 : 8, OUT = P == 2 ? 2 : 4;
        return (w00 * q[0] + w01 * q[1] + w10 * q[uw] + w11 * q[uw + 1] + RND) >> OUT;
    }
};

template <int P>
__device__ __forceinline__ float subpel_cost_p(const int16_t* pic, int pw, const int16_t* up, int uw, int uh,
                                               const Blim& b, int mx, int my, float start) {
    const int lane = threadIdx.x & 31;
    FloatSeq f = float_seq_start(start);
    const int n = b.xl * b.yl;
    const UpFast<P> fast(b, uw, uh, mx, my);
    PixWalk w(b.xl);
    for (int k0 = 0; k0 < n; k0 += 256) {
        int d[8];
        int tot = 0;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            d[s] = 0;
            if (k0 + 32 * s + lane < n) {
                const int x = b.xp + w.col, y = b.yp + w.row;
                const int pr = fast.inside ? fast.at(up, uw, x, y) : up_pred(up, uw, uh, P, x, y, mx, my);
                d[s] = abs(pr - pic[(size_t)y * pw + x]);
            }
            tot += d[s];
            w.next();
        }
        tot = __reduce_add_sync(0xffffffffu, tot);
        if (!float_seq_add_exact(f, tot)) {
#pragma unroll
            for (int s = 0; s < 8; ++s) float_seq_add(f, d[s]);
        }
    }
    return (float)f.c;
}

__device__ __noinline__ float subpel_cost(const int16_t* pic, int pw, const int16_t* up, int uw, int uh, int p,
                                          const Blim& b, int mx, int my, float start) {
    if (b.xl <= 0 || b.yl <= 0) return start;
    if (p == 1) return subpel_cost_p<1>(pic, pw, up, uw, uh, b, mx, my, start);
    if (p == 2) return subpel_cost_p<2>(pic, pw, up, uw, uh, b, mx, my, start);
    return subpel_cost_p<3>(pic, pw, up, uw, uh, b, mx, my, start);
}

// Integer total of |pred - pic| over a block for one candidate (the terms the cost loop adds),
// over the block's pixels [kb, ke) in raster order (kb a multiple of 32; integer, so a block's
// total may be split between warps).
template <int P>
__device__ __forceinline__ int subpel_total_p(const int16_t* pic, int pw, const int16_t* up, int uw, int uh,
                                              const Blim& b, int mx, int my, int kb, int ke) {
    const int lane = threadIdx.x & 31;
    const int n = ke;
    const UpFast<P> fast(b, uw, uh, mx, my);
    PixWalk w(b.xl, kb);
    int tot = 0;
    if (fast.inside) {
        for (int k0 = kb; k0 < n; k0 += 256) {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (k0 + 32 * s + lane < n) {
                    const int x = b.xp + w.col, y = b.yp + w.row;
                    tot += abs(fast.at(up, uw, x, y) - pic[(size_t)y * pw + x]);
                }
                w.next();
            }
        }
        return __reduce_add_sync(0xffffffffu, tot);
    }
    for (int k0 = kb; k0 < n; k0 += 256) {
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            if (k0 + 32 * s + lane < n) {
                const int x = b.xp + w.col, y = b.yp + w.row;
                tot += abs(up_pred(up, uw, uh, P, x, y, mx, my) - pic[(size_t)y * pw + x]);
            }
            w.next();
        }
    }
    return __reduce_add_sync(0xffffffffu, tot);
}

__device__ __noinline__ int subpel_total(const int16_t* pic, int pw, const int16_t* up, int uw, int uh, int p,
                                         const Blim& b, int mx, int my, int kb = 0, int ke = -1) {
    if (b.xl <= 0 || b.yl <= 0) return 0;
    if (ke < 0) ke = b.xl * b.yl;
    if (ke <= kb) return 0;
    if (p == 1) return subpel_total_p<1>(pic, pw, up, uw, uh, b, mx, my, kb, ke);
    if (p == 2) return subpel_total_p<2>(pic, pw, up, uw, uh, b, mx, my, kb, ke);
    return subpel_total_p<3>(pic, pw, up, uw, uh, b, mx, my, kb, ke);
}

// Copies the h x w region at (x0, y0) of a pw x ph plane into shared memory (rows of w),
// coordinates clamped to the plane; each lane keeps eight loads in flight before storing.
__device__ __forceinline__ void stage_rect(int16_t* dst, const int16_t* __restrict__ src, int pw, int ph, int x0,
                                           int y0, int w, int h) {
    const int lane = threadIdx.x & 31;
    const int n = w * h;
    if (n <= 0) return;
    // this lane's element i = 32 k + lane sits at row r, column c; both advance by fixed
    // steps per 32 elements, so no division per element
    int r = lane / w, c = lane - r * w;
    const int dr = 32 / w, dc = 32 - dr * w;
    for (int i0 = 0; i0 < n; i0 += 256) {
        int16_t v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int i = i0 + 32 * k + lane;
            v[k] = 0;
            if (i < n)
                v[k] = __ldg(&src[(size_t)clampi(y0 + r, 0, ph - 1) * pw + clampi(x0 + c, 0, pw - 1)]);
            c += dc;
            r += dr;
            if (c >= w) {
                c -= w;
                ++r;
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int i = i0 + 32 * k + lane;
            if (i < n) dst[i] = v[k];
        }
    }
}

// A block staged in shared memory for the sub-pel search around its pel vector (mvx, mvy):
// the block's picture samples and the upconverted reference window that every candidate
// within +-((2 + SUB_EXTRA) 2^(prec-1) - 1) of (mvx, mvy) << prec reads (prec 1..3: the
// refinement's own candidates, within +-(2^prec - 1), and most predictors): up rows
// 2 (yp + mvy) - 2 - SUB_EXTRA .. 2 (yp + yl + mvy) + SUB_EXTRA and the same columns, each
// coordinate clamped to the array as up_at does, so reads need no clamping.  The staged
// columns start at the 8-sample boundary at or below the first one (16-byte loads) and a
// row holds sub_win_pitch(xl) samples, a pitch of 16 words modulo 32 so that the two
// half-warps of the fused passes (two block rows, two window rows apart) use disjoint banks.
constexpr int SUB_EXTRA = 2;

__host__ __device__ constexpr int sub_win_pitch(int xl) {
    // at least 2 xl + 3 + 2 SUB_EXTRA columns plus up to 7 of alignment, = 16 modulo 32
    return ((2 * xl + 3 + 2 * SUB_EXTRA + 7) + 15) / 32 * 32 + 16;
}

struct SubWin {
    int16_t* pic;  // xl * yl, raster order
    int16_t* up;   // (2 yl + 3 + 2 SUB_EXTRA) rows of ww samples
    int ww, wx0, wy0;
};

template <int P>
__device__ __forceinline__ int win_pred(const SubWin& S, int x, int y, int mx, int my) {
    if (P == 1) return S.up[(2 * y + my - S.wy0) * S.ww + 2 * x + mx - S.wx0];
    if (P == 2) {
        const int rx = mx & 1, ry = my & 1;
        const int16_t* q = S.up + (2 * y + (my >> 1) - S.wy0) * S.ww + 2 * x + (mx >> 1) - S.wx0;
        return ((2 - rx) * (2 - ry) * q[0] + rx * (2 - ry) * q[1] + (2 - rx) * ry * q[S.ww] + rx * ry * q[S.ww + 1] +
                2) >> 2;
    }
    const int rx = mx & 3, ry = my & 3;
    const int16_t* q = S.up + (2 * y + (my >> 2) - S.wy0) * S.ww + 2 * x + (mx >> 2) - S.wx0;
    return ((4 - rx) * (4 - ry) * q[0] + rx * (4 - ry) * q[1] + (4 - rx) * ry * q[S.ww] + rx * ry * q[S.ww + 1] + 8) >>
           4;
}

__device__ __noinline__ void stage_subwin(SubWin& S, int16_t* mem, const int16_t* pic, int pw, const int16_t* up, int uw, int uh,
                             const Blim& b, short2 mv) {
    const int lane = threadIdx.x & 31;
    S.pic = mem;
    S.up = mem + ((b.xl * b.yl + 7) & ~7);
    S.ww = sub_win_pitch(b.xl);
    S.wx0 = (2 * (b.xp + mv.x) - 2 - SUB_EXTRA) & ~7;
    S.wy0 = 2 * (b.yp + mv.y) - 2 - SUB_EXTRA;
    const int wh = 2 * b.yl + 3 + 2 * SUB_EXTRA;
    stage_rect(S.pic, pic, pw, 1 << 30, b.xp, b.yp, b.xl, b.yl);
    const bool aligned = (uw & 7) == 0 && (reinterpret_cast<uintptr_t>(up) & 15) == 0;
    if (aligned && S.wx0 >= 0 && S.wx0 + S.ww <= uw && S.wy0 >= 0 && S.wy0 + wh <= uh) {
        // the window lies inside the plane: 16-byte loads, four per lane in flight
        const int per_row = S.ww >> 3, n = per_row * wh;
        for (int i0 = 0; i0 < n; i0 += 128) {
            int4 v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int i = i0 + 32 * k + lane;
                if (i < n) {
                    const int r = i / per_row, c = i - r * per_row;
                    v[k] = __ldg(reinterpret_cast<const int4*>(up + (size_t)(S.wy0 + r) * uw + S.wx0) + c);
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int i = i0 + 32 * k + lane;
                if (i < n) reinterpret_cast<int4*>(S.up)[i] = v[k];
            }
        }
    } else {
        for (int r = 0; r < wh; ++r)
            for (int c = lane; c < S.ww; c += 32)
                S.up[r * S.ww + c] = __ldg(&up[(size_t)clampi(S.wy0 + r, 0, uh - 1) * uw + clampi(S.wx0 + c, 0, uw - 1)]);
    }
    __syncwarp();
}

// subpel_cost over a staged block (same arithmetic and order).
template <int P>
__device__ __forceinline__ float subpel_cost_win_p(const SubWin& S, const Blim& b, int mx, int my, float start) {
    const int lane = threadIdx.x & 31;
    FloatSeq f = float_seq_start(start);
    const int n = b.xl * b.yl;
    PixWalk w(b.xl);
    for (int k0 = 0; k0 < n; k0 += 256) {
        int d[8];
        int tot = 0;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            d[s] = 0;
            const int k = k0 + 32 * s + lane;
            if (k < n) d[s] = abs(win_pred<P>(S, b.xp + w.col, b.yp + w.row, mx, my) - S.pic[k]);
            tot += d[s];
            w.next();
        }
        tot = __reduce_add_sync(0xffffffffu, tot);
        if (!float_seq_add_exact(f, tot)) {
#pragma unroll
            for (int s = 0; s < 8; ++s) float_seq_add(f, d[s]);
        }
    }
    return (float)f.c;
}

__device__ __noinline__ float subpel_cost_win(const SubWin S, int p, const Blim b, int mx, int my, float start) {
    if (p == 1) return subpel_cost_win_p<1>(S, b, mx, my, start);
    if (p == 2) return subpel_cost_win_p<2>(S, b, mx, my, start);
    return subpel_cost_win_p<3>(S, b, mx, my, start);
}

// Integer totals of |pred - pic| over a staged block for the eight neighbours
// (cx + dx, cy + dy), dx, dy in {-1, 0, 1}, of a centre at precision P, all in one pass over
// the block: P = 1, the half-pel neighbours of a pel position (each prediction a window
// sample); P = 2, the quarter-pel neighbours of a half-pel position (cx, cy even: each
// prediction the rounded mean of two or four samples of the centre's 3 x 3 window
// neighbourhood, which is what win_pred<2> computes for those offsets).  Lane k returns the
// total of neighbour k = (dy + 1) * 3 + dx + 1 (lane 4, the centre: 0).
template <int P>
__device__ __forceinline__ int neighbour_totals(const SubWin S, const Blim& b, int cx, int cy) {
    const int lane = threadIdx.x & 31;
    const int n = b.xl * b.yl;
    const int ww = S.ww;
    const int ox = (P == 1 ? cx : cx >> 1) - S.wx0, oy = (P == 1 ? cy : cy >> 1) - S.wy0;
    PixWalk w(b.xl);
    int t0 = 0, t1 = 0, t2 = 0, t3 = 0, t5 = 0, t6 = 0, t7 = 0, t8 = 0;
#pragma unroll 4
    for (int k = lane; k < n; k += 32) {
        const int16_t* q = S.up + (2 * (b.yp + w.row) + oy) * ww + 2 * (b.xp + w.col) + ox;
        const int p = S.pic[k];
        const int a = q[-ww - 1], bb = q[-ww], c = q[-ww + 1], d = q[-1], f = q[1], g = q[ww - 1], h = q[ww],
                  i = q[ww + 1];
        if (P == 1) {
            t0 += abs(a - p);
            t1 += abs(bb - p);
            t2 += abs(c - p);
            t3 += abs(d - p);
            t5 += abs(f - p);
            t6 += abs(g - p);
            t7 += abs(h - p);
            t8 += abs(i - p);
        } else {
            const int e = q[0];
            t0 += abs(((a + bb + d + e + 2) >> 2) - p);
            t1 += abs(((bb + e + 1) >> 1) - p);
            t2 += abs(((bb + c + e + f + 2) >> 2) - p);
            t3 += abs(((d + e + 1) >> 1) - p);
            t5 += abs(((e + f + 1) >> 1) - p);
            t6 += abs(((d + e + g + h + 2) >> 2) - p);
            t7 += abs(((e + h + 1) >> 1) - p);
            t8 += abs(((e + f + h + i + 2) >> 2) - p);
        }
        w.next();
    }
    int mine = 0;
    const int r0 = __reduce_add_sync(0xffffffffu, t0), r1 = __reduce_add_sync(0xffffffffu, t1),
              r2 = __reduce_add_sync(0xffffffffu, t2), r3 = __reduce_add_sync(0xffffffffu, t3),
              r5 = __reduce_add_sync(0xffffffffu, t5), r6 = __reduce_add_sync(0xffffffffu, t6),
              r7 = __reduce_add_sync(0xffffffffu, t7), r8 = __reduce_add_sync(0xffffffffu, t8);
    mine = lane == 0 ? r0 : lane == 1 ? r1 : lane == 2 ? r2 : lane == 3 ? r3 : lane == 5 ? r5 : lane == 6 ? r6
         : lane == 7 ? r7 : lane == 8 ? r8 : 0;
    return mine;
}

__device__ __noinline__ int half_pel_totals(const SubWin S, const Blim b, short2 mv) {
    return neighbour_totals<1>(S, b, 2 * mv.x, 2 * mv.y);
}

__device__ __noinline__ int quarter_pel_totals(const SubWin S, const Blim b, short2 c) {
    return neighbour_totals<2>(S, b, c.x, c.y);
}

// BiBlock*Pel::Diff (me_utils.cpp:1172-1785): |((2 pic - p1) - p2) >> 1| with int16
// intermediates, summed in float from 0 (exact: integer sums below 2^24).  The eighth-pel
// version walks the second reference from the first one's integer start position when the
// second one needs bounds checking (me_utils.cpp:1764-1768); reproduced here.
__device__ __noinline__ int bi_sad_range(const int16_t* pic, int pw, const int16_t* up1, const int16_t* up2, int uw, int uh,
                            int p, const Blim& b, short2 mv1, short2 mv2, int kb, int ke);

__device__ float bi_cost(const int16_t* pic, int pw, const int16_t* up1, const int16_t* up2, int uw, int uh, int p,
                         const Blim& b, short2 mv1, short2 mv2) {
    if (b.xl <= 0 || b.yl <= 0) return 0.0f;
    return (float)bi_sad_range(pic, pw, up1, up2, uw, uh, p, b, mv1, mv2, 0, b.xl * b.yl);
}

// Pixels [kb, ke) (raster order) of the bi-prediction SAD; integer, so it splits freely.
__device__ __noinline__ int bi_sad_range(const int16_t* pic, int pw, const int16_t* up1, const int16_t* up2, int uw, int uh,
                            int p, const Blim& b, short2 mv1, short2 mv2, int kb, int ke) {
    if (b.xl <= 0 || b.yl <= 0 || ke <= kb) return 0;
    int m2x = mv2.x, m2y = mv2.y;
    if (p == 3) {
        const int sx = (b.xp << 1) + (mv2.x >> 2), sy = (b.yp << 1) + (mv2.y >> 2);
        if (sx < 0 || sx + (b.xl << 1) >= uw || sy < 0 || sy + (b.yl << 1) >= uh) {
            m2x = ((mv1.x >> 2) << 2) | (mv2.x & 3);
            m2y = ((mv1.y >> 2) << 2) | (mv2.y & 3);
        }
    }
    const int lane = threadIdx.x & 31;
    PixWalk w(b.xl, kb);
    int s = 0;
    if (p == 2) {
        // quarter-pel with both predictions inside their planes: no clamping
        const UpFast<2> f1(b, uw, uh, mv1.x, mv1.y), f2(b, uw, uh, m2x, m2y);
        if (f1.inside && f2.inside) {
#pragma unroll 4
            for (int k = kb + lane; k < ke; k += 32) {
                const int x = b.xp + w.col, y = b.yp + w.row;
                const int16_t dd = (int16_t)((pic[(size_t)y * pw + x] << 1) - f1.at(up1, uw, x, y));
                const int16_t t = (int16_t)((dd - f2.at(up2, uw, x, y)) >> 1);
                s += abs((int)t);
                w.next();
            }
            return __reduce_add_sync(0xffffffffu, s);
        }
    }
#pragma unroll 4
    for (int k = kb + lane; k < ke; k += 32) {
        const int x = b.xp + w.col, y = b.yp + w.row;
        const int16_t dd = (int16_t)((pic[(size_t)y * pw + x] << 1) - up_pred(up1, uw, uh, p, x, y, mv1.x, mv1.y));
        const int16_t t = (int16_t)((dd - up_pred(up2, uw, uh, p, x, y, m2x, m2y)) >> 1);
        s += abs((int)t);
        w.next();
    }
    return __reduce_add_sync(0xffffffffu, s);
}

// IntraBlockDiff::CalcDC and ::Diff (me_utils.cpp:284-408): truncating mean, SAD against it.
__device__ int block_dc(const int16_t* pic, int pw, const Blim& b) {
    if (b.xl <= 0 || b.yl <= 0) return 0;
    const int lane = threadIdx.x & 31;
    const int n = b.xl * b.yl;
    PixWalk w(b.xl);
    int s = 0;
#pragma unroll 8
    for (int k = lane; k < n; k += 32) {
        s += pic[(size_t)(b.yp + w.row) * pw + b.xp + w.col];
        w.next();
    }
    s = __reduce_add_sync(0xffffffffu, s);
    return (int)(int16_t)(s / n);
}

__device__ __noinline__ float intra_cost(const int16_t* pic, int pw, const Blim& b, int16_t& dc) {
    if (b.xl <= 0 || b.yl <= 0) {
        dc = 0;
        return 0.0f;
    }
    dc = (int16_t)block_dc(pic, pw, b);
    const int lane = threadIdx.x & 31;
    const int n = b.xl * b.yl;
    PixWalk w(b.xl);
    int s = 0;
#pragma unroll 8
    for (int k = lane; k < n; k += 32) {
        s += abs(pic[(size_t)(b.yp + w.row) * pw + b.xp + w.col] - dc);
        w.next();
    }
    return (float)__reduce_add_sync(0xffffffffu, s);
}

// ============================================================================================
// Pel search (pixel_match.cpp)
// ============================================================================================

struct PelJob {
    const int16_t* pic;     // this level's picture plane (dense, pw x ph)
    const int16_t* ref;     // this level's reference plane
    int pw, ph;
    int xnb, ynb;           // block grid of this level
    short2* mv;             // vectors of this level (output)
    float* cost;            // (SAD, mvcost, total) per block (output)
    const short2* guide;    // vectors of the coarser level, or null at the coarsest
    int gxnb, gynb;
    int radius;             // min(level + 1, 5)
    int* best_sad;          // zero + guide lists: best SAD (INT_MAX if the block is empty)
    short2* best_mv;
    int* flags;             // completion flags of the wavefront
};

// All jobs of a launch share one block grid (xnb x ynb = per_job units).
struct PelLaunch {
    int total, per_job;
    int win_elems;          // int16 elements of shared memory per warp (block + search window)
    Olb o;
    int* ticket;
    int* err;
    const PelJob* jobs;     // device table
    Wave wave;
    WaveDebug dbg;
};

// Best candidate of one list (BlockMatcher::FindBestMatchPel over the list, PelBlockDiff::Diff
// per candidate): the block and the reference window the list covers (coordinates clamped as
// BChk does) are copied to the warp's shared memory, then groups of G lanes each take one
// candidate (G = the largest power of two with 2 G n <= 32, so small lists still use most
// lanes).  The list's minimum with the earliest index replaces (best, bmv) only when strictly
// smaller: the same result as the reference's sequential strict-< scan.
// Earlier lists: the square of radius r around each of n centres (AddVect drops a candidate
// already listed, block_match.cpp:170-190).
struct SeenLists {
    short2 c[2];
    int n;
    __device__ __forceinline__ bool has(short2 v, int r) const {
        for (int k = 0; k < n; ++k)
            if (abs(v.x - c[k].x) <= r && abs(v.y - c[k].y) <= r) return true;
        return false;
    }
};

__device__ __noinline__ void pel_list_best(const int16_t* pic, const int16_t* ref, int pw, int ph, const Blim& b, short2 centre,
                              int r, int16_t* mem, int& best, short2& bmv, bool blk_staged = false,
                              SeenLists seen = SeenLists{{}, 0}, unsigned long long* ops = nullptr) {
    const int lane = threadIdx.x & 31;
    const int n_all = (2 * r + 1) * (2 * r + 1);
    if (seen.n) {
        // a list wholly inside the earlier lists adds no candidate: nothing to stage or sum
        bool fresh = false;
        for (int k = lane; k < n_all; k += 32) fresh |= !seen.has(cand_at(centre, r, k), r);
        if (!__any_sync(0xffffffffu, fresh)) return;
    }
    if (ops) {
        int fresh = 0;
        for (int k = lane; k < n_all; k += 32) fresh += !(seen.n && seen.has(cand_at(centre, r, k), r));
        count_ops(ops, 3LL * __reduce_add_sync(0xffffffffu, fresh) * b.xl * b.yl);
    }
    const int ww = b.xl + 2 * r, wh = b.yl + 2 * r;
    int16_t* blk = mem;
    int16_t* win = mem + b.xl * b.yl;
    if (!blk_staged) stage_rect(blk, pic, pw, ph, b.xp, b.yp, b.xl, b.yl);
    stage_rect(win, ref, pw, ph, b.xp + centre.x - r, b.yp + centre.y - r, ww, wh);
    __syncwarp();
    const int n = (2 * r + 1) * (2 * r + 1);
    // G lanes per candidate, each summing every G-th row: as many lanes busy as the list
    // allows (9 candidates: 27 lanes)
    const int G = n >= 32 ? 1 : 32 / n;
    const int per_round = 32 / G;
    const int grp = lane / G, g = lane - grp * G;
    int my_best = INT_MAX, my_k = INT_MAX;
    for (int k0 = 0; k0 < n; k0 += per_round) {
        const int k = k0 + grp;
        int sad = 0;
        bool dup = false;
        if (k < n && grp < per_round) {
            const short2 c = cand_at(centre, r, k);
            dup = seen.n && seen.has(c, r);
        }
        if (k < n && grp < per_round && !dup) {
            const short2 c = cand_at(centre, r, k);
            const int dx = c.x - centre.x + r, dy = c.y - centre.y + r;
            for (int y = g; y < b.yl; y += G) {
                const int16_t* pr = blk + y * b.xl;
                const int16_t* wr = win + (y + dy) * ww + dx;
#pragma unroll 4
                for (int x = 0; x < b.xl; ++x) sad += abs((int)(int16_t)(pr[x] - wr[x]));
            }
        }
        // the group's leader (g == 0) gathers its G - 1 partners, which sit just above it
        int tot = sad;
        for (int o = 1; o < G; ++o) {
            const int v = __shfl_down_sync(0xffffffffu, sad, o);
            tot += v;
        }
        sad = tot;
        if (k < n && grp < per_round && !dup && g == 0 && sad < my_best) {
            my_best = sad;
            my_k = k;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int ob = __shfl_xor_sync(0xffffffffu, my_best, o);
        const int ok = __shfl_xor_sync(0xffffffffu, my_k, o);
        if (ob < my_best || (ob == my_best && ok < my_k)) {
            my_best = ob;
            my_k = ok;
        }
    }
    if (my_best < best) {
        best = my_best;
        bmv = cand_at(centre, r, my_k);
    }
    __syncwarp();
}

// Parallel phase: the zero-centred and the guide-centred lists of every block.
__global__ void __launch_bounds__(ME_THREADS) pel_lists_kernel(const __grid_constant__ PelLaunch L) {
    extern __shared__ __align__(16) int16_t pel_smem[];
    int16_t* const wmem = pel_smem + (size_t)(threadIdx.x >> 5) * L.win_elems;
    const int u = blockIdx.x * WARPS_PER_CTA + (threadIdx.x >> 5);
    if (u >= L.total) return;
    const int jn = u / L.per_job;
    const PelJob& J = L.jobs[jn];
    const int b = u - jn * L.per_job;
    const int by = b / J.xnb, bx = b - by * J.xnb;
    const Blim bl = block_limits(L.o, J.pw, J.ph, bx, by);
    int best = INT_MAX;
    short2 bmv = make_short2(0, 0);
    if (bl.xl > 0 && bl.yl > 0) {
        pel_list_best(J.pic, J.ref, J.pw, J.ph, bl, make_short2(0, 0), J.radius, wmem, best, bmv, false,
                      SeenLists{{}, 0}, L.dbg.ops);
        if (J.guide) {
            const int gx = clampi(bx >> 1, 0, J.gxnb - 1), gy = clampi(by >> 1, 0, J.gynb - 1);
            const short2 gv = J.guide[(size_t)gy * J.gxnb + gx];
            // candidates already in the zero-centred list are not listed again
            pel_list_best(J.pic, J.ref, J.pw, J.ph, bl, make_short2((short)(gv.x * 2), (short)(gv.y * 2)), J.radius,
                          wmem, best, bmv, true, SeenLists{{make_short2(0, 0), make_short2(0, 0)}, 1}, L.dbg.ops);
        }
    }
    if ((threadIdx.x & 31) == 0) {
        J.best_sad[b] = best;
        J.best_mv[b] = bmv;
    }
}

// Wavefront phase: raster predictor, predictor-centred list, final vectors and costs
// (PixelMatcher::MatchPic / DoBlock, BlockMatcher::FindBestMatchPel).
__global__ void __launch_bounds__(ME_THREADS) pel_wavefront_kernel(const __grid_constant__ PelLaunch L) {
    extern __shared__ __align__(16) int16_t pel_smem[];
    int16_t* const wmem = pel_smem + (size_t)(threadIdx.x >> 5) * L.win_elems;
    for (int it = 0; it < L.wave.life; ++it) {
        const int u = warp_ticket(L.ticket);
        if (u >= L.total) return;
        int jn, bx, by;
        wave_unit(L.wave, u, jn, bx, by);
        const PelJob& J = L.jobs[jn];
        const int W = J.xnb;
        const int b = by * W + bx;
        // the block's own samples do not depend on the neighbours: load them before waiting
        const Blim bl = block_limits(L.o, J.pw, J.ph, bx, by);
        if (bl.xl > 0 && bl.yl > 0) stage_rect(wmem, J.pic, J.pw, J.ph, bl.xp, bl.yp, bl.xl, bl.yl);
        if (bx > 0) wait_flag(&J.flags[b - 1], L.err, L.dbg.spin_limit);
        if (by > 0) {
            wait_flag(&J.flags[b - W], L.err, L.dbg.spin_limit);
            if (bx < W - 1) wait_flag(&J.flags[b - W + 1], L.err, L.dbg.spin_limit);
        }
        const short2* mv = J.mv;
        short2 pred = make_short2(0, 0);
        if (by == 0) {
            if (bx > 0) pred = __ldcg(&mv[b - 1]);
        } else if (bx == 0) {
            pred = __ldcg(&mv[b - W]);
        } else if (bx < W - 1) {
            pred = mv_median3(__ldcg(&mv[b - 1]), __ldcg(&mv[b - W]), __ldcg(&mv[b - W + 1]));
        } else {
            pred = mv_mean(__ldcg(&mv[b - W]), __ldcg(&mv[b - 1]));
        }
        int best = J.best_sad[b];
        short2 bmv = J.best_mv[b];
        float sad;
        if (bl.xl > 0 && bl.yl > 0) {
            // the zero- and guide-centred lists (pel_lists_kernel) came first
            SeenLists seen{{make_short2(0, 0), make_short2(0, 0)}, 1};
            if (J.guide) {
                const int gx = clampi(bx >> 1, 0, J.gxnb - 1), gy = clampi(by >> 1, 0, J.gynb - 1);
                const short2 gv = J.guide[(size_t)gy * J.gxnb + gx];
                seen.c[1] = make_short2((short)(gv.x * 2), (short)(gv.y * 2));
                seen.n = 2;
            }
            pel_list_best(J.pic, J.ref, J.pw, J.ph, bl, pred, J.radius, wmem, best, bmv, true, seen, L.dbg.ops);
            sad = (float)best;
        } else {
            bmv = make_short2(0, 0);
            sad = 10000000.0f;
        }
        if ((threadIdx.x & 31) == 0) {
            const float mvcost = (float)norm1(bmv.x - pred.x, bmv.y - pred.y);
            J.mv[b] = bmv;
            J.cost[3 * b] = sad;
            J.cost[3 * b + 1] = mvcost;
            J.cost[3 * b + 2] = sad + 0.0f * mvcost;
            audit_unit(L.dbg, jn, b);
            if (u != L.dbg.skip_unit) publish(&J.flags[b]);
        }
        __syncwarp();
    }
}

// ============================================================================================
// Sub-pel refinement (me_subpel.cpp:65-176, block_match.cpp:327-467)
// ============================================================================================

struct SubJob {
    const int16_t* pic;  // luma, pw x ph
    const int16_t* up;   // upconverted original reference, 2pw x 2ph
    int pw, ph, xnb, ynb;
    short2* mv;          // in: pel vectors; out: sub-pel vectors
    float* cost;         // (SAD, mvcost, total) per block, in and out
    const float* lambda; // lambda map
    int* flags;
};

struct SubLaunch {
    int total, prec;
    int win_elems;       // int16 elements of shared memory per warp for SubWin; 0: no staging
    Olb o;
    int* ticket;
    int* err;
    const SubJob* jobs;  // device table
    Wave wave;
    WaveDebug dbg;
};

struct Cost3 {
    float SAD, mvcost, total;
};

// One candidate of the refinement at precision i: from its integer total when the step's
// neighbour totals are known (fused) and no addition of the reference's loop could round,
// else from the staged window when there is one, else from global memory; (best, best_mv)
// updated on a strictly smaller total.
__device__ __forceinline__ void eval_subpel_cand(const SubJob& J, const SubWin& S, bool staged, bool fused,
                                                 int total, int i, int sh, const Blim& bl, short2 c, short2 pred,
                                                 float lambda, Cost3& best, short2& best_mv,
                                                 unsigned long long* ops) {
    const float mvcost = (float)getvarup(pred, c.x << sh, c.y << sh);
    if (bl.xl <= 0 || bl.yl <= 0) return;
    count_ops(ops, (long long)(3 + interp_ops(i)) * bl.xl * bl.yl);
    const float start = mvcost * lambda;
    float sum;
    FloatSeq f = float_seq_start(start);
    if (fused && float_seq_add_exact(f, total))
        sum = (float)f.c;
    else
        sum = staged ? subpel_cost_win(S, i, bl, c.x, c.y, start)
                     : subpel_cost(J.pic, J.pw, J.up, 2 * J.pw, 2 * J.ph, i, bl, c.x, c.y, start);
    if (sum < best.total) {
        best_mv = c;
        best.total = sum;
        best.mvcost = mvcost;
        best.SAD = sum - start;
    }
}

__global__ void __launch_bounds__(ME_THREADS, 4) subpel_wavefront_kernel(const __grid_constant__ SubLaunch L) {
    extern __shared__ __align__(16) int16_t sub_smem[];
    int16_t* const wmem = sub_smem + (size_t)(threadIdx.x >> 5) * L.win_elems;
    const int prec = L.prec;
    for (int it = 0; it < L.wave.life; ++it) {
        const int u = warp_ticket(L.ticket);
        if (u >= L.total) return;
        int jn, bx, by;
        wave_unit(L.wave, u, jn, bx, by);
        const SubJob& J = L.jobs[jn];
        const int W = J.xnb, H = J.ynb;
        const int b = by * W + bx;
        // Everything that depends only on this block comes before the neighbour waits: its
        // limits, pel vector and cost, and (when the full search is likely) the staged search
        // window, whose loads then overlap the wait instead of following it.
        const Blim bl = block_limits(L.o, J.pw, J.ph, bx, by);
        const short2 mv = J.mv[b];
        const float pel_sad = J.cost[3 * b];
        const float area2 = (float)(2 * bl.xl * bl.yl);
        const float lambda = J.lambda[b];
        const bool staged = L.win_elems > 0 && bl.xl > 0 && bl.yl > 0 && !(pel_sad < area2);
        SubWin S{};
        int half_tot = 0;  // lane k: total of half-pel neighbour k of the pel vector
        if (staged) {
            stage_subwin(S, wmem, J.pic, J.pw, J.up, 2 * J.pw, 2 * J.ph, bl, mv);
            // the first refinement step's candidates are all among these eight
            half_tot = half_pel_totals(S, bl, mv);
        }
        // neighbours in SubpelRefine::m_nshift order: left, top-left, top, top-right
        const int nsx[4] = {-1, -1, 0, 1}, nsy[4] = {0, -1, -1, -1};
        short2 nbr[4];
        int n = 0;
        const bool all = bx > 0 && by > 0 && bx < W - 1;
        for (int i = 0; i < 4; ++i) {
            const int x = bx + nsx[i], y = by + nsy[i];
            if (all || (x >= 0 && y >= 0 && x < W && y < H)) {
                wait_flag(&J.flags[y * W + x], L.err, L.dbg.spin_limit);
                nbr[n++] = __ldcg(&J.mv[y * W + x]);
            }
        }
        const short2 pred = mv_median_list(nbr, n);
        Cost3 cost{pel_sad, 0.0f, 0.0f};
        cost.mvcost = (float)getvarup(pred, mv.x << prec, mv.y << prec);
        cost.total = cost.SAD + lambda * cost.mvcost;
        short2 out_mv;
        Cost3 out_cost;
        if (cost.SAD < area2) {
            out_mv = make_short2((short)(mv.x << prec), (short)(mv.y << prec));
            out_cost = cost;
        } else {
            Cost3 pc{0.0f, 0.0f, 0.0f};
            // the predictor reads the staged window when it lies within the search range
            const int reach = (2 + SUB_EXTRA) * (1 << (prec - 1)) - 1;
            const bool pred_in_win = staged && abs(pred.x - (mv.x << prec)) <= reach &&
                                     abs(pred.y - (mv.y << prec)) <= reach;
            if (bl.xl > 0 && bl.yl > 0) count_ops(L.dbg.ops, (long long)(3 + interp_ops(prec)) * bl.xl * bl.yl);
            if (bl.xl <= 0 || bl.yl <= 0)
                pc.SAD = 0.0f;
            else if (pred_in_win)
                pc.SAD = subpel_cost_win(S, prec, bl, pred.x, pred.y, 0.0f);
            else
                pc.SAD = subpel_cost(J.pic, J.pw, J.up, 2 * J.pw, 2 * J.ph, prec, bl, pred.x, pred.y, 0.0f);
            pc.total = pc.SAD;
            if (pc.SAD < area2) {
                out_mv = pred;
                out_cost = pc;
            } else {
                Cost3 best = cost;
                short2 bmv = mv;
                bool bailed = false;
                // candidates stay within +-(2^prec - 1) of mv << prec: the window staged above
                for (int i = 1; i <= prec; ++i) {
                    bmv = make_short2((short)(bmv.x << 1), (short)(bmv.y << 1));
                    short2 tb = bmv;
                    const int sh = prec - i;
                    // every candidate of the step is one of bmv's eight neighbours: their
                    // integer totals in one pass (half-pel: computed before the waits)
                    const bool fused = staged && i <= 2;
                    const int step_tot = !fused ? 0 : i == 1 ? half_tot : quarter_pel_totals(S, bl, bmv);
                    // the four neighbours, then (after a move) the two across the move
                    int mx = 0, my = 0;  // the move of the first four (0, 0: none)
                    for (int q = 0; q < 6; ++q) {
                        int dx, dy;
                        if (q == 4) {
                            mx = tb.x - bmv.x;
                            my = tb.y - bmv.y;
                            if (mx == 0 && my == 0) break;
                        }
                        if (q < 4) {
                            dx = q == 0 ? -1 : q == 1 ? 1 : 0;
                            dy = q == 2 ? -1 : q == 3 ? 1 : 0;
                        } else if (mx != 0) {
                            dx = mx;
                            dy = q == 4 ? -1 : 1;
                        } else {
                            dx = q == 4 ? -1 : 1;
                            dy = my;
                        }
                        const int total = __shfl_sync(0xffffffffu, step_tot, (dy + 1) * 3 + dx + 1);
                        const short2 c = make_short2((short)(bmv.x + dx), (short)(bmv.y + dy));
                        eval_subpel_cand(J, S, staged, fused, total, i, sh, bl, c, pred, lambda, best, tb,
                                         L.dbg.ops);
                    }
                    bmv = tb;
                    if ((double)best.total > 1.1 * (double)pc.total) {
                        bailed = true;
                        break;
                    }
                }
                if (bailed) {
                    out_mv = pred;
                    out_cost = pc;
                } else {
                    out_mv = bmv;
                    out_cost = best;
                }
            }
        }
        if ((threadIdx.x & 31) == 0) {
            J.mv[b] = out_mv;
            J.cost[3 * b] = out_cost.SAD;
            J.cost[3 * b + 1] = out_cost.mvcost;
            J.cost[3 * b + 2] = out_cost.total;
            audit_unit(L.dbg, jn, b);
            publish(&J.flags[b]);
        }
        __syncwarp();
    }
}

// ============================================================================================
// Mode decision (me_mode_decn.cpp:66-537)
// ============================================================================================

// Data of one level (0 superblocks, 1 sub-superblocks, 2 blocks).
struct LevelData {
    int xnb, ynb;
    short2* mv[2];
    float* cost[2];     // (SAD, mvcost, total)
    uint8_t* mode;
    int16_t* dcy;       // DC of Y (level 2: the picture's DC(Y_COMP) array)
    const float* lambda;
};

struct ModeJob {
    const int16_t* pic;  // luma pw x ph
    const int16_t* up[2];
    int pw, ph;
    LevelData lev[3];
    float* sbcost;
    uint8_t* split;
    int xnsb, ynsb;
    int* flags;          // per superblock
    float* bcost;        // level-2 (block) decision costs, from mode_blocks_kernel
    int nref;            // references of this picture (1 or 2)
};

struct ModeLaunch {
    int total, prec;
    Olb lb[3];
    float level_factor[3];
    int* ticket;
    int* err;
    const ModeJob* jobs;  // device table
    Wave wave;
    WaveDebug dbg;
};

// ModeDecider::DoME: the unit's four guide vectors as candidates (BlockMatcher::FindBestMatchSubp).
// Candidate list of ModeDecider::DoME for unit (x, y) and reference r: the four guide
// vectors of the next finer level, duplicates dropped, in the reference's order.
__device__ __forceinline__ int dome_candidates(const ModeJob& J, int x, int y, int level, int r, short2* c) {
    const LevelData& guide = J.lev[level + 1];
    const int gx = x << 1, gy = y << 1;
    int nc = 0;
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            const short2 v = __ldcg(&guide.mv[r][(size_t)(gy + j) * guide.xnb + gx + i]);
            bool dup = false;
            for (int q = 0; q < nc; ++q) dup |= (c[q].x == v.x && c[q].y == v.y);
            if (!dup) c[nc++] = v;
        }
    return nc;
}

// Integer totals of every DoME candidate of unit (x, y), computed before the superblock's
// neighbours are done (the candidates do not depend on them; only the vector costs do).
__device__ __noinline__ void dome_totals(const ModeLaunch& L, const ModeJob& J, int x, int y, int level, int* tot) {
    const Blim bl = block_limits(L.lb[level], J.pw, J.ph, x, y);
    for (int r = 0; r < J.nref; ++r) {
        short2 c[4];
        const int nc = dome_candidates(J, x, y, level, r, c);
        for (int q = 0; q < nc; ++q) {
            const int t = subpel_total(J.pic, J.pw, J.up[r], 2 * J.pw, 2 * J.ph, L.prec, bl, c[q].x, c[q].y);
            if ((threadIdx.x & 31) == 0) tot[4 * r + q] = t;
        }
    }
    __syncwarp();
}

__device__ __noinline__ void do_me(const ModeLaunch& L, const ModeJob& J, int x, int y, int level,
                                   const int* pre_tot = nullptr) {
    const LevelData& me = J.lev[level];
    const LevelData& guide = J.lev[level + 1];
    const LevelData& blk = J.lev[2];
    const int gx = x << 1, gy = y << 1;
    const int xb = x << (2 - level), yb = y << (2 - level);
    const size_t k = (size_t)y * me.xnb + x;
    const float lambda = me.lambda[k];
    const Blim bl = block_limits(L.lb[level], J.pw, J.ph, x, y);
    for (int r = 0; r < J.nref; ++r) {
        short2 c[4];
        int nc = 0;
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 2; ++i) {
                const short2 v = __ldcg(&guide.mv[r][(size_t)(gy + j) * guide.xnb + gx + i]);
                bool dup = false;
                for (int q = 0; q < nc; ++q) dup |= (c[q].x == v.x && c[q].y == v.y);
                if (!dup) c[nc++] = v;
            }
        const short2* bv = blk.mv[r];
        const int W = blk.xnb;
        short2 pred = make_short2(0, 0);
        if (xb > 0 && yb > 0)
            pred = mv_median3(__ldcg(&bv[(size_t)yb * W + xb - 1]), __ldcg(&bv[(size_t)(yb - 1) * W + xb - 1]),
                              __ldcg(&bv[(size_t)(yb - 1) * W + xb]));
        else if (xb == 0 && yb > 0)
            pred = mv_mean(__ldcg(&bv[(size_t)(yb - 1) * W + xb]), __ldcg(&bv[(size_t)(yb - 1) * W + xb + 1]));
        else if (xb > 0 && yb == 0)
            pred = mv_mean(__ldcg(&bv[(size_t)yb * W + xb - 1]), __ldcg(&bv[(size_t)(yb + 1) * W + xb - 1]));
        Cost3 best{me.cost[r][3 * k], me.cost[r][3 * k + 1], 100000000.0f};
        short2 bmv = me.mv[r][k];
        if (bl.xl > 0 && bl.yl > 0)
            count_ops(L.dbg.ops, (long long)nc * (3 + interp_ops(L.prec)) * bl.xl * bl.yl);
        for (int q = 0; q < nc; ++q) {
            if (bl.xl <= 0 || bl.yl <= 0) break;
            const float mvcost = (float)getvarup(pred, c[q].x, c[q].y);
            const float start = mvcost * lambda;
            float sum;
            FloatSeq f = float_seq_start(start);
            if (pre_tot && float_seq_add_exact(f, pre_tot[4 * r + q]))
                sum = (float)f.c;  // no addition of the loop could round
            else
                sum = subpel_cost(J.pic, J.pw, J.up[r], 2 * J.pw, 2 * J.ph, L.prec, bl, c[q].x, c[q].y, start);
            if (sum < best.total) {
                bmv = c[q];
                best.total = sum;
                best.mvcost = mvcost;
                best.SAD = sum - start;
            }
        }
        if ((threadIdx.x & 31) == 0) {
            me.mv[r][k] = bmv;
            me.cost[r][3 * k] = best.SAD;
            me.cost[r][3 * k + 1] = best.mvcost;
            me.cost[r][3 * k + 2] = best.total;
        }
        __syncwarp();
    }
}

// ModeDecider::DoUnitDecn: best of REF1 / REF2 / bi-prediction / intra for one unit.
__device__ __noinline__ float do_unit_decn(const ModeLaunch& L, const ModeJob& J, int x, int y, int level, float bsad_in = -1.0f) {
    const LevelData& me = J.lev[level];
    const size_t k = (size_t)y * me.xnb + x;
    const float lambda = me.lambda[k];
    const float mode_cost = 0.0f;
    const float f = L.level_factor[level];
    const Blim bl = block_limits(L.lb[level], J.pw, J.ph, x, y);
    int mode = 1;
    const float t1 = __ldcg(&me.cost[0][3 * k + 2]) * f;
    float min_cost = t1 + mode_cost;
    float best_sad = __ldcg(&me.cost[0][3 * k]);
    float t2 = 0.0f;
    if (J.nref > 1) {
        t2 = __ldcg(&me.cost[1][3 * k + 2]) * f;
        float unit = t2 + mode_cost;
        if (unit < min_cost) {
            mode = 2;
            min_cost = unit;
            best_sad = __ldcg(&me.cost[1][3 * k]);
        }
        const float bmvcost = __ldcg(&me.cost[0][3 * k + 1]) + __ldcg(&me.cost[1][3 * k + 1]);
        // the bi-prediction difference: two predictions, 2 pic - p1 - p2, halve, absolute value, add
        if (bl.xl > 0 && bl.yl > 0)
            count_ops(L.dbg.ops, (long long)(5 + 2 * interp_ops(L.prec)) * bl.xl * bl.yl);
        const float bsad = bsad_in >= 0.0f ? bsad_in
                                           : bi_cost(J.pic, J.pw, J.up[0], J.up[1], 2 * J.pw, 2 * J.ph, L.prec, bl,
                                                     __ldcg(&me.mv[0][k]), __ldcg(&me.mv[1][k]));
        float btotal = bsad + lambda * bmvcost;
        btotal *= f;
        unit = btotal + mode_cost;
        if (unit < min_cost) {
            mode = 3;
            min_cost = unit;
            best_sad = bsad;
        }
    }
    int16_t dc = 0;
    bool set_dc = false;
    if (level == 2 && (double)best_sad > 4.0 * L.lb[level].xblen * L.lb[level].yblen) {
        float ic = intra_cost(J.pic, J.pw, bl, dc);
        count_ops(L.dbg.ops, 4LL * bl.xl * bl.yl);  // the DC sum, then subtract, absolute value, add
        set_dc = true;
        ic *= f;
        const float unit = ic + mode_cost;
        if (unit < min_cost && (double)ic < 0.85 * (double)best_sad) {
            mode = 0;
            min_cost = unit;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        me.cost[0][3 * k + 2] = t1;
        if (J.nref > 1) me.cost[1][3 * k + 2] = t2;
        me.mode[k] = (uint8_t)mode;
        if (set_dc) me.dcy[k] = dc;
    }
    __syncwarp();
    return min_cost;
}

// Writes the decisions of one level's units over the superblock's 16 blocks
// (ModeDecider::DoLevelDecn's propagation) and the superblock's split and cost.  Called by a
// whole warp: lanes 0-15 take one block each; the fence makes the writes visible device-wide
// before the CTA barrier that precedes thread 0's release of the superblock's flag.
__device__ void propagate_level(const ModeLaunch& L, const ModeJob& J, int xsb, int ysb, int level, float sb_cost) {
    const LevelData& lv = J.lev[level];
    const LevelData& bl = J.lev[2];
    const int span = 1 << (2 - level);
    const int t = threadIdx.x & 31;
    if (t < 16) {
        const int v = (ysb << 2) + (t >> 2), u = (xsb << 2) + (t & 3);
        const int j = v / span, i = u / span;
        const size_t src = (size_t)j * lv.xnb + i, dst = (size_t)v * bl.xnb + u;
        bl.mode[dst] = __ldcg(&lv.mode[src]);
        bl.dcy[dst] = __ldcg(&lv.dcy[src]);
        bl.mv[0][dst] = __ldcg(&lv.mv[0][src]);
        if (J.nref > 1) bl.mv[1][dst] = __ldcg(&lv.mv[1][src]);
    }
    if (t == 0) {
        const size_t sb = (size_t)ysb * J.xnsb + xsb;
        J.sbcost[sb] = sb_cost;
        J.split[sb] = (uint8_t)level;
    }
    __threadfence();
    __syncwarp();
}

// Level-2 decisions (every block: REF1 / REF2 / bi / intra) depend on nothing outside the block,
// so they run for all blocks of all jobs before the superblock wavefront.  One warp per block;
// the unit cost goes to bcost for the superblock sums.
__global__ void __launch_bounds__(ME_THREADS) mode_blocks_kernel(const __grid_constant__ ModeLaunch L, int per_job) {
    const int u = blockIdx.x * WARPS_PER_CTA + (threadIdx.x >> 5);
    if (u >= L.total) return;
    const int jn = u / per_job;
    const ModeJob& J = L.jobs[jn];
    const int k = u - jn * per_job;
    const int xnb = J.lev[2].xnb;
    const int y = k / xnb, x = k - y * xnb;
    const float c = do_unit_decn(L, J, x, y, 2);
    if ((threadIdx.x & 31) == 0) J.bcost[k] = c;
}

// Superblock wavefront (ModeDecider::DoModeDecn per superblock): one CTA of WARPS_PER_CTA
// warps per superblock.  Level 2 sums the precomputed block costs; level 1 gives one
// sub-superblock to each warp; level 0 spreads its motion-search candidates and the
// bi-prediction SAD over the warps.  Float sums keep the reference's order.
__global__ void __launch_bounds__(ME_THREADS, 5) mode_wavefront_kernel(const __grid_constant__ ModeLaunch L) {
    static_assert(WARPS_PER_CTA == 4, "level 1 has four sub-superblocks");
    __shared__ int s_u;
    __shared__ float s_cost[WARPS_PER_CTA];
    __shared__ float s_sum[2][WARPS_PER_CTA];
    __shared__ float s_mvc[2][WARPS_PER_CTA];
    __shared__ int s_bi[WARPS_PER_CTA];
    constexpr int MAX_V0 = 8;               // distinct block vectors per reference worth precomputing
    __shared__ short2 s_v0[2][MAX_V0];      // the superblock's distinct block vectors per reference
    __shared__ int s_t0[2][MAX_V0];         // their integer totals at superblock size
    __shared__ int s_n0[2];                 // how many (0: none precomputed)
    __shared__ int s_pre1[WARPS_PER_CTA][8];  // each warp's level-1 candidate totals
    __shared__ short2 s_cand[2][4];           // level-0 candidates per reference
    __shared__ int s_ncand[2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int it = 0; it < L.wave.life; ++it) {
        __syncthreads();
        if (threadIdx.x == 0) s_u = atomicAdd(L.ticket, 1);
        __syncthreads();
        const int u = s_u;
        if (u >= L.total) return;
        int jn, xsb, ysb;
        wave_unit(L.wave, u, jn, xsb, ysb);
        const ModeJob& J = L.jobs[jn];
        const int s = ysb * J.xnsb + xsb;
        // level-1 candidate totals of this warp's sub-superblock while the neighbours finish
        // (in shared memory: the totals are read back by every lane of the warp)
        int* const pre1 = s_pre1[warp];
        dome_totals(L, J, (xsb << 1) + (warp & 1), (ysb << 1) + (warp >> 1), 1, pre1);
        // Level-0 candidates are level-1 vectors, each chosen among its sub-superblock's block
        // vectors: the integer totals at superblock size of the distinct block vectors (when
        // few) are computed here too, also before the waits.
        {
            const LevelData& bk = J.lev[2];
            if (warp == 0) {
                // lanes 0-15: reference 1's block vectors in raster order, lanes 16-31:
                // reference 2's; a lane keeps its vector when no earlier lane of its half has it
                const int r = lane >> 4, t = lane & 15;
                const bool valid = r < J.nref;
                const short2 v = valid ? __ldcg(&bk.mv[r][(size_t)((ysb << 2) + (t >> 2)) * bk.xnb + (xsb << 2) +
                                                       (t & 3)])
                                       : make_short2(0, 0);
                const unsigned long long key = ((unsigned long long)r << 32) |
                                               ((unsigned)(uint16_t)v.x << 16) | (unsigned)(uint16_t)v.y;
                const unsigned same = __match_any_sync(0xffffffffu, key);
                const bool first = valid && (same & ((1u << lane) - 1)) == 0;
                const unsigned half = r ? 0xffff0000u : 0x0000ffffu;
                const unsigned firsts = __ballot_sync(0xffffffffu, first) & half;
                const int n0 = __popc(firsts);
                if (first && n0 <= MAX_V0) s_v0[r][__popc(firsts & ((1u << lane) - 1))] = v;
                if (t == 0) s_n0[r] = valid && n0 <= MAX_V0 ? n0 : 0;
            }
            __syncthreads();
            const Blim bl0 = block_limits(L.lb[0], J.pw, J.ph, xsb, ysb);
            for (int r = 0; r < J.nref; ++r)
                for (int q = warp; q < s_n0[r]; q += WARPS_PER_CTA) {
                    const int t = (bl0.xl > 0 && bl0.yl > 0)
                                      ? subpel_total(J.pic, J.pw, J.up[r], 2 * J.pw, 2 * J.ph, L.prec, bl0,
                                                     s_v0[r][q].x, s_v0[r][q].y)
                                      : 0;
                    if (lane == 0) s_t0[r][q] = t;
                }
        }
        if (threadIdx.x == 0) {
            if (xsb > 0) wait_flag(&J.flags[s - 1], L.err, L.dbg.spin_limit);
            if (ysb > 0) {
                wait_flag(&J.flags[s - J.xnsb], L.err, L.dbg.spin_limit);
                if (xsb > 0) wait_flag(&J.flags[s - J.xnsb - 1], L.err, L.dbg.spin_limit);
            }
        }
        __syncthreads();
        // ---- level 2: the 16 block costs in raster order ----
        const LevelData& blk = J.lev[2];
        float c2 = 0.0f;
        for (int j = 0; j < 4; ++j)
            for (int i = 0; i < 4; ++i) c2 += __ldcg(&J.bcost[(size_t)((ysb << 2) + j) * blk.xnb + (xsb << 2) + i]);
        // ---- level 1: sub-superblock (2 xsb + (warp & 1), 2 ysb + (warp >> 1)) per warp ----
        {
            const int i = (xsb << 1) + (warp & 1), j = (ysb << 1) + (warp >> 1);
            do_me(L, J, i, j, 1, pre1);
            const float c = do_unit_decn(L, J, i, j, 1);
            if (lane == 0) s_cost[warp] = c;
        }
        __syncthreads();
        float sb_cur = c2;
        if (warp == 0) {
            const float c1 = ((s_cost[0] + s_cost[1]) + s_cost[2]) + s_cost[3];
            if (lane == 0) {
                J.split[s] = 2;
                J.sbcost[s] = c2;
            }
            if (c1 <= c2) {
                propagate_level(L, J, xsb, ysb, 1, c1);
                sb_cur = c1;
            }
            __syncwarp();
            if (lane == 0) s_cost[0] = sb_cur;
        }
        __syncthreads();
        sb_cur = s_cost[0];
        // ---- level 0: the whole superblock as one unit (always evaluated: sb_cur <= c2) ----
        if (sb_cur <= c2) {
            const LevelData& me = J.lev[0];
            const LevelData& guide = J.lev[1];
            const size_t k = (size_t)ysb * me.xnb + xsb;
            const float lambda = me.lambda[k];
            const Blim bl = block_limits(L.lb[0], J.pw, J.ph, xsb, ysb);
            const int xb = xsb << 2, yb = ysb << 2;
            // the candidates (the four level-1 vectors, duplicates dropped) in shared memory, so
            // that warp q reads its own without a dynamically indexed local array
            if (threadIdx.x < J.nref) {
                const int r = threadIdx.x;
                int nc = 0;
                for (int jj = 0; jj < 2; ++jj)
                    for (int ii = 0; ii < 2; ++ii) {
                        const short2 v = __ldcg(&guide.mv[r][(size_t)((ysb << 1) + jj) * guide.xnb + (xsb << 1) + ii]);
                        bool dup = false;
                        for (int q = 0; q < nc; ++q) dup |= (s_cand[r][q].x == v.x && s_cand[r][q].y == v.y);
                        if (!dup) s_cand[r][nc++] = v;
                    }
                s_ncand[r] = nc;
            }
            __syncthreads();
            for (int r = 0; r < J.nref; ++r) {
                const int nc = s_ncand[r];
                const short2* bv = blk.mv[r];
                const int W = blk.xnb;
                short2 pr = make_short2(0, 0);
                if (xb > 0 && yb > 0)
                    pr = mv_median3(__ldcg(&bv[(size_t)yb * W + xb - 1]), __ldcg(&bv[(size_t)(yb - 1) * W + xb - 1]),
                                    __ldcg(&bv[(size_t)(yb - 1) * W + xb]));
                else if (xb == 0 && yb > 0)
                    pr = mv_mean(__ldcg(&bv[(size_t)(yb - 1) * W + xb]), __ldcg(&bv[(size_t)(yb - 1) * W + xb + 1]));
                else if (xb > 0 && yb == 0)
                    pr = mv_mean(__ldcg(&bv[(size_t)yb * W + xb - 1]), __ldcg(&bv[(size_t)(yb + 1) * W + xb - 1]));
                // warp q evaluates candidate q (BlockMatcher::FindBestMatchSubp's loop body)
                if (warp < nc && bl.xl > 0 && bl.yl > 0) {
                    const short2 cw = s_cand[r][warp];
                    const float mvcost = (float)getvarup(pr, cw.x, cw.y);
                    const float start = mvcost * lambda;
                    int pre = -1;
                    for (int q = 0; q < s_n0[r]; ++q)
                        if (s_v0[r][q].x == cw.x && s_v0[r][q].y == cw.y) pre = q;
                    FloatSeq f = float_seq_start(start);
                    float sum;
                    if (pre >= 0 && float_seq_add_exact(f, s_t0[r][pre]))
                        sum = (float)f.c;  // precomputed total, and no addition of the loop could round
                    else
                        sum = subpel_cost(J.pic, J.pw, J.up[r], 2 * J.pw, 2 * J.ph, L.prec, bl, cw.x, cw.y, start);
                    if (lane == 0) {
                        s_sum[r][warp] = sum;
                        s_mvc[r][warp] = mvcost;
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int r = 0; r < J.nref; ++r) {
                    Cost3 best{me.cost[r][3 * k], me.cost[r][3 * k + 1], 100000000.0f};
                    short2 bmv = me.mv[r][k];
                    for (int q = 0; q < s_ncand[r]; ++q) {
                        if (bl.xl <= 0 || bl.yl <= 0) break;
                        const float sum = s_sum[r][q], mvcost = s_mvc[r][q];
                        if (sum < best.total) {
                            bmv = s_cand[r][q];
                            best.total = sum;
                            best.mvcost = mvcost;
                            best.SAD = sum - mvcost * lambda;
                        }
                    }
                    me.mv[r][k] = bmv;
                    me.cost[r][3 * k] = best.SAD;
                    me.cost[r][3 * k + 1] = best.mvcost;
                    me.cost[r][3 * k + 2] = best.total;
                }
            }
            __syncthreads();
            float bsad = -1.0f;
            if (J.nref > 1) {
                const int n = bl.xl * bl.yl;
                const int per = ((n + WARPS_PER_CTA - 1) / WARPS_PER_CTA + 31) / 32 * 32;
                const int part = bi_sad_range(J.pic, J.pw, J.up[0], J.up[1], 2 * J.pw, 2 * J.ph, L.prec, bl,
                                              __ldcg(&me.mv[0][k]), __ldcg(&me.mv[1][k]), warp * per,
                                              min(n, (warp + 1) * per));
                if (lane == 0) s_bi[warp] = part;
                __syncthreads();
                bsad = (float)(s_bi[0] + s_bi[1] + s_bi[2] + s_bi[3]);
            }
            if (warp == 0) {
                const float c0 = do_unit_decn(L, J, xsb, ysb, 0, bsad);
                if (c0 <= sb_cur) propagate_level(L, J, xsb, ysb, 0, c0);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            audit_unit(L.dbg, jn, s);
            publish(&J.flags[s]);
        }
    }
}

// ============================================================================================
// DC values (ModeDecider::SetDC, me_mode_decn.cpp:540-573)
// ============================================================================================

struct DcJob {
    const int16_t* pic;
    int pw, ph;
    Olb o;
    int16_t* tmp;   // block DCs
    int16_t* dc;    // output plane (last row left as it is)
    int xnb, ynb;
};

struct DcLaunch {
    int total, per_job;
    const DcJob* jobs;  // device table
};

__global__ void __launch_bounds__(ME_THREADS) block_dc_kernel(const __grid_constant__ DcLaunch L) {
    const int u = blockIdx.x * WARPS_PER_CTA + (threadIdx.x >> 5);
    if (u >= L.total) return;
    const int j = u / L.per_job;
    const DcJob& J = L.jobs[j];
    const int b = u - j * L.per_job;
    const int by = b / J.xnb, bx = b - by * J.xnb;
    const int dc = block_dc(J.pic, J.pw, block_limits(J.o, J.pw, J.ph, bx, by));
    if ((threadIdx.x & 31) == 0) J.tmp[b] = (int16_t)dc;
}

__global__ void smooth_dc_kernel(const __grid_constant__ DcLaunch L) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= L.total) return;
    const int j = u / L.per_job;
    const DcJob& J = L.jobs[j];
    const int b = u - j * L.per_job;
    const int y = b / J.xnb, x = b - y * J.xnb;
    const int W = J.xnb;
    if (y == J.ynb - 1) return;
    const int16_t* t = J.tmp;
    int16_t v;
    if (y == 0 || x == 0 || x == W - 1) {
        v = t[b];
    } else {
        v = (int16_t)((t[b - W - 1] + 3 * t[b - W] + t[b - W + 1] + 3 * t[b - 1] + 3 * t[b + 1] + t[b + W - 1] +
                       3 * t[b + W] + t[b + W + 1] + 8) >> 4);
    }
    J.dc[b] = v;
}

}  // namespace

// ============================================================================================
// Host side
// ============================================================================================

namespace {

// FindTransitions (motion.cpp:201-333) for one reference: the vector-variation map (the SAD
// map computed first is overwritten in the reference and has no effect), widened to whole
// superblocks.  long double as in the reference.
void find_transitions(const short2* mv, int W, int H, std::vector<uint8_t>& trans) {
    std::vector<double> val((size_t)W * H, 0.0);
    long double total = 0.0;
    for (int j = 1; j < H - 1; ++j)
        for (int i = 1; i < W - 1; ++i) {
            double v = 0.0;
            const short2 c = mv[(size_t)j * W + i];
            for (int q = -1; q <= 1; ++q)
                for (int p = -1; p <= 1; ++p) {
                    const short2 o = mv[(size_t)(j + q) * W + i + p];
                    const double d = (double)(std::abs(o.x - c.x) + std::abs(o.y - c.y));
                    if (d > v) v = d;
                }
            val[(size_t)j * W + i] = v;
            total += v;
        }
    const long double mean = total / (long double)(W * H);
    long double sd = 0.0;
    for (int j = 1; j < H - 1; ++j)
        for (int i = 1; i < W - 1; ++i) {
            double diff = (double)(val[(size_t)j * W + i] - mean);
            diff *= diff;
            sd += diff;
        }
    sd /= (long double)(W * H);
    sd = std::sqrt(sd);
    const double threshold = (double)(mean + 3 * sd);
    trans.assign((size_t)W * H, 0);
    for (size_t k = 0; k < (size_t)W * H; ++k) trans[k] = val[k] >= threshold;
    for (int j = 0; j < H / 4; ++j)
        for (int i = 0; i < W / 4; ++i) {
            uint8_t any = 0;
            for (int q = 4 * j; q < 4 * (j + 1); ++q)
                for (int p = 4 * i; p < 4 * (i + 1); ++p) any |= trans[(size_t)q * W + p];
            for (int q = 4 * j; q < 4 * (j + 1); ++q)
                for (int p = 4 * i; p < 4 * (i + 1); ++p) trans[(size_t)q * W + p] = any;
        }
}

// MEData::SetLambdaMap(num_refs, lambda) (motion.cpp:128-171).
void lambda_map(const short2* mv1, const short2* mv2, int nref, int W, int H, float lambda, float* out) {
    std::vector<uint8_t> t1, t2;
    find_transitions(mv1, W, H, t1);
    if (nref > 1) find_transitions(mv2, W, H, t2);
    for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
            const size_t k = (size_t)j * W + i;
            float l;
            if (nref == 1) {
                l = t1[k] ? 0.0f : lambda;
            } else if (t1[k] && t2[k]) {
                l = 0.0f;
            } else if (t1[k] || t2[k]) {
                l = (float)(lambda / 4.0);
            } else {
                l = lambda;
            }
            if (i < 4 || j < 4) l = (float)(l / 5.0);
            out[k] = l;
        }
}

// Page-locked host staging for the batch's vector read-back and lambda maps, one growing
// buffer per host thread (released at thread exit).
struct MePinned {
    void* p = nullptr;
    size_t n = 0;
    ~MePinned() {
        if (p) cudaFreeHost(p);
    }
};

int me_pinned(size_t bytes, char** out) {
    thread_local MePinned buf;
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

// MEData::SetLambdaMap(level, block map, wt) (motion.cpp:173-196).
void level_lambda_map(const float* blk, int W, int level, int lw, int lh, float wt, float* out) {
    const int f = 1 << (2 - level);
    for (int j = 0; j < lh; ++j)
        for (int i = 0; i < lw; ++i) {
            float l = blk[(size_t)(f * j) * W + f * i];
            for (int q = f * j; q < f * (j + 1); ++q)
                for (int p = f * i; p < f * (i + 1); ++p) l = std::max(blk[(size_t)q * W + p], l);
            out[(size_t)j * lw + i] = l * wt;
        }
}

// A bump allocator over the caller's (or the library's) workspace.
struct Arena {
    char* base;
    size_t used, cap;
    template <class T>
    T* take(size_t n) {
        used = align_up(used, 256);
        T* p = reinterpret_cast<T*>(base ? base + used : nullptr);
        used += n * sizeof(T);
        return p;
    }
};

struct MeGeometry {
    int w, h, depth, nref, cformat;
    Olb lb[3];
    int xnb[13], ynb[13], pw[13], ph[13];
    int xnsb, ynsb;
};

int me_depth(int w, int h) {
    return (int)std::min(std::log((double)w / 12.0) / std::log(2.0), std::log((double)h / 12.0) / std::log(2.0));
}

int me_geometry(int cformat, int w, int h, const dgpu_block_params* bp, int nref, MeGeometry& g) {
    if (!bp || nref < 1 || nref > 2 || bp->precision < 1 || bp->precision > 3) return DGPU_ERR_ARG;
    if (bp->xbsep <= 0 || bp->ybsep <= 0 || bp->xblen < bp->xbsep || bp->yblen < bp->ybsep ||
        bp->xblen > 2 * bp->xbsep || bp->yblen > 2 * bp->ybsep || bp->xnum_sb <= 0 || bp->ynum_sb <= 0)
        return DGPU_ERR_SIZE;
    g.w = w;
    g.h = h;
    g.nref = nref;
    g.cformat = cformat;
    g.lb[2] = make_olb(bp->xblen, bp->yblen, bp->xbsep, bp->ybsep);
    g.lb[1] = make_olb(g.lb[2].xblen + g.lb[2].xbsep, g.lb[2].yblen + g.lb[2].xbsep, 2 * g.lb[2].xbsep,
                       2 * g.lb[2].ybsep);
    g.lb[0] = make_olb(g.lb[1].xblen + g.lb[1].xbsep, g.lb[1].yblen + g.lb[1].xbsep, 2 * g.lb[1].xbsep,
                       2 * g.lb[1].ybsep);
    g.depth = me_depth(w, h);
    if (g.depth < 1 || g.depth > 12) return DGPU_ERR_SIZE;
    g.xnsb = bp->xnum_sb;
    g.ynsb = bp->ynum_sb;
    g.xnb[0] = 4 * bp->xnum_sb;
    g.ynb[0] = 4 * bp->ynum_sb;
    g.pw[0] = w;
    g.ph[0] = h;
    for (int l = 1; l <= g.depth; ++l) {
        g.pw[l] = w / (1 << l);
        g.ph[l] = h / (1 << l);
        if (g.pw[l] / 2 < 12 && l < g.depth) return DGPU_ERR_SIZE;
        g.xnb[l] = (g.xnb[l - 1] >> 1) + (g.pw[l] % g.lb[2].xbsep != 0);
        g.ynb[l] = (g.ynb[l - 1] >> 1) + (g.ph[l] % g.lb[2].ybsep != 0);
        // the reference reads outside its vector array when a level has a single column
        if (g.xnb[l] < 2) return DGPU_ERR_SIZE;
    }
    return DGPU_OK;
}

// Device buffers of one batch: per picture (pyramid planes, upconverted luma) and per
// task (the per-level search state, flags, lambda maps, mode-decision levels).
struct PicBufs {
    int16_t* down[13];   // pyramid levels >= 1 of the picture's luma
    int16_t* up;         // upconverted luma (used when the picture is a reference)
};

struct TaskBufs {
    short2* mv[13][2];   // level >= 1 vectors
    float* cost[13][2];
    int* best_sad[13][2];
    short2* best_mv[13][2];
    int* flags;          // 2 * max units of any level
    float* lambda[3];    // level maps 0, 1, 2
    short2* lmv[2][2];   // mode-decision levels 0 and 1
    float* lcost[2][2];
    uint8_t* lmode[2];
    int16_t* ldcy[2];
    int16_t* dctmp;      // block DCs of the three components
    float* bcost;        // level-2 mode-decision costs per block
};

size_t pic_layout(const MeGeometry& g, PicBufs& P, Arena& a, bool need_up) {
    for (int l = 1; l <= g.depth; ++l) P.down[l] = a.take<int16_t>((size_t)g.pw[l] * g.ph[l]);
    P.up = need_up ? a.take<int16_t>(4 * (size_t)g.w * g.h) : nullptr;
    return a.used;
}

// fa / za: arenas over regions shared by all tasks of a batch, so that the wavefront flags and
// the mode-decision level data each clear with one memset.
size_t task_layout(const MeGeometry& g, TaskBufs& T, Arena& a, Arena& fa, Arena& za) {
    for (int l = 0; l <= g.depth; ++l)
        for (int r = 0; r < 2; ++r) {
            const size_t n = (size_t)g.xnb[l] * g.ynb[l];
            T.mv[l][r] = l ? a.take<short2>(n) : nullptr;
            T.cost[l][r] = l ? a.take<float>(3 * n) : nullptr;
            T.best_sad[l][r] = a.take<int>(n);
            T.best_mv[l][r] = a.take<short2>(n);
        }
    size_t maxunits = 0;
    for (int l = 0; l <= g.depth; ++l) maxunits = std::max(maxunits, (size_t)g.xnb[l] * g.ynb[l]);
    T.flags = fa.take<int>(2 * maxunits);
    const size_t nb = (size_t)g.xnb[0] * g.ynb[0];
    T.lambda[2] = a.take<float>(nb);
    T.lambda[1] = a.take<float>(nb / 4);
    T.lambda[0] = a.take<float>(nb / 16);
    for (int lv = 0; lv < 2; ++lv) {
        const size_t n = lv ? nb / 4 : nb / 16;
        for (int r = 0; r < 2; ++r) {
            T.lmv[lv][r] = za.take<short2>(n);
            T.lcost[lv][r] = za.take<float>(3 * n);
        }
        T.lmode[lv] = za.take<uint8_t>(n);
        T.ldcy[lv] = za.take<int16_t>(n);
    }
    T.dctmp = a.take<int16_t>(3 * nb);
    T.bcost = a.take<float>(nb);
    return a.used;
}

struct BatchArgs {
    int cformat, w, h, luma_depth, stages, prec;
    int npics, ntasks;
    const int16_t* const* pics;  // npics * 3 planes
    const int* task_pic;
    const int* task_ref[2];      // second may hold -1 entries
    const float* task_lambda;
    int16_t* const* mv_out;
    float* const* cost_out;
    uint8_t* const* mode_out;
    int16_t* const* dc_out;
    uint8_t* const* split_out;
    float* const* sbcost_out;
};

// Wave-order prefix table of a W x H grid (see Wave): units of one job on diagonals < t.
void wave_prefix(int W, int H, int slope, std::vector<int>& pre) {
    const int T = (W - 1) + slope * (H - 1) + 1;
    pre.assign(T + 1, 0);
    for (int t = 0; t < T; ++t) {
        const int ex = t - (W - 1);
        const int ylo = ex > 0 ? (ex + slope - 1) / slope : 0;
        const int yhi = std::min(H - 1, t / slope);
        pre[t + 1] = pre[t] + std::max(0, yhi - ylo + 1);
    }
}

// Device tables of one batch: the jobs of every launch and the wave-order prefixes.
struct BatchTables {
    PelJob* pel;      // (depth + 1) levels x 2 * ntasks
    SubJob* sub;      // 2 * ntasks
    ModeJob* mode;    // ntasks
    DcJob* dc;        // 3 * ntasks
    int* prefix;      // levels 0..depth (slope 2), then superblocks (slope 1)
    size_t prefix_off[14];
    size_t prefix_len;
    char* flags;      // every task's wavefront flags
    size_t flags_bytes;
    char* zero;       // every task's mode-decision level data (cleared per batch)
    size_t zero_bytes;
};

size_t prefix_layout(const MeGeometry& g, size_t* off) {
    size_t n = 0;
    for (int l = 0; l <= g.depth; ++l) {
        off[l] = n;
        n += (size_t)(g.xnb[l] - 1) + 2 * (size_t)(g.ynb[l] - 1) + 2;
    }
    off[g.depth + 1] = n;
    n += (size_t)(g.xnsb - 1) + (size_t)(g.ynsb - 1) + 2;
    return n;
}

size_t batch_bytes(const MeGeometry& g, const BatchArgs& A, std::vector<PicBufs>* P, std::vector<TaskBufs>* T,
                   char* base, int** ctl, BatchTables* tabs = nullptr) {
    Arena a{base, 0, 0};
    {
        BatchTables bt{};
        bt.pel = a.take<PelJob>((size_t)(g.depth + 1) * 2 * A.ntasks);
        bt.sub = a.take<SubJob>((size_t)2 * A.ntasks);
        bt.mode = a.take<ModeJob>((size_t)A.ntasks);
        bt.dc = a.take<DcJob>((size_t)3 * A.ntasks);
        bt.prefix_len = prefix_layout(g, bt.prefix_off);
        bt.prefix = a.take<int>(bt.prefix_len);
        if (tabs) *tabs = bt;
    }
    std::vector<char> is_ref(A.npics, 0);
    for (int t = 0; t < A.ntasks; ++t)
        for (int r = 0; r < 2; ++r)
            if (A.task_ref[r][t] >= 0) is_ref[A.task_ref[r][t]] = 1;
    PicBufs pb;
    for (int p = 0; p < A.npics; ++p) {
        pic_layout(g, pb, a, is_ref[p] && A.stages >= 2);
        if (P) P->push_back(pb);
    }
    TaskBufs tb;
    {
        Arena sa{nullptr, 0, 0}, sf{nullptr, 0, 0}, sz{nullptr, 0, 0};
        task_layout(g, tb, sa, sf, sz);
        const size_t fper = align_up(sf.used, 256), zper = align_up(sz.used, 256);
        char* fbase = a.take<char>(fper * A.ntasks);
        char* zbase = a.take<char>(zper * A.ntasks);
        if (tabs) {
            tabs->flags = fbase;
            tabs->flags_bytes = fper * A.ntasks;
            tabs->zero = zbase;
            tabs->zero_bytes = zper * A.ntasks;
        }
        Arena fa{fbase, 0, 0}, za{zbase, 0, 0};
        for (int t = 0; t < A.ntasks; ++t) {
            task_layout(g, tb, a, fa, za);
            if (T) T->push_back(tb);
        }
    }
    int* c = a.take<int>(64);
    if (ctl) *ctl = c;
    return a.used + 256;
}

// Largest per-CTA window staging of the pel kernels: blocks up to 64 x 64 (check_args) and a
// search radius of at most 5, for each of the CTA's warps.
constexpr size_t PEL_SMEM_MAX = align_up((size_t)64 * 64 + (size_t)(64 + 10) * (64 + 10), 8) * 2 * WARPS_PER_CTA;

// Opts the pel kernels into PEL_SMEM_MAX bytes of dynamic shared memory once per device.  One
// fixed value set under a lock, so a host thread never launches while another lowers it.
int pel_smem_setup() {
    static std::mutex mu;
    static uint64_t done = 0;  // devices 0..63 already set up
    int dev = 0;
    DGPU_CHECK_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
    std::lock_guard<std::mutex> lock(mu);
    if (bit && (done & bit)) return DGPU_OK;
    DGPU_CHECK_CUDA(
        cudaFuncSetAttribute(pel_lists_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PEL_SMEM_MAX));
    DGPU_CHECK_CUDA(
        cudaFuncSetAttribute(pel_wavefront_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PEL_SMEM_MAX));
    done |= bit;
    return DGPU_OK;
}

// Resident CTAs per SM of the persistent wavefront kernels (dgpu_me_set_occupancy): at 8 a
// launch holds every register of every SM until its last unit is done; fewer leave room on
// each SM for other streams' kernels.  Any number is free of deadlock: a CTA waits only on
// units whose tickets were taken before its own, by CTAs already resident.
std::atomic<int> g_wave_ctas_per_sm{8};

int wave_grid(int ctas_needed) {
    static std::atomic<int> sms[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    std::atomic<int>& n = sms[dev & 63];
    if (n.load() <= 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
            cudaGetLastError();
            v = 148;
        }
        n.store(v);
    }
    return std::max(1, std::min(ctas_needed, n.load() * g_wave_ctas_per_sm.load()));
}

// Units a warp (pel and sub-pel wavefronts) or a CTA (mode wavefront) takes before it exits
// (dgpu_me_set_unit_lifetime; 0: until the tickets run out).  A bounded lifetime hands the SMs
// back to the block scheduler every few units, so that kernels of higher-priority streams
// start within that time instead of after the whole launch.  Also free of deadlock: a unit
// waits only on units with earlier tickets, held by warps that are resident and finish them.
std::atomic<int> g_wave_life{0};

// Grid of a wavefront launch over `total` units, `slots` ticket takers per CTA (warps, or 1),
// with w.life set: the persistent grid, or with a lifetime at least enough CTAs that
// grid x slots x life covers every unit.
int wave_launch_grid(Wave& w, int total, int slots) {
    const int persistent = wave_grid((total + slots - 1) / slots);
    const int life = g_wave_life.load();
    if (life <= 0) {
        w.life = INT_MAX;
        return persistent;
    }
    w.life = life;
    const long long per = (long long)slots * life;
    const long long need = ((long long)total + per - 1) / per;
    return (int)std::max<long long>(persistent, need);
}

// Process-wide settings of dgpu_debug_wavefront, read once by each motion-estimation call.
struct DebugSettings {
    int skip_unit = -1;
    long long spin_limit = SPIN_LIMIT;
    int* audit[3] = {nullptr, nullptr, nullptr};  // pel (finest level), sub-pel, mode decision
    unsigned long long* ops = nullptr;             // [3]: pel, sub-pel, mode decision
};
std::mutex g_debug_mu;
DebugSettings g_debug;

DebugSettings debug_settings() {
    std::lock_guard<std::mutex> lk(g_debug_mu);
    return g_debug;
}

// Device time per kernel class of the estimation calls made while dgpu_me_profile is on, in
// the order of DGPU_ME_NKERNELS.
constexpr int MEK_N = DGPU_ME_NKERNELS;
struct MeProfile {
    bool on = false;
    double ms[MEK_N] = {};
    int launches[MEK_N] = {};
};
MeProfile g_me_prof;  // guarded by g_debug_mu

// Events around each kernel class of one call; elapsed times are added to g_me_prof once
// the call has synchronised (flush), and the events are released in any case.
class MeTimer {
   public:
    MeTimer(bool on, cudaStream_t st) : on_(on), st_(st) {}
    ~MeTimer() {
        for (auto& r : rec_) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
    }
    void start(int k) {
        if (!on_) return;
        Rec r{k, nullptr, nullptr};
        if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) {
            cudaGetLastError();
            on_ = false;
            return;
        }
        cudaEventRecord(r.a, st_);
        rec_.push_back(r);
    }
    void stop() {
        if (on_ && !rec_.empty()) cudaEventRecord(rec_.back().b, st_);
    }
    void flush() {
        if (!on_) return;
        std::lock_guard<std::mutex> lk(g_debug_mu);
        for (auto& r : rec_) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
                g_me_prof.ms[r.k] += ms;
                g_me_prof.launches[r.k] += 1;
            } else {
                cudaGetLastError();
            }
        }
    }

   private:
    struct Rec {
        int k;
        cudaEvent_t a, b;
    };
    bool on_;
    cudaStream_t st_;
    std::vector<Rec> rec_;
};

bool me_profile_on() {
    std::lock_guard<std::mutex> lk(g_debug_mu);
    return g_me_prof.on;
}

int run_batch(const MeGeometry& g, const BatchArgs& A, void* workspace, cudaStream_t st) {
    const DebugSettings dbg = debug_settings();
    MeTimer tm(me_profile_on(), st);
    std::vector<PicBufs> P;
    std::vector<TaskBufs> T;
    int* ctl = nullptr;
    BatchTables tabs{};
    batch_bytes(g, A, &P, &T, static_cast<char*>(workspace), &ctl, &tabs);
    {
        std::vector<int> all(tabs.prefix_len), pre;
        for (int l = 0; l <= g.depth; ++l) {
            wave_prefix(g.xnb[l], g.ynb[l], 2, pre);
            std::copy(pre.begin(), pre.end(), all.begin() + tabs.prefix_off[l]);
        }
        wave_prefix(g.xnsb, g.ynsb, 1, pre);
        std::copy(pre.begin(), pre.end(), all.begin() + tabs.prefix_off[g.depth + 1]);
        DGPU_CHECK_CUDA(cudaMemcpyAsync(tabs.prefix, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice, st));
    }
    auto wave_of = [&](int slot, int W, int slope, int njobs) {
        Wave w;
        w.prefix = tabs.prefix + tabs.prefix_off[slot];
        w.W = W;
        w.slope = slope;
        w.njobs = njobs;
        w.T = 0;
        w.life = INT_MAX;
        return w;
    };
    DGPU_CHECK_CUDA(cudaMemsetAsync(ctl, 0, 2 * sizeof(int), st));
    const size_t nb = (size_t)g.xnb[0] * g.ynb[0];
    auto luma = [&](int p) { return A.pics[3 * p]; };
    auto nref_of = [&](int t) { return A.task_ref[1][t] >= 0 ? 2 : 1; };
    auto ref_of = [&](int t, int r) { return r == 1 && A.task_ref[1][t] >= 0 ? A.task_ref[1][t] : A.task_ref[0][t]; };
    auto mv0 = [&](int t, int r) { return reinterpret_cast<short2*>(A.mv_out[t]) + (size_t)r * nb; };
    auto cost0 = [&](int t, int r) { return A.cost_out[t] + (size_t)r * 3 * nb; };
    std::vector<char> used(A.npics, 0);
    for (int t = 0; t < A.ntasks; ++t) {
        used[A.task_pic[t]] = 1;
        for (int r = 0; r < nref_of(t); ++r) used[ref_of(t, r)] = 1;
    }
    // ---- pyramids of every picture involved (PixelMatcher::MakePicHierarchy) ----
    tm.start(0);
    for (int l = 1; l <= g.depth; ++l) {
        std::vector<const int16_t*> in;
        std::vector<int16_t*> out;
        for (int p = 0; p < A.npics; ++p) {
            if (!used[p]) continue;
            in.push_back(l == 1 ? luma(p) : P[p].down[l - 1]);
            out.push_back(P[p].down[l]);
        }
        for (size_t i = 0; i < in.size(); i += 32) {
            const int k = (int)std::min<size_t>(32, in.size() - i);
            std::vector<int> iw(k, g.pw[l - 1]), ih(k, g.ph[l - 1]), os(k, g.pw[l]);
            const int rc = dgpu_downconvert_batch(k, in.data() + i, iw.data(), ih.data(), iw.data(), out.data() + i,
                                                  os.data(), st);
            if (rc) return rc;
        }
    }
    tm.stop();
    // ---- pel search, coarsest level first: every job of a level in one wavefront ----
    for (int l = g.depth; l >= 0; --l) {
        std::vector<PelJob> jobs;
        for (int t = 0; t < A.ntasks; ++t)
            for (int r = 0; r < nref_of(t); ++r) {
                PelJob J{};
                const int pp = A.task_pic[t], rp = ref_of(t, r);
                J.pic = l ? P[pp].down[l] : luma(pp);
                J.ref = l ? P[rp].down[l] : luma(rp);
                J.pw = g.pw[l];
                J.ph = g.ph[l];
                J.xnb = g.xnb[l];
                J.ynb = g.ynb[l];
                J.mv = l ? T[t].mv[l][r] : mv0(t, r);
                J.cost = l ? T[t].cost[l][r] : cost0(t, r);
                J.guide = l < g.depth ? T[t].mv[l + 1][r] : nullptr;
                J.gxnb = l < g.depth ? g.xnb[l + 1] : 0;
                J.gynb = l < g.depth ? g.ynb[l + 1] : 0;
                J.radius = std::min(l + 1, 5);
                J.best_sad = T[t].best_sad[l][r];
                J.best_mv = T[t].best_mv[l][r];
                J.flags = T[t].flags + (size_t)r * g.xnb[l] * g.ynb[l];
                jobs.push_back(J);
            }
        DGPU_CHECK_CUDA(cudaMemsetAsync(tabs.flags, 0, tabs.flags_bytes, st));
        PelJob* dj = tabs.pel + (size_t)l * 2 * A.ntasks;
        DGPU_CHECK_CUDA(cudaMemcpyAsync(dj, jobs.data(), sizeof(PelJob) * jobs.size(), cudaMemcpyHostToDevice, st));
        PelLaunch L{};
        L.dbg = WaveDebug{dbg.spin_limit, dbg.skip_unit, l == 0 ? dbg.audit[0] : nullptr, dbg.ops};
        L.o = g.lb[2];
        L.per_job = g.xnb[l] * g.ynb[l];
        L.total = L.per_job * (int)jobs.size();
        L.jobs = dj;
        L.wave = wave_of(l, g.xnb[l], 2, (int)jobs.size());
        L.wave.T = (g.xnb[l] - 1) + 2 * (g.ynb[l] - 1) + 1;
        // per-warp shared memory: the block and its search window (radius <= 5)
        const int xl = g.lb[2].xblen, yl = g.lb[2].yblen, rr = std::min(l + 1, 5);
        L.win_elems = (int)align_up((size_t)xl * yl + (size_t)(xl + 2 * rr) * (yl + 2 * rr), 8);
        const size_t smem = (size_t)L.win_elems * 2 * WARPS_PER_CTA;
        if (smem > PEL_SMEM_MAX) return DGPU_ERR_SIZE;
        {
            const int rc = pel_smem_setup();
            if (rc) return rc;
        }
        // the candidate-list phase covers every unit: one warp per unit
        tm.start(1);
        pel_lists_kernel<<<(L.total + WARPS_PER_CTA - 1) / WARPS_PER_CTA, ME_THREADS, smem, st>>>(L);
        tm.stop();
        DGPU_CHECK_LAUNCH();
        L.ticket = ctl;
        L.err = ctl + 1;
        DGPU_CHECK_CUDA(cudaMemsetAsync(ctl, 0, sizeof(int), st));
        tm.start(2);
        const int grid = wave_launch_grid(L.wave, L.total, WARPS_PER_CTA);
        pel_wavefront_kernel<<<grid, ME_THREADS, smem, st>>>(L);
        tm.stop();
        DGPU_CHECK_LAUNCH();
    }
    int err_host = 0;
    if (A.stages >= 2) {
        // ---- lambda maps on the host (long double statistics, as the reference) ----
        // vectors come back and maps go out through page-locked memory; the tasks' maps are
        // independent, so host threads share them
        char* pin = nullptr;
        {
            const int rc = me_pinned((sizeof(short2) * 2 * nb + sizeof(float) * nb) * A.ntasks + 256, &pin);
            if (rc) return rc;
        }
        short2* hmv_all = reinterpret_cast<short2*>(pin);
        float* hl_all = reinterpret_cast<float*>(pin + sizeof(short2) * 2 * nb * A.ntasks);
        auto hmv = [&](int t) { return hmv_all + (size_t)t * 2 * nb; };
        auto hlm = [&](int t) { return hl_all + (size_t)t * nb; };
        for (int t = 0; t < A.ntasks; ++t)
            DGPU_CHECK_CUDA(cudaMemcpyAsync(hmv(t), A.mv_out[t], sizeof(short2) * nref_of(t) * nb,
                                            cudaMemcpyDeviceToHost, st));
        DGPU_CHECK_CUDA(cudaMemcpyAsync(&err_host, ctl + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        DGPU_CHECK_CUDA(host_wait(st));
        if (err_host) return DGPU_ERR_CUDA;
        {
            const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
            const int nth = std::min(A.ntasks, std::min(hw, 16));
            auto work = [&](int first) {
                for (int t = first; t < A.ntasks; t += nth)
                    lambda_map(hmv(t), hmv(t) + nb, nref_of(t), g.xnb[0], g.ynb[0], A.task_lambda[t], hlm(t));
            };
            std::vector<std::thread> pool;
            for (int k = 1; k < nth; ++k) pool.emplace_back(work, k);
            work(0);
            for (auto& th : pool) th.join();
        }
        for (int t = 0; t < A.ntasks; ++t)
            DGPU_CHECK_CUDA(cudaMemcpyAsync(T[t].lambda[2], hlm(t), sizeof(float) * nb, cudaMemcpyHostToDevice, st));
        // ---- upconverted original references (EncPicture::UpOrigData) ----
        tm.start(0);
        {
            std::vector<const int16_t*> in;
            std::vector<int16_t*> out;
            for (int p = 0; p < A.npics; ++p)
                if (P[p].up) {
                    in.push_back(luma(p));
                    out.push_back(P[p].up);
                }
            for (size_t i = 0; i < in.size(); i += 32) {
                const int k = (int)std::min<size_t>(32, in.size() - i);
                std::vector<int> iw(k, g.w), ih(k, g.h), bd(k, A.luma_depth), us(k, 2 * g.w);
                const int rc = dgpu_upconvert_batch(k, in.data() + i, iw.data(), ih.data(), iw.data(), bd.data(),
                                                    out.data() + i, us.data(), st);
                if (rc) return rc;
            }
        }
        tm.stop();
        // ---- sub-pel refinement: every job in one wavefront ----
        {
            std::vector<SubJob> jobs;
            for (int t = 0; t < A.ntasks; ++t)
                for (int r = 0; r < nref_of(t); ++r) {
                    SubJob J{};
                    J.pic = luma(A.task_pic[t]);
                    J.up = P[ref_of(t, r)].up;
                    J.pw = g.w;
                    J.ph = g.h;
                    J.xnb = g.xnb[0];
                    J.ynb = g.ynb[0];
                    J.mv = mv0(t, r);
                    J.cost = cost0(t, r);
                    J.lambda = T[t].lambda[2];
                    J.flags = T[t].flags + (size_t)r * nb;
                    jobs.push_back(J);
                }
            DGPU_CHECK_CUDA(cudaMemsetAsync(tabs.flags, 0, tabs.flags_bytes, st));
            DGPU_CHECK_CUDA(cudaMemcpyAsync(tabs.sub, jobs.data(), sizeof(SubJob) * jobs.size(),
                                            cudaMemcpyHostToDevice, st));
            SubLaunch S{};
            S.dbg = WaveDebug{dbg.spin_limit, -1, dbg.audit[1], dbg.ops ? dbg.ops + 1 : nullptr};
            S.o = g.lb[2];
            S.prec = A.prec;
            S.total = (int)nb * (int)jobs.size();
            S.jobs = tabs.sub;
            S.wave = wave_of(0, g.xnb[0], 2, (int)jobs.size());
            S.wave.T = (g.xnb[0] - 1) + 2 * (g.ynb[0] - 1) + 1;
            // per-warp staging of the block and its window when it fits a modest budget
            const int xl = g.lb[2].xblen, yl = g.lb[2].yblen;
            const int elems = (int)align_up(align_up((size_t)xl * yl, 8) +
                                                (size_t)sub_win_pitch(xl) * (2 * yl + 3 + 2 * SUB_EXTRA), 8);
            S.win_elems = elems * 2 * WARPS_PER_CTA <= 24 * 1024 ? elems : 0;
            S.ticket = ctl;
            S.err = ctl + 1;
            DGPU_CHECK_CUDA(cudaMemsetAsync(ctl, 0, sizeof(int), st));
            const int grid = wave_launch_grid(S.wave, S.total, WARPS_PER_CTA);
            tm.start(3);
            subpel_wavefront_kernel<<<grid, ME_THREADS, (size_t)S.win_elems * 2 * WARPS_PER_CTA, st>>>(S);
            tm.stop();
            DGPU_CHECK_LAUNCH();
        }
        if (A.stages >= 3) {
            const float f0 = (float)(16 * g.lb[2].xblen * g.lb[2].yblen) / (float)(g.lb[0].xblen * g.lb[0].yblen);
            const float f1 = (float)(4 * g.lb[2].xblen * g.lb[2].yblen) / (float)(g.lb[1].xblen * g.lb[1].yblen);
            // fresh level data for every task (a new MEData per picture in the reference)
            DGPU_CHECK_CUDA(cudaMemsetAsync(tabs.zero, 0, tabs.zero_bytes, st));
            std::vector<std::vector<float>> l0(A.ntasks), l1(A.ntasks);
            for (int t = 0; t < A.ntasks; ++t) {
                l0[t].resize(nb / 16);
                l1[t].resize(nb / 4);
                level_lambda_map(hlm(t), g.xnb[0], 0, g.xnb[0] / 4, g.ynb[0] / 4, (float)(1.0 / f0), l0[t].data());
                level_lambda_map(hlm(t), g.xnb[0], 1, g.xnb[0] / 2, g.ynb[0] / 2, (float)(1.0 / f1), l1[t].data());
                DGPU_CHECK_CUDA(cudaMemcpyAsync(T[t].lambda[0], l0[t].data(), sizeof(float) * l0[t].size(),
                                                cudaMemcpyHostToDevice, st));
                DGPU_CHECK_CUDA(cudaMemcpyAsync(T[t].lambda[1], l1[t].data(), sizeof(float) * l1[t].size(),
                                                cudaMemcpyHostToDevice, st));
                // zero DC arrays (a fresh MvData)
                DGPU_CHECK_CUDA(cudaMemsetAsync(A.dc_out[t], 0, sizeof(int16_t) * 3 * nb, st));
            }
            ModeLaunch M{};
            M.dbg = WaveDebug{dbg.spin_limit, -1, dbg.audit[2], dbg.ops ? dbg.ops + 2 : nullptr};
            M.prec = A.prec;
            for (int i = 0; i < 3; ++i) M.lb[i] = g.lb[i];
            M.level_factor[0] = f0;
            M.level_factor[1] = f1;
            M.level_factor[2] = 1.0f;
            std::vector<ModeJob> jobs;
            // one launch per reference count (the kernel takes nref per launch); each launch
            // runs all its pictures' superblock wavefronts together
            // every picture's superblock wavefront in one launch (nref per job)
            for (int t = 0; t < A.ntasks; ++t) {
                const int want_nref = nref_of(t);
                ModeJob J{};
                J.nref = want_nref;
                J.pic = luma(A.task_pic[t]);
                J.up[0] = P[ref_of(t, 0)].up;
                J.up[1] = P[ref_of(t, 1)].up;
                J.pw = g.w;
                J.ph = g.h;
                for (int lv = 0; lv < 3; ++lv) {
                    LevelData& D = J.lev[lv];
                    D.xnb = g.xnb[0] >> (2 - lv);
                    D.ynb = g.ynb[0] >> (2 - lv);
                    D.lambda = T[t].lambda[lv];
                    if (lv == 2) {
                        D.mv[0] = mv0(t, 0);
                        D.mv[1] = want_nref > 1 ? mv0(t, 1) : mv0(t, 0);
                        D.cost[0] = cost0(t, 0);
                        D.cost[1] = want_nref > 1 ? cost0(t, 1) : cost0(t, 0);
                        D.mode = A.mode_out[t];
                        D.dcy = A.dc_out[t];
                    } else {
                        D.mv[0] = T[t].lmv[lv][0];
                        D.mv[1] = T[t].lmv[lv][1];
                        D.cost[0] = T[t].lcost[lv][0];
                        D.cost[1] = T[t].lcost[lv][1];
                        D.mode = T[t].lmode[lv];
                        D.dcy = T[t].ldcy[lv];
                    }
                }
                J.sbcost = A.sbcost_out[t];
                J.split = A.split_out[t];
                J.xnsb = g.xnsb;
                J.ynsb = g.ynsb;
                J.flags = T[t].flags;
                J.bcost = T[t].bcost;
                jobs.push_back(J);
            }
            DGPU_CHECK_CUDA(cudaMemsetAsync(tabs.flags, 0, tabs.flags_bytes, st));
            {
                const int nj = (int)jobs.size();
                DGPU_CHECK_CUDA(cudaMemcpyAsync(tabs.mode, jobs.data(), sizeof(ModeJob) * nj, cudaMemcpyHostToDevice,
                                                st));
                M.jobs = tabs.mode;
                // level 2 for every block of every job, then the superblock wavefront
                M.total = (int)nb * nj;
                tm.start(4);
                mode_blocks_kernel<<<(M.total + WARPS_PER_CTA - 1) / WARPS_PER_CTA, ME_THREADS, 0, st>>>(M, (int)nb);
                tm.stop();
                DGPU_CHECK_LAUNCH();
                M.total = g.xnsb * g.ynsb * nj;
                M.wave = wave_of(g.depth + 1, g.xnsb, 1, nj);
                M.wave.T = (g.xnsb - 1) + (g.ynsb - 1) + 1;
                M.ticket = ctl;
                M.err = ctl + 1;
                DGPU_CHECK_CUDA(cudaMemsetAsync(ctl, 0, sizeof(int), st));
                const int grid = wave_launch_grid(M.wave, M.total, 1);
                tm.start(5);
                mode_wavefront_kernel<<<grid, ME_THREADS, 0, st>>>(M);
                tm.stop();
                DGPU_CHECK_LAUNCH();
            }
            // ---- DC values of all three components ----
            {
                std::vector<DcJob> jobs;
                for (int t = 0; t < A.ntasks; ++t)
                    for (int c = 0; c < 3; ++c) {
                        const int xs = (c && A.cformat != 0) ? 1 : 0, ys = (c && A.cformat == 2) ? 1 : 0;
                        DcJob Jd{};
                        Jd.pic = A.pics[3 * A.task_pic[t] + c];
                        Jd.pw = g.w >> xs;
                        Jd.ph = g.h >> ys;
                        Jd.o = make_olb(g.lb[2].xblen >> xs, g.lb[2].yblen >> ys, g.lb[2].xbsep >> xs,
                                        g.lb[2].ybsep >> ys);
                        Jd.tmp = T[t].dctmp + (size_t)c * nb;
                        Jd.dc = A.dc_out[t] + (size_t)c * nb;
                        Jd.xnb = g.xnb[0];
                        Jd.ynb = g.ynb[0];
                        jobs.push_back(Jd);
                    }
                DGPU_CHECK_CUDA(cudaMemcpyAsync(tabs.dc, jobs.data(), sizeof(DcJob) * jobs.size(),
                                                cudaMemcpyHostToDevice, st));
                DcLaunch D{};
                D.per_job = (int)nb;
                D.total = (int)nb * (int)jobs.size();
                D.jobs = tabs.dc;
                tm.start(6);
                block_dc_kernel<<<(D.total + WARPS_PER_CTA - 1) / WARPS_PER_CTA, ME_THREADS, 0, st>>>(D);
                DGPU_CHECK_LAUNCH();
                smooth_dc_kernel<<<(D.total + 255) / 256, 256, 0, st>>>(D);
                tm.stop();
                DGPU_CHECK_LAUNCH();
            }
        }
    }
    DGPU_CHECK_CUDA(cudaMemcpyAsync(&err_host, ctl + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    DGPU_CHECK_CUDA(host_wait(st));
    if (err_host) return DGPU_ERR_CUDA;
    tm.flush();
    return DGPU_OK;
}

int check_args(int cformat, int luma_depth, const MeGeometry& g) {
    if (cformat < 0 || cformat > 2 || luma_depth < 2 || luma_depth > 15) return DGPU_ERR_ARG;
    if (g.lb[2].xblen > 64 || g.lb[2].yblen > 64) return DGPU_ERR_SIZE;
    return DGPU_OK;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_me_depth(int w, int h) { return me_depth(w, h); }

extern "C" int dgpu_me_profile(int enable, double* kernel_ms, int* launches) {
    std::lock_guard<std::mutex> lk(g_debug_mu);
    for (int k = 0; k < MEK_N; ++k) {
        if (kernel_ms) kernel_ms[k] = g_me_prof.ms[k];
        if (launches) launches[k] = g_me_prof.launches[k];
        g_me_prof.ms[k] = 0.0;
        g_me_prof.launches[k] = 0;
    }
    g_me_prof.on = enable != 0;
    return DGPU_OK;
}

extern "C" int dgpu_me_set_occupancy(int ctas_per_sm) {
    if (ctas_per_sm < 1 || ctas_per_sm > 8) return DGPU_ERR_ARG;
    g_wave_ctas_per_sm.store(ctas_per_sm);
    return DGPU_OK;
}

extern "C" int dgpu_me_set_unit_lifetime(int units) {
    if (units < 0) return DGPU_ERR_ARG;
    g_wave_life.store(units);
    return DGPU_OK;
}

extern "C" int dgpu_debug_wavefront(int skip_unit, long long spin_limit, int* audit_pel, int* audit_subpel,
                                    int* audit_mode, unsigned long long* ops) {
    if (skip_unit < -1 || spin_limit < 0) return DGPU_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_debug_mu);
    g_debug.skip_unit = skip_unit;
    g_debug.spin_limit = spin_limit == 0 ? SPIN_LIMIT : std::min(spin_limit, SPIN_LIMIT);
    g_debug.audit[0] = audit_pel;
    g_debug.audit[1] = audit_subpel;
    g_debug.audit[2] = audit_mode;
    g_debug.ops = ops;
    return DGPU_OK;
}

extern "C" size_t dgpu_me_batch_workspace_bytes(int cformat, int w, int h, const dgpu_block_params* bp, int npics,
                                                int ntasks, const int* task_ref2, int stages) {
    MeGeometry g;
    if (me_geometry(cformat, w, h, bp, 2, g) != DGPU_OK || npics <= 0 || ntasks <= 0) return 0;
    std::vector<int> zeros(ntasks, 0);
    BatchArgs A{};
    A.npics = npics;
    A.ntasks = ntasks;
    A.stages = stages;
    A.task_ref[0] = zeros.data();
    A.task_ref[1] = task_ref2 ? task_ref2 : zeros.data();
    // every picture may be a reference: size for the worst case
    std::vector<int> all(npics);
    for (int p = 0; p < npics; ++p) all[p] = p;
    BatchArgs B = A;
    std::vector<int> r0(std::max(npics, ntasks), 0);
    for (int t = 0; t < std::max(npics, ntasks); ++t) r0[t] = t % npics;
    B.ntasks = std::max(npics, ntasks);
    B.task_ref[0] = r0.data();
    std::vector<int> none(B.ntasks, -1);
    B.task_ref[1] = none.data();
    return batch_bytes(g, B, nullptr, nullptr, nullptr, nullptr);
}

extern "C" size_t dgpu_me_workspace_bytes(int cformat, int w, int h, const dgpu_block_params* bp, int nref) {
    return dgpu_me_batch_workspace_bytes(cformat, w, h, bp, 3, 1, nullptr, 3);
}

extern "C" int dgpu_motion_estimate_batch(int cformat, int w, int h, const dgpu_block_params* bp, int luma_depth,
                                          int npics, const int16_t* const* pics, int ntasks, const int* task_pic,
                                          const int* task_ref1, const int* task_ref2, const float* task_lambda,
                                          int stages, int16_t* const* mv_out, float* const* cost_out,
                                          uint8_t* const* mode_out, int16_t* const* dc_out, uint8_t* const* split_out,
                                          float* const* sbcost_out, void* workspace, size_t ws_bytes, void* stream) {
    if (npics <= 0 || ntasks <= 0 || !pics || !task_pic || !task_ref1 || !task_ref2 || !task_lambda || !mv_out ||
        !cost_out)
        return DGPU_ERR_ARG;
    if (stages >= 3 && (!mode_out || !dc_out || !split_out || !sbcost_out)) return DGPU_ERR_ARG;
    MeGeometry g;
    int rc = me_geometry(cformat, w, h, bp, 2, g);
    if (rc) return rc;
    rc = check_args(cformat, luma_depth, g);
    if (rc) return rc;
    for (int p = 0; p < npics; ++p)
        for (int c = 0; c < (stages >= 3 ? 3 : 1); ++c)
            if (!pics[3 * p + c]) return DGPU_ERR_ARG;
    for (int t = 0; t < ntasks; ++t) {
        if (task_pic[t] < 0 || task_pic[t] >= npics || task_ref1[t] < 0 || task_ref1[t] >= npics ||
            task_ref2[t] >= npics || !mv_out[t] || !cost_out[t])
            return DGPU_ERR_ARG;
        if (stages >= 3 && (!mode_out[t] || !dc_out[t] || !split_out[t] || !sbcost_out[t])) return DGPU_ERR_ARG;
    }
    BatchArgs A{};
    A.cformat = cformat;
    A.w = w;
    A.h = h;
    A.luma_depth = luma_depth;
    A.stages = stages;
    A.prec = bp->precision;
    A.npics = npics;
    A.ntasks = ntasks;
    A.pics = pics;
    A.task_pic = task_pic;
    A.task_ref[0] = task_ref1;
    A.task_ref[1] = task_ref2;
    A.task_lambda = task_lambda;
    A.mv_out = mv_out;
    A.cost_out = cost_out;
    A.mode_out = mode_out;
    A.dc_out = dc_out;
    A.split_out = split_out;
    A.sbcost_out = sbcost_out;
    const size_t need = batch_bytes(g, A, nullptr, nullptr, nullptr, nullptr);
    if (!workspace) {
        rc = library_scratch(need, stream, &workspace);
        if (rc) return rc;
    } else if (ws_bytes < need) {
        return DGPU_ERR_NOMEM;
    }
    return run_batch(g, A, workspace, as_stream(stream));
}

extern "C" int dgpu_motion_estimate(int cformat, int w, int h, const dgpu_block_params* bp, int nref,
                                    const int16_t* const* pic, const int16_t* const* ref1,
                                    const int16_t* const* ref2, int luma_depth, float lambda, int stages,
                                    int16_t* mv_out, float* cost_out, uint8_t* mode_out, int16_t* dc_out,
                                    uint8_t* split_out, float* sbcost_out, void* workspace, size_t ws_bytes,
                                    void* stream) {
    if (!pic || !ref1 || (nref == 2 && !ref2) || nref < 1 || nref > 2) return DGPU_ERR_ARG;
    const int16_t* pics[9] = {pic[0], pic[1], pic[2], ref1[0], ref1[1], ref1[2],
                              nref == 2 ? ref2[0] : nullptr, nref == 2 ? ref2[1] : nullptr,
                              nref == 2 ? ref2[2] : nullptr};
    const int task_pic = 0, task_ref1 = 1, task_ref2 = nref == 2 ? 2 : -1;
    return dgpu_motion_estimate_batch(cformat, w, h, bp, luma_depth, nref == 2 ? 3 : 2, pics, 1, &task_pic,
                                      &task_ref1, &task_ref2, &lambda, stages, &mv_out, &cost_out, &mode_out, &dc_out,
                                      &split_out, &sbcost_out, workspace, ws_bytes, stream);
}
