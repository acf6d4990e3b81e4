// Integer lifting wavelet transform (all Dirac filters), forward and inverse, for sm_100a.
//
// Replaces WaveletTransform::Transform and the VHFilter*::Split / Synth family
// (libdirac_common/wavelet_utils.cpp:440-1567).
//
// Design.  One launch per decomposition level covers every component / picture of a
// call (a job table in the kernel parameters maps CTAs to (job, tile)).  A CTA owns a
// TX x TY tile of the level region in the interleaved (pre-Mallat) domain.  It stages
// the tile plus an 8-sample halo on every side in shared memory, runs all lifting steps
// of both directions there, and scatters the result straight into the four Mallat
// quadrants (forward) or into natural order (inverse).  The halo covers the widest
// lifting reach (6 samples, DD13_7), so tiles are independent and each level reads its
// input and writes its output exactly once from HBM.  The reference's irregular edge
// formulas are all one rule -- a neighbour index is clamped inside its own parity
// subsequence -- which the kernel applies with global coordinates, so edge tiles need no
// special code.  Level 1 reads the int16 picture and applies the reference's
// replicate-padding and ShiftRowLeft on load; the inverse applies ShiftRowRight and the
// truncating int16 cast on store.  The low-pass band of every level but the last goes to
// a scratch buffer (ping-pong between two regions), which the next level reads.
//
// Shared-memory layout: rows of SP = SW + 1 int32 (odd pitch), so that consecutive
// threads walking consecutive rows (horizontal lifting) or consecutive columns (vertical
// lifting) hit distinct banks.

#include <new>

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int TX = 64;          // tile width  (interleaved samples, even)
constexpr int TY = 32;          // tile height (even)
constexpr int HALO = 8;         // >= widest lifting reach (6), even
constexpr int SW = TX + 2 * HALO;
constexpr int SH = TY + 2 * HALO;
constexpr int SP = SW + 1;      // odd pitch: conflict-free row and column walks
constexpr int NTHREADS = 256;
constexpr int MAXJ = 32;        // jobs per launch (kernel parameter table)

enum Kind { K_SHIFT2 = 0, K_FOURTAP = 1, K_97 = 2, K_HAAR = 3 };

// One level of one component.
struct LevelJob {
    const int16_t* in16;   // forward level 1: int16 picture (replicate-padded on load)
    const int32_t* in32;   // forward level > 1: low-pass band of the previous level
    int in_stride;
    int32_t* coeff;        // Mallat coefficient array (high-pass bands live here)
    int coeff_stride;
    int32_t* ll;           // forward: low-pass destination; inverse: low-pass source
    int ll_stride;
    int16_t* out16;        // inverse level 1: int16 picture (truncating store)
    int32_t* out32;        // inverse level > 1: synthesised region (next level's low-pass)
    int out_stride;
    int w, h;              // true picture size (level 1)
    int xl, yl;            // level region (interleaved domain), even
    int filter;
    int tiles_x;
    int tile_begin;
};

struct LevelJobs {
    int njobs;
    LevelJob job[MAXJ];
};

// Lifting update for one target given its neighbours (libdirac_common/wavelet_utils.h:490-616).
template <int PAR, int KIND, int SH_, int T1, int T2, int G>
__device__ __forceinline__ int lift_delta(int a, int b, int c, int e) {
    if constexpr (KIND == K_SHIFT2) {
        return (a + b + (1 << (SH_ - 1))) >> SH_;
    } else if constexpr (KIND == K_FOURTAP) {
        return (T1 * (a + b) + T2 * (c + e) + (1 << (SH_ - 1))) >> SH_;
    } else if constexpr (KIND == K_97) {
        return (G * (a + b)) >> 12;
    } else {
        return PAR ? a : ((b + 1) >> 1);
    }
}

// One lifting step along AXIS (0: along x within rows, 1: along y within columns) for the
// lines [l0, l1) of the orthogonal axis.  g0 = global coordinate (along AXIS) of shared
// index 0 (even); n = region length along AXIS; len = shared extent along AXIS.
// Targets k = 2m + PAR; neighbours are the other parity at subsequence indices
// m-1+PAR, m+PAR (near) and m-2+PAR, m+1+PAR (far), clamped to [0, n/2 - 1].  Targets
// whose neighbours fall outside shared memory are skipped: they lie in the halo, at a
// distance from the tile that no later step's reach crosses.
template <int AXIS, int PAR, int SIGN, int KIND, int SH_, int T1, int T2, int G>
__device__ __forceinline__ void lift_pass(int32_t* s, int len, int g0, int n, int l0, int l1) {
    const int nlines = l1 - l0;
    const int half_len = len >> 1;
    const int total = nlines * half_len;
    const int nh = n >> 1;
    constexpr int OTH = 1 - PAR;
    for (int idx = threadIdx.x; idx < total; idx += NTHREADS) {
        const int line = l0 + idx % nlines;
        const int mm = idx / nlines;
        const int c = 2 * mm + PAR;
        const int g = g0 + c;
        if (g < 0 || g >= n) continue;
        const int m = g >> 1;
        const int ca = 2 * clampi(m - 1 + PAR, 0, nh - 1) + OTH - g0;
        const int cb = 2 * clampi(m + PAR, 0, nh - 1) + OTH - g0;
        int cc = ca, ce = cb;
        if constexpr (KIND == K_FOURTAP) {
            cc = 2 * clampi(m - 2 + PAR, 0, nh - 1) + OTH - g0;
            ce = 2 * clampi(m + 1 + PAR, 0, nh - 1) + OTH - g0;
        }
        const int lo = min(min(ca, cb), min(cc, ce));
        const int hi = max(max(ca, cb), max(cc, ce));
        if (lo < 0 || hi >= len) continue;
        auto at = [&](int pos) -> int32_t& {
            return AXIS == 0 ? s[line * SP + pos] : s[pos * SP + line];
        };
        const int a = at(ca), b = at(cb);
        int cv = 0, ev = 0;
        if constexpr (KIND == K_FOURTAP) {
            cv = at(cc);
            ev = at(ce);
        }
        const int d = lift_delta<PAR, KIND, SH_, T1, T2, G>(a, b, cv, ev);
        int32_t& t = at(c);
        t = (SIGN < 0) ? (t - d) : (t + d);
    }
}

// Per-filter analysis (Split) and synthesis (Synth) step sequences.
//   DD9_7     wavelet_utils.cpp:952-1133     LEGALL5_3 :805-949     DD13_7 :1136-1339
//   HAAR0/1   :1342-1489                     DAUB9_7   :575-800 (also FIDELITY / unknown)
template <int F>
struct Filter;

template <>
struct Filter<DGPU_DD9_7> {
    static constexpr int SHIFT = 1;
    template <int AX>
    __device__ static void analysis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 1, -1, K_FOURTAP, 4, 9, -1, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 0, +1, K_SHIFT2, 2, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
    template <int AX>
    __device__ static void synthesis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 0, -1, K_SHIFT2, 2, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 1, +1, K_FOURTAP, 4, 9, -1, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
};

template <>
struct Filter<DGPU_LEGALL5_3> {
    static constexpr int SHIFT = 1;
    template <int AX>
    __device__ static void analysis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 1, -1, K_SHIFT2, 1, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 0, +1, K_SHIFT2, 2, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
    template <int AX>
    __device__ static void synthesis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 0, -1, K_SHIFT2, 2, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 1, +1, K_SHIFT2, 1, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
};

template <>
struct Filter<DGPU_DD13_7> {
    static constexpr int SHIFT = 1;
    template <int AX>
    __device__ static void analysis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 1, -1, K_FOURTAP, 4, 9, -1, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 0, +1, K_FOURTAP, 5, 9, -1, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
    template <int AX>
    __device__ static void synthesis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 0, -1, K_FOURTAP, 5, 9, -1, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 1, +1, K_FOURTAP, 4, 9, -1, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
};

template <int SHIFTBITS>
struct HaarFilter {
    static constexpr int SHIFT = SHIFTBITS;
    template <int AX>
    __device__ static void analysis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 1, -1, K_HAAR, 0, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 0, +1, K_HAAR, 0, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
    template <int AX>
    __device__ static void synthesis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 0, -1, K_HAAR, 0, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 1, +1, K_HAAR, 0, 0, 0, 0>(s, len, g0, n, l0, l1); __syncthreads();
    }
};
template <> struct Filter<DGPU_HAAR0> : HaarFilter<0> {};
template <> struct Filter<DGPU_HAAR1> : HaarFilter<1> {};

template <>
struct Filter<DGPU_DAUB9_7> {
    static constexpr int SHIFT = 1;
    template <int AX>
    __device__ static void analysis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 1, -1, K_97, 0, 0, 0, 6497>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 0, -1, K_97, 0, 0, 0, 217>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 1, +1, K_97, 0, 0, 0, 3616>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 0, +1, K_97, 0, 0, 0, 1817>(s, len, g0, n, l0, l1); __syncthreads();
    }
    template <int AX>
    __device__ static void synthesis(int32_t* s, int len, int g0, int n, int l0, int l1) {
        lift_pass<AX, 0, -1, K_97, 0, 0, 0, 1817>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 1, -1, K_97, 0, 0, 0, 3616>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 0, +1, K_97, 0, 0, 0, 217>(s, len, g0, n, l0, l1); __syncthreads();
        lift_pass<AX, 1, +1, K_97, 0, 0, 0, 6497>(s, len, g0, n, l0, l1); __syncthreads();
    }
};

__device__ __forceinline__ int find_job(const LevelJobs& jobs, int tile) {
    int j = 0;
    while (j + 1 < jobs.njobs && jobs.job[j + 1].tile_begin <= tile) ++j;
    return j;
}

// ---- forward level ------------------------------------------------------------------

template <int F>
__device__ void forward_tile(int32_t* s, const LevelJob& jb, int tx0, int ty0) {
    using Flt = Filter<F>;
    const int gx0 = tx0 - HALO, gy0 = ty0 - HALO;
    // Stage the tile + halo.  Level 1 reads the int16 picture with the reference's
    // replicate padding (wavelet_utils.cpp:451-460); every level applies ShiftRowLeft.
    for (int idx = threadIdx.x; idx < SH * SW; idx += NTHREADS) {
        const int r = idx / SW, c = idx - r * SW;
        const int gy = gy0 + r, gx = gx0 + c;
        if (gy < 0 || gy >= jb.yl || gx < 0 || gx >= jb.xl) continue;
        int v;
        if (jb.in16) {
            v = jb.in16[(size_t)min(gy, jb.h - 1) * jb.in_stride + min(gx, jb.w - 1)];
        } else {
            v = jb.in32[(size_t)gy * jb.in_stride + gx];
        }
        s[r * SP + c] = (int32_t)((uint32_t)v << Flt::SHIFT);
    }
    __syncthreads();
    // Horizontal lifting on every staged row (the vertical steps need the halo rows),
    // then vertical lifting on the tile's own columns.
    Flt::template analysis<0>(s, SW, gx0, jb.xl, 0, SH);
    Flt::template analysis<1>(s, SH, gy0, jb.yl, HALO, HALO + TX);
    // Scatter into the Mallat quadrants (VHFilter::DeInterleave, wavelet_utils.cpp:540-573).
    const int xl2 = jb.xl >> 1, yl2 = jb.yl >> 1;
    for (int idx = threadIdx.x; idx < TY * (TX / 2); idx += NTHREADS) {
        const int r = idx / (TX / 2), i = idx - r * (TX / 2);
        const int gy = ty0 + r, gx = tx0 + 2 * i;
        if (gy >= jb.yl || gx >= jb.xl) continue;
        const int32_t ev = s[(HALO + r) * SP + HALO + 2 * i];
        const int32_t od = s[(HALO + r) * SP + HALO + 2 * i + 1];
        const int ox = gx >> 1;
        if ((gy & 1) == 0) {
            const int oy = gy >> 1;
            jb.ll[(size_t)oy * jb.ll_stride + ox] = ev;
            jb.coeff[(size_t)oy * jb.coeff_stride + xl2 + ox] = od;
        } else {
            const int oy = yl2 + (gy >> 1);
            jb.coeff[(size_t)oy * jb.coeff_stride + ox] = ev;
            jb.coeff[(size_t)oy * jb.coeff_stride + xl2 + ox] = od;
        }
    }
}

__global__ void __launch_bounds__(NTHREADS) dwt_forward_level_kernel(const __grid_constant__ LevelJobs jobs) {
    __shared__ int32_t s[SH * SP];
    const int j = find_job(jobs, blockIdx.x);
    const LevelJob& jb = jobs.job[j];
    const int t = blockIdx.x - jb.tile_begin;
    const int ty = t / jb.tiles_x, tx = t - ty * jb.tiles_x;
    const int tx0 = tx * TX, ty0 = ty * TY;
    switch (jb.filter) {
        case DGPU_DD9_7: forward_tile<DGPU_DD9_7>(s, jb, tx0, ty0); break;
        case DGPU_LEGALL5_3: forward_tile<DGPU_LEGALL5_3>(s, jb, tx0, ty0); break;
        case DGPU_DD13_7: forward_tile<DGPU_DD13_7>(s, jb, tx0, ty0); break;
        case DGPU_HAAR0: forward_tile<DGPU_HAAR0>(s, jb, tx0, ty0); break;
        case DGPU_HAAR1: forward_tile<DGPU_HAAR1>(s, jb, tx0, ty0); break;
        default: forward_tile<DGPU_DAUB9_7>(s, jb, tx0, ty0); break;
    }
}

// ---- inverse level ------------------------------------------------------------------

template <int F>
__device__ void inverse_tile(int32_t* s, const LevelJob& jb, int tx0, int ty0) {
    using Flt = Filter<F>;
    const int gx0 = tx0 - HALO, gy0 = ty0 - HALO;
    const int xl2 = jb.xl >> 1, yl2 = jb.yl >> 1;
    // Gather from the Mallat quadrants into interleaved order (VHFilter::Interleave,
    // wavelet_utils.cpp:491-523); the low-pass quadrant comes from jb.ll.
    for (int idx = threadIdx.x; idx < SH * SW; idx += NTHREADS) {
        const int r = idx / SW, c = idx - r * SW;
        const int gy = gy0 + r, gx = gx0 + c;
        if (gy < 0 || gy >= jb.yl || gx < 0 || gx >= jb.xl) continue;
        const int qy = gy >> 1, qx = gx >> 1;
        int32_t v;
        if (((gx | gy) & 1) == 0) {
            v = jb.ll[(size_t)qy * jb.ll_stride + qx];
        } else {
            v = jb.coeff[(size_t)((gy & 1) * yl2 + qy) * jb.coeff_stride + (gx & 1) * xl2 + qx];
        }
        s[r * SP + c] = v;
    }
    __syncthreads();
    // Vertical synthesis on every staged column, then horizontal on the tile's own rows.
    Flt::template synthesis<1>(s, SH, gy0, jb.yl, 0, SW);
    Flt::template synthesis<0>(s, SW, gx0, jb.xl, HALO, HALO + TY);
    // ShiftRowRight and store in natural order.
    for (int idx = threadIdx.x; idx < TY * TX; idx += NTHREADS) {
        const int r = idx / TX, c = idx - r * TX;
        const int gy = ty0 + r, gx = tx0 + c;
        int32_t v = s[(HALO + r) * SP + HALO + c];
        if constexpr (Flt::SHIFT > 0) v = (v + (1 << (Flt::SHIFT - 1))) >> Flt::SHIFT;
        if (jb.out16) {
            if (gy < jb.h && gx < jb.w) jb.out16[(size_t)gy * jb.out_stride + gx] = (int16_t)v;
        } else if (gy < jb.yl && gx < jb.xl) {
            jb.out32[(size_t)gy * jb.out_stride + gx] = v;
        }
    }
}

__global__ void __launch_bounds__(NTHREADS) dwt_inverse_level_kernel(const __grid_constant__ LevelJobs jobs) {
    __shared__ int32_t s[SH * SP];
    const int j = find_job(jobs, blockIdx.x);
    const LevelJob& jb = jobs.job[j];
    const int t = blockIdx.x - jb.tile_begin;
    const int ty = t / jb.tiles_x, tx = t - ty * jb.tiles_x;
    const int tx0 = tx * TX, ty0 = ty * TY;
    switch (jb.filter) {
        case DGPU_DD9_7: inverse_tile<DGPU_DD9_7>(s, jb, tx0, ty0); break;
        case DGPU_LEGALL5_3: inverse_tile<DGPU_LEGALL5_3>(s, jb, tx0, ty0); break;
        case DGPU_DD13_7: inverse_tile<DGPU_DD13_7>(s, jb, tx0, ty0); break;
        case DGPU_HAAR0: inverse_tile<DGPU_HAAR0>(s, jb, tx0, ty0); break;
        case DGPU_HAAR1: inverse_tile<DGPU_HAAR1>(s, jb, tx0, ty0); break;
        default: inverse_tile<DGPU_DAUB9_7>(s, jb, tx0, ty0); break;
    }
}

// ---- host side --------------------------------------------------------------------------

int normalise_filter(int f) {
    switch (f) {
        case DGPU_DD9_7: case DGPU_LEGALL5_3: case DGPU_DD13_7: case DGPU_HAAR0: case DGPU_HAAR1:
            return f;
        default:
            return DGPU_DAUB9_7;
    }
}

int min_level_len(int f) {
    switch (normalise_filter(f)) {
        case DGPU_DD9_7: case DGPU_DD13_7: return 6;
        case DGPU_HAAR0: case DGPU_HAAR1: return 2;
        default: return 4;
    }
}

// The two low-pass scratch regions of one transform: A holds levels 1, 3, 5.. (forward)
// and the outputs of synthesis levels 2, 4, ..; B the others.
struct ScratchSplit {
    int32_t* a;
    int32_t* b;
};

size_t scratch_a_elems(int cw, int ch) { return (size_t)(cw / 2) * (ch / 2); }
size_t scratch_b_elems(int cw, int ch) { return (size_t)(cw / 4) * (ch / 4); }

struct Entry {
    int filter, depth;
    int16_t* pic;
    int w, h, pic_stride;
    int32_t* coeff;
    int cw, ch, coeff_stride;
    ScratchSplit scr;
};

int validate(const Entry& e) {
    if (!e.pic || !e.coeff) return DGPU_ERR_ARG;
    if (e.depth < 1 || e.depth > 10) return DGPU_ERR_SIZE;
    if (e.w <= 0 || e.h <= 0 || e.w > e.cw || e.h > e.ch) return DGPU_ERR_SIZE;
    const int mul = 1 << e.depth;
    if (e.cw % mul || e.ch % mul) return DGPU_ERR_SIZE;
    const int minlen = min_level_len(e.filter);
    if ((e.cw >> (e.depth - 1)) < minlen || (e.ch >> (e.depth - 1)) < minlen) return DGPU_ERR_SIZE;
    if (e.pic_stride < e.w || e.coeff_stride < e.cw) return DGPU_ERR_ARG;
    return DGPU_OK;
}

int launch_jobs(bool forward, LevelJobs& jobs, int& total_tiles, cudaStream_t st) {
    if (jobs.njobs == 0) return DGPU_OK;
    if (forward) {
        dwt_forward_level_kernel<<<total_tiles, NTHREADS, 0, st>>>(jobs);
    } else {
        dwt_inverse_level_kernel<<<total_tiles, NTHREADS, 0, st>>>(jobs);
    }
    DGPU_CHECK_LAUNCH();
    jobs.njobs = 0;
    total_tiles = 0;
    return DGPU_OK;
}

int add_job(bool forward, LevelJobs& jobs, int& total_tiles, const LevelJob& jb, cudaStream_t st) {
    if (jobs.njobs == MAXJ) {
        int rc = launch_jobs(forward, jobs, total_tiles, st);
        if (rc) return rc;
    }
    LevelJob j = jb;
    j.tiles_x = (j.xl + TX - 1) / TX;
    const int tiles_y = (j.yl + TY - 1) / TY;
    j.tile_begin = total_tiles;
    total_tiles += j.tiles_x * tiles_y;
    jobs.job[jobs.njobs++] = j;
    return DGPU_OK;
}

int run_entries(int direction, Entry* e, int n, cudaStream_t st) {
    int maxd = 0;
    for (int i = 0; i < n; ++i) maxd = e[i].depth > maxd ? e[i].depth : maxd;
    LevelJobs jobs;
    jobs.njobs = 0;
    int total_tiles = 0;
    const bool fwd = direction == DGPU_FORWARD;
    if (fwd) {
        for (int l = 1; l <= maxd; ++l) {
            for (int i = 0; i < n; ++i) {
                const Entry& E = e[i];
                if (l > E.depth) continue;
                LevelJob jb = {};
                jb.xl = E.cw >> (l - 1);
                jb.yl = E.ch >> (l - 1);
                jb.w = E.w;
                jb.h = E.h;
                jb.filter = normalise_filter(E.filter);
                jb.coeff = E.coeff;
                jb.coeff_stride = E.coeff_stride;
                if (l == 1) {
                    jb.in16 = E.pic;
                    jb.in_stride = E.pic_stride;
                } else {
                    jb.in32 = ((l - 1) & 1) ? E.scr.a : E.scr.b;
                    jb.in_stride = jb.xl;
                }
                if (l == E.depth) {
                    jb.ll = E.coeff;
                    jb.ll_stride = E.coeff_stride;
                } else {
                    jb.ll = (l & 1) ? E.scr.a : E.scr.b;
                    jb.ll_stride = jb.xl >> 1;
                }
                int rc = add_job(true, jobs, total_tiles, jb, st);
                if (rc) return rc;
            }
            int rc = launch_jobs(true, jobs, total_tiles, st);
            if (rc) return rc;
        }
    } else {
        for (int l = maxd; l >= 1; --l) {
            for (int i = 0; i < n; ++i) {
                const Entry& E = e[i];
                if (l > E.depth) continue;
                LevelJob jb = {};
                jb.xl = E.cw >> (l - 1);
                jb.yl = E.ch >> (l - 1);
                jb.w = E.w;
                jb.h = E.h;
                jb.filter = normalise_filter(E.filter);
                jb.coeff = E.coeff;
                jb.coeff_stride = E.coeff_stride;
                if (l == E.depth) {
                    jb.ll = E.coeff;
                    jb.ll_stride = E.coeff_stride;
                } else {
                    // low-pass = output of synthesis level l+1
                    jb.ll = ((l + 1) & 1) ? E.scr.b : E.scr.a;
                    jb.ll_stride = jb.xl >> 1;
                }
                if (l == 1) {
                    jb.out16 = E.pic;
                    jb.out_stride = E.pic_stride;
                } else {
                    jb.out32 = (l & 1) ? E.scr.b : E.scr.a;
                    jb.out_stride = jb.xl;
                }
                int rc = add_job(false, jobs, total_tiles, jb, st);
                if (rc) return rc;
            }
            int rc = launch_jobs(false, jobs, total_tiles, st);
            if (rc) return rc;
        }
    }
    return DGPU_OK;
}

size_t entry_scratch_bytes(int cw, int ch) {
    return align_up(scratch_a_elems(cw, ch) * 4, 256) + align_up(scratch_b_elems(cw, ch) * 4, 256);
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" size_t dgpu_dwt_scratch_bytes(int cw, int ch, int depth) {
    if (cw <= 0 || ch <= 0 || depth < 1) return 0;
    return entry_scratch_bytes(cw, ch);
}

extern "C" int dgpu_wavelet_transform_batch(int direction, int n, const int* filter, const int* depth,
                                            int16_t* const* pic, const int* w, const int* h,
                                            const int* pic_stride, int32_t* const* coeff, const int* cw,
                                            const int* ch, const int* coeff_stride, void* scratch,
                                            size_t scratch_bytes, void* stream) {
    if (n <= 0 || !filter || !depth || !pic || !w || !h || !pic_stride || !coeff || !cw || !ch || !coeff_stride)
        return DGPU_ERR_ARG;
    if (direction != DGPU_FORWARD && direction != DGPU_BACKWARD) return DGPU_ERR_ARG;
    Entry* e = new (std::nothrow) Entry[n];
    if (!e) return DGPU_ERR_NOMEM;
    size_t need = 0;
    int rc = DGPU_OK;
    for (int i = 0; i < n && rc == DGPU_OK; ++i) {
        e[i] = Entry{filter[i], depth[i], pic[i], w[i], h[i], pic_stride[i], coeff[i], cw[i], ch[i], coeff_stride[i], {}};
        rc = validate(e[i]);
        need += entry_scratch_bytes(cw[i], ch[i]);
    }
    if (rc == DGPU_OK) {
        if (!scratch) {
            rc = library_scratch(need, &scratch);
        } else if (scratch_bytes < need) {
            rc = DGPU_ERR_NOMEM;
        }
    }
    if (rc == DGPU_OK) {
        char* p = static_cast<char*>(scratch);
        for (int i = 0; i < n; ++i) {
            e[i].scr.a = reinterpret_cast<int32_t*>(p);
            p += align_up(scratch_a_elems(e[i].cw, e[i].ch) * 4, 256);
            e[i].scr.b = reinterpret_cast<int32_t*>(p);
            p += align_up(scratch_b_elems(e[i].cw, e[i].ch) * 4, 256);
        }
        rc = run_entries(direction, e, n, as_stream(stream));
    }
    delete[] e;
    return rc;
}

extern "C" int dgpu_wavelet_transform(int direction, int filter, int depth, int16_t* pic, int w, int h,
                                      int pic_stride, int32_t* coeff, int cw, int ch, int coeff_stride,
                                      void* scratch, size_t scratch_bytes, void* stream) {
    return dgpu_wavelet_transform_batch(direction, 1, &filter, &depth, &pic, &w, &h, &pic_stride, &coeff, &cw,
                                        &ch, &coeff_stride, scratch, scratch_bytes, stream);
}

extern "C" int dgpu_wavelet_transform_host(int direction, int filter, int depth, int16_t* pic, int w, int h,
                                           int pic_stride, int32_t* coeff, int cw, int ch, int coeff_stride) {
    if (!pic || !coeff || pic_stride < w || coeff_stride < cw || w <= 0 || h <= 0 || cw <= 0 || ch <= 0)
        return DGPU_ERR_ARG;
    int16_t* dpic = nullptr;
    int32_t* dcoeff = nullptr;
    const size_t pic_bytes = (size_t)h * pic_stride * sizeof(int16_t);
    const size_t coeff_bytes = (size_t)ch * coeff_stride * sizeof(int32_t);
    int rc = DGPU_OK;
    if (cudaMalloc(&dpic, pic_bytes) != cudaSuccess || cudaMalloc(&dcoeff, coeff_bytes) != cudaSuccess) {
        rc = DGPU_ERR_NOMEM;
    }
    if (rc == DGPU_OK) {
        cudaError_t ce = (direction == DGPU_FORWARD) ? cudaMemcpy(dpic, pic, pic_bytes, cudaMemcpyHostToDevice)
                                                     : cudaMemcpy(dcoeff, coeff, coeff_bytes, cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) rc = DGPU_ERR_CUDA;
    }
    if (rc == DGPU_OK)
        rc = dgpu_wavelet_transform(direction, filter, depth, dpic, w, h, pic_stride, dcoeff, cw, ch, coeff_stride,
                                    nullptr, 0, nullptr);
    if (rc == DGPU_OK) {
        cudaError_t ce = (direction == DGPU_FORWARD) ? cudaMemcpy(coeff, dcoeff, coeff_bytes, cudaMemcpyDeviceToHost)
                                                     : cudaMemcpy(pic, dpic, pic_bytes, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) rc = DGPU_ERR_CUDA;
    }
    cudaFree(dpic);
    cudaFree(dcoeff);
    return rc;
}
