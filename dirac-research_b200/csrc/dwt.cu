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

#include <mutex>
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

// A lifting step as a type, so that step sequences can drive both the shared-memory and
// the register code paths.
template <int PAR_, int SIGN_, int KIND_, int SH__, int T1_, int T2_, int G_>
struct Step {
    static constexpr int PAR = PAR_, SIGN = SIGN_, KIND = KIND_, SHF = SH__, T1 = T1_, T2 = T2_, G = G_;
};
template <class S>
using Inv = Step<S::PAR, -S::SIGN, S::KIND, S::SHF, S::T1, S::T2, S::G>;
template <class... S>
struct Steps {};

// Per-filter analysis (Split) step sequences; synthesis (Synth) runs them in reverse with the
// opposite sign.
//   DD9_7     wavelet_utils.cpp:952-1133     LEGALL5_3 :805-949     DD13_7 :1136-1339
//   HAAR0/1   :1342-1489                     DAUB9_7   :575-800 (also FIDELITY / unknown)
template <int F>
struct Filter;

template <>
struct Filter<DGPU_DD9_7> {
    static constexpr int SHIFT = 1;
    using S1 = Step<1, -1, K_FOURTAP, 4, 9, -1, 0>;
    using S2 = Step<0, +1, K_SHIFT2, 2, 0, 0, 0>;
    using Analysis = Steps<S1, S2>;
    using Synthesis = Steps<Inv<S2>, Inv<S1>>;
};

template <>
struct Filter<DGPU_LEGALL5_3> {
    static constexpr int SHIFT = 1;
    using S1 = Step<1, -1, K_SHIFT2, 1, 0, 0, 0>;
    using S2 = Step<0, +1, K_SHIFT2, 2, 0, 0, 0>;
    using Analysis = Steps<S1, S2>;
    using Synthesis = Steps<Inv<S2>, Inv<S1>>;
};

template <>
struct Filter<DGPU_DD13_7> {
    static constexpr int SHIFT = 1;
    using S1 = Step<1, -1, K_FOURTAP, 4, 9, -1, 0>;
    using S2 = Step<0, +1, K_FOURTAP, 5, 9, -1, 0>;
    using Analysis = Steps<S1, S2>;
    using Synthesis = Steps<Inv<S2>, Inv<S1>>;
};

template <int SHIFTBITS>
struct HaarFilter {
    static constexpr int SHIFT = SHIFTBITS;
    using S1 = Step<1, -1, K_HAAR, 0, 0, 0, 0>;
    using S2 = Step<0, +1, K_HAAR, 0, 0, 0, 0>;
    using Analysis = Steps<S1, S2>;
    using Synthesis = Steps<Inv<S2>, Inv<S1>>;
};
template <> struct Filter<DGPU_HAAR0> : HaarFilter<0> {};
template <> struct Filter<DGPU_HAAR1> : HaarFilter<1> {};

template <>
struct Filter<DGPU_DAUB9_7> {
    static constexpr int SHIFT = 1;
    using S1 = Step<1, -1, K_97, 0, 0, 0, 6497>;
    using S2 = Step<0, -1, K_97, 0, 0, 0, 217>;
    using S3 = Step<1, +1, K_97, 0, 0, 0, 3616>;
    using S4 = Step<0, +1, K_97, 0, 0, 0, 1817>;
    using Analysis = Steps<S1, S2, S3, S4>;
    using Synthesis = Steps<Inv<S4>, Inv<S3>, Inv<S2>, Inv<S1>>;
};

// Shared-memory path: every step is one pass over the tile followed by a barrier.
template <int AX, class... S>
__device__ __forceinline__ void run_smem(Steps<S...>, int32_t* s, int len, int g0, int n, int l0, int l1) {
    ((lift_pass<AX, S::PAR, S::SIGN, S::KIND, S::SHF, S::T1, S::T2, S::G>(s, len, g0, n, l0, l1),
      __syncthreads()),
     ...);
}

// Register path: a thread holds a segment of N consecutive samples of one line (SEG_HALO
// halo samples on each side of its outputs).  All indices are compile-time.  A segment that
// starts at the region's first sample (lo) or ends at its last (hi) holds SEG_HALO samples
// outside the region; after loading and after every step they are overwritten with the
// sample the reference's edge rule reads instead (the nearest in-region sample of the same
// parity), which makes the in-region results identical to the clamped-index formulation.
constexpr int SEG_HALO = 6;

template <class S, int N>
__device__ __forceinline__ void lift_regs(int (&v)[N]) {
    constexpr int R = (S::KIND == K_FOURTAP) ? 3 : 1;
#pragma unroll
    for (int i = S::PAR; i < N; i += 2) {
        if (i - R < 0 || i + R >= N) continue;
        int d;
        if constexpr (S::KIND == K_FOURTAP) {
            d = lift_delta<S::PAR, S::KIND, S::SHF, S::T1, S::T2, S::G>(v[i - 1], v[i + 1], v[i - 3], v[i + 3]);
        } else {
            d = lift_delta<S::PAR, S::KIND, S::SHF, S::T1, S::T2, S::G>(v[i - 1], v[i + 1], 0, 0);
        }
        v[i] = (S::SIGN < 0) ? (v[i] - d) : (v[i] + d);
    }
}

template <int N>
__device__ __forceinline__ void repad(int (&v)[N], bool lo, bool hi) {
    if (lo) {
#pragma unroll
        for (int i = 0; i < SEG_HALO; ++i) v[i] = v[SEG_HALO + (i & 1)];
    }
    if (hi) {
#pragma unroll
        for (int j = 0; j < SEG_HALO; ++j) v[N - SEG_HALO + j] = v[N - SEG_HALO - 2 + (j & 1)];
    }
}

template <int N, class... S>
__device__ __forceinline__ void run_regs(Steps<S...>, int (&v)[N], bool lo, bool hi) {
    repad(v, lo, hi);
    ((lift_regs<S>(v), repad(v, lo, hi)), ...);
}

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
    run_smem<0>(typename Flt::Analysis{}, s, SW, gx0, jb.xl, 0, SH);
    run_smem<1>(typename Flt::Analysis{}, s, SH, gy0, jb.yl, HALO, HALO + TX);
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
    run_smem<1>(typename Flt::Synthesis{}, s, SH, gy0, jb.yl, 0, SW);
    run_smem<0>(typename Flt::Synthesis{}, s, SW, gx0, jb.xl, HALO, HALO + TY);
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

// ---- register-segment fast path (regions at least 64 x 64) ---------------------------
//
// A CTA owns a 64 x 64 tile (the last tile of a row / column is moved back to end exactly at
// the region's edge, overlapping its neighbour, so every tile is full and every edge lies at
// a fixed position inside a segment).  Each lifting direction is run by threads that each hold
// a 44-sample segment (32 outputs + a 6-sample halo on each side) of one line in registers.
// The first direction's segments are loaded straight from global memory (16-byte vector loads
// when the window is aligned and inside the picture, clamped scalar loads otherwise, so every
// load of a thread is in flight at once); its 32 outputs go to shared memory, where the second
// direction's segments are read from.  Forward: rows first, then columns stored straight into
// the Mallat quadrants.  Inverse: columns first (gathered from the quadrants), then rows.

constexpr int FT = 64;                    // tile side
constexpr int FH = 8;                     // halo lines above / left of the tile
constexpr int SEG = 32;                   // outputs per segment
constexpr int SEGN = SEG + 2 * SEG_HALO;  // registers per segment (44)
constexpr int FLINES = FT + 2 * FH;       // lines the first direction covers (80)
constexpr int FAST_THREADS = 2 * FLINES;  // 160: two segments per line
constexpr int FWD_P = FT + 1;             // forward shared pitch: 80 rows x 64 columns
constexpr int INV_P = FLINES + 1;         // inverse shared pitch: 64 rows x 80 columns

// Load the 44-sample window [x - 6, x + 38) of one row into v (converted to int, << shift).
// Columns are clamped to [0, xmax] and the row to [0, ymax]: in-region samples get the
// reference's replicate padding, out-of-region ones get don't-care values that the edge
// re-padding overwrites.
template <class T, int SHIFT>
__device__ __forceinline__ void load_row_window(int (&v)[SEGN], const T* base, int stride, int y, int ymax, int x,
                                                int xmax) {
    const T* row = base + (size_t)clampi(y, 0, ymax) * stride;
    constexpr int PER16 = 16 / sizeof(T);  // elements per 16-byte vector
    const int x8 = x - 8;                  // vector window [x - 8, x + 40)
    const bool vec = x8 >= 0 && x + 40 <= xmax + 1 && ((reinterpret_cast<uintptr_t>(row + x8) & 15) == 0);
    if (vec) {
        T w[48];
#pragma unroll
        for (int k = 0; k < 48 / PER16; ++k)
            *reinterpret_cast<int4*>(&w[k * PER16]) = *reinterpret_cast<const int4*>(row + x8 + k * PER16);
#pragma unroll
        for (int i = 0; i < SEGN; ++i) v[i] = (int)((uint32_t)(int)w[i + 2] << SHIFT);
    } else {
#pragma unroll
        for (int i = 0; i < SEGN; ++i) v[i] = (int)((uint32_t)(int)row[clampi(x - SEG_HALO + i, 0, xmax)] << SHIFT);
    }
}

template <int F>
__device__ void forward_fast(int32_t* s, const LevelJob& jb, int x0, int y0) {
    using Flt = Filter<F>;
    const int tid = threadIdx.x;
    // rows: 80 lines (the tile's 64 plus 8 above and below), two segments each
    {
        const int seg = tid / FLINES, r = tid - seg * FLINES;
        const int xs = x0 + SEG * seg;
        const int gy = y0 - FH + r;
        int v[SEGN];
        if (jb.in16) {
            load_row_window<int16_t, Flt::SHIFT>(v, jb.in16, jb.in_stride, gy, jb.h - 1, xs, jb.w - 1);
        } else {
            load_row_window<int32_t, Flt::SHIFT>(v, jb.in32, jb.in_stride, gy, jb.yl - 1, xs, jb.xl - 1);
        }
        run_regs(typename Flt::Analysis{}, v, xs == 0, xs + SEG == jb.xl);
        int32_t* dst = s + r * FWD_P + SEG * seg;
#pragma unroll
        for (int k = 0; k < SEG; ++k) dst[k] = v[SEG_HALO + k];
    }
    __syncthreads();
    // columns: the tile's 64, two segments each, stored straight into the Mallat quadrants
    if (tid < 2 * FT) {
        const int seg = tid / FT, c = tid - seg * FT;
        int v[SEGN];
        const int32_t* src = s + ((FH - SEG_HALO) + SEG * seg) * FWD_P + c;
#pragma unroll
        for (int i = 0; i < SEGN; ++i) v[i] = src[i * FWD_P];
        const int ys = y0 + SEG * seg;
        run_regs(typename Flt::Analysis{}, v, ys == 0, ys + SEG == jb.yl);
        const int gx = x0 + c;
        const int xl2 = jb.xl >> 1, yl2 = jb.yl >> 1;
        const int ox = gx >> 1;
        const bool odd_x = gx & 1;
        int32_t* even_row_dst = odd_x ? (jb.coeff + xl2 + ox) : (jb.ll + ox);
        const int even_row_stride = odd_x ? jb.coeff_stride : jb.ll_stride;
        int32_t* odd_row_dst = jb.coeff + (size_t)yl2 * jb.coeff_stride + (odd_x ? xl2 : 0) + ox;
#pragma unroll
        for (int k = 0; k < SEG; k += 2) {
            const int oy = (ys + k) >> 1;
            even_row_dst[(size_t)oy * even_row_stride] = v[SEG_HALO + k];
            odd_row_dst[(size_t)oy * jb.coeff_stride] = v[SEG_HALO + k + 1];
        }
    }
}

template <int F>
__device__ void inverse_fast(int32_t* s, const LevelJob& jb, int x0, int y0) {
    using Flt = Filter<F>;
    const int tid = threadIdx.x;
    const int xl2 = jb.xl >> 1, yl2 = jb.yl >> 1;
    // columns: 80 lines (the tile's 64 plus 8 left and right), gathered from the quadrants
    {
        const int seg = tid / FLINES, c = tid - seg * FLINES;
        const int gx = clampi(x0 - FH + c, 0, jb.xl - 1);
        const int qx = gx >> 1;
        // even rows come from LL (even column) or HL (odd column), odd rows from LH or HH
        const int32_t* even_src = (gx & 1) ? (jb.coeff + xl2 + qx) : (jb.ll + qx);
        const int even_stride = (gx & 1) ? jb.coeff_stride : jb.ll_stride;
        const int32_t* odd_src = jb.coeff + (size_t)yl2 * jb.coeff_stride + (gx & 1) * xl2 + qx;
        const int ys = y0 + SEG * seg;
        int v[SEGN];
#pragma unroll
        for (int i = 0; i < SEGN; ++i) {
            const int gy = clampi(ys - SEG_HALO + i, 0, jb.yl - 1);
            v[i] = (gy & 1) ? odd_src[(size_t)(gy >> 1) * jb.coeff_stride] : even_src[(size_t)(gy >> 1) * even_stride];
        }
        run_regs(typename Flt::Synthesis{}, v, ys == 0, ys + SEG == jb.yl);
        int32_t* dst = s + (SEG * seg) * INV_P + c;
#pragma unroll
        for (int k = 0; k < SEG; ++k) dst[k * INV_P] = v[SEG_HALO + k];
    }
    __syncthreads();
    // rows: the tile's 64, two segments each, then ShiftRowRight and the store
    if (tid < 2 * FT) {
        const int seg = tid / FT, r = tid - seg * FT;
        int v[SEGN];
        const int32_t* src = s + r * INV_P + (FH - SEG_HALO) + SEG * seg;
#pragma unroll
        for (int i = 0; i < SEGN; ++i) v[i] = src[i];
        const int xs = x0 + SEG * seg;
        run_regs(typename Flt::Synthesis{}, v, xs == 0, xs + SEG == jb.xl);
        int o[SEG];
#pragma unroll
        for (int k = 0; k < SEG; ++k) {
            int32_t x = v[SEG_HALO + k];
            if constexpr (Flt::SHIFT > 0) x = (x + (1 << (Flt::SHIFT - 1))) >> Flt::SHIFT;
            o[k] = x;
        }
        const int gy = y0 + r;
        if (jb.out16) {
            if (gy < jb.h) {
                int16_t* row = jb.out16 + (size_t)gy * jb.out_stride + xs;
                if (xs + SEG <= jb.w && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
#pragma unroll
                    for (int k = 0; k < SEG; k += 8) {
                        int4 q;
                        q.x = (int)(uint16_t)(int16_t)o[k] | ((int)(uint16_t)(int16_t)o[k + 1] << 16);
                        q.y = (int)(uint16_t)(int16_t)o[k + 2] | ((int)(uint16_t)(int16_t)o[k + 3] << 16);
                        q.z = (int)(uint16_t)(int16_t)o[k + 4] | ((int)(uint16_t)(int16_t)o[k + 5] << 16);
                        q.w = (int)(uint16_t)(int16_t)o[k + 6] | ((int)(uint16_t)(int16_t)o[k + 7] << 16);
                        *reinterpret_cast<int4*>(row + k) = q;
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < SEG; ++k)
                        if (xs + k < jb.w) row[k] = (int16_t)o[k];
                }
            }
        } else {
            int32_t* row = jb.out32 + (size_t)gy * jb.out_stride + xs;
            if ((reinterpret_cast<uintptr_t>(row) & 15) == 0) {
#pragma unroll
                for (int k = 0; k < SEG; k += 4)
                    *reinterpret_cast<int4*>(row + k) = make_int4(o[k], o[k + 1], o[k + 2], o[k + 3]);
            } else {
#pragma unroll
                for (int k = 0; k < SEG; ++k) row[k] = o[k];
            }
        }
    }
}

__device__ __forceinline__ void fast_tile_origin(const LevelJob& jb, int t, int& x0, int& y0) {
    const int ty = t / jb.tiles_x, tx = t - ty * jb.tiles_x;
    x0 = min(tx * FT, jb.xl - FT);
    y0 = min(ty * FT, jb.yl - FT);
}

__global__ void __launch_bounds__(FAST_THREADS) dwt_forward_fast_kernel(const __grid_constant__ LevelJobs jobs) {
    __shared__ int32_t s[FLINES * FWD_P];
    const int j = find_job(jobs, blockIdx.x);
    const LevelJob& jb = jobs.job[j];
    int x0, y0;
    fast_tile_origin(jb, blockIdx.x - jb.tile_begin, x0, y0);
    switch (jb.filter) {
        case DGPU_DD9_7: forward_fast<DGPU_DD9_7>(s, jb, x0, y0); break;
        case DGPU_LEGALL5_3: forward_fast<DGPU_LEGALL5_3>(s, jb, x0, y0); break;
        case DGPU_DD13_7: forward_fast<DGPU_DD13_7>(s, jb, x0, y0); break;
        case DGPU_HAAR0: forward_fast<DGPU_HAAR0>(s, jb, x0, y0); break;
        case DGPU_HAAR1: forward_fast<DGPU_HAAR1>(s, jb, x0, y0); break;
        default: forward_fast<DGPU_DAUB9_7>(s, jb, x0, y0); break;
    }
}

__global__ void __launch_bounds__(FAST_THREADS) dwt_inverse_fast_kernel(const __grid_constant__ LevelJobs jobs) {
    __shared__ int32_t s[FT * INV_P];
    const int j = find_job(jobs, blockIdx.x);
    const LevelJob& jb = jobs.job[j];
    int x0, y0;
    fast_tile_origin(jb, blockIdx.x - jb.tile_begin, x0, y0);
    switch (jb.filter) {
        case DGPU_DD9_7: inverse_fast<DGPU_DD9_7>(s, jb, x0, y0); break;
        case DGPU_LEGALL5_3: inverse_fast<DGPU_LEGALL5_3>(s, jb, x0, y0); break;
        case DGPU_DD13_7: inverse_fast<DGPU_DD13_7>(s, jb, x0, y0); break;
        case DGPU_HAAR0: inverse_fast<DGPU_HAAR0>(s, jb, x0, y0); break;
        case DGPU_HAAR1: inverse_fast<DGPU_HAAR1>(s, jb, x0, y0); break;
        default: inverse_fast<DGPU_DAUB9_7>(s, jb, x0, y0); break;
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

// Jobs of one level go to the register fast path when their region is at least one full
// tile in each direction, to the generic shared-memory path otherwise.
struct LevelBatch {
    LevelJobs fast, slow;
    int fast_tiles = 0, slow_tiles = 0;
    LevelBatch() { fast.njobs = slow.njobs = 0; }
};

int flush(bool forward, LevelBatch& b, bool fast_table, cudaStream_t st) {
    LevelJobs& jobs = fast_table ? b.fast : b.slow;
    int& tiles = fast_table ? b.fast_tiles : b.slow_tiles;
    if (jobs.njobs == 0) return DGPU_OK;
    if (fast_table) {
        if (forward) dwt_forward_fast_kernel<<<tiles, FAST_THREADS, 0, st>>>(jobs);
        else dwt_inverse_fast_kernel<<<tiles, FAST_THREADS, 0, st>>>(jobs);
    } else {
        if (forward) dwt_forward_level_kernel<<<tiles, NTHREADS, 0, st>>>(jobs);
        else dwt_inverse_level_kernel<<<tiles, NTHREADS, 0, st>>>(jobs);
    }
    DGPU_CHECK_LAUNCH();
    jobs.njobs = 0;
    tiles = 0;
    return DGPU_OK;
}

int launch_jobs(bool forward, LevelBatch& b, cudaStream_t st) {
    int rc = flush(forward, b, true, st);
    if (rc) return rc;
    return flush(forward, b, false, st);
}

// A side qualifies for the fast path when the tiles laid from 0 in steps of FT, with the last
// one moved back to end at the edge, leave every non-edge segment's halo inside the region.
bool fast_side(int n) { return n >= FT && (n % FT == 0 || n % FT >= SEG_HALO); }

int add_job(bool forward, LevelBatch& b, const LevelJob& jb, cudaStream_t st) {
    const bool fast = fast_side(jb.xl) && fast_side(jb.yl);
    LevelJobs& jobs = fast ? b.fast : b.slow;
    if (jobs.njobs == MAXJ) {
        int rc = flush(forward, b, fast, st);
        if (rc) return rc;
    }
    int& tiles = fast ? b.fast_tiles : b.slow_tiles;
    LevelJob j = jb;
    const int tw = fast ? FT : TX, th = fast ? FT : TY;
    j.tiles_x = (j.xl + tw - 1) / tw;
    const int tiles_y = (j.yl + th - 1) / th;
    j.tile_begin = tiles;
    tiles += j.tiles_x * tiles_y;
    jobs.job[jobs.njobs++] = j;
    return DGPU_OK;
}

int run_entries(int direction, Entry* e, int n, cudaStream_t st) {
    int maxd = 0;
    for (int i = 0; i < n; ++i) maxd = e[i].depth > maxd ? e[i].depth : maxd;
    LevelBatch batch;
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
                int rc = add_job(true, batch, jb, st);
                if (rc) return rc;
            }
            int rc = launch_jobs(true, batch, st);
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
                int rc = add_job(false, batch, jb, st);
                if (rc) return rc;
            }
            int rc = launch_jobs(false, batch, st);
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
            rc = library_scratch(need, stream, &scratch);
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

// ---------------------------------------------------------------------------------------------
// Allocation-free wavelet transform.
//
// Some callers cannot allocate device memory at the point where they transform: code running
// under a device-memory budget that is already fully reserved, host threads that must not
// synchronise the device (cudaMalloc / cudaFree may), or embedders whose allocator owns every
// device byte.  dgpu_wavelet_transform_static serves them: the low-pass intermediates live in
// the fixed array below, so the call needs neither a caller scratch buffer nor the library's
// growable one.  The array costs DGPU_DWT_STATIC_SCRATCH_BYTES of memory on every GPU that
// loads this library, for as long as the process lives.
//
// The array is shared by all calls on a device and keeps whatever the last call left in it.
// Every level writes its low-pass band before the next level reads it, so nothing in it has
// to start at zero.  Calls whose kernels overlap on the GPU (on different streams, or from
// different host threads) race on the array and corrupt each other's results: serialise them.
// ---------------------------------------------------------------------------------------------

static __device__ __align__(256) unsigned char g_dwt_static_scratch[DGPU_DWT_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
void* g_static_scratch_addr[kStaticMaxDevices] = {};
}  // namespace

// Device address of g_dwt_static_scratch on the current device; looked up once per device
// (the host-side name of a __device__ array is not a device address).
static int static_scratch_address(void** out) {
    int dev = 0;
    DGPU_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kStaticMaxDevices) return DGPU_ERR_DEVICE;
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_scratch_addr[dev]) {
        void* p = nullptr;
        DGPU_CHECK_CUDA(cudaGetSymbolAddress(&p, g_dwt_static_scratch));
        g_static_scratch_addr[dev] = p;
    }
    *out = g_static_scratch_addr[dev];
    return DGPU_OK;
}

extern "C" int dgpu_wavelet_transform_static(int direction, int filter, int depth, int16_t* pic, int w, int h,
                                             int pic_stride, int32_t* coeff, int cw, int ch, int coeff_stride,
                                             void* stream) {
    if (direction != DGPU_FORWARD && direction != DGPU_BACKWARD) return DGPU_ERR_ARG;
    Entry e{filter, depth, pic, w, h, pic_stride, coeff, cw, ch, coeff_stride, {}};
    int rc = validate(e);
    if (rc) return rc;
    const size_t need = entry_scratch_bytes(cw, ch);
    if (need > DGPU_DWT_STATIC_SCRATCH_BYTES) return DGPU_ERR_SIZE;
    void* base = nullptr;
    rc = static_scratch_address(&base);
    if (rc) return rc;
    char* p = static_cast<char*>(base);
    e.scr.a = reinterpret_cast<int32_t*>(p);
    e.scr.b = reinterpret_cast<int32_t*>(p + align_up(scratch_a_elems(cw, ch) * 4, 256));
    return run_entries(direction, &e, 1, as_stream(stream));
}
