// Overlapped-block motion compensation (OBMC) for sm_100a.
//
// Replaces MotionCompensator::CompensatePicture and its per-precision BlockPixelPred
// (libdirac_common/mot_comp.cpp:63-1239).  The reference walks blocks in raster order,
// scatters each block's weighted prediction into an int16 strip and flushes finished rows;
// here every output sample gathers the contributions of the (at most 2 x 2) prediction
// units covering it, which is the same integer sum with no write conflicts, so one thread
// owns one sample and the picture is updated in place.
//
// A unit is one block row high and 1, 2 or 4 blocks wide, as the superblock split level
// dictates (mot_comp.cpp:327-394); its mode, vectors and DC come from its first block.
// Its weight is separable: V[y] * H[x] from the 1-D windows of CreateBlock
// (mot_comp.cpp:735-804), with the leading ramp padded flat on the picture's left / top
// edge and the trailing ramp on the right / bottom edge (CalculateWeights, :710-724;
// selection :353-383).  Products and sums are truncated to int16 where the reference
// stores them in ValueType.  Prediction samples come from the upconverted reference with
// coordinates clamped to [0, 2*size-2] (the reference's BChk(., 2*size-1)).
//
// CTAs of 256 threads map to 32 x 32 sample tiles of one component (four rows per thread).  A tile first tabulates, in shared
// memory, the block rows covering each of its rows (with their vertical weights) and, for each
// column and each of the three split modes, the units covering it (with their horizontal
// weights), so that no sample divides; then each thread reads the block data of its units
// (L1-resident) and 1-4 upconverted samples per prediction, at compile-time precision.

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int MTX = 32;             // tile columns; tile rows (8, 16 or 32) are a template parameter
constexpr int MT_THREADS = 256;     // eight rows at a time
constexpr int MC_ROWS[3] = {32, 16, 8};  // tile-height variants (index 0 is the default)

struct McComp {
    int16_t* pic;
    const int16_t* up1;
    const int16_t* up2;
    int w, h, stride;          // component size and picture stride
    int xblen, yblen, xbsep, ybsep, xoff, yoff;
    int x_used, y_used;        // NUM_USED_BLKS limits
    int xshift, yshift;        // chroma MV scaling
    int comp;                  // 0 Y, 1 U, 2 V (DC plane)
    int clip_lo, clip_hi;      // clip after ADD when clip_lo <= clip_hi
    int tiles_x, tile_begin;
};

struct McParams {
    const int16_t* mv1;
    const int16_t* mv2;
    const uint8_t* mode;
    const int16_t* dc;
    const uint8_t* split;
    int xnb, ynb, xnum_sb;
    int precision;
    int add_or_sub;            // 0 ADD, 1 SUBTRACT
    int ncomp;
    // reference picture weights (PicturePredParams::Ref1Weight, Ref2Weight,
    // PictureWeightsBits); wt_custom unless they are the defaults 1, 1, 1
    int wt_custom, wt1, wt2, wt_bits, wt_bias;
    McComp comp[3];
};

// AdjustBlockByRefWeights (mot_comp.cpp:620-680) with custom weights, for one sample of a
// predicted block: the reference scales its int16 block values by ref1 + ref2 weights (one
// reference) or each by its own weight and adds them (two), then (v + bias) >> bits.
__device__ __forceinline__ int ref_weighted(const McParams& P, int md, int p1, int p2) {
    const int16_t v = md == 3 ? (int16_t)((int16_t)(p1 * P.wt1) + (int16_t)(p2 * P.wt2))
                              : (int16_t)(p1 * (P.wt1 + P.wt2));
    return (int16_t)((v + P.wt_bias) >> P.wt_bits);
}

// 1-D window value (CreateBlock) at position pos of a window of length len and
// separation sep; cls 0 pads the leading ramp flat, 2 is the mirror of 0 (trailing flat).
__device__ __forceinline__ int obmc_window(int len, int sep, int cls, int pos) {
    const int o = (len - sep) >> 1;
    int flat = (cls == 0);
    if (cls == 2) {
        pos = len - 1 - pos;
        flat = 1;
    }
    auto ramp = [&](int x) -> int {
        if (o == 1) return x == 0 ? 3 : 5;
        return 1 + (6 * x + o - 1) / (2 * o - 1);
    };
    if (pos < 2 * o) return flat ? 8 : ramp(pos);
    if (pos < sep) return 8;
    return 8 - ramp(pos - sep);
}

__device__ __forceinline__ int up_at(const int16_t* up, int stride2, int W2, int H2, int yy, int xx) {
    return up[(size_t)clampi(yy, 0, H2 - 1) * stride2 + clampi(xx, 0, W2 - 1)];
}

// BlockPixelPred for one sample (mot_comp.cpp:846-1239) at compile-time precision PREC.
template <int PREC>
__device__ __forceinline__ int pixel_pred(const int16_t* up, int w, int h, int px, int py, int mvx, int mvy) {
    const int W2 = 2 * w - 1, H2 = 2 * h - 1, s2 = 2 * w;
    if (PREC == 0) return up_at(up, s2, W2, H2, 2 * (py + mvy), 2 * (px + mvx));
    if (PREC == 1) return up_at(up, s2, W2, H2, 2 * py + mvy, 2 * px + mvx);
    constexpr int M = PREC == 2 ? 1 : 3, SH = PREC == 2 ? 1 : 2, ONE = M + 1, RND = PREC == 2 ? 2 : 8,
                  OUT = PREC == 2 ? 2 : 4;
    const int rx = mvx & M, ry = mvy & M;
    const int bx = 2 * px + (mvx >> SH), by = 2 * py + (mvy >> SH);
    // clamped rows and columns of the 2 x 2 neighbourhood (BChk)
    const int x0 = clampi(bx, 0, W2 - 1), x1 = clampi(bx + 1, 0, W2 - 1);
    const int16_t* r0 = up + (size_t)clampi(by, 0, H2 - 1) * s2;
    const int16_t* r1 = up + (size_t)clampi(by + 1, 0, H2 - 1) * s2;
    return (int16_t)(((ONE - rx) * (ONE - ry) * r0[x0] + rx * (ONE - ry) * r0[x1] + (ONE - rx) * ry * r1[x0] +
                      rx * ry * r1[x1] + RND) >> OUT);
}

// Per tile row: the (at most two) block rows covering it, with their vertical weights.
struct McRow {
    int yb[2];
    int V[2];  // 0: the block row does not cover this row
};

// Per tile column and superblock split mode: the (at most two) units covering it.
struct McCol {
    int xb[2];   // candidate block column (-1: none); its superblock gives the split mode
    int xs0[2];  // first block of the unit under this split mode (-1: not used)
    int H[2];
};

// Tile-local cache of the block data: for block (yb, xb) of the tile's range, the unit
// (yb, xs0) covering it under its superblock's split, with that unit's mode, vectors (scaled
// to the component) and DC.
// Each reference's prediction is also precomputed as an offset into the upconverted plane
// and four bilinear weights; `inside` says that every prediction of the unit reads within the
// plane, so that its samples need no clamping.
constexpr int CBY = 10, CBX = 12;  // CBY * CBX <= 128 threads fill it
struct McUnit {
    short2 mv1, mv2;
    int delta[2];      // (2 py + oy) * 2w + 2 px + ox - (2 py * 2w + 2 px) per reference
    uint32_t wts[2];   // bilinear weights w00 | w01 << 8 | w10 << 16 | w11 << 24 per reference
    int16_t dc;
    uint8_t mode, sm, inside;
};

// Offset and weights of one reference's prediction (pixel_pred's arithmetic, split so that
// only the sample position remains per sample); returns whether the unit's sample rectangle
// [x0, x1] x [y0, y1] reads inside the (2w - 1) x (2h - 1) upconverted plane.
template <int PREC>
__device__ __forceinline__ bool pred_params(int mvx, int mvy, int s2, int W2, int H2, int x0, int x1, int y0, int y1,
                                            int& delta, uint32_t& wts) {
    int ox, oy, span;
    if (PREC <= 1) {
        ox = PREC == 0 ? 2 * mvx : mvx;
        oy = PREC == 0 ? 2 * mvy : mvy;
        wts = 1u;
        span = 0;
    } else {
        constexpr int M = PREC == 2 ? 1 : 3, SH = PREC == 2 ? 1 : 2, ONE = M + 1;
        const int rx = mvx & M, ry = mvy & M;
        ox = mvx >> SH;
        oy = mvy >> SH;
        wts = (uint32_t)((ONE - rx) * (ONE - ry)) | ((uint32_t)(rx * (ONE - ry)) << 8) |
              ((uint32_t)((ONE - rx) * ry) << 16) | ((uint32_t)(rx * ry) << 24);
        span = 1;
    }
    delta = oy * s2 + ox;
    return 2 * x0 + ox >= 0 && 2 * x1 + ox + span <= W2 - 1 && 2 * y0 + oy >= 0 && 2 * y1 + oy + span <= H2 - 1;
}

// The prediction at q (the unit's base sample for this position) from the packed weights.
template <int PREC>
__device__ __forceinline__ int pred_fast(const int16_t* q, int s2, uint32_t wts) {
    if (PREC <= 1) return q[0];
    constexpr int RND = PREC == 2 ? 2 : 8, OUT = PREC == 2 ? 2 : 4;
    return (int16_t)(((int)(wts & 0xff) * q[0] + (int)((wts >> 8) & 0xff) * q[1] +
                      (int)((wts >> 16) & 0xff) * q[s2] + (int)(wts >> 24) * q[s2 + 1] + RND) >> OUT);
}

template <int PREC, int MTY>
__global__ void __launch_bounds__(MT_THREADS) obmc_kernel(const __grid_constant__ McParams P) {
    __shared__ McRow rows[MTY];
    __shared__ McCol cols[3][MTX];
    __shared__ McUnit cache[CBY][CBX];
    int ci = 0;
    while (ci + 1 < P.ncomp && P.comp[ci + 1].tile_begin <= (int)blockIdx.x) ++ci;
    const McComp& C = P.comp[ci];
    const int t = blockIdx.x - C.tile_begin;
    const int ty = t / C.tiles_x, tx = t - ty * C.tiles_x;
    const int tid = threadIdx.x;
    // the tile's block range: cached when it fits (it does for block separations >= 4 / 6)
    const int yb_lo = (ty * MTY + C.yoff) / C.ybsep - 1, yb_hi = (ty * MTY + MTY - 1 + C.yoff) / C.ybsep;
    const int xb_lo = (tx * MTX + C.xoff) / C.xbsep - 1, xb_hi = (tx * MTX + MTX - 1 + C.xoff) / C.xbsep;
    const bool cached = yb_hi - yb_lo < CBY && xb_hi - xb_lo < CBX;
    // ---- tables of the tile: block rows per row, units per column and split mode ----
    if (cached && tid >= 128 && tid < 128 + CBY * CBX) {
        const int i = tid - 128, yr = i / CBX, xr = i - yr * CBX;
        const int yb = yb_lo + yr, xb = xb_lo + xr;
        McUnit u{};
        if (yb >= 0 && yb < P.ynb && xb >= 0 && xb < P.xnb) {
            const int sm = P.split[(size_t)(yb >> 2) * P.xnum_sb + (xb >> 2)];
            const int nb = sm == 0 ? 4 : (sm == 1 ? 2 : 1);
            const int xs0 = xb - (xb % nb);
            const size_t b = (size_t)yb * P.xnb + xs0;
            u.sm = (uint8_t)sm;
            u.mode = P.mode[b];
            const short2 m1 = reinterpret_cast<const short2*>(P.mv1)[b];
            const short2 m2 = reinterpret_cast<const short2*>(P.mv2)[b];
            u.mv1 = make_short2((short)(m1.x >> C.xshift), (short)(m1.y >> C.yshift));
            u.mv2 = make_short2((short)(m2.x >> C.xshift), (short)(m2.y >> C.yshift));
            u.dc = P.dc[(size_t)C.comp * P.xnb * P.ynb + b];
            // the unit's samples: columns pos_x .. pos_x + len - 1, rows pos_y .. + yblen - 1
            const int pos_x = xs0 * C.xbsep - C.xoff, len = nb * C.xbsep + 2 * C.xoff;
            const int pos_y = yb * C.ybsep - C.yoff;
            const int x0 = max(pos_x, 0), x1 = min(pos_x + len, C.w) - 1;
            const int y0 = max(pos_y, 0), y1 = min(pos_y + C.yblen, C.h) - 1;
            const int s2 = 2 * C.w, W2 = 2 * C.w - 1, H2 = 2 * C.h - 1;
            const bool in1 = pred_params<PREC>(u.mv1.x, u.mv1.y, s2, W2, H2, x0, x1, y0, y1, u.delta[0], u.wts[0]);
            const bool in2 = pred_params<PREC>(u.mv2.x, u.mv2.y, s2, W2, H2, x0, x1, y0, y1, u.delta[1], u.wts[1]);
            u.inside = (uint8_t)(u.mode == 0 || (u.mode == 1 && in1) || (u.mode == 2 && in2) || (in1 && in2));
        }
        cache[yr][xr] = u;
    }
    if (tid < MTY) {
        const int py = ty * MTY + tid;
        const int yb_hi = (py + C.yoff) / C.ybsep;
        McRow r;
        for (int k = 0; k < 2; ++k) {
            const int yb = yb_hi - 1 + k;
            const int pos_y = yb * C.ybsep - C.yoff;
            r.yb[k] = yb;
            r.V[k] = 0;
            if (yb < 0 || yb >= C.y_used || py < pos_y || py >= pos_y + C.yblen) continue;
            const int rcls = pos_y < 0 ? 0 : (yb + 1 < C.y_used ? 1 : 2);
            r.V[k] = obmc_window(C.yblen, C.ybsep, rcls, py - pos_y);
        }
        rows[tid] = r;
    } else if (tid >= 32 && tid < 32 + 3 * MTX) {
        const int sm = (tid - 32) / MTX, col = (tid - 32) - sm * MTX;
        const int px = tx * MTX + col;
        const int nb = sm == 0 ? 4 : (sm == 1 ? 2 : 1);
        const int xb_hi = (px + C.xoff) / C.xbsep;
        McCol c;
        for (int k = 0; k < 2; ++k) {
            const int xb = xb_hi - 1 + k;
            c.xb[k] = -1;
            c.xs0[k] = -1;
            c.H[k] = 0;
            if (xb < 0 || xb >= P.xnb) continue;
            if (px < xb * C.xbsep - C.xoff || px >= xb * C.xbsep - C.xoff + C.xblen) continue;
            c.xb[k] = xb;
            const int xs0 = xb - (xb % nb);
            if (xs0 >= C.x_used) continue;
            const int pos_x = xs0 * C.xbsep - C.xoff;
            const int len = nb * C.xbsep + 2 * C.xoff;
            const int ccls = (pos_x >= 0 && xs0 + nb < C.x_used) ? 1 : (pos_x < 0 ? 0 : 2);
            c.xs0[k] = xs0;
            c.H[k] = obmc_window(len, nb * C.xbsep, ccls, px - pos_x);
        }
        cols[sm][col] = c;
    }
    __syncthreads();
    const int col = tid % MTX;
    const int px = tx * MTX + col;
    for (int row = tid / MTX; row < MTY; row += MT_THREADS / MTX) {
    const int py = ty * MTY + row;
    if (px >= C.w || py >= C.h) return;

    int acc = 0;
    const McRow& R = rows[row];
    if (cached) {
#pragma unroll
        for (int ky = 0; ky < 2; ++ky) {
            if (R.V[ky] == 0) continue;
            const McUnit* crow = cache[R.yb[ky] - yb_lo];
            int last_unit = -1;
#pragma unroll
            for (int kx = 0; kx < 2; ++kx) {
                const int xb = cols[0][col].xb[kx];
                if (xb < 0) continue;
                const McUnit& u = crow[xb - xb_lo];
                const McCol& U = cols[u.sm][col];
                const int xs0 = U.xs0[kx];
                if (xs0 < 0 || xs0 == last_unit) continue;
                last_unit = xs0;
                const int16_t wgt = (int16_t)(R.V[ky] * U.H[kx]);
                int pred;
                if (u.mode == 0) {
                    pred = u.dc;
                } else if (u.inside) {
                    const int base = 2 * py * (2 * C.w) + 2 * px;
                    const int r = u.mode == 2 ? 1 : 0;
                    pred = pred_fast<PREC>((r ? C.up2 : C.up1) + base + u.delta[r], 2 * C.w, u.wts[r]);
                    if (u.mode == 3) {
                        const int p2 = pred_fast<PREC>(C.up2 + base + u.delta[1], 2 * C.w, u.wts[1]);
                        pred = P.wt_custom ? ref_weighted(P, 3, pred, p2) : (int16_t)((pred + p2 + 1) >> 1);
                    } else if (P.wt_custom) {
                        pred = ref_weighted(P, u.mode, pred, 0);
                    }
                } else {
                    const short2 m = u.mode == 2 ? u.mv2 : u.mv1;
                    pred = pixel_pred<PREC>(u.mode == 2 ? C.up2 : C.up1, C.w, C.h, px, py, m.x, m.y);
                    if (u.mode == 3) {
                        const int p2 = pixel_pred<PREC>(C.up2, C.w, C.h, px, py, u.mv2.x, u.mv2.y);
                        pred = P.wt_custom ? ref_weighted(P, 3, pred, p2) : (int16_t)((pred + p2 + 1) >> 1);
                    } else if (P.wt_custom) {
                        pred = ref_weighted(P, u.mode, pred, 0);
                    }
                }
                acc = (int16_t)(acc + (int16_t)(pred * wgt));
            }
        }
    }
    const short2* mv1 = reinterpret_cast<const short2*>(P.mv1);
    const short2* mv2 = reinterpret_cast<const short2*>(P.mv2);
#pragma unroll
    for (int ky = 0; ky < 2 && !cached; ++ky) {
        if (R.V[ky] == 0) continue;
        const int yb = R.yb[ky];
        const uint8_t* split_row = P.split + (size_t)(yb >> 2) * P.xnum_sb;
        int last_unit = -1;
#pragma unroll
        for (int kx = 0; kx < 2; ++kx) {
            const int xb = cols[0][col].xb[kx];
            if (xb < 0) continue;
            const int sm = split_row[xb >> 2];
            const McCol& U = cols[sm][col];
            const int xs0 = U.xs0[kx];
            if (xs0 < 0 || xs0 == last_unit) continue;
            last_unit = xs0;
            const int16_t wgt = (int16_t)(R.V[ky] * U.H[kx]);
            const size_t b = (size_t)yb * P.xnb + xs0;
            const int md = P.mode[b];
            int pred;
            if (md == 0) {
                pred = P.dc[(size_t)C.comp * P.xnb * P.ynb + b];
            } else {
                const short2 m = (md == 2) ? mv2[b] : mv1[b];
                const int16_t* u = (md == 2) ? C.up2 : C.up1;
                pred = pixel_pred<PREC>(u, C.w, C.h, px, py, m.x >> C.xshift, m.y >> C.yshift);
                if (md == 3) {
                    const short2 m2 = mv2[b];
                    const int p2 = pixel_pred<PREC>(C.up2, C.w, C.h, px, py, m2.x >> C.xshift, m2.y >> C.yshift);
                    pred = P.wt_custom ? ref_weighted(P, 3, pred, p2) : (int16_t)((pred + p2 + 1) >> 1);
                } else if (P.wt_custom) {
                    pred = ref_weighted(P, md, pred, 0);
                }
            }
            acc = (int16_t)(acc + (int16_t)(pred * wgt));
        }
    }
    const int v = (int16_t)(((int16_t)acc + 32) >> 6);
    int16_t* o = C.pic + (size_t)py * C.stride + px;
    int r = P.add_or_sub ? (*o - v) : (*o + v);
    r = (int16_t)r;
    if (C.clip_lo <= C.clip_hi) r = clampi(r, C.clip_lo, C.clip_hi);
    *o = (int16_t)r;
    }
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

namespace dgpu {

template <int MTY>
void launch_obmc(int tiles, const McParams& P, cudaStream_t st) {
    switch (P.precision) {
        case 0: obmc_kernel<0, MTY><<<tiles, MT_THREADS, 0, st>>>(P); break;
        case 1: obmc_kernel<1, MTY><<<tiles, MT_THREADS, 0, st>>>(P); break;
        case 2: obmc_kernel<2, MTY><<<tiles, MT_THREADS, 0, st>>>(P); break;
        default: obmc_kernel<3, MTY><<<tiles, MT_THREADS, 0, st>>>(P); break;
    }
}

int mc_tile_variants() { return 3; }

// dgpu_motion_compensate[_weighted] with a chosen tile height (variant indexes MC_ROWS).
int motion_compensate_impl(int variant, int add_or_sub, int cformat, int w, int h, const dgpu_block_params* bp,
                           const int16_t* mv1, const int16_t* mv2, const uint8_t* mode, const int16_t* dc,
                           const uint8_t* split, int16_t* const* pic, const int* pic_stride,
                           const int16_t* const* ref1up, const int16_t* const* ref2up, int clip_luma_depth,
                           int clip_chroma_depth, int wt1, int wt2, int wt_bits, cudaStream_t st) {
    if (variant < 0 || variant >= 3) return DGPU_ERR_ARG;
    if (wt_bits < 0 || wt_bits > 16) return DGPU_ERR_ARG;
    const int MTY = MC_ROWS[variant];
    if (!bp || !mv1 || !mode || !dc || !split || !pic || !pic_stride || !ref1up) return DGPU_ERR_ARG;
    if (add_or_sub != 0 && add_or_sub != 1) return DGPU_ERR_ARG;
    if (cformat < 0 || cformat > 2) return DGPU_ERR_ARG;
    if (bp->precision < 0 || bp->precision > 3) return DGPU_ERR_ARG;
    if (bp->xbsep <= 0 || bp->ybsep <= 0 || bp->xblen < bp->xbsep || bp->yblen < bp->ybsep ||
        bp->xblen > 2 * bp->xbsep || bp->yblen > 2 * bp->ybsep || (bp->xbsep & 3) || (bp->ybsep & 3) ||
        (bp->xblen & 3) || (bp->yblen & 3) || bp->xnum_sb <= 0 || bp->ynum_sb <= 0)
        return DGPU_ERR_SIZE;
    if (w < 8 || h < 8) return DGPU_ERR_SIZE;
    McParams P = {};
    P.mv1 = mv1;
    P.mv2 = mv2 ? mv2 : mv1;
    P.mode = mode;
    P.dc = dc;
    P.split = split;
    P.xnb = 4 * bp->xnum_sb;
    P.ynb = 4 * bp->ynum_sb;
    P.xnum_sb = bp->xnum_sb;
    P.precision = bp->precision;
    P.add_or_sub = add_or_sub;
    P.ncomp = 3;
    P.wt_custom = wt_bits != 1 || wt1 != 1 || wt2 != 1;  // PicturePredParams::CustomRefWeights
    P.wt1 = wt1;
    P.wt2 = wt2;
    P.wt_bits = wt_bits;
    P.wt_bias = 1;  // 2^(bits - 1), built as the reference builds it: 1 when bits is 0
    for (int i = wt_bits - 1; i > 0; --i) P.wt_bias <<= 1;
    int tiles = 0;
    for (int c = 0; c < 3; ++c) {
        McComp& C = P.comp[c];
        C.xshift = (c && cformat != 0) ? 1 : 0;  // ChromaFormat: 0 444, 1 422, 2 420
        C.yshift = (c && cformat == 2) ? 1 : 0;
        C.w = w >> C.xshift;
        C.h = h >> C.yshift;
        if (!pic[c] || !ref1up[c] || pic_stride[c] < C.w) return DGPU_ERR_ARG;
        C.pic = pic[c];
        C.stride = pic_stride[c];
        C.up1 = ref1up[c];
        C.up2 = (ref2up && ref2up[c]) ? ref2up[c] : ref1up[c];
        C.xblen = bp->xblen >> C.xshift;
        C.xbsep = bp->xbsep >> C.xshift;
        C.yblen = bp->yblen >> C.yshift;
        C.ybsep = bp->ybsep >> C.yshift;
        C.xoff = (C.xblen - C.xbsep) / 2;
        C.yoff = (C.yblen - C.ybsep) / 2;
        C.x_used = (C.w + C.xbsep + (C.xblen - C.xbsep) / 2 - 1) / C.xbsep;
        C.y_used = (C.h + C.ybsep + (C.yblen - C.ybsep) / 2 - 1) / C.ybsep;
        if (C.x_used > P.xnb) C.x_used = P.xnb;
        if (C.y_used > P.ynb) C.y_used = P.ynb;
        C.comp = c;
        const int depth = c ? clip_chroma_depth : clip_luma_depth;
        if (add_or_sub == 0 && depth > 0) {
            C.clip_lo = -(1 << (depth - 1));
            C.clip_hi = (1 << (depth - 1)) - 1;
        } else {
            C.clip_lo = 1;
            C.clip_hi = 0;
        }
        C.tiles_x = (C.w + MTX - 1) / MTX;
        C.tile_begin = tiles;
        tiles += C.tiles_x * ((C.h + MTY - 1) / MTY);
    }
    if (MTY == 32) launch_obmc<32>(tiles, P, st);
    else if (MTY == 16) launch_obmc<16>(tiles, P, st);
    else launch_obmc<8>(tiles, P, st);
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}

int motion_compensate_tiled(int variant, int add_or_sub, int cformat, int w, int h, const dgpu_block_params* bp,
                            const int16_t* mv1, const int16_t* mv2, const uint8_t* mode, const int16_t* dc,
                            const uint8_t* split, int16_t* const* pic, const int* pic_stride,
                            const int16_t* const* ref1up, const int16_t* const* ref2up, int clip_luma_depth,
                            int clip_chroma_depth, cudaStream_t st) {
    return motion_compensate_impl(variant, add_or_sub, cformat, w, h, bp, mv1, mv2, mode, dc, split, pic, pic_stride,
                                  ref1up, ref2up, clip_luma_depth, clip_chroma_depth, 1, 1, 1, st);
}

}  // namespace dgpu

extern "C" int dgpu_motion_compensate(int add_or_sub, int cformat, int w, int h, const dgpu_block_params* bp,
                                      const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                                      const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                                      const int* pic_stride, const int16_t* const* ref1up,
                                      const int16_t* const* ref2up, int clip_luma_depth, int clip_chroma_depth,
                                      void* stream) {
    return motion_compensate_tiled(0, add_or_sub, cformat, w, h, bp, mv1, mv2, mode, dc, split, pic, pic_stride,
                                   ref1up, ref2up, clip_luma_depth, clip_chroma_depth, as_stream(stream));
}

extern "C" int dgpu_motion_compensate_weighted(int add_or_sub, int cformat, int w, int h,
                                               const dgpu_block_params* bp, const int16_t* mv1, const int16_t* mv2,
                                               const uint8_t* mode, const int16_t* dc, const uint8_t* split,
                                               int16_t* const* pic, const int* pic_stride,
                                               const int16_t* const* ref1up, const int16_t* const* ref2up,
                                               int clip_luma_depth, int clip_chroma_depth, int ref1_weight,
                                               int ref2_weight, int weight_bits, void* stream) {
    return motion_compensate_impl(0, add_or_sub, cformat, w, h, bp, mv1, mv2, mode, dc, split, pic, pic_stride,
                                  ref1up, ref2up, clip_luma_depth, clip_chroma_depth, ref1_weight, ref2_weight,
                                  weight_bits, as_stream(stream));
}
