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
// Threads map to 32 x 8 sample tiles of one component; each thread reads the block data
// of its units (L1-resident) and 1-4 upconverted samples per prediction.

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int MTX = 32, MTY = 8;

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
    McComp comp[3];
};

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

// BlockPixelPred for one sample (mot_comp.cpp:846-1239)
__device__ __forceinline__ int pixel_pred(int prec, const int16_t* up, int w, int h, int px, int py, int mvx,
                                          int mvy) {
    const int W2 = 2 * w - 1, H2 = 2 * h - 1, s2 = 2 * w;
    switch (prec) {
        case 0:
            return up_at(up, s2, W2, H2, 2 * (py + mvy), 2 * (px + mvx));
        case 1:
            return up_at(up, s2, W2, H2, 2 * py + mvy, 2 * px + mvx);
        case 2: {
            const int rx = mvx & 1, ry = mvy & 1;
            const int bx = 2 * px + (mvx >> 1), by = 2 * py + (mvy >> 1);
            return (int16_t)(((2 - rx) * (2 - ry) * up_at(up, s2, W2, H2, by, bx) +
                              rx * (2 - ry) * up_at(up, s2, W2, H2, by, bx + 1) +
                              (2 - rx) * ry * up_at(up, s2, W2, H2, by + 1, bx) +
                              rx * ry * up_at(up, s2, W2, H2, by + 1, bx + 1) + 2) >> 2);
        }
        default: {
            const int rx = mvx & 3, ry = mvy & 3;
            const int bx = 2 * px + (mvx >> 2), by = 2 * py + (mvy >> 2);
            return (int16_t)(((4 - rx) * (4 - ry) * up_at(up, s2, W2, H2, by, bx) +
                              rx * (4 - ry) * up_at(up, s2, W2, H2, by, bx + 1) +
                              (4 - rx) * ry * up_at(up, s2, W2, H2, by + 1, bx) +
                              rx * ry * up_at(up, s2, W2, H2, by + 1, bx + 1) + 8) >> 4);
        }
    }
}

__global__ void __launch_bounds__(MTX* MTY) obmc_kernel(const __grid_constant__ McParams P) {
    int ci = 0;
    while (ci + 1 < P.ncomp && P.comp[ci + 1].tile_begin <= (int)blockIdx.x) ++ci;
    const McComp& C = P.comp[ci];
    const int t = blockIdx.x - C.tile_begin;
    const int ty = t / C.tiles_x, tx = t - ty * C.tiles_x;
    const int px = tx * MTX + threadIdx.x % MTX;
    const int py = ty * MTY + threadIdx.x / MTX;
    if (px >= C.w || py >= C.h) return;

    int acc = 0;
    const int yb_hi = (py + C.yoff) / C.ybsep;
    for (int yb = yb_hi - 1; yb <= yb_hi; ++yb) {
        if (yb < 0 || yb >= C.y_used) continue;
        const int pos_y = yb * C.ybsep - C.yoff;
        if (py < pos_y || py >= pos_y + C.yblen) continue;
        const int rcls = pos_y < 0 ? 0 : (yb + 1 < C.y_used ? 1 : 2);
        const int V = obmc_window(C.yblen, C.ybsep, rcls, py - pos_y);
        const int xb_hi = (px + C.xoff) / C.xbsep;
        int last_unit = -1;
        for (int xb = xb_hi - 1; xb <= xb_hi; ++xb) {
            if (xb < 0 || xb >= P.xnb) continue;
            if (px < xb * C.xbsep - C.xoff || px >= xb * C.xbsep - C.xoff + C.xblen) continue;
            const int sm = P.split[(size_t)(yb >> 2) * P.xnum_sb + (xb >> 2)];
            const int nb = sm == 0 ? 4 : (sm == 1 ? 2 : 1);
            const int xs0 = xb - (xb % nb);
            if (xs0 == last_unit || xs0 >= C.x_used) continue;
            last_unit = xs0;
            const int pos_x = xs0 * C.xbsep - C.xoff;
            const int len = nb * C.xbsep + 2 * C.xoff;
            const int ccls = (pos_x >= 0 && xs0 + nb < C.x_used) ? 1 : (pos_x < 0 ? 0 : 2);
            const int H = obmc_window(len, nb * C.xbsep, ccls, px - pos_x);
            const int16_t wgt = (int16_t)(V * H);
            const size_t b = (size_t)yb * P.xnb + xs0;
            const int md = P.mode[b];
            int pred;
            if (md == 0) {
                pred = P.dc[(size_t)C.comp * P.xnb * P.ynb + b];
            } else {
                const int16_t* m = (md == 2) ? P.mv2 : P.mv1;
                const int16_t* u = (md == 2) ? C.up2 : C.up1;
                pred = pixel_pred(P.precision, u, C.w, C.h, px, py, m[2 * b] >> C.xshift, m[2 * b + 1] >> C.yshift);
                if (md == 3) {
                    const int p2 = pixel_pred(P.precision, C.up2, C.w, C.h, px, py, P.mv2[2 * b] >> C.xshift,
                                              P.mv2[2 * b + 1] >> C.yshift);
                    pred = (int16_t)((pred + p2 + 1) >> 1);
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

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_motion_compensate(int add_or_sub, int cformat, int w, int h, const dgpu_block_params* bp,
                                      const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                                      const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                                      const int* pic_stride, const int16_t* const* ref1up,
                                      const int16_t* const* ref2up, int clip_luma_depth, int clip_chroma_depth,
                                      void* stream) {
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
    obmc_kernel<<<tiles, MTX * MTY, 0, as_stream(stream)>>>(P);
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}
