/*
 * dirac_oracle.c -- TEST INFRASTRUCTURE ONLY (see dirac_oracle.h).
 *
 * Plain-C restatement of the Dirac hot path used as the parity oracle for the CUDA
 * kernels and as the timed CPU baseline.  Written from the reference's behaviour, not
 * copied: the per-filter edge formulas of libdirac_common/wavelet_utils.cpp are expressed
 * through a single rule (a neighbour index is clamped inside its own parity
 * subsequence), which reproduces every explicit edge case of the reference for level
 * sides >= orc_dwt_min_len(filter).
 */
#include "dirac_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------ */
/* Wavelet transform                                                                     */
/* ------------------------------------------------------------------------------------ */

/* Kinds of lifting step (libdirac_common/wavelet_utils.h:490-616). */
enum { LIFT_SHIFT2 = 0,  /* PredictStepShift/UpdateStepShift: (a+b+2^(s-1))>>s      */
       LIFT_FOURTAP = 1, /* *StepFourTap<s,t1,t2>: (t1(a+b)+t2(c+d)+2^(s-1))>>s      */
       LIFT_97 = 2,      /* *Step97<g>: (g*(a+b))>>12                                */
       LIFT_HAAR = 3 };  /* Haar pair step (wavelet_utils.cpp:1342-1489)             */

typedef struct {
    int parity; /* 1: odd samples are updated from even ones; 0: the reverse */
    int sign;   /* -1: "predict" (subtract), +1: "update" (add) */
    int kind;
    int shift, t1, t2, gain;
} lift_step;

typedef struct {
    int nsteps;
    int shift; /* ShiftRowLeft before analysis / ShiftRowRight after synthesis */
    lift_step step[4];
} filter_def;

/* Analysis steps in order; synthesis runs them in reverse with the opposite sign.
 * DD9_7   wavelet_utils.cpp:952-1042   LEGALL5_3 :805-877   DD13_7 :1136-1233
 * HAAR0/1 :1342-1450                   DAUB9_7  :575-690 (also FIDELITY and unknown
 * filters, which the WaveletTransform constructor maps to DAUB9_7, :406-435). */
static filter_def get_filter(int filter) {
    filter_def f;
    memset(&f, 0, sizeof(f));
    switch (filter) {
    case ORC_DD9_7:
        f.nsteps = 2; f.shift = 1;
        f.step[0] = (lift_step){1, -1, LIFT_FOURTAP, 4, 9, -1, 0};
        f.step[1] = (lift_step){0, +1, LIFT_SHIFT2, 2, 0, 0, 0};
        break;
    case ORC_LEGALL5_3:
        f.nsteps = 2; f.shift = 1;
        f.step[0] = (lift_step){1, -1, LIFT_SHIFT2, 1, 0, 0, 0};
        f.step[1] = (lift_step){0, +1, LIFT_SHIFT2, 2, 0, 0, 0};
        break;
    case ORC_DD13_7:
        f.nsteps = 2; f.shift = 1;
        f.step[0] = (lift_step){1, -1, LIFT_FOURTAP, 4, 9, -1, 0};
        f.step[1] = (lift_step){0, +1, LIFT_FOURTAP, 5, 9, -1, 0};
        break;
    case ORC_HAAR0:
    case ORC_HAAR1:
        f.nsteps = 2; f.shift = (filter == ORC_HAAR1) ? 1 : 0;
        f.step[0] = (lift_step){1, -1, LIFT_HAAR, 0, 0, 0, 0};
        f.step[1] = (lift_step){0, +1, LIFT_HAAR, 0, 0, 0, 0};
        break;
    default: /* DAUB9_7, FIDELITY, anything else */
        f.nsteps = 4; f.shift = 1;
        f.step[0] = (lift_step){1, -1, LIFT_97, 0, 0, 0, 6497};
        f.step[1] = (lift_step){0, -1, LIFT_97, 0, 0, 0, 217};
        f.step[2] = (lift_step){1, +1, LIFT_97, 0, 0, 0, 3616};
        f.step[3] = (lift_step){0, +1, LIFT_97, 0, 0, 0, 1817};
        break;
    }
    return f;
}

int orc_dwt_min_len(int filter) {
    switch (filter) {
    case ORC_DD9_7:
    case ORC_DD13_7: return 6;
    case ORC_HAAR0:
    case ORC_HAAR1: return 2;
    default: return 4;
    }
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* One lifting step over a 1-D sequence x[0], x[s], ... x[(n-1)s] (n even).
 * Target sample k = 2m+parity reads the other parity's subsequence q at
 *   near: q[m-1+parity], q[m+parity]      far: q[m-2+parity], q[m+1+parity]
 * with the subsequence index clamped to [0, n/2-1]. */
static void lift_1d(int32_t* x, int n, int s, const lift_step* st, int sign) {
    const int half = n >> 1;
    const int other = 1 - st->parity;
    for (int m = 0; m < half; ++m) {
        const int p = st->parity;
        const int ia = clampi(m - 1 + p, 0, half - 1);
        const int ib = clampi(m + p, 0, half - 1);
        const int a = x[(2 * ia + other) * s];
        const int b = x[(2 * ib + other) * s];
        int d;
        switch (st->kind) {
        case LIFT_SHIFT2:
            d = (a + b + (1 << (st->shift - 1))) >> st->shift;
            break;
        case LIFT_FOURTAP: {
            const int ic = clampi(m - 2 + p, 0, half - 1);
            const int id = clampi(m + 1 + p, 0, half - 1);
            const int c = x[(2 * ic + other) * s];
            const int e = x[(2 * id + other) * s];
            d = (st->t1 * (a + b) + st->t2 * (c + e) + (1 << (st->shift - 1))) >> st->shift;
            break;
        }
        case LIFT_97:
            d = (st->gain * (a + b)) >> 12;
            break;
        default: /* Haar: odd uses its left even partner, even uses its right odd partner */
            d = p ? a : ((b + 1) >> 1);
            break;
        }
        int32_t* t = &x[(2 * m + p) * s];
        *t = (sign < 0) ? (*t - d) : (*t + d);
    }
}

/* Mallat reorder of an xl x yl region (VHFilter::DeInterleave, wavelet_utils.cpp:540-573). */
static void deinterleave(int32_t* c, int stride, int xl, int yl, int32_t* tmp) {
    for (int j = 0; j < yl; ++j) memcpy(tmp + (size_t)j * xl, c + (size_t)j * stride, sizeof(int32_t) * xl);
    const int xl2 = xl >> 1, yl2 = yl >> 1;
    for (int j = 0; j < yl; ++j)
        for (int i = 0; i < xl; ++i)
            c[(size_t)((j & 1) * yl2 + (j >> 1)) * stride + (i & 1) * xl2 + (i >> 1)] = tmp[(size_t)j * xl + i];
}

/* VHFilter::Interleave, wavelet_utils.cpp:491-523. */
static void interleave(int32_t* c, int stride, int xl, int yl, int32_t* tmp) {
    for (int j = 0; j < yl; ++j) memcpy(tmp + (size_t)j * xl, c + (size_t)j * stride, sizeof(int32_t) * xl);
    const int xl2 = xl >> 1, yl2 = yl >> 1;
    for (int j = 0; j < yl; ++j)
        for (int i = 0; i < xl; ++i)
            c[(size_t)j * stride + i] = tmp[(size_t)((j & 1) * yl2 + (j >> 1)) * xl + (i & 1) * xl2 + (i >> 1)];
}

/* One analysis level on the top-left xl x yl region (VHFilter*::Split). */
static void split_level(const filter_def* f, int32_t* c, int stride, int xl, int yl, int32_t* tmp) {
    for (int j = 0; j < yl; ++j) {
        int32_t* row = c + (size_t)j * stride;
        if (f->shift)
            for (int i = 0; i < xl; ++i) row[i] = (int32_t)((uint32_t)row[i] << f->shift);
        for (int k = 0; k < f->nsteps; ++k) lift_1d(row, xl, 1, &f->step[k], f->step[k].sign);
    }
    for (int i = 0; i < xl; ++i)
        for (int k = 0; k < f->nsteps; ++k) lift_1d(c + i, yl, stride, &f->step[k], f->step[k].sign);
    deinterleave(c, stride, xl, yl, tmp);
}

/* One synthesis level (VHFilter*::Synth): vertical then horizontal, then ShiftRowRight. */
static void synth_level(const filter_def* f, int32_t* c, int stride, int xl, int yl, int32_t* tmp) {
    interleave(c, stride, xl, yl, tmp);
    for (int i = 0; i < xl; ++i)
        for (int k = f->nsteps - 1; k >= 0; --k) lift_1d(c + i, yl, stride, &f->step[k], -f->step[k].sign);
    for (int j = 0; j < yl; ++j) {
        int32_t* row = c + (size_t)j * stride;
        for (int k = f->nsteps - 1; k >= 0; --k) lift_1d(row, xl, 1, &f->step[k], -f->step[k].sign);
        if (f->shift) {
            const int half = 1 << (f->shift - 1);
            for (int i = 0; i < xl; ++i) row[i] = (row[i] + half) >> f->shift;
        }
    }
}

static int dwt_check(int filter, int depth, int cw, int ch) {
    if (depth < 1 || depth > 8 || cw <= 0 || ch <= 0) return -1;
    const int mul = 1 << depth;
    if (cw % mul || ch % mul) return -2;
    const int minlen = orc_dwt_min_len(filter);
    if ((cw >> (depth - 1)) < minlen || (ch >> (depth - 1)) < minlen) return -3;
    return 0;
}

/* WaveletTransform::Transform FORWARD (wavelet_utils.cpp:446-466). */
int orc_dwt_forward(int filter, int depth, const int16_t* pic, int w, int h, int pic_stride,
                    int32_t* coeff, int cw, int ch, int coeff_stride) {
    int rc = dwt_check(filter, depth, cw, ch);
    if (rc) return rc;
    if (w <= 0 || h <= 0 || w > cw || h > ch) return -4;
    /* pad-copy: the last column and row are replicated into the padding */
    for (int j = 0; j < ch; ++j) {
        const int16_t* src = pic + (size_t)(j < h ? j : h - 1) * pic_stride;
        int32_t* dst = coeff + (size_t)j * coeff_stride;
        for (int i = 0; i < cw; ++i) dst[i] = src[i < w ? i : w - 1];
    }
    const filter_def f = get_filter(filter);
    int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)cw * ch);
    if (!tmp) return -5;
    for (int l = 1, xl = cw, yl = ch; l <= depth; ++l, xl >>= 1, yl >>= 1)
        split_level(&f, coeff, coeff_stride, xl, yl, tmp);
    free(tmp);
    return 0;
}

/* WaveletTransform::Transform BACKWARD (wavelet_utils.cpp:467-484). */
int orc_dwt_backward(int filter, int depth, int32_t* coeff, int cw, int ch, int coeff_stride,
                     int16_t* pic, int w, int h, int pic_stride) {
    int rc = dwt_check(filter, depth, cw, ch);
    if (rc) return rc;
    if (w <= 0 || h <= 0 || w > cw || h > ch) return -4;
    const filter_def f = get_filter(filter);
    int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)cw * ch);
    if (!tmp) return -5;
    for (int l = 1, xl = cw >> (depth - 1), yl = ch >> (depth - 1); l <= depth; ++l, xl <<= 1, yl <<= 1)
        synth_level(&f, coeff, coeff_stride, xl, yl, tmp);
    free(tmp);
    for (int j = 0; j < h; ++j)
        for (int i = 0; i < w; ++i) pic[(size_t)j * pic_stride + i] = (int16_t)coeff[(size_t)j * coeff_stride + i];
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Half-pel upconversion (UpConverter::DoUpConverter / RowLoop, upconvert.cpp:55-200)     */
/* ------------------------------------------------------------------------------------ */

static const int up_taps[4] = {21, -7, 3, -1};

/* The reference accumulates in a ValueType (int16) `sum`, truncating after every add;
   the casts below reproduce that. */
int orc_upconvert(const int16_t* pic, int w, int h, int stride, int bit_depth, int16_t* up, int up_stride) {
    if (w < 8 || h < 8 || bit_depth < 2 || bit_depth > 16) return -1;
    const int lo = -(1 << (bit_depth - 1)), hi = (1 << (bit_depth - 1)) - 1;
    /* vertical pass: even up-rows copy, odd up-rows interpolate between source rows y, y+1
       (source row indices clamped to [0, h-1]); only even up-columns are written here */
    for (int y = 0; y < h; ++y) {
        int16_t* even_row = up + (size_t)(2 * y) * up_stride;
        int16_t* odd_row = up + (size_t)(2 * y + 1) * up_stride;
        for (int x = 0; x < w; ++x) {
            even_row[2 * x] = pic[(size_t)y * stride + x];
            int16_t sum = 16;
            for (int t = 0; t < 4; ++t) {
                const int ya = clampi(y - t, 0, h - 1), yb = clampi(y + 1 + t, 0, h - 1);
                sum = (int16_t)(sum + (pic[(size_t)ya * stride + x] + pic[(size_t)yb * stride + x]) * up_taps[t]);
            }
            sum = (int16_t)(sum >> 5);
            odd_row[2 * x] = (int16_t)clampi(sum, lo, hi);
        }
    }
    /* horizontal pass on every up-row: odd columns from the even ones (even-column index
       clamped to [0, w-1]) */
    for (int r = 0; r < 2 * h; ++r) {
        int16_t* row = up + (size_t)r * up_stride;
        for (int x = 0; x < w; ++x) {
            int16_t sum = 16;
            for (int t = 0; t < 4; ++t) {
                const int xa = clampi(x - t, 0, w - 1), xb = clampi(x + 1 + t, 0, w - 1);
                sum = (int16_t)(sum + (row[2 * xa] + row[2 * xb]) * up_taps[t]);
            }
            sum = (int16_t)(sum >> 5);
            row[2 * x + 1] = (int16_t)clampi(sum, lo, hi);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* 2x decimation (DownConverter::DoDownConvert / RowLoop, downconvert.cpp:51-204,        */
/* taps downconvert.h:82-89)                                                             */
/* ------------------------------------------------------------------------------------ */

static const int down_taps[6] = {86, 46, 4, -8, -4, 4};

int orc_downconvert(const int16_t* pic, int w, int h, int stride, int16_t* out, int out_stride) {
    const int ow = w / 2, oh = h / 2;
    const int xlen = 2 * ow, ylen = 2 * oh; /* an odd last row/column is not used */
    if (ow < 12 || oh < 12) return -1;
    int16_t* rowbuf = (int16_t*)malloc(sizeof(int16_t) * (size_t)xlen);
    if (!rowbuf) return -5;
    for (int r = 0; r < oh; ++r) {
        const int y = 2 * r;
        for (int x = 0; x < xlen; ++x) {
            int sum = 128;
            for (int t = 0; t < 6; ++t) {
                const int ya = clampi(y - t, 0, ylen - 1), yb = clampi(y + 1 + t, 0, ylen - 1);
                sum += (pic[(size_t)ya * stride + x] + pic[(size_t)yb * stride + x]) * down_taps[t];
            }
            rowbuf[x] = (int16_t)(sum >> 8);
        }
        for (int c = 0; c < ow; ++c) {
            const int x = 2 * c;
            int sum = 128;
            for (int t = 0; t < 6; ++t) {
                const int xa = clampi(x - t, 0, xlen - 1), xb = clampi(x + 1 + t, 0, xlen - 1);
                sum += (rowbuf[xa] + rowbuf[xb]) * down_taps[t];
            }
            out[(size_t)r * out_stride + c] = (int16_t)(sum >> 8);
        }
    }
    free(rowbuf);
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Overlapped-block motion compensation (MotionCompensator, mot_comp.cpp:63-1239)         */
/* ------------------------------------------------------------------------------------ */
/*
 * The reference scatters each block's weighted prediction into a strip buffer in block
 * raster order and flushes finished rows.  The restatement below gathers instead: every
 * output sample sums the contributions of the (at most 2 x 2) prediction units that cover
 * it, which is the same integer sum.  A unit is a block, a sub-superblock (2 blocks wide)
 * or a whole superblock row segment (4 blocks wide), chosen by the superblock's split
 * level (mot_comp.cpp:327-394); units are one block row high.  Weights are separable,
 * V[y] * H[x], from the 1-D windows of MotionCompensator::CreateBlock (:735-804) with the
 * edge variants of CalculateWeights (:710-724) chosen as at :353-383.
 */

/* One 1-D window (CreateBlock): length len, separation sep; flat_start pads the leading
 * ramp to 8 (a block on the picture's left / top edge). */
static void obmc_window(int len, int sep, int flat_start, int16_t* out) {
    const int o = (len - sep) / 2;
    if (o != 1) {
        for (int x = 0; x < 2 * o; ++x) {
            out[x] = (int16_t)(1 + (6 * x + o - 1) / (2 * o - 1));
            out[x + sep] = (int16_t)(8 - out[x]);
        }
    } else {
        out[0] = out[1 + sep] = 3;
        out[1] = out[sep] = 5;
    }
    for (int x = 2 * o; x < sep; ++x) out[x] = 8;
    if (flat_start)
        for (int x = 0; x < 2 * o; ++x) out[x] = 8;
}

/* window value for edge class cls (0 leading edge, 1 interior, 2 trailing edge) */
static int16_t obmc_weight(int len, int sep, int cls, int pos) {
    int16_t buf[512];
    if (cls == 2) {
        obmc_window(len, sep, 1, buf);
        return buf[len - 1 - pos];
    }
    obmc_window(len, sep, cls == 0, buf);
    return buf[pos];
}

static inline int bchk(int v, int max) { return v < 0 ? 0 : (v >= max ? max - 1 : v); }

/* BlockPixelPred for one sample (mot_comp.cpp:846-1239): the reference clamps upconverted
 * coordinates with BChk(., 2*size - 1), i.e. to [0, 2*size - 2], whenever any sample of
 * the block would leave that range, and the unclamped paths never leave it. */
static int16_t pixel_pred(int prec, const int16_t* up, int cw, int ch, int px, int py, int mvx, int mvy) {
    const int W2 = 2 * cw - 1, H2 = 2 * ch - 1, stride = 2 * cw;
#define UP(yy, xx) ((int)up[(size_t)bchk((yy), H2) * stride + bchk((xx), W2)])
    switch (prec) {
    case 0:
        return (int16_t)UP(2 * (py + mvy), 2 * (px + mvx));
    case 1:
        return (int16_t)UP(2 * py + mvy, 2 * px + mvx);
    case 2: {
        const int rx = mvx & 1, ry = mvy & 1;
        const int bx = 2 * px + (mvx >> 1), by = 2 * py + (mvy >> 1);
        return (int16_t)(((2 - rx) * (2 - ry) * UP(by, bx) + rx * (2 - ry) * UP(by, bx + 1) +
                          (2 - rx) * ry * UP(by + 1, bx) + rx * ry * UP(by + 1, bx + 1) + 2) >> 2);
    }
    default: {
        const int rx = mvx & 3, ry = mvy & 3;
        const int bx = 2 * px + (mvx >> 2), by = 2 * py + (mvy >> 2);
        return (int16_t)(((4 - rx) * (4 - ry) * UP(by, bx) + rx * (4 - ry) * UP(by, bx + 1) +
                          (4 - rx) * ry * UP(by + 1, bx) + rx * ry * UP(by + 1, bx + 1) + 8) >> 4);
    }
    }
#undef UP
}

/* AdjustBlockByRefWeights (mot_comp.cpp:620-680) for one sample of a predicted block, with
 * custom picture weights: the block's values (ValueType, int16) scaled by ref1 + ref2 weights
 * for one reference, or each by its own weight and added for two, then (v + bias) >> bits,
 * the bias 2^(bits - 1) built by a loop that leaves it 1 when bits is 0. */
static int16_t ref_weighted(int md, int16_t p1, int16_t p2, int wt1, int wt2, int wt_bits) {
    int bias = 1;
    for (int i = wt_bits - 1; i > 0; --i) bias <<= 1;
    int16_t v;
    if (md == 3)
        v = (int16_t)((int16_t)(p1 * wt1) + (int16_t)(p2 * wt2));
    else
        v = (int16_t)(p1 * (wt1 + wt2));
    return (int16_t)((v + bias) >> wt_bits);
}

int orc_motion_compensate(int add_or_sub, int cformat, int w, int h, const orc_block_params* bp,
                          const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                          const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                          const int16_t* const* ref1up, const int16_t* const* ref2up) {
    return orc_motion_compensate_wt(add_or_sub, cformat, w, h, bp, mv1, mv2, mode, dc, split, pic, ref1up, ref2up,
                                    1, 1, 1);
}

int orc_motion_compensate_wt(int add_or_sub, int cformat, int w, int h, const orc_block_params* bp,
                             const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                             const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                             const int16_t* const* ref1up, const int16_t* const* ref2up, int wt1, int wt2,
                             int wt_bits) {
    /* PicturePredParams::CustomRefWeights (common.h:986-991) */
    const int custom = wt_bits != 1 || wt1 != 1 || wt2 != 1;
    if (wt_bits < 0 || wt_bits > 16) return -1;
    if (!bp || bp->xbsep <= 0 || bp->ybsep <= 0 || bp->xblen < bp->xbsep || bp->yblen < bp->ybsep ||
        bp->xblen > 2 * bp->xbsep || bp->yblen > 2 * bp->ybsep || bp->xnum_sb <= 0 || bp->ynum_sb <= 0)
        return -1;
    const int xnb = 4 * bp->xnum_sb, ynb = 4 * bp->ynum_sb;
    for (int c = 0; c < 3; ++c) {
        const int xs = (c && cformat != ORC_444) ? 1 : 0;
        const int ys = (c && cformat == ORC_420) ? 1 : 0;
        const int cw = w >> xs, ch = h >> ys;
        const int xblen = bp->xblen >> xs, xbsep = bp->xbsep >> xs;
        const int yblen = bp->yblen >> ys, ybsep = bp->ybsep >> ys;
        const int xoff = (xblen - xbsep) / 2, yoff = (yblen - ybsep) / 2;
        int x_used = (cw + xbsep + (xblen - xbsep) / 2 - 1) / xbsep; /* NUM_USED_BLKS, :54 */
        int y_used = (ch + ybsep + (yblen - ybsep) / 2 - 1) / ybsep;
        if (x_used > xnb) x_used = xnb;
        if (y_used > ynb) y_used = ynb;
        int16_t* out = pic[c];
        for (int py = 0; py < ch; ++py) {
            for (int px = 0; px < cw; ++px) {
                int acc = 0;
                const int yb_hi = (py + yoff) / ybsep;
                for (int yb = yb_hi - 1; yb <= yb_hi; ++yb) {
                    if (yb < 0 || yb >= y_used) continue;
                    const int pos_y = yb * ybsep - yoff;
                    if (py < pos_y || py >= pos_y + yblen) continue;
                    const int rcls = pos_y < 0 ? 0 : (yb + 1 < y_used ? 1 : 2);
                    const int16_t V = obmc_weight(yblen, ybsep, rcls, py - pos_y);
                    const int xb_hi = (px + xoff) / xbsep;
                    int last_unit = -1;
                    for (int xb = xb_hi - 1; xb <= xb_hi; ++xb) {
                        if (xb < 0 || xb >= xnb) continue;
                        if (px < xb * xbsep - xoff || px >= xb * xbsep - xoff + xblen) continue;
                        const int sm = split[(size_t)(yb / 4) * bp->xnum_sb + xb / 4];
                        const int nb = sm == 0 ? 4 : (sm == 1 ? 2 : 1);
                        const int xs0 = xb - (xb % nb);
                        if (xs0 == last_unit || xs0 >= x_used) continue;
                        last_unit = xs0;
                        const int pos_x = xs0 * xbsep - xoff;
                        const int len = nb * xbsep + 2 * xoff;
                        const int ccls = (pos_x >= 0 && xs0 + nb < x_used) ? 1 : (pos_x < 0 ? 0 : 2);
                        const int16_t H = obmc_weight(len, nb * xbsep, ccls, px - pos_x);
                        const int16_t wgt = (int16_t)(V * H);
                        const size_t b = (size_t)yb * xnb + xs0;
                        const int md = mode[b];
                        int16_t pred;
                        if (md == 0) {
                            pred = dc[(size_t)c * xnb * ynb + b];
                        } else {
                            const int16_t* m1 = (md == 2) ? mv2 : mv1;
                            const int16_t* u1 = (md == 2) ? ref2up[c] : ref1up[c];
                            pred = pixel_pred(bp->precision, u1, cw, ch, px, py, m1[2 * b] >> xs, m1[2 * b + 1] >> ys);
                            if (md == 3) {
                                const int16_t p2 = pixel_pred(bp->precision, ref2up[c], cw, ch, px, py,
                                                              mv2[2 * b] >> xs, mv2[2 * b + 1] >> ys);
                                pred = custom ? ref_weighted(3, pred, p2, wt1, wt2, wt_bits)
                                              : (int16_t)((pred + p2 + 1) >> 1);
                            } else if (custom) {
                                pred = ref_weighted(md, pred, 0, wt1, wt2, wt_bits);
                            }
                        }
                        acc = (int16_t)(acc + (int16_t)(pred * wgt));
                    }
                }
                const int16_t v = (int16_t)(((int16_t)acc + 32) >> 6);
                int16_t* o = &out[(size_t)py * cw + px];
                *o = add_or_sub ? (int16_t)(*o - v) : (int16_t)(*o + v);
            }
        }
    }
    return 0;
}

void orc_clip(int16_t* pic, size_t n, int bit_depth) {
    const int lo = -(1 << (bit_depth - 1)), hi = (1 << (bit_depth - 1)) - 1;
    for (size_t i = 0; i < n; ++i) pic[i] = (int16_t)clampi(pic[i], lo, hi);
}

/* CWMFilterComponent (libdirac_encoder/prefilter.cpp:50-125): the median of the list made of
 * the centre sample repeated max(1, 10 - strength) - 1 times and the nine samples of its 3 x 3
 * window, for rows 1 .. h-2 and columns 1 .. w-3 (the reference's column loop ends at
 * LastX() - 1); an even-length list gives the rounded mean of its two middle values.  Reads
 * `in`, writes every sample of `out` (unfiltered ones copied). */
int orc_cwm_filter(const int16_t* in, int16_t* out, int w, int h, int strength) {
    if (!in || !out || w < 1 || h < 1) return -1;
    const int weight = (10 - strength) > 1 ? 10 - strength : 1;
    const int len = weight + 8;
    int16_t* list = (int16_t*)malloc(sizeof(int16_t) * (size_t)len);
    if (!list) return -4;
    memcpy(out, in, sizeof(int16_t) * (size_t)w * h);
    for (int y = 1; y < h - 1; ++y)
        for (int x = 1; x < w - 2; ++x) {
            int n = 0;
            for (int k = 0; k < weight - 1; ++k) list[n++] = in[(size_t)y * w + x];
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) list[n++] = in[(size_t)(y + dy) * w + x + dx];
            for (int i = 1; i < n; ++i) { /* insertion sort */
                const int16_t t = list[i];
                int j = i - 1;
                while (j >= 0 && list[j] > t) {
                    list[j + 1] = list[j];
                    --j;
                }
                list[j + 1] = t;
            }
            out[(size_t)y * w + x] = (len & 1) ? list[(len - 1) / 2]
                                               : (int16_t)((list[len / 2 - 1] + list[len / 2] + 1) >> 1);
        }
    free(list);
    return 0;
}

/* LPFilter (libdirac_encoder/prefilter.cpp:141-306), the RECTLP residue prefilter: taps of a
 * 17-point Hanning-windowed sinc designed in double (MakeLPRectFilter with 14-bit accuracy and
 * LPFilter's bandwidth), then HFilter and VFilter: each output (sum + 2^13) >> 14 clamped to
 * [-128, 127], source indices clamped to the component.  In place; w, h >= 17. */
int orc_rect_lp_filter(int16_t* pic, int w, int h, float qf, int strength) {
    if (!pic || w < 17 || h < 17) return -1;
    float bw = qf + 3.0f - (float)strength;
    bw = bw < 1.0f ? 1.0f : (bw > 10.0f ? 10.0f : bw);
    bw /= 10.0f;
    const float pi = 3.1415926535f;
    double d[17], sum = 0.0;
    int t[17];
    for (int i = -8; i <= 8; ++i) {
        const float a = (pi * i) / 18;
        const double v = pi * 1.0 * bw * i;
        d[i + 8] = cos((double)a) * (v == 0.0 ? 1.0 : sin(v) / v);
    }
    for (int i = 0; i < 17; ++i) sum += d[i];
    for (int i = 0; i < 17; ++i) {
        const double x = d[i] * (double)(1 << 18) / sum;
        const int r = x > 0 ? (int)(x + 0.5) : -(int)(-x + 0.5);
        t[i] = (r + 8) >> 4;
    }
    int16_t* tmp = (int16_t*)malloc(sizeof(int16_t) * (size_t)w * h);
    if (!tmp) return -4;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int s = 1 << 13;
            for (int k = -8; k <= 8; ++k) s += t[k + 8] * pic[(size_t)y * w + clampi(x - k, 0, w - 1)];
            s >>= 14;
            tmp[(size_t)y * w + x] = (int16_t)clampi(s, -128, 127);
        }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int s = 1 << 13;
            for (int k = -8; k <= 8; ++k) s += t[k + 8] * tmp[(size_t)clampi(y - k, 0, h - 1) * w + x];
            s >>= 14;
            pic[(size_t)y * w + x] = (int16_t)clampi(s, -128, 127);
        }
    free(tmp);
    return 0;
}

/* DiagFilter (libdirac_encoder/prefilter.cpp:535-588), the DIAGLP residue prefilter: the taps
 * quadrant of GetDiagLPFilter (:395-530) for the bandwidth, mixed with a unit impulse by the
 * factor, then every output (2^15 + sum over the 13 x 13 neighbourhood) >> 16 as int16 with
 * source indices clamped (DiagFilterBchkD, :307-354; DiagFilterD reads the same samples in
 * the interior).  The expressions keep the reference's float / double mix.  In place; w, h >= 7;
 * a bandwidth above 0.9 leaves the component unchanged. */
static const int diag_tables[8][7][7] = {
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

int orc_diag_lp_filter(int16_t* pic, int w, int h, float qf, int strength) {
    if (!pic || w < 7 || h < 7) return -1;
    const float ffactor = (8.0 + strength - 4.0 - qf) / 5.0;
    int factor = (int)(ffactor * 256.0);
    factor = factor < 0 ? 0 : (factor > 256 ? 256 : factor);
    const float bw = (1.0 - ffactor) * 0.6 + 0.4;
    if (bw > 0.9) return 0;
    int qbf = (int)(bw * 10.0 + 0.5);
    qbf = qbf < 2 ? 2 : (qbf > 10 ? 10 : qbf);
    int f[7][7];
    for (int j = 0; j < 7; ++j)
        for (int i = 0; i < 7; ++i) f[j][i] = qbf == 10 ? (i == 0 && j == 0 ? 65536 : 0) : diag_tables[qbf - 2][j][i];
    for (int j = 0; j < 7; ++j)
        for (int i = 0; i < 7; ++i)
            f[j][i] = (factor * f[j][i] + (j == 0 && i == 0 ? (256 - factor) * 65536 : 0) + 128) >> 8;
    int16_t* src = (int16_t*)malloc(sizeof(int16_t) * (size_t)w * h);
    if (!src) return -4;
    memcpy(src, pic, sizeof(int16_t) * (size_t)w * h);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int val = 1 << 15;
            for (int j = -6; j <= 6; ++j)
                for (int i = -6; i <= 6; ++i)
                    val += f[abs(j)][abs(i)] * src[(size_t)clampi(y + j, 0, h - 1) * w + clampi(x + i, 0, w - 1)];
            pic[(size_t)y * w + x] = (int16_t)(val >> 16);
        }
    free(src);
    return 0;
}
