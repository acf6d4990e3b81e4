/*
 * dirac_oracle_quant.c -- TEST INFRASTRUCTURE ONLY (see dirac_oracle.h).
 *
 * Plain-C restatement of per-subband quantiser selection (QuantChooser,
 * libdirac_encoder/quant_chooser.cpp:62-362, driven as PictureCompressor::SelectMultiQuants
 * does, picture_compress.cpp:632-709) and of quantisation with in-place reconstruction
 * (GenericBandCodec::CodeVal / CodeCoeffBlock / ClearBlock, band_codec_template.h:53-174 and
 * 470-557; IntraDCBandCodec::CodeCoeff, band_codec.cpp:81-96; CompCompressor::Compress,
 * comp_compress.cpp:64-156).  Floating-point arithmetic follows the reference's types and
 * operation order (float weights, lambda and entropy factors; double statistics).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dirac_oracle.h"

/* QuantiserLists (libdirac_common/common.cpp:931-981) */
int orc_qf4(int q) {
    if (q == 0) return 4;
    if (q == 1) return 5;
    const uint64_t base = (uint64_t)1 << (q / 4);
    uint64_t f;
    switch (q % 4) {
    case 0: f = 4 * base; break;
    case 1: f = (503829 * base + 52958) / 105917; break;
    case 2: f = (665857 * base + 58854) / 117708; break;
    default: f = (440253 * base + 32722) / 65444; break;
    }
    return (int)f;
}
int orc_intra_offset4(int q) { return q == 0 ? 1 : (q == 1 ? 2 : (orc_qf4(q) + 1) >> 1); }
int orc_inter_offset4(int q) { return q == 0 ? 1 : (q == 1 ? 2 : (3 * orc_qf4(q) + 4) >> 3); }

/* SubbandList::Init (wavelet_utils.cpp:144-190): band b (1-based) geometry. */
void orc_band_rect(int depth, int cw, int ch, int b, int* xp, int* yp, int* xl, int* yl) {
    if (b == 3 * depth + 1) {
        *xp = 0; *yp = 0; *xl = cw >> depth; *yl = ch >> depth;
        return;
    }
    const int level = (b - 1) / 3 + 1, kind = (b - 1) % 3;
    const int l_x = cw >> level, l_y = ch >> level;
    *xl = l_x;
    *yl = l_y;
    *xp = (kind == 0 || kind == 2) ? l_x : 0; /* HH, HL */
    *yp = (kind == 0 || kind == 1) ? l_y : 0; /* HH, LH */
}

typedef struct {
    double error;
    int count0, pos, neg;
} qstat;

static double pow4(double x) { return x * x * x * x; }

/* Error and counts for one quantiser over the band sampled every xr columns / yr rows
 * (Integral/NonIntegralErrorCalc; the two coincide for multiples of 4). */
static qstat band_stat(const int32_t* c, int stride, int xp, int yp, int xl, int yl, int xr, int yr, int q) {
    qstat s = {0.0, 0, 0, 0};
    const int qf = orc_qf4(q), off = orc_inter_offset4(q);
    for (int j = yp; j < yp + yl; j += yr)
        for (int i = xp; i < xp + xl; i += xr) {
            const int val = c[(size_t)j * stride + i];
            const int a = abs(val);
            int qv = (a << 2) / qf;
            if (!qv) {
                s.error += pow4((double)a);
                continue;
            }
            s.count0 += qv;
            qv = (qv * qf + off + 2) >> 2;
            if (val > 0) s.pos++; else s.neg++;
            s.error += pow4((double)(a - qv));
        }
    return s;
}

typedef struct {
    double Error, ENTROPY, TOTAL;
} costt;

static costt lagrangian(qstat s, int count1, float wt, float lambda, float ecf) {
    costt c;
    c.Error = s.error / (double)count1;
    c.Error = sqrt(c.Error) / (wt * wt);
    double p0 = (double)s.count0 / (double)(s.count0 + count1);
    double p1 = 1.0 - p0;
    if (p0 != 0.0 && p1 != 0.0)
        c.ENTROPY = -(p0 * log(p0) + p1 * log(p1)) / log(2.0);
    else
        c.ENTROPY = 0.0;
    c.ENTROPY *= (double)(s.count0 + count1);
    c.ENTROPY /= (double)count1;
    double se;
    if (s.pos + s.neg != 0) {
        p0 = (double)s.neg / (double)(s.pos + s.neg);
        p1 = 1.0 - p0;
        if (p0 != 0.0 && p1 != 0.0)
            se = -((p0 * log(p0) + p1 * log(p1)) / log(2.0));
        else
            se = 0.0;
    } else {
        se = 0.0;
    }
    se *= (double)(s.neg + s.pos);
    se /= (double)count1;
    c.ENTROPY += se;
    c.ENTROPY *= ecf;
    c.TOTAL = c.Error + lambda * c.ENTROPY;
    return c;
}

/* QuantChooser::GetBestQuant for one band: returns the estimated bits and sets *qidx (the
 * band's quantiser; left at *qidx's incoming value when the band is all zero). */
static int best_quant(const int32_t* c, int stride, int xp, int yp, int xl, int yl, float wt, float lambda, float ecf,
                      int* qidx) {
    int maxv = 0;
    for (int j = yp; j < yp + yl; ++j)
        for (int i = xp; i < xp + xl; ++i) {
            const int a = abs(c[(size_t)j * stride + i]);
            if (a > maxv) maxv = a;
        }
    if (maxv < 1) return 0;
    const int max_bit = (int)floor(logf((float)maxv) / log(2.0));
    const int nq = 4 * max_bit + 5;
    costt* cost = (costt*)calloc((size_t)nq, sizeof(costt));
    int lo = 0, hi = nq - 1, step = 4, xr = 2, yr = 2, mn = 0;
    for (int pass = 0; pass < 3; ++pass) {
        if (pass == 1) {
            lo = mn - 2 > 0 ? mn - 2 : 0;
            hi = mn + 2 < nq - 1 ? mn + 2 : nq - 1;
            step = 2;
        } else if (pass == 2) {
            lo = mn - 1 > 0 ? mn - 1 : 0;
            hi = mn + 1 < nq - 1 ? mn + 1 : nq - 1;
            step = 1;
            xr = 1;
        }
        const int count1 = (xl / xr) * (yl / yr);
        for (int q = lo; q <= hi; q += step)
            cost[q] = lagrangian(band_stat(c, stride, xp, yp, xl, yl, xr, yr, q), count1, wt, lambda, ecf);
        mn = lo;
        for (int q = lo + step; q <= hi; q += step)
            if (cost[q].TOTAL < cost[mn].TOTAL) mn = q;
    }
    const double bit_sum = cost[mn].ENTROPY * xl * yl;
    free(cost);
    *qidx = mn;
    return (int)bit_sum;
}

/* GenericIntraDCBandCodec::GetPrediction (band_codec_template.h:531-557). */
static int dc_prediction(const int32_t* d, int stride, int x, int y) {
    if (y != 0) {
        if (x != 0) {
            const int sum = d[(size_t)y * stride + x - 1] + d[(size_t)(y - 1) * stride + x - 1] +
                            d[(size_t)(y - 1) * stride + x] + 3 / 2;
            return sum < 0 ? (sum - 2) / 3 : sum / 3;
        }
        return d[(size_t)(y - 1) * stride];
    }
    return x != 0 ? d[x - 1] : 0;
}

static int recon_mag(int q, int qf, int off) { return (q * qf + off + 2) >> 2; }

/* CodeVal: quantise val, return the quantised magnitude, write the reconstruction. */
static int code_val(int val, int qf, int off, int32_t* out) {
    const unsigned a = (unsigned)abs(val);
    const unsigned qv = (a << 2) / (unsigned)qf;
    int r = 0;
    if (qv) {
        r = recon_mag((int)qv, qf, off);
        if (val <= 0) r = -r;
    }
    *out = r;
    return (int)qv;
}

int orc_code_residue(int intra, int depth, int32_t* c, int cw, int ch, float lambda, const float* band_wt,
                     const float* band_ecf, const int* band_ncb, int* band_qidx, int* band_skip, int* band_bits,
                     uint8_t* cb_skip, int32_t* qout) {
    const int nb = 3 * depth + 1;
    if (depth < 1 || cw % (1 << depth) || ch % (1 << depth)) return -1;
    /* quantiser choice, DC band first (SelectQuantisers) */
    size_t cbk = 0;
    size_t* cb_first = (size_t*)malloc(sizeof(size_t) * (size_t)(nb + 1));
    for (int b = 1; b <= nb; ++b) {
        cb_first[b - 1] = cbk;
        cbk += (size_t)band_ncb[2 * (b - 1)] * band_ncb[2 * (b - 1) + 1];
    }
    cb_first[nb] = cbk;
    for (int b = nb; b >= 1; --b) {
        int xp, yp, xl, yl;
        orc_band_rect(depth, cw, ch, b, &xp, &yp, &xl, &yl);
        const int dc_intra = (b == nb) && intra;
        int32_t* saved = NULL;
        if (dc_intra) { /* AddSubAverage(SUBTRACT): DPCM against the previous (int16) value */
            saved = (int32_t*)malloc(sizeof(int32_t) * (size_t)xl * yl);
            int16_t last = 0;
            for (int j = 0; j < yl; ++j)
                for (int i = 0; i < xl; ++i) {
                    int32_t* v = &c[(size_t)j * cw + i];
                    saved[(size_t)j * xl + i] = *v;
                    const int16_t keep = (int16_t)*v;
                    *v -= last;
                    last = keep;
                }
        }
        int q = 0;
        const int bits = best_quant(c, cw, xp, yp, xl, yl, band_wt[b - 1], lambda, band_ecf[b - 1], &q);
        band_bits[b - 1] = bits;
        band_skip[b - 1] = bits == 0;
        band_qidx[b - 1] = q;
        /* code-block skip flags (QuantChooser::SetSkip), only set when the band has data */
        const int xn = band_ncb[2 * (b - 1)], yn = band_ncb[2 * (b - 1) + 1];
        const int qf = orc_qf4(q);
        int maxv = 0;
        for (int j = yp; j < yp + yl; ++j)
            for (int i = xp; i < xp + xl; ++i) maxv = abs(c[(size_t)j * cw + i]) > maxv ? abs(c[(size_t)j * cw + i]) : maxv;
        for (int by = 0; by < yn; ++by)
            for (int bx = 0; bx < xn; ++bx) {
                const int x0 = bx * xl / xn + xp, x1 = (bx + 1) * xl / xn + xp;
                const int y0 = by * yl / yn + yp, y1 = (by + 1) * yl / yn + yp;
                int skip = 1;
                for (int j = y0; j < y1; ++j)
                    for (int i = x0; i < x1; ++i)
                        if ((abs(c[(size_t)j * cw + i]) << 2) >= qf) skip = 0;
                cb_skip[cb_first[b - 1] + (size_t)by * xn + bx] = maxv >= 1 ? (uint8_t)skip : 0;
            }
        if (dc_intra) { /* AddSubAverage(ADD) restores the values as int16 */
            int16_t last = 0;
            for (int j = 0; j < yl; ++j)
                for (int i = 0; i < xl; ++i) {
                    int32_t* v = &c[(size_t)j * cw + i];
                    *v += last;
                    last = (int16_t)*v;
                }
            free(saved);
        }
    }
    /* quantise and reconstruct, DC band first (CompCompressor::Compress) */
    for (int b = nb; b >= 1; --b) {
        int xp, yp, xl, yl;
        orc_band_rect(depth, cw, ch, b, &xp, &yp, &xl, &yl);
        if (band_skip[b - 1]) {
            for (int j = yp; j < yp + yl; ++j)
                for (int i = xp; i < xp + xl; ++i) {
                    c[(size_t)j * cw + i] = 0;
                    if (qout) qout[(size_t)j * cw + i] = 0;
                }
            continue;
        }
        const int q = band_qidx[b - 1];
        const int qf = orc_qf4(q), off = intra ? orc_intra_offset4(q) : orc_inter_offset4(q);
        const int dc_intra = (b == nb) && intra;
        const int xn = band_ncb[2 * (b - 1)], yn = band_ncb[2 * (b - 1) + 1];
        for (int by = 0; by < yn; ++by)
            for (int bx = 0; bx < xn; ++bx) {
                const int x0 = bx * xl / xn + xp, x1 = (bx + 1) * xl / xn + xp;
                const int y0 = by * yl / yn + yp, y1 = (by + 1) * yl / yn + yp;
                const int skip = cb_skip[cb_first[b - 1] + (size_t)by * xn + bx];
                for (int j = y0; j < y1; ++j)
                    for (int i = x0; i < x1; ++i) {
                        int32_t* v = &c[(size_t)j * cw + i];
                        if (dc_intra) {
                            const int16_t pred = (int16_t)dc_prediction(c, cw, i, j);
                            if (skip) {
                                *v = pred;
                                if (qout) qout[(size_t)j * cw + i] = 0;
                            } else {
                                const int16_t val = (int16_t)(*v - pred);
                                int32_t r;
                                const int qv = code_val(val, qf, off, &r);
                                if (qout) qout[(size_t)j * cw + i] = val < 0 ? -qv : qv;
                                *v = r + pred;
                            }
                        } else if (skip) {
                            *v = 0;
                            if (qout) qout[(size_t)j * cw + i] = 0;
                        } else {
                            const int val = *v;
                            int32_t r;
                            const int qv = code_val(val, qf, off, &r);
                            if (qout) qout[(size_t)j * cw + i] = val < 0 ? -qv : qv;
                            *v = r;
                        }
                    }
            }
    }
    free(cb_first);
    return 0;
}

/* Dequantisation of one entropy-decoded component, in the reference decoder's order:
 * CompDecompressor::Decompress walks the bands from the DC band down to band 1
 * (libdirac_decoder/comp_decompress.cpp:64-127) and zeroes a skipped band (SetToVal,
 * :121-125, 154-163); a band decoder walks its code blocks in raster order
 * (GenericBandCodec::DoWorkDecode, band_codec_template.h:204-228), decodes each value as
 * (q * qf4 + offset + 2) >> 2 with its sign (DecodeVal, :330-356; quantiser and offset from
 * DecodeCoeffBlock, :231-270) and zeroes a skipped code block (ClearBlock, :488-496).  The
 * intra DC band first decodes a code block's residues, then adds, in raster order, the
 * prediction from the reconstructed neighbours; a skipped code block takes the prediction
 * alone (GenericIntraDCBandCodec::DecodeCoeffBlock / ClearBlock / GetPrediction, :500-557;
 * int32 arithmetic, CoeffType).  Code block (i, j) of a band covers columns
 * [i * xl / xn, (i + 1) * xl / xn) (Subband::SetNumBlocks, wavelet_utils.cpp:116-140).
 * qindex and coeff are cw x ch, dense; they may be the same array. */
static int decode_val(int q, int qf, int off) {
    if (q == 0) return 0;
    const int mag = q < 0 ? -q : q;
    const int v = (int)((unsigned)mag * (unsigned)qf + (unsigned)(off + 2)) >> 2;
    return q < 0 ? -v : v;
}

int orc_dequantise(int intra, int depth, const int32_t* qindex, int32_t* coeff, int cw, int ch,
                   const int* band_ncb, const int* band_qidx, const int* band_skip, const uint8_t* cb_skip) {
    const int nb = 3 * depth + 1;
    int* cb_first = (int*)malloc(sizeof(int) * (nb + 1));
    if (!cb_first) return -4;
    cb_first[0] = 0;
    for (int b = 0; b < nb; ++b) cb_first[b + 1] = cb_first[b] + band_ncb[2 * b] * band_ncb[2 * b + 1];
    for (int b = nb; b >= 1; --b) {
        int xp, yp, xl, yl;
        orc_band_rect(depth, cw, ch, b, &xp, &yp, &xl, &yl);
        if (band_skip[b - 1]) {
            for (int j = yp; j < yp + yl; ++j)
                for (int i = xp; i < xp + xl; ++i) coeff[(size_t)j * cw + i] = 0;
            continue;
        }
        const int q = band_qidx[b - 1];
        if (q < 0 || q > 119) {
            free(cb_first);
            return -1;
        }
        const int qf = orc_qf4(q), off = intra ? orc_intra_offset4(q) : orc_inter_offset4(q);
        const int xn = band_ncb[2 * (b - 1)], yn = band_ncb[2 * (b - 1) + 1];
        const int dc_intra = intra && b == nb;
        for (int by = 0; by < yn; ++by)
            for (int bx = 0; bx < xn; ++bx) {
                const int skip = cb_skip[cb_first[b - 1] + by * xn + bx];
                const int x0 = xp + bx * xl / xn, x1 = xp + (bx + 1) * xl / xn;
                const int y0 = yp + by * yl / yn, y1 = yp + (by + 1) * yl / yn;
                for (int j = y0; j < y1; ++j)
                    for (int i = x0; i < x1; ++i) {
                        const size_t at = (size_t)j * cw + i;
                        coeff[at] = skip ? 0 : decode_val(qindex[at], qf, off);
                    }
                if (dc_intra)
                    for (int j = y0; j < y1; ++j)
                        for (int i = x0; i < x1; ++i) {
                            const size_t at = (size_t)j * cw + i;
                            const int pred = dc_prediction(coeff, cw, i, j);
                            coeff[at] = skip ? pred : coeff[at] + pred;
                        }
            }
    }
    free(cb_first);
    return 0;
}
