/*
 * dirac_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the Dirac research codec's data-parallel hot path, written
 * for this project from the reference's behaviour (each function cites the reference
 * file:line it restates).  It is the oracle the tests compare the CUDA path against and
 * the CPU baseline bench.py times; nothing in the product links or loads it.
 *
 * Conventions: pictures are int16 (the reference's ValueType), wavelet coefficients int32
 * (CoeffType of the plain-C build), arrays dense row-major with an explicit stride in
 * elements.  Functions return 0 on success and a negative value on invalid arguments.
 */
#ifndef DIRAC_ORACLE_H
#define DIRAC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Filter numbering follows the reference's WltFilter (libdirac_common/common_types.h:61-71). */
enum { ORC_DD9_7 = 0, ORC_LEGALL5_3 = 1, ORC_DD13_7 = 2, ORC_HAAR0 = 3, ORC_HAAR1 = 4,
       ORC_FIDELITY = 5, ORC_DAUB9_7 = 6 };

/* Smallest level-region side a filter handles with its regular edge rule. */
int orc_dwt_min_len(int filter);

/* Forward transform: pad-copy pic (w x h) into coeff (cw x ch, multiples of 2^depth),
 * then depth analysis levels in place (Mallat layout). */
int orc_dwt_forward(int filter, int depth, const int16_t* pic, int w, int h, int pic_stride,
                    int32_t* coeff, int cw, int ch, int coeff_stride);

/* Inverse transform: depth synthesis levels in place on coeff, then truncating copy of the
 * top-left w x h into pic. */
int orc_dwt_backward(int filter, int depth, int32_t* coeff, int cw, int ch, int coeff_stride,
                     int16_t* pic, int w, int h, int pic_stride);

/* 2x half-pel upconversion, up is (2h) x (2w). */
int orc_upconvert(const int16_t* pic, int w, int h, int stride, int bit_depth, int16_t* up,
                  int up_stride);

/* 2x decimation; out is (h/2) x (w/2). */
int orc_downconvert(const int16_t* pic, int w, int h, int stride, int16_t* out, int out_stride);

/* Overlapped-block parameters of a picture (luma, level 2 = single blocks), already in the
 * form PicturePredParams::SetBlockSizes accepts unchanged (libdirac_common/common.cpp:207-330):
 * lengths and separations multiples of 4, sep <= len <= 2 sep.  Blocks = 4 x superblocks. */
typedef struct {
    int precision; /* MVPrecisionType: 0 pel, 1 half, 2 quarter, 3 eighth */
    int xblen, yblen, xbsep, ybsep;
    int xnum_sb, ynum_sb;
} orc_block_params;

/* Chroma format numbering of the reference's ChromaFormat (format444 0, 422 1, 420 2). */
enum { ORC_444 = 0, ORC_422 = 1, ORC_420 = 2 };

/* Overlapped-block motion compensation of one picture (all three components):
 * pic[c] (w_c x h_c, dense) -= / += the OBMC prediction built from the upconverted references
 * ref1up[c] / ref2up[c] ((2 h_c) x (2 w_c)).  add_or_sub: 0 ADD, 1 SUBTRACT.  Block data:
 * mv1/mv2 int16 (x,y) pairs per block, mode uint8 per block (0 INTRA, 1 REF1, 2 REF2,
 * 3 REF1AND2), dc int16 [3][blocks], split uint8 per superblock.  No clipping. */
int orc_motion_compensate(int add_or_sub, int cformat, int w, int h, const orc_block_params* bp,
                          const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                          const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                          const int16_t* const* ref1up, const int16_t* const* ref2up);
/* The same with custom reference picture weights (ref1, ref2, precision bits; 1, 1, 1 is the
 * default). */
int orc_motion_compensate_wt(int add_or_sub, int cformat, int w, int h, const orc_block_params* bp,
                          const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                          const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                          const int16_t* const* ref1up, const int16_t* const* ref2up, int wt1, int wt2, int wt_bits);

/* Number of pyramid levels PixelMatcher uses for a w x h picture (pixel_match.cpp:94-95). */
int orc_me_depth(int w, int h);

/* Motion estimation of one picture against one (nref 1) or two references, as
 * PictureCompressor::PixelME / SubPixelME / ModeDecisionME run it: stage 1 pel search over the
 * pyramid, stage 2 lambda map + sub-pel refinement, stage 3 mode decision + DC.  Planes pic,
 * ref1, ref2 are the three original components.  Outputs (blocks = 16 x superblocks):
 * mv_out [nref][blocks][2] int16, cost_out [nref][blocks][3] = SAD, mvcost, total; after
 * stage 3 mode_out [blocks], dc_out [3][blocks], split_out / sbcost_out [superblocks].
 * MV precision must be half, quarter or eighth pel. */
int orc_motion_estimate(int cformat, int w, int h, const orc_block_params* bp, int nref,
                        const int16_t* const* pic, const int16_t* const* ref1, const int16_t* const* ref2,
                        int luma_depth, float lambda, int stages, int16_t* mv_out, float* cost_out,
                        uint8_t* mode_out, int16_t* dc_out, uint8_t* split_out, float* sbcost_out);

/* QuantiserLists (common.cpp:931-981): quantisation factor x4 and reconstruction offsets x4. */
int orc_qf4(int q);
int orc_intra_offset4(int q);
int orc_inter_offset4(int q);
/* Subband b (1-based, SubbandList order: per level HH, LH, HL; DC last) of a cw x ch array. */
void orc_band_rect(int depth, int cw, int ch, int b, int* xp, int* yp, int* xl, int* yl);

/* Residue coding of one transformed component: quantiser choice per band (band weights,
 * entropy factors and the code-block grid per band are inputs), then quantisation with
 * in-place reconstruction of c (cw x ch, dense).  Outputs per band: quantiser, skip flag,
 * estimated bits; per code block (bands concatenated, raster) the skip flag; optionally the
 * signed quantised indices qout (cw x ch; the intra DC band holds its prediction residues). */
int orc_code_residue(int intra, int depth, int32_t* c, int cw, int ch, float lambda, const float* band_wt,
                     const float* band_ecf, const int* band_ncb, int* band_qidx, int* band_skip, int* band_bits,
                     uint8_t* cb_skip, int32_t* qout);

/* The decoder's dequantisation of one component from its signed quantised indices (the intra
 * DC band holding its prediction residues' indices), band quantisers and skip flags, and
 * code-block skip flags (layouts as orc_code_residue writes them); coeff may equal qindex.
 * Returns -1 for a coded band's quantiser index outside 0..119. */
int orc_dequantise(int intra, int depth, const int32_t* qindex, int32_t* coeff, int cw, int ch,
                   const int* band_ncb, const int* band_qidx, const int* band_skip, const uint8_t* cb_skip);

/* CWMFilterComponent: centre-weighted median prefilter of a dense w x h component. */
int orc_cwm_filter(const int16_t* in, int16_t* out, int w, int h, int strength);

/* LPFilter: the RECTLP residue prefilter of a dense w x h component, in place (w, h >= 17). */
int orc_rect_lp_filter(int16_t* pic, int w, int h, float qf, int strength);

/* DiagFilter: the DIAGLP residue prefilter of a dense w x h component, in place (w, h >= 7). */
int orc_diag_lp_filter(int16_t* pic, int w, int h, float qf, int strength);

/* Picture::ClipComponent: clamp to [-2^(d-1), 2^(d-1)-1]. */
void orc_clip(int16_t* pic, size_t n, int bit_depth);

#ifdef __cplusplus
}
#endif
#endif
