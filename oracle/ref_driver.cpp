// Test infrastructure only: an extern "C" stage driver over the reference codec's own
// classes, compiled together with the reference sources into oracle/_ref/libdirac_ref.so.
// The tests and the golden-fixture generator call it to run the reference itself on the
// same bytes the CUDA path sees.  Nothing in the product links or loads this file.
//
// Every array crossing this boundary is dense row-major with the stated width as stride.

#include <cstring>
#include <vector>

#include <libdirac_common/common.h>
#include <libdirac_common/wavelet_utils.h>
#include <libdirac_common/upconvert.h>
#include <libdirac_motionest/downconvert.h>
#include <libdirac_common/picture.h>
#include <libdirac_common/mot_comp.h>
#include <libdirac_common/motion.h>
#include <libdirac_encoder/enc_queue.h>
#include <libdirac_encoder/enc_picture.h>
#include <libdirac_motionest/pixel_match.h>
#include <libdirac_motionest/me_subpel.h>
#include <libdirac_motionest/me_mode_decn.h>
#include <libdirac_encoder/quant_chooser.h>
#include <libdirac_encoder/comp_compress.h>
#include <libdirac_byteio/component_byteio.h>
#include <libdirac_byteio/subband_byteio.h>
#include <libdirac_common/band_codec.h>
#include <libdirac_common/band_vlc.h>
#include <libdirac_encoder/prefilter.h>

using namespace dirac;

namespace {

void fill_pic(PicArray& a, const short* src) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(&a[j][0], src + (size_t)j * a.LengthX(), sizeof(short) * a.LengthX());
}

void read_pic(const PicArray& a, short* dst) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(dst + (size_t)j * a.LengthX(), &a[j][0], sizeof(short) * a.LengthX());
}

template <class A, class T>
void fill_arr(A& a, const T* src) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(&a[j][0], src + (size_t)j * a.LengthX(), sizeof(T) * a.LengthX());
}

template <class A, class T>
void read_arr(const A& a, T* dst) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(dst + (size_t)j * a.LengthX(), &a[j][0], sizeof(T) * a.LengthX());
}

}  // namespace

extern "C" {

// WaveletTransform(depth, filter).Transform(FORWARD, pic, coeff)
// (libdirac_common/wavelet_utils.cpp:440-466).  pic is h x w int16, coeff is ch x cw int32
// (the padded size, a multiple of 2^depth).  Returns 0, or -1 on an exception.
int ref_dwt_forward(int filter, int depth, const short* pic, int w, int h, int* coeff, int cw, int ch) {
    try {
        PicArray p(h, w);
        fill_pic(p, pic);
        CoeffArray c(ch, cw);
        WaveletTransform wt(depth, (WltFilter)filter);
        wt.Transform(FORWARD, p, c);
        read_arr(c, coeff);
        return 0;
    } catch (...) {
        return -1;
    }
}

// WaveletTransform(depth, filter).Transform(BACKWARD, pic, coeff)
// (wavelet_utils.cpp:467-484): synthesises coeff in place and writes the truncated
// int16 picture.  coeff is read and overwritten.
int ref_dwt_backward(int filter, int depth, int* coeff, int cw, int ch, short* pic, int w, int h) {
    try {
        PicArray p(h, w);
        CoeffArray c(ch, cw);
        fill_arr(c, coeff);
        WaveletTransform wt(depth, (WltFilter)filter);
        wt.Transform(BACKWARD, p, c);
        read_arr(c, coeff);
        read_pic(p, pic);
        return 0;
    } catch (...) {
        return -1;
    }
}

// UpConverter(min,max,orig_w,orig_h).DoUpConverter (libdirac_common/upconvert.cpp:55-145).
// up is (2h) x (2w).
int ref_upconvert(const short* pic, int w, int h, int depth, short* up) {
    try {
        PicArray p(h, w);
        fill_pic(p, pic);
        PicArray u(2 * h, 2 * w);
        u.Fill(0);
        UpConverter uc(-(1 << (depth - 1)), (1 << (depth - 1)) - 1, w, h);
        uc.DoUpConverter(p, u);
        read_pic(u, up);
        return 0;
    } catch (...) {
        return -1;
    }
}

// DownConverter::DoDownConvert (libdirac_motionest/downconvert.cpp:51-147); out is
// (h/2) x (w/2), as PixelMatcher::MakePicHierarchy sizes it (pixel_match.cpp:158-167).
int ref_downconvert(const short* pic, int w, int h, short* out) {
    try {
        PicArray p(h, w);
        fill_pic(p, pic);
        PicArray o(h / 2, w / 2);
        DownConverter dc;
        dc.DoDownConvert(p, o);
        read_pic(o, out);
        return 0;
    } catch (...) {
        return -1;
    }
}

// Block-motion description shared by the MC / ME stage drivers: per block (row-major over
// ynb x xnb) int16 MV pairs (x, y) for reference 1 and 2, uint8 prediction mode
// (PredMode: INTRA 0, REF1_ONLY 1, REF2_ONLY 2, REF1AND2 3), int16 DC per component, and a
// uint8 superblock split level per superblock (ynsb x xnsb).
struct RefBlockDesc {
    int precision;          // MVPrecisionType: 0 pel, 1 half, 2 quarter, 3 eighth
    int xblen, yblen, xbsep, ybsep;  // luma OLB parameters (level 2)
    int xnum_sb, ynum_sb;   // blocks = 4 * superblocks in each direction
};

static void setup_ppp(PicturePredParams& ppp, const RefBlockDesc& d, ChromaFormat cf) {
    ppp.SetMVPrecision((MVPrecisionType)d.precision);
    ppp.SetBlockSizes(OLBParams(d.xblen, d.yblen, d.xbsep, d.ybsep), cf);
    ppp.SetXNumSB(d.xnum_sb);
    ppp.SetYNumSB(d.ynum_sb);
    ppp.SetXNumBlocks(4 * d.xnum_sb);
    ppp.SetYNumBlocks(4 * d.ynum_sb);
}

static void fill_mvdata(MvData& mv, const short* mv1, const short* mv2, const unsigned char* mode,
                        const short* dc, const unsigned char* split, int nref) {
    const int ynb = mv.Mode().LengthY(), xnb = mv.Mode().LengthX();
    for (int j = 0; j < ynb; ++j)
        for (int i = 0; i < xnb; ++i) {
            const size_t b = (size_t)j * xnb + i;
            mv.Vectors(1)[j][i] = MVector(mv1[2 * b], mv1[2 * b + 1]);
            if (nref > 1) mv.Vectors(2)[j][i] = MVector(mv2[2 * b], mv2[2 * b + 1]);
            mv.Mode()[j][i] = (PredMode)mode[b];
            for (int c = 0; c < 3; ++c) mv.DC((CompSort)c)[j][i] = dc[(size_t)c * ynb * xnb + b];
        }
    for (int j = 0; j < mv.SBSplit().LengthY(); ++j)
        for (int i = 0; i < mv.SBSplit().LengthX(); ++i)
            mv.SBSplit()[j][i] = split[(size_t)j * mv.SBSplit().LengthX() + i];
}

// MotionCompensator::CompensatePicture (libdirac_common/mot_comp.cpp:63-192) on one picture:
// pic[3] (in/out, component planes) gets the OBMC prediction from ref1[3]/ref2[3] (plain,
// not upconverted: the reference upconverts them itself through Picture::UpData) added
// (add_or_sub = 0) or subtracted (1).  cformat: ChromaFormat (0 444, 1 422, 2 420).
int ref_motion_compensate_wt(int add_or_sub, int cformat, int w, int h, int luma_depth, int chroma_depth,
                             const RefBlockDesc* d, int nref, const short* mv1, const short* mv2,
                             const unsigned char* mode, const short* dc, const unsigned char* split,
                             short* const* pic, const short* const* ref1, const short* const* ref2, int wt1,
                             int wt2, int wt_bits);

int ref_motion_compensate(int add_or_sub, int cformat, int w, int h, int luma_depth, int chroma_depth,
                          const RefBlockDesc* d, int nref, const short* mv1, const short* mv2,
                          const unsigned char* mode, const short* dc, const unsigned char* split,
                          short* const* pic, const short* const* ref1, const short* const* ref2) {
    return ref_motion_compensate_wt(add_or_sub, cformat, w, h, luma_depth, chroma_depth, d, nref, mv1, mv2, mode, dc,
                                    split, pic, ref1, ref2, 1, 1, 1);
}

// The same with the picture's reference weights set (PicturePredParams::SetRef1Weight,
// SetRef2Weight, SetPictureWeightsPrecision; 1, 1, 1 are the defaults).
int ref_motion_compensate_wt(int add_or_sub, int cformat, int w, int h, int luma_depth, int chroma_depth,
                             const RefBlockDesc* d, int nref, const short* mv1, const short* mv2,
                             const unsigned char* mode, const short* dc, const unsigned char* split,
                             short* const* pic, const short* const* ref1, const short* const* ref2, int wt1,
                             int wt2, int wt_bits) {
    try {
        const ChromaFormat cf = (ChromaFormat)cformat;
        CodecParams cp(VIDEO_FORMAT_CIF, INTER_PICTURE, nref, true);
        PicturePredParams& ppp = cp.GetPicPredParams();
        setup_ppp(ppp, *d, cf);
        ppp.SetRef1Weight(wt1);
        ppp.SetRef2Weight(wt2);
        ppp.SetPictureWeightsPrecision((unsigned int)wt_bits);
        MvData mv(ppp, 2);
        fill_mvdata(mv, mv1, mv2, mode, dc, split, nref);

        PictureParams pp(cf, w, h, luma_depth, chroma_depth);
        pp.SetPicSort(PictureSort::InterRefPictureSort());
        pp.SetPictureNum(1);
        Picture r1(pp), r2(pp);
        pp.SetPictureNum(5);
        pp.Refs().push_back(1);
        if (nref > 1) pp.Refs().push_back(2);
        Picture cur(pp);
        for (int c = 0; c < 3; ++c) {
            fill_pic(cur.Data((CompSort)c), pic[c]);
            fill_pic(r1.Data((CompSort)c), ref1[c]);
            fill_pic(r2.Data((CompSort)c), nref > 1 ? ref2[c] : ref1[c]);
        }
        r1.GetPparams().SetPictureNum(1);
        r2.GetPparams().SetPictureNum(2);
        Picture* refs[2] = {&r1, &r2};
        MotionCompensator::CompensatePicture(ppp, add_or_sub == 0 ? ADD : SUBTRACT, mv, &cur, refs);
        for (int c = 0; c < 3; ++c) read_pic(cur.Data((CompSort)c), pic[c]);
        return 0;
    } catch (...) {
        return -1;
    }
}

// Motion estimation of one picture against one or two references, run through the
// reference's own classes as PictureCompressor::PixelME / SubPixelME / ModeDecisionME do
// (libdirac_encoder/picture_compress.cpp:76-300): PixelMatcher::DoSearch (stage 1), then
// MEData::SetLambdaMap(num_refs, lambda) and SubpelRefine::DoSubpel (stage 2), then
// ModeDecider::DoModeDecn (stage 3).  Component planes pic/ref1/ref2[3] are the original
// pictures (ME uses luma; mode decision's SetDC uses all three).  Outputs after the last
// stage run: mv[ref][block] (x,y) int16, cost[ref][block] = (SAD, mvcost, total) float,
// and after stage 3 mode, dc[3][block], split[sb], sbcost[sb].
int ref_motion_estimate(int cformat, int w, int h, int luma_depth, int chroma_depth, const RefBlockDesc* d,
                        int nref, const short* const* pic, const short* const* ref1, const short* const* ref2,
                        float lambda, int stages, short* mv_out, float* cost_out, unsigned char* mode_out,
                        short* dc_out, unsigned char* split_out, float* sbcost_out) {
    try {
        const ChromaFormat cf = (ChromaFormat)cformat;
        EncoderParams ep(VIDEO_FORMAT_CIF, INTER_PICTURE, nref, true);
        ep.SetFullSearch(false);
        ep.SetCombinedME(false);
        PicturePredParams& ppp = ep.GetPicPredParams();
        setup_ppp(ppp, *d, cf);

        EncQueue q;
        PictureParams pp(cf, w, h, luma_depth, chroma_depth);
        pp.SetPicSort(PictureSort::IntraRefPictureSort());
        pp.SetPictureNum(0);
        q.PushPicture(pp);
        pp.SetPicSort(PictureSort::InterRefPictureSort());
        pp.SetPictureNum(2);
        q.PushPicture(pp);
        pp.SetPictureNum(1);
        pp.Refs().push_back(0);
        if (nref > 1) pp.Refs().push_back(2);
        q.PushPicture(pp);
        const short* const* src[3] = {ref1, nref > 1 ? ref2 : ref1, pic};
        const int pnum[3] = {0, 2, 1};
        for (int k = 0; k < 3; ++k) {
            EncPicture& ep_k = q.GetPicture(pnum[k]);
            for (int c = 0; c < 3; ++c) fill_pic(ep_k.Data((CompSort)c), src[k][c]);
            ep_k.SetOrigData();
        }
        EncPicture& cur = q.GetPicture(1);
        cur.InitMEData(ppp, nref);
        PixelMatcher pm(ep);
        pm.DoSearch(q, 1);
        MEData& me = cur.GetMEData();
        if (stages >= 2) {
            me.SetLambdaMap(nref, lambda);
            if (d->precision != MV_PRECISION_PIXEL) {
                SubpelRefine sr(ep);
                sr.DoSubpel(q, 1);
            }
        }
        if (stages >= 3) {
            ModeDecider md(ep);
            md.DoModeDecn(q, 1);
        }
        const int ynb = me.Mode().LengthY(), xnb = me.Mode().LengthX();
        const size_t nb = (size_t)ynb * xnb;
        for (int r = 1; r <= nref; ++r)
            for (int j = 0; j < ynb; ++j)
                for (int i = 0; i < xnb; ++i) {
                    const size_t b = (size_t)j * xnb + i;
                    const MVector& v = me.Vectors(r)[j][i];
                    mv_out[((r - 1) * nb + b) * 2] = (short)v.x;
                    mv_out[((r - 1) * nb + b) * 2 + 1] = (short)v.y;
                    const MvCostData& cd = me.PredCosts(r)[j][i];
                    cost_out[((r - 1) * nb + b) * 3] = cd.SAD;
                    cost_out[((r - 1) * nb + b) * 3 + 1] = cd.mvcost;
                    cost_out[((r - 1) * nb + b) * 3 + 2] = cd.total;
                }
        if (stages >= 3) {
            for (int j = 0; j < ynb; ++j)
                for (int i = 0; i < xnb; ++i) {
                    const size_t b = (size_t)j * xnb + i;
                    mode_out[b] = (unsigned char)me.Mode()[j][i];
                    for (int c = 0; c < 3; ++c) dc_out[c * nb + b] = me.DC((CompSort)c)[j][i];
                }
            for (int j = 0; j < me.SBSplit().LengthY(); ++j)
                for (int i = 0; i < me.SBSplit().LengthX(); ++i) {
                    split_out[(size_t)j * me.SBSplit().LengthX() + i] = (unsigned char)me.SBSplit()[j][i];
                    sbcost_out[(size_t)j * me.SBSplit().LengthX() + i] = me.SBCosts()[j][i];
                }
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// Residue coding of one transformed component, as PictureCompressor::CodeResidue runs it
// (libdirac_encoder/picture_compress.cpp:391-461): band weights (CoeffArray::SetBandWeights),
// code blocks (SetupCodeBlocks :582-601), quantiser choice per band from DC to HF
// (SelectQuantisers / SelectMultiQuants :603-677, with the intra DC band's AddSubAverage
// :679-709 restated here because those PictureCompressor members are private), then
// CompCompressor::Compress, which quantises and reconstructs every coefficient in place.
// coeff (ch x cw) is read and overwritten with the reconstruction.  Per band (band-list
// order, 1-based band b at index b-1): quantiser index, skip flag, weight, entropy factor,
// estimated bits, code-block grid (x, y) and the code blocks' skip flags (concatenated).
}  // extern "C"

namespace {

// The band loop of CompCompressor::Compress (comp_compress.cpp:64-140) with each band's coded
// data captured: the same codec per band (IntraDCBandCodec for an intra DC band,
// LFBandCodec for the other low-frequency bands, BandCodec otherwise), coding the bands from
// DC to HF; skipped bands set to zero.  band_data receives the bands' data (the bytes their
// SubbandByteIO carries after its header) in that order; band_bytes[b - 1] their lengths.
// vlc: the variable-length band coders (BandVLC / IntraDCBandVLC, comp_compress.cpp:105-120);
// compress_bytes (optional) receives what each coder's Compress returned (whole bytes written
// before the final alignment).
int code_bands_capture(CoeffArray& c, SubbandList& bands, bool intra, unsigned char* band_data, long long cap,
                       int* band_bytes, bool vlc = false, int* compress_bytes = nullptr) {
    long long at = 0;
    for (int b = bands.Length(); b >= 1; --b) {
        band_bytes[b - 1] = 0;
        if (bands(b).Skipped()) {
            for (int j = bands(b).Yp(); j < bands(b).Yp() + bands(b).Yl(); ++j)
                for (int i = bands(b).Xp(); i < bands(b).Xp() + bands(b).Xl(); ++i) c[j][i] = 0;
            continue;
        }
        SubbandByteIO sb(bands(b));
        int n;
        if (vlc) {
            BandVLC* bc;
            if (intra && b == bands.Length())
                bc = new IntraDCBandVLC(&sb, bands);
            else
                bc = new BandVLC(&sb, 0, bands, b, intra);
            const int whole = bc->Compress(c);
            delete bc;
            if (compress_bytes) compress_bytes[b - 1] = whole;
            sb.ByteAlignOutput();
            n = sb.GetSize();
        } else {
            BandCodec* bc;
            if (b >= bands.Length() - 3) {
                if (intra && b == bands.Length())
                    bc = new IntraDCBandCodec(&sb, TOTAL_COEFF_CTXS, bands);
                else
                    bc = new LFBandCodec(&sb, TOTAL_COEFF_CTXS, bands, b, intra);
            } else {
                bc = new BandCodec(&sb, TOTAL_COEFF_CTXS, bands, b, intra);
            }
            n = bc->Compress(c);
            delete bc;
        }
        const std::string data = sb.ByteIO::GetBytes();
        if ((long long)data.size() != n) return -2;
        if (at + n > cap) return -3;
        std::memcpy(band_data + at, data.data(), n);
        at += n;
        band_bytes[b - 1] = n;
    }
    return 0;
}

int code_residue_impl(int cformat, int w, int h, int comp, int intra, int filter, int depth, int* coeff, int cw,
                      int ch, float lambda, float cpd_scale, int* band_qidx, int* band_skip, double* band_wt,
                      float* band_ecf, int* band_bits, int* band_ncb, unsigned char* cb_skip,
                      unsigned char* band_data, long long cap, int* band_bytes, bool vlc = false,
                      int* compress_bytes = nullptr) {
    try {
        const ChromaFormat cf = (ChromaFormat)cformat;
        const PictureType pt = intra ? INTRA_PICTURE : INTER_PICTURE;
        EncoderParams ep(VIDEO_FORMAT_CUSTOM, pt, 2, true);
        ep.SetXl(w);
        ep.SetYl(h);
        ep.SetTransformDepth(depth);
        ep.SetTransformFilter((WltFilter)filter);
        ep.SetUsualCodeBlocks(pt);
        EntropyCorrector* ec = new EntropyCorrector(depth);
        ep.SetEntropyFactors(ec);
        PictureParams pp(cf, w, h, 8, 8);
        pp.SetPicSort(intra ? PictureSort::IntraRefPictureSort() : PictureSort::InterRefPictureSort());
        if (!intra) pp.Refs().push_back(0);
        CoeffArray c(ch, cw, (CompSort)comp);
        fill_arr(c, coeff);
        SubbandList& bands = c.BandList();
        bands.Init(depth, cw, ch);
        c.SetBandWeights(ep, pp, (CompSort)comp, cpd_scale);
        for (int b = 1; b <= bands.Length(); ++b) {
            int xr = 1, yr = 1;
            if (ep.SpatialPartition()) {
                const int level = depth - (b - 1) / 3;
                const CodeBlocks& cb = ep.GetCodeBlocks(level);
                xr = cb.HorizontalCodeBlocks();
                yr = cb.VerticalCodeBlocks();
            }
            bands(b).SetNumBlocks(yr, xr);
        }
        OneDArray<unsigned int> est_bits(Range(1, 3 * depth + 1));
        for (int b = bands.Length(); b >= 1; --b) {
            Subband& node = bands(b);
            node.SetUsingMultiQuants(ep.GetCodeBlockMode() == QUANT_MULTIPLE &&
                                     (node.GetCodeBlocks().LengthX() > 1 || node.GetCodeBlocks().LengthY() > 1));
        }
        for (int b = bands.Length(); b >= 1; --b) {
            Subband& node = bands(b);
            QuantChooser qc(c, lambda);
            const bool dc_intra = (b == bands.Length()) && intra;
            if (dc_intra) {  // AddSubAverage(SUBTRACT): raster DPCM of the DC band
                ValueType last = 0;
                for (int j = 0; j < node.Yl(); ++j)
                    for (int i = 0; i < node.Xl(); ++i) {
                        const ValueType keep = c[j][i];
                        c[j][i] -= last;
                        last = keep;
                    }
            }
            const float ecf = ep.EntropyFactors().Factor(b, pp, (CompSort)comp);
            qc.SetEntropyCorrection(ecf);
            const int bits = qc.GetBestQuant(node);
            if (dc_intra) {  // AddSubAverage(ADD)
                ValueType last = 0;
                for (int j = 0; j < node.Yl(); ++j)
                    for (int i = 0; i < node.Xl(); ++i) {
                        c[j][i] += last;
                        last = c[j][i];
                    }
            }
            node.SetSkip(bits == 0);
            est_bits[b] = bits;
            band_ecf[b - 1] = ecf;
            band_bits[b - 1] = bits;
        }
        size_t k = 0;
        for (int b = 1; b <= bands.Length(); ++b) {
            const Subband& node = bands(b);
            band_qidx[b - 1] = node.QuantIndex();
            band_skip[b - 1] = node.Skipped() ? 1 : 0;
            band_wt[b - 1] = node.Wt();
            const TwoDArray<CodeBlock>& cbs = node.GetCodeBlocks();
            band_ncb[2 * (b - 1)] = cbs.LengthX();
            band_ncb[2 * (b - 1) + 1] = cbs.LengthY();
            for (int j = 0; j < cbs.LengthY(); ++j)
                for (int i = 0; i < cbs.LengthX(); ++i) cb_skip[k++] = cbs[j][i].Skipped() ? 1 : 0;
        }
        if (band_data) {
            const int rc = code_bands_capture(c, bands, intra != 0, band_data, cap, band_bytes, vlc, compress_bytes);
            if (rc) {
                delete ec;
                return rc;
            }
        } else {
            CompCompressor cc(ep, pp);
            ComponentByteIO* out = cc.Compress(c, bands, (CompSort)comp, est_bits);
            delete out;
        }
        read_arr(c, coeff);
        delete ec;
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // namespace

extern "C" {

int ref_code_residue(int cformat, int w, int h, int comp, int intra, int filter, int depth, int* coeff, int cw,
                     int ch, float lambda, float cpd_scale, int* band_qidx, int* band_skip, double* band_wt,
                     float* band_ecf, int* band_bits, int* band_ncb, unsigned char* cb_skip) {
    return code_residue_impl(cformat, w, h, comp, intra, filter, depth, coeff, cw, ch, lambda, cpd_scale, band_qidx,
                             band_skip, band_wt, band_ecf, band_bits, band_ncb, cb_skip, nullptr, 0, nullptr);
}

// The reference's band coders (BandCodec, LFBandCodec; band_codec_template.h:24-200) on given
// signed indices of an inter picture's component: every band and code block at quantiser index
// 0, whose factor is 1 (CodeVal's abs << 2 / 4), so the coded values are the indices
// themselves.  band_ncb: per band the code blocks across and down; a code block is skipped
// when all its indices are zero (cb_skip receives the flags).  Coded data DC band first, as
// ref_code_residue_bytes.
int ref_code_inter_indices_bytes(int depth, const int* idx, int cw, int ch, const int* band_ncb,
                                 unsigned char* cb_skip, unsigned char* band_data, long long cap, int* band_bytes) {
    try {
        CoeffArray c(ch, cw, Y_COMP);
        fill_arr(c, idx);
        SubbandList& bands = c.BandList();
        bands.Init(depth, cw, ch);
        size_t k = 0;
        for (int b = 1; b <= bands.Length(); ++b) {
            Subband& node = bands(b);
            node.SetNumBlocks(band_ncb[2 * (b - 1) + 1], band_ncb[2 * (b - 1)]);
            node.SetQuantIndex(0);
            node.SetSkip(false);
            node.SetUsingMultiQuants(false);
            TwoDArray<CodeBlock>& cbs = node.GetCodeBlocks();
            for (int j = 0; j < cbs.LengthY(); ++j)
                for (int i = 0; i < cbs.LengthX(); ++i) {
                    CodeBlock& blk = cbs[j][i];
                    blk.SetQuantIndex(0);
                    bool zero = true;
                    for (int y = blk.Ystart(); y < blk.Yend() && zero; ++y)
                        for (int x = blk.Xstart(); x < blk.Xend(); ++x)
                            if (c[y][x] != 0) {
                                zero = false;
                                break;
                            }
                    blk.SetSkip(zero);
                    cb_skip[k++] = zero ? 1 : 0;
                }
        }
        return code_bands_capture(c, bands, false, band_data, cap, band_bytes);
    } catch (...) {
        return -1;
    }
}

// As ref_code_residue, and each coded band's arithmetic-coded data captured (DC band first).
int ref_code_residue_bytes(int cformat, int w, int h, int comp, int intra, int filter, int depth, int* coeff, int cw,
                           int ch, float lambda, float cpd_scale, int* band_qidx, int* band_skip, double* band_wt,
                           float* band_ecf, int* band_bits, int* band_ncb, unsigned char* cb_skip,
                           unsigned char* band_data, long long cap, int* band_bytes) {
    return code_residue_impl(cformat, w, h, comp, intra, filter, depth, coeff, cw, ch, lambda, cpd_scale, band_qidx,
                             band_skip, band_wt, band_ecf, band_bits, band_ncb, cb_skip, band_data, cap, band_bytes);
}

// The variable-length band coders' data (-use_vlc), and each coder's Compress result.
int ref_code_residue_vlc_bytes(int cformat, int w, int h, int comp, int intra, int filter, int depth, int* coeff,
                               int cw, int ch, float lambda, float cpd_scale, int* band_qidx, int* band_skip,
                               double* band_wt, float* band_ecf, int* band_bits, int* band_ncb,
                               unsigned char* cb_skip, unsigned char* band_data, long long cap, int* band_bytes,
                               int* compress_bytes) {
    return code_residue_impl(cformat, w, h, comp, intra, filter, depth, coeff, cw, ch, lambda, cpd_scale, band_qidx,
                             band_skip, band_wt, band_ecf, band_bits, band_ncb, cb_skip, band_data, cap, band_bytes,
                             true, compress_bytes);
}

// CWMFilterComponent on a dense w x h component, in place.
int ref_cwm_filter(short* pic, int w, int h, int strength) {
    try {
        PicArray a(h, w);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) a[y][x] = pic[y * w + x];
        CWMFilterComponent(a, strength);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) pic[y * w + x] = a[y][x];
        return 0;
    } catch (...) {
        return -1;
    }
}

// LPFilter (the RECTLP residue prefilter) on a dense w x h component, in place.
int ref_lp_filter(short* pic, int w, int h, float qf, int strength) {
    try {
        PicArray a(h, w);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) a[y][x] = pic[y * w + x];
        LPFilter(a, qf, strength);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) pic[y * w + x] = a[y][x];
        return 0;
    } catch (...) {
        return -1;
    }
}

// DiagFilter (the DIAGLP residue prefilter) on a dense w x h component, in place.
int ref_diag_filter(short* pic, int w, int h, float qf, int strength) {
    try {
        PicArray a(h, w);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) a[y][x] = pic[y * w + x];
        DiagFilter(a, qf, strength);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) pic[y * w + x] = a[y][x];
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
