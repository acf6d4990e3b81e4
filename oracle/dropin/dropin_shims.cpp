// The reference-side binding of the hot path, as a maintainer would add it: the bodies of the
// reference's hot-path methods replaced by calls into libdiracgpu's C ABI, everything else of
// the reference unchanged.  Compiled only into oracle/_ref/libdirac_dropin.so, together with
// the reference's own sources (oracle/Makefile weakens the replaced definitions in the
// reference's objects, so these strong ones take their place at link time); test
// infrastructure that shows the drop-in: the stock dirac_encoder_* / dirac_decoder_* API,
// driven unchanged, produces the stock reference's bitstream and pictures.
//
// Replaced (reference file:line):
//   WaveletTransform::Transform               libdirac_common/wavelet_utils.cpp:440-485
//   MotionCompensator::CompensatePicture      libdirac_common/mot_comp.cpp:63-104 (static form)
//   PictureCompressor::PixelME                libdirac_encoder/picture_compress.cpp:76-80
//   PictureCompressor::SubPixelME             libdirac_encoder/picture_compress.cpp:198-250
//   PictureCompressor::ModeDecisionME         libdirac_encoder/picture_compress.cpp:252-285
//   PictureCompressor::SelectQuantisers       libdirac_encoder/picture_compress.cpp:603-646
// The decoder reaches the GPU through the same WaveletTransform::Transform (BACKWARD) and
// MotionCompensator::CompensatePicture (ADD) that PictureDecompressor::Decompress calls
// (libdirac_decoder/picture_decompress.cpp:73-212).
//
// Every call copies its arrays to the device and back on the legacy default stream: the
// reference keeps its pictures in host memory, and this binding changes none of its data
// structures.  A failure is raised as a DiracException, which the reference's C API turns
// into its error return (dirac_encoder.cpp:1074-1085).

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <dirac_gpu.h>
#include <libdirac_common/dirac_exception.h>
#include <libdirac_common/mot_comp.h>
#include <libdirac_common/motion.h>
#include <libdirac_common/picture.h>
#include <libdirac_common/wavelet_utils.h>
#include <libdirac_encoder/enc_picture.h>
#include <libdirac_encoder/enc_queue.h>
#include <libdirac_encoder/picture_compress.h>

using namespace dirac;

namespace {

void fail(const std::string& what) {
    DIRAC_THROW_EXCEPTION(ERR_UNSUPPORTED_STREAM_DATA, "libdiracgpu: " + what, SEVERITY_TERMINATE);
}

void check(int rc, const char* what) {
    if (rc != DGPU_OK) fail(std::string(what) + " returned " + std::to_string(rc) + " (" + dgpu_last_error() + ")");
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(std::string(what) + ": " + cudaGetErrorString(e));
}

// One device allocation, freed with the object.
struct DevMem {
    void* p = nullptr;
    explicit DevMem(size_t bytes) { check_cuda(cudaMalloc(&p, bytes ? bytes : 1), "cudaMalloc"); }
    ~DevMem() { cudaFree(p); }
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// A PicArray (one contiguous block, rows of LengthX samples) on the device.
struct DevPlane {
    int w, h;
    DevMem mem;
    explicit DevPlane(const PicArray& a)
        : w(a.LengthX()), h(a.LengthY()), mem((size_t)a.LengthX() * a.LengthY() * sizeof(int16_t)) {
        check_cuda(cudaMemcpy(mem.p, &a[0][0], (size_t)w * h * sizeof(int16_t), cudaMemcpyHostToDevice), "upload");
    }
    void download(PicArray& a) const {
        check_cuda(cudaMemcpy(&a[0][0], mem.p, (size_t)w * h * sizeof(int16_t), cudaMemcpyDeviceToHost), "download");
    }
    int16_t* ptr() const { return mem.as<int16_t>(); }
};

dgpu_block_params block_params(const PicturePredParams& ppp) {
    const OLBParams& o = ppp.LumaBParams(2);
    dgpu_block_params bp;
    bp.precision = (int)ppp.MVPrecision();
    bp.xblen = o.Xblen();
    bp.yblen = o.Yblen();
    bp.xbsep = o.Xbsep();
    bp.ybsep = o.Ybsep();
    bp.xnum_sb = ppp.XNumSB();
    bp.ynum_sb = ppp.YNumSB();
    return bp;
}

// Motion estimation of picture pnum through the given stage (1 pel search, 2 + lambda map and
// sub-pel refinement, 3 + mode decision and DC values), from the original pictures as the
// reference's PixelMatcher / SubpelRefine / ModeDecider read them, results written into the
// picture's MEData where those classes leave theirs.
void estimate(EncQueue& q, int pnum, int stages, float lambda) {
    EncPicture& cur = q.GetPicture(pnum);
    const PictureParams& pp = cur.GetPparams();
    MEData& me = cur.GetMEData();
    const PicturePredParams& ppp = me.GetPicPredParams();
    const std::vector<int>& refs = pp.Refs();
    const int nref = (int)refs.size();
    if (nref < 1 || nref > 2) fail("motion estimation needs one or two references");
    if (ppp.MVPrecision() == MV_PRECISION_PIXEL) fail("pixel-accurate motion vectors are not supported");
    const dgpu_block_params bp = block_params(ppp);
    const int xnb = me.Mode().LengthX(), ynb = me.Mode().LengthY();
    if (xnb != 4 * bp.xnum_sb || ynb != 4 * bp.ynum_sb) fail("unexpected block grid");
    const size_t nb = (size_t)xnb * ynb, nsb = (size_t)bp.xnum_sb * bp.ynum_sb;

    std::vector<DevPlane*> planes;
    auto upload = [&](const EncPicture& p, const int16_t** out) {
        for (int c = 0; c < 3; ++c) {
            planes.push_back(new DevPlane(p.OrigData((CompSort)c)));
            out[c] = planes.back()->ptr();
        }
    };
    const int16_t* dpic[3];
    const int16_t* dref1[3];
    const int16_t* dref2[3];
    upload(cur, dpic);
    upload(q.GetPicture(refs[0]), dref1);
    if (nref > 1) upload(q.GetPicture(refs[1]), dref2);
    DevMem mv(nref * nb * 2 * sizeof(int16_t)), cost(nref * nb * 3 * sizeof(float)), mode(nb),
        dc(3 * nb * sizeof(int16_t)), split(nsb), sbcost(nsb * sizeof(float));
    const int rc = dgpu_motion_estimate((int)pp.CFormat(), pp.Xl(), pp.Yl(), &bp, nref, dpic, dref1,
                                        nref > 1 ? dref2 : nullptr, (int)pp.LumaDepth(), lambda, stages,
                                        mv.as<int16_t>(), cost.as<float>(), mode.as<uint8_t>(), dc.as<int16_t>(),
                                        split.as<uint8_t>(), sbcost.as<float>(), nullptr, 0, nullptr);
    for (DevPlane* p : planes) delete p;
    check(rc, "dgpu_motion_estimate");

    std::vector<int16_t> hmv(nref * nb * 2);
    std::vector<float> hcost(nref * nb * 3);
    check_cuda(cudaMemcpy(hmv.data(), mv.p, hmv.size() * sizeof(int16_t), cudaMemcpyDeviceToHost), "download");
    check_cuda(cudaMemcpy(hcost.data(), cost.p, hcost.size() * sizeof(float), cudaMemcpyDeviceToHost), "download");
    for (int r = 1; r <= nref; ++r) {
        MvArray& v = me.Vectors(r);
        TwoDArray<MvCostData>& pc = me.PredCosts(r);
        for (int j = 0; j < ynb; ++j)
            for (int i = 0; i < xnb; ++i) {
                const size_t b = (size_t)(r - 1) * nb + (size_t)j * xnb + i;
                v[j][i].x = hmv[2 * b];
                v[j][i].y = hmv[2 * b + 1];
                pc[j][i].SAD = hcost[3 * b];
                pc[j][i].mvcost = hcost[3 * b + 1];
                pc[j][i].total = hcost[3 * b + 2];
            }
    }
    if (stages < 3) return;
    std::vector<uint8_t> hmode(nb), hsplit(nsb);
    std::vector<int16_t> hdc(3 * nb);
    std::vector<float> hsbcost(nsb);
    check_cuda(cudaMemcpy(hmode.data(), mode.p, nb, cudaMemcpyDeviceToHost), "download");
    check_cuda(cudaMemcpy(hdc.data(), dc.p, hdc.size() * sizeof(int16_t), cudaMemcpyDeviceToHost), "download");
    check_cuda(cudaMemcpy(hsplit.data(), split.p, nsb, cudaMemcpyDeviceToHost), "download");
    check_cuda(cudaMemcpy(hsbcost.data(), sbcost.p, nsb * sizeof(float), cudaMemcpyDeviceToHost), "download");
    for (int j = 0; j < ynb; ++j)
        for (int i = 0; i < xnb; ++i) {
            const size_t b = (size_t)j * xnb + i;
            me.Mode()[j][i] = (PredMode)hmode[b];
            for (int c = 0; c < 3; ++c) me.DC((CompSort)c)[j][i] = hdc[c * nb + b];
        }
    for (int j = 0; j < bp.ynum_sb; ++j)
        for (int i = 0; i < bp.xnum_sb; ++i) {
            me.SBSplit()[j][i] = hsplit[(size_t)j * bp.xnum_sb + i];
            me.SBCosts()[j][i] = hsbcost[(size_t)j * bp.xnum_sb + i];
        }
}

}  // namespace

namespace dirac {

void WaveletTransform::Transform(const Direction d, PicArray& pic_data, CoeffArray& coeff_data) {
    check(dgpu_wavelet_transform_host(d == FORWARD ? DGPU_FORWARD : DGPU_BACKWARD, (int)m_filt_sort, m_depth,
                                      &pic_data[0][0], pic_data.LengthX(), pic_data.LengthY(), pic_data.LengthX(),
                                      &coeff_data[0][0], coeff_data.LengthX(), coeff_data.LengthY(),
                                      coeff_data.LengthX()),
          "dgpu_wavelet_transform_host");
    if (d == FORWARD)
        coeff_data.BandList().Init(m_depth, coeff_data.LengthX(), coeff_data.LengthY());
    else
        coeff_data.BandList().Clear();  // as the reference: the band list no longer describes the data
}

void MotionCompensator::CompensatePicture(const PicturePredParams& ppp, const AddOrSub direction,
                                          const MvData& mv_data, Picture* in_pic, Picture* refsptr[2]) {
    const PictureParams& pp = in_pic->GetPparams();
    if (!pp.PicSort().IsInter()) return;  // only inter pictures are compensated
    const int nref = (int)pp.Refs().size();
    if (nref < 2) refsptr[1] = refsptr[0];
    const dgpu_block_params bp = block_params(ppp);
    const int xnb = mv_data.Mode().LengthX(), ynb = mv_data.Mode().LengthY();
    const size_t nb = (size_t)xnb * ynb, nsb = (size_t)bp.xnum_sb * bp.ynum_sb;

    std::vector<int16_t> hmv[2];
    for (int r = 0; r < nref; ++r) {
        const MvArray& v = mv_data.Vectors(r + 1);
        hmv[r].resize(2 * nb);
        for (int j = 0; j < ynb; ++j)
            for (int i = 0; i < xnb; ++i) {
                hmv[r][2 * ((size_t)j * xnb + i)] = (int16_t)v[j][i].x;
                hmv[r][2 * ((size_t)j * xnb + i) + 1] = (int16_t)v[j][i].y;
            }
    }
    std::vector<uint8_t> hmode(nb), hsplit(nsb);
    std::vector<int16_t> hdc(3 * nb);
    for (int j = 0; j < ynb; ++j)
        for (int i = 0; i < xnb; ++i) {
            hmode[(size_t)j * xnb + i] = (uint8_t)mv_data.Mode()[j][i];
            for (int c = 0; c < 3; ++c) hdc[c * nb + (size_t)j * xnb + i] = mv_data.DC((CompSort)c)[j][i];
        }
    for (int j = 0; j < bp.ynum_sb; ++j)
        for (int i = 0; i < bp.xnum_sb; ++i) hsplit[(size_t)j * bp.xnum_sb + i] = (uint8_t)mv_data.SBSplit()[j][i];

    DevMem mv1(2 * nb * sizeof(int16_t)), mv2(2 * nb * sizeof(int16_t)), mode(nb), dc(3 * nb * sizeof(int16_t)),
        split(nsb);
    check_cuda(cudaMemcpy(mv1.p, hmv[0].data(), 2 * nb * sizeof(int16_t), cudaMemcpyHostToDevice), "upload");
    if (nref > 1)
        check_cuda(cudaMemcpy(mv2.p, hmv[1].data(), 2 * nb * sizeof(int16_t), cudaMemcpyHostToDevice), "upload");
    check_cuda(cudaMemcpy(mode.p, hmode.data(), nb, cudaMemcpyHostToDevice), "upload");
    check_cuda(cudaMemcpy(dc.p, hdc.data(), hdc.size() * sizeof(int16_t), cudaMemcpyHostToDevice), "upload");
    check_cuda(cudaMemcpy(split.p, hsplit.data(), nsb, cudaMemcpyHostToDevice), "upload");

    // the references' upconverted reconstructed planes (Picture::UpData, picture.cpp:141-199)
    std::vector<DevPlane*> keep;
    std::vector<DevMem*> ups;
    int16_t* dpic[3];
    int pstride[3];
    const int16_t* up[2][3];
    for (int c = 0; c < 3; ++c) {
        keep.push_back(new DevPlane(in_pic->Data((CompSort)c)));
        dpic[c] = keep.back()->ptr();
        pstride[c] = keep.back()->w;
        const int depth = (int)(c == 0 ? pp.LumaDepth() : pp.ChromaDepth());
        for (int r = 0; r < (nref > 1 ? 2 : 1); ++r) {
            DevPlane src(refsptr[r]->Data((CompSort)c));
            ups.push_back(new DevMem((size_t)4 * src.w * src.h * sizeof(int16_t)));
            check(dgpu_upconvert(src.ptr(), src.w, src.h, src.w, depth, ups.back()->as<int16_t>(), 2 * src.w, nullptr),
                  "dgpu_upconvert");
            up[r][c] = ups.back()->as<int16_t>();
        }
    }
    // the picture's reference weights (the defaults 1, 1, 1 unless the stream sets others)
    const int rc = dgpu_motion_compensate_weighted(
        direction == ADD ? DGPU_ADD : DGPU_SUBTRACT, (int)pp.CFormat(), pp.Xl(), pp.Yl(), &bp, mv1.as<int16_t>(),
        nref > 1 ? mv2.as<int16_t>() : nullptr, mode.as<uint8_t>(), dc.as<int16_t>(), split.as<uint8_t>(), dpic,
        pstride, up[0], nref > 1 ? up[1] : nullptr, 0, 0, ppp.Ref1Weight(), ppp.Ref2Weight(),
        (int)ppp.PictureWeightsBits(), nullptr);
    if (rc == DGPU_OK)
        for (int c = 0; c < 3; ++c) keep[c]->download(in_pic->Data((CompSort)c));
    for (DevPlane* p : keep) delete p;
    for (DevMem* m : ups) delete m;
    check(rc, "dgpu_motion_compensate_weighted");
}

void PictureCompressor::PixelME(EncQueue& my_buffer, int pnum) { estimate(my_buffer, pnum, 1, 0.0f); }

void PictureCompressor::SubPixelME(EncQueue& my_buffer, int pnum) {
    EncPicture& pic = my_buffer.GetPicture(pnum);
    const PictureParams& pparams = pic.GetPparams();
    MEData& me_data = pic.GetMEData();
    const float lambda = pparams.IsBPicture() ? m_encparams.L2MELambda() : m_encparams.L1MELambda();
    // the reference's own lambda map stays in the MEData for its other readers; the device
    // computes the same map from the same lambda
    me_data.SetLambdaMap(pparams.NumRefs(), lambda);
    m_orig_prec = me_data.GetPicPredParams().MVPrecision();
    estimate(my_buffer, pnum, 2, lambda);
}

void PictureCompressor::ModeDecisionME(EncQueue& my_buffer, int pnum) {
    const PictureParams& pparams = my_buffer.GetPicture(pnum).GetPparams();
    const float lambda = pparams.IsBPicture() ? m_encparams.L2MELambda() : m_encparams.L1MELambda();
    estimate(my_buffer, pnum, 3, lambda);
}

void PictureCompressor::SelectQuantisers(CoeffArray& coeff_data, SubbandList& bands, const float lambda,
                                         OneDArray<unsigned int>& est_bits, const CodeBlockMode cb_mode,
                                         const PictureParams& pp, const CompSort csort) {
    const int nb = bands.Length();
    for (int b = nb; b >= 1; --b)
        bands(b).SetUsingMultiQuants(cb_mode == QUANT_MULTIPLE && (bands(b).GetCodeBlocks().LengthX() > 1 ||
                                                                   bands(b).GetCodeBlocks().LengthY() > 1));
    if (m_encparams.Lossless()) {  // the reference's lossless branch: quantiser 0 everywhere
        for (int b = nb; b >= 1; --b) {
            bands(b).SetQuantIndex(0);
            est_bits[b] = 0;
            TwoDArray<CodeBlock>& blocks = bands(b).GetCodeBlocks();
            for (int j = 0; j < blocks.LengthY(); ++j)
                for (int i = 0; i < blocks.LengthX(); ++i) blocks[j][i].SetQuantIndex(0);
        }
        return;
    }
    const int depth = (nb - 1) / 3, intra = pp.PicSort().IsIntra() ? 1 : 0;
    const int cw = coeff_data.LengthX(), ch = coeff_data.LengthY();
    std::vector<float> wt(nb), ecf(nb);
    std::vector<int> ncb(2 * nb), qidx(nb), skip(nb), bits(nb);
    size_t ncb_total = 0;
    for (int b = 1; b <= nb; ++b) {
        wt[b - 1] = (float)bands(b).Wt();
        ecf[b - 1] = m_encparams.EntropyFactors().Factor(b, pp, csort);
        ncb[2 * (b - 1)] = bands(b).GetCodeBlocks().LengthX();
        ncb[2 * (b - 1) + 1] = bands(b).GetCodeBlocks().LengthY();
        ncb_total += (size_t)ncb[2 * (b - 1)] * ncb[2 * (b - 1) + 1];
    }
    std::vector<uint8_t> cb_skip(ncb_total);
    // the device reconstructs its copy in place; the reference's band coders quantise the
    // original coefficients again, so the host array stays as it is
    DevMem dcoeff((size_t)cw * ch * sizeof(int32_t));
    check_cuda(cudaMemcpy(dcoeff.p, &coeff_data[0][0], (size_t)cw * ch * sizeof(int32_t), cudaMemcpyHostToDevice),
               "upload");
    int32_t* dptr = dcoeff.as<int32_t>();
    check(dgpu_code_residue_batch(1, &intra, &depth, &dptr, &cw, &ch, &lambda, wt.data(), ecf.data(), ncb.data(),
                                  qidx.data(), skip.data(), bits.data(), cb_skip.data(), nullptr, nullptr, 0, nullptr),
          "dgpu_code_residue_batch");
    size_t k = 0;
    for (int b = 1; b <= nb; ++b) {
        Subband& node = bands(b);
        TwoDArray<CodeBlock>& blocks = node.GetCodeBlocks();
        est_bits[b] = (unsigned int)bits[b - 1];
        if (bits[b - 1] != 0) {  // QuantChooser::GetBestQuant's choices (quant_chooser.cpp:127-142)
            node.SetQuantIndex(qidx[b - 1]);
            for (int j = 0; j < blocks.LengthY(); ++j)
                for (int i = 0; i < blocks.LengthX(); ++i) {
                    blocks[j][i].SetQuantIndex(qidx[b - 1]);
                    blocks[j][i].SetSkip(cb_skip[k + (size_t)j * blocks.LengthX() + i] != 0);
                }
        }
        node.SetSkip(bits[b - 1] == 0);
        k += (size_t)blocks.LengthX() * blocks.LengthY();
    }
}

}  // namespace dirac
