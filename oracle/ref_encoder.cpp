// Test infrastructure only: runs the reference encoder through its own public C API
// (libdirac_encoder/dirac_encoder.h: dirac_encoder_context_init, dirac_encoder_init,
// dirac_encoder_load, dirac_encoder_output, dirac_encoder_end_sequence, dirac_encoder_close)
// and returns its locally decoded pictures (and, from ref_encode_stream, its bitstream), so
// that the tests can pin a whole coding loop
// (GOP structure, cut detection, lambdas, motion estimation, compensation, transform and
// quantisation) against the reference itself.  Linked into oracle/_ref/libdirac_ref.so.
//
// Entropy-correction factors.  The reference adapts EntropyCorrector's factors after each
// coded band from the arithmetic coder's actual byte counts (comp_compress.cpp:128,
// common.cpp:134-151).  Arithmetic coding is not part of the data-parallel path, so a
// coding loop without it keeps the initial factors (common.cpp:79-131).  With freeze != 0 this
// driver makes the reference do the same: the library is linked with
// --wrap=<EntropyCorrector::Update>, and the wrapper below skips the update while frozen.
// Everything else in the encoder runs unmodified.

#include <cstdint>
#include <cstring>
#include <vector>

#include <libdirac_common/common.h>
#include <libdirac_encoder/dirac_encoder.h>

using namespace dirac;

namespace {
bool g_freeze_factors = false;
}

extern "C" {

// The linker routes every call of EntropyCorrector::Update from other objects here
// (-Wl,--wrap=_ZN5dirac16EntropyCorrector6UpdateEiRKNS_13PictureParamsENS_8CompSortEii).
void __real__ZN5dirac16EntropyCorrector6UpdateEiRKNS_13PictureParamsENS_8CompSortEii(
    EntropyCorrector* self, int bandnum, const PictureParams& pp, CompSort c, int est_bits, int actual_bits);

void __wrap__ZN5dirac16EntropyCorrector6UpdateEiRKNS_13PictureParamsENS_8CompSortEii(
    EntropyCorrector* self, int bandnum, const PictureParams& pp, CompSort c, int est_bits, int actual_bits) {
    if (g_freeze_factors) return;
    __real__ZN5dirac16EntropyCorrector6UpdateEiRKNS_13PictureParamsENS_8CompSortEii(self, bandnum, pp, c, est_bits,
                                                                                   actual_bits);
}

struct RefEncParams {
    int video_format;   // VideoFormat preset the context starts from
    int cformat;        // ChromaFormat (0 4:4:4, 1 4:2:2, 2 4:2:0)
    int width, height;
    float qf;
    int l1_sep, num_l1;
    float cpd;
    int xblen, yblen, xbsep, ybsep;
    int mv_precision;
    int intra_filter, inter_filter, wlt_depth;
    int use_vlc;        // 1: variable-length coefficient coding (-use_vlc), 0: arithmetic coding
    int field_coding;   // 1: interlaced frames coded as fields (picture_coding_mode 1)
};

// Encodes nframes 8-bit planar frames (Y then U then V, dense, frame after frame).
// recon (nframes frames, same layout) receives the locally decoded pictures by picture
// number (field coding: 2 nframes fields of half height, each Y then U then V, dense);
// ptype[pnum] = 1 for intra, 0 for inter, -1 if never returned, -2 for a first field (the
// encoder reports a frame's type by its second field); *bytes = total
// bitstream bytes.  freeze: keep the initial entropy-correction factors.
// Returns 0, or -1 on an encoder failure.
}  // extern "C"

namespace {

// The encode of ref_encode_sequence; the coded bitstream is appended to *stream when given.
int encode_impl(const RefEncParams* p, int nframes, const unsigned char* frames, int freeze, unsigned char* recon,
                int* ptype, long long* bytes, std::vector<unsigned char>* stream) {
    g_freeze_factors = freeze != 0;
    dirac_encoder_context_t ctx;
    dirac_encoder_context_init(&ctx, static_cast<dirac_encoder_presets_t>(p->video_format));
    ctx.src_params.width = p->width;
    ctx.src_params.height = p->height;
    ctx.src_params.chroma = static_cast<dirac_chroma_t>(p->cformat);
    ctx.src_params.source_sampling = 0;
    ctx.enc_params.qf = p->qf;
    ctx.enc_params.L1_sep = p->l1_sep;
    ctx.enc_params.num_L1 = p->num_l1;
    ctx.enc_params.cpd = p->cpd;
    ctx.enc_params.xblen = p->xblen;
    ctx.enc_params.yblen = p->yblen;
    ctx.enc_params.xbsep = p->xbsep;
    ctx.enc_params.ybsep = p->ybsep;
    ctx.enc_params.mv_precision = static_cast<dirac_mvprecision_t>(p->mv_precision);
    ctx.enc_params.intra_wlt_filter = static_cast<dirac_wlt_filter_t>(p->intra_filter);
    ctx.enc_params.inter_wlt_filter = static_cast<dirac_wlt_filter_t>(p->inter_filter);
    ctx.enc_params.wlt_depth = p->wlt_depth;
    ctx.enc_params.spatial_partition = 1;
    ctx.enc_params.multi_quants = 0;
    ctx.enc_params.using_ac = p->use_vlc ? 0 : 1;
    ctx.enc_params.trate = 0;
    ctx.enc_params.lossless = 0;
    ctx.enc_params.full_search = 0;
    ctx.enc_params.picture_coding_mode = p->field_coding ? 1 : 0;
    ctx.enc_params.prefilter = NO_PF;
    ctx.instr_flag = 0;
    ctx.decode_flag = 1;

    dirac_encoder_t* enc = dirac_encoder_init(&ctx, 0);
    if (!enc) {
        g_freeze_factors = false;
        return -1;
    }
    const int cw = p->cformat == 0 ? p->width : p->width / 2;
    const int ch = p->cformat == 2 ? p->height / 2 : p->height;
    const size_t fsize = (size_t)p->width * p->height + 2 * (size_t)cw * ch;
    // pictures: frames, or two fields per frame; top field first as the video format's
    // defaults set it (the context's field is not read back by the encoder)
    const int npics = p->field_coding ? 2 * nframes : nframes;
    const bool tff = ctx.src_params.topfieldfirst != 0;
    for (int i = 0; i < npics; ++i) ptype[i] = -1;
    std::vector<unsigned char> out(1 << 24);
    long long total = 0;
    int rc = 0;
    // every output call either codes a picture or reports BUFFER / EOS, so a bounded
    // number of calls per loaded frame always suffices
    auto drain = [&](bool to_eos) -> int {
        for (int guard = 0; guard < 4 * npics + 64; ++guard) {
            enc->enc_buf.buffer = out.data();
            enc->enc_buf.size = (int)out.size();
            const dirac_encoder_state_t st = dirac_encoder_output(enc);
            if (st == ENC_STATE_INVALID) return -1;
            if (st == ENC_STATE_AVAIL || st == ENC_STATE_EOS) {
                total += enc->enc_buf.size;
                if (stream) stream->insert(stream->end(), out.data(), out.data() + enc->enc_buf.size);
            }
            if (enc->decoded_frame_avail) {
                const int pn = enc->dec_pparams.pnum;
                if (pn >= 0 && pn < npics && !p->field_coding) {
                    unsigned char* dst = recon + (size_t)pn * fsize;
                    std::memcpy(dst, enc->dec_buf.buf[0], (size_t)p->width * p->height);
                    std::memcpy(dst + (size_t)p->width * p->height, enc->dec_buf.buf[1], (size_t)cw * ch);
                    std::memcpy(dst + (size_t)p->width * p->height + (size_t)cw * ch, enc->dec_buf.buf[2],
                                (size_t)cw * ch);
                    ptype[pn] = enc->dec_pparams.ptype == INTRA_PICTURE ? 1 : 0;
                } else if (pn >= 1 && pn < npics && pn % 2 == 1) {
                    // the API reports a frame once its second field is written
                    // (StreamFieldOutput::WriteFieldComponent, pic_io.cpp:150-240): the output
                    // frame then holds fields pn - 1 and pn in alternate rows
                    for (int f = pn - 1; f <= pn; ++f) {
                        const int row0 = tff ? (f % 2) : 1 - (f % 2);
                        unsigned char* dst = recon + (size_t)f * (fsize / 2);
                        const int ws[3] = {p->width, cw, cw}, hs[3] = {p->height, ch, ch};
                        for (int c = 0; c < 3; ++c) {
                            for (int y = 0; y < hs[c] / 2; ++y)
                                std::memcpy(dst + (size_t)y * ws[c],
                                            enc->dec_buf.buf[c] + (size_t)(2 * y + row0) * ws[c], (size_t)ws[c]);
                            dst += (size_t)ws[c] * (hs[c] / 2);
                        }
                    }
                    // only the second field's type is reported
                    ptype[pn - 1] = -2;
                    ptype[pn] = enc->dec_pparams.ptype == INTRA_PICTURE ? 1 : 0;
                }
            }
            if (st == ENC_STATE_EOS) return 1;
            if (st == ENC_STATE_BUFFER && !to_eos) return 0;
        }
        return -1;
    };
    for (int i = 0; i < nframes && rc == 0; ++i) {
        unsigned char* src = const_cast<unsigned char*>(frames + (size_t)i * fsize);
        if (dirac_encoder_load(enc, src, (int)fsize) < 0) rc = -1;
        else if (drain(false) < 0) rc = -1;
    }
    if (rc == 0) {
        dirac_encoder_end_sequence(enc);
        if (drain(true) < 0) rc = -1;
    }
    dirac_encoder_close(enc);
    g_freeze_factors = false;
    *bytes = total;
    return rc;
}

}  // namespace

extern "C" {

int ref_encode_sequence(const RefEncParams* p, int nframes, const unsigned char* frames, int freeze,
                        unsigned char* recon, int* ptype, long long* bytes) {
    return encode_impl(p, nframes, frames, freeze, recon, ptype, bytes, nullptr);
}

// As ref_encode_sequence, and the coded bitstream copied to stream (capacity cap bytes;
// *bytes is its length).  Returns -2 when the stream does not fit.
int ref_encode_stream(const RefEncParams* p, int nframes, const unsigned char* frames, int freeze,
                      unsigned char* recon, int* ptype, unsigned char* stream, long long cap, long long* bytes) {
    std::vector<unsigned char> s;
    const int rc = encode_impl(p, nframes, frames, freeze, recon, ptype, bytes, &s);
    if (rc) return rc;
    if ((long long)s.size() > cap) return -2;
    std::memcpy(stream, s.data(), s.size());
    *bytes = (long long)s.size();
    return 0;
}

}  // extern "C"
