// Sequence decoder: the data-parallel part of the reference decoder's picture decoding over
// the library's kernels, every picture resident on the device.
//
// Per picture, on the decoder's stream (PictureDecompressor::Decompress,
// libdirac_decoder/picture_decompress.cpp:73-212): dequantisation of the three components'
// entropy-decoded indices (dgpu_dequantise_batch: the band decoders' arithmetic, the intra
// DC prediction, skipped bands and code blocks), the inverse transform
// (WaveletTransform::Transform BACKWARD), or zero samples for a picture without coded
// coefficients; for inter pictures motion compensation ADD against the references'
// upconverted samples (MotionCompensator::CompensatePicture; the upconversion,
// Picture::UpData, libdirac_common/picture.cpp:141-199, made once per reference picture)
// with the clip (Picture::Clip) fused, for intra pictures the clip alone.  Output samples
// (set_frame_component, libdirac_decoder/dirac_parser.cpp:159-226: value + 2^(depth-1) as
// unsigned samples) are converted when read.
//
// Device memory: one arena, cut into picture slots (reconstructed planes, coefficients,
// upconverted planes) plus one staging area for a picture's host inputs (indices, code-block
// flags, motion data) and the transform scratch.  Work is ordered on one stream, so the
// staging area is reused picture after picture.

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

template <typename T>
__global__ void dec_output_kernel(const int16_t* __restrict__ rec, int n, int off, T* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = (T)((int)rec[i] + off);
}

struct DSlot {
    int16_t* data[3];
    int32_t* coeff[3];
    int16_t* up[3];
    int pnum = -1;  // -1: free
    bool up_valid = false;
    bool has_coeff = false;
};

struct Decoder {
    dgpu_decoder_params P{};
    cudaStream_t st = nullptr;
    int w[3]{}, h[3]{}, pw[3]{}, ph[3]{};
    int nb = 0, nblocks = 0, nsb = 0;
    std::vector<int> ncb;   // [3][nb][2]: (x, y) code blocks per band, per component
    int ncb_comp = 0;       // code blocks of one component's bands
    void* arena = nullptr;
    std::vector<DSlot> slots;
    std::map<int, int> pics;  // picture number -> slot
    // staging for host inputs
    int32_t* s_q[3]{};
    uint8_t* s_cb = nullptr;
    int16_t* s_mv = nullptr;  // [2][nblocks][2]
    uint8_t* s_mode = nullptr;
    int16_t* s_dc = nullptr;
    uint8_t* s_split = nullptr;
    void* dwt_ws = nullptr;
    size_t dwt_ws_bytes = 0;
    void* out_stage = nullptr;  // one output component for host reads
    size_t out_stage_bytes = 0;

    ~Decoder() {
        if (arena) cudaFree(arena);
    }
};

int comp_depth(const Decoder& D, int c) { return c == 0 ? D.P.luma_depth : D.P.chroma_depth; }

size_t sample_bytes(const Decoder& D) { return D.P.luma_depth > 8 || D.P.chroma_depth > 8 ? 2 : 1; }

int decoder_setup(const dgpu_decoder_params& P, int max_pictures, Decoder* D, size_t* total, size_t* slot_bytes,
                  int* nslots) {
    const dgpu_block_params& bp = P.bp;
    if (P.cformat < 0 || P.cformat > 2 || P.width < 16 || P.height < 16 || P.luma_depth < 8 || P.luma_depth > 14 ||
        P.chroma_depth < 8 || P.chroma_depth > 14 || P.wlt_depth < 1 || P.wlt_depth > 6 || max_pictures < 1 ||
        max_pictures > 4096 || bp.precision < 0 || bp.precision > 3 || bp.xbsep < 1 || bp.ybsep < 1 ||
        bp.xblen < bp.xbsep || bp.yblen < bp.ybsep || bp.xnum_sb < 1 || bp.ynum_sb < 1)
        return DGPU_ERR_ARG;
    D->P = P;
    const int xs = P.cformat == 0 ? 0 : 1, ys = P.cformat == 2 ? 1 : 0;
    D->w[0] = P.width;
    D->h[0] = P.height;
    D->w[1] = D->w[2] = P.width >> xs;
    D->h[1] = D->h[2] = P.height >> ys;
    const int mul = 1 << P.wlt_depth;
    for (int c = 0; c < 3; ++c) {
        D->pw[c] = (D->w[c] + mul - 1) / mul * mul;
        D->ph[c] = (D->h[c] + mul - 1) / mul * mul;
    }
    D->nb = 3 * P.wlt_depth + 1;
    D->nsb = bp.xnum_sb * bp.ynum_sb;
    D->nblocks = 16 * D->nsb;
    std::vector<int> one((size_t)2 * D->nb);
    int rc = dgpu_code_blocks(P.wlt_depth, P.width, P.height, P.spatial_partition ? 1 : 0, one.data());
    if (rc) return rc;
    D->ncb.clear();
    for (int c = 0; c < 3; ++c) D->ncb.insert(D->ncb.end(), one.begin(), one.end());
    D->ncb_comp = 0;
    for (int b = 0; b < D->nb; ++b) D->ncb_comp += one[2 * b] * one[2 * b + 1];
    *nslots = max_pictures;
    size_t plane16 = 0, plane32 = 0, up16 = 0;
    for (int c = 0; c < 3; ++c) {
        plane16 += align_up((size_t)D->w[c] * D->h[c] * 2, 256);
        plane32 += align_up((size_t)D->pw[c] * D->ph[c] * 4, 256);
        up16 += align_up((size_t)4 * D->w[c] * D->h[c] * 2, 256);
    }
    *slot_bytes = plane16 + plane32 + up16;
    D->dwt_ws_bytes = 0;
    for (int c = 0; c < 3; ++c)
        D->dwt_ws_bytes += align_up(dgpu_dwt_scratch_bytes(D->pw[c], D->ph[c], P.wlt_depth), 256);
    const size_t staging = plane32 + align_up((size_t)3 * D->ncb_comp, 256) +
                           align_up((size_t)D->nblocks * 2 * 2 * 2, 256) + align_up(D->nblocks, 256) +
                           align_up((size_t)D->nblocks * 3 * 2, 256) + align_up(D->nsb, 256);
    D->out_stage_bytes = align_up((size_t)D->w[0] * D->h[0] * 2, 256);
    *total = (size_t)*nslots * align_up(*slot_bytes, 256) + staging + align_up(D->dwt_ws_bytes, 256) +
             D->out_stage_bytes;
    return DGPU_OK;
}

int ensure_up(Decoder& D, DSlot& r) {
    if (r.up_valid) return DGPU_OK;
    const int16_t* pic[3] = {r.data[0], r.data[1], r.data[2]};
    int16_t* up[3] = {r.up[0], r.up[1], r.up[2]};
    int ups[3], bd[3];
    for (int c = 0; c < 3; ++c) {
        ups[c] = 2 * D.w[c];
        bd[c] = comp_depth(D, c);
    }
    const int rc = dgpu_upconvert_batch(3, pic, D.w, D.h, D.w, bd, up, ups, D.st);
    if (rc) return rc;
    r.up_valid = true;
    return DGPU_OK;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" size_t dgpu_decoder_device_bytes(const dgpu_decoder_params* params, int max_pictures) {
    if (!params) return 0;
    Decoder D;
    size_t total = 0, slot = 0;
    int n = 0;
    return decoder_setup(*params, max_pictures, &D, &total, &slot, &n) == DGPU_OK ? total : 0;
}

extern "C" int dgpu_decoder_create(const dgpu_decoder_params* params, int max_pictures, void* stream, void** out) {
    if (!params || !out) return DGPU_ERR_ARG;
    *out = nullptr;
    Decoder* D = new (std::nothrow) Decoder();
    if (!D) return DGPU_ERR_NOMEM;
    size_t total = 0, slot_bytes = 0;
    int nslots = 0;
    int rc = decoder_setup(*params, max_pictures, D, &total, &slot_bytes, &nslots);
    if (rc) {
        delete D;
        return rc;
    }
    D->st = as_stream(stream);
    if (cudaMalloc(&D->arena, total) != cudaSuccess) {
        cudaGetLastError();
        D->arena = nullptr;
        delete D;
        return DGPU_ERR_NOMEM;
    }
    char* q = static_cast<char*>(D->arena);
    auto take = [&](size_t bytes) {
        char* r = q;
        q += align_up(bytes, 256);
        return r;
    };
    D->slots.resize(nslots);
    for (int k = 0; k < nslots; ++k) {
        DSlot& s = D->slots[k];
        for (int c = 0; c < 3; ++c) s.data[c] = reinterpret_cast<int16_t*>(take((size_t)D->w[c] * D->h[c] * 2));
        for (int c = 0; c < 3; ++c) s.coeff[c] = reinterpret_cast<int32_t*>(take((size_t)D->pw[c] * D->ph[c] * 4));
        for (int c = 0; c < 3; ++c) s.up[c] = reinterpret_cast<int16_t*>(take((size_t)4 * D->w[c] * D->h[c] * 2));
        q = static_cast<char*>(D->arena) + (size_t)(k + 1) * align_up(slot_bytes, 256);
    }
    for (int c = 0; c < 3; ++c) D->s_q[c] = reinterpret_cast<int32_t*>(take((size_t)D->pw[c] * D->ph[c] * 4));
    D->s_cb = reinterpret_cast<uint8_t*>(take((size_t)3 * D->ncb_comp));
    D->s_mv = reinterpret_cast<int16_t*>(take((size_t)D->nblocks * 2 * 2 * 2));
    D->s_mode = reinterpret_cast<uint8_t*>(take(D->nblocks));
    D->s_dc = reinterpret_cast<int16_t*>(take((size_t)D->nblocks * 3 * 2));
    D->s_split = reinterpret_cast<uint8_t*>(take(D->nsb));
    D->dwt_ws = take(D->dwt_ws_bytes);
    D->out_stage = take(D->out_stage_bytes);
    *out = D;
    return DGPU_OK;
}

extern "C" int dgpu_decoder_destroy(void* dec) {
    Decoder* D = static_cast<Decoder*>(dec);
    if (!D) return DGPU_ERR_ARG;
    cudaStreamSynchronize(D->st);
    delete D;
    return DGPU_OK;
}

extern "C" int dgpu_decoder_release(void* dec, int pnum) {
    Decoder* D = static_cast<Decoder*>(dec);
    if (!D) return DGPU_ERR_ARG;
    auto it = D->pics.find(pnum);
    if (it == D->pics.end()) return DGPU_ERR_ARG;
    DSlot& s = D->slots[it->second];
    s.pnum = -1;
    s.up_valid = false;
    s.has_coeff = false;
    D->pics.erase(it);
    return DGPU_OK;
}

extern "C" int dgpu_decoder_decode(void* dec, const dgpu_decode_input* in) {
    Decoder* D = static_cast<Decoder*>(dec);
    if (!D || !in) return DGPU_ERR_ARG;
    const dgpu_decode_input& I = *in;
    if (D->pics.count(I.pnum)) return DGPU_ERR_ARG;
    const bool inter = !I.intra;
    if (inter) {
        if (I.num_refs < 1 || I.num_refs > 2 || !I.mv1 || !I.mode || !I.dc || !I.split ||
            (I.num_refs == 2 && !I.mv2))
            return DGPU_ERR_ARG;
        if (!D->pics.count(I.ref1) || (I.num_refs == 2 && !D->pics.count(I.ref2))) return DGPU_ERR_ARG;
    }
    // intra pictures always carry coefficients (picture_decompress.cpp:137-142)
    if (I.intra && I.zero_residual) return DGPU_ERR_ARG;
    if (I.index_bits != 0 && I.index_bits != 16 && I.index_bits != 32) return DGPU_ERR_ARG;
    const bool idx16 = I.index_bits == 16;
    if (!I.zero_residual && (!I.band_qidx || !I.band_skip || !I.cb_skip || !I.qindex[0] || !I.qindex[1] ||
                             !I.qindex[2]))
        return DGPU_ERR_ARG;
    int k = -1;
    for (int i = 0; i < (int)D->slots.size(); ++i)
        if (D->slots[i].pnum < 0) {
            k = i;
            break;
        }
    if (k < 0) return DGPU_ERR_SIZE;
    DSlot& s = D->slots[k];
    cudaStream_t st = D->st;
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    int rc;
    // 1. residue: dequantisation and inverse transform, or zero samples
    if (!I.zero_residual) {
        // int16 indices (index_bits 16) occupy the first half of the int32 staging area
        const size_t isz = idx16 ? 2 : 4;
        const void* q[3];
        const uint8_t* cb = I.cb_skip;
        if (I.on_host) {
            for (int c = 0; c < 3; ++c) {
                DGPU_CHECK_CUDA(cudaMemcpyAsync(D->s_q[c], I.qindex[c], (size_t)D->pw[c] * D->ph[c] * isz, h2d, st));
                q[c] = D->s_q[c];
            }
            DGPU_CHECK_CUDA(cudaMemcpyAsync(D->s_cb, I.cb_skip, (size_t)3 * D->ncb_comp, h2d, st));
            cb = D->s_cb;
        } else {
            for (int c = 0; c < 3; ++c) q[c] = I.qindex[c];
        }
        const int intra[3] = {I.intra ? 1 : 0, I.intra ? 1 : 0, I.intra ? 1 : 0};
        const int depth[3] = {D->P.wlt_depth, D->P.wlt_depth, D->P.wlt_depth};
        int32_t* coeff[3] = {s.coeff[0], s.coeff[1], s.coeff[2]};
        if (idx16) {
            const int16_t* q16[3] = {static_cast<const int16_t*>(q[0]), static_cast<const int16_t*>(q[1]),
                                     static_cast<const int16_t*>(q[2])};
            rc = dgpu_dequantise_batch16(3, intra, depth, q16, coeff, D->pw, D->ph, D->ncb.data(), I.band_qidx,
                                         I.band_skip, cb, st);
        } else {
            const int32_t* q32[3] = {static_cast<const int32_t*>(q[0]), static_cast<const int32_t*>(q[1]),
                                     static_cast<const int32_t*>(q[2])};
            rc = dgpu_dequantise_batch(3, intra, depth, q32, coeff, D->pw, D->ph, D->ncb.data(), I.band_qidx,
                                       I.band_skip, cb, st);
        }
        if (rc) return rc;
        const int filt[3] = {I.filter, I.filter, I.filter};
        int16_t* pic[3] = {s.data[0], s.data[1], s.data[2]};
        rc = dgpu_wavelet_transform_batch(DGPU_BACKWARD, 3, filt, depth, pic, D->w, D->h, D->w, coeff, D->pw, D->ph,
                                          D->pw, D->dwt_ws, D->dwt_ws_bytes, st);
        if (rc) return rc;
        s.has_coeff = true;
    } else {
        for (int c = 0; c < 3; ++c)
            DGPU_CHECK_CUDA(cudaMemsetAsync(s.data[c], 0, (size_t)D->w[c] * D->h[c] * 2, st));
        s.has_coeff = false;
    }
    // 2. prediction and clip
    if (inter) {
        DSlot& r1 = D->slots[D->pics[I.ref1]];
        rc = ensure_up(*D, r1);
        if (rc) return rc;
        const int16_t* up1[3] = {r1.up[0], r1.up[1], r1.up[2]};
        const int16_t* up2[3] = {nullptr, nullptr, nullptr};
        const bool two = I.num_refs == 2;
        if (two) {
            DSlot& r2 = D->slots[D->pics[I.ref2]];
            rc = ensure_up(*D, r2);
            if (rc) return rc;
            for (int c = 0; c < 3; ++c) up2[c] = r2.up[c];
        }
        const int16_t* mv1 = I.mv1;
        const int16_t* mv2 = two ? I.mv2 : nullptr;
        const uint8_t* mode = I.mode;
        const int16_t* dcv = I.dc;
        const uint8_t* split = I.split;
        if (I.on_host) {
            const size_t mvb = (size_t)D->nblocks * 2 * 2;
            DGPU_CHECK_CUDA(cudaMemcpyAsync(D->s_mv, I.mv1, mvb, h2d, st));
            if (two) DGPU_CHECK_CUDA(cudaMemcpyAsync(D->s_mv + 2 * D->nblocks, I.mv2, mvb, h2d, st));
            DGPU_CHECK_CUDA(cudaMemcpyAsync(D->s_mode, I.mode, D->nblocks, h2d, st));
            DGPU_CHECK_CUDA(cudaMemcpyAsync(D->s_dc, I.dc, (size_t)D->nblocks * 3 * 2, h2d, st));
            DGPU_CHECK_CUDA(cudaMemcpyAsync(D->s_split, I.split, D->nsb, h2d, st));
            mv1 = D->s_mv;
            mv2 = two ? D->s_mv + 2 * D->nblocks : nullptr;
            mode = D->s_mode;
            dcv = D->s_dc;
            split = D->s_split;
        }
        int16_t* pic[3] = {s.data[0], s.data[1], s.data[2]};
        rc = dgpu_motion_compensate(DGPU_ADD, D->P.cformat, D->w[0], D->h[0], &D->P.bp, mv1, mv2, mode, dcv, split,
                                    pic, D->w, up1, two ? up2 : nullptr, D->P.luma_depth, D->P.chroma_depth, st);
        if (rc) return rc;
    } else {
        for (int c = 0; c < 3; ++c) {
            rc = dgpu_clip(s.data[c], D->w[c], D->h[c], D->w[c], comp_depth(*D, c), st);
            if (rc) return rc;
        }
    }
    s.pnum = I.pnum;
    s.up_valid = false;
    D->pics[I.pnum] = k;
    return DGPU_OK;
}

extern "C" size_t dgpu_decoder_item_bytes(void* dec, int pnum, int what, int comp) {
    Decoder* D = static_cast<Decoder*>(dec);
    if (!D || comp < 0 || comp > 2) return 0;
    auto it = D->pics.find(pnum);
    if (it == D->pics.end()) return 0;
    switch (what) {
        case DGPU_ENC_RECON: return (size_t)D->w[comp] * D->h[comp] * 2;
        case DGPU_ENC_COEFF: return D->slots[it->second].has_coeff ? (size_t)D->pw[comp] * D->ph[comp] * 4 : 0;
        case DGPU_ENC_OUTPUT: return (size_t)D->w[comp] * D->h[comp] * sample_bytes(*D);
        default: return 0;
    }
}

extern "C" int dgpu_decoder_read(void* dec, int pnum, int what, int comp, void* dst, size_t bytes, int on_host) {
    Decoder* D = static_cast<Decoder*>(dec);
    if (!D || !dst) return DGPU_ERR_ARG;
    const size_t need = dgpu_decoder_item_bytes(dec, pnum, what, comp);
    if (need == 0 || bytes != need) return DGPU_ERR_ARG;
    const DSlot& s = D->slots[D->pics[pnum]];
    const void* src = nullptr;
    if (what == DGPU_ENC_OUTPUT) {
        const int n = D->w[comp] * D->h[comp];
        const int off = 1 << (comp_depth(*D, comp) - 1);
        void* out = on_host ? D->out_stage : dst;
        const int grid = std::min((n + 255) / 256, 148 * 8);
        if (sample_bytes(*D) == 1)
            dec_output_kernel<uint8_t><<<grid, 256, 0, D->st>>>(s.data[comp], n, off, static_cast<uint8_t*>(out));
        else
            dec_output_kernel<uint16_t><<<grid, 256, 0, D->st>>>(s.data[comp], n, off, static_cast<uint16_t*>(out));
        DGPU_CHECK_LAUNCH();
        if (!on_host) return DGPU_OK;
        src = D->out_stage;
    } else {
        src = what == DGPU_ENC_RECON ? (const void*)s.data[comp] : (const void*)s.coeff[comp];
    }
    DGPU_CHECK_CUDA(
        cudaMemcpyAsync(dst, src, bytes, on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, D->st));
    if (on_host) DGPU_CHECK_CUDA(host_wait(D->st));
    return DGPU_OK;
}
