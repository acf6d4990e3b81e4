// Heterogeneous picture batch: the coding hot path of many pictures of different sizes,
// chroma formats, bit depths, transform filters and depths in shared launches.
//
// Per picture the steps are those PictureCompressor applies to one picture once its motion
// data is known (libdirac_encoder/picture_compress.cpp:92-180 Compress, 418-531 CodeResidue):
// motion compensation SUBTRACT against the upconverted references (inter pictures), the
// forward transform, quantiser choice with quantisation and reconstruction, the inverse
// transform, then motion compensation ADD with the clip (inter) or the clip alone (intra).
// Each picture's results equal its own coding by the single-picture entry points.
//
// Device side: the reference upconversions and both motion compensations of every picture,
// and each transform level of every component, are enqueued once and captured in two CUDA
// graphs (before and after the quantiser choice) on the first run; later runs replay them.
// Between the two graphs the residue coder handles every component of the batch in one call:
// statistics on the device, the reference's double-precision Lagrangian on the host, then
// quantisation on the device.  Motion-compensation tiles are chosen per picture size and
// block parameters by a small autotuner on the first run (timed with CUDA events before the
// capture); the choice changes only the launch shape, never a result.

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "coding_params.h"
#include "dgpu_internal.cuh"

namespace dgpu {

int mc_tile_variants();
int motion_compensate_tiled(int variant, int add_or_sub, int cformat, int w, int h, const dgpu_block_params* bp,
                            const int16_t* mv1, const int16_t* mv2, const uint8_t* mode, const int16_t* dc,
                            const uint8_t* split, int16_t* const* pic, const int* pic_stride,
                            const int16_t* const* ref1up, const int16_t* const* ref2up, int clip_luma_depth,
                            int clip_chroma_depth, cudaStream_t st);

namespace {

struct BPic {
    dgpu_batch_picture P{};
    dgpu_batch_motion M{};
    int w[3]{}, h[3]{}, pw[3]{}, ph[3]{};
    int nb = 0, ncb_total = 0, nref = 0;
    std::vector<int> ncb;          // [nb][2], identical for the three components
    int16_t* data[3]{};
    int32_t* coeff[3]{};
    int32_t* qout[3]{};
    int16_t* up[2][3]{};           // upconverted references
    int mc_variant = 0;
    std::vector<int> bands;        // [3][nb][3]: quantiser index, skip, estimated bits
    std::vector<uint8_t> cb_skip;  // [3][ncb_total]
};

struct UpSrc {
    const int16_t* src;
    int16_t* dst;
    int w, h, depth;
};

struct Batch {
    std::vector<BPic> pics;
    cudaStream_t user = nullptr;     // the caller's stream (loads, reads, ordering)
    cudaStream_t st = nullptr;       // the batch's own stream (captured; the legacy stream cannot be)
    cudaEvent_t ev = nullptr;
    void* arena = nullptr;
    void* dwt_ws = nullptr;
    size_t dwt_ws_bytes = 0;
    void* q_ws = nullptr;
    size_t q_ws_bytes = 0;
    std::vector<UpSrc> ups;
    cudaGraphExec_t pre = nullptr, post = nullptr;
    unsigned long long pre_kernels = 0, post_kernels = 0;  // kernels each graph replays
    bool tuned = false;
    // every component of the batch, for the batched transform and residue calls
    std::vector<int> c_filter, c_depth, c_intra, c_w, c_h, c_pw, c_ph, c_ncb;
    std::vector<int16_t*> c_pic;
    std::vector<int32_t*> c_coeff, c_qout;
    std::vector<float> c_lam, c_wt, c_ecf;
    std::vector<int> r_qidx, r_skip, r_bits;
    std::vector<uint8_t> r_cbskip;

    ~Batch() {
        if (st) cudaStreamSynchronize(st);
        if (user) cudaStreamSynchronize(user);
        if (pre) cudaGraphExecDestroy(pre);
        if (post) cudaGraphExecDestroy(post);
        if (arena) cudaFree(arena);
        if (ev) cudaEventDestroy(ev);
        if (st) cudaStreamDestroy(st);
    }
};

int check_picture(const dgpu_batch_picture& P, const dgpu_batch_motion* M) {
    if (P.cformat < 0 || P.cformat > 2 || P.width < 16 || P.height < 16 || P.luma_depth < 8 || P.luma_depth > 14 ||
        P.chroma_depth < 8 || P.chroma_depth > 14 || P.filter < 0 || P.filter > 6 || P.wlt_depth < 1 ||
        P.wlt_depth > 6)
        return DGPU_ERR_ARG;
    if (!P.intra) {
        const dgpu_block_params& b = P.bp;
        if (!M || !M->ref1[0] || !M->ref1[1] || !M->ref1[2] || !M->mv1 || !M->mode || !M->dc || !M->split)
            return DGPU_ERR_ARG;
        if (M->ref2[0] && (!M->ref2[1] || !M->ref2[2] || !M->mv2)) return DGPU_ERR_ARG;
        if (b.precision < 0 || b.precision > 3 || b.xbsep <= 0 || b.ybsep <= 0 || b.xnum_sb <= 0 || b.ynum_sb <= 0)
            return DGPU_ERR_ARG;
    }
    return DGPU_OK;
}

// Geometry, per-band parameters and device sizes of the batch; with base set, also carves the
// arena.  Returns the arena bytes in *total.
int layout(Batch& B, int n, const dgpu_batch_picture* pics, const dgpu_batch_motion* motion, char* base,
           size_t* total) {
    size_t off = 0;
    auto take = [&](size_t bytes) -> char* {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes, 256);
        return p;
    };
    B.pics.assign(n, BPic());
    std::map<const int16_t*, int16_t*> up_of;  // distinct reference planes
    B.ups.clear();
    for (int k = 0; k < n; ++k) {
        BPic& Q = B.pics[k];
        Q.P = pics[k];
        const dgpu_batch_motion* M = motion ? &motion[k] : nullptr;
        int rc = check_picture(Q.P, M);
        if (rc) return rc;
        if (M) Q.M = *M;
        const int xs = Q.P.cformat == 0 ? 0 : 1, ys = Q.P.cformat == 2 ? 1 : 0;
        Q.w[0] = Q.P.width;
        Q.h[0] = Q.P.height;
        Q.w[1] = Q.w[2] = Q.P.width >> xs;
        Q.h[1] = Q.h[2] = Q.P.height >> ys;
        const int mul = 1 << Q.P.wlt_depth;
        for (int c = 0; c < 3; ++c) {
            Q.pw[c] = (Q.w[c] + mul - 1) / mul * mul;
            Q.ph[c] = (Q.h[c] + mul - 1) / mul * mul;
            Q.data[c] = reinterpret_cast<int16_t*>(take((size_t)Q.w[c] * Q.h[c] * 2));
            Q.coeff[c] = reinterpret_cast<int32_t*>(take((size_t)Q.pw[c] * Q.ph[c] * 4));
            Q.qout[c] = reinterpret_cast<int32_t*>(take((size_t)Q.pw[c] * Q.ph[c] * 4));
        }
        Q.nb = 3 * Q.P.wlt_depth + 1;
        Q.ncb.assign((size_t)2 * Q.nb, 0);
        rc = dgpu_code_blocks(Q.P.wlt_depth, Q.P.width, Q.P.height, 1, Q.ncb.data());
        if (rc) return rc;
        Q.ncb_total = 0;
        for (int b = 0; b < Q.nb; ++b) Q.ncb_total += Q.ncb[2 * b] * Q.ncb[2 * b + 1];
        if (!Q.P.intra) {
            Q.nref = Q.M.ref2[0] ? 2 : 1;
            for (int r = 0; r < Q.nref; ++r)
                for (int c = 0; c < 3; ++c) {
                    const int16_t* src = r ? Q.M.ref2[c] : Q.M.ref1[c];
                    auto it = up_of.find(src);
                    if (it == up_of.end()) {
                        int16_t* dst = reinterpret_cast<int16_t*>(take((size_t)4 * Q.w[c] * Q.h[c] * 2));
                        it = up_of.emplace(src, dst).first;
                        B.ups.push_back({src, dst, Q.w[c], Q.h[c], c ? Q.P.chroma_depth : Q.P.luma_depth});
                    }
                    Q.up[r][c] = it->second;
                }
        }
    }
    // batched transform and residue tables over every component
    B.c_filter.clear();
    B.c_depth.clear();
    B.c_intra.clear();
    B.c_w.clear();
    B.c_h.clear();
    B.c_pw.clear();
    B.c_ph.clear();
    B.c_ncb.clear();
    B.c_pic.clear();
    B.c_coeff.clear();
    B.c_qout.clear();
    B.c_lam.clear();
    B.c_wt.clear();
    B.c_ecf.clear();
    size_t dwt = 0;
    std::vector<double> wd;
    for (BPic& Q : B.pics) {
        const Lambdas L = calc_lambdas(Q.P.qf);
        const double cpd_scale = perceptual_scale(Q.P.intra != 0, Q.P.intra_ratio);
        wd.assign(Q.nb, 0.0);
        std::vector<float> ecf(Q.nb);
        initial_ecf(Q.P.wlt_depth, Q.P.intra != 0, ecf.data());
        for (int c = 0; c < 3; ++c) {
            B.c_filter.push_back(Q.P.filter);
            B.c_depth.push_back(Q.P.wlt_depth);
            B.c_intra.push_back(Q.P.intra ? 1 : 0);
            B.c_w.push_back(Q.w[c]);
            B.c_h.push_back(Q.h[c]);
            B.c_pw.push_back(Q.pw[c]);
            B.c_ph.push_back(Q.ph[c]);
            B.c_pic.push_back(Q.data[c]);
            B.c_coeff.push_back(Q.coeff[c]);
            B.c_qout.push_back(Q.qout[c]);
            B.c_ncb.insert(B.c_ncb.end(), Q.ncb.begin(), Q.ncb.end());
            B.c_lam.push_back(component_lambda(L, Q.P.intra != 0, Q.P.is_b != 0, Q.P.intra_ratio, c));
            const int rc = dgpu_band_weights(Q.P.filter, Q.P.wlt_depth, Q.pw[c], Q.ph[c], c, Q.P.cformat, Q.P.cpd,
                                             (float)cpd_scale, 0, wd.data());
            if (rc) return rc;
            for (int b = 0; b < Q.nb; ++b) B.c_wt.push_back((float)wd[b]);
            B.c_ecf.insert(B.c_ecf.end(), ecf.begin(), ecf.end());
            dwt += align_up(dgpu_dwt_scratch_bytes(Q.pw[c], Q.ph[c], Q.P.wlt_depth), 256);
        }
    }
    const int nc = (int)B.c_pic.size();
    B.dwt_ws_bytes = dwt;
    B.dwt_ws = take(dwt);
    B.q_ws_bytes = dgpu_code_residue_workspace_bytes(nc, B.c_intra.data(), B.c_depth.data(), B.c_pw.data(),
                                                     B.c_ph.data(), B.c_ncb.data());
    if (B.q_ws_bytes == 0) return DGPU_ERR_SIZE;
    B.q_ws = take(B.q_ws_bytes);
    *total = off;
    return DGPU_OK;
}

// Every distinct reference plane upconverted once (Picture::UpData).
int upconvert_refs(Batch& B) {
    const int n = (int)B.ups.size();
    if (n == 0) return DGPU_OK;
    std::vector<const int16_t*> src(n);
    std::vector<int16_t*> dst(n);
    std::vector<int> w(n), h(n), d(n), us(n);
    for (int i = 0; i < n; ++i) {
        src[i] = B.ups[i].src;
        dst[i] = B.ups[i].dst;
        w[i] = B.ups[i].w;
        h[i] = B.ups[i].h;
        d[i] = B.ups[i].depth;
        us[i] = 2 * w[i];
    }
    return dgpu_upconvert_batch(n, src.data(), w.data(), h.data(), w.data(), d.data(), dst.data(), us.data(), B.st);
}

// Upconversions, motion compensation SUBTRACT and the forward transform of every picture.
int enqueue_pre(Batch& B) {
    cudaStream_t st = B.st;
    int rc = upconvert_refs(B);
    if (rc) return rc;
    for (BPic& Q : B.pics) {
        if (Q.P.intra) continue;
        const int16_t* up1[3] = {Q.up[0][0], Q.up[0][1], Q.up[0][2]};
        const int16_t* up2[3] = {Q.up[1][0], Q.up[1][1], Q.up[1][2]};
        rc = motion_compensate_tiled(Q.mc_variant, DGPU_SUBTRACT, Q.P.cformat, Q.w[0], Q.h[0], &Q.P.bp, Q.M.mv1,
                                         Q.nref > 1 ? Q.M.mv2 : nullptr, Q.M.mode, Q.M.dc, Q.M.split, Q.data, Q.w,
                                         up1, Q.nref > 1 ? up2 : nullptr, 0, 0, st);
        if (rc) return rc;
    }
    return dgpu_wavelet_transform_batch(DGPU_FORWARD, (int)B.c_pic.size(), B.c_filter.data(), B.c_depth.data(),
                                        B.c_pic.data(), B.c_w.data(), B.c_h.data(), B.c_w.data(), B.c_coeff.data(),
                                        B.c_pw.data(), B.c_ph.data(), B.c_pw.data(), B.dwt_ws, B.dwt_ws_bytes, st);
}

// The inverse transform, then motion compensation ADD with the clip (inter) or the clip.
int enqueue_post(Batch& B) {
    cudaStream_t st = B.st;
    int rc = dgpu_wavelet_transform_batch(DGPU_BACKWARD, (int)B.c_pic.size(), B.c_filter.data(), B.c_depth.data(),
                                          B.c_pic.data(), B.c_w.data(), B.c_h.data(), B.c_w.data(),
                                          B.c_coeff.data(), B.c_pw.data(), B.c_ph.data(), B.c_pw.data(), B.dwt_ws,
                                          B.dwt_ws_bytes, st);
    if (rc) return rc;
    for (BPic& Q : B.pics) {
        if (Q.P.intra) {
            for (int c = 0; c < 3; ++c) {
                rc = dgpu_clip(Q.data[c], Q.w[c], Q.h[c], Q.w[c], c ? Q.P.chroma_depth : Q.P.luma_depth, st);
                if (rc) return rc;
            }
            continue;
        }
        const int16_t* up1[3] = {Q.up[0][0], Q.up[0][1], Q.up[0][2]};
        const int16_t* up2[3] = {Q.up[1][0], Q.up[1][1], Q.up[1][2]};
        rc = motion_compensate_tiled(Q.mc_variant, DGPU_ADD, Q.P.cformat, Q.w[0], Q.h[0], &Q.P.bp, Q.M.mv1,
                                     Q.nref > 1 ? Q.M.mv2 : nullptr, Q.M.mode, Q.M.dc, Q.M.split, Q.data, Q.w, up1,
                                     Q.nref > 1 ? up2 : nullptr, Q.P.luma_depth, Q.P.chroma_depth, st);
        if (rc) return rc;
    }
    return DGPU_OK;
}

int capture(Batch& B, int (*enqueue)(Batch&), cudaGraphExec_t* out, unsigned long long* kernels) {
    DGPU_CHECK_CUDA(cudaStreamBeginCapture(B.st, cudaStreamCaptureModeThreadLocal));
    const unsigned long long before = dgpu_launch_count();
    const int rc = enqueue(B);
    *kernels = dgpu_launch_count() - before;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(B.st, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc;
    }
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        return DGPU_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        set_last_cuda_error(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
        return DGPU_ERR_CUDA;
    }
    return DGPU_OK;
}

// Autotuner of the motion-compensation tile shape, keyed on (component size, chroma format,
// block parameters): each variant runs twice on the picture's own buffers (the second run
// timed) and the fastest is kept for the process.  Runs before the graphs are captured; the
// tuning runs only touch the picture's working planes, which the first run overwrites.
struct TuneKey {
    int cformat, w, h, prec, xblen, yblen, xbsep, ybsep, nref;
    bool operator<(const TuneKey& o) const {
        return std::tie(cformat, w, h, prec, xblen, yblen, xbsep, ybsep, nref) <
               std::tie(o.cformat, o.w, o.h, o.prec, o.xblen, o.yblen, o.xbsep, o.ybsep, o.nref);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tuned;

int autotune(Batch& B) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DGPU_CHECK_CUDA(cudaEventCreate(&e0));
    DGPU_CHECK_CUDA(cudaEventCreate(&e1));
    // the references' upconverted planes must exist for the trial runs
    int rc = upconvert_refs(B);
    for (BPic& Q : B.pics) {
        if (rc || Q.P.intra) continue;
        const TuneKey key{Q.P.cformat, Q.w[0], Q.h[0], Q.P.bp.precision, Q.P.bp.xblen, Q.P.bp.yblen,
                          Q.P.bp.xbsep, Q.P.bp.ybsep, Q.nref};
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tuned.find(key);
            if (it != g_tuned.end()) {
                Q.mc_variant = it->second;
                continue;
            }
        }
        const int16_t* up1[3] = {Q.up[0][0], Q.up[0][1], Q.up[0][2]};
        const int16_t* up2[3] = {Q.up[1][0], Q.up[1][1], Q.up[1][2]};
        float best_ms = 1e30f;
        int best = 0;
        for (int v = 0; v < mc_tile_variants() && !rc; ++v) {
            // SUBTRACT then ADD without the clip leaves the planes exactly as they were (int16
            // wrap-around arithmetic), so the caller's input survives the trials
            float ms = 0.f;
            for (int rep = 0; rep < 2 && !rc; ++rep) {
                if (rep == 1 && cudaEventRecord(e0, B.st) != cudaSuccess) rc = DGPU_ERR_CUDA;
                if (!rc)
                    rc = motion_compensate_tiled(v, DGPU_SUBTRACT, Q.P.cformat, Q.w[0], Q.h[0], &Q.P.bp, Q.M.mv1,
                                                 Q.nref > 1 ? Q.M.mv2 : nullptr, Q.M.mode, Q.M.dc, Q.M.split, Q.data,
                                                 Q.w, up1, Q.nref > 1 ? up2 : nullptr, 0, 0, B.st);
                if (!rc && rep == 1 && cudaEventRecord(e1, B.st) != cudaSuccess) rc = DGPU_ERR_CUDA;
                if (!rc)
                    rc = motion_compensate_tiled(v, DGPU_ADD, Q.P.cformat, Q.w[0], Q.h[0], &Q.P.bp, Q.M.mv1,
                                                 Q.nref > 1 ? Q.M.mv2 : nullptr, Q.M.mode, Q.M.dc, Q.M.split, Q.data,
                                                 Q.w, up1, Q.nref > 1 ? up2 : nullptr, 0, 0, B.st);
            }
            if (rc) break;
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = DGPU_ERR_CUDA;
                break;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = v;
            }
        }
        if (rc) break;
        Q.mc_variant = best;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGetLastError();
    return rc;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" size_t dgpu_batch_device_bytes(int n, const dgpu_batch_picture* pics, const dgpu_batch_motion* motion) {
    if (n <= 0 || !pics) return 0;
    Batch B;
    size_t total = 0;
    return layout(B, n, pics, motion, nullptr, &total) == DGPU_OK ? total : 0;
}

extern "C" int dgpu_batch_create(int n, const dgpu_batch_picture* pics, const dgpu_batch_motion* motion,
                                 void* stream, void** out) {
    if (n <= 0 || !pics || !out) return DGPU_ERR_ARG;
    *out = nullptr;
    Batch* B = new (std::nothrow) Batch();
    if (!B) return DGPU_ERR_NOMEM;
    size_t total = 0;
    int rc = layout(*B, n, pics, motion, nullptr, &total);
    if (rc) {
        delete B;
        return rc;
    }
    if (cudaMalloc(&B->arena, total) != cudaSuccess) {
        cudaGetLastError();
        B->arena = nullptr;
        delete B;
        return DGPU_ERR_NOMEM;
    }
    rc = layout(*B, n, pics, motion, static_cast<char*>(B->arena), &total);
    if (rc) {
        delete B;
        return rc;
    }
    B->user = as_stream(stream);
    if (cudaStreamCreateWithFlags(&B->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&B->ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        delete B;
        return DGPU_ERR_CUDA;
    }
    int nbt = 0, ncbt = 0;
    for (const BPic& Q : B->pics) {
        nbt += 3 * Q.nb;
        ncbt += 3 * Q.ncb_total;
    }
    B->r_qidx.assign(nbt, 0);
    B->r_skip.assign(nbt, 0);
    B->r_bits.assign(nbt, 0);
    B->r_cbskip.assign(ncbt, 0);
    *out = B;
    return DGPU_OK;
}

extern "C" int dgpu_batch_destroy(void* batch) {
    Batch* B = static_cast<Batch*>(batch);
    if (!B) return DGPU_ERR_ARG;
    delete B;
    return DGPU_OK;
}

extern "C" int dgpu_batch_planes(void* batch, int k, int16_t** planes) {
    Batch* B = static_cast<Batch*>(batch);
    if (!B || !planes || k < 0 || k >= (int)B->pics.size()) return DGPU_ERR_ARG;
    for (int c = 0; c < 3; ++c) planes[c] = B->pics[k].data[c];
    return DGPU_OK;
}

extern "C" int dgpu_batch_load(void* batch, int k, const int16_t* const* planes, int on_host) {
    Batch* B = static_cast<Batch*>(batch);
    if (!B || !planes || k < 0 || k >= (int)B->pics.size()) return DGPU_ERR_ARG;
    const BPic& Q = B->pics[k];
    for (int c = 0; c < 3; ++c) {
        if (!planes[c]) return DGPU_ERR_ARG;
        DGPU_CHECK_CUDA(cudaMemcpyAsync(Q.data[c], planes[c], (size_t)Q.w[c] * Q.h[c] * 2,
                                        on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, B->user));
    }
    return DGPU_OK;
}

extern "C" int dgpu_batch_run(void* batch) {
    Batch* B = static_cast<Batch*>(batch);
    if (!B) return DGPU_ERR_ARG;
    int rc;
    // the batch's stream follows the caller's (its loads), and the caller's follows the run
    DGPU_CHECK_CUDA(cudaEventRecord(B->ev, B->user));
    DGPU_CHECK_CUDA(cudaStreamWaitEvent(B->st, B->ev, 0));
    if (!B->tuned) {
        rc = autotune(*B);
        if (rc) return rc;
        B->tuned = true;
    }
    if (!B->pre) {
        rc = capture(*B, enqueue_pre, &B->pre, &B->pre_kernels);
        if (rc) return rc;
    }
    if (!B->post) {
        rc = capture(*B, enqueue_post, &B->post, &B->post_kernels);
        if (rc) return rc;
    }
    DGPU_CHECK_CUDA(cudaGraphLaunch(B->pre, B->st));
    count_launches(B->pre_kernels);
    rc = dgpu_code_residue_batch((int)B->c_pic.size(), B->c_intra.data(), B->c_depth.data(), B->c_coeff.data(),
                                 B->c_pw.data(), B->c_ph.data(), B->c_lam.data(), B->c_wt.data(), B->c_ecf.data(),
                                 B->c_ncb.data(), B->r_qidx.data(), B->r_skip.data(), B->r_bits.data(),
                                 B->r_cbskip.data(), B->c_qout.data(), B->q_ws, B->q_ws_bytes, B->st);
    if (rc) return rc;
    DGPU_CHECK_CUDA(cudaGraphLaunch(B->post, B->st));
    count_launches(B->post_kernels);
    DGPU_CHECK_CUDA(cudaEventRecord(B->ev, B->st));
    DGPU_CHECK_CUDA(cudaStreamWaitEvent(B->user, B->ev, 0));
    // per-picture results (band choices and code-block skips) in the encoder's layout
    int bo = 0, co = 0;
    for (BPic& Q : B->pics) {
        Q.bands.resize((size_t)9 * Q.nb);
        for (int k = 0; k < 3 * Q.nb; ++k) {
            Q.bands[3 * k] = B->r_qidx[bo + k];
            Q.bands[3 * k + 1] = B->r_skip[bo + k];
            Q.bands[3 * k + 2] = B->r_bits[bo + k];
        }
        Q.cb_skip.assign(B->r_cbskip.begin() + co, B->r_cbskip.begin() + co + 3 * Q.ncb_total);
        bo += 3 * Q.nb;
        co += 3 * Q.ncb_total;
    }
    return DGPU_OK;
}

extern "C" int dgpu_batch_stage_times(void* batch, float* ms) {
    Batch* B = static_cast<Batch*>(batch);
    if (!B || !ms) return DGPU_ERR_ARG;
    if (!B->pre || !B->post) {
        const int rc = dgpu_batch_run(batch);  // tunes and captures
        if (rc) return rc;
    }
    cudaEvent_t e[4] = {};
    for (auto& x : e) DGPU_CHECK_CUDA(cudaEventCreate(&x));
    int rc = DGPU_OK;
    if (cudaEventRecord(B->ev, B->user) != cudaSuccess || cudaStreamWaitEvent(B->st, B->ev, 0) != cudaSuccess ||
        cudaEventRecord(e[0], B->st) != cudaSuccess || cudaGraphLaunch(B->pre, B->st) != cudaSuccess ||
        cudaEventRecord(e[1], B->st) != cudaSuccess)
        rc = DGPU_ERR_CUDA;
    if (!rc)
        rc = dgpu_code_residue_batch((int)B->c_pic.size(), B->c_intra.data(), B->c_depth.data(), B->c_coeff.data(),
                                     B->c_pw.data(), B->c_ph.data(), B->c_lam.data(), B->c_wt.data(),
                                     B->c_ecf.data(), B->c_ncb.data(), B->r_qidx.data(), B->r_skip.data(),
                                     B->r_bits.data(), B->r_cbskip.data(), B->c_qout.data(), B->q_ws, B->q_ws_bytes,
                                     B->st);
    if (!rc && (cudaEventRecord(e[2], B->st) != cudaSuccess || cudaGraphLaunch(B->post, B->st) != cudaSuccess ||
                cudaEventRecord(e[3], B->st) != cudaSuccess || cudaEventSynchronize(e[3]) != cudaSuccess))
        rc = DGPU_ERR_CUDA;
    for (int k = 0; k < 3 && !rc; ++k)
        if (cudaEventElapsedTime(&ms[k], e[k], e[k + 1]) != cudaSuccess) rc = DGPU_ERR_CUDA;
    for (auto& x : e) cudaEventDestroy(x);
    cudaGetLastError();
    return rc;
}

extern "C" size_t dgpu_batch_item_bytes(void* batch, int k, int what, int comp) {
    Batch* B = static_cast<Batch*>(batch);
    if (!B || k < 0 || k >= (int)B->pics.size() || comp < 0 || comp > 2) return 0;
    const BPic& Q = B->pics[k];
    switch (what) {
        case DGPU_ENC_RECON: return (size_t)Q.w[comp] * Q.h[comp] * 2;
        case DGPU_ENC_COEFF:
        case DGPU_ENC_QINDEX: return (size_t)Q.pw[comp] * Q.ph[comp] * 4;
        case DGPU_ENC_BANDS: return Q.bands.empty() ? 0 : (size_t)Q.nb * 3 * sizeof(int);
        case DGPU_ENC_CBSKIP: return Q.cb_skip.empty() ? 0 : (size_t)Q.ncb_total;
        default: return 0;
    }
}

extern "C" int dgpu_batch_read(void* batch, int k, int what, int comp, void* dst, size_t bytes, int on_host) {
    Batch* B = static_cast<Batch*>(batch);
    if (!B || !dst) return DGPU_ERR_ARG;
    const size_t need = dgpu_batch_item_bytes(batch, k, what, comp);
    if (need == 0 || bytes != need) return DGPU_ERR_ARG;
    const BPic& Q = B->pics[k];
    if (what == DGPU_ENC_BANDS || what == DGPU_ENC_CBSKIP) {
        const void* src = what == DGPU_ENC_BANDS ? (const void*)&Q.bands[(size_t)comp * Q.nb * 3]
                                                 : (const void*)&Q.cb_skip[(size_t)comp * Q.ncb_total];
        if (on_host) {
            std::memcpy(dst, src, bytes);
            return DGPU_OK;
        }
        DGPU_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, B->user));
        DGPU_CHECK_CUDA(host_wait(B->user));
        return DGPU_OK;
    }
    const void* src = what == DGPU_ENC_RECON ? (const void*)Q.data[comp]
                      : what == DGPU_ENC_COEFF ? (const void*)Q.coeff[comp] : (const void*)Q.qout[comp];
    DGPU_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                    B->user));
    if (on_host) DGPU_CHECK_CUDA(host_wait(B->user));
    return DGPU_OK;
}
