// Sequence encoder: the reference's frame-coding loop over the library's kernels, with all
// picture data resident on the device.
//
// Host side: the GOP state machine of FrameSequenceCompressor / SequenceCompressor
// (libdirac_encoder/seq_compress.cpp:151-192 CanEncode, 194-499 CompressNextPicture,
// 563-632 SetPicTypeAndRefs, 664-686 CodedToDisplay), the lambdas of
// EncoderParams::CalcLambdas (libdirac_common/common.cpp:451-476) and
// PictureCompressor::GetCompLambda (libdirac_encoder/picture_compress.cpp:532-580), the
// perceptual-weight scale and intra-block ratio of PictureCompressor::CodeResidue /
// IntraModeAnalyse (picture_compress.cpp:300-320, 418-428).
//
// Device side, per picture: motion estimation (batched over every picture whose references
// are known, ahead of coding order: estimation reads only original pictures), motion
// compensation (SUBTRACT) against the upconverted reconstructed references, the forward
// transform of the three components in one batch, quantiser choice and quantisation, the
// inverse transform, motion compensation (ADD) with the clip fused, and the upconversion of
// reference pictures when a later picture first needs them (Picture::UpData,
// libdirac_common/picture.cpp:141-199).
//
// Device memory: one arena per encoder, cut into max_pictures picture slots (original,
// working / reconstructed planes, coefficients, quantised indices, upconverted planes, motion
// data) plus the workspaces of motion estimation, transform and quantisation, all sized at
// creation.  A 1080p 4:2:0 slot is about 64 MB.

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <future>
#include <new>
#include <vector>

#include "coding_params.h"
#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int kIntraMode = 0;  // PredMode INTRA (libdirac_common/common.h:84)
constexpr int kMaxCountTasks = 64;

// ---------------------------------------------------------------------------------------
// small kernels: input conversion, output conversion, intra-block counts
// ---------------------------------------------------------------------------------------
struct Planes3 {
    const void* src[3];
    int16_t* orig[3];
    int16_t* data[3];
    int n[3];
    int w[3];      // picture width
    int pitch[3];  // source row pitch in samples (2 w for a field of a frame)
};

// Unsigned input samples to codec samples (value - 2^(depth-1)), as StreamFrameInput reads
// them (libdirac_common/pic_io.cpp:388-399), written to the original and working planes.
template <typename T>
__global__ void load_kernel(const __grid_constant__ Planes3 P, int off_luma, int off_chroma) {
    const int c = blockIdx.y;
    const T* __restrict__ src = static_cast<const T*>(P.src[c]);
    const int off = c == 0 ? off_luma : off_chroma;
    const int n = P.n[c], w = P.w[c], pitch = P.pitch[c];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int y = i / w;
        const int16_t v = (int16_t)((int)src[(size_t)y * pitch + (i - y * w)] - off);
        P.orig[c][i] = v;
        P.data[c][i] = v;
    }
}

template <typename T>
__global__ void output_kernel(const int16_t* __restrict__ rec, int n, int off, T* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = (T)((int)rec[i] + off);
}

struct CountArgs {
    const uint8_t* mode[kMaxCountTasks];
    int n;
};

// Number of INTRA blocks per task (PictureCompressor::IntraModeAnalyse's count).
__global__ void count_intra_kernel(const __grid_constant__ CountArgs A, int* __restrict__ counts) {
    const uint8_t* __restrict__ m = A.mode[blockIdx.x];
    int c = 0;
    for (int i = threadIdx.x; i < A.n; i += blockDim.x) c += m[i] == kIntraMode;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += part[k];
        counts[blockIdx.x] = t;
    }
}

// The three components' quantised indices narrowed to int16, laid end to end in dst; an index
// outside int16 sets *overflow (the caller's coefficient bound rules that out: a check).
struct NarrowArgs {
    const int32_t* src[3];
    int n[3];  // elements per component
};

__global__ void narrow_kernel(const __grid_constant__ NarrowArgs A, int16_t* __restrict__ dst,
                              int* __restrict__ overflow) {
    const int n01 = A.n[0] + A.n[1], total = n01 + A.n[2];
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int c = i < A.n[0] ? 0 : (i < n01 ? 1 : 2);
        const int v = A.src[c][i - (c == 0 ? 0 : (c == 1 ? A.n[0] : n01))];
        bad |= v < -32768 || v > 32767;
        dst[i] = (int16_t)v;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(overflow, 1);
}

// ---------------------------------------------------------------------------------------
// host structures
// ---------------------------------------------------------------------------------------
struct Slot {
    int16_t* orig[3];
    int16_t* data[3];
    int32_t* coeff[3];
    int32_t* qout[3];
    int16_t* up[3];
    int16_t* mv;
    float* cost;
    uint8_t* mode;
    int16_t* dc;
    uint8_t* split;
    float* sbcost;
    int pnum = -1;  // -1: free
};

struct Pic {
    int pnum = -1;
    int slot = -1;
    bool typed = false, intra = true, is_ref = true, coded = false, cut = false;
    std::vector<int> refs;
    bool me_valid = false;
    std::vector<int> me_refs;
    double ratio = 0.0;
    bool up_valid = false;
    dgpu_picture_info info{};
    std::vector<int> bands;        // [3][nb][3]
    std::vector<uint8_t> cb_skip;  // [3][ncb]
    int coeff_max = INT_MAX;       // the quantiser's largest band maximum (INT_MAX: unknown)

    bool is_b() const {
        return refs.size() == 2 && ((refs[0] < pnum && refs[1] > pnum) || (refs[0] > pnum && refs[1] < pnum));
    }
};

struct Encoder {
    dgpu_encoder_params P{};
    cudaStream_t st = nullptr;
    Lambdas L{};
    int xs = 0, ys = 0;          // chroma shifts
    int w[3]{}, h[3]{};          // component sizes
    int pw[3]{}, ph[3]{};        // padded (transform) sizes
    dgpu_block_params bp{};
    int nblocks = 0, nsb = 0, nb = 0;
    std::vector<int> ncb;        // per band (x, y), identical for the three components
    int ncb_total = 0;

    // GOP state (seq_compress.cpp member names in comments)
    int L1Sep = 0, num_L1 = 0, gop_len = 0;
    int m_L1_sep = 0;            // m_L1_sep
    int gop_start = 0;           // m_gop_start_num
    int code = 0;                // m_current_code_pnum
    int cur = -1;                // m_current_display_pnum
    int last_read = -1;          // m_last_picture_read
    int prepared = -1;           // picture prepared by dgpu_encoder_prepare_next, or -1
    int failed = DGPU_OK;        // first failure of a picture's coding; sticky until reset
    bool field = false;          // field coding: pictures are fields, two per loaded frame
    bool tff = false;            // top field first
    bool eos = false;            // m_eos_signalled
    std::map<int, Pic> pics;

    // device memory
    void* arena = nullptr;
    std::vector<Slot> slots;
    void* me_ws = nullptr;
    size_t me_ws_bytes = 0;
    int me_max_tasks = 0;
    void* dwt_ws = nullptr;
    size_t dwt_ws_bytes = 0;
    void* q_ws = nullptr;
    size_t q_ws_bytes = 0;
    int* d_counts = nullptr;
    void* stage = nullptr;       // one input / output frame of samples
    size_t stage_bytes = 0;
    int* h_counts = nullptr;     // pinned

    // optional per-stage timing with CUDA events on the encoder's stream
    bool profile = false;
    cudaEvent_t ev[2 * DGPU_ENC_NSTAGES] = {};
    double stage_ms[DGPU_ENC_NSTAGES] = {};
    int stage_calls[DGPU_ENC_NSTAGES] = {};

    // dgpu_encoder_code_adaptive: per picture kind (intra, B, other inter) page-locked copies
    // of a finished picture's indices and motion data, and the event after their copies
    uint8_t* kind_stage[3] = {};
    size_t kind_stage_bytes[3] = {};
    cudaEvent_t kind_ev[3] = {};
    // the three components' indices narrowed to int16 for the copy, then the overflow flag
    void* q16 = nullptr;
    size_t q16_bytes = 0;
    std::vector<uint8_t> adaptive_data;  // the last call's coded data, coding order

    ~Encoder() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (int k = 0; k < 3; ++k) {
            if (kind_ev[k]) cudaEventDestroy(kind_ev[k]);
            if (kind_stage[k]) cudaFreeHost(kind_stage[k]);
        }
        if (q16) cudaFree(q16);
        if (arena) cudaFree(arena);
        if (h_counts) cudaFreeHost(h_counts);
    }
};

// Brackets one stage with events when profiling; the elapsed time is collected at the
// stage's end (a host wait, so profiling perturbs the pipeline: use it outside timed runs).
struct StageTimer {
    Encoder& E;
    int k;
    StageTimer(Encoder& e, int stage) : E(e), k(stage) {
        if (E.profile) cudaEventRecord(E.ev[2 * k], E.st);
    }
    ~StageTimer() {
        if (!E.profile) return;
        cudaEventRecord(E.ev[2 * k + 1], E.st);
        if (cudaEventSynchronize(E.ev[2 * k + 1]) == cudaSuccess) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, E.ev[2 * k], E.ev[2 * k + 1]) == cudaSuccess) {
                E.stage_ms[k] += ms;
                E.stage_calls[k] += 1;
            }
        }
        cudaGetLastError();
    }
};

int comp_depth(const Encoder& E, int c) { return c == 0 ? E.P.luma_depth : E.P.chroma_depth; }

size_t sample_bytes(const Encoder& E) { return E.P.luma_depth > 8 || E.P.chroma_depth > 8 ? 2 : 1; }

// ---- GOP structure ----------------------------------------------------------------------
int coded_to_display(const Encoder& E, int cnum) {
    const int s = E.m_L1_sep;
    if (E.field) {  // FieldSequenceCompressor::CodedToDisplay (seq_compress.cpp:859-879)
        const int fnum = cnum >> 1;
        if (s > 0) {
            if (fnum == 0) return cnum;
            if ((fnum - 1) % s == 0) return cnum + (s - 1) * 2;
            return cnum - 2;
        }
        return cnum;
    }
    if (s > 0) {
        if (cnum == 0) return 0;
        if ((cnum - 1) % s == 0) return cnum + s - 1;
        return cnum - 1;
    }
    return cnum;
}

bool can_encode(Encoder& E) {
    if (E.eos) {
        if (E.num_L1 > 0) {
            // in frames: two fields to a frame when field coding (seq_compress.cpp:162-164)
            const int ff = E.field ? 2 : 1;
            const int last_frame = E.last_read / ff, code_frame = E.code / ff;
            if (last_frame >= code_frame + (last_frame % E.L1Sep)) return true;
            if (code_frame <= last_frame) {
                E.cur = E.code;
                return true;
            }
            return false;
        }
        return E.last_read >= E.cur;
    }
    return E.last_read >= E.cur + std::max(4, 2 * E.L1Sep);
}

// FrameSequenceCompressor::SetPicTypeAndRefs with the given separation; `avail` is the last
// loaded picture number (IsPictureAvail).
void type_refs(const Encoder& E, int pnum, int sep, int avail, bool& intra, bool& is_ref, std::vector<int>& refs) {
    const int rel = pnum - E.gop_start;
    refs.clear();
    if (E.num_L1 > 0) {
        if (rel % E.gop_len == 0) {
            intra = true;
            is_ref = E.gop_len > 1;
        } else if (rel % sep == 0) {
            intra = false;
            is_ref = true;
            refs.push_back(pnum - sep);
            if ((rel - sep) % E.gop_len > 0 && sep > 1) refs.push_back(pnum - 2 * sep);
        } else if ((rel + 1) % sep == 0) {
            intra = false;
            is_ref = false;
            refs.push_back(pnum - 1);
            if (pnum + 1 <= avail) refs.push_back(pnum + 1);
        } else {
            intra = false;
            is_ref = true;
            refs.push_back(pnum - 1);
            const int next_ref = (pnum / sep + 1) * sep;
            if (next_ref <= avail) refs.push_back(next_ref);
        }
    } else {
        intra = true;
        is_ref = false;
    }
}

// FieldSequenceCompressor::SetPicTypeAndRefs (seq_compress.cpp:767-852): fields 2n and 2n + 1
// of frame n; the second field of an I frame is predicted from the first.
void type_refs_field(const Encoder& E, int pnum, int sep, int avail, bool& intra, bool& is_ref,
                     std::vector<int>& refs) {
    const int rel = pnum - E.gop_start;
    refs.clear();
    if (E.num_L1 <= 0) {
        intra = true;
        is_ref = false;
        return;
    }
    const bool second = pnum % 2 != 0;
    if ((rel / 2) % E.gop_len == 0) {
        if (E.gop_len > 1) {
            intra = !second;
            is_ref = true;
            if (second) refs.push_back(pnum - 1);
        } else {
            intra = true;
            is_ref = false;
        }
    } else if ((rel / 2) % sep == 0) {
        intra = false;
        is_ref = true;
        if (second) {
            refs.push_back(pnum - 1);
            refs.push_back(pnum - sep * 2);
        } else {
            refs.push_back(pnum - sep * 2);
            refs.push_back(pnum - sep * 2 + 1);
        }
    } else if ((rel / 2 + 1) % sep == 0) {
        intra = false;
        is_ref = !second;
        refs.push_back(pnum - 1);
        if (pnum + 2 <= avail) refs.push_back(pnum + 2);
    } else {
        intra = false;
        is_ref = true;
        refs.push_back(pnum - 1);
        const int next_ref = (((pnum / 2) / sep + 1) * sep) * 2 + (pnum % 2);
        if (next_ref <= avail) refs.push_back(next_ref);
    }
}

void set_type(Encoder& E, Pic& p) {
    if (E.field)
        type_refs_field(E, p.pnum, E.m_L1_sep, E.last_read, p.intra, p.is_ref, p.refs);
    else
        type_refs(E, p.pnum, E.m_L1_sep, E.last_read, p.intra, p.is_ref, p.refs);
    p.typed = true;
}

// ---- device helpers ---------------------------------------------------------------------
Slot& slot_of(Encoder& E, const Pic& p) { return E.slots[p.slot]; }

int ensure_up(Encoder& E, Pic& r) {
    if (r.up_valid) return DGPU_OK;
    StageTimer timer(E, DGPU_STAGE_UPCONVERT);
    Slot& s = slot_of(E, r);
    const int16_t* pic[3] = {s.data[0], s.data[1], s.data[2]};
    int16_t* up[3] = {s.up[0], s.up[1], s.up[2]};
    int ups[3], bd[3];
    for (int c = 0; c < 3; ++c) {
        ups[c] = 2 * E.w[c];
        bd[c] = comp_depth(E, c);
    }
    const int rc = dgpu_upconvert_batch(3, pic, E.w, E.h, E.w, bd, up, ups, E.st);
    if (rc) return rc;
    r.up_valid = true;
    return DGPU_OK;
}

// Refs a not-yet-typed picture will most likely get (the normal separation): used only to
// estimate ahead; results are keyed by the references they were computed with.
bool predicted_refs(const Encoder& E, const Pic& q, std::vector<int>& refs) {
    if (q.typed) {
        if (q.intra) return false;
        refs = q.refs;
        return true;
    }
    bool intra, is_ref;
    type_refs(E, q.pnum, E.L1Sep, E.last_read, intra, is_ref, refs);
    return !intra;
}

struct MeTask {
    Encoder* E;
    int pnum;
    std::vector<int> refs;
};

// Motion-estimation tasks of E: `first` (when given) against its current references, then
// every other loaded, uncoded picture whose references are (or will most likely be) known and
// already loaded and whose estimate is missing or was made against other references; at most
// `cap` tasks.
void collect_me_tasks(Encoder& E, const Pic* first, int cap, std::vector<MeTask>& tasks) {
    int n = 0;
    if (first) {
        tasks.push_back({&E, first->pnum, first->refs});
        ++n;
    }
    for (auto& kv : E.pics) {
        Pic& q = kv.second;
        if (n >= cap) break;
        if ((first && q.pnum == first->pnum) || q.coded || q.slot < 0) continue;
        // without the end of the sequence, a picture's references may still change as
        // pictures arrive: only look at pictures a full sub-group before the last loaded
        if (!E.eos && q.pnum + std::max(E.L1Sep, 1) > E.last_read) continue;
        std::vector<int> refs;
        if (!predicted_refs(E, q, refs)) continue;
        if (q.me_valid && q.me_refs == refs) continue;
        bool ok = true;
        for (int r : refs) ok = ok && r >= 0 && r <= E.last_read && E.pics.count(r) && E.pics[r].slot >= 0;
        if (ok) {
            tasks.push_back({&E, q.pnum, refs});
            ++n;
        }
    }
}

// Runs the tasks (of one or several encoders with the same picture size, chroma format,
// block parameters and luma depth) in one batched estimation on stream st, then records each
// picture's estimate and intra-block ratio.  ws: workspace of ws_bytes; d_counts / h_counts:
// device / pinned host ints, one per task.
int run_me_tasks(const std::vector<MeTask>& tasks, cudaStream_t st, void* ws, size_t ws_bytes, int* d_counts,
                 int* h_counts) {
    if (tasks.empty()) return DGPU_OK;
    Encoder& E0 = *tasks[0].E;
    // pictures involved, in first-use order
    std::vector<std::pair<Encoder*, int>> pics_used;
    auto index_of = [&](Encoder* e, int pn) {
        for (size_t k = 0; k < pics_used.size(); ++k)
            if (pics_used[k].first == e && pics_used[k].second == pn) return (int)k;
        pics_used.push_back({e, pn});
        return (int)pics_used.size() - 1;
    };
    const int nt = (int)tasks.size();
    std::vector<int> tp(nt), t1(nt), t2(nt);
    std::vector<float> tl(nt);
    for (int t = 0; t < nt; ++t) {
        tp[t] = index_of(tasks[t].E, tasks[t].pnum);
        t1[t] = index_of(tasks[t].E, tasks[t].refs[0]);
        t2[t] = tasks[t].refs.size() > 1 ? index_of(tasks[t].E, tasks[t].refs[1]) : -1;
        tl[t] = tasks[t].E->L.me;  // L1MELambda == L2MELambda (common.cpp:464-465)
    }
    std::vector<const int16_t*> planes;
    for (auto& pu : pics_used) {
        Slot& s = pu.first->slots[pu.first->pics[pu.second].slot];
        for (int c = 0; c < 3; ++c) planes.push_back(s.orig[c]);
    }
    std::vector<int16_t*> mv(nt), dc(nt);
    std::vector<float*> cost(nt), sbc(nt);
    std::vector<uint8_t*> mode(nt), split(nt);
    for (int t = 0; t < nt; ++t) {
        Encoder& E = *tasks[t].E;
        Slot& s = E.slots[E.pics[tasks[t].pnum].slot];
        mv[t] = s.mv;
        cost[t] = s.cost;
        mode[t] = s.mode;
        dc[t] = s.dc;
        split[t] = s.split;
        sbc[t] = s.sbcost;
    }
    int rc = dgpu_motion_estimate_batch(E0.P.cformat, E0.w[0], E0.h[0], &E0.bp, E0.P.luma_depth,
                                        (int)pics_used.size(), planes.data(), nt, tp.data(), t1.data(), t2.data(),
                                        tl.data(), 3, mv.data(), cost.data(), mode.data(), dc.data(), split.data(),
                                        sbc.data(), ws, ws_bytes, st);
    if (rc) return rc;
    for (int t0 = 0; t0 < nt; t0 += kMaxCountTasks) {
        CountArgs A{};
        const int k = std::min(kMaxCountTasks, nt - t0);
        for (int t = 0; t < k; ++t) A.mode[t] = mode[t0 + t];
        A.n = E0.nblocks;
        count_intra_kernel<<<k, 256, 0, st>>>(A, d_counts + t0);
        DGPU_CHECK_LAUNCH();
    }
    DGPU_CHECK_CUDA(cudaMemcpyAsync(h_counts, d_counts, sizeof(int) * nt, cudaMemcpyDeviceToHost, st));
    DGPU_CHECK_CUDA(host_wait(st));
    for (int t = 0; t < nt; ++t) {
        Encoder& E = *tasks[t].E;
        Pic& q = E.pics[tasks[t].pnum];
        q.me_valid = true;
        q.me_refs = tasks[t].refs;
        q.ratio = (double)h_counts[t] / (double)E.nblocks;
    }
    return DGPU_OK;
}

// Motion estimation of p against its current references, batched with every other loaded
// picture whose references are (or will most likely be) known and already loaded.
int ensure_me(Encoder& E, Pic& p) {
    if (p.me_valid && p.me_refs == p.refs) return DGPU_OK;
    StageTimer timer(E, DGPU_STAGE_ME);
    std::vector<MeTask> tasks;
    collect_me_tasks(E, &p, E.me_max_tasks, tasks);
    return run_me_tasks(tasks, E.st, E.me_ws, E.me_ws_bytes, E.d_counts, E.h_counts);
}

int motion_compensate(Encoder& E, Pic& p, int add_or_sub, bool clip) {
    Slot& s = slot_of(E, p);
    Pic& r1 = E.pics[p.refs[0]];
    int rc = ensure_up(E, r1);
    if (rc) return rc;
    const int16_t* up1[3] = {E.slots[r1.slot].up[0], E.slots[r1.slot].up[1], E.slots[r1.slot].up[2]};
    const int16_t* up2[3] = {nullptr, nullptr, nullptr};
    const bool two = p.refs.size() > 1;
    if (two) {
        Pic& r2 = E.pics[p.refs[1]];
        rc = ensure_up(E, r2);
        if (rc) return rc;
        for (int c = 0; c < 3; ++c) up2[c] = E.slots[r2.slot].up[c];
    }
    int16_t* pic[3] = {s.data[0], s.data[1], s.data[2]};
    StageTimer timer(E, add_or_sub == DGPU_SUBTRACT ? DGPU_STAGE_MC_SUBTRACT : DGPU_STAGE_MC_ADD);
    return dgpu_motion_compensate(add_or_sub, E.P.cformat, E.w[0], E.h[0], &E.bp, s.mv,
                                  two ? s.mv + 2 * E.nblocks : nullptr, s.mode, s.dc, s.split, pic, E.w, up1,
                                  two ? up2 : nullptr, clip ? E.P.luma_depth : 0, clip ? E.P.chroma_depth : 0, E.st);
}

int transform(Encoder& E, Pic& p, int dir, int filter) {
    StageTimer timer(E, dir == DGPU_FORWARD ? DGPU_STAGE_DWT_FORWARD : DGPU_STAGE_DWT_INVERSE);
    Slot& s = slot_of(E, p);
    int filt[3] = {filter, filter, filter};
    int depth[3] = {E.P.wlt_depth, E.P.wlt_depth, E.P.wlt_depth};
    int16_t* pic[3] = {s.data[0], s.data[1], s.data[2]};
    int32_t* coeff[3] = {s.coeff[0], s.coeff[1], s.coeff[2]};
    return dgpu_wavelet_transform_batch(dir, 3, filt, depth, pic, E.w, E.h, E.w, coeff, E.pw, E.ph, E.pw, E.dwt_ws,
                                        E.dwt_ws_bytes, E.st);
}

float comp_lambda(const Encoder& E, const Pic& p, int comp) {
    return component_lambda(E.L, p.intra, p.is_b(), p.ratio, comp);
}

// Transform (unless done already, forward_done), quantiser choice and quantisation, inverse
// transform.
int code_residue(Encoder& E, Pic& p, const float* ecf_in, bool forward_done = false) {
    Slot& s = slot_of(E, p);
    const int depth = E.P.wlt_depth;
    const int filter = p.intra ? E.P.intra_filter : E.P.inter_filter;
    const double cpd_scale = perceptual_scale(p.intra, p.ratio);
    const int nb = E.nb;
    std::vector<float> wt(3 * nb), ecf(3 * nb);
    std::vector<int> ncb(6 * nb);
    std::vector<double> wd(nb);
    float lam[3];
    int intra[3], dep[3];
    for (int c = 0; c < 3; ++c) {
        int rc = dgpu_band_weights(filter, depth, E.pw[c], E.ph[c], c, E.P.cformat, E.P.cpd, (float)cpd_scale, E.field ? 1 : 0,
                                   wd.data());
        if (rc) return rc;
        for (int b = 0; b < nb; ++b) wt[c * nb + b] = (float)wd[b];
        if (ecf_in)
            std::memcpy(&ecf[c * nb], ecf_in + c * nb, sizeof(float) * nb);
        else
            initial_ecf(depth, p.intra, &ecf[c * nb]);
        std::memcpy(&ncb[2 * c * nb], E.ncb.data(), sizeof(int) * 2 * nb);
        lam[c] = comp_lambda(E, p, c);
        intra[c] = p.intra ? 1 : 0;
        dep[c] = depth;
    }
    std::vector<int> qidx(3 * nb), skip(3 * nb), bits(3 * nb);
    p.cb_skip.assign((size_t)3 * E.ncb_total, 0);
    int32_t* coeff[3] = {s.coeff[0], s.coeff[1], s.coeff[2]};
    int32_t* qout[3] = {s.qout[0], s.qout[1], s.qout[2]};
    int rc = forward_done ? DGPU_OK : transform(E, p, DGPU_FORWARD, filter);
    if (rc) return rc;
    {
        StageTimer timer(E, DGPU_STAGE_QUANT);
        rc = code_residue_batch(3, intra, dep, coeff, E.pw, E.ph, lam, wt.data(), ecf.data(), ncb.data(), qidx.data(),
                                skip.data(), bits.data(), p.cb_skip.data(), qout, E.q_ws, E.q_ws_bytes, E.st,
                                &p.coeff_max);
    }
    if (rc) return rc;
    rc = transform(E, p, DGPU_BACKWARD, filter);
    if (rc) return rc;
    p.bands.resize((size_t)9 * nb);
    for (int k = 0; k < 3 * nb; ++k) {
        p.bands[3 * k] = qidx[k];
        p.bands[3 * k + 1] = skip[k];
        p.bands[3 * k + 2] = bits[k];
    }
    dgpu_picture_info& I = p.info;
    I.filter = filter;
    I.cpd_scale = cpd_scale;
    for (int c = 0; c < 3; ++c) I.lambda[c] = lam[c];
    return DGPU_OK;
}

// A coded picture no later picture can reference: references reach back at most
// 2 * L1 separation pictures from the earliest picture not yet coded.
bool releasable(const Encoder& E, const Pic& p) {
    if (!p.coded) return false;
    int first_uncoded = E.last_read + 1;
    for (const auto& kv : E.pics)
        if (!kv.second.coded) {
            first_uncoded = kv.first;
            break;
        }
    return p.pnum < first_uncoded - 2 * std::max(E.L1Sep, 1);
}

int take_slot(Encoder& E) {
    for (size_t k = 0; k < E.slots.size(); ++k)
        if (E.slots[k].pnum < 0) return (int)k;
    for (auto it = E.pics.begin(); it != E.pics.end(); ++it) {
        if (releasable(E, it->second)) {
            const int k = it->second.slot;
            E.slots[k].pnum = -1;
            E.pics.erase(it);
            return k;
        }
    }
    return -1;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

// Checks the parameters and fills the encoder's geometry, GOP constants and workspace sizes;
// *total receives the bytes of its device arena.  Allocates nothing.
static int encoder_setup(const dgpu_encoder_params& P, int max_pictures, void* stream, Encoder* E, size_t* total,
                         size_t* slot_bytes, int* nslots_out) {
    if (P.cformat < 0 || P.cformat > 2 || P.width < 16 || P.height < 16 || P.luma_depth < 8 || P.luma_depth > 14 ||
        P.chroma_depth < 8 || P.chroma_depth > 14 || P.num_l1 < 0 || (P.num_l1 > 0 && P.l1_sep < 1) ||
        P.mv_precision < 1 || P.mv_precision > 3 || P.wlt_depth < 1 || P.wlt_depth > 6 || P.intra_filter < 0 ||
        P.intra_filter > 6 || P.inter_filter < 0 || P.inter_filter > 6 || P.xbsep < 1 || P.ybsep < 1 ||
        P.xblen < P.xbsep || P.yblen < P.ybsep || P.field_coding < 0 || P.field_coding > 1)
        return DGPU_ERR_ARG;
    E->P = P;
    E->field = P.field_coding == 1;
    E->tff = P.top_field_first != 0;
    E->st = as_stream(stream);
    E->L = calc_lambdas(P.qf);
    E->xs = P.cformat == 0 ? 0 : 1;
    E->ys = P.cformat == 2 ? 1 : 0;
    // field coding codes pictures of half the frame's height (dirac_encoder.cpp:525-530)
    if (E->field && (P.height % (2 << E->ys) != 0 || P.height < 32)) return DGPU_ERR_SIZE;
    const int pic_h = E->field ? P.height / 2 : P.height;
    E->w[0] = P.width;
    E->h[0] = pic_h;
    E->w[1] = E->w[2] = P.width >> E->xs;
    E->h[1] = E->h[2] = pic_h >> E->ys;
    const int mul = 1 << P.wlt_depth;
    for (int c = 0; c < 3; ++c) {
        E->pw[c] = (E->w[c] + mul - 1) / mul * mul;
        E->ph[c] = (E->h[c] + mul - 1) / mul * mul;
    }
    // SequenceCompressor::SetMotionParameters (seq_compress.cpp:104-133)
    E->bp.precision = P.mv_precision;
    E->bp.xblen = P.xblen;
    E->bp.yblen = P.yblen;
    E->bp.xbsep = P.xbsep;
    E->bp.ybsep = P.ybsep;
    E->bp.xnum_sb = (P.width + 4 * P.xbsep - 1) / (4 * P.xbsep);
    E->bp.ynum_sb = (pic_h + 4 * P.ybsep - 1) / (4 * P.ybsep);
    E->nsb = E->bp.xnum_sb * E->bp.ynum_sb;
    E->nblocks = 16 * E->nsb;
    E->nb = 3 * P.wlt_depth + 1;
    E->ncb.assign((size_t)2 * E->nb, 0);
    int rc = dgpu_code_blocks(P.wlt_depth, P.width, pic_h, 1, E->ncb.data());
    if (rc) return rc;
    for (int b = 0; b < E->nb; ++b) E->ncb_total += E->ncb[2 * b] * E->ncb[2 * b + 1];
    // GOP (dirac_encoder.cpp:562-572, common.cpp:512-518)
    E->num_L1 = P.num_l1;
    E->L1Sep = P.num_l1 > 0 ? P.l1_sep : 0;
    E->gop_len = P.num_l1 > 0 ? (P.num_l1 + 1) * P.l1_sep : 10;
    E->m_L1_sep = E->L1Sep;
    const int min_slots = 4 * std::max(E->L1Sep, 1) + 8;
    *nslots_out = std::max(max_pictures, min_slots);
    const int nslots = *nslots_out;

    // ---- sizes ----
    size_t plane16 = 0, plane32 = 0, up16 = 0;
    for (int c = 0; c < 3; ++c) {
        plane16 += align_up((size_t)E->w[c] * E->h[c] * 2, 256);
        plane32 += align_up((size_t)E->pw[c] * E->ph[c] * 4, 256);
        up16 += align_up((size_t)4 * E->w[c] * E->h[c] * 2, 256);
    }
    const size_t me_out = align_up((size_t)E->nblocks * 2 * 2 * 2, 256) + align_up((size_t)E->nblocks * 2 * 3 * 4, 256) +
                          align_up(E->nblocks, 256) + align_up((size_t)E->nblocks * 3 * 2, 256) +
                          align_up(E->nsb, 256) + align_up((size_t)E->nsb * 4, 256);
    *slot_bytes = 2 * plane16 + 2 * plane32 + up16 + me_out;
    E->me_max_tasks = std::min(nslots, 64);
    {
        std::vector<int> r2(E->me_max_tasks, 0);
        const int npics_max = std::min(nslots, 3 * E->me_max_tasks);
        E->me_ws_bytes = dgpu_me_batch_workspace_bytes(P.cformat, P.width, pic_h, &E->bp, npics_max,
                                                       E->me_max_tasks, r2.data(), 3);
        if (E->me_ws_bytes == 0) return DGPU_ERR_ARG;
    }
    for (int c = 0; c < 3; ++c) E->dwt_ws_bytes += align_up(dgpu_dwt_scratch_bytes(E->pw[c], E->ph[c], P.wlt_depth), 256);
    {
        int intra[3] = {1, 1, 1}, dep[3] = {P.wlt_depth, P.wlt_depth, P.wlt_depth};
        std::vector<int> ncb3(6 * E->nb);
        for (int c = 0; c < 3; ++c) std::memcpy(&ncb3[2 * c * E->nb], E->ncb.data(), sizeof(int) * 2 * E->nb);
        E->q_ws_bytes = dgpu_code_residue_workspace_bytes(3, intra, dep, E->pw, E->ph, ncb3.data());
        if (E->q_ws_bytes == 0) return DGPU_ERR_ARG;
    }
    // one input frame (two fields when field coding) or one output picture
    for (int c = 0; c < 3; ++c)
        E->stage_bytes += align_up((size_t)E->w[c] * E->h[c] * 2 * (E->field ? 2 : 1), 256);
    *total = (size_t)nslots * align_up(*slot_bytes, 256) + align_up(E->me_ws_bytes, 256) +
             align_up(E->dwt_ws_bytes, 256) + align_up(E->q_ws_bytes, 256) +
             align_up(sizeof(int) * E->me_max_tasks, 256) + E->stage_bytes;
    return DGPU_OK;
}

extern "C" size_t dgpu_encoder_device_bytes(const dgpu_encoder_params* params, int max_pictures) {
    if (!params) return 0;
    Encoder E;
    size_t total = 0, slot = 0;
    int nslots = 0;
    return encoder_setup(*params, max_pictures, nullptr, &E, &total, &slot, &nslots) == DGPU_OK ? total : 0;
}

extern "C" int dgpu_encoder_create(const dgpu_encoder_params* params, int max_pictures, void* stream, void** out) {
    if (!params || !out) return DGPU_ERR_ARG;
    *out = nullptr;
    Encoder* E = new (std::nothrow) Encoder();
    if (!E) return DGPU_ERR_NOMEM;
    size_t total = 0, slot_bytes = 0;
    int nslots = 0;
    {
        const int rc = encoder_setup(*params, max_pictures, stream, E, &total, &slot_bytes, &nslots);
        if (rc) {
            delete E;
            return rc;
        }
    }
    if (cudaMalloc(&E->arena, total) != cudaSuccess) {
        cudaGetLastError();
        E->arena = nullptr;
        delete E;
        return DGPU_ERR_NOMEM;
    }
    if (cudaMallocHost(&E->h_counts, sizeof(int) * E->me_max_tasks) != cudaSuccess) {
        cudaGetLastError();
        E->h_counts = nullptr;
        delete E;
        return DGPU_ERR_NOMEM;
    }
    char* q = static_cast<char*>(E->arena);
    auto take = [&](size_t bytes) {
        char* r = q;
        q += align_up(bytes, 256);
        return r;
    };
    E->slots.resize(nslots);
    for (int k = 0; k < nslots; ++k) {
        Slot& s = E->slots[k];
        for (int c = 0; c < 3; ++c) s.orig[c] = reinterpret_cast<int16_t*>(take((size_t)E->w[c] * E->h[c] * 2));
        for (int c = 0; c < 3; ++c) s.data[c] = reinterpret_cast<int16_t*>(take((size_t)E->w[c] * E->h[c] * 2));
        for (int c = 0; c < 3; ++c) s.coeff[c] = reinterpret_cast<int32_t*>(take((size_t)E->pw[c] * E->ph[c] * 4));
        for (int c = 0; c < 3; ++c) s.qout[c] = reinterpret_cast<int32_t*>(take((size_t)E->pw[c] * E->ph[c] * 4));
        for (int c = 0; c < 3; ++c) s.up[c] = reinterpret_cast<int16_t*>(take((size_t)4 * E->w[c] * E->h[c] * 2));
        s.mv = reinterpret_cast<int16_t*>(take((size_t)E->nblocks * 2 * 2 * 2));
        s.cost = reinterpret_cast<float*>(take((size_t)E->nblocks * 2 * 3 * 4));
        s.mode = reinterpret_cast<uint8_t*>(take(E->nblocks));
        s.dc = reinterpret_cast<int16_t*>(take((size_t)E->nblocks * 3 * 2));
        s.split = reinterpret_cast<uint8_t*>(take(E->nsb));
        s.sbcost = reinterpret_cast<float*>(take((size_t)E->nsb * 4));
        q = static_cast<char*>(E->arena) + (size_t)(k + 1) * align_up(slot_bytes, 256);
    }
    E->me_ws = take(E->me_ws_bytes);
    E->dwt_ws = take(E->dwt_ws_bytes);
    E->q_ws = take(E->q_ws_bytes);
    E->d_counts = reinterpret_cast<int*>(take(sizeof(int) * E->me_max_tasks));
    E->stage = take(E->stage_bytes);
    *out = E;
    return DGPU_OK;
}

extern "C" int dgpu_encoder_destroy(void* enc) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E) return DGPU_ERR_ARG;
    cudaStreamSynchronize(E->st);
    delete E;
    return DGPU_OK;
}

namespace dgpu {
namespace {

// One picture into slot k from device planes src[c] with row pitch pitch[c] (samples).
int load_slot(Encoder& E, int k, const void* const* src, const int* pitch) {
    Slot& s = E.slots[k];
    Planes3 P3{};
    for (int c = 0; c < 3; ++c) {
        P3.src[c] = src[c];
        P3.orig[c] = s.orig[c];
        P3.data[c] = s.data[c];
        P3.n[c] = E.w[c] * E.h[c];
        P3.w[c] = E.w[c];
        P3.pitch[c] = pitch[c];
    }
    StageTimer timer(E, DGPU_STAGE_LOAD);
    dim3 grid(std::min((E.w[0] * E.h[0] + 255) / 256, 148 * 8), 3);
    const int offl = 1 << (E.P.luma_depth - 1), offc = 1 << (E.P.chroma_depth - 1);
    if (sample_bytes(E) == 1)
        load_kernel<uint8_t><<<grid, 256, 0, E.st>>>(P3, offl, offc);
    else
        load_kernel<uint16_t><<<grid, 256, 0, E.st>>>(P3, offl, offc);
    DGPU_CHECK_LAUNCH();
    const int pnum = ++E.last_read;
    s.pnum = pnum;
    Pic& p = E.pics[pnum];
    p = Pic();
    p.pnum = pnum;
    p.slot = k;
    return DGPU_OK;
}

}  // namespace
}  // namespace dgpu

extern "C" int dgpu_encoder_load(void* enc, const void* const* planes, int on_host) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E || !planes || !planes[0] || !planes[1] || !planes[2]) return DGPU_ERR_ARG;
    if (E->eos) return DGPU_ERR_ARG;
    // a frame, or the two fields of an interlaced frame (StreamFieldInput::ReadFieldComponent,
    // pic_io.cpp:464-530): each field takes every other row of the frame
    const int npics = E->field ? 2 : 1;
    int k[2] = {-1, -1};
    for (int f = 0; f < npics; ++f) {
        k[f] = take_slot(*E);
        if (k[f] < 0) {
            if (f == 1) E->slots[k[0]].pnum = -1;  // nothing loaded: give the first slot back
            return DGPU_ERR_SIZE;
        }
        E->slots[k[f]].pnum = 0x7fffffff;  // reserved, so that the second take finds another slot
    }
    const size_t sb = sample_bytes(*E);
    const void* src[3];
    size_t off = 0;
    for (int c = 0; c < 3; ++c) {
        const size_t bytes = (size_t)E->w[c] * E->h[c] * npics * sb;  // the whole frame
        if (on_host) {
            void* dst = static_cast<char*>(E->stage) + off;
            DGPU_CHECK_CUDA(cudaMemcpyAsync(dst, planes[c], bytes, cudaMemcpyHostToDevice, E->st));
            src[c] = dst;
            off += align_up(bytes, 256);
        } else {
            src[c] = planes[c];
        }
    }
    for (int f = 0; f < npics; ++f) {
        const void* fsrc[3];
        int pitch[3];
        // field f of the frame: the even rows for the first field when the top field is first
        const int parity = E->field ? (f == 0 ? (E->tff ? 0 : 1) : (E->tff ? 1 : 0)) : 0;
        for (int c = 0; c < 3; ++c) {
            pitch[c] = E->w[c] * npics;
            fsrc[c] = static_cast<const char*>(src[c]) + (size_t)parity * E->w[c] * sb;
        }
        const int rc = load_slot(*E, k[f], fsrc, pitch);
        if (rc) return rc;
    }
    return DGPU_OK;
}

extern "C" int dgpu_encoder_reset(void* enc) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E) return DGPU_ERR_ARG;
    DGPU_CHECK_CUDA(cudaStreamSynchronize(E->st));
    E->pics.clear();
    for (Slot& s : E->slots) s.pnum = -1;
    E->m_L1_sep = E->L1Sep;
    E->gop_start = 0;
    E->code = 0;
    E->cur = -1;
    E->last_read = -1;
    E->prepared = -1;
    E->failed = DGPU_OK;
    E->eos = false;
    return DGPU_OK;
}

extern "C" int dgpu_encoder_profile(void* enc, int enable, double* stage_ms, int* stage_calls) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E) return DGPU_ERR_ARG;
    if (stage_ms)
        for (int k = 0; k < DGPU_ENC_NSTAGES; ++k) stage_ms[k] = E->stage_ms[k];
    if (stage_calls)
        for (int k = 0; k < DGPU_ENC_NSTAGES; ++k) stage_calls[k] = E->stage_calls[k];
    if (enable && !E->ev[0])
        for (auto& e : E->ev) DGPU_CHECK_CUDA(cudaEventCreate(&e));
    E->profile = enable != 0;
    for (int k = 0; k < DGPU_ENC_NSTAGES; ++k) {
        E->stage_ms[k] = 0.0;
        E->stage_calls[k] = 0;
    }
    return DGPU_OK;
}

extern "C" int dgpu_encoder_end_sequence(void* enc) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E) return DGPU_ERR_ARG;
    E->eos = true;
    return DGPU_OK;
}

namespace dgpu {
namespace {
int code_next_impl(Encoder* E, const float* ecf, const float* ecf_state, dgpu_picture_info* info);
int prepare_impl(Encoder* E, dgpu_picture_info* info);
int finish_impl(Encoder* E, const float* ecf, const float* ecf_state, dgpu_picture_info* info);
}  // namespace
}  // namespace dgpu

namespace dgpu {
namespace {
// A failure part-way through a picture's coding leaves its slot holding half-coded data (the
// residue after SUBTRACT, or coefficients); coding on from there would be silently wrong, so
// the failure is recorded and every later coding call returns it until dgpu_encoder_reset.
int sticky(Encoder* E, int rc) {
    if (rc < 0) E->failed = rc;
    return rc;
}
}  // namespace
}  // namespace dgpu

extern "C" int dgpu_encoder_prepare_next(void* enc, dgpu_picture_info* info) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E) return DGPU_ERR_ARG;
    if (E->failed) return E->failed;
    return sticky(E, prepare_impl(E, info));
}

extern "C" int dgpu_encoder_finish_next(void* enc, const float* ecf, const float* ecf_state, dgpu_picture_info* info) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E) return DGPU_ERR_ARG;
    if (E->failed) return E->failed;
    if (E->prepared < 0) return DGPU_ERR_ARG;  // nothing prepared: no state was touched
    return sticky(E, finish_impl(E, ecf, ecf_state, info));
}

extern "C" int dgpu_encoder_code_next(void* enc, const float* ecf, dgpu_picture_info* info) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E) return DGPU_ERR_ARG;
    if (E->failed) return E->failed;
    return sticky(E, code_next_impl(E, ecf, nullptr, info));
}

extern "C" int dgpu_encoder_code_next_adaptive(void* enc, const float* ecf_state, dgpu_picture_info* info) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E || !ecf_state) return DGPU_ERR_ARG;
    if (E->failed) return E->failed;
    return sticky(E, code_next_impl(E, nullptr, ecf_state, info));
}

namespace dgpu {
namespace {

// dgpu_encoder_code_next; with ecf_state, the picture's factors are taken from it once its
// kind is final (after cut detection): EntropyCorrector::Factor's index, intra 0, B 1, other
// inter 2 (common.cpp:65-75).
// Steps of a picture's coding that do not depend on the entropy-correction factors: picture
// types, motion estimation, intra analysis, the P-only switch and cut detection, motion
// compensation SUBTRACT and the forward transform.  Returns 1 with the picture's provisional
// info (its kind is final), 0 when more input is needed.
int prepare_impl(Encoder* E, dgpu_picture_info* info) {
    if (E->prepared >= 0) {  // already prepared
        if (info) *info = E->pics[E->prepared].info;
        return 1;
    }
    if (E->last_read < 0) return 0;
    // a scheduled return to the normal L1 separation (seq_compress.cpp:212-219); ff fields to a
    // frame when field coding
    const int ff = E->field ? 2 : 1;
    if (E->L1Sep > 0 && E->L1Sep != E->m_L1_sep && (E->code - ff) % (E->L1Sep * ff) == 0) E->m_L1_sep = E->L1Sep;
    E->cur = coded_to_display(*E, E->code);
    if (!can_encode(*E)) return 0;
    if (!E->pics.count(E->cur) || E->pics[E->cur].coded) return 0;
    // 1. picture types one sub-group ahead
    for (auto& kv : E->pics) {
        Pic& q = kv.second;
        if (!q.typed && !q.coded && (E->num_L1 == 0 || q.pnum < E->cur + E->L1Sep)) set_type(*E, q);
    }
    Pic* p = &E->pics[E->cur];
    int rc;
    if (!p->intra) {
        // 8.-11. estimation, intra analysis, switch to P-only sub-groups
        for (;;) {
            rc = ensure_me(*E, *p);
            if (rc) return rc;
            if (E->m_L1_sep > 1 && p->ratio > 0.25 && E->cur % (E->L1Sep * ff) == 0) {
                E->m_L1_sep = 1;
                for (int i = 0; i < ff * E->L1Sep; ++i) {
                    auto it = E->pics.find(E->cur - i + (ff - 1));
                    if (it == E->pics.end()) return DGPU_ERR_ARG;
                    set_type(*E, it->second);
                }
                p->me_valid = false;
                E->cur = coded_to_display(*E, E->code);
                p = &E->pics[E->cur];
                continue;
            }
            break;
        }
        // cut detection
        if (p->ratio > 0.3333) {
            p->cut = true;
            if (E->L1Sep > 1 && E->cur % (ff * E->L1Sep) == 0) E->gop_start = p->pnum;
            p->intra = true;
        } else {
            rc = motion_compensate(*E, *p, DGPU_SUBTRACT, false);
            if (rc) return rc;
        }
    }
    // 16. forward transform
    rc = transform(*E, *p, DGPU_FORWARD, p->intra ? E->P.intra_filter : E->P.inter_filter);
    if (rc) return rc;
    dgpu_picture_info& I = p->info;
    I.pnum = p->pnum;
    I.coded_num = E->code;
    I.intra = p->intra ? 1 : 0;
    I.is_ref = p->is_ref ? 1 : 0;
    I.cut = p->cut ? 1 : 0;
    I.num_refs = (int)p->refs.size();
    I.ref1 = p->refs.size() > 0 ? p->refs[0] : -1;
    I.ref2 = p->refs.size() > 1 ? p->refs[1] : -1;
    I.is_b = p->is_b() ? 1 : 0;
    I.intra_ratio = p->ratio;
    I.filter = p->intra ? E->P.intra_filter : E->P.inter_filter;
    E->prepared = p->pnum;
    if (info) *info = I;
    return 1;
}

// The rest of the prepared picture's coding: quantiser choice with the given factors (or the
// picture kind's factors from ecf_state), quantisation, inverse transform, reconstruction.
int finish_impl(Encoder* E, const float* ecf, const float* ecf_state, dgpu_picture_info* info) {
    if (E->prepared < 0) return DGPU_ERR_ARG;
    Pic* p = &E->pics[E->prepared];
    E->prepared = -1;
    int rc;
    // 17.-19. quantisation, inverse transform
    if (ecf_state) ecf = ecf_state + (size_t)(p->intra ? 0 : (p->is_b() ? 1 : 2)) * 3 * E->nb;
    rc = code_residue(*E, *p, ecf, true);
    if (rc) return rc;
    // 20.-21. reconstruction and clip
    if (!p->intra) {
        rc = motion_compensate(*E, *p, DGPU_ADD, true);
        if (rc) return rc;
    } else {
        StageTimer timer(*E, DGPU_STAGE_MC_ADD);
        Slot& s = slot_of(*E, *p);
        for (int c = 0; c < 3; ++c) {
            rc = dgpu_clip(s.data[c], E->w[c], E->h[c], E->w[c], comp_depth(*E, c), E->st);
            if (rc) return rc;
        }
    }
    p->up_valid = false;
    p->coded = true;
    if (info) *info = p->info;
    ++E->code;
    return 1;
}

int code_next_impl(Encoder* E, const float* ecf, const float* ecf_state, dgpu_picture_info* info) {
    const int rc = prepare_impl(E, nullptr);
    if (rc != 1) return rc;
    return finish_impl(E, ecf, ecf_state, info);
}

}  // namespace
}  // namespace dgpu

extern "C" size_t dgpu_encoder_item_bytes(void* enc, int pnum, int what, int comp) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E || comp < 0 || comp > 2) return 0;
    auto it = E->pics.find(pnum);
    if (it == E->pics.end() || !it->second.coded) return 0;
    const Pic& p = it->second;
    const bool inter = !p.intra || p.cut;
    switch (what) {
        case DGPU_ENC_RECON: return (size_t)E->w[comp] * E->h[comp] * 2;
        case DGPU_ENC_COEFF:
        case DGPU_ENC_QINDEX: return (size_t)E->pw[comp] * E->ph[comp] * 4;
        case DGPU_ENC_MV: return inter ? (size_t)p.refs.size() * E->nblocks * 4 : 0;
        case DGPU_ENC_MODE: return inter ? (size_t)E->nblocks : 0;
        case DGPU_ENC_DC: return inter ? (size_t)3 * E->nblocks * 2 : 0;
        case DGPU_ENC_SPLIT: return inter ? (size_t)E->nsb : 0;
        case DGPU_ENC_BANDS: return (size_t)E->nb * 3 * sizeof(int);
        case DGPU_ENC_CBSKIP: return (size_t)E->ncb_total;
        case DGPU_ENC_OUTPUT: return (size_t)E->w[comp] * E->h[comp] * sample_bytes(*E);
        default: return 0;
    }
}

extern "C" int dgpu_encoder_read(void* enc, int pnum, int what, int comp, void* dst, size_t bytes, int on_host) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E || !dst || on_host < 0 || on_host > 2) return DGPU_ERR_ARG;
    const size_t need = dgpu_encoder_item_bytes(enc, pnum, what, comp);
    if (need == 0 || bytes != need) return DGPU_ERR_ARG;
    if (on_host == 2 && what == DGPU_ENC_OUTPUT) return DGPU_ERR_ARG;  // staged through one buffer
    const Pic& p = E->pics[pnum];
    const Slot& s = E->slots[p.slot];
    if (what == DGPU_ENC_BANDS || what == DGPU_ENC_CBSKIP) {
        const void* src = what == DGPU_ENC_BANDS ? (const void*)&p.bands[(size_t)comp * E->nb * 3]
                                                 : (const void*)&p.cb_skip[(size_t)comp * E->ncb_total];
        if (on_host) {
            std::memcpy(dst, src, bytes);
            return DGPU_OK;
        }
        DGPU_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, E->st));
        DGPU_CHECK_CUDA(host_wait(E->st));
        return DGPU_OK;
    }
    const void* src = nullptr;
    if (what == DGPU_ENC_OUTPUT) {
        const int n = E->w[comp] * E->h[comp];
        const int off = 1 << (comp_depth(*E, comp) - 1);
        void* out = on_host ? E->stage : dst;
        const int grid = std::min((n + 255) / 256, 148 * 8);
        if (sample_bytes(*E) == 1)
            output_kernel<uint8_t><<<grid, 256, 0, E->st>>>(s.data[comp], n, off, static_cast<uint8_t*>(out));
        else
            output_kernel<uint16_t><<<grid, 256, 0, E->st>>>(s.data[comp], n, off, static_cast<uint16_t*>(out));
        DGPU_CHECK_LAUNCH();
        if (!on_host) return DGPU_OK;
        src = E->stage;
    } else {
        switch (what) {
            case DGPU_ENC_RECON: src = s.data[comp]; break;
            case DGPU_ENC_COEFF: src = s.coeff[comp]; break;
            case DGPU_ENC_QINDEX: src = s.qout[comp]; break;
            case DGPU_ENC_MV: src = s.mv; break;
            case DGPU_ENC_MODE: src = s.mode; break;
            case DGPU_ENC_DC: src = s.dc; break;
            case DGPU_ENC_SPLIT: src = s.split; break;
            default: return DGPU_ERR_ARG;
        }
    }
    DGPU_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, E->st));
    if (on_host == 1) DGPU_CHECK_CUDA(host_wait(E->st));
    return DGPU_OK;
}

// ---------------------------------------------------------------------------------------
// Stock-encoder coding with the host band coder, pipelined by picture kind
// ---------------------------------------------------------------------------------------
namespace dgpu {
namespace {

// One finished picture on its way through the host band coder.
struct CodedPicture {
    dgpu_picture_info info{};
    bool idx16 = false;            // indices staged as int16 (then the overflow flag)
    std::vector<int> bands;        // [3][nb][3] quantiser index, skip, estimated bits
    std::vector<uint8_t> cb_skip;  // [3][ncb_total]
    std::vector<uint8_t> data;     // coded subbands (dgpu_code_bands_host's layout)
    std::vector<int> band_bytes;   // [3][nb]
};

// Codes one picture's subbands from its page-locked indices and adapts its kind's factors.
int code_picture(const Encoder& E, CodedPicture& C, const uint8_t* stage, float* ecf_state) {
    const int nb = E.nb, depth = E.P.wlt_depth;
    const int intra[3] = {C.info.intra, C.info.intra, C.info.intra}, dep[3] = {depth, depth, depth};
    const void* q[3];
    size_t off = 0;
    for (int c = 0; c < 3; ++c) {
        q[c] = stage + off;
        off += (size_t)E.pw[c] * E.ph[c] * (C.idx16 ? 2 : 4);
    }
    // the narrowing's overflow flag: set only if the coefficient bound failed
    if (C.idx16 && *reinterpret_cast<const int*>(stage + align_up(off, 16))) return DGPU_ERR_CUDA;
    const int16_t* q16[3];
    const int32_t* q32[3];
    for (int c = 0; c < 3; ++c) {
        q16[c] = static_cast<const int16_t*>(q[c]);
        q32[c] = static_cast<const int32_t*>(q[c]);
    }
    std::vector<int> ncb3(6 * nb), qidx(3 * nb), skip(3 * nb), est(3 * nb);
    for (int c = 0; c < 3; ++c)
        for (int b = 0; b < nb; ++b) {
            ncb3[2 * (c * nb + b)] = E.ncb[2 * b];
            ncb3[2 * (c * nb + b) + 1] = E.ncb[2 * b + 1];
            qidx[c * nb + b] = C.bands[(size_t)(c * nb + b) * 3];
            skip[c * nb + b] = C.bands[(size_t)(c * nb + b) * 3 + 1];
            est[c * nb + b] = C.bands[(size_t)(c * nb + b) * 3 + 2];
        }
    C.band_bytes.assign(3 * nb, 0);
    size_t cap = C.data.size() ? C.data.size() : (size_t)E.pw[0] * E.ph[0] / 4 + 4096;
    for (;;) {
        C.data.resize(cap);
        const int rc =
            C.idx16 ? dgpu_code_bands_host16(3, intra, dep, q16, E.pw, E.ph, ncb3.data(), qidx.data(), skip.data(),
                                             C.cb_skip.data(), C.data.data(), cap, C.band_bytes.data())
                    : dgpu_code_bands_host(3, intra, dep, q32, E.pw, E.ph, ncb3.data(), qidx.data(), skip.data(),
                                           C.cb_skip.data(), C.data.data(), cap, C.band_bytes.data());
        if (rc == DGPU_OK) break;
        if (rc != DGPU_ERR_SIZE) return rc;
        size_t need = 0;
        for (int v : C.band_bytes) need += (size_t)v;
        if (need <= cap) return DGPU_ERR_SIZE;
        cap = need;
    }
    size_t used = 0;
    for (int v : C.band_bytes) used += (size_t)v;
    C.data.resize(used);
    for (int c = 0; c < 3; ++c) {
        const int rc = dgpu_entropy_update(depth, ecf_state, C.info.intra, C.info.is_b, c, skip.data() + c * nb,
                                           est.data() + c * nb, C.band_bytes.data() + c * nb);
        if (rc) return rc;
    }
    return DGPU_OK;
}

}  // namespace
}  // namespace dgpu

extern "C" int dgpu_encoder_code_adaptive(void* enc, float* ecf_state, int max_pictures, dgpu_picture_info* infos,
                                          uint8_t* out, size_t out_cap, size_t* out_bytes, int* band_bytes,
                                          size_t* d2h_bytes, int* npictures) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E || !ecf_state || max_pictures < 0 || !npictures || !out_bytes) return DGPU_ERR_ARG;
    if (E->failed) return E->failed;
    *npictures = 0;
    *out_bytes = 0;
    if (d2h_bytes) *d2h_bytes = 0;
    int dev = 0;
    DGPU_CHECK_CUDA(cudaGetDevice(&dev));
    const int nb = E->nb;
    std::vector<std::unique_ptr<CodedPicture>> done;
    std::future<int> last[3];
    int rc = DGPU_OK;
    size_t copied = 0;
    for (;;) {
        dgpu_picture_info nxt{};
        int r = dgpu_encoder_prepare_next(enc, &nxt);
        if (r <= 0) {
            rc = r;
            break;
        }
        if ((int)done.size() >= max_pictures) {
            rc = DGPU_ERR_SIZE;
            break;
        }
        // the stock encoder's factors and their updates are per picture kind: wait only for
        // the coding of the last picture of this one's kind
        const int kind = nxt.intra ? 0 : (nxt.is_b ? 1 : 2);
        if (last[kind].valid() && (r = last[kind].get()) != DGPU_OK) {
            rc = r;
            break;
        }
        auto C = std::make_unique<CodedPicture>();
        if ((r = dgpu_encoder_finish_next(enc, nullptr, ecf_state, &C->info)) < 0) {
            rc = r;
            break;
        }
        const int pn = C->info.pnum;
        const Pic& p = E->pics[pn];
        C->bands = p.bands;
        C->cb_skip = p.cb_skip;
        // indices and motion data into the kind's page-locked buffer, without waiting.  An
        // inter picture's indices are at most its largest |coefficient| (no DC prediction):
        // when that fits int16 they go as int16, followed by the narrowing's overflow flag;
        // an intra picture's (DC prediction residues) go as int32.
        const bool idx16 = !C->info.intra && p.coeff_max <= 32767;
        C->idx16 = idx16;
        size_t nq = 0;
        for (int c = 0; c < 3; ++c) nq += (size_t)E->pw[c] * E->ph[c];
        const size_t q16_off = align_up(nq * 2, 16);  // the flag's offset
        const int items[] = {DGPU_ENC_QINDEX, DGPU_ENC_QINDEX, DGPU_ENC_QINDEX, DGPU_ENC_MV,
                             DGPU_ENC_MODE, DGPU_ENC_DC, DGPU_ENC_SPLIT};
        size_t need = idx16 ? q16_off + 16 : 0;
        for (int k = idx16 ? 3 : 0; k < 7; ++k) need += dgpu_encoder_item_bytes(enc, pn, items[k], k < 3 ? k : 0);
        if (E->kind_stage_bytes[kind] < need) {
            if (E->kind_stage[kind]) cudaFreeHost(E->kind_stage[kind]);
            E->kind_stage[kind] = nullptr;
            E->kind_stage_bytes[kind] = 0;
            if (cudaHostAlloc(reinterpret_cast<void**>(&E->kind_stage[kind]), need, cudaHostAllocDefault) !=
                cudaSuccess) {
                cudaGetLastError();
                rc = DGPU_ERR_NOMEM;
                break;
            }
            E->kind_stage_bytes[kind] = need;
        }
        if (!E->kind_ev[kind] &&
            cudaEventCreateWithFlags(&E->kind_ev[kind], cudaEventDisableTiming | cudaEventBlockingSync) !=
                cudaSuccess) {
            cudaGetLastError();
            rc = DGPU_ERR_CUDA;
            break;
        }
        size_t off = 0;
        if (idx16) {
            if (E->q16_bytes < q16_off + 16) {
                if (E->q16) cudaFree(E->q16);
                E->q16 = nullptr;
                E->q16_bytes = 0;
                if (cudaMalloc(&E->q16, q16_off + 16) != cudaSuccess) {
                    cudaGetLastError();
                    rc = DGPU_ERR_NOMEM;
                    break;
                }
                E->q16_bytes = q16_off + 16;
            }
            const Slot& s = E->slots[p.slot];
            NarrowArgs A;
            for (int c = 0; c < 3; ++c) {
                A.src[c] = s.qout[c];
                A.n[c] = E->pw[c] * E->ph[c];
            }
            int16_t* d16 = static_cast<int16_t*>(E->q16);
            int* dflag = reinterpret_cast<int*>(static_cast<char*>(E->q16) + q16_off);
            if (cudaMemsetAsync(dflag, 0, sizeof(int), E->st) != cudaSuccess) {
                cudaGetLastError();
                rc = DGPU_ERR_CUDA;
                break;
            }
            narrow_kernel<<<(int)std::min<size_t>((nq + 255) / 256, 148 * 8), 256, 0, E->st>>>(A, d16, dflag);
            count_launch();
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(E->kind_stage[kind], d16, nq * 2, cudaMemcpyDeviceToHost, E->st) != cudaSuccess ||
                cudaMemcpyAsync(E->kind_stage[kind] + q16_off, dflag, sizeof(int), cudaMemcpyDeviceToHost, E->st) !=
                    cudaSuccess) {
                cudaGetLastError();
                rc = DGPU_ERR_CUDA;
                break;
            }
            off = q16_off + 16;
        }
        for (int k = idx16 ? 3 : 0; k < 7 && r >= 0; ++k) {
            const size_t n = dgpu_encoder_item_bytes(enc, pn, items[k], k < 3 ? k : 0);
            if (n == 0) continue;
            r = dgpu_encoder_read(enc, pn, items[k], k < 3 ? k : 0, E->kind_stage[kind] + off, n, 2);
            off += n;
        }
        if (r < 0) {
            rc = r;
            break;
        }
        copied += idx16 ? off - (q16_off + 16) + nq * 2 + sizeof(int) : off;
        if (cudaEventRecord(E->kind_ev[kind], E->st) != cudaSuccess) {
            cudaGetLastError();
            rc = DGPU_ERR_CUDA;
            break;
        }
        CodedPicture* cp = C.get();
        done.push_back(std::move(C));
        const uint8_t* stage = E->kind_stage[kind];
        const cudaEvent_t ev = E->kind_ev[kind];
        last[kind] = std::async(std::launch::async, [E, cp, stage, ev, ecf_state, dev]() -> int {
            try {
                if (cudaSetDevice(dev) != cudaSuccess || cudaEventSynchronize(ev) != cudaSuccess) {
                    cudaGetLastError();
                    return DGPU_ERR_CUDA;
                }
                return code_picture(*E, *cp, stage, ecf_state);
            } catch (const std::bad_alloc&) {
                return DGPU_ERR_NOMEM;
            }
        });
    }
    for (auto& f : last)
        if (f.valid()) {
            const int r = f.get();
            if (rc == DGPU_OK && r != DGPU_OK) rc = r;
        }
    // a failure leaves pictures finished but not coded: sticky until dgpu_encoder_reset
    if (rc < 0) return sticky(E, rc);
    size_t at = 0;
    for (const auto& C : done) at += C->data.size();
    E->adaptive_data.resize(at);
    at = 0;
    for (size_t i = 0; i < done.size(); ++i) {
        const CodedPicture& C = *done[i];
        if (infos) infos[i] = C.info;
        if (band_bytes) std::memcpy(band_bytes + i * 3 * nb, C.band_bytes.data(), sizeof(int) * 3 * nb);
        if (!C.data.empty()) std::memcpy(E->adaptive_data.data() + at, C.data.data(), C.data.size());
        at += C.data.size();
    }
    *npictures = (int)done.size();
    *out_bytes = at;
    if (d2h_bytes) *d2h_bytes = copied;
    if (!out) return DGPU_OK;
    if (at > out_cap) return DGPU_ERR_SIZE;
    if (at) std::memcpy(out, E->adaptive_data.data(), at);
    return DGPU_OK;
}

extern "C" int dgpu_encoder_adaptive_data(void* enc, uint8_t* out, size_t out_cap, size_t* out_bytes) {
    Encoder* E = static_cast<Encoder*>(enc);
    if (!E || !out_bytes) return DGPU_ERR_ARG;
    *out_bytes = E->adaptive_data.size();
    if (!out) return DGPU_OK;
    if (E->adaptive_data.size() > out_cap) return DGPU_ERR_SIZE;
    if (!E->adaptive_data.empty()) std::memcpy(out, E->adaptive_data.data(), E->adaptive_data.size());
    return DGPU_OK;
}

// ---------------------------------------------------------------------------------------
// Encoder groups: the motion estimation of several sequences in one batched launch
// ---------------------------------------------------------------------------------------
namespace dgpu {
namespace {

struct Group {
    std::vector<Encoder*> enc;
    cudaStream_t st = nullptr;   // owned
    cudaEvent_t ev = nullptr;    // ordering between the encoders' streams and st
    void* ws = nullptr;
    size_t ws_bytes = 0;
    int max_tasks = 0;
    int* d_counts = nullptr;
    int* h_counts = nullptr;     // pinned

    ~Group() {
        if (st) cudaStreamSynchronize(st);
        if (ws) cudaFree(ws);
        if (d_counts) cudaFree(d_counts);
        if (h_counts) cudaFreeHost(h_counts);
        if (ev) cudaEventDestroy(ev);
        if (st) cudaStreamDestroy(st);
    }
};

bool same_geometry(const Encoder& a, const Encoder& b) {
    return a.P.cformat == b.P.cformat && a.P.width == b.P.width && a.P.height == b.P.height && a.field == b.field &&
           a.P.luma_depth == b.P.luma_depth && a.bp.precision == b.bp.precision && a.bp.xblen == b.bp.xblen &&
           a.bp.yblen == b.bp.yblen && a.bp.xbsep == b.bp.xbsep && a.bp.ybsep == b.bp.ybsep;
}

// Workspace of one batch holding every member's largest estimation batch.
size_t group_ws_bytes(const std::vector<Encoder*>& enc, int* max_tasks) {
    int nt = 0, np = 0;
    for (Encoder* E : enc) {
        nt += E->me_max_tasks;
        np += std::min((int)E->slots.size(), 3 * E->me_max_tasks);
    }
    *max_tasks = nt;
    std::vector<int> r2(nt, 0);
    const Encoder& E0 = *enc[0];
    return dgpu_me_batch_workspace_bytes(E0.P.cformat, E0.P.width, E0.h[0], &E0.bp, np, nt, r2.data(), 3);
}

}  // namespace
}  // namespace dgpu

extern "C" size_t dgpu_encoder_group_device_bytes(void* const* encoders, int n) {
    if (!encoders || n < 1) return 0;
    std::vector<Encoder*> enc;
    for (int k = 0; k < n; ++k) {
        Encoder* E = static_cast<Encoder*>(encoders[k]);
        if (!E || !same_geometry(*E, *static_cast<Encoder*>(encoders[0]))) return 0;
        enc.push_back(E);
    }
    int nt = 0;
    const size_t ws = group_ws_bytes(enc, &nt);
    return ws ? align_up(ws, 256) + align_up(sizeof(int) * nt, 256) : 0;
}

extern "C" int dgpu_encoder_group_create(void* const* encoders, int n, void** out) {
    if (!encoders || n < 1 || !out) return DGPU_ERR_ARG;
    *out = nullptr;
    Group* G = new (std::nothrow) Group();
    if (!G) return DGPU_ERR_NOMEM;
    for (int k = 0; k < n; ++k) {
        Encoder* E = static_cast<Encoder*>(encoders[k]);
        bool dup = false;
        for (Encoder* e : G->enc) dup = dup || e == E;
        if (!E || dup || !same_geometry(*E, *static_cast<Encoder*>(encoders[0]))) {
            delete G;
            return DGPU_ERR_ARG;
        }
        G->enc.push_back(E);
    }
    G->ws_bytes = group_ws_bytes(G->enc, &G->max_tasks);
    if (G->ws_bytes == 0) {
        delete G;
        return DGPU_ERR_ARG;
    }
    if (cudaStreamCreateWithFlags(&G->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&G->ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&G->ws, G->ws_bytes) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&G->d_counts), sizeof(int) * G->max_tasks) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&G->h_counts), sizeof(int) * G->max_tasks) != cudaSuccess) {
        cudaGetLastError();
        delete G;
        return DGPU_ERR_NOMEM;
    }
    *out = G;
    return DGPU_OK;
}

extern "C" int dgpu_encoder_group_destroy(void* group) {
    Group* G = static_cast<Group*>(group);
    if (!G) return DGPU_ERR_ARG;
    delete G;
    return DGPU_OK;
}

namespace dgpu {
namespace {

// Estimates, for every listed encoder, each loaded and uncoded inter picture whose references
// are known, in one batched launch on st after the encoders' pending work; their streams then
// follow the estimation.  ev orders the streams.
int estimate_members(const std::vector<Encoder*>& enc, cudaStream_t st, cudaEvent_t ev, void* ws, size_t ws_bytes,
                     int* d_counts, int* h_counts, int* ntasks) {
    std::vector<MeTask> tasks;
    for (Encoder* E : enc) {
        if (E->last_read < 0) continue;
        // the loop's picture types are set one sub-group ahead of the coded picture, exactly
        // as dgpu_encoder_code_next sets them; untyped pictures get their likely references
        collect_me_tasks(*E, nullptr, E->me_max_tasks, tasks);
    }
    if (tasks.empty()) return DGPU_OK;
    // the estimation's stream follows every member's stream (their loads), and each member's
    // stream follows the estimation (the host waits for it below as well)
    for (Encoder* E : enc) {
        DGPU_CHECK_CUDA(cudaEventRecord(ev, E->st));
        DGPU_CHECK_CUDA(cudaStreamWaitEvent(st, ev, 0));
    }
    const int rc = run_me_tasks(tasks, st, ws, ws_bytes, d_counts, h_counts);
    if (rc) return rc;
    DGPU_CHECK_CUDA(cudaEventRecord(ev, st));
    for (Encoder* E : enc) DGPU_CHECK_CUDA(cudaStreamWaitEvent(E->st, ev, 0));
    if (ntasks) *ntasks = (int)tasks.size();
    return DGPU_OK;
}

// Page-locked task counts and an ordering event per host thread, for dgpu_encoders_estimate.
struct EstimateHostState {
    int* h_counts = nullptr;
    int cap = 0;
    cudaEvent_t ev = nullptr;
    ~EstimateHostState() {
        if (h_counts) cudaFreeHost(h_counts);
        if (ev) cudaEventDestroy(ev);
    }
};

}  // namespace
}  // namespace dgpu

extern "C" int dgpu_encoder_group_estimate(void* group, int* ntasks) {
    Group* G = static_cast<Group*>(group);
    if (ntasks) *ntasks = 0;
    if (!G) return DGPU_ERR_ARG;
    return estimate_members(G->enc, G->st, G->ev, G->ws, G->ws_bytes, G->d_counts, G->h_counts, ntasks);
}

extern "C" int dgpu_encoders_estimate(void* const* encoders, int n, void* workspace, size_t ws_bytes, void* stream,
                                      int* ntasks) {
    if (ntasks) *ntasks = 0;
    if (!encoders || n < 1 || !workspace) return DGPU_ERR_ARG;
    std::vector<Encoder*> enc;
    for (int k = 0; k < n; ++k) {
        Encoder* E = static_cast<Encoder*>(encoders[k]);
        bool dup = false;
        for (Encoder* e : enc) dup = dup || e == E;
        if (!E || dup || !same_geometry(*E, *static_cast<Encoder*>(encoders[0]))) return DGPU_ERR_ARG;
        enc.push_back(E);
    }
    int nt = 0;
    const size_t me_ws = group_ws_bytes(enc, &nt);
    if (me_ws == 0) return DGPU_ERR_ARG;
    const size_t need = align_up(me_ws, 256) + align_up(sizeof(int) * nt, 256);
    if (ws_bytes < need) return DGPU_ERR_NOMEM;
    thread_local EstimateHostState hs;
    if (hs.cap < nt) {
        if (hs.h_counts) cudaFreeHost(hs.h_counts);
        hs.h_counts = nullptr;
        hs.cap = 0;
        DGPU_CHECK_CUDA(cudaMallocHost(reinterpret_cast<void**>(&hs.h_counts), sizeof(int) * nt));
        hs.cap = nt;
    }
    if (!hs.ev) DGPU_CHECK_CUDA(cudaEventCreateWithFlags(&hs.ev, cudaEventDisableTiming));
    char* base = static_cast<char*>(workspace);
    int* d_counts = reinterpret_cast<int*>(base + align_up(me_ws, 256));
    return estimate_members(enc, as_stream(stream), hs.ev, workspace, me_ws, d_counts, hs.h_counts, ntasks);
}
