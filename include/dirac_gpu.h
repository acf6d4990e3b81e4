/*
 * dirac_gpu.h -- C ABI of the B200 (sm_100a) implementation of the Dirac research codec's
 * data-parallel coding hot path.
 *
 * Every entry point takes plain pointers and sizes.  Unless the name ends in _host, array
 * pointers are CUDA device pointers, `stream` is a cudaStream_t passed as void* (NULL =
 * the legacy default stream) and the call is asynchronous on that stream.  Entry points
 * return DGPU_OK (0) or a negative DGPU_ERR_* code; no C++ exception or CUDA error crosses
 * this boundary (the reference turns its DiracException into return codes at its own C API
 * the same way, libdirac_encoder/dirac_encoder.cpp:1074-1085).
 *
 * Sample conventions follow the reference: pictures are int16 (ValueType, 8-bit video is
 * stored as u8 - 128, libdirac_common/pic_io.cpp:388-399) and wavelet coefficients are int32
 * (CoeffType of the reference's plain-C build, libdirac_common/common.h:72-78).  Strides are
 * in elements.
 *
 * Scratch passed as NULL: the entry points that take a scratch or workspace pointer
 * (dgpu_wavelet_transform[_batch], dgpu_motion_estimate[_batch], dgpu_code_residue_batch,
 * dgpu_rect_lp_filter, dgpu_diag_lp_filter) then use a buffer the library owns, one per (device, stream), grown
 * with cudaMalloc on first use and on growth.  Calls on one stream are ordered by it, so they
 * may share that buffer; calls on the same stream issued from several host threads at once
 * race on it and must be serialised by the caller.  Calls on different streams use different
 * buffers.  An outgrown buffer is never freed while the process runs (another thread may
 * still hold it), so the library's scratch grows to at most twice the largest need per stream.
 * Callers that must not allocate pass their own scratch.
 */
#ifndef DIRAC_GPU_H
#define DIRAC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGPU_OK 0
#define DGPU_ERR_ARG (-1)     /* invalid argument (null pointer, bad enum, bad stride)   */
#define DGPU_ERR_SIZE (-2)    /* size outside what the reference's algorithm defines     */
#define DGPU_ERR_CUDA (-3)    /* a CUDA runtime call or kernel launch failed            */
#define DGPU_ERR_NOMEM (-4)   /* device or host allocation failed / scratch too small    */
#define DGPU_ERR_DEVICE (-5)  /* no usable sm_100 device                                 */

/* Filters: numbering of the reference's WltFilter (libdirac_common/common_types.h:61-71).
 * FIDELITY and any unknown value select DAUB9_7, as the reference's WaveletTransform
 * constructor does (libdirac_common/wavelet_utils.cpp:406-435). */
#define DGPU_DD9_7 0
#define DGPU_LEGALL5_3 1
#define DGPU_DD13_7 2
#define DGPU_HAAR0 3
#define DGPU_HAAR1 4
#define DGPU_FIDELITY 5
#define DGPU_DAUB9_7 6

/* Direction: numbering of the reference's Direction (libdirac_common/common.h:93). */
#define DGPU_FORWARD 0
#define DGPU_BACKWARD 1

/* Library version string; the compute capability (e.g. 100) of the current device, or
 * DGPU_ERR_DEVICE when it is not an sm_100 part; text of the last CUDA failure. */
const char* dgpu_version(void);
int dgpu_device_check(void);
const char* dgpu_last_error(void);

/* Running total of kernel launches issued by this library in this process. */
unsigned long long dgpu_launch_count(void);

/* How the library's host threads wait for the device where a call needs a result on the host
 * (the quantiser's round trips, motion-estimation error words, host reads): 0 (the default)
 * polls the stream (cudaStreamSynchronize under the default device flags), 1 sleeps on an
 * event created with cudaEventBlockingSync, 2 polls with cudaStreamQuery and yields the core
 * between polls.  Sleeping or yielding leaves the host cores to other threads when many
 * streams wait at once; polling wakes sooner, which a sequence coded alone, with two
 * quantiser round trips per picture, needs.  Process-wide; DGPU_ERR_ARG for other values.
 * No counterpart in the reference.
 *
 * The library's host worker pool (band coding, the quantiser's Lagrangian) has one worker
 * fewer than the hardware threads, at most 15, or DGPU_HOST_THREADS (1..256) workers when
 * that environment variable is set before the pool's first use. */
int dgpu_set_blocking_waits(int on);

/* Measures, on the current device, the rate of the integer block-difference operation
 * acc += |a - b| (counted as 3 operations: subtract, absolute value, add) on register-resident
 * data with every SM busy: the integer roofline the motion-estimation kernels' algorithmic
 * operation counts are compared with.  No counterpart in the reference.  Synchronous; about
 * 10 ms of GPU time. */
int dgpu_measure_int_rate(double* ops_per_second);

/* ---------------------------------------------------------------------------------------
 * Wavelet transform
 * Replaces WaveletTransform::Transform(Direction, PicArray&, CoeffArray&)
 * (libdirac_common/wavelet_utils.h:700-718, wavelet_utils.cpp:440-485).
 *
 * pic: h x w int16 picture component.  coeff: ch x cw int32 array whose sides are the
 * picture sides padded up to a multiple of 2^depth (Picture::InitWltData,
 * libdirac_common/picture.cpp:201-219).  FORWARD replicates the last column/row into the
 * padding and leaves coeff in the reference's Mallat layout (LL top-left, then HL, LH, HH
 * per level).  BACKWARD reads coeff (left unchanged, unlike the reference's in-place
 * synthesis, whose leftover contents no caller reads) and writes pic with the reference's
 * truncating int32 -> int16 cast.  Every level side (cw >> (depth-1), ch >> (depth-1)) must
 * be at least 6 for DD9_7/DD13_7, 4 for LEGALL5_3/DAUB9_7 and 2 for HAAR0/HAAR1.
 *
 * scratch: device memory of at least dgpu_dwt_scratch_bytes(cw, ch, depth) bytes holding the
 * intermediate low-pass bands, or NULL to let the library use its own buffer for the stream
 * (see "Scratch passed as NULL" above).
 * ------------------------------------------------------------------------------------- */
size_t dgpu_dwt_scratch_bytes(int cw, int ch, int depth);

int dgpu_wavelet_transform(int direction, int filter, int depth,
                           int16_t* pic, int w, int h, int pic_stride,
                           int32_t* coeff, int cw, int ch, int coeff_stride,
                           void* scratch, size_t scratch_bytes, void* stream);

/* Several components / pictures in one launch per level: n transforms described by
 * parallel arrays (each entry as in dgpu_wavelet_transform; all share `direction`).
 * scratch must hold the sum of dgpu_dwt_scratch_bytes over the entries (each entry's share
 * starting on a 256-byte boundary), or be NULL. */
int dgpu_wavelet_transform_batch(int direction, int n, const int* filter, const int* depth,
                                 int16_t* const* pic, const int* w, const int* h,
                                 const int* pic_stride, int32_t* const* coeff, const int* cw,
                                 const int* ch, const int* coeff_stride, void* scratch,
                                 size_t scratch_bytes, void* stream);

/* Host-buffer form of dgpu_wavelet_transform (the reference's calling convention: caller
 * memory in host RAM).  Copies in, transforms, copies out, synchronises. */
int dgpu_wavelet_transform_host(int direction, int filter, int depth,
                                int16_t* pic, int w, int h, int pic_stride,
                                int32_t* coeff, int cw, int ch, int coeff_stride);

/* Allocation-free form of dgpu_wavelet_transform, for callers that cannot allocate device
 * memory when they transform (a fully reserved device-memory budget, threads that must not
 * synchronise the device as cudaMalloc/cudaFree may, or an embedding allocator that owns
 * all device memory).  It has no counterpart in the reference, which always transforms in
 * host memory.  The low-pass intermediates live in one fixed device array of
 * DGPU_DWT_STATIC_SCRATCH_BYTES per GPU, held from library load to process exit; it fits
 * components with dgpu_dwt_scratch_bytes(cw, ch, depth) <= that size (any component up to
 * 1920 x 1088, i.e. HD luma); larger ones return DGPU_ERR_SIZE.  The first call on a device
 * looks the array's device address up (cudaGetSymbolAddress); make that first call before
 * any stream capture.  All calls on a device share the array: calls whose kernels overlap
 * on the GPU race and must be serialised by the caller.  No allocation of any kind. */
#define DGPU_DWT_STATIC_SCRATCH_BYTES (4u << 20)
int dgpu_wavelet_transform_static(int direction, int filter, int depth,
                                  int16_t* pic, int w, int h, int pic_stride,
                                  int32_t* coeff, int cw, int ch, int coeff_stride,
                                  void* stream);

/* ---------------------------------------------------------------------------------------
 * Half-pel upconversion
 * Replaces UpConverter::DoUpConverter (libdirac_common/upconvert.cpp:55-200), as called by
 * Picture::UpData (libdirac_common/picture.cpp:141-199) and EncPicture::UpOrigData
 * (libdirac_encoder/enc_picture.cpp:131-159).  pic: h x w int16; up: (2h) x (2w) int16,
 * up_stride even and up 4-byte aligned; samples clipped to [-2^(bit_depth-1),
 * 2^(bit_depth-1)-1].  w, h >= 8 (the reference's edge loops overlap below that).
 * ------------------------------------------------------------------------------------- */
int dgpu_upconvert(const int16_t* pic, int w, int h, int stride, int bit_depth, int16_t* up,
                   int up_stride, void* stream);
int dgpu_upconvert_batch(int n, const int16_t* const* pic, const int* w, const int* h,
                         const int* stride, const int* bit_depth, int16_t* const* up,
                         const int* up_stride, void* stream);

/* ---------------------------------------------------------------------------------------
 * 2x decimation (one level of the motion-estimation pyramid)
 * Replaces DownConverter::DoDownConvert (libdirac_motionest/downconvert.cpp:51-204) as
 * PixelMatcher::MakePicHierarchy uses it (libdirac_motionest/pixel_match.cpp:158-182):
 * out is (h/2) x (w/2); both output sides must be >= 12.
 * ------------------------------------------------------------------------------------- */
int dgpu_downconvert(const int16_t* pic, int w, int h, int stride, int16_t* out,
                     int out_stride, void* stream);
int dgpu_downconvert_batch(int n, const int16_t* const* pic, const int* w, const int* h,
                           const int* stride, int16_t* const* out, const int* out_stride,
                           void* stream);

/* Picture::ClipComponent (libdirac_common/picture.cpp:221-283): clamp to the sample range. */
int dgpu_clip(int16_t* pic, int w, int h, int stride, int bit_depth, void* stream);

/* ---------------------------------------------------------------------------------------
 * Centre-weighted median prefilter of one component
 * Replaces CWMFilterComponent (libdirac_encoder/prefilter.cpp:50-125), which the encoder
 * applies to each input picture's working data when the CWM prefilter is selected
 * (seq_compress.cpp:649-651, 725-726; the original data, used by motion estimation, stays
 * unfiltered).  in and out: h x w int16 (distinct buffers: the reference filters from a copy);
 * strength as EncoderParams::PrefilterStrength.  Rows 1 .. h-2 and columns 1 .. w-3 are
 * filtered (the reference's loop leaves the last two columns), the rest copied.
 * ------------------------------------------------------------------------------------- */
int dgpu_cwm_filter(const int16_t* in, int in_stride, int16_t* out, int out_stride, int w, int h,
                    int strength, void* stream);

/* RECTLP residue prefilter of one component, in place: replaces LPFilter
 * (libdirac_encoder/prefilter.cpp:141-306), which PictureCompressor::Prefilter applies to each
 * component before the forward transform when RECTLP is selected (picture_compress.cpp:
 * 340-355).  The 17 taps are designed on the host in double from qf and strength as the
 * reference does; rows, then columns, outputs clamped to [-128, 127] as in the reference.
 * scratch: device w x h int16, or NULL for the library's own buffer.  DGPU_ERR_SIZE below
 * 17 x 17 (the reference's edge loops need 17 samples). */
int dgpu_rect_lp_filter(int16_t* pic, int w, int h, int stride, float qf, int strength, int16_t* scratch,
                        void* stream);

/* DIAGLP residue prefilter of one component, in place: replaces DiagFilter
 * (libdirac_encoder/prefilter.cpp:535-588, DiagFilterBchkD / DiagFilterD :307-392), which
 * PictureCompressor::Prefilter applies to each component before the forward transform when
 * DIAGLP is selected (picture_compress.cpp:340-355).  A 13 x 13 two-dimensional filter whose
 * quadrant of taps comes from the reference's tables for the bandwidth the quality factor and
 * strength give (GetDiagLPFilter, :395-530), mixed with a unit impulse; outputs
 * (2^15 + sum) >> 16 as int16, source indices clamped to the component.  When that bandwidth
 * is above 0.9 the reference leaves the component as it is, and so does this call.  scratch:
 * device w x h int16, or NULL for the library's own buffer.  DGPU_ERR_SIZE below 7 x 7 (the
 * reference's edge loops need 7 samples). */
int dgpu_diag_lp_filter(int16_t* pic, int w, int h, int stride, float qf, int strength, int16_t* scratch,
                        void* stream);

/* ---------------------------------------------------------------------------------------
 * Overlapped-block motion compensation
 * Replaces MotionCompensator::CompensatePicture(const PicturePredParams&, AddOrSub,
 * const MvData&, Picture*, Picture*[2]) (libdirac_common/mot_comp.h, mot_comp.cpp:63-1239).
 *
 * Block parameters are the luma level-2 OLBParams in the form
 * PicturePredParams::SetBlockSizes keeps unchanged (lengths and separations multiples of 4,
 * sep <= len <= 2 sep; libdirac_common/common.cpp:207-330); chroma parameters are derived
 * from them by the chroma format as there.  Blocks = 4 x superblocks per direction.
 * Block data (MvData, libdirac_common/motion.h:219-300), row-major over blocks:
 *   mv1, mv2  int16 (x, y) per block, in units of the MV precision (mv2 may be NULL)
 *   mode      uint8 per block: PredMode INTRA 0, REF1_ONLY 1, REF2_ONLY 2, REF1AND2 3
 *   dc        int16 per block for Y, then U, then V (3 planes of blocks)
 *   split     uint8 per superblock: 0 whole superblock, 1 four sub-superblocks, 2 blocks
 * pic[3]: the picture's component planes, updated in place (add_or_sub 0 ADD, 1 SUBTRACT).
 * ref1up/ref2up[3]: the references' upconverted planes ((2h_c) x (2w_c), dense), as
 * produced by dgpu_upconvert; ref2up may be NULL for single-reference pictures.
 * clip_*_depth > 0 clamps the ADD result to that bit depth (Picture::Clip fused);
 * 0 leaves it unclipped.  dgpu_motion_compensate uses the default reference picture weights;
 * dgpu_motion_compensate_weighted takes the picture's (PicturePredParams::Ref1Weight,
 * Ref2Weight, PictureWeightsBits, 0..16 bits) and applies them as AdjustBlockByRefWeights
 * does (mot_comp.cpp:620-680) when they are not the defaults 1, 1, 1.
 * ------------------------------------------------------------------------------------- */
typedef struct {
    int precision; /* MVPrecisionType: 0 pel, 1 half, 2 quarter, 3 eighth */
    int xblen, yblen, xbsep, ybsep;
    int xnum_sb, ynum_sb;
} dgpu_block_params;

#define DGPU_ADD 0
#define DGPU_SUBTRACT 1

int dgpu_motion_compensate(int add_or_sub, int cformat, int w, int h, const dgpu_block_params* bp,
                           const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                           const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                           const int* pic_stride, const int16_t* const* ref1up,
                           const int16_t* const* ref2up, int clip_luma_depth,
                           int clip_chroma_depth, void* stream);
int dgpu_motion_compensate_weighted(int add_or_sub, int cformat, int w, int h, const dgpu_block_params* bp,
                                    const int16_t* mv1, const int16_t* mv2, const uint8_t* mode,
                                    const int16_t* dc, const uint8_t* split, int16_t* const* pic,
                                    const int* pic_stride, const int16_t* const* ref1up,
                                    const int16_t* const* ref2up, int clip_luma_depth, int clip_chroma_depth,
                                    int ref1_weight, int ref2_weight, int weight_bits, void* stream);

/* ---------------------------------------------------------------------------------------
 * Motion estimation of one picture
 * Replaces PictureCompressor::PixelME / SubPixelME / ModeDecisionME
 * (libdirac_encoder/picture_compress.cpp:76-300) and the classes they drive: PixelMatcher
 * (libdirac_motionest/pixel_match.cpp:59-380), MEData::SetLambdaMap
 * (libdirac_common/motion.cpp:128-196), SubpelRefine (me_subpel.cpp:65-176) and ModeDecider
 * (me_mode_decn.cpp:66-573).
 *
 * pic, ref1, ref2: the original (not reconstructed) component planes, dense (stride = width),
 * device memory; only luma is searched, all three feed the DC values.  nref 1 or 2.  stages:
 * 1 pel search over the pyramid, 2 adds the lambda map (lambda: the picture's ME lambda,
 * e.g. EncoderParams::L1MELambda) and sub-pel refinement, 3 adds mode decision and DC values.
 * MV precision (bp->precision) must be 1 (half), 2 (quarter) or 3 (eighth).
 * Outputs, device memory, blocks = 16 x superblocks, row-major:
 *   mv_out    int16 [nref][blocks][2]           cost_out  float [nref][blocks][3] (SAD, mvcost, total)
 *   mode_out  uint8 [blocks]    dc_out int16 [3][blocks]    split_out uint8 / sbcost_out float [superblocks]
 * The call synchronises the stream once (between stages 1 and 2, where the host computes the
 * lambda map's statistics as the reference does in long double) and at its end.
 * workspace: at least dgpu_me_workspace_bytes(...) bytes of device memory, or NULL for the
 * library's own buffer.  A wait that times out inside a kernel returns DGPU_ERR_CUDA.
 * ------------------------------------------------------------------------------------- */
int dgpu_me_depth(int w, int h);
size_t dgpu_me_workspace_bytes(int cformat, int w, int h, const dgpu_block_params* bp, int nref);

/* Batched form: ntasks pictures estimated in the same launches (a GOP's pictures, all the
 * same size, format and block parameters).  pics holds npics pictures' three planes
 * (pics[3*p + c]); task t estimates picture task_pic[t] against task_ref1[t] and, when
 * task_ref2[t] >= 0, task_ref2[t], with lambda task_lambda[t].  Each picture's pyramid and
 * (for references) upconverted luma are computed once for all tasks.  Outputs per task as in
 * dgpu_motion_estimate (arrays of per-task device pointers).  One synchronisation for all
 * lambda maps, one at the end. */
size_t dgpu_me_batch_workspace_bytes(int cformat, int w, int h, const dgpu_block_params* bp, int npics,
                                     int ntasks, const int* task_ref2, int stages);
int dgpu_motion_estimate_batch(int cformat, int w, int h, const dgpu_block_params* bp, int luma_depth,
                               int npics, const int16_t* const* pics, int ntasks, const int* task_pic,
                               const int* task_ref1, const int* task_ref2, const float* task_lambda,
                               int stages, int16_t* const* mv_out, float* const* cost_out,
                               uint8_t* const* mode_out, int16_t* const* dc_out, uint8_t* const* split_out,
                               float* const* sbcost_out, void* workspace, size_t ws_bytes, void* stream);
int dgpu_motion_estimate(int cformat, int w, int h, const dgpu_block_params* bp, int nref,
                         const int16_t* const* pic, const int16_t* const* ref1,
                         const int16_t* const* ref2, int luma_depth, float lambda, int stages,
                         int16_t* mv_out, float* cost_out, uint8_t* mode_out, int16_t* dc_out,
                         uint8_t* split_out, float* sbcost_out, void* workspace, size_t ws_bytes,
                         void* stream);

/* Device time of the motion-estimation kernels by class, for measurement: while enabled,
 * every estimation call times each class with CUDA events on its stream (one event pair per
 * launch, so profiled calls are slower).  kernel_ms / launches (NULL or DGPU_ME_NKERNELS
 * entries) receive the totals accumulated since the previous call, which are then cleared.
 * Classes: 0 resampling (pyramid downconversion and upconversion of the references),
 * 1 pel candidate lists (pel_lists_kernel), 2 pel wavefront, 3 sub-pel wavefront, 4 mode
 * decision's block pass, 5 mode-decision wavefront, 6 DC values. */
#define DGPU_ME_NKERNELS 7
int dgpu_me_profile(int enable, double* kernel_ms, int* launches);

/* Resident CTAs per SM (1..8, default 8) of the persistent motion-estimation wavefront
 * kernels (pel search, sub-pel refinement, mode decision), process-wide, read by later
 * estimation calls.  At 8 a wavefront launch occupies every SM's registers until it ends, so
 * work on other streams (another encoder's coding) waits for it; fewer leave room for that
 * work on every SM.  Results do not depend on it.  No counterpart in the reference. */
int dgpu_me_set_occupancy(int ctas_per_sm);

/* Units (blocks or superblocks) one warp of the pel and sub-pel wavefronts, or one CTA of the
 * mode-decision wavefront, takes before it exits, process-wide, read by later estimation
 * calls (0, the default: until the launch's units run out).  With a lifetime the grid grows
 * so that every unit is still taken, and CTAs leave their SMs every few units: kernels on
 * streams of higher priority (an encoder's coding while a group estimates) start within that
 * time instead of after the whole launch.  Results do not depend on it.  DGPU_ERR_ARG for a
 * negative count.  No counterpart in the reference. */
int dgpu_me_set_unit_lifetime(int units);

/* Failure-detection and ordering checks of the motion-estimation wavefronts.  No counterpart
 * in the reference, whose search is sequential.  Process-wide settings, read by every later
 * dgpu_motion_estimate[_batch] call (and the encoders' estimation) until changed; set them
 * only while no estimation runs.
 *   skip_unit >= 0: every pel-search wavefront launch leaves the completion flag of that unit
 *   (its position in the launch's wavefront order) unset, so the waits of its dependants run
 *   out and the call returns DGPU_ERR_CUDA, with the device context intact; -1: normal.
 *   spin_limit: polls before a wait gives up (0: the normal limit of about 2 s; larger values
 *   are clamped to it).
 *   audit_pel / audit_subpel / audit_mode: NULL, or zeroed device int arrays of 1 + the
 *   finest level's blocks (pel, sub-pel) or 1 + the superblocks (mode decision); the first
 *   task's wavefront records there, for each unit (row-major), the position at which it was
 *   decided (element 0 counts), so a caller can check every unit came after the neighbours
 *   the reference's raster order makes it depend on.
 *   ops: NULL, or a zeroed device array of three counters that accumulate the algorithmic
 *   integer operations of the pel search, the sub-pel refinement and mode decision: for every
 *   block difference the reference's search evaluates, 3 per pixel (subtract, absolute value,
 *   add) plus the sub-pel interpolation (0 half-pel, 4 quarter-pel, 8 eighth-pel per pixel);
 *   bi-prediction differences 5 + 2 x interpolation, intra costs 4 per pixel.  Counting adds an
 *   atomic per evaluation: use it in a separate pass, not a timed one. */
int dgpu_debug_wavefront(int skip_unit, long long spin_limit, int* audit_pel, int* audit_subpel,
                         int* audit_mode, unsigned long long* ops);

/* ---------------------------------------------------------------------------------------
 * Quantiser selection and quantisation of transformed components
 * Replaces PictureCompressor::SelectQuantisers / SelectMultiQuants with QuantChooser
 * (libdirac_encoder/picture_compress.cpp:603-709, quant_chooser.cpp:62-362) and the
 * quantise-and-reconstruct arithmetic of CompCompressor::Compress and the band coders
 * (comp_compress.cpp:64-156, band_codec_template.h:53-174, 470-557, band_codec.cpp:81-96).
 *
 * n components per call (up to 48).  coeff[c]: device, dense cw[c] x ch[c] int32 in the
 * Mallat layout (the forward transform's output); reconstructed in place.  Per component:
 * intra flag, transform depth, lambda (the component's quantiser lambda,
 * PictureCompressor::GetCompLambda).  Per band, for all components concatenated in band-list
 * order (band b of component c at index sum of earlier components' 3*depth+1, plus b-1):
 * band_wt (CoeffArray::SetBandWeights, as float), band_ecf (EntropyCorrector::Factor) and
 * band_ncb (code blocks x, y: EncoderParams::SetUsualCodeBlocks / SetupCodeBlocks) are host
 * inputs; band_qidx, band_skip, band_bits (estimated bits) are host outputs, and cb_skip
 * (host, all code blocks concatenated in raster order) receives the code-block skip flags.
 * qout[c] (device, optional, same layout as coeff) receives the signed quantised indices (the
 * intra DC band holds its prediction residues' indices).  The call synchronises the stream:
 * the Lagrangian choice runs on the host in double precision like the reference's.
 * ------------------------------------------------------------------------------------- */
int dgpu_quant_factor4(int q);

/* Host-only helpers (no GPU use) for the inputs above: CoeffArray::SetBandWeights
 * (libdirac_common/wavelet_utils.cpp:192-395; cpd = EncoderParams::CPD(), cpd_scale as
 * PictureCompressor::CodeResidue computes it) and the code-block grid of
 * EncoderParams::SetUsualCodeBlocks (common.cpp:488-510; luma size, as the reference uses it
 * for every component). */
int dgpu_band_weights(int filter, int depth, int cw, int ch, int comp, int cformat, float cpd,
                      float cpd_scale, int field_coding, double* out);
int dgpu_code_blocks(int depth, int luma_w, int luma_h, int spatial_partition, int* ncb);
/* Device workspace bytes one dgpu_code_residue_batch call with these components needs
 * (0 on invalid arguments). */
size_t dgpu_code_residue_workspace_bytes(int n, const int* intra, const int* depth, const int* cw,
                                         const int* ch, const int* band_ncb);
int dgpu_code_residue_batch(int n, const int* intra, const int* depth, int32_t* const* coeff,
                            const int* cw, const int* ch, const float* lambda, const float* band_wt,
                            const float* band_ecf, const int* band_ncb, int* band_qidx, int* band_skip,
                            int* band_bits, uint8_t* cb_skip, int32_t* const* qout, void* workspace,
                            size_t ws_bytes, void* stream);

/* ---------------------------------------------------------------------------------------
 * Dequantisation of entropy-decoded components (the decoder's side of the residue coding).
 * Replaces the arithmetic the band decoders apply after decoding each magnitude and sign:
 * GenericBandCodec::DecodeVal with the band's quantiser (band_codec_template.h:231-270,
 * 330-356), ClearBlock for skipped code blocks (:488-496), the intra DC band's prediction
 * from reconstructed neighbours (GenericIntraDCBandCodec, :500-557) and
 * CompDecompressor::SetToVal for skipped bands (libdirac_decoder/comp_decompress.cpp:64-163).
 * A host binding makes DecodeVal store the signed index instead of the dequantised value.
 *
 * n components.  qindex[c] (device, dense cw[c] x ch[c] int32, Mallat layout): signed
 * quantised indices, the intra DC band holding its prediction residues' indices (the layout
 * dgpu_code_residue_batch writes to qout); coeff[c] (device, same layout) receives the
 * coefficients and may equal qindex[c] (in place).  Per band, components concatenated in
 * band-list order as for dgpu_code_residue_batch: band_ncb, band_qidx, band_skip (host);
 * cb_skip (DEVICE): the code-block skip flags of every band in that order.  Asynchronous on
 * the stream, no workspace, no synchronisation.  DGPU_ERR_ARG (nothing launched) when a
 * coded band's quantiser index is outside 0..119, as the reference decoder refuses it.
 * ------------------------------------------------------------------------------------- */
int dgpu_dequantise_batch(int n, const int* intra, const int* depth, const int32_t* const* qindex,
                          int32_t* const* coeff, const int* cw, const int* ch, const int* band_ncb,
                          const int* band_qidx, const int* band_skip, const uint8_t* cb_skip, void* stream);
/* As dgpu_dequantise_batch, over int16 index arrays (same layout); coeff[c] must not overlap
 * qindex[c] (no in-place form). */
int dgpu_dequantise_batch16(int n, const int* intra, const int* depth, const int16_t* const* qindex,
                            int32_t* const* coeff, const int* cw, const int* ch, const int* band_ncb,
                            const int* band_qidx, const int* band_skip, const uint8_t* cb_skip, void* stream);

/* ---------------------------------------------------------------------------------------
 * Sequence encoder: the data-parallel part of the reference's frame-coding loop
 * SequenceCompressor::CompressNextPicture (libdirac_encoder/seq_compress.cpp:194-499) with
 * FrameSequenceCompressor's GOP structure (seq_compress.cpp:151-192, 563-686) and the
 * PictureCompressor steps it drives (picture_compress.cpp:76-580): motion estimation on
 * the original pictures, intra-block analysis, P-only sub-group switch and cut detection,
 * motion compensation against the reconstructed references, forward transform, quantiser
 * choice and quantisation, inverse transform, reconstruction and clipping.  Everything stays
 * resident on the device; the host keeps the GOP state machine and the lambdas.
 *
 * What stays with the caller (serial host code in the reference): the arithmetic coding of
 * the coefficients and motion data, and therefore the adaptation of the entropy-correction
 * factors (EntropyCorrector::Update, common.cpp:134-151), which dgpu_encoder_code_next
 * takes as an input (NULL: the initial factors of EntropyCorrector::Init,
 * common.cpp:79-131).  Not supported: rate control (trate), prefilters, lossless coding,
 * num_l1 < 0.
 *
 * Field coding (field_coding = 1; FieldSequenceCompressor, seq_compress.cpp:697-892): each
 * dgpu_encoder_load takes an interlaced frame and makes two pictures of half its height, the
 * fields (StreamFieldInput::ReadFieldComponent, pic_io.cpp:464-530: the first field the even
 * rows when top_field_first, else the odd ones), numbered 2n and 2n + 1; their types,
 * references and coding order follow the field GOP, and every result is per field.  The frame
 * height must be a multiple of 4 for 4:2:0 (of 2 otherwise).
 *
 * Use: dgpu_encoder_create; dgpu_encoder_load for each picture in display order;
 * dgpu_encoder_code_next until it returns 0 (it needs the same look-ahead as the reference:
 * 2 * l1_sep pictures, or dgpu_encoder_end_sequence); dgpu_encoder_read for results.  A
 * picture's results stay readable until its slot is reused by a later load (never, when
 * max_pictures >= the sequence length).  A handle is not thread-safe; different handles
 * may run on different streams concurrently.
 * ------------------------------------------------------------------------------------- */
typedef struct {
    int cformat;                  /* ChromaFormat: 0 4:4:4, 1 4:2:2, 2 4:2:0 */
    int width, height;            /* luma picture size */
    int luma_depth, chroma_depth; /* bits per sample, 8..14 */
    float qf;                     /* quality factor (EncoderParams::Qf) */
    int l1_sep, num_l1;           /* GOP: L1 separation and L1 pictures per GOP (0: I only) */
    float cpd;                    /* perceptual weighting, cycles per degree */
    int xblen, yblen, xbsep, ybsep; /* luma OBMC block length and separation */
    int mv_precision;             /* 1 half, 2 quarter, 3 eighth pel */
    int intra_filter, inter_filter, wlt_depth; /* WltFilter numbering, transform depth */
    int field_coding;             /* 1: interlaced frames coded as two field pictures each
                                     (FieldSequenceCompressor); height is the frame's */
    int top_field_first;          /* with field_coding: the first field holds the even rows */
} dgpu_encoder_params;

typedef struct {
    int pnum;         /* picture (display) number */
    int coded_num;    /* position in coding order */
    int intra;        /* 1: coded intra (I picture or a detected cut) */
    int is_ref;       /* 1: reference picture */
    int cut;          /* 1: an inter picture re-coded as intra by cut detection */
    int num_refs, ref1, ref2;  /* references (-1 when absent) */
    int is_b;         /* PictureParams::IsBPicture */
    int filter;       /* transform filter used */
    double intra_ratio;   /* MEData::IntraBlockRatio (inter pictures) */
    double cpd_scale;     /* perceptual-weight scale used for the band weights */
    float lambda[3];      /* quantiser lambdas (PictureCompressor::GetCompLambda) */
} dgpu_picture_info;

/* dgpu_encoder_read items; comp selects the component where it applies */
#define DGPU_ENC_RECON 0    /* int16 [h][w] reconstructed component (codec samples) */
#define DGPU_ENC_COEFF 1    /* int32 [ch][cw] reconstructed coefficients (padded size) */
#define DGPU_ENC_QINDEX 2   /* int32 [ch][cw] signed quantised indices */
#define DGPU_ENC_MV 3       /* int16 [num_refs][blocks][2] motion vectors */
#define DGPU_ENC_MODE 4     /* uint8 [blocks] prediction modes (0 intra, 1 ref1, 2 ref2, 3 bi) */
#define DGPU_ENC_DC 5       /* int16 [3][blocks] intra-block DC values */
#define DGPU_ENC_SPLIT 6    /* uint8 [superblocks] superblock splitting levels */
#define DGPU_ENC_BANDS 7    /* int32 [3*depth+1][3] per band: quantiser index, skip, estimated bits */
#define DGPU_ENC_CBSKIP 8   /* uint8 code-block skip flags of all bands, band-list order */
#define DGPU_ENC_OUTPUT 9   /* uint8 (depth 8) / uint16 [h][w] output samples: recon + 2^(d-1) */

/* stages timed by dgpu_encoder_profile */
#define DGPU_STAGE_LOAD 0
#define DGPU_STAGE_ME 1
#define DGPU_STAGE_MC_SUBTRACT 2
#define DGPU_STAGE_DWT_FORWARD 3
#define DGPU_STAGE_QUANT 4
#define DGPU_STAGE_DWT_INVERSE 5
#define DGPU_STAGE_MC_ADD 6   /* motion compensation ADD with the clip, or the clip alone */
#define DGPU_STAGE_UPCONVERT 7
#define DGPU_ENC_NSTAGES 8

/* Device bytes dgpu_encoder_create would allocate for these parameters (0 if they are
 * invalid); no GPU use, so a scheduler can admit sequences against a memory budget. */
size_t dgpu_encoder_device_bytes(const dgpu_encoder_params* params, int max_pictures);
int dgpu_encoder_create(const dgpu_encoder_params* params, int max_pictures, void* stream, void** encoder);
int dgpu_encoder_destroy(void* encoder);
/* Forgets every picture and the GOP state (a new sequence), keeping the device memory. */
int dgpu_encoder_reset(void* encoder);
/* Stage timing with CUDA events on the encoder's stream (each stage waits for its end event,
 * so profiled runs are slower).  Copies the accumulated milliseconds and call counts per
 * stage (DGPU_STAGE_*) to stage_ms / stage_calls when not NULL, clears them, and turns
 * profiling on or off. */
int dgpu_encoder_profile(void* encoder, int enable, double* stage_ms, int* stage_calls);
/* Loads the next picture in display order: three dense planes of unsigned samples (uint8 for
 * depth 8, uint16 otherwise), in host memory (on_host = 1) or device memory (0). */
int dgpu_encoder_load(void* encoder, const void* const* planes, int on_host);
int dgpu_encoder_end_sequence(void* encoder);
/* Codes the next picture in coding order.  ecf: NULL, or [3][3*depth+1] entropy-correction
 * factors for this picture (the caller's EntropyCorrector::Factor values).  Returns 1 and
 * fills info when a picture was coded, 0 when more input (or nothing) remains.
 * A failure part-way through a picture (this call, _adaptive, prepare_next or finish_next)
 * leaves that picture half coded; it is sticky: every later coding call of the encoder
 * returns the same error code until dgpu_encoder_reset. */
int dgpu_encoder_code_next(void* encoder, const float* ecf, dgpu_picture_info* info);
/* As dgpu_encoder_code_next, with the caller's whole EntropyCorrector state (the
 * [3][3][3*depth+1] layout of dgpu_entropy_init): the encoder takes the picture's factors
 * from it once the picture's kind (intra, B, other inter) is final, cut detection included,
 * as the reference's quantiser choice does.  With the state adapted after each coded picture
 * (dgpu_code_bands_host's byte counts, dgpu_entropy_update) the choices are the stock
 * reference encoder's. */
int dgpu_encoder_code_next_adaptive(void* encoder, const float* ecf_state, dgpu_picture_info* info);
/* dgpu_encoder_code_next in two halves, so that a caller can arithmetic-code picture n on the
 * host while the device works on picture n + 1.  prepare_next runs what does not depend on
 * the entropy-correction factors (picture types, motion estimation, intra analysis, the
 * P-only switch and cut detection, motion compensation SUBTRACT, the forward transform) and
 * returns 1 with the picture's info (its kind final; lambdas and cpd scale follow at finish),
 * 0 when more input is needed; calling it again before finish_next returns the same picture.
 * finish_next completes it with ecf (as dgpu_encoder_code_next) or, when ecf_state is not
 * NULL, the kind's factors from that state (as dgpu_encoder_code_next_adaptive); it returns 1
 * and the final info, DGPU_ERR_ARG when no picture is prepared. */
int dgpu_encoder_prepare_next(void* encoder, dgpu_picture_info* info);
int dgpu_encoder_finish_next(void* encoder, const float* ecf, const float* ecf_state, dgpu_picture_info* info);
size_t dgpu_encoder_item_bytes(void* encoder, int pnum, int what, int comp);
/* Copies one result of a coded picture to dst; bytes must equal dgpu_encoder_item_bytes.
 * on_host = 0: dst is device memory, the copy queued on the encoder's stream.  1: host
 * memory, the encoder's stream synchronised.  2: page-locked host memory, the copy queued on
 * the encoder's stream and not waited for: the data is there once that stream has reached an
 * event the caller records after the call (DGPU_ENC_BANDS and DGPU_ENC_CBSKIP, kept on the
 * host, are copied at once; DGPU_ENC_OUTPUT, staged through one buffer, is refused). */
int dgpu_encoder_read(void* encoder, int pnum, int what, int comp, void* dst, size_t bytes, int on_host);

/* ---------------------------------------------------------------------------------------
 * Heterogeneous picture batch (batched form): many pictures of different sizes, chroma
 * formats, bit depths, filters and depths coded together, each exactly as
 * PictureCompressor codes one picture once its motion data is known
 * (libdirac_encoder/picture_compress.cpp:92-180, 418-531): motion compensation SUBTRACT
 * against the upconverted references (Picture::UpData), forward transform, quantiser choice
 * with quantisation and reconstruction (CodeResidue), inverse transform, motion
 * compensation ADD with the clip (inter) or the clip (intra).
 *
 * Per picture: the coding parameters below; for inter pictures the references' planes
 * (codec samples, dense, device memory; distinct planes are upconverted once per run) and
 * the motion data in the layout of dgpu_motion_compensate.  The batch keeps the given
 * device pointers, which must stay valid while it lives.  The lambdas, band weights and
 * initial entropy-correction factors are the encoder's (GetCompLambda with the given intra
 * ratio and B flag; CodeResidue's perceptual scale; EntropyCorrector::Init).
 *
 * dgpu_batch_planes gives picture k's three device planes: the caller writes the picture's
 * codec samples there (or loads them with dgpu_batch_load) before a run and reads the
 * reconstruction after it.  dgpu_batch_run
 * codes every picture: on its first call it tunes the motion-compensation tile shape
 * (keeping the planes' contents) and captures the device work before and after the
 * quantiser choice in two CUDA graphs, which later calls replay; the quantiser choice
 * synchronises the stream (host Lagrangian, as the reference).  On return the band results
 * are readable with dgpu_batch_read (DGPU_ENC_BANDS / CBSKIP); the reconstruction
 * (DGPU_ENC_RECON), coefficients and quantised indices are complete once the stream reaches
 * the end of the run.  The first call must not be made during a stream capture.  A batch is
 * not thread-safe; different batches may run on different threads and streams.
 * ------------------------------------------------------------------------------------- */
typedef struct {
    int cformat, width, height;   /* ChromaFormat and luma size */
    int luma_depth, chroma_depth; /* bits per sample, 8..14 */
    int filter, wlt_depth;        /* WltFilter and transform depth */
    int intra;                    /* 1: intra picture */
    int is_b;                     /* inter: PictureParams::IsBPicture (quantiser lambda) */
    float qf, cpd;                /* quality factor, perceptual cycles per degree */
    double intra_ratio;           /* inter: MEData::IntraBlockRatio of the motion data */
    dgpu_block_params bp;         /* inter: block parameters */
} dgpu_batch_picture;

typedef struct {
    const int16_t* ref1[3];       /* first reference's planes */
    const int16_t* ref2[3];       /* second reference's planes, or NULLs */
    const int16_t* mv1;
    const int16_t* mv2;           /* NULL with one reference */
    const uint8_t* mode;
    const int16_t* dc;
    const uint8_t* split;
} dgpu_batch_motion;

/* motion: n entries (read for inter pictures only), or NULL when every picture is intra */
size_t dgpu_batch_device_bytes(int n, const dgpu_batch_picture* pics, const dgpu_batch_motion* motion);
int dgpu_batch_create(int n, const dgpu_batch_picture* pics, const dgpu_batch_motion* motion, void* stream,
                      void** batch);
int dgpu_batch_destroy(void* batch);
int dgpu_batch_planes(void* batch, int k, int16_t** planes);
/* Copies picture k's three planes (int16 codec samples, dense) into the batch, from host
 * (on_host = 1; page-locked memory keeps the copy asynchronous) or device memory. */
int dgpu_batch_load(void* batch, int k, const int16_t* const* planes, int on_host);
int dgpu_batch_run(void* batch);
/* One run timed by stage with CUDA events on the batch's stream (synchronises): ms[0] the
 * upconversions, motion compensation SUBTRACT and forward transforms, ms[1] the quantiser
 * choice with quantisation (host Lagrangian included), ms[2] the inverse transforms and
 * motion compensation ADD / clips. */
int dgpu_batch_stage_times(void* batch, float* ms);
size_t dgpu_batch_item_bytes(void* batch, int k, int what, int comp);
int dgpu_batch_read(void* batch, int k, int what, int comp, void* dst, size_t bytes, int on_host);


/* ---------------------------------------------------------------------------------------
 * Encoder groups (batched form): the motion estimation of several sequences in one launch.
 * Replaces nothing in the reference, which codes one sequence per SequenceCompressor; each
 * member's results are those of PictureCompressor::PixelME / SubPixelME / ModeDecisionME
 * (libdirac_encoder/picture_compress.cpp:180-298) for the same picture and references.
 *
 * Members must share picture size, chroma format, luma depth and block parameters.
 * dgpu_encoder_group_estimate estimates, for every member, each loaded and uncoded inter
 * picture whose references are known (a full sub-group behind the last loaded picture, or
 * any after dgpu_encoder_end_sequence) in one batched launch on the group's own stream, after
 * the members' pending work; the members' later dgpu_encoder_code_next calls reuse those
 * estimates (pictures whose references change, e.g. by cut detection, are re-estimated by
 * their encoder).  *ntasks receives the number of picture estimates made.  The call
 * synchronises with the estimation; no member may be used by another thread meanwhile.
 * The group holds a workspace for every member's largest estimation batch.
 * ------------------------------------------------------------------------------------- */
size_t dgpu_encoder_group_device_bytes(void* const* encoders, int n);
int dgpu_encoder_group_create(void* const* encoders, int n, void** group);
int dgpu_encoder_group_destroy(void* group);
int dgpu_encoder_group_estimate(void* group, int* ntasks);
/* The same estimation for a set of encoders chosen per call (e.g. the live streams of one
 * picture format a serving loop has on the GPU at that moment), with a workspace the caller
 * holds: at least dgpu_encoder_group_device_bytes(encoders, n) bytes of device memory.  Runs
 * on `stream` after the encoders' pending work; their streams follow it.  Synchronises with
 * the estimation; none of the encoders may be used by another thread meanwhile. */
int dgpu_encoders_estimate(void* const* encoders, int n, void* workspace, size_t ws_bytes, void* stream,
                           int* ntasks);

/* Codes every picture the encoder has input for as the stock reference encoder does: each
 * picture's subbands arithmetic-coded on the host (dgpu_code_bands_host) and its kind's
 * entropy-correction factors in ecf_state (dgpu_entropy_init) adapted from the coded bytes
 * (dgpu_entropy_update) before the next picture of that kind is quantised
 * (SequenceCompressor::CompressNextPicture, seq_compress.cpp:194-499; EntropyCorrector,
 * common.cpp:57-151).  The reference's factors and their updates are per picture kind
 * (intra, B, other inter), so a picture waits only for the host coding of the last picture of
 * its kind: the coding runs on host threads while the pictures after it are prepared and
 * finished on the device, their indices and motion data copied to page-locked memory without
 * a wait.  An inter picture whose largest |coefficient| fits 16 bits (so does every index:
 * no DC prediction) has its indices narrowed to int16 on the device and copied at half the
 * bytes (dgpu_code_bands_host16); intra pictures' go as int32.  The results equal a serial
 * loop of dgpu_encoder_code_next_adaptive and
 * dgpu_code_bands_host.  At most max_pictures pictures (DGPU_ERR_SIZE beyond); per picture in
 * coding order: infos (optional), band_bytes (optional, [3][3*depth+1] as
 * dgpu_code_bands_host), its coded data in out (optional); out_bytes receives the data's total
 * length.  The encoder keeps the data until its next such call: when out is smaller the call
 * returns DGPU_ERR_SIZE after coding every picture, and dgpu_encoder_adaptive_data copies the
 * data once the caller has room.  d2h_bytes (optional): the device-to-host bytes copied
 * (indices and motion data); npictures: the count.  A failure is sticky, as for
 * dgpu_encoder_code_next. */
int dgpu_encoder_code_adaptive(void* encoder, float* ecf_state, int max_pictures, dgpu_picture_info* infos,
                               uint8_t* out, size_t out_cap, size_t* out_bytes, int* band_bytes,
                               size_t* d2h_bytes, int* npictures);
int dgpu_encoder_adaptive_data(void* encoder, uint8_t* out, size_t out_cap, size_t* out_bytes);

/* ---------------------------------------------------------------------------------------
 * Arithmetic coding of quantised subbands on the host, and entropy-correction factors.
 * dgpu_code_bands_host replaces the entropy coding of the reference's band coders
 * (CompCompressor::Compress, libdirac_encoder/comp_compress.cpp:64-140; GenericBandCodec /
 * IntraDCBandCodec, libdirac_common/band_codec_template.h:24-200, band_codec.cpp:81-96;
 * ArithCodecBase, arith_codec.h:65-360, arith_codec.cpp:40-120): the same bytes, from the
 * signed quantised indices instead of the coefficients.  No GPU use; the bands are coded in
 * parallel on the library's host threads.
 *
 * n components; qindex[c] (HOST, dense cw[c] x ch[c] int32): the signed quantised indices
 * as dgpu_code_residue_batch writes them (DGPU_ENC_QINDEX; the intra DC band its prediction
 * residues' indices).  Per band, components concatenated in band-list order: band_ncb,
 * band_qidx, band_skip (as for dgpu_code_residue_batch); cb_skip: the code-block skip flags
 * (host, as it writes them).  out (out_cap bytes) receives every coded band's data (the bytes
 * the reference's SubbandByteIO carries after its header), component by component, each
 * component's bands from the DC band down (the reference's coding order); band_bytes[g] is
 * band g's length (0 when skipped).  DGPU_ERR_SIZE when out is too small (band_bytes is still
 * filled, so a caller can size the buffer).
 *
 * EntropyCorrector (libdirac_common/common.cpp:57-151): state holds [3][3][3*depth+1] floats
 * (picture kind: intra, B, other inter; component; band).  dgpu_entropy_factors gives the
 * [3][3*depth+1] factors dgpu_encoder_code_next takes for a picture; dgpu_entropy_update
 * applies one coded component's bands (EntropyCorrector::Update with the quantiser's estimated
 * bits, DGPU_ENC_BANDS, and 8 x the coded bytes).
 * ------------------------------------------------------------------------------------- */
int dgpu_code_bands_host(int n, const int* intra, const int* depth, const int32_t* const* qindex,
                         const int* cw, const int* ch, const int* band_ncb, const int* band_qidx,
                         const int* band_skip, const uint8_t* cb_skip, uint8_t* out, size_t out_cap,
                         int* band_bytes);
/* As dgpu_code_bands_host over int16 index arrays (same layout, indices that fit 16 bits):
 * the same bytes, half the index bytes read. */
int dgpu_code_bands_host16(int n, const int* intra, const int* depth, const int16_t* const* qindex,
                           const int* cw, const int* ch, const int* band_ncb, const int* band_qidx,
                           const int* band_skip, const uint8_t* cb_skip, uint8_t* out, size_t out_cap,
                           int* band_bytes);
/* The variable-length form of the band coders (-use_vlc: BandVLC / IntraDCBandVLC over
 * ArithCodecToVLCAdapter, libdirac_common/band_vlc.cpp:49-100): the same symbols as plain
 * bits, each band's data padded to a byte.  band_bits (optional) receives each band's exact
 * bit count (the reference's EntropyCorrector update after a VLC band counts its whole bytes,
 * 8 * (band_bits / 8)). */
int dgpu_code_bands_vlc_host(int n, const int* intra, const int* depth, const int32_t* const* qindex,
                             const int* cw, const int* ch, const int* band_ncb, const int* band_qidx,
                             const int* band_skip, const uint8_t* cb_skip, uint8_t* out, size_t out_cap,
                             int* band_bytes, long long* band_bits);
/* The variable-length form on the device: the same bytes as dgpu_code_bands_vlc_host from
 * device-resident indices (qindex[c] device, dense cw[c] x ch[c] int32); band_ncb,
 * band_skip and cb_skip are host arrays as there, out device memory, 4-byte aligned, holding
 * the data rounded up to 4 bytes (DGPU_ERR_SIZE otherwise, band_bytes filled).  One pass sums
 * each code block's code lengths, a second places every coefficient's code at its offset
 * (the codes are independent).  band_bytes / band_bits (host) receive the bands' byte and
 * exact bit counts; synchronises the stream between the passes (the sizes come back to the
 * host), the writes then queued on it.  scratch: NULL or at least 64 bytes per code block
 * plus 512. */
int dgpu_code_bands_vlc(int n, const int* depth, const int32_t* const* qindex, const int* cw, const int* ch,
                        const int* band_ncb, const int* band_skip, const uint8_t* cb_skip, uint8_t* out,
                        size_t out_cap, int* band_bytes, long long* band_bits, void* scratch,
                        size_t scratch_bytes, void* stream);
/* The decoding side (the band decoders' symbol decoding: band_codec_template.h:204-357,
 * 500-557 over ArithCodecBase's decoder, arith_codec.h:200-250, arith_codec.cpp:132-165, or
 * the VLC adapter when vlc != 0): from the coded bands' data (the layout dgpu_code_bands_host
 * writes: per component, bands from the DC band down; band_bytes as the subband headers give
 * them) to the signed quantised indices dgpu_dequantise_batch takes.  qindex[c] (host, dense
 * cw[c] x ch[c] int32) is written in full (zeros in skipped bands and code blocks); cb_skip
 * receives the decoded code-block skip flags (band-list order, components concatenated).  The
 * bands of a level are decoded in parallel, levels from coarse to fine (a band's contexts
 * read its parent band).  data_bytes is the length of data: band lengths that add up to more
 * (a corrupt or truncated stream) return DGPU_ERR_ARG before any band is decoded.  No GPU use. */
int dgpu_decode_bands_host(int n, const int* depth, const int* cw, const int* ch, const int* band_ncb,
                           const int* band_skip, const uint8_t* data, size_t data_bytes,
                           const int* band_bytes, int vlc, int32_t* const* qindex, uint8_t* cb_skip);
int dgpu_entropy_init(int depth, float* state);
int dgpu_entropy_factors(int depth, const float* state, int intra, int is_b, float* ecf);
int dgpu_entropy_update(int depth, float* state, int intra, int is_b, int comp, const int* band_skip,
                        const int* est_bits, const int* band_bytes);

/* ---------------------------------------------------------------------------------------
 * Sequence decoder: the data-parallel part of PictureDecompressor::Decompress
 * (libdirac_decoder/picture_decompress.cpp:73-212) and of the frame output of dirac_parse
 * (set_frame_component, libdirac_decoder/dirac_parser.cpp:159-226): dequantisation (as
 * dgpu_dequantise_batch), the inverse transform of the three components, motion
 * compensation ADD against the upconverted reference pictures (Picture::UpData, made once
 * per reference) with the clip, or the clip alone for intra pictures, and the conversion to
 * unsigned output samples.  What stays with the caller (serial host code in the reference):
 * parsing, the entropy decoding of coefficients (to signed quantised indices) and of motion
 * data, and the picture buffer's policy (dgpu_decoder_release drops a picture).
 *
 * Per picture (dgpu_decode_input): its number, intra flag, references, transform filter,
 * the zero-residual flag (no coefficients coded: the residue is zero), per band the
 * quantiser indices and skip flags (host, components concatenated), and, in host memory
 * (on_host = 1) or device memory (on_host = 0): the signed quantised indices of the three
 * components (int32 [ch][cw] padded to the transform depth: the layout of DGPU_ENC_QINDEX;
 * int16 in the same layout with index_bits = 16, for a caller that has checked every index
 * fits 16 bits: half the bytes to copy),
 * the code-block skip flags (per component in band-list order as DGPU_ENC_CBSKIP, components
 * concatenated) and, for inter pictures, the motion data in the layout of
 * dgpu_motion_compensate.  Transform depth, code blocks and block parameters are fixed per
 * decoder (as the reference encoder keeps them), the filter is per picture.  Host inputs are
 * copied on the decoder's stream: page-locked ones must stay unchanged until the stream has
 * passed the call, pageable ones may be reused on return.
 *
 * dgpu_decoder_decode returns DGPU_ERR_ARG for invalid arguments and for a reference that is
 * not in the buffer (the reference decoder does not decode such a picture,
 * picture_decompress.cpp:107-113), DGPU_ERR_SIZE when every picture slot is taken.  Results
 * are read with dgpu_decoder_read (DGPU_ENC_RECON, DGPU_ENC_COEFF, DGPU_ENC_OUTPUT), which
 * synchronises the stream for host copies.  A handle is not thread-safe; different handles
 * may run on different streams concurrently.
 * ------------------------------------------------------------------------------------- */
typedef struct {
    int cformat, width, height;   /* ChromaFormat and luma size */
    int luma_depth, chroma_depth; /* bits per sample, 8..14 */
    int wlt_depth;                /* transform depth */
    int spatial_partition;        /* 1: SetUsualCodeBlocks' code blocks (dgpu_code_blocks), 0: one per band */
    dgpu_block_params bp;         /* block parameters of the inter pictures */
} dgpu_decoder_params;

typedef struct {
    int pnum;                     /* picture number */
    int intra;                    /* 1: intra picture (no motion data) */
    int num_refs, ref1, ref2;     /* inter: references (picture numbers) */
    int filter;                   /* WltFilter of the picture's transform */
    int zero_residual;            /* 1: no coefficients coded */
    const int* band_qidx;         /* host, [3][3*depth+1] quantiser indices */
    const int* band_skip;         /* host, [3][3*depth+1] band skip flags */
    int on_host;                  /* 1: the arrays below are in host memory */
    const void* qindex[3];        /* int32 elements, or int16 with index_bits = 16 */
    const uint8_t* cb_skip;
    const int16_t* mv1;
    const int16_t* mv2;           /* NULL with one reference */
    const uint8_t* mode;
    const int16_t* dc;
    const uint8_t* split;
    int index_bits;               /* 0 or 32: int32 indices; 16: int16 (half the bytes copied) */
} dgpu_decode_input;

size_t dgpu_decoder_device_bytes(const dgpu_decoder_params* params, int max_pictures);
int dgpu_decoder_create(const dgpu_decoder_params* params, int max_pictures, void* stream, void** decoder);
int dgpu_decoder_destroy(void* decoder);
int dgpu_decoder_decode(void* decoder, const dgpu_decode_input* in);
/* Drops a picture from the buffer (PictureBuffer::Remove); its slot is reused by a later decode. */
int dgpu_decoder_release(void* decoder, int pnum);
size_t dgpu_decoder_item_bytes(void* decoder, int pnum, int what, int comp);
int dgpu_decoder_read(void* decoder, int pnum, int what, int comp, void* dst, size_t bytes, int on_host);

#ifdef __cplusplus
}
#endif
#endif /* DIRAC_GPU_H */
