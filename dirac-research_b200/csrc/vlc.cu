// Variable-length coding of quantised subbands on the device (-use_vlc).
//
// The reference's variable-length band coders (BandVLC / IntraDCBandVLC over
// ArithCodecToVLCAdapter, libdirac_common/band_vlc.cpp:49-100, band_vlc.h:55-140) write the
// arithmetic coder's binary symbols as plain bits: per code block its skip flag (when the band
// has more than one code block), then per coefficient in raster order the interleaved
// exp-Golomb code of |v| + 1 (for each bit below the top one: a 0 follow bit and the bit
// itself; then a terminating 1) and, for a non-zero value, its sign (1 for negative).  Each
// band's data ends on a byte boundary (SubbandByteIO::GetBytes).  No symbol depends on another,
// so every coefficient's code is placed independently: one pass sums the code lengths of each
// code block, the host turns the sums into bit offsets (bands byte-aligned, components one after
// the other, each component's bands from the DC band down), and a second pass ORs each code
// into big-endian 32-bit words at its offset (a block-wide scan of the lengths within a code
// block).  The bytes equal dgpu_code_bands_vlc_host's.

#include <algorithm>
#include <vector>

#include "dgpu_internal.cuh"

namespace dgpu {
namespace {

constexpr int VLC_THREADS = 256;

// One code block of one component's band: its rectangle in the component's indices, its skip
// flag, and where its bits start in the output (set for the second pass).
struct VlcBlock {
    const int32_t* q;   // the component's indices
    int cw;             // row pitch
    int x0, x1, y0, y1;
    int code_skip;      // 1: a skip flag precedes the block
    int skipped;        // 1: skipped (flag 1, no coefficients)
    long long bit0;     // first bit of the block in the output (second pass)
};

__device__ __forceinline__ unsigned magnitude(int v) { return v < 0 ? 0u - (unsigned)v : (unsigned)v; }

__device__ __forceinline__ int vlc_len(int v) {
    const unsigned n1 = magnitude(v) + 1u;
    const int top = 31 - __clz(n1);
    return 2 * top + 1 + (v != 0);
}

// The code of v, most significant bit first, in the low vlc_len(v) bits.
__device__ __forceinline__ unsigned long long vlc_code(int v) {
    const unsigned n1 = magnitude(v) + 1u;
    const int top = 31 - __clz(n1);
    unsigned long long c = 0;
    for (int i = top - 1; i >= 0; --i) c = (c << 2) | ((n1 >> i) & 1u);  // 0 follow bit, info bit
    c = (c << 1) | 1u;                                                    // terminator
    if (v != 0) c = (c << 1) | (v < 0 ? 1u : 0u);                         // sign
    return c;
}

// ORs the low len bits of code into the stream at bit position p (words big-endian in memory).
__device__ __forceinline__ void put_bits(uint32_t* words, long long p, unsigned long long code, int len) {
    while (len > 0) {
        const long long k = p >> 5;
        const int o = (int)(p & 31);
        const int take = min(32 - o, len);
        const unsigned bits = (unsigned)((code >> (len - take)) & ((1ull << take) - 1));
        const unsigned w = bits << (32 - o - take);
        atomicOr(&words[k], __byte_perm(w, 0, 0x0123));
        p += take;
        len -= take;
    }
}

__device__ __forceinline__ long long block_sum(long long v, long long* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    long long t = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < VLC_THREADS / 32; ++i) t += red[i];
    __syncthreads();
    return t;
}

// First pass: bits per code block (skip flag included).
__global__ void __launch_bounds__(VLC_THREADS) vlc_count_kernel(const VlcBlock* blocks, long long* bits) {
    __shared__ long long red[VLC_THREADS / 32];
    const VlcBlock B = blocks[blockIdx.x];
    long long s = 0;
    if (!B.skipped) {
        const int w = B.x1 - B.x0, n = w * (B.y1 - B.y0);
        for (int i = threadIdx.x; i < n; i += VLC_THREADS) {
            const int y = B.y0 + i / w, x = B.x0 + i % w;
            s += vlc_len(B.q[(size_t)y * B.cw + x]);
        }
    }
    const long long t = block_sum(s, red);
    if (threadIdx.x == 0) bits[blockIdx.x] = t + B.code_skip;
}

// Second pass: every code at its offset.  Chunks of VLC_THREADS coefficients in raster order;
// a block-wide exclusive scan of their lengths gives each one's position.
__global__ void __launch_bounds__(VLC_THREADS) vlc_write_kernel(const VlcBlock* blocks, uint32_t* words) {
    __shared__ int warp_tot[VLC_THREADS / 32];
    __shared__ long long base;
    const VlcBlock B = blocks[blockIdx.x];
    if (threadIdx.x == 0) {
        if (B.code_skip) put_bits(words, B.bit0, B.skipped ? 1u : 0u, 1);
        base = B.bit0 + B.code_skip;
    }
    __syncthreads();
    if (B.skipped) return;
    const int w = B.x1 - B.x0, n = w * (B.y1 - B.y0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c0 = 0; c0 < n; c0 += VLC_THREADS) {
        const int i = c0 + threadIdx.x;
        int v = 0, len = 0;
        if (i < n) {
            v = B.q[(size_t)(B.y0 + i / w) * B.cw + B.x0 + i % w];
            len = vlc_len(v);
        }
        // exclusive scan of len over the block
        int incl = len;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        int before = 0, total = 0;
        for (int k = 0; k < VLC_THREADS / 32; ++k) {
            if (k < warp) before += warp_tot[k];
            total += warp_tot[k];
        }
        if (i < n) put_bits(words, base + before + incl - len, vlc_code(v), len);
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
}

// SubbandList::Init (wavelet_utils.cpp:144-190): band b (1-based) of a cw x ch array.
void vlc_band_rect(int depth, int cw, int ch, int b, int& xp, int& yp, int& xl, int& yl) {
    if (b == 3 * depth + 1) {
        xp = yp = 0;
        xl = cw >> depth;
        yl = ch >> depth;
        return;
    }
    const int level = (b - 1) / 3 + 1, kind = (b - 1) % 3;
    xl = cw >> level;
    yl = ch >> level;
    xp = (kind == 0 || kind == 2) ? xl : 0;
    yp = (kind == 0 || kind == 1) ? yl : 0;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_code_bands_vlc(int n, const int* depth, const int32_t* const* qindex, const int* cw,
                                   const int* ch, const int* band_ncb, const int* band_skip, const uint8_t* cb_skip,
                                   uint8_t* out, size_t out_cap, int* band_bytes, long long* band_bits,
                                   void* scratch, size_t scratch_bytes, void* stream) {
    if (n <= 0 || !depth || !qindex || !cw || !ch || !band_ncb || !band_skip || !cb_skip || !band_bytes)
        return DGPU_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    // the code blocks of every coded band, in output order: component by component, each
    // component's bands from the DC band down, a band's blocks in raster order
    std::vector<VlcBlock> blocks;
    std::vector<int> band_of;        // per block: global band index
    std::vector<int> first_global(n);
    int g = 0;
    size_t cbo_total = 0;
    std::vector<size_t> cb_first;    // per global band: its first code-block flag
    for (int c = 0; c < n; ++c) {
        const int d = depth[c];
        if (d < 1 || d > 8 || !qindex[c] || cw[c] <= 0 || ch[c] <= 0 || cw[c] % (1 << d) || ch[c] % (1 << d))
            return DGPU_ERR_ARG;
        first_global[c] = g;
        for (int b = 1; b <= 3 * d + 1; ++b, ++g) {
            if (band_ncb[2 * g] < 1 || band_ncb[2 * g + 1] < 1) return DGPU_ERR_ARG;
            cb_first.push_back(cbo_total);
            cbo_total += (size_t)band_ncb[2 * g] * band_ncb[2 * g + 1];
        }
    }
    for (int c = 0; c < n; ++c) {
        const int d = depth[c], nb = 3 * d + 1;
        for (int b = nb; b >= 1; --b) {
            const int gb = first_global[c] + b - 1;
            if (band_skip[gb]) continue;
            int xp, yp, xl, yl;
            vlc_band_rect(d, cw[c], ch[c], b, xp, yp, xl, yl);
            const int xn = band_ncb[2 * gb], yn = band_ncb[2 * gb + 1];
            for (int by = 0; by < yn; ++by)
                for (int bx = 0; bx < xn; ++bx) {
                    VlcBlock B{};
                    B.q = qindex[c];
                    B.cw = cw[c];
                    B.x0 = xp + bx * xl / xn;
                    B.x1 = xp + (bx + 1) * xl / xn;
                    B.y0 = yp + by * yl / yn;
                    B.y1 = yp + (by + 1) * yl / yn;
                    B.code_skip = (xn > 1 || yn > 1) ? 1 : 0;
                    B.skipped = cb_skip[cb_first[gb] + (size_t)by * xn + bx] != 0;
                    blocks.push_back(B);
                    band_of.push_back(gb);
                }
        }
    }
    const int nblk = (int)blocks.size();
    for (int k = 0; k < g; ++k) {
        band_bytes[k] = 0;
        if (band_bits) band_bits[k] = 0;
    }
    if (nblk == 0) return DGPU_OK;
    // device tables: the blocks and their bit counts
    const size_t need = align_up(sizeof(VlcBlock) * nblk, 256) + align_up(sizeof(long long) * nblk, 256);
    void* ws = scratch;
    if (!ws) {
        const int rc = library_scratch(need, stream, &ws);
        if (rc) return rc;
    } else if (scratch_bytes < need) {
        return DGPU_ERR_NOMEM;
    }
    VlcBlock* d_blocks = static_cast<VlcBlock*>(ws);
    long long* d_bits = reinterpret_cast<long long*>(static_cast<char*>(ws) + align_up(sizeof(VlcBlock) * nblk, 256));
    DGPU_CHECK_CUDA(cudaMemcpyAsync(d_blocks, blocks.data(), sizeof(VlcBlock) * nblk, cudaMemcpyHostToDevice, st));
    vlc_count_kernel<<<nblk, VLC_THREADS, 0, st>>>(d_blocks, d_bits);
    DGPU_CHECK_LAUNCH();
    std::vector<long long> bits(nblk);
    DGPU_CHECK_CUDA(cudaMemcpyAsync(bits.data(), d_bits, sizeof(long long) * nblk, cudaMemcpyDeviceToHost, st));
    DGPU_CHECK_CUDA(host_wait(st));
    // bit offsets: each band starts on a byte boundary
    std::vector<long long> bbits(g, 0);
    for (int i = 0; i < nblk; ++i) bbits[band_of[i]] += bits[i];
    long long at = 0;  // bytes
    int prev_band = -1;
    long long in_band = 0;
    for (int i = 0; i < nblk; ++i) {
        const int gb = band_of[i];
        if (gb != prev_band) {
            if (prev_band >= 0) at += (bbits[prev_band] + 7) / 8;
            prev_band = gb;
            in_band = 0;
        }
        blocks[i].bit0 = 8 * at + in_band;
        in_band += bits[i];
    }
    const long long total = at + (bbits[prev_band] + 7) / 8;
    for (int k = 0; k < g; ++k) {
        band_bytes[k] = (int)((bbits[k] + 7) / 8);
        if (band_bits) band_bits[k] = bbits[k];
    }
    if (!out) return DGPU_OK;
    // the writes OR into whole 32-bit words: out holds the data rounded up to 4 bytes
    const size_t words_bytes = align_up((size_t)total, 4);
    if (words_bytes > out_cap) return DGPU_ERR_SIZE;
    if (reinterpret_cast<size_t>(out) % 4) return DGPU_ERR_ARG;
    DGPU_CHECK_CUDA(cudaMemsetAsync(out, 0, words_bytes, st));
    DGPU_CHECK_CUDA(cudaMemcpyAsync(d_blocks, blocks.data(), sizeof(VlcBlock) * nblk, cudaMemcpyHostToDevice, st));
    vlc_write_kernel<<<nblk, VLC_THREADS, 0, st>>>(d_blocks, reinterpret_cast<uint32_t*>(out));
    DGPU_CHECK_LAUNCH();
    return DGPU_OK;
}
