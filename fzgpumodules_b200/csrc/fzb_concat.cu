// fzb_concat.cu -- gathers a pipeline's output segments into one buffer:
// [u32 n][u64 size_i x n] padded to 16 bytes, then every segment padded to
// 16 bytes (the layout of the reference's Pipeline::concatOutputs,
// src/pipeline/compressor.cpp:760-875, ConcatLayout in
// src/pipeline/pipeline_utils.h:35-46).  One launch copies every segment;
// pad bytes are written as zeros.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/fzb.h"

namespace {

constexpr int kMaxSeg = FZB_CONCAT_MAX_SEGMENTS;

struct ConcatParams {
    int n;
    const uint8_t* src[kMaxSeg];
    uint64_t bytes[kMaxSeg];
    uint64_t dst_off[kMaxSeg];
    uint64_t header_bytes;
};

__host__ __device__ inline uint64_t pad16(uint64_t v) { return (v + 15) & ~15ull; }

__global__ void concat_kernel(ConcatParams p, uint8_t* __restrict__ out) {
    const int seg = blockIdx.y;
    if (seg == p.n) {  // header
        if (blockIdx.x != 0) return;
        for (uint64_t i = threadIdx.x; i < p.header_bytes; i += blockDim.x) {
            uint8_t v = 0;
            if (i < 4) v = (uint8_t)((uint32_t)p.n >> (8 * i));
            else if (i < 4 + 8ull * p.n) {
                const uint64_t k = (i - 4) / 8, b = (i - 4) % 8;
                v = (uint8_t)(p.bytes[k] >> (8 * b));
            }
            out[i] = v;
        }
        return;
    }
    const uint8_t* s = p.src[seg];
    uint8_t* d = out + p.dst_off[seg];
    const uint64_t len = p.bytes[seg], plen = pad16(len);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if ((reinterpret_cast<uintptr_t>(s) & 15) == 0) {
        const uint64_t nv = len / 16;
        const uint4* s4 = reinterpret_cast<const uint4*>(s);
        uint4* d4 = reinterpret_cast<uint4*>(d);
        for (uint64_t i = t0; i < nv; i += stride) d4[i] = s4[i];
        for (uint64_t i = 16 * nv + t0; i < plen; i += stride) d[i] = i < len ? s[i] : 0;
    } else {
        for (uint64_t i = t0; i < plen; i += stride) d[i] = i < len ? s[i] : 0;
    }
}

}  // namespace

extern "C" uint64_t fzb_concat_bytes(const uint64_t* sizes, int n) {
    if (!sizes || n <= 0 || n > kMaxSeg) return 0;
    uint64_t total = pad16(4 + 8ull * (uint64_t)n);
    for (int i = 0; i < n; i++) total += pad16(sizes[i]);
    return total;
}

extern "C" int fzb_concat(const void* const* d_srcs, const uint64_t* sizes, int n, void* d_out,
                          void* stream) {
    if (!d_srcs || !sizes || !d_out || n <= 0 || n > kMaxSeg) return FZB_E_INVALID;
    if (reinterpret_cast<uintptr_t>(d_out) & 15) return FZB_E_INVALID;
    ConcatParams p{};
    p.n = n;
    p.header_bytes = pad16(4 + 8ull * (uint64_t)n);
    uint64_t off = p.header_bytes, maxlen = 0;
    for (int i = 0; i < n; i++) {
        if (sizes[i] && !d_srcs[i]) return FZB_E_INVALID;
        p.src[i] = static_cast<const uint8_t*>(d_srcs[i]);
        p.bytes[i] = sizes[i];
        p.dst_off[i] = off;
        off += pad16(sizes[i]);
        if (sizes[i] > maxlen) maxlen = sizes[i];
    }
    uint64_t blocks = (maxlen / 16 + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > 1024) blocks = 1024;
    dim3 grid((unsigned)blocks, (unsigned)(n + 1), 1);
    concat_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(p, static_cast<uint8_t*>(d_out));
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

// ---------------------------------------------------------------------------
// The inverse: a container whose segment sizes only the device knows is cut
// back into per-segment buffers.  Every CTA parses the header itself (n and
// the u64 sizes), checks it against the expected count, the destination
// capacities and the container capacity, and copies its share of every
// segment with 16-byte words (segments start on 16-byte boundaries).  A bad
// header sets FZB's malformed bit in *err and copies nothing.
// ---------------------------------------------------------------------------
namespace {

struct SplitParams {
    int n;
    uint8_t* dst[kMaxSeg];
    uint64_t cap[kMaxSeg];
    uint64_t in_cap;
};

constexpr uint32_t kSplitMalformed = 2u;  // the status bit fzb_workspace_status reports as malformed

__global__ void split_kernel(const uint8_t* __restrict__ in, SplitParams p, uint32_t* err) {
    __shared__ uint64_t s_off[kMaxSeg + 1], s_len[kMaxSeg];
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        const uint32_t n = *reinterpret_cast<const uint32_t*>(in);
        bool ok = n == (uint32_t)p.n && pad16(4 + 8ull * n) <= p.in_cap;
        uint64_t off = pad16(4 + 8ull * (uint64_t)p.n);
        for (int k = 0; ok && k < p.n; k++) {
            uint64_t len;
            memcpy(&len, in + 4 + 8 * k, 8);
            ok = len <= p.cap[k] && off + pad16(len) <= p.in_cap;
            s_off[k] = off;
            s_len[k] = len;
            off += pad16(len);
        }
        s_ok = ok;
        if (!ok && blockIdx.x == 0) atomicOr(err, kSplitMalformed);
    }
    __syncthreads();
    if (!s_ok) return;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < p.n; k++) {
        const uint4* s4 = reinterpret_cast<const uint4*>(in + s_off[k]);
        uint4* d4 = reinterpret_cast<uint4*>(p.dst[k]);
        const uint64_t nv = pad16(s_len[k]) / 16;
        for (uint64_t i = t0; i < nv; i += stride) d4[i] = s4[i];
    }
}

}  // namespace

extern "C" int fzb_concat_split(const void* d_in, uint64_t in_capacity, void* const* d_dsts,
                                const uint64_t* capacities, int n, uint32_t* d_err, void* stream) {
    if (!d_in || !d_dsts || !capacities || !d_err || n <= 0 || n > kMaxSeg) return FZB_E_INVALID;
    if (reinterpret_cast<uintptr_t>(d_in) & 15) return FZB_E_INVALID;
    SplitParams p{};
    p.n = n;
    p.in_cap = in_capacity;
    uint64_t maxcap = 0;
    for (int i = 0; i < n; i++) {
        // whole 16-byte words are copied: capacities are multiples of 16
        if (!d_dsts[i] || (reinterpret_cast<uintptr_t>(d_dsts[i]) & 15) || (capacities[i] & 15))
            return FZB_E_INVALID;
        p.dst[i] = static_cast<uint8_t*>(d_dsts[i]);
        p.cap[i] = capacities[i];
        if (capacities[i] > maxcap) maxcap = capacities[i];
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t blocks = (maxcap / 16 + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > 4ull * (uint64_t)sms) blocks = 4ull * (uint64_t)sms;
    split_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const uint8_t*>(d_in), p, d_err);
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

// ---------------------------------------------------------------------------
// Concatenation enqueued before the segment sizes reach the host.  The first
// warp of every CTA turns the size words into lengths and offsets (at most
// 32 segments), so no CTA waits for another; each CTA then copies its
// grid-stride share of every segment with 16-byte words.
// ---------------------------------------------------------------------------
namespace {

struct ConcatDevParams {
    int n;
    const uint8_t* src[kMaxSeg];
    const void* word[kMaxSeg];
    uint64_t cap[kMaxSeg];
    uint64_t scale[kMaxSeg];
    uint64_t wmax[kMaxSeg];
    uint8_t wbytes[kMaxSeg];
};

__global__ void concat_dev_kernel(ConcatDevParams p, uint8_t* __restrict__ out) {
    __shared__ uint64_t s_len[kMaxSeg], s_off[kMaxSeg];
    static_assert(kMaxSeg <= 32, "one warp lays the segments out");
    if (threadIdx.x < 32) {  // lane k: segment k's length, then an exclusive scan of the padded lengths
        const int k = threadIdx.x;
        uint64_t len = 0;
        if (k < p.n) {
            len = p.cap[k];
            if (p.word[k]) {
                uint64_t w = p.wbytes[k] == 8 ? *static_cast<const uint64_t*>(p.word[k])
                                              : (uint64_t)*static_cast<const uint32_t*>(p.word[k]);
                if (w > p.wmax[k]) w = p.wmax[k];
                // w * scale cannot wrap: the host checked wmax * scale
                len = w * p.scale[k];
                if (len > p.cap[k]) len = p.cap[k];
            }
        }
        uint64_t incl = pad16(len);
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t v = __shfl_up_sync(0xffffffffu, incl, d);
            if (k >= d) incl += v;
        }
        if (k < p.n) {
            s_len[k] = len;
            s_off[k] = pad16(4 + 8ull * (uint64_t)p.n) + incl - pad16(len);
        }
    }
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0) {  // header
        const uint64_t hb = pad16(4 + 8ull * (uint64_t)p.n);
        for (uint64_t i = threadIdx.x; i < hb; i += blockDim.x) {
            uint8_t v = 0;
            if (i < 4) v = (uint8_t)((uint32_t)p.n >> (8 * i));
            else if (i < 4 + 8ull * p.n) v = (uint8_t)(s_len[(i - 4) / 8] >> (8 * ((i - 4) % 8)));
            out[i] = v;
        }
    }
    for (int seg = 0; seg < p.n; seg++) {  // every CTA takes a share of every segment
        const uint8_t* s = p.src[seg];
        uint8_t* d = out + s_off[seg];
        const uint64_t len = s_len[seg], plen = pad16(len);
        if ((reinterpret_cast<uintptr_t>(s) & 15) == 0) {
            const uint64_t nv = len / 16;
            const uint4* s4 = reinterpret_cast<const uint4*>(s);
            uint4* d4 = reinterpret_cast<uint4*>(d);
            uint64_t i = t0;
            for (; i + 3 * stride < nv; i += 4 * stride) {  // four loads in flight per thread
                const uint4 a = __ldcs(s4 + i), b = __ldcs(s4 + i + stride);
                const uint4 c = __ldcs(s4 + i + 2 * stride), e = __ldcs(s4 + i + 3 * stride);
                d4[i] = a;
                d4[i + stride] = b;
                d4[i + 2 * stride] = c;
                d4[i + 3 * stride] = e;
            }
            for (; i < nv; i += stride) d4[i] = s4[i];
            for (uint64_t j = 16 * nv + t0; j < plen; j += stride) d[j] = j < len ? s[j] : 0;
        } else {
            for (uint64_t i = t0; i < plen; i += stride) d[i] = i < len ? s[i] : 0;
        }
    }
}

constexpr int kMaxGather = FZB_GATHER_MAX;

struct GatherParams {
    int n;
    uint32_t* src[kMaxGather];
    uint32_t words[kMaxGather];
    uint32_t dst_word[kMaxGather];
    uint32_t clear_mask;
};

// One warp per item; a lane reads a word, stores it and, for a status word,
// clears the source.
__global__ void gather_words_kernel(GatherParams p, uint32_t* dst) {
    const int lane = threadIdx.x & 31;
    for (int k = threadIdx.x >> 5; k < p.n; k += blockDim.x >> 5) {
        for (uint32_t i = lane; i < p.words[k]; i += 32) {
            const uint32_t v = p.src[k][i];
            dst[p.dst_word[k] + i] = v;
            if ((p.clear_mask >> k) & 1u) p.src[k][i] = 0;
        }
    }
}

}  // namespace

extern "C" int fzb_concat_dev(const void* const* d_srcs, const uint64_t* caps, const void* const* d_size_words,
                              const uint32_t* size_word_bytes, const uint64_t* size_scale,
                              const uint64_t* size_max, int n, void* d_out, void* stream) {
    if (!d_srcs || !caps || !d_size_words || !size_word_bytes || !size_scale || !size_max || !d_out || n <= 0 ||
        n > kMaxSeg)
        return FZB_E_INVALID;
    if (reinterpret_cast<uintptr_t>(d_out) & 15) return FZB_E_INVALID;
    ConcatDevParams p{};
    p.n = n;
    uint64_t maxcap = 0;
    for (int i = 0; i < n; i++) {
        if (caps[i] && !d_srcs[i]) return FZB_E_INVALID;
        p.src[i] = static_cast<const uint8_t*>(d_srcs[i]);
        p.word[i] = d_size_words[i];
        p.cap[i] = caps[i];
        if (d_size_words[i]) {
            const uint32_t wb = size_word_bytes[i];
            if ((wb != 4 && wb != 8) || (reinterpret_cast<uintptr_t>(d_size_words[i]) & (wb - 1)) ||
                size_scale[i] == 0 || size_max[i] > ~0ull / size_scale[i])
                return FZB_E_INVALID;
            p.wbytes[i] = (uint8_t)wb;
            p.scale[i] = size_scale[i];
            p.wmax[i] = size_max[i];
        }
        if (caps[i] > maxcap) maxcap = caps[i];
    }
    // one grid over all segments: the lengths are on the device, so it is
    // sized for the largest (a few waves of the SMs at most)
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t blocks = (maxcap / 16 + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > 8ull * (uint64_t)sms) blocks = 8ull * (uint64_t)sms;
    concat_dev_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p, static_cast<uint8_t*>(d_out));
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

extern "C" int fzb_gather_words(const void* const* d_srcs, const uint32_t* bytes, const uint8_t* clear, int n,
                                void* dst, void* stream) {
    if (!d_srcs || !bytes || !clear || !dst || n <= 0 || n > kMaxGather) return FZB_E_INVALID;
    if (reinterpret_cast<uintptr_t>(dst) & 7) return FZB_E_INVALID;
    GatherParams p{};
    p.n = n;
    uint32_t off = 0;
    for (int i = 0; i < n; i++) {
        if (!d_srcs[i] || (reinterpret_cast<uintptr_t>(d_srcs[i]) & 3) || bytes[i] == 0 || (bytes[i] & 3) ||
            bytes[i] > 256)
            return FZB_E_INVALID;
        p.src[i] = static_cast<uint32_t*>(const_cast<void*>(d_srcs[i]));
        p.words[i] = bytes[i] / 4;
        p.dst_word[i] = off / 4;
        off += (bytes[i] + 7) & ~7u;
        if (clear[i]) p.clear_mask |= 1u << i;
    }
    gather_words_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(p, static_cast<uint32_t*>(dst));
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}
