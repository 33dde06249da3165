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
