// fzb_common.cuh -- device helpers shared by the sm_100a hot-path kernels.
//
// Rounding, code mapping, block scans, the 16x16 in-register bit transpose
// used by Bitshuffle, byte-mask helpers used by RZE, and the bounded
// decoupled look-back used to place variable-size chunk outputs.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fzb {

constexpr int kThreads = 256;            // threads per chunk CTA
constexpr int kChunkBytes = 16384;       // Bitshuffle block == RZE chunk
constexpr int kChunkCodes = kChunkBytes / 2;  // u16 codes per chunk
constexpr int kRzeAvail = kChunkBytes - 2;    // rze_stage.cu:369

// Device error word bits (workspace[0]); read by the host after the launch.
constexpr uint32_t kErrLookbackTimeout = 1u;
constexpr uint32_t kErrMalformed = 2u;
constexpr uint32_t kErrInexact = 4u;      // fused inverse left the exact-integer regime
constexpr uint32_t kErrUnsorted = 8u;     // outlier indices not ascending
constexpr uint32_t kErrTmaTimeout = 16u;  // a TMA copy did not complete within its bound

// Round half away from zero (the float overload of `round` that the
// reference applies to x * ebx2_r).  v - trunc(v) is exact in FP32.
__device__ __forceinline__ float round_half_away(float v) {
    float t = truncf(v);
    float d = __fsub_rn(v, t);
    float s = __int_as_float((__float_as_int(v) & 0x80000000) | 0x3f800000);  // +-1
    return (fabsf(d) >= 0.5f) ? __fadd_rn(t, s) : t;
}

// Code of a quantizable delta: (TCode)(int)delta or its zigzag
// (lorenzo_quant.cu:326-334, zigzag.h:70-74).
__device__ __forceinline__ uint32_t encode_code(float c, bool zigzag) {
    int iv = __float2int_rz(c);
    if (zigzag) {
        int s = (int)(int16_t)iv;
        return (((uint32_t)s << 1) ^ (uint32_t)(s >> 15)) & 0xffffu;
    }
    return (uint32_t)iv & 0xffffu;
}

// Inverse of encode_code as the dequantize kernels read it (zigzag.h:80-84).
__device__ __forceinline__ float decode_code(uint32_t u, bool zigzag) {
    if (zigzag) {
        int s = (int)((u >> 1) ^ (0u - (u & 1u)));
        return (float)(int16_t)s;
    }
    return (float)(int16_t)u;
}

// ---------------------------------------------------------------- scans

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t n = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += n;
    }
    return v;
}

// Block-wide exclusive scan for kThreads threads.  `ws` needs 9 u32 of smem.
// Returns the exclusive prefix; *total receives the block sum.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* ws, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = (lane < kThreads / 32) ? ws[lane] : 0u;
        uint32_t ti = warp_incl_scan(t);
        if (lane < kThreads / 32) ws[lane] = ti - t;  // exclusive warp offsets
        if (lane == kThreads / 32 - 1) ws[8] = ti;
    }
    __syncthreads();
    uint32_t r = ws[warp] + inc - v;
    *total = ws[8];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------- bit transpose

// In-place transpose of two 16x16 bit matrices held in the low and high
// halves of x[0..15]: afterwards bit i of x[j] (per half) is what bit j of
// x[i] was.  With x[l] = code[l] | code[l+16] << 16 the result is
// x[b] = plane word of bit b over the 32 codes, i.e. exactly the word the
// reference's ballot bitshuffle (bitshuffle_stage.cu:299-323) stores at
// plane (15-b).  The transform is its own inverse.
__device__ __forceinline__ void transpose16x2(uint32_t (&x)[16]) {
    // 8x8 block swap: exchange byte 1 of x[i] with byte 0 of x[i+8] in both
    // halves (one byte permute per output word).
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t a = x[i], b = x[i + 8];
        x[i] = __byte_perm(a, b, 0x6240);      // a.b0, b.b0, a.b2, b.b2
        x[i + 8] = __byte_perm(a, b, 0x7351);  // a.b1, b.b1, a.b3, b.b3
    }
#pragma unroll
    for (int s = 4; s >= 1; s >>= 1) {
        const uint32_t m = (s == 4) ? 0x0f0f0f0fu : (s == 2) ? 0x33333333u : 0x55555555u;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            if (i & s) continue;
            uint32_t t = ((x[i] >> s) ^ x[i + s]) & m;
            x[i + s] ^= t;
            x[i] ^= t << s;
        }
    }
}

// ---------------------------------------------------------------- byte masks

// 4-bit mask of the nonzero bytes of w (bit k <-> byte k).
__device__ __forceinline__ uint32_t nz_nibble(uint32_t w) {
    uint32_t hi = (((w & 0x7f7f7f7fu) + 0x7f7f7f7fu) | w) & 0x80808080u;
    return (hi * 0x00204081u) >> 28;
}

__device__ __forceinline__ uint32_t nz_byte_mask64(uint64_t w) {
    return nz_nibble((uint32_t)w) | (nz_nibble((uint32_t)(w >> 32)) << 4);
}

// ---------------------------------------------------------------- look-back
//
// One u64 status word per chunk: bits 63..62 = 0 empty, 1 aggregate,
// 2 inclusive prefix; bits 61..0 = value.  Chunks are taken in ticket
// order, so a chunk only ever waits on chunks whose CTAs are running or
// done; every wait is bounded and raises kErrLookbackTimeout instead of
// spinning forever.

constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagPre = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ void lb_store(unsigned long long* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t lb_load(const unsigned long long* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Called by all kThreads threads of the CTA owning `chunk`: one round trip
// inspects 256 predecessors.  Publishes `agg`, walks back to the nearest
// inclusive prefix, publishes this chunk's inclusive prefix and returns the
// exclusive prefix (identical in all threads).  `red` needs 2*(kThreads/32)+2
// u64 of shared memory.
__device__ __noinline__ static uint64_t lookback(unsigned long long* st, uint32_t chunk,
                                                 uint64_t agg, uint32_t* err,
                                                 unsigned long long* red) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr int W = kThreads / 32;
    if (chunk == 0) {
        if (t == 0) lb_store(st, kFlagPre | agg);
        return 0;
    }
    if (t == 0) lb_store(st + chunk, kFlagAgg | agg);
    uint64_t excl = 0;
    int64_t base = (int64_t)chunk - 1;
    bool timed_out = false;
    while (true) {
        const int64_t idx = base - t;
        uint64_t s = kFlagPre;  // positions before chunk 0 read as an empty prefix
        if (idx >= 0) {
            int spins = 0;
            while (true) {
                s = lb_load(st + idx);
                if ((s >> 62) != 0) break;
                if (++spins > kSpinLimit) {
                    timed_out = true;
                    s = kFlagPre;
                    break;
                }
                __nanosleep(32);
            }
        }
        // nearest inclusive prefix: smallest t whose status carries one
        const uint32_t pre = __ballot_sync(0xffffffffu, (s >> 62) == 2);
        if (lane == 0) red[warp] = pre ? (unsigned long long)(warp * 32 + __ffs(pre) - 1) : 1000ull;
        __syncthreads();
        unsigned long long tmin = 1000ull;
#pragma unroll
        for (int w = 0; w < W; w++) tmin = min(tmin, red[w]);
        uint64_t v = ((unsigned long long)t <= tmin) ? (s & kValMask) : 0ull;
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        if (lane == 0) red[W + warp] = v;
        __syncthreads();
        uint64_t sum = 0;
#pragma unroll
        for (int w = 0; w < W; w++) sum += red[W + w];
        excl += sum;
        __syncthreads();
        if (tmin < 1000ull) break;
        base -= kThreads;
    }
    if (timed_out) atomicOr(err, kErrLookbackTimeout);
    if (t == 0) lb_store(st + chunk, kFlagPre | ((excl + agg) & kValMask));
    return excl;
}

}  // namespace fzb
