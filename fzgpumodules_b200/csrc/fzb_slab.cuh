// fzb_slab.cuh -- device helpers shared by the slab kernels (fzb_slab.cu,
// fzb_slab_inv.cu): mbarrier and TMA wrappers, packed f32x2 helpers, the
// 128-byte swizzle of a slab-plane buffer, and the 8-lane byte transpose that
// converts between per-thread plane nibbles and RZE level-1 bitmap words.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "fzb_kernels.cuh"

namespace fzb {
namespace {

constexpr int kStageBytes = kChunkCodes * 4;  // one slab plane of f32
constexpr int kSmemAlign = 1024;              // 128-byte swizzle atom
constexpr uint32_t kWaitLimit = 1u << 26;     // mbarrier polls (also bounded by a 2 s clock)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t v;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
    return v;
}

// Bounded wait for phase `parity` of `bar` (2 s of global time at most):
// false when the bound ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < kWaitLimit; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > 2000000000ull) break;
    }
    return false;
}

// 2-D tiled TMA load (no multicast) of box {32 floats, 256 rows} at row `y`.
__device__ __forceinline__ void tma_load_rows(void* dst, const CUtensorMap* map, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Orders this thread's earlier generic shared-memory accesses before later
// async-proxy (TMA) writes to the same bytes.
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// max that returns NaN when either input is NaN.
__device__ __forceinline__ float max_nan(float a, float b) {
    float d;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// a - b for both lanes, one rounding each (fma(b, -1, a) == a - b exactly).
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}

constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: c + kMagic holds integer c in its low bits

// Round half away from zero of y: trunc(y + copysign(0.49999997, y)) with the
// add rounded to nearest equals round(y) for every float (for |y| >= 2^23 y is
// already integral and the add returns y).  `sv` supplies the sign (of v, the
// same as y's since the scale is positive).
__device__ __forceinline__ uint32_t half_bits(float sv) {
    return (__float_as_uint(sv) & 0x80000000u) | 0x3effffffu;
}

struct Q4 {
    float2 a, b;  // elements 0,1 and 2,3 of a granule
};

// q of a granule: round half away from zero of v * r.
__device__ __forceinline__ Q4 quant4(float4 v, float r) {
    // scalar products: a packed multiply followed by the packed add could be
    // contracted into one fused multiply-add, which rounds differently
    const float2 y0 = f2(__fmul_rn(v.x, r), __fmul_rn(v.y, r));
    const float2 y1 = f2(__fmul_rn(v.z, r), __fmul_rn(v.w, r));
    const float2 s0 = __fadd2_rn(y0, f2(__uint_as_float(half_bits(v.x)), __uint_as_float(half_bits(v.y))));
    const float2 s1 = __fadd2_rn(y1, f2(__uint_as_float(half_bits(v.z)), __uint_as_float(half_bits(v.w))));
    return {f2(truncf(s0.x), truncf(s0.y)), f2(truncf(s1.x), truncf(s1.y))};
}

// Codes of two integer-valued deltas |c| < 2^22 packed as c0 | c1 << 16
// (int16 or zigzag), through the magic-number add: c + 1.5 * 2^23 holds c in
// its low mantissa bits.
template <bool ZZ>
__device__ __forceinline__ uint32_t code_pair(float2 c) {
    const float2 m = __fadd2_rn(c, f2(kMagic, kMagic));
    uint32_t p = __byte_perm(__float_as_uint(m.x), __float_as_uint(m.y), 0x5410);
    if (ZZ) {
        uint32_t s;
        asm("prmt.b32 %0, %1, %1, 0xBB99;" : "=r"(s) : "r"(p));  // per-half sign mask
        p = ((p << 1) & 0xfffefffeu) ^ s;
    }
    return p;
}

// Byte offset in a 128-byte-swizzled buffer of 16-byte granule g of row `row`
// (the TMA SWIZZLE_128B layout: granule index XOR row % 8).  Thread t of a
// slab kernel owns row t (32 floats).
__device__ __forceinline__ uint32_t swz_off(uint32_t row, uint32_t g) {
    return row * 128u + 16u * (g ^ (row & 7u));
}

// Transpose of an 8x8 byte matrix across the 8-lane group of `lane`: lane i
// holds row i (bytes 0-3 in lo, 4-7 in hi); afterwards lane j holds column j
// with the bytes of even source lanes 0,2,4,6 in lo and of odd source lanes
// 1,3,5,7 in hi.  Three butterfly stages (partner lane ^4, ^2, ^1).
__device__ __forceinline__ void group_transpose8(uint32_t& lo, uint32_t& hi, uint32_t lane) {
    const uint32_t full = 0xffffffffu;
    uint32_t w0, w1;
    {   // word s2 <- bytes of source lane with bit 2 = s2
        const bool b2 = lane & 4;
        const uint32_t r = __shfl_xor_sync(full, b2 ? lo : hi, 4);
        w0 = b2 ? r : lo;
        w1 = b2 ? hi : r;
    }
    {   // half s1 of word s2 <- source lane (s2, s1)
        const bool b1 = lane & 2;
        const uint32_t send = b1 ? __byte_perm(w0, w1, 0x5410) : __byte_perm(w0, w1, 0x7632);
        const uint32_t r = __shfl_xor_sync(full, send, 2);
        const uint32_t n0 = b1 ? __byte_perm(r, w0, 0x7610) : __byte_perm(w0, r, 0x5410);
        const uint32_t n1 = b1 ? __byte_perm(r, w1, 0x7632) : __byte_perm(w1, r, 0x7610);
        w0 = n0;
        w1 = n1;
    }
    {   // lo <- source lanes 0,2,4,6; hi <- 1,3,5,7
        const bool b0 = lane & 1;
        const uint32_t even = __byte_perm(w0, w1, 0x6420), odd = __byte_perm(w0, w1, 0x7531);
        const uint32_t r = __shfl_xor_sync(full, b0 ? even : odd, 1);
        lo = b0 ? r : even;
        hi = b0 ? odd : r;
    }
}

// Level-1 bitmap words of this lane's 8-lane group: lane j (= lane & 7) gets
// the words of planes 2j (.x) and 2j+1 (.y); nibble i of each word is the
// nonzero-byte nibble of lane i of the group.  nib64 byte u holds the
// nibbles of planes 2u (low) and 2u+1 (high).
__device__ __forceinline__ uint2 bm1_words(uint64_t nib64, uint32_t lane) {
    uint32_t lo = (uint32_t)nib64, hi = (uint32_t)(nib64 >> 32);
    group_transpose8(lo, hi, lane);
    // byte k of lo = source 2k, of hi = source 2k+1: nibble i of the word = source i
    uint2 out;
    out.x = (lo & 0x0f0f0f0fu) | ((hi << 4) & 0xf0f0f0f0u);
    out.y = ((lo >> 4) & 0x0f0f0f0fu) | (hi & 0xf0f0f0f0u);
    return out;
}

// Inverse of bm1_words: from this lane's words of planes 2j and 2j+1 to its
// own 16 plane nibbles (nib64 layout as above).
__device__ __forceinline__ uint64_t nibs_from_bm1(uint32_t w_even, uint32_t w_odd, uint32_t lane) {
    // byte i = (nibble i of the even word) | (nibble i of the odd word) << 4, natural order
    const uint32_t a = (w_even & 0x0f0f0f0fu) | ((w_odd << 4) & 0xf0f0f0f0u);         // sources 0,2,4,6
    const uint32_t b = ((w_even >> 4) & 0x0f0f0f0fu) | (w_odd & 0xf0f0f0f0u);          // sources 1,3,5,7
    uint32_t lo = __byte_perm(a, b, 0x5140), hi = __byte_perm(a, b, 0x7362);           // bytes by source 0..7
    group_transpose8(lo, hi, lane);
    const uint32_t nlo = __byte_perm(lo, hi, 0x5140), nhi = __byte_perm(lo, hi, 0x7362);
    return ((uint64_t)nhi << 32) | nlo;
}

// Exclusive warp scans of four packed-count words at once (independent
// chains interleaved for latency).  `active` bit j: word j is scanned (all
// lanes agree); inactive words return 0.  inc[j] receives the inclusive value.
__device__ __forceinline__ void warp_scan4(const uint32_t (&v)[4], uint32_t active, uint32_t (&inc)[4]) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 4; j++) inc[j] = v[j];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t n[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((active >> j) & 1u) n[j] = __shfl_up_sync(0xffffffffu, inc[j], d);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (((active >> j) & 1u) && lane >= (uint32_t)d) inc[j] += n[j];
    }
}

}  // namespace
}  // namespace fzb
