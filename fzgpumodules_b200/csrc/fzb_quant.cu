// fzb_quant.cu -- QuantizerStage<float, TCode> (quantizers/quantizer/
// quantizer.cu): prediction-free quantisation of each value, TCode = u16 or
// u32.
//   ABS / NOA (:30-70): q = rint(x / (2 abs_eb)); representable when
//       -R < q < R and |x| < threshold, stored as q (two's complement in
//       TCode) or zigzag(q) in the signed type of TCode's width; else an
//       outlier with stored code 0.  NOA scales the bound by max - min.
//   ABS / NOA in place (:83-107, TCode = u32 only, zigzag required): valid
//       codes are (q << 1) ^ (q >> 31); outliers keep the value's raw bits.
//       Inverse (:147-167): (code >> 1) >= R marks an outlier.
//   REL (:232-327): |x| >= threshold, zero, denormal, inf and NaN are
//       outliers; else bin = rint(__log2f(|x|) / log2eb) with log2eb =
//       2 log2(1 + eb), packed as ((|bin| << 2) | (bin < 0) << 1 | sign) + 1
//       and kept when |bin| < R, the packed word fits TCode and
//       exp2f(bin * log2eb) lies within |x| / (1 + eb) .. |x| (1 + eb).
//       Inverse (:330-356): sign * exp2f(bin * log2eb), 0 for code 0.
// Outliers go to (value, index) lists in ascending index order -- one of the
// orders the reference's atomicAdd slots can produce; when more than `cap`
// occur, the first `cap` by index are kept and the count is capped (the
// reference's postStreamSync caps it the same way, :651-676).
//
// This file is built with the compiler's default floating-point contraction,
// like the reference's kernels: its REL path calls __log2f and exp2f, and the
// codes must come out bit-identical.
//
// Forward: two kernels and no inter-CTA waits.  quantizer_codes_kernel
// streams tiles of 4096 values (256 threads x four 16-byte loads; element
// k*1024 + 4t + j in thread t), writes the codes with vector stores and
// records each tile's outlier count, summed per group of 256 tiles.
// quantizer_outliers_kernel then revisits only the tiles that hold outliers
// (the first kernel appends them to a list):
// it takes the tile's offset from the group and tile counts before it,
// recomputes the outlier flags from the input and writes (value, index)
// pairs in index order; its block 0 stores min(total, cap) as the count.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "../../include/fzb.h"
#include "fzb_common.cuh"
#include "fzb_kernels.cuh"

namespace fzb {
namespace {

constexpr uint32_t kQTile = 4096;   // values per tile: 256 threads x 4 granules of 4
constexpr uint32_t kQGroup = 256;   // tiles per group count
constexpr int kQWarps = kThreads / 32;
constexpr int kQMaxParts = 1024;

struct QArgs {
    const float* in;
    uint64_t n;
    const float* st;  // resolved bound: [1] abs_eb, [2] 1 / (2 abs_eb)
    float log2eb, log2eb_r, opp, oopp;
    float threshold;
    uint32_t radius;  // as stored in TCode
    int zigzag;
    void* codes;
    float* ovals;
    uint32_t* oidx;
    uint32_t* count;
    uint64_t cap;
    uint32_t* tile_cnt;   // outliers per tile
    uint32_t* group_cnt;  // outliers per group of kQGroup tiles (zeroed per launch)
    uint32_t* list;       // tiles holding outliers, in completion order
    uint32_t* list_len;   // zeroed per launch
    uint32_t ntiles, ngroups;
    int vec;              // input 16-byte aligned, codes aligned for 4-code stores
};

template <typename TC>
__device__ __forceinline__ TC zigzag_code(int q) {
    using S = typename std::make_signed<TC>::type;
    const S v = (S)q;
    return (TC)((TC)((TC)v << 1) ^ (TC)(v >> (sizeof(TC) * 8 - 1)));
}

template <typename TC>
__device__ __forceinline__ int unzigzag_code(TC u) {
    using S = typename std::make_signed<TC>::type;
    return (int)(S)(TC)((TC)(u >> 1) ^ (TC)(0 - (u & 1)));
}

// One value -> stored code; `outlier` reports the outlier path.
template <typename TC, bool REL>
__device__ __forceinline__ TC quantize_one(const QArgs& a, float x, float ebx2_r, bool& outlier) {
    const int R = (int)a.radius;
    if (!REL) {
        const int q = __float2int_rn(x * ebx2_r);
        outlier = !(q > -R && q < R && fabsf(x) < a.threshold);
        if (outlier) return (TC)0;
        return a.zigzag ? zigzag_code<TC>(q) : (TC)q;
    }
    outlier = true;
    if (fabsf(x) >= a.threshold) return (TC)0;
    const int expo = (int)((__float_as_uint(x) >> 23) & 0xffu);
    if (expo == 0 || expo == 255) return (TC)0;
    const bool neg = x < 0.0f;
    const float ax = neg ? -x : x;
    const int lb = __float2int_rn(__log2f(ax) * a.log2eb_r);
    const uint32_t alb = (uint32_t)(lb < 0 ? -lb : lb);
    const uint32_t stored = ((alb << 2) | ((lb < 0 ? 1u : 0u) << 1) | (neg ? 1u : 0u)) + 1u;
    if (alb < (uint32_t)R && stored <= (uint32_t)(TC)~(TC)0) {
        const float ar = exp2f((float)lb * a.log2eb);
        const float lo = ax * a.oopp, hi = ax * a.opp;
        if (ar >= lo && ar <= hi) {
            outlier = false;
            return (TC)stored;
        }
    }
    return (TC)0;
}

// Four consecutive values of granule k of this thread's tile (zero past n).
__device__ __forceinline__ float4 load_granule(const QArgs& a, uint64_t i0, bool full) {
    if (full) return __ldcs(reinterpret_cast<const float4*>(a.in + i0));
    float4 v;
    v.x = i0 < a.n ? a.in[i0] : 0.0f;
    v.y = i0 + 1 < a.n ? a.in[i0 + 1] : 0.0f;
    v.z = i0 + 2 < a.n ? a.in[i0 + 2] : 0.0f;
    v.w = i0 + 3 < a.n ? a.in[i0 + 3] : 0.0f;
    return v;
}

// Quantises granule k; returns the 4-bit outlier mask of its valid values.
template <typename TC, bool REL>
__device__ __forceinline__ uint32_t quantize_granule(const QArgs& a, const float4& v, uint64_t i0, float r,
                                                     TC (&c)[4]) {
    const float x[4] = {v.x, v.y, v.z, v.w};
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        bool o;
        c[j] = quantize_one<TC, REL>(a, x[j], r, o);
        if (o && i0 + j < a.n) m |= 1u << j;
    }
    return m;
}

template <typename TC, bool REL>
__global__ void __launch_bounds__(kThreads) quantizer_codes_kernel(QArgs a) {
    __shared__ uint32_t s_w[kQWarps];
    const int t = threadIdx.x;
    const uint64_t base = (uint64_t)blockIdx.x * kQTile;
    const bool full = a.vec && base + kQTile <= a.n;
    const float r = REL ? 0.0f : a.st[2];
    TC* codes = static_cast<TC*>(a.codes);
    float4 v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = load_granule(a, base + (uint64_t)k * 1024 + 4 * t, full);
    uint32_t cnt = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint64_t i0 = base + (uint64_t)k * 1024 + 4 * t;
        TC c[4];
        cnt += __popc(quantize_granule<TC, REL>(a, v[k], i0, r, c));
        if (full) {
            if (sizeof(TC) == 4) {
                *reinterpret_cast<uint4*>(codes + i0) = make_uint4(c[0], c[1], c[2], c[3]);
            } else {
                *reinterpret_cast<uint2*>(codes + i0) =
                    make_uint2((uint32_t)c[0] | ((uint32_t)c[1] << 16), (uint32_t)c[2] | ((uint32_t)c[3] << 16));
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (i0 + j < a.n) codes[i0 + j] = c[j];
        }
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
    if ((t & 31) == 0) s_w[t >> 5] = cnt;
    __syncthreads();
    if (t == 0) {
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kQWarps; w++) total += s_w[w];
        a.tile_cnt[blockIdx.x] = total;
        if (total) {
            atomicAdd(a.group_cnt + blockIdx.x / kQGroup, total);
            a.list[atomicAdd(a.list_len, 1u)] = blockIdx.x;
        }
    }
}

// Block-wide sum of one value per thread (result in every thread).
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* s_w) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < kQWarps; w++) t += s_w[w];
    return t;
}

template <typename TC, bool REL>
__device__ __forceinline__ void write_tile_outliers(const QArgs& a, uint32_t tile, uint32_t* s_w,
                                                    unsigned long long* s_wx) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    // offset: every outlier in earlier groups and in earlier tiles of this group
    const uint32_t g = tile / kQGroup;
    uint32_t part = 0;
    for (uint32_t i = t; i < g; i += kThreads) part += a.group_cnt[i];
    for (uint32_t i = g * kQGroup + t; i < tile; i += kThreads) part += a.tile_cnt[i];
    const uint64_t prefix = block_sum(part, s_w);
    if (prefix >= a.cap) return;
    const uint64_t base = (uint64_t)tile * kQTile;
    const bool full = a.vec && base + kQTile <= a.n;
    const float r = REL ? 0.0f : a.st[2];
    float4 v[4];
    uint32_t m[4];
    unsigned long long packed = 0;  // 16-bit outlier count of granule k in bits 16k..16k+15
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = load_granule(a, base + (uint64_t)k * 1024 + 4 * t, full);
        TC c[4];
        m[k] = quantize_granule<TC, REL>(a, v[k], base + (uint64_t)k * 1024 + 4 * t, r, c);
        packed |= (unsigned long long)__popc(m[k]) << (16 * k);
    }
    // exclusive block scan of the packed counts: four independent 16-bit lanes
    unsigned long long inc = packed;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += o;
    }
    __syncthreads();
    if (lane == 31) s_wx[warp] = inc;
    __syncthreads();
    unsigned long long before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kQWarps; w++) {
        if (w < warp) before += s_wx[w];
        all += s_wx[w];
    }
    const unsigned long long excl = before + inc - packed;
    uint64_t kbase = prefix;  // outliers of granules < k across the tile come first
#pragma unroll
    for (int k = 0; k < 4; k++) {
        uint64_t slot = kbase + ((excl >> (16 * k)) & 0xffffu);
        const float x[4] = {v[k].x, v[k].y, v[k].z, v[k].w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if ((m[k] >> j) & 1u) {
                if (slot < a.cap) {
                    a.ovals[slot] = x[j];
                    a.oidx[slot] = (uint32_t)(base + (uint64_t)k * 1024 + 4 * t + j);
                }
                slot++;
            }
        }
        kbase += (all >> (16 * k)) & 0xffffu;
    }
}

// The grid walks the list of tiles that hold outliers.  A tile's slots
// depend only on the counts before it, so the list order does not matter.
template <typename TC, bool REL>
__global__ void __launch_bounds__(kThreads) quantizer_outliers_kernel(QArgs a) {
    __shared__ uint32_t s_w[kQWarps];
    __shared__ unsigned long long s_wx[kQWarps];
    if (blockIdx.x == 0) {  // the stored count: min(total, cap)
        uint32_t part = 0;
        for (uint32_t g = threadIdx.x; g < a.ngroups; g += kThreads) part += a.group_cnt[g];
        const uint32_t total = block_sum(part, s_w);
        if (threadIdx.x == 0) *a.count = (uint32_t)((uint64_t)total < a.cap ? total : a.cap);
    }
    const uint32_t len = *a.list_len;
    for (uint32_t i = blockIdx.x; i < len; i += gridDim.x) write_tile_outliers<TC, REL>(a, a.list[i], s_w, s_wx);
}

__global__ void __launch_bounds__(256) quantizer_fwd_inplace_kernel(const float* __restrict__ in, uint64_t n,
                                                                    const float* __restrict__ st, float threshold,
                                                                    uint32_t radius, uint32_t* __restrict__ codes) {
    const float r = st[2];
    const int R = (int)radius;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = __ldcs(in + i);
        const int q = __float2int_rn(x * r);
        codes[i] = (q > -R && q < R && fabsf(x) < threshold) ? (((uint32_t)q << 1) ^ (uint32_t)(q >> 31))
                                                             : __float_as_uint(x);
    }
}

template <typename TC, bool REL>
__device__ __forceinline__ float dequant_one(TC c, float ebx2, float log2eb, int zigzag) {
    if (!REL) {
        using S = typename std::make_signed<TC>::type;
        const int q = zigzag ? unzigzag_code<TC>(c) : (int)(S)c;
        return (float)q * ebx2;
    }
    if (c == 0) return 0.0f;
    const uint32_t cv = (uint32_t)c - 1u;
    const int alb = (int)(cv >> 2);
    const int lb = ((cv >> 1) & 1u) ? -alb : alb;
    const float ar = exp2f((float)lb * log2eb);
    return (cv & 1u) ? -ar : ar;
}

__device__ __forceinline__ float dequant_inplace(uint32_t c, float ebx2, uint32_t radius) {
    if ((c >> 1) >= radius) return __uint_as_float(c);
    const int32_t ci = (int32_t)c;
    const int q = (ci & 1) ? -((ci + 1) >> 1) : (ci >> 1);
    return (float)q * ebx2;
}

// Four codes of granule i0 (zero past n).
template <typename TC>
__device__ __forceinline__ void load_codes(const TC* __restrict__ codes, uint64_t i0, uint64_t n, bool full,
                                           TC (&c)[4]) {
    if (full) {
        if (sizeof(TC) == 4) {
            const uint4 u = __ldcs(reinterpret_cast<const uint4*>(codes + i0));
            c[0] = (TC)u.x, c[1] = (TC)u.y, c[2] = (TC)u.z, c[3] = (TC)u.w;
        } else {
            const uint2 u = __ldcs(reinterpret_cast<const uint2*>(codes + i0));
            c[0] = (TC)(u.x & 0xffffu), c[1] = (TC)(u.x >> 16), c[2] = (TC)(u.y & 0xffffu), c[3] = (TC)(u.y >> 16);
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) c[j] = i0 + j < n ? codes[i0 + j] : (TC)0;
}

__device__ __forceinline__ void store_values(float* __restrict__ out, uint64_t i0, uint64_t n, bool full,
                                             const float (&y)[4]) {
    if (full) {
        __stcs(reinterpret_cast<float4*>(out + i0), make_float4(y[0], y[1], y[2], y[3]));
        return;
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (i0 + j < n) out[i0 + j] = y[j];
}

// One block per tile of 4096 codes (granule k*1024 + 4t in thread t); all
// loads are issued before any value is computed.  MODE 0 ABS/NOA, 1 REL,
// 2 in-place outliers.
template <typename TC, int MODE>
__global__ void __launch_bounds__(256) quantizer_inv_kernel(const TC* __restrict__ codes, uint64_t n, float ebx2,
                                                            float log2eb, int zigzag, uint32_t radius, int vec,
                                                            float* __restrict__ out) {
    const uint64_t base = (uint64_t)blockIdx.x * kQTile;
    const bool full = vec && base + kQTile <= n;
    TC c[4][4];
#pragma unroll
    for (int k = 0; k < 4; k++) load_codes(codes, base + (uint64_t)k * 1024 + 4 * threadIdx.x, n, full, c[k]);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float y[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            y[j] = MODE == 2 ? dequant_inplace((uint32_t)c[k][j], ebx2, radius)
                             : dequant_one<TC, MODE == 1>(c[k][j], ebx2, log2eb, zigzag);
        store_values(out, base + (uint64_t)k * 1024 + 4 * threadIdx.x, n, full, y);
    }
}

// out[idx[k]] = vals[k] for k < min(*count, cap); indices past n are skipped.
__global__ void __launch_bounds__(256) scatter_assign_kernel(const float* __restrict__ vals,
                                                             const uint32_t* __restrict__ idx,
                                                             const uint32_t* __restrict__ count, uint64_t cap,
                                                             uint64_t n, float* __restrict__ out) {
    const uint64_t m = *count < cap ? *count : cap;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride) {
        const uint32_t j = idx[k];
        if (j < n) out[j] = vals[k];
    }
}

// Workspace: [256 B control: word 0 device status (fzb_workspace_status),
// word 2 the value-range scan's completion counter, word 3 the outlier tile
// list length][group counts][min / max partials][tile counts][tile list].  The control block and the group counts are
// cleared by one memset per call.
struct QWork {
    uint32_t* err;
    uint32_t* mm_done;
    uint32_t* list_len;
    uint32_t* group_cnt;
    float* pmin;
    float* pmax;
    uint32_t* tile_cnt;
    uint32_t* list;
    size_t head;  // bytes cleared per call
    size_t need;
};

QWork carve_q(void* base, uint64_t n) {
    uint8_t* p = static_cast<uint8_t*>(base);
    const uint64_t ntiles = (n + kQTile - 1) / kQTile, ngroups = (ntiles + kQGroup - 1) / kQGroup;
    QWork w{};
    w.err = reinterpret_cast<uint32_t*>(p);
    w.mm_done = w.err ? w.err + 2 : nullptr;
    w.list_len = w.err ? w.err + 3 : nullptr;
    size_t off = 256;
    w.group_cnt = p ? reinterpret_cast<uint32_t*>(p + off) : nullptr;
    off += (ngroups * 4 + 255) / 256 * 256;
    w.head = off;
    w.pmin = p ? reinterpret_cast<float*>(p + off) : nullptr;
    off += kQMaxParts * 4;
    w.pmax = p ? reinterpret_cast<float*>(p + off) : nullptr;
    off += kQMaxParts * 4;
    w.tile_cnt = p ? reinterpret_cast<uint32_t*>(p + off) : nullptr;
    off += (ntiles * 4 + 255) / 256 * 256;
    w.list = p ? reinterpret_cast<uint32_t*>(p + off) : nullptr;
    off += (ntiles * 4 + 255) / 256 * 256;
    w.need = off;
    return w;
}

// REL parameters exactly as QuantizerStage::execute computes them on the host
// (quantizer.cu:566-571, inverse :423).
void rel_params(float eb, float* log2eb, float* log2eb_r, float* opp, float* oopp) {
    *log2eb = 2.0f * std::log2(1.0f + eb);
    *log2eb_r = 1.0f / *log2eb;
    *opp = 1.0f + eb;
    *oopp = 1.0f / *opp;
}

unsigned elem_grid(uint64_t n) {
    uint64_t g = (n + 255) / 256, cap = (uint64_t)device_sms() * 16;
    if (g > cap) g = cap;
    return (unsigned)(g ? g : 1);
}

}  // namespace
}  // namespace fzb

using namespace fzb;

extern "C" {

size_t fzb_quantizer_workspace_bytes(uint64_t n) { return carve_q(nullptr, n).need; }

int fzb_quantizer_forward(const float* d_in, uint64_t n, int code_bytes, float eb, int eb_mode, float value_base,
                          uint32_t radius, int zigzag, float threshold, int inplace, void* d_codes, float* d_ovals,
                          uint32_t* d_oidx, uint32_t* d_count, uint64_t cap, float* d_eb_state, void* d_work,
                          size_t work_bytes, void* stream) {
    if (code_bytes != 2 && code_bytes != 4) return FZB_E_INVALID;
    if (eb_mode != FZB_ABS && eb_mode != FZB_REL && eb_mode != FZB_NOA) return FZB_E_INVALID;
    if (n >= (1ull << 32) || !d_eb_state || (n && (!d_in || !d_codes))) return FZB_E_INVALID;
    const bool rel = eb_mode == FZB_REL;
    const bool inpl = inplace && !rel;  // REL always keeps outlier lists (quantizer.h:246-249)
    if (inpl && (!zigzag || code_bytes != 4)) return FZB_E_INVALID;  // quantizer.cu:602-611
    if (!inpl && (!d_count || (cap && (!d_ovals || !d_oidx)))) return FZB_E_INVALID;
    const QWork w = carve_q(d_work, n);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the stored radius is the TCode conversion of quant_radius
    const uint32_t R = code_bytes == 2 ? (uint32_t)(uint16_t)radius : radius;
    if (cudaMemsetAsync(d_work, 0, w.head, s) != cudaSuccess) return FZB_E_CUDA;
    if (n == 0) return (inpl || cudaMemsetAsync(d_count, 0, 4, s) == cudaSuccess) ? FZB_OK : FZB_E_CUDA;
    {
        TraceScope ts(s, "quantizer_resolve_eb");
        if (eb_mode == FZB_NOA && !(value_base > 0.0f)) {
            uint64_t parts = (n / 4 + 255) / 256, lim = (uint64_t)device_sms() * 7;
            if (parts > lim) parts = lim;
            if (parts > (uint64_t)kQMaxParts) parts = kQMaxParts;
            if (parts < 1) parts = 1;
            minmax_kernel<<<(unsigned)parts, 256, 0, s>>>(d_in, n, w.pmin, w.pmax, w.mm_done, FZB_NOA, eb, d_eb_state);
        } else {
            resolve_eb_kernel<<<1, 32, 0, s>>>(rel ? FZB_ABS : eb_mode, eb, value_base, d_eb_state);
        }
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    if (inpl) {
        TraceScope ts(s, "quantizer_fwd_inplace");
        quantizer_fwd_inplace_kernel<<<elem_grid(n), 256, 0, s>>>(d_in, n, d_eb_state, threshold, R,
                                                                  static_cast<uint32_t*>(d_codes));
        return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
    }
    QArgs a{};
    a.in = d_in;
    a.n = n;
    a.st = d_eb_state;
    rel_params(eb, &a.log2eb, &a.log2eb_r, &a.opp, &a.oopp);
    a.threshold = threshold;
    a.radius = R;
    a.zigzag = zigzag;
    a.codes = d_codes;
    a.ovals = d_ovals;
    a.oidx = d_oidx;
    a.count = d_count;
    a.cap = cap;
    a.tile_cnt = w.tile_cnt;
    a.group_cnt = w.group_cnt;
    a.list = w.list;
    a.list_len = w.list_len;
    a.ntiles = (uint32_t)((n + kQTile - 1) / kQTile);
    a.ngroups = (a.ntiles + kQGroup - 1) / kQGroup;
    a.vec = ((reinterpret_cast<uintptr_t>(d_in) & 15) == 0) &&
            ((reinterpret_cast<uintptr_t>(d_codes) & (uintptr_t)(4 * code_bytes - 1)) == 0);
    {
        TraceScope ts(s, "quantizer_fwd");
        if (code_bytes == 2) {
            if (rel) quantizer_codes_kernel<uint16_t, true><<<a.ntiles, kThreads, 0, s>>>(a);
            else quantizer_codes_kernel<uint16_t, false><<<a.ntiles, kThreads, 0, s>>>(a);
        } else {
            if (rel) quantizer_codes_kernel<uint32_t, true><<<a.ntiles, kThreads, 0, s>>>(a);
            else quantizer_codes_kernel<uint32_t, false><<<a.ntiles, kThreads, 0, s>>>(a);
        }
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    TraceScope ts(s, "quantizer_outliers");
    const unsigned og = a.ntiles < (uint32_t)device_sms() * 8 ? a.ntiles : (unsigned)device_sms() * 8;
    if (code_bytes == 2) {
        if (rel) quantizer_outliers_kernel<uint16_t, true><<<og, kThreads, 0, s>>>(a);
        else quantizer_outliers_kernel<uint16_t, false><<<og, kThreads, 0, s>>>(a);
    } else {
        if (rel) quantizer_outliers_kernel<uint32_t, true><<<og, kThreads, 0, s>>>(a);
        else quantizer_outliers_kernel<uint32_t, false><<<og, kThreads, 0, s>>>(a);
    }
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

int fzb_quantizer_inverse(const void* d_codes, uint64_t n, int code_bytes, float eb, int eb_mode, float abs_eb,
                          uint32_t radius, int zigzag, int inplace, const float* d_ovals, const uint32_t* d_oidx,
                          const uint32_t* d_count, uint64_t cap, float* d_out, void* stream) {
    if (code_bytes != 2 && code_bytes != 4) return FZB_E_INVALID;
    if (eb_mode != FZB_ABS && eb_mode != FZB_REL && eb_mode != FZB_NOA) return FZB_E_INVALID;
    if (n && (!d_codes || !d_out)) return FZB_E_INVALID;
    const bool rel = eb_mode == FZB_REL;
    const bool inpl = inplace && !rel;
    if (inpl && code_bytes != 4) return FZB_E_INVALID;
    if (!inpl && cap && (!d_ovals || !d_oidx || !d_count)) return FZB_E_INVALID;
    if (n == 0) return FZB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const float ebx2 = 2.0f * abs_eb;
    const uint32_t R = code_bytes == 2 ? (uint32_t)(uint16_t)radius : radius;
    float log2eb = 0.0f, r_, o_, oo_;
    rel_params(eb, &log2eb, &r_, &o_, &oo_);
    const uint64_t ntiles = (n + kQTile - 1) / kQTile;
    if (ntiles > 0x7fffffffull) return FZB_E_INVALID;
    const unsigned g = (unsigned)ntiles;
    const int vec = ((reinterpret_cast<uintptr_t>(d_out) & 15) == 0) &&
                    ((reinterpret_cast<uintptr_t>(d_codes) & (uintptr_t)(4 * code_bytes - 1)) == 0);
    TraceScope ts(s, "quantizer_inv");
    if (inpl) {
        quantizer_inv_kernel<uint32_t, 2><<<g, 256, 0, s>>>(static_cast<const uint32_t*>(d_codes), n, ebx2, log2eb,
                                                             zigzag, R, vec, d_out);
        return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
    }
    if (code_bytes == 2) {
        const uint16_t* c = static_cast<const uint16_t*>(d_codes);
        if (rel) quantizer_inv_kernel<uint16_t, 1><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, R, vec, d_out);
        else quantizer_inv_kernel<uint16_t, 0><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, R, vec, d_out);
    } else {
        const uint32_t* c = static_cast<const uint32_t*>(d_codes);
        if (rel) quantizer_inv_kernel<uint32_t, 1><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, R, vec, d_out);
        else quantizer_inv_kernel<uint32_t, 0><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, R, vec, d_out);
    }
    if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    if (cap) {
        uint64_t sg = (cap + 255) / 256;
        if (sg > 4096) sg = 4096;
        scatter_assign_kernel<<<(unsigned)sg, 256, 0, s>>>(d_ovals, d_oidx, d_count, cap, n, d_out);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    return FZB_OK;
}

}  // extern "C"
