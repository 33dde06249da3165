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
// Forward kernel: tiles of 2048 elements (256 threads x 8, element k*256 + t
// of the tile in thread t) taken in ticket order; codes are written
// coalesced; outlier slots come from per-(k, warp) ballot counts ordered by
// index and a decoupled look-back over the tiles' outlier counts.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "../../include/fzb.h"
#include "fzb_common.cuh"
#include "fzb_kernels.cuh"

namespace fzb {
namespace {

constexpr int kQPer = 8;
constexpr uint32_t kQTile = (uint32_t)kThreads * kQPer;  // 2048
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
    unsigned long long* status;
    uint32_t* ticket;
    uint32_t* err;
    uint32_t ntiles;
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

template <typename TC, bool REL>
__global__ void __launch_bounds__(kThreads) quantizer_fwd_kernel(QArgs a) {
    __shared__ uint32_t s_tile, s_total;
    __shared__ uint32_t s_off[kQPer * kQWarps];  // (k, warp) counts, then exclusive offsets
    __shared__ unsigned long long s_red[2 * kQWarps + 2];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_tile = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kQTile;
    const float ebx2_r = REL ? 0.0f : a.st[2];
    TC* codes = static_cast<TC*>(a.codes);
    float xv[kQPer];
#pragma unroll
    for (int k = 0; k < kQPer; k++) {
        const uint64_t i = base + (uint64_t)k * kThreads + t;
        xv[k] = i < a.n ? __ldcs(a.in + i) : 0.0f;
    }
    uint32_t om = 0;
#pragma unroll
    for (int k = 0; k < kQPer; k++) {
        const uint64_t i = base + (uint64_t)k * kThreads + t;
        if (i < a.n) {
            bool o;
            codes[i] = quantize_one<TC, REL>(a, xv[k], ebx2_r, o);
            om |= (o ? 1u : 0u) << k;
        }
    }
#pragma unroll
    for (int k = 0; k < kQPer; k++) {
        const uint32_t b = __ballot_sync(0xffffffffu, (om >> k) & 1u);
        if (lane == 0) s_off[k * kQWarps + warp] = __popc(b);
    }
    __syncthreads();
    if (warp == 0) {  // 64 (k, warp) entries in index order, two per lane
        const uint32_t c0 = s_off[2 * lane], c1 = s_off[2 * lane + 1];
        const uint32_t inc = warp_incl_scan(c0 + c1);
        const uint32_t ex = inc - c0 - c1;
        s_off[2 * lane] = ex;
        s_off[2 * lane + 1] = ex + c0;
        if (lane == 31) s_total = inc;
    }
    __syncthreads();
    const uint32_t total = s_total;
    const uint64_t prefix = lookback(a.status, tile, total, a.err, s_red);
    if (total) {
        const uint32_t below = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < kQPer; k++) {
            const uint32_t b = __ballot_sync(0xffffffffu, (om >> k) & 1u);
            if ((om >> k) & 1u) {
                const uint64_t slot = prefix + s_off[k * kQWarps + warp] + __popc(b & below);
                if (slot < a.cap) {
                    a.ovals[slot] = xv[k];
                    a.oidx[slot] = (uint32_t)(base + (uint64_t)k * kThreads + t);
                }
            }
        }
    }
    if (tile == a.ntiles - 1 && t == 0) {
        const uint64_t all = prefix + total;
        *a.count = (uint32_t)(all < a.cap ? all : a.cap);
    }
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
__global__ void __launch_bounds__(256) quantizer_inv_kernel(const TC* __restrict__ codes, uint64_t n, float ebx2,
                                                            float log2eb, int zigzag, float* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const TC c = codes[i];
        float v;
        if (!REL) {
            using S = typename std::make_signed<TC>::type;
            const int q = zigzag ? unzigzag_code<TC>(c) : (int)(S)c;
            v = (float)q * ebx2;
        } else if (c == 0) {
            v = 0.0f;
        } else {
            const uint32_t cv = (uint32_t)c - 1u;
            const int alb = (int)(cv >> 2);
            const int lb = ((cv >> 1) & 1u) ? -alb : alb;
            const float ar = exp2f((float)lb * log2eb);
            v = (cv & 1u) ? -ar : ar;
        }
        out[i] = v;
    }
}

__global__ void __launch_bounds__(256) quantizer_inv_inplace_kernel(const uint32_t* __restrict__ codes, uint64_t n,
                                                                    float ebx2, uint32_t radius,
                                                                    float* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t c = codes[i];
        if ((c >> 1) >= radius) {
            out[i] = __uint_as_float(c);
        } else {
            const int32_t ci = (int32_t)c;
            const int q = (ci & 1) ? -((ci + 1) >> 1) : (ci >> 1);
            out[i] = (float)q * ebx2;
        }
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

struct QWork {
    uint32_t* err;     // word 0: device status bits (read by fzb_workspace_status)
    uint32_t* ticket;  // word 1
    uint32_t* mm_done; // word 2
    float* pmin;
    float* pmax;
    unsigned long long* status;
    size_t need;
};

QWork carve_q(void* base, uint64_t n) {
    uint8_t* p = static_cast<uint8_t*>(base);
    const uint64_t ntiles = (n + kQTile - 1) / kQTile;
    QWork w{};
    w.err = reinterpret_cast<uint32_t*>(p);
    w.ticket = w.err ? w.err + 1 : nullptr;
    w.mm_done = w.err ? w.err + 2 : nullptr;
    size_t off = 256;
    w.pmin = p ? reinterpret_cast<float*>(p + off) : nullptr;
    off += kQMaxParts * 4;
    w.pmax = p ? reinterpret_cast<float*>(p + off) : nullptr;
    off += kQMaxParts * 4;
    w.status = p ? reinterpret_cast<unsigned long long*>(p + off) : nullptr;
    off += ((ntiles + 1) * 8 + 255) / 256 * 256;
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
    if (cudaMemsetAsync(d_work, 0, 256, s) != cudaSuccess) return FZB_E_CUDA;
    if (!inpl && cudaMemsetAsync(d_count, 0, 4, s) != cudaSuccess) return FZB_E_CUDA;
    if (n == 0) return FZB_OK;
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
    a.status = w.status;
    a.ticket = w.ticket;
    a.err = w.err;
    a.ntiles = (uint32_t)((n + kQTile - 1) / kQTile);
    if (cudaMemsetAsync(w.status, 0, (size_t)a.ntiles * 8, s) != cudaSuccess) return FZB_E_CUDA;
    TraceScope ts(s, "quantizer_fwd");
    if (code_bytes == 2) {
        if (rel) quantizer_fwd_kernel<uint16_t, true><<<a.ntiles, kThreads, 0, s>>>(a);
        else quantizer_fwd_kernel<uint16_t, false><<<a.ntiles, kThreads, 0, s>>>(a);
    } else {
        if (rel) quantizer_fwd_kernel<uint32_t, true><<<a.ntiles, kThreads, 0, s>>>(a);
        else quantizer_fwd_kernel<uint32_t, false><<<a.ntiles, kThreads, 0, s>>>(a);
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
    const unsigned g = elem_grid(n);
    TraceScope ts(s, "quantizer_inv");
    if (inpl) {
        quantizer_inv_inplace_kernel<<<g, 256, 0, s>>>(static_cast<const uint32_t*>(d_codes), n, ebx2, R, d_out);
        return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
    }
    if (code_bytes == 2) {
        const uint16_t* c = static_cast<const uint16_t*>(d_codes);
        if (rel) quantizer_inv_kernel<uint16_t, true><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, d_out);
        else quantizer_inv_kernel<uint16_t, false><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, d_out);
    } else {
        const uint32_t* c = static_cast<const uint32_t*>(d_codes);
        if (rel) quantizer_inv_kernel<uint32_t, true><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, d_out);
        else quantizer_inv_kernel<uint32_t, false><<<g, 256, 0, s>>>(c, n, ebx2, log2eb, zigzag, d_out);
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
