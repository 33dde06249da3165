// fzb_pfpl.cu -- the pfpl preset's chain in one pass per direction:
//   Quantizer<float, uint32_t> (quantizers/quantizer/quantizer.cu)
//   -> DifferenceStage<int32_t, uint32_t> with 16 KiB chunks (predictors/diff/diff.cu)
//   -> Bitshuffle(16384, ew 2) (shufflers/bitshuffle/bitshuffle_stage.cu)
//   -> RZE(16384, 4 levels) (coders/rze/rze_stage.cu)
// (examples/presets/pfpl.toml).  The stages' blocks line up: one 16 KiB RZE
// chunk is one Bitshuffle block and one Difference chunk of 4096 codes, so a
// CTA takes 4096 values, quantises them, differences and negabinary-codes
// them inside the chunk, transposes the 8192 half-words into bit planes and
// codes the chunk with RZE, without writing the codes to HBM.  Thread t owns
// values 16t..16t+15 of the chunk, which are half-words 32t..32t+31 of the
// Bitshuffle block: the layout the LorenzoQuant chain's chunk coder takes.
// Outliers are staged per chunk and assembled in chunk order (index order
// unless more than `cap` occur), as in the LorenzoQuant chain.
//
// The inverse decodes a chunk, undoes the bit transpose, negabinary and the
// chunk's prefix sum in registers and dequantises, then scatters the
// outliers.  Both directions give the bytes and values of the four stages
// run one after another.
//
// Built with the default floating-point contraction, like fzb_quant.cu: the
// REL codes come from __log2f and exp2f.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/fzb.h"
#include "fzb_common.cuh"
#include "fzb_kernels.cuh"

namespace fzb {
namespace {

constexpr uint32_t kPVals = 4096;  // values (u32 codes) per chunk
constexpr int kPSmem = 2 * kChunkBytes + 16 + 2048 + 256 + 32;
constexpr int kPMaxParts = 1024;

struct PArgs {
    const float* in;
    uint64_t n;
    uint32_t n_chunks;
    const float* st;  // resolved bound: [2] 1 / (2 abs_eb)
    float log2eb, log2eb_r, opp, oopp, threshold;
    int radius;
    int zigzag;
    uint8_t* slots;
    uint32_t* sizes;
    uint32_t* ostage_ctr;
    uint32_t* obase;
    uint32_t* ocnt;
    float* ostage_val;
    uint32_t* ostage_idx;
    uint32_t ostage_cap;
};

__device__ __forceinline__ uint32_t nb_enc32(uint32_t u) { return (u + 0xAAAAAAAAu) ^ 0xAAAAAAAAu; }
__device__ __forceinline__ uint32_t nb_dec32(uint32_t u) { return (u ^ 0xAAAAAAAAu) - 0xAAAAAAAAu; }

// QuantizerStage<float, uint32_t> code of one value (quantizer.cu:30-70,
// :232-327); `outlier` reports the outlier path (stored code 0).
template <bool REL>
__device__ __forceinline__ uint32_t pfpl_code(const PArgs& a, float x, float r, bool& outlier) {
    if (!REL) {
        const int q = __float2int_rn(x * r);
        outlier = !(q > -a.radius && q < a.radius && fabsf(x) < a.threshold);
        if (outlier) return 0u;
        return a.zigzag ? (((uint32_t)q << 1) ^ (uint32_t)(q >> 31)) : (uint32_t)q;
    }
    outlier = true;
    if (fabsf(x) >= a.threshold) return 0u;
    const int expo = (int)((__float_as_uint(x) >> 23) & 0xffu);
    if (expo == 0 || expo == 255) return 0u;
    const bool neg = x < 0.0f;
    const float ax = neg ? -x : x;
    const int lb = __float2int_rn(__log2f(ax) * a.log2eb_r);
    const uint32_t alb = (uint32_t)(lb < 0 ? -lb : lb);
    const uint32_t stored = ((alb << 2) | ((lb < 0 ? 1u : 0u) << 1) | (neg ? 1u : 0u)) + 1u;
    if (alb < (uint32_t)a.radius) {
        const float ar = exp2f((float)lb * a.log2eb);
        const float lo = ax * a.oopp, hi = ax * a.opp;
        if (ar >= lo && ar <= hi) {
            outlier = false;
            return stored;
        }
    }
    return 0u;
}

// A chunk's encoded bytes (S when stored raw, else O) to its 16 KiB slot,
// its size word to sizes[c] (the slot layout the assembly kernels read).
__device__ __forceinline__ void store_slot(uint8_t* __restrict__ slots, uint32_t* __restrict__ sizes, uint32_t c,
                                           uint32_t sw, const uint8_t* payload) {
    const uint32_t clean = sw & 0x7fffffffu;
    uint4* d4 = reinterpret_cast<uint4*>(slots + (size_t)c * kChunkBytes);
    const uint4* s4 = reinterpret_cast<const uint4*>(payload);
    for (uint32_t i = threadIdx.x; i < (clean + 15) / 16; i += kThreads) d4[i] = s4[i];
    if (threadIdx.x == 0) sizes[c] = sw;
}

template <bool REL>
__global__ void __launch_bounds__(kThreads, 5) pfpl_chunk_kernel(PArgs a) {
    extern __shared__ float4 smraw[];
    __shared__ uint32_t s_ws[16];
    __shared__ uint32_t s_last[kThreads / 32];
    __shared__ uint32_t s_obase;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t c = blockIdx.x;
    const uint64_t i0 = (uint64_t)c * kPVals;
    const uint32_t cnt = (uint32_t)min((uint64_t)kPVals, a.n - i0);
    const uint32_t e0 = 16u * t;
    const float r = REL ? 0.0f : a.st[2];

    float v[16];
    if (e0 + 16 <= cnt && (reinterpret_cast<uintptr_t>(a.in) & 15) == 0) {
        const float4* p = reinterpret_cast<const float4*>(a.in + i0 + e0);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float4 q = __ldcs(p + k);
            v[4 * k] = q.x, v[4 * k + 1] = q.y, v[4 * k + 2] = q.z, v[4 * k + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int e = 0; e < 16; e++) v[e] = (e0 + e < cnt) ? a.in[i0 + e0 + e] : 0.0f;
    }
    uint32_t q[16];
    uint32_t om = 0;
#pragma unroll
    for (int e = 0; e < 16; e++) {
        bool o;
        q[e] = pfpl_code<REL>(a, v[e], r, o);
        if (e0 + e >= cnt) q[e] = 0u, o = false;
        om |= (o ? 1u : 0u) << e;
    }
    // predecessor of this thread's first code (the chunk starts a new run)
    uint32_t prev = __shfl_up_sync(0xffffffffu, q[15], 1);
    if (lane == 31) s_last[warp] = q[15];
    __syncthreads();
    if (lane == 0) prev = warp ? s_last[warp - 1] : 0u;
    uint32_t d[16];
#pragma unroll
    for (int e = 0; e < 16; e++) {
        const uint32_t p = e ? q[e - 1] : prev;
        const uint32_t diff = (e0 + e == 0) ? q[e] : q[e] - p;
        d[e] = (e0 + e < cnt) ? nb_enc32(diff) : 0u;
    }

    // outliers: block scan, one staging allocation per chunk
    const uint32_t nout = __popc(om);
    uint32_t ototal;
    const uint32_t ooff = block_excl_scan(nout, s_ws, &ototal);
    if (t == 0) {
        const uint32_t b = ototal ? atomicAdd(a.ostage_ctr, ototal) : 0u;
        a.obase[c] = b;
        a.ocnt[c] = ototal;
        s_obase = b;
    }
    __syncthreads();
    if (nout) {
        uint32_t pos = s_obase + ooff;
#pragma unroll
        for (int e = 0; e < 16; e++) {
            if ((om >> e) & 1u) {
                if (pos < a.ostage_cap) {
                    a.ostage_val[pos] = v[e];
                    a.ostage_idx[pos] = (uint32_t)(i0 + e0 + e);
                }
                pos++;
            }
        }
    }

    // Bitshuffle (ew 2) of the chunk's 8192 half-words, then RZE
    uint8_t* base = reinterpret_cast<uint8_t*>(smraw);
    RzeSmem sm;
    sm.S = reinterpret_cast<uint32_t*>(base);
    sm.O = base + kChunkBytes;
    sm.bm1 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16);
    sm.bm2 = base + 2 * kChunkBytes + 16 + 2048;
    sm.bm3 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16 + 2048 + 256);
    sm.ws = s_ws;
    if (cnt == kPVals) {
        // x[l] = half-word l | half-word (16 + l) << 16 of this thread's 32
        uint32_t x[16];
#pragma unroll
        for (int l = 0; l < 8; l++) {
            x[2 * l] = __byte_perm(d[l], d[8 + l], 0x5410);
            x[2 * l + 1] = __byte_perm(d[l], d[8 + l], 0x7632);
        }
        transpose16x2(x);
#pragma unroll
        for (int b = 0; b < 16; b++) sm.S[(15 - b) * 256 + t] = x[b];
    } else {  // partial last block: Bitshuffle leaves it unchanged
#pragma unroll
        for (int e = 0; e < 16; e++) sm.S[16 * t + e] = d[e];
    }
    __syncthreads();
    const uint32_t sw = rze_encode_chunk(sm, (int)(4 * cnt));
    store_slot(a.slots, a.sizes, c, sw, (sw >> 31) ? reinterpret_cast<const uint8_t*>(sm.S) : sm.O);
}

__global__ void pfpl_cap_count_kernel(uint32_t* count, uint32_t cap) {
    if (*count > cap) *count = cap;
}

struct PDec {
    const uint8_t* rze;
    uint64_t rze_bytes;
    const unsigned long long* in_off;
    uint32_t n_chunks;
    uint32_t orig_bytes;
    uint64_t n;
    float ebx2, log2eb;
    int zigzag;
    float* out;
    uint32_t* err;
};

template <bool REL>
__device__ __forceinline__ float pfpl_value(uint32_t c, float ebx2, float log2eb, int zigzag) {
    if (!REL) {
        const int q = zigzag ? (int)((c >> 1) ^ (0u - (c & 1u))) : (int)c;
        return (float)q * ebx2;
    }
    if (c == 0) return 0.0f;
    const uint32_t cv = c - 1u;
    const int alb = (int)(cv >> 2);
    const int lb = ((cv >> 1) & 1u) ? -alb : alb;
    const float ar = exp2f((float)lb * log2eb);
    return (cv & 1u) ? -ar : ar;
}

template <bool REL>
__global__ void __launch_bounds__(kThreads, 3) pfpl_decode_kernel(PDec a) {
    extern __shared__ float4 smraw[];
    __shared__ uint32_t s_ws[16];
    const int t = threadIdx.x;
    const uint32_t c = blockIdx.x;
    uint8_t* base = reinterpret_cast<uint8_t*>(smraw);
    RzeDecSmem sm;
    sm.C = base;
    sm.S = reinterpret_cast<uint32_t*>(base + kChunkBytes + 16);
    sm.bm1 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16);
    sm.bm2 = base + 2 * kChunkBytes + 16 + 2048;
    sm.bm3 = base + 2 * kChunkBytes + 16 + 2048 + 256;
    sm.ws = s_ws;
    uint32_t e = reinterpret_cast<const uint32_t*>(a.rze + 8)[c];
    const int osz = (c + 1 < a.n_chunks) ? kChunkBytes : (int)(a.orig_bytes - c * (uint32_t)kChunkBytes);
    const uint64_t off = a.in_off[c];
    if (off + (e & 0x7fffffffu) > a.rze_bytes) {
        if (t == 0) atomicOr(a.err, kErrMalformed);
        e = 2;  // decode as zeros
    }
    rze_decode_chunk(a.rze + off, e, osz, sm, a.err);
    const uint32_t cnt = (uint32_t)osz / 4;
    const uint32_t e0 = 16u * t;
    uint32_t d[16];
    if (osz == kChunkBytes) {
        uint32_t x[16];
#pragma unroll
        for (int b = 0; b < 16; b++) x[b] = sm.S[(15 - b) * 256 + t];
        transpose16x2(x);
#pragma unroll
        for (int l = 0; l < 8; l++) {
            d[l] = __byte_perm(x[2 * l], x[2 * l + 1], 0x5410);
            d[8 + l] = __byte_perm(x[2 * l], x[2 * l + 1], 0x7632);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) d[k] = (e0 + k < cnt) ? sm.S[16 * t + k] : 0u;
    }
    // negabinary, then the chunk's inclusive prefix sum
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        run += nb_dec32(d[k]);
        d[k] = run;
    }
    uint32_t total;
    const uint32_t excl = block_excl_scan(run, s_ws, &total);
    const uint64_t i0 = (uint64_t)c * kPVals + e0;
    float y[16];
#pragma unroll
    for (int k = 0; k < 16; k++) y[k] = pfpl_value<REL>(d[k] + excl, a.ebx2, a.log2eb, a.zigzag);
    if (e0 + 16 <= cnt && (reinterpret_cast<uintptr_t>(a.out) & 15) == 0) {
        float4* p = reinterpret_cast<float4*>(a.out + i0);
#pragma unroll
        for (int k = 0; k < 4; k++) __stcs(p + k, make_float4(y[4 * k], y[4 * k + 1], y[4 * k + 2], y[4 * k + 3]));
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++)
            if (e0 + k < cnt && i0 + k < a.n) a.out[i0 + k] = y[k];
    }
}

__global__ void __launch_bounds__(256) pfpl_scatter_kernel(const float* __restrict__ vals,
                                                           const uint32_t* __restrict__ idx,
                                                           const uint32_t* __restrict__ count, uint64_t cap,
                                                           uint64_t n, float* __restrict__ out) {
    const uint64_t m = *count < cap ? *count : cap;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = idx[k];
        if (j < n) out[j] = vals[k];
    }
}

// Workspace of the compressor: [256 B control: word 0 device status, word 1
// outlier staging counter, word 2 value-range scan counter][min / max
// partials][payload offsets][outlier ends][sizes][outlier counts][outlier
// bases][chunk slots][staged outliers].
struct PWork {
    uint32_t* err;
    uint32_t* ostage_ctr;
    unsigned int* mm_done;
    float* pmin;
    float* pmax;
    unsigned long long* pay_off;
    uint32_t* ofin;
    uint32_t* sizes;
    uint32_t* ocnt;
    uint32_t* obase;
    uint8_t* slots;
    float* ostage_val;
    uint32_t* ostage_idx;
    size_t need;
};

inline size_t a256(size_t v) { return (v + 255) & ~(size_t)255; }

PWork carve_p(void* basep, uint64_t n, uint64_t cap) {
    const uint64_t nch = (n + kPVals - 1) / kPVals;
    uint8_t* p = static_cast<uint8_t*>(basep);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        uint8_t* q = p ? p + off : nullptr;
        off += a256(bytes);
        return q;
    };
    PWork w{};
    uint8_t* ctrl = take(256);
    w.err = reinterpret_cast<uint32_t*>(ctrl);
    w.ostage_ctr = ctrl ? w.err + 1 : nullptr;
    w.mm_done = ctrl ? reinterpret_cast<unsigned int*>(w.err + 2) : nullptr;
    w.pmin = reinterpret_cast<float*>(take(4 * kPMaxParts));
    w.pmax = reinterpret_cast<float*>(take(4 * kPMaxParts));
    w.pay_off = reinterpret_cast<unsigned long long*>(take(8 * (nch + 2)));
    w.ofin = reinterpret_cast<uint32_t*>(take(4 * (nch + 2)));
    w.sizes = reinterpret_cast<uint32_t*>(take(4 * (nch + 1)));
    w.ocnt = reinterpret_cast<uint32_t*>(take(4 * (nch + 1)));
    w.obase = reinterpret_cast<uint32_t*>(take(4 * (nch + 1)));
    w.slots = take(nch * (uint64_t)kChunkBytes);
    w.ostage_val = reinterpret_cast<float*>(take(4 * (cap + 1)));
    w.ostage_idx = reinterpret_cast<uint32_t*>(take(4 * (cap + 1)));
    w.need = off;
    return w;
}

void rel_params_p(float eb, float* log2eb, float* log2eb_r, float* opp, float* oopp) {
    *log2eb = 2.0f * std::log2(1.0f + eb);
    *log2eb_r = 1.0f / *log2eb;
    *opp = 1.0f + eb;
    *oopp = 1.0f / *opp;
}

}  // namespace
}  // namespace fzb

using namespace fzb;

extern "C" {

size_t fzb_pfpl_workspace_bytes(uint64_t n, uint64_t cap) { return carve_p(nullptr, n, cap).need; }

int fzb_pfpl_compress(const float* d_in, uint64_t n, float eb, int eb_mode, float value_base, uint32_t radius,
                      int zigzag, float threshold, float* d_ovals, uint32_t* d_oidx, uint64_t cap,
                      uint32_t* d_count, void* d_rze, uint64_t* d_rze_size, float* d_eb_state, void* d_work,
                      size_t work_bytes, void* stream) {
    if (!d_in || !d_rze || !d_rze_size || !d_count || !d_eb_state || n == 0 || n >= (1ull << 30)) return FZB_E_INVALID;
    if (eb_mode != FZB_ABS && eb_mode != FZB_REL && eb_mode != FZB_NOA) return FZB_E_INVALID;
    if (cap && (!d_ovals || !d_oidx)) return FZB_E_INVALID;
    if (cap >= 0xffffffffull) return FZB_E_INVALID;
    const PWork w = carve_p(d_work, n, cap);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool rel = eb_mode == FZB_REL;
    if (cudaMemsetAsync(d_work, 0, 256, s) != cudaSuccess) return FZB_E_CUDA;
    {
        TraceScope ts(s, "pfpl_resolve_eb");
        if (eb_mode == FZB_NOA && !(value_base > 0.0f)) {
            uint64_t parts = (n / 4 + 255) / 256, lim = (uint64_t)device_sms() * 7;
            if (parts > lim) parts = lim;
            if (parts > (uint64_t)kPMaxParts) parts = kPMaxParts;
            if (parts < 1) parts = 1;
            minmax_kernel<<<(unsigned)parts, 256, 0, s>>>(d_in, n, w.pmin, w.pmax, w.mm_done, FZB_NOA, eb, d_eb_state);
        } else {
            resolve_eb_kernel<<<1, 32, 0, s>>>(rel ? FZB_ABS : eb_mode, eb, value_base, d_eb_state);
        }
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    PArgs a{};
    a.in = d_in;
    a.n = n;
    a.n_chunks = (uint32_t)((n + kPVals - 1) / kPVals);
    a.st = d_eb_state;
    rel_params_p(eb, &a.log2eb, &a.log2eb_r, &a.opp, &a.oopp);
    a.threshold = threshold;
    a.radius = (int)radius;
    a.zigzag = zigzag;
    a.slots = w.slots;
    a.sizes = w.sizes;
    a.ostage_ctr = w.ostage_ctr;
    a.obase = w.obase;
    a.ocnt = w.ocnt;
    a.ostage_val = w.ostage_val;
    a.ostage_idx = w.ostage_idx;
    a.ostage_cap = (uint32_t)cap;
    {
        TraceScope ts(s, "pfpl_chunk");
        if (rel) pfpl_chunk_kernel<true><<<a.n_chunks, kThreads, kPSmem, s>>>(a);
        else pfpl_chunk_kernel<false><<<a.n_chunks, kThreads, kPSmem, s>>>(a);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    AsmArgs m{};
    m.slots = w.slots;
    m.sizes = w.sizes;
    m.n_chunks = a.n_chunks;
    m.orig_bytes = (uint32_t)(4 * n);
    m.out = static_cast<uint8_t*>(d_rze);
    m.out_size = reinterpret_cast<unsigned long long*>(d_rze_size);
    m.pay_off = w.pay_off;
    m.ocnt = w.ocnt;
    m.obase = w.obase;
    m.ofin = w.ofin;
    m.ostage_err = w.ostage_val;
    m.ostage_idx = w.ostage_idx;
    m.ostage_cap = (uint32_t)cap;
    m.out_err = d_ovals;
    m.out_idx = d_oidx;
    m.cap = (uint32_t)cap;
    m.out_count = d_count;
    {
        TraceScope ts(s, "assemble_scan");
        if (launch_assemble_scan(m, s) != 0) return FZB_E_CUDA;
    }
    {
        TraceScope ts(s, "assemble_copy");
        unsigned g = a.n_chunks < 4u * (unsigned)device_sms() * 8u ? a.n_chunks : 4u * (unsigned)device_sms() * 8u;
        assemble_copy_kernel<<<g, 256, 0, s>>>(m);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    pfpl_cap_count_kernel<<<1, 1, 0, s>>>(d_count, (uint32_t)cap);
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

size_t fzb_pfpl_decompress_workspace_bytes(uint64_t n) {
    const uint64_t nch = (n + kPVals - 1) / kPVals;
    return 256 + a256(8 * (nch + 2));
}

int fzb_pfpl_decompress(const void* d_rze, uint64_t rze_bytes, const float* d_ovals, const uint32_t* d_oidx,
                        const uint32_t* d_count, uint64_t cap, uint64_t n, float eb, int eb_mode, float abs_eb,
                        int zigzag, float* d_out, void* d_work, size_t work_bytes, void* stream) {
    if (!d_rze || !d_out || n == 0 || n >= (1ull << 30)) return FZB_E_INVALID;
    if (eb_mode != FZB_ABS && eb_mode != FZB_REL && eb_mode != FZB_NOA) return FZB_E_INVALID;
    if (cap && (!d_ovals || !d_oidx || !d_count)) return FZB_E_INVALID;
    if (!d_work || work_bytes < fzb_pfpl_decompress_workspace_bytes(n)) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* err = static_cast<uint32_t*>(d_work);
    unsigned long long* in_off = reinterpret_cast<unsigned long long*>(static_cast<uint8_t*>(d_work) + 256);
    const uint32_t nch = (uint32_t)((n + kPVals - 1) / kPVals);
    if (cudaMemsetAsync(d_work, 0, 256, s) != cudaSuccess) return FZB_E_CUDA;
    {
        TraceScope ts(s, "rze_prepass");
        if (launch_rze_prepass(static_cast<const uint8_t*>(d_rze), rze_bytes, nch, (uint32_t)(4 * n), in_off, err,
                               s) != 0)
            return FZB_E_CUDA;
    }
    PDec a{};
    a.rze = static_cast<const uint8_t*>(d_rze);
    a.rze_bytes = rze_bytes;
    a.in_off = in_off;
    a.n_chunks = nch;
    a.orig_bytes = (uint32_t)(4 * n);
    a.n = n;
    a.ebx2 = 2.0f * abs_eb;
    float r_, o_, oo_;
    rel_params_p(eb, &a.log2eb, &r_, &o_, &oo_);
    a.zigzag = zigzag;
    a.out = d_out;
    a.err = err;
    {
        TraceScope ts(s, "pfpl_decode");
        if (eb_mode == FZB_REL) pfpl_decode_kernel<true><<<nch, kThreads, kPSmem, s>>>(a);
        else pfpl_decode_kernel<false><<<nch, kThreads, kPSmem, s>>>(a);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    if (cap) {
        uint64_t sg = (cap + 255) / 256;
        if (sg > 4096) sg = 4096;
        pfpl_scatter_kernel<<<(unsigned)sg, 256, 0, s>>>(d_ovals, d_oidx, d_count, cap, n, d_out);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    return FZB_OK;
}

}  // extern "C"
