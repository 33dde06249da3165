// fzb_transforms.cu -- the integer stages that sit around the quantisation
// codes in the shipped pipelines:
//   Zigzag      (transforms/zigzag/zigzag.h:33-57, zigzag_stage.cu:19-96)
//   Negabinary  (transforms/negabinary/negabinary.h:30-56, negabinary_stage.cu)
//   Difference  (predictors/diff/diff.cu:26-220): first differences inside
//               power-of-two chunks, optionally negabinary-coded; inverse is a
//               chunked inclusive prefix sum
//   Lorenzo     (predictors/lorenzo/lorenzo_stage.cu:18-400): lossless
//               integer Lorenzo deltas; 1-D inside 256-element blocks, 2-D
//               and 3-D inclusion-exclusion over the whole field; inverse is
//               the matching prefix sums (x, then y, then z)
// All arithmetic is on the unsigned bit pattern modulo 2^(8*width), which is
// what the reference's signed arithmetic produces on two's-complement
// hardware, so every result is bit-exact and independent of summation order.
//
// Scans.  A segmented inclusive scan over a flat array runs in tiles of 4096
// elements (256 threads x 16).  When every tile begins a segment (segment
// length divides 4096: the 1-D Lorenzo blocks, the 16 KiB Difference chunks
// of int32 data) one kernel does it.  Otherwise a reduce / carry / apply
// sequence carries (value, has-start) pairs between tiles with the segmented
// operator (a, b) -> (b.start ? b.v : a.v + b.v, a.start | b.start).  Scans
// along y and z (stride nx or nx*ny) run one thread per column over 64-row
// tiles, with the same three-phase carry when a column is longer than 64.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "../../include/fzb.h"
#include "fzb_kernels.cuh"

namespace fzb {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanPer = 16;
constexpr uint64_t kScanTile = (uint64_t)kScanThreads * kScanPer;  // 4096
constexpr int kColThreads = 256;
constexpr uint64_t kColRows = 64;

// Accumulator: 32-bit for widths up to 4 bytes (sums mod 2^32 truncate to the
// element width), 64-bit for 8-byte elements.
template <typename U>
using Acc = typename std::conditional<sizeof(U) == 8, uint64_t, uint32_t>::type;

template <typename U>
__device__ __forceinline__ U zz_enc(U u) {
    using S = typename std::make_signed<U>::type;
    return (U)((U)(u << 1) ^ (U)((S)u >> (sizeof(U) * 8 - 1)));
}
template <typename U>
__device__ __forceinline__ U zz_dec(U u) {
    return (U)((U)(u >> 1) ^ (U)(0 - (u & 1)));
}
template <typename U>
__device__ __forceinline__ U nb_mask() {
    return (U)0xAAAAAAAAAAAAAAAAull;
}
template <typename U>
__device__ __forceinline__ U nb_enc(U u) {
    return (U)((U)(u + nb_mask<U>()) ^ nb_mask<U>());
}
template <typename U>
__device__ __forceinline__ U nb_dec(U u) {
    return (U)((U)(u ^ nb_mask<U>()) - nb_mask<U>());
}

enum { kZzEnc = 0, kZzDec = 1, kNbEnc = 2, kNbDec = 3 };

template <typename U, int OP>
__device__ __forceinline__ U apply_op(U v) {
    if (OP == kZzEnc) return zz_enc(v);
    if (OP == kZzDec) return zz_dec(v);
    if (OP == kNbEnc) return nb_enc(v);
    return nb_dec(v);
}

template <typename U>
union Granule {
    uint4 q;
    U e[16 / sizeof(U)];
};

// ------------------------------------------------------------ elementwise

// in == out is allowed (each element is read before it is written by the
// same thread).
template <typename U, int OP>
__global__ void __launch_bounds__(256) xform_kernel(const U* in, U* out, uint64_t n, int vec) {
    constexpr int kPer = 16 / sizeof(U);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t done = 0;
    if (vec) {
        const uint64_t nv = n / kPer;
        for (uint64_t g = t; g < nv; g += stride) {
            Granule<U> b;
            b.q = reinterpret_cast<const uint4*>(in)[g];
#pragma unroll
            for (int k = 0; k < kPer; k++) b.e[k] = apply_op<U, OP>(b.e[k]);
            reinterpret_cast<uint4*>(out)[g] = b.q;
        }
        done = nv * kPer;
    }
    for (uint64_t i = done + t; i < n; i += stride) out[i] = apply_op<U, OP>(in[i]);
}

// Difference forward: out[i] = in[i] - in[i-1], except at i = 0 and at
// multiples of the power-of-two chunk (cmask = chunk - 1; 0 chunk -> no
// boundaries but i = 0), optionally negabinary-coded.  in != out.
template <typename U, bool NB>
__global__ void __launch_bounds__(256) diff_fwd_kernel(const U* __restrict__ in, U* __restrict__ out, uint64_t n,
                                                       uint64_t chunk, int vec) {
    constexpr int kPer = 16 / sizeof(U);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t cmask = chunk ? chunk - 1 : ~0ull;
    uint64_t done = 0;
    if (vec) {
        const uint64_t nv = n / kPer;
        for (uint64_t g = t; g < nv; g += stride) {
            Granule<U> b, o;
            b.q = reinterpret_cast<const uint4*>(in)[g];
            const uint64_t i0 = g * kPer;
            U prev = i0 ? in[i0 - 1] : (U)0;
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const uint64_t i = i0 + k;
                const bool start = (i == 0) || (chunk && (i & cmask) == 0);
                const U d = start ? b.e[k] : (U)(b.e[k] - prev);
                o.e[k] = NB ? nb_enc(d) : d;
                prev = b.e[k];
            }
            reinterpret_cast<uint4*>(out)[g] = o.q;
        }
        done = nv * kPer;
    }
    for (uint64_t i = done + t; i < n; i += stride) {
        const bool start = (i == 0) || (chunk && (i & cmask) == 0);
        const U d = start ? in[i] : (U)(in[i] - in[i - 1]);
        out[i] = NB ? nb_enc(d) : d;
    }
}

// 1-D Lorenzo delta inside 256-element blocks (lorenzo_stage.cu:23-33).
template <typename U>
__global__ void __launch_bounds__(256) lorenzo1_fwd_kernel(const U* __restrict__ in, U* __restrict__ out,
                                                           uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = (U)(in[i] - ((i & 255) ? in[i - 1] : (U)0));
}

// 2-D / 3-D Lorenzo delta (lorenzo_stage.cu:100-118, :215-243).  One block
// covers 256 x-positions of one row; row r = z * ny + y.
template <typename U>
__global__ void __launch_bounds__(256) lorenzo_nd_fwd_kernel(const U* __restrict__ in, U* __restrict__ out,
                                                             uint64_t nx, uint64_t ny, uint32_t xtiles) {
    const uint32_t row = blockIdx.x / xtiles;
    const uint64_t x = (uint64_t)(blockIdx.x - row * xtiles) * 256 + threadIdx.x;
    if (x >= nx) return;
    const uint64_t y = row % ny, z = row / ny;
    const uint64_t sy = nx, sz = nx * ny;
    const uint64_t i = z * sz + y * nx + x;
    using A = Acc<U>;
    const bool hx = x > 0, hy = y > 0, hz = z > 0;
    A v = (A)in[i];
    if (hx) v -= (A)in[i - 1];
    if (hy) v -= (A)in[i - sy];
    if (hx && hy) v += (A)in[i - sy - 1];
    if (hz) {
        v -= (A)in[i - sz];
        if (hx) v += (A)in[i - sz - 1];
        if (hy) v += (A)in[i - sz - sy];
        if (hx && hy) v -= (A)in[i - sz - sy - 1];
    }
    out[i] = (U)v;
}

// ------------------------------------------------------------ segmented scan

struct SegScan {
    const void* in;
    void* out;
    uint64_t n;
    uint64_t seg;        // segment length (0: one segment)
    int vec;             // 16-byte aligned in and out
    void* tile_v;        // Acc per tile: aggregate, then exclusive carry
    uint32_t* tile_f;    // per tile: a segment starts inside
};

template <typename U>
__device__ __forceinline__ void load_run(const U* p, uint64_t i0, uint64_t n, bool vec, U (&x)[kScanPer]) {
    if (vec && i0 + kScanPer <= n) {
        constexpr int NQ = kScanPer * sizeof(U) / 16;
        union {
            uint4 q[NQ];
            U e[kScanPer];
        } b;
        const uint4* q = reinterpret_cast<const uint4*>(p + i0);
#pragma unroll
        for (int j = 0; j < NQ; j++) b.q[j] = q[j];
#pragma unroll
        for (int k = 0; k < kScanPer; k++) x[k] = b.e[k];
    } else {
#pragma unroll
        for (int k = 0; k < kScanPer; k++) x[k] = (i0 + k < n) ? p[i0 + k] : (U)0;
    }
}

template <typename U>
__device__ __forceinline__ void store_run(U* p, uint64_t i0, uint64_t n, bool vec, const U (&x)[kScanPer]) {
    if (vec && i0 + kScanPer <= n) {
        constexpr int NQ = kScanPer * sizeof(U) / 16;
        union {
            uint4 q[NQ];
            U e[kScanPer];
        } b;
#pragma unroll
        for (int k = 0; k < kScanPer; k++) b.e[k] = x[k];
        uint4* q = reinterpret_cast<uint4*>(p + i0);
#pragma unroll
        for (int j = 0; j < NQ; j++) q[j] = b.q[j];
    } else {
#pragma unroll
        for (int k = 0; k < kScanPer; k++)
            if (i0 + k < n) p[i0 + k] = x[k];
    }
}

// Exclusive segmented scan of one (v, f) pair per thread across the block;
// also returns the block aggregate.  sv / sf: one slot per warp.
template <typename A>
__device__ __forceinline__ void block_seg_scan(A v, uint32_t f, A& ev, uint32_t& ef, A& tv, uint32_t& tf, A* sv,
                                               uint32_t* sf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    A iv = v;
    uint32_t ifl = f;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const A pv = __shfl_up_sync(0xffffffffu, iv, d);
        const uint32_t pf = __shfl_up_sync(0xffffffffu, ifl, d);
        if (lane >= d) {
            if (!ifl) iv = (A)(pv + iv);
            ifl |= pf;
        }
    }
    if (lane == 31) {
        sv[warp] = iv;
        sf[warp] = ifl;
    }
    A xv = __shfl_up_sync(0xffffffffu, iv, 1);
    uint32_t xf = __shfl_up_sync(0xffffffffu, ifl, 1);
    if (lane == 0) {
        xv = 0;
        xf = 0;
    }
    __syncthreads();
    A wv = 0;
    uint32_t wf = 0;
    for (int w = 0; w < nw; w++) {
        if (w == warp) {
            ev = xf ? xv : (A)(wv + xv);
            ef = wf | xf;
        }
        wv = sf[w] ? sv[w] : (A)(wv + sv[w]);
        wf |= sf[w];
    }
    tv = wv;
    tf = wf;
    __syncthreads();
}

// PHASE 0: one-pass scan (every tile starts a segment) or apply with the
// tile carries; PHASE 1: tile aggregates only.
template <typename U, bool NB, int PHASE>
__global__ void __launch_bounds__(kScanThreads, 4) segscan_kernel(SegScan a) {
    using A = Acc<U>;
    __shared__ A sv[kScanThreads / 32];
    __shared__ uint32_t sf[kScanThreads / 32];
    const uint64_t tile = blockIdx.x;
    const uint64_t i0 = tile * kScanTile + (uint64_t)threadIdx.x * kScanPer;
    U x[kScanPer];
    load_run(static_cast<const U*>(a.in), i0, a.n, a.vec, x);
    // starts: i % seg == 0 (seg == 0: only i == 0)
    uint64_t r = a.seg ? i0 % a.seg : i0;
    A acc = 0;
    uint32_t smask = 0;  // bit k: a start at or before element k in this run
    uint32_t any = 0;
    A loc[kScanPer];
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        const bool st = (r == 0) && (i0 + k < a.n);
        const A v = (A)(NB ? nb_dec(x[k]) : x[k]);
        acc = st ? v : (A)(acc + v);
        any |= st ? 1u : 0u;
        smask |= any << k;
        loc[k] = acc;
        if (a.seg) {
            if (++r == a.seg) r = 0;
        } else {
            r = 1;
        }
    }
    A ev, tv;
    uint32_t ef, tf;
    block_seg_scan<A>(acc, any, ev, ef, tv, tf, sv, sf);
    if (PHASE == 1) {
        if (threadIdx.x == 0) {
            static_cast<A*>(a.tile_v)[tile] = tv;
            a.tile_f[tile] = tf;
        }
        return;
    }
    const A carry = a.tile_v ? static_cast<const A*>(a.tile_v)[tile] : (A)0;
    // elements with no start before them in the tile take the tile carry
    const A pre = ef ? ev : (A)(carry + ev);
#pragma unroll
    for (int k = 0; k < kScanPer; k++) x[k] = (U)(((smask >> k) & 1) ? loc[k] : (A)(pre + loc[k]));
    store_run(static_cast<U*>(a.out), i0, a.n, a.vec, x);
}

// Tile aggregates -> exclusive carries, one block of 1024 threads walking the
// tile list in rounds.
template <typename A>
__global__ void __launch_bounds__(1024) segscan_carry_kernel(A* tv, uint32_t* tf, uint64_t ntiles) {
    __shared__ A sv[32];
    __shared__ uint32_t sf[32];
    A rv = 0;
    uint32_t rf = 0;
    for (uint64_t base = 0; base < ntiles; base += 1024) {
        const uint64_t i = base + threadIdx.x;
        const A v = i < ntiles ? tv[i] : (A)0;
        const uint32_t f = i < ntiles ? tf[i] : 0u;
        A ev, tot;
        uint32_t ef, totf;
        block_seg_scan<A>(v, f, ev, ef, tot, totf, sv, sf);
        if (i < ntiles) tv[i] = ef ? ev : (A)(rv + ev);
        rv = totf ? tot : (A)(rv + tot);
        rf |= totf;
    }
}

// ------------------------------------------------------------ column scan

struct ColScan {
    void* data;       // scanned in place
    uint64_t s;       // stride between consecutive elements of a column
    uint64_t L;       // column length
    uint64_t nlt;     // 64-row tiles per column
    uint64_t ncg;     // 256-column groups
    void* tot;        // [outer][nlt][s] tile totals, then exclusive carries
};

// PHASE 0: apply (carry from tot when nlt > 1); PHASE 1: tile totals.
template <typename U, int PHASE>
__global__ void __launch_bounds__(kColThreads) colscan_kernel(ColScan a) {
    using A = Acc<U>;
    uint64_t b = blockIdx.x;
    const uint64_t cg = b % a.ncg;
    b /= a.ncg;
    const uint64_t lt = b % a.nlt, o = b / a.nlt;
    const uint64_t c = cg * kColThreads + threadIdx.x;
    if (c >= a.s) return;
    const uint64_t l0 = lt * kColRows, l1 = (l0 + kColRows < a.L) ? l0 + kColRows : a.L;
    U* p = static_cast<U*>(a.data) + o * a.L * a.s + c;
    A* tot = static_cast<A*>(a.tot);
    const uint64_t ti = (o * a.nlt + lt) * a.s + c;
    A acc = (PHASE == 0 && a.nlt > 1) ? tot[ti] : (A)0;
    for (uint64_t l = l0; l < l1; l += 8) {
        U v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = (l + k < l1) ? p[(l + k) * a.s] : (U)0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            acc = (A)(acc + (A)v[k]);
            if (PHASE == 0 && l + k < l1) p[(l + k) * a.s] = (U)acc;
        }
    }
    if (PHASE == 1) tot[ti] = acc;
}

// Per (outer, column): tile totals -> exclusive carries.
template <typename A>
__global__ void __launch_bounds__(256) colscan_carry_kernel(A* tot, uint64_t s, uint64_t nlt, uint64_t lines) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= lines) return;
    const uint64_t o = t / s, c = t - o * s;
    A run = 0;
    for (uint64_t lt = 0; lt < nlt; lt++) {
        const uint64_t i = (o * nlt + lt) * s + c;
        const A v = tot[i];
        tot[i] = run;
        run = (A)(run + v);
    }
}

// ------------------------------------------------------------ host helpers

unsigned grid_for(uint64_t items, int per_sm) {
    const uint64_t cap = (uint64_t)device_sms() * per_sm;
    uint64_t g = (items + 255) / 256;
    if (g > cap) g = cap;
    return (unsigned)(g ? g : 1);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

uint64_t round_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

struct ScanWork {
    void* tile_v;
    uint32_t* tile_f;
    void* col;
    size_t need;
};

ScanWork carve_scan(void* base, uint64_t n) {
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    uint8_t* p = static_cast<uint8_t*>(base);
    ScanWork w{};
    size_t off = 0;
    w.tile_v = p ? p + off : nullptr;
    off += round_up(ntiles * 8 + 8, 256);
    w.tile_f = p ? reinterpret_cast<uint32_t*>(p + off) : nullptr;
    off += round_up(ntiles * 4 + 4, 256);
    w.col = p ? p + off : nullptr;
    off += round_up((n / 32 + 2) * 8, 256);
    w.need = off;
    return w;
}

template <typename U, bool NB>
int seg_scan(const void* in, void* out, uint64_t n, uint64_t seg, const ScanWork& w, cudaStream_t s) {
    if (n == 0) return FZB_OK;
    using A = Acc<U>;
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles > 0x7fffffffull) return FZB_E_INVALID;
    SegScan a{in, out, n, seg, (aligned16(in) && aligned16(out)) ? 1 : 0, nullptr, nullptr};
    const bool local = seg && (kScanTile % seg == 0);
    if (!local && ntiles > 1) {
        a.tile_v = w.tile_v;
        a.tile_f = w.tile_f;
        segscan_kernel<U, NB, 1><<<(unsigned)ntiles, kScanThreads, 0, s>>>(a);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
        segscan_carry_kernel<A><<<1, 1024, 0, s>>>(static_cast<A*>(w.tile_v), w.tile_f, ntiles);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    segscan_kernel<U, NB, 0><<<(unsigned)ntiles, kScanThreads, 0, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

// In-place inclusive scan along an axis of stride `stride` and length L,
// repeated over `outer` blocks of L * stride elements.
template <typename U>
int col_scan(void* data, uint64_t stride, uint64_t L, uint64_t outer, const ScanWork& w, cudaStream_t s) {
    using A = Acc<U>;
    if (L <= 1 || stride == 0 || outer == 0) return FZB_OK;
    ColScan a{data, stride, L, (L + kColRows - 1) / kColRows, (stride + kColThreads - 1) / kColThreads, w.col};
    const uint64_t blocks = outer * a.nlt * a.ncg;
    if (blocks > 0x7fffffffull) return FZB_E_INVALID;
    if (a.nlt > 1) {
        colscan_kernel<U, 1><<<(unsigned)blocks, kColThreads, 0, s>>>(a);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
        const uint64_t lines = outer * stride;
        colscan_carry_kernel<A><<<(unsigned)((lines + 255) / 256), 256, 0, s>>>(static_cast<A*>(w.col), stride,
                                                                                 a.nlt, lines);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    colscan_kernel<U, 0><<<(unsigned)blocks, kColThreads, 0, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

template <typename U, int OP>
int run_xform(const void* in, void* out, uint64_t n, cudaStream_t s) {
    if (n == 0) return FZB_OK;
    const int vec = aligned16(in) && aligned16(out);
    const uint64_t items = vec ? (n * sizeof(U) + 15) / 16 : n;
    xform_kernel<U, OP><<<grid_for(items, 16), 256, 0, s>>>(static_cast<const U*>(in), static_cast<U*>(out), n, vec);
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

template <int OP>
int xform_dispatch(const void* in, uint64_t n, int ew, void* out, cudaStream_t s) {
    switch (ew) {
        case 1: return run_xform<uint8_t, OP>(in, out, n, s);
        case 2: return run_xform<uint16_t, OP>(in, out, n, s);
        case 4: return run_xform<uint32_t, OP>(in, out, n, s);
        case 8: return run_xform<uint64_t, OP>(in, out, n, s);
        default: return FZB_E_INVALID;
    }
}

template <typename U>
int diff_typed(const void* in, uint64_t n, uint64_t chunk, int nb, int inverse, void* out, const ScanWork& w,
               cudaStream_t s) {
    if (!inverse) {
        const int vec = aligned16(in) && aligned16(out);
        const uint64_t items = vec ? (n * sizeof(U) + 15) / 16 : n;
        const unsigned g = grid_for(items, 16);
        if (nb)
            diff_fwd_kernel<U, true><<<g, 256, 0, s>>>(static_cast<const U*>(in), static_cast<U*>(out), n, chunk, vec);
        else
            diff_fwd_kernel<U, false><<<g, 256, 0, s>>>(static_cast<const U*>(in), static_cast<U*>(out), n, chunk, vec);
        return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
    }
    return nb ? seg_scan<U, true>(in, out, n, chunk, w, s) : seg_scan<U, false>(in, out, n, chunk, w, s);
}

template <typename U>
int lorenzo_typed(const void* in, const uint64_t d[3], uint64_t n, int inverse, void* out, const ScanWork& w,
                  cudaStream_t s) {
    const uint64_t nx = d[0], ny = d[1], nz = d[2];
    const int ndim = nz > 1 ? 3 : (ny > 1 ? 2 : 1);
    if (ndim == 1) {
        if (!inverse) {
            lorenzo1_fwd_kernel<U><<<grid_for(n, 16), 256, 0, s>>>(static_cast<const U*>(in), static_cast<U*>(out), n);
            return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
        }
        return seg_scan<U, false>(in, out, n, 256, w, s);
    }
    const uint64_t nfield = nx * ny * nz;
    if (!inverse) {
        const uint64_t xtiles = (nx + 255) / 256, blocks = xtiles * ny * nz;
        if (blocks > 0x7fffffffull) return FZB_E_INVALID;
        lorenzo_nd_fwd_kernel<U><<<(unsigned)blocks, 256, 0, s>>>(static_cast<const U*>(in), static_cast<U*>(out), nx,
                                                                  ny, (uint32_t)xtiles);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    } else {
        int rc = seg_scan<U, false>(in, out, nfield, nx, w, s);
        if (rc == FZB_OK) rc = col_scan<U>(out, nx, ny, nz, w, s);
        if (rc == FZB_OK && ndim == 3) rc = col_scan<U>(out, nx * ny, nz, 1, w, s);
        if (rc != FZB_OK) return rc;
    }
    // elements past the field pass through unchanged
    if (n > nfield && in != out &&
        cudaMemcpyAsync(static_cast<U*>(out) + nfield, static_cast<const U*>(in) + nfield, (n - nfield) * sizeof(U),
                        cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return FZB_E_CUDA;
    return FZB_OK;
}

}  // namespace
}  // namespace fzb

using namespace fzb;

extern "C" {

int fzb_zigzag(const void* d_in, uint64_t n, int elem_bytes, int inverse, void* d_out, void* stream) {
    if ((!d_in || !d_out) && n) return FZB_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    TraceScope ts(s, "zigzag");
    return inverse ? xform_dispatch<kZzDec>(d_in, n, elem_bytes, d_out, s)
                   : xform_dispatch<kZzEnc>(d_in, n, elem_bytes, d_out, s);
}

int fzb_negabinary(const void* d_in, uint64_t n, int elem_bytes, int inverse, void* d_out, void* stream) {
    if ((!d_in || !d_out) && n) return FZB_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    TraceScope ts(s, "negabinary");
    return inverse ? xform_dispatch<kNbDec>(d_in, n, elem_bytes, d_out, s)
                   : xform_dispatch<kNbEnc>(d_in, n, elem_bytes, d_out, s);
}

size_t fzb_scan_workspace_bytes(uint64_t n, int elem_bytes) {
    (void)elem_bytes;
    return carve_scan(nullptr, n).need;
}

int fzb_diff(const void* d_in, uint64_t n, int elem_bytes, uint64_t chunk_elems, int negabinary, int inverse,
             void* d_out, void* d_work, size_t work_bytes, void* stream) {
    if ((!d_in || !d_out) && n) return FZB_E_INVALID;
    if (chunk_elems & (chunk_elems - 1)) return FZB_E_INVALID;  // diff.cu:116-117: power of two
    if (!inverse && d_in == d_out && n) return FZB_E_INVALID;
    if (n == 0) return FZB_OK;
    const ScanWork w = carve_scan(d_work, n);
    if (inverse && (!d_work || work_bytes < w.need)) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    TraceScope ts(s, inverse ? "diff_inv" : "diff_fwd");
    switch (elem_bytes) {
        case 1: return diff_typed<uint8_t>(d_in, n, chunk_elems, negabinary, inverse, d_out, w, s);
        case 2: return diff_typed<uint16_t>(d_in, n, chunk_elems, negabinary, inverse, d_out, w, s);
        case 4: return diff_typed<uint32_t>(d_in, n, chunk_elems, negabinary, inverse, d_out, w, s);
        case 8: return diff_typed<uint64_t>(d_in, n, chunk_elems, negabinary, inverse, d_out, w, s);
        default: return FZB_E_INVALID;
    }
}

int fzb_lorenzo_int(const void* d_in, const uint64_t dims[3], uint64_t n, int elem_bytes, int inverse, void* d_out,
                    void* d_work, size_t work_bytes, void* stream) {
    if (!dims || ((!d_in || !d_out) && n)) return FZB_E_INVALID;
    uint64_t d[3] = {dims[0] ? dims[0] : n, dims[1] ? dims[1] : 1, dims[2] ? dims[2] : 1};
    const bool nd = d[1] > 1 || d[2] > 1;
    if (nd && d[0] * d[1] * d[2] > n) return FZB_E_INVALID;
    if (!inverse && d_in == d_out && n) return FZB_E_INVALID;
    if (n == 0) return FZB_OK;
    const ScanWork w = carve_scan(d_work, n);
    if (inverse && nd && (!d_work || work_bytes < w.need)) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    TraceScope ts(s, inverse ? "lorenzo_int_inv" : "lorenzo_int_fwd");
    switch (elem_bytes) {
        case 1: return lorenzo_typed<uint8_t>(d_in, d, n, inverse, d_out, w, s);
        case 2: return lorenzo_typed<uint16_t>(d_in, d, n, inverse, d_out, w, s);
        case 4: return lorenzo_typed<uint32_t>(d_in, d, n, inverse, d_out, w, s);
        case 8: return lorenzo_typed<uint64_t>(d_in, d, n, inverse, d_out, w, s);
        default: return FZB_E_INVALID;
    }
}

}  // extern "C"
