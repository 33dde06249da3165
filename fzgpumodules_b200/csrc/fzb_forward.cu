// fzb_forward.cu -- forward kernels: value base, fused Lorenzo predict +
// quantize (codes only, or fused with Bitshuffle and RZE into the final
// stream), standalone Bitshuffle and RZE encode.
//
// One CTA of 256 threads per 8192-element chunk (= one 16 KiB Bitshuffle
// block = one RZE chunk).  Placement is two-phase so no chunk ever waits on
// another: each chunk writes its encoded bytes to a fixed slot and its
// outliers to staging, then assemble_scan/assemble_copy build the ordered
// stream and outlier list.
#include "fzb_kernels.cuh"
#include "fzb_slab.cuh"

namespace fzb {

// ---------------------------------------------------------------------------
// value base (predictor_utils.cuh:27-117) and error-bound resolution on the
// device, so REL/NOA need no host round trip.
// ---------------------------------------------------------------------------

// Grid-stride min/max with eight independent 16-byte loads in flight per
// thread; the last block to finish reduces the partials and resolves
// abs_eb / ebx2_r into st (lorenzo_quant.cu:612-644).  st layout:
// [0] value_base, [1] abs_eb, [2] ebx2_r, [3] ebx2.
__device__ __forceinline__ void resolve_eb_store(float lo, float hi, int mode, float user_eb,
                                                 float vb, bool have_minmax, float* st) {
    if (mode != 0 && have_minmax) {
        if (mode == 2) {
            vb = __fsub_rn(hi, lo);
        } else {
            const float al = lo < 0.0f ? -lo : lo, ah = hi < 0.0f ? -hi : hi;
            vb = al > ah ? al : ah;
        }
    }
    if (mode == 0) vb = 0.0f;
    // ABS, or value_base <= 0 -> fall back to ABS
    const float abs_eb = (mode == 0 || !(vb > 0.0f)) ? user_eb : __fmul_rn(user_eb, vb);
    st[0] = vb;
    st[1] = abs_eb;
    st[2] = __fdiv_rn(1.0f, __fmul_rn(2.0f, abs_eb));
    st[3] = __fmul_rn(2.0f, abs_eb);
}

// Block `blk` of `nblk` cooperating blocks: partial min/max into
// pmin/pmax[blk]; the last block to finish reduces the partials and resolves
// the error bound into st, then re-arms `done` for the next launch.
__device__ __forceinline__ void minmax_body(const float* __restrict__ x, uint64_t n, float* __restrict__ pmin,
                                            float* __restrict__ pmax, unsigned int* __restrict__ done, int mode,
                                            float user_eb, float* __restrict__ st, const unsigned blk,
                                            const unsigned nblk) {
    float lo = INFINITY, hi = -INFINITY;
    const bool vec = ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
    const uint64_t nv = vec ? n / 4 : 0;
    const float4* x4 = reinterpret_cast<const float4*>(x);
    const uint64_t stride = (uint64_t)nblk * blockDim.x;
    uint64_t i = (uint64_t)blk * blockDim.x + threadIdx.x;
    // sixteen 16-byte loads in flight per thread, streamed past L1 with a
    // 256-byte L2 fetch (a read-once scan)
    for (; i + 15 * stride < nv; i += 16 * stride) {
        float4 v[16];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const float4* q = x4 + i + k * stride;
            asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v4.f32 {%0,%1,%2,%3}, [%4];"
                         : "=f"(v[k].x), "=f"(v[k].y), "=f"(v[k].z), "=f"(v[k].w) : "l"(q));
        }
#pragma unroll
        for (int k = 0; k < 16; k++) {
            lo = fminf(lo, fminf(fminf(v[k].x, v[k].y), fminf(v[k].z, v[k].w)));
            hi = fmaxf(hi, fmaxf(fmaxf(v[k].x, v[k].y), fmaxf(v[k].z, v[k].w)));
        }
    }
    for (; i < nv; i += stride) {
        const float4 v = __ldg(x4 + i);
        lo = fminf(lo, fminf(fminf(v.x, v.y), fminf(v.z, v.w)));
        hi = fmaxf(hi, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
    }
    for (uint64_t k = 4 * nv + (uint64_t)blk * blockDim.x + threadIdx.x; k < n; k += stride) {
        lo = fminf(lo, x[k]);
        hi = fmaxf(hi, x[k]);
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, d));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    __shared__ float slo[8], shi[8];
    __shared__ bool s_last;
    if ((threadIdx.x & 31) == 0) {
        slo[threadIdx.x >> 5] = lo;
        shi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; w++) {
            lo = fminf(lo, slo[w]);
            hi = fmaxf(hi, shi[w]);
        }
        pmin[blk] = lo;
        pmax[blk] = hi;
        __threadfence();
        s_last = (atomicAdd(done, 1u) == nblk - 1);
    }
    __syncthreads();
    // this block's share is written: a programmatic dependent (the slab
    // compressor) may start its set-up while the last block resolves the
    // bound, which it reads only after this grid has ended
    asm volatile("griddepcontrol.launch_dependents;");
    if (!s_last) return;
    __threadfence();
    lo = INFINITY;
    hi = -INFINITY;
    for (unsigned b = threadIdx.x; b < nblk; b += blockDim.x) {
        lo = fminf(lo, __ldcg(pmin + b));
        hi = fmaxf(hi, __ldcg(pmax + b));
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, d));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    if ((threadIdx.x & 31) == 0) {
        slo[threadIdx.x >> 5] = lo;
        shi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; w++) {
            lo = fminf(lo, slo[w]);
            hi = fmaxf(hi, shi[w]);
        }
        resolve_eb_store(lo, hi, mode, user_eb, 0.0f, true, st);
        *done = 0;  // ready for the next launch
    }
}

__global__ void __launch_bounds__(256) minmax_kernel(const float* __restrict__ x, uint64_t n,
                                                     float* __restrict__ pmin, float* __restrict__ pmax,
                                                     unsigned int* __restrict__ done, int mode, float user_eb,
                                                     float* __restrict__ st) {
    minmax_body(x, n, pmin, pmax, done, mode, user_eb, st, blockIdx.x, gridDim.x);
}

// Error-bound resolution without a scan (ABS, or a caller-provided base).
__global__ void resolve_eb_kernel(int mode, float user_eb, float vb_given, float* __restrict__ st) {
    if (threadIdx.x == 0) resolve_eb_store(0.f, 0.f, mode, user_eb, vb_given, false, st);
}

// ---------------------------------------------------------------------------
// Lorenzo windows.  Each role (current / up neighbour row, plane z / z-1)
// stages q = round(x * ebx2_r) for a contiguous index range into shared
// memory as 16-byte granules; granule r of a window lives at
// soff + (r ^ ((r >> 3) & 7)) so that the per-thread 32-element reads of a
// warp hit distinct banks.
// ---------------------------------------------------------------------------

struct Win {
    long long gbase;  // first element (multiple of 4, may be negative)
    int ngran;        // granules
    int soff;         // granule offset in shared memory (multiple of 8)
};

__device__ __forceinline__ int swz(int r) { return r ^ ((r >> 3) & 7); }

__device__ __forceinline__ float q_of(float v, float r) { return round_half_away(__fmul_rn(v, r)); }

__device__ __forceinline__ void load_window(float4* Q, const Win& w, const float* __restrict__ in,
                                            uint32_t nfield, float r, bool vec_ok) {
    constexpr int kPer = 9;  // granules in flight per thread
    for (int base = 0; base < w.ngran; base += kPer * kThreads) {
        float4 buf[kPer];
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const int gi = base + threadIdx.x + i * kThreads;
            buf[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gi < w.ngran) {
                const long long g = w.gbase + 4LL * gi;
                if (vec_ok && g >= 0 && g + 4 <= (long long)nfield) {
                    buf[i] = __ldg(reinterpret_cast<const float4*>(in + g));
                } else {
                    float e[4];
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        e[k] = (g + k >= 0 && g + k < (long long)nfield) ? __ldg(in + g + k) : 0.0f;
                    buf[i] = make_float4(e[0], e[1], e[2], e[3]);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const int gi = base + threadIdx.x + i * kThreads;
            if (gi < w.ngran) {
                const long long g = w.gbase + 4LL * gi;
                float4 v = buf[i];
                if (g >= 0 && g + 4 <= (long long)nfield) {
                    v.x = q_of(v.x, r);
                    v.y = q_of(v.y, r);
                    v.z = q_of(v.z, r);
                    v.w = q_of(v.w, r);
                } else {  // field edge: positions outside stage as 0 (never read by a valid element)
                    v.x = (g + 0 >= 0 && g + 0 < (long long)nfield) ? q_of(v.x, r) : 0.0f;
                    v.y = (g + 1 >= 0 && g + 1 < (long long)nfield) ? q_of(v.y, r) : 0.0f;
                    v.z = (g + 2 >= 0 && g + 2 < (long long)nfield) ? q_of(v.z, r) : 0.0f;
                    v.w = (g + 3 >= 0 && g + 3 < (long long)nfield) ? q_of(v.w, r) : 0.0f;
                }
                Q[w.soff + swz(gi)] = v;
            }
        }
    }
}

// Windows a chunk needs: q(k) (cur) and q(k - nx) (up) for plane z and, in
// 3-D when some element has z % 8 != 0, for plane z - 1.  Union mode covers
// cur and up with one window per plane; rows wider than a chunk use two.
struct Roles {
    Win cur0, up0, cur1, up1;
    bool two, z;  // separate up windows / plane z-1 present
};

__device__ __forceinline__ Win make_win(long long start, long long end, int& soff) {
    const long long gb = start >= 0 ? (start & ~3LL) : -(((-start) + 3) & ~3LL);
    const int ng = (int)((end - gb + 3) >> 2);
    Win w{gb, ng, soff};
    soff += (ng + 7) & ~7;
    return w;
}

__device__ __forceinline__ void make_roles(const FwdArgs& a, int ndim, uint32_t i0, uint32_t cnt,
                                           bool need_z, Roles& R) {
    int soff = 0;
    R.two = (ndim >= 2) && a.two_piece;
    R.z = (ndim == 3) && need_z;
    for (int p = 0; p < (R.z ? 2 : 1); p++) {
        const long long sh = p ? (long long)a.plane : 0;
        const long long s0 = (long long)i0 - sh, e0 = (long long)i0 + cnt - sh;
        Win cur, up;
        if (ndim == 1) {
            cur = up = make_win(s0 - 1, e0, soff);
        } else if (!R.two) {
            cur = up = make_win(s0 - (long long)a.nx - 1, e0, soff);
        } else {
            up = make_win(s0 - (long long)a.nx - 1, e0 - (long long)a.nx, soff);
            cur = make_win(s0 - 1, e0, soff);
        }
        if (p == 0) { R.cur0 = cur; R.up0 = up; }
        else { R.cur1 = cur; R.up1 = up; }
    }
}

__device__ __forceinline__ void load_roles(float4* Q, const Roles& R, const float* in, uint32_t nfield,
                                           float r, bool vec_ok) {
    load_window(Q, R.cur0, in, nfield, r, vec_ok);
    if (R.two) load_window(Q, R.up0, in, nfield, r, vec_ok);
    if (R.z) {
        load_window(Q, R.cur1, in, nfield, r, vec_ok);
        if (R.two) load_window(Q, R.up1, in, nfield, r, vec_ok);
    }
}

// Single-element q read of element k from role window w.
__device__ __forceinline__ float qread(const float4* Q, const Win& w, long long k) {
    const int m = (int)(k - w.gbase);
    const float* Qf = reinterpret_cast<const float*>(Q);
    return Qf[4 * (w.soff + swz(m >> 2)) + (m & 3)];
}

// Lorenzo delta of element k in the reference's operation order
// (3-D: z, x, y -- lorenzo_quant_nd.cu:234-246; 2-D: y, x -- :72-77;
// 1-D: x -- lorenzo_quant.cu:308-321).
template <int NDIM>
__device__ __forceinline__ float delta_xyz(const FwdArgs& a, const float4* Q, const Roles& R, uint32_t k,
                                           uint32_t x, uint32_t y, uint32_t z) {
    if (NDIM == 1) {
        const float q = qread(Q, R.cur0, k);
        return (k & 1023u) ? __fsub_rn(q, qread(Q, R.cur0, (long long)k - 1)) : q;
    }
    const Win& wc = R.cur0;
    const Win& wu = R.up0;
    const long long ku = (long long)k - a.nx;
    if (NDIM == 2) {
        const uint32_t tx = x & 31u, ty = y & 31u;
        float v0 = qread(Q, wc, k);
        if (ty) v0 = __fsub_rn(v0, qread(Q, wu, ku));
        if (!tx) return v0;
        float v1 = qread(Q, wc, (long long)k - 1);
        if (ty) v1 = __fsub_rn(v1, qread(Q, wu, ku - 1));
        return __fsub_rn(v0, v1);
    }
    const uint32_t tx = x & 7u, ty = y & 7u, tz = z & 7u;
    const long long kz = (long long)k - a.plane, kuz = ku - a.plane;
    auto A = [&](const Win& w, long long kk, long long kkz, const Win* wz) -> float {
        float v = qread(Q, w, kk);
        return tz ? __fsub_rn(v, qread(Q, *wz, kkz)) : v;
    };
    const Win* wcz = &R.cur1;
    const Win* wuz = &R.up1;
    float b0 = A(wc, k, kz, wcz);
    if (tx) b0 = __fsub_rn(b0, A(wc, (long long)k - 1, kz - 1, wcz));
    if (!ty) return b0;
    float b1 = A(wu, ku, kuz, wuz);
    if (tx) b1 = __fsub_rn(b1, A(wu, ku - 1, kuz - 1, wuz));
    return __fsub_rn(b0, b1);
}

// Along a run of consecutive elements the x neighbour's terms are the previous
// element's own, so the run carries them: Run::a0 = A(x, y) and a1 = A(x, y-1)
// of the last element, with A the z-differenced value (3-D), the y-differenced
// value (2-D, a0 only) or q itself (1-D).  delta_run gives the same float
// operations in the same order as delta_xyz.
struct Run {
    float a0, a1;
};
template <int NDIM>
__device__ __forceinline__ void run_terms(const FwdArgs& a, const float4* Q, const Roles& R, long long k,
                                          uint32_t y, uint32_t z, float& a0, float& a1) {
    if (NDIM == 1) {
        a0 = qread(Q, R.cur0, k);
        a1 = 0.0f;
    } else if (NDIM == 2) {
        a0 = qread(Q, R.cur0, k);
        if (y & 31u) a0 = __fsub_rn(a0, qread(Q, R.up0, k - a.nx));
        a1 = 0.0f;
    } else {
        const bool tz = (z & 7u) != 0;
        a0 = qread(Q, R.cur0, k);
        if (tz) a0 = __fsub_rn(a0, qread(Q, R.cur1, k - a.plane));
        a1 = 0.0f;
        if (y & 7u) {
            a1 = qread(Q, R.up0, k - a.nx);
            if (tz) a1 = __fsub_rn(a1, qread(Q, R.up1, k - a.nx - a.plane));
        }
    }
}
template <int NDIM>
__device__ __forceinline__ float delta_run(const FwdArgs& a, const float4* Q, const Roles& R, uint32_t k,
                                           uint32_t x, uint32_t y, uint32_t z, Run& run) {
    float a0, a1;
    run_terms<NDIM>(a, Q, R, k, y, z, a0, a1);
    float d;
    if (NDIM == 1) {
        d = (k & 1023u) ? __fsub_rn(a0, run.a0) : a0;
    } else if (NDIM == 2) {
        d = (x & 31u) ? __fsub_rn(a0, run.a0) : a0;
    } else {
        const bool tx = (x & 7u) != 0;
        const float b0 = tx ? __fsub_rn(a0, run.a0) : a0;
        if (y & 7u) {
            const float b1 = tx ? __fsub_rn(a1, run.a1) : a1;
            d = __fsub_rn(b0, b1);
        } else {
            d = b0;
        }
    }
    run.a0 = a0;
    run.a1 = a1;
    return d;
}

// The granule of 4 window values starting at k (k - gbase a multiple of 4).
__device__ __forceinline__ float4 qread4(const float4* Q, const Win& w, long long k) {
    return Q[w.soff + swz((int)((k - w.gbase) >> 2))];
}

// Element coordinates of field index k, and the step to k + 1 (x fastest),
// so that a run of consecutive elements needs no divisions.
struct Xyz {
    uint32_t x, y, z;
};
template <int NDIM>
__device__ __forceinline__ Xyz xyz_of(const FwdArgs& a, uint32_t k) {
    if (NDIM == 1) return Xyz{k, 0u, 0u};
    const uint32_t z = (NDIM == 3) ? k / a.plane : 0u;
    const uint32_t rem = k - z * a.plane;
    const uint32_t y = rem / a.nx;
    return Xyz{rem - y * a.nx, y, z};
}
template <int NDIM>
__device__ __forceinline__ void xyz_next(const FwdArgs& a, Xyz& c) {
    if (NDIM == 1) return;
    if (++c.x == a.nx) {
        c.x = 0;
        if (++c.y == a.ny && NDIM == 3) {
            c.y = 0;
            c.z++;
        }
    }
}

// Raw little-endian code words of a 32-code group from the packed form
// x[l] = code[l] | code[l+16] << 16.
__device__ __forceinline__ void packed_to_raw(const uint32_t (&x)[16], uint32_t (&rw)[16]) {
#pragma unroll
    for (int l = 0; l < 8; l++) rw[l] = __byte_perm(x[2 * l], x[2 * l + 1], 0x5410);
#pragma unroll
    for (int l = 8; l < 16; l++) rw[l] = __byte_perm(x[2 * l - 16], x[2 * l - 15], 0x7632);
}

__device__ __forceinline__ void raw_to_packed(const uint32_t (&rw)[16], uint32_t (&x)[16]) {
#pragma unroll
    for (int l = 0; l < 8; l++) {
        x[2 * l] = __byte_perm(rw[l], rw[l + 8], 0x5410);
        x[2 * l + 1] = __byte_perm(rw[l], rw[l + 8], 0x7632);
    }
}

// Writes a chunk's encoded bytes (S when stored raw, else O) to its 16 KiB
// slot and its size word to sizes[c].
__device__ __forceinline__ void write_slot(uint8_t* __restrict__ slots, uint32_t* __restrict__ sizes,
                                           uint32_t c, uint32_t sw, const uint8_t* payload) {
    const uint32_t clean = sw & 0x7fffffffu;
    uint4* d4 = reinterpret_cast<uint4*>(slots + (size_t)c * kChunkBytes);
    const uint4* s4 = reinterpret_cast<const uint4*>(payload);
    for (uint32_t i = threadIdx.x; i < (clean + 15) / 16; i += kThreads) d4[i] = s4[i];
    if (threadIdx.x == 0) sizes[c] = sw;
}

// Exclusive scans over chunks (one CTA of 1024 threads): payload offsets,
// outlier offsets, RZE header, total sizes.
template <uint32_t kTile>
__device__ __forceinline__ void assemble_scan_body(const AsmArgs& a, uint32_t* sp, uint32_t* so) {
    // Tiles of kTile chunks: loads issued in batches of eight per thread (all
    // in flight at once) into shared memory, kTile/1024 chunks per thread, a
    // warp-shuffle block scan, coalesced writes, carry to the next tile.
    // sp / so hold pad32-indexed entries (kTile + kTile / 32 words each).
    constexpr uint32_t kPer = kTile / 1024;
    __shared__ uint32_t wp[32], wo[32], s_tile[2];
    const uint32_t n = a.n_chunks, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    // outliers that found room in staging (an overflowing run keeps those,
    // the count still reports every outlier found)
    auto staged = [&](uint32_t b0, uint32_t n0) -> uint32_t {
        return b0 >= a.ostage_cap ? 0u : min(n0, a.ostage_cap - b0);
    };
    uint32_t* hdr = reinterpret_cast<uint32_t*>(a.out);
    unsigned long long carry_p = 0;
    uint32_t carry_o = 0, ot = 0;
    for (uint32_t t0 = 0; t0 < n; t0 += kTile) {
        const uint32_t cnt = min(kTile, n - t0);
        for (uint32_t j0 = 0; j0 < kPer; j0 += (kPer < 8 ? kPer : 8)) {
            constexpr uint32_t kB = kPer < 8 ? kPer : 8;
            uint32_t vs[kB], vb[kB], vc[kB];
#pragma unroll
            for (uint32_t j = 0; j < kB; j++) {
                const uint32_t i = t + 1024u * (j0 + j);
                const bool in = i < cnt;
                vs[j] = (in && a.sizes) ? a.sizes[t0 + i] : 0u;
                vb[j] = (in && a.ocnt) ? a.obase[t0 + i] : 0u;
                vc[j] = (in && a.ocnt) ? a.ocnt[t0 + i] : 0u;
            }
#pragma unroll
            for (uint32_t j = 0; j < kB; j++) {
                const uint32_t i = t + 1024u * (j0 + j);
                sp[pad32(i)] = vs[j] & 0x7fffffffu;
                so[pad32(i)] = a.ocnt ? staged(vb[j], vc[j]) : 0u;
                ot += vc[j];
                if (a.sizes && i < cnt) hdr[2 + t0 + i] = vs[j];  // the stream's size table
            }
        }
        __syncthreads();
        uint32_t lp = 0, lo = 0;
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++) {
            lp += sp[pad32(kPer * t + j)];
            lo += so[pad32(kPer * t + j)];
        }
        uint32_t ip = lp, io = lo;  // inclusive warp scans
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t np = __shfl_up_sync(0xffffffffu, ip, d), no = __shfl_up_sync(0xffffffffu, io, d);
            if (lane >= (uint32_t)d) {
                ip += np;
                io += no;
            }
        }
        if (lane == 31) {
            wp[warp] = ip;
            wo[warp] = io;
        }
        __syncthreads();
        if (warp == 0) {
            const uint32_t vp = wp[lane], vo = wo[lane];
            uint32_t xp = vp, xo = vo;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t np = __shfl_up_sync(0xffffffffu, xp, d), no = __shfl_up_sync(0xffffffffu, xo, d);
                if (lane >= (uint32_t)d) {
                    xp += np;
                    xo += no;
                }
            }
            wp[lane] = xp - vp;  // exclusive warp offsets
            wo[lane] = xo - vo;
        }
        __syncthreads();
        uint32_t rp = wp[warp] + ip - lp, ro = wo[warp] + io - lo;
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++) {  // exclusive prefixes in place
            const uint32_t k = pad32(kPer * t + j);
            const uint32_t vp = sp[k], vo = so[k];
            sp[k] = rp;
            so[k] = ro;
            rp += vp;
            ro += vo;
        }
        if (t == 1023) {
            s_tile[0] = rp;
            s_tile[1] = ro;
        }
        __syncthreads();
        for (uint32_t i = t; i < cnt; i += 1024) {
            if (a.sizes) a.pay_off[t0 + i] = carry_p + sp[pad32(i)];
            if (a.ocnt) a.ofin[t0 + i] = carry_o + so[pad32(i)];
        }
        carry_p += s_tile[0];
        carry_o += s_tile[1];
        __syncthreads();  // the next tile reuses the arrays
    }
    __shared__ unsigned int s_tot;
    if (t == 0) s_tot = 0;
    __syncthreads();
    if (a.ocnt && ot) atomicAdd(&s_tot, ot);
    __syncthreads();
    if (t == 1023) {
        if (a.sizes) {
            hdr[0] = a.orig_bytes;
            hdr[1] = n;
            const unsigned long long total = 8ull + 4ull * n + carry_p;
            const unsigned long long padded = (total + 3) & ~3ull;
            for (unsigned long long i = total; i < padded; i++) a.out[i] = 0;
            *a.out_size = padded;
        }
        if (a.ocnt) *a.out_count = s_tot;
    }
}

// Both assembly kernels are launched as programmatic dependents: each waits
// for the kernel before it (the chunk sizes, then the offsets) and the scan
// lets the copy start launching once it is done.
__global__ void __launch_bounds__(1024) assemble_scan_kernel(AsmArgs a) {
    extern __shared__ uint32_t asm_dyn[];
    asm volatile("griddepcontrol.wait;" ::: "memory");
    assemble_scan_body<kAsmTile>(a, asm_dyn, asm_dyn + kAsmTile + kAsmTile / 32);
    asm volatile("griddepcontrol.launch_dependents;");
}

// The same scans for up to kTiledScanMax chunks, a CTA per 1024 chunks:
// each CTA first sums the payload sizes, staged outlier counts and outlier
// counts of every chunk before its tile (at most 63 K words each, from L2),
// then scans its own tile; the last CTA writes the stream header's totals.
__global__ void __launch_bounds__(1024) assemble_scan_tiles_kernel(AsmArgs a) {
    __shared__ uint32_t ws[66];
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const uint32_t n = a.n_chunks, t = threadIdx.x, base = blockIdx.x * 1024u;
    const bool last = base + 1024u >= n;
    auto staged = [&](uint32_t i) -> uint32_t {
        const uint32_t b0 = a.obase[i], n0 = a.ocnt[i];
        return b0 >= a.ostage_cap ? 0u : min(n0, a.ostage_cap - b0);
    };
    uint32_t sp = 0, so = 0, sc = 0;  // before the tile: payload bytes, staged outliers, outliers found
    for (uint32_t i = t; i < base; i += 1024u) {
        if (a.sizes) sp += a.sizes[i] & 0x7fffffffu;
        if (a.ocnt) {
            so += staged(i);
            sc += a.ocnt[i];
        }
    }
    const uint32_t i = base + t;
    const bool in = i < n;
    const uint32_t vs = (in && a.sizes) ? a.sizes[i] : 0u;
    const uint32_t vo = (in && a.ocnt) ? staged(i) : 0u;
    const uint32_t vc = (in && a.ocnt) ? a.ocnt[i] : 0u;
    uint32_t e0, e1, SP, SO, ep, eo, TP, TO;
    block_scan2_1024(sp, so, e0, e1, SP, SO, ws);  // SP, SO: the sums before the tile
    block_scan2_1024(vs & 0x7fffffffu, vo, ep, eo, TP, TO, ws);
    uint32_t* hdr = reinterpret_cast<uint32_t*>(a.out);
    if (in) {
        if (a.sizes) {
            a.pay_off[i] = (unsigned long long)SP + ep;
            hdr[2 + i] = vs;  // the stream's size table
        }
        if (a.ocnt) a.ofin[i] = SO + eo;
    }
    if (last) {
        uint32_t c0, c1, SC, TC;
        block_scan2_1024(sc, vc, c0, c1, SC, TC, ws);
        if (t == 0) {
            if (a.sizes) {
                hdr[0] = a.orig_bytes;
                hdr[1] = n;
                const unsigned long long total = 8ull + 4ull * n + (unsigned long long)SP + TP;
                const unsigned long long padded = (total + 3) & ~3ull;
                for (unsigned long long k = total; k < padded; k++) a.out[k] = 0;
                *a.out_size = padded;
            }
            if (a.ocnt) *a.out_count = SC + TC;
        }
    }
    asm volatile("griddepcontrol.launch_dependents;");
}

int launch_assemble_scan(const AsmArgs& a, cudaStream_t s) {
    if (a.n_chunks <= kTiledScanMax && !(flags_env() & 16))
        return (int)launch_dependent(assemble_scan_tiles_kernel, (a.n_chunks + 1023u) / 1024u + (a.n_chunks == 0),
                                     1024, 0, s, a);
    const int smem = (int)(2 * (kAsmTile + kAsmTile / 32) * sizeof(uint32_t));
    static SmemAttr attr;
    const cudaError_t e = ensure_dyn_smem(attr, (const void*)assemble_scan_kernel, smem);
    if (e != cudaSuccess) return (int)e;
    return (int)launch_dependent(assemble_scan_kernel, 1, 1024, (size_t)smem, s, a);
}

// One chunk per group of `nth` threads (thread `tid` of the group): payload
// from its slot to the final stream position
// (any byte alignment), and its outliers from staging to their sorted
// position (chunks are index ranges and each chunk's block is sorted).
__device__ __forceinline__ void assemble_copy_body(const AsmArgs& a, const uint32_t c, const uint32_t tid,
                                                   const uint32_t nth) {
    if (a.sizes) {
        const uint32_t len = a.sizes[c] & 0x7fffffffu;
        uint8_t* dst = a.out + 8ull + 4ull * a.n_chunks + a.pay_off[c];
        const uint8_t* src = a.slots + (size_t)c * kChunkBytes;
        const uint32_t* s32 = reinterpret_cast<const uint32_t*>(src);
        const uintptr_t d0 = reinterpret_cast<uintptr_t>(dst), d1 = d0 + len;
        const uintptr_t a0 = (d0 + 3) & ~(uintptr_t)3, a1 = d1 & ~(uintptr_t)3;
        if (a0 >= a1) {
            for (uint32_t i = tid; i < len; i += nth) dst[i] = src[i];
        } else {
            const uint32_t head = (uint32_t)(a0 - d0), tail = (uint32_t)(d1 - a1);
            if (tid < head) dst[tid] = src[tid];
            if (tid < tail) dst[(a1 - d0) + tid] = src[(a1 - d0) + tid];
            uint32_t* dw = reinterpret_cast<uint32_t*>(a0);
            const uint32_t nw = (uint32_t)((a1 - a0) >> 2), r = head & 3;
            for (uint32_t i0 = tid; i0 < nw; i0 += 4 * nth) {  // four words per thread in flight
                uint32_t lo[4], hi[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const uint32_t i = i0 + k * nth;
                    const uint32_t w0 = (head + 4 * i) >> 2;  // source word of destination word i
                    lo[k] = i < nw ? __ldg(s32 + w0) : 0u;
                    hi[k] = (i < nw && r) ? __ldg(s32 + w0 + 1) : 0u;
                }
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const uint32_t i = i0 + k * nth;
                    if (i < nw) dw[i] = r ? __funnelshift_r(lo[k], hi[k], 8 * r) : lo[k];
                }
            }
        }
    }
    if (a.ocnt) {
        const uint32_t b = a.obase[c], f = a.ofin[c];
        const uint32_t n = b >= a.ostage_cap ? 0u : min(a.ocnt[c], a.ostage_cap - b);
        for (uint32_t i = tid; i < n; i += nth) {
            const uint32_t s = b + i, d = f + i;
            if (d < a.cap) {
                a.out_err[d] = a.ostage_err[s];
                a.out_idx[d] = a.ostage_idx[s];
            }
        }
    }
}

// One warp per chunk, grid-stride over the chunks.
__global__ void __launch_bounds__(256) assemble_copy_kernel(AsmArgs a) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    for (uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < a.n_chunks; c += nw)
        assemble_copy_body(a, c, lane, 32);
}

// Row-vector path: one thread, 32 consecutive elements of one row, all
// operands staged in shared memory.  TZ/TY say whether the z / y predecessor
// lies inside the tile (z % 8 != 0, y % 8 != 0; 2-D: y % 32 != 0).
struct GroupIn {
    const float4 *Qc, *Qu, *Qcz, *Quz;
    int rc, ru, rcz, ruz;
    float p0;
    uint32_t j0;
    float radius;
};

template <bool ZZ>
__device__ __forceinline__ uint32_t code_of(float c) {
    const int iv = __float2int_rz(c);
    if (ZZ) {
        const int s = (int)(int16_t)iv;
        return (((uint32_t)s << 1) ^ (uint32_t)(s >> 15)) & 0xffffu;
    }
    return (uint32_t)iv & 0xffffu;
}

__device__ __forceinline__ void unpack4(float4 v, float* d) {
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
}

template <int NDIM, bool ZZ, bool TZ, bool TY>
__device__ __forceinline__ void group_codes(const GroupIn& g, uint32_t (&x)[16], uint32_t& om) {
    float p0 = g.p0, p1 = 0.0f;  // carried a00 / a01 (3-D), v0 (2-D), q (1-D)
#pragma unroll
    for (int h = 0; h < 2; h++) {
        float qc[16], qu[16], qcz[16], quz[16];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            unpack4(g.Qc[swz(g.rc + 4 * h + k)], qc + 4 * k);
            if (NDIM >= 2 && TY) unpack4(g.Qu[swz(g.ru + 4 * h + k)], qu + 4 * k);
            if (NDIM == 3 && TZ) {
                unpack4(g.Qcz[swz(g.rcz + 4 * h + k)], qcz + 4 * k);
                if (TY) unpack4(g.Quz[swz(g.ruz + 4 * h + k)], quz + 4 * k);
            }
        }
#pragma unroll
        for (int e = 0; e < 16; e++) {
            const int E = 16 * h + e;
            float cc;
            if (NDIM == 3) {
                const float a00 = TZ ? __fsub_rn(qc[e], qcz[e]) : qc[e];
                const float b0 = (E & 7) ? __fsub_rn(a00, p0) : a00;
                p0 = a00;
                if (TY) {
                    const float a01 = TZ ? __fsub_rn(qu[e], quz[e]) : qu[e];
                    const float b1 = (E & 7) ? __fsub_rn(a01, p1) : a01;
                    p1 = a01;
                    cc = __fsub_rn(b0, b1);
                } else {
                    cc = b0;
                }
            } else if (NDIM == 2) {
                const float v0 = TY ? __fsub_rn(qc[e], qu[e]) : qc[e];
                cc = E ? __fsub_rn(v0, p0) : v0;
                p0 = v0;
            } else {
                cc = ((g.j0 + E) & 1023u) ? __fsub_rn(qc[e], p0) : qc[e];
                p0 = qc[e];
            }
            const bool qz = fabsf(cc) < g.radius;
            const uint32_t code = qz ? code_of<ZZ>(cc) : 0u;
            om |= (qz ? 0u : 1u) << E;
            if (h == 0) x[e] = code;
            else x[e] = __byte_perm(x[e], code, 0x5410);
        }
    }
}

template <int NDIM, bool ZZ>
__device__ __forceinline__ void group_dispatch(const GroupIn& g, bool tz, bool ty, uint32_t (&x)[16],
                                               uint32_t& om) {
    if (NDIM == 3) {
        if (tz) {
            if (ty) group_codes<NDIM, ZZ, true, true>(g, x, om);
            else group_codes<NDIM, ZZ, true, false>(g, x, om);
        } else {
            if (ty) group_codes<NDIM, ZZ, false, true>(g, x, om);
            else group_codes<NDIM, ZZ, false, false>(g, x, om);
        }
    } else if (NDIM == 2) {
        if (ty) group_codes<NDIM, ZZ, false, true>(g, x, om);
        else group_codes<NDIM, ZZ, false, false>(g, x, om);
    } else {
        group_codes<NDIM, ZZ, false, false>(g, x, om);
    }
}

// Codes of one thread's whole 32-element run when rows are a multiple of 4
// elements but not of 32 (the element path's case): every window value of the
// run comes in 16-byte granules (k, k - nx, k - plane and k - plane - nx are
// all multiples of 4 from the window bases), the coordinates step along the
// run, and the x neighbour's terms are carried as in delta_run, with the same
// float operations in the same order.
template <int NDIM>
__device__ __forceinline__ void run_codes_vec(const FwdArgs& a, const float4* Q, const Roles& R, uint32_t k0,
                                              Xyz cz, bool zz, uint32_t (&x)[16], uint32_t& om) {
    Run run{0.0f, 0.0f};
    if ((cz.x & (NDIM == 2 ? 31u : 7u)) != 0) run_terms<NDIM>(a, Q, R, (long long)k0 - 1, cz.y, cz.z, run.a0, run.a1);
#pragma unroll
    for (int g = 0; g < 8; g++) {
        const long long kg = (long long)k0 + 4 * g;
        const float4 c4 = qread4(Q, R.cur0, kg);
        const float4 u4 = qread4(Q, R.up0, kg - a.nx);
        float4 cz4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), uz4 = cz4;
        if (NDIM == 3 && R.z) {
            cz4 = qread4(Q, R.cur1, kg - a.plane);
            uz4 = qread4(Q, R.up1, kg - a.plane - a.nx);
        }
        const float cv[4] = {c4.x, c4.y, c4.z, c4.w}, uv[4] = {u4.x, u4.y, u4.z, u4.w};
        const float czv[4] = {cz4.x, cz4.y, cz4.z, cz4.w}, uzv[4] = {uz4.x, uz4.y, uz4.z, uz4.w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int E = 4 * g + e;
            float a0 = cv[e], a1 = 0.0f, d;
            if (NDIM == 2) {
                if (cz.y & 31u) a0 = __fsub_rn(a0, uv[e]);
                d = (cz.x & 31u) ? __fsub_rn(a0, run.a0) : a0;
            } else {
                const bool tz = (cz.z & 7u) != 0, tx = (cz.x & 7u) != 0;
                if (tz) a0 = __fsub_rn(a0, czv[e]);
                const float b0 = tx ? __fsub_rn(a0, run.a0) : a0;
                if (cz.y & 7u) {
                    a1 = uv[e];
                    if (tz) a1 = __fsub_rn(a1, uzv[e]);
                    d = __fsub_rn(b0, tx ? __fsub_rn(a1, run.a1) : a1);
                } else {
                    d = b0;
                }
            }
            run.a0 = a0;
            run.a1 = a1;
            const bool qz = fabsf(d) < a.radius;
            const uint32_t code = qz ? encode_code(d, zz) : 0u;
            om |= (qz ? 0u : 1u) << E;
            x[E & 15] |= code << (16 * (E >> 4));
            xyz_next<NDIM>(a, cz);
        }
    }
}

// ---------------------------------------------------------------------------
// The chunk kernel.  FUSED=false writes codes; FUSED=true bitshuffles them
// (16 KiB blocks, element width 2, ballot layout) and RZE-encodes the block
// straight into the final stream.  ROWAL: rows are multiples of 32 elements,
// so each thread's 32 codes share (y, z) and the row-vector path applies.
// ---------------------------------------------------------------------------

// One 8192-code chunk `c` of the field `a` (every thread of the block
// calls it; it contains block-wide barriers).  Q: dynamic shared memory,
// s_ws: 16 words, s_obase: one word.  `preset`: windows the caller has
// already staged (and synchronised), in place of the chunk's own.
// Register front end for full chunks of 1-D fields (16-byte aligned input):
// thread t's 32 elements k0 .. k0 + 31 come straight from HBM into
// registers, are quantized with the packed round (trunc(y + copysign(
// 0.49999997, y))) and differenced there; a 1024-element block starts at
// every lane 0, and element k0 - 1 is lane t - 1's last.  Codes come from the
// magic-number add; per 4-element granule a NaN-propagating max flags
// outliers, confirmed element by element.  Same codes and outlier set as the
// window path (group_codes).  (The same front end for 2-D rows, reading the
// row above from L2, made the batch slower: 3.98 against 3.73 ms.)
template <int NDIM>
__device__ __forceinline__ bool reg_front_ok(const FwdArgs& a, uint32_t i0, uint32_t cnt) {
    return NDIM == 1 && cnt == (uint32_t)kChunkCodes && i0 + (uint32_t)kChunkCodes <= a.nfield &&
           (reinterpret_cast<uintptr_t>(a.in) & 15) == 0;
}

template <bool ZZ>
__device__ __forceinline__ void reg_codes_1d(const FwdArgs& a, uint32_t k0, float r, uint32_t (&x)[16],
                                             uint32_t& om) {
    const float4* src = reinterpret_cast<const float4*>(a.in + k0);
    const float R = a.radius;
    Q4 q[8];
#pragma unroll
    for (int g = 0; g < 8; g++) q[g] = quant4(__ldg(src + g), r);
    const float pl = __shfl_up_sync(0xffffffffu, q[7].b.y, 1);
    float left = (threadIdx.x & 31u) ? pl : 0.0f;  // the x predecessor of element 0
    uint32_t rw[16];
    om = 0;
#pragma unroll
    for (int g = 0; g < 8; g++) {
        const Q4 c = {sub2(q[g].a, f2(left, q[g].a.x)), sub2(q[g].b, f2(q[g].a.y, q[g].b.x))};
        left = q[g].b.y;
        const float mx = max_nan(max_nan(fabsf(c.a.x), fabsf(c.a.y)), max_nan(fabsf(c.b.x), fabsf(c.b.y)));
        uint32_t p0 = code_pair<ZZ>(c.a), p1 = code_pair<ZZ>(c.b);
        if (!(mx < R)) {  // outliers: their codes are 0
            const uint32_t b = (fabsf(c.a.x) < R ? 0u : 1u) | (fabsf(c.a.y) < R ? 0u : 2u) |
                               (fabsf(c.b.x) < R ? 0u : 4u) | (fabsf(c.b.y) < R ? 0u : 8u);
            om |= b << (4 * g);
            p0 &= ((b & 1u) ? 0xffff0000u : 0xffffffffu) & ((b & 2u) ? 0x0000ffffu : 0xffffffffu);
            p1 &= ((b & 4u) ? 0xffff0000u : 0xffffffffu) & ((b & 8u) ? 0x0000ffffu : 0xffffffffu);
        }
        rw[2 * g] = p0;
        rw[2 * g + 1] = p1;
    }
    raw_to_packed(rw, x);
}

// 1-D delta of element k recomputed from the input, for the register front
// end's outlier records (the window path reads its windows instead).
__device__ __forceinline__ float reg_delta_1d(const FwdArgs& a, uint32_t k, float r) {
    const float q = q_of(__ldg(a.in + k), r);
    return (k & 1023u) ? __fsub_rn(q, q_of(__ldg(a.in + k - 1), r)) : q;
}

template <int NDIM, bool FUSED, bool ROWAL>
__device__ __forceinline__ void lq_chunk_body(const FwdArgs& a, const uint32_t c, float4* Q, uint32_t* s_ws,
                                              uint32_t& s_obase, const Roles* preset = nullptr) {
    const int t = threadIdx.x;
    const uint32_t i0 = c * (uint32_t)kChunkCodes;
    const uint32_t cnt = min((uint32_t)kChunkCodes, a.n_total - i0);
    const float r = *a.ebx2_r;
    const bool zz = a.zigzag != 0;

    bool need_z = false;
    if (NDIM == 3 && i0 < a.nfield) {
        const uint32_t last = min(i0 + cnt, a.nfield) - 1;
        const uint32_t z0 = i0 / a.plane, z1 = last / a.plane;
        need_z = (z0 & 7u) || (z1 != z0);
    }
    Roles R;
    const bool reg = !preset && reg_front_ok<NDIM>(a, i0, cnt);  // the same for every thread of the chunk
    if (preset) {
        R = *preset;
    } else if (!reg) {
        make_roles(a, NDIM, i0, cnt, need_z, R);
        const bool vec_ok = (reinterpret_cast<uintptr_t>(a.in) & 15) == 0;
        load_roles(Q, R, a.in, a.nfield, r, vec_ok);
        __syncthreads();
    }

    // ---- pass 1: codes of this thread's 32 consecutive elements ----
    const uint32_t j0 = 32u * t;
    const uint32_t k0 = i0 + j0;
    uint32_t x[16];
#pragma unroll
    for (int l = 0; l < 16; l++) x[l] = 0;
    // row-vector path only for whole groups; partial groups use the element path
    const bool whole = ROWAL && (j0 + 32 <= cnt) && (k0 + 32 <= a.nfield);
    uint32_t om = 0;  // outlier bit per element
    if (reg) {
        if (zz) reg_codes_1d<true>(a, k0, r, x, om);
        else reg_codes_1d<false>(a, k0, r, x, om);
    } else if (whole) {
        uint32_t ty = 0, tz = 0;
        if (NDIM == 3) {
            const uint32_t z = k0 / a.plane, y = (k0 - z * a.plane) / a.nx;
            ty = y & 7u;
            tz = z & 7u;
        } else if (NDIM == 2) {
            ty = (k0 / a.nx) & 31u;
        }
        GroupIn g;
        g.Qc = Q + R.cur0.soff;
        g.Qu = Q + R.up0.soff;
        g.rc = (int)(((long long)k0 - R.cur0.gbase) >> 2);
        g.ru = (int)(((long long)k0 - a.nx - R.up0.gbase) >> 2);
        g.Qcz = g.Qc;
        g.Quz = g.Qu;
        g.rcz = g.ruz = 0;
        if (NDIM == 3 && tz) {
            g.Qcz = Q + R.cur1.soff;
            g.Quz = Q + R.up1.soff;
            g.rcz = (int)(((long long)k0 - a.plane - R.cur1.gbase) >> 2);
            g.ruz = (int)(((long long)k0 - a.plane - a.nx - R.up1.gbase) >> 2);
        }
        g.p0 = (NDIM == 1 && (j0 & 1023u)) ? qread(Q, R.cur0, (long long)k0 - 1) : 0.0f;
        g.j0 = j0;
        g.radius = a.radius;
        if (zz) group_dispatch<NDIM, true>(g, tz != 0, ty != 0, x, om);
        else group_dispatch<NDIM, false>(g, tz != 0, ty != 0, x, om);
    } else if (NDIM >= 2 && (a.nx & 3u) == 0 && j0 + 32 <= cnt && k0 + 32 <= a.nfield) {
        run_codes_vec<NDIM>(a, Q, R, k0, xyz_of<NDIM>(a, k0), zz, x, om);
    } else if (j0 < cnt && k0 < a.nfield) {
        // element path (rows not a multiple of 4, partial groups): coordinates
        // step along the run; the unrolled loop keeps x[] in registers
        Xyz cz = xyz_of<NDIM>(a, k0);
        Run run{0.0f, 0.0f};
        {   // the x neighbour of the run's first element, when its tile uses it
            const bool tx = NDIM == 1 ? (k0 & 1023u) != 0 : (cz.x & (NDIM == 2 ? 31u : 7u)) != 0;
            if (tx) run_terms<NDIM>(a, Q, R, (long long)k0 - 1, cz.y, cz.z, run.a0, run.a1);
        }
#pragma unroll
        for (int E = 0; E < 32; E++) {
            const uint32_t k = k0 + E;
            if (j0 + E < cnt && k < a.nfield) {
                const float cc = delta_run<NDIM>(a, Q, R, k, cz.x, cz.y, cz.z, run);
                const bool qz = fabsf(cc) < a.radius;
                const uint32_t code = qz ? encode_code(cc, zz) : 0u;
                om |= (qz ? 0u : 1u) << E;
                x[E & 15] |= code << (16 * (E >> 4));
            }
            xyz_next<NDIM>(a, cz);
        }
    }
    const uint32_t nout = __popc(om);

    // ---- outliers: block scan, one staging allocation per chunk ----
    uint32_t ototal;
    const uint32_t ooff = block_excl_scan(nout, s_ws, &ototal);
    if (t == 0) {
        const uint32_t b = ototal ? atomicAdd(a.ostage_ctr, ototal) : 0u;
        a.obase[c] = b;
        a.ocnt[c] = ototal;
        s_obase = b;
    }
    __syncthreads();
    if (nout && reg) {  // pass 2, register front end: the deltas again from the input
        uint32_t pos = s_obase + ooff;
        for (int E = 0; E < 32; E++) {
            if (!((om >> E) & 1u)) continue;
            if (pos < a.ostage_cap) {
                a.ostage_err[pos] = reg_delta_1d(a, k0 + E, r);
                a.ostage_idx[pos] = k0 + E;
            }
            pos++;
        }
    } else if (nout) {  // pass 2: recompute this thread's deltas and stage its outliers
        uint32_t pos = s_obase + ooff;
        Xyz cz = xyz_of<NDIM>(a, k0);
        for (int E = 0; E < 32; E++, xyz_next<NDIM>(a, cz)) {
            const uint32_t k = k0 + E;
            if (j0 + E < cnt && k < a.nfield) {
                const float cc = delta_xyz<NDIM>(a, Q, R, k, cz.x, cz.y, cz.z);
                if (!(fabsf(cc) < a.radius)) {
                    if (pos < a.ostage_cap) {
                        a.ostage_err[pos] = cc;
                        a.ostage_idx[pos] = k;
                    }
                    pos++;
                }
            }
        }
    }

    if (!FUSED) {
        uint32_t rw[16];
        packed_to_raw(x, rw);
        uint16_t* dst = a.codes + k0;
        if (j0 + 32 <= cnt && (reinterpret_cast<uintptr_t>(a.codes) & 15) == 0) {
            uint4* d4 = reinterpret_cast<uint4*>(dst);
#pragma unroll
            for (int v = 0; v < 4; v++)
                d4[v] = make_uint4(rw[4 * v], rw[4 * v + 1], rw[4 * v + 2], rw[4 * v + 3]);
        } else {
#pragma unroll
            for (int E = 0; E < 32; E++)
                if (j0 + E < cnt) dst[E] = (uint16_t)(x[E & 15] >> (16 * (E >> 4)));
        }
        return;
    }

    // ---- Bitshuffle into S, then RZE ----
    __syncthreads();  // windows are dead past this point
    uint8_t* base = reinterpret_cast<uint8_t*>(Q);
    RzeSmem sm;
    sm.S = reinterpret_cast<uint32_t*>(base);
    sm.O = base + kChunkBytes;
    sm.bm1 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16);
    sm.bm2 = base + 2 * kChunkBytes + 16 + 2048;
    sm.bm3 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16 + 2048 + 256);
    sm.ws = s_ws;
    if (cnt == (uint32_t)kChunkCodes) {
        transpose16x2(x);
#pragma unroll
        for (int b = 0; b < 16; b++) sm.S[(15 - b) * 256 + t] = x[b];
    } else {  // partial tail block: Bitshuffle copies it unchanged
        uint32_t rw[16];
        packed_to_raw(x, rw);
#pragma unroll
        for (int l = 0; l < 16; l++) sm.S[16 * t + l] = rw[l];
    }
    __syncthreads();
    const uint32_t sw = rze_encode_chunk(sm, (int)(2 * cnt));
    write_slot(a.slots, a.sizes, c, sw, (sw >> 31) ? reinterpret_cast<const uint8_t*>(sm.S) : sm.O);
}

template <int NDIM, bool FUSED, bool ROWAL>
__global__ void __launch_bounds__(kThreads, 3) lq_chunk_kernel(FwdArgs a) {
    extern __shared__ float4 Q[];
    __shared__ uint32_t s_ws[16];
    __shared__ uint32_t s_obase;
    lq_chunk_body<NDIM, FUSED, ROWAL>(a, blockIdx.x, Q, s_ws, s_obase);
}

// ---------------------------------------------------------------------------
// Batched fused compression: many fields, one persistent launch.  CTAs take
// (field, chunk) units from a global counter in the order `unit_order`
// lists the fields; every unit runs the same chunk body as the single-field
// kernel, so each field's bytes equal its own fzb_lq_bs_rze_compress output.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 3) lq_batch_kernel(BatchArgs b) {
    extern __shared__ float4 Q[];
    __shared__ uint32_t s_ws[16];
    __shared__ uint32_t s_obase;
    __shared__ uint32_t s_unit;
    // thread 0 takes the next unit's ticket as this one starts, so the
    // dispenser's round trip overlaps the chunk instead of preceding it
    uint32_t next = 0;
    if (threadIdx.x == 0) s_unit = atomicAdd(b.counter, 1u);
    for (;;) {
        __syncthreads();
        const uint32_t u = s_unit;
        __syncthreads();  // s_unit is rewritten at the end of this iteration
        if (u >= b.lq_units) break;
        if (threadIdx.x == 0) next = atomicAdd(b.counter, 1u);
        // field = last slot whose unit_begin <= u (fields in unit_order)
        uint32_t lo = 0, hi = b.nfields;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (b.unit_begin[mid] <= u) lo = mid;
            else hi = mid;
        }
        const BatchField& f = b.fields[b.unit_order[lo]];
        const uint32_t c = u - b.unit_begin[lo];
        switch (f.kind) {
            case 0: lq_chunk_body<1, true, true>(f.a, c, Q, s_ws, s_obase); break;
            case 1: lq_chunk_body<2, true, true>(f.a, c, Q, s_ws, s_obase); break;
            case 2: lq_chunk_body<2, true, false>(f.a, c, Q, s_ws, s_obase); break;
            case 3: lq_chunk_body<3, true, true>(f.a, c, Q, s_ws, s_obase); break;
            default: lq_chunk_body<3, true, false>(f.a, c, Q, s_ws, s_obase); break;
        }
        if (threadIdx.x == 0) s_unit = next;  // read after the barrier that opens the next iteration
    }
}

// REL/NOA value bases of every field in one launch: blockIdx.y = field,
// blockIdx.x < parts(field) take part; the last block of a field resolves it.
__global__ void __launch_bounds__(256) batch_minmax_kernel(BatchArgs b) {
    const BatchField& f = b.fields[blockIdx.y];
    if (blockIdx.x >= f.mm_parts) return;
    if (f.mm_parts == 1 && f.scan == 0) {  // ABS, or a caller-provided value base
        if (threadIdx.x == 0) resolve_eb_store(0.f, 0.f, f.mode, f.user_eb, f.vb_given, false, f.eb_state);
        return;
    }
    minmax_body(f.in, f.n, f.pmin, f.pmax, f.mm_done, f.mode, f.user_eb, f.eb_state, blockIdx.x, f.mm_parts);
}

__global__ void __launch_bounds__(1024) batch_assemble_scan_kernel(BatchArgs b) {
    __shared__ uint32_t sp[4096 + 128], so[4096 + 128];
    assemble_scan_body<4096>(b.fields[blockIdx.x].m, sp, so);
}

__global__ void __launch_bounds__(256) batch_assemble_copy_kernel(BatchArgs b) {
    const uint32_t u = blockIdx.x;
    uint32_t lo = 0, hi = b.nfields;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (b.unit_begin[mid] <= u) lo = mid;
        else hi = mid;
    }
    assemble_copy_body(b.fields[b.unit_order[lo]].m, u - b.unit_begin[lo], threadIdx.x, blockDim.x);
}

// Per launch: the unit dispenser, every field's error word and outlier
// staging counter start at zero.
__global__ void batch_reset_kernel(BatchArgs b) {
    const BatchField& f = b.fields[blockIdx.x];
    if (threadIdx.x == 0) {
        *f.a.ostage_ctr = 0;
        *f.a.err = 0;
        if (blockIdx.x == 0) *b.counter = 0;
    }
}

int launch_batch_scan(const BatchArgs& b, uint32_t mm_grid_x, cudaStream_t s) {
    batch_reset_kernel<<<b.nfields, 32, 0, s>>>(b);
    batch_minmax_kernel<<<dim3(mm_grid_x, b.nfields), 256, 0, s>>>(b);
    return (int)cudaGetLastError();
}

int launch_batch_code(const BatchArgs& b, unsigned lq_grid, size_t smem, cudaStream_t s) {
    if (b.lq_units) {
        cudaError_t e = cudaFuncSetAttribute(lq_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        lq_batch_kernel<<<lq_grid, kThreads, smem, s>>>(b);
    }
    batch_assemble_scan_kernel<<<b.nfields, 1024, 0, s>>>(b);
    batch_assemble_copy_kernel<<<b.total_units, 256, 0, s>>>(b);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Slab-column kernel for 3-D fields whose chunks are R = 8192/nx whole rows
// (nx a power of two in [32, 1024], ny % R == 0, no padding).  A work unit is
// one R-row slab across one 8-plane z tile; its chunks are produced plane by
// plane.  Every element is rounded once (plane z-1's q stays in registers),
// no halo is read (slab and tile origins have y % 8 == 0 and z % 8 == 0), and
// plane z+1 is prefetched into registers while plane z is encoded.  Units
// run last-to-first so the tail of the field, still in L2 after the
// value-base scan, is consumed first.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int gswz(int g) { return g ^ ((g >> 3) & 7); }

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <bool ZZ>
__global__ void __launch_bounds__(kThreads, 2) lq3d_slab_kernel(FwdArgs a, uint32_t slabs,
                                                               uint32_t units) {
    extern __shared__ float4 smem4[];
    __shared__ uint32_t s_ws[16];
    __shared__ uint32_t s_obase;
    uint8_t* base = reinterpret_cast<uint8_t*>(smem4);
    float4* A4 = smem4;                       // A plane: 8192 floats, swizzled granules
    float4* Rw = smem4 + kChunkCodes / 4;     // raw plane prefetch: 8192 floats, swizzled
    const float* Af = reinterpret_cast<const float*>(smem4);
    RzeSmem sm;
    uint8_t* rz = base + 8 * kChunkCodes;
    sm.S = reinterpret_cast<uint32_t*>(rz);
    sm.O = rz + kChunkBytes;
    sm.bm1 = reinterpret_cast<uint32_t*>(rz + 2 * kChunkBytes + 16);
    sm.bm2 = rz + 2 * kChunkBytes + 16 + 2048;
    sm.bm3 = reinterpret_cast<uint32_t*>(rz + 2 * kChunkBytes + 16 + 2048 + 256);
    sm.ws = s_ws;

    const int t = threadIdx.x;
    const uint32_t nx = a.nx, R = kChunkCodes / nx;
    const float r = *a.ebx2_r;
    const uint32_t e0 = 32u * t;             // this thread's 32 elements of the slab plane
    const uint32_t ty = (e0 / nx) & 7u;      // slab origin has y % 8 == 0
    const int gup = ((int)e0 - (int)nx) >> 2;
    auto dswz = [](int m) { const int g = m >> 2; return (gswz(g) << 2) | (m & 3); };
    auto prefetch = [&](uint32_t z, uint32_t s) {
        const float4* src = reinterpret_cast<const float4*>(
            a.in + ((size_t)z * a.ny + (size_t)s * R) * nx + e0);
#pragma unroll
        for (int g = 0; g < 8; g++) cp_async16(Rw + gswz(8 * t + g), src + g);
        cp_async_commit();
    };

    uint32_t uu = blockIdx.x;
    if (uu < units) {
        const uint32_t u = units - 1 - uu;
        prefetch((u / slabs) * 8, u % slabs);
    }
    for (; uu < units; uu += gridDim.x) {
        const uint32_t u = units - 1 - uu;
        const uint32_t s = u % slabs, zt = u / slabs;
        const uint32_t z0 = zt * 8, z1 = min(z0 + 8, a.nz);
        float qprev[32];
        for (uint32_t z = z0; z < z1; z++) {
            const uint32_t c = z * slabs + s;
            const bool tz = (z != z0);
            cp_async_wait_all();
            float4 cur[8];
#pragma unroll
            for (int g = 0; g < 8; g++) cur[g] = Rw[gswz(8 * t + g)];
            // each thread refills only its own granules, so no barrier is needed
            if (z + 1 < z1) prefetch(z + 1, s);
            else if (uu + gridDim.x < units) {
                const uint32_t un = units - 1 - (uu + gridDim.x);
                prefetch((un / slabs) * 8, un % slabs);
            }
            // A = q(z) - q(z-1): the z difference first (lorenzo_quant_nd.cu:236)
#pragma unroll
            for (int g = 0; g < 8; g++) {
                float v[4] = {cur[g].x, cur[g].y, cur[g].z, cur[g].w};
                float w[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int e = 4 * g + k;
                    const float q = q_of(v[k], r);
                    w[k] = tz ? __fsub_rn(q, qprev[e]) : q;
                    qprev[e] = q;
                }
                A4[gswz(8 * t + g)] = make_float4(w[0], w[1], w[2], w[3]);
            }
            __syncthreads();
            // x then y differences (lorenzo_quant_nd.cu:239-246), quantize
            uint32_t x[16];
            uint32_t om = 0;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float av[16], up[16];
#pragma unroll
                for (int g = 0; g < 4; g++) {
                    const float4 w = A4[gswz(8 * t + 4 * h + g)];
                    av[4 * g] = w.x; av[4 * g + 1] = w.y; av[4 * g + 2] = w.z; av[4 * g + 3] = w.w;
                    if (ty) {
                        const float4 q = A4[gswz(gup + 4 * h + g)];
                        up[4 * g] = q.x; up[4 * g + 1] = q.y; up[4 * g + 2] = q.z; up[4 * g + 3] = q.w;
                    }
                }
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int e = 16 * h + k;
                    float cc;
                    const float b0 = (e & 7) ? __fsub_rn(av[k], av[k - 1]) : av[k];
                    if (ty) {
                        const float b1 = (e & 7) ? __fsub_rn(up[k], up[k - 1]) : up[k];
                        cc = __fsub_rn(b0, b1);
                    } else {
                        cc = b0;
                    }
                    const bool qz = fabsf(cc) < a.radius;
                    const uint32_t code = qz ? code_of<ZZ>(cc) : 0u;
                    om |= (qz ? 0u : 1u) << e;
                    if (h == 0) x[k] = code;
                    else x[k] = __byte_perm(x[k], code, 0x5410);
                }
            }
            // outliers: one staging allocation per chunk; values recomputed
            // from the staged A plane (rare path)
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
                const uint32_t kbase = c * (uint32_t)kChunkCodes + e0;
                for (int e = 0; e < 32; e++) {
                    if (!((om >> e) & 1u)) continue;
                    const int m = (int)e0 + e;
                    const float a0 = Af[dswz(m)];
                    const float b0 = (e & 7) ? __fsub_rn(a0, Af[dswz(m - 1)]) : a0;
                    float cc = b0;
                    if (ty) {
                        const float u0 = Af[dswz(m - (int)nx)];
                        const float b1 = (e & 7) ? __fsub_rn(u0, Af[dswz(m - (int)nx - 1)]) : u0;
                        cc = __fsub_rn(b0, b1);
                    }
                    if (pos < a.ostage_cap) {
                        a.ostage_err[pos] = cc;
                        a.ostage_idx[pos] = kbase + e;
                    }
                    pos++;
                }
            }
            // Bitshuffle (full chunk) and RZE
            transpose16x2(x);
#pragma unroll
            for (int b = 0; b < 16; b++) sm.S[(15 - b) * 256 + t] = x[b];
            __syncthreads();
            const uint32_t sw = rze_encode_chunk(sm, kChunkBytes);
            write_slot(a.slots, a.sizes, c, sw, (sw >> 31) ? reinterpret_cast<const uint8_t*>(sm.S) : sm.O);
            __syncthreads();
        }
    }
    cp_async_wait_all();
}

int launch_lq3d_slab(const FwdArgs& a, unsigned grid, cudaStream_t s) {
    const size_t smem = 8 * kChunkCodes + 2 * kChunkBytes + 16 + 2048 + 256 + 32;
    const uint32_t slabs = a.ny / (kChunkCodes / a.nx), units = slabs * ((a.nz + 7) / 8);
    cudaError_t e;
    if (a.zigzag) {
        e = cudaFuncSetAttribute(lq3d_slab_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        lq3d_slab_kernel<true><<<grid, kThreads, smem, s>>>(a, slabs, units);
    } else {
        e = cudaFuncSetAttribute(lq3d_slab_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        lq3d_slab_kernel<false><<<grid, kThreads, smem, s>>>(a, slabs, units);
    }
    return (int)cudaGetLastError();
}

template <int NDIM, bool FUSED, bool ROWAL>
static int launch_lq_t(const FwdArgs& a, size_t smem, unsigned grid, cudaStream_t s) {
    auto k = lq_chunk_kernel<NDIM, FUSED, ROWAL>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    k<<<grid, kThreads, smem, s>>>(a);
    return (int)cudaGetLastError();
}

int launch_lq_chunk(int ndim, bool fused, bool rowal, const FwdArgs& a, size_t smem,
                    unsigned grid, cudaStream_t s) {
    if (ndim == 1) return fused ? launch_lq_t<1, true, true>(a, smem, grid, s)
                                : launch_lq_t<1, false, true>(a, smem, grid, s);
    if (ndim == 2) {
        if (fused) return rowal ? launch_lq_t<2, true, true>(a, smem, grid, s)
                                : launch_lq_t<2, true, false>(a, smem, grid, s);
        return rowal ? launch_lq_t<2, false, true>(a, smem, grid, s)
                     : launch_lq_t<2, false, false>(a, smem, grid, s);
    }
    if (fused) return rowal ? launch_lq_t<3, true, true>(a, smem, grid, s)
                            : launch_lq_t<3, true, false>(a, smem, grid, s);
    return rowal ? launch_lq_t<3, false, true>(a, smem, grid, s)
                 : launch_lq_t<3, false, false>(a, smem, grid, s);
}

// ---------------------------------------------------------------------------
// Standalone Bitshuffle, element width 2 (ballot layout, MSB plane first).
// One CTA per 16 KiB block; thread t owns codes 32t..32t+31.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) bitshuffle2_kernel(const uint8_t* __restrict__ in,
                                                               uint8_t* __restrict__ out,
                                                               int inverse) {
    const size_t blk = (size_t)blockIdx.x * kChunkBytes;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(in + blk);
    uint32_t* dst = reinterpret_cast<uint32_t*>(out + blk);
    const int t = threadIdx.x;
    uint32_t x[16];
    if (!inverse) {
        uint32_t rw[16];
        const uint4* s4 = reinterpret_cast<const uint4*>(src + 16 * t);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            uint4 q = __ldg(s4 + v);
            rw[4 * v] = q.x; rw[4 * v + 1] = q.y; rw[4 * v + 2] = q.z; rw[4 * v + 3] = q.w;
        }
        raw_to_packed(rw, x);
        transpose16x2(x);
#pragma unroll
        for (int b = 0; b < 16; b++) dst[(15 - b) * 256 + t] = x[b];
    } else {
#pragma unroll
        for (int b = 0; b < 16; b++) x[b] = __ldg(src + (15 - b) * 256 + t);
        transpose16x2(x);
        uint32_t rw[16];
        packed_to_raw(x, rw);
        uint4* d4 = reinterpret_cast<uint4*>(dst + 16 * t);
#pragma unroll
        for (int v = 0; v < 4; v++) d4[v] = make_uint4(rw[4 * v], rw[4 * v + 1], rw[4 * v + 2], rw[4 * v + 3]);
    }
}

// Element width 1 or 2, any block size that is a multiple of 1024 * ew:
// one warp ballot per bit plane (bitshuffle_stage.cu:299-349).
__global__ void bitshuffle_ballot_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                                         uint32_t block, int ew, int inverse) {
    const uint32_t W = 8u * ew, n_chunk = block / ew, npp = n_chunk / 32u;
    const uint8_t* src = in + (size_t)blockIdx.x * block;
    uint8_t* dst = out + (size_t)blockIdx.x * block;
    const int lane = threadIdx.x & 31;
    for (uint32_t i = threadIdx.x; i < n_chunk; i += blockDim.x) {
        const uint32_t wg = i / 32u;
        if (!inverse) {
            uint32_t v = (ew == 1) ? src[i] : reinterpret_cast<const uint16_t*>(src)[i];
            for (uint32_t b = 0; b < W; b++) {
                uint32_t bal = __ballot_sync(0xffffffffu, (v >> b) & 1u);
                if (lane == 0) reinterpret_cast<uint32_t*>(dst)[(W - 1 - b) * npp + wg] = bal;
            }
        } else {
            uint32_t v = 0;
            for (uint32_t b = 0; b < W; b++) {
                uint32_t word = reinterpret_cast<const uint32_t*>(src)[(W - 1 - b) * npp + wg];
                v |= ((word >> lane) & 1u) << b;
            }
            if (ew == 1) dst[i] = (uint8_t)v;
            else reinterpret_cast<uint16_t*>(dst)[i] = (uint16_t)v;
        }
    }
}

// Element widths 4 and 8 (the reference's butterfly kernels,
// bitshuffle_stage.cu:66-110 and :175-278): plane p holds bit W-1-p; a plane
// word (u32 for width 4, u64 for width 8) covers a group of 32 / 64
// elements with element e at the word's top bit minus e.  A warp handles one
// group per step: lane l loads element l (width 8: also l + 32), a 5-stage
// shuffle transpose (plus a register swap stage for 64 rows) gives lane j
// column j, and the plane word of plane p is column W-1-p bit-reversed,
// taken from lane 31-p.  The inverse runs the same steps backwards.
template <int EW>
__device__ __forceinline__ uint64_t bs_lo_mask(int s) {
    const uint32_t m = s == 16 ? 0x0000ffffu : s == 8 ? 0x00ff00ffu : s == 4 ? 0x0f0f0f0fu : s == 2 ? 0x33333333u
                                                                                                : 0x55555555u;
    return EW == 4 ? (uint64_t)m : ((uint64_t)m << 32) | m;
}

// Transpose of the 32 x 32 bit matrix whose row l is lane l's word.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, uint32_t lane) {
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const uint32_t m = (uint32_t)bs_lo_mask<4>(s);
        const uint32_t q = __shfl_xor_sync(0xffffffffu, x, s);
        x = (lane & s) ? ((x & ~m) | ((q & ~m) >> s)) : ((x & m) | ((q & m) << s));
    }
    return x;
}

// Transpose of the 64 x 64 bit matrix whose rows l and l + 32 are lane l's
// a0 and a1; afterwards a0 / a1 of lane j are columns j / j + 32.
__device__ __forceinline__ void warp_transpose64(uint64_t& a0, uint64_t& a1, uint32_t lane) {
    const uint64_t lo = 0x00000000ffffffffull;
    const uint64_t n0 = (a0 & lo) | ((a1 & lo) << 32), n1 = (a1 & ~lo) | ((a0 & ~lo) >> 32);
    a0 = n0;
    a1 = n1;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const uint64_t m = bs_lo_mask<8>(s);
        const uint64_t q0 = __shfl_xor_sync(0xffffffffu, a0, s), q1 = __shfl_xor_sync(0xffffffffu, a1, s);
        if (lane & s) {
            a0 = (a0 & ~m) | ((q0 & ~m) >> s);
            a1 = (a1 & ~m) | ((q1 & ~m) >> s);
        } else {
            a0 = (a0 & m) | ((q0 & m) << s);
            a1 = (a1 & m) | ((q1 & m) << s);
        }
    }
}

template <int EW>
__global__ void __launch_bounds__(1024) bitshuffle_wide_kernel(const uint8_t* __restrict__ in,
                                                               uint8_t* __restrict__ out, uint32_t block,
                                                               int inverse) {
    constexpr uint32_t GW = EW == 4 ? 32u : 64u;  // elements per plane word
    const uint32_t n_chunk = block / EW, npp = n_chunk / GW, groups = n_chunk / GW;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t rl = 31 - lane;
    if (EW == 4) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(in + (size_t)blockIdx.x * block);
        uint32_t* dst = reinterpret_cast<uint32_t*>(out + (size_t)blockIdx.x * block);
        for (uint32_t g = warp; g < groups; g += nwarps) {
            if (!inverse) {
                const uint32_t t = warp_transpose32(__ldg(src + GW * g + lane), lane);
                dst[(size_t)lane * npp + g] = __brev(__shfl_sync(0xffffffffu, t, rl));
            } else {
                const uint32_t t = __shfl_sync(0xffffffffu, __brev(__ldg(src + (size_t)lane * npp + g)), rl);
                dst[GW * g + lane] = warp_transpose32(t, lane);
            }
        }
    } else {
        const uint64_t* src = reinterpret_cast<const uint64_t*>(in + (size_t)blockIdx.x * block);
        uint64_t* dst = reinterpret_cast<uint64_t*>(out + (size_t)blockIdx.x * block);
        for (uint32_t g = warp; g < groups; g += nwarps) {
            if (!inverse) {
                uint64_t a0 = __ldg(src + GW * g + lane), a1 = __ldg(src + GW * g + 32 + lane);
                warp_transpose64(a0, a1, lane);
                const uint64_t r0 = __shfl_sync(0xffffffffu, a0, rl), r1 = __shfl_sync(0xffffffffu, a1, rl);
                dst[(size_t)lane * npp + g] = __brevll(r1);          // plane lane: column 63 - lane
                dst[(size_t)(lane + 32) * npp + g] = __brevll(r0);   // plane lane + 32: column 31 - lane
            } else {
                const uint64_t w0 = __ldg(src + (size_t)lane * npp + g), w1 = __ldg(src + (size_t)(lane + 32) * npp + g);
                uint64_t a1 = __shfl_sync(0xffffffffu, __brevll(w0), rl);
                uint64_t a0 = __shfl_sync(0xffffffffu, __brevll(w1), rl);
                warp_transpose64(a0, a1, lane);
                dst[GW * g + lane] = a0;
                dst[GW * g + 32 + lane] = a1;
            }
        }
    }
}

int launch_bitshuffle_wide(const uint8_t* in, uint8_t* out, uint64_t nfull, uint32_t block, int ew, int inverse,
                           cudaStream_t s) {
    if (ew == 4) bitshuffle_wide_kernel<4><<<(unsigned)nfull, 1024, 0, s>>>(in, out, block, inverse);
    else bitshuffle_wide_kernel<8><<<(unsigned)nfull, 1024, 0, s>>>(in, out, block, inverse);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Standalone RZE encode of a byte stream (rze_stage.cu:774-843 semantics,
// one pass: chunk encode + look-back placement).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) rze_encode_kernel(RzeEncArgs a) {
    extern __shared__ float4 Q[];
    __shared__ uint32_t s_ws[16];
    const int t = threadIdx.x;
    const uint32_t c = blockIdx.x;
    const uint64_t off = (uint64_t)c * kChunkBytes;
    const int in_size = (int)min((uint64_t)kChunkBytes, a.bytes - off);
    uint8_t* base = reinterpret_cast<uint8_t*>(Q);
    RzeSmem sm;
    sm.S = reinterpret_cast<uint32_t*>(base);
    sm.O = base + kChunkBytes;
    sm.bm1 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16);
    sm.bm2 = base + 2 * kChunkBytes + 16 + 2048;
    sm.bm3 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16 + 2048 + 256);
    sm.ws = s_ws;
    const uint8_t* src = a.in + off;
    if (in_size == kChunkBytes && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
        const uint4* s4 = reinterpret_cast<const uint4*>(src);
        uint4* d4 = reinterpret_cast<uint4*>(sm.S);
        for (int i = t; i < kChunkBytes / 16; i += kThreads) d4[i] = __ldg(s4 + i);
    } else {
        uint8_t* Sb = reinterpret_cast<uint8_t*>(sm.S);
        for (int i = t; i < kChunkBytes; i += kThreads) Sb[i] = (i < in_size) ? src[i] : 0;
    }
    __syncthreads();
    const uint32_t sw = rze_encode_chunk(sm, in_size);
    write_slot(a.slots, a.sizes, c, sw, (sw >> 31) ? reinterpret_cast<const uint8_t*>(sm.S) : sm.O);
}

}  // namespace fzb
