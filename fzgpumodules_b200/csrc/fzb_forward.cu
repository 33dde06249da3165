// fzb_forward.cu -- forward kernels: value base, fused Lorenzo predict +
// quantize (codes only, or fused with Bitshuffle and RZE into the final
// stream), standalone Bitshuffle and RZE encode.
//
// One CTA of 256 threads per 8192-element chunk (= one 16 KiB Bitshuffle
// block = one RZE chunk).  Chunks are claimed through a ticket counter so the
// decoupled look-back that places outliers and compressed bytes only waits on
// chunks that are already running.
#include "fzb_kernels.cuh"

namespace fzb {

// ---------------------------------------------------------------------------
// value base (predictor_utils.cuh:27-117) and error-bound resolution on the
// device, so REL/NOA need no host round trip.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) minmax_kernel(const float* __restrict__ x, uint64_t n,
                                                     float* __restrict__ pmin,
                                                     float* __restrict__ pmax) {
    float lo = INFINITY, hi = -INFINITY;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * 4;
    const bool vec = ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4; i < n; i += stride) {
        if (vec && i + 4 <= n) {
            float4 v = __ldg(reinterpret_cast<const float4*>(x + i));
            lo = fminf(lo, fminf(fminf(v.x, v.y), fminf(v.z, v.w)));
            hi = fmaxf(hi, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
        } else {
            for (uint64_t k = i; k < n && k < i + 4; k++) {
                lo = fminf(lo, x[k]);
                hi = fmaxf(hi, x[k]);
            }
        }
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, d));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    __shared__ float slo[8], shi[8];
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
        pmin[blockIdx.x] = lo;
        pmax[blockIdx.x] = hi;
    }
}

// EbState layout (device): [0] value_base, [1] abs_eb, [2] ebx2_r, [3] ebx2.
// nparts == 0: value_base = vb_given (ABS, or a caller-provided base).
// Launched with one warp.
__global__ void resolve_eb_kernel(const float* __restrict__ pmin, const float* __restrict__ pmax,
                                  int nparts, int mode, float user_eb, float vb_given,
                                  float* __restrict__ st) {
    float vb = (mode != 0) ? vb_given : 0.0f;
    float lo = INFINITY, hi = -INFINITY;
    if (mode != 0 && nparts > 0) {
        for (int i = threadIdx.x; i < nparts; i += 32) {
            lo = fminf(lo, pmin[i]);
            hi = fmaxf(hi, pmax[i]);
        }
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, d));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, d));
        }
    }
    if (threadIdx.x != 0) return;
    if (mode != 0 && nparts > 0) {
        if (mode == 2) {
            vb = __fsub_rn(hi, lo);
        } else {
            float al = lo < 0.0f ? -lo : lo, ah = hi < 0.0f ? -hi : hi;
            vb = al > ah ? al : ah;
        }
    }
    // lorenzo_quant.cu:612-644: ABS, or value_base <= 0 -> fall back to ABS
    float abs_eb = (mode == 0 || !(vb > 0.0f)) ? user_eb : __fmul_rn(user_eb, vb);
    st[0] = vb;
    st[1] = abs_eb;
    st[2] = __fdiv_rn(1.0f, __fmul_rn(2.0f, abs_eb));
    st[3] = __fmul_rn(2.0f, abs_eb);
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
__device__ __forceinline__ float delta_at(const FwdArgs& a, const float4* Q, const Roles& R,
                                          uint32_t k) {
    if (NDIM == 1) {
        const float q = qread(Q, R.cur0, k);
        return (k & 1023u) ? __fsub_rn(q, qread(Q, R.cur0, (long long)k - 1)) : q;
    }
    const uint32_t z = (NDIM == 3) ? k / a.plane : 0u;
    const uint32_t rem = k - z * a.plane;
    const uint32_t y = rem / a.nx, x = rem - y * a.nx;
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

// Shared epilogue: look-back for the compressed byte offset, copy out,
// header words, trailing pad.  `sw` is the chunk's size word.
__device__ __forceinline__ void rze_place_chunk(uint8_t* __restrict__ out, uint32_t n_chunks,
                                                uint32_t orig_bytes, uint32_t c, uint32_t sw,
                                                const uint8_t* payload,
                                                unsigned long long* st, uint32_t* err,
                                                unsigned long long* out_size,
                                                unsigned long long* s_b) {
    const uint32_t clean = sw & 0x7fffffffu;
    if (threadIdx.x < 32) {
        uint64_t ex = lookback(st, c, clean, err);
        if (threadIdx.x == 0) *s_b = ex;
    }
    __syncthreads();
    const uint64_t boff = *s_b;
    const uint64_t hdr = 8ull + 4ull * n_chunks;
    copy_out_bytes(out + hdr + boff, payload, clean);
    if (threadIdx.x == 0) {
        reinterpret_cast<uint32_t*>(out + 8)[c] = sw;
        if (c == 0) {
            reinterpret_cast<uint32_t*>(out)[0] = orig_bytes;
            reinterpret_cast<uint32_t*>(out)[1] = n_chunks;
        }
    }
    if (c == n_chunks - 1) {
        const uint64_t total = hdr + boff + clean;
        const uint64_t padded = (total + 3) & ~3ull;
        if (threadIdx.x < padded - total) out[total + threadIdx.x] = 0;
        if (threadIdx.x == 0) *out_size = padded;
    }
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

// ---------------------------------------------------------------------------
// The chunk kernel.  FUSED=false writes codes; FUSED=true bitshuffles them
// (16 KiB blocks, element width 2, ballot layout) and RZE-encodes the block
// straight into the final stream.  ROWAL: rows are multiples of 32 elements,
// so each thread's 32 codes share (y, z) and the row-vector path applies.
// ---------------------------------------------------------------------------

template <int NDIM, bool FUSED, bool ROWAL>
__global__ void __launch_bounds__(kThreads, 3) lq_chunk_kernel(FwdArgs a) {
    extern __shared__ float4 Q[];
    __shared__ uint32_t s_ws[16];
    __shared__ uint32_t s_chunk;
    __shared__ unsigned long long s_b;
    const int t = threadIdx.x;
    if (t == 0) s_chunk = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t c = s_chunk;
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
    make_roles(a, NDIM, i0, cnt, need_z, R);
    const bool vec_ok = (reinterpret_cast<uintptr_t>(a.in) & 15) == 0;
    load_roles(Q, R, a.in, a.nfield, r, vec_ok);
    __syncthreads();

    // ---- pass 1: codes of this thread's 32 consecutive elements ----
    const uint32_t j0 = 32u * t;
    const uint32_t k0 = i0 + j0;
    uint32_t x[16];
#pragma unroll
    for (int l = 0; l < 16; l++) x[l] = 0;
    // row-vector path only for whole groups; partial groups use the element path
    const bool whole = ROWAL && (j0 + 32 <= cnt) && (k0 + 32 <= a.nfield);
    uint32_t om = 0;  // outlier bit per element
    if (whole) {
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
    } else if (j0 < cnt && k0 < a.nfield) {
        for (int E = 0; E < 32; E++) {
            const uint32_t k = k0 + E;
            if (j0 + E < cnt && k < a.nfield) {
                const float cc = delta_at<NDIM>(a, Q, R, k);
                const bool qz = fabsf(cc) < a.radius;
                const uint32_t code = qz ? encode_code(cc, zz) : 0u;
                om |= (qz ? 0u : 1u) << E;
#pragma unroll
                for (int l = 0; l < 16; l++)
                    if (l == (E & 15)) x[l] |= code << (16 * (E >> 4));
            }
        }
    }
    const uint32_t nout = __popc(om);

    // ---- outliers: block scan + look-back for their global offset ----
    uint32_t ototal;
    const uint32_t ooff = block_excl_scan(nout, s_ws, &ototal);
    if (t < 32) {
        uint64_t ex = lookback(a.st_outl, c, ototal, a.err);
        if (t == 0) s_b = ex;
    }
    __syncthreads();
    const uint64_t obase = s_b;
    if (nout) {  // pass 2: recompute this thread's deltas and store outliers
        uint64_t pos = obase + ooff;
        for (int E = 0; E < 32; E++) {
            const uint32_t k = k0 + E;
            if (j0 + E < cnt && k < a.nfield) {
                const float cc = delta_at<NDIM>(a, Q, R, k);
                if (!(fabsf(cc) < a.radius)) {
                    if (pos < a.cap) {
                        a.out_err[pos] = cc;
                        a.out_idx[pos] = k;
                    }
                    pos++;
                }
            }
        }
    }
    if (c == a.n_chunks - 1 && t == 0) *a.out_count = (uint32_t)((obase + ototal) < 0xffffffffull ? (obase + ototal) : 0xffffffffull);

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
    rze_place_chunk(a.rze, a.n_chunks, a.codes_bytes, c, sw,
                    (sw >> 31) ? reinterpret_cast<const uint8_t*>(sm.S) : sm.O, a.st_bytes, a.err,
                    a.rze_size, &s_b);
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

// ---------------------------------------------------------------------------
// Standalone RZE encode of a byte stream (rze_stage.cu:774-843 semantics,
// one pass: chunk encode + look-back placement).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) rze_encode_kernel(RzeEncArgs a) {
    extern __shared__ float4 Q[];
    __shared__ uint32_t s_ws[16];
    __shared__ uint32_t s_chunk;
    __shared__ unsigned long long s_b;
    const int t = threadIdx.x;
    if (t == 0) s_chunk = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t c = s_chunk;
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
    rze_place_chunk(a.out, a.n_chunks, (uint32_t)a.bytes, c, sw,
                    (sw >> 31) ? reinterpret_cast<const uint8_t*>(sm.S) : sm.O, a.st_bytes, a.err,
                    a.out_size, &s_b);
}

}  // namespace fzb
