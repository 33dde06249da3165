// fzb_slab_inv.cu -- fused single-pass inverse RZE -> Bitshuffle inverse ->
// 3-D Lorenzo inverse for the slab geometry (nx a power of two in [32, 1024],
// ny % (8192/nx) == 0): persistent CTAs walk (R-row slab, 8-plane z tile)
// units plane by plane, mirroring the slab compressor (fzb_slab.cu).
//
// Per chunk (= one slab plane):
//   * the chunk's payload is staged into shared memory with 16-byte cp.async
//     copies (4-byte ones for a stream that is not 16-byte aligned) one plane
//     ahead (double buffer);
//   * warp 0 rebuilds RZE levels 4 -> 2 (bm3, bm2 and the per-byte prefix
//     counts of bm2), all threads rebuild bm1 (rze_stage.cu:871-994);
//   * thread t owns chunk elements 32t..32t+31: its 16 plane nibbles come
//     from the 8-lane byte transpose of the bm1 words, the per-plane
//     level-1 byte offsets from warp scans of the nibble popcounts plus
//     per-warp bases, and each plane word is read with one funnel shift and
//     re-expanded with a byte permute; the words are bit-transposed back to
//     32 codes (bitshuffle_stage.cu:299-323 layout);
//   * codes -> deltas through the float magic-number conversion, outliers of
//     the segment are added, the x prefix runs in registers; after the next
//     chunk's first barrier (so that this pass overlaps warp 0's level
//     decoding of that chunk) each thread takes a 4-wide, 8-row column strip
//     for the y prefix, the running z sum (registers, across the unit's
//     planes) and the 16-byte output stores (value * 2 * eb).
//
// Three CTAs of 256 threads run per SM (80 registers a thread).
//
// The reference scans x, y and z with Hillis-Steele add trees
// (lorenzo_quant_nd.cu inverse); this kernel sums sequentially.  Every
// partial sum of either order is an integer of magnitude <= 2^24 when the
// deltas are codes (|d| <= 32768: 8, 64 and 512 terms), so both are exact and
// equal.  Chunks that carry outliers are checked: |d|, |x prefix| and
// |xy prefix| must stay below 2^21, else kErrInexact is raised and the host
// reruns the exact kernels.
#include "fzb_slab.cuh"

namespace fzb {
namespace {

constexpr int kCBytes = kChunkBytes + 64;  // one staged chunk (+ lead bytes and a slack word)
constexpr size_t kInvSmem = kSmemAlign + kStageBytes + 2 * kCBytes + 2048 + 256 + 1024;
constexpr float kExact = 2097152.0f;       // 2^21
constexpr int kInvCtasPerSm = 3;           // 80 registers a thread, 3 x 73 KB of shared memory an SM

// Expansion selectors: __byte_perm(v, 0, kExpandInit[m]) moves the low
// popc(m) bytes of v to the byte positions flagged in the 4-bit mask m.
__constant__ uint32_t kExpandInit[16] = {
    0x4444, 0x4440, 0x4404, 0x4410, 0x4044, 0x4140, 0x4104, 0x4210,
    0x0444, 0x1440, 0x1404, 0x2410, 0x1044, 0x2140, 0x2104, 0x3210};

__device__ __forceinline__ void cp_async4(uint32_t* dst, const uint32_t* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16s(uint32_t* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Stages chunk c's payload (from the 16-byte boundary at or below its first
// byte when the stream is 16-byte aligned, else the 4-byte one) into Cw.
// Returns the header word in e, the first byte's offset from that boundary in
// lead, and ok = the payload lies inside the stream.
__device__ __forceinline__ void stage_chunk(const InvArgs& a, uint32_t c, uint32_t* Cw, uint32_t& e,
                                            uint32_t& lead, bool& ok) {
    e = reinterpret_cast<const uint32_t*>(a.rze + 8)[c];
    const uint64_t off = a.in_off[c];
    const uint32_t comp = e & 0x7fffffffu;
    ok = off + comp <= a.rze_bytes;
    const uint8_t* src = a.rze + (ok ? off : 0);
    const uint32_t ncopy = ok ? min(comp, (uint32_t)kChunkBytes) : 0u;
    const uint8_t* end = a.rze + a.rze_bytes;
    if ((reinterpret_cast<uintptr_t>(a.rze) & 15u) == 0) {
        // a 16-byte aligned stream: 16-byte copies from the 16-byte boundary
        // at or below the first byte (never below the stream's start)
        lead = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 15u);
        const uint32_t ng = (lead + ncopy + 15) >> 4;
        const uint8_t* g0 = src - lead;
        for (uint32_t i = threadIdx.x; i < ng; i += kThreads) {
            const uint8_t* p = g0 + 16u * i;
            if (p + 16 <= end) {
                cp_async16s(Cw + 4u * i, p);
            } else {  // the stream's last bytes: only those inside it
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    uint32_t v = 0;
                    for (int b = 0; b < 4; b++)
                        if (p + 4 * w + b < end) v |= (uint32_t)p[4 * w + b] << (8 * b);
                    Cw[4u * i + w] = v;
                }
            }
        }
        cp_async_commit();
        return;
    }
    lead = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 3u);
    const uint32_t nw = (lead + ncopy + 3) >> 2;
    const uint32_t* gw = reinterpret_cast<const uint32_t*>(src - lead);
    for (uint32_t i = threadIdx.x; i < nw; i += kThreads) {
        const uint8_t* p = reinterpret_cast<const uint8_t*>(gw + i);
        if (p + 4 <= end) {
            cp_async4(Cw + i, gw + i);
        } else {  // last word of the stream: only the bytes inside it
            uint32_t v = 0;
            for (int b = 0; b < 4; b++)
                if (p + b < end) v |= (uint32_t)p[b] << (8 * b);
            Cw[i] = v;
        }
    }
    cp_async_commit();
}

// 4 bytes of the staged chunk starting at payload byte q (lead included).
__device__ __forceinline__ uint32_t staged_word(const uint32_t* Cw, uint32_t q) {
    return __funnelshift_r(Cw[q >> 2], Cw[(q >> 2) + 1], 8u * (q & 3u));
}

__device__ __forceinline__ uint32_t staged_byte(const uint32_t* Cw, uint32_t q) {
    return (Cw[q >> 2] >> (8u * (q & 3u))) & 0xffu;
}

// Packed code pair -> two biased 16-bit values u = s + 32768 (s the signed
// delta): zigzag inverse (zigzag.h:80-84) or plain int16.
template <bool ZZ>
__device__ __forceinline__ uint32_t biased_pair(uint32_t x) {
    if (ZZ) {
        const uint32_t nb = 0x80008000u - (x & 0x00010001u);  // per half: bit0 ? 0x7fff : 0x8000
        return ((x >> 1) & 0x7fff7fffu) ^ nb;
    }
    return x ^ 0x80008000u;
}

}  // namespace

namespace {

template <bool ZZ>
__global__ void __launch_bounds__(kThreads, kInvCtasPerSm) lq3d_inv_slab_kernel(InvArgs a, uint32_t slabs, uint32_t units) {
    extern __shared__ uint8_t dsm[];
    __shared__ uint32_t s_exp[16];
    __shared__ uint32_t s_tot[8][4];    // per warp: inclusive plane counts, 8-bit fields
    __shared__ uint32_t s_base[8][16];  // per warp, per plane: level-1 byte offset
    __shared__ uint32_t s_om[kThreads];     // per segment: outlier positions of the chunk
    __shared__ uint32_t s_first[kThreads];  // per segment: its first outlier list entry
    __shared__ uint32_t s_misc[4];          // 0 level-1 size s1, 1 malformed flag

    // launched as a programmatic dependent: the prepass offsets, outlier
    // ranges and error word are read after the kernels before have ended
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (*a.err & (kErrUnsorted | kErrMalformed)) return;
    uint8_t* base = dsm + ((kSmemAlign - (smem_u32(dsm) & (kSmemAlign - 1))) & (kSmemAlign - 1));
    uint8_t* X = base;  // x-prefixed plane, 128-byte swizzled rows (one per thread)
    uint32_t* Cbuf = reinterpret_cast<uint32_t*>(base + kStageBytes);
    uint32_t* bm1 = reinterpret_cast<uint32_t*>(base + kStageBytes + 2 * kCBytes);
    uint8_t* bm2 = reinterpret_cast<uint8_t*>(bm1) + 2048;
    uint32_t* pfx2 = reinterpret_cast<uint32_t*>(bm2 + 256);

    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t full = 0xffffffffu;
    const uint32_t nx = a.nx, R = kChunkCodes / nx, S = nx / 32, G = gridDim.x;
    const uint32_t xq = nx / 4, band = t / xq, x4 = t % xq;  // column strip of this thread
    const float ebx2 = inv_ebx2(a);
    const uint32_t nout = min(*a.out_count, a.cap);
    bool inexact = false, malformed = false;

    if (t < 16) s_exp[t] = kExpandInit[t];
    s_om[t] = 0;

    auto unit_z0 = [&](uint32_t uu) { return ((units - 1 - uu) / slabs) * 8u; };
    uint32_t ce = 0, clead = 0;
    bool cok = false;
    if (blockIdx.x < units) {
        const uint32_t u = units - 1 - blockIdx.x;
        stage_chunk(a, unit_z0(blockIdx.x) * slabs + u % slabs, Cbuf, ce, clead, cok);
    }

    // Output pass of one decoded plane (x-prefixed rows in X): the thread's
    // column strip gets its y prefix, the running z sum and 16-byte stores.
    float acc[32];
#pragma unroll
    for (int i = 0; i < 32; i++) acc[i] = 0.0f;
    auto strip = [&](uint32_t sz, uint32_t ss, bool chk) {
        float2 y0 = f2(0.0f, 0.0f), y1 = y0;
        float mx = 0.0f;
        const float2 e2 = f2(ebx2, ebx2);
        float* orow = a.out + ((size_t)sz * a.ny + (size_t)ss * R + band * 8u) * nx + 4u * x4;
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const uint32_t own = (band * 8u + r) * S + (x4 >> 3);
            const float4 v = *reinterpret_cast<const float4*>(X + swz_off(own, x4 & 7u));
            if (r == 0) {
                y0 = f2(v.x, v.y);
                y1 = f2(v.z, v.w);
            } else {
                y0 = __fadd2_rn(y0, f2(v.x, v.y));
                y1 = __fadd2_rn(y1, f2(v.z, v.w));
            }
            if (chk) mx = max_nan(max_nan(mx, fmaxf(fabsf(y0.x), fabsf(y0.y))), fmaxf(fabsf(y1.x), fabsf(y1.y)));
            const float2 a0 = __fadd2_rn(f2(acc[4 * r], acc[4 * r + 1]), y0);
            const float2 a1 = __fadd2_rn(f2(acc[4 * r + 2], acc[4 * r + 3]), y1);
            acc[4 * r] = a0.x;
            acc[4 * r + 1] = a0.y;
            acc[4 * r + 2] = a1.x;
            acc[4 * r + 3] = a1.y;
            const float2 o0v = __fmul2_rn(a0, e2), o1v = __fmul2_rn(a1, e2);
            *reinterpret_cast<float4*>(orow + (size_t)r * nx) = make_float4(o0v.x, o0v.y, o1v.x, o1v.y);
        }
        if (chk && !(mx < kExact)) inexact = true;
    };
    bool pend = false, pchk = false;
    uint32_t pz = 0, ps = 0;

    uint32_t k = 0;
    for (uint32_t uu = blockIdx.x; uu < units; uu += G) {
        const uint32_t u = units - 1 - uu, s = u % slabs;
        const uint32_t z0 = (u / slabs) * 8u, z1 = min(z0 + 8u, a.nz);
        for (uint32_t z = z0; z < z1; z++, k++) {
            const uint32_t c = z * slabs + s;
            const uint32_t* Cw = Cbuf + (k & 1) * (kCBytes / 4);
            cp_async_wait_all();
            __syncthreads();  // B0: chunk c staged; the previous plane's X rows are complete
            const uint32_t e = ce, lead = clead;
            const bool ok = cok;
            {   // stage the next plane's chunk into the other buffer
                uint32_t nu = uu, nz = z + 1;
                if (nz >= z1) {
                    nu = uu + G;
                    nz = nu < units ? unit_z0(nu) : 0u;
                }
                if (nu < units)
                    stage_chunk(a, nz * slabs + (units - 1 - nu) % slabs, Cbuf + ((k + 1) & 1) * (kCBytes / 4), ce,
                                clead, cok);
            }
            if (pend) strip(pz, ps, pchk);  // the previous plane (X is complete since B0)
            if (z == z0) {
#pragma unroll
                for (int i = 0; i < 32; i++) acc[i] = 0.0f;
            }

            // 0: RZE levels, 1: zeros, 2: stored raw (rze_stage.cu:904-930 cases)
            const uint32_t comp = e & 0x7fffffffu;
            int kind;
            bool bad = !ok;
            if (bad) kind = 1;
            else if (e >> 31) {
                kind = 2;
                if (comp < (uint32_t)kChunkBytes) { bad = true; kind = 1; }
            } else if (comp <= 2) kind = 1;
            else if (comp > (uint32_t)kChunkBytes || comp < 7) { bad = true; kind = 1; }
            else kind = 0;

            if (kind == 0 && warp == 0) {  // levels 4 -> 2
                const uint32_t q4 = lead + comp - 6;
                const uint32_t bm4 = staged_word(Cw, q4);
                const int t3 = (int)comp - 6 - __popc(bm4);
                bool b = t3 < 0;
                // bm3 byte `lane` (b3 = 32)
                const uint32_t r3 = __popc(bm4 & (0xffffffffu >> (31 - lane)));
                const uint32_t v3 = (r3 && !b) ? staged_byte(Cw, lead + (uint32_t)t3 + r3 - 1) : 0u;
                const uint32_t p3 = __popc(v3);
                uint32_t i3 = p3;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t n = __shfl_up_sync(full, i3, d);
                    if (lane >= (uint32_t)d) i3 += n;
                }
                const int t2 = t3 - (int)__shfl_sync(full, i3, 31);
                b = b || t2 < 0;
                // bm2 bytes 8*lane .. 8*lane+7 from bm3 byte `lane`
                uint32_t w2[2] = {0u, 0u}, q2[8];
                uint32_t run = 0;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const uint32_t rk = i3 - p3 + __popc(v3 & (0xffu >> (7 - j)));
                    const uint32_t v = (rk && !b) ? staged_byte(Cw, lead + (uint32_t)t2 + rk - 1) : 0u;
                    w2[j >> 2] |= v << (8 * (j & 3));
                    q2[j] = run;
                    run += __popc(v);
                }
                uint32_t i2 = run;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t n = __shfl_up_sync(full, i2, d);
                    if (lane >= (uint32_t)d) i2 += n;
                }
                const int t1 = t2 - (int)__shfl_sync(full, i2, 31);
                b = b || t1 < 0;
                reinterpret_cast<uint2*>(bm2)[lane] = make_uint2(w2[0], w2[1]);
#pragma unroll
                for (int j = 0; j < 8; j++) pfx2[8 * lane + j] = i2 - run + q2[j];
                if (lane == 0) {
                    s_misc[0] = b ? 0u : (uint32_t)t1;
                    s_misc[1] = b ? 1u : 0u;
                }
            }
            // mark this chunk's outliers per 32-element segment
            const uint32_t o0 = a.ostart[c], o1 = min(a.ostart[c + 1], nout);
            const uint32_t kbase = c * (uint32_t)kChunkCodes;
            for (uint32_t i = o0 + t; i < o1; i += kThreads) {
                const uint32_t m = a.out_idx[i] - kbase;
                if (m < (uint32_t)kChunkCodes) {
                    atomicOr(&s_om[m >> 5], 1u << (m & 31));
                    if (i == o0 || ((a.out_idx[i - 1] - kbase) >> 5) != (m >> 5)) s_first[m >> 5] = i;
                }
            }
            __syncthreads();  // B1

            uint32_t s1 = 0;
            if (kind == 0) {
                s1 = s_misc[0];
                if (s_misc[1]) { bad = true; kind = 1; }
            }
            if (kind == 0) {  // bm1 bytes 8t .. 8t+7
                const uint32_t m2 = bm2[t], ex = pfx2[t];
                uint32_t w1[2] = {0u, 0u};
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const uint32_t rk = ex + __popc(m2 & (0xffu >> (7 - j)));
                    const uint32_t v = rk ? staged_byte(Cw, lead + s1 + rk - 1) : 0u;
                    w1[j >> 2] |= v << (8 * (j & 3));
                }
                reinterpret_cast<uint2*>(bm1)[t] = make_uint2(w1[0], w1[1]);
            }
            __syncthreads();  // B2

            // this thread's 16 plane nibbles and the per-plane level-1 offsets
            uint64_t nib64 = 0;
            uint32_t pm = 0, KX[4] = {0u, 0u, 0u, 0u};
            if (kind == 0) {
                const uint32_t j = lane & 7u;
                nib64 = nibs_from_bm1(bm1[(15 - 2 * j) * 32 + (t >> 3)], bm1[(14 - 2 * j) * 32 + (t >> 3)], lane);
                uint32_t K[4] = {0u, 0u, 0u, 0u}, mine = 0;
#pragma unroll
                for (int b = 0; b < 16; b++) {
                    const uint32_t nb = (uint32_t)(nib64 >> (4 * b)) & 15u;
                    K[b >> 2] += (uint32_t)__popc(nb) << (8 * (b & 3));
                    mine |= (nb ? 1u : 0u) << b;
                }
                pm = __reduce_or_sync(full, mine);
                uint32_t act = 0;
#pragma unroll
                for (int jj = 0; jj < 4; jj++) act |= (((pm >> (4 * jj)) & 15u) ? 1u : 0u) << jj;
                warp_scan4(K, act, KX);
                if (lane == 31) {
#pragma unroll
                    for (int jj = 0; jj < 4; jj++) s_tot[warp][jj] = ((act >> jj) & 1u) ? KX[jj] : 0u;
                }
#pragma unroll
                for (int jj = 0; jj < 4; jj++) KX[jj] = ((act >> jj) & 1u) ? KX[jj] - K[jj] : 0u;
            }
            __syncthreads();  // B3
            if (kind == 0 && warp == 0) {
                const uint32_t b = lane & 15u, h = lane >> 4;
                uint32_t cnt[4];
#pragma unroll
                for (int i = 0; i < 4; i++) cnt[i] = (s_tot[4 * h + i][b >> 2] >> (8 * (b & 3u))) & 0xffu;
                const uint32_t gs = cnt[0] + cnt[1] + cnt[2] + cnt[3];
                const uint32_t other = __shfl_xor_sync(full, gs, 16);
                const uint32_t T = gs + other;
                uint32_t suf = T;  // planes >= b come first (plane 15 leads)
#pragma unroll
                for (uint32_t d = 1; d < 16; d <<= 1) {
                    const uint32_t n = __shfl_down_sync(full, suf, d, 16);
                    if (b + d < 16) suf += n;
                }
                uint32_t off = suf - T + (h ? other : 0u);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    s_base[4 * h + i][b] = off;
                    off += cnt[i];
                }
                if (lane == 0 && suf != s1) s_misc[1] = 1u;  // bitmap and payload disagree
            }
            __syncthreads();  // B4
            if (kind == 0 && s_misc[1]) { bad = true; kind = 1; }
            if (bad) malformed = true;

            // plane words -> codes
            uint32_t x[16];
#pragma unroll
            for (int b = 0; b < 16; b++) x[b] = 0u;
            if (kind == 0) {
#pragma unroll
                for (int b = 0; b < 16; b++) {
                    if ((pm >> b) & 1u) {
                        const uint32_t nb = (uint32_t)(nib64 >> (4 * b)) & 15u;
                        const uint32_t pos = s_base[warp][b] + ((KX[b >> 2] >> (8 * (b & 3))) & 0xffu);
                        x[b] = __byte_perm(staged_word(Cw, lead + pos), 0u, s_exp[nb]);
                    }
                }
            } else if (kind == 2) {
#pragma unroll
                for (int b = 0; b < 16; b++) x[b] = staged_word(Cw, lead + 4u * ((15u - b) * 256u + t));
            }
            transpose16x2(x);

            // codes -> deltas (u - 32768 through 1.5*2^23 + u), outliers, x prefix.
            // Words x[8h..8h+7] hold elements 8h..8h+7 (low halves) and
            // 16+8h..23+8h (high halves): one x-prefix group each, so only
            // sixteen deltas are live at a time.
            const float2 nb2 = f2(-(kMagic + 32768.0f), -(kMagic + 32768.0f));
            auto deltas = [&](int h, float (&lo)[8], float (&hi)[8]) {
#pragma unroll
                for (int kk = 0; kk < 8; kk += 2) {
                    const uint32_t p0 = biased_pair<ZZ>(x[8 * h + kk]), p1 = biased_pair<ZZ>(x[8 * h + kk + 1]);
                    const float2 l = __fadd2_rn(f2(__uint_as_float(__byte_perm(p0, 0x4b400000u, 0x7610)),
                                                   __uint_as_float(__byte_perm(p1, 0x4b400000u, 0x7610))), nb2);
                    const float2 u = __fadd2_rn(f2(__uint_as_float(__byte_perm(p0, 0x4b400000u, 0x7632)),
                                                   __uint_as_float(__byte_perm(p1, 0x4b400000u, 0x7632))), nb2);
                    lo[kk] = l.x;
                    lo[kk + 1] = l.y;
                    hi[kk] = u.x;
                    hi[kk + 1] = u.y;
                }
            };
            // group i (elements 8i..8i+7) <-> granules 2i, 2i+1 of the thread's row of X
            auto put = [&](int i, const float (&v)[8]) {
                *reinterpret_cast<float4*>(X + swz_off(t, 2 * i)) = make_float4(v[0], v[1], v[2], v[3]);
                *reinterpret_cast<float4*>(X + swz_off(t, 2 * i + 1)) = make_float4(v[4], v[5], v[6], v[7]);
            };
            auto scan8 = [](float (&v)[8]) {
#pragma unroll
                for (int jj = 1; jj < 8; jj++) v[jj] = __fadd_rn(v[jj], v[jj - 1]);
            };
            const bool checked = o1 > o0;  // uniform: the chunk carries outliers
            if (!checked) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    float lo[8], hi[8];
                    deltas(h, lo, hi);
                    scan8(lo);
                    scan8(hi);
                    put(h, lo);
                    put(2 + h, hi);
                }
            } else {  // add the outliers through the thread's own row of X
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    float lo[8], hi[8];
                    deltas(h, lo, hi);
                    put(h, lo);
                    put(2 + h, hi);
                }
                const uint32_t om = s_om[t];
                if (om) {
                    s_om[t] = 0;
                    for (uint32_t p = s_first[t]; p < o1; p++) {
                        const uint32_t m = a.out_idx[p] - kbase;
                        if ((m >> 5) != t) break;
                        float* q = reinterpret_cast<float*>(X + swz_off(t, (m & 31u) >> 2)) + (m & 3u);
                        const float v = __fadd_rn(a.out_err[p], *q);
                        *q = v;
                        if (!(fabsf(v) < kExact)) inexact = true;
                    }
                }
                float mx = 0.0f;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float4 v0 = *reinterpret_cast<const float4*>(X + swz_off(t, 2 * i));
                    const float4 v1 = *reinterpret_cast<const float4*>(X + swz_off(t, 2 * i + 1));
                    float v[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
                    scan8(v);
#pragma unroll
                    for (int jj = 0; jj < 8; jj++) mx = max_nan(mx, fabsf(v[jj]));
                    put(i, v);
                }
                if (!(mx < kExact)) inexact = true;
            }
            // this plane's output pass runs after the next B0
            pend = true;
            pz = z;
            ps = s;
            pchk = checked;
        }
    }
    if (pend) {  // the last plane
        __syncthreads();
        strip(pz, ps, pchk);
    }
    cp_async_wait_all();
    if (__any_sync(full, inexact) && lane == 0) atomicOr(a.err, kErrInexact);
    if (__any_sync(full, malformed) && lane == 0) atomicOr(a.err, kErrMalformed);
}

}  // namespace

int launch_lq3d_inv_slab(const InvArgs& a, unsigned sms, cudaStream_t s) {
    const uint32_t slabs = a.ny / (kChunkCodes / a.nx), units = slabs * ((a.nz + 7) / 8);
    unsigned grid = sms * kInvCtasPerSm;
    grid = grid < units ? grid : units;
    cudaError_t e;
    if (a.zigzag) {
        static SmemAttr attr;
        e = ensure_dyn_smem(attr, (const void*)lq3d_inv_slab_kernel<true>, (int)kInvSmem);
        if (e != cudaSuccess) return (int)e;
        e = launch_dependent(lq3d_inv_slab_kernel<true>, grid, kThreads, kInvSmem, s, a, slabs, units);
        if (e != cudaSuccess) return (int)e;
    } else {
        static SmemAttr attr;
        e = ensure_dyn_smem(attr, (const void*)lq3d_inv_slab_kernel<false>, (int)kInvSmem);
        if (e != cudaSuccess) return (int)e;
        e = launch_dependent(lq3d_inv_slab_kernel<false>, grid, kThreads, kInvSmem, s, a, slabs, units);
        if (e != cudaSuccess) return (int)e;
    }
    return (int)cudaGetLastError();
}

}  // namespace fzb
