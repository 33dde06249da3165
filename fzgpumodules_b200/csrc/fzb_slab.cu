// fzb_slab.cu -- TMA-fed slab kernel for the fused 3-D chain
// LorenzoQuant(3-D) -> Bitshuffle(16 KiB, element width 2) -> RZE(16 KiB).
//
// Applies to 3-D fields whose 8192-element chunks are R = 8192/nx whole rows
// (nx a power of two in [32, 1024], ny % R == 0, no padding).  A work unit is
// one R-row slab across one 8-plane z tile; the unit's chunks are produced
// plane by plane by one persistent CTA of 512 threads (two CTAs per SM).
//
// Data flow per chunk (= one slab plane), four CTA barriers:
//   * one thread issues a 2-D TMA copy of the 32 KiB plane into a 128-byte
//     swizzled shared buffer one plane ahead of use (double buffer, mbarrier
//     completion, bounded waits);
//   * thread t owns chunk elements 16t..16t+15 (half of one 32-wide x
//     segment of one row).  It quantizes them (f32x2 adds, scalar products),
//     forms the z difference against the previous plane's q held in
//     registers and the x difference in registers, writes B = (z, x)-
//     differenced values back over its own bytes of the buffer, and after
//     barrier B1 reads the row above for the y difference
//     (lorenzo_quant_nd.cu:236-246 order);
//   * codes come from the exact integer-valued deltas through the float
//     magic-number conversion (c + 1.5*2^23 holds c in its low mantissa
//     bits), zigzag works on packed code pairs, outliers are found per
//     4-element granule with a NaN-propagating max;
//   * the 16 codes are bit-transposed in registers (the Bitshuffle ballot
//     layout, bitshuffle_stage.cu:299-323) and stored as the shuffled chunk S
//     in shared memory (B2);
//   * RZE (rze_stage.cu:324-445): thread t reads S words 8t..8t+7, forms
//     their nonzero-byte nibbles (level-1 bitmap word t) and the level-2 bits
//     of its four bm1 bytes; one packed warp scan counts both levels, and
//     after B3 the warp totals give every thread its payload offsets.  Each
//     thread compacts the nonzero bytes of its word pairs (two byte permutes
//     from a 256-entry selector table) into a zeroed payload buffer with
//     shared atomics; meanwhile warp 0 codes levels 3 and 4 and the trailer;
//   * after B4 the encoded chunk goes to its 16 KiB slot; assemble_scan /
//     assemble_copy (fzb_forward.cu) place slots and staged outliers exactly
//     as for the other chunk kernels.
#include "fzb_slab.cuh"

namespace fzb {
namespace {

constexpr int kOBytes = kChunkBytes + 128;    // level payload (+ slack for the second atomic word)
constexpr size_t kSlabSmem = kSmemAlign + 2 * kStageBytes + kOBytes + kChunkBytes + 256;

}  // namespace

namespace {

constexpr int kTT = 512;  // threads of a slab-compressor CTA: 16 chunk elements each

// Byte offset of 16-byte granule g (0..3) of thread t's elements 16t..16t+15
// in a swizzled plane buffer (two threads per 128-byte row).
__device__ __forceinline__ uint32_t thr_off(uint32_t t, uint32_t g) {
    return swz_off(t >> 1, 4u * (t & 1u) + g);
}

// ---------------------------------------------------------------------------
// Codes of one thread's 16 elements from B (z- and x-differenced) and the
// row above (read from the swizzled exchange buffer when ty != 0).
// x[k] = code[k] | code[k + 8] << 16; om4 bit g = granule g (elements
// 4g..4g+3) may hold an outlier.  Outlier codes are not zeroed here.
// ---------------------------------------------------------------------------
template <bool ZZ>
__device__ __forceinline__ void make_codes16(const float (&B)[16], const uint8_t* stg, uint32_t tu, bool ty,
                                             float R, uint32_t (&x)[8], uint32_t& om4) {
    om4 = 0;
#pragma unroll
    for (int g = 0; g < 2; g++) {
        float c[8];  // elements 4g..4g+3 and 8+4g..8+4g+3
        if (ty) {
            const float4 u0 = *reinterpret_cast<const float4*>(stg + thr_off(tu, g));
            const float4 u1 = *reinterpret_cast<const float4*>(stg + thr_off(tu, g + 2));
            float2 d;
            d = sub2(f2(B[4 * g], B[4 * g + 1]), f2(u0.x, u0.y));  c[0] = d.x; c[1] = d.y;
            d = sub2(f2(B[4 * g + 2], B[4 * g + 3]), f2(u0.z, u0.w));  c[2] = d.x; c[3] = d.y;
            d = sub2(f2(B[8 + 4 * g], B[9 + 4 * g]), f2(u1.x, u1.y));  c[4] = d.x; c[5] = d.y;
            d = sub2(f2(B[10 + 4 * g], B[11 + 4 * g]), f2(u1.z, u1.w));  c[6] = d.x; c[7] = d.y;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                c[k] = B[4 * g + k];
                c[4 + k] = B[8 + 4 * g + k];
            }
        }
        const float m0 = max_nan(max_nan(fabsf(c[0]), fabsf(c[1])), max_nan(fabsf(c[2]), fabsf(c[3])));
        const float m1 = max_nan(max_nan(fabsf(c[4]), fabsf(c[5])), max_nan(fabsf(c[6]), fabsf(c[7])));
        if (!(m0 < R)) om4 |= 1u << g;
        if (!(m1 < R)) om4 |= 1u << (g + 2);
        const float2 M2 = make_float2(kMagic, kMagic);
        float cm[8];
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
            const float2 d = __fadd2_rn(f2(c[k], c[k + 1]), M2);
            cm[k] = d.x;
            cm[k + 1] = d.y;
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            uint32_t p = __byte_perm(__float_as_uint(cm[k]), __float_as_uint(cm[4 + k]), 0x5410);
            if (ZZ) {
                uint32_t s;
                asm("prmt.b32 %0, %1, %1, 0xBB99;" : "=r"(s) : "r"(p));  // per-half sign mask
                p = ((p << 1) & 0xfffefffeu) ^ s;
            }
            x[4 * g + k] = p;
        }
    }
}

// Exact outlier mask (bit e = element e) for the granules flagged in om4,
// recomputed from the exchange buffer (the thread's own B and the row above).
__device__ __forceinline__ uint32_t outlier_mask16(const uint8_t* stg, uint32_t t, uint32_t tu, bool ty, float R,
                                                   uint32_t om4) {
    uint32_t om = 0;
    while (om4) {
        const uint32_t g = __ffs(om4) - 1;
        om4 &= om4 - 1;
        const float4 b = *reinterpret_cast<const float4*>(stg + thr_off(t, g));
        float c[4] = {b.x, b.y, b.z, b.w};
        if (ty) {
            const float4 u = *reinterpret_cast<const float4*>(stg + thr_off(tu, g));
            c[0] = __fsub_rn(c[0], u.x);
            c[1] = __fsub_rn(c[1], u.y);
            c[2] = __fsub_rn(c[2], u.z);
            c[3] = __fsub_rn(c[3], u.w);
        }
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (!(fabsf(c[k]) < R)) om |= 1u << (4 * g + k);
    }
    return om;
}

// Delta of element e (the value an outlier record stores).
__device__ __forceinline__ float delta_at16(const uint8_t* stg, uint32_t t, uint32_t tu, bool ty, uint32_t e) {
    float c = *(reinterpret_cast<const float*>(stg + thr_off(t, e >> 2)) + (e & 3));
    if (ty) c = __fsub_rn(c, *(reinterpret_cast<const float*>(stg + thr_off(tu, e >> 2)) + (e & 3)));
    return c;
}

// In-place transpose of a 16x16 bit matrix held as x[k] = row k | row (k+8)
// << 16: afterwards x[m] = column m | column (m+8) << 16, bit i of a column
// = bit of row i.  With rows = codes this yields the bit planes of the 16
// codes (the Bitshuffle ballot layout, bitshuffle_stage.cu:299-323, for half
// of a 32-code group).  The 8x8 off-diagonal blocks swap by a byte permute,
// then each byte lane transposes its 8x8 block in three stages.
__device__ __forceinline__ void transpose16(uint32_t (&x)[8]) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = __byte_perm(x[k], 0u, 0x3120);
#pragma unroll
    for (int s = 4; s >= 1; s >>= 1) {
        const uint32_t m = (s == 4) ? 0x0f0f0f0fu : (s == 2) ? 0x33333333u : 0x55555555u;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (i & s) continue;
            const uint32_t d = ((x[i] >> s) ^ x[i + s]) & m;
            x[i + s] ^= d;
            x[i] ^= d << s;
        }
    }
}

// Compaction selectors: __byte_perm(w, 0, kSelInit[m]) moves the bytes of w
// flagged in the 4-bit mask m to the low end, in order, zero-filled.
__constant__ uint32_t kSelInit[16] = {
    0x4444, 0x4440, 0x4441, 0x4410, 0x4442, 0x4420, 0x4421, 0x4210,
    0x4443, 0x4430, 0x4431, 0x4310, 0x4432, 0x4320, 0x4321, 0x3210};

// ORs the 4 bytes of `packed` (the low popc bytes meaningful) into the
// zeroed byte stream O at byte offset pos.
__device__ __forceinline__ void or_bytes_at(uint32_t* Ow, uint32_t pos, uint32_t packed) {
    const uint32_t sh = (pos & 3u) * 8u;
    atomicOr(&Ow[pos >> 2], packed << sh);
    atomicOr(&Ow[(pos >> 2) + 1], __funnelshift_l(packed, 0u, sh));
}

}  // namespace

namespace {

template <bool ZZ>
__global__ void __launch_bounds__(kTT, 2)
    lq3d_tma_kernel(const FwdArgs a, const __grid_constant__ CUtensorMap map, uint32_t slabs, uint32_t units) {
    extern __shared__ uint8_t dsm[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_sel[16];
    __shared__ uint2 s_sel8[256];  // pair compaction selectors: set bytes first, then a zero byte
    __shared__ uint32_t s_wout[kTT / 32];  // per warp: outlier count
    __shared__ uint32_t s_l1[kTT / 32];    // per warp: level-1 | level-2 << 16 byte counts
    __shared__ uint32_t s_misc[4];         // 1 outlier staging base, 2 size word

    uint8_t* base = dsm + ((kSmemAlign - (smem_u32(dsm) & (kSmemAlign - 1))) & (kSmemAlign - 1));
    uint8_t* O = base + 2 * kStageBytes;
    uint32_t* Ow = reinterpret_cast<uint32_t*>(O);
    uint8_t* Sbuf = O + kOBytes;  // the shuffled chunk (16 KiB)
    uint32_t* Sw = reinterpret_cast<uint32_t*>(Sbuf);
    uint16_t* Sh = reinterpret_cast<uint16_t*>(Sbuf);
    uint8_t* bm2 = Sbuf + kChunkBytes;

    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t full = 0xffffffffu;
    const uint32_t nx = a.nx, R = kChunkCodes / nx, S16 = nx / 16;  // threads per row
    const bool ty = ((t / S16) & 7u) != 0;  // slab origins have y % 8 == 0
    const uint32_t tu = ty ? t - S16 : t;   // thread holding the row above
    const float rad = a.radius;
    const uint32_t G = gridDim.x;

    if (t < 16) s_sel[t] = kSelInit[t];
    if (t < 256) {  // mask t: the flagged bytes of a word pair in order, then a zero (unflagged) byte
        uint32_t sel = 0, k = 0, zb = 0;
        for (uint32_t b = 0; b < 8; b++)
            if (!((t >> b) & 1u)) {
                zb = b;
                break;
            }
        for (uint32_t b = 0; b < 8; b++)
            if ((t >> b) & 1u) sel |= b << (4 * k++);
        for (; k < 8; k++) sel |= zb << (4 * k);
        s_sel8[t] = make_uint2(sel & 0xffffu, sel >> 16);  // output bytes 0-3 and 4-7
    }
    for (uint32_t i = t; i < (uint32_t)kOBytes / 16; i += kTT) reinterpret_cast<uint4*>(O)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (t == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // plane sequence of this CTA: units blockIdx.x, +G, ... (last to first),
    // each from its tile's first plane; thread 0 keeps the issue cursor
    auto unit_z0 = [&](uint32_t uu) { return ((units - 1 - uu) / slabs) * 8u; };
    uint32_t iu = blockIdx.x, iz = iu < units ? unit_z0(iu) : 0u;
    auto issue_next = [&](uint32_t seq) {
        if (iu >= units) return;
        const uint32_t s = (units - 1 - iu) % slabs;
        const int row = (int)((((size_t)iz * a.ny + (size_t)s * R) * nx) >> 5);
        uint64_t* bar = &s_bar[seq & 1];
        mbar_expect_tx(bar, kStageBytes);
        tma_load_rows(base + (seq & 1) * kStageBytes, &map, row, bar);
        if (++iz >= min(unit_z0(iu) + 8u, a.nz)) {
            iu += G;
            if (iu < units) iz = unit_z0(iu);
        }
    };
    if (t == 0) {
        issue_next(0);
        issue_next(1);
    }
    // Launched as a programmatic dependent of the value-base scan: the set-up
    // above and the first two plane copies (the field is not the scan's
    // output) overlap the scan's tail; the error bound is read after it.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const float r = *a.ebx2_r;

    uint32_t k = 0;  // plane sequence number
    for (uint32_t uu = blockIdx.x; uu < units; uu += G) {
        const uint32_t u = units - 1 - uu, s = u % slabs;
        const uint32_t z0 = (u / slabs) * 8u, z1 = min(z0 + 8u, a.nz);
        float qp[16];
        for (uint32_t z = z0; z < z1; z++, k++) {
            const uint32_t c = z * slabs + s;
            const bool tz = z != z0;
            uint8_t* stg = base + (k & 1) * kStageBytes;
            const bool bad = !mbar_wait_bounded(&s_bar[k & 1], (k >> 1) & 1u);

            // q, z difference, x difference; B over the thread's own bytes
            float B[16];
            float alast = 0.0f;
#pragma unroll
            for (int g = 0; g < 4; g++) {
                const float4 v = *reinterpret_cast<const float4*>(stg + thr_off(t, g));
                // scalar products: a packed multiply followed by the packed add
                // below can be contracted into one fused multiply-add, which
                // rounds differently when v*r lies next to a rounding midpoint
                const float2 y0 = f2(__fmul_rn(v.x, r), __fmul_rn(v.y, r));
                const float2 y1 = f2(__fmul_rn(v.z, r), __fmul_rn(v.w, r));
                const float2 s0 = __fadd2_rn(y0, f2(__uint_as_float(half_bits(v.x)), __uint_as_float(half_bits(v.y))));
                const float2 s1 = __fadd2_rn(y1, f2(__uint_as_float(half_bits(v.z)), __uint_as_float(half_bits(v.w))));
                const float2 q0 = f2(truncf(s0.x), truncf(s0.y)), q1 = f2(truncf(s1.x), truncf(s1.y));
                float2 A0 = q0, A1 = q1;
                if (tz) {
                    A0 = sub2(q0, f2(qp[4 * g], qp[4 * g + 1]));
                    A1 = sub2(q1, f2(qp[4 * g + 2], qp[4 * g + 3]));
                }
                qp[4 * g] = q0.x;
                qp[4 * g + 1] = q0.y;
                qp[4 * g + 2] = q1.x;
                qp[4 * g + 3] = q1.y;
                // x % 8 == 0 starts a tile: elements 0 and 8 of the thread
                B[4 * g] = (g & 1) ? __fsub_rn(A0.x, alast) : A0.x;
                B[4 * g + 1] = __fsub_rn(A0.y, A0.x);
                B[4 * g + 2] = __fsub_rn(A1.x, A0.y);
                B[4 * g + 3] = __fsub_rn(A1.y, A1.x);
                alast = A1.y;
                *reinterpret_cast<float4*>(stg + thr_off(t, g)) = make_float4(B[4 * g], B[4 * g + 1], B[4 * g + 2], B[4 * g + 3]);
            }
            if (__syncthreads_or(bad)) {  // B1 (a copy did not arrive: give up)
                if (t == 0) {
                    atomicOr(a.err, kErrTmaTimeout);
                    // bounded drain of the copies still in flight
                    mbar_wait_bounded(&s_bar[k & 1], (k >> 1) & 1u);
                    if (k == 0) mbar_wait_bounded(&s_bar[1], 0u);
                }
                __syncthreads();
                return;
            }
            if (t == 0 && k >= 1) issue_next(k + 1);

            // codes, outliers, bit planes
            uint32_t x[8], om4;
            make_codes16<ZZ>(B, stg, tu, ty, rad, x, om4);
            const uint32_t om = om4 ? outlier_mask16(stg, t, tu, ty, rad, om4) : 0u;
            transpose16(x);
            if (__any_sync(full, om != 0u)) {
                const uint32_t keep = ~(om | (om << 16));  // outlier codes are 0
#pragma unroll
                for (int b = 0; b < 8; b++) x[b] &= keep;
            }
            const uint32_t nout = __popc(om);
            uint32_t oex = 0;
            if (__any_sync(full, nout != 0u)) {
                const uint32_t inc = warp_incl_scan(nout);
                oex = inc - nout;
                if (lane == 31) s_wout[warp] = inc;
            } else if (lane == 0) {
                s_wout[warp] = 0;
            }
            // the shuffled chunk S: plane b of the 32-code group j is word
            // (15-b)*256 + j, its low half from thread 2j, high half from 2j+1
#pragma unroll
            for (int b = 0; b < 8; b++) {
                Sh[(15 - b) * 512 + t] = (uint16_t)x[b];
                Sh[(7 - b) * 512 + t] = (uint16_t)(x[b] >> 16);
            }
            __syncthreads();  // B2
            if (t == 0) {  // staging for this chunk's outliers
                uint32_t tot = 0;
#pragma unroll
                for (int w = 0; w < kTT / 32; w++) tot += s_wout[w];
                const uint32_t ob = tot ? atomicAdd(a.ostage_ctr, tot) : 0u;
                a.obase[c] = ob;
                a.ocnt[c] = tot;
                s_misc[1] = ob;
            }

            // RZE levels 1 and 2: thread t takes S words 8t..8t+7 (warp w =
            // plane region w); their nonzero-byte nibbles are bm1 word t
            uint32_t w[8];
            {
                const uint4 q0 = reinterpret_cast<const uint4*>(Sw)[2 * t], q1 = reinterpret_cast<const uint4*>(Sw)[2 * t + 1];
                w[0] = q0.x; w[1] = q0.y; w[2] = q0.z; w[3] = q0.w;
                w[4] = q1.x; w[5] = q1.y; w[6] = q1.z; w[7] = q1.w;
            }
            uint32_t nb1 = 0;
            if (__any_sync(full, (w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7]) != 0u)) {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const uint32_t hb = (((w[i] & 0x7f7f7f7fu) + 0x7f7f7f7fu) | w[i]) & 0x80808080u;
                    nb1 |= ((hb * 0x00204081u) >> (28 - 4 * i)) & (15u << (4 * i));
                }
            }
            // level 2: bm1 bytes that differ from their predecessor
            uint32_t prev = __shfl_up_sync(full, nb1, 1) >> 24;
            if (lane == 0) prev = t ? (nz_nibble(Sw[8 * t - 2]) | (nz_nibble(Sw[8 * t - 1]) << 4)) : 0u;
            const uint32_t m2 = nz_nibble(nb1 ^ ((nb1 << 8) | prev));
            const uint32_t v12 = (uint32_t)__popc(nb1) | ((uint32_t)__popc(m2) << 16);
            const uint32_t inc12 = warp_incl_scan(v12);
            if (lane == 31) s_l1[warp] = inc12;
            {   // bm2 byte t/2 = bm2 bits of bm1 bytes 8(t/2)..: two lanes per byte
                const uint32_t pair = m2 | (__shfl_down_sync(full, m2, 1) << 4);
                if (!(lane & 1u)) bm2[t >> 1] = (uint8_t)pair;
            }
            __syncthreads();  // B3
            uint32_t tot12, pre12 = inc12 - v12;
            {   // warp totals: lane l scans warps 0..l
                const uint32_t v = lane < kTT / 32 ? s_l1[lane] : 0u;
                uint32_t iv = v;
#pragma unroll
                for (int d = 1; d < kTT / 32; d <<= 1) {
                    const uint32_t n = __shfl_up_sync(full, iv, d);
                    if (lane >= (uint32_t)d) iv += n;
                }
                pre12 += __shfl_sync(full, iv - v, warp);
                tot12 = __shfl_sync(full, iv, kTT / 32 - 1);
            }
            const uint32_t nzT = tot12 & 0xffffu, n2T = tot12 >> 16;

            if (om) {  // outlier records, ascending index within the chunk
                uint32_t pos = s_misc[1] + oex;
                for (uint32_t w8 = 0; w8 < warp; w8++) pos += s_wout[w8];
                const uint32_t kb = c * (uint32_t)kChunkCodes + 16u * t;
                uint32_t m = om;
                while (m) {
                    const uint32_t e = __ffs(m) - 1;
                    m &= m - 1;
                    if (pos < a.ostage_cap) {
                        a.ostage_err[pos] = delta_at16(stg, t, tu, ty, e);
                        a.ostage_idx[pos] = kb + e;
                    }
                    pos++;
                }
            }

            // 0: encode, 1: all-zero chunk, 2: stored raw (rze_stage.cu:365-389)
            int mode = nzT == 0 ? 1 : ((nzT >= (uint32_t)kRzeAvail || nzT > (uint32_t)(kRzeAvail - 2048)) ? 2 : 0);
            const uint32_t wpos = nzT + n2T;
            if (mode == 0 && (wpos >= (uint32_t)kRzeAvail || wpos > (uint32_t)(kRzeAvail - 256))) mode = 2;
            if (mode == 0) {
                // level-1 payload: the nonzero bytes of each word pair, compacted
                // by two byte permutes and ORed into the zeroed payload buffer
                uint32_t pos = pre12 & 0xffffu;
                if (nb1)  // threads of all-zero plane regions skip the loop
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const uint32_t m8 = (nb1 >> (8 * i)) & 0xffu;
                    if (m8) {
                        const uint2 sel = s_sel8[m8];
                        const uint32_t lo = __byte_perm(w[2 * i], w[2 * i + 1], sel.x);
                        const uint32_t hi = __byte_perm(w[2 * i], w[2 * i + 1], sel.y);
                        const uint32_t sh = (pos & 3u) * 8u;
                        uint32_t* dst = Ow + (pos >> 2);
                        atomicOr(dst, lo << sh);
                        atomicOr(dst + 1, __funnelshift_l(lo, hi, sh));
                        atomicOr(dst + 2, __funnelshift_l(hi, 0u, sh));
                    }
                    pos += __popc(m8);
                }
                // level-2 payload: the non-repeated bm1 bytes
                if (m2) or_bytes_at(Ow, nzT + (pre12 >> 16), __byte_perm(nb1, 0u, s_sel[m2]));
            }

            // levels 3 and 4 and the chunk trailer (warp 0, while the other
            // warps compact): bm2 and the payload end wpos are known since B3;
            // bytes at and after wpos go in by atomics too, since the last
            // level-2 payload word may be shared
            if (mode == 0 && warp == 0) {
                const uint2 mw = reinterpret_cast<const uint2*>(bm2)[lane];
                const uint64_t M3 = ((uint64_t)mw.y << 32) | mw.x;
                uint32_t p3 = __shfl_up_sync(full, mw.y, 1) >> 24;
                if (lane == 0) p3 = 0;
                const uint32_t m3 = nz_byte_mask64(M3 ^ ((M3 << 8) | p3));  // bm3 byte `lane`
                const uint32_t n3 = __popc(m3), inc = warp_incl_scan(n3);
                const uint32_t n3T = __shfl_sync(full, inc, 31);
                {
                    uint32_t p = wpos + inc - n3, m = m3;
                    while (m) {
                        const uint32_t b = __ffs(m) - 1;
                        m &= m - 1;
                        atomicOr(&Ow[p >> 2], (uint32_t)(uint8_t)(M3 >> (8 * b)) << (8 * (p & 3u)));
                        p++;
                    }
                }
                uint32_t pb = __shfl_up_sync(full, m3, 1);
                if (lane == 0) pb = 0;
                const bool nr4 = m3 != pb;
                const uint32_t bm4 = __ballot_sync(full, nr4);
                uint32_t wp = wpos + n3T;
                uint32_t sw = 0x80000000u | (uint32_t)kChunkBytes;
                if (!(wp >= (uint32_t)kRzeAvail || wp >= (uint32_t)(kRzeAvail - 4) ||
                      wp > (uint32_t)(kRzeAvail - 4 - 32))) {
                    if (nr4) {
                        const uint32_t q = wp + __popc(bm4 & ((1u << lane) - 1u));
                        atomicOr(&Ow[q >> 2], (m3 & 0xffu) << (8 * (q & 3u)));
                    }
                    wp += __popc(bm4);
                    if (wp < (uint32_t)(kRzeAvail - 4)) {
                        if (lane == 0) {  // bm4 word and the original size, 6 bytes from wp
                            const uint32_t sh = 8 * (wp & 3u);
                            const uint32_t lo = bm4, hi = (uint32_t)kChunkBytes;
                            atomicOr(&Ow[wp >> 2], lo << sh);
                            atomicOr(&Ow[(wp >> 2) + 1], __funnelshift_l(lo, hi, sh));
                            atomicOr(&Ow[(wp >> 2) + 2], __funnelshift_l(hi, 0u, sh));
                        }
                        sw = wp + 6;
                    }
                }
                if (lane == 0) s_misc[2] = sw;
            }
            if (t == 0) {
                if (mode == 1) {
                    O[0] = (uint8_t)(kChunkBytes & 0xff);
                    O[1] = (uint8_t)(kChunkBytes >> 8);
                    s_misc[2] = 2u;
                } else if (mode == 2) {
                    s_misc[2] = 0x80000000u | (uint32_t)kChunkBytes;
                }
            }
            __syncthreads();  // B4

            const uint32_t sw = s_misc[2];
            uint4* d4 = reinterpret_cast<uint4*>(a.slots + (size_t)c * kChunkBytes);
            uint4* o4 = reinterpret_cast<uint4*>(O);
            if (sw >> 31) {  // stored raw: the shuffled chunk itself
                const uint4* s4 = reinterpret_cast<const uint4*>(Sbuf);
                for (uint32_t i = t; i < (uint32_t)kChunkBytes / 16; i += kTT) d4[i] = s4[i];
                for (uint32_t i = t; i < (uint32_t)kOBytes / 16; i += kTT) o4[i] = make_uint4(0u, 0u, 0u, 0u);
            } else {
                for (uint32_t i = t; i < (sw + 15) / 16; i += kTT) {
                    d4[i] = o4[i];
                    o4[i] = make_uint4(0u, 0u, 0u, 0u);
                }
            }
            if (t == 0) a.sizes[c] = sw;
            fence_proxy_async();  // this plane's generic accesses before the buffer's next TMA fill
        }
    }
    asm volatile("griddepcontrol.launch_dependents;");  // the assembly scan may start launching
}

}  // namespace

// Host: a 2-D view of the field as rows of 32 floats, box = one slab plane.
namespace {
using EncodeTiled = PFN_cuTensorMapEncodeTiled_v12000;

EncodeTiled encode_tiled() {
    static EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiled) nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}
}  // namespace

bool lq3d_tma_supported(const FwdArgs& a) {
    return encode_tiled() != nullptr && (reinterpret_cast<uintptr_t>(a.in) & 15u) == 0 &&
           a.radius <= 2097152.0f && a.nfield % 8192u == 0;
}

int launch_lq3d_tma(const FwdArgs& a, unsigned grid, cudaStream_t s) {
    EncodeTiled enc = encode_tiled();
    if (!enc) return (int)cudaErrorNotSupported;
    CUtensorMap map;
    const cuuint64_t gdim[2] = {32, (cuuint64_t)(a.nfield / 32)};
    const cuuint64_t gstride[1] = {128};
    const cuuint32_t box[2] = {32, 256};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(a.in), gdim, gstride, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return (int)cudaErrorInvalidValue;
    const uint32_t slabs = a.ny / (kChunkCodes / a.nx), units = slabs * ((a.nz + 7) / 8);
    grid = grid < units ? grid : units;
    cudaError_t e;
    if (a.zigzag) {
        static SmemAttr attr;
        e = ensure_dyn_smem(attr, (const void*)lq3d_tma_kernel<true>, (int)kSlabSmem);
        if (e != cudaSuccess) return (int)e;
        e = launch_dependent(lq3d_tma_kernel<true>, grid, kTT, kSlabSmem, s, a, map, slabs, units);
    } else {
        static SmemAttr attr;
        e = ensure_dyn_smem(attr, (const void*)lq3d_tma_kernel<false>, (int)kSlabSmem);
        if (e != cudaSuccess) return (int)e;
        e = launch_dependent(lq3d_tma_kernel<false>, grid, kTT, kSlabSmem, s, a, map, slabs, units);
    }
    return (int)e;
}

}  // namespace fzb
