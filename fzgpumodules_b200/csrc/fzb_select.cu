// fzb_select.cu -- per-chunk lossless coding of quantization codes with a
// learned coder selector.
//
// The code array is cut into 64 KiB chunks (32768 u16 codes; the last may
// be shorter).  Each chunk is coded on its own by one of four coders, each
// producing exactly the bytes its reference stage would produce on that
// chunk alone:
//   0  Bitshuffle(16 KiB, ew 2) -> RZE(16 KiB, 4 levels)   (RZE stream)
//   1  RLE<uint16_t>                                        (RLE stream)
//   2  Bitpack<uint16_t>, nbits detected                    (packed bytes)
//   3  Huffman<uint16_t>, bklen 1024, coarse                (PHF blob)
// A coder whose output would exceed 64 KiB, or Huffman with a symbol >= 1024,
// is never chosen (Bitpack always fits).  Choice: exhaustive trial (smallest
// size, lowest coder index on ties) or a 16 -> 64 -> 64 -> 4 FP32 MLP on 16
// per-chunk statistics that predicts each coder's log2 size.
//
// Container: [u32 'FZSC'][u32 nchunks][u32 n_codes][u32 32768]
//            [u8 tag x nchunks, padded to 4][u8 param x nchunks, padded to 4]
//            [u32 size x nchunks][payload_i padded to 4 bytes] ...
// (param = Bitpack nbits, 0 otherwise).
#include "fzb_kernels.cuh"

namespace fzb {

namespace {

__device__ __forceinline__ void sel_raw_to_packed(const uint32_t (&rw)[16], uint32_t (&x)[16]) {
#pragma unroll
    for (int l = 0; l < 8; l++) {
        x[2 * l] = __byte_perm(rw[l], rw[l + 8], 0x5410);
        x[2 * l + 1] = __byte_perm(rw[l], rw[l + 8], 0x7632);
    }
}

__device__ __forceinline__ uint32_t chunk_count(uint64_t n, uint32_t c) {
    const uint64_t b = (uint64_t)c * kSelCodes;
    return (uint32_t)(n - b < (uint64_t)kSelCodes ? n - b : (uint64_t)kSelCodes);
}

// chunk id of this block, or -1 when coder k is not wanted for it
__device__ __forceinline__ int sel_chunk(const SelArgs& s, int k) {
    const uint32_t c = s.list ? s.list[blockIdx.x] : blockIdx.x;
    if (s.want && !((s.want[c] >> k) & 1u)) return -1;
    return (int)c;
}

__device__ __forceinline__ float bin_entropy(float p) {
    if (p <= 0.0f || p >= 1.0f) return 0.0f;
    return -(p * __log2f(p) + (1.0f - p) * __log2f(1.0f - p));
}

// Block-wide float sum (256 threads), fixed reduction order.

__device__ __forceinline__ uint32_t block_max_u32(uint32_t v, uint32_t* red) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, d));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t m = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) m = max(m, red[w]);
    __syncthreads();
    return m;
}

}  // namespace

// ---------------------------------------------------------------------------
// Features: 16 statistics per chunk (CTA per chunk).  Per code the kernel only
// histograms the code (1024 bins of min(code, 1023): lane-private bins for
// codes < 16, where nearly all codes fall, shared bins above), compares it
// with its predecessor and ORs it into its 8-code group; everything that is a
// function of the code alone (log moments, zero codes, zero bytes, bit-plane
// counts, the maximum, both byte histograms) is then summed over the bins,
// with the rare codes >= 1023 handled one by one.  Thread t takes the 8-code
// groups t, t+256, ... with 16-byte loads.
// ---------------------------------------------------------------------------
// Block-wide sums of K values per thread (256 threads, K <= 32), in place;
// two barriers for all K.
template <int K>
__device__ __forceinline__ void block_sum_n(float (&v)[K], float* red) {
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], d);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < K; k++) red[(threadIdx.x >> 5) * 32 + k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) {
        float s = 0.0f;
#pragma unroll
        for (int w = 0; w < 8; w++) s += red[w * 32 + k];
        v[k] = s;
    }
    __syncthreads();
}

struct FeatAcc {
    float sd = 0;                      // sum of log2(1 + |delta|)
    uint32_t same = 0, nzb = 0;        // equal neighbours, nonzero bit-plane bytes
    float s1 = 0, s2 = 0;              // codes >= 1023: log moments
    uint32_t vmax = 0, bits[16] = {};  // codes >= 1023: maximum, bit counts
};

__device__ __forceinline__ void feat_code(FeatAcc& f, uint32_t u, uint32_t pv, bool has_prev, uint32_t* h1024,
                                          uint32_t* priv, uint32_t* hlo_x, uint32_t* hhi_x) {
    atomicAdd(u < 16 ? priv + 32 * u : h1024 + min(u, 1023u), 1u);
    if (has_prev) {
        f.same += (u == pv);
        f.sd += __log2f(1.0f + (float)(u > pv ? u - pv : pv - u));
    }
    if (u >= 1023) {  // rare: the bin holds every code >= 1023
        const float lg = __log2f(1.0f + (float)u);
        f.s1 += lg;
        f.s2 += lg * lg;
        f.vmax = max(f.vmax, u);
#pragma unroll
        for (int b = 0; b < 16; b++) f.bits[b] += (u >> b) & 1u;
        atomicAdd(hlo_x + (u & 0xffu), 1u);
        if (u >= 1024) atomicAdd(hhi_x + (u >> 8), 1u);
    } else if (u >= 256) {
        atomicAdd(hlo_x + (u & 0xffu), 1u);
    }
}

__global__ void __launch_bounds__(256) sel_features_kernel(const uint16_t* __restrict__ codes, uint64_t n,
                                                           float* __restrict__ feats) {
    __shared__ uint32_t h1024[1024];
    __shared__ uint32_t hlo_x[256], hhi_x[256];  // low bytes of codes >= 256, high bytes of codes >= 1024
    __shared__ uint32_t priv[8 * 16 * 32];     // [warp][bin][lane]
    __shared__ float redn[8 * 32];
    __shared__ uint32_t ured[8];
    const uint32_t c = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t cnt = chunk_count(n, c);
    const uint16_t* src = codes + (uint64_t)c * kSelCodes;
    for (uint32_t i = t; i < 1024; i += 256) h1024[i] = 0;
    hlo_x[t] = 0;
    hhi_x[t] = 0;
    uint32_t* mypriv = priv + warp * 512 + lane;
#pragma unroll
    for (int b = 0; b < 16; b++) mypriv[32 * b] = 0;
    __syncthreads();
    FeatAcc f;
    const bool vec = (reinterpret_cast<uintptr_t>(src) & 15u) == 0;
    for (uint32_t g = t; 8 * g < cnt; g += 256) {
        const uint32_t i0 = 8 * g;
        uint32_t pv = i0 ? src[i0 - 1] : 0u;
        uint32_t o = 0;
        if (vec && i0 + 8 <= cnt) {
            const uint4 q = *reinterpret_cast<const uint4*>(src + i0);
            const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                o |= w[k];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint32_t u = h ? w[k] >> 16 : w[k] & 0xffffu;
                    feat_code(f, u, pv, i0 + 2 * k + h > 0, h1024, mypriv, hlo_x, hhi_x);
                    pv = u;
                }
            }
            o |= o >> 16;
        } else {  // partial group (or unaligned codes): code by code
            for (uint32_t k = 0; k < 8 && i0 + k < cnt; k++) {
                const uint32_t u = src[i0 + k];
                feat_code(f, u, pv, i0 + k > 0, h1024, mypriv, hlo_x, hhi_x);
                pv = u;
                o |= u;
            }
        }
        f.nzb += __popc(o & 0xffffu);  // nonzero bit-plane bytes of the 8 codes
    }
    // lane-private bins -> h1024[0..15]
#pragma unroll
    for (int b = 0; b < 16; b++) {
        const uint32_t v = __reduce_add_sync(0xffffffffu, mypriv[32 * b]);
        if (lane == 0 && v) atomicAdd(h1024 + b, v);
    }
    __syncthreads();  // the histogram is complete
    const float fn = (float)max(cnt, 1u);
    // per-code sums plus the bins of this thread (t, t+256, t+512, t+768; bin
    // 1023 holds every code >= 1023 and was summed code by code)
    float r1[29];
    r1[0] = f.s1;
    r1[1] = f.s2;
    r1[2] = (float)f.same;
    r1[3] = f.sd;
    r1[4] = (float)f.nzb;
#pragma unroll
    for (int b = 0; b < 16; b++) r1[5 + b] = (float)f.bits[b];
    uint32_t vmax = f.vmax;
    float e1024 = 0;
#pragma unroll
    for (int qq = 0; qq < 4; qq++) {
        const uint32_t bin = t + 256u * qq;
        const uint32_t h = h1024[bin];
        const float p = h / fn;
        if (p > 0) e1024 -= p * __log2f(p);
        r1[25 + qq] = (float)h;  // quarter sums of the histogram
        if (h && bin < 1023) {
            const float lg = __log2f(1.0f + (float)bin), fh = (float)h;
            r1[0] += fh * lg;
            r1[1] += fh * lg * lg;
            vmax = max(vmax, bin);
#pragma unroll
            for (int b = 0; b < 10; b++)
                if ((bin >> b) & 1u) r1[5 + b] += fh;
        }
    }
    const float pl = (h1024[t] + hlo_x[t]) / fn;  // low byte b: codes equal to b plus codes >= 256
    r1[21] = pl > 0 ? -pl * __log2f(pl) : 0.0f;
    r1[22] = e1024;
    r1[23] = (float)hhi_x[t];                     // codes >= 1024
    r1[24] = (float)hlo_x[0] * (t == 0);          // codes >= 256 with a zero low byte
    block_sum_n(r1, redn);
    vmax = block_max_u32(vmax, ured);
    const float m1 = r1[0] / fn, m2 = r1[1] / fn;
    float out[16];
    out[0] = m1 / 16.0f;
    out[1] = sqrtf(fmaxf(m2 - m1 * m1, 0.0f)) / 8.0f;
    out[2] = (float)h1024[0] / fn;
    out[3] = 1.0f - r1[2] / fn;  // runs per code
    // zero low bytes: codes 0 and codes >= 256 with a zero low byte; zero high bytes: codes < 256
    out[4] = ((float)h1024[0] + r1[24] + r1[25]) / (2.0f * fn);
    out[5] = r1[3] / fn / 16.0f;
    float hb[4] = {0, 0, 0, 0};
#pragma unroll
    for (int b = 0; b < 16; b++) hb[b >> 2] += bin_entropy(r1[5 + b] / fn) * 0.25f;
    out[6] = hb[0];
    out[7] = hb[1];
    out[8] = hb[2];
    out[9] = hb[3];
    out[10] = __log2f(1.0f + (float)vmax) / 16.0f;
    out[11] = r1[21] / 8.0f;
    out[13] = vmax >= 1024 ? 1.0f : 0.0f;  // Huffman (bklen 1024) not applicable
    out[14] = r1[4] / (2.0f * fn);
    out[15] = r1[22] / 10.0f;
    // high-byte entropy: bins 0..3 = quarters of h1024 less the codes >= 1024
    // folded into its last bin, bins >= 4 from the rare codes
    float r3[1];
    {
        const float qv = t == 0 ? r1[25] : t == 1 ? r1[26] : t == 2 ? r1[27] : r1[28] - r1[23];
        const float ph = (t < 4 ? qv : (float)hhi_x[t]) / fn;
        r3[0] = ph > 0 ? -ph * __log2f(ph) : 0.0f;
    }
    block_sum_n(r3, redn);
    out[12] = r3[0] / 8.0f;
    if (t < 16) {
        float v = 0;
#pragma unroll
        for (int k = 0; k < 16; k++)
            if (k == (int)t) v = out[k];
        feats[(uint64_t)c * kSelFeat + t] = v;
    }
}

// ---------------------------------------------------------------------------
// Coder 0: Bitshuffle + RZE.  Sub-chunk kernel (grid nlist x 4) encodes one
// 16 KiB block into scratch; the assembly kernel writes the chunk's RZE
// stream ([u32 orig][u32 nsub][u32 size x nsub][payloads], padded to 4).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) sel_rze_sub_kernel(SelArgs s) {
    extern __shared__ uint4 sm4[];
    __shared__ uint32_t s_ws[16];
    const int ci = sel_chunk(s, 0);
    if (ci < 0) return;
    const uint32_t c = (uint32_t)ci;
    const uint32_t j = blockIdx.y, t = threadIdx.x;
    const uint32_t cnt = chunk_count(s.n, c);
    const uint32_t sb = j * (uint32_t)kChunkCodes;  // first code of the block within the chunk
    if (sb >= cnt) return;
    const uint32_t bc = min((uint32_t)kChunkCodes, cnt - sb);
    uint8_t* base = reinterpret_cast<uint8_t*>(sm4);
    RzeSmem sm;
    sm.S = reinterpret_cast<uint32_t*>(base);
    sm.O = base + kChunkBytes;
    sm.bm1 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16);
    sm.bm2 = base + 2 * kChunkBytes + 16 + 2048;
    sm.bm3 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16 + 2048 + 256);
    sm.ws = s_ws;
    const uint16_t* src = s.codes + (uint64_t)c * kSelCodes + sb;
    uint32_t rw[16];
    if (bc == (uint32_t)kChunkCodes && (reinterpret_cast<uintptr_t>(s.codes) & 15) == 0) {
        const uint4* s4 = reinterpret_cast<const uint4*>(src) + 4 * t;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const uint4 q = __ldg(s4 + v);
            rw[4 * v] = q.x;
            rw[4 * v + 1] = q.y;
            rw[4 * v + 2] = q.z;
            rw[4 * v + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int l = 0; l < 16; l++) {
            const uint32_t e = 32 * t + 2 * l;
            const uint32_t lo = e < bc ? src[e] : 0u, hi = e + 1 < bc ? src[e + 1] : 0u;
            rw[l] = lo | (hi << 16);
        }
    }
    if (bc == (uint32_t)kChunkCodes) {
        uint32_t x[16];
        sel_raw_to_packed(rw, x);
        transpose16x2(x);
#pragma unroll
        for (int b = 0; b < 16; b++) sm.S[(15 - b) * 256 + t] = x[b];
    } else {  // the block shorter than 16 KiB is copied unchanged
#pragma unroll
        for (int l = 0; l < 16; l++) sm.S[16 * t + l] = rw[l];
    }
    __syncthreads();
    const uint32_t sw = rze_encode_chunk(sm, (int)(2 * bc));
    const uint32_t clean = sw & 0x7fffffffu;
    const uint8_t* payload = (sw >> 31) ? reinterpret_cast<const uint8_t*>(sm.S) : sm.O;
    uint4* d4 = reinterpret_cast<uint4*>(s.scratch + ((size_t)c * 4 + j) * kChunkBytes);
    const uint4* p4 = reinterpret_cast<const uint4*>(payload);
    for (uint32_t i = t; i < (clean + 15) / 16; i += kThreads) d4[i] = p4[i];
    if (t == 0) s.subsizes[(size_t)c * 4 + j] = sw;
}

__global__ void __launch_bounds__(256) sel_rze_assemble_kernel(SelArgs s) {
    const int ci = sel_chunk(s, 0);
    if (ci < 0) return;
    const uint32_t c = (uint32_t)ci;
    const uint32_t cnt = chunk_count(s.n, c);
    const uint32_t nsub = (2 * cnt + kChunkBytes - 1) / kChunkBytes;
    uint32_t sw[4], off[4], tot = 8 + 4 * nsub;
    for (uint32_t j = 0; j < 4; j++) {
        sw[j] = j < nsub ? s.subsizes[(size_t)c * 4 + j] : 0u;
        off[j] = tot;
        tot += sw[j] & 0x7fffffffu;
    }
    const uint32_t padded = (tot + 3) & ~3u;
    if (padded > (uint32_t)kSelBytes) {
        if (threadIdx.x == 0) s.sizes[(size_t)c * kSelCoders + 0] = kSelNoFit;
        return;
    }
    uint8_t* dst = s.slots + ((size_t)c * kSelCoders + 0) * kSelSlot;
    if (threadIdx.x == 0) {
        uint32_t* h = reinterpret_cast<uint32_t*>(dst);
        h[0] = 2 * cnt;
        h[1] = nsub;
        for (uint32_t j = 0; j < nsub; j++) h[2 + j] = sw[j];
        for (uint32_t i = tot; i < padded; i++) dst[i] = 0;
        s.sizes[(size_t)c * kSelCoders + 0] = padded;
    }
    for (uint32_t j = 0; j < nsub; j++) {
        const uint8_t* src = s.scratch + ((size_t)c * 4 + j) * kChunkBytes;
        const uint32_t len = sw[j] & 0x7fffffffu;
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) dst[off[j] + i] = src[i];
    }
}

// ---------------------------------------------------------------------------
// Coder 1: RLE  [u32 runs][u16 values, padded to 4][u32 lengths]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) sel_rle_kernel(SelArgs s) {
    __shared__ uint32_t ws[16];
    __shared__ uint32_t first_start[256];
    const int ci = sel_chunk(s, 1);
    if (ci < 0) return;
    const uint32_t c = (uint32_t)ci;
    const uint32_t cnt = chunk_count(s.n, c), t = threadIdx.x;
    const uint16_t* src = s.codes + (uint64_t)c * kSelCodes;
    const uint32_t b0 = 128 * t;
    uint32_t nstart = 0, fs = 0xffffffffu;
    for (uint32_t k = 0; k < 128; k++) {
        const uint32_t i = b0 + k;
        if (i >= cnt) break;
        if (i == 0 || src[i] != src[i - 1]) {
            nstart++;
            if (fs == 0xffffffffu) fs = i;
        }
    }
    uint32_t runs;
    const uint32_t r0 = block_excl_scan(nstart, ws, &runs);
    first_start[t] = fs;
    __syncthreads();
    const uint32_t vbytes = (2 * runs + 3) & ~3u;
    const uint32_t total = 4 + vbytes + 4 * runs;
    if (total > (uint32_t)kSelBytes) {
        if (t == 0) s.sizes[(size_t)c * kSelCoders + 1] = kSelNoFit;
        return;
    }
    // next run start after this thread's range
    uint32_t next = cnt;
    for (uint32_t u = t + 1; u < 256; u++)
        if (first_start[u] != 0xffffffffu) {
            next = first_start[u];
            break;
        }
    uint8_t* dst = s.slots + ((size_t)c * kSelCoders + 1) * kSelSlot;
    uint16_t* vals = reinterpret_cast<uint16_t*>(dst + 4);
    uint32_t* lens = reinterpret_cast<uint32_t*>(dst + 4 + vbytes);
    uint32_t r = r0, last = 0xffffffffu;
    for (uint32_t k = 0; k < 128; k++) {
        const uint32_t i = b0 + k;
        if (i >= cnt) break;
        if (i == 0 || src[i] != src[i - 1]) {
            if (last != 0xffffffffu) lens[r - 1] = i - last;
            vals[r] = src[i];
            last = i;
            r++;
        }
    }
    if (last != 0xffffffffu) lens[r - 1] = next - last;
    if (t == 0) {
        *reinterpret_cast<uint32_t*>(dst) = runs;
        if (runs & 1) vals[runs] = 0;  // pad the values to 4 bytes
        s.sizes[(size_t)c * kSelCoders + 1] = total;
    }
}

// ---------------------------------------------------------------------------
// Coder 2: Bitpack with detected nbits (smallest power of two whose range
// holds the maximum), LSB-first below 8 bits.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) sel_bitpack_kernel(SelArgs s) {
    __shared__ uint32_t red[8];
    const int ci = sel_chunk(s, 2);
    if (ci < 0) return;
    const uint32_t c = (uint32_t)ci;
    const uint32_t cnt = chunk_count(s.n, c), t = threadIdx.x;
    const uint16_t* src = s.codes + (uint64_t)c * kSelCodes;
    uint32_t m = 0;
    for (uint32_t i = t; i < cnt; i += 256) m = max(m, (uint32_t)src[i]);
    m = block_max_u32(m, red);
    uint32_t nb = 16;
    for (uint32_t b = 1; b < 16; b *= 2)
        if (m < (1u << b)) {
            nb = b;
            break;
        }
    const uint32_t out_bytes = (cnt * nb + 7) / 8;
    uint8_t* dst = s.slots + ((size_t)c * kSelCoders + 2) * kSelSlot;
    if (nb >= 8) {
        const uint32_t per = nb / 8;
        for (uint32_t i = t; i < cnt; i += 256) {
            const uint32_t v = src[i];
            for (uint32_t b = 0; b < per; b++) dst[i * per + b] = (uint8_t)(v >> (8 * b));
        }
    } else {
        const uint32_t per = 8 / nb, mask = (1u << nb) - 1u;
        for (uint32_t o = t; o < out_bytes; o += 256) {
            uint32_t packed = 0;
            for (uint32_t k = 0; k < per; k++) {
                const uint32_t e = o * per + k;
                if (e < cnt) packed |= ((uint32_t)src[e] & mask) << (k * nb);
            }
            dst[o] = (uint8_t)packed;
        }
    }
    if (t == 0) {
        s.sizes[(size_t)c * kSelCoders + 2] = out_bytes;
        s.params[c * kSelCoders + 2] = (uint8_t)nb;
    }
}

// ---------------------------------------------------------------------------
// Coder 3: Huffman (bklen 1024).  Histogram (CTA per chunk), canonical
// codebook (one warp per chunk; lane 0 replays the reference's heap
// construction, the warp gathers leaves and canonizes), coarse encode into
// the PHF blob.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) sel_hf_hist_kernel(SelArgs s) {
    __shared__ uint32_t h[kSelBk];
    __shared__ uint32_t bad;
    const int ci = sel_chunk(s, 3);
    if (ci < 0) return;
    const uint32_t c = (uint32_t)ci;
    const uint32_t cnt = chunk_count(s.n, c), t = threadIdx.x;
    const uint16_t* src = s.codes + (uint64_t)c * kSelCodes;
    for (uint32_t i = t; i < kSelBk; i += 256) h[i] = 0;
    if (t == 0) bad = 0;
    __syncthreads();
    for (uint32_t i = t; i < cnt; i += 256) {
        const uint32_t u = src[i];
        if (u < (uint32_t)kSelBk) atomicAdd(&h[u], 1u);
        else bad = 1;
    }
    __syncthreads();
    uint32_t* f = s.hf_freq + (size_t)c * kSelBk;
    for (uint32_t i = t; i < kSelBk; i += 256) f[i] = h[i];
    if (t == 0 && bad) s.sizes[(size_t)c * kSelCoders + 3] = kSelNoFit;
    else if (t == 0) s.sizes[(size_t)c * kSelCoders + 3] = 0;
}

// Book for one chunk (one warp).  Lane 0 replays the reference's heap
// construction exactly (same keys, same sift rules, the first popped node
// becomes the right child); each merge records the parent of the two merged
// nodes, and one pass from the root down turns the parents into depths (the
// code lengths of the reference's tree walk).  The leaf gather and the
// canonical codebook are warp-parallel.  Dynamic shared memory (8 KB, so
// about 25 chunks run per SM): the heap (later the per-symbol lengths), then
// the parent/depth array.
__global__ void __launch_bounds__(32) sel_hf_book_kernel(SelArgs s) {
    extern __shared__ uint32_t smb[];
    __shared__ int numl[32], entry[32], first[32], nxt[32];
    __shared__ uint32_t nzmask[32], leafbase[32];
    __shared__ int s_ok, s_nsym;
    const int ci = sel_chunk(s, 3);
    if (ci < 0) return;
    const uint32_t c = (uint32_t)ci;
    if (s.sizes[(size_t)c * kSelCoders + 3] == kSelNoFit) return;
    uint32_t* hk = smb;                                                      // kSelBk + 2 keys, 1-indexed
    uint16_t* par = reinterpret_cast<uint16_t*>(smb + kSelBk + 2);           // 2 * kSelBk: parent, then depth
    uint8_t* len = reinterpret_cast<uint8_t*>(smb);                          // kSelBk, over the dead heap
    const uint32_t* freq = s.hf_freq + (size_t)c * kSelBk;
    const uint32_t lane = threadIdx.x, full = 0xffffffffu, lt = (1u << lane) - 1u;

    // leaves in symbol order: leaf id = rank of the symbol among the present
    // ones; par[leaf] holds its frequency until the heap is built
    uint32_t fq[kSelBk / 32];
#pragma unroll
    for (int g = 0; g < kSelBk / 32; g++) fq[g] = freq[g * 32 + lane];
    uint32_t mine = 0;  // lane g: present-symbol mask of group g
#pragma unroll
    for (int g = 0; g < kSelBk / 32; g++) {
        const uint32_t b = __ballot_sync(full, fq[g] != 0);
        if (lane == (uint32_t)g) mine = b;
    }
    const uint32_t pc = __popc(mine);
    uint32_t inc = pc;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(full, inc, d);
        if (lane >= (uint32_t)d) inc += v;
    }
    nzmask[lane] = mine;
    leafbase[lane] = inc - pc;
    numl[lane] = 0;
    const int leaves = (int)__shfl_sync(full, inc, 31);
    __syncwarp();
#pragma unroll
    for (int g = 0; g < kSelBk / 32; g++)
        if (fq[g]) par[leafbase[g] + __popc(nzmask[g] & lt)] = (uint16_t)fq[g];
    __syncwarp();

    if (lane == 0) {
        // binary min-heap, 1-indexed, of keys freq << 11 | node id (freq <=
        // 32768, ids < 2048; comparisons look at the frequency only):
        // insertion stops at a parent whose frequency is <= the new node's;
        // removal sinks the moved node, taking the right child only when
        // strictly smaller and swapping only when strictly larger
        int hs = 0;
        auto push = [&](uint32_t key) {
            const uint32_t kf = key >> 11;
            int i = ++hs;
            while (i > 1) {
                const int p = i >> 1;
                const uint32_t kp = hk[p];
                if ((kp >> 11) <= kf) break;
                hk[i] = kp;
                i = p;
            }
            hk[i] = key;
        };
        auto pop = [&]() -> uint32_t {
            const uint32_t top = hk[1];
            const uint32_t moved = hk[hs];
            hs--;
            const uint32_t mf = moved >> 11;
            int i = 1;
            while (2 * i <= hs) {
                const uint2 kk = *reinterpret_cast<const uint2*>(hk + 2 * i);  // both children
                int ch = 2 * i;
                uint32_t kc = kk.x;
                if (ch + 1 <= hs && (kk.y >> 11) < (kc >> 11)) {
                    ch++;
                    kc = kk.y;
                }
                if (mf > (kc >> 11)) {
                    hk[i] = kc;
                    i = ch;
                } else {
                    break;
                }
            }
            hk[i] = moved;
            return top;
        };
        for (int i = 0; i < leaves; i++) push(((uint32_t)par[i] << 11) | (uint32_t)i);
        int nn = leaves;
        while (hs > 1) {  // the first popped node becomes the right child
            const uint32_t kr = pop();
            const uint32_t kl = pop();
            par[kr & 0x7ffu] = (uint16_t)nn;
            par[kl & 0x7ffu] = (uint16_t)nn;
            push((((kr >> 11) + (kl >> 11)) << 11) | (uint32_t)nn);
            nn++;
        }
        // depths: every parent id is above its children's, so one pass from
        // the root down, in place; the walk's 58-level stack limit fails the
        // book when any node lies deeper
        int maxd = 0;
        if (nn > 0) {
            par[nn - 1] = 0;
            for (int id = nn - 2; id >= 0; id--) {
                const int d = par[par[id]] + 1;
                par[id] = (uint16_t)d;
                maxd = max(maxd, d);
            }
        }
        s_ok = maxd <= 58;
        s_nsym = leaves;
    }
    __syncwarp();
    if (!s_ok) {
        if (lane == 0) s.sizes[(size_t)c * kSelCoders + 3] = kSelNoFit;
        return;
    }
    // lengths (above 27: the cutoff length 28) and their counts
    for (int g = 0; g < kSelBk / 32; g++) {
        uint32_t l = 0xffu;
        const uint32_t m = nzmask[g];
        if ((m >> lane) & 1u) {
            const uint32_t d = par[leafbase[g] + __popc(m & lt)];
            l = d > 27 ? 28u : d;
        }
        len[g * 32 + lane] = (uint8_t)l;
        const uint32_t same = __match_any_sync(full, l);
        if (l != 0xffu && (same >> lane) == 1u) numl[l] += __popc(same);  // highest lane of the group
        __syncwarp();
    }
    // canonical form: entry = exclusive scan of the counts; first[l] from the
    // longest length down
    {
        const int cnt_l = numl[lane];
        int e = cnt_l;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(full, e, d);
            if (lane >= (uint32_t)d) e += v;
        }
        entry[lane] = e - cnt_l;
        const uint32_t used = __ballot_sync(full, cnt_l != 0);
        const int max_l = used ? 31 - __clz(used) : 0;
        if (lane == 0) {
            for (int i = 0; i < 32; i++) first[i] = 0;
            for (int l = max_l - 1; l >= 1; l--) first[l] = (first[l + 1] + numl[l + 1] + 1) >> 1;
            first[0] = 0xff;
        }
    }
    __syncwarp();
    // slots in symbol order within each length: book words and keys
    uint32_t* bk4 = s.hf_book + (size_t)c * kSelBk;
    uint8_t* blob = s.slots + ((size_t)c * kSelCoders + 3) * kSelSlot;
    int* rb_first = reinterpret_cast<int*>(blob + 128);
    uint16_t* keys = reinterpret_cast<uint16_t*>(blob + 128 + 256);
    nxt[lane] = entry[lane];
    __syncwarp();
    for (int g = 0; g < kSelBk / 32; g++) {
        const uint32_t sym = g * 32 + lane;
        const uint32_t l = len[sym];
        const uint32_t same = __match_any_sync(full, l);
        uint32_t w = 0xffffffffu;
        if (l != 0xffu) {
            const int slot = nxt[l] + __popc(same & lt);
            w = ((uint32_t)(first[l] + slot - entry[l]) & 0x7ffffffu) | (l << 27);
            keys[slot] = (uint16_t)sym;
        }
        bk4[sym] = w;
        __syncwarp();
        if (l != 0xffu && (same >> lane) == 1u) nxt[l] += __popc(same);
        __syncwarp();
    }
    for (int i = s_nsym + (int)lane; i < kSelBk; i += 32) keys[i] = 0;
    rb_first[lane] = first[lane];
    rb_first[32 + lane] = entry[lane];
}

__global__ void __launch_bounds__(256) sel_hf_encode_kernel(SelArgs s) {
    __shared__ uint32_t book[kSelBk];
    __shared__ uint32_t cells[kHfSublen];
    __shared__ uint32_t pnbit[kSelParts], pent[kSelParts + 1];
    __shared__ uint32_t ws[16];
    const int ci = sel_chunk(s, 3);
    if (ci < 0) return;
    const uint32_t c = (uint32_t)ci;
    if (s.sizes[(size_t)c * kSelCoders + 3] == kSelNoFit) return;
    const uint32_t cnt = chunk_count(s.n, c), t = threadIdx.x;
    const uint16_t* src = s.codes + (uint64_t)c * kSelCodes;
    const uint32_t* bk4 = s.hf_book + (size_t)c * kSelBk;
    for (uint32_t i = t; i < (uint32_t)kSelBk; i += 256) book[i] = bk4[i];
    __syncthreads();
    const uint32_t pardeg = (cnt + kHfSublen - 1) / kHfSublen;
    // pass 1: bits per partition
    for (uint32_t p = 0; p < pardeg; p++) {
        uint32_t bits = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint32_t i = p * kHfSublen + 3 * t + k;
            if (i < cnt) bits += book[src[i]] >> 27;
        }
        uint32_t tot;
        block_excl_scan(bits, ws, &tot);
        if (t == 0) pnbit[p] = tot;
        __syncthreads();
    }
    if (t == 0) {
        uint32_t e = 0;
        for (uint32_t p = 0; p < pardeg; p++) {
            pent[p] = e;
            e += (pnbit[p] + 31) / 32;
        }
        pent[pardeg] = e;
    }
    __syncthreads();
    const uint32_t ncell = pent[pardeg];
    const uint32_t rb = 256 + 2 * kSelBk;
    const uint32_t e1 = 128, e2 = e1 + rb, e3 = e2 + 4 * pardeg, e4 = e3 + 4 * pardeg, e5 = e4 + 4 * ncell;
    if (e5 > (uint32_t)kSelBytes) {
        if (t == 0) s.sizes[(size_t)c * kSelCoders + 3] = kSelNoFit;
        return;
    }
    uint8_t* blob = s.slots + ((size_t)c * kSelCoders + 3) * kSelSlot;
    uint32_t* bitstream = reinterpret_cast<uint32_t*>(blob + e4);
    // pass 2: partitions into their cells
    for (uint32_t p = 0; p < pardeg; p++) {
        for (uint32_t i = t; i < (uint32_t)kHfSublen; i += 256) cells[i] = 0;
        __syncthreads();
        uint32_t w[3], bits = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint32_t i = p * kHfSublen + 3 * t + k;
            w[k] = i < cnt ? book[src[i]] : 0u;
            bits += w[k] >> 27;
        }
        uint32_t tot;
        uint32_t off = block_excl_scan(bits, ws, &tot);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint32_t ln = w[k] >> 27, cd = w[k] & 0x7ffffffu;
            if (ln) {
                const uint32_t cell = off >> 5, pos = off & 31;
                if (pos + ln <= 32) {
                    atomicOr(&cells[cell], cd << (32 - pos - ln));
                } else {
                    const uint32_t spill = pos + ln - 32;
                    atomicOr(&cells[cell], cd >> spill);
                    atomicOr(&cells[cell + 1], cd << (32 - spill));
                }
            }
            off += ln;
        }
        __syncthreads();
        const uint32_t nc = (tot + 31) / 32;
        for (uint32_t i = t; i < nc; i += 256) bitstream[pent[p] + i] = cells[i];
        __syncthreads();
    }
    uint32_t* h32 = reinterpret_cast<uint32_t*>(blob);
    if (t < 32) h32[t] = 0;
    __syncthreads();
    for (uint32_t p = t; p < pardeg; p += 256) {  // per-partition tables
        reinterpret_cast<uint32_t*>(blob + e2)[p] = pnbit[p];
        reinterpret_cast<uint32_t*>(blob + e3)[p] = pent[p];
    }
    if (t == 0) {
        uint64_t nbit = 0;
        for (uint32_t p = 0; p < pardeg; p++) nbit += pnbit[p];
        h32[0] = kSelBk;
        h32[1] = kHfSublen;
        h32[2] = pardeg;
        h32[4] = cnt;
        h32[5] = 0;
        h32[6] = (uint32_t)nbit;
        h32[7] = (uint32_t)(nbit >> 32);
        h32[8] = ncell;
        h32[9] = 0;
        h32[10] = 0;
        h32[11] = e1;
        h32[12] = e2;
        h32[13] = e3;
        h32[14] = e4;
        h32[15] = e5;
        s.sizes[(size_t)c * kSelCoders + 3] = e5;
    }
}

// ---------------------------------------------------------------------------
// Choice and container.
// ---------------------------------------------------------------------------
// mode 0: smallest size; mode 1: smallest predicted log-size (pred[c][4]);
// mode 2 + k: coder k when it fits, else the smallest.
__global__ void sel_choose_kernel(SelArgs s, uint32_t nchunks, int mode, const float* __restrict__ pred) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const uint32_t* sz = s.sizes + (size_t)c * kSelCoders;
    int best = -1;
    if (mode == 1) {
        float bp = INFINITY;
        for (int k = 0; k < kSelCoders; k++) {
            const float v = pred[(size_t)c * kSelCoders + k];
            if (v < bp) {
                bp = v;
                best = k;
            }
        }
    } else if (mode >= 2) {
        best = mode - 2;
    }
    if (best < 0 || sz[best] == kSelNoFit) {  // exhaustive, or the predicted coder does not fit
        uint32_t bs = kSelNoFit;
        for (int k = 0; k < kSelCoders; k++)
            if (sz[k] < bs) {
                bs = sz[k];
                best = k;
            }
    }
    s.tags[c] = (uint8_t)best;
}

// want[c] = the chosen coder only.
__global__ void sel_tag_mask_kernel(SelArgs s, uint32_t nchunks, uint8_t* __restrict__ want) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nchunks) want[c] = (uint8_t)(1u << s.tags[c]);
}

// Learned choices whose coder did not fit get the other coders tried.
__global__ void sel_fallback_kernel(SelArgs s, uint32_t nchunks, uint8_t* __restrict__ want) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const uint32_t k = s.tags[c];
    want[c] = s.sizes[(size_t)c * kSelCoders + k] == kSelNoFit ? (uint8_t)(0xFu & ~(1u << k)) : (uint8_t)0;
}

__global__ void __launch_bounds__(1024) sel_header_kernel(SelArgs s, uint32_t nchunks, uint8_t* __restrict__ out,
                                                          unsigned long long* __restrict__ out_size,
                                                          unsigned long long* __restrict__ offs) {
    // offs: exclusive scan of the padded chosen sizes.  Tiles of 4096 chunks:
    // coalesced loads (and header writes), a warp-shuffle block scan, carry.
    constexpr uint32_t kTile = 4096, kPer = kTile / 1024;
    __shared__ uint32_t sz[kTile];
    __shared__ uint32_t wsum[32], s_tile;
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t hdr = 16 + 2 * ((nchunks + 3) & ~3u) + 4 * nchunks;
    uint32_t* h32 = reinterpret_cast<uint32_t*>(out);
    uint8_t* tags = out + 16;
    uint8_t* params = tags + ((nchunks + 3) & ~3u);
    uint32_t* sizes = reinterpret_cast<uint32_t*>(params + ((nchunks + 3) & ~3u));
    unsigned long long carry = hdr;
    for (uint32_t t0 = 0; t0 < nchunks; t0 += kTile) {
        const uint32_t cnt = min(kTile, nchunks - t0);
        for (uint32_t i = t; i < kTile; i += 1024) {
            uint32_t v = 0;
            if (i < cnt) {
                const uint32_t c = t0 + i, k = s.tags[c];
                const uint32_t len = s.sizes[(size_t)c * kSelCoders + k];
                v = (len + 3u) & ~3u;
                tags[c] = (uint8_t)k;
                params[c] = s.params[c * kSelCoders + k];
                sizes[c] = len;
            }
            sz[i] = v;
        }
        __syncthreads();
        uint32_t l = 0;
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++) l += sz[kPer * t + j];
        uint32_t inc = l;  // a tile's padded sizes fit 32 bits (4096 x 64 KiB)
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= (uint32_t)d) inc += v;
        }
        if (lane == 31) wsum[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint32_t v = wsum[lane];
            uint32_t x = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t u = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= (uint32_t)d) x += u;
            }
            wsum[lane] = x - v;
        }
        __syncthreads();
        uint32_t r = wsum[warp] + inc - l;
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++) {
            const uint32_t v = sz[kPer * t + j];
            sz[kPer * t + j] = r;
            r += v;
        }
        if (t == 1023) s_tile = r;
        __syncthreads();
        for (uint32_t i = t; i < cnt; i += 1024) offs[t0 + i] = carry + sz[i];
        carry += s_tile;
        __syncthreads();
    }
    for (uint32_t c = nchunks + t; c < ((nchunks + 3) & ~3u); c += 1024) {
        tags[c] = 0;
        params[c] = 0;
    }
    if (t == 0) {
        h32[0] = 0x43535A46u;  // "FZSC"
        h32[1] = nchunks;
        h32[2] = (uint32_t)s.n;
        h32[3] = kSelCodes;
        *out_size = carry;
    }
}

__global__ void __launch_bounds__(256) sel_copy_kernel(SelArgs s, uint8_t* __restrict__ out,
                                                       const unsigned long long* __restrict__ offs) {
    // payload words: offsets are multiples of 4 and slots 16-byte aligned; the
    // bytes past len in the last word are zero padding
    const uint32_t c = blockIdx.x;
    const uint32_t k = s.tags[c];
    const uint32_t len = s.sizes[(size_t)c * kSelCoders + k], nw = (len + 3u) >> 2;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(s.slots + ((size_t)c * kSelCoders + k) * kSelSlot);
    uint32_t* dst = reinterpret_cast<uint32_t*>(out + offs[c]);
    for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x) {
        uint32_t v = src[i];
        if (4 * i + 4 > len) v &= 0xffffffffu >> (8 * (4 * i + 4 - len));
        dst[i] = v;
    }
}

// ---------------------------------------------------------------------------
// MLP 16 -> 64 -> 64 -> 4, FP32, ReLU.  Parameters packed as
// W1[16][64] b1[64] W2[64][64] b2[64] W3[64][4] b3[4] (row = input).
// One thread per sample; the parameters sit in shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                                          float* __restrict__ Y, uint32_t batch) {
    __shared__ float w[kMlpParams];
    for (uint32_t i = threadIdx.x; i < (uint32_t)kMlpParams; i += blockDim.x) w[i] = P[i];
    __syncthreads();
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const float* W1 = w;
    const float* B1 = W1 + 16 * 64;
    const float* W2 = B1 + 64;
    const float* B2 = W2 + 64 * 64;
    const float* W3 = B2 + 64;
    const float* B3 = W3 + 64 * 4;
    float x[16], h1[64], h2[64];
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = X[(size_t)b * 16 + i];
    for (int j = 0; j < 64; j++) {
        float a = B1[j];
#pragma unroll
        for (int i = 0; i < 16; i++) a = __fadd_rn(a, __fmul_rn(x[i], W1[i * 64 + j]));
        h1[j] = fmaxf(a, 0.0f);
    }
    for (int j = 0; j < 64; j++) {
        float a = B2[j];
        for (int i = 0; i < 64; i++) a = __fadd_rn(a, __fmul_rn(h1[i], W2[i * 64 + j]));
        h2[j] = fmaxf(a, 0.0f);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float a = B3[j];
        for (int i = 0; i < 64; i++) a = __fadd_rn(a, __fmul_rn(h2[i], W3[i * 4 + j]));
        Y[(size_t)b * 4 + j] = a;
    }
}

// Gradients of the mean squared error 1/(4B) sum (Y - T)^2 over the batch,
// accumulated into G (same packing as P, zeroed by the caller); *loss +=
// the batch's loss.  Per-sample gradients are summed in shared memory, then
// added to G once per block.
__global__ void __launch_bounds__(128) mlp_backward_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                                           const float* __restrict__ T, uint32_t batch,
                                                           float* __restrict__ G, float* __restrict__ loss,
                                                           const int kind) {
    __shared__ float w[kMlpParams];
    __shared__ float g[kMlpParams];
    __shared__ float sl[4];
    for (uint32_t i = threadIdx.x; i < (uint32_t)kMlpParams; i += blockDim.x) {
        w[i] = P[i];
        g[i] = 0.0f;
    }
    __syncthreads();
    const float* W1 = w;
    const float* B1 = W1 + 16 * 64;
    const float* W2 = B1 + 64;
    const float* B2 = W2 + 64 * 64;
    const float* W3 = B2 + 64;
    const float* B3 = W3 + 64 * 4;
    float* gW1 = g;
    float* gB1 = gW1 + 16 * 64;
    float* gW2 = gB1 + 64;
    float* gB2 = gW2 + 64 * 64;
    float* gW3 = gB2 + 64;
    float* gB3 = gW3 + 64 * 4;
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (b < batch) {
        float x[16], h1[64], h2[64], dy[4];
#pragma unroll
        for (int i = 0; i < 16; i++) x[i] = X[(size_t)b * 16 + i];
        for (int j = 0; j < 64; j++) {
            float a = B1[j];
#pragma unroll
            for (int i = 0; i < 16; i++) a = __fadd_rn(a, __fmul_rn(x[i], W1[i * 64 + j]));
            h1[j] = fmaxf(a, 0.0f);
        }
        for (int j = 0; j < 64; j++) {
            float a = B2[j];
            for (int i = 0; i < 64; i++) a = __fadd_rn(a, __fmul_rn(h1[i], W2[i * 64 + j]));
            h2[j] = fmaxf(a, 0.0f);
        }
        float y[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float a = B3[j];
            for (int i = 0; i < 64; i++) a = __fadd_rn(a, __fmul_rn(h2[i], W3[i * 4 + j]));
            y[j] = a;
        }
        if (kind == 0) {  // mean squared error against T
            const float scale = 2.0f / (4.0f * (float)batch);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float d = y[j] - T[(size_t)b * 4 + j];
                l += d * d / 4.0f;
                dy[j] = scale * d;
            }
        } else {  // cross-entropy of p = softmax(-y) against q = softmax(-T / tau), T = regrets
            const float m = fminf(fminf(y[0], y[1]), fminf(y[2], y[3]));
            float tr[4], e[4], qv[4], z = 0.0f, zq = 0.0f, tmin = INFINITY;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                tr[j] = T[(size_t)b * 4 + j];
                tmin = fminf(tmin, tr[j]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                e[j] = __expf(m - y[j]);
                z += e[j];
                qv[j] = __expf((tmin - tr[j]) * (1.0f / kMlpTau));
                zq += qv[j];
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float p = e[j] / z, q = qv[j] / zq;
                l -= q * (__logf(e[j]) - __logf(z));
                dy[j] = (q - p) / (float)batch;
            }
        }
        // layer 3
        float dh2[64];
        for (int i = 0; i < 64; i++) {
            float a = 0.0f;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                atomicAdd(&gW3[i * 4 + j], h2[i] * dy[j]);
                a += W3[i * 4 + j] * dy[j];
            }
            dh2[i] = h2[i] > 0.0f ? a : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 4; j++) atomicAdd(&gB3[j], dy[j]);
        // layer 2 (dh1 reuses h1's storage after its use)
        float dh1[64];
        for (int i = 0; i < 64; i++) dh1[i] = 0.0f;
        for (int j = 0; j < 64; j++) {
            const float d = dh2[j];
            if (d == 0.0f) continue;
            atomicAdd(&gB2[j], d);
            for (int i = 0; i < 64; i++) {
                atomicAdd(&gW2[i * 64 + j], h1[i] * d);
                dh1[i] += W2[i * 64 + j] * d;
            }
        }
        for (int j = 0; j < 64; j++) {
            const float d = h1[j] > 0.0f ? dh1[j] : 0.0f;
            if (d == 0.0f) continue;
            atomicAdd(&gB1[j], d);
#pragma unroll
            for (int i = 0; i < 16; i++) atomicAdd(&gW1[i * 64 + j], x[i] * d);
        }
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) l += __shfl_xor_sync(0xffffffffu, l, d);
    if ((threadIdx.x & 31) == 0) sl[threadIdx.x >> 5] = l;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < (uint32_t)kMlpParams; i += blockDim.x)
        if (g[i] != 0.0f) atomicAdd(&G[i], g[i]);
    if (threadIdx.x == 0) atomicAdd(loss, (sl[0] + sl[1] + sl[2] + sl[3]) / (float)batch);
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8); step counts from 1.
__global__ void mlp_adam_kernel(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                                float* __restrict__ V, float lr, int step) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint32_t)kMlpParams) return;
    const float b1 = 0.9f, b2 = 0.999f;
    const float g = G[i];
    const float m = b1 * M[i] + (1.0f - b1) * g;
    const float v = b2 * V[i] + (1.0f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    const float mh = m / (1.0f - powf(b1, (float)step));
    const float vh = v / (1.0f - powf(b2, (float)step));
    P[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
int launch_sel_features(const uint16_t* codes, uint64_t n, float* feats, cudaStream_t s) {
    const uint32_t nch = (uint32_t)((n + kSelCodes - 1) / kSelCodes);
    sel_features_kernel<<<nch, 256, 0, s>>>(codes, n, feats);
    return (int)cudaGetLastError();
}

// F[NN] L[NN] R[NN] S[NN] heap[kSelBk+2] len[kSelBk] code[kSelBk] meta[192]
// stk_code[64] stk_len[64] ok
size_t sel_book_smem() {
    return (kSelBk + 2) * 4 + 2 * kSelBk * 2;  // heap (later the lengths), parent/depth array
}

int launch_sel_tag_mask(const SelArgs& a, uint32_t nchunks, uint8_t* want, cudaStream_t s) {
    sel_tag_mask_kernel<<<(nchunks + 255) / 256, 256, 0, s>>>(a, nchunks, want);
    return (int)cudaGetLastError();
}

int launch_sel_fallback_mask(const SelArgs& a, uint32_t nchunks, uint8_t* want, cudaStream_t s) {
    sel_fallback_kernel<<<(nchunks + 255) / 256, 256, 0, s>>>(a, nchunks, want);
    return (int)cudaGetLastError();
}

int launch_sel_coders(const SelArgs& a, uint32_t nlist, unsigned coder_mask, cudaStream_t s) {
    if (nlist == 0) return 0;
    cudaError_t e;
    if (coder_mask & 1u) {
        TraceScope ts(s, "sel_rze");
        const int smem = 2 * kChunkBytes + 16 + 2048 + 256 + 32;
        e = cudaFuncSetAttribute(sel_rze_sub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return (int)e;
        sel_rze_sub_kernel<<<dim3(nlist, 4), kThreads, smem, s>>>(a);
        sel_rze_assemble_kernel<<<nlist, 256, 0, s>>>(a);
    }
    if (coder_mask & 2u) {
        TraceScope ts(s, "sel_rle");
        sel_rle_kernel<<<nlist, 256, 0, s>>>(a);
    }
    if (coder_mask & 4u) {
        TraceScope ts(s, "sel_bitpack");
        sel_bitpack_kernel<<<nlist, 256, 0, s>>>(a);
    }
    if (coder_mask & 8u) {
        {
            TraceScope ts(s, "sel_hf_hist");
            sel_hf_hist_kernel<<<nlist, 256, 0, s>>>(a);
        }
        const int smem = (int)sel_book_smem();
        e = cudaFuncSetAttribute(sel_hf_book_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return (int)e;
        {
            TraceScope ts(s, "sel_hf_book");
            sel_hf_book_kernel<<<nlist, 32, smem, s>>>(a);
        }
        TraceScope ts(s, "sel_hf_encode");
        sel_hf_encode_kernel<<<nlist, 256, 0, s>>>(a);
    }
    return (int)cudaGetLastError();
}

int launch_sel_choose(const SelArgs& a, uint32_t nchunks, int mode, const float* pred, cudaStream_t s) {
    sel_choose_kernel<<<(nchunks + 255) / 256, 256, 0, s>>>(a, nchunks, mode, pred);
    return (int)cudaGetLastError();
}

int launch_sel_container(const SelArgs& a, uint32_t nchunks, uint8_t* out, unsigned long long* out_size,
                         unsigned long long* offs, cudaStream_t s) {
    sel_header_kernel<<<1, 1024, 0, s>>>(a, nchunks, out, out_size, offs);
    sel_copy_kernel<<<nchunks, 256, 0, s>>>(a, out, offs);
    return (int)cudaGetLastError();
}

int launch_mlp_forward(const float* P, const float* X, float* Y, uint32_t batch, cudaStream_t s) {
    mlp_forward_kernel<<<(batch + 127) / 128, 128, 0, s>>>(P, X, Y, batch);
    return (int)cudaGetLastError();
}

int launch_mlp_backward(const float* P, const float* X, const float* T, uint32_t batch, float* G, float* loss,
                        int kind, cudaStream_t s) {
    mlp_backward_kernel<<<(batch + 127) / 128, 128, 0, s>>>(P, X, T, batch, G, loss, kind);
    return (int)cudaGetLastError();
}

int launch_mlp_adam(float* P, const float* G, float* M, float* V, float lr, int step, cudaStream_t s) {
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, s>>>(P, G, M, V, lr, step);
    return (int)cudaGetLastError();
}

}  // namespace fzb
