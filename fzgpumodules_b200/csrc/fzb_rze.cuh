// fzb_rze.cuh -- block-level RZE chunk encoder/decoder (256 threads).
//
// Format of one chunk (modules/coders/rze/rze_stage.cu:324-445):
//   [nonzero bytes][non-repeated bm1 bytes][non-repeated bm2 bytes]
//   [non-repeated bm3 bytes][bm4, 4 bytes][u16 input size]
// bmL+1 marks the bytes of bmL that differ from their predecessor (byte 0
// compared with 0); bm1 marks nonzero input bytes.  An all-zero chunk is the
// 2-byte size tag alone; a chunk that overflows any level is stored raw and
// its header size word carries bit 31.
//
// Work split: thread t owns input bytes [64t, 64t+64) (bm1 bytes 8t..8t+7 =
// bm2 byte t); levels 3 and 4 run in warp 0.
#pragma once

#include "fzb_common.cuh"

namespace fzb {

// Compaction selectors: __byte_perm(w, 0, kRzeSel[m]) moves the bytes of w
// flagged in the 4-bit mask m to the low end, in order, zero-filled.
__constant__ static uint32_t kRzeSel[16] = {0x4444, 0x4440, 0x4441, 0x4410, 0x4442, 0x4420, 0x4421, 0x4210,
                                            0x4443, 0x4430, 0x4431, 0x4310, 0x4432, 0x4320, 0x4321, 0x3210};

struct RzeSmem {
    uint32_t* S;    // 4096 words: chunk bytes (zero past in_size)
    uint8_t* O;     // >= kChunkBytes + 8 bytes: encoded chunk
    uint32_t* bm1;  // 512 words
    uint8_t* bm2;   // 256 bytes
    uint32_t* bm3;  // 8 words
    uint32_t* ws;   // 16 words scan workspace
};

// Encodes the chunk held in sm.S (in_size bytes, rest zero).  Returns the
// header size word (bit 31 = stored raw; then the payload is S itself).
// Uniform across the block; ends with a barrier.
//
// Thread t takes S words 16t..16t+15 (bytes 64t..64t+63): their nonzero-byte
// nibbles are bm1 bytes 8t..8t+7, so levels 1 and 2 need one packed warp scan
// of both byte counts and one barrier for the per-warp totals.  Nonzero bytes
// are compacted per word by a byte permute and OR-ed into the zeroed output
// with two shared atomics (an output word can straddle two threads).  Levels
// 3 and 4 run in warp 0.  Same bytes and raw decisions as rze_stage.cu:324-445.
__device__ static uint32_t rze_encode_chunk(const RzeSmem& sm, int in_size) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t full = 0xffffffffu;
    const uint32_t raw_word = 0x80000000u | (uint32_t)in_size;
    const int b1 = (in_size + 7) >> 3, b2 = (b1 + 7) >> 3, b3 = (b2 + 7) >> 3;
    uint32_t* Ow = reinterpret_cast<uint32_t*>(sm.O);
    const uint32_t sel_tbl = kRzeSel[lane & 15];  // lane l holds selector l (read with a shuffle)
    // output zeroed for the atomics: payloads stay below kRzeAvail, so the
    // second word of an atomic pair stays below kChunkBytes + 4
    for (int i = t; i < (kChunkBytes + 16) / 16; i += kThreads)
        reinterpret_cast<uint4*>(sm.O)[i] = make_uint4(0u, 0u, 0u, 0u);
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const uint4 q = reinterpret_cast<const uint4*>(sm.S)[4 * t + i];
        w[4 * i] = q.x;
        w[4 * i + 1] = q.y;
        w[4 * i + 2] = q.z;
        w[4 * i + 3] = q.w;
    }
    uint32_t nlo = 0, nhi = 0;
    {
        uint32_t o = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) o |= w[i];
        if (__any_sync(full, o != 0u)) {
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const uint32_t hb = (((w[i] & 0x7f7f7f7fu) + 0x7f7f7f7fu) | w[i]) & 0x80808080u;
                const uint32_t nb = ((hb * 0x00204081u) >> (28 - 4 * (i & 7))) & (15u << (4 * (i & 7)));
                if (i < 8) nlo |= nb;
                else nhi |= nb;
            }
        }
    }
    // level 2: the bm1 bytes (< b1) that differ from their predecessor
    uint32_t prev = __shfl_up_sync(full, nhi, 1) >> 24;
    if (lane == 0) prev = t ? (nz_nibble(sm.S[16 * t - 2]) | (nz_nibble(sm.S[16 * t - 1]) << 4)) : 0u;
    const uint64_t M = ((uint64_t)nhi << 32) | nlo;
    uint32_t m2 = nz_byte_mask64(M ^ ((M << 8) | prev));
    {
        const int valid = b1 - 8 * t;
        m2 &= (valid >= 8) ? 0xffu : (valid <= 0 ? 0u : ((1u << valid) - 1u));
    }
    const uint32_t v12 = (uint32_t)(__popc(nlo) + __popc(nhi)) | ((uint32_t)__popc(m2) << 16);
    const uint32_t inc12 = warp_incl_scan(v12);
    if (lane == 31) sm.ws[warp] = inc12;
    sm.bm2[t] = (uint8_t)m2;
    __syncthreads();
    uint32_t tot12 = 0, pre12 = inc12 - v12;
#pragma unroll
    for (int w8 = 0; w8 < kThreads / 32; w8++) {
        const uint32_t v = sm.ws[w8];
        tot12 += v;
        if (w8 < warp) pre12 += v;
    }
    const uint32_t nzT = tot12 & 0xffffu, n2T = tot12 >> 16;
    if (nzT == 0) {  // all-zero chunk: the 2-byte size tag alone
        if (t == 0) {
            sm.O[0] = (uint8_t)(in_size & 0xff);
            sm.O[1] = (uint8_t)((in_size >> 8) & 0xff);
        }
        __syncthreads();
        return 2u;
    }
    const uint32_t wpos = nzT + n2T;
    if ((int)nzT >= kRzeAvail || (int)nzT > kRzeAvail - b1 || (int)wpos >= kRzeAvail ||
        (int)wpos > kRzeAvail - b2) {
        __syncthreads();
        return raw_word;
    }
    {   // level-1 payload: nonzero bytes in byte order; level-2: non-repeated bm1 bytes
        uint32_t pos = pre12 & 0xffffu;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const uint32_t nb = ((i < 8 ? nlo : nhi) >> (4 * (i & 7))) & 15u;
            const uint32_t sel = __shfl_sync(full, sel_tbl, nb);
            if (nb) {
                const uint32_t packed = __byte_perm(w[i], 0u, sel);
                const uint32_t sh = (pos & 3u) * 8u;
                atomicOr(&Ow[pos >> 2], packed << sh);
                atomicOr(&Ow[(pos >> 2) + 1], __funnelshift_l(packed, 0u, sh));
            }
            pos += __popc(nb);
        }
        uint32_t q = nzT + (pre12 >> 16);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t mb = (m2 >> (4 * h)) & 15u;
            const uint32_t sel = __shfl_sync(full, sel_tbl, mb);
            if (mb) {
                const uint32_t packed = __byte_perm(h ? nhi : nlo, 0u, sel);
                const uint32_t sh = (q & 3u) * 8u;
                atomicOr(&Ow[q >> 2], packed << sh);
                atomicOr(&Ow[(q >> 2) + 1], __funnelshift_l(packed, 0u, sh));
            }
            q += __popc(mb);
        }
    }
    __syncthreads();
    // levels 3 and 4 (warp 0), header
    if (warp == 0) {
        const uint2 mw = reinterpret_cast<const uint2*>(sm.bm2)[lane];
        const uint64_t M3 = ((uint64_t)mw.y << 32) | mw.x;
        uint32_t p3 = __shfl_up_sync(full, mw.y, 1) >> 24;
        if (lane == 0) p3 = 0;
        uint32_t m3 = nz_byte_mask64(M3 ^ ((M3 << 8) | p3));  // bm3 byte `lane`
        {
            const int valid = b2 - 8 * lane;
            m3 &= (valid >= 8) ? 0xffu : (valid <= 0 ? 0u : ((1u << valid) - 1u));
        }
        const uint32_t n3 = __popc(m3), inc = warp_incl_scan(n3);
        const uint32_t n3T = __shfl_sync(full, inc, 31);
        {
            uint32_t p = wpos + inc - n3, m = m3;
            while (m) {
                const uint32_t b = __ffs(m) - 1;
                m &= m - 1;
                sm.O[p++] = (uint8_t)(M3 >> (8 * b));
            }
        }
        uint32_t pb = __shfl_up_sync(full, m3, 1);
        if (lane == 0) pb = 0;
        const bool nr4 = (lane < b3) && (m3 != pb);
        const uint32_t bm4 = __ballot_sync(full, nr4);
        uint32_t wp = wpos + n3T;
        uint32_t sw = raw_word;
        if (!((int)wp >= kRzeAvail || (int)wp >= kRzeAvail - 4 || (int)wp > (kRzeAvail - 4) - b3)) {
            if (nr4) sm.O[wp + __popc(bm4 & ((1u << lane) - 1u))] = (uint8_t)m3;
            wp += __popc(bm4);
            if ((int)wp < kRzeAvail - 4) {
                if (lane == 0) {
                    sm.O[wp + 0] = (uint8_t)(bm4);
                    sm.O[wp + 1] = (uint8_t)(bm4 >> 8);
                    sm.O[wp + 2] = (uint8_t)(bm4 >> 16);
                    sm.O[wp + 3] = (uint8_t)(bm4 >> 24);
                    sm.O[wp + 4] = (uint8_t)(in_size & 0xff);
                    sm.O[wp + 5] = (uint8_t)((in_size >> 8) & 0xff);
                }
                sw = wp + 6;
            }
        }
        if (lane == 0) sm.ws[12] = sw;
    }
    __syncthreads();
    return sm.ws[12];
}

// Copies `len` bytes from shared memory `src` to global `dst` (any byte
// alignment).  Words shared with a neighbouring chunk are written bytewise so
// concurrent chunks never overwrite each other's bytes.
__device__ __forceinline__ void copy_out_bytes(uint8_t* dst, const uint8_t* src, uint32_t len) {
    if (len == 0) return;
    const uintptr_t d0 = reinterpret_cast<uintptr_t>(dst);
    const uintptr_t d1 = d0 + len;
    const uintptr_t a0 = (d0 + 3) & ~(uintptr_t)3;  // first full word
    const uintptr_t a1 = d1 & ~(uintptr_t)3;        // end of last full word
    if (a0 >= a1) {
        for (uint32_t i = threadIdx.x; i < len; i += kThreads) dst[i] = src[i];
        return;
    }
    const uint32_t head = (uint32_t)(a0 - d0), tail = (uint32_t)(d1 - a1);
    if (threadIdx.x < head) dst[threadIdx.x] = src[threadIdx.x];
    if (threadIdx.x < tail) dst[(a1 - d0) + threadIdx.x] = src[(a1 - d0) + threadIdx.x];
    const uint32_t nwords = (uint32_t)((a1 - a0) >> 2);
    uint32_t* dw = reinterpret_cast<uint32_t*>(a0);
    const uint8_t* s = src + head;
    for (uint32_t i = threadIdx.x; i < nwords; i += kThreads) {
        const uint8_t* p = s + 4 * i;
        dw[i] = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    }
}

struct RzeDecSmem {
    uint8_t* C;     // >= kChunkBytes + 8: staged compressed chunk
    uint32_t* S;    // 4096 words: decoded chunk bytes
    uint32_t* bm1;  // 512 words
    uint8_t* bm2;   // 256 bytes
    uint8_t* bm3;   // 32 bytes
    uint32_t* ws;   // 16 words
};

// Decodes one chunk (header word `e`, `osz` original bytes) from global
// `src` into sm.S (bytes past osz zeroed).  Sets kErrMalformed on an
// inconsistent chunk (and leaves zeros).  Ends with a barrier.
__device__ static void rze_decode_chunk(const uint8_t* __restrict__ src, uint32_t e, int osz,
                                 const RzeDecSmem& sm, uint32_t* err) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t comp = e & 0x7fffffffu;
    uint8_t* Sb = reinterpret_cast<uint8_t*>(sm.S);
    if (e & 0x80000000u) {  // raw chunk: copy the original bytes
        const int n = min((int)comp, osz);
        if (n != osz && t == 0) atomicOr(err, kErrMalformed);
        for (int i = t; i < kChunkBytes; i += kThreads) Sb[i] = (i < n) ? src[i] : 0;
        __syncthreads();
        return;
    }
    if (comp <= 2) {  // all-zero chunk
        for (int i = t; i < kChunkBytes / 4; i += kThreads) sm.S[i] = 0;
        __syncthreads();
        return;
    }
    if (comp > (uint32_t)kChunkBytes || comp < 7u) {
        if (t == 0) atomicOr(err, kErrMalformed);
        for (int i = t; i < kChunkBytes / 4; i += kThreads) sm.S[i] = 0;
        __syncthreads();
        return;
    }
    // stage the compressed bytes (aligned word loads, unaligned start)
    {
        const uintptr_t s0 = reinterpret_cast<uintptr_t>(src);
        const uintptr_t a0 = s0 & ~(uintptr_t)3;
        const uint32_t lead = (uint32_t)(s0 - a0);
        const uint32_t nw = (lead + comp + 3) >> 2;
        const uint32_t* sw = reinterpret_cast<const uint32_t*>(a0);
        for (uint32_t i = t; i < nw; i += kThreads) {
            uint32_t v = __ldg(sw + i);
#pragma unroll
            for (int b = 0; b < 4; b++) {
                int32_t pos = (int32_t)(4 * i + b) - (int32_t)lead;
                if (pos >= 0 && pos < (int32_t)comp) sm.C[pos] = (uint8_t)(v >> (8 * b));
            }
        }
    }
    __syncthreads();
    const int b1 = (osz + 7) >> 3, b2 = (b1 + 7) >> 3, b3 = (b2 + 7) >> 3;
    const int bm4_start = (int)comp - 6;
    const uint32_t bm4 = (uint32_t)sm.C[bm4_start] | ((uint32_t)sm.C[bm4_start + 1] << 8) |
                         ((uint32_t)sm.C[bm4_start + 2] << 16) | ((uint32_t)sm.C[bm4_start + 3] << 24);
    const int s3 = bm4_start - __popc(bm4);
    bool bad = s3 < 0;
    // bm3 from bm4: byte l = data3[rank(l)-1] if any set bit at <= l
    if (warp == 0) {
        uint32_t r = __popc(bm4 & (0xffffffffu >> (31 - lane)));
        uint32_t v = (r && lane < b3 && !bad) ? sm.C[s3 + (int)r - 1] : 0u;
        sm.bm3[lane] = (uint8_t)v;
        uint32_t pc = __popc(v);
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) pc += __shfl_xor_sync(0xffffffffu, pc, d);
        if (lane == 0) sm.ws[12] = pc;
    }
    __syncthreads();
    const int s2 = s3 - (int)sm.ws[12];
    bad = bad || s2 < 0;
    // bm2 from bm3: thread t produces bm2 byte t from bm3 bit t
    {
        const uint32_t* b3w = reinterpret_cast<const uint32_t*>(sm.bm3);
        uint32_t r = 0;
        for (int k = 0; k < (t >> 5); k++) r += __popc(b3w[k]);
        r += __popc(b3w[t >> 5] & (0xffffffffu >> (31 - lane)));
        uint32_t v = (r && t < b2 && !bad) ? sm.C[s2 + (int)r - 1] : 0u;
        sm.bm2[t] = (uint8_t)v;
        uint32_t n2;
        const uint32_t ex = block_excl_scan((uint32_t)__popc(v), sm.ws, &n2);
        const int s1 = s2 - (int)n2;
        bad = bad || s1 < 0;
        // bm1 from bm2: thread t produces bm1 bytes 8t..8t+7 from bm2 byte t
        uint64_t M = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            uint32_t rk = ex + __popc(v & (0xffu >> (7 - k)));
            uint32_t byte = (rk && (8 * t + k) < b1 && !bad) ? sm.C[s1 + (int)rk - 1] : 0u;
            M |= (uint64_t)byte << (8 * k);
        }
        // level-1 zero elimination: bytes 64t..64t+63 from bits of M
        uint32_t nzT;
        uint32_t pos = block_excl_scan((uint32_t)__popcll(M), sm.ws, &nzT);
        bad = bad || ((int)nzT != s1);
        if (bad) M = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            uint32_t nib = (uint32_t)(M >> (4 * i)) & 15u;
            uint32_t wv = 0;
            while (nib) {
                int b = __ffs(nib) - 1;
                nib &= nib - 1;
                wv |= (uint32_t)sm.C[pos++] << (8 * b);
            }
            sm.S[16 * t + i] = wv;
        }
    }
    if (bad && t == 0) atomicOr(err, kErrMalformed);
    __syncthreads();
}

}  // namespace fzb
