// fzb_huffman.cu -- PHF-layout Huffman coder (HuffmanStage<uint16_t>, coarse
// mode): device histogram, partition encode, blob assembly, decode.
//
// Blob layout (modules/coders/huffman/phf/hf.h:38-44, hf_hl.cc:50-67,
// hf_buf.cc:152-176):
//   [phf_header, 128-byte slot][revbook][par_nbit u32 x pardeg]
//   [par_entry u32 x pardeg][bitstream u32 x total_ncell]
// phf_header: int bklen(16-bit field) | int sublen | int pardeg | pad |
// size_t original_len | size_t total_nbit | size_t total_ncell |
// u32 entry[6].  Bytes 64..127 of the slot (stale encoder scratch in the
// reference) and the upper half of the first word are written as zero.
// Partitions hold sublen = 768 symbols in coarse mode (hf_bk.cc:28-37) and
// 1024 in fine mode (hf_buf.cc:46-49); within a partition codes are
// concatenated MSB-first into u32 cells (hf_kernels.cu:73-122).  Fine mode's
// ReVISIT-lite kernel (hf_kernels.cu:145-250) packs four codes of at most 8
// bits per thread and merges the shards into exactly those cells; when the
// longest code is over 8 bits the reference deflates coarsely at sublen 1024
// (hf_hl.cc:69-103).  Here one kernel serves both modes: a warp codes a
// partition, each lane sublen/32 consecutive symbols packed at its scanned
// bit offset.
#include "fzb_kernels.cuh"

namespace fzb {

constexpr uint32_t kHfSmemBook = 16384;  // books up to this size are staged in shared memory

// Privatised histogram: each CTA counts into `copies` shared-memory copies
// (warp w into copy w % copies, so a frequent symbol's atomics spread), then
// merges.  Symbols 0..3 -- the small deltas, most of a zigzag code stream --
// are counted in registers (16-bit fields, two to a word) and added once per
// warp at the end; a thread adds each run of equal other symbols among its
// eight with one atomic, four 16-byte loads in flight.  (Combining equal
// symbols across a warp with match.any first was slower: 0.109 against 0.085
// ms on C3's codes.)  Symbols >= bklen are skipped (histogram.cu:47-51).
__global__ void __launch_bounds__(512) hf_histogram_kernel(const uint16_t* __restrict__ in, uint64_t n,
                                                           uint32_t bklen, uint32_t copies,
                                                           uint32_t* __restrict__ freq) {
    extern __shared__ uint32_t hs[];
    const bool priv = bklen <= kHfSmemBook;  // larger books count straight into freq
    uint32_t* h = priv ? hs + bklen * ((threadIdx.x >> 5) % copies) : freq;
    if (priv)
        for (uint32_t i = threadIdx.x; i < bklen * copies; i += blockDim.x) hs[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const bool vec = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    const uint64_t nv = vec ? n / 8 : 0;
    const uint4* in8 = reinterpret_cast<const uint4*>(in);
    // symbols 0..3 (the small deltas of zigzag codes) count in registers, two
    // 16-bit fields per word, flushed before a field can wrap; the others go
    // to the shared copies, equal neighbours merged into one add
    uint32_t c01 = 0, c23 = 0, since = 0;
    const bool small_ok = bklen >= 4;
    constexpr int kU = 4;  // 16-byte loads in flight per thread
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < nv; i0 += kU * stride) {
        uint4 v[kU];
#pragma unroll
        for (int u = 0; u < kU; u++) v[u] = i0 + u * stride < nv ? __ldg(in8 + i0 + u * stride) : make_uint4(~0u, ~0u, ~0u, ~0u);
#pragma unroll
        for (int u = 0; u < kU; u++) {
            if (i0 + u * stride >= nv) break;
            const uint32_t w[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
            uint32_t cur = 0xffffffffu, run = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t a = (w[k >> 1] >> (16 * (k & 1))) & 0xffffu;
                if (small_ok && a < 4u) {
                    const uint32_t inc = 1u << ((a & 1u) << 4);
                    if (a < 2u) c01 += inc;
                    else c23 += inc;
                    continue;
                }
                if (a != cur) {
                    if (cur < bklen) atomicAdd(&h[cur], run);
                    cur = a;
                    run = 0;
                }
                run++;
            }
            if (cur < bklen) atomicAdd(&h[cur], run);
            since += 8;
        }
        if (since >= 65536 - 8 * kU) {  // a 16-bit field could wrap in the next round
            atomicAdd(&h[0], c01 & 0xffffu);
            atomicAdd(&h[1], c01 >> 16);
            atomicAdd(&h[2], c23 & 0xffffu);
            atomicAdd(&h[3], c23 >> 16);
            c01 = c23 = since = 0;
        }
    }
    if (small_ok) {  // every lane of the block reaches this point
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t t0 = __reduce_add_sync(0xffffffffu, c01 & 0xffffu), t1 = __reduce_add_sync(0xffffffffu, c01 >> 16);
        const uint32_t t2 = __reduce_add_sync(0xffffffffu, c23 & 0xffffu), t3 = __reduce_add_sync(0xffffffffu, c23 >> 16);
        if (lane == 0) {
            if (t0) atomicAdd(&h[0], t0);
            if (t1) atomicAdd(&h[1], t1);
            if (t2) atomicAdd(&h[2], t2);
            if (t3) atomicAdd(&h[3], t3);
        }
    }
    for (uint64_t i = 8 * nv + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t a = in[i];
        if (a < bklen) atomicAdd(&h[a], 1u);
    }
    if (!priv) return;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < bklen; i += blockDim.x) {
        uint32_t t = 0;
        for (uint32_t c = 0; c < copies; c++) t += hs[c * bklen + i];
        if (t) atomicAdd(&freq[i], t);
    }
}

// Encode, a warp per partition (static interleave over all warps).  Lane l
// codes the partition's symbols l*PER .. l*PER + PER - 1 (PER = SUB / 32):
// it looks up their codewords, a warp scan of the code lengths gives its
// first bit, and it packs its codes MSB-first into 32-bit words that it ORs
// into the warp's shared-memory cells (only a lane's first and last word
// can be shared with a neighbour).  The warp then copies the cells to the
// partition's slot and clears them for its next partition.
constexpr int kHfEncWarps = 8;

template <int SUB>
__global__ void __launch_bounds__(32 * kHfEncWarps) hf_encode_kernel(const uint16_t* __restrict__ in, uint64_t n,
                                                                     const uint32_t* __restrict__ bk4, uint32_t bklen,
                                                                     uint32_t pardeg, uint32_t* __restrict__ slots,
                                                                     uint32_t* __restrict__ par_nbit,
                                                                     uint32_t* __restrict__ par_ncell) {
    constexpr int PER = SUB / 32;  // 24 (coarse) or 32 (fine)
    static_assert(PER % 8 == 0, "whole 16-byte loads per lane");
    extern __shared__ uint32_t sm[];
    const bool staged = bklen <= kHfSmemBook;
    const uint32_t* book = staged ? sm + kHfEncWarps * SUB : bk4;  // bklen words when staged
    if (staged)
        for (uint32_t i = threadIdx.x; i < bklen; i += blockDim.x) sm[kHfEncWarps * SUB + i] = bk4[i];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t* cells = sm + warp * SUB;
    for (uint32_t i = lane; i < (uint32_t)SUB; i += 32) cells[i] = 0;
    __syncthreads();
    const bool vec = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    for (uint32_t p = blockIdx.x * kHfEncWarps + warp; p < pardeg; p += gridDim.x * kHfEncWarps) {
        const uint64_t base = (uint64_t)p * SUB + (uint64_t)PER * lane;
        uint32_t w[PER];
        if (vec && base + PER <= n) {
            const uint4* src = reinterpret_cast<const uint4*>(in + base);
#pragma unroll
            for (int q = 0; q < PER / 8; q++) {
                const uint4 v = __ldg(src + q);
                const uint32_t h[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    w[8 * q + 2 * k] = h[k] & 0xffffu;
                    w[8 * q + 2 * k + 1] = h[k] >> 16;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < PER; k++) w[k] = base + k < n ? (uint32_t)in[base + k] : 0xffffffffu;
        }
        uint32_t bits = 0;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            w[k] = w[k] < bklen ? book[w[k]] : 0u;  // symbols past the book (or the input) are not coded
            bits += w[k] >> 27;
        }
        uint32_t inc = bits;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(~0u, inc, d);
            if (lane >= (uint32_t)d) inc += y;
        }
        const uint32_t total = __shfl_sync(~0u, inc, 31);
        const uint32_t off = inc - bits;
        uint32_t cw = off >> 5, nb = off & 31u;  // acc holds the cell's first nb bits, MSB-aligned
        uint64_t acc = 0;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t len = w[k] >> 27;
            if (len) acc |= (uint64_t)(w[k] & 0x7ffffffu) << (64 - nb - len);
            nb += len;
            if (nb >= 32) {
                atomicOr(&cells[cw], (uint32_t)(acc >> 32));
                cw++;
                acc <<= 32;
                nb -= 32;
            }
        }
        if (nb) atomicOr(&cells[cw], (uint32_t)(acc >> 32));  // zero bits of other lanes OR in harmlessly
        __syncwarp();
        const uint32_t ncell = (total + 31) / 32;
        uint32_t* dst = slots + (size_t)p * SUB;
        for (uint32_t i = lane; i < ncell; i += 32) {
            dst[i] = cells[i];
            cells[i] = 0;
        }
        if (lane == 0) {
            par_nbit[p] = total;
            par_ncell[p] = ncell;
        }
        __syncwarp();
    }
    asm volatile("griddepcontrol.launch_dependents;");  // the cell-count scan may start launching
}

// Header + revbook (one CTA of 1024 threads).  hf_concat_kernel adds up the
// total bit count and writes par_nbit and par_entry.
// *ncell_total must already hold the cell count.
__global__ void __launch_bounds__(1024) hf_header_kernel(uint8_t* __restrict__ out, uint32_t bklen,
                                                         uint32_t sublen, uint32_t pardeg, uint64_t n,
                                                         const uint8_t* __restrict__ revbook,
                                                         uint32_t revbook_bytes,
                                                         const uint32_t* __restrict__ ncell_total,
                                                         unsigned long long* __restrict__ out_size) {
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the scan's cell total
    const uint32_t e1 = 128, e2 = e1 + revbook_bytes, e3 = e2 + 4 * pardeg, e4 = e3 + 4 * pardeg;
    for (uint32_t i = threadIdx.x; i < revbook_bytes; i += blockDim.x) out[e1 + i] = revbook[i];
    if (threadIdx.x == 0) {
        const uint64_t ncell = *ncell_total;
        uint32_t* h32 = reinterpret_cast<uint32_t*>(out);
        for (int i = 0; i < 32; i++) h32[i] = 0;
        h32[0] = bklen & 0xffffu;
        h32[1] = sublen;
        h32[2] = pardeg;
        // 64-bit fields as word pairs (the blob is only 4-byte aligned)
        h32[4] = (uint32_t)n;
        h32[5] = (uint32_t)(n >> 32);
        h32[6] = h32[7] = 0;  // total bits, written by hf_concat_kernel
        h32[8] = (uint32_t)ncell;
        h32[9] = (uint32_t)(ncell >> 32);
        uint32_t* ent = reinterpret_cast<uint32_t*>(out + 40);
        ent[0] = 0;
        ent[1] = e1;
        ent[2] = e2;
        ent[3] = e3;
        ent[4] = e4;
        ent[5] = e4 + (uint32_t)(4 * ncell);
        *out_size = e4 + 4 * ncell;
    }
    asm volatile("griddepcontrol.launch_dependents;");
}

// Partition cells from their slots to the bitstream (u32 aligned), with
// the par_nbit and par_entry words and the total bit count.  A warp takes
// kHfCatGroup consecutive partitions, lane l < kHfCatGroup holding the header
// of the l-th, and copies four at a time so that their loads are in flight
// together; small groups give enough warps to cover the load latency.
constexpr int kHfCatWarps = 8;
constexpr int kHfCatGroup = 8;
constexpr int kHfCatWords = 96;  // words per partition copied in the unrolled pass

__global__ void __launch_bounds__(32 * kHfCatWarps) hf_concat_kernel(
    const uint32_t* __restrict__ slots, const uint32_t* __restrict__ par_nbit,
    const uint32_t* __restrict__ par_ncell, const uint32_t* __restrict__ par_entry, uint32_t pardeg, uint32_t sublen,
    uint32_t* __restrict__ out_nbit, uint32_t* __restrict__ out_entry, uint32_t* __restrict__ bitstream,
    uint32_t* __restrict__ ctrl, uint32_t* __restrict__ head_nbit) {
    __shared__ unsigned long long s_bits[kHfCatWarps];
    asm volatile("griddepcontrol.wait;" ::: "memory");  // offsets and header of the kernels before
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned long long bits = 0;
    for (uint32_t g = blockIdx.x * kHfCatWarps + warp; (uint64_t)kHfCatGroup * g < pardeg;
         g += gridDim.x * kHfCatWarps) {
        const uint32_t pl = kHfCatGroup * g + lane;
        uint32_t nc = 0, e = 0;
        if (lane < (uint32_t)kHfCatGroup && pl < pardeg) {
            const uint32_t nb = par_nbit[pl];
            nc = par_ncell[pl];
            e = par_entry[pl];
            out_nbit[pl] = nb;
            out_entry[pl] = e;
            bits += nb;
        }
#pragma unroll
        for (int j = 0; j < kHfCatGroup; j += 4) {
            uint32_t v[4][kHfCatWords / 32];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t ncj = __shfl_sync(~0u, nc, j + q);
                const uint32_t* src = slots + (size_t)(kHfCatGroup * g + j + q) * sublen;
#pragma unroll
                for (int r = 0; r < kHfCatWords / 32; r++) {
                    const uint32_t i = lane + 32 * r;
                    v[q][r] = i < ncj ? src[i] : 0u;
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t ncj = __shfl_sync(~0u, nc, j + q), ej = __shfl_sync(~0u, e, j + q);
#pragma unroll
                for (int r = 0; r < kHfCatWords / 32; r++) {
                    const uint32_t i = lane + 32 * r;
                    if (i < ncj) bitstream[ej + i] = v[q][r];
                }
                const uint32_t* src = slots + (size_t)(kHfCatGroup * g + j + q) * sublen;
                for (uint32_t i = kHfCatWords + lane; i < ncj; i += 32) bitstream[ej + i] = src[i];
            }
        }
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) bits += __shfl_xor_sync(~0u, bits, d);
    if (lane == 0) s_bits[warp] = bits;
    __syncthreads();
    // the CTA's bits (under 2^32) go into the 64-bit count ctrl[2] (low) /
    // ctrl[3] (high); the last CTA writes it to the header as two words
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kHfCatWarps; w++) t += s_bits[w];
        const uint32_t lo = (uint32_t)t, old = atomicAdd(&ctrl[2], lo);
        if (old + lo < old) atomicAdd(&ctrl[3], 1u);
        __threadfence();
        if (atomicAdd(&ctrl[4], 1u) == gridDim.x - 1) {
            __threadfence();
            head_nbit[0] = atomicAdd(&ctrl[2], 0u);
            head_nbit[1] = atomicAdd(&ctrl[3], 0u);
        }
    }
}

// Canonical decode (hf_kernels.cu:258-312).  The reference gives each
// partition to one thread.  Here, when the book has short codes, a warp
// decodes one partition at a time, so every lane has work in proportion to
// the partition's bits rather than its symbols and the output leaves in
// coalesced 16-byte stores:
//   * tables: each CTA builds a multi-symbol lookup table indexed by the next
//     kHfLutBits bits.  Entry u holds up to kHfMultiMax whole codes that lie
//     inside those bits: their symbols, their total length, their end
//     offsets and an error flag.  A first-code table built with the canonical
//     walk's own comparisons (the shortest l with v >= first[l]) feeds it, so
//     symbols and error flags are identical to the walk's.  A second table
//     gives every whole code in the window (count and end offsets) for
//     counting.  A code longer than the table continues the walk from length
//     kHfLutBits + 1;
//   * count: the partition's nbit bits are cut into up to 32 equal segments
//     of at least 32 bits.  Lane j decodes from its segment's first bit
//     (possibly inside a code) to the first code boundary at or past the
//     segment's end, counting codes and noting its code starts over its first
//     64 bits (F);
//   * synchronise: Huffman codes resynchronise.  Lane j - 1, if it decoded
//     from a true boundary, decodes on past its end and notes the true starts
//     (T) until one of them is also in lane j's F, at most 64 bits.  From the
//     first shared start lane j's decode is the true decode: its count is
//     corrected for the codes before that start, and its end is a true
//     boundary.  A lane with no shared start inside its segment decodes again
//     from its predecessor's true end;
//   * emit: a warp prefix sum of the counts places each lane's symbols; each
//     lane decodes its codes from its true start into the warp's staging
//     strip, and the warp copies the partition out.
// A book whose shortest code has more than kHfCoopMaxShortest bits (codes of
// nearly one length resynchronise slowly, if ever) is decoded one partition
// per lane instead, straight to the output.
// A well-formed partition decodes its want symbols in exactly nbit bits;
// anything else (a length past 31, a table index past the book, a bit count
// that does not match) raises kErrMalformed.  CTA b owns partitions b, b + G,
// b + 2G, ... (G CTAs), spread over the field, and its warps take them in
// turn from a shared-memory counter, so no global counter is contended.
constexpr int kHfLutBits = 12;
constexpr uint32_t kHfLutSize = 1u << kHfLutBits;
constexpr int kHfMultiMax = 4;
constexpr int kHfDecWarps = 16;
constexpr int kHfDecThreads = 32 * kHfDecWarps;
constexpr int kHfCoopMaxShortest = 4;
constexpr uint32_t kHfStage = kHfSublenFine;  // symbols staged per warp
// symbols (8 B), meta (4 B) and counts (4 B) per window, then the warps'
// staging strips, which hold the first-code table while the CTA builds
constexpr size_t kHfDecSmem = 16 * (size_t)kHfLutSize + 2 * (size_t)kHfStage * kHfDecWarps;
static_assert(2 * kHfStage * kHfDecWarps >= 4 * kHfLutSize, "first-code table fits the strips");

// The partition's cells (MSB-first u32 words) from any bit: w0:w1 hold the
// next 64 - off bits, w2 the word after them.
struct HfBits {
    const uint32_t* cells;
    uint32_t ncells, wi, w0, w1, w2, off;
    __device__ __forceinline__ uint32_t word(uint32_t i) const { return i < ncells ? __ldg(cells + i) : 0u; }
    __device__ __forceinline__ void seek(uint32_t c0, uint32_t bit) {
        const uint32_t w = c0 + (bit >> 5);
        w0 = word(w);
        w1 = word(w + 1);
        w2 = word(w + 2);
        wi = w + 3;
        off = bit & 31u;
    }
    // the next 32 bits, MSB first
    __device__ __forceinline__ uint32_t win() const { return __funnelshift_l(w1, w0, off); }
    // l <= 31; moves to the next word without a branch
    __device__ __forceinline__ void advance(uint32_t l) {
        off += l;
        const bool step = off >= 32;
        const uint32_t nw = step && wi < ncells ? __ldg(cells + wi) : 0u;
        w0 = step ? w1 : w0;
        w1 = step ? w2 : w1;
        w2 = step ? nw : w2;
        wi += step ? 1u : 0u;
        off &= 31u;
    }
};

struct HfDecTables {
    const uint2* sym;
    const uint32_t* meta;  // total length | count << 4 | bad << 7 | first length << 8 | end offsets << 12
    const uint32_t* cmeta;  // every whole code in the window: total length | count << 4 | end offsets << 8
    const uint32_t* first;
    const int* entry;
    const uint16_t* keys;
    uint32_t bklen;
};

// the canonical walk from length kHfLutBits + 1 over the next 32 bits w;
// 32 when no code matches
__device__ __forceinline__ int hf_walk(uint32_t w, const uint32_t* first, uint32_t& v) {
    int l = kHfLutBits + 1;
    v = w >> (32 - l);
    while (l < 32 && v < first[l]) {
        l++;
        v = w >> (32 - l);
    }
    return l;
}

// One probe for counting: total length, codes, end offsets (bit k-1 = a code
// ends k bits on).  A missing code counts as one of 31 bits.
__device__ __forceinline__ void hf_probe(uint32_t w, const HfDecTables& t, uint32_t& tot, uint32_t& c,
                                         uint32_t& E) {
    const uint32_t m = t.cmeta[w >> (32 - kHfLutBits)];
    c = (m >> 4) & 15u;
    tot = m & 15u;
    E = m >> 8;
    if (c == 0) {
        uint32_t v;
        const int l = hf_walk(w, t.first, v);
        tot = l >= 32 ? 31u : (uint32_t)l;
        E = 1u << (tot - 1);
        c = 1;
    }
}

// the code starts in a probe's window, relative to its first bit
__device__ __forceinline__ uint32_t hf_starts(uint32_t tot, uint32_t E) {
    return 1u | ((E << 1) & ((1u << tot) - 1u));
}

// Decodes from bit `start` to the first code boundary at or past s_end (e),
// counting the codes (cnt); F: the code starts in [rec, rec + 64).
__device__ __forceinline__ void hf_count(HfBits& r, const HfDecTables& t, uint32_t start, uint32_t s_end,
                                         uint32_t rec, uint32_t& e, uint32_t& cnt, uint64_t& F) {
    uint32_t pos = start;
    cnt = 0;
    F = 0;
    // while a whole window lies before s_end every code in it counts (a
    // longer code is a single code, so its end is the boundary sought)
    while (pos + kHfLutBits <= s_end) {
        uint32_t tot, c, E;
        hf_probe(r.win(), t, tot, c, E);
        const uint32_t d = pos - rec;
        if (d < 64) F |= (uint64_t)hf_starts(tot, E) << d;
        cnt += c;
        r.advance(tot);
        pos += tot;
    }
    while (pos < s_end) {
        uint32_t tot, c, E;
        hf_probe(r.win(), t, tot, c, E);
        const uint32_t d = pos - rec;
        if (d < 64) F |= (uint64_t)hf_starts(tot, E) << d;
        const uint32_t rr = s_end - pos;
        uint32_t adv = tot;
        if (tot > rr) {  // the first code end at or past s_end
            adv = rr - 1 + (uint32_t)__ffs(E >> (rr - 1));
            c = (uint32_t)__popc(E & ((1u << adv) - 1u));
        }
        cnt += c;
        r.advance(adv);
        pos += adv;
    }
    e = pos;
}

// Decodes `count` codes from the reader, handing symbol i to put(i, s);
// returns the bits used.
template <class Put>
__device__ __forceinline__ uint32_t hf_emit(HfBits& r, const HfDecTables& t, uint32_t count, uint32_t& eacc,
                                            bool& bad, Put put) {
    uint32_t i = 0, used = 0;
    // while kHfMultiMax symbols remain every probe's codes are all taken, and
    // symbols past a probe's count are overwritten by the next probe
    while (i + kHfMultiMax <= count) {
        const uint32_t w = r.win();
        const uint32_t u = w >> (32 - kHfLutBits);
        const uint32_t m = t.meta[u];
        uint32_t cm = (m >> 4) & 7u;
        uint32_t adv = m & 15u;
        if (cm == 0) {
            uint32_t v;
            int l = hf_walk(w, t.first, v);
            uint32_t s = 0;
            if (l >= 32) {  // no code: flag it and move on by 31 bits
                bad = true;
                l = 31;
            } else {
                const int k = t.entry[l] + (int)v - (int)t.first[l];
                const bool kin = k >= 0 && k < (int)t.bklen;
                bad |= !kin;
                s = kin ? __ldg(t.keys + k) : 0u;
            }
            put(i, s);
            cm = 1;
            adv = (uint32_t)l;
        } else {
            const uint2 sy = t.sym[u];
            put(i, sy.x);
            put(i + 1, sy.x >> 16);
            put(i + 2, sy.y);
            put(i + 3, sy.y >> 16);
            eacc |= m;
        }
        i += cm;
        r.advance(adv);
        used += adv;
    }
    while (i < count) {
        const uint32_t w = r.win();
        const uint32_t u = w >> (32 - kHfLutBits);
        const uint32_t m = t.meta[u];
        const uint32_t cm = (m >> 4) & 7u;
        uint32_t adv;
        if (cm == 0) {
            uint32_t v;
            int l = hf_walk(w, t.first, v);
            uint32_t s = 0;
            if (l >= 32) {  // no code: flag it and move on by 31 bits
                bad = true;
                l = 31;
            } else {
                const int k = t.entry[l] + (int)v - (int)t.first[l];
                const bool kin = k >= 0 && k < (int)t.bklen;
                bad |= !kin;
                s = kin ? __ldg(t.keys + k) : 0u;
            }
            put(i, s);
            i++;
            adv = (uint32_t)l;
        } else {
            const uint2 sy = t.sym[u];
            const uint32_t take = min(cm, count - i);
            put(i, sy.x);
            if (take > 1) put(i + 1, sy.x >> 16);
            if (take > 2) put(i + 2, sy.y);
            if (take > 3) put(i + 3, sy.y >> 16);
            if (take == cm) {
                adv = m & 15u;
            } else {  // the end of the take-th code
                uint32_t E = m >> 12;
                if (take > 1) E &= E - 1;
                if (take > 2) E &= E - 1;
                adv = (uint32_t)__ffs(E);
            }
            eacc |= m;
            i += take;
        }
        r.advance(adv);
        used += adv;
    }
    return used;
}

__global__ void __launch_bounds__(kHfDecThreads, 2)
    hf_decode_kernel(const uint8_t* __restrict__ blob, uint64_t blob_bytes, uint64_t n, uint32_t bklen_expect,
                     uint16_t* __restrict__ out, uint32_t* err) {
    __shared__ uint32_t s_first[32];
    __shared__ int s_entry[32];
    __shared__ uint32_t s_next;  // the CTA's next partition (or group of 32), in its own numbering
    extern __shared__ __align__(16) uint8_t hf_smem[];
    uint2* msym = reinterpret_cast<uint2*>(hf_smem);
    uint32_t* mmeta = reinterpret_cast<uint32_t*>(hf_smem + 8 * kHfLutSize);
    uint32_t* cmeta = reinterpret_cast<uint32_t*>(hf_smem + 12 * kHfLutSize);
    uint8_t* strips = hf_smem + 16 * kHfLutSize;

    const uint32_t* ent = reinterpret_cast<const uint32_t*>(blob + 40);
    const uint32_t e1 = ent[1], e2 = ent[2], e3 = ent[3], e4 = ent[4], e5 = ent[5];
    const uint32_t* h32 = reinterpret_cast<const uint32_t*>(blob);
    const uint32_t bklen = h32[0] & 0xffffu, sublen = h32[1];
    const bool sub_ok = sublen == (uint32_t)kHfSublen || sublen == (uint32_t)kHfSublenFine;
    const uint32_t pardeg = sub_ok ? (uint32_t)((n - 1) / sublen + 1) : 0u;
    const bool ok = bklen == bklen_expect && sub_ok && h32[2] == pardeg &&
                    h32[4] == (uint32_t)n && h32[5] == (uint32_t)(n >> 32) && e1 == 128 &&
                    e2 == e1 + 256 + 2 * bklen && e3 == e2 + 4 * pardeg && e4 == e3 + 4 * pardeg &&
                    e4 <= e5 && e5 <= blob_bytes;
    if (!ok) {
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(err, kErrMalformed);
        return;
    }
    const int* rb = reinterpret_cast<const int*>(blob + e1);
    if (threadIdx.x < 32) {
        s_first[threadIdx.x] = (uint32_t)rb[threadIdx.x];
        s_entry[threadIdx.x] = rb[32 + threadIdx.x];
    }
    if (threadIdx.x == 0) s_next = 0;
    const uint16_t* keys = reinterpret_cast<const uint16_t*>(blob + e1 + 256);
    __syncthreads();
    // first-code table: symbol << 16 | bad << 8 | length (length 0: a longer code)
    uint32_t* first = reinterpret_cast<uint32_t*>(strips);
    for (uint32_t u = threadIdx.x; u < kHfLutSize; u += blockDim.x) {
        uint32_t e = 0;
        for (int l = 1; l <= kHfLutBits; l++) {
            const uint32_t v = u >> (kHfLutBits - l);
            if (v >= s_first[l]) {
                const int k = s_entry[l] + (int)v - (int)s_first[l];
                const bool kin = k >= 0 && k < (int)bklen;
                e = (kin ? ((uint32_t)__ldg(keys + k) << 16) : (1u << 8)) | (uint32_t)l;
                break;
            }
        }
        first[u] = e;
    }
    __syncthreads();
    // multi-symbol table; a code with an out-of-book index ends the entry and,
    // as the entry's first code, is emitted as symbol 0 with the bad flag
    for (uint32_t u = threadIdx.x; u < kHfLutSize; u += blockDim.x) {
        uint64_t syms = 0;
        uint32_t tot = 0, cnt = 0, bad = 0, len1 = 0, ends = 0;
        while (cnt < (uint32_t)kHfMultiMax) {
            const uint32_t e = first[(u << tot) & (kHfLutSize - 1)];
            const uint32_t l = e & 0xffu;
            if (l == 0 || tot + l > (uint32_t)kHfLutBits) break;
            if (e & (1u << 8)) {
                if (cnt == 0) {
                    bad = 1;
                    tot = len1 = l;
                    ends = 1u << (l - 1);
                    cnt = 1;
                }
                break;
            }
            syms |= (uint64_t)(e >> 16) << (16 * cnt);
            if (cnt == 0) len1 = l;
            tot += l;
            ends |= 1u << (tot - 1);
            cnt++;
        }
        msym[u] = make_uint2((uint32_t)syms, (uint32_t)(syms >> 32));
        mmeta[u] = tot | cnt << 4 | bad << 7 | len1 << 8 | ends << 12;
        // counting ignores the error flag and the kHfMultiMax cap
        uint32_t ctot = 0, ccnt = 0, cends = 0;
        while (true) {
            const uint32_t l = first[(u << ctot) & (kHfLutSize - 1)] & 0xffu;
            if (l == 0 || ctot + l > (uint32_t)kHfLutBits) break;
            ctot += l;
            cends |= 1u << (ctot - 1);
            ccnt++;
        }
        cmeta[u] = ctot | ccnt << 4 | cends << 8;
    }
    // the shortest code length in the book (lengths l with entry[l + 1] > entry[l])
    int shortest = 32;
    for (int l = 30; l >= 1; l--)
        if (s_entry[l + 1] > s_entry[l]) shortest = l;
    __syncthreads();

    const HfDecTables tb{msym, mmeta, cmeta, s_first, s_entry, keys, bklen};
    const uint32_t* nbits_g = reinterpret_cast<const uint32_t*>(blob + e2);
    const uint32_t* entry_g = reinterpret_cast<const uint32_t*>(blob + e3);
    const uint32_t ncells = (e5 - e4) / 4;
    const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint16_t* stage = reinterpret_cast<uint16_t*>(strips + 2 * kHfStage * warp);
    HfBits r;
    r.cells = reinterpret_cast<const uint32_t*>(blob + e4);
    r.ncells = ncells;
    bool bad = false;

    if (shortest > kHfCoopMaxShortest) {
        // one partition per lane, 32 per take from the counter
        while (true) {
            uint32_t g = 0;
            if (lane == 0) g = blockIdx.x + atomicAdd(&s_next, 1u) * gridDim.x;
            g = __shfl_sync(~0u, g, 0);
            if (g >= (pardeg + 31) / 32) break;
            const uint32_t p = 32 * g + lane;
            if (p < pardeg) {
                const uint32_t nbit = __ldg(nbits_g + p);
                const uint64_t o0 = (uint64_t)p * sublen;
                const uint32_t want = (uint32_t)min((uint64_t)sublen, n - o0);
                if (nbit == 0) {
                    if (s_entry[1] == 1) {
                        const uint16_t k0 = __ldg(keys);
                        for (uint32_t i = 0; i < want; i++) out[o0 + i] = k0;
                    } else {
                        bad = true;
                    }
                } else {
                    r.seek(min(__ldg(entry_g + p), ncells), 0);
                    uint32_t eacc = 0;
                    const uint32_t used =
                        hf_emit(r, tb, want, eacc, bad, [&](uint32_t i, uint32_t s) { out[o0 + i] = (uint16_t)s; });
                    bad |= ((eacc >> 7) & 1u) != 0 || used != nbit;
                }
            }
        }
        if (bad) atomicOr(err, kErrMalformed);
        return;
    }

    while (true) {
        uint32_t p = 0;
        if (lane == 0) p = blockIdx.x + atomicAdd(&s_next, 1u) * gridDim.x;
        p = __shfl_sync(~0u, p, 0);
        if (p >= pardeg) break;
        const uint32_t nbit = __ldg(nbits_g + p);
        const uint32_t c0 = min(__ldg(entry_g + p), ncells);
        const uint64_t o0 = (uint64_t)p * sublen;
        const uint32_t want = (uint32_t)min((uint64_t)sublen, n - o0);
        if (nbit == 0) {
            if (s_entry[1] == 1) {
                // a single symbol in the book gets a zero-length code: every
                // output is that symbol (the reference leaves this case undecoded)
                const uint16_t k0 = __ldg(keys);
                for (uint32_t i = lane; i < want; i += 32) out[o0 + i] = k0;
            } else {
                bad = true;
            }
            continue;
        }
        if (nbit > 31u * sublen) {  // longer than want codes of 31 bits
            bad = true;
            continue;
        }
        const uint32_t seg = max(32u, (nbit + 31) / 32), nact = (nbit + seg - 1) / seg;
        const bool act = lane < nact;
        const uint32_t sj = min(lane * seg, nbit), send = min(sj + seg, nbit);
        // the next lane's segment bits that a shared start may fall in
        const uint32_t lim = min(64u, min(send + seg, nbit) - send);
        uint32_t e = nbit, cnt = 0;
        uint64_t F = 0, T = 0;
        if (act) {
            r.seek(c0, sj);
            hf_count(r, tb, sj, send, sj, e, cnt, F);
        }
        const uint64_t Fn = __shfl_down_sync(~0u, F, 1);
        // lanes in `go` decode on from their end, noting true starts for the
        // next lane until one is in its F
        auto extend = [&](bool go) {
            uint32_t x = e;
            T = 0;
            while (__any_sync(~0u, go)) {
                if (go) {
                    uint32_t tot, c, E;
                    hf_probe(r.win(), tb, tot, c, E);
                    T |= (uint64_t)hf_starts(tot, E) << (x - send);
                    r.advance(tot);
                    x += tot;
                    go = (T & Fn) == 0 && x < send + lim;
                }
            }
        };
        extend(act && lane + 1 < nact && e < send + lim);
        // lane j's count from its first start shared with lane j - 1's true starts
        auto check = [&](uint64_t tprev, uint32_t& ct) -> bool {
            const uint64_t both = tprev & F;
            if (!both) return false;
            const uint32_t q = (uint32_t)__ffsll((long long)both) - 1;
            if (sj + q >= send) return false;
            const uint64_t below = (1ull << q) - 1ull;
            ct = cnt - (uint32_t)__popcll(F & below) + (uint32_t)__popcll(tprev & below);
            return true;
        };
        uint32_t ct = cnt;
        bool good = true;
        {
            const uint64_t tprev = __shfl_up_sync(~0u, T, 1);
            if (act && lane > 0) good = check(tprev, ct);
        }
        uint32_t fails = __ballot_sync(~0u, !good);
        while (fails) {
            const uint32_t k = (uint32_t)__ffs(fails) - 1;  // lanes below k are true
            const uint32_t tk = __shfl_sync(~0u, e, k - 1);
            if (lane == k) {
                r.seek(c0, tk);
                uint64_t Fk;
                hf_count(r, tb, tk, send, sj, e, cnt, Fk);
                ct = cnt;
            }
            extend(lane == k && k + 1 < nact && e < send + lim);
            fails &= ~(1u << k);
            const uint64_t tnew = __shfl_sync(~0u, T, k);
            bool recheck_fail = false;
            if (lane == k + 1 && act && !((fails >> lane) & 1u)) recheck_fail = !check(tnew, ct);
            fails |= __ballot_sync(~0u, recheck_fail);
        }
        // place each lane's symbols
        const uint32_t mine = act ? ct : 0u;
        uint32_t inc = mine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(~0u, inc, d);
            if (lane >= (uint32_t)d) inc += y;
        }
        const uint32_t total = __shfl_sync(~0u, inc, 31);
        const uint32_t elast = __shfl_sync(~0u, e, nact - 1);
        const uint32_t tstart = __shfl_up_sync(~0u, e, 1);
        if (total != want || elast != nbit) {
            bad = true;
            continue;
        }
        if (act) {
            const uint32_t t0 = lane == 0 ? 0u : tstart;
            const uint32_t off = inc - mine;
            if (mine) {
                r.seek(c0, t0);
                uint32_t eacc = 0;
                const uint32_t used =
                    hf_emit(r, tb, mine, eacc, bad, [&](uint32_t i, uint32_t s) { stage[off + i] = (uint16_t)s; });
                bad |= ((eacc >> 7) & 1u) != 0 || t0 + used != e;
            } else {
                bad |= t0 != e;
            }
        }
        __syncwarp();
        if (aligned) {
            const uint32_t n8 = want >> 3;
            uint4* d4 = reinterpret_cast<uint4*>(out + o0);
            const uint4* s4 = reinterpret_cast<const uint4*>(stage);
            for (uint32_t i = lane; i < n8; i += 32) d4[i] = s4[i];
            for (uint32_t i = (n8 << 3) + lane; i < want; i += 32) out[o0 + i] = stage[i];
        } else {
            for (uint32_t i = lane; i < want; i += 32) out[o0 + i] = stage[i];
        }
        __syncwarp();
    }
    if (bad) atomicOr(err, kErrMalformed);
}

int launch_hf_histogram(const uint16_t* in, uint64_t n, uint32_t bklen, uint32_t* freq, int sms,
                        cudaStream_t s) {
    cudaMemsetAsync(freq, 0, 4 * (size_t)bklen, s);
    const uint32_t copies = bklen <= 4096 ? 4u : 1u;
    const int smem = bklen <= kHfSmemBook ? 4 * (int)(bklen * copies) : 0;
    cudaFuncSetAttribute(hf_histogram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    TraceScope ts(s, "hf_histogram");
    hf_histogram_kernel<<<2 * sms, 512, smem, s>>>(in, n, bklen, copies, freq);
    return (int)cudaGetLastError();
}

int launch_hf_encode(const uint16_t* in, uint64_t n, const uint32_t* bk4, uint32_t bklen, uint32_t sublen,
                     const uint8_t* d_revbook, uint8_t* out, unsigned long long* out_size,
                     uint32_t* slots, uint32_t* par_nbit, uint32_t* par_ncell, uint32_t* par_entry,
                     uint32_t* tiles, uint32_t* ncell_total, uint32_t* ctrl, int sms, cudaStream_t s) {
    if (sublen != (uint32_t)kHfSublen && sublen != (uint32_t)kHfSublenFine) return (int)cudaErrorInvalidValue;
    const uint32_t pardeg = (uint32_t)((n - 1) / sublen + 1);
    const int smem = 4 * (kHfEncWarps * (int)sublen + (bklen <= kHfSmemBook ? (int)bklen : 0));
    const unsigned grid =
        (unsigned)max((uint64_t)1, min((uint64_t)(pardeg + kHfEncWarps - 1) / kHfEncWarps, (uint64_t)4 * sms));
    cudaError_t e;
    {
        TraceScope ts(s, "hf_encode");
        if (sublen == (uint32_t)kHfSublenFine) {
            e = cudaFuncSetAttribute(hf_encode_kernel<kHfSublenFine>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     smem);
            if (e != cudaSuccess) return (int)e;
            hf_encode_kernel<kHfSublenFine><<<grid, 32 * kHfEncWarps, smem, s>>>(in, n, bk4, bklen, pardeg, slots,
                                                                                 par_nbit, par_ncell);
        } else {
            e = cudaFuncSetAttribute(hf_encode_kernel<kHfSublen>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return (int)e;
            hf_encode_kernel<kHfSublen><<<grid, 32 * kHfEncWarps, smem, s>>>(in, n, bk4, bklen, pardeg, slots,
                                                                             par_nbit, par_ncell);
        }
    }
    ScanSrc sc{};
    sc.base = par_ncell;
    sc.n = pardeg;
    int rc = launch_scan_u32(sc, par_entry, tiles, ncell_total, s);
    if (rc) return rc;
    const uint32_t rb = 256 + 2 * bklen;
    cudaError_t eh = launch_dependent(hf_header_kernel, 1, 1024, 0, s, out, bklen, sublen, pardeg, n, d_revbook, rb,
                                      (const uint32_t*)ncell_total, out_size);
    if (eh != cudaSuccess) return (int)eh;
    uint32_t* out_nbit = reinterpret_cast<uint32_t*>(out + 128 + rb);
    uint32_t* bitstream = reinterpret_cast<uint32_t*>(out + 128 + rb + 8 * (size_t)pardeg);
    const uint32_t groups = (pardeg + kHfCatGroup - 1) / kHfCatGroup;
    TraceScope tc(s, "hf_concat");
    return (int)launch_dependent(hf_concat_kernel, (groups + kHfCatWarps - 1) / kHfCatWarps, 32 * kHfCatWarps, 0, s,
                                 (const uint32_t*)slots, (const uint32_t*)par_nbit, (const uint32_t*)par_ncell,
                                 (const uint32_t*)par_entry, pardeg, sublen, out_nbit, out_nbit + pardeg, bitstream,
                                 ctrl, reinterpret_cast<uint32_t*>(out + 24));
}

int launch_hf_decode(const uint8_t* blob, uint64_t blob_bytes, uint64_t n, uint32_t bklen,
                     uint16_t* out, uint32_t* err, cudaStream_t s) {
    const uint32_t pardeg = (uint32_t)((n - 1) / kHfSublen + 1);  // the larger partition count
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // two CTAs per SM, fewer for small inputs; warps take partitions from a counter
    const uint32_t grid = max(1u, min(2u * (uint32_t)sms, (pardeg + kHfDecWarps - 1) / kHfDecWarps));
    cudaError_t e = cudaFuncSetAttribute(hf_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHfDecSmem);
    if (e != cudaSuccess) return (int)e;
    TraceScope ts(s, "hf_decode");
    hf_decode_kernel<<<grid, kHfDecThreads, kHfDecSmem, s>>>(blob, blob_bytes, n, bklen, out, err);
    return (int)cudaGetLastError();
}

}  // namespace fzb
