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
// (hf_hl.cc:69-103).  Here one kernel serves both modes: a thread takes
// sublen/256 consecutive symbols and, when they fit one 32-bit word (every
// code at most 32/(sublen/256) bits), packs them and ORs the word into the
// cells; otherwise each code is ORed in on its own.
#include "fzb_kernels.cuh"

namespace fzb {

constexpr int kHfThreads = 256;  // sublen / 256 symbols per thread per partition
constexpr uint32_t kHfSmemBook = 16384;  // books up to this size are staged in shared memory

// Privatised histogram: each CTA counts into shared memory, then merges.
// Symbols >= bklen are skipped (histogram.cu:47-51).
__global__ void __launch_bounds__(512) hf_histogram_kernel(const uint16_t* __restrict__ in, uint64_t n,
                                                           uint32_t bklen, uint32_t* __restrict__ freq) {
    extern __shared__ uint32_t hs[];
    const bool priv = bklen <= kHfSmemBook;  // larger books count straight into freq
    uint32_t* h = priv ? hs : freq;
    if (priv)
        for (uint32_t i = threadIdx.x; i < bklen; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const bool vec = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    const uint64_t nv = vec ? n / 8 : 0;
    const uint4* in8 = reinterpret_cast<const uint4*>(in);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
        const uint4 v = __ldg(in8 + i);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t a = w[k] & 0xffffu, b = w[k] >> 16;
            if (a < bklen) atomicAdd(&h[a], 1u);
            if (b < bklen) atomicAdd(&h[b], 1u);
        }
    }
    for (uint64_t i = 8 * nv + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t a = in[i];
        if (a < bklen) atomicAdd(&h[a], 1u);
    }
    if (!priv) return;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < bklen; i += blockDim.x)
        if (h[i]) atomicAdd(&freq[i], h[i]);
}

// One CTA per partition group (persistent loop): look up the codewords,
// prefix-sum their lengths, OR the codes into shared-memory cells at their
// bit offsets, write the cells to the partition's slot.
template <int SUB>
__global__ void __launch_bounds__(kHfThreads) hf_encode_kernel(const uint16_t* __restrict__ in, uint64_t n,
                                                               const uint32_t* __restrict__ bk4, uint32_t bklen,
                                                               uint32_t pardeg, uint32_t* __restrict__ slots,
                                                               uint32_t* __restrict__ par_nbit,
                                                               uint32_t* __restrict__ par_ncell) {
    constexpr int PER = SUB / kHfThreads;  // 3 (coarse) or 4 (fine)
    extern __shared__ uint32_t sm[];
    const bool staged = bklen <= kHfSmemBook;
    uint32_t* cells = sm;                             // SUB words
    const uint32_t* book = staged ? sm + SUB : bk4;   // bklen words when staged
    __shared__ uint32_t ws[16];
    uint32_t lmax = 0;
    if (staged)
        for (uint32_t i = threadIdx.x; i < bklen; i += blockDim.x) {
            const uint32_t v = bk4[i];
            sm[SUB + i] = v;
            lmax = max(lmax, v >> 27);
        }
    // the PER codes of a thread fit one word when every code is short enough
    const bool packed = staged && !__syncthreads_or(lmax * PER > 32);
    const int t = threadIdx.x;
    for (uint32_t p = blockIdx.x; p < pardeg; p += gridDim.x) {
        for (int i = t; i < SUB; i += kHfThreads) cells[i] = 0;
        __syncthreads();
        const uint64_t base = (uint64_t)p * SUB + PER * t;
        uint32_t w[PER], bits = 0;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            w[k] = 0;
            if (base + k < n) {
                const uint32_t sym = in[base + k];
                w[k] = (sym < bklen) ? book[sym] : 0u;
            }
            bits += w[k] >> 27;
        }
        uint32_t total;
        uint32_t off = block_excl_scan(bits, ws, &total);
        if (packed) {  // MSB-first concatenation of the thread's codes in one word
            uint32_t acc = 0, nb = 0;
#pragma unroll
            for (int k = 0; k < PER; k++) {
                const uint32_t len = w[k] >> 27;
                if (len) acc |= (w[k] & 0x7ffffffu) << (32 - nb - len);
                nb += len;
            }
            if (nb) {
                const uint32_t cell = off >> 5, pos = off & 31;
                atomicOr(&cells[cell], acc >> pos);
                if (pos + nb > 32) atomicOr(&cells[cell + 1], acc << (32 - pos));
            }
        } else {
#pragma unroll
            for (int k = 0; k < PER; k++) {
                const uint32_t len = w[k] >> 27, code = w[k] & 0x7ffffffu;
                if (len) {
                    const uint32_t cell = off >> 5, pos = off & 31;  // pos = bits already used in the cell
                    if (pos + len <= 32) {
                        atomicOr(&cells[cell], code << (32 - pos - len));
                    } else {
                        const uint32_t spill = pos + len - 32;  // bits going to the next cell
                        atomicOr(&cells[cell], code >> spill);
                        atomicOr(&cells[cell + 1], code << (32 - spill));
                    }
                }
                off += len;
            }
        }
        __syncthreads();
        const uint32_t ncell = (total + 31) / 32;
        uint32_t* dst = slots + (size_t)p * SUB;
        for (uint32_t i = t; i < ncell; i += kHfThreads) dst[i] = cells[i];
        if (t == 0) {
            par_nbit[p] = total;
            par_ncell[p] = ncell;
        }
        __syncthreads();
    }
}

// Header + revbook + par_nbit + par_entry (one CTA of 1024 threads).
// par_entry must already hold the exclusive scan of par_ncell and
// *ncell_total its sum.
__global__ void __launch_bounds__(1024) hf_header_kernel(uint8_t* __restrict__ out, uint32_t bklen,
                                                         uint32_t sublen, uint32_t pardeg, uint64_t n,
                                                         const uint8_t* __restrict__ revbook,
                                                         uint32_t revbook_bytes,
                                                         const uint32_t* __restrict__ par_nbit,
                                                         const uint32_t* __restrict__ par_entry,
                                                         const uint32_t* __restrict__ ncell_total,
                                                         unsigned long long* __restrict__ out_size) {
    __shared__ unsigned long long part[32];
    const uint32_t e1 = 128, e2 = e1 + revbook_bytes, e3 = e2 + 4 * pardeg, e4 = e3 + 4 * pardeg;
    unsigned long long nbit = 0;
    for (uint32_t p = threadIdx.x; p < pardeg; p += blockDim.x) {
        const uint32_t v = par_nbit[p];
        nbit += v;
        reinterpret_cast<uint32_t*>(out + e2)[p] = v;
        reinterpret_cast<uint32_t*>(out + e3)[p] = par_entry[p];
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) nbit += __shfl_xor_sync(0xffffffffu, nbit, d);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = nbit;
    for (uint32_t i = threadIdx.x; i < revbook_bytes; i += blockDim.x) out[e1 + i] = revbook[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long tot = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) tot += part[i];
        const uint64_t ncell = *ncell_total;
        uint32_t* h32 = reinterpret_cast<uint32_t*>(out);
        for (int i = 0; i < 32; i++) h32[i] = 0;
        h32[0] = bklen & 0xffffu;
        h32[1] = sublen;
        h32[2] = pardeg;
        uint64_t* h64 = reinterpret_cast<uint64_t*>(out + 16);
        h64[0] = n;
        h64[1] = tot;
        h64[2] = ncell;
        uint32_t* ent = reinterpret_cast<uint32_t*>(out + 40);
        ent[0] = 0;
        ent[1] = e1;
        ent[2] = e2;
        ent[3] = e3;
        ent[4] = e4;
        ent[5] = e4 + (uint32_t)(4 * ncell);
        *out_size = e4 + 4 * ncell;
    }
}

// Partition cells from their slots to the bitstream (u32 aligned).
__global__ void hf_concat_kernel(const uint32_t* __restrict__ slots, const uint32_t* __restrict__ par_ncell,
                                 const uint32_t* __restrict__ par_entry, uint32_t pardeg, uint32_t sublen,
                                 uint32_t* __restrict__ bitstream) {
    for (uint32_t p = blockIdx.x; p < pardeg; p += gridDim.x) {
        const uint32_t nc = par_ncell[p], e = par_entry[p];
        for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) bitstream[e + i] = slots[(size_t)p * sublen + i];
    }
}

// Canonical decode (hf_kernels.cu:258-312), one thread per partition as in
// the reference, reorganised for throughput:
//   * a per-CTA lookup table indexed by the next kHfLutBits bits gives
//     (symbol, length) of every code of at most kHfLutBits bits in one probe;
//     longer codes continue the canonical first[] walk from length
//     kHfLutBits + 1.  The table is built with the walk's own comparisons
//     (the shortest l with v >= first[l]), so both give identical symbols and
//     error flags;
//   * the partition's cells stream through registers in 16-byte blocks, the
//     next block loaded while the current one is consumed, so a load has some
//     fifty symbols of work to hide behind;
//   * symbols are decoded 16 at a time into eight registers and leave as two
//     16-byte stores.
// A well-formed partition decodes its want symbols in exactly nbit bits;
// anything else (a length past 31, a table index past the book, a bit count
// that does not match) raises kErrMalformed.
constexpr int kHfLutBits = 12;
constexpr int kHfDecThreads = 256;

struct HfBlockReader {
    const uint8_t* blk;  // next 16-byte block to load
    const uint8_t* end;  // one past the last blob byte
    uint32_t c0, c1, c2, c3, inq;
    uint4 nxt;

    __device__ __forceinline__ uint4 load(const uint8_t* p) const {
        if (p + 16 <= end) return __ldg(reinterpret_cast<const uint4*>(p));
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint8_t* q = p + 4 * i;
            w[i] = q + 4 <= end ? __ldg(reinterpret_cast<const uint32_t*>(q)) : 0u;
        }
        return make_uint4(w[0], w[1], w[2], w[3]);
    }
    // starts at cell address a (4-byte aligned)
    __device__ __forceinline__ void start(const uint8_t* a, const uint8_t* e) {
        end = e;
        const uint8_t* b0 = reinterpret_cast<const uint8_t*>(reinterpret_cast<uintptr_t>(a) & ~(uintptr_t)15);
        const uint4 cur = load(b0);
        nxt = load(b0 + 16);
        blk = b0 + 32;
        c0 = cur.x;
        c1 = cur.y;
        c2 = cur.z;
        c3 = cur.w;
        inq = 4;
        for (uint32_t k = (uint32_t)((reinterpret_cast<uintptr_t>(a) & 15) >> 2); k; k--) take();
    }
    __device__ __forceinline__ uint32_t take() {
        const uint32_t v = c0;
        c0 = c1;
        c1 = c2;
        c2 = c3;
        if (--inq == 0) {
            c0 = nxt.x;
            c1 = nxt.y;
            c2 = nxt.z;
            c3 = nxt.w;
            inq = 4;
            nxt = load(blk);
            blk += 16;
        }
        return v;
    }
};

__global__ void __launch_bounds__(kHfDecThreads, 4)
    hf_decode_kernel(const uint8_t* __restrict__ blob, uint64_t blob_bytes, uint64_t n, uint32_t bklen_expect,
                     uint16_t* __restrict__ out, uint32_t* err) {
    __shared__ uint32_t s_first[32];
    __shared__ int s_entry[32];
    __shared__ uint32_t lut[1u << kHfLutBits];

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
    const uint16_t* keys = reinterpret_cast<const uint16_t*>(blob + e1 + 256);
    __syncthreads();
    // lookup table: entry = symbol << 16 | bad << 8 | length (length 0: a longer code)
    for (uint32_t u = threadIdx.x; u < (1u << kHfLutBits); u += blockDim.x) {
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
        lut[u] = e;
    }
    __syncthreads();

    const uint32_t* nbits_g = reinterpret_cast<const uint32_t*>(blob + e2);
    const uint32_t* entry_g = reinterpret_cast<const uint32_t*>(blob + e3);
    const uint8_t* cells = blob + e4;
    const uint8_t* blob_end = blob + e5;
    const uint32_t ncells = (e5 - e4) / 4;
    const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    bool bad = false;

    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pardeg; p += gridDim.x * blockDim.x) {
        const uint32_t nbit = __ldg(nbits_g + p);
        const uint32_t c0 = __ldg(entry_g + p);
        const uint64_t o0 = (uint64_t)p * sublen;
        const uint32_t want = (uint32_t)min((uint64_t)sublen, n - o0);
        if (nbit == 0 && want > 0 && s_entry[1] == 1) {
            // a single symbol in the book gets a zero-length code: every
            // output is that symbol (the reference leaves this case undecoded)
            const uint16_t k0 = __ldg(keys);
            for (uint32_t i = 0; i < want; i++) out[o0 + i] = k0;
            continue;
        }
        HfBlockReader rd;
        rd.start(cells + 4 * (size_t)min(c0, ncells), blob_end);
        uint64_t buf = 0;  // the next `have` bits, MSB-aligned
        int have = 0;
        uint32_t used = 0, eacc = 0;
        while (have <= 32) {
            buf |= (uint64_t)rd.take() << (32 - have);
            have += 32;
        }
        auto next_symbol = [&]() -> uint32_t {
            if (have <= 32) {
                buf |= (uint64_t)rd.take() << (32 - have);
                have += 32;
            }
            const uint32_t e = lut[(uint32_t)(buf >> (64 - kHfLutBits))];
            int l = (int)(e & 0xffu);
            uint32_t sym;
            if (l != 0) {
                eacc |= e;
                sym = e >> 16;
            } else {  // longer than the table: continue the walk
                l = kHfLutBits + 1;
                uint32_t v = (uint32_t)(buf >> (64 - l));
                while (l < 32 && v < s_first[l]) {
                    l++;
                    v = (uint32_t)(buf >> (64 - l));
                }
                if (l >= 32) {  // no code: flag it and move on by a full word
                    bad = true;
                    l = 31;
                    sym = 0;
                } else {
                    const int k = s_entry[l] + (int)v - (int)s_first[l];
                    const bool kin = k >= 0 && k < (int)bklen;
                    bad |= !kin;
                    sym = kin ? __ldg(keys + k) : 0u;
                }
            }
            buf <<= l;
            have -= l;
            used += l;
            return sym;
        };
        uint32_t i = 0;
        if (aligned) {
            for (; i + 16 <= want; i += 16) {
                uint32_t w[8];
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const uint32_t sym = next_symbol();
                    if (j & 1) w[j >> 1] |= sym << 16;
                    else w[j >> 1] = sym;
                }
                uint4* d4 = reinterpret_cast<uint4*>(out + o0 + i);
                d4[0] = make_uint4(w[0], w[1], w[2], w[3]);
                d4[1] = make_uint4(w[4], w[5], w[6], w[7]);
            }
        }
        for (; i < want; i++) out[o0 + i] = (uint16_t)next_symbol();
        bad |= ((eacc >> 8) & 1u) != 0 || used != nbit;
    }
    if (bad) atomicOr(err, kErrMalformed);
}

int launch_hf_histogram(const uint16_t* in, uint64_t n, uint32_t bklen, uint32_t* freq, int sms,
                        cudaStream_t s) {
    cudaMemsetAsync(freq, 0, 4 * (size_t)bklen, s);
    const int smem = bklen <= kHfSmemBook ? 4 * (int)bklen : 0;
    cudaFuncSetAttribute(hf_histogram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    hf_histogram_kernel<<<2 * sms, 512, smem, s>>>(in, n, bklen, freq);
    return (int)cudaGetLastError();
}

int launch_hf_encode(const uint16_t* in, uint64_t n, const uint32_t* bk4, uint32_t bklen, uint32_t sublen,
                     const uint8_t* d_revbook, uint8_t* out, unsigned long long* out_size,
                     uint32_t* slots, uint32_t* par_nbit, uint32_t* par_ncell, uint32_t* par_entry,
                     uint32_t* tiles, uint32_t* ncell_total, int sms, cudaStream_t s) {
    if (sublen != (uint32_t)kHfSublen && sublen != (uint32_t)kHfSublenFine) return (int)cudaErrorInvalidValue;
    const uint32_t pardeg = (uint32_t)((n - 1) / sublen + 1);
    const int smem = 4 * ((int)sublen + (bklen <= kHfSmemBook ? (int)bklen : 0));
    const unsigned grid = (unsigned)min((uint64_t)pardeg, (uint64_t)8 * sms);
    cudaError_t e;
    if (sublen == (uint32_t)kHfSublenFine) {
        e = cudaFuncSetAttribute(hf_encode_kernel<kHfSublenFine>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return (int)e;
        hf_encode_kernel<kHfSublenFine><<<grid, kHfThreads, smem, s>>>(in, n, bk4, bklen, pardeg, slots, par_nbit,
                                                                       par_ncell);
    } else {
        e = cudaFuncSetAttribute(hf_encode_kernel<kHfSublen>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return (int)e;
        hf_encode_kernel<kHfSublen><<<grid, kHfThreads, smem, s>>>(in, n, bk4, bklen, pardeg, slots, par_nbit,
                                                                   par_ncell);
    }
    ScanSrc sc{};
    sc.base = par_ncell;
    sc.n = pardeg;
    int rc = launch_scan_u32(sc, par_entry, tiles, ncell_total, s);
    if (rc) return rc;
    const uint32_t rb = 256 + 2 * bklen;
    hf_header_kernel<<<1, 1024, 0, s>>>(out, bklen, sublen, pardeg, n, d_revbook, rb, par_nbit, par_entry,
                                       ncell_total, out_size);
    uint32_t* bitstream = reinterpret_cast<uint32_t*>(out + 128 + rb + 8 * (size_t)pardeg);
    hf_concat_kernel<<<(unsigned)min((uint64_t)pardeg, (uint64_t)8 * sms), 128, 0, s>>>(
        slots, par_ncell, par_entry, pardeg, sublen, bitstream);
    return (int)cudaGetLastError();
}

int launch_hf_decode(const uint8_t* blob, uint64_t blob_bytes, uint64_t n, uint32_t bklen,
                     uint16_t* out, uint32_t* err, cudaStream_t s) {
    const uint32_t pardeg = (uint32_t)((n - 1) / kHfSublen + 1);  // the larger partition count
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t need = (pardeg + kHfDecThreads - 1) / kHfDecThreads;
    const uint32_t grid = min(need, (uint32_t)sms * 4u);
    TraceScope ts(s, "hf_decode");
    hf_decode_kernel<<<grid ? grid : 1u, kHfDecThreads, 0, s>>>(blob, blob_bytes, n, bklen, out, err);
    return (int)cudaGetLastError();
}

}  // namespace fzb
