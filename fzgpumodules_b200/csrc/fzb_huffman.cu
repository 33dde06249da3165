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

// One thread per partition: canonical decode (hf_kernels.cu:267-298) with a
// 64-bit bit reader; 16 symbols are gathered before each 32-byte store.  The
// partition length comes from the blob header (768 coarse, 1024 fine); the
// grid covers the coarse partition count, the larger of the two.
__global__ void __launch_bounds__(128) hf_decode_kernel(const uint8_t* __restrict__ blob, uint64_t blob_bytes,
                                                        uint64_t n, uint32_t bklen_expect,
                                                        uint16_t* __restrict__ out, uint32_t* err) {
    __shared__ int s_first[32], s_entry[32];
    extern __shared__ uint16_t s_keys[];
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
        s_first[threadIdx.x] = rb[threadIdx.x];
        s_entry[threadIdx.x] = rb[32 + threadIdx.x];
    }
    const uint16_t* keys = reinterpret_cast<const uint16_t*>(blob + e1 + 256);
    for (uint32_t i = threadIdx.x; i < bklen; i += blockDim.x) s_keys[i] = keys[i];
    __syncthreads();
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pardeg) return;
    const uint32_t nbit = reinterpret_cast<const uint32_t*>(blob + e2)[p];
    const uint32_t entry = reinterpret_cast<const uint32_t*>(blob + e3)[p];
    const uint32_t ncells = (e5 - e4) / 4;
    const uint32_t* bits = reinterpret_cast<const uint32_t*>(blob + e4) + entry;
    const uint32_t avail = entry < ncells ? ncells - entry : 0u;
    const uint64_t o0 = (uint64_t)p * sublen;
    const uint32_t want = (uint32_t)min((uint64_t)sublen, n - o0);
    // bit reader: buf holds the next `have` bits MSB-aligned
    uint64_t buf = 0;
    int have = 0;
    uint32_t cell = 0;
    auto refill = [&]() {
        while (have <= 32) {
            const uint32_t v = cell < avail ? __ldg(bits + cell) : 0u;
            buf |= (uint64_t)v << (32 - have);
            have += 32;
            cell++;
        }
    };
    const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    uint32_t used = 0, outn = 0;
    uint16_t stage[16];
    bool bad = false;
    if (nbit == 0 && want > 0 && s_entry[1] == 1) {
        // a single symbol in the book gets a zero-length code: every output
        // is that symbol (the reference leaves this case undecoded)
        for (uint32_t i = 0; i < want; i++) out[o0 + i] = s_keys[0];
        return;
    }
    while (used < nbit && outn < want) {
        refill();
        uint32_t v = (uint32_t)(buf >> 63);
        int l = 1;
        while (l < 32 && v < (uint32_t)s_first[l]) {
            v = (uint32_t)(buf >> (63 - l));
            l++;
        }
        if (l >= 32) {
            bad = true;
            break;
        }
        buf <<= l;
        have -= l;
        used += l;
        const int k = s_entry[l] + (int)v - s_first[l];
        const bool kin = k >= 0 && k < (int)bklen;
        bad |= !kin;
        stage[outn & 15] = kin ? s_keys[k] : (uint16_t)0;
        outn++;
        if ((outn & 15) == 0 && aligned) {
            uint4* d4 = reinterpret_cast<uint4*>(out + o0 + outn - 16);
            uint32_t w[8];
#pragma unroll
            for (int j = 0; j < 8; j++) w[j] = (uint32_t)stage[2 * j] | ((uint32_t)stage[2 * j + 1] << 16);
            d4[0] = make_uint4(w[0], w[1], w[2], w[3]);
            d4[1] = make_uint4(w[4], w[5], w[6], w[7]);
        } else if (!aligned) {
            out[o0 + outn - 1] = stage[(outn - 1) & 15];
        }
    }
    if (aligned)
        for (uint32_t i = outn & ~15u; i < outn; i++) out[o0 + i] = stage[i & 15];
    if (bad || outn != want || used != nbit) atomicOr(err, kErrMalformed);
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
    const int smem = 2 * (int)bklen + 16;
    cudaFuncSetAttribute(hf_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    hf_decode_kernel<<<(pardeg + 127) / 128, 128, smem, s>>>(blob, blob_bytes, n, bklen, out, err);
    return (int)cudaGetLastError();
}

}  // namespace fzb
