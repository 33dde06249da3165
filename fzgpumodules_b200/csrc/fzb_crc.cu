// fzb_crc.cu -- CRC-32 (IEEE 802.3: reflected polynomial 0xEDB88320, initial
// register and final inversion 0xFFFFFFFF), the FZM data checksum
// (src/pipeline/compressor_io.cpp:25-52, used at :218-228), over device memory.
//
// The CRC of a message with a zero register and no final inversion ("raw
// CRC") is linear in the message bits:
//     raw(A || B) = shift(raw(A), |B|) xor raw(B),
// where shift(r, n) feeds n zero bytes through the register; and zero bytes in
// front of a message leave its raw CRC unchanged.  So:
//   * each thread computes the raw CRC of one 512-byte segment with a
//     slice-by-8 table held in shared memory;
//   * a CTA folds its 256 segments pairwise in 8 rounds (round k shifts the
//     left half by 512 * 2^k bytes) into the raw CRC of a 128 KiB block; the
//     tail block (under 128 KiB) is read zero-prefixed;
//   * one or two further rounds of 1024-wide folds combine the blocks (the list
//     is zero-padded at the front to a multiple of 1024 entries);
//   * the standard CRC is ~(shift(raw(full blocks), |tail|) xor raw(tail)
//     xor shift(0xFFFFFFFF, |M|)).
// shift by n bytes is a 32x32 GF(2) operator, stored as its 32 column words
// (column i = image of bit i); the host builds the operators by repeated
// squaring of the one-zero-bit operator.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/fzb.h"
#include "fzb_kernels.cuh"

namespace fzb {
namespace {

constexpr uint32_t kPoly = 0xEDB88320u;
constexpr int kSegBytes = 512;
constexpr int kSegs = 256;                                  // threads (segments) per block
constexpr uint64_t kBlockBytes = (uint64_t)kSegBytes * kSegs;  // 128 KiB
constexpr int kFold = 1024;                                 // entries per combine CTA

struct CrcOp {
    uint32_t c[32];
};
struct CrcOps8 {
    CrcOp op[8];
};
struct CrcOps10 {
    CrcOp op[10];
};

// ---------------------------------------------------------------- host side

uint32_t op_apply(const CrcOp& a, uint32_t v) {
    uint32_t r = 0;
    for (int i = 0; v; i++, v >>= 1)
        if (v & 1u) r ^= a.c[i];
    return r;
}

CrcOp op_compose(const CrcOp& a, const CrcOp& b) {  // a after b
    CrcOp r;
    for (int i = 0; i < 32; i++) r.c[i] = op_apply(a, b.c[i]);
    return r;
}

CrcOp op_identity() {
    CrcOp r;
    for (int i = 0; i < 32; i++) r.c[i] = 1u << i;
    return r;
}

// Feeding n zero bytes through the register: the composition of the
// operators for 2^j zero bytes over the set bits j of n (a table built once).
CrcOp op_zero_bytes(uint64_t n) {
    struct Pow {
        CrcOp op[64];
    };
    static const Pow pw = [] {
        Pow t;
        CrcOp p;  // one zero bit: bit 0 leaves as the polynomial, the rest shift down
        p.c[0] = kPoly;
        for (int i = 1; i < 32; i++) p.c[i] = 1u << (i - 1);
        for (int k = 0; k < 3; k++) p = op_compose(p, p);  // one zero byte
        for (int j = 0; j < 64; j++) {
            t.op[j] = p;
            p = op_compose(p, p);
        }
        return t;
    }();
    CrcOp r = op_identity();
    for (int j = 0; n; j++, n >>= 1)
        if (n & 1u) r = op_compose(pw.op[j], r);
    return r;
}

// ---------------------------------------------------------------- device side

__device__ __forceinline__ uint32_t dev_apply(const uint32_t* op, uint32_t v) {
    uint32_t r = 0;
    while (v) {
        const int i = __ffs(v) - 1;
        r ^= op[i];
        v &= v - 1;
    }
    return r;
}

// Slice-by-8 tables: t[k][b] = raw CRC of byte b followed by k zero bytes.
__device__ void build_tables(uint32_t (*t)[256]) {
    for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x) {
        uint32_t c = b;
        for (int k = 0; k < 8; k++) c = (c >> 1) ^ ((c & 1u) ? kPoly : 0u);
        t[0][b] = c;
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x) {
        uint32_t c = t[0][b];
        for (int k = 1; k < 8; k++) {
            c = (c >> 8) ^ t[0][c & 0xffu];
            t[k][b] = c;
        }
    }
    __syncthreads();
}

// Raw CRC of the 128 KiB block b (the tail block zero-prefixed), one CTA of
// kSegs threads.
__global__ void __launch_bounds__(kSegs) crc_block_kernel(const uint8_t* __restrict__ p, uint64_t bytes,
                                                          uint64_t nfull, const __grid_constant__ CrcOps8 ops,
                                                          uint32_t* __restrict__ block_crc) {
    __shared__ uint32_t tab[8][256];
    __shared__ uint32_t sop[8][32];
    __shared__ uint32_t part[kSegs];
    build_tables(tab);
    for (int i = threadIdx.x; i < 8 * 32; i += kSegs) sop[i / 32][i % 32] = ops.op[i / 32].c[i % 32];
    const uint64_t b = blockIdx.x, t = threadIdx.x;
    uint32_t crc = 0;
    if (b < nfull) {
        const uint8_t* s = p + b * kBlockBytes + t * kSegBytes;
        if ((reinterpret_cast<uintptr_t>(p) & 7u) == 0) {
            const uint2* s8 = reinterpret_cast<const uint2*>(s);
#pragma unroll 4
            for (int i = 0; i < kSegBytes / 8; i++) {
                const uint2 w = __ldg(s8 + i);
                const uint32_t lo = crc ^ w.x, hi = w.y;
                crc = tab[7][lo & 0xffu] ^ tab[6][(lo >> 8) & 0xffu] ^ tab[5][(lo >> 16) & 0xffu] ^ tab[4][lo >> 24] ^
                      tab[3][hi & 0xffu] ^ tab[2][(hi >> 8) & 0xffu] ^ tab[1][(hi >> 16) & 0xffu] ^ tab[0][hi >> 24];
            }
        } else {
            for (int i = 0; i < kSegBytes; i++) crc = (crc >> 8) ^ tab[0][(crc ^ __ldg(s + i)) & 0xffu];
        }
    } else {  // tail: bytes [nfull * 128K, bytes) as the end of a zero-prefixed block
        const uint64_t start = nfull * kBlockBytes;
        const uint64_t tail = bytes - start;
        const uint64_t vbase = kBlockBytes - tail;  // virtual offset of the first real byte
        for (uint64_t v = t * kSegBytes; v < (t + 1) * kSegBytes; v++)
            if (v >= vbase) crc = (crc >> 8) ^ tab[0][(crc ^ p[start + (v - vbase)]) & 0xffu];
    }
    part[t] = crc;
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < 8; k++) {
        const uint32_t half = 1u << k;
        if ((t & (2 * half - 1)) == 0) part[t] = dev_apply(sop[k], part[t]) ^ part[t + half];
        __syncthreads();
    }
    if (t == 0) block_crc[b] = part[0];
}

// Folds kFold consecutive raw CRCs of equal-length units (the list zero-padded
// at the front by `pad` entries) into one.
__global__ void __launch_bounds__(kFold) crc_fold_kernel(const uint32_t* __restrict__ in, uint64_t count,
                                                         uint64_t pad, const __grid_constant__ CrcOps10 ops,
                                                         uint32_t* __restrict__ out) {
    __shared__ uint32_t sop[10][32];
    __shared__ uint32_t part[kFold];
    for (int i = threadIdx.x; i < 10 * 32; i += kFold) sop[i / 32][i % 32] = ops.op[i / 32].c[i % 32];
    const uint64_t j = (uint64_t)blockIdx.x * kFold + threadIdx.x;  // position in the padded list
    part[threadIdx.x] = (j >= pad && j - pad < count) ? in[j - pad] : 0u;
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < 10; k++) {
        const uint32_t half = 1u << k, t = threadIdx.x;
        if ((t & (2 * half - 1)) == 0) part[t] = dev_apply(sop[k], part[t]) ^ part[t + half];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = part[0];
}

// total = ~(shift(full, |tail|) ^ tail ^ shift(~0, |M|))
__global__ void crc_finish_kernel(const uint32_t* __restrict__ full, const uint32_t* __restrict__ tail,
                                  const __grid_constant__ CrcOp op_tail, const __grid_constant__ CrcOp op_all,
                                  uint32_t* __restrict__ out) {
    if (threadIdx.x != 0) return;
    const uint32_t f = full ? *full : 0u, tl = tail ? *tail : 0u;
    uint32_t r = 0, v = f;
    for (int i = 0; v; i++, v >>= 1)
        if (v & 1u) r ^= op_tail.c[i];
    r ^= tl;
    uint32_t s = 0;
    v = 0xFFFFFFFFu;
    for (int i = 0; i < 32; i++, v >>= 1)
        if (v & 1u) s ^= op_all.c[i];
    *out = ~(r ^ s);
}

uint64_t crc_nfull(uint64_t bytes) { return bytes / kBlockBytes; }
uint64_t crc_groups(uint64_t n) { return (n + kFold - 1) / kFold; }

}  // namespace
}  // namespace fzb

using namespace fzb;

extern "C" {

size_t fzb_crc32_workspace_bytes(uint64_t bytes) {
    const uint64_t nfull = crc_nfull(bytes), g1 = crc_groups(nfull);
    return 256 + 4 * (nfull + 1) + 256 + 4 * (g1 + 1) + 256 + 256;
}

int fzb_crc32(const void* d_data, uint64_t bytes, uint32_t* d_crc, void* d_work, size_t work_bytes, void* stream) {
    if ((!d_data && bytes) || !d_crc) return FZB_E_INVALID;
    const uint64_t nfull = crc_nfull(bytes), tail = bytes - nfull * kBlockBytes, g1 = crc_groups(nfull);
    if (g1 > (uint64_t)kFold) return FZB_E_INVALID;  // more than 128 GiB
    if (!d_work || work_bytes < fzb_crc32_workspace_bytes(bytes)) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(d_work);
    uint32_t* block_crc = reinterpret_cast<uint32_t*>(w);
    uint32_t* lvl1 = reinterpret_cast<uint32_t*>(w + ((4 * (nfull + 1) + 255) & ~255ull) + 256);
    uint32_t* lvl2 = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(lvl1) + ((4 * (g1 + 1) + 255) & ~255ull) + 256);
    const uint8_t* p = static_cast<const uint8_t*>(d_data);

    // fixed operators, built once: shifts by 512 * 2^k, 128 KiB * 2^k and 128 MiB * 2^k bytes
    static const CrcOps8 seg = [] {
        CrcOps8 o;
        for (int k = 0; k < 8; k++) o.op[k] = op_zero_bytes((uint64_t)kSegBytes << k);
        return o;
    }();
    static const CrcOps10 o1 = [] {
        CrcOps10 o;
        for (int k = 0; k < 10; k++) o.op[k] = op_zero_bytes(kBlockBytes << k);
        return o;
    }();
    static const CrcOps10 o2 = [] {
        CrcOps10 o;
        for (int k = 0; k < 10; k++) o.op[k] = op_zero_bytes((kBlockBytes * kFold) << k);
        return o;
    }();
    const uint64_t nblk = nfull + (tail ? 1 : 0);
    if (nblk) {
        crc_block_kernel<<<(unsigned)nblk, kSegs, 0, s>>>(p, bytes, nfull, seg, block_crc);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    }
    const uint32_t* full = nullptr;
    if (nfull) {
        const uint64_t pad1 = g1 * kFold - nfull;
        crc_fold_kernel<<<(unsigned)g1, kFold, 0, s>>>(block_crc, nfull, pad1, o1, lvl1);
        if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
        full = lvl1;
        if (g1 > 1) {
            crc_fold_kernel<<<1, kFold, 0, s>>>(lvl1, g1, kFold - g1, o2, lvl2);
            if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
            full = lvl2;
        }
    }
    const CrcOp op_tail = op_zero_bytes(tail), op_all = op_zero_bytes(bytes);
    crc_finish_kernel<<<1, 32, 0, s>>>(full, tail ? block_crc + nfull : nullptr, op_tail, op_all, d_crc);
    return cudaGetLastError() == cudaSuccess ? FZB_OK : FZB_E_CUDA;
}

}  // extern "C"
