// fzb_inverse.cu -- inverse kernels: RZE stream prepass, chunk decode
// (bytes, or bytes + Bitshuffle inverse -> codes), outlier scatter, the
// exact tile-local Lorenzo inverse (1-D/2-D/3-D) and the fused single-pass
// RZE -> Bitshuffle -> 3-D Lorenzo inverse.
#include "fzb_kernels.cuh"

namespace fzb {

// ---------------------------------------------------------------------------
// Payload offsets of every chunk of an RZE stream (rze_stage.cu:871-900),
// one CTA of 1024 threads.  in_off[n] receives the end of the payload.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) rze_prepass_kernel(const uint8_t* __restrict__ rze,
                                                           uint64_t rze_bytes, uint32_t n_expect,
                                                           uint32_t orig_expect,
                                                           unsigned long long* __restrict__ in_off,
                                                           uint32_t* err) {
    // Tiles of kAsmTile size words: loads issued in batches of eight per
    // thread (all in flight at once) into shared memory, 16 per thread, a
    // warp-shuffle block scan, coalesced writes, carry between tiles.
    constexpr uint32_t kTile = kAsmTile, kPer = kTile / 1024;
    extern __shared__ uint32_t sz[];  // pad32-indexed
    __shared__ uint32_t wsum[32], s_tile;
    const uint32_t* h = reinterpret_cast<const uint32_t*>(rze);
    const uint32_t n = n_expect, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint64_t hdr = 8ull + 4ull * n;
    if (h[0] != orig_expect || h[1] != n_expect || hdr > rze_bytes) {
        // inconsistent header: flag it and point every chunk at the header end
        if (t == 0) atomicOr(err, kErrMalformed);
        for (uint32_t i = t; i <= n; i += blockDim.x) in_off[i] = rze_bytes + 1;
        return;
    }
    unsigned long long carry = hdr;
    for (uint32_t t0 = 0; t0 < n; t0 += kTile) {
        const uint32_t cnt = min(kTile, n - t0);
        for (uint32_t j0 = 0; j0 < kPer; j0 += 8) {
            uint32_t v[8];
#pragma unroll
            for (uint32_t j = 0; j < 8; j++) {
                const uint32_t i = t + 1024u * (j0 + j);
                v[j] = i < cnt ? h[2 + t0 + i] : 0u;
            }
#pragma unroll
            for (uint32_t j = 0; j < 8; j++) sz[pad32(t + 1024u * (j0 + j))] = v[j] & 0x7fffffffu;
        }
        __syncthreads();
        uint32_t l = 0;
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++) l += sz[pad32(kPer * t + j)];
        uint32_t inc = l;  // tile sums fit 32 bits: 4096 chunks of at most 16 KiB
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
            const uint32_t v = sz[pad32(kPer * t + j)];
            sz[pad32(kPer * t + j)] = r;
            r += v;
        }
        if (t == 1023) s_tile = r;
        __syncthreads();
        for (uint32_t i = t; i < cnt; i += 1024) in_off[t0 + i] = carry + sz[pad32(i)];
        carry += s_tile;
        __syncthreads();
    }
    if (t == 0) {
        in_off[n] = carry;
        if (carry > rze_bytes) atomicOr(err, kErrMalformed);
    }
    asm volatile("griddepcontrol.launch_dependents;");  // outlier_ranges_kernel may start
}

// The same offsets for up to kTiledScanMax chunks, a CTA per 1024 chunks,
// each summing the size words before its tile itself (no CTA waits for
// another); the last CTA writes the end offset and checks it.
__global__ void __launch_bounds__(1024) rze_prepass_tiles_kernel(const uint8_t* __restrict__ rze,
                                                                 uint64_t rze_bytes, uint32_t n_expect,
                                                                 uint32_t orig_expect,
                                                                 unsigned long long* __restrict__ in_off,
                                                                 uint32_t* err) {
    __shared__ uint32_t ws[66];
    const uint32_t* h = reinterpret_cast<const uint32_t*>(rze);
    const uint32_t n = n_expect, t = threadIdx.x, base = blockIdx.x * 1024u;
    const bool last = base + 1024u >= n;
    const uint64_t hdr = 8ull + 4ull * n;
    if (h[0] != orig_expect || h[1] != n_expect || hdr > rze_bytes) {
        // inconsistent header: flag it and point every chunk at the header end
        if (blockIdx.x == 0 && t == 0) atomicOr(err, kErrMalformed);
        if (base + t < n) in_off[base + t] = rze_bytes + 1;
        if (last && t == 0) in_off[n] = rze_bytes + 1;
        asm volatile("griddepcontrol.launch_dependents;");
        return;
    }
    uint32_t sp = 0;  // bytes of the chunks before the tile (at most 2^30)
    for (uint32_t i = t; i < base; i += 1024u) sp += h[2 + i] & 0x7fffffffu;
    const uint32_t i = base + t;
    const uint32_t v = i < n ? h[2 + i] & 0x7fffffffu : 0u;
    uint32_t e0, e1, SP, S1, ev, e2, TV, T2;
    block_scan2_1024(sp, 0u, e0, e1, SP, S1, ws);
    block_scan2_1024(v, 0u, ev, e2, TV, T2, ws);
    if (i < n) in_off[i] = hdr + SP + ev;
    if (last && t == 0) {
        const unsigned long long end = hdr + (unsigned long long)SP + TV;
        in_off[n] = end;
        if (end > rze_bytes) atomicOr(err, kErrMalformed);
    }
    asm volatile("griddepcontrol.launch_dependents;");  // outlier_ranges_kernel may start
}

int launch_rze_prepass(const uint8_t* rze, uint64_t rze_bytes, uint32_t n_expect, uint32_t orig_expect,
                       unsigned long long* in_off, uint32_t* err, cudaStream_t s) {
    if (n_expect <= kTiledScanMax && !(flags_env() & 16)) {
        rze_prepass_tiles_kernel<<<(n_expect + 1023u) / 1024u + (n_expect == 0), 1024, 0, s>>>(
            rze, rze_bytes, n_expect, orig_expect, in_off, err);
        return (int)cudaGetLastError();
    }
    const int smem = (int)((kAsmTile + kAsmTile / 32) * sizeof(uint32_t));
    static SmemAttr attr;
    const cudaError_t e = ensure_dyn_smem(attr, (const void*)rze_prepass_kernel, smem);
    if (e != cudaSuccess) return (int)e;
    rze_prepass_kernel<<<1, 1024, smem, s>>>(rze, rze_bytes, n_expect, orig_expect, in_off, err);
    return (int)cudaGetLastError();
}

// Per-chunk start of the (index-sorted) outlier list, and a sortedness check.
__global__ void outlier_ranges_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                                      uint32_t cap, uint32_t n_chunks, uint32_t* __restrict__ ostart,
                                      uint32_t* err) {
    const uint32_t nout = min(*count, cap);
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t c = tid; c <= n_chunks; c += stride) {
        const uint64_t key = (uint64_t)c * kChunkCodes;
        uint32_t lo = 0, hi = nout;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if ((uint64_t)idx[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        ostart[c] = lo;
    }
    for (uint32_t i = tid; i + 1 < nout; i += stride)
        if (idx[i] >= idx[i + 1]) atomicOr(err, kErrUnsorted);
    // launched as a programmatic dependent of the RZE prepass, whose offsets it
    // does not read: the fused inverse may start launching now, and this grid
    // ends only after the prepass has, so the inverse's wait covers both
    asm volatile("griddepcontrol.launch_dependents;");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ RzeDecSmem dec_smem(uint8_t* base, uint32_t* ws) {
    RzeDecSmem sm;
    sm.C = base;
    sm.S = reinterpret_cast<uint32_t*>(base + kChunkBytes + 16);
    sm.bm1 = reinterpret_cast<uint32_t*>(base + 2 * kChunkBytes + 16);
    sm.bm2 = base + 2 * kChunkBytes + 16 + 2048;
    sm.bm3 = base + 2 * kChunkBytes + 16 + 2048 + 256;
    sm.ws = ws;
    return sm;
}
constexpr int kDecSmemBytes = 2 * kChunkBytes + 16 + 2048 + 256 + 32;

__device__ __forceinline__ bool chunk_src(const InvArgs& a, uint32_t c, uint32_t* e, int* osz,
                                          const uint8_t** src) {
    *e = reinterpret_cast<const uint32_t*>(a.rze + 8)[c];
    *osz = (c + 1 < a.n_chunks) ? kChunkBytes : (int)(a.orig_bytes - c * (uint32_t)kChunkBytes);
    const uint64_t off = a.in_off[c];
    *src = a.rze + off;
    return off + (*e & 0x7fffffffu) <= a.rze_bytes;
}

// Plain RZE decode: one CTA per chunk, decoded bytes to bytes_out.
__global__ void __launch_bounds__(kThreads) rze_decode_kernel(InvArgs a) {
    extern __shared__ float4 smraw[];
    __shared__ uint32_t s_ws[16];
    const uint32_t c = blockIdx.x;
    const RzeDecSmem sm = dec_smem(reinterpret_cast<uint8_t*>(smraw), s_ws);
    uint32_t e;
    int osz;
    const uint8_t* src;
    if (!chunk_src(a, c, &e, &osz, &src)) {
        if (threadIdx.x == 0) atomicOr(a.err, kErrMalformed);
        e = 2;  // decode as zeros
    }
    rze_decode_chunk(src, e, osz, sm, a.err);
    uint8_t* dst = a.bytes_out + (size_t)c * kChunkBytes;
    if (osz == kChunkBytes && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        const uint4* s4 = reinterpret_cast<const uint4*>(sm.S);
        uint4* d4 = reinterpret_cast<uint4*>(dst);
        for (int i = threadIdx.x; i < kChunkBytes / 16; i += kThreads) d4[i] = s4[i];
    } else {
        const uint8_t* Sb = reinterpret_cast<const uint8_t*>(sm.S);
        for (int i = threadIdx.x; i < osz; i += kThreads) dst[i] = Sb[i];
    }
}

// RZE decode + Bitshuffle inverse: one CTA per chunk (grid-stride over the
// chunks when the grid is smaller), codes to a.codes.
__global__ void __launch_bounds__(kThreads) rze_decode_codes_kernel(InvArgs a) {
    extern __shared__ float4 smraw[];
    __shared__ uint32_t s_ws[16];
    if (inv_gated_off(a)) return;
    const RzeDecSmem sm = dec_smem(reinterpret_cast<uint8_t*>(smraw), s_ws);
    for (uint32_t c = blockIdx.x; c < a.n_chunks; c += gridDim.x) {
        uint32_t e;
        int osz;
        const uint8_t* src;
        if (!chunk_src(a, c, &e, &osz, &src)) {
            if (threadIdx.x == 0) atomicOr(a.err, kErrMalformed);
            e = 2;
        }
        rze_decode_chunk(src, e, osz, sm, a.err);
        const int t = threadIdx.x;
        if (osz == kChunkBytes) {
            uint32_t x[16];
            if (a.shuffled) {
#pragma unroll
                for (int b = 0; b < 16; b++) x[b] = sm.S[(15 - b) * 256 + t];
                transpose16x2(x);
                uint32_t rw[16];
#pragma unroll
                for (int l = 0; l < 8; l++) rw[l] = __byte_perm(x[2 * l], x[2 * l + 1], 0x5410);
#pragma unroll
                for (int l = 8; l < 16; l++) rw[l] = __byte_perm(x[2 * l - 16], x[2 * l - 15], 0x7632);
#pragma unroll
                for (int l = 0; l < 16; l++) x[l] = rw[l];
            } else {
#pragma unroll
                for (int l = 0; l < 16; l++) x[l] = sm.S[16 * t + l];
            }
            uint4* d4 = reinterpret_cast<uint4*>(a.codes + (size_t)c * kChunkCodes + 32 * t);
#pragma unroll
            for (int v = 0; v < 4; v++) d4[v] = make_uint4(x[4 * v], x[4 * v + 1], x[4 * v + 2], x[4 * v + 3]);
        } else {  // tail block: stored unshuffled
            uint8_t* dst = reinterpret_cast<uint8_t*>(a.codes) + (size_t)c * kChunkBytes;
            const uint8_t* Sb = reinterpret_cast<const uint8_t*>(sm.S);
            for (int i = t; i < osz; i += kThreads) dst[i] = Sb[i];
        }
        __syncthreads();  // the shared buffers are reused by the next chunk
    }
}

// Zeroes the n_total outputs (the exact path's first step; a kernel rather
// than a memset so that it can be gated).
__global__ void zero_out_kernel(InvArgs a) {
    if (inv_gated_off(a)) return;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total;
         i += (uint64_t)gridDim.x * blockDim.x)
        a.out[i] = 0.0f;
}

// out must be zeroed; writes each outlier's delta at its index
// (lorenzo_quant_kernels.cuh:23-40).
__global__ void scatter_outliers_kernel(InvArgs a) {
    if (inv_gated_off(a)) return;
    const uint32_t n = min(*a.out_count, a.cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = a.out_idx[i];
        if (k < a.n_total) a.out[k] = a.out_err[i];
    }
}

// ---------------------------------------------------------------------------
// Exact inverse kernels.  `out` holds the scattered outlier deltas (zero
// elsewhere); each tile is reconstructed with the reference's add tree.
// ---------------------------------------------------------------------------

// 1-D: 1024-element tiles, thread t owns elements 4t..4t+3
// (lorenzo_quant.cu:155-244).
__global__ void __launch_bounds__(256) lq_inverse_1d_kernel(InvArgs a) {
    __shared__ float s_w[8];
    if (inv_gated_off(a)) return;
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const float ebx2 = inv_ebx2(a);
    const bool zz = a.zigzag != 0;
    const uint32_t ntiles = (a.nfield + 1023) / 1024;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t base = (uint64_t)tile * 1024 + 4 * t;
        float v[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint64_t g = base + i;
            v[i] = (g < a.nfield) ? __fadd_rn(a.out[g], decode_code(a.codes[g], zz)) : 0.0f;
        }
#pragma unroll
        for (int i = 1; i < 4; i++) v[i] = __fadd_rn(v[i], v[i - 1]);
        float ts = v[3];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            float n = __shfl_up_sync(0xffffffffu, ts, d);
            if ((int)lane >= d) ts = __fadd_rn(ts, n);
        }
        float pre = __shfl_up_sync(0xffffffffu, ts, 1);
        if (lane > 0) {
#pragma unroll
            for (int i = 0; i < 4; i++) v[i] = __fadd_rn(v[i], pre);
        }
        if (lane == 31) s_w[warp] = v[3];
        __syncthreads();
        if (warp > 0) {
            float w[8];
#pragma unroll
            for (int i = 0; i < 8; i++) w[i] = s_w[i];
            // Hillis-Steele over the 8 warp totals, evaluated as a tree
#pragma unroll
            for (int d = 1; d < 8; d <<= 1)
#pragma unroll
                for (int i = 7; i >= 1; i--)
                    if (i >= d) w[i] = __fadd_rn(w[i], w[i - d]);
            const float add = w[warp - 1];
#pragma unroll
            for (int i = 0; i < 4; i++) v[i] = __fadd_rn(v[i], add);
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint64_t g = base + i;
            if (g < a.nfield) a.out[g] = __fmul_rn(v[i], ebx2);
        }
        __syncthreads();  // s_w is rewritten by the next tile
    }
}

// 2-D: 32x32 tiles, 128 threads = 32 x 4 row groups of 8
// (lorenzo_quant_nd.cu:112-190).
__global__ void __launch_bounds__(128) lq_inverse_2d_kernel(InvArgs a) {
    __shared__ float s_tot[4][32];
    if (inv_gated_off(a)) return;
    const uint32_t lx = threadIdx.x & 31, wy = threadIdx.x >> 5;
    const float ebx2 = inv_ebx2(a);
    const bool zz = a.zigzag != 0;
    const uint32_t tx = (a.nx + 31) / 32, ntiles = tx * ((a.ny + 31) / 32);
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t gx = (tile % tx) * 32 + lx, gy0 = (tile / tx) * 32 + wy * 8;
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint32_t gy = gy0 + i;
            v[i] = 0.0f;
            if (gx < a.nx && gy < a.ny) {
                const uint64_t g = (uint64_t)gy * a.nx + gx;
                v[i] = __fadd_rn(a.out[g], decode_code(a.codes[g], zz));
            }
        }
#pragma unroll
        for (int i = 1; i < 8; i++) v[i] = __fadd_rn(v[i], v[i - 1]);
        s_tot[wy][lx] = v[7];
        __syncthreads();
        if (wy > 0) {
            const float t0 = s_tot[0][lx];
            const float t1 = __fadd_rn(t0, s_tot[1][lx]);
            const float add = (wy == 1) ? t0 : (wy == 2) ? t1 : __fadd_rn(t1, s_tot[2][lx]);
#pragma unroll
            for (int i = 0; i < 8; i++) v[i] = __fadd_rn(v[i], add);
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                float n = __shfl_up_sync(0xffffffffu, v[i], d);
                if ((int)lx >= d) v[i] = __fadd_rn(v[i], n);
            }
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint32_t gy = gy0 + i;
            if (gx < a.nx && gy < a.ny) a.out[(uint64_t)gy * a.nx + gx] = __fmul_rn(v[i], ebx2);
        }
        __syncthreads();  // s_tot is rewritten by the next tile
    }
}

// 3-D: one CTA per 32x8x8 brick (four 8x8x8 tiles); thread (x, z) scans y
// sequentially and x as an 8-lane Hillis-Steele, then thread (x, y) runs the
// z Hillis-Steele tree in registers (lorenzo_quant_nd.cu:281-364).
__global__ void __launch_bounds__(256) lq_inverse_3d_kernel(InvArgs a) {
    __shared__ float V[8][8][33];  // [z][y][x]
    if (inv_gated_off(a)) return;
    const uint32_t lx = threadIdx.x & 31, lz = threadIdx.x >> 5;
    const float ebx2 = inv_ebx2(a);
    const bool zz = a.zigzag != 0;
    const uint32_t tx = (a.nx + 31) / 32, ty = (a.ny + 7) / 8, ntiles = tx * ty * ((a.nz + 7) / 8);
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t bx = tile % tx, by = (tile / tx) % ty, bz = tile / (tx * ty);
        const uint32_t gx = bx * 32 + lx, gy0 = by * 8, gz = bz * 8 + lz;
        float v[8];
#pragma unroll
        for (int y = 0; y < 8; y++) {
            v[y] = 0.0f;
            const uint32_t gy = gy0 + y;
            if (gx < a.nx && gy < a.ny && gz < a.nz) {
                const uint64_t g = ((uint64_t)gz * a.ny + gy) * a.nx + gx;
                v[y] = __fadd_rn(a.out[g], decode_code(a.codes[g], zz));
            }
        }
#pragma unroll
        for (int y = 1; y < 8; y++) v[y] = __fadd_rn(v[y], v[y - 1]);
        const uint32_t sx = lx & 7;
#pragma unroll
        for (int y = 0; y < 8; y++) {
#pragma unroll
            for (int d = 1; d < 8; d <<= 1) {
                float n = __shfl_up_sync(0xffffffffu, v[y], d, 8);
                if ((int)sx >= d) v[y] = __fadd_rn(v[y], n);
            }
            V[lz][y][lx] = v[y];
        }
        __syncthreads();
        const uint32_t ly = lz;  // second phase: thread (x, y)
        float w[8];
#pragma unroll
        for (int z = 0; z < 8; z++) w[z] = V[z][ly][lx];
#pragma unroll
        for (int d = 1; d < 8; d <<= 1)
#pragma unroll
            for (int z = 7; z >= 1; z--)
                if (z >= d) w[z] = __fadd_rn(w[z], w[z - d]);
        const uint32_t gy = gy0 + ly;
#pragma unroll
        for (int z = 0; z < 8; z++) {
            const uint32_t gzz = bz * 8 + z;
            if (gx < a.nx && gy < a.ny && gzz < a.nz)
                a.out[((uint64_t)gzz * a.ny + gy) * a.nx + gx] = __fmul_rn(w[z], ebx2);
        }
        __syncthreads();  // V is rewritten by the next brick
    }
}

// ---------------------------------------------------------------------------
// Fused inverse for 3-D fields whose 8192-code chunks are R = 8192/nx whole
// rows (nx a power of two <= 1024, ny % R == 0).  One CTA per (R-row slab,
// 8-plane z tile): for each plane it decodes the chunk (RZE -> Bitshuffle
// inverse -> deltas in shared memory), adds that chunk's outliers, scans y
// and x with the reference's add tree and keeps a running z sum in
// registers.  The running z sum equals the reference's z Hillis-Steele tree
// whenever every partial sum is an integer below 2^24; the kernel checks
// max|v| < 2^21 (8 planes) and otherwise raises kErrInexact so the host
// reruns the exact kernels.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int dswz(int m) {  // swizzled float index in D
    const int g = m >> 2;
    return ((g ^ ((g >> 3) & 7)) << 2) | (m & 3);
}

__global__ void __launch_bounds__(kThreads, 2) fused_inverse_3d_kernel(InvArgs a) {
    extern __shared__ float4 smraw[];
    __shared__ uint32_t s_ws[16];
    if (*a.err & (kErrUnsorted | kErrMalformed)) return;
    uint8_t* base = reinterpret_cast<uint8_t*>(smraw);
    const RzeDecSmem sm = dec_smem(base, s_ws);
    float* D = reinterpret_cast<float*>(base + kDecSmemBytes);
    const int t = threadIdx.x;
    const uint32_t nx = a.nx, R = kChunkCodes / nx, slabs = a.ny / R;
    const uint32_t s = blockIdx.x, zt = blockIdx.y;
    const uint32_t lognx = 31 - __clz(nx);
    const float ebx2 = inv_ebx2(a);
    const bool zz = a.zigzag != 0;
    const uint32_t nout = min(*a.out_count, a.cap);

    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int y = 0; y < 8; y++) acc[i][y] = 0.0f;
    // Exactness guard: every partial sum of the z tree (reference) and of the
    // running sum (here) adds at most 8 plane values, so max|v| < 2^21 keeps
    // all of them integers below 2^24.
    float vmax = 0.0f;

    const uint32_t z0 = zt * 8, z1 = min(z0 + 8, a.nz);
    for (uint32_t z = z0; z < z1; z++) {
        const uint32_t c = z * slabs + s;
        uint32_t e;
        int osz;
        const uint8_t* src;
        if (!chunk_src(a, c, &e, &osz, &src)) {
            if (t == 0) atomicOr(a.err, kErrMalformed);
            e = 2;
        }
        rze_decode_chunk(src, e, osz, sm, a.err);
        {   // Bitshuffle inverse + code -> float delta, thread t owns codes 32t..
            uint32_t x[16];
#pragma unroll
            for (int b = 0; b < 16; b++) x[b] = sm.S[(15 - b) * 256 + t];
            transpose16x2(x);
            float4* D4 = reinterpret_cast<float4*>(D);
#pragma unroll
            for (int g = 0; g < 8; g++) {
                float f[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int E = 4 * g + k;
                    f[k] = decode_code((x[E & 15] >> (16 * (E >> 4))) & 0xffffu, zz);
                }
                const int gi = 8 * t + g;
                D4[gi ^ ((gi >> 3) & 7)] = make_float4(f[0], f[1], f[2], f[3]);
            }
        }
        __syncthreads();
        {   // outliers of this chunk: delta = outlier + decoded code
            const uint32_t o0 = a.ostart[c], o1 = min(a.ostart[c + 1], nout);
            const uint32_t kbase = c * (uint32_t)kChunkCodes;
            for (uint32_t i = o0 + t; i < o1; i += kThreads) {
                const int m = (int)(a.out_idx[i] - kbase);
                D[dswz(m)] = __fadd_rn(a.out_err[i], D[dswz(m)]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t col = t + kThreads * i;
            const uint32_t ytile = col >> lognx, x = col & (nx - 1);
            float v[8];
#pragma unroll
            for (int y = 0; y < 8; y++) v[y] = D[dswz((int)(((ytile * 8 + y) << lognx) + x))];
#pragma unroll
            for (int y = 1; y < 8; y++) v[y] = __fadd_rn(v[y], v[y - 1]);
            const uint32_t tx = x & 7;
#pragma unroll
            for (int y = 0; y < 8; y++) {
#pragma unroll
                for (int d = 1; d < 8; d <<= 1) {
                    float n = __shfl_up_sync(0xffffffffu, v[y], d, 8);
                    if ((int)tx >= d) v[y] = __fadd_rn(v[y], n);
                }
                acc[i][y] = __fadd_rn(acc[i][y], v[y]);
                vmax = fmaxf(vmax, fabsf(v[y]));
                const uint32_t gy = s * R + ytile * 8 + y;
                a.out[((uint64_t)z * a.ny + gy) * nx + x] = __fmul_rn(acc[i][y], ebx2);
            }
        }
        __syncthreads();
    }
    const bool inexact = !(vmax < 2097152.0f);  // NaN counts as inexact
    if (__any_sync(0xffffffffu, inexact) && (t & 31) == 0) atomicOr(a.err, kErrInexact);
}

}  // namespace fzb
