// fzb_coders.cu -- RLE and Bitpack coders plus the device-wide scan they use.
//
// RLE wire format (modules/coders/rle/rle.h:22, rle.cu:119-148):
//   [u32 runs][values T x runs, padded to 4 bytes with zeros][u32 lengths x runs]
// Bitpack (modules/coders/bitpack/bitpack_stage.cu:30-124): low nbits of each
// element, LSB-first inside a byte for nbits < 8, little-endian bytes above.
//
// Every element count that is only known on the device (run count, detected
// nbits) is read by the kernels from device memory, so no call needs a host
// round trip.
#include "fzb_kernels.cuh"

namespace fzb {

constexpr int kScanTile = 4096;  // elements per CTA in the scan passes

// ---------------------------------------------------------------------------
// Exclusive scan of u32 values, three passes: tile sums, one-CTA scan of
// the tile sums, tile scan + offset.  The source is either a plain array
// (count given or read from *cptr) or the run-length array of an RLE stream
// (count and position read from the stream's header on the device).
// ---------------------------------------------------------------------------
__device__ __forceinline__ const uint32_t* scan_src(const ScanSrc& a, uint32_t* cnt) {
    if (a.rle) {
        const uint32_t R = *reinterpret_cast<const uint32_t*>(a.rle);
        *cnt = min(R, a.n);
        return reinterpret_cast<const uint32_t*>(a.rle + 4 + ((R * (uint32_t)a.elem + 3u) & ~3u));
    }
    *cnt = a.cptr ? min(*a.cptr, a.n) : a.n;
    return a.base;
}

__global__ void __launch_bounds__(256) scan_tile_sums(ScanSrc a, uint32_t* __restrict__ tsum) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    uint32_t cnt;
    const uint32_t* in = scan_src(a, &cnt);
    const uint32_t b = blockIdx.x * kScanTile;
    uint32_t s = 0;
    for (uint32_t i = b + threadIdx.x; i < min(cnt, b + kScanTile); i += 256) s += in[i];
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    __shared__ uint32_t w[8];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < 8; i++) t += w[i];
        tsum[blockIdx.x] = t;
    }
    asm volatile("griddepcontrol.launch_dependents;");
}

__global__ void __launch_bounds__(1024) scan_tile_offsets(uint32_t* __restrict__ tsum, uint32_t ntiles,
                                                          uint32_t* __restrict__ total) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __shared__ uint32_t s[1024];
    const uint32_t t = threadIdx.x, per = (ntiles + 1023) / 1024;
    const uint32_t b = t * per, e = min(ntiles, b + per);
    uint32_t sum = 0;
    for (uint32_t i = b; i < e; i++) sum += tsum[i];
    s[t] = sum;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        uint32_t v = (t >= (unsigned)d) ? s[t - d] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    uint32_t run = s[t] - sum;
    for (uint32_t i = b; i < e; i++) {
        const uint32_t v = tsum[i];
        tsum[i] = run;
        run += v;
    }
    if (t == 1023 && total) *total = s[1023];
    asm volatile("griddepcontrol.launch_dependents;");
}

__global__ void __launch_bounds__(256) scan_tile_apply(ScanSrc a, const uint32_t* __restrict__ toff,
                                                       uint32_t* __restrict__ out) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __shared__ uint32_t ws[16];
    uint32_t cnt;
    const uint32_t* in = scan_src(a, &cnt);
    const uint32_t b = blockIdx.x * kScanTile + threadIdx.x * 16;
    uint32_t v[16], s = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        v[i] = (b + i < cnt) ? in[b + i] : 0u;
        s += v[i];
    }
    uint32_t tot;
    uint32_t run = toff[blockIdx.x] + block_excl_scan(s, ws, &tot);
#pragma unroll
    for (int i = 0; i < 16; i++) {
        if (b + i < cnt) out[b + i] = run;
        run += v[i];
    }
    asm volatile("griddepcontrol.launch_dependents;");
}

int launch_scan_u32(const ScanSrc& a, uint32_t* out, uint32_t* tile_scratch, uint32_t* total,
                    cudaStream_t s) {
    if (a.n == 0) return 0;
    const uint32_t ntiles = (a.n + kScanTile - 1) / kScanTile;
    // programmatic dependents: each waits for the kernel before it (the
    // first for whatever produced the input) and lets the next one launch
    cudaError_t e = launch_dependent(scan_tile_sums, ntiles, 256, 0, s, a, tile_scratch);
    if (e == cudaSuccess) e = launch_dependent(scan_tile_offsets, 1, 1024, 0, s, tile_scratch, ntiles, total);
    if (e == cudaSuccess) e = launch_dependent(scan_tile_apply, ntiles, 256, 0, s, a, (const uint32_t*)tile_scratch, out);
    return (int)e;
}

// ---------------------------------------------------------------------------
// RLE encode.  Pass 1 counts run starts per 4096-element tile; the tile
// counts are scanned; pass 2 writes each run's value and start position;
// pass 3 turns start positions into lengths.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ uint32_t run_starts16(const T* __restrict__ in, uint32_t n, uint32_t b,
                                                 T (&v)[16]) {
    uint32_t m = 0;
    T prev = (b > 0 && b - 1 < n) ? in[b - 1] : T(0);
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t k = b + i;
        v[i] = (k < n) ? in[k] : T(0);
        const bool start = (k < n) && (k == 0 || v[i] != prev);
        m |= (start ? 1u : 0u) << i;
        prev = v[i];
    }
    return m;
}

template <typename T>
__global__ void __launch_bounds__(256) rle_count_kernel(const T* __restrict__ in, uint32_t n,
                                                        uint32_t* __restrict__ tcnt) {
    T v[16];
    const uint32_t m = run_starts16(in, n, blockIdx.x * kScanTile + threadIdx.x * 16, v);
    uint32_t s = __popc(m);
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    __shared__ uint32_t w[8];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < 8; i++) t += w[i];
        tcnt[blockIdx.x] = t;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) rle_emit_kernel(const T* __restrict__ in, uint32_t n,
                                                       const uint32_t* __restrict__ toff,
                                                       uint8_t* __restrict__ out,
                                                       uint32_t* __restrict__ starts) {
    __shared__ uint32_t ws[16];
    T v[16];
    const uint32_t b = blockIdx.x * kScanTile + threadIdx.x * 16;
    const uint32_t m = run_starts16(in, n, b, v);
    uint32_t tot;
    uint32_t r = toff[blockIdx.x] + block_excl_scan(__popc(m), ws, &tot);
    T* values = reinterpret_cast<T*>(out + 4);
#pragma unroll
    for (int i = 0; i < 16; i++) {
        if ((m >> i) & 1u) {
            values[r] = v[i];
            starts[r] = b + i;
            r++;
        }
    }
}

template <typename T>
__global__ void rle_lengths_kernel(const uint32_t* __restrict__ runs_ptr, uint32_t n,
                                   const uint32_t* __restrict__ starts, uint8_t* __restrict__ out,
                                   unsigned long long* __restrict__ out_size) {
    const uint32_t R = *runs_ptr;
    const uint32_t vbytes = R * (uint32_t)sizeof(T), valigned = (vbytes + 3u) & ~3u;
    uint32_t* lens = reinterpret_cast<uint32_t*>(out + 4 + valigned);
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t r = tid; r < R; r += gridDim.x * blockDim.x)
        lens[r] = ((r + 1 < R) ? starts[r + 1] : n) - starts[r];
    if (tid == 0) {
        reinterpret_cast<uint32_t*>(out)[0] = R;
        for (uint32_t i = vbytes; i < valigned; i++) out[4 + i] = 0;
        *out_size = 4ull + valigned + 4ull * R;
    }
}

// ---------------------------------------------------------------------------
// RLE decode: scan of run lengths, then each 4096-element output tile
// gathers the runs that overlap it into shared memory and every element
// binary-searches its run there.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) rle_expand_kernel(const uint8_t* __restrict__ in,
                                                         const uint32_t* __restrict__ offs,
                                                         uint32_t n, T* __restrict__ out,
                                                         uint32_t* err) {
    __shared__ uint32_t s_off[kScanTile + 2];
    __shared__ T s_val[kScanTile + 2];
    __shared__ uint32_t s_nr;
    const uint32_t R = min(*reinterpret_cast<const uint32_t*>(in), n);
    const T* values = reinterpret_cast<const T*>(in + 4);
    const uint32_t t0 = blockIdx.x * kScanTile, t1 = min(n, t0 + kScanTile);
    if (t0 >= n) return;
    if (R == 0) {
        if (threadIdx.x == 0) atomicOr(err, kErrMalformed);
        for (uint32_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) out[i] = T(0);
        return;
    }
    // last run whose start <= t0: every round all threads probe evenly spaced
    // starts and the count of starts <= t0 narrows the range about blockDim-fold
    uint32_t lo = 0, hi = R;
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + blockDim.x - 1) / blockDim.x;
        const uint32_t p = lo + threadIdx.x * step;
        const int c = __syncthreads_count(p < hi && offs[p] <= t0);
        const uint32_t nlo = lo + (uint32_t)(c > 0 ? c - 1 : 0) * step;
        hi = min(hi, lo + (uint32_t)(c > 0 ? c : 1) * step);
        lo = nlo;
    }
    // the runs overlapping the tile: at most kScanTile + 1 from r0
    const uint32_t r0 = lo, win = min(R - r0, (uint32_t)kScanTile + 1);
    if (threadIdx.x == 0) s_nr = 0;
    __syncthreads();
    uint32_t mine = 0;
    for (uint32_t i = threadIdx.x; i < win; i += blockDim.x) {
        const uint32_t o = offs[r0 + i];
        s_off[i] = o;
        s_val[i] = values[r0 + i];
        mine += o < t1;
    }
    if (mine) atomicAdd(&s_nr, mine);
    __syncthreads();
    const uint32_t nr = s_nr;
    if (nr == 0) {
        for (uint32_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) out[i] = T(0);
        return;
    }
    for (uint32_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
        uint32_t lo = 0, hi = nr;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_off[mid] <= i) lo = mid;
            else hi = mid;
        }
        out[i] = s_val[lo];
    }
}

template <typename T>
int launch_rle_encode_t(const T* in, uint32_t n, uint8_t* out, unsigned long long* out_size,
                        uint32_t* tcnt, uint32_t* starts, uint32_t* runs_total, cudaStream_t s) {
    const uint32_t ntiles = (n + kScanTile - 1) / kScanTile;
    rle_count_kernel<T><<<ntiles, 256, 0, s>>>(in, n, tcnt);
    scan_tile_offsets<<<1, 1024, 0, s>>>(tcnt, ntiles, runs_total);
    rle_emit_kernel<T><<<ntiles, 256, 0, s>>>(in, n, tcnt, out, starts);
    rle_lengths_kernel<T><<<592, 256, 0, s>>>(runs_total, n, starts, out, out_size);
    return (int)cudaGetLastError();
}

int launch_rle_encode(const void* in, uint32_t n, int elem, uint8_t* out, unsigned long long* out_size,
                      uint32_t* tcnt, uint32_t* starts, uint32_t* runs_total, cudaStream_t s) {
    if (elem == 1) return launch_rle_encode_t<uint8_t>((const uint8_t*)in, n, out, out_size, tcnt, starts, runs_total, s);
    if (elem == 2) return launch_rle_encode_t<uint16_t>((const uint16_t*)in, n, out, out_size, tcnt, starts, runs_total, s);
    return launch_rle_encode_t<uint32_t>((const uint32_t*)in, n, out, out_size, tcnt, starts, runs_total, s);
}

// Run lengths must add up to n; checked on the device.
__global__ void rle_check_total(const uint32_t* __restrict__ total, uint32_t n, uint32_t* err) {
    if (*total != n) atomicOr(err, kErrMalformed);
}

int launch_rle_decode(const uint8_t* in, uint32_t n, int elem, void* out, uint32_t* offs,
                      uint32_t* tile_scratch, uint32_t* total, uint32_t* err, cudaStream_t s) {
    ScanSrc a{};
    a.rle = in;
    a.elem = elem;
    a.n = n;  // at most n runs in a valid stream
    int rc = launch_scan_u32(a, offs, tile_scratch, total, s);
    if (rc) return rc;
    rle_check_total<<<1, 1, 0, s>>>(total, n, err);
    const uint32_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (elem == 1) rle_expand_kernel<uint8_t><<<ntiles, 256, 0, s>>>(in, offs, n, (uint8_t*)out, err);
    else if (elem == 2) rle_expand_kernel<uint16_t><<<ntiles, 256, 0, s>>>(in, offs, n, (uint16_t*)out, err);
    else rle_expand_kernel<uint32_t><<<ntiles, 256, 0, s>>>(in, offs, n, (uint32_t*)out, err);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Bitpack.  nbits may be detected on the device (smallest power of two whose
// range holds the maximum, bitpack_stage.cu:118-124); kernels read it there.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) bitpack_max_kernel(const T* __restrict__ in, uint64_t n,
                                                          uint32_t* __restrict__ pmax,
                                                          unsigned int* __restrict__ done,
                                                          uint8_t* __restrict__ nbits_out) {
    uint32_t m = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, (uint32_t)in[i]);
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, d));
    __shared__ uint32_t w[8];
    __shared__ bool s_last;
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < 8; i++) m = max(m, w[i]);
        pmax[blockIdx.x] = m;
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    m = 0;
    for (unsigned b = 0; b < gridDim.x; b++) m = max(m, __ldcg(pmax + b));
    const int full = 8 * (int)sizeof(T);
    int nb = full;
    for (int b = 1; b < full; b *= 2)
        if ((uint64_t)m < (1ull << b)) { nb = b; break; }
    *nbits_out = (uint8_t)nb;
    *done = 0;
}

template <typename T>
__global__ void bitpack_encode_kernel(const T* __restrict__ in, uint64_t n,
                                      const uint8_t* __restrict__ nbits_ptr, uint8_t* __restrict__ out,
                                      unsigned long long* __restrict__ out_size) {
    const int nbits = *nbits_ptr;
    const uint64_t nout = (n * (uint64_t)nbits + 7) / 8;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    if (tid == 0 && out_size) *out_size = nout;
    if (nbits < 8) {
        const int per = 8 / nbits;
        const uint32_t mask = (1u << nbits) - 1u;
        for (uint64_t b = tid; b < nout; b += stride) {
            uint32_t packed = 0;
            for (int k = 0; k < per; k++) {
                const uint64_t e = b * per + k;
                if (e < n) packed |= ((uint32_t)in[e] & mask) << (k * nbits);
            }
            out[b] = (uint8_t)packed;
        }
    } else {
        const int bytes = nbits / 8;
        for (uint64_t i = tid; i < n; i += stride) {
            uint32_t v = (uint32_t)in[i];
            if (nbits < 32) v &= (1u << nbits) - 1u;
            for (int b = 0; b < bytes; b++) out[i * bytes + b] = (uint8_t)(v >> (8 * b));
        }
    }
}

template <typename T>
__global__ void bitpack_decode_kernel(const uint8_t* __restrict__ in, uint64_t n, int nbits,
                                      T* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t v = 0;
        if (nbits < 8) {
            const int per = 8 / nbits;
            v = (in[i / per] >> ((i % per) * nbits)) & ((1u << nbits) - 1u);
        } else {
            for (int b = 0; b < nbits / 8; b++) v |= (uint32_t)in[i * (nbits / 8) + b] << (8 * b);
        }
        out[i] = (T)v;
    }
}

__global__ void set_byte_kernel(uint8_t* p, uint8_t v) { *p = v; }

int launch_bitpack_encode(const void* in, uint64_t n, int elem, int nbits, uint8_t* nbits_dev,
                          uint8_t* out, unsigned long long* out_size, uint32_t* pmax,
                          unsigned int* done, cudaStream_t s) {
    const unsigned grid = 1184;
    if (nbits == 0) {
        if (elem == 1) bitpack_max_kernel<uint8_t><<<grid, 256, 0, s>>>((const uint8_t*)in, n, pmax, done, nbits_dev);
        else if (elem == 2) bitpack_max_kernel<uint16_t><<<grid, 256, 0, s>>>((const uint16_t*)in, n, pmax, done, nbits_dev);
        else bitpack_max_kernel<uint32_t><<<grid, 256, 0, s>>>((const uint32_t*)in, n, pmax, done, nbits_dev);
    } else {
        set_byte_kernel<<<1, 1, 0, s>>>(nbits_dev, (uint8_t)nbits);
    }
    if (elem == 1) bitpack_encode_kernel<uint8_t><<<grid, 256, 0, s>>>((const uint8_t*)in, n, nbits_dev, out, out_size);
    else if (elem == 2) bitpack_encode_kernel<uint16_t><<<grid, 256, 0, s>>>((const uint16_t*)in, n, nbits_dev, out, out_size);
    else bitpack_encode_kernel<uint32_t><<<grid, 256, 0, s>>>((const uint32_t*)in, n, nbits_dev, out, out_size);
    return (int)cudaGetLastError();
}

int launch_bitpack_decode(const uint8_t* in, uint64_t n, int elem, int nbits, void* out, cudaStream_t s) {
    const unsigned grid = 1184;
    if (elem == 1) bitpack_decode_kernel<uint8_t><<<grid, 256, 0, s>>>(in, n, nbits, (uint8_t*)out);
    else if (elem == 2) bitpack_decode_kernel<uint16_t><<<grid, 256, 0, s>>>(in, n, nbits, (uint16_t*)out);
    else bitpack_decode_kernel<uint32_t><<<grid, 256, 0, s>>>(in, n, nbits, (uint32_t*)out);
    return (int)cudaGetLastError();
}

}  // namespace fzb
