// fzb_rows2d.cu -- LorenzoQuant 2-D codes for fields whose rows are whole
// 8192-element chunks (nx a multiple of 8192): the codes-only forward of
// LorenzoQuantStage (lorenzo_quant_nd.cu:199-274, 2-D: 32x32 tiles, the y
// difference then the x difference) in one pass from HBM to HBM, no shared
// memory windows.
//
// A CTA of 256 threads walks down a run of rows of one chunk column.  Thread
// t owns granules t + 256 i (i = 0..7) of its chunk, four elements each, so
// every load and store of a warp is 512 / 256 contiguous bytes and a 32-wide
// x tile is the granules of 8 consecutive lanes.  Per row the thread
//   * quantizes its 32 values (scalar products, round half away from zero as
//     trunc(y + copysign(0.49999997, y)), packed adds),
//   * subtracts the row above, whose q it holds in registers from the
//     previous row (y % 32 == 0 starts a tile: no y difference),
//   * takes the x difference inside the granule and, for its first element,
//     against lane - 1's last one (a shuffle; lane % 8 == 0 starts a tile),
//   * converts the integer-valued deltas to codes with the float magic-number
//     add and zigzags them as packed pairs, flags outliers per granule with a
//     NaN-propagating max and confirms them element by element.
// A chunk with outliers stages them in index order (granule-major, one block
// scan per granule slot); the values are recomputed from the input with the
// same operations.  Codes and outliers equal lq_chunk_kernel's; the run's
// first row reloads the row above when the run starts inside a tile.
#include "fzb_slab.cuh"

namespace fzb {
namespace {

constexpr int kRowThreads = 256;
constexpr int kRowGran = kChunkCodes / 4 / kRowThreads;  // granules a thread owns per chunk (8)
constexpr int kRowCtasPerSm = 2;

// Deltas of a granule from its q, the row above's q (ty) and the previous
// element's y difference `left` (0 at a tile start): c = (q - q_up) - left.
__device__ __forceinline__ Q4 deltas4(Q4 q, Q4 qu, bool ty, float left) {
    const Q4 v = ty ? Q4{sub2(q.a, qu.a), sub2(q.b, qu.b)} : q;
    return {sub2(v.a, f2(left, v.a.x)), sub2(v.b, f2(v.a.y, v.b.x))};
}

// The y-differenced value of the element before granule g's first (lane - 1
// of the tile), recomputed from the input for the outlier records.
__device__ __forceinline__ float left_v(const float* __restrict__ row, const float* __restrict__ up, bool ty,
                                        uint32_t e, float r) {
    const float q = round_half_away(__fmul_rn(__ldg(row + e), r));
    return ty ? __fsub_rn(q, round_half_away(__fmul_rn(__ldg(up + e), r))) : q;
}

__device__ __forceinline__ void stage_outlier(const FwdArgs& a, uint32_t flag, float c, uint32_t k, uint32_t& pos) {
    if (!flag) return;
    if (pos < a.ostage_cap) {
        a.ostage_err[pos] = c;
        a.ostage_idx[pos] = k;
    }
    pos++;
}

template <bool ZZ>
__global__ void __launch_bounds__(kRowThreads, kRowCtasPerSm) lq2d_rows_kernel(FwdArgs a, uint32_t m, uint32_t rpr,
                                                                             uint32_t units) {
    __shared__ uint32_t s_ws[16];
    __shared__ uint32_t s_obase;
    const uint32_t t = threadIdx.x, lane = t & 31u;
    const float r = __ldcg(a.ebx2_r);
    const float R = a.radius;
    const uint32_t ny = a.nfield / a.nx;
    const bool tile_start = (lane & 7u) == 0;
    for (uint32_t u = blockIdx.x; u < units; u += gridDim.x) {
        const uint32_t col = u % m, y0 = (u / m) * rpr, y1 = min(ny, y0 + rpr);
        Q4 qp[kRowGran];  // q of the row above, this thread's granules
        if (y0 & 31u) {   // the run starts inside a tile: q of row y0 - 1
            const float4* up4 = reinterpret_cast<const float4*>(a.in + (size_t)(y0 - 1) * a.nx + (size_t)col * kChunkCodes);
#pragma unroll
            for (int i = 0; i < kRowGran; i++) qp[i] = quant4(__ldg(up4 + t + kRowThreads * i), r);
        } else {
#pragma unroll
            for (int i = 0; i < kRowGran; i++) qp[i] = {f2(0.f, 0.f), f2(0.f, 0.f)};
        }
        for (uint32_t y = y0; y < y1; y++) {
            const uint32_t c = y * m + col;
            const size_t rowbase = (size_t)y * a.nx + (size_t)col * kChunkCodes;
            const float4* in4 = reinterpret_cast<const float4*>(a.in + rowbase);
            const bool ty = (y & 31u) != 0;
            float4 xv[kRowGran];
#pragma unroll
            for (int i = 0; i < kRowGran; i++) xv[i] = __ldcs(in4 + t + kRowThreads * i);
            uint2 cw[kRowGran];
            uint32_t om = 0;  // outlier bit per element: granule i, element k -> bit 4i + k
#pragma unroll
            for (int i = 0; i < kRowGran; i++) {
                const Q4 q = quant4(xv[i], r);
                const Q4 qu = qp[i];
                qp[i] = q;
                const float vlast = ty ? __fsub_rn(q.b.y, qu.b.y) : q.b.y;
                const float vprev = __shfl_up_sync(0xffffffffu, vlast, 1);
                const Q4 cc = deltas4(q, qu, ty, tile_start ? 0.0f : vprev);
                const float mx = max_nan(max_nan(fabsf(cc.a.x), fabsf(cc.a.y)), max_nan(fabsf(cc.b.x), fabsf(cc.b.y)));
                uint32_t p0 = code_pair<ZZ>(cc.a), p1 = code_pair<ZZ>(cc.b);
                if (!(mx < R)) {  // outliers: exact per-element test, their codes are 0
                    const uint32_t b = (fabsf(cc.a.x) < R ? 0u : 1u) | (fabsf(cc.a.y) < R ? 0u : 2u) |
                                       (fabsf(cc.b.x) < R ? 0u : 4u) | (fabsf(cc.b.y) < R ? 0u : 8u);
                    om |= b << (4 * i);
                    p0 &= ((b & 1u) ? 0xffff0000u : 0xffffffffu) & ((b & 2u) ? 0x0000ffffu : 0xffffffffu);
                    p1 &= ((b & 4u) ? 0xffff0000u : 0xffffffffu) & ((b & 8u) ? 0x0000ffffu : 0xffffffffu);
                }
                cw[i] = make_uint2(p0, p1);
            }
            uint2* out2 = reinterpret_cast<uint2*>(a.codes + rowbase);
#pragma unroll
            for (int i = 0; i < kRowGran; i++) __stcs(out2 + t + kRowThreads * i, cw[i]);

            // outliers, in index order: granule slot i major, thread minor
            if (__syncthreads_or(om != 0u)) {
                uint32_t off[kRowGran], run = 0;
#pragma unroll
                for (int i = 0; i < kRowGran; i++) {
                    uint32_t tot;
                    off[i] = block_excl_scan(__popc((om >> (4 * i)) & 15u), s_ws, &tot) + run;
                    run += tot;
                }
                if (t == 0) {
                    const uint32_t b = atomicAdd(a.ostage_ctr, run);
                    a.obase[c] = b;
                    a.ocnt[c] = run;
                    s_obase = b;
                }
                __syncthreads();
                const float* row = a.in + rowbase;
                const float* up = row - a.nx;
#pragma unroll
                for (int i = 0; i < kRowGran; i++) {
                    const uint32_t bits = (om >> (4 * i)) & 15u;
                    if (bits) {
                        const uint32_t g = t + kRowThreads * i;
                        const Q4 q = quant4(__ldg(reinterpret_cast<const float4*>(row) + g), r);
                        Q4 qu = {f2(0.f, 0.f), f2(0.f, 0.f)};
                        if (ty) qu = quant4(__ldg(reinterpret_cast<const float4*>(up) + g), r);
                        const float left = tile_start ? 0.0f : left_v(row, up, ty, 4 * g - 1, r);
                        const Q4 cc = deltas4(q, qu, ty, left);
                        uint32_t pos = s_obase + off[i];
                        const uint32_t k0 = (uint32_t)(rowbase + 4 * g);
                        stage_outlier(a, bits & 1u, cc.a.x, k0, pos);
                        stage_outlier(a, bits & 2u, cc.a.y, k0 + 1, pos);
                        stage_outlier(a, bits & 4u, cc.b.x, k0 + 2, pos);
                        stage_outlier(a, bits & 8u, cc.b.y, k0 + 3, pos);
                    }
                }
            } else if (t == 0) {
                a.obase[c] = 0;
                a.ocnt[c] = 0;
            }
        }
    }
}

}  // namespace

// float4 loads, uint2 code stores; the magic-number conversion is exact for
// |c| < 2^22, and codes are only formed for |c| < radius
bool lq_rows_supported(const FwdArgs& a) {
    return (reinterpret_cast<uintptr_t>(a.in) & 15) == 0 && (reinterpret_cast<uintptr_t>(a.codes) & 7) == 0 &&
           a.radius <= 2097152.0f;
}

int launch_lq_rows(const FwdArgs& a, unsigned sms, cudaStream_t s) {
    const uint32_t m = a.nx / (uint32_t)kChunkCodes, ny = a.nfield / a.nx;
    const uint32_t want = (uint32_t)kRowCtasPerSm * sms;
    // runs of whole 32-row tiles where that still fills the GPU
    uint32_t rpr = (uint32_t)(((uint64_t)m * ny + want - 1) / want);
    if (rpr < 1) rpr = 1;
    if (rpr >= 32) rpr = (rpr + 31) & ~31u;
    const uint32_t runs = (ny + rpr - 1) / rpr, units = m * runs;
    const unsigned grid = units < want ? units : want;
    if (a.zigzag) lq2d_rows_kernel<true><<<grid, kRowThreads, 0, s>>>(a, m, rpr, units);
    else lq2d_rows_kernel<false><<<grid, kRowThreads, 0, s>>>(a, m, rpr, units);
    return (int)cudaGetLastError();
}

}  // namespace fzb
