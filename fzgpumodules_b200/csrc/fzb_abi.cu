// fzb_abi.cu -- the extern "C" boundary (include/fzb.h).  Host-side
// argument checking, workspace carving and kernel launches; no allocation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/fzb.h"
#include "fzb_kernels.cuh"

using namespace fzb;

namespace {

constexpr int kVersion = 100;
constexpr size_t kCtrlBytes = 256;   // err, ticket, scalars
constexpr int kMaxParts = 1024;      // min/max partials

struct Work {
    uint32_t* err;
    uint32_t* ostage_ctr;
    unsigned int* mm_done;
    float* pmin;
    float* pmax;
    unsigned long long* in_off;   // decode: payload offsets; encode: pay_off
    uint32_t* ostart;             // decode: per-chunk outlier start; encode: ofin
    uint32_t* sizes;
    uint32_t* ocnt;
    uint32_t* obase;
    uint16_t* codes;   // 2 * n_total bytes: chunk slots (encode) / codes (exact inverse)
    float* ostage_err;
    uint32_t* ostage_idx;
    uint64_t ostage_cap;
    uint32_t* big;      // n_total u32 (RLE run starts / offsets)
    uint32_t* tiles;    // per-4096-element tile scratch
    uint32_t* total;    // device scalar
    unsigned int* done; // last-block counter
    uint8_t* nbits;     // device byte
    size_t need;
};

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

inline uint64_t chunks_of(uint64_t n_total) { return (n_total + kChunkCodes - 1) / kChunkCodes; }

Work carve(void* base, uint64_t n_total, uint64_t cap) {
    Work w{};
    const uint64_t nch = chunks_of(n_total) + 1;
    uint8_t* p = static_cast<uint8_t*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        uint8_t* q = p ? p + off : nullptr;
        off += align256(bytes);
        return q;
    };
    uint8_t* ctrl = take(kCtrlBytes);
    w.err = reinterpret_cast<uint32_t*>(ctrl);
    w.ostage_ctr = reinterpret_cast<uint32_t*>(ctrl ? ctrl + 4 : nullptr);
    w.mm_done = reinterpret_cast<unsigned int*>(ctrl ? ctrl + 8 : nullptr);
    w.pmin = reinterpret_cast<float*>(take(sizeof(float) * kMaxParts));
    w.pmax = reinterpret_cast<float*>(take(sizeof(float) * kMaxParts));
    w.in_off = reinterpret_cast<unsigned long long*>(take(8 * (nch + 1)));
    w.ostart = reinterpret_cast<uint32_t*>(take(4 * (nch + 1)));
    w.sizes = reinterpret_cast<uint32_t*>(take(4 * nch));
    w.ocnt = reinterpret_cast<uint32_t*>(take(4 * nch));
    w.obase = reinterpret_cast<uint32_t*>(take(4 * nch));
    w.codes = reinterpret_cast<uint16_t*>(take(2 * (n_total + kChunkCodes) + 64));
    w.ostage_cap = cap;
    w.ostage_err = reinterpret_cast<float*>(take(4 * (cap + 1)));
    w.ostage_idx = reinterpret_cast<uint32_t*>(take(4 * (cap + 1)));
    w.big = reinterpret_cast<uint32_t*>(take(4 * (n_total + 64)));
    w.tiles = reinterpret_cast<uint32_t*>(take(4 * (n_total / 4096 + 64)));
    w.total = reinterpret_cast<uint32_t*>(ctrl ? ctrl + 12 : nullptr);
    w.done = reinterpret_cast<unsigned int*>(ctrl ? ctrl + 16 : nullptr);
    w.nbits = ctrl ? ctrl + 20 : nullptr;
    w.need = off;
    return w;
}

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

// FZB_DISABLE_SLAB is a bit mask selecting the alternative kernels (all
// produce identical results; tests exercise each): 1 = 3-D fused compression
// through the per-chunk kernel, 2 = the cp.async slab kernel instead of the
// TMA one, 4 = the per-(slab, tile) fused inverse instead of the persistent
// slab inverse, 8 = codes of 2-D fields with chunk-wide rows through the
// per-chunk kernel instead of the row walk.
#define CK(call)                                          \
    do {                                                  \
        if ((call) != cudaSuccess) return FZB_E_CUDA;     \
    } while (0)

struct Geometry {
    uint32_t nx, ny, nz, ndim, nfield;
};

int geometry(uint64_t n_total, const uint32_t dims[3], Geometry* g) {
    if (n_total == 0 || n_total >= (1ull << 31) || dims == nullptr) return FZB_E_INVALID;
    uint32_t ny = dims[1] ? dims[1] : 1, nz = dims[2] ? dims[2] : 1;
    uint64_t nx = dims[0];
    if (nx == 0) nx = n_total / ((uint64_t)ny * nz);  // LorenzoQuantStage infers x
    const uint64_t nf = nx * ny * nz;
    if (nx == 0 || nf == 0 || nf > n_total) return FZB_E_INVALID;
    g->nx = (uint32_t)nx;
    g->ny = ny;
    g->nz = nz;
    g->nfield = (uint32_t)nf;
    g->ndim = nz > 1 ? 3 : (ny > 1 ? 2 : 1);  // LorenzoQuantStage::ndim()
    return FZB_OK;
}

// Dynamic shared memory of the chunk kernel: the staged windows, at least
// the RZE working set when fused.
size_t lq_smem_bytes(const Geometry& g, bool fused) {
    auto gran = [](uint64_t len) { return (((len + 3) / 4 + 1) + 7) & ~(uint64_t)7; };
    uint64_t per_plane;
    if (g.ndim == 1) per_plane = gran(kChunkCodes + 1);
    else if (g.nx <= kChunkCodes) per_plane = gran((uint64_t)g.nx + 1 + kChunkCodes);
    else per_plane = 2 * gran(kChunkCodes + 1);
    const uint64_t planes = (g.ndim == 3) ? 2 : 1;
    size_t bytes = (size_t)(per_plane * planes * 16);
    const size_t rze_set = 2 * kChunkBytes + 16 + 2048 + 256 + 32;
    if (fused && bytes < rze_set) bytes = rze_set;
    return bytes;
}

int launch_lq(const Geometry& g, bool fused, const FwdArgs& a, size_t smem, uint32_t grid,
              cudaStream_t s) {
    const bool rowal = (g.ndim == 1) || (g.nx % 32 == 0);
    return launch_lq_chunk((int)g.ndim, fused, rowal, a, smem, grid, s) == 0 ? FZB_OK : FZB_E_CUDA;
}

// Resolves abs_eb / ebx2_r on the device into eb_state (no host sync).
int resolve_eb(const float* d_in, uint64_t n_total, float eb, int mode, float value_base,
               const Work& w, float* d_eb_state, cudaStream_t s) {
    if (mode != FZB_ABS && !(value_base > 0.0f)) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        uint64_t want = (n_total / 4 + 255) / 256;
        int parts = (int)(want < (uint64_t)(7 * sms) ? want : (uint64_t)(7 * sms));
        if (parts < 1) parts = 1;
        if (parts > kMaxParts) parts = kMaxParts;
        TraceScope ts(s, "minmax_resolve_eb");
        minmax_kernel<<<parts, 256, 0, s>>>(d_in, n_total, w.pmin, w.pmax, w.mm_done, mode, eb,
                                            d_eb_state);
    } else {
        TraceScope ts(s, "resolve_eb");
        resolve_eb_kernel<<<1, 32, 0, s>>>(mode, eb, value_base, d_eb_state);
    }
    CK(cudaGetLastError());
    return FZB_OK;
}

// Chunk-kernel arguments of one field whose workspace is `w`.
FwdArgs fwd_args(const Geometry& g, const Work& w, const float* d_in, uint64_t n_total, float* d_eb_state,
                 uint32_t radius, int zigzag, uint16_t* d_codes, uint64_t cap) {
    FwdArgs a{};
    a.in = d_in;
    a.n_total = (uint32_t)n_total;
    a.nfield = g.nfield;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.plane = g.nx * g.ny;
    a.ebx2_r = d_eb_state + 2;
    a.radius = (float)(uint16_t)radius;  // the kernel compares against TCode(radius)
    a.zigzag = zigzag;
    a.two_piece = (g.ndim >= 2 && g.nx > (uint32_t)kChunkCodes) ? 1 : 0;
    a.codes = d_codes;
    a.n_chunks = (uint32_t)chunks_of(n_total);
    a.slots = reinterpret_cast<uint8_t*>(w.codes);
    a.sizes = w.sizes;
    a.ocnt = w.ocnt;
    a.obase = w.obase;
    a.ostage_ctr = w.ostage_ctr;
    a.ostage_err = w.ostage_err;
    a.ostage_idx = w.ostage_idx;
    a.ostage_cap = (uint32_t)(cap < 0xffffffffull ? cap : 0xffffffffull);
    a.err = w.err;
    return a;
}

// Assembly arguments matching fwd_args().
AsmArgs asm_args(const Work& w, const FwdArgs& a, bool fused, void* d_rze, uint64_t* d_rze_size, float* d_err,
                 uint32_t* d_idx, uint32_t* d_count) {
    AsmArgs m{};
    m.slots = a.slots;
    m.sizes = fused ? w.sizes : nullptr;
    m.n_chunks = a.n_chunks;
    m.orig_bytes = 2u * a.n_total;
    m.out = static_cast<uint8_t*>(d_rze);
    m.out_size = reinterpret_cast<unsigned long long*>(d_rze_size);
    m.pay_off = w.in_off;
    m.ocnt = w.ocnt;
    m.obase = w.obase;
    m.ofin = w.ostart;
    m.ostage_err = w.ostage_err;
    m.ostage_idx = w.ostage_idx;
    m.ostage_cap = a.ostage_cap;
    m.out_err = d_err;
    m.out_idx = d_idx;
    m.cap = a.ostage_cap;
    m.out_count = d_count;
    return m;
}

int forward_common(bool fused, const float* d_in, uint64_t n_total, const uint32_t dims[3],
                   float eb, int eb_mode, float value_base, uint32_t radius, int zigzag,
                   uint16_t* d_codes, float* d_err, uint32_t* d_idx, uint64_t cap,
                   uint32_t* d_count, void* d_rze, uint64_t* d_rze_size, float* d_eb_state,
                   void* d_work, size_t work_bytes, void* stream) {
    Geometry g;
    int rc = geometry(n_total, dims, &g);
    if (rc) return rc;
    if (!d_in || !d_count || !d_eb_state || (cap && (!d_err || !d_idx))) return FZB_E_INVALID;
    if (fused ? (!d_rze || !d_rze_size) : !d_codes) return FZB_E_INVALID;
    if (eb_mode < FZB_ABS || eb_mode > FZB_NOA || !(eb > 0.0f)) return FZB_E_INVALID;
    Work w = carve(d_work, n_total, cap);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    const uint64_t nch = chunks_of(n_total);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    rc = resolve_eb(d_in, n_total, eb, eb_mode, value_base, w, d_eb_state, s);
    if (rc) return rc;
    const FwdArgs a = fwd_args(g, w, d_in, n_total, d_eb_state, radius, zigzag, d_codes, cap);
    const uint32_t nx = g.nx;
    const bool slab = fused && g.ndim == 3 && nx >= 32 && nx <= 1024 && (nx & (nx - 1)) == 0 &&
                      g.ny % ((uint32_t)kChunkCodes / nx) == 0 && g.nfield == n_total &&
                      !(flags_env() & 1);
    if (slab) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (lq3d_tma_supported(a) && !(flags_env() & 2)) {
            TraceScope ts(s, "lq3d_tma_bs_rze");
            rc = launch_lq3d_tma(a, (unsigned)(2 * sms), s) == 0 ? FZB_OK : FZB_E_CUDA;
        } else {
            TraceScope ts(s, "lq3d_slab_bs_rze");
            rc = launch_lq3d_slab(a, (unsigned)(2 * sms), s) == 0 ? FZB_OK : FZB_E_CUDA;
        }
    } else if (!fused && g.ndim == 2 && nx % (uint32_t)kChunkCodes == 0 && g.nfield == n_total &&
               lq_rows_supported(a) && !(flags_env() & 8)) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        TraceScope ts(s, "lq_rows");
        rc = launch_lq_rows(a, (unsigned)sms, s) == 0 ? FZB_OK : FZB_E_CUDA;
    } else {
        TraceScope ts(s, fused ? "lq_chunk_bs_rze" : "lq_chunk");
        rc = launch_lq(g, fused, a, lq_smem_bytes(g, fused), (uint32_t)nch, s);
    }
    if (rc) return rc;
    const AsmArgs m = asm_args(w, a, fused, d_rze, d_rze_size, d_err, d_idx, d_count);
    {
        TraceScope ts(s, "assemble_scan");
        if (launch_assemble_scan(m, s) != 0) return FZB_E_CUDA;
    }
    CK(cudaGetLastError());
    {
        TraceScope ts(s, "assemble_copy");
        CK(launch_dependent(assemble_copy_kernel, copy_grid(nch), 256, 0, s, m));
    }
    CK(cudaGetLastError());
    return FZB_OK;
}

InvArgs inv_args(const Work& w, const Geometry& g, uint64_t n_total) {
    InvArgs a{};
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.plane = g.nx * g.ny;
    a.nfield = g.nfield;
    a.n_total = (uint32_t)n_total;
    a.err = w.err;
    a.in_off = w.in_off;
    a.ostart = w.ostart;
    return a;
}

int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// zero(out) + scatter + tile kernels (the exact path).  Every kernel walks
// its tiles grid-stride: one tile per CTA normally; when the launch is gated
// on the device status (a.gate) the grids are a few CTAs per SM, so a gate
// that says "not needed" costs a few microseconds.
int exact_inverse(const InvArgs& a, const Geometry& g, cudaStream_t s) {
    const uint32_t lim = a.gate ? 2u * (uint32_t)sm_count() : 0xffffffffu;
    auto grid = [&](uint64_t tiles) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, lim)); };
    if (a.gate) {
        TraceScope ts(s, "zero_out");
        zero_out_kernel<<<grid(((uint64_t)a.n_total + 1023) / 1024), 256, 0, s>>>(a);
        CK(cudaGetLastError());
    } else {
        CK(cudaMemsetAsync(a.out, 0, sizeof(float) * (size_t)a.n_total, s));
    }
    if (a.cap) {
        TraceScope ts(s, "scatter_outliers");
        scatter_outliers_kernel<<<std::min(grid((a.cap + 255) / 256), 4096u), 256, 0, s>>>(a);
        CK(cudaGetLastError());
    }
    TraceScope ts(s, "lq_inverse");
    if (g.ndim == 1) {
        lq_inverse_1d_kernel<<<grid((g.nfield + 1023) / 1024), 256, 0, s>>>(a);
    } else if (g.ndim == 2) {
        lq_inverse_2d_kernel<<<grid((uint64_t)((g.nx + 31) / 32) * ((g.ny + 31) / 32)), 128, 0, s>>>(a);
    } else {
        lq_inverse_3d_kernel<<<grid((uint64_t)((g.nx + 31) / 32) * ((g.ny + 7) / 8) * ((g.nz + 7) / 8)), 256, 0, s>>>(a);
    }
    CK(cudaGetLastError());
    return FZB_OK;
}

int read_status(const Work& w, cudaStream_t s, uint32_t* bits) {
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpy(bits, w.err, 4, cudaMemcpyDeviceToHost));
    return FZB_OK;
}

int status_of(uint32_t bits) {
    if (bits & kErrMalformed) return FZB_E_MALFORMED;
    if (bits & (kErrLookbackTimeout | kErrTmaTimeout)) return FZB_E_TIMEOUT;
    return FZB_OK;
}

}  // namespace

extern "C" {

int fzb_version(void) { return kVersion; }

const char* fzb_status_string(int st) {
    switch (st) {
        case FZB_OK: return "ok";
        case FZB_E_INVALID: return "invalid argument or unsupported configuration";
        case FZB_E_CUDA: return "CUDA runtime error";
        case FZB_E_WORKSPACE: return "workspace too small";
        case FZB_E_CAPACITY: return "output buffer too small";
        case FZB_E_MALFORMED: return "malformed compressed input";
        case FZB_E_TIMEOUT: return "device wait timed out";
        case FZB_E_RANGE: return "input symbol outside [0, bklen)";
        default: return "unknown status";
    }
}

size_t fzb_workspace_bytes(uint64_t n_total, uint64_t cap) { return carve(nullptr, n_total, cap).need; }

int fzb_workspace_status(void* d_work, void* stream) {
    if (!d_work) return FZB_E_INVALID;
    uint32_t* err = static_cast<uint32_t*>(d_work);
    uint32_t bits = 0;
    CK(cudaStreamSynchronize(S(stream)));
    CK(cudaMemcpy(&bits, err, 4, cudaMemcpyDeviceToHost));
    CK(cudaMemset(err, 0, 4));
    return status_of(bits);
}

int fzb_status_from_bits(uint32_t bits, int* rerun_exact) {
    if (rerun_exact) *rerun_exact = (bits & (kErrInexact | kErrUnsorted)) ? 1 : 0;
    return status_of(bits);
}

int fzb_lq_forward(const float* d_in, uint64_t n_total, const uint32_t dims[3], float eb,
                   int eb_mode, float value_base, uint32_t radius, int zigzag, uint16_t* d_codes,
                   float* d_err, uint32_t* d_idx, uint64_t cap, uint32_t* d_count,
                   float* d_eb_state, void* d_work, size_t work_bytes, void* stream) {
    return forward_common(false, d_in, n_total, dims, eb, eb_mode, value_base, radius, zigzag,
                          d_codes, d_err, d_idx, cap, d_count, nullptr, nullptr, d_eb_state,
                          d_work, work_bytes, stream);
}

int fzb_lq_bs_rze_compress(const float* d_in, uint64_t n_total, const uint32_t dims[3], float eb,
                           int eb_mode, float value_base, uint32_t radius, int zigzag,
                           float* d_err, uint32_t* d_idx, uint64_t cap, uint32_t* d_count,
                           void* d_rze, uint64_t* d_rze_size, float* d_eb_state, void* d_work,
                           size_t work_bytes, void* stream) {
    return forward_common(true, d_in, n_total, dims, eb, eb_mode, value_base, radius, zigzag,
                          nullptr, d_err, d_idx, cap, d_count, d_rze, d_rze_size, d_eb_state,
                          d_work, work_bytes, stream);
}

namespace {
int lq_inverse_common(const uint16_t* d_codes, const float* d_err, const uint32_t* d_idx, const uint32_t* d_count,
                      uint64_t cap, uint64_t n_total, const uint32_t dims[3], float abs_eb, const float* d_abs_eb,
                      int zigzag, float* d_out, void* d_work, size_t work_bytes, void* stream) {
    Geometry g;
    int rc = geometry(n_total, dims, &g);
    if (rc) return rc;
    if (!d_codes || !d_out || !d_count || (cap && (!d_err || !d_idx))) return FZB_E_INVALID;
    Work w = carve(d_work, n_total, 0);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    InvArgs a = inv_args(w, g, n_total);
    a.codes = const_cast<uint16_t*>(d_codes);
    a.out_err = d_err;
    a.out_idx = d_idx;
    a.out_count = d_count;
    a.cap = (uint32_t)(cap < 0xffffffffull ? cap : 0xffffffffull);
    a.ebx2 = 2.0f * abs_eb;
    a.abs_eb_src = d_abs_eb;
    a.zigzag = zigzag;
    a.out = d_out;
    return exact_inverse(a, g, s);
}
}  // namespace

int fzb_lq_inverse(const uint16_t* d_codes, const float* d_err, const uint32_t* d_idx,
                   const uint32_t* d_count, uint64_t cap, uint64_t n_total, const uint32_t dims[3],
                   float abs_eb, int zigzag, float* d_out, void* d_work, size_t work_bytes,
                   void* stream) {
    return lq_inverse_common(d_codes, d_err, d_idx, d_count, cap, n_total, dims, abs_eb, nullptr, zigzag, d_out,
                             d_work, work_bytes, stream);
}

int fzb_lq_inverse_dev(const uint16_t* d_codes, const float* d_err, const uint32_t* d_idx,
                       const uint32_t* d_count, uint64_t cap, uint64_t n_total, const uint32_t dims[3],
                       const float* d_abs_eb, int zigzag, float* d_out, void* d_work, size_t work_bytes,
                       void* stream) {
    if (!d_abs_eb) return FZB_E_INVALID;
    return lq_inverse_common(d_codes, d_err, d_idx, d_count, cap, n_total, dims, 0.0f, d_abs_eb, zigzag, d_out,
                             d_work, work_bytes, stream);
}

int fzb_bitshuffle(const void* d_in, uint64_t bytes, uint32_t block, int ew, int inverse,
                   void* d_out, void* stream) {
    if (!d_in || !d_out || (ew != 1 && ew != 2 && ew != 4 && ew != 8)) return FZB_E_INVALID;
    if (block == 0 || block % (1024u * (uint32_t)ew) != 0) return FZB_E_INVALID;
    cudaStream_t s = S(stream);
    const uint64_t nfull = bytes / block;
    const uint8_t* in = static_cast<const uint8_t*>(d_in);
    uint8_t* out = static_cast<uint8_t*>(d_out);
    if (nfull) {
        if (ew == 2 && block == (uint32_t)kChunkBytes &&
            ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0) {
            bitshuffle2_kernel<<<(unsigned)nfull, kThreads, 0, s>>>(in, out, inverse);
        } else if (ew == 4 || ew == 8) {
            if (((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & (uintptr_t)(ew - 1)) != 0)
                return FZB_E_INVALID;  // the reference reads and writes u32 / u64 words
            if (launch_bitshuffle_wide(in, out, nfull, block, ew, inverse, s) != 0) return FZB_E_CUDA;
        } else {
            const uint32_t nchunk = block / (uint32_t)ew;
            bitshuffle_ballot_kernel<<<(unsigned)nfull, nchunk < 1024 ? nchunk : 1024, 0, s>>>(
                in, out, block, ew, inverse);
        }
        CK(cudaGetLastError());
    }
    const uint64_t tail = bytes - nfull * block;
    if (tail) CK(cudaMemcpyAsync(out + nfull * block, in + nfull * block, tail,
                                 cudaMemcpyDeviceToDevice, s));
    return FZB_OK;
}

uint64_t fzb_rze_max_bytes(uint64_t bytes) {
    const uint64_t nch = (bytes + kChunkBytes - 1) / kChunkBytes;
    return 8 + 4 * nch + nch * (uint64_t)kChunkBytes + 4;
}

int fzb_rze_encode(const void* d_in, uint64_t bytes, void* d_out, uint64_t* d_out_size,
                   void* d_work, size_t work_bytes, void* stream) {
    if (!d_in || !d_out || !d_out_size || bytes == 0 || bytes >= (1ull << 32)) return FZB_E_INVALID;
    const uint64_t n_equiv = (bytes + 1) / 2;
    Work w = carve(d_work, n_equiv, 0);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    const uint64_t nch = (bytes + kChunkBytes - 1) / kChunkBytes;
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    RzeEncArgs a{};
    a.in = static_cast<const uint8_t*>(d_in);
    a.bytes = bytes;
    a.slots = reinterpret_cast<uint8_t*>(w.codes);
    a.sizes = w.sizes;
    const int smem = 2 * kChunkBytes + 16 + 2048 + 256 + 32;
    CK(cudaFuncSetAttribute(rze_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    rze_encode_kernel<<<(unsigned)nch, kThreads, smem, s>>>(a);
    CK(cudaGetLastError());
    AsmArgs m{};
    m.slots = a.slots;
    m.sizes = w.sizes;
    m.n_chunks = (uint32_t)nch;
    m.orig_bytes = (uint32_t)bytes;
    m.out = static_cast<uint8_t*>(d_out);
    m.out_size = reinterpret_cast<unsigned long long*>(d_out_size);
    m.pay_off = w.in_off;
    if (launch_assemble_scan(m, s) != 0) return FZB_E_CUDA;
    CK(cudaGetLastError());
    assemble_copy_kernel<<<copy_grid(nch), 256, 0, s>>>(m);
    CK(cudaGetLastError());
    return FZB_OK;
}

int fzb_rze_decode(const void* d_in, uint64_t in_bytes, uint64_t orig_bytes, void* d_out,
                   void* d_work, size_t work_bytes, void* stream) {
    if (!d_in || !d_out || orig_bytes == 0 || orig_bytes >= (1ull << 32)) return FZB_E_INVALID;
    const uint64_t nch = (orig_bytes + kChunkBytes - 1) / kChunkBytes;
    if (in_bytes < 8 + 4 * nch) return FZB_E_MALFORMED;
    const uint64_t n_equiv = (orig_bytes + 1) / 2;
    Work w = carve(d_work, n_equiv, 0);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    if (launch_rze_prepass(static_cast<const uint8_t*>(d_in), in_bytes, (uint32_t)nch, (uint32_t)orig_bytes,
                           w.in_off, w.err, s) != 0)
        return FZB_E_CUDA;
    CK(cudaGetLastError());
    InvArgs a{};
    a.rze = static_cast<const uint8_t*>(d_in);
    a.rze_bytes = in_bytes;
    a.in_off = w.in_off;
    a.n_chunks = (uint32_t)nch;
    a.orig_bytes = (uint32_t)orig_bytes;
    a.bytes_out = static_cast<uint8_t*>(d_out);
    a.err = w.err;
    const int smem = kChunkBytes * 2 + 16 + 2048 + 256 + 32;
    CK(cudaFuncSetAttribute(rze_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    rze_decode_kernel<<<(unsigned)nch, kThreads, smem, s>>>(a);
    CK(cudaGetLastError());
    return FZB_OK;
}

namespace {
int lq_bs_rze_decompress_common(const void* d_rze, uint64_t rze_bytes, const float* d_err,
                                const uint32_t* d_idx, const uint32_t* d_count, uint64_t cap,
                                uint64_t n_total, const uint32_t dims[3], float abs_eb, const float* d_abs_eb,
                                int zigzag, float* d_out, unsigned flags, void* d_work, size_t work_bytes,
                                void* stream) {
    Geometry g;
    int rc = geometry(n_total, dims, &g);
    if (rc) return rc;
    if (!d_rze || !d_out || !d_count || (cap && (!d_err || !d_idx))) return FZB_E_INVALID;
    const uint64_t nch = chunks_of(n_total);
    if (rze_bytes < 8 + 4 * nch) return FZB_E_MALFORMED;
    Work w = carve(d_work, n_total, 0);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    {
        TraceScope ts(s, "rze_prepass");
        if (launch_rze_prepass(static_cast<const uint8_t*>(d_rze), rze_bytes, (uint32_t)nch,
                               (uint32_t)(2 * n_total), w.in_off, w.err, s) != 0)
            return FZB_E_CUDA;
    }
    CK(cudaGetLastError());
    InvArgs a = inv_args(w, g, n_total);
    a.rze = static_cast<const uint8_t*>(d_rze);
    a.rze_bytes = rze_bytes;
    a.n_chunks = (uint32_t)nch;
    a.orig_bytes = (uint32_t)(2 * n_total);
    a.out_err = d_err;
    a.out_idx = d_idx;
    a.out_count = d_count;
    a.cap = (uint32_t)(cap < 0xffffffffull ? cap : 0xffffffffull);
    a.ebx2 = 2.0f * abs_eb;
    a.abs_eb_src = d_abs_eb;
    a.zigzag = zigzag;
    a.shuffled = 1;
    a.out = d_out;
    const bool dev_fallback = (flags & FZB_DEVICE_FALLBACK) != 0;

    const uint32_t nx = g.nx;
    const bool pow2 = nx >= 8 && nx <= 1024 && (nx & (nx - 1)) == 0;
    const uint32_t R = pow2 ? (uint32_t)kChunkCodes / nx : 0;
    const bool fused = !(flags & FZB_FORCE_EXACT) && g.ndim == 3 && pow2 && g.ny % R == 0;
    if (fused) {
        {
            TraceScope ts(s, "outlier_ranges");
            CK(launch_dependent(outlier_ranges_kernel, (unsigned)((nch + 256) / 256 + 1), 256, 0, s, d_idx, d_count,
                                a.cap, (uint32_t)nch, w.ostart, w.err));
        }
        CK(cudaGetLastError());
        const int smem = 2 * kChunkBytes + 16 + 2048 + 256 + 32 + 4 * kChunkCodes;
        CK(cudaFuncSetAttribute(fused_inverse_3d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem));
        if (nx >= 32 && !(flags_env() & 4)) {
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            TraceScope ts(s, "lq3d_inv_slab");
            if (launch_lq3d_inv_slab(a, (unsigned)sms, s) != 0) return FZB_E_CUDA;
        } else {
            dim3 grid(g.ny / R, (g.nz + 7) / 8, 1);
            TraceScope ts(s, "fused_inverse_3d");
            fused_inverse_3d_kernel<<<grid, kThreads, smem, s>>>(a);
        }
        CK(cudaGetLastError());
        if (n_total > g.nfield)
            CK(cudaMemsetAsync(d_out + g.nfield, 0, sizeof(float) * (n_total - g.nfield), s));
        if (dev_fallback) {
            // the exact kernels follow, gated on the flags the fused kernel set
            a.gate = w.err;
            a.gate_mask = kErrInexact | kErrUnsorted;
        } else {
            if (flags & FZB_NO_SYNC) return FZB_OK;
            uint32_t bits = 0;
            rc = read_status(w, s, &bits);
            if (rc) return rc;
            if (status_of(bits) != FZB_OK) return status_of(bits);
            if (!(bits & (kErrInexact | kErrUnsorted))) return FZB_OK;
            CK(cudaMemsetAsync(w.err, 0, 4, s));  // rerun exactly below
        }
    }
    a.codes = w.codes;
    const int smem = 2 * kChunkBytes + 16 + 2048 + 256 + 32;
    CK(cudaFuncSetAttribute(rze_decode_codes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            smem));
    {
        TraceScope ts(s, "rze_decode_bitunshuffle");
        const uint64_t lim = a.gate ? 4ull * (uint64_t)sm_count() : nch;
        rze_decode_codes_kernel<<<(unsigned)std::min<uint64_t>(nch, lim), kThreads, smem, s>>>(a);
    }
    CK(cudaGetLastError());
    rc = exact_inverse(a, g, s);
    if (rc || (flags & (FZB_NO_SYNC | FZB_DEVICE_FALLBACK))) return rc;
    uint32_t bits = 0;
    rc = read_status(w, s, &bits);
    return rc ? rc : status_of(bits);
}

}  // namespace

int fzb_lq_bs_rze_decompress(const void* d_rze, uint64_t rze_bytes, const float* d_err,
                             const uint32_t* d_idx, const uint32_t* d_count, uint64_t cap,
                             uint64_t n_total, const uint32_t dims[3], float abs_eb, int zigzag,
                             float* d_out, unsigned flags, void* d_work, size_t work_bytes,
                             void* stream) {
    return lq_bs_rze_decompress_common(d_rze, rze_bytes, d_err, d_idx, d_count, cap, n_total, dims, abs_eb,
                                       nullptr, zigzag, d_out, flags, d_work, work_bytes, stream);
}

int fzb_lq_bs_rze_decompress_dev(const void* d_rze, uint64_t rze_capacity, const float* d_err,
                                 const uint32_t* d_idx, const uint32_t* d_count, uint64_t cap,
                                 uint64_t n_total, const uint32_t dims[3], const float* d_abs_eb, int zigzag,
                                 float* d_out, void* d_work, size_t work_bytes, void* stream) {
    if (!d_abs_eb) return FZB_E_INVALID;
    return lq_bs_rze_decompress_common(d_rze, rze_capacity, d_err, d_idx, d_count, cap, n_total, dims, 0.0f,
                                       d_abs_eb, zigzag, d_out, FZB_DEVICE_FALLBACK, d_work, work_bytes, stream);
}

uint64_t fzb_rle_max_bytes(uint64_t n, int elem) {
    return 4 + ((n * (uint64_t)elem + 3) & ~3ull) + 4 * n;
}

int fzb_rle_encode(const void* d_in, uint64_t n, int elem, void* d_out, uint64_t* d_out_size,
                   void* d_work, size_t work_bytes, void* stream) {
    if (!d_in || !d_out || !d_out_size || (elem != 1 && elem != 2 && elem != 4)) return FZB_E_INVALID;
    if (n == 0 || n >= (1ull << 31)) return FZB_E_INVALID;
    Work w = carve(d_work, n, 0);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    return launch_rle_encode(d_in, (uint32_t)n, elem, static_cast<uint8_t*>(d_out),
                             reinterpret_cast<unsigned long long*>(d_out_size), w.tiles, w.big,
                             w.total, s) == 0 ? FZB_OK : FZB_E_CUDA;
}

int fzb_rle_decode(const void* d_in, uint64_t n, int elem, void* d_out, void* d_work,
                   size_t work_bytes, void* stream) {
    if (!d_in || !d_out || (elem != 1 && elem != 2 && elem != 4)) return FZB_E_INVALID;
    if (n == 0 || n >= (1ull << 31)) return FZB_E_INVALID;
    Work w = carve(d_work, n, 0);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    return launch_rle_decode(static_cast<const uint8_t*>(d_in), (uint32_t)n, elem, d_out, w.big,
                             w.tiles, w.total, w.err, s) == 0 ? FZB_OK : FZB_E_CUDA;
}

int fzb_bitpack_encode(const void* d_in, uint64_t n, int elem, int nbits, void* d_out,
                       uint8_t* d_nbits, uint64_t* d_out_size, void* d_work, size_t work_bytes,
                       void* stream) {
    if (!d_in || !d_out || (elem != 1 && elem != 2 && elem != 4) || n == 0) return FZB_E_INVALID;
    if (nbits < 0 || nbits > 8 * elem || (nbits & (nbits - 1)) != 0) return FZB_E_INVALID;
    Work w = carve(d_work, 1, 0);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    uint8_t* nb = d_nbits ? d_nbits : w.nbits;
    return launch_bitpack_encode(d_in, n, elem, nbits, nb, static_cast<uint8_t*>(d_out),
                                 reinterpret_cast<unsigned long long*>(d_out_size),
                                 reinterpret_cast<uint32_t*>(w.pmin), w.done, s) == 0 ? FZB_OK : FZB_E_CUDA;
}

int fzb_bitpack_decode(const void* d_in, uint64_t n, int elem, int nbits, void* d_out, void* stream) {
    if (!d_in || !d_out || (elem != 1 && elem != 2 && elem != 4) || n == 0) return FZB_E_INVALID;
    if (nbits <= 0 || nbits > 8 * elem || (nbits & (nbits - 1)) != 0) return FZB_E_INVALID;
    return launch_bitpack_decode(static_cast<const uint8_t*>(d_in), n, elem, nbits, d_out, S(stream)) == 0
               ? FZB_OK : FZB_E_CUDA;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// PHF Huffman (HuffmanStage<uint16_t>, coarse mode).
// ---------------------------------------------------------------------------
namespace {

struct HfWork {
    uint32_t* err;
    uint32_t* ncell_total;
    uint32_t* freq;
    uint32_t* bk4;
    uint8_t* revbook;
    uint32_t* par_nbit;
    uint32_t* par_ncell;
    uint32_t* par_entry;
    uint32_t* tiles;
    uint32_t* slots;
    size_t need;
};

inline uint64_t hf_pardeg(uint64_t n) { return (n - 1) / kHfSublen + 1; }
inline size_t hf_revbook_bytes(uint32_t bklen) { return 256 + 2 * (size_t)bklen; }

// ctrl first, so fzb_workspace_status reads the same error word
HfWork carve_hf(void* base, uint64_t n, uint32_t bklen) {
    HfWork w{};
    const uint64_t pd = hf_pardeg(n);
    uint8_t* p = static_cast<uint8_t*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        uint8_t* q = p ? p + off : nullptr;
        off += align256(bytes);
        return q;
    };
    uint8_t* ctrl = take(kCtrlBytes);
    w.err = reinterpret_cast<uint32_t*>(ctrl);
    w.ncell_total = reinterpret_cast<uint32_t*>(ctrl ? ctrl + 4 : nullptr);
    w.freq = reinterpret_cast<uint32_t*>(take(4 * (size_t)bklen));
    w.bk4 = reinterpret_cast<uint32_t*>(take(4 * (size_t)bklen));
    w.revbook = take(hf_revbook_bytes(bklen));
    w.par_nbit = reinterpret_cast<uint32_t*>(take(4 * pd));
    w.par_ncell = reinterpret_cast<uint32_t*>(take(4 * pd));
    w.par_entry = reinterpret_cast<uint32_t*>(take(4 * pd));
    w.tiles = reinterpret_cast<uint32_t*>(take(4 * (pd / 4096 + 64)));
    // partition slots for either partition length
    const uint64_t pd_fine = (n - 1) / kHfSublenFine + 1;
    w.slots = reinterpret_cast<uint32_t*>(take(4 * std::max(pd * kHfSublen, pd_fine * kHfSublenFine)));
    w.need = off;
    return w;
}

// bklen even keeps every u32 table of the blob 4-byte aligned
inline bool hf_args_ok(uint64_t n, uint32_t bklen) {
    return n > 0 && n < (1ull << 31) && bklen >= 2 && bklen <= 65534 && (bklen & 1) == 0;
}

}  // namespace

extern "C" {

size_t fzb_huff_workspace_bytes(uint64_t n, uint32_t bklen) {
    if (!hf_args_ok(n, bklen)) return 0;
    return carve_hf(nullptr, n, bklen).need;
}

uint64_t fzb_huff_max_bytes(uint64_t n, uint32_t bklen) {
    if (!hf_args_ok(n, bklen)) return 0;
    const uint64_t pd = hf_pardeg(n);
    return 128 + hf_revbook_bytes(bklen) + 8 * pd + 4 * (n + pd) + 16;
}

int fzb_huff_histogram(const uint16_t* d_in, uint64_t n, uint32_t bklen, uint32_t* d_freq,
                       void* stream) {
    if (!d_in || !d_freq || n == 0 || n >= (1ull << 31) || bklen < 1 || bklen > 65535) return FZB_E_INVALID;
    return launch_hf_histogram(d_in, n, bklen, d_freq, sm_count(), S(stream)) == 0 ? FZB_OK : FZB_E_CUDA;
}

int fzb_huff_book(const uint32_t* h_freq, uint32_t bklen, uint32_t* h_bk4, uint8_t* h_revbook) {
    if (!h_freq || !h_bk4 || !h_revbook || bklen < 1 || bklen > 65535) return FZB_E_INVALID;
    return build_huffman_book(h_freq, bklen, h_bk4, h_revbook) == 0 ? FZB_OK : FZB_E_INVALID;
}

}  // extern "C"

namespace {

int huff_encode_sub(const uint16_t* d_in, uint64_t n, uint32_t bklen, const uint32_t* d_bk4,
                    const uint8_t* d_revbook, uint32_t sublen, void* d_out, uint64_t* d_out_size, void* d_work,
                    size_t work_bytes, void* stream) {
    if (!d_in || !d_bk4 || !d_revbook || !d_out || !d_out_size || !hf_args_ok(n, bklen))
        return FZB_E_INVALID;
    if (reinterpret_cast<uintptr_t>(d_out) & 3) return FZB_E_INVALID;
    HfWork w = carve_hf(d_work, n, bklen);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(w.err, 0, kCtrlBytes, s));
    return launch_hf_encode(d_in, n, d_bk4, bklen, sublen, d_revbook, static_cast<uint8_t*>(d_out),
                            reinterpret_cast<unsigned long long*>(d_out_size), w.slots, w.par_nbit,
                            w.par_ncell, w.par_entry, w.tiles, w.ncell_total, w.err, sm_count(), s) == 0
               ? FZB_OK : FZB_E_CUDA;
}

// Pinned host staging of the codebook round trip, one per host thread: the
// histogram comes back and the book goes out with asynchronous copies (a
// pageable copy stages through a driver buffer and blocks).  `done` marks
// the end of the last upload, waited for before the buffers are rewritten.
struct HfHostStage {
    uint32_t* freq = nullptr;
    uint32_t* bk4 = nullptr;
    uint8_t* revbook = nullptr;
    uint32_t bklen = 0;
    int dev = -1;  // the device `done` belongs to
    cudaEvent_t done = nullptr;
    bool pending = false;
    ~HfHostStage() { release(); }
    void release() {
        if (done) {
            if (pending) cudaEventSynchronize(done);
            cudaEventDestroy(done);
        }
        if (freq) cudaFreeHost(freq);
        freq = nullptr;
        bk4 = nullptr;
        revbook = nullptr;
        done = nullptr;
        pending = false;
        bklen = 0;
        dev = -1;
    }
    // false: no pinned memory (the caller stages through vectors)
    bool ensure(uint32_t n) {
        int d = 0;
        if (cudaGetDevice(&d) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (freq && bklen >= n && d == dev) {
            if (pending) cudaEventSynchronize(done);
            pending = false;
            return true;
        }
        release();
        const size_t bytes = 8 * (size_t)n + hf_revbook_bytes(n);
        void* h = nullptr;
        if (cudaHostAlloc(&h, bytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            cudaFreeHost(h);
            done = nullptr;
            return false;
        }
        dev = d;
        freq = static_cast<uint32_t*>(h);
        bk4 = freq + n;
        revbook = reinterpret_cast<uint8_t*>(bk4 + n);
        bklen = n;
        return true;
    }
};

int huff_compress_sub(const uint16_t* d_in, uint64_t n, uint32_t bklen, uint32_t sublen, void* d_out,
                      uint64_t* d_out_size, void* d_work, size_t work_bytes, void* stream) {
    if (!d_in || !d_out || !d_out_size || !hf_args_ok(n, bklen)) return FZB_E_INVALID;
    if (reinterpret_cast<uintptr_t>(d_out) & 3) return FZB_E_INVALID;
    HfWork w = carve_hf(d_work, n, bklen);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    int rc = fzb_huff_histogram(d_in, n, bklen, w.freq, stream);
    if (rc) return rc;
    static thread_local HfHostStage stage;
    std::vector<uint32_t> vfreq, vbk4;
    std::vector<uint8_t> vrev;
    uint32_t *freq, *bk4;
    uint8_t* revbook;
    const bool pinned = stage.ensure(bklen);
    if (pinned) {
        freq = stage.freq;
        bk4 = stage.bk4;
        revbook = stage.revbook;
    } else {
        vfreq.resize(bklen);
        vbk4.resize(bklen);
        vrev.resize(hf_revbook_bytes(bklen));
        freq = vfreq.data();
        bk4 = vbk4.data();
        revbook = vrev.data();
    }
    CK(cudaMemcpyAsync(freq, w.freq, 4 * (size_t)bklen, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    uint64_t sum = 0;
    for (uint32_t i = 0; i < bklen; i++) sum += freq[i];
    if (sum != n) return FZB_E_RANGE;
    if (build_huffman_book(freq, bklen, bk4, revbook) != 0) return FZB_E_INVALID;
    CK(cudaMemcpyAsync(w.bk4, bk4, 4 * (size_t)bklen, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(w.revbook, revbook, hf_revbook_bytes(bklen), cudaMemcpyHostToDevice, s));
    if (pinned) {  // the uploads read the pinned buffers until they have run
        CK(cudaEventRecord(stage.done, s));
        stage.pending = true;
    }
    return huff_encode_sub(d_in, n, bklen, w.bk4, w.revbook, sublen, d_out, d_out_size, d_work, work_bytes,
                           stream);
}

}  // namespace

extern "C" {

int fzb_huff_encode(const uint16_t* d_in, uint64_t n, uint32_t bklen, const uint32_t* d_bk4,
                    const uint8_t* d_revbook, void* d_out, uint64_t* d_out_size, void* d_work,
                    size_t work_bytes, void* stream) {
    return huff_encode_sub(d_in, n, bklen, d_bk4, d_revbook, kHfSublen, d_out, d_out_size, d_work, work_bytes,
                           stream);
}

int fzb_huff_encode_fine(const uint16_t* d_in, uint64_t n, uint32_t bklen, const uint32_t* d_bk4,
                         const uint8_t* d_revbook, void* d_out, uint64_t* d_out_size, void* d_work,
                         size_t work_bytes, void* stream) {
    return huff_encode_sub(d_in, n, bklen, d_bk4, d_revbook, kHfSublenFine, d_out, d_out_size, d_work,
                           work_bytes, stream);
}

int fzb_huff_compress(const uint16_t* d_in, uint64_t n, uint32_t bklen, void* d_out,
                      uint64_t* d_out_size, void* d_work, size_t work_bytes, void* stream) {
    return huff_compress_sub(d_in, n, bklen, kHfSublen, d_out, d_out_size, d_work, work_bytes, stream);
}

int fzb_huff_compress_fine(const uint16_t* d_in, uint64_t n, uint32_t bklen, void* d_out,
                           uint64_t* d_out_size, void* d_work, size_t work_bytes, void* stream) {
    return huff_compress_sub(d_in, n, bklen, kHfSublenFine, d_out, d_out_size, d_work, work_bytes, stream);
}

int fzb_huff_decode(const void* d_in, uint64_t in_bytes, uint64_t n, uint32_t bklen, uint16_t* d_out,
                    void* d_work, size_t work_bytes, void* stream) {
    if (!d_in || !d_out || !hf_args_ok(n, bklen) || in_bytes < 128) return FZB_E_INVALID;
    if (reinterpret_cast<uintptr_t>(d_in) & 3) return FZB_E_INVALID;
    if (!d_work || work_bytes < kCtrlBytes) return FZB_E_WORKSPACE;
    cudaStream_t s = S(stream);
    uint32_t* err = static_cast<uint32_t*>(d_work);
    CK(cudaMemsetAsync(err, 0, kCtrlBytes, s));
    return launch_hf_decode(static_cast<const uint8_t*>(d_in), in_bytes, n, bklen, d_out, err, s) == 0
               ? FZB_OK : FZB_E_CUDA;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched LorenzoQuant -> Bitshuffle -> RZE over many fields: one reset
// kernel, one value-base kernel for every field, the slab kernel of each
// field the single-field call codes with one, one persistent chunk kernel
// over the (field, chunk) units of the others and two assembly kernels,
// capturable in a CUDA graph.
// ---------------------------------------------------------------------------
namespace {

struct BatchPlan {
    BatchArgs args;
    uint32_t mm_grid_x;
    unsigned lq_grid;
    size_t smem;
    std::vector<FwdArgs> slab;  // fields coded by a slab kernel (host copies of their arguments)
    unsigned sms = 148;
};

// A field the single-field call would code with a slab kernel (3-D, nx a
// power of two in [32, 1024], whole-row chunks, no padding).
bool batch_slab_field(const Geometry& g, uint64_t n_total) {
    const uint32_t nx = g.nx;
    return g.ndim == 3 && nx >= 32 && nx <= 1024 && (nx & (nx - 1)) == 0 &&
           g.ny % ((uint32_t)kChunkCodes / nx) == 0 && g.nfield == n_total;
}

struct BatchLayout {
    size_t desc_bytes;
    std::vector<size_t> field_off;
    size_t total;
};

BatchLayout batch_layout(const fzb_batch_field* f, int nf) {
    BatchLayout L;
    L.desc_bytes = align256(sizeof(BatchField) * (size_t)nf) + align256(8ull * nf + 64);
    size_t off = L.desc_bytes;
    for (int i = 0; i < nf; i++) {
        L.field_off.push_back(off);
        off += align256(carve(nullptr, f[i].n_total, f[i].cap).need);
    }
    L.total = off;
    return L;
}

int batch_check(const fzb_batch_field& f, Geometry* g) {
    int rc = geometry(f.n_total, f.dims, g);
    if (rc) return rc;
    if (!f.d_in || !f.d_count || !f.d_eb_state || !f.d_rze || !f.d_rze_size) return FZB_E_INVALID;
    if (f.cap && (!f.d_err || !f.d_idx)) return FZB_E_INVALID;
    if (f.eb_mode < FZB_ABS || f.eb_mode > FZB_NOA || !(f.eb > 0.0f)) return FZB_E_INVALID;
    return FZB_OK;
}

}  // namespace

extern "C" {

size_t fzb_batch_workspace_bytes(const fzb_batch_field* fields, int nfields) {
    if (!fields || nfields <= 0) return 0;
    return batch_layout(fields, nfields).total;
}

void* fzb_batch_create(const fzb_batch_field* fields, int nfields, const fzb_batch_tuning* tuning, void* d_work,
                       size_t work_bytes, int* status) {
    int dummy = 0;
    int* st = status ? status : &dummy;
    *st = FZB_E_INVALID;
    if (!fields || nfields <= 0 || !d_work) return nullptr;
    const BatchLayout L = batch_layout(fields, nfields);
    if (work_bytes < L.total) {
        *st = FZB_E_WORKSPACE;
        return nullptr;
    }
    int dev = 0, sms = 148, max_smem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    uint8_t* base = static_cast<uint8_t*>(d_work);
    std::vector<BatchField> hf((size_t)nfields);
    std::vector<char> is_slab((size_t)nfields, 0);
    size_t smem = 0;
    uint32_t mm_grid = 1;
    for (int i = 0; i < nfields; i++) {
        const fzb_batch_field& f = fields[i];
        Geometry g;
        const int rc = batch_check(f, &g);
        if (rc) {
            *st = rc;
            return nullptr;
        }
        const Work w = carve(base + L.field_off[i], f.n_total, f.cap);
        BatchField& b = hf[i];
        b.a = fwd_args(g, w, f.d_in, f.n_total, f.d_eb_state, f.radius, f.zigzag, nullptr, f.cap);
        b.m = asm_args(w, b.a, true, f.d_rze, f.d_rze_size, f.d_err, f.d_idx, f.d_count);
        b.in = f.d_in;
        b.n = f.n_total;
        b.pmin = w.pmin;
        b.pmax = w.pmax;
        b.mm_done = w.mm_done;
        b.eb_state = f.d_eb_state;
        b.mode = f.eb_mode;
        b.user_eb = f.eb;
        b.vb_given = f.value_base;
        b.scan = (f.eb_mode != FZB_ABS && !(f.value_base > 0.0f)) ? 1u : 0u;
        const uint64_t per_sm_parts = (tuning && tuning->scan_parts > 0) ? (uint64_t)tuning->scan_parts : 4u;
        uint64_t want = (f.n_total / 4 + 255) / 256;
        uint64_t parts = want < per_sm_parts * sms ? want : per_sm_parts * sms;
        if (parts < 1) parts = 1;
        if (parts > (uint64_t)kMaxParts) parts = kMaxParts;
        b.mm_parts = b.scan ? (uint32_t)parts : 1u;
        if (b.mm_parts > mm_grid) mm_grid = b.mm_parts;
        const bool rowal = (g.ndim == 1) || (g.nx % 32 == 0);
        b.kind = g.ndim == 1 ? 0u : g.ndim == 2 ? (rowal ? 1u : 2u) : (rowal ? 3u : 4u);
        b.n_chunks = (uint32_t)chunks_of(f.n_total);
        is_slab[i] = batch_slab_field(g, f.n_total) && !(flags_env() & 1) && !(tuning && tuning->flat_tiles);
        if (!is_slab[i]) {
            const size_t sm = lq_smem_bytes(g, true);
            if (sm > smem) smem = sm;
        }
    }
    if ((int)smem > max_smem) {
        *st = FZB_E_INVALID;
        return nullptr;
    }
    // field order of the unit ranges: the chunk kernel's fields first (in
    // the tuned order), the slab kernels' fields after them
    std::vector<uint32_t> order((size_t)nfields), begin((size_t)nfields);
    for (int i = 0; i < nfields; i++) order[i] = (uint32_t)i;
    if (tuning && tuning->order == 1)
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t x, uint32_t y) { return hf[x].n_chunks > hf[y].n_chunks; });
    std::stable_partition(order.begin(), order.end(), [&](uint32_t x) { return !is_slab[x]; });
    uint64_t units = 0, lq_units = 0;
    for (int i = 0; i < nfields; i++) {
        begin[i] = (uint32_t)units;
        units += hf[order[i]].n_chunks;
        if (!is_slab[order[i]]) lq_units = units;
    }
    if (units >= (1ull << 31)) return nullptr;
    // descriptors: [BatchField x n][order x n][begin x n][counter]
    std::vector<uint8_t> desc(L.desc_bytes, 0);
    std::memcpy(desc.data(), hf.data(), sizeof(BatchField) * hf.size());
    const size_t o_order = align256(sizeof(BatchField) * (size_t)nfields);
    std::memcpy(desc.data() + o_order, order.data(), 4ull * nfields);
    std::memcpy(desc.data() + o_order + 4ull * nfields, begin.data(), 4ull * nfields);
    const size_t o_counter = o_order + 8ull * nfields;
    if (cudaMemcpy(base, desc.data(), desc.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        *st = FZB_E_CUDA;
        return nullptr;
    }
    for (int i = 0; i < nfields; i++)  // control words (scan counters start at zero)
        if (cudaMemset(base + L.field_off[i], 0, kCtrlBytes) != cudaSuccess) {
            *st = FZB_E_CUDA;
            return nullptr;
        }
    auto* p = new BatchPlan();
    p->args.fields = reinterpret_cast<const BatchField*>(base);
    p->args.nfields = (uint32_t)nfields;
    p->args.unit_order = reinterpret_cast<const uint32_t*>(base + o_order);
    p->args.unit_begin = reinterpret_cast<const uint32_t*>(base + o_order + 4ull * nfields);
    p->args.total_units = (uint32_t)units;
    p->args.lq_units = (uint32_t)lq_units;
    p->args.counter = reinterpret_cast<uint32_t*>(base + o_counter);
    p->mm_grid_x = mm_grid;
    p->sms = (unsigned)sms;
    for (int i = 0; i < nfields; i++)
        if (is_slab[order[i]]) p->slab.push_back(hf[order[i]].a);
    const int per_sm = (tuning && tuning->ctas_per_sm > 0) ? tuning->ctas_per_sm : 2;
    const uint64_t grid = (uint64_t)per_sm * (uint64_t)sms;
    p->lq_grid = (unsigned)(grid < lq_units ? grid : lq_units);
    if (p->lq_grid == 0) p->lq_grid = 1;
    p->smem = smem;
    *st = FZB_OK;
    return p;
}

int fzb_batch_launch(void* batch, void* stream) {
    if (!batch) return FZB_E_INVALID;
    const BatchPlan* p = static_cast<const BatchPlan*>(batch);
    cudaStream_t s = S(stream);
    TraceScope ts(s, "batch_lq_bs_rze");
    if (launch_batch_scan(p->args, p->mm_grid_x, s) != 0) return FZB_E_CUDA;
    for (const FwdArgs& a : p->slab) {  // the slab kernels of the single-field call
        const int rc = (lq3d_tma_supported(a) && !(flags_env() & 2)) ? launch_lq3d_tma(a, 2 * p->sms, s)
                                                                      : launch_lq3d_slab(a, 2 * p->sms, s);
        if (rc != 0) return FZB_E_CUDA;
    }
    return launch_batch_code(p->args, p->lq_grid, p->smem, s) == 0 ? FZB_OK : FZB_E_CUDA;
}

void fzb_batch_destroy(void* batch) { delete static_cast<BatchPlan*>(batch); }

int fzb_batch_autotune(const fzb_batch_field* fields, int nfields, void* d_work, size_t work_bytes, void* stream,
                       fzb_batch_tuning* best, float* best_ms) {
    if (!best) return FZB_E_INVALID;
    cudaStream_t s = S(stream);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best_t = 1e30f;
    int rc = FZB_OK;
    auto trial = [&](const fzb_batch_tuning& t) {
        if (rc != FZB_OK) return;
        int st = 0;
        void* p = fzb_batch_create(fields, nfields, &t, d_work, work_bytes, &st);
        if (!p) {
            rc = st;
            return;
        }
        float tmin = 1e30f;
        for (int rep = 0; rep < 3 && rc == FZB_OK; rep++) {  // first run warms up
            if (cudaEventRecord(e0, s) != cudaSuccess) rc = FZB_E_CUDA;
            if (rc == FZB_OK) rc = fzb_batch_launch(p, stream);
            if (rc == FZB_OK && cudaEventRecord(e1, s) != cudaSuccess) rc = FZB_E_CUDA;
            if (rc == FZB_OK && cudaEventSynchronize(e1) != cudaSuccess) rc = FZB_E_CUDA;
            float ms = 0;
            if (rc == FZB_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = FZB_E_CUDA;
            if (rc == FZB_OK && rep > 0 && ms < tmin) tmin = ms;
        }
        fzb_batch_destroy(p);
        if (rc == FZB_OK && tmin < best_t) {
            best_t = tmin;
            *best = t;
        }
    };
    // coordinate search: CTAs per SM x order, then the tile shape, then the
    // scan granularity, each from the best shape so far
    for (int order = 0; order < 2; order++)
        for (int per_sm = 1; per_sm <= 3; per_sm++) trial(fzb_batch_tuning{per_sm, order, 0, 4});
    if (rc == FZB_OK) {
        fzb_batch_tuning t = *best;
        t.flat_tiles = 1;
        trial(t);
    }
    if (rc == FZB_OK) {
        const fzb_batch_tuning b = *best;
        for (int parts : {1, 2, 8}) {
            fzb_batch_tuning t = b;
            t.scan_parts = parts;
            trial(t);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_ms) *best_ms = best_t;
    return rc;
}

}  // extern "C"
