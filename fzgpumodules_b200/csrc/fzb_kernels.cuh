// fzb_kernels.cuh -- kernel argument blocks and declarations shared by the
// kernel translation units and the C-ABI layer.
#pragma once

#include "fzb_rze.cuh"

#include <atomic>
#include <cstdlib>

namespace fzb {

// Raises a kernel's dynamic shared memory limit once per device: the
// attribute outlasts the call, so later launches skip the driver call.  One
// SmemAttr per kernel (a static at the launch site); devices past the eighth
// set it on every call.
struct SmemAttr {
    std::atomic<int> bytes[8] = {};
};
inline cudaError_t ensure_dyn_smem(SmemAttr& st, const void* func, int bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    if (dev >= 0 && dev < 8 && st.bytes[dev].load(std::memory_order_relaxed) >= bytes) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && dev >= 0 && dev < 8) st.bytes[dev].store(bytes, std::memory_order_relaxed);
    return e;
}

// Multiprocessor count of the current device, queried once per device (the
// first eight devices; later ones query on every call).
inline int device_sms() {
    static std::atomic<int> cache[8] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    if (dev >= 0 && dev < 8) {
        const int v = cache[dev].load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    int sms = 0;
    if (dev < 0 || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return 1;
    if (dev < 8) cache[dev].store(sms, std::memory_order_relaxed);
    return sms;
}

struct FwdArgs {
    const float* in;
    uint32_t n_total;  // elements in the code domain (>= nfield when padded)
    uint32_t nfield;   // nx * ny * nz
    uint32_t nx, ny, nz;
    uint32_t plane;        // nx * ny
    const float* ebx2_r;   // device scalar
    float radius;
    int zigzag;
    int two_piece;         // separate windows for q(k) and q(k - nx)
    uint16_t* codes;       // codes-only output
    float* out_err;
    uint32_t* out_idx;
    uint32_t cap;
    uint32_t* out_count;
    uint32_t n_chunks;
    // two-phase placement: chunk payloads go to fixed 16 KiB slots and
    // outliers to an atomically allocated staging area; assemble_* kernels
    // then write the final, ordered outputs
    uint8_t* slots;        // n_chunks * 16 KiB (+16)
    uint32_t* sizes;       // per-chunk RZE size words
    uint32_t* ocnt;        // per-chunk outlier counts
    uint32_t* obase;       // per-chunk staging offsets
    uint32_t* ostage_ctr;
    float* ostage_err;
    uint32_t* ostage_idx;
    uint32_t ostage_cap;
    uint32_t* err;
};

// Final placement of slot payloads and staged outliers.
struct AsmArgs {
    const uint8_t* slots;
    const uint32_t* sizes;   // null: outliers only
    uint32_t n_chunks;
    uint32_t orig_bytes;
    uint8_t* out;            // RZE stream
    unsigned long long* out_size;
    unsigned long long* pay_off;  // n_chunks (scratch)
    const uint32_t* ocnt;
    const uint32_t* obase;
    uint32_t* ofin;          // n_chunks (scratch)
    const float* ostage_err;
    const uint32_t* ostage_idx;
    uint32_t ostage_cap;
    float* out_err;
    uint32_t* out_idx;
    uint32_t cap;
    uint32_t* out_count;
};

struct RzeEncArgs {
    const uint8_t* in;
    uint64_t bytes;
    uint8_t* slots;
    uint32_t* sizes;
};

// Inverse-side arguments.
struct InvArgs {
    const uint8_t* rze;           // RZE stream (fused / codes path)
    uint64_t rze_bytes;
    const unsigned long long* in_off;  // per-chunk payload offsets (prepass)
    uint32_t n_chunks;
    uint32_t orig_bytes;          // RZE original byte count
    uint16_t* codes;              // codes output (codes path)
    uint8_t* bytes_out;           // plain RZE decode output
    const float* out_err;
    const uint32_t* out_idx;
    const uint32_t* out_count;
    uint32_t cap;
    const uint32_t* ostart;       // per-chunk outlier start (n_chunks + 1)
    uint32_t nx, ny, nz, plane, nfield, n_total;
    float ebx2;                   // 2 * abs_eb
    int zigzag;
    int shuffled;                 // full chunks are bitshuffled (ew = 2)
    float* out;
    uint32_t* err;
    // device-resident error bound: when set, kernels take 2 * *abs_eb_src
    // (the compressor's eb state) instead of ebx2
    const float* abs_eb_src;
    // device-side fallback: when set, a kernel does its work only if
    // *gate & gate_mask (the fused inverse flagged a case it leaves to the
    // exact kernels), so the decision needs no host round trip
    const uint32_t* gate;
    uint32_t gate_mask;
};

__device__ __forceinline__ float inv_ebx2(const InvArgs& a) {
    return a.abs_eb_src ? 2.0f * *a.abs_eb_src : a.ebx2;
}

__device__ __forceinline__ bool inv_gated_off(const InvArgs& a) {
    return a.gate != nullptr && !(*reinterpret_cast<const volatile uint32_t*>(a.gate) & a.gate_mask);
}

__global__ void minmax_kernel(const float* x, uint64_t n, float* pmin, float* pmax,
                              unsigned int* done, int mode, float user_eb, float* st);
__global__ void resolve_eb_kernel(int mode, float user_eb, float vb_given, float* st);
// Launches the chunk kernel instance for (ndim, fused, row-aligned); returns
// a cudaError_t value.
int launch_lq_chunk(int ndim, bool fused, bool rowal, const FwdArgs& a, size_t smem,
                    unsigned grid, cudaStream_t s);
// Slab-column fused 3-D kernel (see fzb_forward.cu); `grid` persistent CTAs.
int launch_lq3d_slab(const FwdArgs& a, unsigned grid, cudaStream_t s);
// Codes of a 2-D field whose rows are whole chunks (nx % 8192 == 0, no
// padding past the field), rows walked down chunk columns (fzb_rows2d.cu);
// needs a 16-byte aligned input, 8-byte aligned codes and radius <= 2^21.
bool lq_rows_supported(const FwdArgs& a);
int launch_lq_rows(const FwdArgs& a, unsigned sms, cudaStream_t s);
// TMA-fed slab kernel (fzb_slab.cu): same applicability and bytes, plus a
// 16-byte aligned input and radius <= 2^21.
bool lq3d_tma_supported(const FwdArgs& a);
int launch_lq3d_tma(const FwdArgs& a, unsigned grid, cudaStream_t s);
__global__ void bitshuffle2_kernel(const uint8_t* in, uint8_t* out, int inverse);
__global__ void bitshuffle_ballot_kernel(const uint8_t* in, uint8_t* out, uint32_t block, int ew,
                                         int inverse);
// Element widths 4 and 8: one CTA per block (fzb_forward.cu).
int launch_bitshuffle_wide(const uint8_t* in, uint8_t* out, uint64_t nfull, uint32_t block, int ew, int inverse,
                           cudaStream_t s);
__global__ void rze_encode_kernel(RzeEncArgs a);
__global__ void assemble_scan_kernel(AsmArgs a);
// Shared-memory index with one pad word per 32 entries: thread t touching
// entries k*t + j (k a power of two up to 32) stays free of bank conflicts.
__device__ __forceinline__ uint32_t pad32(uint32_t i) { return i + (i >> 5); }

// Fields of up to this many chunks take the tiled scans (assemble_scan,
// rze_prepass): one CTA per 1024 chunks, each summing the chunks before its
// tile itself, so no CTA waits for another.
constexpr uint32_t kTiledScanMax = 65536;

// FZB_DISABLE_SLAB (a test and measurement switch, default 0): bit 1 codes
// slab-shaped 3-D fields with the chunk kernel, 2 takes the cp.async slab
// kernel instead of the TMA one, 4 the per-tile fused inverse instead of the
// inverse slab kernel, 8 2-D codes with the chunk kernel instead of the row
// walk, 16 the single-CTA assembly scan and prepass instead of the tiled ones.
inline unsigned flags_env() {
    const char* v = getenv("FZB_DISABLE_SLAB");
    return v ? (unsigned)strtoul(v, nullptr, 10) & 31u : 0u;
}

// Exclusive scans of two values over a block of 1024 threads, with their
// totals (ws: 64 words of shared memory).
__device__ __forceinline__ void block_scan2_1024(uint32_t a, uint32_t b, uint32_t& ea, uint32_t& eb, uint32_t& ta,
                                                 uint32_t& tb, uint32_t* ws) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t ia = a, ib = b;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t na = __shfl_up_sync(0xffffffffu, ia, d), nb = __shfl_up_sync(0xffffffffu, ib, d);
        if (lane >= (uint32_t)d) {
            ia += na;
            ib += nb;
        }
    }
    if (lane == 31) {
        ws[warp] = ia;
        ws[32 + warp] = ib;
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t va = ws[lane], vb = ws[32 + lane];
        uint32_t xa = va, xb = vb;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t na = __shfl_up_sync(0xffffffffu, xa, d), nb = __shfl_up_sync(0xffffffffu, xb, d);
            if (lane >= (uint32_t)d) {
                xa += na;
                xb += nb;
            }
        }
        __syncwarp();
        ws[lane] = xa - va;
        ws[32 + lane] = xb - vb;
        if (lane == 31) {
            ws[64] = xa;
            ws[65] = xb;
        }
    }
    __syncthreads();
    ea = ws[warp] + ia - a;
    eb = ws[32 + warp] + ib - b;
    ta = ws[64];
    tb = ws[65];
    __syncthreads();  // ws may be reused
}
constexpr uint32_t kAsmTile = 16384;  // chunks per tile of the single-CTA assembly scan (shared memory: 2 words each)
int launch_assemble_scan(const AsmArgs& a, cudaStream_t s);
__global__ void assemble_copy_kernel(AsmArgs a);  // one warp per chunk, grid-stride
inline unsigned copy_grid(uint64_t n_chunks) {
    const uint64_t g = (n_chunks + 7) / 8;
    return (unsigned)(g < 1184 ? (g ? g : 1) : 1184);
}

__global__ void rze_prepass_kernel(const uint8_t* rze, uint64_t rze_bytes, uint32_t n_expect,
                                   uint32_t orig_expect, unsigned long long* in_off, uint32_t* err);
int launch_rze_prepass(const uint8_t* rze, uint64_t rze_bytes, uint32_t n_expect, uint32_t orig_expect,
                       unsigned long long* in_off, uint32_t* err, cudaStream_t s);
__global__ void outlier_ranges_kernel(const uint32_t* idx, const uint32_t* count, uint32_t cap,
                                      uint32_t n_chunks, uint32_t* ostart, uint32_t* err);
__global__ void rze_decode_kernel(InvArgs a);
__global__ void rze_decode_codes_kernel(InvArgs a);
__global__ void scatter_outliers_kernel(InvArgs a);
__global__ void zero_out_kernel(InvArgs a);
__global__ void lq_inverse_1d_kernel(InvArgs a);
__global__ void lq_inverse_2d_kernel(InvArgs a);
__global__ void lq_inverse_3d_kernel(InvArgs a);
__global__ void fused_inverse_3d_kernel(InvArgs a);
// Persistent slab inverse (fzb_slab_inv.cu) for nx >= 32; same results.
int launch_lq3d_inv_slab(const InvArgs& a, unsigned sms, cudaStream_t s);  // persistent grid: 3 CTAs per SM

// Exclusive scan of u32 values (fzb_coders.cu).  The source is a plain
// array (count given, or read from *cptr on the device) or the run-length
// array of an RLE stream.
struct ScanSrc {
    const uint32_t* base;     // plain array
    const uint32_t* cptr;     // optional device count
    const uint8_t* rle;       // RLE stream instead of base
    int elem;                 // RLE value width
    uint32_t n;               // upper bound of the count
};
int launch_scan_u32(const ScanSrc& a, uint32_t* out, uint32_t* tile_scratch, uint32_t* total,
                    cudaStream_t s);

// RLE and Bitpack (fzb_coders.cu); return cudaError_t values.
int launch_rle_encode(const void* in, uint32_t n, int elem, uint8_t* out, unsigned long long* out_size,
                      uint32_t* tcnt, uint32_t* starts, uint32_t* runs_total, cudaStream_t s);
int launch_rle_decode(const uint8_t* in, uint32_t n, int elem, void* out, uint32_t* offs,
                      uint32_t* tile_scratch, uint32_t* total, uint32_t* err, cudaStream_t s);
int launch_bitpack_encode(const void* in, uint64_t n, int elem, int nbits, uint8_t* nbits_dev,
                          uint8_t* out, unsigned long long* out_size, uint32_t* pmax,
                          unsigned int* done, cudaStream_t s);
int launch_bitpack_decode(const uint8_t* in, uint64_t n, int elem, int nbits, void* out, cudaStream_t s);

// Batched fused compression (fzb_forward.cu): one field's arguments.
struct BatchField {
    FwdArgs a;               // chunk kernel arguments (slots, staging, ...)
    AsmArgs m;               // assembly arguments
    const float* in;         // value-base scan
    uint64_t n;
    float* pmin;
    float* pmax;
    unsigned int* mm_done;
    float* eb_state;
    int mode;
    float user_eb;
    float vb_given;
    uint32_t mm_parts;       // blocks of the scan (1 when no scan)
    uint32_t scan;           // 1: REL/NOA scan, 0: resolve only
    uint32_t kind;           // 0 1-D, 1 2-D rows %32, 2 2-D, 3 3-D rows %32, 4 3-D
    uint32_t n_chunks;
};

struct BatchArgs {
    const BatchField* fields;
    uint32_t nfields;
    const uint32_t* unit_order;  // field index per slot
    const uint32_t* unit_begin;  // first unit (chunk) of each slot
    uint32_t total_units;        // chunks of every field (the assembly's units)
    uint32_t lq_units;           // the chunk kernel's units: the leading slots, slab fields excluded
    uint32_t* counter;           // unit dispenser
};

// Reset and the value-base scan of every field; then the chunk kernel over
// the first lq_units units and the assembly of every field.  Fields that take
// a slab kernel are launched between the two.
int launch_batch_scan(const BatchArgs& b, uint32_t mm_grid_x, cudaStream_t s);
int launch_batch_code(const BatchArgs& b, unsigned lq_grid, size_t smem, cudaStream_t s);

// Per-chunk coding with a learned selector (fzb_select.cu).
constexpr int kSelCodes = 32768;            // codes per 64 KiB chunk
constexpr int kSelBytes = 65536;
constexpr int kSelCoders = 4;               // Bitshuffle+RZE, RLE, Bitpack, Huffman
constexpr uint32_t kSelSlot = 65536 + 256;  // per (chunk, coder) output slot
constexpr uint32_t kSelNoFit = 0xffffffffu; // coder output larger than the chunk / not applicable
constexpr int kSelFeat = 16;
constexpr int kSelBk = 1024;                // Huffman book length
constexpr int kSelParts = (kSelCodes + 767) / 768;
constexpr int kMlpParams = 16 * 64 + 64 + 64 * 64 + 64 + 64 * 4 + 4;
constexpr float kMlpTau = 0.02f;            // soft-label temperature on log2 regrets

struct SelArgs {
    const uint16_t* codes;
    uint64_t n;
    const uint32_t* list;    // chunk ids (null: blockIdx)
    const uint8_t* want;     // per chunk: bit k = run coder k (null: all)
    uint8_t* slots;          // nchunks * 4 * kSelSlot
    uint32_t* sizes;         // nchunks * 4 (kSelNoFit = no output)
    uint8_t* params;         // nchunks * 4
    uint8_t* scratch;        // nchunks * 4 * 16 KiB (RZE blocks)
    uint32_t* subsizes;      // nchunks * 4
    uint32_t* hf_freq;       // nchunks * kSelBk
    uint32_t* hf_book;       // nchunks * kSelBk
    uint8_t* tags;           // nchunks
};

int launch_sel_features(const uint16_t* codes, uint64_t n, float* feats, cudaStream_t s);
int launch_sel_coders(const SelArgs& a, uint32_t nchunks, unsigned coder_mask, cudaStream_t s);
int launch_sel_choose(const SelArgs& a, uint32_t nchunks, int mode, const float* pred, cudaStream_t s);
int launch_sel_fallback_mask(const SelArgs& a, uint32_t nchunks, uint8_t* want, cudaStream_t s);
int launch_sel_tag_mask(const SelArgs& a, uint32_t nchunks, uint8_t* want, cudaStream_t s);
int launch_sel_container(const SelArgs& a, uint32_t nchunks, uint8_t* out, unsigned long long* out_size,
                         unsigned long long* offs, cudaStream_t s);
int launch_mlp_forward(const float* P, const float* X, float* Y, uint32_t batch, cudaStream_t s);
int launch_mlp_backward(const float* P, const float* X, const float* T, uint32_t batch, float* G, float* loss,
                        int kind, cudaStream_t s);
int launch_mlp_adam(float* P, const float* G, float* M, float* V, float lr, int step, cudaStream_t s);

// Launches `kernel` as a programmatic dependent of the previous kernel on
// `s` (it may start before that kernel ends and must wait with
// griddepcontrol.wait before reading its results); a plain launch when the
// attribute is refused.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem,
                                    cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
        e = cudaGetLastError();
    }
    return e;
}

// Per-kernel CUDA-event timing (fzb_trace.cu): a TraceScope around a launch
// records an event pair on the launching stream while tracing is enabled.
extern bool g_trace_on;
class TraceScope {
public:
    TraceScope(cudaStream_t s, const char* name);
    ~TraceScope();
    TraceScope(const TraceScope&) = delete;
    TraceScope& operator=(const TraceScope&) = delete;

private:
    cudaStream_t s_;
    cudaEvent_t end_;
};

// PHF Huffman, coarse mode (fzb_huffman.cu, codebook in fzb_hfbook.cpp).
constexpr int kHfSublen = 768;       // coarse mode partition (hf_bk.cc:28-37)
constexpr int kHfSublenFine = 1024;  // fine mode partition (hf_buf.cc:46-49)
int launch_hf_histogram(const uint16_t* in, uint64_t n, uint32_t bklen, uint32_t* freq, int sms,
                        cudaStream_t s);
int launch_hf_encode(const uint16_t* in, uint64_t n, const uint32_t* bk4, uint32_t bklen, uint32_t sublen,
                     const uint8_t* d_revbook, uint8_t* out, unsigned long long* out_size,
                     uint32_t* slots, uint32_t* par_nbit, uint32_t* par_ncell, uint32_t* par_entry,
                     uint32_t* tiles, uint32_t* ncell_total, uint32_t* ctrl, int sms, cudaStream_t s);
int launch_hf_decode(const uint8_t* blob, uint64_t blob_bytes, uint64_t n, uint32_t bklen,
                     uint16_t* out, uint32_t* err, cudaStream_t s);
int build_huffman_book(const uint32_t* freq, uint32_t bklen, uint32_t* bk4, uint8_t* revbook);

}  // namespace fzb
