// fzb_select_abi.cu -- C ABI of the per-chunk coder selector (fzb_sel_*,
// fzb_mlp_*): workspace layout, the exhaustive / learned / fixed encode
// paths and the chunk-container decoder.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/fzb.h"
#include "fzb_kernels.cuh"

using namespace fzb;

namespace {

inline size_t a256(size_t v) { return (v + 255) & ~(size_t)255; }

struct SelWork {
    uint8_t* slots;
    uint32_t* sizes;
    uint8_t* params;
    uint8_t* scratch;
    uint32_t* subsizes;
    uint32_t* hf_freq;
    uint32_t* hf_book;
    uint8_t* tags;
    uint8_t* want;
    float* feats;
    float* pred;
    unsigned long long* offs;
    unsigned long long* out_size_tmp;
    size_t need;
};

SelWork sel_carve(void* base, uint64_t nch) {
    SelWork w{};
    uint8_t* p = static_cast<uint8_t*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        uint8_t* q = p ? p + off : nullptr;
        off += a256(bytes);
        return q;
    };
    w.slots = take(nch * kSelCoders * (size_t)kSelSlot);
    w.sizes = reinterpret_cast<uint32_t*>(take(4 * nch * kSelCoders));
    w.params = take(nch * kSelCoders);
    w.scratch = take(nch * 4 * (size_t)kChunkBytes);
    w.subsizes = reinterpret_cast<uint32_t*>(take(4 * nch * 4));
    w.hf_freq = reinterpret_cast<uint32_t*>(take(4 * nch * kSelBk));
    w.hf_book = reinterpret_cast<uint32_t*>(take(4 * nch * kSelBk));
    w.tags = take(nch);
    w.want = take(nch);
    w.feats = reinterpret_cast<float*>(take(4 * nch * kSelFeat));
    w.pred = reinterpret_cast<float*>(take(4 * nch * kSelCoders));
    w.offs = reinterpret_cast<unsigned long long*>(take(8 * nch));
    w.out_size_tmp = reinterpret_cast<unsigned long long*>(take(8));
    w.need = off;
    return w;
}

inline uint64_t sel_chunks(uint64_t n) { return (n + kSelCodes - 1) / kSelCodes; }

SelArgs sel_args(const SelWork& w, const uint16_t* codes, uint64_t n) {
    SelArgs a{};
    a.codes = codes;
    a.n = n;
    a.slots = w.slots;
    a.sizes = w.sizes;
    a.params = w.params;
    a.scratch = w.scratch;
    a.subsizes = w.subsizes;
    a.hf_freq = w.hf_freq;
    a.hf_book = w.hf_book;
    a.tags = w.tags;
    return a;
}

#define CK(call)                                      \
    do {                                              \
        if ((call) != cudaSuccess) return FZB_E_CUDA; \
    } while (0)

inline int rc_of(int e) { return e == 0 ? FZB_OK : FZB_E_CUDA; }

bool args_ok(const uint16_t* d_codes, uint64_t n) { return d_codes && n > 0 && n < (1ull << 31); }

}  // namespace

extern "C" {

uint64_t fzb_sel_chunks(uint64_t n) { return sel_chunks(n); }

size_t fzb_sel_workspace_bytes(uint64_t n) {
    if (n == 0 || n >= (1ull << 31)) return 0;
    return sel_carve(nullptr, sel_chunks(n)).need;
}

uint64_t fzb_sel_max_bytes(uint64_t n) {
    const uint64_t nch = sel_chunks(n);
    return 16 + 2 * ((nch + 3) & ~3ull) + 4 * nch + nch * (uint64_t)kSelBytes;
}

int fzb_sel_features(const uint16_t* d_codes, uint64_t n, float* d_feats, void* stream) {
    if (!args_ok(d_codes, n) || !d_feats) return FZB_E_INVALID;
    TraceScope ts(static_cast<cudaStream_t>(stream), "sel_features");
    return rc_of(launch_sel_features(d_codes, n, d_feats, static_cast<cudaStream_t>(stream)));
}

int fzb_sel_trial(const uint16_t* d_codes, uint64_t n, uint32_t* d_sizes, void* d_work, size_t work_bytes,
                  void* stream) {
    if (!args_ok(d_codes, n) || !d_sizes) return FZB_E_INVALID;
    const uint64_t nch = sel_chunks(n);
    SelWork w = sel_carve(d_work, nch);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SelArgs a = sel_args(w, d_codes, n);
    CK(cudaMemsetAsync(w.sizes, 0xff, 4 * nch * kSelCoders, s));
    int rc;
    {
        TraceScope ts(s, "sel_trial_coders");
        rc = launch_sel_coders(a, (uint32_t)nch, 0xFu, s);
    }
    if (rc) return FZB_E_CUDA;
    CK(cudaMemcpyAsync(d_sizes, w.sizes, 4 * nch * kSelCoders, cudaMemcpyDeviceToDevice, s));
    return FZB_OK;
}

int fzb_sel_encode(const uint16_t* d_codes, uint64_t n, int mode, const float* d_params, void* d_out,
                   uint64_t* d_out_size, uint8_t* d_tags, void* d_work, size_t work_bytes, void* stream) {
    if (!args_ok(d_codes, n) || !d_out || !d_out_size) return FZB_E_INVALID;
    if (mode < FZB_SEL_EXHAUSTIVE || mode > FZB_SEL_FIXED(3)) return FZB_E_INVALID;
    if (mode == FZB_SEL_LEARNED && !d_params) return FZB_E_INVALID;
    const uint64_t nch = sel_chunks(n);
    SelWork w = sel_carve(d_work, nch);
    if (!d_work || work_bytes < w.need) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SelArgs a = sel_args(w, d_codes, n);
    const uint32_t nc = (uint32_t)nch;
    CK(cudaMemsetAsync(w.sizes, 0xff, 4 * nch * kSelCoders, s));
    CK(cudaMemsetAsync(w.params, 0, nch * kSelCoders, s));
    int rc = 0;
    if (mode == FZB_SEL_EXHAUSTIVE) {  // every coder on every chunk, keep the smallest
        {
            TraceScope ts(s, "sel_coders_all");
            rc = launch_sel_coders(a, nc, 0xFu, s);
        }
        if (!rc) rc = launch_sel_choose(a, nc, 0, nullptr, s);
    } else {
        const float* pred = nullptr;
        if (mode == FZB_SEL_LEARNED) {
            {
                TraceScope ts(s, "sel_features");
                rc = launch_sel_features(d_codes, n, w.feats, s);
            }
            if (!rc) {
                TraceScope ts(s, "mlp_forward");
                rc = launch_mlp_forward(d_params, w.feats, w.pred, nc, s);
            }
            pred = w.pred;
        }
        // pick, run the picked coder only, then try the others where it did not fit
        if (!rc) rc = launch_sel_choose(a, nc, mode, pred, s);
        if (!rc) rc = launch_sel_tag_mask(a, nc, w.want, s);
        if (!rc) {
            SelArgs b = a;
            b.want = w.want;
            TraceScope ts(s, "sel_coders_chosen");
            rc = launch_sel_coders(b, nc, 0xFu, s);
        }
        if (!rc) rc = launch_sel_fallback_mask(a, nc, w.want, s);
        if (!rc) {
            SelArgs b = a;
            b.want = w.want;
            rc = launch_sel_coders(b, nc, 0xFu, s);
        }
        if (!rc) rc = launch_sel_choose(a, nc, mode, pred, s);
    }
    if (!rc) {
        TraceScope ts(s, "sel_container");
        rc = launch_sel_container(a, nc, static_cast<uint8_t*>(d_out), reinterpret_cast<unsigned long long*>(d_out_size),
                                  w.offs, s);
    }
    if (rc) return FZB_E_CUDA;
    if (d_tags) CK(cudaMemcpyAsync(d_tags, w.tags, nch, cudaMemcpyDeviceToDevice, s));
    return FZB_OK;
}

// Host-driven decoder: reads the container header, then decodes every
// chunk with its coder's decoder into d_codes (n codes).
int fzb_sel_decode(const void* d_in, uint64_t in_bytes, uint16_t* d_codes, uint64_t n, void* d_work,
                   size_t work_bytes, void* stream) {
    if (!d_in || !d_codes || n == 0 || n >= (1ull << 31) || in_bytes < 16) return FZB_E_INVALID;
    const uint64_t nch = sel_chunks(n);
    const size_t need = fzb_workspace_bytes(kSelCodes, 0) + 2 * kSelBytes + 256;
    if (!d_work || work_bytes < need) return FZB_E_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint8_t* in = static_cast<const uint8_t*>(d_in);
    uint32_t h[4];
    CK(cudaMemcpyAsync(h, in, 16, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h[0] != 0x43535A46u || h[1] != nch || h[2] != (uint32_t)n || h[3] != (uint32_t)kSelCodes)
        return FZB_E_MALFORMED;
    const uint64_t pad = (nch + 3) & ~3ull;
    const uint64_t hdr = 16 + 2 * pad + 4 * nch;
    if (in_bytes < hdr) return FZB_E_MALFORMED;
    std::vector<uint8_t> meta(hdr);
    CK(cudaMemcpyAsync(meta.data(), in, hdr, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const uint8_t* tags = meta.data() + 16;
    const uint8_t* params = tags + pad;
    const uint32_t* sizes = reinterpret_cast<const uint32_t*>(params + pad);
    uint8_t* ws = static_cast<uint8_t*>(d_work);
    uint8_t* tmp = ws + a256(fzb_workspace_bytes(kSelCodes, 0));  // 64 KiB staging
    const size_t wsz = fzb_workspace_bytes(kSelCodes, 0);
    uint64_t off = hdr;
    for (uint64_t c = 0; c < nch; c++) {
        const uint32_t cnt = (uint32_t)((n - c * kSelCodes) < (uint64_t)kSelCodes ? n - c * kSelCodes : kSelCodes);
        const uint32_t sz = sizes[c];
        if (off + sz > in_bytes) return FZB_E_MALFORMED;
        uint16_t* dst = d_codes + c * kSelCodes;
        int rc = FZB_OK;
        switch (tags[c]) {
            case 0:  // RZE stream of the bitshuffled chunk
                rc = fzb_rze_decode(in + off, sz, 2ull * cnt, tmp, ws, wsz, stream);
                if (!rc) rc = fzb_bitshuffle(tmp, 2ull * cnt, kChunkBytes, 2, 1, dst, stream);
                break;
            case 1: rc = fzb_rle_decode(in + off, cnt, 2, dst, ws, wsz, stream); break;
            case 2: rc = fzb_bitpack_decode(in + off, cnt, 2, params[c], dst, stream); break;
            case 3: rc = fzb_huff_decode(in + off, sz, cnt, kSelBk, dst, ws, wsz, stream); break;
            default: return FZB_E_MALFORMED;
        }
        if (rc) return rc;
        const int st = fzb_workspace_status(ws, stream);
        if (st) return st;
        off += (sz + 3) & ~3u;
    }
    return FZB_OK;
}

int fzb_mlp_forward(const float* d_params, const float* d_x, float* d_y, uint32_t batch, void* stream) {
    if (!d_params || !d_x || !d_y || batch == 0) return FZB_E_INVALID;
    return rc_of(launch_mlp_forward(d_params, d_x, d_y, batch, static_cast<cudaStream_t>(stream)));
}

int fzb_mlp_grad(const float* d_params, const float* d_x, const float* d_t, uint32_t batch, int loss_kind,
                 float* d_grad, float* d_loss, void* stream) {
    if (!d_params || !d_x || !d_t || !d_grad || !d_loss || batch == 0) return FZB_E_INVALID;
    if (loss_kind != FZB_MLP_MSE && loss_kind != FZB_MLP_REGRET) return FZB_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CK(cudaMemsetAsync(d_grad, 0, sizeof(float) * kMlpParams, s));
    CK(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
    return rc_of(launch_mlp_backward(d_params, d_x, d_t, batch, d_grad, d_loss, loss_kind, s));
}

int fzb_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, float lr, int step, void* stream) {
    if (!d_params || !d_grad || !d_m || !d_v || step < 1) return FZB_E_INVALID;
    return rc_of(launch_mlp_adam(d_params, d_grad, d_m, d_v, lr, step, static_cast<cudaStream_t>(stream)));
}

}  // extern "C"
