// Test infrastructure: drives the reference's own stage classes (compiled
// from the reference sources into oracle/_ref/libfzref.so) on caller-owned
// device buffers, so GPU tests can compare our kernels with the reference
// kernels on identical inputs.  Never linked into the product.
//
// Each entry point returns 0 on success, -1 on a reference exception (the
// message is available from ref_last_error()).
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "coders/bitpack/bitpack_stage.h"
#include "coders/huffman/huffman_stage.h"
#include "coders/rle/rle.h"
#include "coders/rze/rze_stage.h"
#include "fused/lorenzo_quant/lorenzo_quant.h"
#include "mem/mempool.h"
#include "predictors/diff/diff.h"
#include "predictors/lorenzo/lorenzo_stage.h"
#include "quantizers/quantizer/quantizer.h"
#include "shufflers/bitshuffle/bitshuffle_stage.h"
#include "transforms/negabinary/negabinary_stage.h"
#include "transforms/zigzag/zigzag_stage.h"
#include "ref_scrub.cuh"

using namespace fz;

static std::string g_err;
// byte written over every SM's shared memory before the reference's
// LorenzoQuant runs (ref_scrub.cuh); -1 leaves shared memory as it is
static int g_fill = 0;

// The reference's Huffman coarse encoder starts its host scan of the
// partition cell counts at h_par_entry[0] without writing it
// (phf/hf_kernels.cu:419-420); that array is pinned memory from
// MemoryPool::allocatePersistentPinned (src/mem/mempool.cpp:258), which a
// recycled pinned allocation can hand over with stale bytes, shifting every
// partition of the bitstream.  The parity build compiles mempool.cpp with
// its cudaMallocHost call routed here (oracle/Makefile), so that the array
// starts at zero as on a fresh allocation.
extern "C" cudaError_t fzref_zeroed_malloc_host(void** ptr, size_t bytes) {
    const cudaError_t e = cudaHostAlloc(ptr, bytes, cudaHostAllocDefault);
    if (e == cudaSuccess && *ptr) std::memset(*ptr, 0, bytes);
    return e;
}

extern "C" const char* ref_last_error() { return g_err.c_str(); }

extern "C" void ref_set_shared_fill(int byte) { g_fill = byte; }

extern "C" int ref_fill_shared(int byte) {
    return ref_scrub::fill_shared((uint8_t)byte, 0) == cudaSuccess ? 0 : -1;
}

#define GUARD_BEGIN try {
#define GUARD_END                                   \
    }                                               \
    catch (const std::exception& e) {               \
        g_err = e.what();                           \
        return -1;                                  \
    }                                               \
    catch (...) {                                   \
        g_err = "unknown exception";                \
        return -1;                                  \
    }

// LorenzoQuantStage<float,uint16_t> forward (lorenzo_quant.cu:583-719) and
// postStreamSync (:722-766).  Writes codes/outlier buffers; *count_out is the
// device outlier counter (may exceed the capacity); hdr receives the 44-byte
// serialized LorenzoQuantConfig.
extern "C" int ref_lq_fwd(const float* d_in, size_t n, size_t nx, size_t ny, size_t nz,
                          float eb, int mode, int radius, float outlier_cap, int zigzag,
                          uint16_t* d_codes, float* d_err, uint32_t* d_idx,
                          uint32_t* d_count, uint8_t* hdr44) {
    GUARD_BEGIN
    if (g_fill >= 0 && ref_scrub::fill_shared((uint8_t)g_fill, 0) != cudaSuccess)
        throw std::runtime_error("shared-memory fill failed");
    MemoryPool pool(MemoryPoolConfig(n * sizeof(float), 3.0f));
    LorenzoQuantStage<float, uint16_t>::Config cfg;
    cfg.error_bound = eb;
    cfg.quant_radius = radius;
    cfg.outlier_capacity = outlier_cap;
    cfg.dims = {nx, ny, nz};
    cfg.eb_mode = static_cast<ErrorBoundMode>(mode);
    cfg.zigzag_codes = zigzag != 0;
    LorenzoQuantStage<float, uint16_t> st(cfg);
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<float*>(d_in)}, {d_codes, d_err, d_idx, d_count},
               {n * sizeof(float)});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    st.postStreamSync(s);
    if (hdr44) st.serializeHeader(0, hdr44, 128);
    GUARD_END
    return 0;
}

extern "C" int ref_lq_inv(const uint16_t* d_codes, const float* d_err, const uint32_t* d_idx,
                          const uint32_t* d_count, size_t n, size_t cap,
                          const uint8_t* hdr44, float* d_out) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(n * sizeof(float), 3.0f));
    LorenzoQuantStage<float, uint16_t> st;
    st.deserializeHeader(hdr44, 44);
    st.setInverse(true);
    cudaStream_t s = 0;
    st.execute(s, &pool,
               {const_cast<uint16_t*>(d_codes), const_cast<float*>(d_err),
                const_cast<uint32_t*>(d_idx), const_cast<uint32_t*>(d_count)},
               {d_out}, {n * sizeof(uint16_t), cap * sizeof(float), cap * sizeof(uint32_t), 4});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    GUARD_END
    return 0;
}

extern "C" int ref_bitshuffle(const void* d_in, size_t bytes, uint32_t block, int ew,
                              int inverse, void* d_out) {
    GUARD_BEGIN
    BitshuffleStage st;
    st.setBlockSize(block);
    st.setElementWidth(ew);
    st.setInverse(inverse != 0);
    cudaStream_t s = 0;
    st.execute(s, nullptr, {const_cast<void*>(d_in)}, {d_out}, {bytes});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    GUARD_END
    return 0;
}

extern "C" int ref_rze_encode(const void* d_in, size_t bytes, void* d_out, size_t* out_bytes) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(bytes, 3.0f));
    RZEStage st;
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<void*>(d_in)}, {d_out}, {bytes});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    st.postStreamSync(s);
    *out_bytes = st.getActualOutputSize(0);
    GUARD_END
    return 0;
}

extern "C" int ref_rze_decode(const void* d_in, size_t bytes, void* d_out, size_t* out_bytes) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(bytes, 3.0f));
    RZEStage st;
    st.setInverse(true);
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<void*>(d_in)}, {d_out}, {bytes});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    *out_bytes = st.getActualOutputSize(0);
    GUARD_END
    return 0;
}

extern "C" int ref_rle_u16(const uint16_t* d_in, size_t n, void* d_out, size_t* out_bytes,
                           uint16_t* d_dec) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(n * 2, 3.0f));
    RLEStage<uint16_t> st;
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<uint16_t*>(d_in)}, {d_out}, {n * 2});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    st.postStreamSync(s);
    *out_bytes = st.getActualOutputSize(0);
    if (d_dec) {
        st.setInverse(true);
        st.execute(s, &pool, {d_out}, {d_dec}, {*out_bytes});
        if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    }
    GUARD_END
    return 0;
}

extern "C" int ref_bitpack_u16(const uint16_t* d_in, size_t n, int nbits, void* d_out,
                               size_t* out_bytes, int* nbits_used, uint16_t* d_dec) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(n * 2, 3.0f));
    BitpackStage<uint16_t> st;
    if (nbits > 0) st.setNBits((uint8_t)nbits);
    else st.setAutoDetect(true);
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<uint16_t*>(d_in)}, {d_out}, {n * 2});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    *out_bytes = st.getActualOutputSize(0);
    *nbits_used = st.getNBits();
    if (d_dec) {
        st.setInverse(true);
        st.execute(s, &pool, {d_out}, {d_dec}, {*out_bytes});
        if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    }
    GUARD_END
    return 0;
}

// Fine mode (setEncodeMode(Fine)).  Only whole 1024-symbol partitions are
// passed here: for a partial last partition the reference's ReVISIT-lite
// kernel reads symbols from shared memory it never filled.
extern "C" int ref_huffman_u16_fine(const uint16_t* d_in, size_t n, int bklen, void* d_out,
                                    size_t* out_bytes, uint16_t* d_dec) {
    if (n == 0 || n % 1024 != 0) return -2;
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(n * 2 + (size_t(1) << 22), 3.0f));
    HuffmanStage<uint16_t> st;
    st.setBklen((uint32_t)bklen);
    st.setEncodeMode(HuffmanEncodeMode::Fine);
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<uint16_t*>(d_in)}, {d_out}, {n * 2});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    *out_bytes = st.getActualOutputSize(0);
    if (d_dec) {
        st.setInverse(true);
        st.execute(s, &pool, {d_out}, {d_dec}, {*out_bytes});
        if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    }
    GUARD_END
    return 0;
}

extern "C" int ref_huffman_u16(const uint16_t* d_in, size_t n, int bklen, void* d_out,
                               size_t* out_bytes, uint16_t* d_dec) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(n * 2 + (size_t(1) << 22), 3.0f));
    HuffmanStage<uint16_t> st;
    st.setBklen((uint32_t)bklen);
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<uint16_t*>(d_in)}, {d_out}, {n * 2});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    *out_bytes = st.getActualOutputSize(0);
    if (d_dec) {
        st.setInverse(true);
        st.execute(s, &pool, {d_out}, {d_dec}, {*out_bytes});
        if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    }
    GUARD_END
    return 0;
}

// DifferenceStage<int32_t> / <int32_t, uint32_t> (predictors/diff/diff.cu).
extern "C" int ref_diff_i32(const void* d_in, size_t n, size_t chunk_bytes, int negabinary, int inverse,
                            void* d_out) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(n * 8 + (size_t(1) << 22), 2.0f));
    cudaStream_t s = 0;
    if (negabinary) {
        DifferenceStage<int32_t, uint32_t> st;
        st.setChunkSize(chunk_bytes);
        st.setInverse(inverse != 0);
        st.execute(s, &pool, {const_cast<void*>(d_in)}, {d_out}, {n * 4});
    } else {
        DifferenceStage<int32_t> st;
        st.setChunkSize(chunk_bytes);
        st.setInverse(inverse != 0);
        st.execute(s, &pool, {const_cast<void*>(d_in)}, {d_out}, {n * 4});
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    GUARD_END
    return 0;
}

// LorenzoStage<int32_t> (predictors/lorenzo/lorenzo_stage.cu).
extern "C" int ref_lorenzo_i32(const void* d_in, size_t n, size_t nx, size_t ny, size_t nz, int inverse,
                               void* d_out) {
    GUARD_BEGIN
    MemoryPool pool(MemoryPoolConfig(n * 8 + (size_t(1) << 22), 2.0f));
    LorenzoStage<int32_t> st;
    st.setDims(nx, ny, nz);
    st.setInverse(inverse != 0);
    cudaStream_t s = 0;
    st.execute(s, &pool, {const_cast<void*>(d_in)}, {d_out}, {n * 4});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    GUARD_END
    return 0;
}

// ZigzagStage<int32_t, uint32_t> / NegabinaryStage<int32_t, uint32_t>.
extern "C" int ref_transform_i32(int negabinary, const void* d_in, size_t n, int inverse, void* d_out) {
    GUARD_BEGIN
    cudaStream_t s = 0;
    if (negabinary) {
        NegabinaryStage<int32_t, uint32_t> st;
        st.setInverse(inverse != 0);
        st.execute(s, nullptr, {const_cast<void*>(d_in)}, {d_out}, {n * 4});
    } else {
        ZigzagStage<int32_t, uint32_t> st;
        st.setInverse(inverse != 0);
        st.execute(s, nullptr, {const_cast<void*>(d_in)}, {d_out}, {n * 4});
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    GUARD_END
    return 0;
}

// QuantizerStage<float, uint16_t / uint32_t> forward, then its inverse from
// the serialized header (quantizers/quantizer/quantizer.cu).  mode: 0 ABS,
// 1 REL, 2 NOA.  hdr receives the 36-byte QuantizerConfig; d_recon may be
// null (forward only).
template <typename TC>
static void ref_quant_run(const float* d_in, size_t n, float eb, int mode, int radius, int zigzag, int inplace,
                          float threshold, float cap_frac, void* d_codes, float* d_vals, uint32_t* d_idx,
                          uint32_t* d_count, float* d_recon, uint8_t* hdr) {
    MemoryPool pool(MemoryPoolConfig(n * 16 + (size_t(1) << 22), 2.0f));
    typename QuantizerStage<float, TC>::Config cfg;
    cfg.error_bound = eb;
    cfg.eb_mode = mode == 0 ? ErrorBoundMode::ABS : (mode == 1 ? ErrorBoundMode::REL : ErrorBoundMode::NOA);
    cfg.quant_radius = radius;
    cfg.outlier_capacity = cap_frac;
    cfg.zigzag_codes = zigzag != 0;
    cfg.inplace_outliers = inplace != 0;
    cfg.outlier_threshold = threshold;
    QuantizerStage<float, TC> st(cfg);
    cudaStream_t s = 0;
    const bool inpl = inplace && mode != 1;
    if (inpl) st.execute(s, &pool, {const_cast<float*>(d_in)}, {d_codes}, {n * 4});
    else st.execute(s, &pool, {const_cast<float*>(d_in)}, {d_codes, d_vals, d_idx, d_count}, {n * 4});
    if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    st.postStreamSync(s);
    const size_t hn = st.serializeHeader(0, hdr, 128);
    if (d_recon) {
        QuantizerStage<float, TC> inv;
        inv.deserializeHeader(hdr, hn);
        inv.setInverse(true);
        if (inpl) {
            inv.execute(s, &pool, {d_codes}, {d_recon}, {n * sizeof(TC)});
        } else {
            QuantizerConfig qc;
            std::memcpy(&qc, hdr, sizeof(qc));
            const size_t k = qc.outlier_count;
            inv.execute(s, &pool, {d_codes, d_vals, d_idx, d_count}, {d_recon}, {n * sizeof(TC), k * 4, k * 4, 4});
        }
        if (cudaStreamSynchronize(s) != cudaSuccess) throw std::runtime_error("sync failed");
    }
}

extern "C" int ref_quantizer_f32(const float* d_in, size_t n, int code_bytes, float eb, int mode, int radius,
                                 int zigzag, int inplace, float threshold, float cap_frac, void* d_codes,
                                 float* d_vals, uint32_t* d_idx, uint32_t* d_count, float* d_recon, uint8_t* hdr) {
    GUARD_BEGIN
    if (code_bytes == 2)
        ref_quant_run<uint16_t>(d_in, n, eb, mode, radius, zigzag, inplace, threshold, cap_frac, d_codes, d_vals,
                                d_idx, d_count, d_recon, hdr);
    else
        ref_quant_run<uint32_t>(d_in, n, eb, mode, radius, zigzag, inplace, threshold, cap_frac, d_codes, d_vals,
                                d_idx, d_count, d_recon, hdr);
    GUARD_END
    return 0;
}
