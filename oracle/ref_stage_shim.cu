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
#include "shufflers/bitshuffle/bitshuffle_stage.h"

using namespace fz;

static std::string g_err;

extern "C" const char* ref_last_error() { return g_err.c_str(); }

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
