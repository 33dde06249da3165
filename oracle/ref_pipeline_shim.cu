// Test infrastructure: runs the reference's own fz::Pipeline (compiled from
// its sources into oracle/_ref/libfzref_pipe.so) on caller-owned device
// buffers and writes its FZM file, so tests can compare the container bytes
// and the decompressed values with this library's pipeline on identical
// inputs.  Never linked into the product.
//
// chain 0: LorenzoQuant -> RLE<uint16_t>              (codes port)
// chain 1: LorenzoQuant -> Bitshuffle(16384, ew 2) -> RZE(16384, 4)
// chain 2: LorenzoQuant -> Huffman<uint16_t>(bklen 1024)
// Returns 0, or -1 with the exception text in ref_pipe_last_error().
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "pipeline/compressor.h"
#include "predictors/diff/diff.h"
#include "predictors/lorenzo/lorenzo_stage.h"
#include "quantizers/quantizer/quantizer.h"
#include "transforms/negabinary/negabinary_stage.h"
#include "transforms/zigzag/zigzag_stage.h"
#include "ref_scrub.cuh"

using namespace fz;

static std::string g_err;
// byte written over every SM's shared memory before each reference compress
// (ref_scrub.cuh); -1 leaves shared memory as it is
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

extern "C" const char* ref_pipe_last_error() { return g_err.c_str(); }

extern "C" void ref_pipe_set_shared_fill(int byte) { g_fill = byte; }

static void fill_shared() {
    if (g_fill >= 0 && ref_scrub::fill_shared((uint8_t)g_fill, 0) != cudaSuccess)
        throw std::runtime_error("shared-memory fill failed");
}

extern "C" int ref_pipeline_fzm(int chain, const float* d_in, size_t n, size_t x, size_t y, size_t z, float eb,
                                int mode, int radius, float outlier_cap, int zigzag, int preallocate,
                                const char* path, float* d_decomp, size_t* decomp_bytes, size_t* comp_bytes) {
    try {
        Pipeline p(n * sizeof(float), preallocate ? MemoryStrategy::PREALLOCATE : MemoryStrategy::MINIMAL, 3.0f);
        p.setDims(x, y, z);
        LorenzoQuantStage<float, uint16_t>::Config cfg;
        cfg.error_bound = eb;
        cfg.quant_radius = radius;
        cfg.outlier_capacity = outlier_cap;
        cfg.eb_mode = static_cast<ErrorBoundMode>(mode);
        cfg.zigzag_codes = zigzag != 0;
        auto* lq = p.addStage<LorenzoQuantStage<float, uint16_t>>(cfg);
        if (chain == 0) {
            auto* rle = p.addStage<RLEStage<uint16_t>>();
            p.connect(rle, lq, "codes");
        } else if (chain == 1) {
            auto* bs = p.addStage<BitshuffleStage>();
            bs->setBlockSize(16384);
            bs->setElementWidth(2);
            auto* rze = p.addStage<RZEStage>();
            p.connect(bs, lq, "codes");
            p.connect(rze, bs);
        } else {
            auto* hf = p.addStage<HuffmanStage<uint16_t>>();
            hf->setBklen(1024);
            p.connect(hf, lq, "codes");
        }
        p.finalize();
        void* out = nullptr;
        size_t sz = 0;
        fill_shared();
        p.compress(d_in, n * sizeof(float), &out, &sz, 0);
        if (cudaStreamSynchronize(0) != cudaSuccess) throw std::runtime_error("sync failed");
        *comp_bytes = sz;
        p.writeToFile(path, 0);
        void* dec = nullptr;
        size_t dsz = 0;
        Pipeline::decompressFromFile(path, &dec, &dsz, 0);
        *decomp_bytes = dsz;
        if (d_decomp && dec) cudaMemcpy(d_decomp, dec, dsz, cudaMemcpyDeviceToDevice);
        if (dec) cudaFree(dec);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device sync failed");
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
    return 0;
}

// Pipelines around the direct Quantizer (the shipped presets
// examples/presets/pfpl.toml, speed.toml, quantizer_lorenzo_bitpack.toml and
// two more codings of the codes):
// chain 3: Quantizer<float,u32>(REL, zigzag) -> Difference<int32,uint32>(16 KiB)
//          -> Bitshuffle(16384, ew 2) -> RZE
// chain 4: Quantizer<float,u32>(REL, zigzag) -> Bitshuffle(16384, ew 4) -> RZE
// chain 5: Quantizer<float,u32>(NOA, radius 512) -> Lorenzo<int32> -> Bitpack<u32>(16)
// chain 6: Quantizer<float,u16>(ABS) -> Negabinary<int16,uint16> -> Bitshuffle(ew 2) -> RZE
// chain 7: Quantizer<float,u32>(ABS, zigzag, in-place outliers) -> Zigzag<int32,uint32>
//          -> Bitshuffle(ew 4) -> RZE
// The reference's stage factory has no Quantizer case, so the file cannot be
// read back by decompressFromFile; decompression runs on the live pipeline.
extern "C" int ref_pipeline_codes(int chain, const float* d_in, size_t n, size_t x, size_t y, size_t z, float eb,
                                  int mode, int radius, float outlier_cap, const char* path, float* d_decomp,
                                  size_t* decomp_bytes, size_t* comp_bytes) {
    try {
        Pipeline p(n * sizeof(float), MemoryStrategy::PREALLOCATE, 3.0f);
        p.setDims(x, y, z);
        auto bs_rze = [&](Stage* from, const char* port, int ew) {
            auto* bs = p.addStage<BitshuffleStage>();
            bs->setBlockSize(16384);
            bs->setElementWidth(ew);
            auto* rze = p.addStage<RZEStage>();
            rze->setLevels(4);
            p.connect(bs, from, port);
            p.connect(rze, bs);
        };
        if (chain == 6) {
            QuantizerStage<float, uint16_t>::Config c(eb, static_cast<ErrorBoundMode>(mode), radius, outlier_cap);
            auto* q = p.addStage<QuantizerStage<float, uint16_t>>(c);
            auto* nb = p.addStage<NegabinaryStage<int16_t, uint16_t>>();
            p.connect(nb, q, "codes");
            bs_rze(nb, "output", 2);
        } else {
            QuantizerStage<float, uint32_t>::Config c(eb, static_cast<ErrorBoundMode>(mode), radius, outlier_cap);
            c.zigzag_codes = chain == 3 || chain == 4 || chain == 7;
            c.inplace_outliers = chain == 7;
            auto* q = p.addStage<QuantizerStage<float, uint32_t>>(c);
            if (chain == 3) {
                auto* d = p.addStage<DifferenceStage<int32_t, uint32_t>>();
                d->setChunkSize(16384);
                p.connect(d, q, "codes");
                bs_rze(d, "output", 2);
            } else if (chain == 4) {
                bs_rze(q, "codes", 4);
            } else if (chain == 5) {
                auto* l = p.addStage<LorenzoStage<int32_t>>();
                auto* bp = p.addStage<BitpackStage<uint32_t>>();
                bp->setNBits(16);
                p.connect(l, q, "codes");
                p.connect(bp, l);
            } else {
                auto* zz = p.addStage<ZigzagStage<int32_t, uint32_t>>();
                p.connect(zz, q, "codes");
                bs_rze(zz, "output", 4);
            }
        }
        p.finalize();
        void* out = nullptr;
        size_t sz = 0;
        fill_shared();
        p.compress(d_in, n * sizeof(float), &out, &sz, 0);
        if (cudaStreamSynchronize(0) != cudaSuccess) throw std::runtime_error("sync failed");
        *comp_bytes = sz;
        p.writeToFile(path, 0);
        void* dec = nullptr;
        size_t dsz = 0;
        p.decompress(nullptr, 0, &dec, &dsz, 0);
        if (cudaStreamSynchronize(0) != cudaSuccess) throw std::runtime_error("sync failed");
        *decomp_bytes = dsz;
        if (d_decomp && dec) cudaMemcpy(d_decomp, dec, dsz, cudaMemcpyDeviceToDevice);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device sync failed");
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
    return 0;
}

// Times the reference's pfpl chain (chain 3 above: Quantizer REL -> Difference
// -> Bitshuffle -> RZE), or the speed chain, through its own
// Pipeline::compress / decompress on
// the default stream: `warmup` untimed calls, then the mean of `steps` calls
// each bracketed by CUDA events.  Every call includes the reference's own
// host synchronisation.  A 256 MiB buffer is rewritten between calls to
// evict L2.
// `speed` = 1 times the speed preset's chain instead (Quantizer REL ->
// Bitshuffle(16384, ew 4) -> RZE, examples/presets/speed.toml).
extern "C" int ref_pipeline_time_pfpl(const float* d_in, size_t n, float eb, float outlier_cap, int steps, int warmup,
                                      float* comp_ms, float* decomp_ms, size_t* comp_bytes, int speed) {
    try {
        Pipeline p(n * sizeof(float), MemoryStrategy::PREALLOCATE, 3.0f);
        p.setDims(n, 1, 1);
        QuantizerStage<float, uint32_t>::Config c(eb, ErrorBoundMode::REL, 32768, outlier_cap);
        c.zigzag_codes = true;
        // stages in topological order: the reference propagates buffer sizes
        // in addStage order
        auto* q = p.addStage<QuantizerStage<float, uint32_t>>(c);
        DifferenceStage<int32_t, uint32_t>* d = nullptr;
        if (!speed) {
            d = p.addStage<DifferenceStage<int32_t, uint32_t>>();
            d->setChunkSize(16384);
        }
        auto* bs = p.addStage<BitshuffleStage>();
        bs->setBlockSize(16384);
        bs->setElementWidth(speed ? 4 : 2);
        auto* rze = p.addStage<RZEStage>();
        rze->setLevels(4);
        if (d) {
            p.connect(d, q, "codes");
            p.connect(bs, d);
        } else {
            p.connect(bs, q, "codes");
        }
        p.connect(rze, bs);
        p.finalize();
        void* flush = nullptr;
        if (cudaMalloc(&flush, 256u << 20) != cudaSuccess) throw std::runtime_error("flush alloc failed");
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        double tc = 0, td = 0;
        void* out = nullptr;
        size_t sz = 0;
        for (int i = 0; i < warmup + steps; i++) {
            cudaMemsetAsync(flush, i & 0xff, 256u << 20, 0);
            cudaEventRecord(a, 0);
            p.compress(d_in, n * sizeof(float), &out, &sz, 0);
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            if (i >= warmup) tc += ms;
            cudaMemsetAsync(flush, i & 0xff, 256u << 20, 0);
            void* dec = nullptr;
            size_t dsz = 0;
            cudaEventRecord(a, 0);
            p.decompress(nullptr, 0, &dec, &dsz, 0);
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            cudaEventElapsedTime(&ms, a, b);
            if (i >= warmup) td += ms;
        }
        *comp_ms = (float)(tc / steps);
        *decomp_ms = (float)(td / steps);
        *comp_bytes = sz;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaFree(flush);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device sync failed");
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
    return 0;
}

// Times the reference's own pipeline for the LorenzoQuant chain (chain 1
// above: LorenzoQuant(REL, zigzag, capacity 0.1) -> Bitshuffle(16384, ew 2)
// -> RZE(16384, 4)) on an x*y*z field, as ref_pipeline_time_pfpl does.
extern "C" int ref_pipeline_time_lq(const float* d_in, size_t x, size_t y, size_t z, float eb, int steps, int warmup,
                                    float* comp_ms, float* decomp_ms, size_t* comp_bytes) {
    try {
        const size_t n = x * y * z;
        Pipeline p(n * sizeof(float), MemoryStrategy::PREALLOCATE, 3.0f);
        p.setDims(x, y, z);
        LorenzoQuantStage<float, uint16_t>::Config cfg;
        cfg.error_bound = eb;
        cfg.quant_radius = 32768;
        cfg.outlier_capacity = 0.1f;
        cfg.eb_mode = ErrorBoundMode::REL;
        cfg.zigzag_codes = true;
        auto* lq = p.addStage<LorenzoQuantStage<float, uint16_t>>(cfg);
        auto* bs = p.addStage<BitshuffleStage>();
        bs->setBlockSize(16384);
        bs->setElementWidth(2);
        auto* rze = p.addStage<RZEStage>();
        rze->setLevels(4);
        p.connect(bs, lq, "codes");
        p.connect(rze, bs);
        p.finalize();
        void* flush = nullptr;
        if (cudaMalloc(&flush, 256u << 20) != cudaSuccess) throw std::runtime_error("flush alloc failed");
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        double tc = 0, td = 0;
        void* out = nullptr;
        size_t sz = 0;
        for (int i = 0; i < warmup + steps; i++) {
            float ms = 0;
            fill_shared();
            cudaMemsetAsync(flush, i & 0xff, 256u << 20, 0);
            cudaEventRecord(a, 0);
            p.compress(d_in, n * sizeof(float), &out, &sz, 0);
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            cudaEventElapsedTime(&ms, a, b);
            if (i >= warmup) tc += ms;
            cudaMemsetAsync(flush, i & 0xff, 256u << 20, 0);
            void* dec = nullptr;
            size_t dsz = 0;
            cudaEventRecord(a, 0);
            p.decompress(nullptr, 0, &dec, &dsz, 0);
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            cudaEventElapsedTime(&ms, a, b);
            if (i >= warmup) td += ms;
        }
        *comp_ms = (float)(tc / steps);
        *decomp_ms = (float)(td / steps);
        *comp_bytes = sz;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaFree(flush);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device sync failed");
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
    return 0;
}

// Loads a TOML configuration with the reference's own Pipeline::loadConfig
// (src/pipeline/config.cpp:534-640), compresses n floats with it, writes the
// FZM file and saves the configuration back with Pipeline::saveConfig.
// `x, y, z` set the dimensions before loading, as a caller of the reference
// does when its file has no `dims` key.
extern "C" int ref_pipeline_config(const char* config_path, size_t x, size_t y, size_t z, const float* d_in,
                                   size_t n, const char* fzm_path, const char* saved_path, size_t* comp_bytes) {
    try {
        Pipeline p;
        if (x) p.setDims(x, y, z);
        p.loadConfig(config_path);
        fill_shared();
        void* out = nullptr;
        size_t sz = 0;
        p.compress(d_in, n * sizeof(float), &out, &sz, 0);
        if (cudaStreamSynchronize(0) != cudaSuccess) throw std::runtime_error("sync failed");
        *comp_bytes = sz;
        p.writeToFile(fzm_path, 0);
        p.saveConfig(saved_path);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device sync failed");
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
    return 0;
}
