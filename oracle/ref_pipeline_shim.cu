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
#include <string>

#include "pipeline/compressor.h"

using namespace fz;

static std::string g_err;

extern "C" const char* ref_pipe_last_error() { return g_err.c_str(); }

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
