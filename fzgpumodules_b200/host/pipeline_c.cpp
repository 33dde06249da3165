// pipeline_c.cpp -- C ABI over fz::Pipeline (fzb_pipeline_* in fzb.h), for
// bindings in languages without C++ interop.  Stages are addressed by the
// index addStage returned; C++ exceptions become FZB_E_PIPELINE with the
// message available from fzb_last_error() on the calling thread.
#include <memory>
#include <string>
#include <vector>

#include "fz/pipeline.h"
#include "fzb.h"

namespace {

thread_local std::string g_last_error;

struct Handle {
    std::unique_ptr<fz::Pipeline> p;
    std::vector<fz::Stage*> stages;
};

template <typename F>
int guarded(F&& f) {
    try {
        g_last_error.clear();
        return f();
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return FZB_E_INVALID;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return FZB_E_PIPELINE;
    } catch (...) {
        g_last_error = "unknown exception";
        return FZB_E_PIPELINE;
    }
}

Handle* H(void* p) { return static_cast<Handle*>(p); }

int add(void* p, fz::Stage* s) {
    Handle* h = H(p);
    h->stages.push_back(s);
    return (int)h->stages.size() - 1;
}

fz::Stage* stage_at(void* p, int i) {
    Handle* h = H(p);
    if (i < 0 || i >= (int)h->stages.size()) throw std::invalid_argument("no stage with index " + std::to_string(i));
    return h->stages[i];
}

}  // namespace

extern "C" {

const char* fzb_last_error(void) { return g_last_error.c_str(); }

void* fzb_pipeline_create(uint64_t input_hint, int strategy, float pool_multiplier) {
    try {
        g_last_error.clear();
        auto* h = new Handle();
        h->p.reset(new fz::Pipeline(input_hint,
                                    strategy == FZB_PREALLOCATE ? fz::MemoryStrategy::PREALLOCATE : fz::MemoryStrategy::MINIMAL,
                                    pool_multiplier > 0.0f ? pool_multiplier : 3.0f));
        return h;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return nullptr;
    }
}

void fzb_pipeline_destroy(void* p) { delete H(p); }

int fzb_pipeline_set_dims(void* p, uint64_t x, uint64_t y, uint64_t z) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->setDims(x, y, z);
        return FZB_OK;
    });
}

int fzb_pipeline_add_lorenzo_quant(void* p, float eb, int eb_mode, int radius, float outlier_capacity, int zigzag,
                                   float value_base) {
    if (!p || eb_mode < FZB_ABS || eb_mode > FZB_NOA || radius <= 0 || radius > 65535) return FZB_E_INVALID;
    return guarded([&] {
        fz::LorenzoQuantStage<float, uint16_t>::Config c;
        c.error_bound = eb;
        c.quant_radius = radius;
        c.outlier_capacity = outlier_capacity;
        c.eb_mode = (fz::ErrorBoundMode)eb_mode;
        c.precomputed_value_base = value_base;
        c.zigzag_codes = zigzag != 0;
        return add(p, H(p)->p->addStage<fz::LorenzoQuantStage<float, uint16_t>>(c));
    });
}

int fzb_pipeline_add_quantizer(void* p, int code_bytes, float eb, int eb_mode, int radius, float outlier_capacity,
                               int zigzag, int inplace, float threshold, float value_base) {
    if (!p || eb_mode < FZB_ABS || eb_mode > FZB_NOA || (code_bytes != 2 && code_bytes != 4) || radius <= 0)
        return FZB_E_INVALID;
    return guarded([&] {
        auto fill = [&](auto& c) {
            c.error_bound = eb;
            c.quant_radius = radius;
            c.outlier_capacity = outlier_capacity;
            c.eb_mode = (fz::ErrorBoundMode)eb_mode;
            c.precomputed_value_base = value_base;
            c.zigzag_codes = zigzag != 0;
            c.inplace_outliers = inplace != 0;
            c.outlier_threshold = threshold;
        };
        if (code_bytes == 2) {
            fz::QuantizerStage<float, uint16_t>::Config c;
            fill(c);
            return add(p, H(p)->p->addStage<fz::QuantizerStage<float, uint16_t>>(c));
        }
        fz::QuantizerStage<float, uint32_t>::Config c;
        fill(c);
        return add(p, H(p)->p->addStage<fz::QuantizerStage<float, uint32_t>>(c));
    });
}

int fzb_pipeline_add_difference(void* p, int in_type, int out_type, uint32_t chunk_size) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        using DT = fz::DataType;
        const DT a = (DT)in_type, b = (DT)out_type;
        fz::Stage* s = nullptr;
        auto mk = [&](auto* st) {
            st->setChunkSize(chunk_size);
            s = st;
        };
        auto& P = *H(p)->p;
        if (a == DT::INT8 && b == DT::UINT8) mk(P.addStage<fz::DifferenceStage<int8_t, uint8_t>>());
        else if (a == DT::INT16 && b == DT::UINT16) mk(P.addStage<fz::DifferenceStage<int16_t, uint16_t>>());
        else if (a == DT::INT32 && b == DT::UINT32) mk(P.addStage<fz::DifferenceStage<int32_t, uint32_t>>());
        else if (a == DT::INT64 && b == DT::UINT64) mk(P.addStage<fz::DifferenceStage<int64_t, uint64_t>>());
        else if (a == b && a == DT::UINT8) mk(P.addStage<fz::DifferenceStage<uint8_t>>());
        else if (a == b && a == DT::UINT16) mk(P.addStage<fz::DifferenceStage<uint16_t>>());
        else if (a == b && a == DT::UINT32) mk(P.addStage<fz::DifferenceStage<uint32_t>>());
        else if (a == b && a == DT::INT32) mk(P.addStage<fz::DifferenceStage<int32_t>>());
        else if (a == b && a == DT::INT64) mk(P.addStage<fz::DifferenceStage<int64_t>>());
        else throw std::invalid_argument("unsupported Difference type combination");
        return add(p, s);
    });
}

int fzb_pipeline_add_lorenzo(void* p, int data_type) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        using DT = fz::DataType;
        auto& P = *H(p)->p;
        switch ((DT)data_type) {
            case DT::INT8: return add(p, P.addStage<fz::LorenzoStage<int8_t>>());
            case DT::INT16: return add(p, P.addStage<fz::LorenzoStage<int16_t>>());
            case DT::INT32: return add(p, P.addStage<fz::LorenzoStage<int32_t>>());
            case DT::INT64: return add(p, P.addStage<fz::LorenzoStage<int64_t>>());
            default: throw std::invalid_argument("unsupported Lorenzo data_type");
        }
    });
}

static int add_sign_coding(void* p, int in_type, bool nb) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        using DT = fz::DataType;
        auto& P = *H(p)->p;
        switch ((DT)in_type) {
            case DT::INT8:
                return add(p, nb ? (fz::Stage*)P.addStage<fz::NegabinaryStage<int8_t, uint8_t>>()
                                 : P.addStage<fz::ZigzagStage<int8_t, uint8_t>>());
            case DT::INT16:
                return add(p, nb ? (fz::Stage*)P.addStage<fz::NegabinaryStage<int16_t, uint16_t>>()
                                 : P.addStage<fz::ZigzagStage<int16_t, uint16_t>>());
            case DT::INT32:
                return add(p, nb ? (fz::Stage*)P.addStage<fz::NegabinaryStage<int32_t, uint32_t>>()
                                 : P.addStage<fz::ZigzagStage<int32_t, uint32_t>>());
            case DT::INT64:
                return add(p, nb ? (fz::Stage*)P.addStage<fz::NegabinaryStage<int64_t, uint64_t>>()
                                 : P.addStage<fz::ZigzagStage<int64_t, uint64_t>>());
            default: throw std::invalid_argument("unsupported input_type (a signed integer type is required)");
        }
    });
}

int fzb_pipeline_add_zigzag(void* p, int in_type) { return add_sign_coding(p, in_type, false); }
int fzb_pipeline_add_negabinary(void* p, int in_type) { return add_sign_coding(p, in_type, true); }

int fzb_pipeline_load_config(void* p, const char* path) {
    if (!p || !path) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->loadConfig(path);
        return FZB_OK;
    });
}

int fzb_pipeline_save_config(void* p, const char* path) {
    if (!p || !path) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->saveConfig(path);
        return FZB_OK;
    });
}

int fzb_pipeline_add_bitshuffle(void* p, uint32_t block_size, int element_width) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        auto* s = H(p)->p->addStage<fz::BitshuffleStage>();
        s->setBlockSize(block_size);
        s->setElementWidth((size_t)element_width);
        return add(p, s);
    });
}

int fzb_pipeline_add_rze(void* p, uint32_t chunk_size, int levels) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        auto* s = H(p)->p->addStage<fz::RZEStage>();
        s->setChunkSize(chunk_size);
        s->setLevels(levels);
        return add(p, s);
    });
}

int fzb_pipeline_add_rle(void* p, int elem) {
    if (!p || (elem != 1 && elem != 2 && elem != 4)) return FZB_E_INVALID;
    return guarded([&] {
        fz::Stage* s = elem == 1   ? (fz::Stage*)H(p)->p->addStage<fz::RLEStage<uint8_t>>()
                       : elem == 2 ? (fz::Stage*)H(p)->p->addStage<fz::RLEStage<uint16_t>>()
                                   : (fz::Stage*)H(p)->p->addStage<fz::RLEStage<uint32_t>>();
        return add(p, s);
    });
}

int fzb_pipeline_add_huffman(void* p, uint32_t bklen) {
    if (!p || bklen < 1 || bklen > 65535) return FZB_E_INVALID;
    return guarded([&] {
        auto* s = H(p)->p->addStage<fz::HuffmanStage<uint16_t>>();
        s->setBklen(bklen);
        return add(p, s);
    });
}

int fzb_pipeline_add_huffman_mode(void* p, uint32_t bklen, int encode_mode) {
    if (!p || bklen < 1 || bklen > 65535 || encode_mode < 0 || encode_mode > 1) return FZB_E_INVALID;
    return guarded([&] {
        auto* s = H(p)->p->addStage<fz::HuffmanStage<uint16_t>>();
        s->setBklen(bklen);
        s->setEncodeMode(encode_mode ? fz::HuffmanEncodeMode::Fine : fz::HuffmanEncodeMode::Coarse);
        return add(p, s);
    });
}

int fzb_pipeline_add_bitpack(void* p, int elem, int nbits) {
    if (!p || (elem != 1 && elem != 2 && elem != 4)) return FZB_E_INVALID;
    return guarded([&] {
        auto setup = [&](auto* s) {
            if (nbits == 0) s->setAutoDetect(true);
            else s->setNBits((uint8_t)nbits);
            return add(p, s);
        };
        if (elem == 1) return setup(H(p)->p->addStage<fz::BitpackStage<uint8_t>>());
        if (elem == 2) return setup(H(p)->p->addStage<fz::BitpackStage<uint16_t>>());
        return setup(H(p)->p->addStage<fz::BitpackStage<uint32_t>>());
    });
}

int fzb_pipeline_connect(void* p, int dependent, int producer, const char* output_name) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        return H(p)->p->connect(stage_at(p, dependent), stage_at(p, producer), output_name ? output_name : "output");
    });
}

int fzb_pipeline_set_fusion(void* p, int on) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->setFusion(on != 0);
        return FZB_OK;
    });
}

int fzb_pipeline_set_num_streams(void* p, int num_streams) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->setNumStreams(num_streams);
        return FZB_OK;
    });
}

int fzb_pipeline_num_streams(void* p) {
    if (!p) return FZB_E_INVALID;
    return H(p)->p->getNumStreams();
}

int fzb_pipeline_enable_bounds_check(void* p, int on) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->enableBoundsCheck(on != 0);
        return FZB_OK;
    });
}

int fzb_pipeline_enable_graph_mode(void* p, int on) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->enableGraphMode(on != 0);
        return FZB_OK;
    });
}

int fzb_pipeline_enable_profiling(void* p, int on) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->enableProfiling(on != 0);
        return FZB_OK;
    });
}

int fzb_pipeline_finalize(void* p) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->finalize();
        return FZB_OK;
    });
}

int fzb_pipeline_is_fused(void* p) { return p && H(p)->p->isFused() ? 1 : 0; }

int fzb_pipeline_capture_graph(void* p, void* stream) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->captureGraph(static_cast<cudaStream_t>(stream));
        return FZB_OK;
    });
}

int fzb_pipeline_decompress_graph_captured(void* p) {
    if (!p) return FZB_E_INVALID;
    return H(p)->p->isDecompressGraphCaptured() ? 1 : 0;
}

int fzb_pipeline_check_decompress(void* p, void* stream) {
    if (!p) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->checkDecompressStatus(static_cast<cudaStream_t>(stream));
        return FZB_OK;
    });
}

int fzb_pipeline_compress(void* p, const void* d_in, uint64_t bytes, void** d_out, uint64_t* out_bytes,
                          void* stream) {
    if (!p || !d_in || !d_out || !out_bytes) return FZB_E_INVALID;
    return guarded([&] {
        size_t sz = 0;
        H(p)->p->compress(d_in, bytes, d_out, &sz, static_cast<cudaStream_t>(stream));
        *out_bytes = sz;
        return FZB_OK;
    });
}

int fzb_pipeline_decompress(void* p, const void* d_in, uint64_t bytes, void** d_out, uint64_t* out_bytes,
                            void* stream) {
    if (!p || !d_out || !out_bytes) return FZB_E_INVALID;
    return guarded([&] {
        size_t sz = 0;
        H(p)->p->decompress(d_in, bytes, d_out, &sz, static_cast<cudaStream_t>(stream));
        *out_bytes = sz;
        return FZB_OK;
    });
}

int fzb_pipeline_decompress_into(void* p, const void* d_in, uint64_t bytes, void* d_out, uint64_t capacity,
                                 uint64_t* out_bytes, void* stream) {
    if (!p || !d_out || !out_bytes) return FZB_E_INVALID;
    return guarded([&] {
        size_t sz = 0;
        H(p)->p->decompress(d_in, bytes, d_out, capacity, &sz, static_cast<cudaStream_t>(stream));
        *out_bytes = sz;
        return FZB_OK;
    });
}

int fzb_pipeline_write_file(void* p, const char* path, void* stream) {
    if (!p || !path) return FZB_E_INVALID;
    return guarded([&] {
        H(p)->p->writeToFile(path, static_cast<cudaStream_t>(stream));
        return FZB_OK;
    });
}

int fzb_pipeline_stage_timings(void* p, double* ms, int max_entries) {
    if (!p || !ms) return FZB_E_INVALID;
    return guarded([&] {
        const auto& r = H(p)->p->getLastPerfResult();
        int n = 0;
        for (const auto& s : r.stages)
            if (n < max_entries) ms[n++] = s.elapsed_ms;
        return n;
    });
}

int fzb_decompress_file(const char* path, void** d_out, uint64_t* out_bytes, void* stream) {
    if (!path || !d_out || !out_bytes) return FZB_E_INVALID;
    return guarded([&] {
        size_t sz = 0;
        fz::Pipeline::decompressFromFile(path, d_out, &sz, static_cast<cudaStream_t>(stream));
        *out_bytes = sz;
        return FZB_OK;
    });
}

int fzb_free(void* d_ptr) { return cudaFree(d_ptr) == cudaSuccess ? FZB_OK : FZB_E_CUDA; }

}  // extern "C"
