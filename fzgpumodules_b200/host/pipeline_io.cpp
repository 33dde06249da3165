// pipeline_io.cpp -- decompression (the inverse DAG) and the FZM container:
// buildHeader / writeToFile / readHeader / decompressFromFile
// (src/pipeline/compressor_io.cpp:90-706, compressor_inverse_dag.cpp).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <functional>
#include <stdexcept>
#include <unordered_set>

#include "fz/pipeline.h"
#include "fzb.h"

namespace fz {

namespace {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

inline size_t pad16(size_t v) { return (v + 15) & ~(size_t)15; }

struct FwdDesc {
    Stage* stage;
    std::vector<int> in_ids, out_ids;
};

using Avail = std::unordered_map<int, std::pair<void*, size_t>>;

// What a Pipeline's decompression keeps between calls: the fused inverse's
// workspace and the mapped block its status word (and the stages' results)
// are gathered into before the call's one wait.  Null for a one-off
// decompression (decompressFromFile), which allocates per call and reads
// each value with its own copy.
struct InverseCtx {
    ResultGather* gather = nullptr;
    void** work = nullptr;
    size_t* work_bytes = nullptr;
    std::function<bool(cudaStream_t)> enqueue_reads;  // the stages' pending results
    std::function<void()> finish_reads;
};

// The fused inverse's workspace: the context's kept buffer (grown when
// needed), else a pool buffer that *temp receives for release.
void* inverse_work(InverseCtx* ctx, MemoryPool* pool, size_t need, cudaStream_t stream, void** temp) {
    *temp = nullptr;
    if (ctx && ctx->work) {
        if (*ctx->work && *ctx->work_bytes >= need) return *ctx->work;
        if (*ctx->work) pool->free(*ctx->work, stream);
        *ctx->work_bytes = 0;
        *ctx->work = pool->allocate(need, stream, "inverse_workspace", true);
        if (!*ctx->work) throw std::runtime_error("decompress: workspace allocation failed");
        *ctx->work_bytes = need;
        return *ctx->work;
    }
    *temp = pool->allocate(need, stream, "inverse_workspace", false);
    if (!*temp) throw std::runtime_error("decompress: workspace allocation failed");
    return *temp;
}

// Waits for the stream and returns the workspace status bits (cleared on the
// device): gathered through the mapped block before the wait when the
// context has one, else copied after it.
uint32_t wait_status(InverseCtx* ctx, void* w, cudaStream_t stream) {
    uint32_t bits = 0;
    std::vector<DeviceRead> rd{{w, 4, &bits, true}};
    const bool g = ctx && ctx->gather && ctx->gather->enqueue(rd, stream);
    cuda_check(cudaStreamSynchronize(stream), "decompress");
    if (g) {
        ctx->gather->finish(rd);
    } else {
        cuda_check(cudaMemcpy(&bits, w, 4, cudaMemcpyDeviceToHost), "decompress status");
        cuda_check(cudaMemset(w, 0, 4), "decompress status");
    }
    return bits;
}

std::string hex8(uint32_t v) {
    char b[16];
    std::snprintf(b, sizeof(b), "%08X", v);
    return b;
}

// The fused inverse applies when the source stage is LorenzoQuant whose codes
// go through Bitshuffle(16 KiB, ew 2) into RZE(16 KiB, 4 levels) and nothing
// else reads the intermediates.
// The pfpl chain, Quantizer<float, uint32_t> -> Difference<int32_t,
// uint32_t>(16 KiB) -> Bitshuffle(16 KiB, ew 2) -> RZE(16 KiB, 4 levels), is
// inverted in one pass the same way.
bool fused_inverse_pfpl(const std::vector<FwdDesc>& fwd, const Avail& avail, const FwdDesc* q,
                        MemoryPool* pool, void* d_result, size_t capacity, size_t* result_size,
                        cudaStream_t stream, InverseCtx* ctx) {
    auto* qs = dynamic_cast<QuantizerStage<float, uint32_t>*>(q->stage);
    if (!qs || q->out_ids.size() != 4) return false;
    auto only = [&](int buf) -> const FwdDesc* {
        const FwdDesc* r = nullptr;
        int k = 0;
        for (const auto& d : fwd)
            for (int i : d.in_ids)
                if (i == buf) r = &d, k++;
        return (k == 1 && r->out_ids.size() == 1 && r->in_ids.size() == 1) ? r : nullptr;
    };
    const FwdDesc* df = only(q->out_ids[0]);
    if (!df) return false;
    auto* dfs = dynamic_cast<DifferenceStage<int32_t, uint32_t>*>(df->stage);
    if (!dfs || dfs->getChunkSize() != 16384) return false;
    const FwdDesc* bs = only(df->out_ids[0]);
    if (!bs) return false;
    auto* bss = dynamic_cast<BitshuffleStage*>(bs->stage);
    if (!bss || bss->getBlockSize() != 16384 || bss->getElementWidth() != 2) return false;
    const FwdDesc* rz = only(bs->out_ids[0]);
    if (!rz) return false;
    auto* rzs = dynamic_cast<RZEStage*>(rz->stage);
    if (!rzs || rzs->getChunkSize() != 16384 || rzs->getLevels() != 4) return false;
    for (int i = 1; i < 4; i++)
        if (!avail.count(q->out_ids[i])) return false;
    if (!avail.count(rz->out_ids[0])) return false;
    const auto& rze = avail.at(rz->out_ids[0]);
    const auto& val = avail.at(q->out_ids[1]);
    const auto& idx = avail.at(q->out_ids[2]);
    const auto& cnt = avail.at(q->out_ids[3]);
    const size_t n = rzs->getCachedOrigBytes() / sizeof(uint32_t);
    *result_size = n * sizeof(float);
    if (n == 0) return true;
    if (*result_size > capacity) throw std::runtime_error("decompress: output buffer too small");
    // the outlier lists and the stream are read with word loads: realign
    std::vector<void*> temps;
    auto aligned = [&](const std::pair<void*, size_t>& b) -> const void* {
        if (!(reinterpret_cast<uintptr_t>(b.first) & 15) || !b.second) return b.first;
        void* t = pool->allocate(b.second, stream, "inverse_realign", false);
        if (!t) throw std::runtime_error("decompress: allocation failed");
        temps.push_back(t);
        cuda_check(cudaMemcpyAsync(t, b.first, b.second, cudaMemcpyDeviceToDevice, stream), "decompress realign");
        return t;
    };
    const size_t need = fzb_pfpl_decompress_workspace_bytes(n);
    void* wtemp = nullptr;
    void* w = inverse_work(ctx, pool, need, stream, &wtemp);
    int rc = FZB_OK;
    try {
        const void* r = aligned(rze);
        const void* v = aligned(val);
        const void* ix = aligned(idx);
        const void* ct = aligned(cnt);
        rc = fzb_pfpl_decompress(r, rze.second, static_cast<const float*>(v), static_cast<const uint32_t*>(ix),
                                 static_cast<const uint32_t*>(ct), val.second / sizeof(float), n,
                                 qs->getErrorBound(), (int)qs->getErrorBoundMode(), qs->computedAbsErrorBound(),
                                 qs->getZigzagCodes() ? 1 : 0, static_cast<float*>(d_result), w, need, stream);
        if (rc == FZB_OK) rc = fzb_status_from_bits(wait_status(ctx, w, stream), nullptr);
    } catch (...) {
        cudaStreamSynchronize(stream);
        for (void* t : temps) pool->free(t, stream);
        if (wtemp) pool->free(wtemp, stream);
        throw;
    }
    cudaStreamSynchronize(stream);
    for (void* t : temps) pool->free(t, stream);
    if (wtemp) pool->free(wtemp, stream);
    if (rc) throw std::runtime_error(std::string("Quantizer<-Difference<-Bitshuffle<-RZE decompress: ") +
                                     fzb_status_string(rc));
    return true;
}

bool fused_inverse(const std::vector<FwdDesc>& fwd, const Avail& avail, int source_buf, MemoryPool* pool,
                   void* d_result, size_t capacity, size_t* result_size, cudaStream_t stream, InverseCtx* ctx) {
    const FwdDesc* lq = nullptr;
    for (const auto& d : fwd)
        if (d.in_ids.size() == 1 && d.in_ids[0] == source_buf) lq = &d;
    if (!lq || lq->out_ids.size() != 4) return false;
    if (fused_inverse_pfpl(fwd, avail, lq, pool, d_result, capacity, result_size, stream, ctx)) return true;
    auto* lqs = dynamic_cast<LorenzoQuantStage<float, uint16_t>*>(lq->stage);
    if (!lqs) return false;
    auto consumers = [&](int buf) {
        std::vector<const FwdDesc*> v;
        for (const auto& d : fwd)
            for (int i : d.in_ids)
                if (i == buf) v.push_back(&d);
        return v;
    };
    const auto c1 = consumers(lq->out_ids[0]);
    if (c1.size() != 1 || c1[0]->out_ids.size() != 1) return false;
    auto* bs = dynamic_cast<BitshuffleStage*>(c1[0]->stage);
    if (!bs || bs->getBlockSize() != 16384 || bs->getElementWidth() != 2) return false;
    const auto c2 = consumers(c1[0]->out_ids[0]);
    if (c2.size() != 1 || c2[0]->out_ids.size() != 1) return false;
    auto* rz = dynamic_cast<RZEStage*>(c2[0]->stage);
    if (!rz || rz->getChunkSize() != 16384 || rz->getLevels() != 4) return false;
    for (int i = 1; i < 4; i++)
        if (!avail.count(lq->out_ids[i])) return false;
    if (!avail.count(c2[0]->out_ids[0])) return false;
    const auto& rze = avail.at(c2[0]->out_ids[0]);
    const auto& err = avail.at(lq->out_ids[1]);
    const auto& idx = avail.at(lq->out_ids[2]);
    const auto& cnt = avail.at(lq->out_ids[3]);
    const size_t n = rz->getCachedOrigBytes() / sizeof(uint16_t);
    *result_size = n * sizeof(float);
    if (n == 0) return true;
    if (*result_size > capacity) throw std::runtime_error("decompress: output buffer too small");
    const auto d = lqs->getDims();
    uint32_t dims[3] = {(uint32_t)d[0], (uint32_t)d[1], (uint32_t)d[2]};
    const size_t need = fzb_workspace_bytes(n, 0);
    void* wtemp = nullptr;
    void* w = inverse_work(ctx, pool, need, stream, &wtemp);
    // the fused pass without a host wait; its status word comes back with
    // the call's one wait, and a case it left to the exact kernels (values
    // outside the exact-integer range, unsorted outliers) runs them after
    auto run = [&](unsigned flags) {
        return fzb_lq_bs_rze_decompress(rze.first, rze.second, static_cast<const float*>(err.first),
                                        static_cast<const uint32_t*>(idx.first),
                                        static_cast<const uint32_t*>(cnt.first), err.second / sizeof(float), n, dims,
                                        lqs->computedAbsErrorBound(), lqs->getZigzagCodes() ? 1 : 0,
                                        static_cast<float*>(d_result), flags, w, need, stream);
    };
    int rc = run(FZB_NO_SYNC);
    if (rc == FZB_OK) {
        int rerun = 0;
        rc = fzb_status_from_bits(wait_status(ctx, w, stream), &rerun);
        if (rc == FZB_OK && rerun) rc = run(FZB_FORCE_EXACT);
    } else {
        cudaStreamSynchronize(stream);
    }
    if (wtemp) pool->free(wtemp, stream);
    if (rc) throw std::runtime_error(std::string("LorenzoQuant<-Bitshuffle<-RZE decompress: ") + fzb_status_string(rc));
    return true;
}

// Runs the inverse of every stage in reverse topological order.  d_result
// receives the source buffer's reconstruction.
void run_inverse(const std::vector<FwdDesc>& fwd, Avail avail, int source_buf, MemoryPool* pool, void* d_result,
                 size_t capacity, size_t* result_size, cudaStream_t stream, bool allow_fused,
                 InverseCtx* ctx = nullptr) {
    for (const auto& d : fwd) d.stage->setInverse(true);
    // the fused inverses end with the stream synchronised
    if (allow_fused && fused_inverse(fwd, avail, source_buf, pool, d_result, capacity, result_size, stream, ctx))
        return;
    std::vector<void*> temps;
    try {
        for (auto it = fwd.rbegin(); it != fwd.rend(); ++it) {
            std::vector<void*> in;
            std::vector<size_t> sizes;
            for (int id : it->out_ids) {
                auto a = avail.find(id);
                if (a == avail.end())
                    throw std::runtime_error("decompress: buffer " + std::to_string(id) + " of stage '" +
                                             it->stage->getName() + "' is not available");
                void* ptr = a->second.first;
                // container segments are packed unpadded; the coders read
                // their headers with word loads, so realign odd starts
                if ((reinterpret_cast<uintptr_t>(ptr) & 15) && a->second.second) {
                    void* t = pool->allocate(a->second.second, stream, "inverse_realign", false);
                    if (!t) throw std::runtime_error("decompress: allocation failed");
                    temps.push_back(t);
                    cuda_check(cudaMemcpyAsync(t, ptr, a->second.second, cudaMemcpyDeviceToDevice, stream),
                               "decompress realign");
                    ptr = t;
                }
                in.push_back(ptr);
                sizes.push_back(a->second.second);
            }
            if (it->in_ids.size() != 1)
                throw std::runtime_error("decompress: stage '" + it->stage->getName() + "' has " +
                                         std::to_string(it->in_ids.size()) + " inputs; one is supported");
            const size_t est = it->stage->estimateOutputSizes(sizes).at(0);
            void* out = nullptr;
            if (it->in_ids[0] == source_buf) {
                if (est > capacity) throw std::runtime_error("decompress: output buffer too small");
                out = d_result;
            } else {
                out = est ? pool->allocate(est, stream, "inverse_intermediate", false) : nullptr;
                if (est && !out) throw std::runtime_error("decompress: allocation failed");
                temps.push_back(out);
            }
            it->stage->execute(stream, pool, in, {out}, sizes);
            avail[it->in_ids[0]] = {out, it->stage->getActualOutputSize(0)};
        }
        const bool gathered = ctx && ctx->enqueue_reads && ctx->enqueue_reads(stream);
        cuda_check(cudaStreamSynchronize(stream), "decompress");
        if (gathered) ctx->finish_reads();
        for (const auto& d : fwd) d.stage->postStreamSync(stream);
    } catch (...) {
        cudaStreamSynchronize(stream);
        for (void* p : temps) pool->free(p, stream);
        throw;
    }
    for (void* p : temps) pool->free(p, stream);
    *result_size = avail.at(source_buf).second;
}

}  // namespace

// ---------------------------------------------------------------- decompress

void Pipeline::runInverse(const std::unordered_map<int, std::pair<void*, size_t>>& outputs, void* d_result,
                          size_t capacity, size_t* result_size, cudaStream_t stream) {
    std::vector<FwdDesc> fwd;
    for (const auto& lv : dag_->getLevels())
        for (auto* n : lv) fwd.push_back({n->stage, n->input_buffer_ids, n->output_buffer_ids});
    for (auto& s : stages_) s->saveState();
    try {
        InverseCtx ctx;
        ctx.gather = &gather_;
        ctx.work = &inv_work_;
        ctx.work_bytes = &inv_work_bytes_;
        ctx.enqueue_reads = [this](cudaStream_t st) { return enqueueResultReads(st); };
        ctx.finish_reads = [this]() { finishResultReads(); };
        run_inverse(fwd, outputs, input_buffer_id_, pool_.get(), d_result, capacity, result_size, stream, fused_,
                    &ctx);
    } catch (...) {
        for (auto& s : stages_) {
            s->setInverse(false);
            s->restoreState();
        }
        throw;
    }
    for (auto& s : stages_) {
        s->setInverse(false);
        s->restoreState();
    }
    if (original_input_size_ && *result_size > original_input_size_) *result_size = original_input_size_;
}

void Pipeline::decompress(const void* d_input, size_t input_size, void** d_output, size_t* output_size,
                          cudaStream_t stream) {
    if (!finalized_) throw std::runtime_error("Pipeline not finalized");
    if (meta_.empty()) throw std::runtime_error("decompress() requires compress() to have been called first");
    std::unordered_map<int, std::pair<void*, size_t>> outs;
    size_t off = pad16(4 + 8 * meta_.size());
    for (const auto& m : meta_) {
        void* p = dag_->getBuffer(m.buffer_id);
        if (d_input) {
            if (meta_.size() == 1) p = const_cast<void*>(d_input);
            else {
                p = static_cast<uint8_t*>(const_cast<void*>(d_input)) + off;
                off += pad16(m.actual_size);
            }
        }
        outs[m.buffer_id] = {p, m.actual_size};
    }
    if (d_input && meta_.size() > 1 && off > input_size)
        throw std::runtime_error("decompress(): input (" + std::to_string(input_size) +
                                 " bytes) is shorter than the compressed layout (" + std::to_string(off) + " bytes)");
    const size_t cap = input_size_;  // the source bytes (padded)
    if (decomp_exec_) {  // replay the captured decompression: no host wait
        const auto t0 = std::chrono::steady_clock::now();
        const void* src = d_input;
        size_t bytes = input_size;
        if (!src) {
            src = concat_buf_;
            bytes = concatSize();
        }
        if (!src || bytes > decomp_in_bytes_)
            throw std::runtime_error("decompress(): the container (" + std::to_string(bytes) +
                                     " bytes) does not fit the decompression graph's slot (" +
                                     std::to_string(decomp_in_bytes_) + " bytes)");
        cuda_check(cudaMemcpyAsync(decomp_in_, src, bytes, cudaMemcpyDeviceToDevice, stream), "decompress input");
        cuda_check(cudaGraphLaunch(decomp_exec_, stream), "decompress graph launch");
        const size_t out = (original_input_size_ && original_input_size_ < cap) ? original_input_size_ : cap;
        if (pool_managed_decomp_) {
            *d_output = decomp_out_;
        } else {
            void* p = nullptr;
            cuda_check(cudaMalloc(&p, out), "cudaMalloc for decompress output");
            cuda_check(cudaMemcpyAsync(p, decomp_out_, out, cudaMemcpyDeviceToDevice, stream), "decompress copy-out");
            *d_output = p;
        }
        *output_size = out;
        last_perf_ = PipelinePerfResult();
        last_perf_.is_compress = false;
        last_perf_.input_bytes = bytes;
        last_perf_.output_bytes = out;
        last_perf_.host_elapsed_ms = last_perf_.dag_elapsed_ms =
            std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return;
    }
    void* d_final = nullptr;
    if (pool_managed_decomp_ && decomp_outputs_.size() == 1 && decomp_output_bytes_ >= cap) {
        // the previous call's output is released by this call: reuse it
        d_final = decomp_outputs_[0];
    } else if (pool_managed_decomp_) {
        for (void* p : decomp_outputs_) pool_->free(p, stream);
        decomp_outputs_.clear();
        decomp_output_bytes_ = 0;
        d_final = pool_->allocate(cap, stream, "decomp_output", true);
        if (!d_final) throw std::runtime_error("Pool allocation for decompress output failed");
        decomp_outputs_.push_back(d_final);
        decomp_output_bytes_ = cap;
    } else {
        cuda_check(cudaMalloc(&d_final, cap), "cudaMalloc for decompress output");
    }
    const auto t0 = std::chrono::steady_clock::now();
    runInverse(outs, d_final, cap, output_size, stream);
    const auto t1 = std::chrono::steady_clock::now();
    *d_output = d_final;
    last_perf_ = PipelinePerfResult();
    last_perf_.is_compress = false;
    last_perf_.input_bytes = input_size;
    last_perf_.output_bytes = *output_size;
    last_perf_.host_elapsed_ms = last_perf_.dag_elapsed_ms = std::chrono::duration<float, std::milli>(t1 - t0).count();
}

void Pipeline::decompress(const void* d_input, size_t input_size, void* d_output_buf, size_t output_buf_capacity,
                          size_t* actual_output_size, cudaStream_t stream) {
    if (!finalized_) throw std::runtime_error("Pipeline not finalized");
    if (meta_.empty()) throw std::runtime_error("decompress() requires compress() to have been called first");
    if (!d_output_buf) throw std::runtime_error("decompress(): null output buffer");
    std::unordered_map<int, std::pair<void*, size_t>> outs;
    size_t off = pad16(4 + 8 * meta_.size());
    for (const auto& m : meta_) {
        void* p = dag_->getBuffer(m.buffer_id);
        if (d_input) {
            if (meta_.size() == 1) p = const_cast<void*>(d_input);
            else {
                p = static_cast<uint8_t*>(const_cast<void*>(d_input)) + off;
                off += pad16(m.actual_size);
            }
        }
        outs[m.buffer_id] = {p, m.actual_size};
    }
    if (decomp_exec_) {
        void* p = nullptr;
        size_t sz = 0;
        const bool managed = pool_managed_decomp_;
        pool_managed_decomp_ = true;
        try {
            decompress(d_input, input_size, &p, &sz, stream);
        } catch (...) {
            pool_managed_decomp_ = managed;
            throw;
        }
        pool_managed_decomp_ = managed;
        if (sz > output_buf_capacity)
            throw std::runtime_error("decompress(): output (" + std::to_string(sz) + " bytes) exceeds the buffer capacity");
        cuda_check(cudaMemcpyAsync(d_output_buf, p, sz, cudaMemcpyDeviceToDevice, stream), "decompress copy-out");
        *actual_output_size = sz;
        return;
    }
    if (output_buf_capacity >= input_size_) {
        runInverse(outs, d_output_buf, output_buf_capacity, actual_output_size, stream);
        return;
    }
    // the padded reconstruction does not fit: stage it and copy the prefix
    void* tmp = pool_->allocate(input_size_, stream, "decomp_stage", false);
    if (!tmp) throw std::runtime_error("decompress staging allocation failed");
    size_t sz = 0;
    try {
        runInverse(outs, tmp, input_size_, &sz, stream);
    } catch (...) {
        pool_->free(tmp, stream);
        throw;
    }
    if (sz > output_buf_capacity) {
        pool_->free(tmp, stream);
        throw std::runtime_error("decompress(): output (" + std::to_string(sz) + " bytes) exceeds the buffer capacity");
    }
    cuda_check(cudaMemcpyAsync(d_output_buf, tmp, sz, cudaMemcpyDeviceToDevice, stream), "decompress copy-out");
    pool_->free(tmp, stream);
    *actual_output_size = sz;
}

// --------------------------------------------------------- captured decompress

namespace {

// Stages whose inverse takes every size from the device or from values fixed
// at capture time (element counts, capacities).
bool inverse_on_device(Stage* s) {
    switch ((StageType)s->getStageTypeId()) {
        case StageType::LORENZO_QUANT:
        case StageType::BITSHUFFLE:
        case StageType::RZE:
        case StageType::RLE:
        case StageType::HUFFMAN:
            return true;
        case StageType::BITPACK:
            return s->isGraphCompatible();  // a fixed bit width
        default:
            return false;
    }
}

}  // namespace

void Pipeline::releaseDecompressGraph() {
    if (decomp_exec_) cudaGraphExecDestroy(decomp_exec_);
    if (decomp_graph_) cudaGraphDestroy(decomp_graph_);
    decomp_exec_ = nullptr;
    decomp_graph_ = nullptr;
    for (void* p : decomp_temps_) pool_->free(p, 0);
    decomp_temps_.clear();
    for (void** p : {&decomp_in_, &decomp_out_, &decomp_work_})
        if (*p) {
            pool_->free(*p, 0);
            *p = nullptr;
        }
    decomp_in_bytes_ = decomp_work_bytes_ = 0;
}

// What the decompression graph runs: the container in decomp_in_ is split on
// the device into the DAG's own output buffers, then the chain is inverted
// into decomp_out_ -- the fused LorenzoQuant <- Bitshuffle <- RZE pass, or
// stage by stage into intermediates kept from the first (uncaptured) pass.
// Sizes passed to the stages are capacities; the kernels read the actual
// sizes from the segments' own headers and counts.
void Pipeline::enqueueGraphInverse(cudaStream_t stream) {
    std::vector<void*> dsts;
    std::vector<uint64_t> caps;
    for (int id : output_buffer_ids_) {
        const BufferInfo& b = dag_->getBufferInfo(id);
        dsts.push_back(b.d_ptr);
        caps.push_back(b.allocated_size);
    }
    uint32_t* status = static_cast<uint32_t*>(decomp_work_);
    cuda_check(cudaMemsetAsync(status, 0, 256, stream), "decompress status");
    int rc = fzb_concat_split(decomp_in_, decomp_in_bytes_, dsts.data(), caps.data(), (int)dsts.size(), status,
                              stream);
    if (rc) throw std::runtime_error(std::string("decompress container split: ") + fzb_status_string(rc));
    auto consumer = [&](int buf) { return dag_->getNodes()[dag_->getBufferInfo(buf).consumer_stage_ids[0]]; };
    if (decomp_fused_) {
        auto* lq = static_cast<LorenzoQuantStage<float, uint16_t>*>(input_node_->stage);
        DAGNode* bsn = consumer(input_node_->output_index_to_buffer_id.at(0));
        DAGNode* rzn = consumer(bsn->output_buffer_ids[0]);
        auto* rz = static_cast<RZEStage*>(rzn->stage);
        const size_t n = rz->getCachedOrigBytes() / sizeof(uint16_t);
        const BufferInfo& rb = dag_->getBufferInfo(rzn->output_buffer_ids[0]);
        const BufferInfo& eb = dag_->getBufferInfo(input_node_->output_buffer_ids[1]);
        const auto d = lq->getDims();
        const uint32_t dims[3] = {(uint32_t)d[0], (uint32_t)d[1], (uint32_t)d[2]};
        rc = fzb_lq_bs_rze_decompress_dev(
            rb.d_ptr, rb.allocated_size, static_cast<const float*>(eb.d_ptr),
            static_cast<const uint32_t*>(dag_->getBuffer(input_node_->output_buffer_ids[2])),
            static_cast<const uint32_t*>(dag_->getBuffer(input_node_->output_buffer_ids[3])),
            eb.estimate / sizeof(float), n, dims, lq->deviceEbState() + 1, lq->getZigzagCodes() ? 1 : 0,
            static_cast<float*>(decomp_out_), static_cast<uint8_t*>(decomp_work_) + 256, decomp_work_bytes_ - 256,
            stream);
        if (rc) throw std::runtime_error(std::string("LorenzoQuant<-Bitshuffle<-RZE decompress: ") +
                                         fzb_status_string(rc));
        return;
    }
    std::unordered_map<int, std::pair<void*, size_t>> avail;
    for (int id : output_buffer_ids_) avail[id] = {dag_->getBuffer(id), dag_->getBufferInfo(id).estimate};
    std::vector<DAGNode*> order;
    for (const auto& lv : dag_->getLevels())
        for (auto* n : lv) order.push_back(n);
    size_t k = 0;
    for (auto it = order.rbegin(); it != order.rend(); ++it) {
        DAGNode* n = *it;
        std::vector<void*> in;
        std::vector<size_t> sizes;
        for (int id : n->output_buffer_ids) {
            const auto& a = avail.at(id);
            in.push_back(a.first);
            sizes.push_back(a.second);
        }
        void* out = nullptr;
        if (n->input_buffer_ids[0] == input_buffer_id_) {
            out = decomp_out_;
        } else {
            if (k == decomp_temps_.size()) {  // the first pass reserves the intermediates
                const size_t est = n->stage->estimateOutputSizes(sizes).at(0);
                void* t = pool_->allocate(est ? est : 256, stream, "graph_decompress_intermediate", true);
                if (!t) throw std::runtime_error("decompress: allocation failed");
                decomp_temps_.push_back(t);
            }
            out = decomp_temps_[k++];
        }
        n->stage->execute(stream, pool_.get(), in, {out}, sizes);
        avail[n->input_buffer_ids[0]] = {out, n->stage->getActualOutputSize(0)};
    }
}

bool Pipeline::captureDecompress(cudaStream_t stream) {
    releaseDecompressGraph();
    const size_t nout = output_buffer_ids_.size();
    if (nout < 2 || nout > FZB_CONCAT_MAX_SEGMENTS || fused_pfpl_) return false;
    for (auto& s : stages_)
        if (!inverse_on_device(s.get())) return false;
    for (int id : output_buffer_ids_) {
        const BufferInfo& b = dag_->getBufferInfo(id);
        if (!b.d_ptr || (b.allocated_size & 15) || (reinterpret_cast<uintptr_t>(b.d_ptr) & 15)) return false;
    }
    auto* lq = dynamic_cast<LorenzoQuantStage<float, uint16_t>*>(input_node_->stage);
    if (lq && !lq->deviceEbState()) return false;
    decomp_fused_ = fused_ && lq != nullptr;
    decomp_in_bytes_ = pad16(getMaxCompressedSize(graph_input_bytes_));
    decomp_in_ = pool_->allocate(decomp_in_bytes_, stream, "graph_decompress_input", true);
    decomp_out_ = pool_->allocate(graph_input_bytes_, stream, "graph_decompress_output", true);
    decomp_work_bytes_ = 256;
    if (decomp_fused_) {
        DAGNode* bsn = dag_->getNodes()[dag_->getBufferInfo(input_node_->output_index_to_buffer_id.at(0))
                                            .consumer_stage_ids[0]];
        DAGNode* rzn = dag_->getNodes()[dag_->getBufferInfo(bsn->output_buffer_ids[0]).consumer_stage_ids[0]];
        decomp_work_bytes_ += fzb_workspace_bytes(static_cast<RZEStage*>(rzn->stage)->getCachedOrigBytes() / 2, 0);
    }
    decomp_work_ = pool_->allocate(decomp_work_bytes_, stream, "graph_decompress_workspace", true);
    if (!decomp_in_ || !decomp_out_ || !decomp_work_) {
        releaseDecompressGraph();
        throw std::runtime_error("Failed to allocate the decompression graph's buffers");
    }
    // a container of the warm pass's outputs: the uncaptured first pass sizes
    // every stage workspace, so that nothing allocates inside the capture
    const auto saved_meta = meta_;
    collectMetadata();
    size_t sz = 0;
    concatOutputs(decomp_in_, decomp_in_bytes_, &sz, stream);
    meta_ = saved_meta;
    for (auto& s : stages_) s->saveState();
    for (auto& s : stages_) s->setInverse(true);
    if (lq) lq->setInverseDeviceErrorBound(true);
    auto restore = [&] {
        if (lq) lq->setInverseDeviceErrorBound(false);
        for (auto& s : stages_) {
            s->setInverse(false);
            s->restoreState();
        }
    };
    try {
        enqueueGraphInverse(stream);
        cuda_check(cudaStreamSynchronize(stream), "decompress graph warm pass");
        for (auto& s : stages_) s->postStreamSync(stream);
        const int st = fzb_workspace_status(decomp_work_, stream);
        if (st) throw std::runtime_error(std::string("decompress graph warm pass: ") + fzb_status_string(st));
        cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        capturing_ = true;
        try {
            enqueueGraphInverse(stream);
        } catch (...) {
            capturing_ = false;
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        capturing_ = false;
        cuda_check(cudaStreamEndCapture(stream, &decomp_graph_), "end capture");
        cuda_check(cudaGraphInstantiate(&decomp_exec_, decomp_graph_, 0), "graph instantiate");
    } catch (...) {
        restore();
        releaseDecompressGraph();
        throw;
    }
    restore();
    return true;
}

void Pipeline::checkDecompressStatus(cudaStream_t stream) {
    cuda_check(cudaStreamSynchronize(stream), "decompress");
    if (!decomp_exec_) return;  // eager decompressions report a bad input when they run
    int st = fzb_workspace_status(decomp_work_, stream);
    if (st == FZB_OK && decomp_fused_) st = fzb_workspace_status(static_cast<uint8_t*>(decomp_work_) + 256, stream);
    if (st != FZB_OK) throw std::runtime_error(std::string("decompress: ") + fzb_status_string(st));
    if (decomp_fused_) return;
    for (auto& s : stages_) s->saveState();
    try {
        for (auto& s : stages_) {
            s->setInverse(true);
            s->postStreamSync(stream);  // the inverse's workspace status
            s->setInverse(false);
        }
    } catch (...) {
        for (auto& s : stages_) {
            s->setInverse(false);
            s->restoreState();
        }
        throw;
    }
    for (auto& s : stages_) s->restoreState();
}

// ----------------------------------------------------------------------- FZM

Pipeline::FZMFileHeader Pipeline::buildHeader() const {
    if (!finalized_) throw std::runtime_error("Cannot build header before finalization");
    if (meta_.empty()) throw std::runtime_error("Cannot build header before compress() is called");
    FZMFileHeader fh;
    fh.core.uncompressed_size = input_size_;
    fh.core.num_sources = 1;
    fh.core.source_uncompressed_sizes[0] = input_size_;
    for (const auto& lv : dag_->getLevels())
        for (auto* n : lv) {
            FZMStageInfo si;
            si.stage_type = (StageType)n->stage->getStageTypeId();
            si.stage_version = 1;
            si.num_inputs = (uint8_t)n->input_buffer_ids.size();
            si.num_outputs = (uint8_t)n->output_buffer_ids.size();
            for (size_t i = 0; i < n->input_buffer_ids.size() && i < FZM_MAX_STAGE_INPUTS; i++)
                si.input_buffer_ids[i] = (uint16_t)n->input_buffer_ids[i];
            for (size_t i = 0; i < n->output_buffer_ids.size() && i < FZM_MAX_STAGE_OUTPUTS; i++)
                si.output_buffer_ids[i] = (uint16_t)n->output_buffer_ids[i];
            if (si.num_outputs) si.config_size = (uint32_t)n->stage->serializeHeader(0, si.stage_config, FZM_STAGE_CONFIG_SIZE);
            fh.stages.push_back(si);
        }
    fh.core.num_stages = (uint32_t)fh.stages.size();
    fh.core.num_buffers = (uint16_t)meta_.size();
    uint64_t off = 0;
    for (const auto& m : meta_) {
        FZMBufferEntry e;
        e.stage_type = (StageType)m.producer->stage->getStageTypeId();
        e.stage_version = 1;
        e.data_type = (DataType)m.producer->stage->getOutputDataType((size_t)m.output_index);
        e.producer_output_idx = (uint8_t)m.output_index;
        e.dag_buffer_id = (uint16_t)m.buffer_id;
        std::strncpy(e.name, m.name.c_str(), FZM_MAX_NAME_LEN - 1);
        e.data_size = m.actual_size;
        e.allocated_size = m.allocated_size;
        e.uncompressed_size = m.actual_size;
        e.byte_offset = off;
        e.config_size = (uint32_t)m.producer->stage->serializeHeader((size_t)m.output_index, e.stage_config,
                                                                     FZM_STAGE_CONFIG_SIZE);
        off += m.actual_size;
        fh.buffers.push_back(e);
    }
    fh.core.compressed_size = off;
    fh.core.header_size = fh.core.computeHeaderSize();
    return fh;
}

namespace {

// CRC-32 of `bytes` bytes of device memory, computed on the device
// (fzb_crc32) with its small workspace from `pool`; one 4-byte read-back.
uint32_t device_crc32(const void* d_data, size_t bytes, MemoryPool* pool, cudaStream_t stream) {
    const size_t need = fzb_crc32_workspace_bytes(bytes) + 256;
    uint8_t* w = static_cast<uint8_t*>(pool->allocate(need, stream, "crc32_workspace", false));
    if (!w) throw std::runtime_error("allocation for the CRC-32 workspace failed");
    uint32_t* d_crc = reinterpret_cast<uint32_t*>(w + need - 256);
    const int rc = fzb_crc32(d_data, bytes, d_crc, w, need - 256, stream);
    uint32_t crc = 0;
    if (rc == 0) cuda_check(cudaMemcpyAsync(&crc, d_crc, 4, cudaMemcpyDeviceToHost, stream), "CRC-32 read-back");
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize failed");
    pool->free(w, stream);
    if (rc) throw std::runtime_error(std::string("fzb_crc32: ") + fzb_status_string(rc));
    return crc;
}

uint32_t header_checksum(const Pipeline::FZMFileHeader& fh) {
    FZMHeaderCore c = fh.core;
    c.header_checksum = 0;
    uint32_t crc = crc32Update(0xFFFFFFFFu, &c, sizeof(c));
    if (!fh.stages.empty()) crc = crc32Update(crc, fh.stages.data(), fh.stages.size() * sizeof(FZMStageInfo));
    if (!fh.buffers.empty()) crc = crc32Update(crc, fh.buffers.data(), fh.buffers.size() * sizeof(FZMBufferEntry));
    return crc ^ 0xFFFFFFFFu;
}

}  // namespace

void Pipeline::writeToFile(const std::string& filename, cudaStream_t stream) {
    if (!finalized_) throw std::runtime_error("Cannot write to file before finalization");
    if (!compressed_) throw std::runtime_error("compress() must be called before writeToFile()");
    FZMFileHeader fh = buildHeader();
    std::vector<uint8_t> payload(fh.core.compressed_size);
    // the payload is the outputs back to back: gather them on the device, take
    // the checksum there, and read the payload back in one copy
    uint8_t* d_payload = nullptr;
    if (!payload.empty()) {
        d_payload = static_cast<uint8_t*>(pool_->allocate(payload.size(), stream, "fzm_payload", false));
        if (!d_payload) throw std::runtime_error("allocation for the FZM payload failed");
    }
    size_t off = 0;
    for (const auto& m : meta_) {
        if (m.actual_size)
            cuda_check(cudaMemcpyAsync(d_payload + off, dag_->getBuffer(m.buffer_id), m.actual_size,
                                       cudaMemcpyDeviceToDevice, stream),
                       "cudaMemcpyAsync failed");
        off += m.actual_size;
    }
    try {
        fh.core.data_checksum = device_crc32(d_payload, payload.size(), pool_.get(), stream);
        if (!payload.empty())
            cuda_check(cudaMemcpyAsync(payload.data(), d_payload, payload.size(), cudaMemcpyDeviceToHost, stream),
                       "cudaMemcpyAsync failed");
        cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize failed");
    } catch (...) {
        if (d_payload) pool_->free(d_payload, stream);
        throw;
    }
    if (d_payload) pool_->free(d_payload, stream);
    fh.core.flags |= FZM_FLAG_HAS_DATA_CHECKSUM | FZM_FLAG_HAS_HEADER_CHECKSUM;
    fh.core.header_checksum = header_checksum(fh);
    std::ofstream f(filename, std::ios::binary);
    if (!f) throw std::runtime_error("Failed to open file for writing: " + filename);
    f.write(reinterpret_cast<const char*>(&fh.core), sizeof(fh.core));
    if (!fh.stages.empty())
        f.write(reinterpret_cast<const char*>(fh.stages.data()), fh.stages.size() * sizeof(FZMStageInfo));
    if (!fh.buffers.empty())
        f.write(reinterpret_cast<const char*>(fh.buffers.data()), fh.buffers.size() * sizeof(FZMBufferEntry));
    if (!payload.empty()) f.write(reinterpret_cast<const char*>(payload.data()), payload.size());
    if (!f) throw std::runtime_error("Failed to write file: " + filename);
}

Pipeline::FZMFileHeader Pipeline::readHeader(const std::string& filename) {
    std::ifstream f(filename, std::ios::binary);
    if (!f) throw std::runtime_error("Failed to open file for reading: " + filename);
    uint32_t magic = 0;
    uint16_t version = 0;
    f.read(reinterpret_cast<char*>(&magic), 4);
    f.read(reinterpret_cast<char*>(&version), 2);
    if (!f) throw std::runtime_error("Failed to read header from file: " + filename);
    if (magic != FZM_MAGIC) throw std::runtime_error("Invalid FZM file format (bad magic number)");
    const uint8_t major = fzmVersionMajor(version), minor = fzmVersionMinor(version);
    if (major != FZM_VERSION_MAJOR)
        throw std::runtime_error("Incompatible FZM major version: file has major " + std::to_string(major) +
                                 ", reader expects major " + std::to_string(FZM_VERSION_MAJOR));
    const bool exact = minor == FZM_VERSION_MINOR, legacy = minor == 0;
    f.seekg(0, std::ios::beg);
    FZMFileHeader fh;
    fh.core = FZMHeaderCore();
    std::memset(static_cast<void*>(&fh.core), 0, sizeof(fh.core));
    f.read(reinterpret_cast<char*>(&fh.core), legacy ? FZM_LEGACY_HEADER_CORE_SIZE : sizeof(FZMHeaderCore));
    if (!f) throw std::runtime_error("Failed to read header from file: " + filename);
    if (fh.core.num_stages > FZM_MAX_BUFFERS || fh.core.num_buffers > FZM_MAX_BUFFERS)
        throw std::runtime_error("FZM header has too many stages/buffers");
    fh.stages.resize(fh.core.num_stages);
    if (fh.core.num_stages) {
        f.read(reinterpret_cast<char*>(fh.stages.data()), fh.core.num_stages * sizeof(FZMStageInfo));
        if (!f) throw std::runtime_error("Failed to read stage data from file: " + filename);
    }
    fh.buffers.resize(fh.core.num_buffers);
    if (fh.core.num_buffers) {
        f.read(reinterpret_cast<char*>(fh.buffers.data()), fh.core.num_buffers * sizeof(FZMBufferEntry));
        if (!f) throw std::runtime_error("Failed to read buffer data from file: " + filename);
    }
    if (!legacy && exact && (fh.core.flags & FZM_FLAG_HAS_HEADER_CHECKSUM)) {
        const uint32_t got = header_checksum(fh);
        if (got != fh.core.header_checksum)
            throw std::runtime_error("FZM header checksum mismatch in '" + filename + "': expected 0x" +
                                     hex8(fh.core.header_checksum) + ", computed 0x" + hex8(got) +
                                     " — file may be corrupted");
    }
    return fh;
}

void Pipeline::decompressFromFile(const std::string& filename, void** d_output, size_t* output_size,
                                  cudaStream_t stream, PipelinePerfResult* perf_out, size_t pool_override_bytes) {
    const auto t0 = std::chrono::steady_clock::now();
    FZMFileHeader fh = readHeader(filename);
    std::vector<uint8_t> payload(fh.core.compressed_size);
    {
        std::ifstream f(filename, std::ios::binary);
        if (!f) throw std::runtime_error("Failed to open file for reading: " + filename);
        f.seekg((std::streamoff)fh.core.header_size, std::ios::beg);
        if (!payload.empty()) f.read(reinterpret_cast<char*>(payload.data()), payload.size());
        if (!f) throw std::runtime_error("Failed to read compressed data from file: " + filename);
    }
    for (const auto& e : fh.buffers)
        if (e.byte_offset + e.data_size > fh.core.compressed_size)
            throw std::runtime_error("FZM buffer '" + std::string(e.name, strnlen(e.name, FZM_MAX_NAME_LEN)) +
                                     "' lies outside the payload");
    size_t max_u = fh.core.uncompressed_size;
    for (const auto& e : fh.buffers) max_u = std::max<size_t>(max_u, e.uncompressed_size);
    const size_t pool_bytes = pool_override_bytes ? pool_override_bytes
                                                  : (size_t)fh.core.compressed_size + (size_t)(2.5 * (double)max_u) +
                                                        (32ull << 20);
    MemoryPool pool(MemoryPoolConfig(pool_bytes, 1.0f));
    void* d_payload = nullptr;
    if (!payload.empty()) {
        d_payload = pool.allocate(payload.size(), stream, "compressed_data_load", false);
        if (!d_payload) throw std::runtime_error("allocation for the compressed data failed");
        cuda_check(cudaMemcpyAsync(d_payload, payload.data(), payload.size(), cudaMemcpyHostToDevice, stream),
                   "cudaMemcpyAsync failed");
        cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize failed");
    }
    if (fh.core.flags & FZM_FLAG_HAS_DATA_CHECKSUM) {  // checked on the device copy
        uint32_t got = 0;
        try {
            got = device_crc32(d_payload, payload.size(), &pool, stream);
        } catch (...) {
            if (d_payload) pool.free(d_payload, stream);
            throw;
        }
        if (got != fh.core.data_checksum) {
            if (d_payload) pool.free(d_payload, stream);
            throw std::runtime_error("FZM data checksum mismatch in '" + filename + "': expected 0x" +
                                     hex8(fh.core.data_checksum) + ", computed 0x" + hex8(got) +
                                     " — compressed data may be corrupted");
        }
    }
    std::vector<std::unique_ptr<Stage>> owned;
    std::vector<FwdDesc> fwd;
    std::unordered_set<int> produced;
    for (const auto& si : fh.stages) {
        owned.emplace_back(createStage(si.stage_type, si.stage_config, si.config_size));
        FwdDesc d{owned.back().get(), {}, {}};
        for (int j = 0; j < si.num_inputs && j < (int)FZM_MAX_STAGE_INPUTS; j++)
            if (si.input_buffer_ids[j] != 0xFFFF) d.in_ids.push_back(si.input_buffer_ids[j]);
        for (int j = 0; j < si.num_outputs && j < (int)FZM_MAX_STAGE_OUTPUTS; j++)
            if (si.output_buffer_ids[j] != 0xFFFF) {
                d.out_ids.push_back(si.output_buffer_ids[j]);
                produced.insert(si.output_buffer_ids[j]);
            }
        fwd.push_back(d);
    }
    int source_buf = -1;
    for (const auto& d : fwd)
        for (int id : d.in_ids)
            if (!produced.count(id) && source_buf < 0) source_buf = id;
    if (source_buf < 0) {
        if (d_payload) pool.free(d_payload, stream);
        throw std::runtime_error("decompressFromFile: could not identify any source stage in topology");
    }
    Avail avail;
    for (const auto& e : fh.buffers)
        avail[(int)e.dag_buffer_id] = {static_cast<uint8_t*>(d_payload) + e.byte_offset, (size_t)e.data_size};
    size_t src_bytes = fh.core.num_sources && fh.core.source_uncompressed_sizes[0] ? fh.core.source_uncompressed_sizes[0]
                                                                                   : fh.core.uncompressed_size;
    void* d_final = nullptr;
    cuda_check(cudaMalloc(&d_final, src_bytes ? src_bytes : 1), "cudaMalloc for decompressed output failed");
    size_t got = 0;
    const auto t1 = std::chrono::steady_clock::now();
    try {
        run_inverse(fwd, avail, source_buf, &pool, d_final, src_bytes, &got, stream, true);
    } catch (...) {
        cudaStreamSynchronize(stream);
        cudaFree(d_final);
        if (d_payload) pool.free(d_payload, stream);
        throw;
    }
    const auto t2 = std::chrono::steady_clock::now();
    if (d_payload) pool.free(d_payload, stream);
    cudaStreamSynchronize(stream);
    *d_output = d_final;
    *output_size = got;
    if (perf_out) {
        *perf_out = PipelinePerfResult();
        perf_out->is_compress = false;
        perf_out->input_bytes = fh.core.compressed_size;
        perf_out->output_bytes = got;
        perf_out->dag_elapsed_ms = std::chrono::duration<float, std::milli>(t2 - t1).count();
        perf_out->host_elapsed_ms = std::chrono::duration<float, std::milli>(t2 - t0).count();
    }
}

}  // namespace fz
