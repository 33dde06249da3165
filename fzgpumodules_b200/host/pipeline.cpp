// pipeline.cpp -- DAG construction and execution for fz::Pipeline.
//
// Buffer ids follow the order the reference assigns them in
// (src/pipeline/compressor.cpp:150-170,536-548; src/pipeline/dag.cpp:79-246):
// every output slot of a stage gets an id when the stage is added, connect()
// reuses the producer's slot, and the source input buffers are numbered at
// finalize().  Levels are longest-path depths (dag.cpp:725-750).
#include "fz/pipeline.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>
#include <queue>
#include <stdexcept>

#include "fzb.h"

namespace fz {

namespace {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

inline size_t pad16(size_t v) { return (v + 15) & ~(size_t)15; }
inline size_t pad256(size_t v) { return (v + 255) & ~(size_t)255; }

bool types_compatible(uint8_t a, uint8_t b) {
    if (a == b) return true;
    const DataType da = (DataType)a, db = (DataType)b;
    const bool af = da == DataType::FLOAT32 || da == DataType::FLOAT64;
    const bool bf = db == DataType::FLOAT32 || db == DataType::FLOAT64;
    if (af || bf) return false;
    return getDataTypeSize(da) == getDataTypeSize(db);
}

}  // namespace

// ============================================================ ResultGather

ResultGather::~ResultGather() {
    if (host_) cudaFreeHost(host_);
}

bool ResultGather::enqueue(const std::vector<DeviceRead>& reads, cudaStream_t stream) {
    if (reads.empty() || reads.size() > FZB_GATHER_MAX) return false;
    size_t total = 0;
    for (const auto& r : reads) total += (r.bytes + 7) & ~(size_t)7;
    if (total > kBytes) return false;
    if (!host_) {
        void* h = nullptr;
        if (cudaHostAlloc(&h, kBytes, cudaHostAllocMapped) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        void* d = nullptr;
        if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
            cudaGetLastError();
            cudaFreeHost(h);
            return false;
        }
        host_ = h;
        dev_ = d;
    }
    const void* src[FZB_GATHER_MAX];
    uint32_t bytes[FZB_GATHER_MAX];
    uint8_t clear[FZB_GATHER_MAX];
    for (size_t i = 0; i < reads.size(); i++) {
        src[i] = reads[i].src;
        bytes[i] = reads[i].bytes;
        clear[i] = reads[i].clear ? 1 : 0;
    }
    return fzb_gather_words(src, bytes, clear, (int)reads.size(), dev_, stream) == FZB_OK;
}

void ResultGather::finish(const std::vector<DeviceRead>& reads) const {
    const uint8_t* h = static_cast<const uint8_t*>(host_);
    size_t off = 0;
    for (const auto& r : reads) {
        std::memcpy(r.dst, h + off, r.bytes);
        off += (r.bytes + 7) & ~(size_t)7;
    }
}

float PipelinePerfResult::throughput_gbs() const {
    float ms = 0.0f;
    for (const auto& s : stages) ms += s.elapsed_ms;
    if (ms <= 0.0f) ms = dag_elapsed_ms;
    const size_t bytes = is_compress ? input_bytes : output_bytes;
    return ms > 0.0f ? (float)bytes / (ms * 1e-3f) / 1e9f : 0.0f;
}

// ======================================================================= DAG

CompressionDAG::CompressionDAG(MemoryPool* pool, MemoryStrategy strategy) : pool_(pool), strategy_(strategy) {}

CompressionDAG::~CompressionDAG() {
    releaseAll(0);
    for (auto* n : nodes_) {
        if (n->start_event) cudaEventDestroy(n->start_event);
        if (n->end_event) cudaEventDestroy(n->end_event);
        delete n;
    }
}

DAGNode* CompressionDAG::addStage(Stage* stage, const std::string& name) {
    auto* n = new DAGNode();
    n->id = (int)nodes_.size();
    n->stage = stage;
    n->name = name.empty() ? "stage_" + std::to_string(n->id) : name;
    nodes_.push_back(n);
    return n;
}

int CompressionDAG::addUnconnectedOutput(DAGNode* node, int output_index, const std::string& tag) {
    const int id = next_buffer_id_++;
    BufferInfo& b = buffers_[id];
    b.size = 1;
    b.tag = tag;
    b.producer_stage_id = node->id;
    b.producer_output_index = output_index;
    node->output_buffer_ids.push_back(id);
    node->output_index_to_buffer_id[output_index] = id;
    return id;
}

bool CompressionDAG::connectExistingOutput(DAGNode* producer, DAGNode* consumer, int output_index) {
    auto it = producer->output_index_to_buffer_id.find(output_index);
    if (it == producer->output_index_to_buffer_id.end()) return false;
    BufferInfo& b = buffers_[it->second];
    consumer->input_buffer_ids.push_back(it->second);
    b.consumer_stage_ids.push_back(consumer->id);
    consumer->dependencies.push_back(producer);
    producer->dependents.push_back(consumer);
    b.tag = producer->name + "_to_" + consumer->name;
    b.is_persistent = false;
    return true;
}

int CompressionDAG::setInputBuffer(DAGNode* node, const std::string& tag) {
    const int id = next_buffer_id_++;
    BufferInfo& b = buffers_[id];
    b.size = 1;
    b.tag = tag;
    b.is_persistent = true;
    b.is_external = true;
    b.producer_stage_id = -1;
    node->input_buffer_ids.push_back(id);
    b.consumer_stage_ids.push_back(node->id);
    return id;
}

void CompressionDAG::finalize() {
    // Kahn order; a leftover node means a cycle
    std::vector<int> indeg(nodes_.size(), 0);
    for (auto* n : nodes_)
        for (auto* d : n->dependents) indeg[d->id]++;
    std::queue<DAGNode*> q;
    for (auto* n : nodes_)
        if (indeg[n->id] == 0) q.push(n);
    std::vector<DAGNode*> order;
    while (!q.empty()) {
        DAGNode* n = q.front();
        q.pop();
        order.push_back(n);
        for (auto* d : n->dependents)
            if (--indeg[d->id] == 0) q.push(d);
    }
    if (order.size() != nodes_.size())
        throw std::runtime_error("Cyclic dependency detected in pipeline graph! Topological sort visited " +
                                 std::to_string(order.size()) + " of " + std::to_string(nodes_.size()) +
                                 " nodes");
    for (auto* n : order) {
        int lv = 0;
        for (auto* d : n->dependencies) lv = std::max(lv, d->level + 1);
        n->level = lv;
    }
    int max_level = 0;
    for (auto* n : nodes_) max_level = std::max(max_level, n->level);
    levels_.assign(max_level + 1, {});
    for (auto* n : nodes_) levels_[n->level].push_back(n);  // insertion order within a level
    // buffer lifetimes in levels: produced at the producer's level, dead
    // after the last consumer's level (pipeline outputs live to the end)
    for (auto& kv : buffers_) {
        BufferInfo& b = kv.second;
        b.first_level = b.producer_stage_id >= 0 ? nodes_[b.producer_stage_id]->level : 0;
        b.last_level = b.first_level;
        for (int c : b.consumer_stage_ids) b.last_level = std::max(b.last_level, nodes_[c]->level);
        if (b.is_persistent) b.last_level = max_level + 1;
    }
}

void CompressionDAG::allocate(int id, cudaStream_t stream) {
    BufferInfo& b = buffers_.at(id);
    if (b.is_external) return;
    if (b.d_ptr && b.allocated_size >= b.size) return;
    if (strategy_ == MemoryStrategy::PREALLOCATE && arena_) {
        if (b.size <= b.allocated_size) return;
        throw std::runtime_error("buffer '" + b.tag + "' outgrew its preallocated slot (" +
                                 std::to_string(b.size) + " > " + std::to_string(b.allocated_size) + " bytes)");
    }
    if (b.d_ptr) release(id, stream);
    if (b.size == 0) {
        b.d_ptr = nullptr;
        b.allocated_size = 0;
        return;
    }
    b.d_ptr = pool_->allocate(b.size, stream, b.tag, b.is_persistent);
    if (!b.d_ptr) throw std::runtime_error("Failed to allocate buffer: " + b.tag);
    b.allocated_size = b.size;
}

void CompressionDAG::release(int id, cudaStream_t stream) {
    BufferInfo& b = buffers_.at(id);
    if (b.is_external || !b.d_ptr) return;
    if (arena_) return;  // arena slots live until the DAG goes away
    pool_->free(b.d_ptr, stream);
    b.d_ptr = nullptr;
    b.allocated_size = 0;
}

void CompressionDAG::releaseAll(cudaStream_t stream) {
    if (arena_) {
        pool_->free(arena_, stream);
        arena_ = nullptr;
        for (auto& kv : buffers_)
            if (!kv.second.is_external) {
                kv.second.d_ptr = nullptr;
                kv.second.allocated_size = 0;
            }
        return;
    }
    for (auto& kv : buffers_) release(kv.first, stream);
}

// Interval colouring: buffers sorted by size (largest first) take the lowest
// arena offset whose occupants' level ranges do not overlap theirs.
void CompressionDAG::preallocate(cudaStream_t stream) {
    if (arena_) return;
    std::vector<int> ids;
    for (auto& kv : buffers_)
        if (!kv.second.is_external && kv.second.size > 0) ids.push_back(kv.first);
    std::sort(ids.begin(), ids.end(), [&](int a, int b) {
        const size_t sa = buffers_[a].size, sb = buffers_[b].size;
        return sa != sb ? sa > sb : a < b;
    });
    struct Placed {
        size_t off, end;
        int lo, hi;
    };
    std::vector<Placed> placed;
    size_t total = 0;
    for (int id : ids) {
        BufferInfo& b = buffers_[id];
        const size_t need = pad256(b.size);
        std::vector<std::pair<size_t, size_t>> busy;
        for (const auto& p : placed)
            if (!(p.hi < b.first_level || b.last_level < p.lo)) busy.push_back({p.off, p.end});
        std::sort(busy.begin(), busy.end());
        size_t off = 0;
        for (const auto& r : busy) {
            if (off + need <= r.first) break;
            off = std::max(off, r.second);
        }
        placed.push_back({off, off + need, b.first_level, b.last_level});
        b.arena_offset = off;
        total = std::max(total, off + need);
    }
    regions_ = 0;
    {
        std::vector<size_t> offs;
        for (const auto& p : placed) offs.push_back(p.off);
        std::sort(offs.begin(), offs.end());
        regions_ = std::unique(offs.begin(), offs.end()) - offs.begin();
    }
    if (total == 0) return;
    arena_ = pool_->allocate(total, stream, "dag_arena", true);
    if (!arena_) throw std::runtime_error("Failed to preallocate the pipeline arena (" + std::to_string(total) + " bytes)");
    arena_bytes_ = total;
    for (int id : ids) {
        BufferInfo& b = buffers_[id];
        b.d_ptr = static_cast<uint8_t*>(arena_) + b.arena_offset;
        b.allocated_size = pad256(b.size);
    }
}

// ================================================================== Pipeline

Pipeline::Pipeline(size_t input_data_size, MemoryStrategy strategy, float pool_multiplier)
    : strategy_(strategy), pool_multiplier_(pool_multiplier), input_size_hint_(input_data_size) {
    pool_.reset(new MemoryPool(MemoryPoolConfig(input_data_size, pool_multiplier)));
    dag_.reset(new CompressionDAG(pool_.get(), strategy));
}

Pipeline::~Pipeline() {
    cudaDeviceSynchronize();
    releaseDecompressGraph();
    for (cudaEvent_t e : fork_events_) cudaEventDestroy(e);
    for (cudaEvent_t e : join_events_) cudaEventDestroy(e);
    for (cudaStream_t st : side_streams_) cudaStreamDestroy(st);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (void* p : decomp_outputs_) pool_->free(p, 0);
    if (pad_buf_) pool_->free(pad_buf_, 0);
    if (concat_buf_) pool_->free(concat_buf_, 0);
    if (graph_input_) pool_->free(graph_input_, 0);
    if (d_fused_size_) pool_->free(d_fused_size_, 0);
    if (inv_work_) pool_->free(inv_work_, 0);
    dag_.reset();
    stages_.clear();
}

void Pipeline::setMemoryStrategy(MemoryStrategy strategy) {
    if (finalized_) throw std::runtime_error("Cannot change strategy after finalization");
    strategy_ = strategy;
    // rebuild the DAG with the same stages and connections
    auto conns = connections_;
    std::vector<Stage*> order;
    for (auto* n : stage_nodes_) order.push_back(n->stage);
    dag_.reset(new CompressionDAG(pool_.get(), strategy));
    stage_nodes_.clear();
    for (Stage* s : order) {
        DAGNode* n = dag_->addStage(s, s->getName());
        const auto names = s->getOutputNames();
        for (size_t i = 0; i < s->getNumOutputs(); i++)
            dag_->addUnconnectedOutput(n, (int)i, s->getName() + "." + (i < names.size() ? names[i] : std::to_string(i)) +
                                                      "_unconnected");
        stage_nodes_.push_back(n);
    }
    connections_.clear();
    for (const auto& c : conns) connect(c.dependent, c.producer, c.output_name);
}

void Pipeline::setNumStreams(int num_streams) {
    if (finalized_) throw std::runtime_error("Cannot configure streams after finalization");
    num_streams_ = num_streams;
}

void Pipeline::enableGraphMode(bool enable) {
    if (finalized_) throw std::runtime_error("Cannot change graph mode after finalization");
    graph_mode_ = enable;
}

Stage* Pipeline::addRawStage(Stage* stage) {
    if (finalized_) {
        delete stage;
        throw std::runtime_error("Cannot add stages after finalization");
    }
    stage->setDims(dims_);
    DAGNode* n = dag_->addStage(stage, stage->getName());
    const auto names = stage->getOutputNames();
    for (size_t i = 0; i < stage->getNumOutputs(); i++)
        dag_->addUnconnectedOutput(n, (int)i,
                                   stage->getName() + "." + (i < names.size() ? names[i] : std::to_string(i)) +
                                       "_unconnected");
    stages_.emplace_back(stage);
    stage_nodes_.push_back(n);
    return stage;
}

int Pipeline::connect(Stage* dependent, Stage* producer, const std::string& output_name) {
    if (finalized_) throw std::runtime_error("Cannot connect stages after finalization");
    DAGNode *dn = nullptr, *pn = nullptr;
    for (auto* n : stage_nodes_) {
        if (n->stage == dependent) dn = n;
        if (n->stage == producer) pn = n;
    }
    if (!dn || !pn) throw std::runtime_error("Cannot connect stages not added to pipeline");
    const int idx = producer->getOutputIndex(output_name);
    if (idx < 0)
        throw std::runtime_error("Stage '" + producer->getName() + "' does not have output '" + output_name + "'");
    connections_.push_back({dependent, producer, output_name, idx});
    if (!dag_->connectExistingOutput(pn, dn, idx))
        throw std::runtime_error("internal: missing output slot for " + producer->getName() + "." + output_name);
    return pn->output_index_to_buffer_id.at(idx);
}

int Pipeline::connect(Stage* dependent, const std::vector<Stage*>& producers) {
    int last = -1;
    for (Stage* p : producers) last = connect(dependent, p);
    return last;
}

void Pipeline::finalize() {
    if (finalized_) throw std::runtime_error("Pipeline already finalized");
    if (stages_.empty()) throw std::runtime_error("Pipeline has no stages");
    for (auto& s : stages_) s->setDims(dims_);
    if (!connections_.empty()) {
        for (auto& s : stages_) {
            bool seen = false;
            for (const auto& c : connections_) seen |= (c.dependent == s.get() || c.producer == s.get());
            if (!seen)
                throw std::runtime_error("Stage '" + s->getName() +
                                         "' has no connections; every stage in a connected pipeline must be "
                                         "linked to at least one other stage via connect()");
        }
    }
    for (const auto& c : connections_) {  // type check (compressor.cpp:211-247)
        const uint8_t pt = c.producer->getOutputDataType((size_t)c.output_index);
        const uint8_t ct = c.dependent->getInputDataType(0);
        if (pt == (uint8_t)DataType::UNKNOWN || ct == (uint8_t)DataType::UNKNOWN) continue;
        if (!types_compatible(pt, ct))
            throw std::runtime_error("Type mismatch: '" + c.producer->getName() + "' output '" + c.output_name +
                                     "' has type " + dataTypeToString((DataType)pt) + " but '" +
                                     c.dependent->getName() + "' expects " + dataTypeToString((DataType)ct));
    }
    std::vector<DAGNode*> sources;
    for (auto* n : stage_nodes_)
        if (n->dependencies.empty()) sources.push_back(n);
    bool has_sink = false;
    for (auto* n : stage_nodes_) has_sink |= n->dependents.empty();
    if (sources.empty() || !has_sink) throw std::runtime_error("Pipeline has no source or sink stages");
    if (sources.size() != 1)
        throw std::runtime_error("only single-source pipelines are supported (" + std::to_string(sources.size()) +
                                 " sources)");
    input_node_ = sources[0];
    input_buffer_id_ = dag_->setInputBuffer(input_node_, "pipeline_input");
    // unconnected outputs become pipeline outputs, in stage order
    for (auto* n : stage_nodes_) {
        const auto names = n->stage->getOutputNames();
        for (size_t i = 0; i < n->stage->getNumOutputs(); i++) {
            const int id = n->output_index_to_buffer_id.at((int)i);
            BufferInfo& b = dag_->buffer(id);
            if (!b.consumer_stage_ids.empty()) continue;
            b.tag = "pipeline_output_" + n->stage->getName() + "." + (i < names.size() ? names[i] : std::to_string(i));
            b.is_persistent = true;
            output_buffer_ids_.push_back(id);
            output_nodes_.push_back(n);
        }
    }
    if (output_buffer_ids_.size() > FZM_MAX_BUFFERS)
        throw std::runtime_error("too many pipeline outputs (" + std::to_string(output_buffer_ids_.size()) + ")");
    dag_->finalize();
    // input alignment: LCM of the stages' requirements (compressor.cpp:249-265)
    size_t align = 1;
    for (auto& s : stages_) {
        const size_t a = s->getRequiredInputAlignment();
        if (a > 1) align = std::lcm(align, a);
    }
    input_alignment_ = align;
    if (align > 1 && input_size_hint_) input_size_hint_ = (input_size_hint_ + align - 1) / align * align;
    detectFusion();
    if (input_size_hint_) propagateBufferSizes(input_size_hint_);
    for (const auto& lv : dag_->getLevels())
        for (auto* n : lv) {
            const size_t inlen = n->input_buffer_ids.empty() ? 0 : dag_->getBufferSize(n->input_buffer_ids[0]);
            n->stage->onFinalize(inlen, pool_.get());
        }
    {   // side streams for levels with several stages (dag.cpp:262-285, 343-369)
        size_t widest = 1;
        for (const auto& lv : dag_->getLevels()) widest = std::max(widest, lv.size());
        const int ns = std::max<int>(num_streams_, (int)widest);
        if (ns > 1 && widest > 1) {
            for (int i = 0; i < ns; i++) {
                cudaStream_t st = nullptr;
                cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "Failed to create CUDA stream");
                side_streams_.push_back(st);
            }
            for (size_t i = 0; i < dag_->getLevels().size(); i++) {
                cudaEvent_t e = nullptr;
                cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "level fork event");
                fork_events_.push_back(e);
            }
            for (size_t i = 0; i < dag_->getNodes().size(); i++) {
                cudaEvent_t e = nullptr;
                cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "stage join event");
                join_events_.push_back(e);
            }
        }
        // the count the pipeline reports (and saveConfig writes) is the
        // reference's: the requested count, or the widest level when larger
        num_streams_ = ns > 1 ? ns : 1;
    }
    d_fused_size_ = static_cast<uint64_t*>(pool_->allocate(256, 0, "fused_stream_size", true));
    if (strategy_ == MemoryStrategy::PREALLOCATE && input_size_hint_) dag_->preallocate(0);
    if (graph_mode_) {
        if (strategy_ != MemoryStrategy::PREALLOCATE)
            throw std::runtime_error("Graph mode requires PREALLOCATE memory strategy.");
        if (!input_size_hint_) throw std::runtime_error("Graph mode requires a non-zero input size hint.");
        for (auto& s : stages_)
            if (!s->isGraphCompatible())
                throw std::runtime_error("stage '" + s->getName() + "' is not graph-compatible");
        graph_input_bytes_ = input_size_hint_;
        graph_input_ = pool_->allocate(graph_input_bytes_, 0, "graph_input_slot", true);
        if (!graph_input_) throw std::runtime_error("Failed to allocate graph input slot");
    }
    cuda_check(cudaStreamSynchronize(0), "finalize");
    finalized_ = true;
    if (warmup_on_finalize_ && input_size_hint_) warmup(0);
}

void Pipeline::detectFusion() {
    fused_ = false;
    fused_pfpl_ = false;
    if (!fusion_enabled_) return;
    auto* lq = dynamic_cast<LorenzoQuantStage<float, uint16_t>*>(input_node_->stage);
    auto* qs = dynamic_cast<QuantizerStage<float, uint32_t>*>(input_node_->stage);
    if (!lq && !(qs && !qs->isInplace())) return;
    const int codes = input_node_->output_index_to_buffer_id.at(0);
    const BufferInfo& cb = dag_->getBufferInfo(codes);
    if (cb.consumer_stage_ids.size() != 1) return;
    DAGNode* bsn = dag_->getNodes()[cb.consumer_stage_ids[0]];
    if (qs) {  // Quantizer -> Difference(int32 -> uint32, 16 KiB) -> ...
        auto* df = dynamic_cast<DifferenceStage<int32_t, uint32_t>*>(bsn->stage);
        if (!df || df->getChunkSize() != 16384 || bsn->input_buffer_ids.size() != 1) return;
        const BufferInfo& db = dag_->getBufferInfo(bsn->output_buffer_ids[0]);
        if (db.consumer_stage_ids.size() != 1) return;
        bsn = dag_->getNodes()[db.consumer_stage_ids[0]];
    }
    auto* bs = dynamic_cast<BitshuffleStage*>(bsn->stage);
    if (!bs || bs->getBlockSize() != 16384 || bs->getElementWidth() != 2 || bsn->input_buffer_ids.size() != 1) return;
    const BufferInfo& bb = dag_->getBufferInfo(bsn->output_buffer_ids[0]);
    if (bb.consumer_stage_ids.size() != 1) return;
    DAGNode* rzn = dag_->getNodes()[bb.consumer_stage_ids[0]];
    auto* rz = dynamic_cast<RZEStage*>(rzn->stage);
    if (!rz || rz->getChunkSize() != 16384 || rz->getLevels() != 4 || rzn->input_buffer_ids.size() != 1) return;
    fused_ = true;
    fused_pfpl_ = qs != nullptr;
}

void Pipeline::propagateBufferSizes(size_t source_bytes) {
    dag_->buffer(input_buffer_id_).size = source_bytes;
    dag_->buffer(input_buffer_id_).estimate = source_bytes;
    for (const auto& lv : dag_->getLevels())
        for (auto* n : lv) {
            std::vector<size_t> in;
            for (int id : n->input_buffer_ids) in.push_back(dag_->getBufferSize(id));
            const auto est = n->stage->estimateOutputSizes(in);
            for (size_t i = 0; i < n->output_buffer_ids.size() && i < est.size(); i++) {
                BufferInfo& b = dag_->buffer(n->output_buffer_ids[i]);
                b.size = est[i];
                b.estimate = est[i];
            }
        }
}

size_t Pipeline::getMaxCompressedSize(size_t input_bytes) const {
    if (!finalized_) throw std::runtime_error("getMaxCompressedSize() requires a finalized pipeline");
    size_t padded = input_alignment_ > 1 ? (input_bytes + input_alignment_ - 1) / input_alignment_ * input_alignment_
                                         : input_bytes;
    std::unordered_map<int, size_t> sz;
    sz[input_buffer_id_] = padded;
    for (const auto& lv : dag_->getLevels())
        for (auto* n : lv) {
            std::vector<size_t> in;
            for (int id : n->input_buffer_ids) in.push_back(sz[id]);
            const auto est = n->stage->estimateOutputSizes(in);
            for (size_t i = 0; i < n->output_buffer_ids.size() && i < est.size(); i++) sz[n->output_buffer_ids[i]] = est[i];
        }
    if (output_buffer_ids_.size() == 1) return sz[output_buffer_ids_[0]];
    size_t total = pad16(4 + 8 * output_buffer_ids_.size());
    for (int id : output_buffer_ids_) total += pad16(sz[id]);
    return total;
}

const void* Pipeline::prepareInput(const void* d_input, size_t input_size, cudaStream_t stream, size_t* padded) {
    original_input_size_ = 0;
    if (input_alignment_ > 1 && input_size % input_alignment_ != 0) {
        const size_t p = (input_size + input_alignment_ - 1) / input_alignment_ * input_alignment_;
        if (p > pad_bytes_) {
            if (pad_buf_) pool_->free(pad_buf_, stream);
            pad_buf_ = pool_->allocate(p, stream, "pipeline_input_pad", true);
            if (!pad_buf_) throw std::runtime_error("Failed to allocate pipeline input pad buffer");
            pad_bytes_ = p;
        }
        cuda_check(cudaMemcpyAsync(pad_buf_, d_input, input_size, cudaMemcpyDeviceToDevice, stream), "input pad");
        cuda_check(cudaMemsetAsync(static_cast<uint8_t*>(pad_buf_) + input_size, 0, p - input_size, stream),
                   "input pad");
        original_input_size_ = input_size;
        *padded = p;
        return pad_buf_;
    }
    *padded = input_size;
    return d_input;
}

// Runs every node level by level, as the reference DAG does
// (dag.cpp:382-510).  Input sizes come from the producer's execute-time size
// (or the propagated estimate when that is 0).  A level with several stages
// forks from `stream` onto the side streams and joins back before the next
// level; everything else runs on `stream`.
void Pipeline::runForward(cudaStream_t stream) {
    std::unordered_map<int, int> remaining;
    for (auto* n : dag_->getNodes())
        for (int id : n->input_buffer_ids) remaining[id]++;
    std::vector<bool> skip(dag_->getNodes().size(), false);
    if (fused_) {
        const BufferInfo& cb = dag_->getBufferInfo(input_node_->output_index_to_buffer_id.at(0));
        DAGNode* bsn = dag_->getNodes()[cb.consumer_stage_ids[0]];
        if (fused_pfpl_) {
            skip[bsn->id] = true;
            bsn = dag_->getNodes()[dag_->getBufferInfo(bsn->output_buffer_ids[0]).consumer_stage_ids[0]];
        }
        DAGNode* rzn = dag_->getNodes()[dag_->getBufferInfo(bsn->output_buffer_ids[0]).consumer_stage_ids[0]];
        skip[bsn->id] = skip[rzn->id] = true;
    }
    const auto& levels = dag_->getLevels();
    for (size_t lv = 0; lv < levels.size(); lv++) {
        std::vector<DAGNode*> run;
        for (auto* n : levels[lv])
            if (!skip[n->id]) run.push_back(n);
        if (run.size() > 1 && !side_streams_.empty()) {
            // outputs are reserved on the caller's stream before the fork
            for (auto* n : run)
                for (int id : n->output_buffer_ids) dag_->allocate(id, stream);
            cuda_check(cudaEventRecord(fork_events_[lv], stream), "level fork");
            for (size_t k = 0; k < run.size(); k++) {
                cudaStream_t s = side_streams_[k % side_streams_.size()];
                cuda_check(cudaStreamWaitEvent(s, fork_events_[lv], 0), "level fork");
                runNode(run[k], s);
                cuda_check(cudaEventRecord(join_events_[run[k]->id], s), "level join");
            }
            for (auto* n : run) cuda_check(cudaStreamWaitEvent(stream, join_events_[n->id], 0), "level join");
        } else {
            for (auto* n : run) runNode(n, stream);
        }
        if (strategy_ == MemoryStrategy::MINIMAL)
            for (auto* n : run)
                for (int id : n->input_buffer_ids)
                    if (--remaining[id] == 0 && !dag_->getBufferInfo(id).is_persistent) dag_->release(id, stream);
    }
}

// One stage on `stream`: the fused chain when `n` starts it, else the
// stage's own execute(); then the sizes its consumers see.
void Pipeline::runNode(DAGNode* n, cudaStream_t stream) {
    std::vector<void*> in, out;
    std::vector<size_t> sizes;
    for (int id : n->input_buffer_ids) {
        const BufferInfo& b = dag_->getBufferInfo(id);
        in.push_back(b.d_ptr);
        sizes.push_back(b.size);
    }
    if (profiling_enabled_) {
        if (!n->start_event) cudaEventCreate(&n->start_event);
        if (!n->end_event) cudaEventCreate(&n->end_event);
        cudaEventRecord(n->start_event, stream);
    }
    if (fused_ && n == input_node_) {
        const BufferInfo& cb = dag_->getBufferInfo(n->output_index_to_buffer_id.at(0));
        DAGNode* bsn = dag_->getNodes()[cb.consumer_stage_ids[0]];
        DAGNode* dfn = nullptr;
        if (fused_pfpl_) {
            dfn = bsn;
            bsn = dag_->getNodes()[dag_->getBufferInfo(dfn->output_buffer_ids[0]).consumer_stage_ids[0]];
        }
        DAGNode* rzn = dag_->getNodes()[dag_->getBufferInfo(bsn->output_buffer_ids[0]).consumer_stage_ids[0]];
        for (int i = 1; i < 4; i++) dag_->allocate(n->output_buffer_ids[i], stream);
        const int rz_out = rzn->output_buffer_ids[0];
        dag_->allocate(rz_out, stream);
        size_t code_bytes;
        if (fused_pfpl_) {
            auto* qs = static_cast<QuantizerStage<float, uint32_t>*>(n->stage);
            qs->fusedForward(stream, pool_.get(), in[0], sizes[0], dag_->getBuffer(n->output_buffer_ids[1]),
                             dag_->getBuffer(n->output_buffer_ids[2]), dag_->getBuffer(n->output_buffer_ids[3]),
                             dag_->getBuffer(rz_out), d_fused_size_);
            code_bytes = sizes[0];  // one uint32 code per float
            static_cast<DifferenceStage<int32_t, uint32_t>*>(dfn->stage)->markFused(code_bytes);
        } else {
            auto* lq = static_cast<LorenzoQuantStage<float, uint16_t>*>(n->stage);
            lq->fusedForward(stream, pool_.get(), in[0], sizes[0], dag_->getBuffer(n->output_buffer_ids[1]),
                             dag_->getBuffer(n->output_buffer_ids[2]), dag_->getBuffer(n->output_buffer_ids[3]),
                             dag_->getBuffer(rz_out), d_fused_size_);
            code_bytes = sizes[0] / sizeof(float) * sizeof(uint16_t);
        }
        static_cast<BitshuffleStage*>(bsn->stage)->markFused(code_bytes);
        static_cast<RZEStage*>(rzn->stage)->markFused(code_bytes, d_fused_size_, stream);
        for (int i = 1; i < 4; i++) {
            const size_t sz = n->stage->getExecuteTimeOutputSize(i);
            if (sz) dag_->buffer(n->output_buffer_ids[i]).size = sz;
        }
        if (profiling_enabled_) cudaEventRecord(n->end_event, stream);
        if (bounds_check_) {
            checkBounds(n);
            checkBounds(rzn);
        }
        return;
    }
    for (int id : n->output_buffer_ids) {
        dag_->allocate(id, stream);
        out.push_back(dag_->getBuffer(id));
    }
    n->stage->execute(stream, pool_.get(), in, out, sizes);
    if (profiling_enabled_) cudaEventRecord(n->end_event, stream);
    // sizes downstream stages see; sinks are read after the sync
    for (size_t k = 0; k < n->output_buffer_ids.size(); k++) {
        BufferInfo& b = dag_->buffer(n->output_buffer_ids[k]);
        if (b.consumer_stage_ids.empty()) continue;
        const size_t sz = n->stage->getExecuteTimeOutputSize((int)k);
        if (sz) b.size = sz;
    }
    if (bounds_check_) checkBounds(n);
}

// The bounds check of dag.cpp:438-462: each output's actual size (read back,
// which synchronises) against the bytes reserved for it.  Skipped while the
// stream is being captured into a graph.
void Pipeline::checkBounds(DAGNode* n) {
    if (capturing_) return;
    const auto names = n->stage->getOutputNames();
    for (size_t k = 0; k < n->output_buffer_ids.size(); k++) {
        const BufferInfo& b = dag_->getBufferInfo(n->output_buffer_ids[k]);
        if (b.allocated_size == 0) continue;
        const size_t sz = n->stage->getActualOutputSize((int)k);
        if (sz > b.allocated_size)
            throw std::runtime_error("Buffer overwrite detected: stage '" + n->name + "' output '" +
                                     (k < names.size() ? names[k] : std::to_string(k)) + "' wrote " +
                                     std::to_string(sz) + " bytes into a " + std::to_string(b.allocated_size) +
                                     "-byte buffer");
    }
}

void Pipeline::collectMetadata() {
    meta_.clear();
    for (size_t i = 0; i < output_buffer_ids_.size(); i++) {
        const int id = output_buffer_ids_[i];
        BufferInfo& b = dag_->buffer(id);
        DAGNode* p = output_nodes_[i];
        BufferMetadata m;
        m.buffer_id = id;
        m.producer = p;
        m.output_index = b.producer_output_index;
        const auto names = p->stage->getOutputNames();
        m.name = (m.output_index >= 0 && m.output_index < (int)names.size()) ? names[m.output_index] : "output";
        const size_t at_exec = p->stage->getExecuteTimeOutputSize(m.output_index);
        if (at_exec) b.size = at_exec;
        m.allocated_size = b.size;
        const auto by_name = p->stage->getActualOutputSizesByName();
        const auto it = by_name.find(m.name);
        m.actual_size = it != by_name.end() ? it->second : b.size;
        meta_.push_back(m);
    }
}

size_t Pipeline::concatSize() const {
    size_t total = pad16(4 + 8 * meta_.size());
    for (const auto& m : meta_) total += pad16(m.actual_size);
    return total;
}

void Pipeline::concatOutputs(void* d_out, size_t capacity, size_t* out_size, cudaStream_t stream) {
    std::vector<const void*> src;
    std::vector<uint64_t> sizes;
    for (const auto& m : meta_) {
        src.push_back(dag_->getBuffer(m.buffer_id));
        sizes.push_back(m.actual_size);
    }
    const size_t total = concatSize();
    if (total > capacity)
        throw std::runtime_error("compress(): output (" + std::to_string(total) + " bytes) exceeds the buffer capacity (" +
                                 std::to_string(capacity) + " bytes)");
    const int rc = fzb_concat(src.data(), sizes.data(), (int)src.size(), d_out, stream);
    if (rc) throw std::runtime_error(std::string("concat: ") + fzb_status_string(rc));
    *out_size = total;
}

bool Pipeline::enqueueResultReads(cudaStream_t stream) {
    reads_.clear();
    read_stages_.clear();
    for (auto& st : stages_) {
        auto* r = dynamic_cast<DeviceResults*>(st.get());
        if (!r) continue;
        const size_t before = reads_.size();
        r->pendingReads(reads_);
        if (reads_.size() > before) read_stages_.push_back(r);
    }
    if (gather_.enqueue(reads_, stream)) return true;
    reads_.clear();
    read_stages_.clear();
    return false;
}

void Pipeline::finishResultReads() {
    gather_.finish(reads_);
    for (auto* r : read_stages_) r->resultsFetched();
    reads_.clear();
    read_stages_.clear();
}

// Every output's bound (the bytes reserved for its buffer) and, where the
// size is still on the device, the word it follows; the container is laid out
// on the device and checked against the host's sizes after the wait.
bool Pipeline::enqueueDeviceConcat(cudaStream_t stream) {
    const size_t n = output_buffer_ids_.size();
    if (n < 2 || n > FZB_CONCAT_MAX_SEGMENTS) return false;
    const void* src[FZB_CONCAT_MAX_SEGMENTS];
    const void* word[FZB_CONCAT_MAX_SEGMENTS];
    uint64_t caps[FZB_CONCAT_MAX_SEGMENTS], scale[FZB_CONCAT_MAX_SEGMENTS], maxc[FZB_CONCAT_MAX_SEGMENTS];
    uint32_t wbytes[FZB_CONCAT_MAX_SEGMENTS];
    for (size_t i = 0; i < n; i++) {
        DAGNode* p = output_nodes_[i];
        const auto* r = dynamic_cast<const DeviceResults*>(p->stage);
        if (!r) return false;  // a stage of another library: its sizes are known after the wait only
        const BufferInfo& b = dag_->getBufferInfo(output_buffer_ids_[i]);
        const int idx = b.producer_output_index;
        src[i] = dag_->getBuffer(output_buffer_ids_[i]);
        DeviceSize ds;
        if (r->deviceOutputSize(idx, &ds)) {
            // the bytes reserved for the output (asking the stage would read
            // its size back, the wait this avoids)
            caps[i] = b.allocated_size ? b.allocated_size : b.size;
            word[i] = ds.word;
            wbytes[i] = ds.word_bytes;
            scale[i] = ds.scale;
            maxc[i] = ds.max_count;
        } else {
            caps[i] = p->stage->getActualOutputSize(idx);
            word[i] = nullptr;
            wbytes[i] = 0;
            scale[i] = 1;
            maxc[i] = 0;
        }
        dev_concat_caps_[i] = caps[i];
        dev_concat_fixed_[i] = word[i] == nullptr;
    }
    const size_t bound = fzb_concat_bytes(caps, (int)n);
    if (!bound) return false;
    if (bound > concat_bytes_) {
        if (concat_buf_) pool_->free(concat_buf_, stream);
        concat_bytes_ = 0;
        concat_buf_ = pool_->allocate(bound, stream, "concat_output", true);
        if (!concat_buf_) throw std::runtime_error("Failed to allocate concat output buffer");
        concat_bytes_ = bound;
    }
    return fzb_concat_dev(src, caps, word, wbytes, scale, maxc, (int)n, concat_buf_, stream) == FZB_OK;
}

void Pipeline::compress(const void* d_input, size_t input_size, void** d_output, size_t* output_size,
                        cudaStream_t stream) {
    if (!finalized_) throw std::runtime_error("Pipeline must be finalized before execution");
    if (!d_input) throw std::runtime_error("compress(): null device pointer passed as input");
    if (input_size_hint_ && input_size > input_size_hint_)
        throw std::runtime_error("compress(): input size (" + std::to_string(input_size) +
                                 " bytes) exceeds the finalize-time buffer size hint (" +
                                 std::to_string(input_size_hint_) + " bytes)");
    const auto t0 = std::chrono::steady_clock::now();
    size_t src_bytes = 0;
    const void* src = nullptr;
    if (graph_exec_) {
        cuda_check(cudaMemcpyAsync(graph_input_, d_input, input_size, cudaMemcpyDeviceToDevice, stream), "graph input");
        if (input_size < graph_input_bytes_)
            cuda_check(cudaMemsetAsync(static_cast<uint8_t*>(graph_input_) + input_size, 0,
                                       graph_input_bytes_ - input_size, stream),
                       "graph input");
        original_input_size_ = (input_alignment_ > 1 && input_size % input_alignment_) ? input_size : 0;
        src = graph_input_;
        src_bytes = graph_input_bytes_;
    } else {
        src = prepareInput(d_input, input_size, stream, &src_bytes);
    }
    BufferInfo& ib = dag_->buffer(input_buffer_id_);
    ib.d_ptr = const_cast<void*>(src);
    ib.size = src_bytes;
    input_size_ = src_bytes;
    if (!input_size_hint_) propagateBufferSizes(src_bytes);
    const auto t1 = std::chrono::steady_clock::now();
    if (graph_exec_) {
        cuda_check(cudaGraphLaunch(graph_exec_, stream), "graph launch");
        for (auto& s : stages_) s->onGraphReplay(stream);
    } else {
        runForward(stream);
    }
    const auto t2 = std::chrono::steady_clock::now();
    // one wait: the container and the stages' results are enqueued first
    concat_enqueued_ = enqueueDeviceConcat(stream);
    const bool gathered = enqueueResultReads(stream);
    cuda_check(cudaStreamSynchronize(stream), "compress");
    if (gathered) finishResultReads();
    for (auto& s : stages_) s->postStreamSync(stream);
    collectMetadata();
    if (profiling_enabled_) {
        last_perf_ = PipelinePerfResult();
        last_perf_.is_compress = true;
        for (const auto& lv : dag_->getLevels())
            for (auto* n : lv)
                if (n->start_event && n->end_event) {
                    float ms = 0.0f;
                    if (cudaEventElapsedTime(&ms, n->start_event, n->end_event) == cudaSuccess)
                        last_perf_.stages.push_back({n->name, n->level, ms});
                    else cudaGetLastError();
                }
    }
    if (concat_enqueued_) {
        // the device laid the container out from its own sizes: a segment
        // whose host size differs (a fixed size that changed, a device size
        // past its buffer) is concatenated again from the host sizes
        bool same = meta_.size() == output_buffer_ids_.size();
        for (size_t i = 0; same && i < meta_.size(); i++)
            same = dev_concat_fixed_[i] ? meta_[i].actual_size == dev_concat_caps_[i]
                                        : meta_[i].actual_size <= dev_concat_caps_[i];
        concat_enqueued_ = same;
    }
    if (concat_enqueued_) {
        *output_size = concatSize();
        *d_output = concat_buf_;
    } else if (meta_.size() > 1) {
        const size_t need = concatSize();
        if (need > concat_bytes_) {
            if (concat_buf_) pool_->free(concat_buf_, stream);
            concat_buf_ = pool_->allocate(need, stream, "concat_output", true);
            if (!concat_buf_) throw std::runtime_error("Failed to allocate concat output buffer");
            concat_bytes_ = need;
        }
        concatOutputs(concat_buf_, concat_bytes_, output_size, stream);
        *d_output = concat_buf_;
    } else {
        *d_output = dag_->getBuffer(meta_[0].buffer_id);
        *output_size = meta_[0].actual_size;
    }
    compressed_ = true;
    const auto t3 = std::chrono::steady_clock::now();
    last_perf_.is_compress = true;
    last_perf_.input_bytes = input_size_;
    last_perf_.output_bytes = *output_size;
    last_perf_.dag_elapsed_ms = std::chrono::duration<float, std::milli>(t2 - t1).count();
    last_perf_.host_elapsed_ms = std::chrono::duration<float, std::milli>(t3 - t0).count();
}

void Pipeline::compress(const void* d_input, size_t input_size, void* d_output_buf, size_t output_buf_capacity,
                        size_t* actual_output_size, cudaStream_t stream) {
    if (graph_mode_) throw std::runtime_error("compress() into a caller buffer is not available in graph mode");
    void* p = nullptr;
    size_t sz = 0;
    if (!d_output_buf) throw std::runtime_error("compress(): null output buffer");
    compress(d_input, input_size, &p, &sz, stream);
    if (sz > output_buf_capacity)
        throw std::runtime_error("compress(): output (" + std::to_string(sz) + " bytes) exceeds the buffer capacity (" +
                                 std::to_string(output_buf_capacity) + " bytes)");
    cuda_check(cudaMemcpyAsync(d_output_buf, p, sz, cudaMemcpyDeviceToDevice, stream), "compress copy-out");
    *actual_output_size = sz;
}

void Pipeline::reset(cudaStream_t stream) {
    if (!finalized_) return;
    if (strategy_ == MemoryStrategy::MINIMAL) {
        for (int i = 0; i < dag_->bufferCount(); i++)
            if (!dag_->getBufferInfo(i).is_persistent) dag_->release(i, stream);
    }
}

void Pipeline::warmup(cudaStream_t stream) {
    if (!finalized_) throw std::runtime_error("Pipeline must be finalized before warmup()");
    if (!input_size_hint_) return;
    void* d = nullptr;
    cuda_check(cudaMalloc(&d, input_size_hint_), "warmup");
    cudaMemsetAsync(d, 0, input_size_hint_, stream);
    void* out = nullptr;
    size_t sz = 0;
    try {
        compress(d, input_size_hint_, &out, &sz, stream);
        void* dec = nullptr;
        size_t dsz = 0;
        decompress(out, sz, &dec, &dsz, stream);
        cudaStreamSynchronize(stream);
        if (!pool_managed_decomp_) cudaFree(dec);
    } catch (...) {
        cudaFree(d);
        throw;
    }
    for (void* p : decomp_outputs_) pool_->free(p, stream);
    decomp_outputs_.clear();
    decomp_output_bytes_ = 0;
    meta_.clear();
    compressed_ = false;
    cudaStreamSynchronize(stream);
    cudaFree(d);
}

void Pipeline::captureGraph(cudaStream_t stream) {
    if (!finalized_) throw std::runtime_error("Pipeline must be finalized before captureGraph()");
    if (!graph_mode_) throw std::runtime_error("Call enableGraphMode(true) before finalize() to use captureGraph()");
    if (stream == 0) throw std::runtime_error("captureGraph() needs a non-default stream");
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    if (graph_) {
        cudaGraphDestroy(graph_);
        graph_ = nullptr;
    }
    BufferInfo& ib = dag_->buffer(input_buffer_id_);
    ib.d_ptr = graph_input_;
    ib.size = graph_input_bytes_;
    input_size_ = graph_input_bytes_;
    // stage workspaces are sized by a first eager run, so nothing allocates inside the capture
    runForward(stream);
    cuda_check(cudaStreamSynchronize(stream), "captureGraph warm pass");
    for (auto& s : stages_) s->postStreamSync(stream);
    const bool prof = profiling_enabled_;
    profiling_enabled_ = false;
    cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    capturing_ = true;
    try {
        runForward(stream);
    } catch (...) {
        capturing_ = false;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        profiling_enabled_ = prof;
        throw;
    }
    capturing_ = false;
    profiling_enabled_ = prof;
    cuda_check(cudaStreamEndCapture(stream, &graph_), "end capture");
    cuda_check(cudaGraphInstantiate(&graph_exec_, graph_, 0), "graph instantiate");
    captureDecompress(stream);
}

std::vector<Pipeline::OutputBuffer> Pipeline::getOutputBuffers() const {
    std::vector<OutputBuffer> v;
    for (const auto& m : meta_) v.push_back({dag_->getBuffer(m.buffer_id), m.actual_size, m.allocated_size, m.name, m.buffer_id});
    return v;
}

}  // namespace fz
