// fz/pipeline.h -- pipeline builder, DAG executor and FZM file I/O with the
// reference's user API (include/pipeline/compressor.h:34-386,
// include/pipeline/dag.h): addStage / connect / finalize / compress /
// decompress / writeToFile / readHeader / decompressFromFile.
//
// Buffer numbering, execution levels, per-buffer sizes and the container
// records follow the reference so files are interchangeable.  Pipeline
// outputs are ordered canonically (stage insertion order, then output
// index); the reference orders them by hash-map iteration, so its segment
// order can differ while every segment's bytes agree.
//
// A LorenzoQuant -> Bitshuffle(16 KiB, ew 2) -> RZE(16 KiB, 4 levels) chain,
// or the pfpl chain Quantizer(uint32 codes) -> Difference(int32 -> uint32,
// 16 KiB) -> Bitshuffle(16 KiB, ew 2) -> RZE(16 KiB, 4 levels), whose
// intermediate buffers feed nothing else runs as one fused kernel pass in
// each direction (the intermediates are never materialised);
// setFusion(false) runs the stages one by one.  Both produce identical bytes.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <memory>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "fz/fzm_format.h"
#include "fz/mempool.h"
#include "fz/stage.h"
#include "fz/stages.h"

namespace fz {

// Mapped pinned host block that small device results (sizes, counts, error
// bounds, status words) are copied into by one kernel enqueued before a
// stream wait (fzb_gather_words), instead of one blocking copy per value.
class ResultGather {
public:
    ResultGather() = default;
    ~ResultGather();
    ResultGather(const ResultGather&) = delete;
    ResultGather& operator=(const ResultGather&) = delete;
    // False when nothing was enqueued (more reads than one launch takes, no
    // mapped memory); the caller then reads the values itself.
    bool enqueue(const std::vector<DeviceRead>& reads, cudaStream_t stream);
    // After the wait: copies each value to its dst.
    void finish(const std::vector<DeviceRead>& reads) const;

private:
    static constexpr size_t kBytes = 4096;
    void* host_ = nullptr;
    void* dev_ = nullptr;
};

enum class MemoryStrategy {
    MINIMAL,      // allocate at first use, free after the last consumer
    PREALLOCATE,  // one arena sized at finalize(); buffers with disjoint lifetimes share it
};

struct BufferInfo {
    size_t size = 0;            // current byte size (estimate, then actual)
    size_t estimate = 0;        // size from the finalize/compress-time propagation
    size_t allocated_size = 0;  // bytes reserved
    void* d_ptr = nullptr;
    std::string tag;
    std::vector<int> consumer_stage_ids;
    int producer_stage_id = -1;
    int producer_output_index = 0;
    bool is_persistent = false;  // pipeline outputs and inputs
    bool is_external = false;    // caller-owned pointer
    int first_level = 0, last_level = 0;  // lifetime, for arena sharing
    size_t arena_offset = 0;
};

struct DAGNode {
    int id = -1;
    Stage* stage = nullptr;
    std::string name;
    std::vector<int> input_buffer_ids;
    std::vector<int> output_buffer_ids;
    std::unordered_map<int, int> output_index_to_buffer_id;
    std::vector<DAGNode*> dependencies;
    std::vector<DAGNode*> dependents;
    int level = -1;
    cudaEvent_t start_event = nullptr, end_event = nullptr;  // profiling
};

struct StageTimingResult {
    std::string name;
    int level = 0;
    float elapsed_ms = 0.0f;
};

struct PipelinePerfResult {
    bool is_compress = true;
    float host_elapsed_ms = 0.0f;
    float dag_elapsed_ms = 0.0f;
    size_t input_bytes = 0;
    size_t output_bytes = 0;
    std::vector<StageTimingResult> stages;
    // uncompressed bytes per second over the summed stage time
    float throughput_gbs() const;
};

class CompressionDAG {
public:
    CompressionDAG(MemoryPool* pool, MemoryStrategy strategy);
    ~CompressionDAG();
    DAGNode* addStage(Stage* stage, const std::string& name);
    int addUnconnectedOutput(DAGNode* node, int output_index, const std::string& tag);
    bool connectExistingOutput(DAGNode* producer, DAGNode* consumer, int output_index);
    int setInputBuffer(DAGNode* node, const std::string& tag);
    void finalize();  // cycle check + levels
    const std::vector<std::vector<DAGNode*>>& getLevels() const { return levels_; }
    const std::vector<DAGNode*>& getNodes() const { return nodes_; }
    BufferInfo& buffer(int id) { return buffers_.at(id); }
    const BufferInfo& getBufferInfo(int id) const { return buffers_.at(id); }
    void* getBuffer(int id) const { return buffers_.at(id).d_ptr; }
    size_t getBufferSize(int id) const { return buffers_.at(id).size; }
    int bufferCount() const { return (int)buffers_.size(); }
    // Reserve every internal buffer (PREALLOCATE: one arena; buffers whose
    // level ranges do not overlap share bytes).
    void preallocate(cudaStream_t stream);
    void allocate(int id, cudaStream_t stream);
    void release(int id, cudaStream_t stream);
    void releaseAll(cudaStream_t stream);
    MemoryStrategy strategy() const { return strategy_; }
    size_t arenaBytes() const { return arena_bytes_; }
    size_t getColorRegionCount() const { return regions_; }

private:
    MemoryPool* pool_;
    MemoryStrategy strategy_;
    std::vector<DAGNode*> nodes_;
    std::vector<std::vector<DAGNode*>> levels_;
    std::unordered_map<int, BufferInfo> buffers_;
    int next_buffer_id_ = 0;
    void* arena_ = nullptr;
    size_t arena_bytes_ = 0;
    size_t regions_ = 0;
};

class Pipeline {
public:
    explicit Pipeline(size_t input_data_size = 0, MemoryStrategy strategy = MemoryStrategy::MINIMAL,
                      float pool_multiplier = 3.0f);
    ~Pipeline();
    Pipeline(const Pipeline&) = delete;
    Pipeline& operator=(const Pipeline&) = delete;

    void setMemoryStrategy(MemoryStrategy strategy);
    // Streams for sibling stages (include/pipeline/compressor.h:64).  At
    // finalize() the pipeline keeps max(n, widest DAG level) side streams
    // when that is above 1; a level with several stages forks from the
    // caller's stream onto them (round-robin within the level, as
    // dag.cpp:752-762) and joins back before the next level.  Levels of one
    // stage, and every linear chain, run on the caller's stream.
    void setNumStreams(int num_streams);
    int getNumStreams() const { return num_streams_; }
    // After each stage, read its actual output sizes (this synchronises) and
    // throw when one exceeds the bytes reserved for it (dag.cpp:438-462).
    void enableBoundsCheck(bool enable) { bounds_check_ = enable; }
    bool isBoundsCheckEnabled() const { return bounds_check_; }
    float getPoolMultiplier() const { return pool_multiplier_; }
    void setDims(size_t x, size_t y = 1, size_t z = 1) { dims_ = {x, y, z}; }
    void setDims(std::array<size_t, 3> dims) { dims_ = dims; }
    std::array<size_t, 3> getDims() const { return dims_; }

    template <typename StageT, typename... Args>
    StageT* addStage(Args&&... args) {
        auto* s = new StageT(std::forward<Args>(args)...);
        if (dims_[0] > 0) s->setDims(dims_);
        addRawStage(s);
        return s;
    }
    // TOML configurations (src/pipeline/config.cpp): loadConfig adds, connects
    // and finalizes the stages a file describes; saveConfig writes a
    // finalized pipeline in the same format.
    void loadConfig(const std::string& path);
    void saveConfig(const std::string& path) const;
    int connect(Stage* dependent, Stage* producer, const std::string& output_name = "output");
    int connect(Stage* dependent, const std::vector<Stage*>& producers);
    void finalize();
    void warmup(cudaStream_t stream = 0);
    void setWarmupOnFinalize(bool enable) { warmup_on_finalize_ = enable; }
    void setPoolManagedDecompOutput(bool enable) { pool_managed_decomp_ = enable; }
    bool isPoolManagedDecompOutput() const { return pool_managed_decomp_; }
    void setFusion(bool enable) { fusion_enabled_ = enable; }
    bool isFused() const { return fused_; }
    size_t getMaxCompressedSize(size_t input_bytes) const;
    size_t getLastUncompressedSize() const { return original_input_size_ ? original_input_size_ : input_size_; }

    // Pool-owned output, valid until the next compress()/reset().
    void compress(const void* d_input, size_t input_size, void** d_output, size_t* output_size,
                  cudaStream_t stream = 0);
    // Caller-owned output buffer.
    void compress(const void* d_input, size_t input_size, void* d_output_buf, size_t output_buf_capacity,
                  size_t* actual_output_size, cudaStream_t stream = 0);
    // d_input = nullptr decompresses the pipeline's own last outputs.
    void decompress(const void* d_input, size_t input_size, void** d_output, size_t* output_size,
                    cudaStream_t stream = 0);
    void decompress(const void* d_input, size_t input_size, void* d_output_buf, size_t output_buf_capacity,
                    size_t* actual_output_size, cudaStream_t stream = 0);
    void reset(cudaStream_t stream = 0);

    void enableProfiling(bool enable) { profiling_enabled_ = enable; }
    bool isProfilingEnabled() const { return profiling_enabled_; }
    const PipelinePerfResult& getLastPerfResult() const { return last_perf_; }
    CompressionDAG* getDAG() { return dag_.get(); }
    MemoryPool* getMemoryPool() { return pool_.get(); }
    size_t getPeakMemoryUsage() const { return pool_ ? pool_->getPeakUsage() : 0; }
    size_t getCurrentMemoryUsage() const { return pool_ ? pool_->getCurrentUsage() : 0; }
    size_t getColorRegionCount() const { return dag_->getColorRegionCount(); }

    // CUDA Graph replay of the compress DAG (PREALLOCATE, graph-compatible
    // stages, a non-default stream).
    void enableGraphMode(bool enable);
    bool isGraphModeEnabled() const { return graph_mode_; }
    // Captures the compress DAG and, where every stage's inverse runs from
    // device-resident sizes (LorenzoQuant, Bitshuffle, RZE, RLE, Bitpack,
    // Huffman; two or more pipeline outputs), the decompression too.  A
    // graph-mode decompress() then copies the container into a fixed slot
    // and replays the graph: the container is split on the device (the
    // segment sizes are read from its header there), the error bound comes
    // from the compressor's device state, and nothing waits on the host.
    // The reference's graph mode covers compression only
    // (include/pipeline/compressor.h:321-341).
    void captureGraph(cudaStream_t stream);
    bool isGraphCaptured() const { return graph_exec_ != nullptr; }
    bool isDecompressGraphCaptured() const { return decomp_exec_ != nullptr; }
    // Waits for the last decompress() and throws if the device found its
    // input malformed (graph-mode decompressions report it only here).
    void checkDecompressStatus(cudaStream_t stream = 0);

    struct FZMFileHeader {
        FZMHeaderCore core;
        std::vector<FZMStageInfo> stages;
        std::vector<FZMBufferEntry> buffers;
    };
    FZMFileHeader buildHeader() const;
    void writeToFile(const std::string& filename, cudaStream_t stream = 0);
    static FZMFileHeader readHeader(const std::string& filename);
    // Rebuilds the stages from the file and decompresses it; *d_output is a
    // cudaMalloc'd buffer the caller frees.
    static void decompressFromFile(const std::string& filename, void** d_output, size_t* output_size,
                                   cudaStream_t stream = 0, PipelinePerfResult* perf_out = nullptr,
                                   size_t pool_override_bytes = 0);

    struct OutputBuffer {
        void* d_ptr;
        size_t actual_size;
        size_t allocated_size;
        std::string name;
        int buffer_id;
    };
    std::vector<OutputBuffer> getOutputBuffers() const;

private:
    struct BufferMetadata {
        int buffer_id;
        size_t actual_size;
        size_t allocated_size;
        DAGNode* producer;
        int output_index;
        std::string name;
    };
    Stage* addRawStage(Stage* stage);
    void propagateBufferSizes(size_t source_bytes);
    void detectFusion();
    void runForward(cudaStream_t stream);
    void runNode(DAGNode* n, cudaStream_t stream);
    void checkBounds(DAGNode* n);
    const void* prepareInput(const void* d_input, size_t input_size, cudaStream_t stream, size_t* padded);
    void collectMetadata();
    void concatOutputs(void* d_out, size_t capacity, size_t* out_size, cudaStream_t stream);
    size_t concatSize() const;
    // Concatenation enqueued before the wait, with the sizes the device
    // holds; false (nothing enqueued) when a stage's sizes are host-only.
    bool enqueueDeviceConcat(cudaStream_t stream);
    // The stages' pending device results, gathered into the mapped block by
    // one kernel before the wait (false: nothing gathered, the stages read
    // their own); distributed after it.
    bool enqueueResultReads(cudaStream_t stream);
    void finishResultReads();
    // Inverse over the forward topology: fwd buffer id -> (pointer, bytes).
    // Returns the reconstructed source buffer (pool- or caller-owned).
    void runInverse(const std::unordered_map<int, std::pair<void*, size_t>>& outputs, void* d_result,
                    size_t result_capacity, size_t* result_size, cudaStream_t stream);

    std::unique_ptr<MemoryPool> pool_;
    std::unique_ptr<CompressionDAG> dag_;
    MemoryStrategy strategy_;
    std::vector<std::unique_ptr<Stage>> stages_;
    std::vector<DAGNode*> stage_nodes_;  // insertion order
    struct Conn {
        Stage* dependent;
        Stage* producer;
        std::string output_name;
        int output_index;
    };
    std::vector<Conn> connections_;
    std::array<size_t, 3> dims_ = {0, 1, 1};
    bool finalized_ = false, compressed_ = false, warmup_on_finalize_ = false;
    bool pool_managed_decomp_ = true, profiling_enabled_ = false;
    bool fusion_enabled_ = true, fused_ = false;
    bool fused_pfpl_ = false;  // the fused chain starts at a Quantizer (pfpl) rather than LorenzoQuant
    bool graph_mode_ = false;
    bool bounds_check_ = false, capturing_ = false;
    float pool_multiplier_ = 3.0f;
    int num_streams_ = 1;
    std::vector<cudaStream_t> side_streams_;
    std::vector<cudaEvent_t> fork_events_;   // one per DAG level
    std::vector<cudaEvent_t> join_events_;   // one per stage
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    // captured decompression: container slot, reconstruction slot, split
    // status word + fused-inverse workspace, stage-by-stage intermediates
    cudaGraph_t decomp_graph_ = nullptr;
    cudaGraphExec_t decomp_exec_ = nullptr;
    void* decomp_in_ = nullptr;
    size_t decomp_in_bytes_ = 0;
    void* decomp_out_ = nullptr;
    void* decomp_work_ = nullptr;
    size_t decomp_work_bytes_ = 0;
    bool decomp_fused_ = false;
    std::vector<void*> decomp_temps_;
    bool captureDecompress(cudaStream_t stream);
    void enqueueGraphInverse(cudaStream_t stream);
    void releaseDecompressGraph();
    void* graph_input_ = nullptr;
    size_t graph_input_bytes_ = 0;
    DAGNode* input_node_ = nullptr;
    int input_buffer_id_ = -1;
    std::vector<int> output_buffer_ids_;
    std::vector<DAGNode*> output_nodes_;
    std::vector<BufferMetadata> meta_;
    size_t input_size_hint_, input_alignment_ = 1, input_size_ = 0, original_input_size_ = 0;
    void* pad_buf_ = nullptr;
    size_t pad_bytes_ = 0;
    void* concat_buf_ = nullptr;
    size_t concat_bytes_ = 0;
    std::vector<void*> decomp_outputs_;
    size_t decomp_output_bytes_ = 0;  // capacity of decomp_outputs_[0]
    uint64_t* d_fused_size_ = nullptr;  // device u64 for the fused path's stream size
    ResultGather gather_;
    std::vector<DeviceRead> reads_;
    std::vector<DeviceResults*> read_stages_;
    bool concat_enqueued_ = false;
    uint64_t dev_concat_caps_[FZM_MAX_BUFFERS] = {};
    bool dev_concat_fixed_[FZM_MAX_BUFFERS] = {};
    // the fused inverse's workspace, kept between decompress calls
    void* inv_work_ = nullptr;
    size_t inv_work_bytes_ = 0;
    PipelinePerfResult last_perf_;
};

}  // namespace fz
