// fz/stages.h -- the hot-path stages behind the fz::Stage interface, with
// the reference's class names, setters, output names and container headers
// (modules/fused/lorenzo_quant/lorenzo_quant.h, shufflers/bitshuffle/
// bitshuffle_stage.h, coders/rze/rze_stage.h, coders/rle/rle.h,
// coders/huffman/huffman_stage.h, coders/bitpack/bitpack_stage.h,
// quantizers/quantizer/quantizer.h, predictors/diff/diff.h,
// predictors/lorenzo/lorenzo_stage.h, transforms/zigzag/zigzag_stage.h,
// transforms/negabinary/negabinary_stage.h).  Every
// stage runs the sm_100a kernels of libfzb through the C ABI in fzb.h; errors
// are thrown as std::runtime_error, as the reference does.
#pragma once

#include <array>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "fz/mempool.h"
#include "fz/stage.h"

namespace fz {

// A small device result that a stage reads on the host after a
// synchronisation: a stream size, an outlier count, the resolved error
// bound, a status word.
struct DeviceRead {
    const void* src = nullptr;  // device address, 4-byte aligned
    uint32_t bytes = 0;         // a multiple of 4, at most 256
    void* dst = nullptr;        // host destination, filled after the wait
    bool clear = false;         // zero the device word once read (status words)
};

// Where an output's size lives on the device before the wait:
// min(*word, max_count) * scale bytes (word a u32 or u64).
struct DeviceSize {
    const void* word = nullptr;
    uint32_t word_bytes = 4;
    uint64_t scale = 1;
    uint64_t max_count = ~0ull;
};

// Implemented by this library's stages.  A pipeline collects the pending
// reads of every stage, copies them into one mapped host block with one
// kernel enqueued before its single stream wait (fzb_gather_words), fills
// each dst and calls resultsFetched(); postStreamSync then uses the copies
// instead of issuing its own blocking copies.  Run alone, a stage reads
// them itself.  A pipeline whose stages all implement this also enqueues
// its output concatenation before the wait (fzb_concat_dev), taking the
// sizes the device holds from deviceOutputSize().
class DeviceResults {
public:
    virtual ~DeviceResults() = default;
    virtual void pendingReads(std::vector<DeviceRead>& out) { (void)out; }
    virtual void resultsFetched() {}
    // False when getActualOutputSize(index) is already exact on the host.
    virtual bool deviceOutputSize(int index, DeviceSize* ds) const {
        (void)index;
        (void)ds;
        return false;
    }
};

// Device workspace owned by a stage, drawn from the pipeline's pool (or
// cudaMalloc when the stage runs without a pool) and grown on demand.
class StageWorkspace {
public:
    StageWorkspace() = default;
    ~StageWorkspace();
    StageWorkspace(const StageWorkspace&) = delete;
    StageWorkspace& operator=(const StageWorkspace&) = delete;
    void* ensure(size_t bytes, MemoryPool* pool, cudaStream_t stream);
    size_t size() const { return bytes_; }
    void* get() const { return ptr_; }
    // Throws when a kernel latched an error (malformed input, a bounded
    // wait that gave up) in this workspace; clears it.  Uses the status
    // word a pipeline fetched (pendingStatus) when there is one.
    void checkStatus(cudaStream_t stream, const char* what) const;
    // Adds the status word to a pipeline's gathered reads.
    void pendingStatus(std::vector<DeviceRead>& out) const;
    void statusFetched() const { fetched_ = ptr_ != nullptr; }

private:
    void release();
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
    MemoryPool* pool_ = nullptr;
    mutable uint32_t h_bits_ = 0;
    mutable bool fetched_ = false;
};

// ---------------------------------------------------------------------------
// LorenzoQuant (1/2/3-D predict + quantize), float -> uint16 codes + outliers.
// ---------------------------------------------------------------------------
enum class ErrorBoundMode : uint8_t { ABS = 0, REL = 1, NOA = 2 };

// 44-byte container record (lorenzo_quant.h:43-67).
struct LorenzoQuantConfig {
    float error_bound;       // absolute bound used by the decompressor
    uint32_t quant_radius;
    uint32_t num_elements;
    uint32_t outlier_count;  // stored outliers
    DataType input_type;
    DataType code_type;
    uint8_t ndim;
    uint8_t eb_mode;
    uint32_t dim_x;
    uint32_t dim_y;
    uint32_t dim_z;
    float user_eb;
    float value_base;
    uint8_t zigzag_codes;
    uint8_t reserved[3];
    LorenzoQuantConfig()
        : error_bound(0.0f), quant_radius(0), num_elements(0), outlier_count(0),
          input_type(DataType::FLOAT32), code_type(DataType::UINT16), ndim(1), eb_mode(0), dim_x(0),
          dim_y(1), dim_z(1), user_eb(0.0f), value_base(0.0f), zigzag_codes(0), reserved{0, 0, 0} {}
};
static_assert(sizeof(LorenzoQuantConfig) == 44, "LorenzoQuantConfig is 44 bytes");

template <typename TInput = float, typename TCode = uint16_t>
class LorenzoQuantStage : public Stage, public DeviceResults {
    static_assert(std::is_same<TInput, float>::value && std::is_same<TCode, uint16_t>::value,
                  "the sm_100a kernels implement LorenzoQuantStage<float, uint16_t>");

public:
    struct Config {
        float error_bound = 1e-3f;
        int quant_radius = 32768;
        float outlier_capacity = 0.2f;
        std::array<size_t, 3> dims = {0, 1, 1};  // {x, y, z}, x fastest; x = 0 infers x
        ErrorBoundMode eb_mode = ErrorBoundMode::ABS;
        float precomputed_value_base = 0.0f;  // > 0 skips the REL/NOA scan
        bool zigzag_codes = false;
        Config() = default;
        Config(TInput eb, TCode radius = 32768, float outlier_cap = 0.2f, std::array<size_t, 3> d = {0, 1, 1})
            : error_bound(eb), quant_radius(radius), outlier_capacity(outlier_cap), dims(d) {}
    };

    explicit LorenzoQuantStage(const Config& config = Config());

    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    void postStreamSync(cudaStream_t stream) override;
    void onGraphReplay(cudaStream_t) override { pending_ = !is_inverse_ && d_count_ != nullptr; }
    void pendingReads(std::vector<DeviceRead>& out) override;
    void resultsFetched() override;
    bool deviceOutputSize(int index, DeviceSize* ds) const override;

    std::string getName() const override { return "LorenzoQuant"; }
    size_t getNumInputs() const override { return is_inverse_ ? 4 : 1; }
    size_t getNumOutputs() const override { return is_inverse_ ? 1 : 4; }
    std::vector<std::string> getOutputNames() const override {
        return {"codes", "outlier_errors", "outlier_indices", "outlier_count"};
    }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& input_sizes) const override;
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override;
    size_t getActualOutputSize(int index) const override {
        return (index >= 0 && index < (int)actual_.size()) ? actual_[index] : 0;
    }
    size_t getExecuteTimeOutputSize(int index) const override {
        if (is_inverse_) return getActualOutputSize(index);
        return (index >= 0 && index < (int)at_execute_.size()) ? at_execute_[index] : 0;
    }
    void saveState() override { saved_ = actual_; }
    void restoreState() override { actual_ = saved_; }

    void setErrorBound(TInput eb) { config_.error_bound = eb; }
    void setQuantRadius(TCode radius) { config_.quant_radius = radius; }
    void setOutlierCapacity(float capacity) { config_.outlier_capacity = capacity; }
    void setDims(const std::array<size_t, 3>& dims) override { config_.dims = dims; }
    void setDims(size_t x, size_t y = 1, size_t z = 1) { config_.dims = {x, y, z}; }
    void setErrorBoundMode(ErrorBoundMode mode) { config_.eb_mode = mode; }
    void setValueBase(float value_base) { config_.precomputed_value_base = value_base; }
    void setZigzagCodes(bool enable) { config_.zigzag_codes = enable; }
    TInput getErrorBound() const { return config_.error_bound; }
    TCode getQuantRadius() const { return (TCode)config_.quant_radius; }
    float getOutlierCapacity() const { return config_.outlier_capacity; }
    std::array<size_t, 3> getDims() const { return config_.dims; }
    ErrorBoundMode getErrorBoundMode() const { return config_.eb_mode; }
    float getValueBase() const { return config_.precomputed_value_base; }
    bool getZigzagCodes() const { return config_.zigzag_codes; }
    int ndim() const { return config_.dims[2] > 1 ? 3 : (config_.dims[1] > 1 ? 2 : 1); }
    void setInverse(bool inverse) override { is_inverse_ = inverse; }
    bool isInverse() const override { return is_inverse_; }

    uint16_t getStageTypeId() const override { return (uint16_t)StageType::LORENZO_QUANT; }
    uint8_t getOutputDataType(size_t i) const override;
    uint8_t getInputDataType(size_t) const override { return (uint8_t)DataType::FLOAT32; }
    size_t serializeHeader(size_t output_index, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return sizeof(LorenzoQuantConfig); }

    // ceil(n * outlier_capacity) in single precision, as the reference
    // computes it (lorenzo_quant.h:333-335).
    size_t getMaxOutlierCount(size_t num_elements) const;
    float computedAbsErrorBound() const { return computed_abs_eb_; }
    float computedValueBase() const { return computed_value_base_; }
    // A captured decompression reads the error bound the compressor left on
    // the device (the second float of deviceEbState()) instead of the host
    // copy, which a graph-replayed compression does not refresh.
    void setInverseDeviceErrorBound(bool on) { inv_dev_eb_ = on; }
    const float* deviceEbState() const { return d_eb_state_; }

    // The fused LorenzoQuant -> Bitshuffle -> RZE path runs this stage's
    // forward kernel itself; it reports back what execute() would record.
    void fusedForward(cudaStream_t stream, MemoryPool* pool, const void* d_in, size_t in_bytes,
                      void* d_err, void* d_idx, void* d_count, void* d_rze, uint64_t* d_rze_size);

private:
    void* forwardWorkspace(size_t n, size_t cap, MemoryPool* pool, cudaStream_t stream);
    Config config_;
    bool is_inverse_ = false;
    std::vector<size_t> actual_, saved_, at_execute_;
    size_t num_elements_ = 0;
    uint32_t actual_outlier_count_ = 0;
    float computed_abs_eb_ = 0.0f;
    float computed_value_base_ = 0.0f;
    const void* d_count_ = nullptr;  // pending read-back (forward)
    float* d_eb_state_ = nullptr;    // inside the workspace
    bool pending_ = false;
    bool fetched_ = false;  // h_count_ / h_state_ hold the pending values
    uint32_t h_count_ = 0;
    float h_state_[4] = {0, 0, 0, 0};
    bool inv_dev_eb_ = false;
    StageWorkspace ws_;
    StageWorkspace inv_ws_;  // the inverse's own, so the forward eb state survives it
};

// ---------------------------------------------------------------------------
// Bitshuffle (bit-plane transpose per block), size-preserving.
// ---------------------------------------------------------------------------
class BitshuffleStage : public Stage, public DeviceResults {
public:
    BitshuffleStage() = default;
    void setInverse(bool inv) override { is_inverse_ = inv; }
    bool isInverse() const override { return is_inverse_; }
    void setBlockSize(size_t bytes) { block_size_ = (uint32_t)bytes; }
    void setElementWidth(size_t bytes) { element_width_ = (uint8_t)bytes; }
    size_t getBlockSize() const { return block_size_; }
    size_t getElementWidth() const { return element_width_; }
    size_t getRequiredInputAlignment() const override { return block_size_; }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    std::string getName() const override { return "Bitshuffle"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override { return {s[0]}; }
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override { return index == 0 ? actual_ : 0; }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::BITSHUFFLE; }
    uint8_t getOutputDataType(size_t) const override { return (uint8_t)DataType::UINT8; }
    // bitshuffle_stage.h:98-106: [u32 block_size][u8 element_width]
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return 5; }
    void saveState() override { saved_ = {block_size_, element_width_, actual_}; }
    void restoreState() override {
        block_size_ = saved_.block;
        element_width_ = saved_.ew;
        actual_ = saved_.actual;
    }
    void markFused(size_t bytes) { actual_ = bytes; }

private:
    struct Saved {
        uint32_t block = 0;
        uint8_t ew = 0;
        size_t actual = 0;
    };
    bool is_inverse_ = false;
    uint32_t block_size_ = 16384;
    uint8_t element_width_ = 4;  // the reference's default; the path uses 2
    size_t actual_ = 0;
    Saved saved_;
};

// ---------------------------------------------------------------------------
// RZE (recursive zero-byte elimination over 16 KiB chunks, 4 levels).
// ---------------------------------------------------------------------------
class RZEStage : public Stage, public DeviceResults {
public:
    RZEStage() = default;
    void setInverse(bool inv) override { is_inverse_ = inv; }
    bool isInverse() const override { return is_inverse_; }
    bool isGraphCompatible() const override { return !is_inverse_; }
    void setChunkSize(size_t bytes) { chunk_size_ = (uint32_t)bytes; }
    void setLevels(int n) { levels_ = (uint8_t)n; }
    size_t getChunkSize() const { return chunk_size_; }
    int getLevels() const { return levels_; }
    uint32_t getCachedOrigBytes() const { return cached_orig_bytes_; }
    size_t getRequiredInputAlignment() const override { return chunk_size_; }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    void postStreamSync(cudaStream_t stream) override;
    void onGraphReplay(cudaStream_t stream) override {
        if (is_inverse_ || !last_size_) return;
        d_size_ = last_size_;
        pending_stream_ = stream;
    }
    void pendingReads(std::vector<DeviceRead>& out) override {
        if (is_inverse_) ws_.pendingStatus(out);
        else if (d_size_) out.push_back({d_size_, 8, &h_size_, false});
    }
    void resultsFetched() override {
        if (is_inverse_) ws_.statusFetched();
        else fetched_ = d_size_ != nullptr;
    }
    bool deviceOutputSize(int index, DeviceSize* ds) const override {
        if (is_inverse_ || !d_size_ || index != 0) return false;
        *ds = {d_size_, 8, 1, ~0ull};
        return true;
    }
    std::string getName() const override { return "RZE"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override;
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        readBack();
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override {
        readBack();
        return index == 0 ? actual_ : 0;
    }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::RZE; }
    uint8_t getOutputDataType(size_t) const override { return (uint8_t)DataType::UINT8; }
    // rze_stage.h:175-184: [u32 chunk_size][u8 levels][u32 original bytes]
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return 9; }
    size_t estimateScratchBytes(const std::vector<size_t>& s) const override;
    void saveState() override { saved_ = {chunk_size_, levels_, cached_orig_bytes_}; }
    void restoreState() override {
        chunk_size_ = saved_.chunk;
        levels_ = saved_.levels;
        cached_orig_bytes_ = saved_.orig;
    }
    // Result of the fused path: the stream size lands in *d_size.
    void markFused(size_t in_bytes, const uint64_t* d_size, cudaStream_t stream);

private:
    void readBack() const;
    struct Saved {
        uint32_t chunk = 0;
        uint8_t levels = 0;
        uint32_t orig = 0;
    };
    bool is_inverse_ = false;
    uint32_t chunk_size_ = 16384;
    uint8_t levels_ = 4;
    uint32_t cached_orig_bytes_ = 0;
    mutable size_t actual_ = 0;
    mutable const uint64_t* d_size_ = nullptr;  // pending read-back
    const uint64_t* last_size_ = nullptr;       // where the last forward run writes its size
    mutable cudaStream_t pending_stream_ = nullptr;
    mutable bool fetched_ = false;  // h_size_ holds *d_size_
    uint64_t h_size_ = 0;
    Saved saved_;
    StageWorkspace ws_;
    uint64_t* d_size_own_ = nullptr;  // inside ws_
};

// ---------------------------------------------------------------------------
// RLE: [u32 runs][values, padded to 4 B][u32 lengths].
// ---------------------------------------------------------------------------
template <typename T>
class RLEStage : public Stage, public DeviceResults {
    static_assert(std::is_same<T, uint8_t>::value || std::is_same<T, uint16_t>::value ||
                      std::is_same<T, uint32_t>::value || std::is_same<T, int32_t>::value,
                  "RLEStage element types: uint8_t, uint16_t, uint32_t, int32_t");

public:
    RLEStage() = default;
    void setInverse(bool inv) override { is_inverse_ = inv; }
    bool isInverse() const override { return is_inverse_; }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    void postStreamSync(cudaStream_t stream) override;
    void onGraphReplay(cudaStream_t stream) override {
        if (is_inverse_ || !last_size_) return;
        d_size_ = last_size_;
        pending_stream_ = stream;
    }
    void pendingReads(std::vector<DeviceRead>& out) override {
        if (is_inverse_) ws_.pendingStatus(out);
        else if (d_size_) out.push_back({d_size_, 8, &h_size_, false});
    }
    void resultsFetched() override {
        if (is_inverse_) ws_.statusFetched();
        else fetched_ = d_size_ != nullptr;
    }
    bool deviceOutputSize(int index, DeviceSize* ds) const override {
        if (is_inverse_ || !d_size_ || index != 0) return false;
        *ds = {d_size_, 8, 1, ~0ull};
        return true;
    }
    std::string getName() const override { return "RLE"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override;
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        readBack();
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override {
        readBack();
        return index == 0 ? actual_ : 0;
    }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::RLE; }
    uint8_t getOutputDataType(size_t) const override { return (uint8_t)dtype(); }
    uint8_t getInputDataType(size_t) const override { return (uint8_t)dtype(); }
    // rle.h:123-131: [u8 data type][u32 element count]
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return 5; }
    size_t estimateScratchBytes(const std::vector<size_t>& s) const override {
        if (is_inverse_ || s.empty()) return 0;
        return (s[0] / sizeof(T)) * (1 + 4 + 4 + sizeof(T) + 4);
    }
    static DataType dtype();

private:
    void readBack() const;
    bool is_inverse_ = false;
    uint32_t cached_num_elements_ = 0;
    mutable size_t actual_ = 0;
    mutable const uint64_t* d_size_ = nullptr;
    const uint64_t* last_size_ = nullptr;
    mutable cudaStream_t pending_stream_ = nullptr;
    mutable bool fetched_ = false;  // h_size_ holds *d_size_
    uint64_t h_size_ = 0;
    StageWorkspace ws_;
};

// ---------------------------------------------------------------------------
// PHF Huffman (coarse or fine mode) over 16-bit symbols.
// ---------------------------------------------------------------------------
enum class HuffmanEncodeMode { Coarse, Fine };

template <typename T>
class HuffmanStage : public Stage, public DeviceResults {
    static_assert(std::is_same<T, uint16_t>::value, "the sm_100a Huffman coder implements uint16_t symbols");

public:
    HuffmanStage() = default;
    void setBklen(uint32_t bklen) { bklen_ = bklen; }
    uint32_t getBklen() const { return bklen_; }
    // Fine mode (huffman_stage.cu:41, hf_buf.cc:46-49): partitions of 1024
    // symbols instead of 768; the decoder reads the length from the blob.
    void setEncodeMode(HuffmanEncodeMode mode) { encode_mode_ = mode; }
    HuffmanEncodeMode getEncodeMode() const { return encode_mode_; }
    void setInverse(bool inv) override { is_inverse_ = inv; }
    bool isInverse() const override { return is_inverse_; }
    bool isGraphCompatible() const override { return false; }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    void postStreamSync(cudaStream_t stream) override {
        if (is_inverse_) ws_.checkStatus(stream, "HuffmanStage (inverse)");
    }
    void pendingReads(std::vector<DeviceRead>& out) override {
        if (is_inverse_) ws_.pendingStatus(out);
    }
    void resultsFetched() override {
        if (is_inverse_) ws_.statusFetched();
    }
    std::string getName() const override { return "Huffman"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override {
        if (s.empty()) return {0};
        return {is_inverse_ ? original_len_ * sizeof(T) : s[0] * 2 + 4096};
    }
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override { return index == 0 ? actual_ : 0; }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::HUFFMAN; }
    uint8_t getOutputDataType(size_t) const override { return (uint8_t)DataType::UNKNOWN; }
    uint8_t getInputDataType(size_t) const override { return (uint8_t)DataType::UNKNOWN; }
    // huffman_stage.h:174-183: [u8 data type][u16 bklen][u64 element count]
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return 11; }
    void saveState() override { saved_ = {bklen_, original_len_, actual_}; }
    void restoreState() override {
        bklen_ = saved_.bklen;
        original_len_ = saved_.len;
        actual_ = saved_.actual;
    }

private:
    struct Saved {
        uint32_t bklen = 1024;
        uint64_t len = 0;
        size_t actual = 0;
    };
    bool is_inverse_ = false;
    uint32_t bklen_ = 1024;
    HuffmanEncodeMode encode_mode_ = HuffmanEncodeMode::Coarse;
    uint64_t original_len_ = 0;
    size_t actual_ = 0;
    Saved saved_;
    StageWorkspace ws_;
};

// ---------------------------------------------------------------------------
// Bitpack: low nbits of each element, nbits a power of two (or detected).
// ---------------------------------------------------------------------------
template <typename T>
class BitpackStage : public Stage, public DeviceResults {
    static_assert(std::is_same<T, uint8_t>::value || std::is_same<T, uint16_t>::value ||
                      std::is_same<T, uint32_t>::value,
                  "BitpackStage: T must be uint8_t, uint16_t or uint32_t");

public:
    BitpackStage() = default;
    void setInverse(bool inv) override { is_inverse_ = inv; }
    bool isInverse() const override { return is_inverse_; }
    void setNBits(uint8_t nbits);
    uint8_t getNBits() const { return nbits_; }
    void setAutoDetect(bool enable) { auto_detect_ = enable; }
    bool isAutoDetect() const { return auto_detect_; }
    bool isGraphCompatible() const override { return !auto_detect_; }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    std::string getName() const override { return "Bitpack"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override;
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override { return index == 0 ? actual_ : 0; }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::BITPACK; }
    uint8_t getOutputDataType(size_t) const override { return (uint8_t)DataType::UNKNOWN; }
    uint8_t getInputDataType(size_t) const override { return (uint8_t)DataType::UNKNOWN; }
    // bitpack_stage.h:160-168: [u8 data type][u8 nbits][u64 element count]
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return 10; }
    void saveState() override { saved_ = {nbits_, num_elements_, actual_}; }
    void restoreState() override {
        nbits_ = saved_.nbits;
        num_elements_ = saved_.n;
        actual_ = saved_.actual;
    }

private:
    struct Saved {
        uint8_t nbits = 8 * sizeof(T);
        uint64_t n = 0;
        size_t actual = 0;
    };
    bool is_inverse_ = false;
    bool auto_detect_ = false;
    uint8_t nbits_ = 8 * sizeof(T);
    uint64_t num_elements_ = 0;
    size_t actual_ = 0;
    Saved saved_;
    StageWorkspace ws_;
};

// ---------------------------------------------------------------------------
// Quantizer: prediction-free quantisation (quantizers/quantizer/quantizer.h).
// Outputs codes, outlier_vals, outlier_idxs, outlier_count (codes only with
// in-place outliers).
// ---------------------------------------------------------------------------
// 36-byte container record (quantizer.h:25-47).
struct QuantizerConfig {
    float abs_error_bound;   // 0 for REL
    float user_error_bound;
    float value_base;        // NOA value range; 0 for ABS / REL
    uint32_t quant_radius;
    uint32_t num_elements;
    uint32_t outlier_count;
    DataType input_type;
    DataType code_type;
    uint8_t eb_mode;
    uint8_t zigzag_codes;
    float outlier_threshold;
    uint8_t inplace_outliers;
    uint8_t pad[3];
    QuantizerConfig()
        : abs_error_bound(0.0f), user_error_bound(0.0f), value_base(0.0f), quant_radius(0), num_elements(0),
          outlier_count(0), input_type(DataType::FLOAT32), code_type(DataType::UINT16), eb_mode(0), zigzag_codes(0),
          outlier_threshold(__builtin_inff()), inplace_outliers(0), pad{0, 0, 0} {}
};
static_assert(sizeof(QuantizerConfig) == 36, "QuantizerConfig is 36 bytes");

template <typename TInput = float, typename TCode = uint16_t>
class QuantizerStage : public Stage, public DeviceResults {
    static_assert(std::is_same<TInput, float>::value &&
                      (std::is_same<TCode, uint16_t>::value || std::is_same<TCode, uint32_t>::value),
                  "the sm_100a kernels implement QuantizerStage<float, uint16_t / uint32_t>");

public:
    struct Config {
        float error_bound = 1e-4f;
        int quant_radius = 32768;
        float outlier_capacity = 0.05f;
        ErrorBoundMode eb_mode = ErrorBoundMode::ABS;
        float precomputed_value_base = 0.0f;       // > 0 skips the NOA scan
        float outlier_threshold = __builtin_inff();  // |x| >= threshold -> outlier
        bool zigzag_codes = false;
        bool inplace_outliers = false;             // ABS / NOA, uint32 codes, zigzag
        Config() = default;
        Config(TInput eb, ErrorBoundMode mode = ErrorBoundMode::ABS, int radius = 32768, float outlier_cap = 0.05f)
            : error_bound(eb), quant_radius(radius), outlier_capacity(outlier_cap), eb_mode(mode) {}
    };

    explicit QuantizerStage(const Config& config = Config());

    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    void postStreamSync(cudaStream_t stream) override;
    void onGraphReplay(cudaStream_t) override { pending_ = !is_inverse_ && d_eb_state_ != nullptr && ran_; }
    void pendingReads(std::vector<DeviceRead>& out) override;
    void resultsFetched() override;
    bool deviceOutputSize(int index, DeviceSize* ds) const override;

    std::string getName() const override { return "Quantizer"; }
    size_t getNumInputs() const override { return is_inverse_ ? (isInplaceMode() ? 1 : 4) : 1; }
    size_t getNumOutputs() const override { return is_inverse_ ? 1 : (isInplaceMode() ? 1 : 4); }
    std::vector<std::string> getOutputNames() const override {
        if (is_inverse_) return {"reconstructed"};
        if (isInplaceMode()) return {"codes"};
        return {"codes", "outlier_vals", "outlier_idxs", "outlier_count"};
    }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& input_sizes) const override;
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override;
    size_t getActualOutputSize(int index) const override {
        return (index >= 0 && index < (int)actual_.size()) ? actual_[index] : 0;
    }
    size_t getExecuteTimeOutputSize(int index) const override {
        if (is_inverse_) return getActualOutputSize(index);
        return (index >= 0 && index < (int)at_execute_.size()) ? at_execute_[index] : 0;
    }
    void setInverse(bool inverse) override { is_inverse_ = inverse; }
    bool isInverse() const override { return is_inverse_; }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::QUANTIZER; }
    uint8_t getOutputDataType(size_t i) const override;
    uint8_t getInputDataType(size_t) const override {
        return (uint8_t)(is_inverse_ ? codeType() : DataType::FLOAT32);
    }
    size_t serializeHeader(size_t output_index, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return sizeof(QuantizerConfig); }
    void saveState() override { saved_ = {config_, num_elements_, actual_outlier_count_, computed_abs_eb_,
                                          computed_value_base_, actual_}; }
    void restoreState() override {
        config_ = saved_.config;
        num_elements_ = saved_.n;
        actual_outlier_count_ = saved_.count;
        computed_abs_eb_ = saved_.abs_eb;
        computed_value_base_ = saved_.vb;
        actual_ = saved_.actual;
    }

    void setErrorBound(TInput eb) { config_.error_bound = eb; }
    void setQuantRadius(int r) { config_.quant_radius = r; }
    void setOutlierCapacity(float c) { config_.outlier_capacity = c; }
    void setErrorBoundMode(ErrorBoundMode m) { config_.eb_mode = m; }
    void setValueBase(float vb) { config_.precomputed_value_base = vb; }
    void setZigzagCodes(bool enable) { config_.zigzag_codes = enable; }
    void setOutlierThreshold(float t) { config_.outlier_threshold = t; }
    void setInplaceOutliers(bool enable) { config_.inplace_outliers = enable; }
    TInput getErrorBound() const { return config_.error_bound; }
    int getQuantRadius() const { return config_.quant_radius; }
    ErrorBoundMode getErrorBoundMode() const { return config_.eb_mode; }
    float getValueBase() const { return config_.precomputed_value_base; }
    float getOutlierCapacity() const { return config_.outlier_capacity; }
    bool getZigzagCodes() const { return config_.zigzag_codes; }
    float getOutlierThreshold() const { return config_.outlier_threshold; }
    bool getInplaceOutliers() const { return config_.inplace_outliers; }
    // ceil(n * outlier_capacity) in single precision (quantizer.h:262-264).
    size_t getMaxOutlierCount(size_t n) const;
    float computedAbsErrorBound() const { return computed_abs_eb_; }
    bool isInplace() const { return isInplaceMode(); }

    // The one-pass Quantizer -> Difference(16 KiB) -> Bitshuffle(ew 2) -> RZE
    // path (uint32 codes) runs this stage's work itself; it records what
    // execute() would.
    void fusedForward(cudaStream_t stream, MemoryPool* pool, const void* d_in, size_t in_bytes, void* d_vals,
                      void* d_idx, void* d_count, void* d_rze, uint64_t* d_rze_size);

private:
    bool isInplaceMode() const { return config_.inplace_outliers && config_.eb_mode != ErrorBoundMode::REL; }
    static DataType codeType() { return sizeof(TCode) == 2 ? DataType::UINT16 : DataType::UINT32; }
    struct Saved {
        Config config;
        size_t n = 0;
        uint32_t count = 0;
        float abs_eb = 0.0f, vb = 0.0f;
        std::vector<size_t> actual;
    };
    Config config_;
    bool is_inverse_ = false;
    bool ran_ = false;
    bool pending_ = false;
    std::vector<size_t> actual_, at_execute_;
    size_t num_elements_ = 0;
    uint32_t actual_outlier_count_ = 0;
    float computed_abs_eb_ = 0.0f;
    float computed_value_base_ = 0.0f;
    const void* d_count_ = nullptr;
    float* d_eb_state_ = nullptr;  // inside the workspace
    bool fetched_ = false;  // h_count_ / h_state_ hold the pending values
    uint32_t h_count_ = 0;
    float h_state_[4] = {0, 0, 0, 0};
    Saved saved_;
    StageWorkspace ws_;
};

// ---------------------------------------------------------------------------
// Difference (predictors/diff/diff.h): first differences in power-of-two
// chunks; TOut the unsigned type of T's width fuses negabinary coding.
// ---------------------------------------------------------------------------
template <typename T, typename TOut = T>
class DifferenceStage : public Stage, public DeviceResults {
    static_assert(std::is_integral<T>::value && sizeof(T) == sizeof(TOut) &&
                      (std::is_same<T, TOut>::value || (std::is_signed<T>::value && std::is_unsigned<TOut>::value)),
                  "the sm_100a kernels implement integer DifferenceStage<T> and <signed, unsigned> pairs");

public:
    DifferenceStage() = default;
    void setInverse(bool inverse) override { is_inverse_ = inverse; }
    bool isInverse() const override { return is_inverse_; }
    void setChunkSize(size_t bytes) { chunk_size_ = bytes; }
    size_t getChunkSize() const { return chunk_size_; }
    size_t getRequiredInputAlignment() const override { return chunk_size_ > 0 ? chunk_size_ : 1; }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    std::string getName() const override { return "Difference"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override { return {s[0]}; }
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override { return index == 0 ? actual_ : 0; }
    void markFused(size_t bytes) { actual_ = bytes; }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::DIFFERENCE; }
    uint8_t getOutputDataType(size_t) const override;
    uint8_t getInputDataType(size_t) const override;
    // diff.h:120-140: [u8 T type][u8 TOut type][u32 chunk_size]
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return 6; }
    void saveState() override { saved_ = {chunk_size_, actual_}; }
    void restoreState() override {
        chunk_size_ = saved_[0];
        actual_ = saved_[1];
    }

private:
    bool is_inverse_ = false;
    size_t chunk_size_ = 0;
    size_t actual_ = 0;
    std::array<size_t, 2> saved_ = {0, 0};
    StageWorkspace ws_;
};

// ---------------------------------------------------------------------------
// Lorenzo (predictors/lorenzo/lorenzo_stage.h): lossless integer Lorenzo.
// ---------------------------------------------------------------------------
// 16-byte container record (lorenzo_stage.h:24-38).
struct LorenzoConfig {
    DataType data_type;
    uint8_t ndim;
    uint8_t reserved[2];
    uint32_t dim_x;
    uint32_t dim_y;
    uint32_t dim_z;
    LorenzoConfig() : data_type(DataType::INT32), ndim(1), reserved{0, 0}, dim_x(0), dim_y(1), dim_z(1) {}
};
static_assert(sizeof(LorenzoConfig) == 16, "LorenzoConfig is 16 bytes");

template <typename T>
class LorenzoStage : public Stage, public DeviceResults {
    static_assert(std::is_integral<T>::value && std::is_signed<T>::value, "LorenzoStage requires a signed integer type");

public:
    LorenzoStage() = default;
    void setInverse(bool inv) override { is_inverse_ = inv; }
    bool isInverse() const override { return is_inverse_; }
    void setDims(const std::array<size_t, 3>& dims) override { dims_ = dims; }
    void setDims(size_t x, size_t y = 1, size_t z = 1) { dims_ = {x, y, z}; }
    std::array<size_t, 3> getDims() const { return dims_; }
    int ndim() const { return dims_[2] > 1 ? 3 : (dims_[1] > 1 ? 2 : 1); }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    std::string getName() const override { return "Lorenzo"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override {
        return {s.empty() ? 0 : s[0]};
    }
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override { return index == 0 ? actual_ : 0; }
    uint16_t getStageTypeId() const override { return (uint16_t)StageType::LORENZO; }
    uint8_t getOutputDataType(size_t) const override { return (uint8_t)elemType(); }
    uint8_t getInputDataType(size_t) const override { return (uint8_t)elemType(); }
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override;
    void deserializeHeader(const uint8_t* buf, size_t size) override;
    size_t getMaxHeaderSize(size_t) const override { return sizeof(LorenzoConfig); }

private:
    static DataType elemType() {
        return sizeof(T) == 1 ? DataType::INT8
               : sizeof(T) == 2 ? DataType::INT16
               : sizeof(T) == 4 ? DataType::INT32
                                : DataType::INT64;
    }
    bool is_inverse_ = false;
    size_t actual_ = 0;
    std::array<size_t, 3> dims_ = {0, 1, 1};
    StageWorkspace ws_;
};

// ---------------------------------------------------------------------------
// Zigzag / Negabinary (transforms/zigzag/zigzag_stage.h,
// transforms/negabinary/negabinary_stage.h): signed <-> unsigned of the same
// width, header [u8 TIn type][u8 TOut type].
// ---------------------------------------------------------------------------
template <typename TIn, typename TOut, bool NEGABINARY>
class SignCodingStage : public Stage, public DeviceResults {
    static_assert(std::is_integral<TIn>::value && std::is_signed<TIn>::value && std::is_unsigned<TOut>::value &&
                      sizeof(TIn) == sizeof(TOut),
                  "TIn signed, TOut its unsigned counterpart");

public:
    void setInverse(bool inv) override { is_inverse_ = inv; }
    bool isInverse() const override { return is_inverse_; }
    void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                 const std::vector<void*>& outputs, const std::vector<size_t>& sizes) override;
    std::string getName() const override { return NEGABINARY ? "Negabinary" : "Zigzag"; }
    size_t getNumInputs() const override { return 1; }
    size_t getNumOutputs() const override { return 1; }
    std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& s) const override {
        return {s.empty() ? 0 : s[0]};
    }
    std::unordered_map<std::string, size_t> getActualOutputSizesByName() const override {
        return {{"output", actual_}};
    }
    size_t getActualOutputSize(int index) const override { return index == 0 ? actual_ : 0; }
    uint16_t getStageTypeId() const override {
        return (uint16_t)(NEGABINARY ? StageType::NEGABINARY : StageType::ZIGZAG);
    }
    uint8_t getOutputDataType(size_t) const override { return (uint8_t)(is_inverse_ ? inType() : outType()); }
    uint8_t getInputDataType(size_t) const override { return (uint8_t)(is_inverse_ ? outType() : inType()); }
    size_t serializeHeader(size_t, uint8_t* buf, size_t max_size) const override {
        if (max_size < 2) return 0;
        buf[0] = (uint8_t)inType();
        buf[1] = (uint8_t)outType();
        return 2;
    }
    void deserializeHeader(const uint8_t*, size_t) override {}
    size_t getMaxHeaderSize(size_t) const override { return 2; }

private:
    static DataType inType() {
        return sizeof(TIn) == 1 ? DataType::INT8
               : sizeof(TIn) == 2 ? DataType::INT16
               : sizeof(TIn) == 4 ? DataType::INT32
                                  : DataType::INT64;
    }
    static DataType outType() {
        return sizeof(TIn) == 1 ? DataType::UINT8
               : sizeof(TIn) == 2 ? DataType::UINT16
               : sizeof(TIn) == 4 ? DataType::UINT32
                                  : DataType::UINT64;
    }
    bool is_inverse_ = false;
    size_t actual_ = 0;
};

template <typename TIn, typename TOut>
using ZigzagStage = SignCodingStage<TIn, TOut, false>;
template <typename TIn, typename TOut>
using NegabinaryStage = SignCodingStage<TIn, TOut, true>;

// Rebuilds a stage from its container record (stage_factory.h:36-...).  The
// stage types of this library's path are supported; others throw.
Stage* createStage(StageType type, const uint8_t* config, size_t config_size);
// The Quantizer / Difference / Lorenzo / Zigzag / Negabinary cases of it;
// nullptr for other types.
Stage* createCodeStage(StageType type, const uint8_t* config, size_t config_size);

}  // namespace fz
