// stages.cpp -- fz:: stages over the libfzb C ABI.  Each stage keeps a
// device workspace from the pipeline's pool; results that only the device
// knows (outlier count, stream sizes, detected nbits) are read back after
// the pipeline synchronises (postStreamSync) or on first request.
#include "fz/stages.h"

#include <algorithm>
#include <cmath>
#include <string>

#include "fzb.h"

namespace fz {

namespace {

void check(int rc, const char* what) {
    if (rc != FZB_OK) throw std::runtime_error(std::string(what) + ": " + fzb_status_string(rc));
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
constexpr DataType dtype_of() {
    return std::is_same<T, uint8_t>::value    ? DataType::UINT8
           : std::is_same<T, uint16_t>::value ? DataType::UINT16
           : std::is_same<T, uint32_t>::value ? DataType::UINT32
           : std::is_same<T, int32_t>::value  ? DataType::INT32
                                              : DataType::UINT8;
}

constexpr size_t kTail = 256;  // per-stage device scalars after the workspace

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

// ---------------------------------------------------------------- workspace

StageWorkspace::~StageWorkspace() { release(); }

void StageWorkspace::release() {
    if (!ptr_) return;
    if (pool_) pool_->free(ptr_, 0);
    else cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
}

void StageWorkspace::checkStatus(cudaStream_t stream, const char* what) const {
    if (!ptr_) return;
    int st;
    if (fetched_) {  // gathered (and cleared on the device) before the pipeline's wait
        fetched_ = false;
        st = fzb_status_from_bits(h_bits_, nullptr);
    } else {
        st = fzb_workspace_status(ptr_, stream);
    }
    if (st != FZB_OK) throw std::runtime_error(std::string(what) + ": " + fzb_status_string(st));
}

// The status word is the workspace's first u32 (what fzb_workspace_status reads).
void StageWorkspace::pendingStatus(std::vector<DeviceRead>& out) const {
    if (!ptr_) return;
    out.push_back({ptr_, 4, &h_bits_, true});
}

void* StageWorkspace::ensure(size_t bytes, MemoryPool* pool, cudaStream_t stream) {
    bytes = align256(bytes ? bytes : 256);
    if (ptr_ && bytes_ >= bytes && pool_ == pool) return ptr_;
    if (ptr_) {
        // the old buffer may still be in use by enqueued work
        cudaStreamSynchronize(stream);
        release();
    }
    if (pool) {
        ptr_ = pool->allocate(bytes, stream, "stage_workspace", true);
    } else if (cudaMalloc(&ptr_, bytes) != cudaSuccess) {
        ptr_ = nullptr;
    }
    if (!ptr_) throw std::runtime_error("stage workspace allocation failed (" + std::to_string(bytes) + " bytes)");
    pool_ = pool;
    bytes_ = bytes;
    return ptr_;
}

// ------------------------------------------------------------- LorenzoQuant

template <typename TInput, typename TCode>
LorenzoQuantStage<TInput, TCode>::LorenzoQuantStage(const Config& config)
    : config_(config), actual_(4, 0), at_execute_(4, 0), computed_abs_eb_(config.error_bound),
      computed_value_base_(config.precomputed_value_base) {}

template <typename TInput, typename TCode>
size_t LorenzoQuantStage<TInput, TCode>::getMaxOutlierCount(size_t num_elements) const {
    const float prod = (float)num_elements * config_.outlier_capacity;  // single precision
    return (size_t)std::ceil(prod);
}

template <typename TInput, typename TCode>
std::vector<size_t> LorenzoQuantStage<TInput, TCode>::estimateOutputSizes(const std::vector<size_t>& s) const {
    if (is_inverse_) {
        const size_t n = s.empty() ? num_elements_ : s[0] / sizeof(TCode);
        return {n * sizeof(TInput)};
    }
    const size_t n = s.empty() ? 0 : s[0] / sizeof(TInput);
    const size_t cap = getMaxOutlierCount(n);
    return {n * sizeof(TCode), cap * sizeof(TInput), cap * sizeof(uint32_t), sizeof(uint32_t)};
}

template <typename TInput, typename TCode>
std::unordered_map<std::string, size_t> LorenzoQuantStage<TInput, TCode>::getActualOutputSizesByName() const {
    const auto names = getOutputNames();
    std::unordered_map<std::string, size_t> m;
    for (size_t i = 0; i < names.size() && i < actual_.size(); i++) m[names[i]] = actual_[i];
    return m;
}

template <typename TInput, typename TCode>
uint8_t LorenzoQuantStage<TInput, TCode>::getOutputDataType(size_t i) const {
    switch (i) {
        case 0: return (uint8_t)DataType::UINT16;
        case 1: return (uint8_t)DataType::FLOAT32;
        case 2:
        case 3: return (uint8_t)DataType::UINT32;
        default: return (uint8_t)DataType::UINT8;
    }
}

template <typename TInput, typename TCode>
void* LorenzoQuantStage<TInput, TCode>::forwardWorkspace(size_t n, size_t cap, MemoryPool* pool,
                                                         cudaStream_t stream) {
    const size_t need = fzb_workspace_bytes(n, cap);
    uint8_t* base = static_cast<uint8_t*>(ws_.ensure(align256(need) + kTail, pool, stream));
    d_eb_state_ = reinterpret_cast<float*>(base + align256(need));
    return base;
}

template <typename TInput, typename TCode>
void LorenzoQuantStage<TInput, TCode>::execute(cudaStream_t stream, MemoryPool* pool,
                                               const std::vector<void*>& inputs,
                                               const std::vector<void*>& outputs,
                                               const std::vector<size_t>& sizes) {
    uint32_t dims[3] = {(uint32_t)config_.dims[0], (uint32_t)config_.dims[1], (uint32_t)config_.dims[2]};
    if (is_inverse_) {
        if (inputs.size() < 4 || outputs.empty() || sizes.size() < 4)
            throw std::runtime_error("LorenzoQuantStage (inverse): Requires 4 inputs and 1 output");
        const size_t n = sizes[0] / sizeof(TCode);
        actual_.assign(1, 0);
        if (n == 0) return;
        const size_t cap = sizes[1] / sizeof(TInput);
        const size_t need = fzb_workspace_bytes(n, 0);
        void* w = inv_ws_.ensure(need, pool, stream);
        if (inv_dev_eb_ && d_eb_state_)
            check(fzb_lq_inverse_dev(static_cast<const uint16_t*>(inputs[0]), static_cast<const float*>(inputs[1]),
                                     static_cast<const uint32_t*>(inputs[2]), static_cast<const uint32_t*>(inputs[3]),
                                     cap, n, dims, d_eb_state_ + 1, config_.zigzag_codes ? 1 : 0,
                                     static_cast<float*>(outputs[0]), w, inv_ws_.size(), stream),
                  "LorenzoQuantStage (inverse)");
        else
            check(fzb_lq_inverse(static_cast<const uint16_t*>(inputs[0]), static_cast<const float*>(inputs[1]),
                                 static_cast<const uint32_t*>(inputs[2]), static_cast<const uint32_t*>(inputs[3]),
                                 cap, n, dims, computed_abs_eb_, config_.zigzag_codes ? 1 : 0,
                                 static_cast<float*>(outputs[0]), w, inv_ws_.size(), stream),
                  "LorenzoQuantStage (inverse)");
        actual_[0] = n * sizeof(TInput);
        return;
    }
    if (inputs.empty() || outputs.size() < 4 || sizes.empty())
        throw std::runtime_error("LorenzoQuantStage: Requires 1 input and 4 outputs");
    const size_t n = sizes[0] / sizeof(TInput);
    num_elements_ = n;
    actual_.assign(4, 0);
    at_execute_.assign(4, 0);
    actual_outlier_count_ = 0;
    pending_ = false;
    if (n == 0) return;
    const size_t cap = getMaxOutlierCount(n);
    void* w = forwardWorkspace(n, cap, pool, stream);
    check(fzb_lq_forward(static_cast<const float*>(inputs[0]), n, dims, config_.error_bound,
                         (int)config_.eb_mode, config_.precomputed_value_base, (uint32_t)config_.quant_radius,
                         config_.zigzag_codes ? 1 : 0, static_cast<uint16_t*>(outputs[0]),
                         static_cast<float*>(outputs[1]), static_cast<uint32_t*>(outputs[2]), cap,
                         static_cast<uint32_t*>(outputs[3]), d_eb_state_, w, ws_.size() - kTail, stream),
          "LorenzoQuantStage");
    d_count_ = outputs[3];
    pending_ = true;
    at_execute_ = {n * sizeof(TCode), cap * sizeof(TInput), cap * sizeof(uint32_t), sizeof(uint32_t)};
    actual_ = at_execute_;
}

template <typename TInput, typename TCode>
void LorenzoQuantStage<TInput, TCode>::fusedForward(cudaStream_t stream, MemoryPool* pool, const void* d_in,
                                                    size_t in_bytes, void* d_err, void* d_idx, void* d_count,
                                                    void* d_rze, uint64_t* d_rze_size) {
    uint32_t dims[3] = {(uint32_t)config_.dims[0], (uint32_t)config_.dims[1], (uint32_t)config_.dims[2]};
    const size_t n = in_bytes / sizeof(TInput);
    num_elements_ = n;
    actual_.assign(4, 0);
    at_execute_.assign(4, 0);
    actual_outlier_count_ = 0;
    pending_ = false;
    if (n == 0) return;
    const size_t cap = getMaxOutlierCount(n);
    void* w = forwardWorkspace(n, cap, pool, stream);
    check(fzb_lq_bs_rze_compress(static_cast<const float*>(d_in), n, dims, config_.error_bound,
                                 (int)config_.eb_mode, config_.precomputed_value_base,
                                 (uint32_t)config_.quant_radius, config_.zigzag_codes ? 1 : 0,
                                 static_cast<float*>(d_err), static_cast<uint32_t*>(d_idx), cap,
                                 static_cast<uint32_t*>(d_count), d_rze, d_rze_size, d_eb_state_, w,
                                 ws_.size() - kTail, stream),
          "LorenzoQuant->Bitshuffle->RZE");
    d_count_ = d_count;
    pending_ = true;
    at_execute_ = {n * sizeof(TCode), cap * sizeof(TInput), cap * sizeof(uint32_t), sizeof(uint32_t)};
    actual_ = at_execute_;
}

template <typename TInput, typename TCode>
void LorenzoQuantStage<TInput, TCode>::postStreamSync(cudaStream_t stream) {
    if (is_inverse_) {
        inv_ws_.checkStatus(stream, "LorenzoQuantStage (inverse)");
        return;
    }
    if (!pending_) return;
    pending_ = false;
    uint32_t count = 0;
    float st[4] = {0, 0, 0, 0};
    if (fetched_) {  // gathered before the pipeline's wait
        fetched_ = false;
        count = h_count_;
        std::memcpy(st, h_state_, sizeof(st));
    } else {
        check_cuda(cudaMemcpy(&count, d_count_, 4, cudaMemcpyDeviceToHost), "LorenzoQuant outlier count");
        check_cuda(cudaMemcpy(st, d_eb_state_, sizeof(st), cudaMemcpyDeviceToHost), "LorenzoQuant eb state");
    }
    computed_abs_eb_ = st[1];
    computed_value_base_ = (config_.eb_mode == ErrorBoundMode::ABS) ? 0.0f : st[0];
    const size_t cap = getMaxOutlierCount(num_elements_);
    if (count > cap) count = (uint32_t)cap;  // outliers past the capacity are dropped
    actual_outlier_count_ = count;
    actual_[1] = count * sizeof(TInput);
    actual_[2] = count * sizeof(uint32_t);
}

template <typename TInput, typename TCode>
void LorenzoQuantStage<TInput, TCode>::pendingReads(std::vector<DeviceRead>& out) {
    if (is_inverse_) {
        inv_ws_.pendingStatus(out);
        return;
    }
    if (!pending_) return;
    out.push_back({d_count_, 4, &h_count_, false});
    out.push_back({d_eb_state_, sizeof(h_state_), h_state_, false});
}

template <typename TInput, typename TCode>
void LorenzoQuantStage<TInput, TCode>::resultsFetched() {
    if (is_inverse_) inv_ws_.statusFetched();
    else fetched_ = pending_;
}

// The outlier lists hold min(count, capacity) entries (postStreamSync's clamp).
template <typename TInput, typename TCode>
bool LorenzoQuantStage<TInput, TCode>::deviceOutputSize(int index, DeviceSize* ds) const {
    if (is_inverse_ || !pending_ || (index != 1 && index != 2)) return false;
    *ds = {d_count_, 4, index == 1 ? sizeof(TInput) : sizeof(uint32_t), getMaxOutlierCount(num_elements_)};
    return true;
}

template <typename TInput, typename TCode>
size_t LorenzoQuantStage<TInput, TCode>::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < sizeof(LorenzoQuantConfig)) throw std::runtime_error("Insufficient buffer for Lorenzo config");
    LorenzoQuantConfig c;
    c.error_bound = computed_abs_eb_;
    c.quant_radius = (uint32_t)config_.quant_radius;
    c.num_elements = (uint32_t)num_elements_;
    c.outlier_count = actual_outlier_count_;
    c.input_type = DataType::FLOAT32;
    c.code_type = DataType::UINT16;
    c.ndim = (uint8_t)ndim();
    c.eb_mode = (uint8_t)config_.eb_mode;
    c.dim_x = (uint32_t)config_.dims[0];
    c.dim_y = (uint32_t)config_.dims[1];
    c.dim_z = (uint32_t)config_.dims[2];
    c.user_eb = config_.error_bound;
    c.value_base = computed_value_base_;
    c.zigzag_codes = config_.zigzag_codes ? 1 : 0;
    std::memcpy(buf, &c, sizeof(c));
    return sizeof(c);
}

template <typename TInput, typename TCode>
void LorenzoQuantStage<TInput, TCode>::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size < 32) throw std::runtime_error("Invalid Lorenzo config size");
    LorenzoQuantConfig c;
    std::memcpy(&c, buf, std::min(size, sizeof(c)));
    config_.error_bound = c.error_bound;
    computed_abs_eb_ = c.error_bound;
    config_.quant_radius = (int)c.quant_radius;
    num_elements_ = c.num_elements;
    actual_outlier_count_ = c.outlier_count;
    if (size >= 40) {  // user_eb / value_base / eb_mode present
        config_.eb_mode = (ErrorBoundMode)c.eb_mode;
        config_.precomputed_value_base = c.value_base;
        computed_value_base_ = c.value_base;
    } else {
        config_.eb_mode = ErrorBoundMode::ABS;
        config_.precomputed_value_base = 0.0f;
        computed_value_base_ = 0.0f;
    }
    config_.zigzag_codes = size >= sizeof(c) && c.zigzag_codes != 0;
    const int nd = c.ndim == 0 ? 1 : c.ndim;
    if (c.dim_x > 0) config_.dims[0] = c.dim_x;
    else if (c.num_elements > 0)
        config_.dims[0] = c.num_elements / (std::max<size_t>(1, c.dim_y) * std::max<size_t>(1, c.dim_z));
    else config_.dims[0] = 0;
    config_.dims[1] = nd >= 2 ? (c.dim_y > 0 ? c.dim_y : 1) : 1;
    config_.dims[2] = nd >= 3 ? (c.dim_z > 0 ? c.dim_z : 1) : 1;
}

template class LorenzoQuantStage<float, uint16_t>;

// --------------------------------------------------------------- Bitshuffle

void BitshuffleStage::execute(cudaStream_t stream, MemoryPool*, const std::vector<void*>& inputs,
                              const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty())
        throw std::runtime_error("BitshuffleStage: invalid inputs/outputs");
    // bitshuffle_stage.h:139-150
    if (element_width_ != 1 && element_width_ != 2 && element_width_ != 4 && element_width_ != 8)
        throw std::invalid_argument("BitshuffleStage: element_width must be 1, 2, 4, or 8");
    if (block_size_ == 0 || block_size_ % (1024u * element_width_) != 0)
        throw std::invalid_argument("BitshuffleStage: block_size must be a positive multiple of 1024 * element_width");
    actual_ = sizes[0];
    if (sizes[0] == 0) return;
    check(fzb_bitshuffle(inputs[0], sizes[0], block_size_, element_width_, is_inverse_ ? 1 : 0, outputs[0],
                         stream),
          "BitshuffleStage");
}

size_t BitshuffleStage::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < 5) return 0;
    std::memcpy(buf, &block_size_, 4);
    buf[4] = element_width_;
    return 5;
}

void BitshuffleStage::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size >= 4) std::memcpy(&block_size_, buf, 4);
    if (size >= 5) element_width_ = buf[4];
}

// ---------------------------------------------------------------------- RZE

std::vector<size_t> RZEStage::estimateOutputSizes(const std::vector<size_t>& s) const {
    if (is_inverse_) return {cached_orig_bytes_ ? (size_t)cached_orig_bytes_ : (s.empty() ? 0 : s[0])};
    const size_t n = s.empty() ? 0 : s[0];
    const size_t nch = (n + chunk_size_ - 1) / chunk_size_;
    return {n + 8 + 4 * nch};
}

size_t RZEStage::estimateScratchBytes(const std::vector<size_t>& s) const {
    if (is_inverse_ || s.empty()) return 0;
    const size_t nch = (s[0] + chunk_size_ - 1) / chunk_size_;
    return nch * ((size_t)chunk_size_ + 12);
}

void RZEStage::readBack() const {
    if (!d_size_) return;
    if (fetched_) {  // gathered before the pipeline's wait
        fetched_ = false;
        actual_ = (size_t)h_size_;
        d_size_ = nullptr;
        return;
    }
    cudaStreamSynchronize(pending_stream_);
    uint64_t v = 0;
    check_cuda(cudaMemcpy(&v, d_size_, 8, cudaMemcpyDeviceToHost), "RZE size read-back");
    actual_ = (size_t)v;
    d_size_ = nullptr;
}

void RZEStage::postStreamSync(cudaStream_t stream) {
    if (is_inverse_) ws_.checkStatus(stream, "RZEStage (inverse)");
    else readBack();
}

void RZEStage::markFused(size_t in_bytes, const uint64_t* d_size, cudaStream_t stream) {
    cached_orig_bytes_ = (uint32_t)in_bytes;
    actual_ = 0;
    d_size_ = d_size;
    last_size_ = d_size;
    pending_stream_ = stream;
}

void RZEStage::execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                       const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty()) throw std::runtime_error("RZEStage: invalid inputs/outputs");
    d_size_ = nullptr;
    if (chunk_size_ != 16384)
        throw std::runtime_error("RZEStage: only chunk_size == 16384 is currently supported; got " +
                                 std::to_string(chunk_size_));
    if (levels_ != 4)
        throw std::runtime_error("RZEStage: only levels == 4 is currently supported; got " +
                                 std::to_string((int)levels_));
    if (is_inverse_) {
        const size_t orig = cached_orig_bytes_;
        actual_ = orig;
        if (orig == 0) return;
        const size_t need = fzb_workspace_bytes((orig + 1) / 2, 0);
        void* w = ws_.ensure(need, pool, stream);
        check(fzb_rze_decode(inputs[0], sizes[0], orig, outputs[0], w, ws_.size(), stream), "RZEStage (inverse)");
        return;
    }
    const size_t in_bytes = sizes[0];
    cached_orig_bytes_ = (uint32_t)in_bytes;
    actual_ = 0;
    if (in_bytes == 0) return;
    const size_t need = fzb_workspace_bytes((in_bytes + 1) / 2, 0);
    uint8_t* w = static_cast<uint8_t*>(ws_.ensure(align256(need) + kTail, pool, stream));
    d_size_own_ = reinterpret_cast<uint64_t*>(w + align256(need));
    check(fzb_rze_encode(inputs[0], in_bytes, outputs[0], d_size_own_, w, align256(need), stream), "RZEStage");
    d_size_ = d_size_own_;
    last_size_ = d_size_own_;
    pending_stream_ = stream;
}

size_t RZEStage::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < 9) return 0;
    std::memcpy(buf, &chunk_size_, 4);
    buf[4] = levels_;
    std::memcpy(buf + 5, &cached_orig_bytes_, 4);
    return 9;
}

void RZEStage::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size >= 4) std::memcpy(&chunk_size_, buf, 4);
    if (size >= 5) levels_ = buf[4];
    if (size >= 9) std::memcpy(&cached_orig_bytes_, buf + 5, 4);
}

// ---------------------------------------------------------------------- RLE

template <typename T>
DataType RLEStage<T>::dtype() {
    return dtype_of<T>();
}

template <typename T>
std::vector<size_t> RLEStage<T>::estimateOutputSizes(const std::vector<size_t>& s) const {
    if (is_inverse_) {
        if (cached_num_elements_ > 0) return {(size_t)cached_num_elements_ * sizeof(T)};
        return {s.empty() ? 0 : s[0] * 2};
    }
    const size_t n = s.empty() ? 0 : s[0] / sizeof(T);
    return {4 + ((n * sizeof(T) + 3) & ~(size_t)3) + 4 * n};
}

template <typename T>
void RLEStage<T>::readBack() const {
    if (!d_size_) return;
    if (fetched_) {  // gathered before the pipeline's wait
        fetched_ = false;
        actual_ = (size_t)h_size_;
        d_size_ = nullptr;
        return;
    }
    cudaStreamSynchronize(pending_stream_);
    uint64_t v = 0;
    check_cuda(cudaMemcpy(&v, d_size_, 8, cudaMemcpyDeviceToHost), "RLE size read-back");
    actual_ = (size_t)v;
    d_size_ = nullptr;
}

template <typename T>
void RLEStage<T>::postStreamSync(cudaStream_t stream) {
    if (is_inverse_) ws_.checkStatus(stream, "RLEStage (inverse)");
    else readBack();
}

template <typename T>
void RLEStage<T>::execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                          const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty()) throw std::runtime_error("RLEStage: invalid inputs/outputs");
    d_size_ = nullptr;
    if (is_inverse_) {
        const size_t n = cached_num_elements_;
        actual_ = n * sizeof(T);
        if (n == 0) return;
        void* w = ws_.ensure(fzb_workspace_bytes(n, 0), pool, stream);
        check(fzb_rle_decode(inputs[0], n, (int)sizeof(T), outputs[0], w, ws_.size(), stream), "RLEStage (inverse)");
        return;
    }
    const size_t n = sizes[0] / sizeof(T);
    cached_num_elements_ = (uint32_t)n;
    actual_ = 0;
    if (n == 0) return;
    const size_t need = fzb_workspace_bytes(n, 0);
    uint8_t* w = static_cast<uint8_t*>(ws_.ensure(align256(need) + kTail, pool, stream));
    uint64_t* d_size = reinterpret_cast<uint64_t*>(w + align256(need));
    check(fzb_rle_encode(inputs[0], n, (int)sizeof(T), outputs[0], d_size, w, align256(need), stream), "RLEStage");
    d_size_ = d_size;
    last_size_ = d_size;
    pending_stream_ = stream;
}

template <typename T>
size_t RLEStage<T>::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < 5) return 0;
    const DataType dt = dtype();
    std::memcpy(buf, &dt, 1);
    std::memcpy(buf + 1, &cached_num_elements_, 4);
    return 5;
}

template <typename T>
void RLEStage<T>::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size >= 5) std::memcpy(&cached_num_elements_, buf + 1, 4);
}

template class RLEStage<uint8_t>;
template class RLEStage<uint16_t>;
template class RLEStage<uint32_t>;
template class RLEStage<int32_t>;

// ------------------------------------------------------------------ Huffman

template <typename T>
void HuffmanStage<T>::execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                              const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty()) throw std::runtime_error("HuffmanStage: invalid inputs/outputs");
    if (is_inverse_) {
        const size_t n = original_len_;
        actual_ = n * sizeof(T);
        if (n == 0) return;
        void* w = ws_.ensure(256, pool, stream);
        check(fzb_huff_decode(inputs[0], sizes[0], n, bklen_, static_cast<uint16_t*>(outputs[0]), w, ws_.size(),
                              stream),
              "HuffmanStage (inverse)");
        return;
    }
    const size_t n = sizes[0] / sizeof(T);
    original_len_ = n;
    actual_ = 0;
    if (n == 0) return;
    const size_t need = fzb_huff_workspace_bytes(n, bklen_);
    if (need == 0) throw std::runtime_error("HuffmanStage: unsupported bklen " + std::to_string(bklen_));
    uint8_t* w = static_cast<uint8_t*>(ws_.ensure(align256(need) + kTail, pool, stream));
    uint64_t* d_size = reinterpret_cast<uint64_t*>(w + align256(need));
    const auto compress = encode_mode_ == HuffmanEncodeMode::Fine ? fzb_huff_compress_fine : fzb_huff_compress;
    const int rc = compress(static_cast<const uint16_t*>(inputs[0]), n, bklen_, outputs[0], d_size, w,
                            align256(need), stream);
    if (rc == FZB_E_RANGE)
        throw std::runtime_error("HuffmanStage: input contains symbols >= bklen (" + std::to_string(bklen_) +
                                 "). Increase bklen or use setZigzagCodes(true) with LorenzoQuantStage.");
    check(rc, "HuffmanStage");
    uint64_t v = 0;
    check_cuda(cudaStreamSynchronize(stream), "HuffmanStage");
    check_cuda(cudaMemcpy(&v, d_size, 8, cudaMemcpyDeviceToHost), "HuffmanStage size read-back");
    actual_ = (size_t)v;
}

template <typename T>
size_t HuffmanStage<T>::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < 11) return 0;
    buf[0] = (uint8_t)dtype_of<T>();
    const uint16_t bk = (uint16_t)bklen_;
    std::memcpy(buf + 1, &bk, 2);
    std::memcpy(buf + 3, &original_len_, 8);
    return 11;
}

template <typename T>
void HuffmanStage<T>::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size >= 3) {
        uint16_t bk;
        std::memcpy(&bk, buf + 1, 2);
        bklen_ = bk;
    }
    if (size >= 11) std::memcpy(&original_len_, buf + 3, 8);
}

template class HuffmanStage<uint16_t>;

// ------------------------------------------------------------------ Bitpack

template <typename T>
void BitpackStage<T>::setNBits(uint8_t nbits) {
    if (nbits == 0 || nbits > 8 * sizeof(T) || (nbits & (nbits - 1)) != 0)
        throw std::invalid_argument("BitpackStage::setNBits: nbits must be a power of two in [1, " +
                                    std::to_string(8 * sizeof(T)) + "], got " + std::to_string(nbits));
    nbits_ = nbits;
}

template <typename T>
std::vector<size_t> BitpackStage<T>::estimateOutputSizes(const std::vector<size_t>& s) const {
    if (s.empty()) return {0};
    if (!is_inverse_) {
        if (auto_detect_) return {s[0]};
        const size_t n = s[0] / sizeof(T);
        return {(n * nbits_ + 7) / 8};
    }
    return {((s[0] * 8 + nbits_ - 1) / nbits_) * sizeof(T)};
}

template <typename T>
void BitpackStage<T>::execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                              const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty()) throw std::runtime_error("BitpackStage: invalid inputs/outputs");
    if (is_inverse_) {
        const size_t n = num_elements_;
        actual_ = n * sizeof(T);
        if (n == 0) return;
        check(fzb_bitpack_decode(inputs[0], n, (int)sizeof(T), nbits_, outputs[0], stream), "BitpackStage (inverse)");
        return;
    }
    const size_t n = sizes[0] / sizeof(T);
    num_elements_ = n;
    actual_ = 0;
    if (n == 0) return;
    uint8_t* w = static_cast<uint8_t*>(ws_.ensure(fzb_workspace_bytes(1, 0) + kTail, pool, stream));
    uint8_t* d_nbits = w + align256(fzb_workspace_bytes(1, 0));
    check(fzb_bitpack_encode(inputs[0], n, (int)sizeof(T), auto_detect_ ? 0 : nbits_, outputs[0], d_nbits, nullptr,
                             w, align256(fzb_workspace_bytes(1, 0)), stream),
          "BitpackStage");
    if (auto_detect_) {  // the detected width is host state (header, output size)
        check_cuda(cudaStreamSynchronize(stream), "BitpackStage");
        check_cuda(cudaMemcpy(&nbits_, d_nbits, 1, cudaMemcpyDeviceToHost), "BitpackStage nbits read-back");
    }
    actual_ = (n * nbits_ + 7) / 8;
}

template <typename T>
size_t BitpackStage<T>::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < 10) return 0;
    buf[0] = (uint8_t)dtype_of<T>();
    buf[1] = nbits_;
    std::memcpy(buf + 2, &num_elements_, 8);
    return 10;
}

template <typename T>
void BitpackStage<T>::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size >= 2) nbits_ = buf[1];
    if (size >= 10) std::memcpy(&num_elements_, buf + 2, 8);
}

template class BitpackStage<uint8_t>;
template class BitpackStage<uint16_t>;
template class BitpackStage<uint32_t>;

// ------------------------------------------------------------------ factory

Stage* createStage(StageType type, const uint8_t* config, size_t config_size) {
    Stage* s = nullptr;
    switch (type) {
        case StageType::LORENZO_QUANT: {
            if (config_size < sizeof(LorenzoQuantConfig))
                throw std::runtime_error("Lorenzo config too small: " + std::to_string(config_size));
            LorenzoQuantConfig c;
            std::memcpy(&c, config, sizeof(c));
            if (c.input_type != DataType::FLOAT32 || c.code_type != DataType::UINT16)
                throw std::runtime_error("Unsupported Lorenzo template instantiation: input_type=" +
                                         std::to_string((int)c.input_type) +
                                         " code_type=" + std::to_string((int)c.code_type));
            s = new LorenzoQuantStage<float, uint16_t>();
            break;
        }
        case StageType::BITSHUFFLE: s = new BitshuffleStage(); break;
        case StageType::RZE: s = new RZEStage(); break;
        case StageType::RLE: {
            const DataType dt = config_size >= 1 ? (DataType)config[0] : DataType::UINT16;
            switch (dt) {
                case DataType::UINT8: s = new RLEStage<uint8_t>(); break;
                case DataType::UINT16: s = new RLEStage<uint16_t>(); break;
                case DataType::UINT32: s = new RLEStage<uint32_t>(); break;
                case DataType::INT32: s = new RLEStage<int32_t>(); break;
                default: throw std::runtime_error("Unsupported RLE data type: " + std::to_string((int)dt));
            }
            break;
        }
        case StageType::HUFFMAN: {
            const DataType dt = config_size >= 1 ? (DataType)config[0] : DataType::UINT16;
            if (dt != DataType::UINT16)
                throw std::runtime_error("Unsupported Huffman symbol type: " + std::to_string((int)dt));
            s = new HuffmanStage<uint16_t>();
            break;
        }
        case StageType::BITPACK: {
            const DataType dt = config_size >= 1 ? (DataType)config[0] : DataType::UINT16;
            switch (dt) {
                case DataType::UINT8: s = new BitpackStage<uint8_t>(); break;
                case DataType::UINT16: s = new BitpackStage<uint16_t>(); break;
                case DataType::UINT32: s = new BitpackStage<uint32_t>(); break;
                default: throw std::runtime_error("Unsupported Bitpack data type: " + std::to_string((int)dt));
            }
            break;
        }
        default:
            s = createCodeStage(type, config, config_size);
            if (!s)
                throw std::runtime_error("Unsupported stage type " + std::to_string((int)type) + " (" +
                                         stageTypeToString(type) + ")");
    }
    if (config_size) s->deserializeHeader(config, config_size);
    return s;
}

}  // namespace fz
