// stages_codes.cpp -- the stages that work on integer codes around the
// quantiser: Quantizer, Difference, Lorenzo (lossless), Zigzag, Negabinary.
// Each runs the sm_100a kernels behind fzb_quantizer_* / fzb_diff /
// fzb_lorenzo_int / fzb_zigzag / fzb_negabinary; messages of the errors the
// reference throws are kept.
#include <algorithm>
#include <cmath>
#include <string>

#include "fz/stages.h"
#include "fzb.h"

namespace fz {

namespace {

void check(int rc, const char* what) {
    if (rc != FZB_OK) throw std::runtime_error(std::string(what) + ": " + fzb_status_string(rc));
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

constexpr size_t kTail = 256;  // eb state after the quantizer workspace

template <typename T>
constexpr DataType int_dtype() {
    return std::is_signed<T>::value
               ? (sizeof(T) == 1 ? DataType::INT8
                  : sizeof(T) == 2 ? DataType::INT16
                  : sizeof(T) == 4 ? DataType::INT32
                                   : DataType::INT64)
               : (sizeof(T) == 1 ? DataType::UINT8
                  : sizeof(T) == 2 ? DataType::UINT16
                  : sizeof(T) == 4 ? DataType::UINT32
                                   : DataType::UINT64);
}

}  // namespace

// ---------------------------------------------------------------- Quantizer

template <typename TInput, typename TCode>
QuantizerStage<TInput, TCode>::QuantizerStage(const Config& config)
    : config_(config), actual_(4, 0), at_execute_(4, 0), computed_abs_eb_(config.error_bound),
      computed_value_base_(config.precomputed_value_base) {}

template <typename TInput, typename TCode>
size_t QuantizerStage<TInput, TCode>::getMaxOutlierCount(size_t n) const {
    return (size_t)std::ceil((float)n * config_.outlier_capacity);
}

template <typename TInput, typename TCode>
std::vector<size_t> QuantizerStage<TInput, TCode>::estimateOutputSizes(const std::vector<size_t>& s) const {
    if (is_inverse_) {
        const size_t n = s.empty() ? 0 : s[0] / sizeof(TCode);
        return {n * sizeof(TInput)};
    }
    const size_t n = s.empty() ? 0 : s[0] / sizeof(TInput);
    if (isInplaceMode()) return {n * sizeof(TCode)};
    const size_t cap = getMaxOutlierCount(n);
    return {n * sizeof(TCode), cap * sizeof(TInput), cap * sizeof(uint32_t), sizeof(uint32_t)};
}

template <typename TInput, typename TCode>
std::unordered_map<std::string, size_t> QuantizerStage<TInput, TCode>::getActualOutputSizesByName() const {
    const auto names = getOutputNames();
    std::unordered_map<std::string, size_t> m;
    for (size_t i = 0; i < names.size() && i < actual_.size(); i++) m[names[i]] = actual_[i];
    return m;
}

template <typename TInput, typename TCode>
uint8_t QuantizerStage<TInput, TCode>::getOutputDataType(size_t i) const {
    if (is_inverse_) return (uint8_t)DataType::FLOAT32;
    if (isInplaceMode()) return (uint8_t)codeType();
    switch (i) {
        case 0: return (uint8_t)codeType();
        case 1: return (uint8_t)DataType::FLOAT32;
        case 2:
        case 3: return (uint8_t)DataType::UINT32;
        default: return (uint8_t)DataType::UINT8;
    }
}

template <typename TInput, typename TCode>
void QuantizerStage<TInput, TCode>::execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                                            const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    const bool inpl = isInplaceMode();
    const int mode = (int)config_.eb_mode;
    if (is_inverse_) {
        const size_t want = inpl ? 1 : 4;
        if (inputs.size() < want || outputs.empty() || sizes.empty())
            throw std::runtime_error(inpl ? "QuantizerStage (inverse, inplace): requires 1 input and 1 output"
                                          : "QuantizerStage (inverse): requires 4 inputs and 1 output");
        const size_t n = sizes[0] / sizeof(TCode);
        actual_.assign(1, 0);
        if (n == 0) return;
        const size_t cap = (!inpl && sizes.size() > 1) ? sizes[1] / sizeof(TInput) : 0;
        check(fzb_quantizer_inverse(inputs[0], n, (int)sizeof(TCode), config_.error_bound, mode, computed_abs_eb_,
                                    (uint32_t)config_.quant_radius, config_.zigzag_codes ? 1 : 0, inpl ? 1 : 0,
                                    inpl ? nullptr : static_cast<const float*>(inputs[1]),
                                    inpl ? nullptr : static_cast<const uint32_t*>(inputs[2]),
                                    inpl ? nullptr : static_cast<const uint32_t*>(inputs[3]), cap,
                                    static_cast<float*>(outputs[0]), stream),
              "QuantizerStage (inverse)");
        actual_[0] = n * sizeof(TInput);
        return;
    }
    if (inputs.empty() || outputs.size() < (inpl ? 1u : 4u) || sizes.empty())
        throw std::runtime_error(inpl ? "QuantizerStage (inplace): requires 1 input and 1 output"
                                      : "QuantizerStage: requires 1 input and 4 outputs");
    if (inpl && !config_.zigzag_codes)
        throw std::runtime_error("QuantizerStage: setInplaceOutliers(true) requires setZigzagCodes(true)");
    if (inpl && sizeof(TCode) != sizeof(TInput))
        throw std::runtime_error(
            "QuantizerStage: setInplaceOutliers(true) requires sizeof(TCode)==sizeof(TInput) "
            "(use QuantizerStage<float, uint32_t>)");
    const size_t n = sizes[0] / sizeof(TInput);
    num_elements_ = n;
    actual_outlier_count_ = 0;
    pending_ = false;
    ran_ = false;
    computed_abs_eb_ = config_.eb_mode == ErrorBoundMode::ABS ? config_.error_bound : 0.0f;
    computed_value_base_ = 0.0f;
    at_execute_.assign(inpl ? 1 : 4, 0);
    actual_ = at_execute_;
    if (n == 0) return;
    const size_t cap = inpl ? 0 : getMaxOutlierCount(n);
    const size_t need = align256(fzb_quantizer_workspace_bytes(n));
    uint8_t* base = static_cast<uint8_t*>(ws_.ensure(need + kTail, pool, stream));
    d_eb_state_ = reinterpret_cast<float*>(base + need);
    check(fzb_quantizer_forward(static_cast<const float*>(inputs[0]), n, (int)sizeof(TCode), config_.error_bound, mode,
                                config_.precomputed_value_base, (uint32_t)config_.quant_radius,
                                config_.zigzag_codes ? 1 : 0, config_.outlier_threshold, inpl ? 1 : 0, outputs[0],
                                inpl ? nullptr : static_cast<float*>(outputs[1]),
                                inpl ? nullptr : static_cast<uint32_t*>(outputs[2]),
                                inpl ? nullptr : static_cast<uint32_t*>(outputs[3]), cap, d_eb_state_, base, need,
                                stream),
          "QuantizerStage");
    d_count_ = inpl ? nullptr : outputs[3];
    pending_ = ran_ = true;
    if (inpl) at_execute_ = {n * sizeof(TCode)};
    else at_execute_ = {n * sizeof(TCode), cap * sizeof(TInput), cap * sizeof(uint32_t), sizeof(uint32_t)};
    actual_ = at_execute_;
}

template <typename TInput, typename TCode>
void QuantizerStage<TInput, TCode>::fusedForward(cudaStream_t stream, MemoryPool* pool, const void* d_in,
                                                 size_t in_bytes, void* d_vals, void* d_idx, void* d_count,
                                                 void* d_rze, uint64_t* d_rze_size) {
    if (sizeof(TCode) != 4 || isInplaceMode())
        throw std::runtime_error("QuantizerStage: the one-pass chain needs uint32 codes and outlier lists");
    const size_t n = in_bytes / sizeof(TInput);
    num_elements_ = n;
    actual_outlier_count_ = 0;
    pending_ = ran_ = false;
    computed_abs_eb_ = config_.eb_mode == ErrorBoundMode::ABS ? config_.error_bound : 0.0f;
    computed_value_base_ = 0.0f;
    at_execute_.assign(4, 0);
    actual_ = at_execute_;
    if (n == 0) return;
    const size_t cap = getMaxOutlierCount(n);
    const size_t need = align256(fzb_pfpl_workspace_bytes(n, cap));
    uint8_t* base = static_cast<uint8_t*>(ws_.ensure(need + kTail, pool, stream));
    d_eb_state_ = reinterpret_cast<float*>(base + need);
    check(fzb_pfpl_compress(static_cast<const float*>(d_in), n, config_.error_bound, (int)config_.eb_mode,
                            config_.precomputed_value_base, (uint32_t)config_.quant_radius,
                            config_.zigzag_codes ? 1 : 0, config_.outlier_threshold, static_cast<float*>(d_vals),
                            static_cast<uint32_t*>(d_idx), cap, static_cast<uint32_t*>(d_count), d_rze, d_rze_size,
                            d_eb_state_, base, need, stream),
          "Quantizer->Difference->Bitshuffle->RZE");
    d_count_ = d_count;
    pending_ = ran_ = true;
    at_execute_ = {n * sizeof(TCode), cap * sizeof(TInput), cap * sizeof(uint32_t), sizeof(uint32_t)};
    actual_ = at_execute_;
}

template <typename TInput, typename TCode>
void QuantizerStage<TInput, TCode>::postStreamSync(cudaStream_t stream) {
    if (is_inverse_ || !pending_) return;
    pending_ = false;
    const bool fetched = fetched_;  // gathered before the pipeline's wait
    fetched_ = false;
    ws_.checkStatus(stream, "QuantizerStage");
    float st[4] = {0, 0, 0, 0};
    if (fetched) std::memcpy(st, h_state_, sizeof(st));
    else check_cuda(cudaMemcpy(st, d_eb_state_, sizeof(st), cudaMemcpyDeviceToHost), "Quantizer eb state");
    if (config_.eb_mode == ErrorBoundMode::NOA) {
        computed_value_base_ = st[0];
        computed_abs_eb_ = st[1];
    }
    if (d_count_) {
        uint32_t count = h_count_;  // already min(outliers, capacity) on the device
        if (!fetched)
            check_cuda(cudaMemcpy(&count, d_count_, 4, cudaMemcpyDeviceToHost), "Quantizer outlier count");
        actual_outlier_count_ = count;
        actual_[1] = count * sizeof(TInput);
        actual_[2] = count * sizeof(uint32_t);
    }
}

template <typename TInput, typename TCode>
void QuantizerStage<TInput, TCode>::pendingReads(std::vector<DeviceRead>& out) {
    if (is_inverse_ || !pending_) return;
    ws_.pendingStatus(out);
    out.push_back({d_eb_state_, sizeof(h_state_), h_state_, false});
    if (d_count_) out.push_back({d_count_, 4, &h_count_, false});
}

template <typename TInput, typename TCode>
void QuantizerStage<TInput, TCode>::resultsFetched() {
    if (is_inverse_ || !pending_) return;
    ws_.statusFetched();
    fetched_ = true;
}

template <typename TInput, typename TCode>
bool QuantizerStage<TInput, TCode>::deviceOutputSize(int index, DeviceSize* ds) const {
    if (is_inverse_ || !pending_ || !d_count_ || (index != 1 && index != 2)) return false;
    *ds = {d_count_, 4, index == 1 ? sizeof(TInput) : sizeof(uint32_t), ~0ull / sizeof(TInput)};
    return true;
}

template <typename TInput, typename TCode>
size_t QuantizerStage<TInput, TCode>::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < sizeof(QuantizerConfig))
        throw std::runtime_error("Insufficient buffer for QuantizerConfig: need " +
                                 std::to_string(sizeof(QuantizerConfig)) + " bytes, got " + std::to_string(max_size));
    QuantizerConfig c;
    c.abs_error_bound = computed_abs_eb_;
    c.user_error_bound = config_.error_bound;
    c.value_base = computed_value_base_;
    c.quant_radius = (uint32_t)config_.quant_radius;
    c.num_elements = (uint32_t)num_elements_;
    c.outlier_count = actual_outlier_count_;
    c.input_type = DataType::FLOAT32;
    c.code_type = codeType();
    c.eb_mode = (uint8_t)config_.eb_mode;
    c.zigzag_codes = config_.zigzag_codes ? 1 : 0;
    c.outlier_threshold = config_.outlier_threshold;
    c.inplace_outliers = config_.inplace_outliers ? 1 : 0;
    std::memcpy(buf, &c, sizeof(c));
    return sizeof(c);
}

template <typename TInput, typename TCode>
void QuantizerStage<TInput, TCode>::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size < 28)  // the record before outlier_threshold / inplace_outliers existed
        throw std::runtime_error("QuantizerConfig header too small: got " + std::to_string(size) +
                                 " bytes, minimum is 28");
    QuantizerConfig c;
    std::memcpy(&c, buf, std::min(size, sizeof(c)));
    config_.error_bound = c.user_error_bound;
    config_.quant_radius = (int)c.quant_radius;
    config_.eb_mode = (ErrorBoundMode)c.eb_mode;
    config_.zigzag_codes = c.zigzag_codes != 0;
    num_elements_ = c.num_elements;
    actual_outlier_count_ = c.outlier_count;
    computed_abs_eb_ = c.abs_error_bound;
    computed_value_base_ = c.value_base;
    if (size >= sizeof(QuantizerConfig)) {
        config_.outlier_threshold = c.outlier_threshold;
        config_.inplace_outliers = c.inplace_outliers != 0;
    } else {
        config_.outlier_threshold = __builtin_inff();
        config_.inplace_outliers = false;
    }
}

template class QuantizerStage<float, uint16_t>;
template class QuantizerStage<float, uint32_t>;

// ---------------------------------------------------------------- Difference

template <typename T, typename TOut>
uint8_t DifferenceStage<T, TOut>::getOutputDataType(size_t) const {
    return (uint8_t)(is_inverse_ ? int_dtype<T>() : int_dtype<TOut>());
}

template <typename T, typename TOut>
uint8_t DifferenceStage<T, TOut>::getInputDataType(size_t) const {
    return (uint8_t)(is_inverse_ ? int_dtype<TOut>() : int_dtype<T>());
}

template <typename T, typename TOut>
void DifferenceStage<T, TOut>::execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                                       const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty())
        throw std::runtime_error("DifferenceStage: inputs, outputs, and sizes vectors must all be non-empty");
    const size_t n = sizes[0] / sizeof(T);
    const size_t chunk = chunk_size_ ? chunk_size_ / sizeof(T) : 0;
    actual_ = 0;
    if (n == 0) return;
    if (chunk & (chunk - 1)) throw std::runtime_error("DifferenceStage: chunk_elems must be a power-of-2");
    const int nb = std::is_same<T, TOut>::value ? 0 : 1;
    if (!is_inverse_) {
        check(fzb_diff(inputs[0], n, (int)sizeof(T), chunk, nb, 0, outputs[0], nullptr, 0, stream), "DifferenceStage");
    } else {
        void* w = ws_.ensure(fzb_scan_workspace_bytes(n, (int)sizeof(T)), pool, stream);
        check(fzb_diff(inputs[0], n, (int)sizeof(T), chunk, nb, 1, outputs[0], w, ws_.size(), stream),
              "DifferenceStage (inverse)");
    }
    actual_ = sizes[0];
}

template <typename T, typename TOut>
size_t DifferenceStage<T, TOut>::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < 6) return 0;
    buf[0] = (uint8_t)int_dtype<T>();
    buf[1] = (uint8_t)int_dtype<TOut>();
    const uint32_t cs = (uint32_t)chunk_size_;
    std::memcpy(buf + 2, &cs, 4);
    return 6;
}

template <typename T, typename TOut>
void DifferenceStage<T, TOut>::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size >= 6) {
        uint32_t cs = 0;
        std::memcpy(&cs, buf + 2, 4);
        chunk_size_ = cs;
    }
}

template class DifferenceStage<uint8_t>;
template class DifferenceStage<uint16_t>;
template class DifferenceStage<uint32_t>;
template class DifferenceStage<int32_t>;
template class DifferenceStage<int64_t>;
template class DifferenceStage<int8_t, uint8_t>;
template class DifferenceStage<int16_t, uint16_t>;
template class DifferenceStage<int32_t, uint32_t>;
template class DifferenceStage<int64_t, uint64_t>;

// ---------------------------------------------------------------- Lorenzo

template <typename T>
void LorenzoStage<T>::execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                              const std::vector<void*>& outputs, const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty())
        throw std::runtime_error("LorenzoStage: inputs, outputs, and sizes must be non-empty");
    actual_ = 0;
    const size_t n = sizes[0] / sizeof(T);
    if (n == 0) return;
    const uint64_t d[3] = {dims_[0] > 0 ? dims_[0] : n, dims_[1], dims_[2]};
    void* w = nullptr;
    size_t wn = 0;
    if (is_inverse_ && ndim() > 1) {
        w = ws_.ensure(fzb_scan_workspace_bytes(n, (int)sizeof(T)), pool, stream);
        wn = ws_.size();
    }
    check(fzb_lorenzo_int(inputs[0], d, n, (int)sizeof(T), is_inverse_ ? 1 : 0, outputs[0], w, wn, stream),
          "LorenzoStage");
    actual_ = sizes[0];
}

template <typename T>
size_t LorenzoStage<T>::serializeHeader(size_t, uint8_t* buf, size_t max_size) const {
    if (max_size < sizeof(LorenzoConfig)) throw std::runtime_error("LorenzoStage: header buffer too small");
    LorenzoConfig c;
    c.data_type = elemType();
    c.ndim = (uint8_t)ndim();
    c.dim_x = (uint32_t)dims_[0];
    c.dim_y = (uint32_t)dims_[1];
    c.dim_z = (uint32_t)dims_[2];
    std::memcpy(buf, &c, sizeof(c));
    return sizeof(c);
}

template <typename T>
void LorenzoStage<T>::deserializeHeader(const uint8_t* buf, size_t size) {
    if (size < sizeof(LorenzoConfig)) throw std::runtime_error("LorenzoStage: header too small");
    LorenzoConfig c;
    std::memcpy(&c, buf, sizeof(c));
    const int nd = c.ndim == 0 ? 1 : (int)c.ndim;
    dims_[0] = c.dim_x;
    dims_[1] = nd >= 2 ? c.dim_y : 1;
    dims_[2] = nd >= 3 ? c.dim_z : 1;
}

template class LorenzoStage<int8_t>;
template class LorenzoStage<int16_t>;
template class LorenzoStage<int32_t>;
template class LorenzoStage<int64_t>;

// ---------------------------------------------------------------- Zigzag / Negabinary

template <typename TIn, typename TOut, bool NEGABINARY>
void SignCodingStage<TIn, TOut, NEGABINARY>::execute(cudaStream_t stream, MemoryPool*,
                                                     const std::vector<void*>& inputs,
                                                     const std::vector<void*>& outputs,
                                                     const std::vector<size_t>& sizes) {
    if (inputs.empty() || outputs.empty() || sizes.empty())
        throw std::runtime_error(NEGABINARY ? "NegabinaryStage: invalid inputs/outputs"
                                            : "ZigzagStage: invalid inputs/outputs");
    actual_ = 0;
    const size_t n = sizes[0] / sizeof(TIn);
    if (n == 0) return;
    const int inv = is_inverse_ ? 1 : 0;
    if (NEGABINARY) check(fzb_negabinary(inputs[0], n, (int)sizeof(TIn), inv, outputs[0], stream), "NegabinaryStage");
    else check(fzb_zigzag(inputs[0], n, (int)sizeof(TIn), inv, outputs[0], stream), "ZigzagStage");
    actual_ = sizes[0];
}

template class SignCodingStage<int8_t, uint8_t, false>;
template class SignCodingStage<int16_t, uint16_t, false>;
template class SignCodingStage<int32_t, uint32_t, false>;
template class SignCodingStage<int64_t, uint64_t, false>;
template class SignCodingStage<int8_t, uint8_t, true>;
template class SignCodingStage<int16_t, uint16_t, true>;
template class SignCodingStage<int32_t, uint32_t, true>;
template class SignCodingStage<int64_t, uint64_t, true>;

// Factory cases for these stages (stage_factory.h:65-100, :134-183,
// :227-240); the Quantizer, absent from the reference's factory, is rebuilt
// from its 36-byte record.
Stage* createCodeStage(StageType type, const uint8_t* config, size_t config_size) {
    auto pair_of = [&](DataType& a, DataType& b) {
        a = config_size >= 1 ? (DataType)config[0] : DataType::INT32;
        b = config_size >= 2 ? (DataType)config[1] : DataType::UINT32;
    };
    DataType a, b;
    switch (type) {
        case StageType::QUANTIZER: {
            if (config_size < 28) throw std::runtime_error("QuantizerConfig header too small");
            QuantizerConfig c;
            std::memcpy(&c, config, std::min(config_size, sizeof(c)));
            if (c.input_type == DataType::FLOAT32 && c.code_type == DataType::UINT16) return new QuantizerStage<float, uint16_t>();
            if (c.input_type == DataType::FLOAT32 && c.code_type == DataType::UINT32) return new QuantizerStage<float, uint32_t>();
            throw std::runtime_error("Unsupported Quantizer type combination: input_type=" +
                                     std::to_string((int)c.input_type) + " code_type=" + std::to_string((int)c.code_type));
        }
        case StageType::DIFFERENCE: {
            pair_of(a, b);
            if (config_size >= 2) {
                if (a == DataType::INT8 && b == DataType::UINT8) return new DifferenceStage<int8_t, uint8_t>();
                if (a == DataType::INT16 && b == DataType::UINT16) return new DifferenceStage<int16_t, uint16_t>();
                if (a == DataType::INT32 && b == DataType::UINT32) return new DifferenceStage<int32_t, uint32_t>();
                if (a == DataType::INT64 && b == DataType::UINT64) return new DifferenceStage<int64_t, uint64_t>();
            }
            switch (a) {
                case DataType::UINT8: return new DifferenceStage<uint8_t>();
                case DataType::UINT16: return new DifferenceStage<uint16_t>();
                case DataType::UINT32: return new DifferenceStage<uint32_t>();
                case DataType::INT32: return new DifferenceStage<int32_t>();
                case DataType::INT64: return new DifferenceStage<int64_t>();
                default:
                    throw std::runtime_error("Unsupported Difference data type: " + std::to_string((int)a));
            }
        }
        case StageType::ZIGZAG:
        case StageType::NEGABINARY: {
            pair_of(a, b);
            const bool nb = type == StageType::NEGABINARY;
            if (a == DataType::INT8 && b == DataType::UINT8)
                return nb ? (Stage*)new NegabinaryStage<int8_t, uint8_t>() : new ZigzagStage<int8_t, uint8_t>();
            if (a == DataType::INT16 && b == DataType::UINT16)
                return nb ? (Stage*)new NegabinaryStage<int16_t, uint16_t>() : new ZigzagStage<int16_t, uint16_t>();
            if (a == DataType::INT32 && b == DataType::UINT32)
                return nb ? (Stage*)new NegabinaryStage<int32_t, uint32_t>() : new ZigzagStage<int32_t, uint32_t>();
            if (a == DataType::INT64 && b == DataType::UINT64)
                return nb ? (Stage*)new NegabinaryStage<int64_t, uint64_t>() : new ZigzagStage<int64_t, uint64_t>();
            throw std::runtime_error(std::string("Unsupported ") + (nb ? "NegabinaryStage" : "ZigzagStage") +
                                     " type pair: TIn=" + std::to_string((int)a) + " TOut=" + std::to_string((int)b));
        }
        case StageType::LORENZO: {
            const DataType dt = config_size >= sizeof(LorenzoConfig) ? (DataType)config[0] : DataType::INT32;
            switch (dt) {
                case DataType::INT8: return new LorenzoStage<int8_t>();
                case DataType::INT16: return new LorenzoStage<int16_t>();
                case DataType::INT32: return new LorenzoStage<int32_t>();
                case DataType::INT64: return new LorenzoStage<int64_t>();
                default: throw std::runtime_error("Unsupported LorenzoStage DataType: " + std::to_string((int)dt));
            }
        }
        default: return nullptr;
    }
}

}  // namespace fz
