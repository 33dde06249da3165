// fz/stage.h -- the stage plugin interface (the reference's fz::Stage,
// include/stage/stage.h:30-242): a stage turns device input buffers into
// device output buffers on a stream, reports its output sizes, and
// serialises the configuration its inverse needs into <= 128 bytes of the
// FZM container.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "fz/fzm_format.h"

namespace fz {

class MemoryPool;

class Stage {
public:
    virtual ~Stage() = default;

    // Enqueue the stage on `stream`.  sizes[i] is the byte size of inputs[i].
    virtual void execute(cudaStream_t stream, MemoryPool* pool, const std::vector<void*>& inputs,
                         const std::vector<void*>& outputs, const std::vector<size_t>& sizes) = 0;

    virtual std::string getName() const = 0;
    virtual size_t getNumInputs() const = 0;
    virtual size_t getNumOutputs() const = 0;
    // Input byte counts must be a multiple of this (the pipeline pads).
    virtual size_t getRequiredInputAlignment() const { return 1; }
    virtual std::vector<std::string> getOutputNames() const { return {"output"}; }
    int getOutputIndex(const std::string& name) const {
        const auto names = getOutputNames();
        for (size_t i = 0; i < names.size(); i++)
            if (names[i] == name) return (int)i;
        return -1;
    }

    // Upper bounds of the output byte sizes for the given input sizes.
    virtual std::vector<size_t> estimateOutputSizes(const std::vector<size_t>& input_sizes) const = 0;
    // Output sizes of the last execute() (may synchronise the stream).
    virtual std::unordered_map<std::string, size_t> getActualOutputSizesByName() const = 0;
    virtual size_t getActualOutputSize(int index) const {
        const auto names = getOutputNames();
        if (index < 0 || index >= (int)names.size()) return 0;
        const auto m = getActualOutputSizesByName();
        const auto it = m.find(names[index]);
        return it == m.end() ? 0 : it->second;
    }

    virtual void setInverse(bool inverse) { (void)inverse; }
    virtual bool isInverse() const { return false; }

    virtual uint16_t getStageTypeId() const = 0;
    virtual uint8_t getOutputDataType(size_t output_index) const = 0;
    virtual uint8_t getInputDataType(size_t /*input_index*/) const { return (uint8_t)DataType::UNKNOWN; }

    // Container metadata (<= FZM_STAGE_CONFIG_SIZE bytes).
    virtual size_t serializeHeader(size_t output_index, uint8_t* buf, size_t max_size) const {
        (void)output_index;
        (void)buf;
        (void)max_size;
        return 0;
    }
    virtual void deserializeHeader(const uint8_t* buf, size_t size) {
        (void)buf;
        (void)size;
    }
    virtual size_t getMaxHeaderSize(size_t /*output_index*/) const { return 0; }

    // Forward state kept across an inverse pass.
    virtual void saveState() {}
    virtual void restoreState() {}

    virtual void setDims(const std::array<size_t, 3>& dims) { (void)dims; }
    virtual void onFinalize(size_t /*estimated_inlen*/, MemoryPool* /*pool*/) {}
    virtual size_t estimateDeviceFootprintBytes(size_t /*inlen*/) const { return 0; }
    virtual size_t estimatePinnedFootprintBytes(size_t /*inlen*/) const { return 0; }
    // Called by the pipeline after the stream has been synchronised.
    virtual void postStreamSync(cudaStream_t stream) { (void)stream; }
    virtual bool isGraphCompatible() const { return true; }
    virtual size_t estimateScratchBytes(const std::vector<size_t>& /*input_sizes*/) const { return 0; }

    // The output size the producing DAG records for output `index` right
    // after execute(), before postStreamSync() refines it (LorenzoQuant
    // reports its outlier capacity there).  Defaults to the actual size.
    virtual size_t getExecuteTimeOutputSize(int index) const { return getActualOutputSize(index); }

    // The work enqueued by the last execute() ran again as part of a CUDA
    // graph replay: results that are read back after the sync are stale.
    virtual void onGraphReplay(cudaStream_t stream) { (void)stream; }
};

}  // namespace fz
