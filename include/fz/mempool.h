// fz/mempool.h -- device memory for pipelines (the reference's MemoryPool,
// include/mem/mempool.h:30-228): a stream-ordered CUDA memory pool sized
// from the input (input bytes x multiplier), falling back to plain
// cudaMalloc where pools are unavailable or FZ_FORCE_MEMPOOL_FALLBACK is set.
// Not thread-safe: one host thread per pipeline.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <string>
#include <unordered_map>
#include <vector>

namespace fz {

struct MemoryPoolConfig {
    size_t input_data_size;
    float pool_size_multiplier;
    int device_id;
    bool enable_reuse;
    bool force_fallback;
    MemoryPoolConfig(size_t input_size = 0, float multiplier = 3.0f, int device = 0, bool reuse = true,
                     bool fallback = false)
        : input_data_size(input_size), pool_size_multiplier(multiplier), device_id(device),
          enable_reuse(reuse), force_fallback(fallback) {}
    // 1 GiB when no size hint was given.
    size_t getPoolSize() const {
        return input_data_size ? (size_t)((double)input_data_size * pool_size_multiplier) : (size_t)1 << 30;
    }
};

class MemoryPool {
public:
    explicit MemoryPool(const MemoryPoolConfig& config = MemoryPoolConfig());
    ~MemoryPool();
    MemoryPool(const MemoryPool&) = delete;
    MemoryPool& operator=(const MemoryPool&) = delete;

    // Stream-ordered allocation; nullptr on failure.
    void* allocate(size_t size, cudaStream_t stream, const std::string& tag = "", bool persistent = false);
    void free(void* ptr, cudaStream_t stream);
    void* allocatePersistentDevice(size_t bytes, const std::string& tag = "");
    void* allocatePersistentPinned(size_t bytes, const std::string& tag = "");
    void freePersistentDevice(void* ptr);
    void freePersistentPinned(void* ptr);
    void setReleaseThreshold(size_t bytes);
    void synchronize(cudaStream_t stream);
    void trim();

    size_t getCurrentUsage() const { return current_; }
    size_t getPeakUsage() const { return peak_; }
    size_t getAllocationCount() const { return live_.size(); }
    size_t getConfiguredSize() const { return config_.getPoolSize(); }
    size_t getPersistentDeviceBytes() const { return persistent_device_bytes_; }
    size_t getPersistentPinnedBytes() const { return persistent_pinned_bytes_; }
    bool isFallbackMode() const { return pool_ == nullptr; }
    int getDeviceId() const { return config_.device_id; }
    cudaMemPool_t getMemPool() const { return pool_; }

private:
    struct Live {
        size_t bytes;
        std::string tag;
        bool persistent;
    };
    MemoryPoolConfig config_;
    cudaMemPool_t pool_ = nullptr;
    std::unordered_map<void*, Live> live_;
    std::unordered_map<void*, size_t> persistent_dev_, persistent_pin_;
    size_t current_ = 0, peak_ = 0;
    size_t persistent_device_bytes_ = 0, persistent_pinned_bytes_ = 0;
};

}  // namespace fz
