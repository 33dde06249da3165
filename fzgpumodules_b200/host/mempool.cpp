// mempool.cpp -- stream-ordered device memory for pipelines: one CUDA
// memory pool per MemoryPool (release threshold pinned high so freed pages
// stay mapped between calls), or cudaMalloc/cudaFree in fallback mode.
#include "fz/mempool.h"

#include <cstdint>
#include <cstdlib>
#include <limits>

namespace fz {

MemoryPool::MemoryPool(const MemoryPoolConfig& config) : config_(config) {
    const char* force = std::getenv("FZ_FORCE_MEMPOOL_FALLBACK");
    if (config_.force_fallback || (force && force[0] && force[0] != '0')) return;
    int supported = 0;
    if (cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, config_.device_id) != cudaSuccess ||
        !supported) {
        cudaGetLastError();
        return;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = config_.device_id;
    if (cudaMemPoolCreate(&pool_, &props) != cudaSuccess) {
        cudaGetLastError();
        pool_ = nullptr;
        return;
    }
    uint64_t threshold = std::numeric_limits<uint64_t>::max();
    cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &threshold);
}

MemoryPool::~MemoryPool() {
    cudaDeviceSynchronize();
    for (auto& kv : live_) {
        if (pool_) cudaFreeAsync(kv.first, 0);
        else cudaFree(kv.first);
    }
    live_.clear();
    for (auto& kv : persistent_dev_) cudaFree(kv.first);
    for (auto& kv : persistent_pin_) cudaFreeHost(kv.first);
    if (pool_) {
        cudaDeviceSynchronize();
        cudaMemPoolDestroy(pool_);
    }
}

void* MemoryPool::allocate(size_t size, cudaStream_t stream, const std::string& tag, bool persistent) {
    if (size == 0) return nullptr;
    void* p = nullptr;
    cudaError_t e = pool_ ? cudaMallocFromPoolAsync(&p, size, pool_, stream) : cudaMalloc(&p, size);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    live_[p] = {size, tag, persistent};
    current_ += size;
    if (current_ > peak_) peak_ = current_;
    return p;
}

void MemoryPool::free(void* ptr, cudaStream_t stream) {
    if (!ptr) return;
    auto it = live_.find(ptr);
    if (it == live_.end()) return;
    current_ -= it->second.bytes;
    live_.erase(it);
    if (pool_) cudaFreeAsync(ptr, stream);
    else {
        cudaStreamSynchronize(stream);
        cudaFree(ptr);
    }
}

void* MemoryPool::allocatePersistentDevice(size_t bytes, const std::string&) {
    void* p = nullptr;
    if (!bytes || cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    persistent_dev_[p] = bytes;
    persistent_device_bytes_ += bytes;
    return p;
}

void* MemoryPool::allocatePersistentPinned(size_t bytes, const std::string&) {
    void* p = nullptr;
    if (!bytes || cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    persistent_pin_[p] = bytes;
    persistent_pinned_bytes_ += bytes;
    return p;
}

void MemoryPool::freePersistentDevice(void* ptr) {
    auto it = persistent_dev_.find(ptr);
    if (it == persistent_dev_.end()) return;
    persistent_device_bytes_ -= it->second;
    persistent_dev_.erase(it);
    cudaFree(ptr);
}

void MemoryPool::freePersistentPinned(void* ptr) {
    auto it = persistent_pin_.find(ptr);
    if (it == persistent_pin_.end()) return;
    persistent_pinned_bytes_ -= it->second;
    persistent_pin_.erase(it);
    cudaFreeHost(ptr);
}

void MemoryPool::setReleaseThreshold(size_t bytes) {
    if (!pool_) return;
    uint64_t t = bytes;
    cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &t);
}

void MemoryPool::synchronize(cudaStream_t stream) { cudaStreamSynchronize(stream); }

void MemoryPool::trim() {
    if (pool_) cudaMemPoolTrimTo(pool_, 0);
}

}  // namespace fz
