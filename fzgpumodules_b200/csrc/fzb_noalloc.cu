// fzb_noalloc.cu -- RZE encode for callers that cannot allocate device memory.
//
// Some callers of this library have no way to obtain device memory for a
// workspace: a plugin invoked through a fixed-signature filter interface
// (an HDF5/NetCDF-style I/O filter or a database UDF handed only its input
// and output buffers), code running inside a stream capture that must not
// allocate, or a host callback that is not allowed to call allocation APIs.
// fzb_rze_encode_noalloc serves them: it runs the same kernels as
// fzb_rze_encode, but its scratch (per-chunk slots, size words and offsets)
// lives in one file-scope device array of fixed size, so the call itself
// allocates nothing.
//
// Limits and rules:
//   * at most kNoAllocMaxBytes input bytes per call (larger inputs are
//     rejected with FZB_E_CAPACITY);
//   * the array exists once per device and stays resident until the process
//     exits;
//   * every call on a device shares it, so calls whose GPU work overlaps
//     (on different streams, or from several host threads) race; serialise
//     them;
//   * the first call on each device resolves the array's device address
//     (cudaGetSymbolAddress with that device current) and caches it; make
//     that first call before any stream capture begins;
//   * the cached address belongs to the device's context: it does not
//     survive cudaDeviceReset, after which this entry point must not be
//     called again in the same process.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/fzb.h"
#include "fzb_kernels.cuh"

using namespace fzb;

namespace {

constexpr uint64_t kNoAllocMaxBytes = FZB_RZE_NOALLOC_MAX_BYTES;  // 8 MiB of input
constexpr uint32_t kNoAllocMaxChunks = kNoAllocMaxBytes / kChunkBytes;  // 512
// slots | size words | payload offsets
constexpr size_t kSlotBytes = (size_t)kNoAllocMaxChunks * kChunkBytes;
constexpr size_t kSizesOff = kSlotBytes;
constexpr size_t kPayOff = kSizesOff + 4 * (size_t)kNoAllocMaxChunks;
constexpr size_t kScratchBytes = kPayOff + 8 * (size_t)kNoAllocMaxChunks + 256;

__device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
uint8_t* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_mu;

// Device address of the scratch array on the current device (resolved once
// per device, with that device current).
int scratch_for_current_device(uint8_t** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FZB_E_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr)
            return FZB_E_CUDA;
        g_scratch_ptr[dev] = static_cast<uint8_t*>(p);
    }
    *out = g_scratch_ptr[dev];
    return FZB_OK;
}

}  // namespace

extern "C" int fzb_rze_encode_noalloc(const void* d_in, uint64_t bytes, void* d_out,
                                      uint64_t* d_out_size, void* stream) {
    if (!d_in || !d_out || !d_out_size || bytes == 0) return FZB_E_INVALID;
    if (bytes > kNoAllocMaxBytes) return FZB_E_CAPACITY;
    uint8_t* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t nch = (uint32_t)((bytes + kChunkBytes - 1) / kChunkBytes);
    // every slot, size word and offset a call reads is written by that call
    // first, so nothing needs clearing between calls
    RzeEncArgs a{};
    a.in = static_cast<const uint8_t*>(d_in);
    a.bytes = bytes;
    a.slots = scratch;
    a.sizes = reinterpret_cast<uint32_t*>(scratch + kSizesOff);
    const int smem = 2 * kChunkBytes + 16 + 2048 + 256 + 32;
    static SmemAttr attr;  // the shared-memory attribute, set once per device
    if (ensure_dyn_smem(attr, (const void*)rze_encode_kernel, smem) != cudaSuccess) return FZB_E_CUDA;
    rze_encode_kernel<<<nch, kThreads, smem, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    AsmArgs m{};
    m.slots = a.slots;
    m.sizes = a.sizes;
    m.n_chunks = nch;
    m.orig_bytes = (uint32_t)bytes;
    m.out = static_cast<uint8_t*>(d_out);
    m.out_size = reinterpret_cast<unsigned long long*>(d_out_size);
    m.pay_off = reinterpret_cast<unsigned long long*>(scratch + kPayOff);
    if (launch_assemble_scan(m, s) != 0) return FZB_E_CUDA;
    if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    assemble_copy_kernel<<<copy_grid(nch), 256, 0, s>>>(m);
    if (cudaGetLastError() != cudaSuccess) return FZB_E_CUDA;
    return FZB_OK;
}
