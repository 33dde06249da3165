// Test infrastructure shared by the reference shims: set every SM's shared
// memory to one byte value before a reference kernel runs.
//
// The reference's 3-D LorenzoQuant kernel (lorenzo_quant_nd.cu:214,246)
// takes its y difference as `delta -= (threadIdx.y > 0) * s[threadIdx.y][tx]`.
// Row 0 of `s` is a ghost row that is never written, so threads with
// threadIdx.y == 0 multiply whatever an earlier kernel left in that shared
// memory by 0.  When those bits are an infinity or a NaN the product is NaN:
// the cell becomes an outlier with code 0 and a NaN error, and decompresses
// to NaN.  Its output therefore depends on the previous kernels on the SM.
// With the ghost row reading zeros (the value the code multiplies away) its
// results are deterministic, so the parity shims scrub shared memory to zero
// first; the ghost-row test fills it with 0xFF to show the dependence.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ref_scrub {

__global__ void fill_shared_kernel(uint32_t words, uint32_t value) {
    extern __shared__ uint32_t s[];
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) s[i] = value;
    __syncthreads();
    // keep the stores: one thread reads a word back into a register sink
    if (threadIdx.x == 0 && s[words - 1] == 0x12345678u && value == 0x87654321u) s[0] = 0;
}

// Fills the dynamic shared memory of several maximum-size CTAs per SM with
// `byte`; returns the CUDA status.
inline cudaError_t fill_shared(uint8_t byte, cudaStream_t stream) {
    int dev = 0, sms = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const int bytes = optin & ~15;
    e = cudaFuncSetAttribute(fill_shared_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    const uint32_t v = 0x01010101u * byte;
    fill_shared_kernel<<<4 * sms, 1024, bytes, stream>>>((uint32_t)bytes / 4u, v);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e;
}

}  // namespace ref_scrub
