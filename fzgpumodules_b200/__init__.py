"""fzgpumodules_b200 -- B200 (sm_100a) rebuild of the FZGPUModules hot path.

The product is libfzb.so (CUDA kernels behind the C ABI in include/fzb.h).
This package loads it (``_lib``), exposes thin calls over torch device
tensors (``kernels``) and seeded synthetic fields (``fields``).
"""
__all__ = ["kernels", "fields"]
