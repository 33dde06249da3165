"""fzb_rze_encode_noalloc: the RZE encoder for callers that cannot allocate
device memory (filter plugins handed only their buffers, code inside a
stream capture, host callbacks).  Checked through the C ABI against the
workspace-based fzb_rze_encode, exact to the byte, on consecutive calls.

Kept in the last-collected test file so a stop-at-first-failure run has
already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _lib():
    from fzgpumodules_b200 import _lib as L
    lib = L.lib()
    lib.fzb_rze_encode_noalloc.restype = C.c_int
    lib.fzb_rze_encode_noalloc.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def _data(n, seed):
    rng = np.random.default_rng(seed)
    d = np.zeros(n, np.uint8)
    d[: n // 3] = rng.integers(0, 256, n // 3, dtype=np.uint8)      # incompressible part
    pos = rng.choice(n, n // 50, replace=False)
    d[pos] = rng.integers(1, 256, pos.size, dtype=np.uint8)         # sparse part
    return d


def test_noalloc_encode_matches_workspace_encode(cuda):
    from fzgpumodules_b200 import kernels as K
    lib = _lib()
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    # a large call, then a smaller one: the second must not see stale bytes
    for call, n in enumerate([16384 * 300 + 77, 16384 * 37 + 1234]):
        d = torch.from_numpy(_data(n, 100 + call)).to(cuda)
        ref, ref_size = K.rze_encode(d)
        out = torch.zeros(int(lib.fzb_rze_max_bytes(n)), dtype=torch.uint8, device=cuda)
        size = torch.zeros(1, dtype=torch.int64, device=cuda)
        rc = lib.fzb_rze_encode_noalloc(C.c_void_p(d.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                        C.c_void_p(size.data_ptr()), stream)
        assert rc == 0
        torch.cuda.synchronize()
        k = int(size.item())
        assert k == int(ref_size.item())
        assert torch.equal(out[:k], ref)


def test_noalloc_encode_rejects_oversize(cuda):
    lib = _lib()
    limit = 8 << 20
    d = torch.zeros(16, dtype=torch.uint8, device=cuda)
    size = torch.zeros(1, dtype=torch.int64, device=cuda)
    # the size check happens on the host before anything touches the device
    rc = lib.fzb_rze_encode_noalloc(C.c_void_p(d.data_ptr()), limit + 1, C.c_void_p(d.data_ptr()),
                                    C.c_void_p(size.data_ptr()), None)
    assert rc == -4  # FZB_E_CAPACITY
