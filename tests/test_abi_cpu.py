"""The C-ABI library loads and exports every symbol include/fzb.h declares
(no device calls)."""
import ctypes as C

from fzgpumodules_b200 import _lib


def test_header_symbols_exported():
    L = _lib.lib()
    syms = _lib.header_symbols()
    assert len(syms) >= 10
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_host_only_queries():
    L = _lib.lib()
    assert L.fzb_version() >= 100
    assert L.fzb_status_string(0) == b"ok"
    assert b"workspace" in L.fzb_status_string(-3)
    a, b = L.fzb_workspace_bytes(1 << 20, 0), L.fzb_workspace_bytes(1 << 27, 1 << 20)
    assert 0 < a < b
    # header + per-chunk sizes + payload bound + pad
    assert L.fzb_rze_max_bytes(16384) == 8 + 4 + 16384 + 4


def test_invalid_arguments_rejected_before_launch():
    L = _lib.lib()
    dims = (C.c_uint32 * 3)(4, 4, 4)
    # null input / zero size are rejected on the host, nothing is enqueued
    rc = L.fzb_lq_forward(None, 64, dims, 1e-3, 0, 0.0, 512, 0, None, None, None, 0, None, None,
                          None, 0, None)
    assert rc == -1
    rc = L.fzb_bitshuffle(None, 100, 16384, 2, 0, None, None)
    assert rc == -1
    rc = L.fzb_rze_encode(None, 0, None, None, None, 0, None)
    assert rc == -1
