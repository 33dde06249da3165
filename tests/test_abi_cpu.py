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


def test_status_bits_and_gather_arguments():
    L = _lib.lib()
    rerun = C.c_int(-1)
    # bit 1 look-back timeout, 2 malformed, 4 inexact, 8 unsorted, 16 TMA timeout
    for bits, st, rr in [(0, 0, 0), (1, -6, 0), (2, -5, 0), (3, -5, 0), (4, 0, 1), (8, 0, 1), (16, -6, 0),
                         (6, -5, 1)]:
        assert L.fzb_status_from_bits(bits, C.byref(rerun)) == st
        assert rerun.value == rr
    assert L.fzb_status_from_bits(2, None) == -5
    # invalid gathers are refused on the host (no pointer is dereferenced)
    fake = 0x10000

    def gather(ptrs, nbytes, dst=fake):
        n = len(ptrs)
        return L.fzb_gather_words((C.c_void_p * n)(*ptrs), (C.c_uint32 * n)(*nbytes), (C.c_uint8 * n)(*([0] * n)),
                                  n, C.c_void_p(dst), None)
    assert gather([fake], [6]) == -1          # not a multiple of 4
    assert gather([fake], [260]) == -1        # above 256 bytes
    assert gather([fake + 2], [4]) == -1      # misaligned source
    assert gather([fake], [4], fake + 4) == -1  # destination not 8-byte aligned
    assert gather([fake] * 33, [4] * 33) == -1  # more than one launch takes
    assert L.fzb_concat_dev(None, None, None, None, None, None, 0, None, None) == -1


def test_huffman_host_codebook_matches_oracle_and_reference():
    """fzb_huff_book is host code: it runs here and must equal the oracle's
    and (when built) the reference's phf_CPU_build_canonized_codebook_v2."""
    import numpy as np
    from fzgpumodules_b200 import kernels as K
    from oracle import oracle as O
    rng = np.random.default_rng(7)
    cases = []
    for _ in range(60):
        bk = int(rng.choice([2, 3, 16, 256, 1024, 4096]))
        f = np.zeros(bk, np.uint32)
        k = int(rng.integers(1, bk + 1))
        pos = rng.choice(bk, k, replace=False)
        f[pos] = rng.geometric(rng.uniform(0.001, 0.5), k).astype(np.uint32) * \
            rng.integers(1, 1000, k).astype(np.uint32)
        cases.append((f, bk))
    fib = [1, 1]
    while len(fib) < 40:
        fib.append(fib[-1] + fib[-2])
    f = np.zeros(1024, np.uint32)
    f[:40] = fib  # tree deeper than 27: lengths truncated to 28
    cases.append((f, 1024))
    f = np.zeros(1024, np.uint32)
    f[7] = 100  # a single symbol
    cases.append((f, 1024))
    # ties everywhere: which equal-frequency node the heap pops decides the tree
    cases.append((np.full(1024, 5, np.uint32), 1024))
    cases.append((rng.integers(1, 4, 1024).astype(np.uint32), 1024))
    f = (np.exp(-0.012 * np.arange(1024)) * 1e5).astype(np.uint32)
    f[:4] *= 200  # C3-like: a few dominant symbols over a long geometric tail
    cases.append((f, 1024))
    for f, bk in cases:
        a = K.huff_book(f, bk)
        b = O.huff_book(f, bk)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        if O.ref_hfbook_available():
            c = O.ref_huff_book(f, bk)
            assert np.array_equal(a[0], c[0]) and np.array_equal(a[1], c[1])


def test_huffman_sizes_and_invalid():
    L = _lib.lib()
    assert L.fzb_huff_max_bytes(768, 1024) == 128 + 256 + 2048 + 8 + 4 * 769 + 16
    assert L.fzb_huff_workspace_bytes(0, 1024) == 0
    assert L.fzb_huff_workspace_bytes(1000, 0) == 0
    assert L.fzb_huff_workspace_bytes(10 ** 6, 1024) > 4 * 10 ** 6
    assert L.fzb_huff_compress(None, 10, 1024, None, None, None, 0, None) == -1
    assert L.fzb_huff_decode(None, 10, 10, 1024, None, None, 0, None) == -1
    assert L.fzb_status_string(-7) == b"input symbol outside [0, bklen)"
