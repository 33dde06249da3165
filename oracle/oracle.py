"""ctypes binding of the CPU oracle (liboracle.so) and the reference-built
checkers under oracle/_ref.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference leg, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HFBOOK = os.path.join(HERE, "_ref", "libref_hfbook.so")
REF_STAGES = os.path.join(HERE, "_ref", "libfzref.so")

ABS, REL, NOA = 0, 1, 2

_lib = None


def build() -> None:
    """Compile liboracle.so (gcc) if it is missing or stale."""
    src = os.path.join(HERE, "fzoracle.c")
    if (not os.path.exists(LIB_PATH)
            or os.path.getmtime(LIB_PATH) < os.path.getmtime(src)):
        subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        p, sz, u32, i32, f32 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_int, C.c_float
        L.orc_round_half_away.restype = f32
        L.orc_round_half_away.argtypes = [f32]
        L.orc_value_base.restype = f32
        L.orc_value_base.argtypes = [p, sz, i32]
        L.orc_resolve_eb.argtypes = [f32, i32, f32, p, p, p]
        L.orc_lq_fwd.restype = u32
        L.orc_lq_fwd.argtypes = [p, sz, u32, u32, u32, i32, f32, u32, i32, p, p, p, sz]
        L.orc_lq_inv.argtypes = [p, sz, p, p, u32, u32, u32, u32, i32, f32, i32, p]
        L.orc_bitshuffle.argtypes = [p, sz, u32, i32, i32, p]
        L.orc_rze_max_bytes.restype = sz
        L.orc_rze_max_bytes.argtypes = [sz]
        L.orc_rze_encode.restype = sz
        L.orc_rze_encode.argtypes = [p, sz, p]
        L.orc_rze_decode.restype = sz
        L.orc_rze_decode.argtypes = [p, sz, p, sz]
        L.orc_rle_max_bytes.restype = sz
        L.orc_rle_max_bytes.argtypes = [sz, i32]
        L.orc_rle_encode.restype = sz
        L.orc_rle_encode.argtypes = [p, sz, i32, p]
        L.orc_rle_decode.restype = sz
        L.orc_rle_decode.argtypes = [p, sz, i32, p, sz]
        L.orc_bitpack_nbits_for_max.restype = i32
        L.orc_bitpack_nbits_for_max.argtypes = [u32, i32]
        L.orc_bitpack_encode.restype = sz
        L.orc_bitpack_encode.argtypes = [p, sz, i32, i32, p]
        L.orc_bitpack_decode.argtypes = [p, sz, i32, i32, p]
        L.orc_histogram.restype = C.c_uint64
        L.orc_histogram.argtypes = [p, sz, u32, p]
        L.orc_huff_book.restype = i32
        L.orc_huff_book.argtypes = [p, u32, p, p]
        L.orc_huff_revbook_bytes.restype = sz
        L.orc_huff_revbook_bytes.argtypes = [u32]
        L.orc_huff_max_bytes.restype = sz
        L.orc_huff_max_bytes.argtypes = [sz, u32]
        L.orc_huff_encode.restype = sz
        L.orc_huff_encode.argtypes = [p, sz, u32, p, p, p]
        L.orc_huff_encode_sub.restype = sz
        L.orc_huff_encode_sub.argtypes = [p, sz, u32, p, p, u32, p]
        L.orc_huff_decode.restype = sz
        L.orc_huff_decode.argtypes = [p, sz, p, sz]
        L.orc_crc32.restype = u32
        L.orc_crc32.argtypes = [p, sz]
        L.orc_zigzag.argtypes = [p, sz, i32, i32, p]
        L.orc_negabinary.argtypes = [p, sz, i32, i32, p]
        L.orc_diff.argtypes = [p, sz, i32, sz, i32, i32, p]
        L.orc_lorenzo_int.argtypes = [p, sz, sz, sz, sz, i32, i32, p]
        L.orc_quantizer_abs.restype = sz
        L.orc_quantizer_abs.argtypes = [p, sz, i32, f32, f32, u32, i32, p, p, p, sz]
        L.orc_quantizer_abs_inv.argtypes = [p, sz, i32, f32, i32, p, p, sz, p]
        L.orc_quantizer_inplace.argtypes = [p, sz, f32, f32, u32, p]
        L.orc_quantizer_inplace_inv.argtypes = [p, sz, f32, u32, p]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- Lorenzo

def value_base(x: np.ndarray, mode: int) -> float:
    x = np.ascontiguousarray(x, dtype=np.float32)
    return float(np.float32(lib().orc_value_base(_p(x), x.size, mode)))


def resolve_eb(user_eb: float, mode: int, value_base: float):
    """(abs_eb, ebx2_r, ebx2) as float32, as the reference host computes them."""
    a, r, e = C.c_float(), C.c_float(), C.c_float()
    lib().orc_resolve_eb(user_eb, mode, value_base, C.byref(a), C.byref(r), C.byref(e))
    return np.float32(a.value), np.float32(r.value), np.float32(e.value)


def lq_fwd(x: np.ndarray, dims, ebx2_r: float, radius: int = 32768,
           zigzag: bool = False, cap: int | None = None, n_total: int | None = None):
    """Returns (codes u16[n_total], err f32[k], idx u32[k], total_count)."""
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    nx, ny, nz = (list(dims) + [1, 1])[:3]
    ndim = 3 if nz > 1 else (2 if ny > 1 else 1)
    n_total = x.size if n_total is None else n_total
    if cap is None:
        cap = n_total
    codes = np.empty(n_total, np.uint16)
    err = np.empty(max(cap, 1), np.float32)
    idx = np.empty(max(cap, 1), np.uint32)
    cnt = lib().orc_lq_fwd(_p(x), n_total, nx, ny, nz, ndim, ebx2_r, radius,
                           int(zigzag), _p(codes), _p(err), _p(idx), cap)
    k = min(cnt, cap)
    return codes, err[:k].copy(), idx[:k].copy(), int(cnt)


def lq_inv(codes, err, idx, dims, ebx2: float, zigzag: bool = False):
    codes = np.ascontiguousarray(codes, dtype=np.uint16)
    err = np.ascontiguousarray(err, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    nx, ny, nz = (list(dims) + [1, 1])[:3]
    ndim = 3 if nz > 1 else (2 if ny > 1 else 1)
    out = np.empty(codes.size, np.float32)
    lib().orc_lq_inv(_p(codes), codes.size, _p(err), _p(idx), idx.size, nx, ny, nz,
                     ndim, ebx2, int(zigzag), _p(out))
    return out


# ---------------------------------------------------------------- lossless

def bitshuffle(data: np.ndarray, block: int = 16384, ew: int = 2, inverse: bool = False):
    b = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    out = np.empty_like(b)
    lib().orc_bitshuffle(_p(b), b.size, block, ew, int(inverse), _p(out))
    return out


def rze_encode(data: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    out = np.empty(lib().orc_rze_max_bytes(b.size), np.uint8)
    n = lib().orc_rze_encode(_p(b), b.size, _p(out))
    return out[:n].copy()


def rze_decode(stream: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(stream, dtype=np.uint8)
    if s.size < 8:
        raise ValueError("RZE stream too short")
    orig = int(s[:4].view(np.uint32)[0])
    out = np.empty(max(orig, 1), np.uint8)
    n = lib().orc_rze_decode(_p(s), s.size, _p(out), orig)
    if n == ctypes_size_max():
        raise ValueError("malformed RZE stream")
    return out[:n].copy()


def ctypes_size_max() -> int:
    return (1 << (8 * C.sizeof(C.c_size_t))) - 1


def rle_encode(data: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(data)
    out = np.empty(lib().orc_rle_max_bytes(d.size, d.itemsize), np.uint8)
    n = lib().orc_rle_encode(_p(d), d.size, d.itemsize, _p(out))
    return out[:n].copy()


def rle_decode(stream: np.ndarray, n: int, dtype=np.uint16) -> np.ndarray:
    s = np.ascontiguousarray(stream, dtype=np.uint8)
    out = np.empty(max(n, 1), dtype)
    k = lib().orc_rle_decode(_p(s), s.size, np.dtype(dtype).itemsize, _p(out), n)
    if k == ctypes_size_max():
        raise ValueError("malformed RLE stream")
    return out[:k].copy()


def bitpack_nbits(max_val: int, elem: int) -> int:
    return lib().orc_bitpack_nbits_for_max(max_val, elem)


def bitpack_encode(data: np.ndarray, nbits: int) -> np.ndarray:
    d = np.ascontiguousarray(data)
    out = np.empty((d.size * nbits + 7) // 8, np.uint8)
    lib().orc_bitpack_encode(_p(d), d.size, d.itemsize, nbits, _p(out))
    return out


def bitpack_decode(packed: np.ndarray, n: int, nbits: int, dtype=np.uint16) -> np.ndarray:
    s = np.ascontiguousarray(packed, dtype=np.uint8)
    out = np.empty(n, dtype)
    lib().orc_bitpack_decode(_p(s), n, np.dtype(dtype).itemsize, nbits, _p(out))
    return out


def histogram(codes: np.ndarray, bklen: int = 1024):
    c = np.ascontiguousarray(codes, dtype=np.uint16)
    f = np.empty(bklen, np.uint32)
    counted = lib().orc_histogram(_p(c), c.size, bklen, _p(f))
    return f, int(counted)


def huff_book(freq: np.ndarray, bklen: int = 1024):
    f = np.ascontiguousarray(freq, dtype=np.uint32)
    bk4 = np.empty(bklen, np.uint32)
    rb = np.zeros(lib().orc_huff_revbook_bytes(bklen), np.uint8)
    rc = lib().orc_huff_book(_p(f), bklen, _p(bk4), _p(rb))
    if rc != 0:
        raise RuntimeError("Huffman tree deeper than the 58-level traversal stack")
    return bk4, rb


def huff_encode(codes: np.ndarray, bklen: int, bk4: np.ndarray, revbook: np.ndarray, sublen: int = 768):
    """PHF blob; sublen 768 is coarse mode, 1024 fine mode (hf_buf.cc:46-49)."""
    c = np.ascontiguousarray(codes, dtype=np.uint16)
    out = np.zeros(lib().orc_huff_max_bytes(c.size, bklen), np.uint8)
    n = lib().orc_huff_encode_sub(_p(c), c.size, bklen, _p(bk4), _p(revbook), sublen, _p(out))
    return out[:n].copy()


def huff_decode(blob: np.ndarray, n: int) -> np.ndarray:
    b = np.ascontiguousarray(blob, dtype=np.uint8)
    out = np.zeros(max(n, 1), np.uint16)
    k = lib().orc_huff_decode(_p(b), b.size, _p(out), n)
    return out[:k].copy()


def crc32(data) -> int:
    b = np.ascontiguousarray(np.frombuffer(bytes(data), np.uint8) if isinstance(data, (bytes, bytearray)) else data).view(np.uint8).reshape(-1)
    return int(lib().orc_crc32(_p(b), b.size))


def _uview(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a).reshape(-1)
    return a.view({1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[a.itemsize])


def zigzag(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    """Zigzag on the element bit patterns; returns the unsigned view."""
    u = _uview(a)
    out = np.empty_like(u)
    lib().orc_zigzag(_p(u), u.size, u.itemsize, int(inverse), _p(out))
    return out


def negabinary(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    u = _uview(a)
    out = np.empty_like(u)
    lib().orc_negabinary(_p(u), u.size, u.itemsize, int(inverse), _p(out))
    return out


def diff(a: np.ndarray, chunk_elems: int = 0, negabinary: bool = False, inverse: bool = False) -> np.ndarray:
    u = _uview(a)
    out = np.empty_like(u)
    lib().orc_diff(_p(u), u.size, u.itemsize, chunk_elems, int(negabinary), int(inverse), _p(out))
    return out


def lorenzo_int(a: np.ndarray, dims, inverse: bool = False) -> np.ndarray:
    """dims = (x, y, z); 1-D when y = z = 1 (blocks of 256 over all n)."""
    u = _uview(a)
    out = np.empty_like(u)
    nx, ny, nz = (int(v) for v in dims)
    lib().orc_lorenzo_int(_p(u), u.size, nx, ny, nz, u.itemsize, int(inverse), _p(out))
    return out


def quantizer_abs(x: np.ndarray, code_bytes: int, ebx2_r, radius: int, zigzag: bool, cap: int,
                  threshold: float = float("inf")):
    """Returns (codes, outlier values, outlier indices, total outliers)."""
    xs = np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    codes = np.empty(xs.size, np.uint16 if code_bytes == 2 else np.uint32)
    vals = np.zeros(max(cap, 1), np.float32)
    idx = np.zeros(max(cap, 1), np.uint32)
    k = lib().orc_quantizer_abs(_p(xs), xs.size, code_bytes, np.float32(ebx2_r), np.float32(threshold), radius,
                                int(zigzag), _p(codes), _p(vals), _p(idx), cap)
    m = min(k, cap)
    return codes, vals[:m].copy(), idx[:m].copy(), int(k)


def quantizer_abs_inv(codes: np.ndarray, ebx2, zigzag: bool, vals: np.ndarray, idx: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(codes).reshape(-1)
    v = np.ascontiguousarray(vals, dtype=np.float32)
    ix = np.ascontiguousarray(idx, dtype=np.uint32)
    out = np.empty(c.size, np.float32)
    lib().orc_quantizer_abs_inv(_p(c), c.size, c.itemsize, np.float32(ebx2), int(zigzag), _p(v), _p(ix), v.size,
                                _p(out))
    return out


def quantizer_inplace(x: np.ndarray, ebx2_r, radius: int, threshold: float = float("inf")) -> np.ndarray:
    xs = np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    codes = np.empty(xs.size, np.uint32)
    lib().orc_quantizer_inplace(_p(xs), xs.size, np.float32(ebx2_r), np.float32(threshold), radius, _p(codes))
    return codes


def quantizer_inplace_inv(codes: np.ndarray, ebx2, radius: int) -> np.ndarray:
    c = np.ascontiguousarray(codes, dtype=np.uint32).reshape(-1)
    out = np.empty(c.size, np.float32)
    lib().orc_quantizer_inplace_inv(_p(c), c.size, np.float32(ebx2), radius, _p(out))
    return out


# ---------------------------------------------------------------- reference builds

_ref_hf = None


def ref_hfbook_available() -> bool:
    return os.path.exists(REF_HFBOOK)


def ref_huff_book(freq: np.ndarray, bklen: int = 1024):
    """The reference's own host codebook builder (built from its sources)."""
    global _ref_hf
    if _ref_hf is None:
        _ref_hf = C.CDLL(REF_HFBOOK)
        _ref_hf.ref_huff_book.restype = C.c_int
        _ref_hf.ref_huff_book.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    f = np.ascontiguousarray(freq, dtype=np.uint32)
    bk4 = np.empty(bklen, np.uint32)
    rb = np.zeros(4 * 64 + 2 * bklen, np.uint8)
    rc = _ref_hf.ref_huff_book(_p(f), bklen, _p(bk4), _p(rb))
    if rc != 0:
        raise RuntimeError("reference codebook builder failed")
    return bk4, rb
