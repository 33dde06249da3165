"""Thin Python calls into the C ABI (include/fzb.h) on torch CUDA tensors.

torch supplies device memory and the current stream; every byte of stage
math runs in libfzb.so.  Each function mirrors one reference stage
``execute`` (cited beside it) and returns torch tensors on the same device.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from ._lib import FzbError, check, lib

ABS, REL, NOA = 0, 1, 2
NO_SYNC, FORCE_EXACT = 1, 2
CHUNK_CODES = 8192
CHUNK_BYTES = 16384


def _ptr(t: torch.Tensor | None):
    return C.c_void_p(t.data_ptr()) if t is not None else None


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def _stream(device=None):
    """The current stream's handle (without building a Stream object when
    torch offers the raw accessor)."""
    if _raw_stream is not None:
        if isinstance(device, str):
            device = torch.device(device)
        idx = device.index if isinstance(device, torch.device) else device
        return C.c_void_p(_raw_stream(torch.cuda.current_device() if idx is None else int(idx)))
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _dims(dims) -> C.Array:
    d = list(dims) + [1, 1, 1]
    return (C.c_uint32 * 3)(int(d[0]), int(d[1]), int(d[2]))


class Workspace:
    """Reusable device workspace sized with fzb_workspace_bytes()."""

    def __init__(self):
        self.buf: torch.Tensor | None = None

    def get(self, n_total: int, device, cap: int = 0) -> tuple[C.c_void_p, int]:
        need = int(lib().fzb_workspace_bytes(int(n_total), int(cap)))
        if self.buf is None or self.buf.numel() < need or self.buf.device != torch.device(device):
            self.buf = torch.empty(need, dtype=torch.uint8, device=device)
        return _ptr(self.buf), self.buf.numel()

    def get_bytes(self, need: int, device) -> tuple[C.c_void_p, int]:
        """Workspace of at least `need` bytes (for the Huffman entry points)."""
        need = max(int(need), 256)
        if self.buf is None or self.buf.numel() < need or self.buf.device != torch.device(device):
            self.buf = torch.empty(need, dtype=torch.uint8, device=device)
        return _ptr(self.buf), self.buf.numel()

    def status(self) -> int:
        if self.buf is None:
            return 0
        return int(lib().fzb_workspace_status(_ptr(self.buf), _stream(self.buf.device)))


_default_ws = Workspace()


def max_outliers(n: int, capacity: float) -> int:
    """LorenzoQuantStage::getMaxOutlierCount (lorenzo_quant.h:333-335):
    ceil(n * capacity) evaluated in single precision."""
    import numpy as np
    return int(math.ceil(float(np.float32(n) * np.float32(capacity))))


def lq_forward(x: torch.Tensor, dims, eb: float, mode: int = ABS, radius: int = 32768,
               zigzag: bool = False, outlier_capacity: float = 0.2, value_base: float = 0.0,
               ws: Workspace | None = None):
    """LorenzoQuantStage<float,uint16_t> forward (lorenzo_quant.cu:583-719)."""
    ws = ws or _default_ws
    n = x.numel()
    cap = max_outliers(n, outlier_capacity)
    dev = x.device
    codes = torch.empty(n, dtype=torch.uint16, device=dev)
    err = torch.empty(max(cap, 1), dtype=torch.float32, device=dev)
    idx = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    eb_state = torch.zeros(4, dtype=torch.float32, device=dev)
    wp, wn = ws.get(n, dev, cap)
    check(lib().fzb_lq_forward(_ptr(x), n, _dims(dims), eb, mode, value_base, radius, int(zigzag),
                               _ptr(codes), _ptr(err), _ptr(idx), cap, _ptr(count), _ptr(eb_state),
                               wp, wn, _stream(dev)), "fzb_lq_forward")
    return dict(codes=codes, err=err, idx=idx, count=count, eb_state=eb_state, cap=cap)


def lq_inverse(codes, err, idx, count, cap: int, dims, abs_eb: float, zigzag: bool = False,
               ws: Workspace | None = None):
    """LorenzoQuantStage inverse (lorenzo_quant.cu:494-581)."""
    ws = ws or _default_ws
    n = codes.numel()
    dev = codes.device
    out = torch.empty(n, dtype=torch.float32, device=dev)
    wp, wn = ws.get(n, dev)
    check(lib().fzb_lq_inverse(_ptr(codes), _ptr(err), _ptr(idx), _ptr(count), cap, n, _dims(dims),
                               abs_eb, int(zigzag), _ptr(out), wp, wn, _stream(dev)), "fzb_lq_inverse")
    return out


def bitshuffle(data: torch.Tensor, block: int = CHUNK_BYTES, ew: int = 2, inverse: bool = False):
    """BitshuffleStage::execute (bitshuffle_stage.cu:355-475)."""
    src = data.view(torch.uint8).reshape(-1)
    out = torch.empty_like(src)
    check(lib().fzb_bitshuffle(_ptr(src), src.numel(), block, ew, int(inverse), _ptr(out),
                               _stream(src.device)), "fzb_bitshuffle")
    return out


def rze_encode(data: torch.Tensor, ws: Workspace | None = None, trim: bool = True):
    """RZEStage forward (rze_stage.cu:774-843).  Returns (stream, size_tensor)."""
    ws = ws or _default_ws
    src = data.view(torch.uint8).reshape(-1)
    nb = src.numel()
    out = torch.empty(int(lib().fzb_rze_max_bytes(nb)), dtype=torch.uint8, device=src.device)
    size = torch.zeros(1, dtype=torch.int64, device=src.device)
    wp, wn = ws.get((nb + 1) // 2, src.device)
    check(lib().fzb_rze_encode(_ptr(src), nb, _ptr(out), _ptr(size), wp, wn, _stream(src.device)),
          "fzb_rze_encode")
    if trim:
        return out[: int(size.item())], size
    return out, size


def rze_decode(stream: torch.Tensor, orig_bytes: int, ws: Workspace | None = None):
    """RZEStage inverse (rze_stage.cu:846-994)."""
    ws = ws or _default_ws
    src = stream.view(torch.uint8).reshape(-1)
    out = torch.empty(orig_bytes, dtype=torch.uint8, device=src.device)
    wp, wn = ws.get((orig_bytes + 1) // 2, src.device)
    check(lib().fzb_rze_decode(_ptr(src), src.numel(), orig_bytes, _ptr(out), wp, wn,
                               _stream(src.device)), "fzb_rze_decode")
    return out


def lq_bs_rze_compress(x: torch.Tensor, dims, eb: float, mode: int = ABS, radius: int = 32768,
                       zigzag: bool = False, outlier_capacity: float = 0.2,
                       value_base: float = 0.0, ws: Workspace | None = None, out=None):
    """Fused LorenzoQuant -> Bitshuffle -> RZE.  Returns a dict of device
    tensors (rze stream at capacity, rze_size, outlier buffers, eb_state)."""
    ws = ws or _default_ws
    n = x.numel()
    cap = max_outliers(n, outlier_capacity)
    dev = x.device
    if out is None:
        out = dict(
            rze=torch.empty(int(lib().fzb_rze_max_bytes(2 * n)), dtype=torch.uint8, device=dev),
            rze_size=torch.zeros(1, dtype=torch.int64, device=dev),
            err=torch.empty(max(cap, 1), dtype=torch.float32, device=dev),
            idx=torch.empty(max(cap, 1), dtype=torch.int32, device=dev),
            count=torch.zeros(1, dtype=torch.int32, device=dev),
            eb_state=torch.zeros(4, dtype=torch.float32, device=dev),
            cap=cap)
    wp, wn = ws.get(n, dev, cap)
    check(lib().fzb_lq_bs_rze_compress(
        _ptr(x), n, _dims(dims), eb, mode, value_base, radius, int(zigzag), _ptr(out["err"]),
        _ptr(out["idx"]), cap, _ptr(out["count"]), _ptr(out["rze"]), _ptr(out["rze_size"]),
        _ptr(out["eb_state"]), wp, wn, _stream(dev)), "fzb_lq_bs_rze_compress")
    return out


def lq_bs_rze_decompress(rze: torch.Tensor, rze_bytes: int, err, idx, count, cap: int, n: int,
                         dims, abs_eb: float, zigzag: bool = False, flags: int = 0,
                         ws: Workspace | None = None, out=None):
    ws = ws or _default_ws
    dev = rze.device
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device=dev)
    wp, wn = ws.get(n, dev)
    check(lib().fzb_lq_bs_rze_decompress(
        _ptr(rze), rze_bytes, _ptr(err), _ptr(idx), _ptr(count), cap, n, _dims(dims), abs_eb,
        int(zigzag), _ptr(out), flags, wp, wn, _stream(dev)), "fzb_lq_bs_rze_decompress")
    return out


def lq_bs_rze_decompress_dev(rze: torch.Tensor, rze_capacity: int, err, idx, count, cap: int, n: int,
                             dims, abs_eb: torch.Tensor, zigzag: bool = False, ws: Workspace | None = None,
                             out=None):
    """The fused inverse with no host wait: the error bound is read on the
    device (abs_eb: a one-float device tensor) and the exact kernels follow
    the fused pass, gated on its status.  Check ws.status() afterwards."""
    ws = ws or _default_ws
    dev = rze.device
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device=dev)
    wp, wn = ws.get(n, dev)
    check(lib().fzb_lq_bs_rze_decompress_dev(
        _ptr(rze), rze_capacity, _ptr(err), _ptr(idx), _ptr(count), cap, n, _dims(dims), _ptr(abs_eb),
        int(zigzag), _ptr(out), wp, wn, _stream(dev)), "fzb_lq_bs_rze_decompress_dev")
    return out


def _elem(t: torch.Tensor) -> int:
    return t.element_size()


def rle_encode(data: torch.Tensor, ws: Workspace | None = None, trim: bool = True):
    """RLEStage<T> forward (rle.cu:261-384).  Returns (stream, size_tensor)."""
    ws = ws or _default_ws
    src = data.reshape(-1)
    n, e = src.numel(), _elem(src)
    out = torch.empty(int(lib().fzb_rle_max_bytes(n, e)), dtype=torch.uint8, device=src.device)
    size = torch.zeros(1, dtype=torch.int64, device=src.device)
    wp, wn = ws.get(n, src.device)
    check(lib().fzb_rle_encode(_ptr(src), n, e, _ptr(out), _ptr(size), wp, wn, _stream(src.device)),
          "fzb_rle_encode")
    if trim:
        return out[: int(size.item())], size
    return out, size


def rle_decode(stream: torch.Tensor, n: int, dtype=torch.uint16, ws: Workspace | None = None,
               out: torch.Tensor | None = None):
    """RLEStage<T> inverse (rle.cu:196-259)."""
    ws = ws or _default_ws
    src = stream.view(torch.uint8).reshape(-1)
    if out is None:
        out = torch.empty(n, dtype=dtype, device=src.device)
    wp, wn = ws.get(n, src.device)
    check(lib().fzb_rle_decode(_ptr(src), n, _elem(out), _ptr(out), wp, wn, _stream(src.device)),
          "fzb_rle_decode")
    return out


def bitpack_encode(data: torch.Tensor, nbits: int = 0, ws: Workspace | None = None):
    """BitpackStage<T> forward (bitpack_stage.cu:169-244).  nbits 0 = detect.
    Returns (packed bytes, nbits used)."""
    ws = ws or _default_ws
    src = data.reshape(-1)
    n, e = src.numel(), _elem(src)
    out = torch.empty(n * e, dtype=torch.uint8, device=src.device)
    nb = torch.zeros(1, dtype=torch.uint8, device=src.device)
    size = torch.zeros(1, dtype=torch.int64, device=src.device)
    wp, wn = ws.get(1, src.device)
    check(lib().fzb_bitpack_encode(_ptr(src), n, e, nbits, _ptr(out), _ptr(nb), _ptr(size), wp, wn,
                                   _stream(src.device)), "fzb_bitpack_encode")
    return out[: int(size.item())], int(nb.item())


def bitpack_decode(packed: torch.Tensor, n: int, nbits: int, dtype=torch.uint16):
    out = torch.empty(n, dtype=dtype, device=packed.device)
    check(lib().fzb_bitpack_decode(_ptr(packed), n, _elem(out), nbits, _ptr(out),
                                   _stream(packed.device)), "fzb_bitpack_decode")
    return out


# ------------------------------------------------------------------ Huffman

# ------------------------------------------------------- stages around the codes

def _flat(data: torch.Tensor) -> torch.Tensor:
    return data.reshape(-1).contiguous()


def zigzag(data: torch.Tensor, inverse: bool = False, out: torch.Tensor | None = None) -> torch.Tensor:
    """ZigzagStage (transforms/zigzag/zigzag_stage.cu) on the element bit
    patterns of `data` (1/2/4/8-byte elements); same dtype out."""
    src = _flat(data)
    dst = torch.empty_like(src) if out is None else out
    check(lib().fzb_zigzag(_ptr(src), src.numel(), src.element_size(), int(inverse), _ptr(dst), _stream(src.device)),
          "fzb_zigzag")
    return dst


def negabinary(data: torch.Tensor, inverse: bool = False, out: torch.Tensor | None = None) -> torch.Tensor:
    """NegabinaryStage (transforms/negabinary/negabinary_stage.cu)."""
    src = _flat(data)
    dst = torch.empty_like(src) if out is None else out
    check(lib().fzb_negabinary(_ptr(src), src.numel(), src.element_size(), int(inverse), _ptr(dst),
                               _stream(src.device)), "fzb_negabinary")
    return dst


def diff(data: torch.Tensor, chunk_bytes: int = 0, negabinary: bool = False, inverse: bool = False,
         ws: Workspace | None = None) -> torch.Tensor:
    """DifferenceStage<T> / <T, TOut> for integer T (predictors/diff/diff.cu);
    chunk_bytes as setChunkSize (0 = one chunk)."""
    ws = ws or _default_ws
    src = _flat(data)
    e = src.element_size()
    dst = torch.empty_like(src)
    wp, wn = ws.get_bytes(lib().fzb_scan_workspace_bytes(src.numel(), e), src.device)
    check(lib().fzb_diff(_ptr(src), src.numel(), e, chunk_bytes // e, int(negabinary), int(inverse), _ptr(dst), wp,
                         wn, _stream(src.device)), "fzb_diff")
    return dst


def lorenzo_int(data: torch.Tensor, dims, inverse: bool = False, ws: Workspace | None = None) -> torch.Tensor:
    """LorenzoStage<T> (predictors/lorenzo/lorenzo_stage.cu); dims = (x, y, z)."""
    ws = ws or _default_ws
    src = _flat(data)
    e = src.element_size()
    dst = torch.empty_like(src)
    d = (C.c_uint64 * 3)(*[int(v) for v in dims])
    wp, wn = ws.get_bytes(lib().fzb_scan_workspace_bytes(src.numel(), e), src.device)
    check(lib().fzb_lorenzo_int(_ptr(src), d, src.numel(), e, int(inverse), _ptr(dst), wp, wn, _stream(src.device)),
          "fzb_lorenzo_int")
    return dst


def quantizer_forward(x: torch.Tensor, eb: float, mode: int = ABS, radius: int = 32768, code_bytes: int = 2,
                      zigzag: bool = False, outlier_capacity: float = 0.05, threshold: float = float("inf"),
                      inplace: bool = False, value_base: float = 0.0, ws: Workspace | None = None,
                      out: dict | None = None, check_status: bool = True) -> dict:
    """QuantizerStage<float, TCode> forward (quantizers/quantizer/quantizer.cu).
    Returns codes, index-ordered outlier lists, capped count, cap and the
    device-resolved bound (value_base, abs_eb, 1/(2 abs_eb), 2 abs_eb).
    check_status=False skips the synchronising read of the device status
    (read it later with ws.status()); `out` reuses a previous result's buffers."""
    ws = ws or _default_ws
    src = _flat(x)
    n, dev = src.numel(), src.device
    cap = 0 if (inplace and mode != REL) else max_outliers(n, outlier_capacity)
    ctype = torch.int16 if code_bytes == 2 else torch.int32
    if out is None:
        out = dict(codes=torch.empty(n, dtype=ctype, device=dev),
                   vals=torch.empty(max(cap, 1), dtype=torch.float32, device=dev),
                   idx=torch.empty(max(cap, 1), dtype=torch.int32, device=dev),
                   count=torch.zeros(1, dtype=torch.int32, device=dev),
                   eb_state=torch.zeros(4, dtype=torch.float32, device=dev), cap=cap)
    wp, wn = ws.get_bytes(lib().fzb_quantizer_workspace_bytes(n), dev)
    check(lib().fzb_quantizer_forward(_ptr(src), n, code_bytes, eb, mode, value_base, radius, int(zigzag), threshold,
                                      int(inplace), _ptr(out["codes"]), _ptr(out["vals"]), _ptr(out["idx"]),
                                      _ptr(out["count"]), cap, _ptr(out["eb_state"]), wp, wn, _stream(dev)),
          "fzb_quantizer_forward")
    if check_status:
        st = lib().fzb_workspace_status(wp, _stream(dev))
        if st != 0:
            raise FzbError(st, "fzb_quantizer_forward")
    return out


def quantizer_inverse(codes: torch.Tensor, eb: float, mode: int, abs_eb: float, radius: int = 32768,
                      zigzag: bool = False, inplace: bool = False, vals=None, idx=None, count=None,
                      cap: int = 0) -> torch.Tensor:
    """QuantizerStage inverse: dequantise, then scatter the outliers."""
    src = _flat(codes)
    n, dev = src.numel(), src.device
    out = torch.empty(n, dtype=torch.float32, device=dev)
    check(lib().fzb_quantizer_inverse(_ptr(src), n, src.element_size(), eb, mode, abs_eb, radius, int(zigzag),
                                      int(inplace), _ptr(vals), _ptr(idx), _ptr(count), cap, _ptr(out),
                                      _stream(dev)), "fzb_quantizer_inverse")
    return out


def pfpl_compress(x: torch.Tensor, eb: float = 1e-3, mode: int = REL, radius: int = 32768, zigzag: bool = True,
                  outlier_capacity: float = 0.1, threshold: float = float("inf"), value_base: float = 0.0,
                  ws: Workspace | None = None, out: dict | None = None) -> dict:
    """The pfpl preset's Quantizer(u32) -> Difference(16 KiB) -> Bitshuffle(ew 2)
    -> RZE chain in one pass.  Returns the RZE stream (max size), its device
    size, the outlier lists, the capped count, cap and eb_state."""
    ws = ws or _default_ws
    src = _flat(x)
    n, dev = src.numel(), src.device
    cap = max_outliers(n, outlier_capacity)
    if out is None:
        out = dict(rze=torch.empty(int(lib().fzb_rze_max_bytes(4 * n)), dtype=torch.uint8, device=dev),
                   rze_size=torch.zeros(1, dtype=torch.int64, device=dev),
                   vals=torch.empty(max(cap, 1), dtype=torch.float32, device=dev),
                   idx=torch.empty(max(cap, 1), dtype=torch.int32, device=dev),
                   count=torch.zeros(1, dtype=torch.int32, device=dev),
                   eb_state=torch.zeros(4, dtype=torch.float32, device=dev), cap=cap)
    wp, wn = ws.get_bytes(lib().fzb_pfpl_workspace_bytes(n, cap), dev)
    check(lib().fzb_pfpl_compress(_ptr(src), n, eb, mode, value_base, radius, int(zigzag), threshold,
                                  _ptr(out["vals"]), _ptr(out["idx"]), cap, _ptr(out["count"]), _ptr(out["rze"]),
                                  _ptr(out["rze_size"]), _ptr(out["eb_state"]), wp, wn, _stream(dev)),
          "fzb_pfpl_compress")
    return out


def pfpl_decompress(rze: torch.Tensor, rze_bytes: int, vals, idx, count, cap: int, n: int, eb: float = 1e-3,
                    mode: int = REL, abs_eb: float = 0.0, zigzag: bool = True, ws: Workspace | None = None,
                    out: torch.Tensor | None = None) -> torch.Tensor:
    ws = ws or _default_ws
    dev = rze.device
    y = torch.empty(n, dtype=torch.float32, device=dev) if out is None else out
    wp, wn = ws.get_bytes(lib().fzb_pfpl_decompress_workspace_bytes(n), dev)
    check(lib().fzb_pfpl_decompress(_ptr(rze), rze_bytes, _ptr(vals), _ptr(idx), _ptr(count), cap, n, eb, mode,
                                    abs_eb, int(zigzag), _ptr(y), wp, wn, _stream(dev)), "fzb_pfpl_decompress")
    return y


def crc32(data: torch.Tensor, ws: Workspace | None = None) -> torch.Tensor:
    """CRC-32 of a device tensor's bytes (the FZM data checksum,
    compressor_io.cpp:25-52).  Returns a 1-element int64 device tensor."""
    ws = ws or _default_ws
    src = data.reshape(-1).view(torch.uint8) if data.numel() else data.reshape(-1)
    out = torch.zeros(1, dtype=torch.int32, device=data.device)
    wp, wn = ws.get_bytes(lib().fzb_crc32_workspace_bytes(src.numel() * src.element_size()), data.device)
    check(lib().fzb_crc32(_ptr(src) if src.numel() else None, src.numel() * src.element_size(), _ptr(out), wp, wn,
                          _stream(data.device)), "fzb_crc32")
    return out.to(torch.int64) & 0xFFFFFFFF


def huff_histogram(codes: torch.Tensor, bklen: int = 1024) -> torch.Tensor:
    """GPU_histogram_generic (util/histogram/histogram.cu): u32 counts."""
    src = codes.reshape(-1)
    freq = torch.empty(bklen, dtype=torch.int32, device=src.device)
    check(lib().fzb_huff_histogram(_ptr(src), src.numel(), bklen, _ptr(freq), _stream(src.device)),
          "fzb_huff_histogram")
    return freq


def huff_book(freq, bklen: int = 1024):
    """phf_CPU_build_canonized_codebook_v2 (phf/hf_bk.cc:84-140) on the host.
    Returns (bk4 u32[bklen], revbook u8[256 + 2*bklen]) as numpy arrays."""
    import numpy as np
    f = np.ascontiguousarray(freq.cpu().numpy() if isinstance(freq, torch.Tensor) else freq).view(np.uint32)
    bk4 = np.empty(bklen, np.uint32)
    rb = np.zeros(256 + 2 * bklen, np.uint8)
    check(lib().fzb_huff_book(f.ctypes.data, bklen, bk4.ctypes.data, rb.ctypes.data), "fzb_huff_book")
    return bk4, rb


def huff_encode(codes: torch.Tensor, bk4, revbook, bklen: int = 1024, ws: Workspace | None = None,
                trim: bool = True, fine: bool = False):
    """GPU_coarse_encode (or, fine=True, GPU_fine_encode with 1024-symbol
    partitions) + blob assembly with a given codebook.  Returns (blob,
    size_tensor)."""
    import numpy as np
    ws = ws or _default_ws
    src = codes.reshape(-1)
    n, dev = src.numel(), src.device
    d_bk4 = torch.from_numpy(np.ascontiguousarray(bk4).view(np.int32)).to(dev)
    d_rb = torch.from_numpy(np.ascontiguousarray(revbook)).to(dev)
    out = torch.empty(int(lib().fzb_huff_max_bytes(n, bklen)), dtype=torch.uint8, device=dev)
    size = torch.zeros(1, dtype=torch.int64, device=dev)
    wp, wn = ws.get_bytes(lib().fzb_huff_workspace_bytes(n, bklen), dev)
    fn = lib().fzb_huff_encode_fine if fine else lib().fzb_huff_encode
    check(fn(_ptr(src), n, bklen, _ptr(d_bk4), _ptr(d_rb), _ptr(out), _ptr(size), wp, wn, _stream(dev)),
          "fzb_huff_encode")
    if trim:
        return out[: int(size.item())], size
    return out, size


def huff_compress(codes: torch.Tensor, bklen: int = 1024, ws: Workspace | None = None,
                  trim: bool = True, fine: bool = False):
    """HuffmanStage<uint16_t>::execute forward (huffman_stage.cu:111-186);
    fine=True is setEncodeMode(Fine).  Returns (blob, size_tensor)."""
    ws = ws or _default_ws
    src = codes.reshape(-1)
    n, dev = src.numel(), src.device
    out = torch.empty(int(lib().fzb_huff_max_bytes(n, bklen)), dtype=torch.uint8, device=dev)
    size = torch.zeros(1, dtype=torch.int64, device=dev)
    wp, wn = ws.get_bytes(lib().fzb_huff_workspace_bytes(n, bklen), dev)
    fn = lib().fzb_huff_compress_fine if fine else lib().fzb_huff_compress
    check(fn(_ptr(src), n, bklen, _ptr(out), _ptr(size), wp, wn, _stream(dev)), "fzb_huff_compress")
    if trim:
        return out[: int(size.item())], size
    return out, size


def huff_decode(blob: torch.Tensor, n: int, bklen: int = 1024, ws: Workspace | None = None,
                out: torch.Tensor | None = None):
    """HuffmanStage<uint16_t> inverse (phf/hf_kernels.cu:267-298)."""
    ws = ws or _default_ws
    src = blob.view(torch.uint8).reshape(-1)
    if out is None:
        out = torch.empty(n, dtype=torch.uint16, device=src.device)
    wp, wn = ws.get_bytes(256, src.device)
    check(lib().fzb_huff_decode(_ptr(src), src.numel(), n, bklen, _ptr(out), wp, wn,
                                _stream(src.device)), "fzb_huff_decode")
    return out


# ------------------------------------------------------------------ tracing

class Trace:
    """Per-kernel CUDA-event timing of the library's launches
    (fzb_trace_*).  Use as a context manager; `kernels()` returns
    {name: (launches, total_ms)} accumulated while enabled."""

    def __enter__(self):
        lib().fzb_trace_collect()
        lib().fzb_trace_reset()
        lib().fzb_trace_enable(1)
        return self

    def __exit__(self, *exc):
        lib().fzb_trace_enable(0)

    @staticmethod
    def kernels() -> dict:
        n = lib().fzb_trace_collect()
        check(min(n, 0), "fzb_trace_collect")
        out = {}
        name = C.create_string_buffer(96)
        launches, ms = C.c_uint64(0), C.c_double(0.0)
        for i in range(n):
            check(lib().fzb_trace_get(i, name, 96, C.byref(launches), C.byref(ms)), "fzb_trace_get")
            out[name.value.decode()] = (int(launches.value), float(ms.value))
        return out


# ------------------------------------------------------------------ batches

class _BatchField(C.Structure):
    _fields_ = [("d_in", C.c_void_p), ("n_total", C.c_uint64), ("dims", C.c_uint32 * 3), ("eb", C.c_float),
                ("eb_mode", C.c_int), ("value_base", C.c_float), ("radius", C.c_uint32), ("zigzag", C.c_int),
                ("d_err", C.c_void_p), ("d_idx", C.c_void_p), ("cap", C.c_uint64), ("d_count", C.c_void_p),
                ("d_rze", C.c_void_p), ("d_rze_size", C.c_void_p), ("d_eb_state", C.c_void_p)]


class BatchTuning(C.Structure):
    """fzb_batch_tuning: CTAs per SM, dispatch order, flat tiles for
    slab-shaped fields, value-base scan blocks per SM (0 = default)."""
    _fields_ = [("ctas_per_sm", C.c_int), ("order", C.c_int), ("flat_tiles", C.c_int), ("scan_parts", C.c_int)]

    def __repr__(self):
        return (f"BatchTuning(ctas_per_sm={self.ctas_per_sm}, order={self.order}, flat_tiles={self.flat_tiles}, "
                f"scan_parts={self.scan_parts})")


class Batch:
    """Batched LorenzoQuant -> Bitshuffle -> RZE over many fields
    (fzb_batch_*).  ``fields``: dicts with x (device float tensor), dims,
    eb, mode, radius, zigzag and optionally outlier_capacity / value_base.
    Outputs per field live in ``self.outputs`` (the same dict layout as
    lq_bs_rze_compress); launch() re-runs the batch into them."""

    def __init__(self, fields: list, tuning: BatchTuning | None = None):
        self.device = fields[0]["x"].device
        self.fields, self.outputs = fields, []
        arr = (_BatchField * len(fields))()
        for i, f in enumerate(fields):
            x = f["x"]
            n = x.numel()
            cap = max_outliers(n, f.get("outlier_capacity", 0.2))
            o = dict(rze=torch.empty(int(lib().fzb_rze_max_bytes(2 * n)), dtype=torch.uint8, device=self.device),
                     rze_size=torch.zeros(1, dtype=torch.int64, device=self.device),
                     err=torch.empty(max(cap, 1), dtype=torch.float32, device=self.device),
                     idx=torch.empty(max(cap, 1), dtype=torch.int32, device=self.device),
                     count=torch.zeros(1, dtype=torch.int32, device=self.device),
                     eb_state=torch.zeros(4, dtype=torch.float32, device=self.device), cap=cap)
            self.outputs.append(o)
            d = f["dims"]
            arr[i] = _BatchField(x.data_ptr(), n, (C.c_uint32 * 3)(*d), f["eb"], f.get("mode", ABS),
                                 f.get("value_base", 0.0), f.get("radius", 32768), int(f.get("zigzag", False)),
                                 o["err"].data_ptr(), o["idx"].data_ptr(), cap, o["count"].data_ptr(),
                                 o["rze"].data_ptr(), o["rze_size"].data_ptr(), o["eb_state"].data_ptr())
        self._arr = arr
        need = int(lib().fzb_batch_workspace_bytes(arr, len(fields)))
        self.work = torch.empty(need, dtype=torch.uint8, device=self.device)
        self._h = None
        self.retune(tuning)

    def retune(self, tuning: BatchTuning | None):
        if self._h:
            lib().fzb_batch_destroy(self._h)
        st = C.c_int(0)
        with torch.cuda.device(self.device):
            h = lib().fzb_batch_create(self._arr, len(self.fields), C.byref(tuning) if tuning else None,
                                       _ptr(self.work), self.work.numel(), C.byref(st))
        if not h:
            check(st.value or -1, "fzb_batch_create")
        self._h = h
        self.tuning = tuning

    def autotune(self) -> tuple:
        best, ms = BatchTuning(), C.c_float(0)
        with torch.cuda.device(self.device):
            check(lib().fzb_batch_autotune(self._arr, len(self.fields), _ptr(self.work), self.work.numel(),
                                           _stream(self.device), C.byref(best), C.byref(ms)), "fzb_batch_autotune")
        self.retune(best)
        return best, ms.value

    def launch(self, stream: torch.cuda.Stream | None = None):
        s = C.c_void_p(stream.cuda_stream) if stream is not None else _stream(self.device)
        check(lib().fzb_batch_launch(self._h, s), "fzb_batch_launch")

    def close(self):
        if self._h:
            lib().fzb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
