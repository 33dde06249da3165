"""Python view of the fz:: pipeline (include/fz/pipeline.h) through the
fzb_pipeline_* C ABI, with the reference's names: stage classes with their
setters, ``Pipeline.addStage / connect / finalize / compress / decompress /
writeToFile / decompressFromFile`` (include/pipeline/compressor.h:34-386).

Stage objects hold their configuration until ``finalize()`` builds the
native pipeline, so setters may be called after ``addStage`` as in C++.
Device buffers are torch tensors; compressed outputs and pool-managed
decompressed outputs are views of pipeline-owned memory, valid until the
next ``compress()`` / ``decompress()`` (copy them to keep them).
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import FzbError, lib

ABS, REL, NOA = 0, 1, 2
MINIMAL, PREALLOCATE = 0, 1


class PipelineError(RuntimeError):
    """A pipeline call failed (the reference throws std::runtime_error)."""


def _check(rc: int, what: str) -> int:
    if rc < 0:
        msg = lib().fzb_last_error().decode(errors="replace")
        if rc == -8:
            raise PipelineError(f"{what}: {msg}")
        raise FzbError(rc, f"{what}: {msg}" if msg else what)
    return rc


class _DeviceView:
    """__cuda_array_interface__ over pipeline-owned device bytes."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


def _view(ptr: int, nbytes: int, device, cache: dict | None = None) -> torch.Tensor:
    """A uint8 tensor over `nbytes` pipeline-owned device bytes at `ptr`.  A
    pipeline reuses its output buffers from call to call, so its views are
    kept by (pointer, size) in `cache` (a few entries) instead of being built
    again through __cuda_array_interface__ on every call."""
    if nbytes == 0 or not ptr:
        return torch.empty(0, dtype=torch.uint8, device=device)
    key = (ptr, nbytes)
    if cache is not None and key in cache:
        return cache[key]
    with torch.cuda.device(device):
        t = torch.as_tensor(_DeviceView(ptr, nbytes), device=device)
    if cache is not None:
        if len(cache) >= 4:
            cache.pop(next(iter(cache)))
        cache[key] = t
    return t


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def _stream(device) -> C.c_void_p:
    if _raw_stream is not None:  # the current stream's handle without a Stream object
        idx = device.index if device.index is not None else torch.cuda.current_device()
        return C.c_void_p(_raw_stream(idx))
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class _OnDevice:
    """torch.cuda.device(d), skipped when d is already current."""

    __slots__ = ("idx", "prev")

    def __init__(self, device):
        self.idx = device.index
        self.prev = None

    def __enter__(self):
        cur = torch.cuda.current_device()
        if cur != self.idx:
            self.prev = cur
            torch.cuda.set_device(self.idx)

    def __exit__(self, *exc):
        if self.prev is not None:
            torch.cuda.set_device(self.prev)


# ------------------------------------------------------------------ stages

class Stage:
    _node = -1

    def getName(self) -> str:
        return type(self).__name__.replace("Stage", "")


class LorenzoQuantStage(Stage):
    """LorenzoQuantStage<float, uint16_t> (fused/lorenzo_quant/lorenzo_quant.h)."""

    def __init__(self, error_bound: float = 1e-3, quant_radius: int = 32768, outlier_capacity: float = 0.2,
                 eb_mode: int = ABS, zigzag_codes: bool = False, value_base: float = 0.0):
        self.error_bound, self.quant_radius = error_bound, quant_radius
        self.outlier_capacity, self.eb_mode = outlier_capacity, eb_mode
        self.zigzag_codes, self.value_base = zigzag_codes, value_base

    def getName(self):
        return "LorenzoQuant"

    def setErrorBound(self, v): self.error_bound = v
    def setQuantRadius(self, v): self.quant_radius = v
    def setOutlierCapacity(self, v): self.outlier_capacity = v
    def setErrorBoundMode(self, v): self.eb_mode = v
    def setValueBase(self, v): self.value_base = v
    def setZigzagCodes(self, v): self.zigzag_codes = bool(v)

    def _add(self, h):
        return lib().fzb_pipeline_add_lorenzo_quant(h, self.error_bound, self.eb_mode, self.quant_radius,
                                                    self.outlier_capacity, int(self.zigzag_codes), self.value_base)


# FZM DataType codes (include/fzm_format.h)
UINT8, UINT16, UINT32, UINT64, INT8, INT16, INT32, INT64, FLOAT32, FLOAT64 = range(10)


class QuantizerStage(Stage):
    """QuantizerStage<float, uint16_t | uint32_t> (quantizers/quantizer/quantizer.h);
    code_bytes = sizeof(TCode).  Outputs: codes, outlier_vals, outlier_idxs,
    outlier_count (codes only with in-place outliers)."""

    def __init__(self, error_bound: float = 1e-4, eb_mode: int = ABS, quant_radius: int = 32768,
                 outlier_capacity: float = 0.05, code_bytes: int = 2, zigzag_codes: bool = False,
                 inplace_outliers: bool = False, outlier_threshold: float = float("inf"), value_base: float = 0.0):
        self.error_bound, self.eb_mode, self.quant_radius = error_bound, eb_mode, quant_radius
        self.outlier_capacity, self.code_bytes, self.zigzag_codes = outlier_capacity, code_bytes, zigzag_codes
        self.inplace_outliers, self.outlier_threshold, self.value_base = inplace_outliers, outlier_threshold, value_base

    def getName(self):
        return "Quantizer"

    def setErrorBound(self, v): self.error_bound = v
    def setQuantRadius(self, v): self.quant_radius = v
    def setOutlierCapacity(self, v): self.outlier_capacity = v
    def setErrorBoundMode(self, v): self.eb_mode = v
    def setValueBase(self, v): self.value_base = v
    def setZigzagCodes(self, v): self.zigzag_codes = bool(v)
    def setOutlierThreshold(self, v): self.outlier_threshold = v
    def setInplaceOutliers(self, v): self.inplace_outliers = bool(v)

    def _add(self, h):
        return lib().fzb_pipeline_add_quantizer(h, self.code_bytes, self.error_bound, self.eb_mode, self.quant_radius,
                                                self.outlier_capacity, int(self.zigzag_codes),
                                                int(self.inplace_outliers), self.outlier_threshold, self.value_base)


class DifferenceStage(Stage):
    """DifferenceStage<T, TOut> (predictors/diff/diff.h) for integer T; TOut the
    unsigned type of a signed T fuses negabinary coding."""

    def __init__(self, input_type: int = INT32, output_type: int | None = None, chunk_size: int = 0):
        self.input_type = input_type
        self.output_type = input_type if output_type is None else output_type
        self.chunk_size = chunk_size

    def setChunkSize(self, v): self.chunk_size = v

    def _add(self, h):
        return lib().fzb_pipeline_add_difference(h, self.input_type, self.output_type, self.chunk_size)


class LorenzoStage(Stage):
    """LorenzoStage<T> (predictors/lorenzo/lorenzo_stage.h), lossless integer
    Lorenzo over the pipeline's dims; T signed."""

    def __init__(self, data_type: int = INT32):
        self.data_type = data_type

    def _add(self, h):
        return lib().fzb_pipeline_add_lorenzo(h, self.data_type)


class ZigzagStage(Stage):
    """ZigzagStage<S, U> (transforms/zigzag/zigzag_stage.h); input_type signed."""

    def __init__(self, input_type: int = INT32):
        self.input_type = input_type

    def _add(self, h):
        return lib().fzb_pipeline_add_zigzag(h, self.input_type)


class NegabinaryStage(Stage):
    """NegabinaryStage<S, U> (transforms/negabinary/negabinary_stage.h)."""

    def __init__(self, input_type: int = INT32):
        self.input_type = input_type

    def _add(self, h):
        return lib().fzb_pipeline_add_negabinary(h, self.input_type)


class BitshuffleStage(Stage):
    """BitshuffleStage (shufflers/bitshuffle/bitshuffle_stage.h); defaults 16 KiB blocks, element width 4."""

    def __init__(self, block_size: int = 16384, element_width: int = 4):
        self.block_size, self.element_width = block_size, element_width

    def setBlockSize(self, v): self.block_size = v
    def setElementWidth(self, v): self.element_width = v

    def _add(self, h):
        return lib().fzb_pipeline_add_bitshuffle(h, self.block_size, self.element_width)


class RZEStage(Stage):
    """RZEStage (coders/rze/rze_stage.h)."""

    def __init__(self, chunk_size: int = 16384, levels: int = 4):
        self.chunk_size, self.levels = chunk_size, levels

    def getName(self):
        return "RZE"

    def setChunkSize(self, v): self.chunk_size = v
    def setLevels(self, v): self.levels = v

    def _add(self, h):
        return lib().fzb_pipeline_add_rze(h, self.chunk_size, self.levels)


class RLEStage(Stage):
    """RLEStage<T> (coders/rle/rle.h); elem = sizeof(T)."""

    def __init__(self, elem: int = 2):
        self.elem = elem

    def getName(self):
        return "RLE"

    def _add(self, h):
        return lib().fzb_pipeline_add_rle(h, self.elem)


class HuffmanEncodeMode:
    """HuffmanEncodeMode (coders/huffman/huffman_stage.h)."""
    Coarse = 0
    Fine = 1


class HuffmanStage(Stage):
    """HuffmanStage<uint16_t> (coders/huffman/huffman_stage.h), coarse or fine mode."""

    def __init__(self, bklen: int = 1024):
        self.bklen = bklen
        self.encode_mode = HuffmanEncodeMode.Coarse

    def setBklen(self, v): self.bklen = v

    def setEncodeMode(self, mode): self.encode_mode = int(mode)

    def _add(self, h):
        return lib().fzb_pipeline_add_huffman_mode(h, self.bklen, self.encode_mode)


class BitpackStage(Stage):
    """BitpackStage<T> (coders/bitpack/bitpack_stage.h); nbits 0 = auto-detect."""

    def __init__(self, elem: int = 2, nbits: int = 0):
        self.elem, self.nbits = elem, nbits

    def setNBits(self, v): self.nbits = v
    def setAutoDetect(self, on): self.nbits = 0 if on else (self.nbits or 8 * self.elem)

    def _add(self, h):
        return lib().fzb_pipeline_add_bitpack(h, self.elem, self.nbits)


# ---------------------------------------------------------------- pipeline

class Pipeline:
    """fz::Pipeline.  ``strategy`` MINIMAL or PREALLOCATE."""

    def __init__(self, input_data_size: int = 0, strategy: int = MINIMAL, pool_multiplier: float = 3.0,
                 device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.device.index is None:  # "cuda": the current device, by index
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._hint, self._strategy, self._mult = int(input_data_size), int(strategy), float(pool_multiplier)
        self._stages: list[Stage] = []
        self._conns: list[tuple[Stage, Stage, str]] = []
        self._dims = (0, 1, 1)
        self._fusion, self._graph, self._profiling = True, False, False
        self._streams, self._bounds = 1, False
        self._h = None
        self._last_in = 0
        self._views: dict = {}  # (pointer, bytes) -> view of pipeline-owned output memory

    # builder ---------------------------------------------------------------
    def loadConfig(self, path: str):
        """Pipeline::loadConfig (src/pipeline/config.cpp:534-640): the
        [pipeline] settings and [[stage]] tables of a TOML file, connected by
        their ``inputs`` and finalized."""
        from . import config
        if self._h is not None:
            raise PipelineError("loadConfig: pipeline is already finalized")
        with open(path) as f:
            cfg = config.parse_config(f.read())
        pl = cfg["pipeline"]
        if "input_size" in pl:
            self._hint = int(pl["input_size"])
        if "dims" in pl:
            d = [int(v) for v in pl["dims"]][:3] + [0, 1, 1][len(pl["dims"][:3]):]
            self.setDims(*d)
        if "memory_strategy" in pl:
            self._strategy = config.strategy(pl["memory_strategy"])
        if "pool_multiplier" in pl:
            self._mult = float(pl["pool_multiplier"])
        if "num_streams" in pl:
            self.setNumStreams(int(pl["num_streams"]))
        for _, st in cfg["stages"]:
            self.addStage(st)
        for dep, prod, port in cfg["connections"]:
            self.connect(dep, prod, port)
        self.finalize()

    def saveConfig(self, path: str):
        """Pipeline::saveConfig (config.cpp:645-...): the finalized pipeline as TOML."""
        from . import config
        if self._h is None:
            raise PipelineError("saveConfig: pipeline must be finalized first")
        params = {"input_size": self._hint,
                  "memory_strategy": "PREALLOCATE" if self._strategy == PREALLOCATE else "MINIMAL",
                  "pool_multiplier": self._mult, "num_streams": self.getNumStreams(), "dims": list(self._dims)}
        with open(path, "w") as f:
            f.write(config.dump_config(params, self._stages, self._conns))

    def setDims(self, x: int, y: int = 1, z: int = 1):
        self._dims = (int(x), int(y), int(z))

    def addStage(self, stage: Stage) -> Stage:
        if self._h is not None:
            raise PipelineError("Cannot add stages after finalization")
        self._stages.append(stage)
        return stage

    def connect(self, dependent: Stage, producer: Stage, output_name: str = "output"):
        if self._h is not None:
            raise PipelineError("Cannot connect stages after finalization")
        self._conns.append((dependent, producer, output_name))

    def setFusion(self, on: bool):
        self._fusion = bool(on)

    def enableGraphMode(self, on: bool):
        self._graph = bool(on)

    def setNumStreams(self, n: int):
        """Side streams for DAG levels with several stages (before finalize)."""
        if self._h is not None:
            raise PipelineError("Cannot configure streams after finalization")
        self._streams = int(n)

    def getNumStreams(self) -> int:
        return lib().fzb_pipeline_num_streams(self._h) if self._h is not None else self._streams

    def enableBoundsCheck(self, on: bool):
        """After each stage, compare its output sizes with the reserved bytes."""
        self._bounds = bool(on)
        if self._h is not None:
            _check(lib().fzb_pipeline_enable_bounds_check(self._h, int(on)), "enableBoundsCheck")

    def enableProfiling(self, on: bool):
        self._profiling = bool(on)
        if self._h is not None:
            _check(lib().fzb_pipeline_enable_profiling(self._h, int(on)), "enableProfiling")

    def finalize(self):
        if self._h is not None:
            raise PipelineError("Pipeline already finalized")
        with torch.cuda.device(self.device):
            h = lib().fzb_pipeline_create(self._hint, self._strategy, self._mult)
            if not h:
                raise PipelineError(lib().fzb_last_error().decode())
            try:
                _check(lib().fzb_pipeline_set_dims(h, *self._dims), "setDims")
                for s in self._stages:
                    s._node = _check(s._add(h), f"addStage({s.getName()})")
                for dep, prod, name in self._conns:
                    _check(lib().fzb_pipeline_connect(h, dep._node, prod._node, name.encode()), "connect")
                _check(lib().fzb_pipeline_set_fusion(h, int(self._fusion)), "setFusion")
                _check(lib().fzb_pipeline_enable_graph_mode(h, int(self._graph)), "enableGraphMode")
                _check(lib().fzb_pipeline_enable_profiling(h, int(self._profiling)), "enableProfiling")
                _check(lib().fzb_pipeline_set_num_streams(h, self._streams), "setNumStreams")
                _check(lib().fzb_pipeline_enable_bounds_check(h, int(self._bounds)), "enableBoundsCheck")
                _check(lib().fzb_pipeline_finalize(h), "finalize")
            except Exception:
                lib().fzb_pipeline_destroy(h)
                raise
        self._h = h

    def isFused(self) -> bool:
        return bool(self._h and lib().fzb_pipeline_is_fused(self._h))

    def captureGraph(self, stream: torch.cuda.Stream):
        _check(lib().fzb_pipeline_capture_graph(self._h, C.c_void_p(stream.cuda_stream)), "captureGraph")

    def isDecompressGraphCaptured(self) -> bool:
        return bool(self._h and lib().fzb_pipeline_decompress_graph_captured(self._h) == 1)

    def checkDecompressStatus(self):
        """Waits for the last decompress and raises if the device found its
        input malformed (graph-mode decompressions report it only here)."""
        with torch.cuda.device(self.device):
            _check(lib().fzb_pipeline_check_decompress(self._h, _stream(self.device)), "decompress")

    # execution -------------------------------------------------------------
    def compress(self, data: torch.Tensor) -> torch.Tensor:
        """Returns a view of the pipeline-owned compressed bytes."""
        if not data.is_contiguous():
            data = data.contiguous()
        nbytes = data.numel() * data.element_size()
        out, nb = C.c_void_p(), C.c_uint64()
        with _OnDevice(self.device):
            _check(lib().fzb_pipeline_compress(self._h, C.c_void_p(data.data_ptr()), nbytes, C.byref(out),
                                               C.byref(nb), _stream(self.device)), "compress")
        self._last_in = nbytes
        return _view(out.value or 0, nb.value, self.device, self._views)

    def decompress(self, compressed: torch.Tensor | None = None, dtype=torch.float32) -> torch.Tensor:
        """Pool-owned reconstruction (``compressed=None`` decompresses the
        pipeline's own last outputs)."""
        out, nb = C.c_void_p(), C.c_uint64()
        if compressed is not None and not compressed.is_contiguous():
            compressed = compressed.contiguous()
        ptr = C.c_void_p(compressed.data_ptr()) if compressed is not None else C.c_void_p()
        n = compressed.numel() * compressed.element_size() if compressed is not None else 0
        with _OnDevice(self.device):
            _check(lib().fzb_pipeline_decompress(self._h, ptr, n, C.byref(out), C.byref(nb), _stream(self.device)),
                   "decompress")
        return _view(out.value or 0, nb.value, self.device, self._views).view(dtype)

    def decompressInto(self, compressed: torch.Tensor | None, out: torch.Tensor) -> int:
        nb = C.c_uint64()
        ptr = C.c_void_p(compressed.data_ptr()) if compressed is not None else C.c_void_p()
        n = compressed.numel() * compressed.element_size() if compressed is not None else 0
        with torch.cuda.device(self.device):
            _check(lib().fzb_pipeline_decompress_into(self._h, ptr, n, C.c_void_p(out.data_ptr()),
                                                      out.numel() * out.element_size(), C.byref(nb),
                                                      _stream(self.device)), "decompress")
        return nb.value

    def stageTimings(self) -> list[float]:
        buf = (C.c_double * 64)()
        k = _check(lib().fzb_pipeline_stage_timings(self._h, buf, 64), "stageTimings")
        return [buf[i] for i in range(k)]

    def writeToFile(self, path: str):
        with torch.cuda.device(self.device):
            _check(lib().fzb_pipeline_write_file(self._h, str(path).encode(), _stream(self.device)), "writeToFile")

    @staticmethod
    def decompressFromFile(path: str, dtype=torch.float32, device=None) -> torch.Tensor:
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        out, nb = C.c_void_p(), C.c_uint64()
        with torch.cuda.device(dev):
            _check(lib().fzb_decompress_file(str(path).encode(), C.byref(out), C.byref(nb), _stream(dev)),
                   "decompressFromFile")
            try:
                t = _view(out.value or 0, nb.value, dev).clone()
            finally:
                if out.value:
                    lib().fzb_free(out)
        return t.view(dtype)

    def close(self):
        self._views = {}
        if self._h is not None:
            torch.cuda.synchronize(self.device)
            lib().fzb_pipeline_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
