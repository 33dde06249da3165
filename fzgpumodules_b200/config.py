"""TOML pipeline configurations: ``Pipeline.loadConfig`` / ``saveConfig``
(src/pipeline/config.cpp:515-640 and the per-stage readers and writers
above them), with the reference's keys, defaults, type names and error
messages, so its preset files (examples/presets/*.toml) load unchanged.

A file has an optional ``[pipeline]`` table (``input_size``, ``dims``,
``memory_strategy``, ``pool_multiplier``, ``num_streams``) and one
``[[stage]]`` table per stage with ``name``, ``type`` and the stage's keys;
``inputs = [{from = "...", port = "..."}]`` connects it (no ``inputs``: a
source stage).  Parsing needs no GPU; building the native pipeline happens
at ``finalize()``.
"""
from __future__ import annotations

import math
import tomllib

from . import pipeline as P

DTYPES = {"uint8": P.UINT8, "uint16": P.UINT16, "uint32": P.UINT32, "uint64": P.UINT64, "int8": P.INT8,
          "int16": P.INT16, "int32": P.INT32, "int64": P.INT64, "float32": P.FLOAT32, "float64": P.FLOAT64}
DTYPE_NAMES = {v: k for k, v in DTYPES.items()}
DTYPE_BYTES = {P.UINT8: 1, P.UINT16: 2, P.UINT32: 4, P.UINT64: 8, P.INT8: 1, P.INT16: 2, P.INT32: 4, P.INT64: 8}
EB_MODES = {"ABS": P.ABS, "REL": P.REL, "NOA": P.NOA}
EB_NAMES = {v: k for k, v in EB_MODES.items()}
STRATEGIES = {"MINIMAL": P.MINIMAL, "PREALLOCATE": P.PREALLOCATE}


class ConfigError(RuntimeError):
    """A configuration the reference's loadConfig would reject."""


def _eb_mode(s: str) -> int:
    if s not in EB_MODES:
        raise ConfigError(f"loadConfig: unknown error_bound_mode \"{s}\"")
    return EB_MODES[s]


def strategy(s: str) -> int:
    if s not in STRATEGIES:
        raise ConfigError(f"loadConfig: unknown memory_strategy \"{s}\"")
    return STRATEGIES[s]


def _huffman_mode(s: str):
    if s not in ("Fine", "Coarse"):
        raise ConfigError(f"loadConfig: unknown Huffman encode_mode \"{s}\"")
    return P.HuffmanEncodeMode.Fine if s == "Fine" else P.HuffmanEncodeMode.Coarse


def _dtype(s: str, what: str) -> int:
    if s not in DTYPES:
        raise ConfigError(f"loadConfig: unknown data type \"{s}\" ({what})")
    return DTYPES[s]


def _stage_from_table(t: dict) -> P.Stage:
    """One [[stage]] table -> a stage object (config.cpp add*Stage)."""
    typ = t["type"]
    g = t.get
    if typ == "LorenzoQuant":
        if g("input_type", "float32") != "float32" or g("code_type", "uint16") != "uint16":
            raise ConfigError("loadConfig: unsupported Lorenzo type combination input_type=\""
                              f"{g('input_type', 'float32')}\" code_type=\"{g('code_type', 'uint16')}\"")
        return P.LorenzoQuantStage(float(g("error_bound", 1e-3)), int(g("quant_radius", 32768)),
                                   float(g("outlier_capacity", 0.2)), _eb_mode(g("error_bound_mode", "ABS")),
                                   bool(g("zigzag_codes", False)))
    if typ == "Quantizer":
        code = g("code_type", "uint32")
        if g("input_type", "float32") != "float32" or code not in ("uint16", "uint32"):
            raise ConfigError("loadConfig: unsupported Quantizer type combination input_type=\""
                              f"{g('input_type', 'float32')}\" code_type=\"{code}\"")
        return P.QuantizerStage(float(g("error_bound", 1e-3)), _eb_mode(g("error_bound_mode", "REL")),
                                int(g("quant_radius", 32768)), float(g("outlier_capacity", 0.05)),
                                code_bytes=2 if code == "uint16" else 4, zigzag_codes=bool(g("zigzag_codes", True)),
                                inplace_outliers=bool(g("inplace_outliers", False)),
                                outlier_threshold=float(g("outlier_threshold", math.inf)))
    if typ == "Lorenzo":
        dt = _dtype(g("data_type", "int32"), "Lorenzo data_type")
        if dt not in (P.INT8, P.INT16, P.INT32, P.INT64):
            raise ConfigError(f"loadConfig: unsupported Lorenzo data_type \"{g('data_type')}\"")
        return P.LorenzoStage(dt)
    if typ == "Bitshuffle":
        return P.BitshuffleStage(int(g("block_size", 16384)), int(g("element_width", 4)))
    if typ == "RZE":
        return P.RZEStage(int(g("chunk_size", 16384)), int(g("levels", 4)))
    if typ == "RLE":
        dt = _dtype(g("data_type", "uint16"), "RLE data_type")
        if dt not in (P.UINT8, P.UINT16, P.UINT32, P.INT32):
            raise ConfigError(f"loadConfig: unsupported RLE data_type \"{g('data_type')}\"")
        return P.RLEStage(DTYPE_BYTES[dt])
    if typ == "Difference":
        a = _dtype(g("input_type", "float32"), "Difference input_type")
        out = g("output_type", "")
        b = _dtype(out, "Difference output_type") if out else a
        return P.DifferenceStage(a, b, int(g("chunk_size", 0)))
    if typ in ("Zigzag", "Negabinary"):
        a = _dtype(g("input_type", "int32"), f"{typ} input_type")
        cls = P.ZigzagStage if typ == "Zigzag" else P.NegabinaryStage
        return cls(a)
    if typ == "Bitpack":
        dt = _dtype(g("input_type", "uint16"), "Bitpack input_type")
        nb = int(g("nbits", 16))
        if nb <= 0 or nb > 8 * DTYPE_BYTES[dt] or nb & (nb - 1):
            raise ConfigError(f"BitpackStage::setNBits: nbits must be a power of two in [1, {8 * DTYPE_BYTES[dt]}], "
                              f"got {nb}")
        return P.BitpackStage(DTYPE_BYTES[dt], nb)
    if typ == "Huffman":
        mode = _huffman_mode(g("encode_mode", "Coarse"))
        s = P.HuffmanStage(int(g("bklen", 1024)))
        s.setEncodeMode(mode)
        return s
    raise ConfigError(f"loadConfig: unknown stage type \"{typ}\"")


def parse_config(text: str) -> dict:
    """Parses a configuration.  Returns {"pipeline": {...}, "stages":
    [(name, stage)], "connections": [(dependent, producer, port)]}."""
    doc = tomllib.loads(text)
    pl = dict(doc.get("pipeline", {}))
    if "memory_strategy" in pl:
        strategy(pl["memory_strategy"])
    arr = doc.get("stage")
    if not arr:
        raise ConfigError("loadConfig: no [[stage]] entries found")
    stages, by_name, tables = [], {}, []
    for t in arr:
        if "name" not in t or "type" not in t:
            raise ConfigError("loadConfig: each [[stage]] must have 'name' and 'type'")
        name = t["name"]
        if name in by_name:
            raise ConfigError(f"loadConfig: duplicate stage name \"{name}\"")
        s = _stage_from_table(t)
        s._config_name = name
        by_name[name] = s
        stages.append((name, s))
        tables.append(t)
    conns = []
    for (name, s), t in zip(stages, tables):
        for inp in t.get("inputs", []) or []:
            if "from" not in inp:
                raise ConfigError(f"loadConfig: stage \"{name}\" input missing 'from' key")
            src = inp["from"]
            if src not in by_name:
                raise ConfigError(f"loadConfig: stage \"{name}\" references unknown stage \"{src}\"")
            conns.append((s, by_name[src], inp.get("port", "output")))
    return {"pipeline": pl, "stages": stages, "connections": conns}


def _fmt(v) -> str:
    """Numbers as the reference's writer prints them: integers plainly,
    floating point with 17 significant digits (std::setprecision(
    max_digits10) on a std::ostream)."""
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, float):
        if math.isinf(v):
            return "inf" if v > 0 else "-inf"
        t = f"{v:.17g}"
        return t
    if isinstance(v, str):
        return f"\"{v}\""
    return str(v)


def _f32(v: float) -> float:
    """The float the stage stores, widened to double as the writer does."""
    import struct
    return struct.unpack("<f", struct.pack("<f", float(v)))[0]


def _stage_table(s: P.Stage) -> dict:
    """The keys config.cpp's save*Stage functions write for a stage, in their
    order; optional keys only when they differ from the loader's defaults."""
    if isinstance(s, P.LorenzoQuantStage):
        return {"type": "LorenzoQuant", "input_type": "float32", "code_type": "uint16",
                "error_bound": _f32(s.error_bound), "error_bound_mode": EB_NAMES[s.eb_mode],
                "quant_radius": int(s.quant_radius), "outlier_capacity": _f32(s.outlier_capacity),
                "zigzag_codes": bool(s.zigzag_codes)}
    if isinstance(s, P.QuantizerStage):
        d = {"type": "Quantizer", "input_type": "float32", "code_type": "uint16" if s.code_bytes == 2 else "uint32",
             "error_bound": _f32(s.error_bound), "error_bound_mode": EB_NAMES[s.eb_mode],
             "quant_radius": int(s.quant_radius), "outlier_capacity": _f32(s.outlier_capacity),
             "zigzag_codes": bool(s.zigzag_codes)}
        if math.isfinite(s.outlier_threshold):
            d["outlier_threshold"] = _f32(s.outlier_threshold)
        if s.inplace_outliers:
            d["inplace_outliers"] = True
        return d
    if isinstance(s, P.LorenzoStage):
        return {"type": "Lorenzo", "data_type": DTYPE_NAMES[s.data_type]}
    if isinstance(s, P.BitshuffleStage):
        return {"type": "Bitshuffle", "block_size": int(s.block_size), "element_width": int(s.element_width)}
    if isinstance(s, P.RZEStage):
        return {"type": "RZE", "chunk_size": int(s.chunk_size), "levels": int(s.levels)}
    if isinstance(s, P.RLEStage):
        return {"type": "RLE", "data_type": {1: "uint8", 2: "uint16", 4: "uint32"}[s.elem]}
    if isinstance(s, P.DifferenceStage):
        return {"type": "Difference", "input_type": DTYPE_NAMES[s.input_type],
                "output_type": DTYPE_NAMES[s.output_type], "chunk_size": int(s.chunk_size)}
    if isinstance(s, P.ZigzagStage):
        return {"type": "Zigzag", "input_type": DTYPE_NAMES[s.input_type],
                "output_type": DTYPE_NAMES[s.input_type].replace("int", "uint", 1)}
    if isinstance(s, P.NegabinaryStage):
        return {"type": "Negabinary", "input_type": DTYPE_NAMES[s.input_type],
                "output_type": DTYPE_NAMES[s.input_type].replace("int", "uint", 1)}
    if isinstance(s, P.BitpackStage):
        return {"type": "Bitpack", "input_type": {1: "uint8", 2: "uint16", 4: "uint32"}[s.elem], "nbits": int(s.nbits)}
    if isinstance(s, P.HuffmanStage):
        d = {"type": "Huffman", "input_type": "uint16", "bklen": int(s.bklen)}
        if s.encode_mode == P.HuffmanEncodeMode.Fine:
            d["encode_mode"] = "Fine"
        return d
    raise ConfigError(f"saveConfig: no TOML form for stage {s.getName()}")


def _esc(v: str) -> str:
    return v.replace("\\", "\\\\").replace('"', '\\"')


def dump_config(pipeline_params: dict, stages: list, connections: list) -> str:
    """TOML text of a pipeline in the layout of the reference's saveConfig
    (config.cpp:645-720): two comment lines, [pipeline], then one [[stage]]
    per stage with its inputs, each table followed by a blank line."""
    names, counts = {}, {}
    for s in stages:
        base = s.getName()
        k = counts.get(base, 0)
        counts[base] = k + 1
        names[id(s)] = base if k == 0 else f"{base}{k}"
    out = ["# FZGPUModules pipeline config",
           "# Generated by Pipeline::saveConfig(). Load with Pipeline::loadConfig().", "", "[pipeline]"]
    for key in ("input_size", "memory_strategy", "pool_multiplier", "num_streams", "dims"):
        if key in pipeline_params:
            v = pipeline_params[key]
            if key == "dims":
                out.append(f"dims = [{', '.join(str(int(d)) for d in v)}]")
            elif key == "pool_multiplier":
                out.append(f"pool_multiplier = {_fmt(_f32(v))}")
            else:
                out.append(f"{key} = {_fmt(v)}")
    out.append("")
    for s in stages:
        out += ["[[stage]]", f"name = \"{_esc(names[id(s)])}\""]
        for k, v in _stage_table(s).items():
            out.append(f"{k} = {_fmt(v)}")
        ins = [(p, port) for (d, p, port) in connections if d is s]
        if ins:
            parts = []
            for p, port in ins:
                e = f"{{ from = \"{_esc(names[id(p)])}\""
                if port != "output":
                    e += f", port = \"{_esc(port)}\""
                parts.append(e + " }")
            out.append("inputs = [" + ", ".join(parts) + "]")
        out.append("")
    return "\n".join(out) + "\n"
