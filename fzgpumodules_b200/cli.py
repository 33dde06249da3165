"""Command-line front end with the reference CLI's options (src/utils/cli/cli.cpp:495-530):

  python -m fzgpumodules_b200.cli -t f32 -m rel -e 1e-3 -i data.f32 -l 3600x1800 -z --report
  python -m fzgpumodules_b200.cli -i data.f32.fzm -x --compare data.f32 --report
  python -m fzgpumodules_b200.cli -c pfpl.toml -i data.f32 -l 512x512x512 -b

-z compresses a raw float32 file into an FZM file (Pipeline::writeToFile), -x decompresses an FZM file
(Pipeline::decompressFromFile) into raw float32, -b times compression and decompression of the file's data.
The pipeline comes from a TOML config (-c) or from --stages, e.g. "lorenzo->bitshuffle->rze" (the default),
"quantizer->diff->bitshuffle->rze", "lorenzo->rle", "lorenzo->huffman".
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time

import numpy as np
import torch

from . import pipeline as P

MODES = {"rel": P.REL, "abs": P.ABS, "noa": P.NOA}


def _dims(s: str | None, n: int):
    if not s:
        return (n, 1, 1)
    d = [int(v) for v in s.lower().split("x")]
    while len(d) < 3:
        d.append(1)
    if d[0] * d[1] * d[2] != n:
        raise SystemExit(f"--len {s} does not match the input's {n} values")
    return tuple(d[:3])


def build_pipeline(args, n: int, dims) -> P.Pipeline:
    """The pipeline the options describe (config file or --stages chain)."""
    pl = P.Pipeline(n * 4, P.PREALLOCATE)
    if args.config:
        pl.setDims(*dims)
        pl.loadConfig(args.config)
        return pl
    pl.setDims(*dims)
    names = [s.strip().lower() for s in args.stages.split("->") if s.strip()]
    prev, port, quant_u32 = None, "output", False
    for name in names:
        if name == "lorenzo":
            s = P.LorenzoQuantStage(args.error_bound, args.radius, 0.2, MODES[args.mode], True)
            nxt = "codes"
        elif name == "quantizer":
            s = P.QuantizerStage(args.error_bound, MODES[args.mode], args.radius, 0.1, code_bytes=4, zigzag_codes=True)
            nxt, quant_u32 = "codes", True
        elif name == "bitshuffle":
            s, nxt = P.BitshuffleStage(args.chunk_size, 2), "output"
        elif name == "rze":
            s, nxt = P.RZEStage(args.chunk_size, args.rze_levels), "output"
        elif name == "diff":
            s, nxt = P.DifferenceStage(P.INT32, P.UINT32, args.chunk_size) if quant_u32 else \
                P.DifferenceStage(P.UINT16, P.UINT16, args.chunk_size), "output"
        elif name == "rle":
            s, nxt = P.RLEStage(4 if quant_u32 else 2), "output"
        elif name == "huffman":
            s, nxt = P.HuffmanStage(1024), "output"
        else:
            raise SystemExit(f"unknown stage \"{name}\" (lorenzo, quantizer, bitshuffle, rze, diff, rle, huffman)")
        pl.addStage(s)
        if prev is not None:
            pl.connect(s, prev, port)
        prev, port = s, nxt
    pl.finalize()
    return pl


def _report(x: np.ndarray, y: np.ndarray, comp_bytes: int):
    d = y.astype(np.float64) - x.astype(np.float64)
    rng = float(x.max() - x.min()) if x.size else 0.0
    mse = float(np.mean(d * d)) if x.size else 0.0
    psnr = 20 * math.log10(rng) - 10 * math.log10(mse) if mse > 0 and rng > 0 else math.inf
    print(f"  ratio:          {x.nbytes / max(comp_bytes, 1):.2f}x")
    print(f"  max abs err:    {float(np.abs(d).max()) if x.size else 0.0:.3e}")
    print(f"  PSNR:           {psnr:.2f} dB")
    print(f"  NRMSE:          {math.sqrt(mse) / rng if rng else 0.0:.3e}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="fzgpumodules_b200.cli")
    mode = ap.add_mutually_exclusive_group(required=True)
    mode.add_argument("-z", "--compress", action="store_true")
    mode.add_argument("-x", "--decompress", action="store_true")
    mode.add_argument("-b", "--benchmark", action="store_true")
    ap.add_argument("-c", "--config")
    ap.add_argument("-R", "--report", action="store_true")
    ap.add_argument("--compare")
    ap.add_argument("--stages", default="lorenzo->bitshuffle->rze")
    ap.add_argument("-m", "--mode", default="rel", choices=list(MODES))
    ap.add_argument("-e", "--error-bound", type=float, default=1e-3)
    ap.add_argument("-t", "--type", default="f32", choices=["f32"])
    ap.add_argument("-r", "--radius", type=int, default=32768)
    ap.add_argument("--chunk-size", type=int, default=16384)
    ap.add_argument("--rze-levels", type=int, default=4)
    ap.add_argument("-l", "--len")
    ap.add_argument("-i", "--input", required=True)
    ap.add_argument("-o", "--output")
    ap.add_argument("--runs", type=int, default=10)
    args = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    if args.decompress:
        t0 = time.perf_counter()
        y = P.Pipeline.decompressFromFile(args.input, device=dev)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        yh = y.cpu().numpy()
        out = args.output or args.input + ".out"
        if args.compare:
            x = np.fromfile(args.compare, dtype=np.float32)
            yh = yh[: x.size]
        yh.tofile(out)
        print(f"decompressed {args.input} -> {out}: {yh.nbytes} bytes in {ms:.3f} ms")
        if args.report and args.compare:
            _report(x, yh, os.path.getsize(args.input))
        return 0
    x = np.fromfile(args.input, dtype=np.float32)
    dims = _dims(args.len, x.size)
    d = torch.from_numpy(x).to(dev)
    pl = build_pipeline(args, x.size, dims)
    if args.compress:
        t0 = time.perf_counter()
        comp = pl.compress(d)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        out = args.output or args.input + ".fzm"
        pl.writeToFile(out)
        print(f"compressed {args.input} -> {out}: {x.nbytes} -> {os.path.getsize(out)} bytes in {ms:.3f} ms "
              f"({x.nbytes / ms / 1e6:.2f} GB/s)")
        if args.report:
            y = pl.decompress()[: x.size].cpu().numpy()
            _report(x, y, comp.numel())
        pl.close()
        return 0
    # benchmark: host-timed calls, as the reference reports them
    comp = pl.compress(d).clone()
    pl.decompress(comp)
    tc, td = [], []
    for _ in range(args.runs):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pl.compress(d)
        torch.cuda.synchronize()
        tc.append((time.perf_counter() - t0) * 1e3)
        t0 = time.perf_counter()
        pl.decompress(comp)
        torch.cuda.synchronize()
        td.append((time.perf_counter() - t0) * 1e3)
    y = pl.decompress(comp)[: x.size].cpu().numpy()
    for name, ts in (("compress", tc), ("decompress", td)):
        m = float(np.mean(ts))
        print(f"{name}:\n  runs:           {args.runs}\n  host ms:        mean={m:.3f}\n"
              f"  throughput:     {x.nbytes / m / 1e6:.2f} GB/s (host mean)")
    if args.report:
        _report(x, y, comp.numel())
    pl.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
