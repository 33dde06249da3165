"""Secondary benchmark workloads (``bench.py --workload ...``), each printed
as one JSON line with the same keys as the headline line:

* ``c1``        LorenzoQuant 2-D (ABS 1e-4) -> RLE on the 1800 x 3600 sinusoid
                field, through fz::Pipeline (the Quick Start chain);
* ``cli``       LorenzoQuant 2-D (REL 1e-3) -> Bitshuffle -> RZE on the same
                1800 x 3600 field through fz::Pipeline: the configuration of the
                reference's only published timing (its CLI documentation);
* ``c3``        LorenzoQuant 2-D (ABS 1e-3, radius 512, zigzag) -> Huffman
                (bklen 1024) on an 8192^2 fractal field, with and without
                the host codebook in the timed region;
* ``batch``     64 fields (log-uniform 1 MB - 256 MB, mixed ranks, REL eb in
                {1e-2, 1e-3, 1e-4}) through the batched chain replayed from one
                CUDA graph, against 64 plain per-field calls;
* ``selector``  2 GiB of mixed fields -> LorenzoQuant (REL 1e-3) codes in 64 KiB
                chunks, coded by exhaustive trial and by the trained MLP selector;
* ``pfpl``      the pfpl preset, Quantizer (REL 1e-3) -> Difference -> Bitshuffle
                -> RZE, on a 512^3 field, as kernels and through fz::Pipeline;
* ``timeline``  a CUPTI timeline (torch.profiler) of fz::Pipeline calls on the
                512^3 chain: host time, GPU busy time, idle gaps and blocking
                calls per call.

Timing: CUDA events on the launching stream after warm-up; inputs larger than
L2 or an L2 flush between timed iterations.
"""
from __future__ import annotations

import json
import time

import numpy as np
import torch

from . import fields as F
from . import kernels as K


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _time(fn, steps: int, warmup: int, flush: torch.Tensor | None = None) -> float:
    """Mean device milliseconds of fn() over `steps` timed calls."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        a, b = _events()
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    return tot / steps


def _line(workload: str, value: float, unit: str, args, extra: dict) -> str:
    d = {"metric": "comp/decomp GB/s and % HBM roofline at fixed eb; ratio, learned vs exhaustive",
         "workload": workload, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "higher_is_better": True, "dtype": "f32", "data": "synthetic"}
    d.update(extra)
    return json.dumps(d)


def run_c1(args, dev):
    from .pipeline import LorenzoQuantStage, Pipeline, RLEStage, ABS, PREALLOCATE
    x = F.sinusoids2d(1800, 3600, seed=1001, device=dev).reshape(-1)
    n = x.numel()
    pl = Pipeline(n * 4, PREALLOCATE)
    pl.setDims(3600, 1800, 1)
    lq = pl.addStage(LorenzoQuantStage(1e-4, 32768, 0.2, ABS, False))
    rle = pl.addStage(RLEStage(2))
    pl.connect(rle, lq, "codes")
    pl.finalize()
    comp = pl.compress(x).clone()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    tc = _time(lambda: pl.compress(x), args.steps, args.warmup, flush)
    td = _time(lambda: pl.decompress(comp), args.steps, args.warmup, flush)
    y = pl.decompress(comp)[:n]
    err = float((y - x).abs().max())
    pl.close()
    return _line("c1: LorenzoQuant2D(ABS 1e-4)->RLE, 1800x3600 sinusoids, fz::Pipeline", 4 * n / tc / 1e6,
                 "GB/s", args, {"compress_ms": tc, "decompress_ms": td, "decompress_gbs": 4 * n / td / 1e6,
                                "ratio": 4 * n / comp.numel(), "max_abs_err": err,
                                "note": "Pipeline calls include their host synchronisation, as the reference's do"})


def run_cli(args, dev):
    from .pipeline import (LorenzoQuantStage, Pipeline, BitshuffleStage, RZEStage, REL, PREALLOCATE)
    x = F.sinusoids2d(1800, 3600, seed=1001, device=dev).reshape(-1)
    n = x.numel()
    pl = Pipeline(n * 4, PREALLOCATE)
    pl.setDims(3600, 1800, 1)
    lq = pl.addStage(LorenzoQuantStage(1e-3, 32768, 0.2, REL, True))
    bs = pl.addStage(BitshuffleStage(16384, 2))
    rz = pl.addStage(RZEStage(16384, 4))
    pl.connect(bs, lq, "codes")
    pl.connect(rz, bs, "output")
    pl.finalize()
    comp = pl.compress(x).clone()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    tc = _time(lambda: pl.compress(x), args.steps, args.warmup, flush)
    td = _time(lambda: pl.decompress(comp), args.steps, args.warmup, flush)
    y = pl.decompress(comp)[:n]
    err = float((y - x).abs().max())
    vb = float(x.abs().max())
    pl.close()
    return _line("cli: LorenzoQuant2D(REL 1e-3, zigzag)->Bitshuffle(16384,ew2)->RZE(16384,4), 1800x3600 sinusoids, fz::Pipeline",
                 4 * n / tc / 1e6, "GB/s", args,
                 {"compress_ms": tc, "decompress_ms": td, "decompress_gbs": 4 * n / td / 1e6, "ratio": 4 * n / comp.numel(),
                  "max_abs_err": err, "abs_eb": 1e-3 * vb,
                  "published_reference": {"compress_gbs_host": 18.85, "compress_gbs_dag": 40.1, "decompress_gbs_host": 14.85,
                                          "decompress_gbs_dag": 19.6, "hardware": "unstated", "input": "CESM CLDHGH 1800x3600",
                                          "source": "docs/cli.md:61-77"},
                  "note": "calls include their host synchronisation, as the reference's host timing does"})


def _peak():
    """Measured HBM copy bandwidth (GB/s) of this GPU pool, or None."""
    import json as _j
    import os as _o
    try:
        with open(_o.path.join(_o.path.dirname(_o.path.dirname(_o.path.abspath(__file__))), "MEASURED_PEAKS.json")) as f:
            return float(_j.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_per_element(kernel: str):
    """DRAM bytes per element of `kernel` from the committed ncu summary
    (profiles/traffic.json), or None."""
    import json as _j
    import os as _o
    try:
        with open(_o.path.join(_o.path.dirname(_o.path.dirname(_o.path.abspath(__file__))), "profiles",
                               "traffic.json")) as f:
            return float(_j.load(f)[kernel]["bytes_per_element"])
    except Exception:
        return None


def c3_summary(dev, steps: int, warmup: int) -> dict:
    """C3: LorenzoQuant 2-D (ABS 1e-3, radius 512, zigzag) -> Huffman (bklen
    1024, coarse) on the 8192^2 fractal field.  Times each step, checks the
    decode, and gives the Huffman decode kernel's roofline: algorithmic bytes
    = blob read + 2 B per code written, over the kernel's own event time;
    traffic = the committed ncu DRAM bytes per code, scaled to n."""
    x = F.fractal2d(8192, seed=1003, device=dev).reshape(-1)
    n = x.numel()
    dims = (8192, 8192, 1)
    ws = K.Workspace()
    out = K.lq_forward(x, dims, 1e-3, K.ABS, 512, True, 0.2, ws=ws)
    codes = out["codes"]
    hws = K.Workspace()
    blob, size = K.huff_compress(codes, 1024, ws=hws)
    freq = K.huff_histogram(codes, 1024)
    bk4, rb = K.huff_book(freq, 1024)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    t_lq = _time(lambda: K.lq_forward(x, dims, 1e-3, K.ABS, 512, True, 0.2, ws=ws), steps, warmup, flush)
    t_hist = _time(lambda: K.huff_histogram(codes, 1024), steps, warmup, flush)
    t_enc = _time(lambda: K.huff_encode(codes, bk4, rb, 1024, ws=hws, trim=False), steps, warmup, flush)
    t_full = _time(lambda: K.huff_compress(codes, 1024, ws=hws, trim=False), steps, warmup, flush)
    dec = torch.empty(n, dtype=torch.uint16, device=dev)
    t_dec = _time(lambda: K.huff_decode(blob, n, 1024, ws=hws, out=dec), steps, warmup, flush)
    with K.Trace():
        for _ in range(steps):
            flush.zero_()
            K.huff_histogram(codes, 1024)
            flush.zero_()
            K.huff_encode(codes, bk4, rb, 1024, ws=hws, trim=False)
            flush.zero_()
            K.huff_decode(blob, n, 1024, ws=hws, out=dec)
        torch.cuda.synchronize()
        kern = K.Trace.kernels()
    t0 = time.perf_counter()
    for _ in range(10):
        K.huff_book(freq, 1024)
    t_book = (time.perf_counter() - t0) / 10 * 1e3
    ok = bool(torch.equal(K.huff_decode(blob, n, 1024), codes))
    comp_bytes = blob.numel() + 8 * min(int(out["count"].item()), out["cap"]) + 4
    dk = next((k for k in kern if k.startswith("hf_decode")), None)
    peak, kind = _peak()
    roof = None
    if dk:
        launches, ms = kern[dk]
        kms = ms / launches
        algo = blob.numel() + 2 * n
        ach = algo / kms / 1e6
        per = _traffic_per_element("hf_decode")
        roof = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": per * n if per else None, "algorithmic_bytes": algo, "peak_kind": kind, "kernel": dk,
                "kernel_ms": kms, "launches": launches}
    return {"workload": "LorenzoQuant2D(ABS 1e-3, r512, zigzag)->Huffman(1024, coarse), 8192^2 fractal",
            "compress_gbs": 4 * n / (t_lq + t_full) / 1e6, "compress_gbs_without_book": 4 * n / (t_lq + t_hist + t_enc) / 1e6,
            "lq_ms": t_lq, "huffman_histogram_ms": t_hist, "huffman_book_host_ms": t_book,
            "huffman_encode_ms": t_enc, "huffman_compress_ms_with_book": t_full, "huffman_decode_ms": t_dec,
            "decode_gbs_codes": 2 * n / t_dec / 1e6, "ratio": 4 * n / comp_bytes,
            "bits_per_code": 8 * blob.numel() / n, "decode_identical": ok,
            "kernels_ms": {k: round(ms / cnt, 4) for k, (cnt, ms) in sorted(kern.items())}, "roofline": roof}


def run_c3(args, dev):
    d = c3_summary(dev, args.steps, args.warmup)
    return _line("c3: " + d.pop("workload"), d["compress_gbs"], "GB/s", args, d)


def batch_fields(dev, count=64, seed=1004, max_mb=256):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nbytes = int(np.exp(rng.uniform(np.log(1 << 20), np.log(max_mb << 20))))
        n = max(nbytes // 4, 1024)
        rank = int(rng.integers(1, 4))
        if rank == 1:
            dims = (n, 1, 1)
        elif rank == 2:
            nx = int(rng.choice([256, 512, 1000, 1024, 2048, 3000]))
            dims = (nx, max(n // nx, 2), 1)
        else:
            nx = int(rng.choice([64, 128, 200, 256, 512]))
            ny = int(rng.choice([64, 128, 256]))
            dims = (nx, ny, max(n // (nx * ny), 2))
        shape = tuple(d for d in reversed(dims) if d > 1) or (dims[0],)
        x = F.grf(shape, seed=seed + i, spike_frac=1e-3, device=dev).reshape(-1).contiguous()
        out.append(dict(x=x, dims=dims, eb=float(rng.choice([1e-2, 1e-3, 1e-4])), mode=K.REL, radius=32768,
                        zigzag=True, outlier_capacity=0.1))
    return out


def _slab_field(f) -> bool:
    """A field the single-field call (and the batch) codes with a slab kernel."""
    nx, ny, nz = f["dims"]
    return (nz > 1 and 32 <= nx <= 1024 and nx & (nx - 1) == 0 and ny % (8192 // nx) == 0
            and f["x"].numel() == nx * ny * nz)


def batch_summary(dev, steps: int, warmup: int) -> dict:
    """C4: the 64-field batch (batch_fields) as one graph-captured launch
    sequence against 64 plain calls, bytes compared field by field."""
    fields = batch_fields(dev)
    total = sum(f["x"].numel() * 4 for f in fields)
    b = K.Batch(fields)
    best, tune_ms = b.autotune()
    s = torch.cuda.Stream(device=dev)
    b.launch(s)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.launch(s)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    t_batch = _time(lambda: g.replay(), steps, warmup, flush)
    ws = K.Workspace()
    plain_out = [None] * len(fields)

    def plain():
        for i, f in enumerate(fields):
            plain_out[i] = K.lq_bs_rze_compress(f["x"], f["dims"], f["eb"], f["mode"], f["radius"], f["zigzag"],
                                                f["outlier_capacity"], ws=ws, out=plain_out[i])
    t_plain = _time(plain, steps, warmup, flush)
    torch.cuda.synchronize()
    same = all(int(o["rze_size"].item()) == int(p["rze_size"].item()) and
               torch.equal(o["rze"][: int(o["rze_size"].item())], p["rze"][: int(p["rze_size"].item())])
               for o, p in zip(b.outputs, plain_out))
    comp = sum(int(o["rze_size"].item()) + 8 * min(int(o["count"].item()), o["cap"]) + 4 for o in b.outputs)
    del g
    b.close()
    return {"workload": "64 fields 1-256 MB, mixed rank, REL {1e-2,1e-3,1e-4}, LQ->BS->RZE",
            "gbs": total / t_batch / 1e6, "batched_ms": t_batch, "plain_ms": t_plain,
            "plain_gbs": total / t_plain / 1e6, "speedup_vs_plain": t_plain / t_batch, "bytes_identical": same,
            "tuning": {"ctas_per_sm": best.ctas_per_sm, "order": best.order, "flat_tiles": best.flat_tiles,
                       "scan_parts": best.scan_parts}, "autotune_best_ms": tune_ms,
            "total_bytes": total, "ratio": total / comp, "launches_per_batch": 5 + sum(map(_slab_field, fields))}


def run_batch(args, dev):
    d = batch_summary(dev, args.steps, args.warmup)
    return _line("batch: " + d.pop("workload"), d.pop("gbs"), "GB/s", args, d)


def selector_summary(dev, steps: int, warmup: int, train_chunks: int = 1 << 20) -> dict:
    """C5: 2 GiB of mixed fields -> LorenzoQuant (REL 1e-3) codes in 64 KiB
    chunks, coded by exhaustive trial and by the MLP selector trained on
    `train_chunks` method-generated chunks (other seeds and field shape than
    the test data) with the library's own kernels."""
    from . import selector as S
    kinds = ("smooth", "piecewise", "noise", "sparse")
    codes = []
    for i in range(32):  # 2 GiB: 32 fields of 64 MiB (256^3), eight per kind
        x = F.mixed_field(kinds[i % 4], (256, 256, 256), 1005 + i, device=dev)
        codes.append(K.lq_forward(x, (256, 256, 256), 1e-3, K.REL, 32768, True, 0.2)["codes"])
        del x
    codes = torch.cat(codes)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    X, T = S.method_training_set(train_chunks, seed=500, device=dev)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    sel = S.CoderSelector(seed=0, device=dev)
    epochs = 60 if train_chunks <= 16384 else 12
    batch = 256 if train_chunks <= 16384 else 4096
    t0 = time.perf_counter()
    losses = sel.train(X, T, epochs=epochs, batch=batch, lr=3e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del X, T
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    t_ex = _time(lambda: S.encode(codes, S.EXHAUSTIVE, trim=False), steps, warmup, flush)
    t_le = _time(lambda: S.encode(codes, S.LEARNED, sel, trim=False), steps, warmup, flush)
    with K.Trace():
        S.encode(codes, S.LEARNED, sel, trim=False)
        torch.cuda.synchronize()
        learned_kernels = {k: round(v[1], 3) for k, v in K.Trace.kernels().items()}
    pre = codes[: 1 << 22]  # decode runs a host loop per chunk: check a 128-chunk prefix
    blob, _ = S.encode(pre, S.LEARNED, sel)
    ok = bool(torch.equal(S.decode(blob, pre.numel()), pre))
    r = S.compare(codes, sel)
    nbytes = codes.numel() * 2
    return {"workload": "2 GiB mixed fields -> LQ(REL 1e-3) codes, 64 KiB chunks, MLP 16-64-64-4",
            "learned_gbs": nbytes / t_le / 1e6, "exhaustive_gbs": nbytes / t_ex / 1e6,
            "learned_ms": t_le, "exhaustive_ms": t_ex, "speedup_vs_exhaustive": t_ex / t_le,
            "ratio_learned": r["ratio_learned"], "ratio_exhaustive": r["ratio_exhaustive"],
            "ratio_best_fixed": r["ratio_best_fixed"],
            "learned_over_exhaustive": r["ratio_learned"] / r["ratio_exhaustive"],
            "gain_over_best_fixed": r["ratio_learned"] / r["ratio_best_fixed"],
            "choice_agreement": r["agreement"], "train_chunks": int(train_chunks),
            "train_generate_seconds": t_gen, "train_seconds": t_train, "train_epochs": epochs,
            "final_loss": losses[-1], "held_out": "test fields use other seeds and a 256^3 shape",
            "chunks": int(S.nchunks(codes.numel())), "learned_kernel_ms": learned_kernels,
            "decode_prefix_identical": ok, "bytes_unit": "GB/s of 16-bit codes (2 B per value)"}


def run_selector(args, dev):
    d = selector_summary(dev, args.steps, args.warmup, getattr(args, "train_chunks", 1 << 20))
    return _line("selector: " + d.pop("workload"), d["learned_gbs"], "GB/s", args, d)


PFPL_DIMS = (512, 512, 512)


def pfpl_field(dev, dims=PFPL_DIMS):
    """The pfpl workload's input: a Gaussian random field (512^3 by default)
    with 0.1 % spikes; dims are (x, y, z)."""
    return F.grf(tuple(dims)[::-1], seed=1006, spike_frac=1e-3, device=dev).reshape(-1)


def run_pfpl(args, dev):
    """The pfpl preset (examples/presets/pfpl.toml): Quantizer(REL 1e-3, u32
    codes, zigzag, outlier capacity 0.1) -> Difference(int32 -> uint32,
    16 KiB chunks) -> Bitshuffle(16384, ew 2) -> RZE(16384, 4), as the stage
    kernels run back to back on device-resident data and through fz::Pipeline."""
    from .pipeline import (BitshuffleStage, DifferenceStage, Pipeline, QuantizerStage, RZEStage, INT32, PREALLOCATE,
                           REL, UINT32)
    dims = tuple(getattr(args, "dims", PFPL_DIMS))
    x = pfpl_field(dev, dims)
    n = x.numel()
    wq, wd, wr = K.Workspace(), K.Workspace(), K.Workspace()
    q = K.quantizer_forward(x, 1e-3, K.REL, 32768, 4, True, 0.1, ws=wq)
    rze, size = K.rze_encode(K.bitshuffle(K.diff(q["codes"], 16384, True, ws=wd), 16384, 2), ws=wr)
    comp_bytes = rze.numel() + 8 * int(q["count"].item()) + 4

    def comp():
        K.quantizer_forward(x, 1e-3, K.REL, 32768, 4, True, 0.1, ws=wq, out=q, check_status=False)
        d = K.diff(q["codes"], 16384, True, ws=wd)
        K.rze_encode(K.bitshuffle(d, 16384, 2), ws=wr, trim=False)

    def decomp():
        b = K.bitshuffle(K.rze_decode(rze, 4 * n, ws=wr), 16384, 2, inverse=True)
        c = K.diff(b.view(torch.int32), 16384, True, inverse=True, ws=wd)
        return K.quantizer_inverse(c, 1e-3, K.REL, 0.0, 32768, True, vals=q["vals"], idx=q["idx"],
                                   count=q["count"], cap=q["cap"])

    y = decomp()
    rel_ok = bool(((y.double() - x.double()).abs() <= x.double().abs() * 1e-3 * 1.01).all())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    tc = _time(comp, args.steps, args.warmup, flush)
    td = _time(decomp, args.steps, args.warmup, flush)
    assert wq.status() == 0 and wr.status() == 0
    # the one-pass chain (fzb_pfpl_compress / fzb_pfpl_decompress)
    wf, wf2 = K.Workspace(), K.Workspace()
    f = K.pfpl_compress(x, 1e-3, K.REL, 32768, True, 0.1, ws=wf)
    fsize = int(f["rze_size"].item())
    same = fsize == rze.numel() and bool(torch.equal(f["rze"][:fsize], rze))
    yf = torch.empty_like(x)

    def fcomp():
        K.pfpl_compress(x, 1e-3, K.REL, 32768, True, 0.1, ws=wf, out=f)

    def fdecomp():
        K.pfpl_decompress(f["rze"], fsize, f["vals"], f["idx"], f["count"], f["cap"], n, ws=wf2, out=yf)

    fdecomp()
    fused_equal = bool(torch.equal(yf.view(torch.int32), y.view(torch.int32)))
    tfc = _time(fcomp, args.steps, args.warmup, flush)
    tfd = _time(fdecomp, args.steps, args.warmup, flush)
    assert wf2.status() == 0
    per_kernel = {}
    for fn in (comp, decomp, fcomp, fdecomp):
        with K.Trace():
            for _ in range(args.steps):
                flush.zero_()
                fn()
            torch.cuda.synchronize()
            for k, (launches, ms) in K.Trace.kernels().items():
                per_kernel[k] = round(ms / launches, 4)
    # through fz::Pipeline (each call includes the pipeline's host synchronisation)
    pl = Pipeline(n * 4, PREALLOCATE)
    qs = pl.addStage(QuantizerStage(1e-3, REL, 32768, 0.1, code_bytes=4, zigzag_codes=True))
    ds = pl.addStage(DifferenceStage(INT32, UINT32, 16384))
    bs = pl.addStage(BitshuffleStage(16384, 2))
    rz = pl.addStage(RZEStage(16384, 4))
    pl.connect(ds, qs, "codes")
    pl.connect(bs, ds)
    pl.connect(rz, bs)
    pl.finalize()
    cp = pl.compress(x).clone()
    tpc = _time(lambda: pl.compress(x), args.steps, args.warmup, flush)
    tpd = _time(lambda: pl.decompress(), args.steps, args.warmup, flush)
    pl.close()
    # the speed preset's chain (Quantizer REL, capacity 0.05 -> Bitshuffle ew 4 -> RZE) through fz::Pipeline
    sp = Pipeline(n * 4, PREALLOCATE)
    sq = sp.addStage(QuantizerStage(1e-3, REL, 32768, 0.05, code_bytes=4, zigzag_codes=True))
    sb = sp.addStage(BitshuffleStage(16384, 4))
    sr = sp.addStage(RZEStage(16384, 4))
    sp.connect(sb, sq, "codes")
    sp.connect(sr, sb)
    sp.finalize()
    scp = sp.compress(x).clone()
    tsc = _time(lambda: sp.compress(x), args.steps, args.warmup, flush)
    tsd = _time(lambda: sp.decompress(), args.steps, args.warmup, flush)
    sp.close()
    peak = None
    try:
        import json as _j
        import os as _o
        with open(_o.path.join(_o.path.dirname(_o.path.dirname(_o.path.abspath(__file__))), "MEASURED_PEAKS.json")) as f:
            peak = float(_j.load(f)["hbm_gbs"])
    except Exception:
        peak = None
    qf = per_kernel.get("quantizer_fwd")
    q_gbs = 8 * n / qf / 1e6 if qf else None  # 4 B read + 4 B code written per value
    ck, dk = per_kernel.get("pfpl_chunk"), per_kernel.get("pfpl_decode")
    # algorithmic bytes: the field read (written) plus the compressed stream written (read)
    ck_gbs = (4 * n + comp_bytes) / ck / 1e6 if ck else None
    dk_gbs = (4 * n + comp_bytes) / dk / 1e6 if dk else None
    return _line("pfpl: Quantizer(REL 1e-3, u32, zigzag)->Difference(i32->u32, 16 KiB)->Bitshuffle(16384, ew2)->RZE, "
                 + "x".join(map(str, dims)) + " GRF", 4 * n / tfc / 1e6, "GB/s", args,
                 {"fused_compress_ms": tfc, "fused_decompress_ms": tfd, "fused_decompress_gbs": 4 * n / tfd / 1e6,
                  "fused_bytes_equal_staged": same, "fused_values_equal_staged": fused_equal,
                  "pfpl_chunk_gbs": ck_gbs, "pfpl_chunk_frac_of_measured_hbm": (ck_gbs / peak) if (ck_gbs and peak) else None,
                  "pfpl_decode_gbs": dk_gbs, "pfpl_decode_frac_of_measured_hbm": (dk_gbs / peak) if (dk_gbs and peak) else None,
                  "staged_compress_ms": tc, "staged_decompress_ms": td, "staged_compress_gbs": 4 * n / tc / 1e6,
                  "staged_decompress_gbs": 4 * n / td / 1e6,
                  "pipeline_compress_gbs": 4 * n / tpc / 1e6, "pipeline_decompress_gbs": 4 * n / tpd / 1e6,
                  "pipeline_compressed_bytes": cp.numel(), "ratio": 4 * n / comp_bytes,
                  "speed_pipeline_compress_gbs": 4 * n / tsc / 1e6, "speed_pipeline_decompress_gbs": 4 * n / tsd / 1e6,
                  "speed_compressed_bytes": scp.numel(),
                  "outliers": int(q["count"].item()), "rel_bound_held": rel_ok, "kernel_ms": per_kernel,
                  "quantizer_fwd_gbs": q_gbs, "quantizer_fwd_frac_of_measured_hbm": (q_gbs / peak) if (q_gbs and peak) else None,
                  "note": "value: the one-pass chain on device-resident data; staged_*: the four stage kernels back to "
                          "back; pipeline_* through fz::Pipeline (which runs the one-pass chain; host syncs included)"})


def _kname(name: str) -> str:
    """A kernel's name without its return type, namespaces' anonymous parts
    and parameter list."""
    n = name.replace("void ", "").replace("(anonymous namespace)::", "")
    return n.split("(")[0][:60].strip()


def pipeline_timeline(dev, calls: int = 3) -> dict:
    """Where the time of a fz::Pipeline call goes, from a CUPTI timeline
    (torch.profiler) of `calls` compress and decompress calls of the 512^3
    LQ3D(REL 1e-3) -> Bitshuffle -> RZE chain (PREALLOCATE), each after an L2
    flush: per call its host duration, the host time before the first GPU
    operation, the GPU busy time and the idle gaps between GPU operations,
    the time from the last GPU operation's end to the call's return, and the
    blocking calls it made (stream / device synchronisations, synchronous
    copies).  Kernel names and durations are listed for the last call."""
    from torch.profiler import ProfilerActivity, profile, record_function

    from .pipeline import PREALLOCATE, REL, BitshuffleStage, LorenzoQuantStage, Pipeline, RZEStage
    x = F.grf((512, 512, 512), seed=1002, spike_frac=1e-3, device=dev).reshape(-1)
    n = x.numel()
    pl = Pipeline(4 * n, PREALLOCATE)
    pl.setDims(512, 512, 512)
    lq = pl.addStage(LorenzoQuantStage(1e-3, 32768, 0.1, REL, True))
    bs = pl.addStage(BitshuffleStage(16384, 2))
    rz = pl.addStage(RZEStage(16384, 4))
    pl.connect(bs, lq, "codes")
    pl.connect(rz, bs)
    pl.finalize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(3):
        pl.compress(x)
        pl.decompress(None)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CPU, ProfilerActivity.CUDA]) as prof:
        for i in range(calls):
            flush.zero_()
            torch.cuda.synchronize()
            with record_function(f"call:compress:{i}"):
                pl.compress(x)
            flush.zero_()
            torch.cuda.synchronize()
            with record_function(f"call:decompress:{i}"):
                pl.decompress(None)
    pl.close()
    import os
    import tempfile
    fd, path = tempfile.mkstemp(suffix=".json")
    os.close(fd)
    try:
        prof.export_chrome_trace(path)
        with open(path) as f:
            trace = json.load(f)
    finally:
        os.remove(path)
    ev = [e for e in trace.get("traceEvents", []) if e.get("ph") == "X"]
    calls_ev = [e for e in ev if str(e.get("name", "")).startswith("call:")]
    gpu = sorted((e["ts"], e["ts"] + e["dur"], e["name"]) for e in ev
                 if e.get("cat") in ("kernel", "gpu_memcpy", "gpu_memset"))
    api = [(e["ts"], e["ts"] + e["dur"], e["name"]) for e in ev if e.get("cat") == "cuda_runtime"]
    out = {}
    for c in sorted(calls_ev, key=lambda e: e["ts"]):
        kind = c["name"].split(":")[1]
        t0, t1 = c["ts"], c["ts"] + c["dur"]
        g = [k for k in gpu if t0 <= k[0] < t1]
        if not g:
            continue
        busy = sum(k[1] - k[0] for k in g)
        gaps, end = 0.0, g[0][1]
        for k in g[1:]:
            gaps += max(0.0, k[0] - end)
            end = max(end, k[1])
        blocking = [a[2] for a in api if t0 <= a[0] < t1 and ("Synchronize" in a[2] or a[2] == "cudaMemcpy")]
        rec = {"call_us": t1 - t0, "host_before_first_gpu_op_us": g[0][0] - t0, "gpu_busy_us": busy,
               "gpu_gaps_us": gaps, "last_gpu_end_to_return_us": t1 - end,
               "gpu_ops": len(g), "blocking_calls": {b: blocking.count(b) for b in sorted(set(blocking))},
               "kernels_us": [[_kname(k[2]), round(k[1] - k[0], 1)] for k in g]}
        out.setdefault(kind, []).append(rec)
    summary = {}
    for kind, recs in out.items():
        m = {k: float(np.mean([r[k] for r in recs])) for k in
             ("call_us", "host_before_first_gpu_op_us", "gpu_busy_us", "gpu_gaps_us", "last_gpu_end_to_return_us")}
        m["gpu_ops"] = recs[-1]["gpu_ops"]
        m["blocking_calls"] = recs[-1]["blocking_calls"]
        m["kernels_us_last_call"] = recs[-1]["kernels_us"]
        m["gbs_by_call"] = 4 * n / m["call_us"] / 1e3
        summary[kind] = m
    return summary


def run_timeline(args, dev):
    d = pipeline_timeline(dev, max(1, min(args.steps, 5)))
    v = d.get("compress", {}).get("gbs_by_call", 0.0)
    return _line("timeline: fz::Pipeline LQ3D(REL 1e-3)->Bitshuffle->RZE 512^3, CUPTI timeline of each call",
                 v, "GB/s", args, {"calls": d, "note": "host clock of the profiled calls (profiler overhead "
                                   "included); the breakdown, not the value, is the point"})


WORKLOADS = {"c1": run_c1, "cli": run_cli, "c3": run_c3, "batch": run_batch, "selector": run_selector,
             "pfpl": run_pfpl, "timeline": run_timeline}
