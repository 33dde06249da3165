"""Benchmark of the LorenzoQuant(3-D, REL 1e-3, radius 32768, zigzag) ->
Bitshuffle(16 KiB, element width 2) -> RZE(16 KiB, 4 levels) chain on a
512^3 FP32 field (seeded Gaussian random field, P(k) ~ k^-3, mean 0, std 1,
0.1% of cells set to +-1e3).

One step = one compression and one decompression of the field, inputs
resident in HBM.  `value` is the compression throughput (uncompressed bytes /
device time of the fused C-ABI call); beside it in the same JSON line:
  decompress       the decompression throughput and its kernel roofline;
  roofline         the compress kernel against the measured HBM peak;
  pipeline         the same chain through this library's fz::Pipeline, each
                   compress / decompress call timed with CUDA events around
                   it (its host synchronisation included), as the reference
                   arm times the reference's own Pipeline;
  e2e              fz::Pipeline with host buffers: H2D of the field,
                   compress, D2H of the container; H2D of the container,
                   decompress, D2H of the field; streamed (step k+1's
                   upload overlaps step k's coding and read-back);
  c3               LorenzoQuant 2-D -> Huffman on 8192^2, with the Huffman
                   decode kernel's roofline;
  batch            64 fields of mixed rank and size as one graph-captured
                   launch sequence, against 64 plain calls;
  selector         the learned per-chunk coder selector against exhaustive
                   trial on 2 GiB of mixed fields (the metric's "ratio,
                   learned vs exhaustive");
  cpu_baseline     the oracle chain on the host cores, on the same field;
  clocks           nvidia-smi samples taken during the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload c1|cli|c3|batch|selector|pfpl|timeline   (secondary
      workloads, one JSON line each; fzgpumodules_b200/benchmarks.py;
      --impl reference --workload pfpl times the reference's own pipeline)

Under torchrun each rank compresses its own field (no data exchange: the
path shards by field); timings are maxed over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

DEFAULT_DIMS = (512, 512, 512)
EB, RADIUS, ZIGZAG, OUTLIER_CAP = 1e-3, 32768, True, 0.1
SEED = 1002
METRIC = "comp/decomp GB/s and % HBM roofline at fixed eb; ratio, learned vs exhaustive"
WORKLOAD = ("LorenzoQuant3D(REL 1e-3, r 32768, zigzag)->Bitshuffle(16384,ew2)->RZE(16384,4) "
            "on 512^3 f32 GRF k^-3 + 0.1% +-1e3 spikes")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 6:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max((float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def dist_setup():
    """One process per GPU under torchrun: NCCL on GPU boxes, gloo where no
    GPU is present (the multi-rank host logic is tested that way)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- CPU side

def host_field(dims, rank: int = 0):
    """The benchmark field as a host float32 array: generated on the GPU,
    so it holds the same values the GPU arm compresses, when one is present."""
    import torch

    from fzgpumodules_b200 import fields
    nx, ny, nz = dims
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    return fields.grf((nz, ny, nx), seed=SEED + rank, spike_frac=1e-3, device=dev).reshape(-1).cpu().numpy()


def cpu_baseline(x, dims, steps: int = 1):
    """The oracle chain (an OpenMP C restatement of the reference's stage
    math) on the host cores, on the whole field `x` (host float32, x
    fastest): value base, LorenzoQuant 3-D, Bitshuffle and RZE, then the
    inverse chain; median seconds of `steps` runs."""
    import numpy as np

    from oracle import oracle as O
    cap = int(np.ceil(x.size * OUTLIER_CAP))
    O.lib()
    tc, td = [], []
    size = 0
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        vb = O.value_base(x, O.REL)
        abs_eb, r, e2 = O.resolve_eb(EB, O.REL, vb)
        codes, err, idx, cnt = O.lq_fwd(x, dims, r, RADIUS, ZIGZAG, cap=cap)
        stream = O.rze_encode(O.bitshuffle(codes, 16384, 2))
        t1 = time.perf_counter()
        c2 = O.bitshuffle(O.rze_decode(stream), 16384, 2, inverse=True).view(np.uint16)
        O.lq_inv(c2, err, idx, dims, e2, ZIGZAG)
        t2 = time.perf_counter()
        tc.append(t1 - t0)
        td.append(t2 - t1)
        size = stream.size + 8 * len(idx) + 4
    nbytes = x.size * 4
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"compress_gbs": nbytes / np.median(tc) / 1e9, "decompress_gbs": nbytes / np.median(td) / 1e9,
            "cores": cores, "sample": "the whole " + "x".join(map(str, dims)) +
            f" field ({nbytes >> 20} MiB), oracle chain, same values as the GPU arm", "ratio": nbytes / size}


def _cpu_2d(x2d, chain: str, eb: float, mode: int, radius: int, zigzag: bool):
    """The oracle on one 2-D field (host cores): compress and decompress GB/s,
    median of three runs."""
    import numpy as np

    from oracle import oracle as O
    O.lib()
    x = np.ascontiguousarray(x2d.reshape(-1).numpy())
    ny, nx = x2d.shape
    dims = (nx, ny, 1)
    cap = int(np.ceil(x.size * 0.2))
    tc, td = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        vb = O.value_base(x, mode) if mode else 0.0
        abs_eb, r, e2 = O.resolve_eb(eb, mode, vb)
        codes, err, idx, cnt = O.lq_fwd(x, dims, r, radius, zigzag, cap=cap)
        if chain == "rle":
            s = O.rle_encode(codes)
        elif chain == "bsrze":
            s = O.rze_encode(O.bitshuffle(codes, 16384, 2))
        else:
            freq, _ = O.histogram(codes, 1024)
            bk4, rb = O.huff_book(freq, 1024)
            s = O.huff_encode(codes, 1024, bk4, rb)
        t1 = time.perf_counter()
        if chain == "rle":
            c2 = O.rle_decode(s, x.size)
        elif chain == "bsrze":
            c2 = O.bitshuffle(O.rze_decode(s), 16384, 2, inverse=True).view(np.uint16)
        else:
            c2 = O.huff_decode(s, x.size)
        O.lq_inv(c2, err, idx, dims, e2, zigzag)
        t2 = time.perf_counter()
        tc.append(t1 - t0)
        td.append(t2 - t1)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": x.size * 4 / np.median(tc) / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
            "decompress_gbs": x.size * 4 / np.median(td) / 1e9, "sample": f"the whole {ny}x{nx} field, oracle chain"}


def _cpu_c1():
    from fzgpumodules_b200 import fields
    from oracle import oracle as O
    return _cpu_2d(fields.sinusoids2d(1800, 3600, seed=1001), "rle", 1e-4, O.ABS, 32768, False)


def _cpu_cli():
    from fzgpumodules_b200 import fields
    from oracle import oracle as O
    return _cpu_2d(fields.sinusoids2d(1800, 3600, seed=1001), "bsrze", 1e-3, O.REL, 32768, True)


def _cpu_c3():
    from fzgpumodules_b200 import fields
    from oracle import oracle as O
    return _cpu_2d(fields.fractal2d(8192, seed=1003), "huff", 1e-3, O.ABS, 512, True)


CPU_WORKLOADS = {"c1": _cpu_c1, "cli": _cpu_cli, "c3": _cpu_c3}


def run_reference(args, world, rank):
    """The reference arm: the reference's stage math on the host cores (the
    reference ships no CPU implementation of this path, so the oracle port),
    on the same field and configuration as this library's arm."""
    if rank != 0:
        return
    import numpy as np
    dims = tuple(args.dims)
    x = host_field(dims)
    res = [cpu_baseline(x, dims, 1) for _ in range(args.warmup + args.steps)][args.warmup:]
    comp = float(np.median([r["compress_gbs"] for r in res]))
    dec = float(np.median([r["decompress_gbs"] for r in res]))
    line = {"metric": METRIC, "value": comp, "unit": "GB/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": _config(dims, 1), "same_config": True,
            "decompress": {"value": dec, "unit": "GB/s"},
            "cpu_baseline": {"value": comp, "unit": "GB/s", "cores": res[0]["cores"], "kind": "port",
                             "sample": res[0]["sample"]},
            "e2e": {"value": comp, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["reference_gpu_pipeline"] = _reference_gpu_lq(args)
    print(json.dumps(line), flush=True)


def _reference_gpu_lq(args):
    """For comparison beside the CPU arm: the reference's own GPU pipeline
    (built from its sources into oracle/_ref) on the full 512^3 workload,
    each Pipeline::compress / decompress call timed with CUDA events."""
    import ctypes as C
    path = os.path.join(ROOT, "oracle", "_ref", "libfzref_pipe.so")
    try:
        import torch
        if not torch.cuda.is_available() or not os.path.exists(path):
            return {"unavailable": "no GPU or no reference pipeline build"}
        from fzgpumodules_b200 import fields
        nx, ny, nz = tuple(args.dims)
        x = fields.grf((nz, ny, nx), seed=SEED, spike_frac=1e-3, device=torch.device("cuda", 0)).reshape(-1)
        L = C.CDLL(path)
        L.ref_pipe_last_error.restype = C.c_char_p
        cm, dm, cb = C.c_float(0), C.c_float(0), C.c_size_t(0)
        steps = max(1, min(args.steps, 10))
        if L.ref_pipeline_time_lq(C.c_void_p(x.data_ptr()), C.c_size_t(nx), C.c_size_t(ny), C.c_size_t(nz),
                                  C.c_float(EB), steps, 3, C.byref(cm), C.byref(dm), C.byref(cb)) != 0:
            return {"unavailable": L.ref_pipe_last_error().decode()}
        nbytes = 4 * x.numel()
        return {"compress_gbs": nbytes / cm.value / 1e6, "decompress_gbs": nbytes / dm.value / 1e6,
                "compress_ms": cm.value, "decompress_ms": dm.value, "compressed_bytes": cb.value, "steps": steps,
                "dims": [nx, ny, nz],
                "note": "the reference's fz::Pipeline::compress / decompress calls timed with CUDA events, host "
                        "synchronisation included; the GPU arm's `pipeline` entry times this library's "
                        "fz::Pipeline the same way"}
    except Exception as e:  # the CPU arm's line stands on its own
        return {"unavailable": str(e)[:200]}


# ---------------------------------------------------------------- GPU side

def _traffic(kernel: str):
    """DRAM bytes per element of `kernel` from the committed ncu summary
    (profiles/traffic.json: dram__bytes_read.sum + dram__bytes_write.sum of
    one captured launch divided by the elements it processed), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)[kernel]
    except Exception:
        return None


def _config(dims, world: int) -> dict:
    return {"workload": WORKLOAD if tuple(dims) == DEFAULT_DIMS else WORKLOAD.replace("512^3", "x".join(map(str, dims))),
            "dims": list(dims), "eb": EB, "eb_mode": "REL", "radius": RADIUS, "zigzag": ZIGZAG,
            "outlier_capacity": OUTLIER_CAP,
            "l2": "input 512 MiB > L2, plus a 256 MiB L2 flush before every timed call",
            "parallelism": f"replicas x{world}"}


def _pipeline(dims, n):
    from fzgpumodules_b200 import pipeline as P
    pl = P.Pipeline(4 * n, P.PREALLOCATE)
    pl.setDims(*dims)
    lq = pl.addStage(P.LorenzoQuantStage(EB, RADIUS, OUTLIER_CAP, P.REL, ZIGZAG))
    bs = pl.addStage(P.BitshuffleStage(16384, 2))
    rz = pl.addStage(P.RZEStage(16384, 4))
    pl.connect(bs, lq, "codes")
    pl.connect(rz, bs)
    pl.finalize()
    return pl


def pipeline_timing(pl, x, steps: int, warmup: int, flush, world: int) -> dict:
    """This library's fz::Pipeline::compress / decompress on the field, each
    call bracketed by CUDA events with its host synchronisation inside, an
    L2 flush before each: the way the reference arm times the reference's
    own Pipeline (ref_pipeline_time_lq)."""
    import torch
    n = x.numel()
    ref = pl.compress(x).clone()
    tc = td = 0.0
    for i in range(warmup + steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        a.record()
        pl.compress(x)
        b.record()
        b.synchronize()
        if i >= warmup:
            tc += a.elapsed_time(b)
        flush.zero_()
        a.record()
        pl.decompress(None)
        b.record()
        b.synchronize()
        if i >= warmup:
            td += a.elapsed_time(b)
    tc = max_over_ranks(tc / steps, world)
    td = max_over_ranks(td / steps, world)
    y = pl.decompress(None)[:n]
    return {"compress_gbs": world * 4 * n / tc / 1e6, "decompress_gbs": world * 4 * n / td / 1e6,
            "compress_ms": tc, "decompress_ms": td, "compressed_bytes": int(ref.numel()),
            "bytes_equal_fused_call": None, "values_equal_fused_call": None, "_y": y, "_comp": ref,
            "note": "fz::Pipeline (PREALLOCATE, fused LQ->BS->RZE execution) through the Python mirror of the C ABI; "
                    "each call includes the pipeline's host synchronisation; the reference arm's "
                    "reference_gpu_pipeline times the reference's fz::Pipeline on the same field the same way"}


def pipeline_e2e(pl, x, steps: int, warmup: int, world: int) -> dict:
    """End to end through fz::Pipeline with host buffers, streamed as a
    service would run it: every step uploads its field from pinned host
    memory, compresses it and reads the container back, and step k+1's upload
    (a second device buffer, its own stream) overlaps step k's compression
    and read-back.  Then the reverse: every step uploads a container,
    decompresses it into one of two device buffers and reads the field back,
    step k+1's upload and decompression overlapping step k's read-back.  Wall
    clock over all steps of a direction, the pipeline fill included."""
    import torch
    n = x.numel()
    dev = x.device
    hx = x.cpu().pin_memory()
    cap = int(pl.compress(x).numel())
    hc = torch.empty(cap + (1 << 20), dtype=torch.uint8).pin_memory()
    hy = torch.empty_like(hx).pin_memory()
    dxs = [torch.empty_like(x) for _ in range(2)]
    dcs = [torch.empty(cap + (1 << 20), dtype=torch.uint8, device=dev) for _ in range(2)]
    ys = [torch.empty_like(x) for _ in range(2)]
    main = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    nb = 0

    def compress_run(k_steps: int) -> float:
        nonlocal nb
        free = [torch.cuda.Event() for _ in range(2)]   # dxs[b] read by its compression
        ready = [torch.cuda.Event() for _ in range(2)]  # dxs[b] uploaded
        for e in free:
            e.record(main)

        def upload(k):
            b = k & 1
            up.wait_event(free[b])
            with torch.cuda.stream(up):
                dxs[b].copy_(hx, non_blocking=True)
            ready[b].record(up)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        upload(0)
        for k in range(k_steps):
            if k + 1 < k_steps:
                upload(k + 1)
            b = k & 1
            main.wait_event(ready[b])
            comp = pl.compress(dxs[b])  # the pipeline's one wait: this compression
            free[b].record(main)
            nb = comp.numel()
            hc[:nb].copy_(comp, non_blocking=True)  # the next compression follows it on `main`
        main.synchronize()
        return time.perf_counter() - t0

    def decompress_run(k_steps: int) -> float:
        used = [torch.cuda.Event() for _ in range(2)]   # dcs[b] consumed
        ready = [torch.cuda.Event() for _ in range(2)]  # dcs[b] uploaded
        done = [torch.cuda.Event() for _ in range(2)]   # ys[b] written
        free = [torch.cuda.Event() for _ in range(2)]   # ys[b] read back
        for e in used + free:
            e.record(main)

        def upload(k):
            b = k & 1
            up.wait_event(used[b])
            with torch.cuda.stream(up):
                dcs[b][:nb].copy_(hc[:nb], non_blocking=True)
            ready[b].record(up)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        upload(0)
        for k in range(k_steps):
            if k + 1 < k_steps:
                upload(k + 1)
            b = k & 1
            main.wait_event(ready[b])
            main.wait_event(free[b])
            pl.decompressInto(dcs[b][:nb], ys[b])  # the pipeline's one wait: this decompression
            used[b].record(main)
            done[b].record(main)
            down.wait_event(done[b])
            with torch.cuda.stream(down):
                hy.copy_(ys[b], non_blocking=True)
            free[b].record(down)
        down.synchronize()
        main.synchronize()
        return time.perf_counter() - t0

    compress_run(max(warmup, 1))
    t_c = max_over_ranks(compress_run(steps) / steps, world)
    decompress_run(max(warmup, 1))
    t_d = max_over_ranks(decompress_run(steps) / steps, world)
    ok = bool(torch.equal(hy.view(torch.int32), pl.decompress(None)[:n].cpu().view(torch.int32)))
    return {"value": world * 4 * n / t_c / 1e9, "unit": "GB/s", "h2d_bytes_per_step": 4 * n + nb,
            "d2h_bytes_per_step": nb + 4 * n, "compress_gbs": world * 4 * n / t_c / 1e9,
            "decompress_gbs": world * 4 * n / t_d / 1e9, "api": "fz::Pipeline compress / decompressInto",
            "streamed": "step k+1's upload overlaps step k's coding and read-back (two device buffers, "
                        "upload / read-back streams); wall clock over all steps, pipeline fill included",
            "values_equal_device_decompress": ok}


def _guard(fn, *a, **k):
    try:
        return fn(*a, **k)
    except Exception as e:  # an extra measurement never takes the headline line down
        return {"error": f"{type(e).__name__}: {str(e)[:300]}"}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    from fzgpumodules_b200 import fields, kernels
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    DIMS = tuple(args.dims)
    nz, ny, nx = DIMS[2], DIMS[1], DIMS[0]
    x = fields.grf((nz, ny, nx), seed=SEED + rank, spike_frac=1e-3, device=dev).reshape(-1)
    n = x.numel()
    nbytes = 4 * n
    ws = kernels.Workspace()
    out = kernels.lq_bs_rze_compress(x, DIMS, EB, kernels.REL, RADIUS, ZIGZAG, OUTLIER_CAP, ws=ws)
    torch.cuda.synchronize()
    size = int(out["rze_size"].item())
    abs_eb = float(out["eb_state"][1].item())
    y = kernels.lq_bs_rze_decompress(out["rze"], size, out["err"], out["idx"], out["count"],
                                     out["cap"], n, DIMS, abs_eb, ZIGZAG, ws=ws)
    torch.cuda.synchronize()
    maxerr = float((y - x).abs().max().item())
    n_out = int(out["count"].item())
    comp_bytes = size + 8 * min(n_out, out["cap"]) + 4  # RZE stream + outlier segments + count
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream()

    def one(kind):
        flush.zero_()  # evict L2 between timed iterations (outside the events)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        if kind == "c":
            kernels.lq_bs_rze_compress(x, DIMS, EB, kernels.REL, RADIUS, ZIGZAG, OUTLIER_CAP, ws=ws, out=out)
        else:
            kernels.lq_bs_rze_decompress(out["rze"], size, out["err"], out["idx"], out["count"],
                                         out["cap"], n, DIMS, abs_eb, ZIGZAG,
                                         flags=kernels.NO_SYNC, ws=ws, out=y)
        e1.record(s)
        return e0, e1

    ev_c, ev_d = [], []
    with ClockSampler(local) as clk:
        time.sleep(0.3)  # let the sampler start before the timed region
        for _ in range(args.warmup):
            one("c"), one("d")
        barrier(world)
        t_wall = time.perf_counter()
        for _ in range(args.steps):  # the timed region: no per-kernel instrumentation
            ev_c.append(one("c"))
            ev_d.append(one("d"))
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
        barrier(world)
        # the same steps again with per-kernel CUDA events on the launching stream
        with kernels.Trace() as trace:
            for _ in range(args.steps):
                one("c"), one("d")
            torch.cuda.synchronize()
        per_kernel = trace.kernels()
    barrier(world)
    st = ws.status()
    tc = [a.elapsed_time(b) / 1e3 for a, b in ev_c]
    td = [a.elapsed_time(b) / 1e3 for a, b in ev_d]
    t_c = max_over_ranks(float(np.mean(tc)), world)
    t_d = max_over_ranks(float(np.mean(td)), world)

    # the dominant kernels, timed by their own events (max over ranks)
    def kern(name):
        launches, ms = per_kernel.get(name, (0, 0.0))
        return launches, max_over_ranks(ms / launches / 1e3 if launches else 0.0, world)

    slab_name = next((k for k in ("lq3d_tma_bs_rze", "lq3d_slab_bs_rze") if k in per_kernel), "lq_chunk_bs_rze")
    inv_name = next((k for k in ("lq3d_inv_slab", "fused_inverse_3d") if k in per_kernel), "lq_inverse")
    n_slab, t_slab = kern(slab_name)
    n_inv, t_inv = kern(inv_name)
    launches = sum(v[0] for v in per_kernel.values())

    # this library's fz::Pipeline, timed as the reference arm times the
    # reference's Pipeline, and end to end with host buffers through it
    pl = _pipeline(DIMS, n)
    pipe = pipeline_timing(pl, x, args.steps, args.warmup, flush, world)
    yp, cp = pipe.pop("_y"), pipe.pop("_comp").cpu().numpy()
    pipe["values_equal_fused_call"] = bool(torch.equal(yp.view(torch.int32), y.view(torch.int32)))
    # the container's last segment is the RZE stream: the same bytes as the fused call's
    nseg = int(cp[:4].view(np.uint32)[0])
    sizes = cp[4:4 + 8 * nseg].view(np.uint64).astype(np.int64)
    off = (4 + 8 * nseg + 15) & ~15
    for k in range(nseg - 1):
        off += (int(sizes[k]) + 15) & ~15
    pipe["bytes_equal_fused_call"] = bool(int(sizes[-1]) == size and np.array_equal(
        cp[off:off + size], out["rze"][:size].cpu().numpy()))
    del cp
    e2e = None if args.no_e2e else pipeline_e2e(pl, x, args.steps, args.warmup, world)
    pl.close()
    del yp

    if rank != 0:
        return
    peak, peak_kind = _peaks()
    algo_c = nbytes + comp_bytes   # read f32 field + write compressed segments
    algo_d = comp_bytes + nbytes   # read compressed segments + write f32 field
    ach_c = algo_c / t_slab / 1e9 if t_slab else 0.0   # dominant compress kernel
    ach_d = algo_d / t_inv / 1e9 if t_inv else 0.0     # dominant decompress kernel
    tr_c, tr_d = _traffic(slab_name), _traffic(inv_name)
    # the host cores run the oracle last, after the GPU extras, so that its
    # OpenMP threads do not share the host with their timed calls
    xh = x.cpu().numpy() if (world == 1 and not args.no_cpu) else None
    line = {
        "metric": METRIC, "value": world * nbytes / t_c / 1e9, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": (t_c + t_d) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": _config(DIMS, world),
        "compress": {"gbs": nbytes / t_c / 1e9, "ms": t_c * 1e3, "ratio": nbytes / comp_bytes,
                     "compressed_bytes": comp_bytes, "outliers": n_out},
        "decompress": {"value": world * nbytes / t_d / 1e9, "unit": "GB/s", "ms": t_d * 1e3,
                       "max_abs_err": maxerr, "abs_eb": abs_eb,
                       "roofline": {"bound": "hbm", "achieved": ach_d, "peak": peak, "unit": "GB/s",
                                    "frac": ach_d / peak,
                                    "traffic": tr_d["bytes_per_element"] * n if tr_d else None,
                                    "algorithmic_bytes": algo_d, "peak_kind": peak_kind,
                                    "kernel": inv_name, "kernel_ms": t_inv * 1e3, "launches": n_inv,
                                    "call_frac": (algo_d / t_d / 1e9) / peak}},
        "roofline": {"bound": "hbm", "achieved": ach_c, "peak": peak, "unit": "GB/s",
                     "frac": ach_c / peak,
                     "traffic": tr_c["bytes_per_element"] * n if tr_c else None,
                     "algorithmic_bytes": algo_c, "peak_kind": peak_kind,
                     "kernel": slab_name, "kernel_ms": t_slab * 1e3, "launches": n_slab,
                     "call_frac": (algo_c / t_c / 1e9) / peak},
        "kernels_ms_per_step": {k: v[1] / args.steps for k, v in per_kernel.items()},
        "pipeline": pipe,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "status": st,
        "wall_s_timed": t_wall,
    }
    if world == 1 and not args.no_extras:
        from fzgpumodules_b200 import benchmarks
        del flush
        torch.cuda.empty_cache()
        line["c3"] = _guard(benchmarks.c3_summary, dev, args.steps, args.warmup)
        torch.cuda.empty_cache()
        line["batch"] = _guard(benchmarks.batch_summary, dev, args.steps, args.warmup)
        torch.cuda.empty_cache()
        line["selector"] = _guard(benchmarks.selector_summary, dev, args.steps, args.warmup, args.train_chunks)
    if xh is not None:
        cpu = cpu_baseline(xh, DIMS, 1)
        line["cpu_baseline"] = {"value": cpu["compress_gbs"], "unit": "GB/s", "cores": cpu["cores"],
                                "kind": "port", "sample": cpu["sample"],
                                "decompress_gbs": cpu["decompress_gbs"]}
    print(json.dumps(line), flush=True)


def run_reference_pfpl(args):
    """Reference arm of the pfpl workload: the reference's own fz::Pipeline
    (built from its sources into oracle/_ref) compressing and decompressing
    the same 512^3 field on this GPU, each call timed with CUDA events."""
    import ctypes as C

    import torch

    from fzgpumodules_b200 import benchmarks
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref", "libfzref_pipe.so")
    base = {"impl": "reference", "workload": "pfpl"}
    if not os.path.exists(path):
        return dict(base, unavailable="the reference pipeline build (oracle/_ref/libfzref_pipe.so) is absent")
    dev = torch.device("cuda", 0)
    x = benchmarks.pfpl_field(dev, tuple(args.dims))
    n = x.numel()
    L = C.CDLL(path)
    L.ref_pipe_last_error.restype = C.c_char_p
    cm, dm, cb = C.c_float(0), C.c_float(0), C.c_size_t(0)
    rc = L.ref_pipeline_time_pfpl(C.c_void_p(x.data_ptr()), C.c_size_t(n), C.c_float(1e-3), C.c_float(0.1),
                                  args.steps, args.warmup, C.byref(cm), C.byref(dm), C.byref(cb), 0)
    if rc != 0:
        return dict(base, unavailable="reference pipeline failed: " + L.ref_pipe_last_error().decode())
    sm, sdm, scb = C.c_float(0), C.c_float(0), C.c_size_t(0)
    rc = L.ref_pipeline_time_pfpl(C.c_void_p(x.data_ptr()), C.c_size_t(n), C.c_float(1e-3), C.c_float(0.05),
                                  args.steps, args.warmup, C.byref(sm), C.byref(sdm), C.byref(scb), 1)
    speed = ({"speed_compress_gbs": 4 * n / sm.value / 1e6, "speed_decompress_gbs": 4 * n / sdm.value / 1e6,
              "speed_compressed_bytes": scb.value} if rc == 0 else
             {"speed_unavailable": L.ref_pipe_last_error().decode()})
    v = 4 * n / cm.value / 1e6
    return dict(base, metric="compress GB/s of the pfpl preset pipeline", value=v, unit="GB/s", n_gpus=1,
                steps=args.steps, warmup=args.warmup, higher_is_better=True, dtype="f32", data="synthetic",
                config={"workload": "pfpl: Quantizer(REL 1e-3)->Difference->Bitshuffle->RZE, 512^3 GRF",
                        "flush": "256 MiB written between calls"},
                compress_ms=cm.value, decompress_ms=dm.value, decompress_gbs=4 * n / dm.value / 1e6,
                compressed_bytes=cb.value, e2e={"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0,
                                                "d2h_bytes_per_step": 0},
                **speed,
                note="the reference's GPU pipeline through its public API (Pipeline::compress / decompress, "
                     "host synchronisation included)")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the c3, batch and selector entries of the headline line")
    ap.add_argument("--train-chunks", type=int, default=1 << 20,
                    help="method-generated chunks the coder selector trains on (selector entry / workload)")
    ap.add_argument("--dims", type=int, nargs=3, default=list(DEFAULT_DIMS), metavar=("NX", "NY", "NZ"),
                    help="field extents (x fastest); the default is the 512^3 workload")
    ap.add_argument("--workload", default="chain",
                    choices=["chain", "c1", "cli", "c3", "batch", "selector", "pfpl", "timeline"],
                    help="chain: the headline LQ3D->BS->RZE line; others: secondary workloads (1 GPU)")
    args = ap.parse_args()
    if args.workload == "pfpl" and args.impl == "reference":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(run_reference_pfpl(args)), flush=True)
        return
    if args.workload != "chain":
        import torch

        from fzgpumodules_b200 import benchmarks
        if int(os.environ.get("RANK", "0")) == 0:
            line = json.loads(benchmarks.WORKLOADS[args.workload](args, torch.device("cuda", 0)))
            if not args.no_cpu and args.workload in CPU_WORKLOADS:
                line["cpu_baseline"] = CPU_WORKLOADS[args.workload]()
            print(json.dumps(line), flush=True)
        return
    world, rank, local = dist_setup() if args.impl == "ours" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
