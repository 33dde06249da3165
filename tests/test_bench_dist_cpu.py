"""The multi-rank host logic of bench.py on CPU: two gloo ranks on
127.0.0.1 (the launch torchrun makes for --gpus 2), the max-over-ranks
timing reduction and barrier, each rank's own replica field, and the
reference arm's rank-0-only rule.  No GPU is used."""
import os
import socket
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    try:
        import torch.distributed as dist

        import bench
        w, r, _ = bench.dist_setup()
        backend = dist.get_backend()
        slowest = bench.max_over_ranks(1.5 * (rank + 1), w)
        bench.barrier(w)
        field = bench.host_field((16, 8, 4), rank)
        dist.destroy_process_group()
        q.put((rank, w, r, backend, slowest, float(field.sum()), field.size))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def test_two_gloo_ranks_reduce_and_shard():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for g in got:
        assert g[1] != "error", g
    (r0, w0, rr0, b0, m0, s0, n0), (r1, w1, rr1, b1, m1, s1, n1) = got
    assert (w0, w1, rr0, rr1) == (2, 2, 0, 1)
    assert b0 == b1 == "gloo"
    assert m0 == m1 == 3.0          # every rank reports the slowest rank's time
    assert n0 == n1 == 16 * 8 * 4
    assert s0 != s1                 # each replica compresses its own field


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench
    args = types.SimpleNamespace(dims=[16, 8, 4], warmup=0, steps=1, gpus=2)
    assert bench.run_reference(args, 2, 1) is None
    assert capsys.readouterr().out == ""
