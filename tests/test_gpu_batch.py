"""Batched compression (fzb_batch_*): many fields of mixed rank, size and
error bound in one persistent launch.  Every field's RZE stream, outliers,
outlier count and resolved error bound must equal its own
fzb_lq_bs_rze_compress call, for every tuning and under CUDA-graph replay."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def K():
    from fzgpumodules_b200 import kernels
    return kernels


def _fields(dev, count=24, seed=1004):
    from fzgpumodules_b200 import fields as F
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nbytes = int(np.exp(rng.uniform(np.log(64 << 10), np.log(4 << 20))))
        n = max(nbytes // 4, 64)
        rank = int(rng.integers(1, 4))
        if rank == 1:
            dims = (n, 1, 1)
        elif rank == 2:
            nx = int(rng.choice([64, 100, 256, 333, 512, 1000]))
            dims = (nx, max(n // nx, 2), 1)
        else:
            nx = int(rng.choice([32, 48, 64, 128, 200]))
            ny = int(rng.choice([16, 32, 40, 64]))
            dims = (nx, ny, max(n // (nx * ny), 2))
        shape = tuple(d for d in reversed(dims) if d > 1) or (dims[0],)
        x = F.grf(shape, seed=seed + i, spike_frac=1e-3, device=dev).reshape(-1).contiguous()
        abs_case = i % 5 == 0  # ABS with a small radius: outliers occur
        out.append(dict(x=x, dims=dims, eb=1e-3 if abs_case else float(rng.choice([1e-2, 1e-3, 1e-4])),
                        mode=K().ABS if abs_case else K().REL, radius=512 if abs_case else 32768, zigzag=True))
    # two slab-shaped fields (the batch gives them the slab kernels)
    for j, dims in enumerate([(128, 64, 9), (256, 32, 17)]):
        x = F.grf(tuple(reversed(dims)), seed=seed + count + j, spike_frac=1e-3, device=dev).reshape(-1).contiguous()
        out.append(dict(x=x, dims=dims, eb=1e-3, mode=K().ABS if j else K().REL, radius=512 if j else 32768,
                        zigzag=True))
    return out


def _expected(f):
    return K().lq_bs_rze_compress(f["x"], f["dims"], f["eb"], f["mode"], f["radius"], f["zigzag"], 0.2)


def _same(o, r):
    sz = int(r["rze_size"].item())
    assert int(o["rze_size"].item()) == sz
    assert torch.equal(o["rze"][:sz], r["rze"][:sz])
    cnt = int(r["count"].item())
    assert int(o["count"].item()) == cnt
    st = min(cnt, r["cap"])
    assert torch.equal(o["err"][:st], r["err"][:st]) and torch.equal(o["idx"][:st], r["idx"][:st])
    assert torch.equal(o["eb_state"], r["eb_state"])


def test_batch_matches_single_field_calls(cuda):
    fields = _fields(cuda)
    ref = [_expected(f) for f in fields]
    assert any(int(r["count"].item()) > 0 for r in ref)
    b = K().Batch(fields)
    for _ in range(2):  # a relaunch re-arms every counter
        b.launch()
        torch.cuda.synchronize()
        for o, r in zip(b.outputs, ref):
            _same(o, r)
    b.close()


@pytest.mark.parametrize("ctas,order,flat,parts", [(1, 0, 0, 0), (3, 1, 1, 1), (2, 1, 0, 8), (2, 0, 1, 2)])
def test_batch_tuning_does_not_change_bytes(cuda, ctas, order, flat, parts):
    # CTAs per SM, dispatch order, tile shape (slab units or flat chunks for
    # slab-shaped fields) and scan granularity change the launch, not the bytes
    fields = _fields(cuda, count=12, seed=77)
    ref = [_expected(f) for f in fields]
    b = K().Batch(fields, K().BatchTuning(ctas, order, flat, parts))
    b.launch()
    torch.cuda.synchronize()
    for o, r in zip(b.outputs, ref):
        _same(o, r)
    best, ms = b.autotune()
    assert 1 <= best.ctas_per_sm <= 3 and best.order in (0, 1) and ms > 0
    assert best.flat_tiles in (0, 1) and best.scan_parts in (1, 2, 4, 8)
    b.launch()
    torch.cuda.synchronize()
    for o, r in zip(b.outputs, ref):
        _same(o, r)
    b.close()


def test_batch_graph_replay(cuda):
    fields = _fields(cuda, count=10, seed=5)
    ref = [_expected(f) for f in fields]
    b = K().Batch(fields)
    s = torch.cuda.Stream(device=cuda)
    b.launch(s)  # warm (lazy module load stays out of the capture)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.launch(s)
    for o in b.outputs:
        o["rze"].zero_()
        o["count"].zero_()
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    for o, r in zip(b.outputs, ref):
        _same(o, r)
    del g
    b.close()
