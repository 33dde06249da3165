"""The one-pass pfpl chain (fzb_pfpl_compress / fzb_pfpl_decompress) against
the same four stages run one after another through the C ABI -- Quantizer
(u32 codes) -> Difference (int32 -> uint32, 16 KiB chunks) -> Bitshuffle
(16384, ew 2) -> RZE -- whose parity with the reference's kernels and
pipeline is established in test_gpu_transforms.py and
test_gpu_pipeline_codes.py: identical RZE bytes, outlier lists and counts,
and bit-identical decompressed values, on whole and partial chunks, in every
error-bound mode, and at full size."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ABS, REL, NOA = 0, 1, 2


def K():
    from fzgpumodules_b200 import kernels
    return kernels


def _field(n, seed, dev):
    g = torch.Generator(device=dev).manual_seed(seed)
    x = torch.cumsum(torch.randn(n, device=dev, generator=g), 0) * 0.05 + 3.0
    idx = torch.randint(0, n, (max(n // 500, 1),), device=dev, generator=g)
    x[idx] = torch.randn(idx.numel(), device=dev, generator=g) * 1e5
    x[idx[: max(idx.numel() // 4, 1)]] = 0.0
    return x.float()


def _staged(x, eb, mode, radius, zz, capf, thr):
    q = K().quantizer_forward(x, eb, mode, radius, 4, zz, capf, thr)
    d = K().diff(q["codes"], 16384, True)
    rze, size = K().rze_encode(K().bitshuffle(d, 16384, 2))
    return q, rze, size


@pytest.mark.parametrize("n", [1, 4095, 4096, 4097, 100_003, 4096 * 37, 700_001])
@pytest.mark.parametrize("mode,radius,zz,thr", [(REL, 32768, True, float("inf")), (ABS, 32768, True, float("inf")),
                                                (NOA, 512, False, float("inf")), (ABS, 1 << 20, False, 50.0)])
def test_pfpl_fused_equals_stages(cuda, n, mode, radius, zz, thr):
    x = _field(n, n % 997 + mode, cuda)
    eb, capf = 1e-3, 0.1
    q, rze, size = _staged(x, eb, mode, radius, zz, capf, thr)
    f = K().pfpl_compress(x, eb, mode, radius, zz, capf, thr)
    fsize = int(f["rze_size"].item())
    assert fsize == int(size.item())
    assert torch.equal(f["rze"][:fsize], rze[:fsize])
    cnt = int(f["count"].item())
    assert cnt == int(q["count"].item())
    assert torch.equal(f["idx"][:cnt], q["idx"][:cnt]) and torch.equal(f["vals"][:cnt], q["vals"][:cnt])
    assert torch.equal(f["eb_state"][:3], q["eb_state"][:3])
    abs_eb = 0.0 if mode == REL else float(q["eb_state"][1].item())
    y = K().pfpl_decompress(f["rze"], fsize, f["vals"], f["idx"], f["count"], f["cap"], n, eb, mode, abs_eb, zz)
    b = K().bitshuffle(K().rze_decode(rze[:fsize], 4 * n), 16384, 2, inverse=True)
    c = K().diff(b.view(torch.int32), 16384, True, inverse=True)
    want = K().quantizer_inverse(c, eb, mode, abs_eb, radius, zz, vals=q["vals"], idx=q["idx"], count=q["count"],
                                 cap=q["cap"])
    assert torch.equal(y.view(torch.int32), want.view(torch.int32))


def test_pfpl_fused_full_size(cuda):
    n = 64 << 20  # 256 MiB of values, above L2
    x = _field(n, 7, cuda)
    q, rze, size = _staged(x, 1e-3, REL, 32768, True, 0.1, float("inf"))
    f = K().pfpl_compress(x, 1e-3, REL, 32768, True, 0.1)
    fsize = int(f["rze_size"].item())
    assert fsize == int(size.item()) and torch.equal(f["rze"][:fsize], rze[:fsize])
    cnt = int(f["count"].item())
    assert torch.equal(f["idx"][:cnt], q["idx"][:cnt])
    y = K().pfpl_decompress(f["rze"], fsize, f["vals"], f["idx"], f["count"], f["cap"], n)
    xd, yd = x.double(), y.double()
    assert bool(((yd - xd).abs() <= xd.abs() * 1e-3 * 1.01).all())
    assert K()._default_ws.status() == 0


@pytest.mark.parametrize("dims", [(128, 128, 64), (3600, 1800, 1)])
def test_pfpl_pipeline_fused_equals_staged(cuda, dims, tmp_path):
    from fzgpumodules_b200 import pipeline as p
    n = dims[0] * dims[1] * dims[2]
    x = _field(n, 11, cuda)
    outs = []
    for fusion in (True, False):
        pl = p.Pipeline(n * 4, p.PREALLOCATE)
        pl.setDims(*dims)
        q = pl.addStage(p.QuantizerStage(1e-3, p.REL, 32768, 0.1, code_bytes=4, zigzag_codes=True))
        d = pl.addStage(p.DifferenceStage(p.INT32, p.UINT32, 16384))
        bs = pl.addStage(p.BitshuffleStage(16384, 2))
        rz = pl.addStage(p.RZEStage(16384, 4))
        pl.connect(d, q, "codes")
        pl.connect(bs, d)
        pl.connect(rz, bs)
        pl.setFusion(fusion)
        pl.finalize()
        assert pl.isFused() == fusion
        comp = pl.compress(x).clone()
        y = pl.decompress().clone()
        path = str(tmp_path / f"f{int(fusion)}.fzm")
        pl.writeToFile(path)
        yf = p.Pipeline.decompressFromFile(path)[:n]
        outs.append((comp, y, yf))
        pl.close()
    (ca, ya, fa), (cb, yb, fb) = outs
    assert torch.equal(ca, cb)
    assert torch.equal(ya.view(torch.int32), yb.view(torch.int32))
    assert torch.equal(fa.view(torch.int32), ya.view(torch.int32)) and torch.equal(fb.view(torch.int32), ya.view(torch.int32))


def _pfpl_pipeline(p, n, dims, graph=False, fusion=True):
    pl = p.Pipeline(n * 4, p.PREALLOCATE)
    pl.setDims(*dims)
    q = pl.addStage(p.QuantizerStage(1e-3, p.REL, 32768, 0.1, code_bytes=4, zigzag_codes=True))
    d = pl.addStage(p.DifferenceStage(p.INT32, p.UINT32, 16384))
    bs = pl.addStage(p.BitshuffleStage(16384, 2))
    rz = pl.addStage(p.RZEStage(16384, 4))
    pl.connect(d, q, "codes")
    pl.connect(bs, d)
    pl.connect(rz, bs)
    pl.enableGraphMode(graph)
    pl.setFusion(fusion)
    pl.finalize()
    return pl


def test_pfpl_pipeline_graph_replay(cuda):
    # one compress captured into a CUDA graph and replayed on new inputs
    # gives the eager pipeline's bytes, outlier counts included
    from fzgpumodules_b200 import pipeline as p
    dims = (256, 256, 32)
    n = dims[0] * dims[1] * dims[2]
    x1 = _field(n, 3, cuda)
    x2 = (x1 * 0.5 + 0.25).contiguous()
    x3 = _field(n, 4, cuda)
    pl = _pfpl_pipeline(p, n, dims, graph=True)
    s = torch.cuda.Stream(device=cuda)
    pl.captureGraph(s)
    eager = _pfpl_pipeline(p, n, dims)
    for x in (x1, x2, x3, x1):
        with torch.cuda.stream(s):
            cg = pl.compress(x).clone()
        s.synchronize()
        ce = eager.compress(x).clone()
        assert torch.equal(cg.cpu(), ce.cpu())
    pl.close()
    eager.close()
