"""The container concatenation and the result gather a pipeline call enqueues
before its single wait (fzb_concat_dev, fzb_gather_words), against the
host-sized concatenation (fzb_concat, the reference's concatOutputs layout)
and a numpy restatement of the layout; and the pipeline's single-wait
decompression when the fused inverse leaves a case to the exact kernels."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def lib():
    from fzgpumodules_b200._lib import lib as _l
    return _l()


def _vp(t: torch.Tensor, off: int = 0):
    return C.c_void_p(t.data_ptr() + off)


def _arr(ctype, vals):
    return (ctype * len(vals))(*vals)


def _layout(segments):
    """[u32 n][u64 len x n] pad16, then each segment pad16 with zero pads."""
    n = len(segments)
    head = np.zeros((4 + 8 * n + 15) & ~15, dtype=np.uint8)
    head[:4] = np.frombuffer(np.uint32(n).tobytes(), dtype=np.uint8)
    head[4:4 + 8 * n] = np.frombuffer(np.array([len(s) for s in segments], dtype=np.uint64).tobytes(),
                                      dtype=np.uint8)
    parts = [head]
    for s in segments:
        pad = np.zeros((len(s) + 15) & ~15, dtype=np.uint8)
        pad[:len(s)] = s
        parts.append(pad)
    return np.concatenate(parts)


def test_concat_dev_matches_concat(cuda):
    L = lib()
    rng = np.random.default_rng(5)
    host = rng.integers(0, 256, size=1 << 20, dtype=np.uint8)
    base = torch.from_numpy(host).to(cuda)
    w32 = torch.tensor([3000, 9000, 0, 0], dtype=torch.int32, device=cuda)
    w64 = torch.tensor([77777, 500000], dtype=torch.int64, device=cuda)
    # (source offset, cap, size word or None, word bytes, scale, max count, expected length)
    segs = [
        (0, 1000, None, 0, 1, 0, 1000),                    # a size the host knows
        (1003, 24000, (w32, 0), 4, 4, 6000, 12000),         # count * 4 from an unaligned source
        (200000, 24000, (w32, 4), 4, 4, 5000, 20000),       # count above its maximum: clamped
        (300000, 100000, (w64, 0), 8, 1, ~0 & (2**64 - 1), 77777),  # a u64 stream size
        (500001, 4096, (w64, 8), 8, 1, 2**64 - 1, 4096),   # device size above the cap: cut
        (0, 0, None, 0, 1, 0, 0),                          # empty
        (700000, 64, (w32, 8), 4, 8, 100, 0),              # a zero count
    ]
    n = len(segs)
    src = _arr(C.c_void_p, [base.data_ptr() + s[0] for s in segs])
    caps = _arr(C.c_uint64, [s[1] for s in segs])
    words = _arr(C.c_void_p, [None if s[2] is None else s[2][0].data_ptr() + s[2][1] for s in segs])
    wbytes = _arr(C.c_uint32, [s[3] for s in segs])
    scale = _arr(C.c_uint64, [s[4] for s in segs])
    maxc = _arr(C.c_uint64, [s[5] for s in segs])
    bound = int(L.fzb_concat_bytes(caps, n))
    out = torch.full((bound,), 0xAA, dtype=torch.uint8, device=cuda)
    assert L.fzb_concat_dev(src, caps, words, wbytes, scale, maxc, n, _vp(out), None) == 0
    lens = _arr(C.c_uint64, [s[6] for s in segs])
    total = int(L.fzb_concat_bytes(lens, n))
    ref = torch.empty(total, dtype=torch.uint8, device=cuda)
    assert L.fzb_concat(src, lens, n, _vp(ref), None) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.array_equal(got[:total], ref.cpu().numpy())
    want = _layout([host[s[0]:s[0] + s[6]] for s in segs])
    assert np.array_equal(got[:total], want)
    assert (got[total:] == 0xAA).all()  # nothing written past the container


def test_concat_dev_rejects_bad_arguments(cuda):
    L = lib()
    buf = torch.zeros(4096, dtype=torch.uint8, device=cuda)
    w = torch.zeros(4, dtype=torch.int64, device=cuda)
    src = _arr(C.c_void_p, [buf.data_ptr(), buf.data_ptr()])
    caps = _arr(C.c_uint64, [64, 64])
    scale = _arr(C.c_uint64, [1, 1])
    maxc = _arr(C.c_uint64, [10, 10])
    for wb, wp, sc, out_off in [(3, w.data_ptr(), 1, 0),          # word width
                                (8, w.data_ptr() + 4, 1, 0),      # misaligned u64 word
                                (4, w.data_ptr(), 0, 0),          # zero scale
                                (4, w.data_ptr(), 1, 8)]:         # output not 16-byte aligned
        words = _arr(C.c_void_p, [wp, None])
        wbytes = _arr(C.c_uint32, [wb, 0])
        sca = _arr(C.c_uint64, [sc, 1])
        assert L.fzb_concat_dev(src, caps, words, wbytes, sca, maxc, 2, _vp(buf, out_off), None) == -1
    big = _arr(C.c_uint64, [2**62, 10])
    words = _arr(C.c_void_p, [w.data_ptr(), None])
    wbytes = _arr(C.c_uint32, [8, 0])
    assert L.fzb_concat_dev(src, caps, words, wbytes, _arr(C.c_uint64, [8, 1]), big, 2, _vp(buf), None) == -1


def test_gather_words(cuda):
    L = lib()
    a = torch.arange(128, dtype=torch.int32, device=cuda)
    status = torch.tensor([5, 7], dtype=torch.int32, device=cuda)
    size = torch.tensor([123456789012], dtype=torch.int64, device=cuda)
    src = _arr(C.c_void_p, [a.data_ptr() + 16, status.data_ptr(), size.data_ptr(), a.data_ptr() + 40])
    nbytes = _arr(C.c_uint32, [12, 4, 8, 256])
    clear = _arr(C.c_uint8, [0, 1, 0, 0])
    for pinned in (False, True):
        status[0] = 5
        if pinned:  # mapped host memory, as the pipeline uses
            dst = torch.zeros(512, dtype=torch.uint8).pin_memory()
        else:
            dst = torch.zeros(512, dtype=torch.uint8, device=cuda)
        assert L.fzb_gather_words(src, nbytes, clear, 4, _vp(dst), None) == 0
        torch.cuda.synchronize()
        d = dst.cpu().numpy()
        # offsets: 0 (12 B, next at 16), 16 (4 B, next at 24), 24 (8 B), 32 (256 B)
        assert np.array_equal(d[0:12].view(np.int32), [4, 5, 6])
        assert d[16:20].view(np.int32)[0] == 5
        assert d[24:32].view(np.int64)[0] == 123456789012
        assert np.array_equal(d[32:288].view(np.int32), np.arange(10, 74))
        assert int(status[0]) == 0 and int(status[1]) == 7  # only the gathered word is cleared
        assert torch.equal(a, torch.arange(128, dtype=torch.int32, device=cuda))


def test_pipeline_decompress_reruns_exact_kernels(cuda):
    # deltas far outside the fused inverse's exact-integer range: the fused
    # pass flags them, the pipeline reads the flag with its one wait and
    # reruns the exact kernels; the result equals the synchronous C-ABI call
    from fzgpumodules_b200 import kernels as K
    from fzgpumodules_b200 import pipeline as P
    dims = (64, 128, 8)  # rows tile a 16 KiB chunk: the fused inverse applies
    n = int(np.prod(dims))
    rng = np.random.default_rng(16)
    x = torch.from_numpy((rng.normal(size=n) * 1e4).astype(np.float32)).to(cuda)
    ref = K.lq_bs_rze_compress(x, dims, 1e-4, K.ABS, 32768, True, 1.0)
    size = int(ref["rze_size"].item())
    abs_eb = float(ref["eb_state"][1].item())
    ws = K.Workspace()
    K.lq_bs_rze_decompress(ref["rze"], size, ref["err"], ref["idx"], ref["count"], ref["cap"], n, dims, abs_eb,
                           True, flags=K.NO_SYNC, ws=ws)
    torch.cuda.synchronize()
    bits = int(ws.buf[:4].view(torch.int32).item())
    assert bits & 12, "the fused pass did not leave this field to the exact kernels"
    ws.status()
    want = K.lq_bs_rze_decompress(ref["rze"], size, ref["err"], ref["idx"], ref["count"], ref["cap"], n, dims,
                                  abs_eb, True)
    pl = P.Pipeline(0, P.MINIMAL)
    pl.setDims(*dims)
    lq = pl.addStage(P.LorenzoQuantStage(1e-4, 32768, 1.0, P.ABS, True))
    bs = pl.addStage(P.BitshuffleStage(16384, 2))
    rz = pl.addStage(P.RZEStage(16384, 4))
    pl.connect(bs, lq, "codes")
    pl.connect(rz, bs)
    pl.finalize()
    assert pl.isFused()
    comp = pl.compress(x).clone()
    for src in (comp, None):
        y = pl.decompress(src).clone()
        assert torch.equal(y.view(torch.int32), want.view(torch.int32))
    pl.close()
