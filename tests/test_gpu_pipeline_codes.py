"""Pipelines built around the direct Quantizer -- the shipped presets
(examples/presets/pfpl.toml, speed.toml, quantizer_lorenzo_bitpack.toml)
and codings of the codes with Negabinary, Zigzag and in-place outliers --
against the reference's own fz::Pipeline compiled from its sources: the FZM
container (header core, stage records, buffer records, segment bytes; the
outlier lists as (index, value) sets) and the decompressed values, which
must be bit-identical.  The reference's stage factory has no Quantizer case,
so its side decompresses on the live pipeline; this library's file is read
back with decompressFromFile."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from test_gpu_pipeline import make_field, parse_fzm

pytestmark = pytest.mark.gpu

ABS, REL, NOA = 0, 1, 2

# name: (chain id, dims, eb, mode, radius, outlier capacity, field)
CHAINS = {
    "pfpl": (3, (128, 128, 64), 1e-3, REL, 32768, 0.1, "grf"),
    "speed": (4, (128, 128, 64), 1e-3, REL, 32768, 0.05, "grf"),
    "quantizer_lorenzo_bitpack": (5, (1024, 1024, 1), 1e-3, NOA, 512, 0.05, "fractal"),
    "quantizer_negabinary_u16": (6, (3600, 1800, 1), 1e-3, ABS, 32768, 0.05, "sin"),
    "quantizer_inplace_zigzag": (7, (256, 64, 32), 1e-3, ABS, 32768, 0.05, "grf"),
}


def P():
    from fzgpumodules_b200 import pipeline
    return pipeline


def build(chain: int, dims, eb, mode, radius, cap, n):
    p = P()
    pl = p.Pipeline(n * 4, p.PREALLOCATE)
    pl.setDims(*dims)

    def bs_rze(src, port, ew):
        bs = pl.addStage(p.BitshuffleStage(16384, ew))
        rz = pl.addStage(p.RZEStage(16384, 4))
        pl.connect(bs, src, port)
        pl.connect(rz, bs)

    if chain == 6:
        q = pl.addStage(p.QuantizerStage(eb, mode, radius, cap, code_bytes=2))
        nb = pl.addStage(p.NegabinaryStage(p.INT16))
        pl.connect(nb, q, "codes")
        bs_rze(nb, "output", 2)
    else:
        q = pl.addStage(p.QuantizerStage(eb, mode, radius, cap, code_bytes=4, zigzag_codes=chain in (3, 4, 7),
                                         inplace_outliers=chain == 7))
        if chain == 3:
            d = pl.addStage(p.DifferenceStage(p.INT32, p.UINT32, 16384))
            pl.connect(d, q, "codes")
            bs_rze(d, "output", 2)
        elif chain == 4:
            bs_rze(q, "codes", 4)
        elif chain == 5:
            lz = pl.addStage(p.LorenzoStage(p.INT32))
            bp = pl.addStage(p.BitpackStage(4, 16))
            pl.connect(lz, q, "codes")
            pl.connect(bp, lz)
        else:
            zz = pl.addStage(p.ZigzagStage(p.INT32))
            pl.connect(zz, q, "codes")
            bs_rze(zz, "output", 4)
    pl.finalize()
    return pl


def _ref_pipe():
    path = os.path.join(os.path.dirname(O.REF_STAGES), "libfzref_pipe.so")
    if not os.path.exists(path):
        pytest.skip("reference pipeline build absent")
    L = C.CDLL(path)
    L.ref_pipe_last_error.restype = C.c_char_p
    return L


@pytest.mark.parametrize("name", list(CHAINS))
def test_quantizer_pipelines_match_reference(cuda, name, tmp_path):
    L = _ref_pipe()
    chain, dims, eb, mode, radius, cap, kind = CHAINS[name]
    x = make_field(kind, dims, cuda)
    n = x.numel()
    ref_path = str(tmp_path / "ref.fzm")
    dec = torch.zeros(n, dtype=torch.float32, device=cuda)
    dsz, csz = C.c_size_t(0), C.c_size_t(0)
    rc = L.ref_pipeline_codes(chain, C.c_void_p(x.data_ptr()), C.c_size_t(n), *[C.c_size_t(v) for v in dims],
                              C.c_float(eb), mode, radius, C.c_float(cap), ref_path.encode(),
                              C.c_void_p(dec.data_ptr()), C.byref(dsz), C.byref(csz))
    assert rc == 0, L.ref_pipe_last_error()
    torch.cuda.synchronize()
    pl = build(chain, dims, eb, mode, radius, cap, n)
    comp = pl.compress(x)
    assert comp.numel() == csz.value
    y_live = pl.decompress().clone()
    ours_path = str(tmp_path / "ours.fzm")
    pl.writeToFile(ours_path)
    y_file = P().Pipeline.decompressFromFile(ours_path)
    a, b = parse_fzm(open(ours_path, "rb").read()), parse_fzm(open(ref_path, "rb").read())
    for k in ("magic", "version", "num_buffers", "uncompressed", "compressed", "header_size", "num_stages",
              "num_sources", "flags", "sources"):
        assert a["core"][k] == b["core"][k], k
    assert a["stages"] == b["stages"]  # stage types and records (QuantizerConfig 36 B, Difference 6 B, ...)
    sa = {(e["type"], e["name"]): e for e in a["buffers"]}
    sb = {(e["type"], e["name"]): e for e in b["buffers"]}
    assert sa.keys() == sb.keys()
    for key in sa:
        ra, rb = bytearray(sa[key]["raw"]), bytearray(sb[key]["raw"])
        for r in (ra, rb):
            r[96:104] = b"\0" * 8   # byte_offset: depends on the segment order
            r[250:256] = b"\0" * 6  # struct tail padding (unset in the reference)
        assert ra == rb, key
        if key[1] in ("outlier_vals", "outlier_idxs"):
            continue
        assert sa[key]["data"] == sb[key]["data"], key
    q = 14  # StageType::QUANTIZER
    if (q, "outlier_idxs") in sa:
        ia = np.frombuffer(sa[(q, "outlier_idxs")]["data"], np.uint32)
        ib = np.frombuffer(sb[(q, "outlier_idxs")]["data"], np.uint32)
        va = np.frombuffer(sa[(q, "outlier_vals")]["data"], np.uint32)
        vb = np.frombuffer(sb[(q, "outlier_vals")]["data"], np.uint32)
        oa, ob = np.argsort(ia, kind="stable"), np.argsort(ib, kind="stable")
        assert np.array_equal(ia[oa], ib[ob]) and np.array_equal(va[oa], vb[ob])
    assert dsz.value == n * 4
    assert torch.equal(y_live.view(torch.int32), dec.view(torch.int32))
    # decompressFromFile returns the source buffer as the container records
    # it: padded to the pipeline's input alignment, as the reference does
    # (compressor_io.cpp:640-673); the values are the prefix
    assert y_file.numel() * 4 == a["core"]["uncompressed"] >= n * 4
    y_file = y_file[:n]
    assert torch.equal(y_file.view(torch.int32), dec.view(torch.int32))
    if chain != 5:  # the 16-bit Bitpack of chain 5 truncates wide deltas in both libraries
        xd, yd = x.double(), y_file.double()
        if mode == REL:
            assert bool(((yd - xd).abs() <= xd.abs() * eb * 1.01).all())
        else:
            assert float((yd - xd).abs().max()) <= eb * 1.01
    pl.close()
