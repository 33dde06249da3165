"""The fz:: pipeline layer on the GPU: Pipeline / DAG / memory pool / FZM
container through the Python mirror of the reference API.

* round trips of the three hot-path chains (LorenzoQuant -> RLE,
  LorenzoQuant -> Bitshuffle -> RZE, LorenzoQuant -> Huffman), with every
  compressed segment equal to the kernel-level entry points' bytes;
* fused vs stage-by-stage execution, PREALLOCATE vs MINIMAL, CUDA-graph
  replay: identical bytes;
* FZM files: write / read / decompressFromFile, CRC and magic checks;
* container parity with the reference's own Pipeline (oracle/_ref): the
  core, stage and buffer records and every payload segment, keyed by
  (stage type, output name) because the reference orders its pipeline
  outputs by hash-map iteration; outlier segments compared as index-sorted
  sets and the Huffman blob with its scratch bytes masked.
"""
import ctypes as C
import os
import struct

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def P():
    from fzgpumodules_b200 import pipeline
    return pipeline


def K():
    from fzgpumodules_b200 import kernels
    return kernels


def F():
    from fzgpumodules_b200 import fields
    return fields


# ------------------------------------------------------------- FZM parsing

CORE = struct.Struct("<IHHQQQIHH4QII")


def parse_fzm(raw: bytes) -> dict:
    c = CORE.unpack_from(raw, 0)
    core = dict(magic=c[0], version=c[1], num_buffers=c[2], uncompressed=c[3], compressed=c[4], header_size=c[5],
                num_stages=c[6], num_sources=c[7], flags=c[8], sources=c[9:13], data_crc=c[13], header_crc=c[14])
    stages, buffers = [], []
    off = 80
    for _ in range(core["num_stages"]):
        stages.append(raw[off:off + 256])
        off += 256
    for _ in range(core["num_buffers"]):
        b = raw[off:off + 256]
        stype, ver, dtype, pidx, bid = struct.unpack_from("<HHBBH", b, 0)
        name = b[8:72].split(b"\0")[0].decode()
        dsize, asize, usize, boff = struct.unpack_from("<QQQQ", b, 72)
        cfg_size = struct.unpack_from("<I", b, 232)[0]
        buffers.append(dict(raw=b, type=stype, version=ver, dtype=dtype, pidx=pidx, bid=bid, name=name,
                            data_size=dsize, alloc=asize, usize=usize, offset=boff, config=b[104:104 + cfg_size]))
        off += 256
    payload = raw[core["header_size"]:]
    for b in buffers:
        b["data"] = payload[b["offset"]:b["offset"] + b["data_size"]]
    return dict(core=core, stages=stages, buffers=buffers, payload=payload)


# ------------------------------------------------------------- pipelines

def build(chain: str, dims, eb, mode, radius, zigzag, cap=0.2, strategy=None, fusion=True, hint=0):
    p = P()
    pl = p.Pipeline(hint, p.PREALLOCATE if strategy == "pre" else p.MINIMAL)
    pl.setDims(*dims)
    lq = pl.addStage(p.LorenzoQuantStage(eb, radius, cap, mode, zigzag))
    if chain == "rle":
        c = pl.addStage(p.RLEStage(2))
        pl.connect(c, lq, "codes")
    elif chain == "bs_rze":
        bs = pl.addStage(p.BitshuffleStage())
        bs.setElementWidth(2)
        rz = pl.addStage(p.RZEStage())
        pl.connect(bs, lq, "codes")
        pl.connect(rz, bs)
    else:
        hf = pl.addStage(p.HuffmanStage(1024))
        if chain == "huffman_fine":
            hf.setEncodeMode(p.HuffmanEncodeMode.Fine)
        pl.connect(hf, lq, "codes")
    pl.setFusion(fusion)
    pl.finalize()
    return pl


def split_concat(buf: np.ndarray):
    n = int(buf[:4].view(np.uint32)[0])
    sizes = buf[4:4 + 8 * n].view(np.uint64).astype(np.int64)
    off = (4 + 8 * n + 15) & ~15
    segs = []
    for s in sizes:
        segs.append(buf[off:off + s])
        off += (int(s) + 15) & ~15
    return segs


CASES = {
    # name: (chain, dims (x, y, z), eb, mode, radius, zigzag, field)
    "c1_rle_2d": ("rle", (3600, 1800, 1), 1e-4, 0, 32768, False, "sin"),
    "bs_rze_3d_rel": ("bs_rze", (128, 128, 64), 1e-3, 1, 32768, True, "grf"),
    "bs_rze_3d_abs_outliers": ("bs_rze", (256, 64, 32), 1e-3, 0, 512, True, "grf"),
    "huffman_2d": ("huffman", (1024, 1024, 1), 1e-3, 0, 512, True, "fractal"),
    "huffman_fine_2d": ("huffman_fine", (1000, 1000, 1), 1e-3, 0, 512, True, "fractal"),
}


def make_field(kind, dims, dev):
    x, y, z = dims
    if kind == "sin":
        return F().sinusoids2d(y, x, seed=1001).reshape(-1).to(dev)
    if kind == "fractal":
        return F().fractal2d(x, seed=1003).reshape(-1).to(dev)
    return F().grf((z, y, x), seed=1002, spike_frac=1e-3, device=dev).reshape(-1)


@pytest.mark.parametrize("case", list(CASES))
def test_pipeline_roundtrip_and_segments(cuda, case):
    chain, dims, eb, mode, radius, zz, kind = CASES[case]
    x = make_field(kind, dims, cuda)
    pl = build(chain, dims, eb, mode, radius, zz)
    assert pl.isFused() == (chain == "bs_rze")
    comp = pl.compress(x).clone()
    segs = split_concat(comp.cpu().numpy())
    assert len(segs) == 4  # outlier_errors, outlier_indices, outlier_count, coder output
    # the kernel-level path on the same field gives the same segments
    if chain == "bs_rze":
        ref = K().lq_bs_rze_compress(x, dims, eb, mode, radius, zz, 0.2)
        cnt = int(ref["count"].item())
        stored = min(cnt, ref["cap"])
        assert np.array_equal(segs[3], ref["rze"][: int(ref["rze_size"].item())].cpu().numpy())
    else:
        ref = K().lq_forward(x, dims, eb, mode, radius, zz, 0.2)
        cnt = int(ref["count"].item())
        stored = min(cnt, ref["cap"])
        if chain == "rle":
            enc, _ = K().rle_encode(ref["codes"])
        else:
            enc, _ = K().huff_compress(ref["codes"], 1024, fine=chain == "huffman_fine")
        assert np.array_equal(segs[3], enc.cpu().numpy())
    assert np.array_equal(segs[0].view(np.float32), ref["err"][:stored].cpu().numpy())
    assert np.array_equal(segs[1].view(np.uint32), ref["idx"][:stored].cpu().numpy().view(np.uint32))
    assert int(segs[2].view(np.uint32)[0]) == cnt
    y = pl.decompress(comp).clone()
    y2 = pl.decompress(None).clone()
    assert torch.equal(y, y2)
    assert y.numel() == x.numel()
    abs_eb = float(ref["eb_state"][1].item())
    assert float((y - x).abs().max()) <= abs_eb * 1.01
    pl.close()


@pytest.mark.parametrize("case", ["bs_rze_3d_rel", "bs_rze_3d_abs_outliers"])
def test_fused_equals_stage_by_stage(cuda, case):
    chain, dims, eb, mode, radius, zz, kind = CASES[case]
    x = make_field(kind, dims, cuda)
    a = build(chain, dims, eb, mode, radius, zz)
    b = build(chain, dims, eb, mode, radius, zz, fusion=False)
    assert a.isFused() and not b.isFused()
    ca, cb = a.compress(x).clone(), b.compress(x).clone()
    assert torch.equal(ca, cb)
    assert torch.equal(a.decompress(ca), b.decompress(cb))
    a.close()
    b.close()


@pytest.mark.parametrize("case", ["c1_rle_2d", "bs_rze_3d_rel", "huffman_2d", "huffman_fine_2d"])
def test_preallocate_equals_minimal(cuda, case):
    chain, dims, eb, mode, radius, zz, kind = CASES[case]
    x = make_field(kind, dims, cuda)
    n4 = x.numel() * 4
    a = build(chain, dims, eb, mode, radius, zz, strategy="pre", hint=n4)
    b = build(chain, dims, eb, mode, radius, zz, strategy="min")
    ca, cb = a.compress(x).clone(), b.compress(x).clone()
    assert torch.equal(ca, cb)
    assert torch.equal(a.decompress(ca), b.decompress(cb))
    a.close()
    b.close()


def test_graph_replay(cuda):
    chain, dims, eb, mode, radius, zz, kind = CASES["bs_rze_3d_rel"]
    x1 = make_field(kind, dims, cuda)
    x2 = (x1 * 0.5 + 0.25).contiguous()
    p = P()
    pl = p.Pipeline(x1.numel() * 4, p.PREALLOCATE)
    pl.setDims(*dims)
    lq = pl.addStage(p.LorenzoQuantStage(eb, radius, 0.2, mode, zz))
    bs = pl.addStage(p.BitshuffleStage(16384, 2))
    rz = pl.addStage(p.RZEStage())
    pl.connect(bs, lq, "codes")
    pl.connect(rz, bs)
    pl.enableGraphMode(True)
    pl.finalize()
    s = torch.cuda.Stream(device=cuda)
    pl.captureGraph(s)
    eager = build(chain, dims, eb, mode, radius, zz)
    for x in (x1, x2, x1):
        with torch.cuda.stream(s):
            cg = pl.compress(x).clone()
        s.synchronize()
        ce = eager.compress(x).clone()
        assert torch.equal(cg.cpu(), ce.cpu())
    pl.close()
    eager.close()


def test_fzm_roundtrip_and_checks(cuda, tmp_path):
    chain, dims, eb, mode, radius, zz, kind = CASES["bs_rze_3d_abs_outliers"]
    x = make_field(kind, dims, cuda)
    pl = build(chain, dims, eb, mode, radius, zz)
    comp = pl.compress(x).clone()
    y = pl.decompress(comp).clone()
    path = tmp_path / "a.fzm"
    pl.writeToFile(str(path))
    raw = path.read_bytes()
    f = parse_fzm(raw)
    c = f["core"]
    assert c["magic"] == 0x464D5A32 and c["version"] == 0x0301 and c["flags"] == 3
    assert c["num_stages"] == 3 and c["num_buffers"] == 4 and c["num_sources"] == 1
    assert c["uncompressed"] == x.numel() * 4 and c["sources"][0] == x.numel() * 4
    assert c["data_crc"] == O.crc32(f["payload"])
    hdr = bytearray(raw[:c["header_size"]])
    hdr[76:80] = b"\0\0\0\0"
    assert c["header_crc"] == O.crc32(bytes(hdr))
    y2 = P().Pipeline.decompressFromFile(str(path))
    assert torch.equal(y2, y)
    # corruptions are rejected on the host
    bad = bytearray(raw)
    bad[c["header_size"] + 10] ^= 0xFF
    (tmp_path / "b.fzm").write_bytes(bytes(bad))
    with pytest.raises(P().PipelineError, match="data checksum"):
        P().Pipeline.decompressFromFile(str(tmp_path / "b.fzm"))
    bad = bytearray(raw)
    bad[100] ^= 0x01
    (tmp_path / "c.fzm").write_bytes(bytes(bad))
    with pytest.raises(P().PipelineError, match="header checksum"):
        P().Pipeline.decompressFromFile(str(tmp_path / "c.fzm"))
    bad = bytearray(raw)
    bad[0] ^= 0x01
    (tmp_path / "d.fzm").write_bytes(bytes(bad))
    with pytest.raises(P().PipelineError, match="magic"):
        P().Pipeline.decompressFromFile(str(tmp_path / "d.fzm"))
    pl.close()


def test_pipeline_errors(cuda):
    p = P()
    a = np.full(40000, 3, np.uint16)
    a[123] = 2000
    pl = p.Pipeline()
    hf = pl.addStage(p.HuffmanStage(1024))
    pl.finalize()
    with pytest.raises(p.PipelineError, match="bklen"):
        pl.compress(torch.from_numpy(a).to(cuda))
    pl.close()
    pl = p.Pipeline()
    lq = pl.addStage(p.LorenzoQuantStage())
    rz = pl.addStage(p.RZEStage())
    pl.connect(rz, lq, "nope")
    with pytest.raises(p.PipelineError, match="does not have output"):
        pl.finalize()
    pl = p.Pipeline()
    with pytest.raises(p.PipelineError, match="no stages"):
        pl.finalize()


# -------------------------------------------------- reference container

def _ref_pipe():
    path = os.path.join(os.path.dirname(O.REF_STAGES), "libfzref_pipe.so")
    if not os.path.exists(path):
        pytest.skip("reference pipeline build absent")
    L = C.CDLL(path)
    L.ref_pipe_last_error.restype = C.c_char_p
    return L


def _segments(f):
    out = {}
    for b in f["buffers"]:
        out[(b["type"], b["name"])] = b
    return out


@pytest.mark.parametrize("case", ["c1_rle_2d", "bs_rze_3d_rel", "bs_rze_3d_abs_outliers", "huffman_2d"])
def test_fzm_matches_reference_pipeline(cuda, case, tmp_path):
    L = _ref_pipe()
    chain, dims, eb, mode, radius, zz, kind = CASES[case]
    x = make_field(kind, dims, cuda)
    n = x.numel()
    chain_id = {"rle": 0, "bs_rze": 1, "huffman": 2}[chain]
    ref_path = str(tmp_path / "ref.fzm")
    dec = torch.zeros(n, dtype=torch.float32, device=cuda)
    dsz, csz = C.c_size_t(0), C.c_size_t(0)
    rc = L.ref_pipeline_fzm(chain_id, C.c_void_p(x.data_ptr()), C.c_size_t(n), C.c_size_t(dims[0]),
                            C.c_size_t(dims[1]), C.c_size_t(dims[2]), C.c_float(eb), mode, radius, C.c_float(0.2),
                            int(zz), 1, ref_path.encode(), C.c_void_p(dec.data_ptr()), C.byref(dsz), C.byref(csz))
    assert rc == 0, L.ref_pipe_last_error()
    torch.cuda.synchronize()
    pl = build(chain, dims, eb, mode, radius, zz, strategy="pre", hint=n * 4)
    pl.compress(x)
    ours_path = str(tmp_path / "ours.fzm")
    pl.writeToFile(ours_path)
    y = P().Pipeline.decompressFromFile(ours_path)
    a, b = parse_fzm(open(ours_path, "rb").read()), parse_fzm(open(ref_path, "rb").read())
    for k in ("magic", "version", "num_buffers", "uncompressed", "compressed", "header_size", "num_stages",
              "num_sources", "flags", "sources"):
        assert a["core"][k] == b["core"][k], k
    assert a["stages"] == b["stages"]  # types, ids, configs (LorenzoQuant 44 B, coder headers)
    sa, sb = _segments(a), _segments(b)
    assert sa.keys() == sb.keys()
    for key in sa:
        ea, eb_ = sa[key], sb[key]
        ra, rb = bytearray(ea["raw"]), bytearray(eb_["raw"])
        for r in (ra, rb):
            r[96:104] = b"\0" * 8     # byte_offset: depends on the segment order
            r[250:256] = b"\0" * 6    # struct tail padding (unset in the reference)
        assert ra == rb, key
        da, db = np.frombuffer(ea["data"], np.uint8), np.frombuffer(eb_["data"], np.uint8)
        assert da.size == db.size, key
        if key[1] in ("outlier_errors", "outlier_indices"):
            continue  # compared as pairs below
        if key[0] == 6:  # Huffman: header scratch bytes
            da, db = da.copy(), db.copy()
            da[2:4] = db[2:4] = 0
            da[64:128] = db[64:128] = 0
        assert np.array_equal(da, db), key
    lq = 1
    ea_err = np.frombuffer(sa[(lq, "outlier_errors")]["data"], np.float32)
    ea_idx = np.frombuffer(sa[(lq, "outlier_indices")]["data"], np.uint32)
    eb_err = np.frombuffer(sb[(lq, "outlier_errors")]["data"], np.float32)
    eb_idx = np.frombuffer(sb[(lq, "outlier_indices")]["data"], np.uint32)
    oa, ob = np.argsort(ea_idx, kind="stable"), np.argsort(eb_idx, kind="stable")
    assert np.array_equal(ea_idx[oa], eb_idx[ob]) and np.array_equal(ea_err[oa], eb_err[ob])
    assert dsz.value == n * 4
    assert torch.equal(y, dec)  # decompressed floats are bit-identical
    pl.close()


def test_sibling_stages_on_side_streams(cuda):
    """A DAG whose codes feed two coders (Bitshuffle -> RZE and RLE): the
    coders share a level, so the pipeline keeps side streams and forks that
    level onto them (Pipeline::setNumStreams, dag.cpp:343-369,752-762).  Each
    branch's segment equals the one its linear pipeline writes, eagerly, with
    the bounds check on, and from a replayed CUDA graph."""
    p = P()
    dims = (128, 64, 32)
    x = make_field("grf", dims, cuda)
    n4 = x.numel() * 4

    def branched(streams, graph=False):
        pl = p.Pipeline(n4, p.PREALLOCATE)
        pl.setDims(*dims)
        lq = pl.addStage(p.LorenzoQuantStage(1e-3, 32768, 0.2, p.REL, True))
        bs = pl.addStage(p.BitshuffleStage(16384, 2))
        rz = pl.addStage(p.RZEStage())
        rl = pl.addStage(p.RLEStage(2))
        pl.connect(bs, lq, "codes")
        pl.connect(rz, bs)
        pl.connect(rl, lq, "codes")
        pl.setNumStreams(streams)
        pl.enableBoundsCheck(True)
        pl.enableGraphMode(graph)
        pl.finalize()
        return pl

    lin_rze = build("bs_rze", dims, 1e-3, 1, 32768, True)
    lin_rle = build("rle", dims, 1e-3, 1, 32768, True)
    seg_rze = split_concat(lin_rze.compress(x).clone().cpu().numpy())[3]
    seg_rle = split_concat(lin_rle.compress(x).clone().cpu().numpy())[3]
    for streams in (1, 3):
        pl = branched(streams)
        assert pl.getNumStreams() == max(streams, 2)
        comp = pl.compress(x).clone()
        segs = split_concat(comp.cpu().numpy())
        assert len(segs) == 5  # three outlier segments, the RZE stream, the RLE stream
        assert np.array_equal(segs[3], seg_rze) and np.array_equal(segs[4], seg_rle)
        y = pl.decompress(comp).clone()
        assert torch.equal(y, lin_rze.decompress(None))
        pl.close()
    g = branched(2, graph=True)
    s = torch.cuda.Stream(device=cuda)
    g.captureGraph(s)
    with torch.cuda.stream(s):
        cg = g.compress(x).clone()
    s.synchronize()
    segs = split_concat(cg.cpu().numpy())
    assert np.array_equal(segs[3], seg_rze) and np.array_equal(segs[4], seg_rle)
    for pl in (g, lin_rze, lin_rle):
        pl.close()


@pytest.mark.parametrize("chain,fusion", [("bs_rze", True), ("bs_rze", False), ("rle", True)])
def test_graph_decompress_on_new_inputs(cuda, chain, fusion):
    """captureGraph also captures the decompression: the container is split on
    the device, the error bound comes from the compressor's device state, and
    decompress() returns without waiting on the host.  For each new field --
    the second one with a different REL value base -- the replayed
    decompression equals an eager pipeline's bit for bit, from the pipeline's
    own outputs and from a copy of the container; a container with a bad
    header is reported by checkDecompressStatus."""
    p = P()
    dims = (128, 128, 64)
    mode = p.REL if chain == "bs_rze" else p.ABS
    x1 = make_field("grf", dims, cuda)
    xs = (x1, (x1 * 0.5 + 0.25).contiguous(), F().grf(dims[::-1], seed=9, spike_frac=1e-3, device=cuda).reshape(-1))
    pl = p.Pipeline(x1.numel() * 4, p.PREALLOCATE)
    pl.setDims(*dims)
    lq = pl.addStage(p.LorenzoQuantStage(1e-3, 32768, 0.2, mode, True))
    if chain == "bs_rze":
        bs = pl.addStage(p.BitshuffleStage(16384, 2))
        rz = pl.addStage(p.RZEStage())
        pl.connect(bs, lq, "codes")
        pl.connect(rz, bs)
    else:
        rl = pl.addStage(p.RLEStage(2))
        pl.connect(rl, lq, "codes")
    pl.enableGraphMode(True)
    pl.setFusion(fusion)
    pl.finalize()
    s = torch.cuda.Stream(device=cuda)
    pl.captureGraph(s)
    assert pl.isDecompressGraphCaptured()
    eager = build(chain, dims, 1e-3, mode, 32768, True, fusion=fusion)
    for x in xs:
        with torch.cuda.stream(s):
            c = pl.compress(x).clone()
            y = pl.decompress(None).clone()
            y2 = pl.decompress(c).clone()
            pl.checkDecompressStatus()
        s.synchronize()
        ce = eager.compress(x).clone()
        ye = eager.decompress(ce).clone()
        assert torch.equal(c, ce)
        assert torch.equal(y.view(torch.int32), ye.view(torch.int32))
        assert torch.equal(y2.view(torch.int32), ye.view(torch.int32))
    bad = c.clone()
    bad[0] = 99  # the header's segment count
    with torch.cuda.stream(s):
        pl.decompress(bad)
        with pytest.raises(p.PipelineError, match="malformed"):
            pl.checkDecompressStatus()
    s.synchronize()
    pl.close()
    eager.close()
