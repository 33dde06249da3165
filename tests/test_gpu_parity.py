"""GPU parity: libfzb.so kernels vs the CPU oracle (bit-exact) and vs the
reference's own stage kernels built from its sources (oracle/_ref), on the
same seeded inputs."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

K = None


def kern():
    global K
    if K is None:
        from fzgpumodules_b200 import kernels
        K = kernels
    return K


def _field(n, seed, kind="smooth"):
    rng = np.random.default_rng(seed)
    if kind == "smooth":
        x = np.cumsum(rng.normal(size=n)).astype(np.float32)
        x /= np.abs(x).max()
        return x.astype(np.float32)
    if kind == "noise":
        return rng.normal(size=n).astype(np.float32)
    if kind == "spiky":
        x = np.cumsum(rng.normal(size=n) * 0.01).astype(np.float32)
        pos = rng.choice(n, max(1, n // 500), replace=False)
        x[pos] = rng.choice([-1e3, 1e3], pos.size)
        return x.astype(np.float32)
    if kind == "blocks":  # zero stretches (all-zero chunks) and constant runs
        x = np.repeat(rng.normal(size=n // 4096 + 1), 4096)[:n].astype(np.float32)
        x[(np.arange(n) // 8192) % 3 == 0] = 0.0
        return x
    if kind == "special":  # NaN / +-inf / huge values among a smooth field
        x = np.cumsum(rng.normal(size=n) * 0.01).astype(np.float32)
        pos = rng.choice(n, max(4, n // 300), replace=False)
        x[pos] = rng.choice(np.array([np.nan, np.inf, -np.inf, 3e30, -2e25, 1e9], np.float32), pos.size)
        return x
    raise ValueError(kind)


def _midpoint_field(n, seed, eb):
    """Values whose float product with ebx2_r = 1/(2 eb) lands exactly on k + 0.5
    while the exact product does not: a fused multiply-add would round them
    to the other integer."""
    r = np.float32(1.0) / (np.float32(2.0) * np.float32(eb))
    rng = np.random.default_rng(seed)
    found = []
    for k in rng.integers(-3000, 3000, 4000):
        t = float(k) + 0.5
        v0 = np.array([t / float(r)], np.float32).view(np.int32)[0]
        for j in range(-3, 4):
            v = np.array([v0 + j], np.int32).view(np.float32)
            if float(v[0] * r) == t and float(v[0]) * float(r) != t:
                found.append(v[0])
    found = np.array(found, np.float32)
    assert found.size > 100
    return found[rng.integers(0, found.size, n)]


def _g(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _h(t):
    return t.cpu().numpy()


def _oracle_forward(x, dims, eb, mode, radius, zz, cap, value_base=0.0):
    vb = value_base if value_base > 0 else (O.value_base(x, mode) if mode else 0.0)
    abs_eb, r, e2 = O.resolve_eb(eb, mode, vb)
    codes, err, idx, cnt = O.lq_fwd(x, dims, r, radius, zz, cap=cap, n_total=x.size)
    return codes, err, idx, cnt, abs_eb, r, e2, vb


GEOMS = [
    (10000, 1, 1), (8192 * 3 + 77, 1, 1),         # 1-D (+ partial chunk)
    (100, 70, 1), (37, 19, 1), (256, 96, 1),      # 2-D odd / row-aligned
    (9000, 3, 1),                                  # 2-D rows wider than a chunk
    (33, 17, 11), (64, 32, 16), (512, 16, 16),    # 3-D odd / row-aligned
    (96, 40, 9),                                   # 3-D chunks spanning planes
    (20, 13, 9), (100, 24, 10),                    # 3-D rows a multiple of 4, not of 32 (16-byte runs)
]


@pytest.mark.parametrize("dims", GEOMS)
@pytest.mark.parametrize("mode,zz,radius,kind", [
    (O.ABS, False, 32768, "smooth"), (O.REL, True, 32768, "spiky"),
    (O.ABS, True, 512, "spiky"), (O.NOA, False, 64, "noise")])
def test_lq_forward_matches_oracle(cuda, dims, mode, zz, radius, kind):
    n = int(np.prod(dims))
    x = _field(n, 11, kind)
    cap = int(np.ceil(n * 0.2))
    codes, err, idx, cnt, abs_eb, r, e2, vb = _oracle_forward(x, dims, 1e-3, mode, radius, zz, cap)
    out = kern().lq_forward(_g(x, cuda), dims, 1e-3, mode, radius, zz, 0.2)
    st = _h(out["eb_state"])
    assert st[1] == abs_eb and st[2] == r and st[3] == e2
    assert np.array_equal(_h(out["codes"]), codes)
    gcnt = int(_h(out["count"])[0])
    assert gcnt == cnt
    _check_outliers(out, x, dims, mode, radius, zz, cap, cnt, idx, err)


@pytest.mark.parametrize("dims", [(37, 19, 5), (3000, 7, 1), (33, 17, 11), (20, 13, 9), (200, 9, 7), (8192, 6, 1),
                                  (40000, 1, 1)])
def test_element_path_large_prequant_values(cuda, dims):
    """Rows that are not a multiple of 32 elements take the element path,
    which carries each element's x-neighbour terms along the run.  With an
    absolute bound of 1e-5 on values up to 1e3 the prequantised values reach
    5e7, above 2^24, so float differences round and their order matters: the
    codes and every outlier's error must still equal the oracle's."""
    n = int(np.prod(dims))
    rng = np.random.default_rng(23)
    x = rng.uniform(-1e3, 1e3, n).astype(np.float32)
    x[::7] = np.float32(0.0)
    cap = n
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-5, O.ABS, 32768, True, cap)
    out = kern().lq_forward(_g(x, cuda), dims, 1e-5, O.ABS, 32768, True, 1.0)
    assert np.array_equal(_h(out["codes"]), codes)
    assert int(_h(out["count"])[0]) == cnt
    _check_outliers(out, x, dims, O.ABS, 32768, True, cap, cnt, idx, err)


def _check_outliers(out, x, dims, mode, radius, zz, cap, cnt, idx, err):
    k = min(cnt, cap)
    gi = _h(out["idx"])[:k].view(np.uint32)
    ge = _h(out["err"])[:k].view(np.uint32)
    if cnt <= cap:  # every outlier stored, sorted by index
        assert np.array_equal(gi, idx)
        assert np.array_equal(ge, err.view(np.uint32))
    else:  # overflow: cap of them stored (which ones depends on order), sorted, exact values
        _, aerr, aidx, _, *_ = _oracle_forward(x, dims, 1e-3, mode, radius, zz, cnt)
        assert np.all(np.diff(gi.astype(np.int64)) > 0)
        pos = np.searchsorted(aidx, gi)
        assert np.all(aidx[pos] == gi)
        assert np.array_equal(aerr.view(np.uint32)[pos], ge)


@pytest.mark.parametrize("dims", GEOMS)
def test_lq_inverse_matches_oracle(cuda, dims):
    n = int(np.prod(dims))
    x = _field(n, 12, "spiky")
    cap = n
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-3, O.ABS, 512, True, cap)
    y = O.lq_inv(codes, err, idx, dims, e2, True)
    dc = kern().lq_inverse(_g(codes, cuda), _g(np.append(err, np.float32(0)), cuda),
                           _g(np.append(idx, 0).astype(np.int32), cuda),
                           _g(np.int32([cnt]), cuda), cap, dims, float(abs_eb), True)
    assert np.array_equal(_h(dc).view(np.uint32), y.view(np.uint32))
    assert np.max(np.abs(y - x)) <= 1e-3 * 1.01


@pytest.mark.parametrize("ew", [1, 2, 4, 8])
def test_bitshuffle_matches_oracle(cuda, ew):
    rng = np.random.default_rng(13)
    d = rng.integers(0, 256, 16384 * 5 + 300, dtype=np.uint8)
    d[: 16384] &= 0x3
    s = kern().bitshuffle(_g(d, cuda), 16384, ew)
    assert np.array_equal(_h(s), O.bitshuffle(d, 16384, ew))
    back = kern().bitshuffle(s, 16384, ew, inverse=True)
    assert np.array_equal(_h(back), d)
    s2 = kern().bitshuffle(_g(d[: 8192 * 3], cuda), 8192, ew)  # non-default block
    assert np.array_equal(_h(s2), O.bitshuffle(d[: 8192 * 3], 8192, ew))
    s3 = kern().bitshuffle(_g(d, cuda), 65536, ew)  # larger block, ragged tail
    assert np.array_equal(_h(s3), O.bitshuffle(d, 65536, ew))
    assert np.array_equal(_h(kern().bitshuffle(s3, 65536, ew, inverse=True)), d)


@pytest.mark.parametrize("ew", [1, 2, 4, 8])
def test_reference_bitshuffle_widths(cuda, ew):
    """The reference's own BitshuffleStage (ballot kernels for widths 1-2,
    butterfly kernels for 4-8) equals the oracle and ours, both ways."""
    L = _ref()
    rng = np.random.default_rng(15 + ew)
    d = rng.integers(0, 256, 16384 * 4, dtype=np.uint8)
    d[:16384] &= 0x11
    din = _g(d, cuda)
    for block in (16384, 8192 * ew):
        ref = torch.empty_like(din)
        assert L.ref_bitshuffle(_vp(din), C.c_size_t(d.size), block, ew, 0, _vp(ref)) == 0, L.ref_last_error()
        want = O.bitshuffle(d, block, ew)
        assert np.array_equal(_h(ref), want)
        ours = kern().bitshuffle(din, block, ew)
        assert np.array_equal(_h(ours), want)
        back = torch.empty_like(din)
        assert L.ref_bitshuffle(_vp(ref), C.c_size_t(d.size), block, ew, 1, _vp(back)) == 0, L.ref_last_error()
        assert np.array_equal(_h(back), d)


def _byte_cases():
    rng = np.random.default_rng(14)
    sparse = np.zeros(16384 * 7, np.uint8)
    sparse[rng.choice(sparse.size, 900, replace=False)] = rng.integers(1, 256, 900)
    return {
        "zeros": np.zeros(16384 * 2, np.uint8),
        "random": rng.integers(0, 256, 16384 * 3, dtype=np.uint8),
        "sparse": sparse,
        "runs": np.repeat(rng.integers(0, 4, 400, dtype=np.uint8), 330),
        "partial": rng.integers(0, 3, 3000, dtype=np.uint8),
        "mixed": np.concatenate([np.zeros(16384, np.uint8), rng.integers(0, 256, 16384, dtype=np.uint8),
                                 np.repeat(np.uint8([1, 2, 3]), 5001)]),
        "near_raw": (rng.random(16384 * 2) < 0.93).astype(np.uint8) * rng.integers(1, 256, 16384 * 2, dtype=np.uint8),
    }


@pytest.mark.parametrize("kind", list(_byte_cases().keys()))
def test_rze_matches_oracle(cuda, kind):
    d = _byte_cases()[kind]
    ref = O.rze_encode(d)
    enc, size = kern().rze_encode(_g(d, cuda))
    assert int(size.item()) == ref.size
    assert np.array_equal(_h(enc), ref)
    dec = kern().rze_decode(enc, d.size)
    assert np.array_equal(_h(dec), d)


FUSED_GEOMS = [(512, 16, 16), (64, 32, 24), (33, 17, 11), (256, 96, 1), (8192 * 2 + 5, 1, 1),
               (1024, 8, 9), (96, 40, 9), (64, 256, 10), (100, 24, 10), (200, 17, 12), (1000, 9, 1)]


@pytest.mark.parametrize("dims", FUSED_GEOMS)
@pytest.mark.parametrize("mode,zz,radius,kind", [
    (O.REL, True, 32768, "spiky"), (O.ABS, True, 512, "spiky"), (O.ABS, False, 32768, "noise")])
def test_fused_compress_matches_oracle_chain(cuda, dims, mode, zz, radius, kind):
    n = int(np.prod(dims))
    x = _field(n, 15, kind)
    cap = int(np.ceil(n * 0.1))
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-3, mode, radius, zz, cap)
    stream = O.rze_encode(O.bitshuffle(codes, 16384, 2))
    out = kern().lq_bs_rze_compress(_g(x, cuda), dims, 1e-3, mode, radius, zz, 0.1)
    size = int(_h(out["rze_size"])[0])
    assert size == stream.size
    assert np.array_equal(_h(out["rze"])[:size], stream)
    assert int(_h(out["count"])[0]) == cnt
    _check_outliers(out, x, dims, mode, radius, zz, cap, cnt, idx, err)
    # inverse: fused single pass (when the geometry allows) and the exact path
    y = O.lq_inv(codes, err, idx, dims, e2, zz)
    for flags in (0, kern().FORCE_EXACT):
        dec = kern().lq_bs_rze_decompress(out["rze"], size, out["err"], out["idx"], out["count"],
                                          out["cap"], n, dims, float(abs_eb), zz, flags=flags)
        assert np.array_equal(_h(dec).view(np.uint32), y.view(np.uint32)), f"flags={flags}"


@pytest.mark.parametrize("dims", [(8192 * 1024 + 5, 1, 1), (256, 256, 130), (37, 19, 5)])
def test_tiled_and_single_cta_scans_agree(cuda, dims, monkeypatch):
    # the assembly scan and the inverse prepass: a CTA per 1024 chunks (each
    # summing the chunks before its tile) and the single-CTA scans equal the
    # oracle's stream, outlier lists and reconstruction (1025 chunks: two tiles)
    n = int(np.prod(dims))
    x = _field(n, 41, "spiky")
    cap = int(np.ceil(n * 0.1))
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-3, O.ABS, 512, True, cap)
    stream = O.rze_encode(O.bitshuffle(codes, 16384, 2))
    y = O.lq_inv(codes, err, idx, dims, e2, True)
    for flag in ("0", "16"):
        monkeypatch.setenv("FZB_DISABLE_SLAB", flag)
        out = kern().lq_bs_rze_compress(_g(x, cuda), dims, 1e-3, O.ABS, 512, True, 0.1)
        size = int(_h(out["rze_size"])[0])
        assert size == stream.size and np.array_equal(_h(out["rze"])[:size], stream), flag
        assert int(_h(out["count"])[0]) == cnt, flag
        _check_outliers(out, x, dims, O.ABS, 512, True, cap, cnt, idx, err)
        dec = kern().lq_bs_rze_decompress(out["rze"], size, out["err"], out["idx"], out["count"],
                                          out["cap"], n, dims, float(abs_eb), True)
        assert np.array_equal(_h(dec).view(np.uint32), y.view(np.uint32)), flag
        got = kern().lq_forward(_g(x, cuda), dims, 1e-3, O.ABS, 512, True, 0.1)
        assert np.array_equal(_h(got["codes"]), codes), flag
        _check_outliers(got, x, dims, O.ABS, 512, True, cap, cnt, idx, err)


@pytest.mark.parametrize("dims", [(512, 32, 16), (64, 256, 10), (32, 256, 9), (1024, 16, 17), (128, 64, 3)])
@pytest.mark.parametrize("kind,eb,radius,zz", [("spiky", 1e-3, 512, True), ("noise", 1e-3, 32768, False),
                                               ("blocks", 1e-3, 32768, True), ("special", 1e-3, 64, True)])
def test_fused_compress_slab_and_chunk_kernels_agree(cuda, dims, kind, eb, radius, zz, monkeypatch):
    # the TMA slab kernel, the cp.async slab kernel and the per-chunk kernel
    # must emit identical bytes (raw, all-zero and outlier-heavy chunks included)
    n = int(np.prod(dims))
    x = _g(_field(n, 18, kind), cuda)
    outs = []
    for flag in ("0", "2", "1"):
        monkeypatch.setenv("FZB_DISABLE_SLAB", flag)
        outs.append(kern().lq_bs_rze_compress(x, dims, eb, O.ABS, radius, zz, 1.0))
    a = outs[0]
    sa = int(_h(a["rze_size"])[0])
    k = int(_h(a["count"])[0])
    if kind in ("spiky", "special"):
        assert k > 0
    for b in outs[1:]:
        sb = int(_h(b["rze_size"])[0])
        assert sa == sb and np.array_equal(_h(a["rze"])[:sa], _h(b["rze"])[:sb])
        assert k == int(_h(b["count"])[0])
        assert np.array_equal(_h(a["idx"])[:k], _h(b["idx"])[:k])
        assert np.array_equal(_h(a["err"])[:k].view(np.uint32), _h(b["err"])[:k].view(np.uint32))
    # inverse: persistent slab kernel, per-tile fused kernel and the exact path agree bit for bit
    abs_eb = float(_h(a["eb_state"])[1])
    decs = []
    for flag, flags in (("0", 0), ("4", 0), ("0", kern().FORCE_EXACT)):
        monkeypatch.setenv("FZB_DISABLE_SLAB", flag)
        decs.append(_h(kern().lq_bs_rze_decompress(a["rze"], sa, a["err"], a["idx"], a["count"], a["cap"], n,
                                                   dims, abs_eb, zz, flags=flags)).view(np.uint32))
    assert np.array_equal(decs[0], decs[2]) and np.array_equal(decs[1], decs[2])


@pytest.mark.parametrize("dims", [(8192, 77, 1), (16384, 40, 1), (8192, 33, 1)])
@pytest.mark.parametrize("mode,zz,radius,kind", [(O.REL, True, 32768, "spiky"), (O.ABS, True, 512, "spiky"),
                                                 (O.NOA, False, 64, "noise")])
def test_row_walk_codes_match_oracle(cuda, dims, mode, zz, radius, kind, monkeypatch):
    """2-D fields whose rows are whole chunks: the row walk (each row's
    q(k - nx) window is the previous row's q(k) window) and the per-chunk
    kernel give the oracle's codes and outliers."""
    n = int(np.prod(dims))
    x = _field(n, 29, kind)
    cap = n
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-3, mode, radius, zz, cap)
    for flag in ("0", "8"):
        monkeypatch.setenv("FZB_DISABLE_SLAB", flag)
        out = kern().lq_forward(_g(x, cuda), dims, 1e-3, mode, radius, zz, 1.0)
        assert np.array_equal(_h(out["codes"]), codes), flag
        assert int(_h(out["count"])[0]) == cnt, flag
        _check_outliers(out, x, dims, mode, radius, zz, cap, cnt, idx, err)


@pytest.mark.parametrize("dims", [(8192, 40, 1), (16384, 9, 1), (65536, 1, 1)])
def test_register_paths_rounding_midpoints(cuda, dims, monkeypatch):
    # the 2-D row walk and the 1-D register front end quantize in registers
    # (round half away from zero as trunc(y + copysign(0.49999997, y))): next
    # to every rounding midpoint their codes equal the oracle's and the
    # per-chunk kernel's
    n = int(np.prod(dims))
    x = _midpoint_field(n, 37, 1e-3)
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-3, O.ABS, 32768, True, n)
    for flag in ("0", "8"):
        monkeypatch.setenv("FZB_DISABLE_SLAB", flag)
        out = kern().lq_forward(_g(x, cuda), dims, 1e-3, O.ABS, 32768, True, 1.0)
        assert np.array_equal(_h(out["codes"]), codes), flag
        assert int(_h(out["count"])[0]) == cnt, flag


@pytest.mark.parametrize("dims", [(256, 64, 9), (512, 16, 8), (96, 40, 9)])
def test_rounding_midpoints_match_oracle(cuda, dims, monkeypatch):
    # every element sits next to a rounding midpoint of x * ebx2_r: codes must
    # come from the rounded product, with no fused multiply-add
    n = int(np.prod(dims))
    eb = 1e-3
    x = _midpoint_field(n, 31, eb)
    cap = n
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, eb, O.ABS, 32768, True, cap)
    stream = O.rze_encode(O.bitshuffle(codes, 16384, 2))
    for flag in ("0", "1"):  # slab kernel where it applies, and the per-chunk kernel
        monkeypatch.setenv("FZB_DISABLE_SLAB", flag)
        out = kern().lq_bs_rze_compress(_g(x, cuda), dims, eb, O.ABS, 32768, True, 1.0)
        size = int(_h(out["rze_size"])[0])
        assert size == stream.size and np.array_equal(_h(out["rze"])[:size], stream), flag
    got = kern().lq_forward(_g(x, cuda), dims, eb, O.ABS, 32768, True, 1.0)
    assert np.array_equal(_h(got["codes"]), codes)


def test_fused_decompress_exactness_fallback(cuda):
    # huge deltas leave the exact-integer regime: the fused inverse must flag
    # it and the host must rerun the exact kernels (same bits as the oracle)
    dims = (64, 16, 16)
    n = int(np.prod(dims))
    rng = np.random.default_rng(16)
    x = (rng.normal(size=n) * 1e4).astype(np.float32)
    cap = n
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-4, O.ABS, 32768, True, cap)
    y = O.lq_inv(codes, err, idx, dims, e2, True)
    out = kern().lq_bs_rze_compress(_g(x, cuda), dims, 1e-4, O.ABS, 32768, True, 1.0)
    size = int(_h(out["rze_size"])[0])
    dec = kern().lq_bs_rze_decompress(out["rze"], size, out["err"], out["idx"], out["count"],
                                      out["cap"], n, dims, float(abs_eb), True)
    assert np.array_equal(_h(dec).view(np.uint32), y.view(np.uint32))


def test_malformed_stream_reports_error(cuda):
    d = _byte_cases()["sparse"]
    enc, size = kern().rze_encode(_g(d, cuda))
    bad = enc.clone()
    bad[8:12] = torch.tensor([0xff, 0xff, 0x00, 0x00], dtype=torch.uint8, device=cuda)  # chunk 0 size
    with pytest.raises(Exception):
        kern().rze_decode(bad, d.size)
        st = kern()._default_ws.status()
        if st != 0:
            raise RuntimeError(st)


# ----------------------------------------------------------- reference kernels

def _ref():
    if not os.path.exists(O.REF_STAGES):
        pytest.skip("reference stage build absent")
    L = C.CDLL(O.REF_STAGES)
    L.ref_last_error.restype = C.c_char_p
    return L


def _vp(t):
    return C.c_void_p(t.data_ptr())


REF_GEOMS = [(10000, 1, 1), (100, 70, 1), (33, 17, 11), (512, 16, 16), (256, 96, 1)]


@pytest.mark.parametrize("dims", REF_GEOMS)
@pytest.mark.parametrize("mode,zz,radius,kind", [
    (O.REL, True, 32768, "spiky"), (O.ABS, True, 512, "spiky"), (O.NOA, False, 32768, "smooth")])
def test_reference_kernels_match_oracle_and_ours(cuda, dims, mode, zz, radius, kind):
    L = _ref()
    n = int(np.prod(dims))
    x = _field(n, 17, kind)
    cap = int(np.ceil(n * 0.2))
    dx = _g(x, cuda)
    codes = torch.empty(n, dtype=torch.int16, device=cuda)
    err = torch.empty(cap, dtype=torch.float32, device=cuda)
    idx = torch.empty(cap, dtype=torch.int32, device=cuda)
    cnt = torch.zeros(1, dtype=torch.int32, device=cuda)
    hdr = (C.c_uint8 * 128)()
    nx, ny, nz = dims
    rc = L.ref_lq_fwd(_vp(dx), C.c_size_t(n), C.c_size_t(nx), C.c_size_t(ny), C.c_size_t(nz),
                      C.c_float(1e-3), mode, radius, C.c_float(0.2), int(zz), _vp(codes), _vp(err),
                      _vp(idx), _vp(cnt), hdr)
    assert rc == 0, L.ref_last_error()
    rcnt = int(_h(cnt)[0])
    ocodes, oerr, oidx, ocnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-3, mode, radius, zz, cap)
    assert rcnt == ocnt
    assert np.array_equal(_h(codes).view(np.uint16), ocodes)
    k = min(rcnt, cap)
    order = np.argsort(_h(idx)[:k].view(np.uint32), kind="stable")
    assert np.array_equal(_h(idx)[:k].view(np.uint32)[order], oidx)  # same set, sorted
    assert np.array_equal(_h(err)[:k].view(np.uint32)[order], oerr.view(np.uint32))
    hv = np.frombuffer(bytes(hdr), np.uint8)
    assert hv[:4].view(np.float32)[0] == abs_eb  # header error_bound
    # reference inverse on its own outputs == oracle inverse == ours
    out = torch.empty(n, dtype=torch.float32, device=cuda)
    rc = L.ref_lq_inv(_vp(codes), _vp(err), _vp(idx), _vp(cnt), C.c_size_t(n), C.c_size_t(cap),
                      hdr, _vp(out))
    assert rc == 0, L.ref_last_error()
    y = O.lq_inv(ocodes, oerr, oidx, dims, e2, zz)
    assert np.array_equal(_h(out).view(np.uint32), y.view(np.uint32))


@pytest.mark.parametrize("kind", ["sparse", "random", "partial", "mixed", "near_raw"])
def test_reference_rze_and_bitshuffle_match(cuda, kind):
    L = _ref()
    d = _byte_cases()[kind]
    n = d.size
    din = _g(d, cuda)
    out = torch.zeros(int(O.lib().orc_rze_max_bytes(n)) + 64, dtype=torch.uint8, device=cuda)
    nb = C.c_size_t(0)
    rc = L.ref_rze_encode(_vp(din), C.c_size_t(n), _vp(out), C.byref(nb))
    assert rc == 0, L.ref_last_error()
    ref_stream = _h(out)[: nb.value]
    assert np.array_equal(ref_stream, O.rze_encode(d))
    if n % 16384 == 0:
        bs = torch.empty_like(din)
        assert L.ref_bitshuffle(_vp(din), C.c_size_t(n), 16384, 2, 0, _vp(bs)) == 0
        assert np.array_equal(_h(bs), O.bitshuffle(d, 16384, 2))


@pytest.mark.parametrize("case", ["in_regime", "inexact", "unsorted"])
def test_device_fallback_decompress(cuda, case):
    # the inverse with no host wait (fzb_lq_bs_rze_decompress_dev): the error
    # bound is read on the device, and the exact kernels follow the fused pass
    # gated on its status -- they take over for huge deltas (inexact) and for
    # outlier lists not in index order (the reference's atomic order), and
    # stay idle otherwise; every case equals the oracle bit for bit
    dims = (64, 16, 16) if case != "in_regime" else (128, 64, 32)
    n = int(np.prod(dims))
    rng = np.random.default_rng(16)
    if case == "inexact":
        x = (rng.normal(size=n) * 1e4).astype(np.float32)
    else:
        x = _field(n, 29, "spiky")
    cap = n
    codes, err, idx, cnt, abs_eb, r, e2, _ = _oracle_forward(x, dims, 1e-4, O.ABS, 512, True, cap)
    y = O.lq_inv(codes, err, idx, dims, e2, True)
    out = kern().lq_bs_rze_compress(_g(x, cuda), dims, 1e-4, O.ABS, 512, True, 1.0)
    k = int(_h(out["count"])[0])
    assert k == cnt and k > 0
    if case == "unsorted":
        order = torch.arange(k - 1, -1, -1, device=cuda)
        out["err"][:k] = out["err"][:k][order].clone()
        out["idx"][:k] = out["idx"][:k][order].clone()
    ws = kern().Workspace()
    dec = kern().lq_bs_rze_decompress_dev(out["rze"], out["rze"].numel(), out["err"], out["idx"], out["count"],
                                          out["cap"], n, dims, out["eb_state"][1:2], True, ws=ws)
    assert ws.status() == 0
    assert np.array_equal(_h(dec).view(np.uint32), y.view(np.uint32))
