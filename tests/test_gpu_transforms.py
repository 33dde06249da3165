"""GPU parity of the stages around the codes: Zigzag, Negabinary, Difference,
lossless integer Lorenzo and the direct Quantizer, through the C ABI.

Integer stages are bit-exact against the oracle at every element width and
against the reference's own kernels (built from its sources) for int32.  The
Quantizer is bit-exact against the oracle for ABS / NOA / in-place and
against the reference's kernels for every mode, REL included (its codes come
from CUDA's __log2f / exp2f, which only the GPU reproduces); outlier lists
are compared as sets because the reference fills them in atomicAdd order."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

UT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}
TT = {1: torch.uint8, 2: torch.int16, 4: torch.int32, 8: torch.int64}


def K():
    from fzgpumodules_b200 import kernels
    return kernels


def _bits(n, ew, seed, lo=None, hi=None):
    rng = np.random.default_rng(seed)
    if lo is None:
        return rng.integers(0, 2**63, n, dtype=np.uint64, endpoint=False).astype(UT[ew])
    return rng.integers(lo, hi, n).astype({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[ew]).view(UT[ew])


def _dev(a: np.ndarray, cuda):
    return torch.from_numpy(a.view({1: np.uint8, 2: np.int16, 4: np.int32, 8: np.int64}[a.itemsize]).copy()).to(cuda)


def _host(t: torch.Tensor, ew: int) -> np.ndarray:
    return t.cpu().numpy().view(UT[ew])


def _ref():
    if not os.path.exists(O.REF_STAGES):
        pytest.skip("reference stage build absent")
    L = C.CDLL(O.REF_STAGES)
    L.ref_last_error.restype = C.c_char_p
    return L


def _vp(t):
    return C.c_void_p(t.data_ptr())


# ------------------------------------------------------------ zigzag / negabinary

@pytest.mark.parametrize("ew", [1, 2, 4, 8])
@pytest.mark.parametrize("n", [0, 1, 17, 4096, 100_003])
def test_zigzag_negabinary_match_oracle(cuda, ew, n):
    a = _bits(n, ew, n + ew)
    d = _dev(a, cuda)
    for fn, orc in ((K().zigzag, O.zigzag), (K().negabinary, O.negabinary)):
        for inv in (False, True):
            got = _host(fn(d, inverse=inv), ew)
            assert np.array_equal(got, orc(a, inverse=inv))


def test_transforms_unaligned_and_in_place(cuda):
    a = _bits(50_001, 4, 5)
    d = _dev(a, cuda)
    for off in (1, 3):  # start off the 16-byte boundary: scalar path
        got = _host(K().zigzag(d[off:]), 4)
        assert np.array_equal(got, O.zigzag(a[off:]))
    e = d.clone()
    K().negabinary(e, out=e)  # in place
    assert np.array_equal(_host(e, 4), O.negabinary(a))


# ------------------------------------------------------------ difference

@pytest.mark.parametrize("ew", [1, 2, 4, 8])
@pytest.mark.parametrize("chunk", [0, 16, 4096, 8192, 1 << 20])
@pytest.mark.parametrize("nb", [False, True])
def test_diff_matches_oracle(cuda, ew, chunk, nb):
    n = 3 * 4096 * 7 + 123  # many scan tiles and a partial one
    a = _bits(n, ew, chunk + ew, -30_000 if ew > 1 else -100, 30_000 if ew > 1 else 100)
    d = _dev(a, cuda)
    fwd = K().diff(d, chunk * ew, nb)
    want = O.diff(a, chunk, nb)
    assert np.array_equal(_host(fwd, ew), want)
    inv = K().diff(fwd, chunk * ew, nb, inverse=True)
    assert np.array_equal(_host(inv, ew), a)


def test_diff_edge_sizes(cuda):
    for n in (1, 2, 15, 16, 4095, 4096, 4097):
        a = _bits(n, 4, n)
        d = _dev(a, cuda)
        for chunk in (0, 4):
            fwd = K().diff(d, chunk * 4, True)
            assert np.array_equal(_host(fwd, 4), O.diff(a, chunk, True))
            assert np.array_equal(_host(K().diff(fwd, chunk * 4, True, inverse=True), 4), a)
    with pytest.raises(Exception):
        K().diff(_dev(_bits(64, 4, 1), cuda), 12)  # chunk of 3 elements: not a power of two


@pytest.mark.parametrize("chunk_bytes,nb", [(0, False), (16384, True), (64, True), (1 << 20, False)])
def test_diff_matches_reference_kernels(cuda, chunk_bytes, nb):
    L = _ref()
    n = 300_007 if chunk_bytes else 40_000  # the reference's unchunked scan is one 512-thread block
    a = _bits(n, 4, 7, -1_000_000, 1_000_000)
    d = _dev(a, cuda)
    r_fwd = torch.empty_like(d)
    assert L.ref_diff_i32(_vp(d), C.c_size_t(n), C.c_size_t(chunk_bytes), int(nb), 0, _vp(r_fwd)) == 0, \
        L.ref_last_error()
    ours = K().diff(d, chunk_bytes, nb)
    assert torch.equal(ours, r_fwd)
    r_inv = torch.empty_like(d)
    assert L.ref_diff_i32(_vp(r_fwd), C.c_size_t(n), C.c_size_t(chunk_bytes), int(nb), 1, _vp(r_inv)) == 0
    assert torch.equal(K().diff(r_fwd, chunk_bytes, nb, inverse=True), r_inv)


# ------------------------------------------------------------ integer Lorenzo

LZ_CASES = [((100_000, 1, 1), 100_000), ((4096, 1, 1), 4096), ((300, 700, 1), 300 * 700 + 55),
            ((67, 45, 90), 67 * 45 * 90), ((16, 16, 16), 4096), ((1000, 3, 130), 1000 * 3 * 130 + 9)]


@pytest.mark.parametrize("ew", [2, 4, 8])
@pytest.mark.parametrize("dims,n", LZ_CASES)
def test_lorenzo_int_matches_oracle(cuda, ew, dims, n):
    a = _bits(n, ew, n % 1000 + ew, -20_000, 20_000)
    d = _dev(a, cuda)
    fwd = K().lorenzo_int(d, dims)
    assert np.array_equal(_host(fwd, ew), O.lorenzo_int(a, dims))
    inv = K().lorenzo_int(fwd, dims, inverse=True)
    assert np.array_equal(_host(inv, ew), a)


@pytest.mark.parametrize("dims", [(4096, 1, 1), (64, 64, 1), (16, 16, 16), (1000, 700, 1), (40, 30, 200)])
def test_lorenzo_int_matches_reference_kernels(cuda, dims):
    L = _ref()
    n = dims[0] * dims[1] * dims[2]
    a = (np.arange(n) % 200).astype(np.int32).view(np.uint32) if n < 10_000 else _bits(n, 4, 9, -99_999, 99_999)
    d = _dev(a, cuda)
    r_fwd = torch.empty_like(d)
    assert L.ref_lorenzo_i32(_vp(d), C.c_size_t(n), *[C.c_size_t(v) for v in dims], 0, _vp(r_fwd)) == 0, \
        L.ref_last_error()
    assert torch.equal(K().lorenzo_int(d, dims), r_fwd)
    r_inv = torch.empty_like(d)
    assert L.ref_lorenzo_i32(_vp(r_fwd), C.c_size_t(n), *[C.c_size_t(v) for v in dims], 1, _vp(r_inv)) == 0
    assert torch.equal(K().lorenzo_int(r_fwd, dims, inverse=True), r_inv)
    assert torch.equal(r_inv, d)


# ------------------------------------------------------------ quantizer

def _field(n, seed, kind="smooth"):
    rng = np.random.default_rng(seed)
    x = (np.sin(np.arange(n) * 0.003) * 40 + rng.standard_normal(n) * 0.5).astype(np.float32)
    if kind == "spiky":
        x[rng.choice(n, n // 200, replace=False)] = rng.standard_normal(n // 200).astype(np.float32) * 1e6
        x[rng.choice(n, 20, replace=False)] = 0.0
    return x


def _ebx2_r(abs_eb):
    return np.float32(1.0) / (np.float32(2.0) * np.float32(abs_eb))


@pytest.mark.parametrize("code_bytes", [2, 4])
@pytest.mark.parametrize("zz", [False, True])
@pytest.mark.parametrize("mode,radius,kind", [(0, 32768, "spiky"), (0, 512, "smooth"), (2, 32768, "spiky")])
def test_quantizer_abs_noa_match_oracle(cuda, code_bytes, zz, mode, radius, kind):
    n = 1_000_003
    x = _field(n, 11, kind)
    dx = torch.from_numpy(x).to(cuda)
    out = K().quantizer_forward(dx, 1e-3, mode, radius, code_bytes, zz, outlier_capacity=0.05)
    st = out["eb_state"].cpu().numpy()
    if mode == 2:
        vb = np.float32(np.float32(x.max()) - np.float32(x.min()))
        assert st[0] == vb and st[1] == np.float32(np.float32(1e-3) * vb)
    codes, vals, idx, k = O.quantizer_abs(x, code_bytes, st[2], radius, zz, out["cap"])
    assert np.array_equal(out["codes"].cpu().numpy().view(UT[code_bytes]), codes)
    cnt = int(out["count"].item())
    assert cnt == min(k, out["cap"])
    assert np.array_equal(out["idx"][:cnt].cpu().numpy().view(np.uint32), idx)
    assert np.array_equal(out["vals"][:cnt].cpu().numpy().view(np.uint32), vals.view(np.uint32))
    y = K().quantizer_inverse(out["codes"], 1e-3, mode, float(st[1]), radius, zz, vals=out["vals"], idx=out["idx"],
                              count=out["count"], cap=out["cap"])
    want = O.quantizer_abs_inv(codes, st[3], zz, vals, idx)
    assert np.array_equal(y.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_quantizer_overflow_threshold_inplace(cuda):
    n = 300_000
    x = _field(n, 12, "spiky")
    dx = torch.from_numpy(x).to(cuda)
    # capacity overflow: the first cap outliers by index are kept, count capped
    out = K().quantizer_forward(dx, 1e-3, 0, 64, 4, True, outlier_capacity=0.001)
    codes, vals, idx, k = O.quantizer_abs(x, 4, _ebx2_r(1e-3), 64, True, out["cap"])
    assert k > out["cap"] and int(out["count"].item()) == out["cap"]
    assert np.array_equal(out["idx"][:out["cap"]].cpu().numpy().view(np.uint32), idx)
    # threshold forces outliers
    out = K().quantizer_forward(dx, 1e-2, 0, 1 << 22, 4, True, outlier_capacity=0.6, threshold=20.0)
    codes, vals, idx, k = O.quantizer_abs(x, 4, _ebx2_r(1e-2), 1 << 22, True, out["cap"], threshold=20.0)
    cnt = int(out["count"].item())
    assert cnt == min(k, out["cap"]) and np.array_equal(out["codes"].cpu().numpy().view(np.uint32), codes)
    assert np.array_equal(out["idx"][:cnt].cpu().numpy().view(np.uint32), idx)
    # in place
    out = K().quantizer_forward(dx, 1e-3, 0, 32768, 4, True, inplace=True)
    want = O.quantizer_inplace(x, _ebx2_r(1e-3), 32768)
    assert np.array_equal(out["codes"].cpu().numpy().view(np.uint32), want)
    y = K().quantizer_inverse(out["codes"], 1e-3, 0, 1e-3, 32768, True, inplace=True)
    assert np.array_equal(y.cpu().numpy(), O.quantizer_inplace_inv(want, np.float32(2e-3), 32768))


@pytest.mark.parametrize("code_bytes", [2, 4])
@pytest.mark.parametrize("mode,radius,zz,inplace,kind", [
    (1, 32768, True, False, "spiky"), (1, 512, False, False, "smooth"), (0, 32768, True, False, "spiky"),
    (2, 512, False, False, "smooth"), (0, 32768, True, True, "spiky")])
def test_quantizer_matches_reference_kernels(cuda, code_bytes, mode, radius, zz, inplace, kind):
    if inplace and code_bytes == 2:
        pytest.skip("in-place outliers need 32-bit codes")
    L = _ref()
    n = 700_001
    x = _field(n, 13, kind)
    dx = torch.from_numpy(x).to(cuda)
    cap_frac = 1.0  # no overflow: past the capacity the reference keeps an arbitrary subset
    cap = K().max_outliers(n, cap_frac)
    ct = torch.int16 if code_bytes == 2 else torch.int32
    r_codes = torch.empty(n, dtype=ct, device=cuda)
    r_vals = torch.zeros(max(cap, 1), dtype=torch.float32, device=cuda)
    r_idx = torch.zeros(max(cap, 1), dtype=torch.int32, device=cuda)
    r_cnt = torch.zeros(1, dtype=torch.int32, device=cuda)
    r_out = torch.empty(n, dtype=torch.float32, device=cuda)
    hdr = (C.c_uint8 * 128)()
    rc = L.ref_quantizer_f32(_vp(dx), C.c_size_t(n), code_bytes, C.c_float(1e-3), mode, radius, int(zz), int(inplace),
                             C.c_float(float("inf")), C.c_float(cap_frac), _vp(r_codes), _vp(r_vals), _vp(r_idx),
                             _vp(r_cnt), _vp(r_out), hdr)
    assert rc == 0, L.ref_last_error()
    out = K().quantizer_forward(dx, 1e-3, mode, radius, code_bytes, zz, outlier_capacity=cap_frac, inplace=inplace)
    assert torch.equal(out["codes"], r_codes)
    h = np.frombuffer(bytes(hdr), np.uint8)
    abs_eb = float(h[0:4].view(np.float32)[0])
    if mode != 1:
        assert abs_eb == float(out["eb_state"][1].item())
    if not inplace:
        k = int(r_cnt.item())
        assert int(out["count"].item()) == k and k == int(h[20:24].view(np.uint32)[0])
        ri = r_idx[:k].cpu().numpy().view(np.uint32)
        order = np.argsort(ri, kind="stable")
        assert np.array_equal(out["idx"][:k].cpu().numpy().view(np.uint32), ri[order])
        assert np.array_equal(out["vals"][:k].cpu().numpy().view(np.uint32),
                              r_vals[:k].cpu().numpy().view(np.uint32)[order])
    y = K().quantizer_inverse(out["codes"], 1e-3, mode, abs_eb, radius, zz, inplace, vals=out["vals"],
                              idx=out["idx"], count=out["count"], cap=out["cap"])
    assert np.array_equal(y.cpu().numpy().view(np.uint32), r_out.cpu().numpy().view(np.uint32))
    if mode == 1:  # pointwise relative bound (test_quantizer.cpp:354-418)
        xs, ys = x.astype(np.float64), y.cpu().numpy().astype(np.float64)
        nz = xs != 0
        assert np.all(np.abs(ys[nz] - xs[nz]) <= np.abs(xs[nz]) * 1e-3 * 1.01)


def test_quantizer_and_diff_at_full_size(cuda):
    # 64 Mi values (256 MiB, above L2): the pfpl front end (REL quantizer ->
    # negabinary difference in 16 KiB chunks) and its inverse round trip.
    n = 64 << 20
    g = torch.Generator(device=cuda).manual_seed(5)
    x = (torch.randn(n, device=cuda, generator=g) * 100).float()
    out = K().quantizer_forward(x, 1e-3, 1, 32768, 4, True, outlier_capacity=0.1)
    d = K().diff(out["codes"], 16384, True)
    back = K().diff(d, 16384, True, inverse=True)
    assert torch.equal(back, out["codes"])
    y = K().quantizer_inverse(back, 1e-3, 1, 0.0, 32768, True, vals=out["vals"], idx=out["idx"], count=out["count"],
                              cap=out["cap"])
    rel = ((y.double() - x.double()).abs() <= x.double().abs() * 1e-3 * 1.01)
    assert bool(rel.all())
    # unchunked carry path at full size
    d0 = K().diff(out["codes"], 0, False)
    assert torch.equal(K().diff(d0, 0, False, inverse=True), out["codes"])
