"""GPU parity for the RLE and Bitpack coders: libfzb.so vs the oracle (exact
bytes) and vs the reference's own stage kernels (oracle/_ref)."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def K():
    from fzgpumodules_b200 import kernels
    return kernels


TDT = {np.uint8: torch.uint8, np.uint16: torch.uint16, np.uint32: torch.int32}


def _g(a, dev):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).to(dev)


def _rle_cases(dtype):
    rng = np.random.default_rng(31)
    return {
        "kat": np.array([7, 7, 7, 42, 42, 1], dtype),               # test_rle.cpp:120-146
        "single": np.array([5], dtype),
        "constant": np.full(50000, 3, dtype),
        "runs": np.repeat(rng.integers(0, 6, 3000).astype(dtype), rng.integers(1, 90, 3000)),
        "random": rng.integers(0, 200, 70001).astype(dtype),
        "long_runs": np.repeat(np.array([1, 2, 1, 0], dtype), [10000, 3, 20000, 7]),
    }


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.uint32])
@pytest.mark.parametrize("case", ["kat", "single", "constant", "runs", "random", "long_runs"])
def test_rle_matches_oracle(cuda, dtype, case):
    a = _rle_cases(dtype)[case]
    ref = O.rle_encode(a)
    enc, size = K().rle_encode(_g(a, cuda))
    assert int(size.item()) == ref.size
    assert np.array_equal(enc.cpu().numpy(), ref)
    dec = K().rle_decode(enc, a.size, TDT[dtype])
    got = dec.cpu().numpy()
    if dtype == np.uint32:
        got = got.view(np.uint32)
    assert np.array_equal(got, a)


def test_rle_malformed_lengths_reported(cuda):
    a = _rle_cases(np.uint16)["runs"]
    enc, _ = K().rle_encode(_g(a, cuda))
    ws = K().Workspace()
    K().rle_decode(enc, a.size + 5, torch.uint16, ws=ws)  # lengths do not add up
    assert ws.status() == -5


@pytest.mark.parametrize("nbits", [0, 1, 2, 4, 8, 16])
def test_bitpack_matches_oracle(cuda, nbits):
    rng = np.random.default_rng(32)
    hi = 1 << (nbits if nbits else 5)
    a = rng.integers(0, hi, 10007).astype(np.uint16)
    use = nbits if nbits else O.bitpack_nbits(int(a.max()), 2)
    ref = O.bitpack_encode(a, use)
    packed, nb = K().bitpack_encode(_g(a, cuda), nbits)
    assert nb == use
    assert np.array_equal(packed.cpu().numpy(), ref)
    back = K().bitpack_decode(packed, a.size, use)
    assert np.array_equal(back.cpu().numpy(), a)


# ----------------------------------------------------------- reference kernels

def _ref():
    if not os.path.exists(O.REF_STAGES):
        pytest.skip("reference stage build absent")
    L = C.CDLL(O.REF_STAGES)
    L.ref_last_error.restype = C.c_char_p
    return L


def _vp(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("case", ["kat", "constant", "runs", "random", "long_runs"])
def test_reference_rle_matches(cuda, case):
    L = _ref()
    a = _rle_cases(np.uint16)[case]
    d = _g(a, cuda)
    out = torch.zeros(int(O.lib().orc_rle_max_bytes(a.size, 2)) + 16, dtype=torch.uint8, device=cuda)
    dec = torch.zeros(a.size, dtype=torch.uint16, device=cuda)
    nb = C.c_size_t(0)
    assert L.ref_rle_u16(_vp(d), C.c_size_t(a.size), _vp(out), C.byref(nb), _vp(dec)) == 0, L.ref_last_error()
    ref = out.cpu().numpy()[: nb.value]
    assert np.array_equal(ref, O.rle_encode(a))
    assert np.array_equal(dec.cpu().numpy(), a)


@pytest.mark.parametrize("nbits", [0, 1, 4, 8, 16])
def test_reference_bitpack_matches(cuda, nbits):
    L = _ref()
    rng = np.random.default_rng(33)
    a = rng.integers(0, 1 << (nbits if nbits else 3), 5003).astype(np.uint16)
    d = _g(a, cuda)
    out = torch.zeros(a.size * 2 + 16, dtype=torch.uint8, device=cuda)
    dec = torch.zeros(a.size, dtype=torch.uint16, device=cuda)
    nb, used = C.c_size_t(0), C.c_int(0)
    assert L.ref_bitpack_u16(_vp(d), C.c_size_t(a.size), nbits, _vp(out), C.byref(nb), C.byref(used),
                             _vp(dec)) == 0, L.ref_last_error()
    assert used.value == (nbits or O.bitpack_nbits(int(a.max()), 2))
    assert np.array_equal(out.cpu().numpy()[: nb.value], O.bitpack_encode(a, used.value))
    assert np.array_equal(dec.cpu().numpy(), a)


def test_quickstart_chain_lq2d_rle(cuda):
    """The Quick Start chain (LorenzoQuant 2-D ABS 1e-4 -> RLE) on the
    1800x3600 sinusoid field: codes and RLE bytes equal the oracle's."""
    from fzgpumodules_b200 import fields
    x = fields.sinusoids2d(1800, 3600, seed=1001).reshape(-1)
    xh = x.numpy()
    dims = (3600, 1800, 1)
    out = K().lq_forward(x.to(cuda), dims, 1e-4, K().ABS, 32768, False, 0.2)
    abs_eb, r, e2 = O.resolve_eb(1e-4, O.ABS, 0.0)
    codes, err, idx, cnt = O.lq_fwd(xh, dims, r, 32768, False, cap=out["cap"])
    assert np.array_equal(out["codes"].cpu().numpy(), codes)
    enc, size = K().rle_encode(out["codes"])
    assert np.array_equal(enc.cpu().numpy(), O.rle_encode(codes))
