"""GPU parity for the PHF Huffman coder (HuffmanStage<uint16_t>, coarse mode):
histogram, codebook, blob bytes and decode of libfzb.so vs the oracle, and
vs the reference's own stage run from oracle/_ref.

Blob bytes 64..127 are compared exactly against the oracle (both write zeros
there) and masked against the reference, whose encoder leaves scratch in
that part of the 128-byte header slot; the upper 16 bits of the first header
word (the reference's int bklen field holds only 16 meaningful bits) are
masked for the same reason."""
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


def _cases():
    rng = np.random.default_rng(41)
    lap = np.clip(np.round(rng.laplace(0, 3.0, 200_003)), -511, 511).astype(np.int64)
    zz = ((lap << 1) ^ (lap >> 63)).astype(np.uint16)  # zigzag Lorenzo-like codes
    return {
        "n1": np.array([5], np.uint16),
        "two_symbols": rng.integers(0, 2, 5000).astype(np.uint16) * 900,
        "partial_partition": rng.integers(0, 40, 767).astype(np.uint16),
        "exact_partitions": rng.integers(0, 40, 768 * 13).astype(np.uint16),
        "ragged": rng.integers(0, 300, 768 * 13 + 5).astype(np.uint16),
        "uniform_1024": rng.integers(0, 1024, 100_000).astype(np.uint16),
        "laplace_zigzag": zz,
        "geometric": np.minimum(rng.geometric(0.02, 300_001), 1023).astype(np.uint16),
    }


def _hist(a, bklen):
    return np.bincount(a[a < bklen], minlength=bklen).astype(np.uint32)


@pytest.mark.parametrize("bklen", [1, 2, 3, 4, 5, 1024, 20000])
def test_histogram_counts(cuda, bklen):
    """Symbols 0..3 counted in registers (SIMD compares on code pairs), the
    others through shared-memory copies (global counts past 16384 symbols):
    every count exact, symbols >= bklen skipped, with tails past the last
    16-byte word and a misaligned start."""
    rng = np.random.default_rng(bklen)
    for n in (1, 7, 8, 9, 1000003):
        small = rng.integers(0, 4, n)
        wide = rng.integers(0, max(2 * bklen, 8), n)
        a = np.where(rng.random(n) < 0.7, small, wide).astype(np.uint16)
        a[rng.random(n) < 0.01] = 65535
        d = torch.from_numpy(np.concatenate([[np.uint16(1)], a])).to(cuda)
        for view, ref in ((d[1:], a), (d, np.concatenate([[np.uint16(1)], a]))):
            freq = K().huff_histogram(view, bklen).cpu().numpy().view(np.uint32)
            assert np.array_equal(freq, _hist(ref, bklen)), (bklen, n)


@pytest.mark.parametrize("case", list(_cases()))
def test_histogram_book_blob_decode(cuda, case):
    a = _cases()[case]
    bklen = 1024
    d = torch.from_numpy(a).to(cuda)
    freq = K().huff_histogram(d, bklen).cpu().numpy().view(np.uint32)
    assert np.array_equal(freq, _hist(a, bklen))
    bk4, rb = O.huff_book(freq, bklen)
    gbk4, grb = K().huff_book(freq, bklen)
    assert np.array_equal(gbk4, bk4) and np.array_equal(grb, rb)
    ref = O.huff_encode(a, bklen, bk4, rb)
    blob, size = K().huff_compress(d, bklen)
    assert int(size.item()) == ref.size
    assert np.array_equal(blob.cpu().numpy(), ref)
    blob2, _ = K().huff_encode(d, bk4, rb, bklen)
    assert np.array_equal(blob2.cpu().numpy(), ref)
    ws = K().Workspace()
    dec = K().huff_decode(blob, a.size, bklen, ws=ws)
    assert ws.status() == 0
    if case != "n1":  # a one-symbol book has a zero-length code (see below)
        assert np.array_equal(O.huff_decode(ref, a.size), a)
    assert np.array_equal(dec.cpu().numpy(), a)


def test_histogram_skips_out_of_range(cuda):
    rng = np.random.default_rng(42)
    a = rng.integers(0, 2000, 123_457).astype(np.uint16)
    for bklen in (1024, 256, 20000, 65535):
        f = K().huff_histogram(torch.from_numpy(a).to(cuda), bklen).cpu().numpy().view(np.uint32)
        assert np.array_equal(f, _hist(a, bklen)), bklen


def test_out_of_range_symbol_rejected(cuda):
    """huffman_stage.cu:151-164: a symbol >= bklen is an error, not data."""
    a = np.full(4000, 3, np.uint16)
    a[1234] = 1024
    with pytest.raises(K().FzbError) as ei:
        K().huff_compress(torch.from_numpy(a).to(cuda), 1024)
    assert ei.value.status == -7


@pytest.mark.parametrize("bklen", [2, 256, 4096, 20000])
def test_other_book_lengths(cuda, bklen):
    rng = np.random.default_rng(bklen)
    a = np.minimum(rng.geometric(0.01, 50_000), bklen - 1).astype(np.uint16)
    freq = _hist(a, bklen)
    bk4, rb = O.huff_book(freq, bklen)
    ref = O.huff_encode(a, bklen, bk4, rb)
    blob, _ = K().huff_compress(torch.from_numpy(a).to(cuda), bklen)
    assert np.array_equal(blob.cpu().numpy(), ref)
    assert np.array_equal(K().huff_decode(blob, a.size, bklen).cpu().numpy(), a)


def test_truncated_blob_reported(cuda):
    a = _cases()["laplace_zigzag"]
    blob, size = K().huff_compress(torch.from_numpy(a).to(cuda), 1024)
    ws = K().Workspace()
    K().huff_decode(blob[: blob.numel() - 64], a.size, 1024, ws=ws)
    assert ws.status() == -5
    ws2 = K().Workspace()
    K().huff_decode(blob, a.size + 1, 1024, ws=ws2)  # header disagrees with n
    assert ws2.status() == -5


def test_unaligned_output_decode(cuda):
    a = _cases()["geometric"][:50_000]
    blob, _ = K().huff_compress(torch.from_numpy(a).to(cuda), 1024)
    buf = torch.zeros(a.size + 1, dtype=torch.uint16, device=cuda)
    K().huff_decode(blob, a.size, 1024, out=buf[1:])
    assert np.array_equal(buf[1:].cpu().numpy(), a)


@pytest.mark.parametrize("fine", [False, True])
@pytest.mark.parametrize("sigma", [0.3, 1.0, 2.0, 4.0, 8.0, 16.0, 64.0])
def test_decode_across_code_lengths(cuda, sigma, fine):
    """Gaussian codes from nearly one symbol to nearly flat: books whose
    shortest code runs from 1 to 7 bits, so the decoder takes both its
    warp-per-partition path (bit segments that resynchronise, a few lanes
    decoding again) and its partition-per-lane path.  Blob bytes and the
    decode are checked against the oracle."""
    rng = np.random.default_rng(int(sigma * 10) + int(fine))
    a = np.clip(np.round(rng.normal(512, sigma, 300_001)), 0, 1023).astype(np.uint16)
    bklen = 1024
    freq = _hist(a, bklen)
    bk4, rb = O.huff_book(freq, bklen)
    ref = O.huff_encode(a, bklen, bk4, rb, sublen=1024 if fine else 768)
    blob, _ = K().huff_compress(torch.from_numpy(a).to(cuda), bklen, fine=fine)
    assert np.array_equal(blob.cpu().numpy(), ref)
    ws = K().Workspace()
    dec = K().huff_decode(blob, a.size, bklen, ws=ws)
    assert ws.status() == 0
    assert np.array_equal(dec.cpu().numpy(), a)


def test_decode_reports_corrupt_cells(cuda):
    """Flipped bits inside the bitstream: every partition whose bit count no
    longer decodes to its symbols is reported, whichever decode path runs."""
    for sigma in (1.0, 64.0):
        rng = np.random.default_rng(7)
        a = np.clip(np.round(rng.normal(512, sigma, 200_000)), 0, 1023).astype(np.uint16)
        blob, _ = K().huff_compress(torch.from_numpy(a).to(cuda), 1024)
        h = blob.cpu().numpy()
        e4, e5 = (int(v) for v in h[40:64].view(np.uint32)[4:6])
        bad = h.copy()
        bad[e4:e5:7] ^= 0x5A
        ws = K().Workspace()
        K().huff_decode(torch.from_numpy(bad).to(cuda), a.size, 1024, ws=ws)
        assert ws.status() == -5, sigma


# ----------------------------------------------------------- reference stage

def _ref():
    if not os.path.exists(O.REF_STAGES):
        pytest.skip("reference stage build absent")
    L = C.CDLL(O.REF_STAGES)
    L.ref_last_error.restype = C.c_char_p
    return L


def _masked(b):
    b = b.copy()
    b[2:4] = 0
    b[64:128] = 0
    return b


# Inputs below about 1300 symbols are left out: the reference's memcpy_merge
# copies the whole bitstream capacity (2*n bytes) to offset entry[4] of a
# 4*n-byte scratch buffer (phf/hf_buf.cc:152-176), which overruns it when the
# header, revbook and partition tables exceed 2*n bytes, and the stage fails
# with "invalid argument".
@pytest.mark.parametrize("case", ["two_symbols", "ragged", "uniform_1024", "laplace_zigzag", "geometric"])
def test_reference_stage_matches(cuda, case):
    L = _ref()
    a = _cases()[case]
    d = torch.from_numpy(a).to(cuda)
    out = torch.zeros(int(O.lib().orc_huff_max_bytes(a.size, 1024)) + 4 * a.size + 4096,
                      dtype=torch.uint8, device=cuda)
    dec = torch.zeros(a.size, dtype=torch.uint16, device=cuda)
    nb = C.c_size_t(0)
    rc = L.ref_huffman_u16(C.c_void_p(d.data_ptr()), C.c_size_t(a.size), 1024, C.c_void_p(out.data_ptr()),
                           C.byref(nb), C.c_void_p(dec.data_ptr()))
    assert rc == 0, L.ref_last_error()
    ref = out.cpu().numpy()[: nb.value]
    ours, _ = K().huff_compress(d, 1024)
    ours = ours.cpu().numpy()
    assert ours.size == ref.size
    assert np.array_equal(_masked(ours), _masked(ref))
    assert np.array_equal(dec.cpu().numpy(), a)


def test_c3_chain_lq2d_huffman(cuda):
    """LorenzoQuant 2-D (ABS 1e-3, radius 512, zigzag) -> Huffman (bklen 1024)
    on a 2048x2048 fractal field in [-50, 50]: codes, outliers and the blob
    equal the oracle's; decode returns the codes."""
    from fzgpumodules_b200 import fields
    x = fields.fractal2d(2048, seed=1003).reshape(-1)
    dims = (2048, 2048, 1)
    out = K().lq_forward(x.to(cuda), dims, 1e-3, K().ABS, 512, True, 0.2)
    _, r, _ = O.resolve_eb(1e-3, O.ABS, 0.0)
    codes, err, idx, cnt = O.lq_fwd(x.numpy(), dims, r, 512, True, cap=out["cap"])
    assert np.array_equal(out["codes"].cpu().numpy(), codes)
    assert int(out["count"].item()) == cnt
    blob, _ = K().huff_compress(out["codes"], 1024)
    freq = _hist(codes, 1024)
    bk4, rb = O.huff_book(freq, 1024)
    ref = O.huff_encode(codes, 1024, bk4, rb)
    assert np.array_equal(blob.cpu().numpy(), ref)
    dec = K().huff_decode(blob, codes.size, 1024)
    assert np.array_equal(dec.cpu().numpy(), codes)


# ----------------------------------------------------------------- fine mode

def _fine_cases():
    rng = np.random.default_rng(43)
    lap = np.clip(np.round(rng.laplace(0, 3.0, 100_000)), -511, 511).astype(np.int64)
    return {
        "n1": np.array([5], np.uint16),
        "short_codes_ragged": rng.integers(0, 16, 1024 * 9 + 333).astype(np.uint16),   # longest code 4 bits
        "short_codes_partial": rng.integers(0, 100, 1000).astype(np.uint16),           # under one partition
        "two_symbols": (rng.integers(0, 2, 4096) * 700).astype(np.uint16),
        "eight_bit_book": rng.integers(0, 200, 1024 * 20).astype(np.uint16),           # lengths 7-8
        "laplace_zigzag": ((lap << 1) ^ (lap >> 63)).astype(np.uint16),                # longer codes
        "uniform_1024_ragged": rng.integers(0, 1024, 50_001).astype(np.uint16),
    }


@pytest.mark.parametrize("case", list(_fine_cases()))
def test_fine_mode_blob_decode(cuda, case):
    """Fine mode (1024-symbol partitions): the blob equals the oracle's at
    sublen 1024 whether the four-codes-per-word packing applies or not, and
    decodes back."""
    a = _fine_cases()[case]
    bklen = 1024
    d = torch.from_numpy(a).to(cuda)
    freq = _hist(a, bklen)
    bk4, rb = O.huff_book(freq, bklen)
    ref = O.huff_encode(a, bklen, bk4, rb, sublen=1024)
    assert ref[4:8].view(np.int32)[0] == 1024
    blob, size = K().huff_compress(d, bklen, fine=True)
    assert int(size.item()) == ref.size
    assert np.array_equal(blob.cpu().numpy(), ref)
    blob2, _ = K().huff_encode(d, bk4, rb, bklen, fine=True)
    assert np.array_equal(blob2.cpu().numpy(), ref)
    ws = K().Workspace()
    dec = K().huff_decode(blob, a.size, bklen, ws=ws)
    assert ws.status() == 0
    assert np.array_equal(dec.cpu().numpy(), a)


def test_fine_mode_header_disagreement_reported(cuda):
    a = _fine_cases()["laplace_zigzag"]
    blob, _ = K().huff_compress(torch.from_numpy(a).to(cuda), 1024, fine=True)
    bad = blob.clone()
    bad[4:8] = torch.tensor(np.array([1000], np.int32).view(np.uint8), device=cuda)  # neither 768 nor 1024
    ws = K().Workspace()
    K().huff_decode(bad, a.size, 1024, ws=ws)
    assert ws.status() == -5


# Whole 1024-symbol partitions only (see ref_huffman_u16_fine), and inputs
# above the reference's small-input limit noted for coarse mode.
@pytest.mark.parametrize("case", ["short", "eight_bit", "long_codes"])
def test_fine_reference_stage_matches(cuda, case):
    L = _ref()
    if not hasattr(L, "ref_huffman_u16_fine"):
        pytest.skip("reference stage build without the fine-mode entry")
    rng = np.random.default_rng(44)
    n = 1024 * 40
    if case == "short":
        a = rng.integers(0, 16, n).astype(np.uint16)
    elif case == "eight_bit":
        a = rng.integers(0, 200, n).astype(np.uint16)
    else:
        lap = np.clip(np.round(rng.laplace(0, 3.0, n)), -511, 511).astype(np.int64)
        a = ((lap << 1) ^ (lap >> 63)).astype(np.uint16)
    d = torch.from_numpy(a).to(cuda)
    out = torch.zeros(int(O.lib().orc_huff_max_bytes(a.size, 1024)) + 4 * a.size + 4096,
                      dtype=torch.uint8, device=cuda)
    dec = torch.zeros(a.size, dtype=torch.uint16, device=cuda)
    nb = C.c_size_t(0)
    rc = L.ref_huffman_u16_fine(C.c_void_p(d.data_ptr()), C.c_size_t(a.size), 1024, C.c_void_p(out.data_ptr()),
                                C.byref(nb), C.c_void_p(dec.data_ptr()))
    assert rc == 0, L.ref_last_error()
    ref = out.cpu().numpy()[: nb.value]
    ours, _ = K().huff_compress(d, 1024, fine=True)
    ours = ours.cpu().numpy()
    assert ours.size == ref.size
    assert np.array_equal(_masked(ours), _masked(ref))
    assert np.array_equal(dec.cpu().numpy(), a)
