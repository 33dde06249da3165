"""CPU tests of the oracle (the parity checker) against the reference's own
known answers and its host codebook builder.  No GPU needed."""
import numpy as np
import pytest

from oracle import oracle as O


def _half_away(v):
    v = np.asarray(v, np.float32).astype(np.float64)
    return (np.sign(v) * np.floor(np.abs(v) + 0.5)).astype(np.float32)


def test_round_half_away():
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.normal(0, 100, 20000).astype(np.float32),
                        np.arange(-10, 10, 0.5, dtype=np.float32),
                        np.float32([0.49999997, -0.49999997, 2.0 ** 23 + 1, 1e30, -0.0])])
    got = np.array([O.lib().orc_round_half_away(float(x)) for x in v], np.float32)
    assert np.array_equal(got, _half_away(v))


@pytest.mark.parametrize("mode", [O.REL, O.NOA])
def test_value_base(mode):
    rng = np.random.default_rng(2)
    x = rng.normal(3, 2, 10001).astype(np.float32)
    vb = O.value_base(x, mode)
    exp = (x.max() - x.min()) if mode == O.NOA else max(abs(x.min()), abs(x.max()))
    assert np.float32(vb) == np.float32(exp)


def _field(shape, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=shape).astype(np.float32)
    for ax in range(len(shape)):
        x = np.cumsum(x, axis=ax)  # smooth-ish
    return (x / np.abs(x).max()).astype(np.float32)


@pytest.mark.parametrize("dims", [(1000, 1, 1), (37, 19, 1), (33, 17, 11), (64, 64, 16)])
@pytest.mark.parametrize("zigzag", [False, True])
def test_lq_roundtrip_error_bound(dims, zigzag):
    nx, ny, nz = dims
    x = _field((nz * ny * nx,), 3)
    eb = 1e-3
    abs_eb, r, e2 = O.resolve_eb(eb, O.ABS, 0.0)
    codes, err, idx, cnt = O.lq_fwd(x, dims, r, 512, zigzag)
    assert cnt == len(idx)
    assert np.all(np.diff(idx.astype(np.int64)) > 0)  # sorted outliers
    y = O.lq_inv(codes, err, idx, dims, e2, zigzag)
    assert np.max(np.abs(y - x)) <= eb * 1.01  # reference tolerance (test_lorenzo.cpp:189)


def test_lq_constant_and_zero_fields():
    for val in (0.0, 3.25):
        x = np.full(4096, val, np.float32)
        _, r, e2 = O.resolve_eb(1e-2, O.ABS, 0.0)
        codes, err, idx, cnt = O.lq_fwd(x, (16, 16, 16), r, 32768, False)
        # only tile origins carry the value itself; everything else predicts exactly
        assert np.count_nonzero(codes) + cnt <= (16 // 8) ** 3
        y = O.lq_inv(codes, err, idx, (16, 16, 16), e2, False)
        assert np.max(np.abs(y - x)) <= 1e-2


def test_lq_padding_codes_zero():
    x = np.linspace(-1, 1, 4096 + 100, dtype=np.float32)
    _, r, e2 = O.resolve_eb(1e-3, O.ABS, 0.0)
    codes, *_ = O.lq_fwd(x, (100, 41, 1), r, 32768, True, n_total=x.size)
    assert np.all(codes[100 * 41:] == 0)


def test_bitshuffle_msb_plane_known_answer():
    # element width 2: every element has only bit 15 set -> plane 0 all ones
    # (the layout pinned by test_bitshuffle_stage.cpp:336-374 for width 4)
    a = np.full(8192, 0x8000, np.uint16)
    s = O.bitshuffle(a, 16384, 2).view(np.uint32)
    assert np.all(s[:256] == 0xFFFFFFFF) and np.all(s[256:] == 0)
    b = np.full(16384, 0x80, np.uint8)
    s = O.bitshuffle(b, 16384, 1).view(np.uint32)
    assert np.all(s[:512] == 0xFFFFFFFF) and np.all(s[512:] == 0)
    # width 4, the reference's own case (test_bitshuffle_stage.cpp:336-374):
    # 1024 elements with only bit 31 set -> plane 0 (32 words) all ones
    c = np.full(1024, 0x80000000, np.uint32)
    s = O.bitshuffle(c.view(np.uint8), 4096, 4).view(np.uint32)
    assert np.all(s[:32] == 0xFFFFFFFF) and np.all(s[32:] == 0)
    e = np.full(1024, 1 << 63, np.uint64)
    s = O.bitshuffle(e.view(np.uint8), 8192, 8).view(np.uint64)
    assert np.all(s[:16] == np.uint64(0xFFFFFFFFFFFFFFFF)) and np.all(s[16:] == 0)


def test_bitshuffle_wide_word_order():
    """Widths 4 and 8 (the reference's butterfly kernels): element e of a
    32- / 64-element group sits at the plane word's bit 31-e / 63-e, the
    reverse of the ballot kernels' order for widths 1 and 2."""
    c = np.zeros(1024, np.uint32)
    c[0] = 1          # element 0, bit 0 -> plane 31, word 0, bit 31
    c[33] = 1 << 5    # element 33 (group 1, e = 1), bit 5 -> plane 26, word 1, bit 30
    s = O.bitshuffle(c.view(np.uint8), 4096, 4).view(np.uint32).reshape(32, 32)
    assert s[31, 0] == 1 << 31 and s[26, 1] == 1 << 30
    assert np.count_nonzero(s) == 2
    e = np.zeros(1024, np.uint64)
    e[65] = 1 << 40   # group 1, e = 1, bit 40 -> plane 23, word 1, bit 62
    s = O.bitshuffle(e.view(np.uint8), 8192, 8).view(np.uint64).reshape(64, 16)
    assert s[23, 1] == np.uint64(1 << 62) and np.count_nonzero(s) == 1
    a = np.zeros(8192, np.uint16)
    a[1] = 1          # width 2: element 1, bit 0 -> plane 15, word 0, bit 1
    s = O.bitshuffle(a, 16384, 2).view(np.uint32).reshape(16, 256)
    assert s[15, 0] == 2 and np.count_nonzero(s) == 1


@pytest.mark.parametrize("ew", [1, 2, 4, 8])
def test_bitshuffle_invariants_and_roundtrip(ew):
    rng = np.random.default_rng(4)
    for fill in (0x00, 0xFF):  # zeros -> zeros, 0xFF -> 0xFF (:235-292)
        d = np.full(16384 * 2, fill, np.uint8)
        assert np.array_equal(O.bitshuffle(d, 16384, ew), d)
    d = rng.integers(0, 256, 16384 * 3 + 1000, dtype=np.uint8)
    s = O.bitshuffle(d, 16384, ew)
    assert np.array_equal(s[-1000:], d[-1000:])  # tail copied unchanged
    assert np.array_equal(O.bitshuffle(s, 16384, ew, inverse=True), d)


def test_rze_all_zero_chunk_small():
    enc = O.rze_encode(np.zeros(16384, np.uint8))
    assert len(enc) <= 17  # test_rze_stage.cpp:197-214
    assert np.array_equal(O.rze_decode(enc), np.zeros(16384, np.uint8))


@pytest.mark.parametrize("kind", ["random", "sparse", "checker", "runs", "partial", "mixed"])
def test_rze_roundtrip(kind):
    rng = np.random.default_rng(5)
    if kind == "random":
        d = rng.integers(0, 256, 16384 * 2, dtype=np.uint8)
    elif kind == "sparse":
        d = np.zeros(16384 * 3, np.uint8)
        d[rng.choice(d.size, 300, replace=False)] = rng.integers(1, 256, 300)
    elif kind == "checker":
        d = np.tile(np.uint8([0, 0xAA]), 16384)
    elif kind == "runs":
        d = np.repeat(rng.integers(0, 4, 200, dtype=np.uint8), 300)
    elif kind == "partial":
        d = rng.integers(0, 3, 3000, dtype=np.uint8)
    else:
        d = np.concatenate([np.zeros(16384, np.uint8), rng.integers(0, 256, 16384, dtype=np.uint8),
                            np.repeat(np.uint8([1, 2, 3]), 5000)])
    enc = O.rze_encode(d)
    assert len(enc) % 4 == 0
    hdr = enc[:8].view(np.uint32)
    assert hdr[0] == d.size and hdr[1] == (d.size + 16383) // 16384
    assert np.array_equal(O.rze_decode(enc), d)
    if kind == "random":  # incompressible chunks are stored raw (flag bit 31)
        assert np.all(enc[8:16].view(np.uint32) & 0x80000000)


def test_rle_known_answer():
    a = np.array([7, 7, 7, 42, 42, 1], np.uint16)  # test_rle.cpp:120-146
    enc = O.rle_encode(a)
    assert enc[:4].view(np.uint32)[0] == 3
    assert np.array_equal(O.rle_decode(enc, a.size), a)


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.uint32])
def test_rle_roundtrip(dtype):
    rng = np.random.default_rng(6)
    a = np.repeat(rng.integers(0, 5, 1000).astype(dtype), rng.integers(1, 50, 1000))
    enc = O.rle_encode(a)
    runs = int(enc[:4].view(np.uint32)[0])
    vb = runs * a.itemsize
    assert len(enc) == 4 + ((vb + 3) & ~3) + 4 * runs
    assert np.array_equal(O.rle_decode(enc, a.size, dtype), a)


def test_bitpack_sizes_and_roundtrip():
    rng = np.random.default_rng(7)
    for nbits in (1, 2, 4, 8, 16):
        a = rng.integers(0, 1 << nbits, 1024).astype(np.uint16)
        p = O.bitpack_encode(a, nbits)
        assert p.size == 1024 * nbits // 8  # test_bitpack.cpp:184-203
        assert np.array_equal(O.bitpack_decode(p, a.size, nbits), a)
    assert O.bitpack_nbits(0, 2) == 1 and O.bitpack_nbits(3, 2) == 2 and O.bitpack_nbits(4, 2) == 4
    assert O.bitpack_nbits(300, 2) == 16 and O.bitpack_nbits(255, 1) == 8


def _histograms(n=200):
    rng = np.random.default_rng(8)
    for t in range(n):
        freq = np.zeros(1024, np.uint32)
        k = int(rng.integers(2, 1024))
        pos = rng.choice(1024, size=k, replace=False)
        if t % 3 == 0:
            freq[pos] = rng.integers(1, 100000, size=k)
        elif t % 3 == 1:
            freq[pos] = (rng.pareto(0.7, size=k) * 10 + 1).astype(np.uint32)
        else:
            freq[pos] = rng.integers(1, 4, size=k)
        yield freq


@pytest.mark.skipif(not O.ref_hfbook_available(), reason="reference codebook build absent")
def test_codebook_matches_reference_build():
    for freq in _histograms():
        a_bk, a_rb = O.huff_book(freq)
        b_bk, b_rb = O.ref_huff_book(freq)
        assert np.array_equal(a_bk, b_bk)
        assert np.array_equal(a_rb, b_rb)


def test_huffman_roundtrip_and_layout():
    rng = np.random.default_rng(9)
    codes = np.clip(np.abs(rng.normal(0, 6, 100000)), 0, 1023).astype(np.uint16)
    freq, counted = O.histogram(codes)
    assert counted == codes.size
    bk, rb = O.huff_book(freq)
    blob = O.huff_encode(codes, 1024, bk, rb)
    ent = blob[40:64].view(np.uint32)
    assert ent[1] == 128 and ent[2] == 128 + 2304 and ent[5] == len(blob)
    assert np.array_equal(O.huff_decode(blob, codes.size), codes)


def test_histogram_skips_out_of_range():
    f, counted = O.histogram(np.array([0, 5, 1023, 1024, 5000], np.uint16))
    assert counted == 3 and f[5] == 1


def test_crc32_known_answer():
    assert O.crc32(b"123456789") == 0xCBF43926


def _revisit_lite_cells(sym, bk4):
    """Cells of one full 1024-symbol partition the way the reference's fine
    encoder builds them (phf/hf_kernels.cu:145-250): 256 shards of 4 codes,
    each packed MSB-first into one word (reduce-merge), then 8 rounds of
    pairwise merges in which the right group's words are shifted in behind the
    left group's bits (shuffle-merge)."""
    M = 0xFFFFFFFF
    buf, cnt = [], []
    for s in range(256):
        acc, nb = 0, 0
        for k in range(4):
            w = int(bk4[sym[4 * s + k]])
            ln, code = w >> 27, w & 0x7FFFFFF
            if ln:
                acc |= ((code << (32 - ln)) & M) >> nb
            nb += ln
        buf.append(acc)
        cnt.append(nb)
    stride = 1
    for _ in range(8):
        for left in range(0, 256, 2 * stride):
            r = left + stride
            units, bits = divmod(cnt[left], 32)
            right = buf[r:r + stride]
            buf[r:r + stride] = [0] * stride
            for i, w in enumerate(right):
                buf[left + units + i] |= w >> bits
                if bits:
                    buf[left + units + i + 1] |= (w << (32 - bits)) & M
            cnt[left] += cnt[r]
        stride *= 2
    return np.array(buf[: (cnt[0] + 31) // 32], np.uint32), cnt[0]


def test_huffman_fine_layout_equals_revisit_lite_merge():
    """Fine mode's ReVISIT-lite shard/merge produces exactly the cells of an
    MSB-first deflate at sublen 1024, which is what the oracle (and the GPU
    coder) write for fine mode; checked on full partitions of books whose
    longest code is at most 8 bits."""
    rng = np.random.default_rng(7)
    cases = [rng.integers(0, hi, 1024 * 3).astype(np.uint16) for hi in (2, 16, 60)]
    cases.append(rng.permutation(np.repeat(np.arange(256), 12)).astype(np.uint16))  # every code 8 bits
    for a in cases:
        freq = np.bincount(a, minlength=1024).astype(np.uint32)
        bk4, rb = O.huff_book(freq, 1024)
        assert int((bk4[freq > 0] >> 27).max()) <= 8
        blob = O.huff_encode(a, 1024, bk4, rb, sublen=1024)
        ent = blob[40:64].view(np.uint32)
        pd = int(blob[8:12].view(np.int32)[0])
        assert pd == 3 and int(blob[4:8].view(np.int32)[0]) == 1024
        nbit = blob[ent[2]:ent[3]].view(np.uint32)
        pent = blob[ent[3]:ent[4]].view(np.uint32)
        bits = blob[ent[4]:ent[5]].view(np.uint32)
        for p in range(pd):
            cells, nb = _revisit_lite_cells(a[1024 * p:1024 * (p + 1)], bk4)
            assert nb == int(nbit[p])
            assert np.array_equal(bits[int(pent[p]):int(pent[p]) + cells.size], cells)
        assert np.array_equal(O.huff_decode(blob, a.size), a)
