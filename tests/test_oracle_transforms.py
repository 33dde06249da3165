"""The oracle's restatements of the stages around the codes (Zigzag,
Negabinary, Difference, lossless Lorenzo, the direct Quantizer) against the
known answers of the reference's own tests (tests/stages/test_zigzag.cpp,
test_negabinary.cpp, test_difference.cpp, test_lorenzo.cpp,
test_quantizer.cpp) and their round-trip properties."""
import numpy as np
import pytest

from oracle import oracle as O


def test_zigzag_known_vectors():
    # ZigzagKnownVectors (test_zigzag.cpp:32-84)
    x = np.array([0, -1, 1, -2, 2, -3, 3, 2**31 - 1, -2**31], np.int32)
    want = np.array([0, 1, 2, 3, 4, 5, 6, (2**31 - 1) * 2, 2**32 - 1], np.uint32)
    assert np.array_equal(O.zigzag(x), want)
    assert np.array_equal(O.zigzag(np.array([0, -1, 1, -2, 2], np.int16)), np.array([0, 1, 2, 3, 4], np.uint16))
    assert np.array_equal(O.zigzag(np.array([0, -1, 1, -63, 63, -128], np.int8)),
                          np.array([0, 1, 2, 125, 126, 255], np.uint8))
    # exhaustive 8- and 16-bit round trips (:87-111), sampled 64-bit (:142-160)
    for dt in (np.int8, np.int16):
        allv = np.arange(np.iinfo(dt).min, np.iinfo(dt).max + 1).astype(dt)
        assert np.array_equal(O.zigzag(O.zigzag(allv), inverse=True).view(dt), allv)
    r = np.random.default_rng(0).integers(-2**63, 2**63 - 1, 10_000, dtype=np.int64, endpoint=True)
    assert np.array_equal(O.zigzag(O.zigzag(r), inverse=True).view(np.int64), r)


def test_negabinary_known_vectors():
    # test_negabinary.cpp:35-69
    x = np.array([0, 1, -1, 2, -2], np.int32)
    assert np.array_equal(O.negabinary(x), np.array([0, 1, 3, 6, 2], np.uint32))
    rng = np.random.default_rng(1)
    for dt in (np.int8, np.int16, np.int32, np.int64):
        a = rng.integers(np.iinfo(dt).min, np.iinfo(dt).max, 5000, dtype=dt, endpoint=True)
        assert np.array_equal(O.negabinary(O.negabinary(a), inverse=True).view(dt), a)


def test_difference_known_answers_and_round_trips():
    # ChunkBoundariesAreIndependent (test_difference.cpp:319-350)
    a = np.array([10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33], np.int32)
    assert list(O.diff(a, chunk_elems=4).view(np.int32)) == [10, 1, 1, 1, 20, 1, 1, 1, 30, 1, 1, 1]
    # ChunksAreIndependentContexts (:411-435)
    b = np.array(list(range(1000, 1008)) + list(range(-500, -492)), np.int32)
    db = O.diff(b, chunk_elems=8).view(np.int32)
    assert db[8] == -500 and np.array_equal(O.diff(db, 8, inverse=True).view(np.int32), b)
    # Uint16WrappingArithmetic (:188-210)
    w = np.array([0, 65535] * 32, np.uint16)
    assert np.array_equal(O.diff(O.diff(w), inverse=True), w)
    # NegabinaryChunkedRoundTrip: chunk starts hold negabinary(value) (:517-555)
    c = (np.arange(4 * 4096) % 97 + np.repeat(np.arange(4) * 100_000, 4096)).astype(np.int32)
    dc = O.diff(c, 4096, negabinary=True)
    for k in range(4):
        assert dc[k * 4096] == O.negabinary(c[k * 4096:k * 4096 + 1])[0]
    rng = np.random.default_rng(2)
    for dt, chunk, nb in ((np.int32, 0, False), (np.int32, 512, True), (np.int16, 1024, True),
                          (np.uint8, 16, False), (np.int64, 1024, True), (np.uint16, 1024, False)):
        lo = -1000 if np.dtype(dt).kind == "i" else 0
        a = rng.integers(lo, 1000, 20_011).astype(dt)
        fwd = O.diff(a, chunk, nb)
        assert np.array_equal(O.diff(fwd, chunk, nb, inverse=True).view(dt), a)


@pytest.mark.parametrize("dims,period", [((4096, 1, 1), None), ((64, 64, 1), 200), ((16, 16, 16), 50),
                                         ((37, 29, 1), None), ((17, 9, 11), None)])
def test_lorenzo_int_round_trip(dims, period):
    # RoundTrip1D / 2D / 3D (test_lorenzo.cpp:35-96) use i % 200 and i % 50
    n = dims[0] * dims[1] * dims[2]
    if period:
        a = (np.arange(n) % period).astype(np.int32)
    else:
        a = np.random.default_rng(3).integers(-50_000, 50_000, n).astype(np.int32)
    d = O.lorenzo_int(a, dims)
    assert np.array_equal(O.lorenzo_int(d, dims, inverse=True).view(np.int32), a)


def test_lorenzo_int_structure():
    # 1-D: every 256-element block starts raw
    a = np.arange(1000, dtype=np.int32) * 3 + 7
    d = O.lorenzo_int(a, (1000, 1, 1)).view(np.int32)
    assert d[0] == 7 and d[256] == a[256] and d[512] == a[512] and np.all(d[1:256] == 3)
    # a linear ramp leaves only the boundary deltas in 2-D / 3-D
    for dims in ((37, 29, 1), (17, 9, 11)):
        x, y, z = np.meshgrid(np.arange(dims[0]), np.arange(dims[1]), np.arange(dims[2]), indexing="ij")
        ramp = (3 * x + 5 * y + 7 * z).transpose(2, 1, 0).reshape(-1).astype(np.int32)
        dr = O.lorenzo_int(ramp, dims).view(np.int32).reshape(dims[2], dims[1], dims[0])
        interior = dr[1:, 1:, 1:] if dims[2] > 1 else dr[0, 1:, 1:]
        assert np.all(interior == 0)
    # elements past the 2-D field pass through
    b = np.arange(40 * 30 + 17, dtype=np.int32)
    db = O.lorenzo_int(b, (40, 30, 1)).view(np.int32)
    assert np.array_equal(db[1200:], b[1200:])


@pytest.mark.parametrize("code_bytes,zigzag", [(2, False), (2, True), (4, False), (4, True)])
def test_quantizer_abs_round_trip_bound(code_bytes, zigzag):
    # SmoothRoundTrip / ZigzagABSRoundTrip (test_quantizer.cpp:168-198, :531-565): |x - x'| <= eb
    rng = np.random.default_rng(4)
    x = (np.sin(np.arange(40_000) * 0.05) * 10).astype(np.float32)
    x[rng.choice(x.size, 50, replace=False)] = 1e6  # forced outliers
    eb = np.float32(1e-2)
    ebx2_r = np.float32(1.0) / (np.float32(2.0) * eb)
    codes, vals, idx, k = O.quantizer_abs(x, code_bytes, ebx2_r, 32768, zigzag, 1000)
    assert k >= 50 and np.all(np.diff(idx.astype(np.int64)) > 0)
    y = O.quantizer_abs_inv(codes, np.float32(2.0) * eb, zigzag, vals, idx)
    assert np.max(np.abs(y - x)) <= eb * 1.01  # the reference tests allow 1 %


def test_quantizer_constant_and_threshold():
    # ConstantInput (test_quantizer.cpp:200-236): no outliers
    c = np.full(512, 5.0, np.float32)
    r = np.float32(1.0) / (np.float32(2.0) * np.float32(1e-3))
    _, _, _, k = O.quantizer_abs(c, 2, r, 32768, False, 51)
    assert k == 0
    # ABSForcesOutliersAboveThreshold (:1070-1117)
    x = (0.5 + (np.arange(1024, dtype=np.float32) / 1024) * 9.0).astype(np.float32)
    want = int(np.sum(np.abs(x) >= 5.0))
    r2 = np.float32(1.0) / (np.float32(2.0) * np.float32(1e-2))
    codes, vals, idx, k = O.quantizer_abs(x, 4, r2, 1 << 22, True, 615, threshold=5.0)
    assert k == want
    y = O.quantizer_abs_inv(codes, np.float32(2e-2), True, vals, idx)
    assert np.max(np.abs(y - x)) <= 1e-2 * 1.01


def test_quantizer_inplace():
    # AllOutliersRoundTrip (test_quantizer.cpp:951-986): radius 8, constant 5.0
    c = np.full(512, 5.0, np.float32)
    r = np.float32(1.0) / (np.float32(2.0) * np.float32(1e-3))
    codes = O.quantizer_inplace(c, r, 8)
    assert np.array_equal(codes, c.view(np.uint32))
    assert np.array_equal(O.quantizer_inplace_inv(codes, np.float32(2e-3), 8), c)
    # ABSRoundTrip (:875-913)
    x = (np.sin(np.arange(8192) * 0.01) * 3).astype(np.float32)
    x[::997] = 1e7
    codes = O.quantizer_inplace(x, r, 32768)
    y = O.quantizer_inplace_inv(codes, np.float32(2e-3), 32768)
    assert np.max(np.abs(y - x)) <= 1e-3 * 1.01 and np.all(y[::997] == x[::997])
