"""CPU checks of the selector oracle: its MLP gradient against central
finite differences, and its per-chunk coder outputs against the oracle's
own decoders (round trips)."""
import numpy as np

from oracle import oracle as O
from oracle import selector_oracle as S


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, S.NP)
    X = rng.uniform(0, 1, (7, 16))
    T = rng.normal(0, 1, (7, 4))
    g, loss = S.mlp_grad(p, X, T)
    assert abs(loss - S.mlp_loss(p, X, T)) < 1e-12
    idx = rng.choice(S.NP, 200, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp = S.mlp_loss(q, X, T)
        q[i] -= 2 * eps
        lm = S.mlp_loss(q, X, T)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-6 * max(1.0, abs(g[i]))


def test_regret_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = rng.normal(0, 0.3, S.NP)
    X = rng.uniform(0, 1, (9, 16))
    R = np.abs(rng.normal(0, 0.5, (9, 4)))
    g, loss = S.regret_grad(p, X, R)
    assert abs(loss - S.regret_loss(p, X, R)) < 1e-12
    eps = 1e-6
    for i in rng.choice(S.NP, 200, replace=False):
        q = p.copy()
        q[i] += eps
        lp = S.regret_loss(q, X, R)
        q[i] -= 2 * eps
        lm = S.regret_loss(q, X, R)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-6 * max(1.0, abs(g[i]))


def _chunks():
    rng = np.random.default_rng(9)
    lap = np.clip(np.round(rng.laplace(0, 2.0, 32768)), -200, 200).astype(np.int64)
    return {
        "laplace_zigzag": ((lap << 1) ^ (lap >> 63)).astype(np.uint16),
        "runs": np.repeat(rng.integers(0, 5, 400), 82)[:32768].astype(np.uint16),
        "zeros_spikes": np.where(rng.random(32768) < 0.03, rng.integers(0, 60000, 32768), 0).astype(np.uint16),
        "uniform16": rng.integers(0, 65536, 32768).astype(np.uint16),
        "partial": rng.integers(0, 7, 5000).astype(np.uint16),
    }


def test_chunk_coders_round_trip():
    for name, c in _chunks().items():
        outs, nb = S.chunk_coder_bytes(c)
        assert outs[2] is not None  # Bitpack always fits
        if outs[0] is not None:
            raw = O.rze_decode(outs[0])
            assert np.array_equal(O.bitshuffle(raw, 16384, 2, inverse=True).view(np.uint16), c), name
        if outs[1] is not None:
            assert np.array_equal(O.rle_decode(outs[1], c.size, np.uint16), c), name
        assert np.array_equal(O.bitpack_decode(outs[2], c.size, nb), c), name
        if outs[3] is not None:
            assert np.array_equal(O.huff_decode(outs[3], c.size), c), name
    # the uniform 16-bit chunk fits only Bitpack / RZE raw-ish; Huffman is not applicable
    outs, nb = S.chunk_coder_bytes(_chunks()["uniform16"])
    assert outs[3] is None and nb == 16
