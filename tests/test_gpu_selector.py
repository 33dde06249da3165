"""The learned per-chunk coder selector on the GPU.

* every coder's bytes on every chunk equal the oracle's restatement of that
  stage on the chunk alone (fixed-coder containers), and the exhaustive
  trial sizes and choices equal the oracle's;
* containers decode back to the codes (exhaustive, learned, fixed);
* features, MLP forward and MLP gradient match the CPU oracle;
* a selector trained with the library's own kernels on method-generated
  chunks keeps the exhaustive trial's compression ratio (within 1 %) on
  held-out data and beats every single fixed coder.
"""
import numpy as np
import pytest
import torch

from oracle import selector_oracle as S

pytestmark = pytest.mark.gpu


def Sel():
    from fzgpumodules_b200 import selector
    return selector


def _codes():
    rng = np.random.default_rng(21)
    lap = np.clip(np.round(rng.laplace(0, 2.0, 32768 * 3)), -300, 300).astype(np.int64)
    parts = [
        ((lap << 1) ^ (lap >> 63)).astype(np.uint16),                                     # Huffman-friendly
        np.repeat(rng.integers(0, 5, 900), 80)[:32768 * 2].astype(np.uint16),            # runs
        np.where(rng.random(32768) < 0.02, rng.integers(0, 60000, 32768), 0).astype(np.uint16),  # sparse spikes
        rng.integers(0, 65536, 32768).astype(np.uint16),                                 # incompressible
        np.zeros(32768, np.uint16),                                                      # constant
        rng.integers(0, 3, 32768).astype(np.uint16),                                     # 2-bit noise
        rng.permutation(np.repeat(np.arange(512), 64)).astype(np.uint16),                # all frequencies tie
        rng.permutation(np.repeat(rng.permutation(1024),                                 # four frequency levels
                                  np.repeat([48, 24, 12, 4], [512, 256, 128, 128]))).astype(np.uint16),
        rng.integers(0, 1200, 20000).astype(np.uint16),                                  # partial, >= 1024
    ]
    return np.concatenate(parts)


def _split(blob: np.ndarray, n: int):
    h = blob[:16].view(np.uint32)
    nch = int(h[1])
    assert h[0] == 0x43535A46 and h[2] == n and h[3] == 32768
    pad = (nch + 3) & ~3
    tags = blob[16:16 + nch]
    params = blob[16 + pad:16 + pad + nch]
    sizes = blob[16 + 2 * pad:16 + 2 * pad + 4 * nch].view(np.uint32)
    off = 16 + 2 * pad + 4 * nch
    pays = []
    for s in sizes:
        pays.append(blob[off:off + int(s)])
        off += (int(s) + 3) & ~3
    assert off == blob.size
    return tags, params, pays


def test_coder_bytes_sizes_and_choices_match_oracle(cuda):
    c = _codes()
    d = torch.from_numpy(c).to(cuda)
    ref_sizes = S.chunk_sizes(c)
    sizes = Sel().trial_sizes(d).cpu().numpy().astype(np.uint32)
    assert np.array_equal(sizes, ref_sizes)
    nch = ref_sizes.shape[0]
    ref_bytes = [S.chunk_coder_bytes(c[i * 32768:(i + 1) * 32768]) for i in range(nch)]
    for k in range(4):
        blob, tags = Sel().encode(d, Sel().fixed(k))
        t, params, pays = _split(blob.cpu().numpy(), c.size)
        for i in range(nch):
            outs, nb = ref_bytes[i]
            if outs[k] is not None:
                assert t[i] == k
                assert np.array_equal(pays[i], outs[k]), (k, i)
                if k == 2:
                    assert params[i] == nb
            else:  # does not fit: the exhaustive fallback picked another coder
                assert t[i] != k
        dec = Sel().decode(blob, c.size).cpu().numpy()
        assert np.array_equal(dec, c)
    blob, tags = Sel().encode(d, Sel().EXHAUSTIVE)
    want = np.argmin(ref_sizes.astype(np.int64), axis=1)  # first minimum = lowest coder index
    assert np.array_equal(tags.cpu().numpy(), want)
    assert np.array_equal(Sel().decode(blob, c.size).cpu().numpy(), c)


def test_features_match_oracle(cuda):
    c = _codes()
    f = Sel().features(torch.from_numpy(c).to(cuda)).cpu().numpy()
    np.testing.assert_allclose(f, S.features(c), rtol=1e-4, atol=2e-5)


def test_features_ragged_and_unaligned(cuda):
    # a length that is not a multiple of 8 codes, and a view 2 bytes off the
    # 16-byte boundary (the scalar path of the features kernel)
    c = _codes()
    dev = torch.from_numpy(c).to(cuda)
    for lo, hi in ((0, 32768 + 13), (1, 1 + 2 * 32768 + 5)):
        f = Sel().features(dev[lo:hi]).cpu().numpy()
        np.testing.assert_allclose(f, S.features(c[lo:hi]), rtol=1e-4, atol=2e-5)


def test_mlp_forward_and_gradient_match_oracle(cuda):
    rng = np.random.default_rng(4)
    sel = Sel().CoderSelector(seed=3, device=cuda)
    X = rng.uniform(0, 1, (1000, 16)).astype(np.float32)
    T = rng.normal(-2, 1, (1000, 4)).astype(np.float32)
    p = sel.params.cpu().numpy().astype(np.float64)
    y = sel.predict(torch.from_numpy(X).to(cuda)).cpu().numpy()
    np.testing.assert_allclose(y, S.mlp_forward(p, X), rtol=1e-5, atol=1e-5)
    g, loss = sel.grad(torch.from_numpy(X).to(cuda), torch.from_numpy(T).to(cuda), Sel().MSE)
    gr, lr = S.mlp_grad(p, X, T)
    np.testing.assert_allclose(g.cpu().numpy(), gr, rtol=1e-3, atol=1e-6)
    assert abs(float(loss.item()) - lr) < 1e-4 * max(1.0, lr)
    R = np.abs(T).astype(np.float32) / 4
    g, loss = sel.grad(torch.from_numpy(X).to(cuda), torch.from_numpy(R).to(cuda), Sel().REGRET)
    gr, lr = S.regret_grad(p, X, R)
    np.testing.assert_allclose(g.cpu().numpy(), gr, rtol=1e-3, atol=1e-7)
    assert abs(float(loss.item()) - lr) < 1e-4 * max(1.0, lr)


def test_trained_selector_keeps_exhaustive_ratio(cuda):
    sel = Sel().CoderSelector(seed=0, device=cuda)
    train = Sel().method_codes(48, seed=500, device=cuda)            # 48 fields x 32 chunks
    x = Sel().features(train)
    t = Sel().regrets_from_sizes(Sel().trial_sizes(train))
    losses = sel.train(x, t, epochs=60, batch=256, lr=3e-3)
    assert losses[-1] < losses[0]
    test = Sel().method_codes(16, seed=9000, device=cuda)
    r = Sel().compare(test, sel)
    assert r["ratio_learned"] >= 0.99 * r["ratio_exhaustive"], r
    assert r["ratio_learned"] > r["ratio_best_fixed"], r
    blob, _ = Sel().encode(test, Sel().LEARNED, sel)
    assert torch.equal(Sel().decode(blob, test.numel()), test)
