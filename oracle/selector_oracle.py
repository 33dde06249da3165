"""Test infrastructure: CPU restatement of the per-chunk coder selector.

* ``mlp_forward`` / ``mlp_grad``: the 16 -> 64 -> 64 -> 4 FP32 ReLU network
  and the gradient of its mean squared error in float64 numpy (the device
  kernels are checked against these within a tolerance; the gradient itself
  is checked against central finite differences in the CPU tests).
* ``chunk_coder_bytes``: each coder's exact output on one 64 KiB chunk of
  codes, built from the oracle's stage restatements (fzoracle.c): Bitshuffle
  (16 KiB, element width 2) -> RZE, RLE, Bitpack with detected nbits, and
  Huffman with bklen 1024 from the chunk's own histogram.
* ``features``: the 16 per-chunk statistics.
Never imported by the product.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

CHUNK = 32768
NP = 16 * 64 + 64 + 64 * 64 + 64 + 64 * 4 + 4


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + 1024].reshape(16, 64); o += 1024
    b1 = p[o:o + 64]; o += 64
    W2 = p[o:o + 4096].reshape(64, 64); o += 4096
    b2 = p[o:o + 64]; o += 64
    W3 = p[o:o + 256].reshape(64, 4); o += 256
    b3 = p[o:o + 4]
    return W1, b1, W2, b2, W3, b3


def mlp_forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    h1 = np.maximum(X @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ W3 + b3


def mlp_loss(p, X, T):
    Y = mlp_forward(p, X)
    return float(np.mean((Y - np.asarray(T, np.float64)) ** 2))


def mlp_grad(p, X, T):
    """Gradient of mean((Y - T)^2) over batch x 4, packed like p."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    B = X.shape[0]
    a1 = X @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    Y = h2 @ W3 + b3
    dY = 2.0 * (Y - T) / (4.0 * B)
    gW3 = h2.T @ dY
    gb3 = dY.sum(0)
    dh2 = (dY @ W3.T) * (a2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (a1 > 0)
    gW1 = X.T @ dh1
    gb1 = dh1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]), float(np.mean((Y - T) ** 2))


TAU = 0.02


def _softmax_rows(z):
    z = z - z.max(axis=1, keepdims=True)
    e = np.exp(z)
    return e / e.sum(axis=1, keepdims=True)


def regret_loss(p, X, R):
    """Cross-entropy of softmax(-y) against the soft labels softmax(-R/TAU)."""
    Y = mlp_forward(p, X)
    P = _softmax_rows(-Y)
    Q = _softmax_rows(-np.asarray(R, np.float64) / TAU)
    return float(np.mean(-np.sum(Q * np.log(P), axis=1)))


def regret_grad(p, X, R):
    """Gradient of regret_loss, packed like p."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    R = np.asarray(R, np.float64)
    B = X.shape[0]
    a1 = X @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    Y = h2 @ W3 + b3
    P = _softmax_rows(-Y)
    Q = _softmax_rows(-R / TAU)
    L = -np.sum(Q * np.log(P), axis=1)
    dY = (Q - P) / B
    gW3 = h2.T @ dY
    gb3 = dY.sum(0)
    dh2 = (dY @ W3.T) * (a2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (a1 > 0)
    gW1 = X.T @ dh1
    gb1 = dh1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]), float(np.mean(L))


# ------------------------------------------------------------------ coders

def _bitpack_nbits(m: int) -> int:
    b = 1
    while b < 16:
        if m < (1 << b):
            return b
        b *= 2
    return 16


def chunk_coder_bytes(codes: np.ndarray):
    """[bytes or None] x 4 for one chunk (None: larger than 64 KiB / not
    applicable), plus the Bitpack nbits."""
    c = np.ascontiguousarray(codes, np.uint16)
    out = []
    shuffled = O.bitshuffle(c, 16384, 2)
    rze = O.rze_encode(shuffled)
    out.append(rze if rze.size <= 65536 else None)
    rle = O.rle_encode(c)
    out.append(rle if rle.size <= 65536 else None)
    nb = _bitpack_nbits(int(c.max()))
    out.append(O.bitpack_encode(c, nb))
    if int(c.max()) < 1024:
        freq = np.bincount(c, minlength=1024).astype(np.uint32)
        bk4, rb = O.huff_book(freq, 1024)
        hf = O.huff_encode(c, 1024, bk4, rb)
        out.append(hf if hf.size <= 65536 else None)
    else:
        out.append(None)
    return out, nb


def chunk_sizes(codes: np.ndarray) -> np.ndarray:
    """Per chunk, the four coders' sizes (0xFFFFFFFF = no fit)."""
    n = codes.size
    res = []
    for b in range(0, n, CHUNK):
        outs, _ = chunk_coder_bytes(codes[b:b + CHUNK])
        res.append([o.size if o is not None else 0xFFFFFFFF for o in outs])
    return np.array(res, np.uint32)


def features(codes: np.ndarray) -> np.ndarray:
    """The 16 per-chunk statistics (float64)."""
    n = codes.size
    out = []
    for b in range(0, n, CHUNK):
        u = codes[b:b + CHUNK].astype(np.int64)
        cnt = u.size
        lg = np.log2(1.0 + u)
        f = np.zeros(16)
        f[0] = lg.mean() / 16
        f[1] = np.sqrt(max(np.mean(lg * lg) - lg.mean() ** 2, 0.0)) / 8
        f[2] = np.mean(u == 0)
        d = np.abs(np.diff(u))
        f[3] = 1.0 - np.sum(d == 0) / cnt
        f[4] = (np.sum((u & 0xFF) == 0) + np.sum((u >> 8) == 0)) / (2 * cnt)
        f[5] = np.sum(np.log2(1.0 + d)) / cnt / 16
        hb = np.zeros(4)
        for bit in range(16):
            pb = np.mean((u >> bit) & 1)
            h = 0.0 if pb <= 0 or pb >= 1 else -(pb * np.log2(pb) + (1 - pb) * np.log2(1 - pb))
            hb[bit >> 2] += 0.25 * h
        f[6:10] = hb
        f[10] = np.log2(1.0 + u.max()) / 16
        for k, v in ((11, u & 0xFF), (12, u >> 8)):
            p = np.bincount(v, minlength=256) / cnt
            p = p[p > 0]
            f[k] = -np.sum(p * np.log2(p)) / 8
        f[13] = 1.0 if np.any(u >= 1024) else 0.0
        ng = (cnt + 7) // 8
        pad = np.zeros(ng * 8, np.int64)
        pad[:cnt] = u
        gor = np.bitwise_or.reduce(pad.reshape(ng, 8), axis=1)
        f[14] = sum(bin(int(v)).count("1") for v in gor) / (2 * cnt)
        p = np.bincount(np.minimum(u, 1023), minlength=1024) / cnt
        p = p[p > 0]
        f[15] = -np.sum(p * np.log2(p)) / 10
        out.append(f)
    return np.array(out)


def targets(sizes: np.ndarray) -> np.ndarray:
    """Regression targets: log2(size / 65536), sizes that do not fit -> 1."""
    s = sizes.astype(np.float64)
    t = np.log2(np.maximum(s, 1.0) / 65536.0)
    t[sizes == 0xFFFFFFFF] = 1.0
    return t
