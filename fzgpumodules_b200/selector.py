"""Learned per-chunk coder selection (fzb_sel_*, fzb_mlp_* in fzb.h).

The quantization codes of a field are cut into 64 KiB chunks; each chunk is
coded by Bitshuffle+RZE, RLE, Bitpack or Huffman.  Exhaustive trial codes
every chunk four ways and keeps the smallest; the learned path computes 16
statistics per chunk, runs a 16 -> 64 -> 64 -> 4 FP32 MLP that predicts the
four coders' log2 sizes, and codes each chunk only with the predicted best
coder (falling back to the others where that coder's output does not fit).
The chosen coder is stored as the chunk's tag; no coder's bytes change.

Training labels come from exhaustive trial on method-generated chunks
(LorenzoQuant codes of seeded smooth / piecewise-constant / noise / sparse
fields); training runs the library's own forward / backward / Adam kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import kernels as K
from ._lib import check, lib

CHUNK_CODES = 32768
NFEAT = 16
NCODERS = 4
NPARAMS = 16 * 64 + 64 + 64 * 64 + 64 + 64 * 4 + 4
EXHAUSTIVE, LEARNED = 0, 1
CODERS = ("bitshuffle+rze", "rle", "bitpack", "huffman")
NOFIT = 0xFFFFFFFF


def fixed(k: int) -> int:
    return 2 + k


def _p(t):
    return C.c_void_p(t.data_ptr())


def _s(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def nchunks(n: int) -> int:
    return (n + CHUNK_CODES - 1) // CHUNK_CODES


class _Work:
    def __init__(self):
        self.buf = None

    def get(self, need: int, dev):
        need = max(int(need), 256)
        if self.buf is None or self.buf.numel() < need or self.buf.device != dev:
            self.buf = torch.empty(need, dtype=torch.uint8, device=dev)
        return _p(self.buf), self.buf.numel()


_work = _Work()


def features(codes: torch.Tensor) -> torch.Tensor:
    c = codes.reshape(-1)
    f = torch.empty(nchunks(c.numel()), NFEAT, dtype=torch.float32, device=c.device)
    check(lib().fzb_sel_features(_p(c), c.numel(), _p(f), _s(c.device)), "fzb_sel_features")
    return f


def trial_sizes(codes: torch.Tensor) -> torch.Tensor:
    """Exhaustive trial: [nchunks, 4] output sizes (NOFIT = does not fit)."""
    c = codes.reshape(-1)
    out = torch.empty(nchunks(c.numel()), NCODERS, dtype=torch.int32, device=c.device)
    wp, wn = _work.get(lib().fzb_sel_workspace_bytes(c.numel()), c.device)
    check(lib().fzb_sel_trial(_p(c), c.numel(), _p(out), wp, wn, _s(c.device)), "fzb_sel_trial")
    return out.to(torch.int64) & 0xFFFFFFFF


MSE, REGRET = 0, 1


def targets_from_sizes(sizes: torch.Tensor) -> torch.Tensor:
    """Regression targets: log2(size / 65536); sizes that do not fit -> 1.0."""
    s = sizes.to(torch.int64) & 0xFFFFFFFF
    t = torch.log2(torch.clamp(s.to(torch.float64), min=1.0) / 65536.0)
    t[s == NOFIT] = 1.0
    return t.to(torch.float32)


def regrets_from_sizes(sizes: torch.Tensor) -> torch.Tensor:
    """Regret of each coder: log2(size / smallest size) (0 for the best);
    coders that do not fit -> 2.0."""
    s = (sizes.to(torch.int64) & 0xFFFFFFFF).to(torch.float64)
    nofit = s == NOFIT
    s = torch.where(nofit, torch.full_like(s, float("inf")), torch.clamp(s, min=1.0))
    r = torch.log2(s / s.min(dim=1, keepdim=True).values)
    r[nofit] = 2.0
    return r.to(torch.float32)


def encode(codes: torch.Tensor, mode: int, selector: "CoderSelector | None" = None, trim: bool = True):
    """Container bytes (trimmed), and the chosen coder per chunk.  With
    trim=False nothing synchronises: returns (buffer at capacity, tags,
    device size)."""
    c = codes.reshape(-1)
    dev = c.device
    nch = nchunks(c.numel())
    out = torch.empty(int(lib().fzb_sel_max_bytes(c.numel())), dtype=torch.uint8, device=dev)
    size = torch.zeros(1, dtype=torch.int64, device=dev)
    tags = torch.empty(nch, dtype=torch.uint8, device=dev)
    wp, wn = _work.get(lib().fzb_sel_workspace_bytes(c.numel()), dev)
    params = _p(selector.params) if selector is not None else None
    check(lib().fzb_sel_encode(_p(c), c.numel(), mode, params, _p(out), _p(size), _p(tags), wp, wn, _s(dev)),
          "fzb_sel_encode")
    if not trim:
        return out, tags, size
    return out[: int(size.item())], tags


def decode(blob: torch.Tensor, n: int) -> torch.Tensor:
    dev = blob.device
    out = torch.empty(n, dtype=torch.uint16, device=dev)
    need = int(lib().fzb_workspace_bytes(CHUNK_CODES, 0)) + 2 * 65536 + 512
    wp, wn = _Work().get(need, dev)
    check(lib().fzb_sel_decode(_p(blob), blob.numel(), _p(out), n, wp, wn, _s(dev)), "fzb_sel_decode")
    return out


class CoderSelector:
    """The 16 -> 64 -> 64 -> 4 MLP; parameters in one device tensor."""

    def __init__(self, seed: int = 0, device=None):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        g = torch.Generator().manual_seed(seed)
        parts = []
        for fan_in, fan_out in ((16, 64), (64, 64), (64, 4)):
            bound = (6.0 / fan_in) ** 0.5 * 0.5
            parts.append((torch.rand(fan_in * fan_out, generator=g) * 2 - 1) * bound)
            parts.append(torch.zeros(fan_out))
        self.params = torch.cat(parts).to(torch.float32).to(dev).contiguous()
        assert self.params.numel() == NPARAMS
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0

    def predict(self, x: torch.Tensor) -> torch.Tensor:
        x = x.contiguous()
        y = torch.empty(x.shape[0], NCODERS, dtype=torch.float32, device=x.device)
        check(lib().fzb_mlp_forward(_p(self.params), _p(x), _p(y), x.shape[0], _s(x.device)), "fzb_mlp_forward")
        return y

    def grad(self, x: torch.Tensor, t: torch.Tensor, kind: int = REGRET):
        x, t = x.contiguous(), t.contiguous()
        g = torch.empty_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device=x.device)
        check(lib().fzb_mlp_grad(_p(self.params), _p(x), _p(t), x.shape[0], kind, _p(g), _p(loss),
                                 _s(x.device)), "fzb_mlp_grad")
        return g, loss

    def adam(self, g: torch.Tensor, lr: float):
        self.step += 1
        check(lib().fzb_mlp_adam(_p(self.params), _p(g), _p(self.m), _p(self.v), lr, self.step,
                                 _s(self.params.device)), "fzb_mlp_adam")

    def train(self, x: torch.Tensor, t: torch.Tensor, epochs: int = 20, batch: int = 2048, lr: float = 3e-3,
              seed: int = 0, kind: int = REGRET) -> list:
        """Adam over shuffled mini-batches; t holds regrets (REGRET) or
        log-size targets (MSE).  Returns the mean loss of every epoch."""
        n = x.shape[0]
        g = torch.Generator(device=x.device).manual_seed(seed)
        losses = []
        acc = torch.zeros(1, dtype=torch.float32, device=x.device)
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g, device=x.device)
            acc.zero_()
            nb = 0
            for b in range(0, n, batch):
                idx = perm[b:b + batch]
                gr, loss = self.grad(x[idx], t[idx], kind)
                self.adam(gr, lr * (0.5 ** (ep // max(1, epochs // 3))))
                acc += loss
                nb += 1
            losses.append(float(acc.item()) / max(nb, 1))
        return losses


def method_codes(count: int, seed: int, device, shape=(64, 128, 128), eb: float = 1e-3) -> torch.Tensor:
    """LorenzoQuant (REL eb, radius 32768, zigzag) codes of `count` seeded
    fields cycling through smooth / piecewise / noise / sparse, concatenated
    (every field is a whole number of chunks)."""
    from . import fields as F
    kinds = ("smooth", "piecewise", "noise", "sparse")
    nz, ny, nx = shape
    out = []
    for i in range(count):
        x = F.mixed_field(kinds[i % 4], shape, seed + i, device=device)
        r = K.lq_forward(x, (nx, ny, nz), eb, K.REL, 32768, True, 0.2)
        out.append(r["codes"])
    return torch.cat(out)


def method_training_set(n_chunks: int, seed: int, device, shape=(128, 256, 256), eb: float = 1e-3):
    """Features and exhaustive-trial regrets of `n_chunks` method-generated
    chunks: LorenzoQuant (REL eb, radius 32768, zigzag) codes of seeded
    fields cycling through smooth / piecewise / noise / sparse, one field at
    a time (each `shape` field is a whole number of chunks), so only the
    16 features and 4 sizes of each chunk are kept.  Returns (X, T) on the
    device."""
    from . import fields as F
    kinds = ("smooth", "piecewise", "noise", "sparse")
    nz, ny, nx = shape
    per = nchunks(nx * ny * nz)
    xs, ts, have, i = [], [], 0, 0
    while have < n_chunks:
        x = F.mixed_field(kinds[i % 4], shape, seed + i, device=device)
        codes = K.lq_forward(x, (nx, ny, nz), eb, K.REL, 32768, True, 0.2)["codes"]
        del x
        take = min(per, n_chunks - have)
        c = codes[: take * CHUNK_CODES]
        xs.append(features(c))
        ts.append(regrets_from_sizes(trial_sizes(c)))
        have += take
        i += 1
    return torch.cat(xs), torch.cat(ts)


def compare(codes: torch.Tensor, sel: CoderSelector) -> dict:
    """Sizes of the exhaustive, learned and fixed-coder containers."""
    ex, tex = encode(codes, EXHAUSTIVE)
    le, tle = encode(codes, LEARNED, sel)
    fixed_sizes = [encode(codes, fixed(k))[0].numel() for k in range(NCODERS)]
    n = codes.numel() * 2
    return dict(exhaustive=ex.numel(), learned=le.numel(), fixed=fixed_sizes,
                ratio_exhaustive=n / ex.numel(), ratio_learned=n / le.numel(),
                ratio_best_fixed=n / min(fixed_sizes),
                agreement=float((tex == tle).float().mean().item()))
