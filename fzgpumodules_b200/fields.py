"""Seeded synthetic scientific fields with the shapes and value distributions
of the benchmark workloads (the reference's CESM sample is not available, so
these stand in for it).  Generated with torch on any device; float32 out.

* ``grf``        Gaussian random field, isotropic P(k) ~ k^-beta, mean 0, std 1,
                 optional +-spike cells (outlier exercise).
* ``sinusoids2d`` sum of 8 seeded 2-D sinusoids (|k| <= 0.05 rad/cell,
                 amplitudes U(0.05, 0.2)) + N(0, 1e-3), offset into [0, 1].
* ``fractal2d``  Perlin-type gradient noise, 6 octaves, persistence 0.5,
                 scaled to [-50, 50].
"""
from __future__ import annotations

import math

import torch


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def grf(shape, seed: int, beta: float = 3.0, spike_frac: float = 0.0, spike: float = 1e3,
        device="cpu") -> torch.Tensor:
    """shape = (nz, ny, nx) or (ny, nx) or (n,), x fastest."""
    shape = tuple(int(s) for s in shape)
    g = _gen(seed, device)
    white = torch.randn(shape, generator=g, device=device, dtype=torch.float32)
    spec = torch.fft.rfftn(white)
    freqs = [torch.fft.fftfreq(s, device=device) for s in shape[:-1]]
    freqs.append(torch.fft.rfftfreq(shape[-1], device=device))
    k2 = torch.zeros(spec.shape, device=device)
    for ax, f in enumerate(freqs):
        view = [1] * len(shape)
        view[ax] = -1
        k2 = k2 + f.reshape(view) ** 2
    k = torch.sqrt(k2)
    k.view(-1)[0] = 1.0
    amp = k ** (-beta / 2.0)
    amp.view(-1)[0] = 0.0
    field = torch.fft.irfftn(spec * amp, s=shape)
    field = (field - field.mean()) / field.std()
    field = field.to(torch.float32)
    if spike_frac > 0:
        n = field.numel()
        m = max(1, int(round(n * spike_frac)))
        pos = torch.randperm(n, generator=g, device=device)[:m]
        sign = torch.where(torch.rand(m, generator=g, device=device) < 0.5, -1.0, 1.0)
        field.view(-1)[pos] = (spike * sign).to(torch.float32)
    return field.contiguous()


def sinusoids2d(ny: int, nx: int, seed: int, device="cpu") -> torch.Tensor:
    g = _gen(seed, device)
    y = torch.arange(ny, device=device, dtype=torch.float64).view(-1, 1)
    x = torch.arange(nx, device=device, dtype=torch.float64).view(1, -1)
    f = torch.zeros(ny, nx, device=device, dtype=torch.float64)
    for _ in range(8):
        r = torch.rand(4, generator=g, device=device, dtype=torch.float64)
        kmag = 0.05 * r[0]
        ang = 2 * math.pi * r[1]
        amp = 0.05 + 0.15 * r[2]
        ph = 2 * math.pi * r[3]
        f += amp * torch.sin(kmag * torch.cos(ang) * x + kmag * torch.sin(ang) * y + ph)
    f += 1e-3 * torch.randn(ny, nx, generator=g, device=device, dtype=torch.float64)
    f = (f - f.min()) / (f.max() - f.min())
    return f.to(torch.float32).contiguous()


def fractal2d(n: int, seed: int, octaves: int = 6, persistence: float = 0.5,
              device="cpu") -> torch.Tensor:
    g = _gen(seed, device)
    out = torch.zeros(n, n, device=device, dtype=torch.float32)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 4 * (2 ** o)
        ang = 2 * math.pi * torch.rand(cells + 1, cells + 1, generator=g, device=device)
        gx, gy = torch.cos(ang), torch.sin(ang)
        coord = torch.arange(n, device=device, dtype=torch.float32) * (cells / n)
        i0 = coord.floor().long().clamp(max=cells - 1)
        fr = coord - i0
        fy, fx = fr.view(-1, 1), fr.view(1, -1)
        iy, ix = i0.view(-1, 1), i0.view(1, -1)

        def dot(dy, dx):
            return gx[iy + dy, ix + dx] * (fx - dx) + gy[iy + dy, ix + dx] * (fy - dy)

        sx = fx * fx * fx * (fx * (fx * 6 - 15) + 10)
        sy = fy * fy * fy * (fy * (fy * 6 - 15) + 10)
        top = dot(0, 0) + sx * (dot(0, 1) - dot(0, 0))
        bot = dot(1, 0) + sx * (dot(1, 1) - dot(1, 0))
        out += amp * (top + sy * (bot - top))
        total += amp
        amp *= persistence
    out = out / total
    out = (out - out.min()) / (out.max() - out.min()) * 100.0 - 50.0
    return out.contiguous()


def piecewise(n: int, seed: int, min_run: int = 10, max_run: int = 1000, device="cpu") -> torch.Tensor:
    """Piecewise-constant values: runs of 10-1000 cells, each run N(0, 1)."""
    g = _gen(seed, device)
    runs = torch.randint(min_run, max_run + 1, (n // min_run + 2,), generator=g, device=device)
    ends = torch.cumsum(runs, 0)
    k = int(torch.searchsorted(ends, torch.tensor([n], device=device)).item()) + 1
    vals = torch.randn(k, generator=g, device=device)
    rid = torch.searchsorted(ends[:k], torch.arange(n, device=device), right=True)
    return vals[rid.clamp(max=k - 1)].to(torch.float32).contiguous()


def noise(n: int, seed: int, device="cpu") -> torch.Tensor:
    """White noise N(0, 1)."""
    return torch.randn(n, generator=_gen(seed, device), device=device, dtype=torch.float32)


def sparse(n: int, seed: int, density: float = 0.05, device="cpu") -> torch.Tensor:
    """95 % zeros, the rest N(0, 1)."""
    g = _gen(seed, device)
    v = torch.randn(n, generator=g, device=device, dtype=torch.float32)
    keep = torch.rand(n, generator=g, device=device) < density
    return torch.where(keep, v, torch.zeros_like(v)).contiguous()


def mixed_field(kind: str, shape, seed: int, device="cpu") -> torch.Tensor:
    """One field of the learned-selector workload: 'smooth' (GRF k^-3),
    'piecewise', 'noise' or 'sparse'; shape (nz, ny, nx)."""
    n = 1
    for s in shape:
        n *= int(s)
    if kind == "smooth":
        return grf(shape, seed=seed, device=device).reshape(-1)
    if kind == "piecewise":
        return piecewise(n, seed, device=device)
    if kind == "noise":
        return noise(n, seed, device=device)
    if kind == "sparse":
        return sparse(n, seed, device=device)
    raise ValueError(kind)
