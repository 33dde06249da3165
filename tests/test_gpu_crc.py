"""fzb_crc32, the FZM data checksum computed on the device, equals zlib's
CRC-32 (the same IEEE polynomial, initial register and final inversion as
compressor_io.cpp:25-52) on sizes around every boundary of the kernel's
segments (512 B), blocks (128 KiB) and fold groups (1024 blocks), on an
unaligned start, and on a buffer large enough for the second fold level."""
import zlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def K():
    from fzgpumodules_b200 import kernels
    return kernels


SIZES = [0, 1, 7, 8, 511, 512, 513, 4096, 131071, 131072, 131073, 5 * 131072 + 777]


@pytest.mark.parametrize("n", SIZES)
def test_crc32_matches_zlib(cuda, n):
    rng = np.random.default_rng(n + 1)
    a = rng.integers(0, 256, n, dtype=np.uint8)
    got = int(K().crc32(torch.from_numpy(a).to(cuda)).item())
    assert got == zlib.crc32(a.tobytes())


def test_crc32_unaligned_and_typed(cuda):
    rng = np.random.default_rng(9)
    a = rng.integers(0, 256, 300_001, dtype=np.uint8)
    d = torch.from_numpy(a).to(cuda)
    for off in (1, 3, 5):  # starts off the 8-byte boundary
        assert int(K().crc32(d[off:]).item()) == zlib.crc32(a[off:].tobytes())
    f = rng.standard_normal(70_000).astype(np.float32)
    assert int(K().crc32(torch.from_numpy(f).to(cuda)).item()) == zlib.crc32(f.tobytes())


def test_crc32_two_fold_levels(cuda):
    n = 1025 * 131072 + 12345  # more than 1024 whole blocks
    g = torch.Generator(device=cuda).manual_seed(3)
    d = torch.randint(0, 256, (n,), dtype=torch.uint8, device=cuda, generator=g)
    want = zlib.crc32(d.cpu().numpy().tobytes())
    assert int(K().crc32(d).item()) == want
