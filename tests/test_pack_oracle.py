"""The oracle's restatement of the fixed-rate lossy wavefield store
(oracle/pack.py) on its own properties, CPU only: per-block error bound, zero
blocks, ragged tails, layout size and idempotence."""
import numpy as np
import pytest

from oracle import pack


@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("shape", [(1, 3, 8, 8), (2, 5, 7, 9), (1, 1, 1, 3)])
def test_error_bound_and_layout(shape, bits):
    rng = np.random.default_rng(sum(shape))
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    x *= np.float32(10.0) ** rng.integers(-6, 6, size=shape)  # a wide dynamic range between blocks
    p = pack.pack(x, bits)
    assert p.dtype == np.uint8 and p.size == pack.packed_bytes(2 * x.size, bits) and p.size % 256 == 0
    y = pack.unpack(p, x.shape, bits)
    f = x.view(np.float32).ravel()
    g = y.view(np.float32).ravel()
    n = f.size
    blk = np.zeros(-(-n // 16) * 16, np.float32)
    blk[:n] = np.abs(f)
    m = np.repeat(blk.reshape(-1, 16).max(axis=1), 16)[:n]
    assert np.all(np.abs(f - g) <= m * 2.0 ** -(bits - 1) * (1 + 1e-6))
    # idempotent: what comes back packs to the same bytes
    assert np.array_equal(pack.pack(y, bits), p)


def test_zero_and_tiny_blocks():
    x = np.zeros((1, 1, 4, 8), np.complex64)
    x[0, 0, 1, :] = 1e-35  # below 2^-100: stored as zero
    x[0, 0, 2, 0] = 3.0
    p = pack.pack(x)
    y = pack.unpack(p, x.shape)
    assert np.all(y[0, 0, 0] == 0) and np.all(y[0, 0, 1] == 0)
    assert y[0, 0, 2, 0] == np.complex64(3.0)
    nblk = 2 * x.size // 16
    assert p[nblk * 16] == 0  # exponent byte of the first (zero) block
