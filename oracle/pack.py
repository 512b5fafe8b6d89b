"""TEST INFRASTRUCTURE: numpy restatement of the library's fixed-rate lossy
wavefield store (pyfwix_b200/csrc/pack.cu), the checker of its bytes.

The reference stores its background wavefields ZFP-compressed at a fixed rate of
8 bits per value (propagator/src/WavefieldPool.cpp:23, :52-60); the library
replaces that with its own block format, restated here: the wavefield's floats in
blocks of 16; per block the largest magnitude m = f 2^E (f in [0.5, 1)), mantissas
q = rint(v 2^(7 - E)) clamped to [-127, 127] (int8), exponent byte E + 128
(clamped to 1..255); blocks with m < 2^-100 are zeros with exponent byte 0.
Blocks with m >= 2^127 and non-finite values are outside the format.
Packed layout: all mantissas (16 bytes per block), then the exponent bytes, padded
to a multiple of 256 bytes.  Parity with the device is bit-exact (powers-of-two
scaling and round-half-even on both sides).  There is no reference code to pin
it against: the reference's ZFP arithmetic is a third-party library (zfp, not
vendored) and its bit stream is a different format; the tests pin this restatement
by its own properties (error bound, zeros, layout, idempotence).
"""
from __future__ import annotations

import numpy as np

BLOCK = 16


def packed_bytes(nfloat):
    nblk = -(-nfloat // BLOCK)
    return -(-(nblk * (BLOCK + 1)) // 256) * 256


def pack(x):
    """complex64 array -> uint8 packed bytes."""
    f = np.ascontiguousarray(x, dtype=np.complex64).view(np.float32).ravel()
    n = f.size
    nblk = -(-n // BLOCK)
    blocks = np.zeros(nblk * BLOCK, np.float32)
    blocks[:n] = f
    blocks = blocks.reshape(nblk, BLOCK)
    m = np.abs(blocks).max(axis=1)
    _, E = np.frexp(m)
    zero = ~(m >= np.float32(2.0 ** -100))
    scale = np.where(zero, np.float32(0), np.ldexp(np.float32(1), (7 - E)).astype(np.float32)).astype(np.float32)
    q = np.rint(blocks * scale[:, None]).astype(np.float32)
    q = np.clip(q, -127, 127).astype(np.int8)
    e = np.clip(E + 128, 1, 255).astype(np.uint8)
    e[zero] = 0
    out = np.zeros(packed_bytes(n), np.uint8)
    out[:nblk * BLOCK] = q.view(np.uint8).ravel()
    out[nblk * BLOCK:nblk * BLOCK + nblk] = e
    return out


def unpack(packed, shape):
    """uint8 packed bytes -> complex64 array of `shape`."""
    n = 2 * int(np.prod(shape))
    nblk = -(-n // BLOCK)
    q = packed[:nblk * BLOCK].view(np.int8).reshape(nblk, BLOCK).astype(np.float32)
    e = packed[nblk * BLOCK:nblk * BLOCK + nblk].astype(np.int64)
    scale = np.where(e == 0, np.float32(0), np.ldexp(np.float32(1), (e - 128 - 7)).astype(np.float32))
    f = (q * scale.astype(np.float32)[:, None]).astype(np.float32).ravel()[:n]
    return f.view(np.complex64).reshape(shape)
