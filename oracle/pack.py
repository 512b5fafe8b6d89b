"""TEST INFRASTRUCTURE: numpy restatement of the library's fixed-rate lossy
wavefield store (pyfwix_b200/csrc/pack.cu), the checker of its bytes.

The reference stores its background wavefields ZFP-compressed at a fixed rate of
8 bits per value (propagator/src/WavefieldPool.cpp:23, :52-60); the library
replaces that with its own block format, restated here, at 8 or 16 bits per
mantissa (``bits``): the wavefield's floats in blocks of 16; per block the
largest magnitude m = f 2^E (f in [0.5, 1)), mantissas q = rint(v 2^(B - E))
clamped to [-(2^B - 1), 2^B - 1] with B = bits - 1 (int8 or int16), exponent byte
E + 128 (clamped to 1..255); blocks with m < 2^-100 are zeros with exponent byte
0.  Blocks with m >= 2^127 and non-finite values are outside the format.
Packed layout: all mantissas (16 or 32 bytes per block), then the exponent bytes,
padded to a multiple of 256 bytes.  Parity with the device is bit-exact (powers-of-two
scaling and round-half-even on both sides).  There is no reference code to pin
it against: the reference's ZFP arithmetic is a third-party library (zfp, not
vendored) and its bit stream is a different format; the tests pin this restatement
by its own properties (error bound, zeros, layout, idempotence).
"""
from __future__ import annotations

import numpy as np

BLOCK = 16


def _mant(bits):
    if bits not in (8, 16):
        raise ValueError("bits must be 8 or 16")
    return (np.int8 if bits == 8 else np.int16), bits - 1


def packed_bytes(nfloat, bits=8):
    nblk = -(-nfloat // BLOCK)
    return -(-(nblk * (BLOCK * bits // 8 + 1)) // 256) * 256


def pack(x, bits=8):
    """complex64 array -> uint8 packed bytes."""
    qt, B = _mant(bits)
    f = np.ascontiguousarray(x, dtype=np.complex64).view(np.float32).ravel()
    n = f.size
    nblk = -(-n // BLOCK)
    blocks = np.zeros(nblk * BLOCK, np.float32)
    blocks[:n] = f
    blocks = blocks.reshape(nblk, BLOCK)
    m = np.abs(blocks).max(axis=1)
    _, E = np.frexp(m)
    zero = ~(m >= np.float32(2.0 ** -100))
    scale = np.where(zero, np.float32(0), np.ldexp(np.float32(1), (B - E)).astype(np.float32)).astype(np.float32)
    q = np.rint(blocks * scale[:, None]).astype(np.float32)
    lim = float(2 ** B - 1)
    q = np.clip(q, -lim, lim).astype(qt)
    e = np.clip(E + 128, 1, 255).astype(np.uint8)
    e[zero] = 0
    mb = nblk * BLOCK * bits // 8
    out = np.zeros(packed_bytes(n, bits), np.uint8)
    out[:mb] = q.view(np.uint8).ravel()
    out[mb:mb + nblk] = e
    return out


def unpack(packed, shape, bits=8):
    """uint8 packed bytes -> complex64 array of `shape`."""
    qt, B = _mant(bits)
    n = 2 * int(np.prod(shape))
    nblk = -(-n // BLOCK)
    mb = nblk * BLOCK * bits // 8
    q = packed[:mb].view(qt).reshape(nblk, BLOCK).astype(np.float32)
    e = packed[mb:mb + nblk].astype(np.int64)
    scale = np.where(e == 0, np.float32(0), np.ldexp(np.float32(1), (e - 128 - B)).astype(np.float32))
    f = (q * scale.astype(np.float32)[:, None]).astype(np.float32).ravel()[:n]
    return f.view(np.complex64).reshape(shape)
