"""B200-native one-way wave-equation depth stepping (PSPI / NSPS, Born scattering,
imaging) behind pyfwix's CudaWEM / CudaOperator surface.

The compute path is libfwix_b200.so (hand-written sm_100a CUDA behind a C ABI,
include/fwix_b200.h); this package is its Python host side.
"""
from . import _lib  # noqa: F401

__version__ = "0.1.0"
