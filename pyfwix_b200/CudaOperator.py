"""Drop-in for pyfwix's ``fwix.CudaOperator`` (``fwix/CudaOperator.py:7-20``).

``cuFFT2d(model, data)``: the unitary 2D DFT over the two fastest axes (y, x) of
every leading index, ``forward`` with e^{-i}, ``adjoint`` with e^{+i}, both scaled
by 1/sqrt(nx ny) (``operator/src/FFT.cpp:5-69``, ``operator/src/fft_callback.cu:7-22``).
It runs this library's own Stockham kernels, not cuFFT.
"""
from __future__ import annotations

import numpy as np
import torch

from .CudaWEM import _dev, _device, _hyper, _store
from .plan import Plan

__all__ = ["CudaOperator", "cuFFT2d"]


class CudaOperator:
    """Base of the device operators: holds the domain / range shapes and the
    device (the reference also creates a CUDA stream here; these operators run
    on torch's current stream)."""

    def __init__(self, model, data):
        self.domain = _hyper(model)
        self.range = _hyper(data)
        self.device = _device(model, data)


class cuFFT2d(CudaOperator):
    def __init__(self, model, data):
        super().__init__(model, data)
        shape = self.domain.shape
        if len(shape) < 2:
            raise ValueError("cuFFT2d needs at least two axes")
        if tuple(self.range.shape) != tuple(shape):
            raise ValueError("cuFFT2d: model and data shapes differ")
        self.shape = tuple(shape)
        ny, nx = shape[-2:]
        nb = int(np.prod(shape[:-2])) if len(shape) > 2 else 1
        with torch.cuda.device(self.device):
            self.plan = Plan(nx=nx, ny=ny, nw=nb, ns=1, nz=1, device=self.device)

    def forward(self, add, model, data):
        with torch.cuda.device(self.device):
            out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
            self.plan.fft2d(_dev(model, self.device), out, inverse=False, add=bool(add))
            _store(data, out)

    def adjoint(self, add, model, data):
        with torch.cuda.device(self.device):
            out = _dev(model, self.device) if add else _dev(model, self.device, zero=True)
            self.plan.fft2d(_dev(data, self.device), out, inverse=True, add=bool(add))
            _store(model, out)
