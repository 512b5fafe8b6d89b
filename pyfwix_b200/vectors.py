"""Hypercubes and vectors for the operator surface.

The reference's Python surface passes SEP vectors (``pyVector`` /
``SepVector``): an array plus a hypercube whose axes are listed fastest first,
each with ``n``, origin ``o`` and sampling ``d`` (``fwix/CudaWEM.py:7-157`` reads
them through ``getHyper()``).  Those packages are not part of this library, so
this module gives the same shape of object on top of a torch tensor:

* :class:`Axis` and :class:`Hypercube` (``getAxis(i)`` is 1-based and counts
  from the fastest axis, ``getNdim()``, ``getN123()``, ``checkSame()``);
* :class:`Vector`: a complex64 torch tensor in numpy order (slowest axis first)
  with its hypercube and the vector operations the reference's callers use
  (``clone``, ``cloneSpace``, ``zero``, ``dot``, ``scaleAdd``, ``norm``);
* :class:`SuperVector`: a list of vectors (the ``[s^2, density]`` model).

The operators also accept bare torch tensors and numpy arrays; their axes then
come from the ``par`` keys ``ox, dx, oy, dy, oz, dz, ow, dw``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch


@dataclass(frozen=True)
class Axis:
    n: int
    o: float = 0.0
    d: float = 1.0
    label: str = ""


class Hypercube:
    """Axes fastest first, as in SEP: a [nz][nw][ny][nx] array has axes (x, y, w, z)."""

    def __init__(self, axes):
        self.axes = [a if isinstance(a, Axis) else Axis(*a) for a in axes]

    @classmethod
    def from_shape(cls, shape):
        """Unit-sampled axes for a numpy-order shape."""
        return cls([Axis(int(n)) for n in reversed(tuple(shape))])

    def getAxis(self, i):
        return self.axes[i - 1]

    def getAxes(self):
        return list(self.axes)

    def getNdim(self):
        return len(self.axes)

    def getN123(self):
        return int(np.prod([a.n for a in self.axes]))

    @property
    def shape(self):
        """numpy-order shape (slowest axis first)."""
        return tuple(a.n for a in reversed(self.axes))

    def checkSame(self, other, tol=1e-6):
        if len(self.axes) != len(other.axes):
            return False
        for a, b in zip(self.axes, other.axes):
            if a.n != b.n or abs(a.o - b.o) > tol * max(1.0, abs(a.o)) or abs(a.d - b.d) > tol * max(1.0, abs(a.d)):
                return False
        return True

    def __repr__(self):
        return "Hypercube(" + ", ".join(f"n={a.n} o={a.o} d={a.d}" for a in self.axes) + ")"


def _as_tensor(x, device=None, dtype=torch.complex64):
    t = torch.as_tensor(x)
    if dtype.is_complex and not t.is_complex():
        t = t.to(torch.float32)
    return t.to(device=device if device is not None else t.device, dtype=dtype)


class Vector:
    """A complex64 tensor (numpy order) with its hypercube."""

    def __init__(self, hyper_or_array, arr=None, device=None, dtype=torch.complex64):
        if isinstance(hyper_or_array, Hypercube):
            self.hyper = hyper_or_array
            if arr is None:
                arr = torch.zeros(self.hyper.shape, dtype=dtype, device=device or "cpu")
        else:
            arr = hyper_or_array if arr is None else arr
            self.hyper = Hypercube.from_shape(np.shape(arr))
        self.arr = _as_tensor(arr, device, dtype).contiguous()
        if tuple(self.arr.shape) != self.hyper.shape:
            raise ValueError(f"array shape {tuple(self.arr.shape)} does not match {self.hyper}")

    # hypercube access in the reference's spelling
    def getHyper(self):
        return self.hyper

    @property
    def shape(self):
        return tuple(self.arr.shape)

    def getNdArray(self):
        return self.arr.cpu().numpy()

    def clone(self):
        return Vector(self.hyper, self.arr.clone())

    def cloneSpace(self):
        return Vector(self.hyper, torch.zeros_like(self.arr))

    def zero(self):
        self.arr.zero_()
        return self

    def scale(self, sc):
        self.arr.mul_(sc)
        return self

    def scaleAdd(self, other, sc1=1.0, sc2=1.0):
        """self = sc1 * self + sc2 * other."""
        self.arr.mul_(sc1).add_(_as_tensor(_arr(other), self.arr.device, self.arr.dtype), alpha=sc2)
        return self

    def dot(self, other):
        """sum conj(self) * other (complex)."""
        o = _as_tensor(_arr(other), self.arr.device, self.arr.dtype)
        return complex(torch.vdot(self.arr.reshape(-1), o.reshape(-1)).item())

    def norm(self):
        return float(torch.linalg.vector_norm(self.arr))

    def __repr__(self):
        return f"Vector({self.hyper}, device={self.arr.device})"


class SuperVector:
    """A list of vectors operated on together (the reference's ``superVector``)."""

    def __init__(self, *vecs):
        if len(vecs) == 1 and isinstance(vecs[0], (list, tuple)):
            vecs = tuple(vecs[0])
        self.vecs = [v if isinstance(v, Vector) else Vector(v) for v in vecs]

    def clone(self):
        return SuperVector([v.clone() for v in self.vecs])

    def cloneSpace(self):
        return SuperVector([v.cloneSpace() for v in self.vecs])

    def zero(self):
        for v in self.vecs:
            v.zero()
        return self

    def dot(self, other):
        return sum(a.dot(b) for a, b in zip(self.vecs, _vecs(other)))

    def scaleAdd(self, other, sc1=1.0, sc2=1.0):
        for a, b in zip(self.vecs, _vecs(other)):
            a.scaleAdd(b, sc1, sc2)
        return self

    def norm(self):
        return float(np.sqrt(sum(v.norm() ** 2 for v in self.vecs)))

    def __getitem__(self, i):
        return self.vecs[i]

    def __len__(self):
        return len(self.vecs)


def _arr(x):
    return x.arr if isinstance(x, Vector) else x


def _vecs(x):
    return x.vecs if isinstance(x, SuperVector) else list(x)
