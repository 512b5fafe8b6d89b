"""Loads a reference-kernel fixture (tests/golden/reference_kernels_<regime>.npz,
made by tests/golden/make_golden.py from pyfwix's own CUDA kernels) and the
oracle grid that matches it."""
import ast
import os

import numpy as np

from oracle import wem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REGIMES = ("real", "complex")


def load(regime):
    path = os.path.join(GOLDEN, f"reference_kernels_{regime}.npz")
    if not os.path.exists(path):
        return None
    f = np.load(path)
    gd = ast.literal_eval(str(f["grid"]))
    g = wem.Grid(nx=gd["nx"], ny=gd["ny"], nw=gd["nw"], nz=2, dx=gd["dx"], dy=gd["dy"], dz=gd["dz"],
                 ox=gd["ox"], oy=gd["oy"], oz=gd["oz"], ow=gd["ow"], dw=gd["dw"], padx=gd["padx"],
                 pady=gd["pady"], nref=gd["nref"], eps=gd["eps"], taperx=gd["taperx"], tapery=gd["tapery"],
                 eps_scat=gd["eps_scat"], taylor=int(f["taylor"]))
    return g, gd, {k: f[k] for k in f.files}


def c128(a):
    return np.asarray(a).astype(np.complex128)
