"""Helpers shared by the GPU parity tests: build matching oracle grids and
device plans from one set of seeded inputs."""
import numpy as np
import torch

from oracle import wem
from tests.conftest import crandn


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def to_dev(x):
    return torch.as_tensor(np.ascontiguousarray(x)).to("cuda").to(torch.complex64)


def to_host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.complex128)


def make_case(seed=0, nx=24, ny=20, nw=5, nz=5, ns=2, padx=0, pady=0, nref=3, eps=0.0,
              taperx=3, tapery=2, taylor=1, complex_refs=False, labels_per_w=True):
    """Seeded grid, references, labels and model for the oracle and the device."""
    rng = np.random.default_rng(seed)
    g = wem.Grid(nx=nx, ny=ny, nw=nw, nz=nz, dx=10.0, dy=12.0, dz=10.0, ox=0.0, oy=0.0, oz=0.0,
                 ow=3.0, dw=2.5, padx=padx, pady=pady, nref=nref, eps=eps, taperx=taperx,
                 tapery=tapery, taylor=taylor)
    s0 = (1.0 / 1800.0) ** 2
    sref = np.empty((nz, nref, nw), dtype=np.complex128)
    for r in range(nref):
        sref[:, r, :] = s0 * (1.0 + 0.15 * r) * (1 + 0.02 * rng.random((nz, 1)))
    if complex_refs:
        sref = sref + 1j * s0 * 0.05 * rng.standard_normal(sref.shape)
    lw = nw if labels_per_w else 1
    labels = rng.integers(0, nref, size=(nz, lw, g.NY, g.NX))
    slow = s0 * (1 + 0.3 * rng.random((nz, nw, ny, nx))) + 1j * s0 * 0.01 * rng.standard_normal((nz, nw, ny, nx))
    den = 1.0 + 0.4 * rng.random((nz, nw, ny, nx)) + 0j
    return g, rng, sref, labels, slow, den


def make_plan(g, ns, sref, labels, slow=None, den=None, step="pspi"):
    from pyfwix_b200.plan import Plan
    p = Plan(nx=g.nx, ny=g.ny, nw=g.nw, ns=ns, nz=g.nz, dx=g.dx, dy=g.dy, dz=g.dz, ox=g.ox,
             oy=g.oy, oz=g.oz, ow=g.ow, dw=g.dw, padx=g.padx, pady=g.pady, nref=g.nref, eps=g.eps,
             taperx=g.taperx, tapery=g.tapery, eps_scat=g.eps_scat, taylor=g.taylor, step=step)
    p.set_refs(sref, labels)
    if slow is not None:
        p.set_model(slow, den)
    return p


def oracle_labels(labels, g):
    """Expand [nz][1][NY][NX] labels to the per-frequency layout of the oracle."""
    if labels.shape[1] == 1:
        return np.repeat(labels, g.nw, axis=1)
    return labels


def wavefield(rng, ns, g):
    return crandn(rng, (ns, g.nw, g.NY, g.NX))
