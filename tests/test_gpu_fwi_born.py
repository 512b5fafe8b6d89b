"""The FWI gradient (``pyfwix_b200.fwi``) tied to the reference's gradient
operator, ExtendedBorn::adjoint (``propagator/src/ExtendedBorn.cpp:122-150``,
called as the gradient in ``fwix/workers.py:62-76``), and checked by central
finite differences on the device.

How the two operators relate.  ExtendedBorn linearises the PSPI modelling in
s^2 per frequency; its gradient with respect to a real, frequency-independent
slowness s is g_s = 2 s sum_w Re g_{s^2}[w].  FWIGradient differentiates the
smooth step's modelling in s.  Both linearise the same Propagator
(``propagator/src/Propagator.cpp:121-221``), but discretise the scattering
differently:

* ExtendedBorn scatters before the step, S(W u ds^2) (``Scattering.cpp:43-52``);
  the smooth step's derivative multiplies after it, -i w dz ds S(u);
* its up scattering takes the perturbation of the level a step leaves
  (``ExtendedBorn.cpp:282-311``), the smooth model that of the level it reaches;
* its linearised reflection carries a factor sqrt(s0 / s1) that the derivative
  of r = (s0 - s1) / (s0 + s1) does not (``lin_reflect.cu:48-92``);
* its Taylor terms beyond the first and eps_scat are not in the split-step
  derivative.

All four differences vanish in a homogeneous background with one reference
(the smooth step is then the PSPI step; no reflection, so no up-going
background), Taylor order 0, eps_scat 0, no taper (the reference's scattering
adjoint omits the taper, ``PSPI.cpp:26-44``), and for perturbations constant
over each depth level (multiplying before or after the step is then the same).
There the two gradients' sums over each depth level must agree for any data
residual: the first test below.  The fields themselves differ by where the
scattering sits inside the step.
"""
import numpy as np
import pytest
import torch

from tests.conftest import crandn
from tests.gpu_helpers import rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _homogeneous(nz=6, n=64, nw=8):
    s = np.float32(1 / 2000.0)
    dx = dz = 10.0
    gx, gy = np.meshgrid(np.arange(4, n - 4, 6) * dx, np.arange(4, n - 4, 6) * dx)
    nr = gx.size
    geom = dict(sx=np.array([n // 2 * dx], np.float32), sy=np.array([n // 2 * dx], np.float32),
                sz=np.array([0.0], np.float32), s_ids=np.array([0], np.int32),
                # receivers on the surface and on level 3 (all on grid nodes)
                rx=np.concatenate([gx.ravel(), gx.ravel()]).astype(np.float32),
                ry=np.concatenate([gy.ravel(), gy.ravel()]).astype(np.float32),
                rz=np.concatenate([np.zeros(nr), np.full(nr, 3 * dz)]).astype(np.float32),
                r_ids=np.zeros(2 * nr, np.int32))
    par = dict(nref=1, padx=0, pady=0, taperx=0, tapery=0, eps=0.0, ox=0.0, oy=0.0, oz=0.0, dx=dx, dy=dx,
               dz=dz, ow=4.0, dw=3.0, checkpoint=None)
    return s, geom, par, (nz, n, n), nw


def test_fwi_gradient_ties_to_born_adjoint():
    from pyfwix_b200.fwi import SmoothFWI
    from pyfwix_b200.plan import Plan
    s, geom, par, shape, nw = _homogeneous()
    nz, ny, nx = shape
    rng = np.random.default_rng(77)
    wav = torch.as_tensor(crandn(rng, (1, nw)).astype(np.complex64)).cuda()
    sfield = torch.full(shape, float(s), dtype=torch.float32)
    refs = torch.full((nz, 1), float(s), dtype=torch.float32)
    prob = SmoothFWI(shape, geom, wav, dict(par, refs=refs))
    d_smooth = prob.model(sfield, keep=True)
    ntr = len(geom["rx"])
    r = torch.as_tensor(crandn(rng, (ntr, nw)).astype(np.complex64)).cuda()
    g_fwi = prob.gradient(r).double().cpu().numpy()

    # the reference's Born on the same modelling: PSPI, one reference per depth
    p = Plan(nx=nx, ny=ny, nw=nw, ns=1, nz=nz, dx=par["dx"], dy=par["dy"], dz=par["dz"], ow=par["ow"],
             dw=par["dw"], nref=1, taperx=0, tapery=0, eps_scat=0.0, taylor=0, step="pspi")
    s2 = (torch.full((nz, 1, ny, nx), float(s), dtype=torch.float64) ** 2).to(torch.complex64)
    p.set_refs(s2[:, :, :1, :1].reshape(nz, 1, 1).expand(nz, 1, nw), torch.zeros((nz, 1, ny, nx), dtype=torch.uint8))
    p.set_model(s2, torch.ones_like(s2))
    src = p.traces(geom["sx"], geom["sy"], geom["sz"], geom["s_ids"])
    rec = p.traces(geom["rx"], geom["ry"], geom["rz"], geom["r_ids"])
    bd = torch.empty((nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d_pspi = torch.empty((ntr, nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, wav, d_pspi, bd, bu)
    # one reference at the local slowness: the smooth step is the PSPI step
    assert float(torch.abs(d_smooth).max()) > 0
    assert rel(to_host(d_smooth), to_host(d_pspi)) < 1e-5
    gs2 = torch.empty((nz, 1, ny, nx), dtype=torch.complex64, device="cuda")
    gr = torch.empty_like(gs2)
    p.born(rec, bd, bu, gs2, gr, r, adjoint=True)
    g_born = (2 * float(s) * to_host(gs2)[:, 0].real)
    sums_fwi = g_fwi.sum(axis=(1, 2))
    sums_born = g_born.sum(axis=(1, 2))
    assert np.abs(sums_born).max() > 0
    assert rel(sums_fwi, sums_born) < 1e-4, (sums_fwi, sums_born)
    # the linearisations agree, the fields do not: scattering before the step
    # (Born) and after it (smooth) put the same sum at different places
    assert rel(g_fwi, g_born) > 1e-3


def test_fwi_gradient_central_differences_on_device():
    """The central finite-difference check of the FWI configuration, on the
    device: 384 x 384 x 96 frequencies, three levels through the first anomaly,
    h = 1e-3 relative.  A single cell moves the FP32 objective by less than its
    rounding, so each of the 16 random cells is the centre of a Gaussian
    perturbation (sigma 16 cells on its level); (J(s + h ds) - J(s - h ds)) / 2h
    must equal <dJ/ds, ds> from the adjoint-state gradient."""
    from pyfwix_b200 import workloads
    from pyfwix_b200.fwi import SmoothFWI
    w, s_true, s0 = workloads.config4()
    z0 = int(np.argmax(np.abs(s_true - s0).sum(axis=(1, 2)))) - 1
    s_true = np.ascontiguousarray(s_true[z0:z0 + 3])
    s0 = np.ascontiguousarray(s0[z0:z0 + 3])
    w.oz, w.nz = z0 * w.dz, 3
    # the receivers off the source's cells: there the data are the reflections
    # alone, whose change with s stands far above the FP32 rounding of the data
    # (with the direct arrival recorded, d(s + h ds) - d(s - h ds) would keep few
    # of its digits)
    g0 = w.geom
    far = (g0["rx"] - g0["sx"][0]) ** 2 + (g0["ry"] - g0["sy"][0]) ** 2 > (4 * w.dx) ** 2
    geom = dict(g0, sz=np.full(1, w.oz, np.float32), rx=g0["rx"][far], ry=g0["ry"][far],
                rz=np.full(int(far.sum()), w.oz, np.float32), r_ids=g0["r_ids"][far])
    par = dict(nref=w.nref, padx=0, pady=0, taperx=w.taperx, tapery=w.tapery, eps=0.0, ox=w.ox, oy=w.oy,
               oz=w.oz, dx=w.dx, dy=w.dy, dz=w.dz, ow=w.ow, dw=w.dw, checkpoint=None)
    wav = torch.as_tensor(w.wavelet).cuda()
    # Fixed references with the starting slowness inside one interval, 2 % from
    # either end: the smooth step is piecewise linear in s between references,
    # so J has kinks at the reference values, and a central difference across
    # one averages two slopes.  The starting model is laterally constant on a
    # level and is an end of the true model's range (the references
    # smooth_refs would take), so every cell would sit on a kink.
    lev = s0.mean(axis=(1, 2)).astype(np.float64)
    refs = torch.as_tensor(lev[:, None] * (1 + np.array([-0.06, -0.02, 0.02, 0.06]))[None, :],
                           dtype=torch.float32).cuda()
    assert w.nref == refs.shape[1] and np.allclose(s0, lev[:, None, None])
    prob = SmoothFWI(s_true.shape, geom, wav, dict(par, refs=refs))
    # J = 1/2 |d(s)|^2 (observed data zero).  Against data of the true model the
    # residual over three levels is small while a perturbation near the source
    # changes the data strongly: the curvature of J (which needs no residual)
    # then outweighs its slope for any h FP32 resolves (in FP64, fd - ad at the
    # source-side bump falls as h^2, 1.4e-8 -> 1.5e-10 -> 2.5e-12 against
    # ad = -1.1e-12 for h = 1e-2, 1e-3, 1e-4).  The gradient's formula does not
    # depend on the data, and with the data as residual the slope dominates.
    d_obs = torch.zeros((int(far.sum()), w.nw), dtype=torch.complex128, device="cuda")
    s0t = torch.as_tensor(s0, dtype=torch.float64)
    data = prob.model(s0t.float(), keep=True)
    grad = prob.gradient(data - d_obs.to(torch.complex64)).double().cpu()

    def objective(s):
        res = prob.model(s.float(), keep=False).to(torch.complex128) - d_obs
        return 0.5 * float(torch.sum(res.real ** 2 + res.imag ** 2))

    rng = np.random.default_rng(1003)
    ny, nx = s0.shape[1:]
    yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    h = 1e-3
    fd, ad, at = [], [], []
    for _ in range(16):
        iz, iy, ix = int(rng.integers(0, 2)), int(rng.integers(24, ny - 24)), int(rng.integers(24, nx - 24))
        bump = np.zeros(s0.shape)
        bump[iz] = np.exp(-((yy - iy) ** 2 + (xx - ix) ** 2) / (2 * 16.0 ** 2))
        ds = s0t * torch.as_tensor(bump)
        fd.append((objective(s0t + h * ds) - objective(s0t - h * ds)) / (2 * h))
        ad.append(float(torch.sum(grad * ds)))
        at.append((iz, iy, ix))
    fd, ad = np.array(fd), np.array(ad)
    err = np.abs(fd - ad) / np.abs(ad).max()
    k = int(np.argmax(err))
    assert np.abs(ad).max() > 0
    assert err.max() < 1e-2, ("worst", at[k], fd[k], ad[k], err[k], "source", g0["sx"][0] / w.dx, g0["sy"][0] / w.dy)
    assert rel(fd, ad) < 1e-2, (fd, ad)
