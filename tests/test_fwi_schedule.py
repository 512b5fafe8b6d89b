"""Sequencing of the FWI gradient driver (``pyfwix_b200.fwi.SmoothFWI``) on the
CPU.  The device plan is replaced by a stand-in that applies the oracle's
operators (smooth step, its adjoint and derivative, injection / recording,
reflection, correlation) to the same torch fields, rounded to complex64 as the
device stores them.  That checks the driver's storage modes -- every depth
stored, or checkpoints every k levels with segments recomputed -- against each
other and against the oracle's adjoint-state gradient without a GPU; the
device operators themselves are checked in ``test_gpu_fwi.py``."""
import numpy as np
import pytest
import torch

from oracle import wem
from pyfwix_b200 import _lib as L
from pyfwix_b200 import fwi
from tests.conftest import crandn


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _put(t, a):
    t.copy_(torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)))
    return t


@pytest.fixture(autouse=True)
def _no_shared_plans():
    """Plans of these tests (counting stand-ins) stay out of later tests' reach."""
    yield
    fwi.clear_plan_cache()


class OraclePlan:
    """The part of ``pyfwix_b200.plan.Plan`` that SmoothFWI calls, on the oracle."""

    def __init__(self, nx, ny, nw, ns, nz, dx, dy, dz, ox, oy, oz, ow, dw, padx, pady, nref, eps, taperx,
                 tapery, step, device):
        assert step == "pspi" and torch.device(device).type == "cpu"
        self.g = wem.Grid(nx=nx, ny=ny, nw=nw, nz=nz, dx=dx, dy=dy, dz=dz, ox=ox, oy=oy, oz=oz, ow=ow, dw=dw,
                          padx=padx, pady=pady, nref=nref, eps=eps, taperx=taperx, tapery=tapery)
        self.nx, self.ny, self.nw, self.ns, self.nz, self.nref = nx, ny, nw, ns, nz, nref
        self.NX, self.NY = nx + padx, ny + pady
        self.wshape = (ns, nw, self.NY, self.NX)
        self.calls = {"step": 0, "pair": 0}

    def traces(self, cx, cy, cz, ids):
        g = self.g
        return wem.make_traces(cx, cy, cz, ids, g.ox, g.oy, g.dx, g.dy, g.oz, g.dz, self.NX, self.NY)

    def ensure_workspace(self, cls=None):
        return None

    def set_smooth(self, slow_pad, sref_real):
        self.sp = slow_pad.double().numpy()
        self.refs = sref_real.double().numpy()

    def set_model(self, slow, den):
        self.s2 = np.repeat(slow.numpy().astype(np.complex128), self.nw, axis=1)
        self.den = np.repeat(den.numpy().astype(np.complex128), self.nw, axis=1)

    def inject(self, tr, iz, traces, wfld, adjoint=False, add=True):
        assert add
        if adjoint:
            _put(traces, wem.record(tr, _np(wfld), _np(traces), iz))
        else:
            _put(wfld, wem.inject(tr, _np(traces), _np(wfld), iz))

    def smooth_step(self, iz, inp, out, mode=L.SMOOTH_FWD, add=False):
        assert not add
        self.calls["step"] += 1
        f = {L.SMOOTH_FWD: wem.smooth_forward, L.SMOOTH_ADJ: wem.smooth_adjoint,
             L.SMOOTH_DERIV: wem.smooth_deriv}[mode]
        return _put(out, f(self.g, self.refs[iz], self.sp[iz], _np(inp)))

    def smooth_step_pair(self, iz, inp, out, deriv, add=False):
        assert not add and out is not deriv
        self.calls["pair"] += 1
        x = _np(inp)
        _put(deriv, wem.smooth_deriv(self.g, self.refs[iz], self.sp[iz], x))
        return _put(out, wem.smooth_forward(self.g, self.refs[iz], self.sp[iz], x)), deriv

    def reflect(self, iz, inp, out, adjoint=False, add=False):
        assert add
        f = wem.reflect_adjoint if adjoint else wem.reflect_forward
        return _put(out, f(self.g, self.s2, self.den, iz, _np(inp), _np(out)))

    def smooth_model_sweep(self, src, rec, wavelet, data, U, Ds, dSU=None):
        """The level loops of fwix_smooth_model_sweep on this stand-in's operators."""
        nz = self.nz
        data.zero_()
        Ds[0].zero_()
        for iz in range(nz):
            self.inject(src, iz, wavelet, Ds[iz])
            self.inject(rec, iz, data, Ds[iz], adjoint=True)
            if iz + 1 < nz:
                self.smooth_step(iz, Ds[iz], Ds[iz + 1])
        U.zero_()
        for iz in range(nz - 1, -1, -1):
            if iz + 1 < nz:
                if dSU is not None:
                    self.smooth_step_pair(iz, U, U, dSU[iz])
                else:
                    self.smooth_step(iz, U, U)
            self.reflect(iz, Ds[iz], U, add=True)
            self.inject(rec, iz, data, U, adjoint=True)

    def smooth_gradient_sweep(self, rec, res, Ds, dSU, mus, nu, G, gpad, crefl):
        """The level loops of fwix_smooth_gradient_sweep on this stand-in's operators."""
        nz = self.nz
        gpad.zero_()
        crefl.zero_()
        mus[0].zero_()
        for iz in range(nz):
            if iz > 0:
                self.smooth_step(iz - 1, mus[iz - 1], mus[iz], mode=L.SMOOTH_ADJ)
            self.inject(rec, iz, res, mus[iz])
            if iz + 1 < nz:
                self.correlate(mus[iz], dSU[iz], gpad[iz], add=True, padded=True)
                self.correlate(mus[iz], Ds[iz], crefl[iz], add=True, padded=False)
        nu.zero_()
        for iz in range(nz - 1, -1, -1):
            if iz + 1 < nz:
                self.smooth_step(iz, Ds[iz], G, mode=L.SMOOTH_DERIV)
                self.correlate(nu, G, gpad[iz], add=True, padded=True)
            if iz == 0:
                break
            self.smooth_step(iz, nu, nu, mode=L.SMOOTH_ADJ)
            self.reflect(iz, mus[iz], nu, adjoint=True, add=True)
            self.inject(rec, iz, res, nu)

    def correlate(self, a, b, out, add=False, padded=True):
        a, b = _np(a), _np(b)
        if not padded:
            a, b = a[:, :, :self.ny, :self.nx], b[:, :, :self.ny, :self.nx]
        c = torch.from_numpy(np.real(np.sum(np.conj(a) * b, axis=(0, 1))).astype(np.float32))
        if add:
            out += c
        else:
            out.copy_(c)
        return out


def _problem(nz=7):
    rng = np.random.default_rng(5)
    nx, ny, nw, nref = 24, 20, 4, 3
    g = wem.Grid(nx=nx, ny=ny, nw=nw, nz=nz, dx=10.0, dy=12.0, dz=10.0, ox=0.0, oy=0.0, oz=0.0, ow=3.0, dw=2.5,
                 padx=4, pady=2, nref=nref, eps=0.0, taperx=3, tapery=2)
    s = (1.0 / 1800.0) * (1 + 0.2 * rng.random((nz, ny, nx)))
    s[nz // 2:] *= 1.3
    s = s.astype(np.float32).astype(np.float64)
    refs = wem.smooth_refs(s, nref).astype(np.float32).astype(np.float64)
    geom = dict(sx=[60.0, 150.0], sy=[96.0, 120.0], sz=[0.0, 5.0], s_ids=[3, 8],
                rx=list(np.linspace(0, 230, 10)), ry=[100.0] * 10, rz=[0.0] * 5 + [12.0] * 5, r_ids=[3, 8] * 5)
    wav = crandn(rng, (2, nw))
    par = dict(dx=g.dx, dy=g.dy, dz=g.dz, ox=g.ox, oy=g.oy, oz=g.oz, ow=g.ow, dw=g.dw, nref=nref, padx=g.padx,
               pady=g.pady, eps=0.0, taperx=g.taperx, tapery=g.tapery, refs=torch.from_numpy(refs))
    acq = wem.make_acquisition(g, geom)
    d_obs = crandn(rng, (len(geom["rx"]), nw)) * 1e-3
    return g, s, refs, geom, wav, par, acq, d_obs


def _driver_gradient(monkeypatch, s, geom, wav, par, d_obs, checkpoint):
    monkeypatch.setattr(fwi, "Plan", OraclePlan)
    fwi.clear_plan_cache()  # a plan (and its step counters) of its own
    prob = fwi.SmoothFWI(s.shape, geom, torch.from_numpy(wav), dict(par, checkpoint=checkpoint), device="cpu")
    data = prob.model(torch.from_numpy(s), keep=True)
    res = data - torch.from_numpy(d_obs).to(torch.complex64)
    g = prob.gradient(res)
    return _np(data), g.double().numpy(), prob


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_every_depth_matches_oracle_gradient(monkeypatch):
    g, s, refs, geom, wav, par, acq, d_obs = _problem()
    data, grad, prob = _driver_gradient(monkeypatch, s, geom, wav, par, d_obs, None)
    assert prob.k is None
    ref_data, _, _ = wem.smooth_propagate(g, refs, s, acq, wav)
    _, ref_grad = wem.smooth_gradient(g, refs, s, acq, wav, d_obs)
    assert _rel(data, ref_data) < 1e-5
    assert _rel(grad, ref_grad) < 1e-4


@pytest.mark.parametrize("k", [2, 3, 7, 16])
def test_checkpoints_match_every_depth(monkeypatch, k):
    """k = 3 leaves a short last segment (7 levels), k = 7 makes one segment and
    k = 16 is deeper than the grid.  With every depth stored the sweeps take
    4 (nz - 1) steps and nz - 1 paired steps (down modelling; up modelling paired
    with the derivative of U; mu steps; nu and its derivative steps; no step whose
    result nothing reads); checkpoints add the recomputed segments."""
    g, s, refs, geom, wav, par, acq, d_obs = _problem()
    data0, grad0, full = _driver_gradient(monkeypatch, s, geom, wav, par, d_obs, None)
    data, grad, prob = _driver_gradient(monkeypatch, s, geom, wav, par, d_obs, k)
    assert prob.k == k
    assert _rel(data, data0) < 1e-6
    assert _rel(grad, grad0) < 1e-5
    nz = g.nz
    assert full.plan.calls["step"] == 4 * (nz - 1) and full.plan.calls["pair"] == nz - 1
    assert prob.plan.calls["step"] + prob.plan.calls["pair"] > full.plan.calls["step"] + full.plan.calls["pair"]


def test_checkpointed_step_count(monkeypatch):
    """With checkpoints every k levels the forward takes about 3 nz steps (down
    pass, and the up pass recomputing each down segment) and the backward about
    5 nz: mu alone, then per segment the down fields with their derivatives and
    the up derivatives as paired steps, the mu fields, and nu."""
    g, s, refs, geom, wav, par, acq, d_obs = _problem(nz=12)
    monkeypatch.setattr(fwi, "Plan", OraclePlan)
    fwi.clear_plan_cache()
    prob = fwi.SmoothFWI(s.shape, geom, torch.from_numpy(wav), dict(par, checkpoint=4), device="cpu")
    data = prob.model(torch.from_numpy(s), keep=True)
    fwd = dict(prob.plan.calls)
    prob.gradient(data - torch.from_numpy(d_obs).to(torch.complex64))
    bwd = {k: prob.plan.calls[k] - fwd[k] for k in fwd}
    nz = g.nz
    assert fwd["pair"] == 0 and fwd["step"] <= 3 * nz
    assert bwd["step"] + bwd["pair"] <= 5 * nz


def test_checkpoint_key():
    """An absent key means "auto"; None (and 0, 1) every depth stored."""
    assert fwi._checkpoint_key({}) == "auto"
    assert fwi._checkpoint_key({"checkpoint": None}) is None
    assert fwi._checkpoint_key({"checkpoint": 8}) == 8

    class Params:
        checkpoint = 4

    assert fwi._checkpoint_key(Params()) == 4
    assert fwi._checkpoint_key(object()) == "auto"
