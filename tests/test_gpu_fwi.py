"""The differentiable step and the FWI gradient on the device against the FP64
oracle (oracle/wem.py, smooth section): the smooth step forward / adjoint /
slowness derivative per depth (1e-5 relative L2, and its dot test), and the
adjoint-state gradient of J = 1/2 |d(s) - d_obs|^2 from full storage and from
depth checkpoints, within the 1e-3 gradient tolerance of the FP64 oracle run of
the same operator; FWIGradient's autograd backward equals that gradient."""
import numpy as np
import pytest
import torch

from oracle import wem
from tests.conftest import crandn
from tests.gpu_helpers import rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _case(nx=32, ny=24, nw=4, nz=5, nref=3, padx=4, pady=4, seed=0):
    rng = np.random.default_rng(seed)
    g = wem.Grid(nx=nx, ny=ny, nw=nw, nz=nz, dx=10.0, dy=10.0, dz=10.0, ow=6.0, dw=3.0, padx=padx, pady=pady,
                 nref=nref, taperx=3, tapery=3)
    s = (1 / 1800.0) * (1 + 0.12 * rng.random((nz, ny, nx)))
    s[nz // 2:] *= 1.25
    geom = dict(sx=np.array([150.0], np.float32), sy=np.array([110.0], np.float32), sz=np.array([0.0], np.float32),
                s_ids=np.array([0], np.int32), rx=np.linspace(0, 300, 14).astype(np.float32),
                ry=np.full(14, 120.0, np.float32), rz=np.zeros(14, np.float32), r_ids=np.zeros(14, np.int32))
    wav = crandn(rng, (1, nw))
    par = dict(nref=nref, padx=padx, pady=pady, taperx=3, tapery=3, eps=0.0, ox=0.0, oy=0.0, oz=0.0, dx=10.0,
               dy=10.0, dz=10.0, ow=6.0, dw=3.0)
    return g, rng, s, geom, wav, par


@pytest.mark.parametrize("nx,ny", [(32, 24), (60, 60)])
def test_smooth_step_modes(nx, ny):
    from pyfwix_b200 import _lib as L
    from pyfwix_b200.fwi import SmoothFWI
    g, rng, s, geom, wav, par = _case(nx=nx, ny=ny)
    prob = SmoothFWI(s.shape, geom, wav, par)
    prob.set_slowness(torch.as_tensor(s, dtype=torch.float32))
    refs = prob.refs.cpu().numpy().astype(np.float64)
    sp = wem.pad_edge(g, s.astype(np.float32).astype(np.float64))
    p = prob.plan
    x = crandn(rng, (1, g.nw, g.NY, g.NX))
    y = crandn(rng, x.shape)
    for iz in (0, 3):
        out = torch.empty_like(to_dev(x))
        got = to_host(p.smooth_step(iz, to_dev(x), out, mode=L.SMOOTH_FWD))
        assert rel(got, wem.smooth_forward(g, refs[iz], sp[iz], x)) < 1e-5
        got = to_host(p.smooth_step(iz, to_dev(y), out, mode=L.SMOOTH_ADJ))
        assert rel(got, wem.smooth_adjoint(g, refs[iz], sp[iz], y)) < 1e-5
        got = to_host(p.smooth_step(iz, to_dev(x), out, mode=L.SMOOTH_DERIV))
        assert rel(got, wem.smooth_deriv(g, refs[iz], sp[iz], x)) < 1e-5
        # dot test of the device pair
        fx = to_host(p.smooth_step(iz, to_dev(x), torch.empty_like(out)))
        ay = to_host(p.smooth_step(iz, to_dev(y), torch.empty_like(out), mode=L.SMOOTH_ADJ))
        assert abs(np.vdot(y, fx) / np.vdot(ay, x) - 1) < 1e-5


@pytest.mark.parametrize("nx,ny,pad", [(56, 60, 4), (32, 24, 4), (384, 384, 0)])
def test_smooth_step_pair(nx, ny, pad):
    """fwix_smooth_step_pair: the forward step into one buffer and its slowness
    derivative into another from one set of transforms, equal to the two separate
    steps (register-resident lengths 64 and 384 sum both weightings in one inverse
    row pass; 36 x 28 runs two generic inverse passes), in and add included."""
    from pyfwix_b200 import _lib as L
    from pyfwix_b200.fwi import SmoothFWI
    g, rng, s, geom, wav, par = _case(nx=nx, ny=ny, nw=3, padx=pad, pady=pad, nz=3)
    prob = SmoothFWI(s.shape, geom, wav, par)
    prob.set_slowness(torch.as_tensor(s, dtype=torch.float32))
    p = prob.plan
    x = to_dev(crandn(rng, (1, g.nw, g.NY, g.NX)))
    fwd = p.smooth_step(1, x, torch.empty_like(x))
    der = p.smooth_step(1, x, torch.empty_like(x), mode=L.SMOOTH_DERIV)
    out, d = torch.empty_like(x), torch.empty_like(x)
    p.smooth_step_pair(1, x, out, d)
    assert rel(to_host(out), to_host(fwd)) < 1e-6 and rel(to_host(d), to_host(der)) < 1e-6
    y = x.clone()
    p.smooth_step_pair(1, y, y, d)            # in place on the forward output
    assert rel(to_host(y), to_host(fwd)) < 1e-6
    out2, d2 = fwd.clone(), der.clone()
    p.smooth_step_pair(1, x, out2, d2, add=True)
    assert rel(to_host(out2), 2 * to_host(fwd)) < 1e-6 and rel(to_host(d2), 2 * to_host(der)) < 1e-6


@pytest.mark.parametrize("checkpoint", [None, 2])
def test_gradient_matches_oracle(checkpoint):
    from pyfwix_b200.fwi import SmoothFWI
    g, rng, s, geom, wav, par = _case()
    s = s.astype(np.float32)
    s_true = (s * (1 + 0.03 * np.exp(-((np.arange(g.nx) - 16) ** 2)[None, None, :] / 20.0))).astype(np.float32)
    prob = SmoothFWI(s.shape, geom, wav, dict(par, checkpoint=checkpoint))
    d_obs = prob.model(torch.as_tensor(s_true), keep=False)
    refs = prob.refs  # references of s_true; hold them fixed for both runs
    prob = SmoothFWI(s.shape, geom, wav, dict(par, checkpoint=checkpoint, refs=refs))
    data = prob.model(torch.as_tensor(s), keep=True)
    res = data - d_obs
    grad = prob.gradient(res).cpu().numpy()
    acq = wem.make_acquisition(g, geom)
    refs64 = refs.cpu().numpy().astype(np.float64)
    d_obs_o = wem.smooth_propagate(g, refs64, s_true.astype(np.float64), acq, wav)[0]
    J_o, grad_o = wem.smooth_gradient(g, refs64, s.astype(np.float64), acq, wav, d_obs_o)
    assert rel(to_host(data), wem.smooth_propagate(g, refs64, s.astype(np.float64), acq, wav)[0]) < 1e-4
    assert rel(grad, grad_o) < 1e-3


@pytest.mark.parametrize("checkpoint", [None, 2])
def test_interleaved_problems_share_plan_and_blocks(checkpoint):
    """Problems of the same sizes share one cached plan, its pool of stored-field
    blocks and its trace lists: interleaved model / gradient calls of two
    problems, and a second gradient call, give each problem's results alone."""
    from pyfwix_b200 import fwi
    g, rng, s, geom, wav, par = _case()
    s = s.astype(np.float32)
    sb = (s * 1.02).astype(np.float32)
    fwi.clear_plan_cache()
    prob = fwi.SmoothFWI(s.shape, geom, wav, dict(par, checkpoint=None))
    d_obs = prob.model(torch.as_tensor(s * 1.01), keep=False)
    par = dict(par, refs=prob.refs, checkpoint=checkpoint)
    del prob

    def alone(sv):
        fwi.clear_plan_cache()
        pr = fwi.SmoothFWI(s.shape, geom, wav, par)
        d = pr.model(torch.as_tensor(sv), keep=True)
        return to_host(d), to_host(pr.gradient(d - d_obs))

    da, ga = alone(s)
    db, gb = alone(sb)
    fwi.clear_plan_cache()
    A = fwi.SmoothFWI(s.shape, geom, wav, par)
    B = fwi.SmoothFWI(s.shape, geom, wav, par)
    assert A.plan is B.plan
    dA = A.model(torch.as_tensor(s), keep=True)
    dB = B.model(torch.as_tensor(sb), keep=True)
    gA = A.gradient(dA - d_obs)
    gB = B.gradient(dB - d_obs)
    gA2 = A.gradient(dA - d_obs)
    for got, ref in ((dA, da), (dB, db), (gA, ga), (gB, gb), (gA2, ga)):
        assert rel(to_host(got), ref) < 1e-6
    fwi.clear_plan_cache()


def test_sweeps_refuse_missing_fields():
    """The every-depth sweeps of the C ABI refuse missing buffers (a gradient of
    more than one level needs the up pass's derivatives) with FWIX_ERR_INVALID
    and leave the plan usable."""
    from pyfwix_b200 import _lib as L
    from pyfwix_b200 import fwi
    g, rng, s, geom, wav, par = _case(nz=3)
    prob = fwi.SmoothFWI(s.shape, geom, wav, dict(par, checkpoint=None))
    data = prob.model(torch.as_tensor(s.astype(np.float32)), keep=True)
    p = prob.plan
    dblk, ublk = prob._blocks
    f = lambda: torch.empty(p.wshape, dtype=torch.complex64, device="cuda")
    gpad = torch.empty((p.nz, p.NY, p.NX), dtype=torch.float32, device="cuda")
    crefl = torch.empty((p.nz, p.ny, p.nx), dtype=torch.float32, device="cuda")
    mus = torch.empty((p.nz,) + tuple(p.wshape), dtype=torch.complex64, device="cuda")
    with pytest.raises(RuntimeError, match="INVALID|null"):
        p.smooth_gradient_sweep(prob.rec, data, dblk, None, mus, f(), f(), gpad, crefl)
    with pytest.raises(RuntimeError, match="INVALID|null"):
        p.smooth_model_sweep(prob.src, prob.rec, prob.wavelet, data, f(), None)
    grad = prob.gradient(data - data)  # zero residual: zero gradient, plan still usable
    assert float(grad.abs().max()) == 0.0
    fwi.clear_plan_cache()


def test_autograd_function():
    from pyfwix_b200.fwi import FWIGradient, SmoothFWI
    g, rng, s, geom, wav, par = _case(nz=4)
    s = s.astype(np.float32)
    prob = SmoothFWI(s.shape, geom, wav, par)
    d_obs = prob.model(torch.as_tensor(s * 1.01), keep=False)
    par = dict(par, refs=prob.refs)
    st = torch.as_tensor(s, device="cuda").requires_grad_(True)
    J = FWIGradient.apply(st, torch.as_tensor(wav).cuda(), geom, d_obs, par)
    J.backward()
    acq = wem.make_acquisition(g, geom)
    refs64 = prob.refs.cpu().numpy().astype(np.float64)
    J_o, grad_o = wem.smooth_gradient(g, refs64, s.astype(np.float64), acq, wav, to_host(d_obs))
    assert abs(float(J.detach()) / J_o - 1) < 1e-4
    assert rel(st.grad.cpu().numpy(), grad_o) < 1e-3


def test_propagator_s_real_and_smooth_mode():
    """Propagator shortcuts: ``s_real`` stands for the model [s^2, 1] (same data
    as passing that model), and ``mode="smooth"`` models with the differentiable
    step (the FP64 oracle's smooth modelling with the same references)."""
    from pyfwix_b200 import CudaWEM
    g, rng, s, geom, wav, par = _case()
    s = s.astype(np.float32)
    # the receivers lie on one line y = 120 m: an aperture (ginsu) that covers the
    # model keeps the parity runs from windowing the model down to two rows
    par = dict(par, ginsu_x=1e4, ginsu_y=1e4)
    d1 = np.zeros((len(geom["rx"]), g.nw), np.complex64)
    p1 = CudaWEM.Propagator(None, d1, wav, par, geom, s_real=s)
    p1.forward(False, None, d1)
    model = CudaWEM.slowness_model(s)
    d2 = np.zeros_like(d1)
    p2 = CudaWEM.Propagator(model, d2, wav, par, geom)
    p2.forward(False, model, d2)
    assert np.abs(d1).max() > 0 and rel(d1, d2) < 1e-6
    d3 = np.zeros_like(d1)
    p3 = CudaWEM.Propagator(None, d3, wav, par, geom, mode="smooth", s_real=s)
    p3.forward(False, None, d3)
    refs64 = p3._smooth.refs.cpu().numpy().astype(np.float64)
    acq = wem.make_acquisition(g, geom)
    ref = wem.smooth_propagate(g, refs64, s.astype(np.float64), acq, wav)[0]
    assert rel(d3, ref) < 1e-4
    d4 = d3.copy()
    p3.forward(True, None, d4)   # add
    assert rel(d4, 2 * ref) < 1e-4
    with pytest.raises(ValueError):
        CudaWEM.Propagator(None, d1, wav, par, geom, mode="bogus", s_real=s)
