"""Parity at the benchmark configurations' sizes.  Each case runs the device path
on a slab of a few depth levels at the configuration's full lateral size and
full frequency count, against the FP64 oracle (``oracle/wem.py``) on the same
inputs: the seeded model of ``pyfwix_b200.workloads``, the reference slownesses
and labels of ``pyfwix_b200.refsampler`` (checked against ``oracle/refs.py``
first), the same acquisition.  Slabs are placed where the model varies
laterally (at the Gaussian anomalies), with the source and receivers on the
slab's top level.

* 128 x 128, 64 frequencies, PSPI nref 4: modelling and migration
  (``propagator/src/Propagator.cpp:121-221``, the lockstep image);
* 256 x 256, 128 frequencies, NSPS nref 4: ExtendedBorn forward and adjoint
  (``propagator/src/ExtendedBorn.cpp:80-453``) and their dot test;
* two shots of the 32-shot batch, 320 x 320 and 384 x 384 with their own bands
  of 48-160 frequencies, PSPI nref 6: migration images through ``fwix_sweep``;
* 384 x 384, 96 frequencies: the autograd FWI gradient, every depth stored and
  from depth checkpoints;
* Born on the register-resident lengths 320, 384 and 640 (small frequency
  counts).

Tolerances (relative L2): data, images and Born outputs 1e-4, gradients 1e-3.
The oracle runs band by band over frequency in worker processes
(``tests/oracle_bands.py``), which gives the same numbers as one run.
"""
import numpy as np
import pytest
import torch

from oracle import refs as oracle_refs
from oracle import wem
from tests import oracle_bands
from tests.conftest import crandn
from tests.gpu_helpers import rel, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL = 1e-4
GTOL = 1e-3


# ----------------------------------------------------------------------------- helpers

def slab(w, z0, nz):
    """The workload restricted to depth levels z0 .. z0 + nz - 1, with the source
    and receivers moved to the slab's top level."""
    w.oz = w.oz + z0 * w.dz
    w.nz = nz
    if w.slow2 is not None and w.anomaly is None and getattr(w, "layers", None) is None:
        w.slow2 = np.ascontiguousarray(w.slow2[z0:z0 + nz])
    g = dict(w.geom)
    g["sz"] = np.full_like(np.asarray(g["sz"], np.float32), w.oz)
    g["rz"] = np.full_like(np.asarray(g["rz"], np.float32), w.oz)
    w.geom = g
    return w


def grid(w):
    return wem.Grid(nx=w.nx, ny=w.ny, nw=w.nw, nz=w.nz, dx=w.dx, dy=w.dy, dz=w.dz, ox=w.ox, oy=w.oy, oz=w.oz,
                    ow=w.ow, dw=w.dw, padx=w.padx, pady=w.pady, nref=w.nref, eps=w.eps, taperx=w.taperx,
                    tapery=w.tapery, eps_scat=w.eps_scat, taylor=w.taylor)


def refs_on_device(w, s2):
    """Reference slownesses and labels of s2 [nz][1][ny][nx] (device), checked
    against the oracle's restatement of the rule."""
    from pyfwix_b200 import refsampler
    sref, labels = refsampler.sample(s2, w.nref, w.padx, w.pady)
    sref_o, lab_o = oracle_refs.sample(s2.double().cpu().numpy(), w.nref, w.padx, w.pady)
    assert np.allclose(sref.cpu().numpy(), sref_o, rtol=1e-6, atol=0)
    # Labels: the nearest reference.  A cell that lies (to float32 rounding)
    # halfway between two references, or at two equal references (the quantiles
    # of a layered level repeat), may take either; any other must agree.
    lab = labels.cpu().numpy().astype(np.int64)
    ny, nx = s2.shape[-2:]
    x = s2.double().cpu().numpy()                                        # [nz][1][ny][nx]
    c = np.asarray(sref_o).real[:, :, 0]                                 # [nz][nref]
    pick = lambda l: np.take_along_axis(c[:, None, None, None, :], l[..., None], axis=-1)[..., 0]
    dev, ora = lab[..., :ny, :nx], lab_o[..., :ny, :nx]
    gap = np.abs(x - pick(dev)) - np.abs(x - pick(ora))
    assert np.all(gap <= 1e-6 * np.abs(x)), gap.max()
    assert np.array_equal(lab[..., ny:, :], lab[..., ny - 1:ny, :].repeat(lab.shape[-2] - ny, axis=-2))
    return refsampler.expand_refs(sref, w.nw), labels


class Case:
    """Device plan and oracle inputs of one single-shot workload."""

    def __init__(self, w, step=None):
        from pyfwix_b200 import workloads
        from pyfwix_b200.plan import Plan
        self.w = w
        kw = w.plan_kwargs()
        if step:
            kw["step"] = step
        self.kind = kw["step"]
        self.s2 = workloads.slow2_on(w, "cuda")[:, None].contiguous()         # [nz][1][ny][nx]
        self.sref, self.labels = refs_on_device(w, self.s2)
        self.p = Plan(ns=1, device="cuda", **kw)
        self.p.set_refs(self.sref, self.labels)
        s2c = self.s2.to(torch.complex64)
        self.p.set_model(s2c, torch.ones_like(s2c))
        g = w.geom
        ids = lambda n: np.zeros(n, np.int32)
        self.src = self.p.traces(g["sx"], g["sy"], g["sz"], ids(len(g["sx"])))
        self.rec = self.p.traces(g["rx"], g["ry"], g["rz"], ids(len(g["rx"])))
        self.ntr = len(g["rx"])
        self.wav = torch.as_tensor(w.wavelet).cuda()
        # oracle side: the same values in FP64 (frequency-independent model and labels)
        self.g = grid(w)
        self.args = dict(geom=w.geom, kind=self.kind, s2=self.s2[:, 0].double().cpu().numpy(),
                         labels=self.labels[:, 0].cpu().numpy(),
                         sref=self.sref.cpu().numpy().astype(np.complex128),
                         wavelet=w.wavelet.astype(np.complex128))

    def oracle(self, task, **extra):
        return oracle_bands.run(task, self.g, dict(self.args, **extra))

    def model(self, keep_up=True):
        p, w = self.p, self.w
        bd = torch.empty((w.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
        bu = torch.empty_like(bd) if keep_up else None
        data = torch.empty((self.ntr, w.nw), dtype=torch.complex64, device="cuda")
        p.propagate(self.src, self.rec, self.wav, data, bd, bu)
        return data, bd, bu


# ----------------------------------------------------------------------------- configurations

def test_config1_modelling_and_migration():
    """128 x 128 x 64 frequencies (2-30 Hz), PSPI nref 4, taper 20: levels 48-51,
    through the +10 % anomaly centred at 500 m."""
    from pyfwix_b200 import workloads
    w = workloads.config1(nz=100)
    w.anomaly = (640.0, 640.0, 500.0)       # the configuration's anomaly, evaluated on the slab's levels
    c = Case(slab(w, 48, 4))
    assert len(np.unique(c.labels.cpu().numpy())) == w.nref
    data, bd, _ = c.model(keep_up=False)
    img = torch.zeros((w.nz, w.ny, w.nx), dtype=torch.float32, device="cuda")
    c.p.migrate(c.src, c.rec, c.wav, data, img)
    torch.cuda.synchronize()
    o = c.oracle("model")
    assert rel(to_host(data), o["data"]) < TOL
    assert rel(to_host(bd), o["bgd"]) < TOL
    o = c.oracle("migrate", data=to_host(data))
    assert rel(img.cpu().numpy(), o["image"]) < TOL


def test_config2_born_forward_adjoint():
    """256 x 256 x 128 frequencies (3-40 Hz), NSPS nref 4, taper 20, levels 0-2 of
    the smooth random model; reflectivity: the configuration's seeded layer
    amplitudes placed on the slab's levels; adjoint of seeded random data."""
    from pyfwix_b200 import workloads
    w = slab(workloads.config2(nz=3), 0, 3)
    c = Case(w)
    rng = np.random.default_rng(1001)
    amps = rng.uniform(-0.1, 0.1, size=w.nz)
    ds = (amps[:, None, None] * w.slow2)[:, None].astype(np.complex64)           # [nz][1][ny][nx]
    _, bd, bu = c.model()
    data = torch.empty((c.ntr, w.nw), dtype=torch.complex64, device="cuda")
    dden = torch.zeros(ds.shape, dtype=torch.complex64, device="cuda")
    c.p.born(c.rec, bd, bu, to_dev(ds), dden, data)
    r = crandn(rng, (c.ntr, w.nw)).astype(np.complex64)
    gs = torch.empty(ds.shape, dtype=torch.complex64, device="cuda")
    gr = torch.empty_like(gs)
    c.p.born(c.rec, bd, bu, gs, gr, to_dev(r), adjoint=True)
    o = c.oracle("born", ds=ds[:, 0], dr=np.zeros_like(ds[:, 0]), r=r)
    assert rel(to_host(data), o["born"]) < TOL
    # the frequency-broadcast model's adjoint is the sum over frequency
    assert rel(to_host(gs)[:, 0], o["gs"]) < TOL
    assert rel(to_host(gr)[:, 0], o["gr"]) < TOL
    # dot test on the device: <r, B m> = <B^T r, m>
    lhs = np.vdot(r.astype(np.complex128).ravel(), to_host(data).ravel())
    rhs = np.vdot(to_host(gs).ravel(), ds.astype(np.complex128).ravel())
    assert abs(lhs / rhs - 1) < 1e-4


def _config3_shot(n):
    from pyfwix_b200 import workloads
    ws = workloads.config3(nshots=32, nz=200)
    w = next(x for x in ws if x.nx == n)
    # the slab sits on the shot's own anomaly depth
    z0 = int(round((w.anomaly[2] - w.oz) / w.dz)) - 1
    return slab(w, z0, 3)


def test_config3_shots_migration():
    """Two shots of the batch -- 320 x 320 and 384 x 384, each with its own band of
    48-160 frequencies, PSPI nref 6, taper 20 -- imaged together through
    fwix_sweep on two streams; every image against the oracle's migration of the
    same data (the shot's modelled data)."""
    from pyfwix_b200 import _lib as L
    from pyfwix_b200.plan import sweep
    cases = [Case(_config3_shot(n)) for n in (320, 384)]
    assert all(48 <= c.w.nw <= 160 for c in cases)
    insts, datas = [], []
    for c in cases:
        data, _, _ = c.model(keep_up=False)
        datas.append(data)
        c.img = torch.zeros((c.w.nz, c.w.ny, c.w.nx), dtype=torch.float32, device="cuda")
        c.p.ensure_workspace(L.WS_SWEEP)
        insts.append(dict(plan=c.p, src=c.src, rec=c.rec, wavelet=c.wav, data=data, image=c.img))
    streams = [torch.cuda.Stream() for _ in range(2)]
    sweep(L.SWEEP_IMAGE, insts, streams)
    torch.cuda.synchronize()
    for c, data in zip(cases, datas):
        o = c.oracle("migrate", data=to_host(data))
        assert rel(to_host(data), o["data"]) < TOL
        assert rel(c.img.cpu().numpy(), o["image"]) < TOL, (c.w.name, rel(c.img.cpu().numpy(), o["image"]))


def test_config4_fwi_gradient():
    """384 x 384 x 96 frequencies (3-30 Hz), the smooth PSPI step with nref 4: three
    levels through the first +-8 % anomaly; true model with the anomalies,
    starting model the background; gradient of J against the oracle's
    adjoint-state gradient, every depth stored and from checkpoints every 2
    levels."""
    from pyfwix_b200 import workloads
    from pyfwix_b200.fwi import SmoothFWI
    w, s_true, s0 = workloads.config4()
    dev = np.abs(s_true - s0).sum(axis=(1, 2))
    z0 = int(np.argmax(dev)) - 1
    w = slab(w, z0, 3)
    s_true = np.ascontiguousarray(s_true[z0:z0 + 3])
    s0 = np.ascontiguousarray(s0[z0:z0 + 3])
    par = dict(nref=w.nref, padx=0, pady=0, taperx=w.taperx, tapery=w.tapery, eps=0.0, ox=w.ox, oy=w.oy,
               oz=w.oz, dx=w.dx, dy=w.dy, dz=w.dz, ow=w.ow, dw=w.dw)
    wav = torch.as_tensor(w.wavelet).cuda()
    prob = SmoothFWI(s_true.shape, w.geom, wav, dict(par, checkpoint=None))
    prob.set_slowness(torch.as_tensor(s_true))
    refs = prob.refs.clone()
    d_obs_o, _, grad_o, data_o = oracle_bands.run("smooth", grid(w), dict(
        geom=w.geom, refs=refs.cpu().numpy().astype(np.float64), s_true=s_true.astype(np.float64),
        s0=s0.astype(np.float64), wavelet=w.wavelet.astype(np.complex128)))
    # Over three levels the data of both models are the same direct arrival up to
    # small reflections, so d(s0) - d_obs keeps only a few of the FP32 digits of
    # either.  The residual is therefore checked on the data's scale, and the
    # gradient (linear in the residual) is taken of the oracle's FP64 residual.
    res_o = data_o - d_obs_o
    res_dev = torch.as_tensor(res_o.astype(np.complex64)).cuda()
    for checkpoint in (None, 2):
        prob = SmoothFWI(s_true.shape, w.geom, wav, dict(par, refs=refs, checkpoint=checkpoint))
        d_obs = prob.model(torch.as_tensor(s_true), keep=False)
        assert rel(to_host(d_obs), d_obs_o) < TOL
        data = prob.model(torch.as_tensor(s0), keep=True)
        assert rel(to_host(data), data_o) < TOL
        assert np.linalg.norm(to_host(data - d_obs) - res_o) < TOL * np.linalg.norm(d_obs_o)
        grad = prob.gradient(res_dev).cpu().numpy()
        assert rel(grad, grad_o) < GTOL, (checkpoint, rel(grad, grad_o))


@pytest.mark.parametrize("n,nw,kind", [(320, 6, "pspi"), (384, 6, "nsps"), (640, 3, "pspi")])
def test_born_on_register_resident_lengths(n, nw, kind):
    """ExtendedBorn forward and adjoint on the plan lengths 320, 384 and 640 (the
    radix-20 and radix-12 first stages), 3 levels of a config1-family model."""
    from pyfwix_b200 import workloads
    w = workloads.Workload(name=f"born-{n}", nx=n, ny=n, nz=3, dx=10.0, dy=10.0, dz=10.0, nw=nw, ow=4.0, dw=3.0,
                           nref=4, step=kind, taperx=20, tapery=20)
    w.anomaly = (n * 4.0, n * 6.0, 20.0)
    w.geom = dict(sx=np.array([n * 5.0], np.float32), sy=np.array([n * 5.0], np.float32),
                  sz=np.array([0.0], np.float32), s_ids=np.array([0], np.int32), **w.surface_receivers())
    rng = np.random.default_rng(n)
    w.wavelet = crandn(rng, (1, nw)).astype(np.complex64)
    c = Case(w)
    _, bd, bu = c.model()
    ds = (crandn(rng, (w.nz, 1, w.ny, w.nx)) * 1e-7).astype(np.complex64)
    dr = (crandn(rng, (w.nz, 1, w.ny, w.nx)) * 1e-2).astype(np.complex64)
    data = torch.empty((c.ntr, w.nw), dtype=torch.complex64, device="cuda")
    c.p.born(c.rec, bd, bu, to_dev(ds), to_dev(dr), data)
    r = crandn(rng, (c.ntr, w.nw)).astype(np.complex64)
    gs = torch.empty(ds.shape, dtype=torch.complex64, device="cuda")
    gr = torch.empty_like(gs)
    c.p.born(c.rec, bd, bu, gs, gr, to_dev(r), adjoint=True)
    o = c.oracle("born", ds=ds[:, 0], dr=dr[:, 0], r=r)
    assert rel(to_host(data), o["born"]) < TOL
    assert rel(to_host(gs)[:, 0], o["gs"]) < TOL
    assert rel(to_host(gr)[:, 0], o["gr"]) < TOL
