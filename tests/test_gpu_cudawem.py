"""The drop-in operator surface (``fwix/CudaWEM.py`` / ``fwix/CudaOperator.py``
class names and ``forward/adjoint(add, model, data)`` calls) against the FP64
oracle, with operands passed the ways the reference's callers pass them:
vectors with hypercubes, host numpy arrays (results written back in place) and
device tensors.  Mirrors the reference's operator tests
(``propagator/tests/*_test.cpp``: forward / adjoint / dot product per operator)."""
import numpy as np
import pytest
import torch

from oracle import wem
from pyfwix_b200 import CudaWEM, vectors
from pyfwix_b200.CudaOperator import cuFFT2d
from tests.conftest import cdot, crandn, dot_err
from tests.gpu_helpers import make_case, oracle_labels, rel

pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_SWEEP = 1e-4


def _axes(g, nz=None):
    return vectors.Hypercube([vectors.Axis(g.nx, g.ox, g.dx), vectors.Axis(g.ny, g.oy, g.dy),
                              vectors.Axis(g.nw, g.ow, g.dw), vectors.Axis(nz or g.nz, g.oz, g.dz)])


def _wf_hyper(g, ns):
    return vectors.Hypercube([vectors.Axis(g.NX, g.ox, g.dx), vectors.Axis(g.NY, g.oy, g.dy),
                              vectors.Axis(g.nw, g.ow, g.dw), vectors.Axis(ns)])


def _par(g, **kw):
    p = dict(nref=g.nref, padx=g.padx, pady=g.pady, eps=g.eps, taperx=g.taperx, tapery=g.tapery,
             eps_scat=g.eps_scat, taylor=g.taylor)
    p.update(kw)
    return p


def test_cufft2d_host_and_device_operands():
    rng = np.random.default_rng(3)
    x = crandn(rng, (3, 2, 40, 48)).astype(np.complex64)
    y = np.zeros_like(x)
    op = cuFFT2d(x, y)
    op.forward(False, x, y)                         # host numpy, written back in place
    assert rel(y, wem.fft2(x.astype(np.complex128))) < TOL
    xd = torch.as_tensor(x).cuda()
    yd = torch.as_tensor(y).cuda()
    op.adjoint(True, xd, yd)                        # device tensors, add
    assert rel(xd.cpu().numpy(), x + wem.ifft2(y.astype(np.complex128))) < TOL


def test_phase_shift_operator():
    g, rng, sref, _, _, _ = make_case(nx=32, ny=24, nw=4, nz=1, eps=0.02, complex_refs=True)
    m = vectors.Vector(_wf_hyper(g, 2), crandn(rng, (2, g.nw, g.NY, g.NX)), device="cuda")
    d = m.cloneSpace()
    op = CudaWEM.PhaseShift(m, d, g.dz, g.eps)
    op.set_slow(sref[0, 1])
    op.forward(False, m, d)
    fac = wem.phase_forward_factor(g.w2(), g.kx(), g.ky(), sref[0, 1], g.dz, g.eps)
    x = m.arr.cpu().numpy()
    assert rel(d.arr.cpu().numpy(), x * fac[None]) < TOL
    y = crandn(rng, x.shape)
    dd = vectors.Vector(_wf_hyper(g, 2), y, device="cuda")
    mm = m.cloneSpace()
    op.adjoint(False, mm, dd)
    adj = wem.phase_adjoint_factor(g.w2(), g.kx(), g.ky(), sref[0, 1], g.dz, g.eps)
    assert rel(mm.arr.cpu().numpy(), y * adj[None]) < TOL


def _slow_model(g, rng, per_w=True):
    s0 = (1 / 1800.0) ** 2
    nwm = g.nw if per_w else 1
    s2 = s0 * (1 + 0.3 * rng.random((g.nz, 1, g.ny, g.nx))) * np.ones((1, nwm, 1, 1))
    return s2.astype(np.complex64)


@pytest.mark.parametrize("cls,kind", [(CudaWEM.PSPI, "pspi"), (CudaWEM.NSPS, "nsps")])
def test_one_step_operators(cls, kind):
    g, rng, _, _, _, _ = make_case(nx=36, ny=30, nw=4, nz=3, nref=3, padx=4, pady=2)
    s2 = vectors.Vector(_axes(g), _slow_model(g, rng), device="cuda")
    m = vectors.Vector(_wf_hyper(g, 2), crandn(rng, (2, g.nw, g.NY, g.NX)), device="cuda")
    d = m.cloneSpace()
    op = cls(m, d, s2, _par(g))
    sref = op.plan._keep["sref"].cpu().numpy().astype(np.complex128)
    lab = oracle_labels(op.plan._keep["labels"].cpu().numpy(), g)
    for iz in range(g.nz):
        op.set_depth(iz)
        op.forward(False, m, d)
        x = m.arr.cpu().numpy().astype(np.complex128)
        ref = (wem.pspi_forward(g, sref[iz], lab[iz], x, taper=True) if kind == "pspi"
               else wem.nsps_forward(g, sref[iz], lab[iz], x))
        assert rel(d.arr.cpu().numpy(), ref) < TOL
        # add-version adjoint (PSPI: no taper, as in the reference)
        y = crandn(rng, x.shape)
        dv = vectors.Vector(_wf_hyper(g, 2), y, device="cuda")
        mv = m.cloneSpace()
        op.adjoint(False, mv, dv)
        ref = (wem.pspi_adjoint(g, sref[iz], lab[iz], y, taper=False) if kind == "pspi"
               else wem.nsps_adjoint(g, sref[iz], lab[iz], y))
        assert rel(mv.arr.cpu().numpy(), ref) < TOL


def test_injection_operator():
    g, rng, _, _, _, _ = make_case(nx=32, ny=24, nw=3, nz=6, padx=4, pady=4)
    cx = rng.uniform(0, 330, 12).astype(np.float32)
    cy = rng.uniform(0, 300, 12).astype(np.float32)
    cz = rng.uniform(0, 35, 12).astype(np.float32)
    ids = rng.integers(0, 2, 12).astype(np.int32)
    tr = crandn(rng, (12, g.nw)).astype(np.complex64)
    wf = np.zeros((2, g.nw, g.NY, g.NX), np.complex64)
    wfv = vectors.Vector(_wf_hyper(g, 2), wf)
    op = CudaWEM.Injection(tr, wfv, g.oz, g.dz, cx, cy, cz, ids)
    otr = wem.make_traces(cx, cy, cz, ids, g.ox, g.oy, g.dx, g.dy, g.oz, g.dz, g.NX, g.NY)
    for iz in range(4):
        op.set_depth(iz)
        op.forward(False, tr, wfv)
        ref = wem.inject(otr, tr.astype(np.complex128), np.zeros(wf.shape, np.complex128), iz)
        assert rel(wfv.arr.numpy(), ref) < TOL
        w = crandn(rng, wf.shape)
        got = np.zeros_like(tr)
        op.adjoint(False, got, w)
        refr = wem.record(otr, w, np.zeros(tr.shape, np.complex128), iz)
        if np.linalg.norm(refr) > 0:
            assert rel(got, refr) < TOL


@pytest.mark.parametrize("cls,fwd,adj", [(CudaWEM.Downward, wem.downward, wem.downward_adjoint),
                                         (CudaWEM.Upward, wem.upward, wem.upward_adjoint)])
def test_sweep_operators(cls, fwd, adj):
    g, rng, _, _, _, _ = make_case(nx=32, ny=24, nw=3, nz=5, nref=3, padx=4, pady=4)
    s2 = _slow_model(g, rng)
    x = crandn(rng, (2, g.nw, g.NY, g.NX)).astype(np.complex64)
    out = np.zeros_like(x)
    par = dict(_par(g), ox=g.ox, dx=g.dx, oy=g.oy, dy=g.dy, oz=g.oz, dz=g.dz, ow=g.ow, dw=g.dw)
    op = cls(x, out, s2, par)                               # bare arrays, axes from par
    sref = op.plan._keep["sref"].cpu().numpy().astype(np.complex128)
    lab = oracle_labels(op.plan._keep["labels"].cpu().numpy(), g)
    st = wem.Stepper(g, sref, lab, "pspi")
    op.forward(False, x, out)
    assert rel(out, fwd(st, g.nz, x.astype(np.complex128))) < TOL_SWEEP
    w = torch.as_tensor(x).cuda()
    op.adjoint(w)                                           # one-argument in-place form
    assert rel(w.cpu().numpy(), adj(st, g.nz, x.astype(np.complex128))) < TOL_SWEEP


def _acq(g, rng):
    # receivers spread over the whole model, so that the acquisition window is the model
    geom = dict(sx=np.array([80.0, 200.0], np.float32), sy=np.array([96.0, 120.0], np.float32),
                sz=np.array([0.0, 5.0], np.float32), s_ids=np.array([7, 3], np.int32),
                rx=np.linspace(0, (g.nx - 1) * g.dx, 16).astype(np.float32),
                ry=np.linspace(0, (g.ny - 1) * g.dy, 16).astype(np.float32),
                rz=np.zeros(16, np.float32), r_ids=np.array([7, 3] * 8, np.int32))
    wav = crandn(rng, (2, g.nw)).astype(np.complex64)
    return geom, wav


def _born_setup(kind="pspi"):
    g, rng, _, _, _, _ = make_case(nx=32, ny=24, nw=3, nz=6, nref=3, padx=4, pady=4, taperx=0, tapery=0)
    s2 = _slow_model(g, rng)
    s2[g.nz - 2:] *= 1.6
    den = (1.0 + 0.2 * rng.random(s2.shape)).astype(np.complex64)
    model = vectors.SuperVector(vectors.Vector(_axes(g), s2), vectors.Vector(_axes(g), den))
    geom, wav = _acq(g, rng)
    data = np.zeros((16, g.nw), np.complex64)
    prop = CudaWEM.Propagator(model, data, wav, _par(g, step=kind), geom)
    return g, rng, s2, den, model, geom, wav, data, prop


def _oracle_of(prop, g, kind="pspi"):
    plan = prop.pairs[0].prop.plan if hasattr(prop, "pairs") else prop.plan
    sref = plan._keep["sref"].cpu().numpy().astype(np.complex128)
    lab = oracle_labels(plan._keep["labels"].cpu().numpy(), g)
    return wem.Stepper(g, sref, lab, kind)


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_propagator_and_born(kind):
    g, rng, s2, den, model, geom, wav, data, prop = _born_setup(kind)
    prop.forward(False, model, data)
    st = _oracle_of(prop, g, kind)
    acq = wem.make_acquisition(g, geom)
    ref, bgd, bgu = wem.propagate(g, st, acq, s2.astype(np.complex128), den.astype(np.complex128),
                                  wav.astype(np.complex128))
    assert rel(data, ref) < TOL_SWEEP
    dm = vectors.SuperVector(vectors.Vector(_axes(g), crandn(rng, s2.shape) * 1e-3),
                             vectors.Vector(_axes(g), crandn(rng, s2.shape) * 1e-2))
    born = CudaWEM.ExtendedBorn(dm, data, model, prop)
    d1 = np.zeros_like(data)
    born.forward(False, dm, d1)
    refb = wem.born_forward(g, st, acq, s2.astype(np.complex128), den.astype(np.complex128), bgd, bgu,
                            dm[0].arr.numpy().astype(np.complex128), dm[1].arr.numpy().astype(np.complex128))
    assert rel(d1, refb) < TOL_SWEEP
    r = crandn(rng, data.shape).astype(np.complex64)
    g_ = dm.cloneSpace()
    born.adjoint(False, g_, r)
    gs, gr = wem.born_adjoint(g, st, acq, s2.astype(np.complex128), den.astype(np.complex128), bgd, bgu,
                              r.astype(np.complex128))
    assert rel(g_[0].arr.numpy(), gs) < TOL_SWEEP
    assert rel(g_[1].arr.numpy(), gr) < TOL_SWEEP
    # dot product through the surface: <B dm, r> vs <dm, B^T r>
    lhs = cdot(r, d1)
    rhs = cdot(g_[0].arr.numpy(), dm[0].arr.numpy()) + cdot(g_[1].arr.numpy(), dm[1].arr.numpy())
    assert abs(lhs / rhs - 1) < 1e-4


def test_born_adjoint_add_and_workers_flow():
    """The call sequence of ``fwix/workers.py:62-76``: forward model, residual,
    objective, Born adjoint into a zeroed gradient."""
    g, rng, s2, den, model, geom, wav, data, prop = _born_setup()
    d_obs = crandn(rng, data.shape).astype(np.complex64) * 1e-3
    res = np.zeros_like(data)
    grad = model.cloneSpace()
    born = CudaWEM.ExtendedBorn(grad, res, model, prop)
    prop.forward(False, model, res)
    res -= d_obs
    obj = float(np.real(np.vdot(res, res)))
    assert obj > 0
    born.adjoint(False, grad, res)
    g1 = [v.arr.clone() for v in grad.vecs]
    born.adjoint(True, grad, res)                             # add doubles it
    for a, b in zip(g1, grad.vecs):
        assert rel(b.arr.numpy(), 2 * a.numpy()) < 1e-6


def test_refsampler_surface():
    g, rng, _, _, _, _ = make_case(nx=32, ny=24, nw=3, nz=4, nref=3, padx=4, pady=2)
    s2 = _slow_model(g, rng)
    rs = CudaWEM.RefSampler(vectors.Vector(_axes(g), s2), dict(nref=3, padx=4, pady=2))
    assert rs.get_ref_slow(2, 1).shape == (g.nw,)
    lab = rs.get_ref_labels(2)
    assert lab.shape == (g.nw, g.NY, g.NX) and lab.min() >= 0 and lab.max() < 3
    # labels pick the nearest reference
    refs = np.stack([rs.get_ref_slow(2, r) for r in range(3)])
    near = np.argmin(np.abs(s2[2][None].astype(np.complex128) - refs[:, :, None, None]), axis=0)
    assert np.mean(lab[:, :g.ny, :g.nx] == near) > 0.999


def test_streaming_batches_windows_and_bands():
    """nbatches = (2 shot groups, 2 frequency bands) with aperture windows
    (ginsu) against the FP64 oracle run on each pair's window and added into
    the global data / gradient at the pair's receivers, band and window
    (StreamingPropagator.cpp:327-470); Born dot test through the surface."""
    from pyfwix_b200 import streaming
    # taper 0: the reference's PSPI Born pair is adjoint only without taper
    g, rng, _, _, _, _ = make_case(nx=56, ny=40, nw=4, nz=5, nref=3, padx=4, pady=4, taperx=0, tapery=0)
    s2 = _slow_model(g, rng)
    s2[g.nz - 2:] *= 1.5
    den = (1.0 + 0.2 * rng.random(s2.shape)).astype(np.complex64)
    model = vectors.SuperVector(vectors.Vector(_axes(g), s2), vectors.Vector(_axes(g), den))
    sx = np.array([60.0, 150.0, 330.0, 430.0], np.float32)
    geom = dict(sx=sx, sy=np.full(4, 180.0, np.float32), sz=np.zeros(4, np.float32),
                s_ids=np.array([11, 12, 13, 14], np.int32))
    rx, ry, rid = [], [], []
    for k, x in enumerate(sx):
        rx += list(x + np.linspace(-40, 40, 5))
        ry += [170.0, 190.0, 200.0, 210.0, 230.0]
        rid += [11 + k] * 5
    geom.update(rx=np.clip(np.array(rx, np.float32), 0, 540), ry=np.array(ry, np.float32),
                rz=np.zeros(len(rx), np.float32), r_ids=np.array(rid, np.int32))
    wav = crandn(rng, (4, g.nw)).astype(np.complex64)
    par = _par(g, ginsu_x=30.0, ginsu_y=20.0)
    data = np.zeros((len(rx), g.nw), np.complex64)
    prop = CudaWEM.Propagator(model, data, wav, par, geom, nbatches=(2, 2))
    assert len(prop.pairs) == 4 and len({p.window for p in prop.pairs}) == 2
    prop.forward(False, model, data)
    ref = np.zeros(data.shape, np.complex128)
    grids = []
    for p in prop.pairs:
        x0, x1, y0, y1 = p.window
        pl = p.prop.plan
        gw = wem.Grid(nx=x1 - x0 + 1, ny=y1 - y0 + 1, nw=p.nf, nz=g.nz, dx=g.dx, dy=g.dy, dz=g.dz,
                      ox=g.ox + x0 * g.dx, oy=g.oy + y0 * g.dy, oz=g.oz, ow=g.ow + p.f0 * g.dw, dw=g.dw,
                      padx=pl.NX - pl.nx, pady=pl.NY - pl.ny, nref=g.nref, taperx=g.taperx, tapery=g.tapery)
        pg = prop._pair_geometry(p)
        acq = wem.make_acquisition(gw, pg)
        st = _oracle_of(p.prop, gw)
        sw = s2[:, p.f0:p.f0 + p.nf, y0:y1 + 1, x0:x1 + 1].astype(np.complex128)
        dw_ = den[:, p.f0:p.f0 + p.nf, y0:y1 + 1, x0:x1 + 1].astype(np.complex128)
        d, bgd, bgu = wem.propagate(gw, st, acq, sw, dw_, wav[p.src_idx][:, p.f0:p.f0 + p.nf].astype(np.complex128))
        ref[np.ix_(p.rec_idx, np.arange(p.f0, p.f0 + p.nf))] += d
        grids.append((gw, st, acq, sw, dw_, bgd, bgu))
    assert rel(data, ref) < TOL_SWEEP
    # Born adjoint against the per-window oracle, and the surface dot test
    born = CudaWEM.ExtendedBorn(model.cloneSpace(), data, model, prop)
    r = crandn(rng, data.shape).astype(np.complex64)
    gmod = model.cloneSpace()
    born.adjoint(False, gmod, r)
    gs_ref = np.zeros(s2.shape, np.complex128)
    for p, (gw, st, acq, sw, dw_, bgd, bgu) in zip(prop.pairs, grids):
        x0, x1, y0, y1 = p.window
        rr = r[p.rec_idx][:, p.f0:p.f0 + p.nf].astype(np.complex128)
        gs, gr = wem.born_adjoint(gw, st, acq, sw, dw_, bgd, bgu, rr)
        gs_ref[:, p.f0:p.f0 + p.nf, y0:y1 + 1, x0:x1 + 1] += gs
    assert rel(gmod[0].arr.numpy(), gs_ref) < TOL_SWEEP
    dm = vectors.SuperVector(vectors.Vector(_axes(g), crandn(rng, s2.shape) * 1e-3),
                             vectors.Vector(_axes(g), crandn(rng, s2.shape) * 1e-2))
    d1 = np.zeros_like(data)
    born.forward(False, dm, d1)
    lhs = cdot(r, d1)
    rhs = cdot(gmod[0].arr.numpy(), dm[0].arr.numpy()) + cdot(gmod[1].arr.numpy(), dm[1].arr.numpy())
    assert abs(lhs / rhs - 1) < 1e-4
    assert streaming.window_indices([60.0], [180.0], (56, 0.0, 10.0), (40, 0.0, 10.0), 30.0, 20.0) == (3, 9, 16, 20)
    assert [streaming.next_fft_length(n) for n in (23, 26, 49, 97)] == [24, 27, 49, 98]


def test_compress_rate_packed_backgrounds():
    """``compress_rate`` 8 (the reference's default rate of its ZFP store) keeps the
    backgrounds in the packed fixed-rate store: data and Born within the store's
    error of the lossless run, the stored bytes 3.7 x fewer; other rates are refused."""
    g, rng, s2, den, model, geom, wav, data, prop = _born_setup("pspi")
    prop.forward(False, model, data)
    par = _par(g, step="pspi", compress_rate=8)
    data_c = np.zeros_like(data)
    prop_c = CudaWEM.Propagator(model, data_c, wav, par, geom)
    prop_c.forward(False, model, data_c)
    assert rel(data_c, data) < 2e-2 and prop_c.get_compression_ratio() > 3.7
    assert prop.get_compression_ratio() == 1.0
    dm = vectors.SuperVector(vectors.Vector(_axes(g), crandn(rng, s2.shape) * 1e-3),
                             vectors.Vector(_axes(g), crandn(rng, s2.shape) * 1e-2))
    d1, d2 = np.zeros_like(data), np.zeros_like(data)
    CudaWEM.ExtendedBorn(dm, d1, model, prop).forward(False, dm, d1)
    CudaWEM.ExtendedBorn(dm, d2, model, prop_c).forward(False, dm, d2)
    assert rel(d2, d1) < 3e-2
    r = crandn(rng, data.shape).astype(np.complex64)
    g1, g2 = dm.cloneSpace(), dm.cloneSpace()
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("error", CudaWEM.PackedGradientWarning)   # lossless: no warning
        CudaWEM.ExtendedBorn(dm, r, model, prop).adjoint(False, g1, r)
    # the gradient on packed backgrounds says that it leaves the lossless tolerance
    with pytest.warns(CudaWEM.PackedGradientWarning, match="1e-3"):
        CudaWEM.ExtendedBorn(dm, r, model, prop_c).adjoint(False, g2, r)
    assert rel(g2[0].arr.numpy(), g1[0].arr.numpy()) < 3e-2
    # rate 16: 1.94 x fewer bytes, the gradient within the 1e-3 bar and no warning
    par16 = _par(g, step="pspi", compress_rate=16)
    data16 = np.zeros_like(data)
    prop16 = CudaWEM.Propagator(model, data16, wav, par16, geom)
    prop16.forward(False, model, data16)
    assert 1.9 < prop16.get_compression_ratio() < 2.0 and rel(data16, data) < 1e-4
    g3 = dm.cloneSpace()
    with warnings.catch_warnings():
        warnings.simplefilter("error", CudaWEM.PackedGradientWarning)
        CudaWEM.ExtendedBorn(dm, r, model, prop16).adjoint(False, g3, r)
    assert rel(g3[0].arr.numpy(), g1[0].arr.numpy()) < 1e-3
    with pytest.raises(ValueError):
        CudaWEM.Propagator(model, data_c, wav, _par(g, compress_rate=4), geom).forward(False, model, data_c)


def test_staged_host_copies(monkeypatch):
    """Large host operands cross the host link through pinned staging buffers
    (pyfwix_b200.hostcopy: chunks, two buffers, host copies on a thread pool):
    the round trip is exact for a length that is no multiple of the chunk, and a
    Born forward + adjoint through the surface with every operand staged equals
    the plain copies bit for bit."""
    from pyfwix_b200 import hostcopy
    monkeypatch.setattr(hostcopy, "CHUNK_BYTES", 4096 + 24)
    monkeypatch.setattr(hostcopy, "THRESHOLD_BYTES", 1)
    rng = np.random.default_rng(3)
    n = 100003
    a = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    t = hostcopy.to_device(a, torch.device("cuda"))
    assert np.array_equal(t.cpu().numpy(), a)
    b = np.empty_like(a)
    hostcopy.to_host(t * 2, b)
    assert np.array_equal(b, 2 * a)
    assert hostcopy.host_view(torch.from_numpy(a)) is not None

    def born_run():
        g, rng2, s2, den, model, geom, wav, data, prop = _born_setup("nsps")
        prop.forward(False, model, data)
        dm = [crandn(rng2, s2.shape).astype(np.complex64) * 1e-3, crandn(rng2, s2.shape).astype(np.complex64) * 1e-2]
        born = CudaWEM.ExtendedBorn(dm, data, model, prop)
        d1 = np.zeros_like(data)
        born.forward(False, dm, d1)
        gs, gr = np.zeros_like(dm[0]), np.zeros_like(dm[1])
        born.adjoint(False, [gs, gr], d1)
        torch.cuda.synchronize()
        return d1, gs, gr

    staged = born_run()
    monkeypatch.setattr(hostcopy, "THRESHOLD_BYTES", 1 << 62)
    plain = born_run()
    for x, y in zip(staged, plain):
        assert np.array_equal(x, y)
