"""Parity of the depth-sweep drivers with the FP64 oracle: Downward / Upward
(OneWay.cpp:24-79), Propagator::forward (Propagator.cpp:121-221), the lockstep
migration image and ExtendedBorn forward / adjoint (ExtendedBorn.cpp:80-453).
Tolerance 1e-4 relative L2 for the swept outputs (image bar of the spec)."""
import numpy as np
import pytest
import torch

from oracle import wem
from tests.conftest import crandn
from tests.gpu_helpers import make_case, make_plan, oracle_labels, rel, to_dev, to_host, wavefield

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_down_up(kind):
    g, rng, sref, labels, _, _ = make_case(nx=32, ny=24, nw=4, nz=6, nref=3, padx=4, pady=4)
    lab = oracle_labels(labels, g)
    st = wem.Stepper(g, sref, lab, kind)
    p = make_plan(g, 2, sref, labels, step=kind)
    x = wavefield(rng, 2, g)
    for adj, fn in ((False, wem.downward), (True, wem.downward_adjoint)):
        y = to_host(p.downward(to_dev(x), adjoint=adj))
        assert rel(y, fn(st, g.nz, x)) < TOL
    for adj, fn in ((False, wem.upward), (True, wem.upward_adjoint)):
        y = to_host(p.upward(to_dev(x), adjoint=adj))
        assert rel(y, fn(st, g.nz, x)) < TOL


def _acq_case(kind="pspi", taper=3, pad=4, nz=7, nx=32, ny=24):
    g, rng, sref, labels, slow, den = make_case(nx=nx, ny=ny, nw=4, nz=nz, nref=3, padx=pad, pady=pad,
                                                taperx=taper, tapery=taper)
    slow = slow.copy()
    slow[nz - 3:] *= 1.8  # reflector
    lab = oracle_labels(labels, g)
    st = wem.Stepper(g, sref, lab, kind)
    geom = dict(sx=[80.0, 200.0, 200.0], sy=[96.0, 120.0, 120.0], sz=[0.0, 5.0, 5.0], s_ids=[4, 9, 9],
                rx=list(np.linspace(0, 300, 16)), ry=[100.0] * 16, rz=[0.0] * 8 + [12.0] * 8,
                r_ids=[4, 9] * 8)
    acq = wem.make_acquisition(g, geom)
    p = make_plan(g, acq.ns, sref, labels, slow, den, step=kind)
    src = p.traces(geom["sx"], geom["sy"], geom["sz"], acq.src.ids)
    rec = p.traces(geom["rx"], geom["ry"], geom["rz"], acq.rec.ids)
    wav = crandn(rng, (3, g.nw))
    return g, rng, st, acq, p, src, rec, wav, slow, den


@pytest.mark.parametrize("kind,nx,ny,pad", [("pspi", 32, 24, 4), ("nsps", 32, 24, 4), ("pspi", 96, 60, 4)])
def test_propagate(kind, nx, ny, pad):
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case(kind, nx=nx, ny=ny, pad=pad)
    data, bgd, bgu = wem.propagate(g, st, acq, slow, den, wav)
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, to_dev(wav), d, bd, bu)
    assert rel(to_host(d), data) < TOL
    assert rel(to_host(bd), np.stack(bgd)) < TOL
    assert rel(to_host(bu), np.stack(bgu)) < TOL
    # add semantics
    d2 = to_dev(data)
    p.propagate(src, rec, to_dev(wav), d2, bd, bu, add=True)
    assert rel(to_host(d2), 2 * data) < TOL


@pytest.mark.parametrize("kind,nx,ny,pad", [("pspi", 32, 24, 4), ("nsps", 32, 24, 4), ("pspi", 64, 64, 0),
                                             ("nsps", 60, 60, 4)])
def test_migrate(kind, nx, ny, pad):
    """Lockstep migration of two shots with receivers at two depths (levels 0-2):
    the image of the levels without receiver injection is summed in the receiver
    step's last pass, the others by a separate correlation; generic and
    register-resident lengths; add semantics."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case(kind, nx=nx, ny=ny, pad=pad)
    data = crandn(rng, (len(acq.rec.ix), g.nw))
    img = wem.migrate(g, st, acq, wav, data)
    out = torch.empty((g.nz, g.ny, g.nx), dtype=torch.float32, device="cuda")
    p.migrate(src, rec, to_dev(wav), to_dev(data), out)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), img) < TOL
    base = torch.ones((g.nz, g.ny, g.nx), dtype=torch.float32, device="cuda")
    p.migrate(src, rec, to_dev(wav), to_dev(data), base, add=True)
    torch.cuda.synchronize()
    assert rel(base.cpu().numpy() - 1, img) < TOL


@pytest.mark.parametrize("kind,taper,nx,ny,pad", [("pspi", 3, 32, 24, 4), ("nsps", 0, 32, 24, 4),
                                                 ("pspi", 3, 64, 64, 0), ("nsps", 2, 60, 44, 4)])
def test_born(kind, taper, nx, ny, pad):
    """Born forward / adjoint; 64 x 64 exercises the register-resident passes,
    the other sizes the generic ones."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case(kind, taper=taper, nx=nx, ny=ny, pad=pad)
    data, bgd, bgu = wem.propagate(g, st, acq, slow, den, wav)
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, to_dev(wav), d, bd, bu)
    ms = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
    mr = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
    ref = wem.born_forward(g, st, acq, slow, den, bgd, bgu, ms, mr)
    out = torch.empty_like(d)
    p.born(rec, bd, bu, to_dev(ms), to_dev(mr), out)
    assert rel(to_host(out), ref) < TOL
    r = crandn(rng, d.shape)
    gs_ref, gr_ref = wem.born_adjoint(g, st, acq, slow, den, bgd, bgu, r)
    gs = torch.empty((g.nz, g.nw, g.ny, g.nx), dtype=torch.complex64, device="cuda")
    gr = torch.empty_like(gs)
    p.born(rec, bd, bu, gs, gr, to_dev(r), adjoint=True)
    assert rel(to_host(gs), gs_ref) < TOL
    assert rel(to_host(gr), gr_ref) < TOL


@pytest.mark.parametrize("kind,taper,nx,ny,pad", [("pspi", 3, 32, 24, 4), ("nsps", 0, 32, 24, 4),
                                                 ("pspi", 3, 64, 64, 0), ("nsps", 2, 64, 64, 0)])
def test_born_broadcast_background(kind, taper, nx, ny, pad):
    """Born forward / adjoint with a background model and a perturbation shared by
    every frequency ([nz][1][ny][nx]): the case in which the per-level
    reflections are added inside the depth steps' row passes (forward: the step's
    output; adjoint: the next step's input) and the adjoint's two frequency sums
    of a level share one pass.  Against the FP64 oracle on per-frequency copies."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case(kind, taper=taper, nx=nx, ny=ny, pad=pad)
    slow1, den1 = slow[:, :1].copy(), den[:, :1].copy()
    slow_w, den_w = np.repeat(slow1, g.nw, 1), np.repeat(den1, g.nw, 1)
    p.set_model(slow1, den1)
    data, bgd, bgu = wem.propagate(g, st, acq, slow_w, den_w, wav)
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, to_dev(wav), d, bd, bu)
    assert rel(to_host(d), data) < TOL
    ms = crandn(rng, (g.nz, 1, g.ny, g.nx))
    mr = crandn(rng, (g.nz, 1, g.ny, g.nx))
    ref = wem.born_forward(g, st, acq, slow_w, den_w, bgd, bgu, np.repeat(ms, g.nw, 1), np.repeat(mr, g.nw, 1))
    out = torch.empty_like(d)
    p.born(rec, bd, bu, to_dev(ms), to_dev(mr), out)
    assert rel(to_host(out), ref) < TOL
    r = crandn(rng, d.shape)
    gs_ref, gr_ref = wem.born_adjoint(g, st, acq, slow_w, den_w, bgd, bgu, r)
    gs = torch.empty((g.nz, 1, g.ny, g.nx), dtype=torch.complex64, device="cuda")
    gr = torch.empty_like(gs)
    p.born(rec, bd, bu, gs, gr, to_dev(r), adjoint=True)
    assert rel(to_host(gs), gs_ref.sum(1, keepdims=True)) < TOL
    assert rel(to_host(gr), gr_ref.sum(1, keepdims=True)) < TOL


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_born_broadcast_background_two_lanes(kind):
    """The reflections inside the steps under the tuner's two-lane form (chunks of
    slices alternating between two streams, each with its own intermediates):
    Born forward and adjoint equal the one-launch plan's."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case(kind, taper=2, nx=64, ny=64, pad=0)
    p.set_model(slow[:, :1].copy(), den[:, :1].copy())
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, to_dev(wav), d, bd, bu)
    ms = to_dev(crandn(rng, (g.nz, 1, g.ny, g.nx)))
    mr = to_dev(crandn(rng, (g.nz, 1, g.ny, g.nx)))
    r = to_dev(crandn(rng, d.shape))

    def run():
        out = torch.empty_like(d)
        p.born(rec, bd, bu, ms, mr, out)
        gs = torch.empty_like(ms)
        gr = torch.empty_like(ms)
        p.born(rec, bd, bu, gs, gr, r, adjoint=True)
        torch.cuda.synchronize()
        return to_host(out), to_host(gs), to_host(gr)

    one = run()
    p.set_tuning(dict(col_tma=True, slices_per_launch=g.nw // 2, streams=2))
    two = run()
    for a, b in zip(two, one):
        assert rel(a, b) < 1e-6


def test_born_dot_product_device():
    """ExtendedBorn dot test (propagator/src/ExtendedBorn.h:61-128) entirely on the
    device, taper off as in born_unit_test.cpp:392-393."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case("pspi", taper=0)
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, to_dev(wav), d, bd, bu)
    ms = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
    mr = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
    r = crandn(rng, d.shape)
    out = torch.empty_like(d)
    p.born(rec, bd, bu, to_dev(ms), to_dev(mr), out)
    gs = torch.empty((g.nz, g.nw, g.ny, g.nx), dtype=torch.complex64, device="cuda")
    gr = torch.empty_like(gs)
    p.born(rec, bd, bu, gs, gr, to_dev(r), adjoint=True)
    lhs = np.vdot(r.ravel(), to_host(out).ravel())
    rhs = np.vdot(to_host(gs).ravel(), ms.ravel()) + np.vdot(to_host(gr).ravel(), mr.ravel())
    assert abs((lhs / rhs).real - 1) < 1e-5


def test_born_frequency_broadcast_model():
    """A [nz][1][ny][nx] perturbation equals its per-frequency copy in the forward,
    and the adjoint returns the frequency sum of the per-frequency gradient."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case("nsps", taper=0)
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, to_dev(wav), d, bd, bu)
    ms = crandn(rng, (g.nz, 1, g.ny, g.nx))
    mr = crandn(rng, (g.nz, 1, g.ny, g.nx))
    out1 = torch.empty_like(d)
    p.born(rec, bd, bu, to_dev(ms), to_dev(mr), out1)
    out2 = torch.empty_like(d)
    p.born(rec, bd, bu, to_dev(np.repeat(ms, g.nw, 1)), to_dev(np.repeat(mr, g.nw, 1)), out2)
    assert rel(to_host(out1), to_host(out2)) < 1e-5
    r = crandn(rng, d.shape)
    gs1 = torch.empty((g.nz, 1, g.ny, g.nx), dtype=torch.complex64, device="cuda")
    gr1 = torch.empty_like(gs1)
    p.born(rec, bd, bu, gs1, gr1, to_dev(r), adjoint=True)
    gs2 = torch.empty((g.nz, g.nw, g.ny, g.nx), dtype=torch.complex64, device="cuda")
    gr2 = torch.empty_like(gs2)
    p.born(rec, bd, bu, gs2, gr2, to_dev(r), adjoint=True)
    assert rel(to_host(gs1), to_host(gs2).sum(1, keepdims=True)) < 1e-5
    assert rel(to_host(gr1), to_host(gr2).sum(1, keepdims=True)) < 1e-5


@pytest.mark.parametrize("nx,ny,pad", [(32, 24, 4), (64, 64, 0)])
def test_phase_cache_rotation(nx, ny, pad):
    """A phase-factor cache of fewer depths than nz (depth iz in slot iz mod k,
    rebuilt when another depth took the slot) gives the same modelling and Born
    forward / adjoint, bit for bit, as the cache of every depth (the Born sweeps
    go down and up, so slots are rebuilt many times), and the same migration
    image to the rounding of its frequency sum (float atomics, no fixed order)."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case("pspi", nx=nx, ny=ny, pad=pad)
    ms = to_dev(crandn(rng, (g.nz, g.nw, g.ny, g.nx)))
    mr = to_dev(crandn(rng, (g.nz, g.nw, g.ny, g.nx)))
    r = to_dev(crandn(rng, (len(acq.rec.ix), g.nw)))

    def run():
        bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
        bu = torch.empty_like(bd)
        d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
        p.propagate(src, rec, to_dev(wav), d, bd, bu)
        out = torch.empty_like(d)
        p.born(rec, bd, bu, ms, mr, out)
        gs = torch.empty_like(ms)
        gr = torch.empty_like(ms)
        p.born(rec, bd, bu, gs, gr, r, adjoint=True)
        img = torch.empty((g.nz, g.ny, g.nx), dtype=torch.float32, device="cuda")
        p.migrate(src, rec, to_dev(wav), r, img)
        torch.cuda.synchronize()
        return [t.clone() for t in (d, out, gs, gr, img)]

    assert p.enable_phase_cache()
    full = run()
    for depths in (1, 3):
        p.disable_phase_cache()
        assert p.enable_phase_cache(depths=depths)
        *rest, img = run()
        for a, b in zip(rest, full[:-1]):
            assert torch.equal(a, b)
        assert rel(img.cpu().numpy(), full[-1].cpu().numpy()) < 1e-6


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_shallow_grids(kind):
    """One and two depth levels: the bottom level reflects nothing and its
    linearised reflection reads the same level twice (propagator/src/LinReflect.h:28-41
    copies level z as level z + 1 there), receivers below the grid are skipped.
    With one level the Born operators add (to rounding) nothing to what the
    output held."""
    for nz in (1, 2):
        g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case(kind, nz=nz)
        data, bgd, bgu = wem.propagate(g, st, acq, slow, den, wav)
        bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
        bu = torch.empty_like(bd)
        d = torch.empty((len(acq.rec.ix), g.nw), dtype=torch.complex64, device="cuda")
        p.propagate(src, rec, to_dev(wav), d, bd, bu)
        assert rel(to_host(d), data) < TOL
        ms = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
        mr = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
        r = crandn(rng, d.shape)
        ref = wem.born_forward(g, st, acq, slow, den, bgd, bgu, ms, mr)
        gs_ref, gr_ref = wem.born_adjoint(g, st, acq, slow, den, bgd, bgu, r)
        d0 = crandn(rng, d.shape)
        g0 = crandn(rng, ms.shape)
        out = to_dev(d0)
        p.born(rec, bd, bu, to_dev(ms), to_dev(mr), out, add=True)
        gs = to_dev(g0)
        gr = to_dev(g0)
        p.born(rec, bd, bu, gs, gr, to_dev(r), adjoint=True, add=True)
        assert rel(to_host(out), d0 + ref) < TOL
        assert rel(to_host(gs), g0 + gs_ref) < TOL
        assert rel(to_host(gr), g0 + gr_ref) < TOL


def test_receivers_all_dropped():
    """Receivers on the last column of the padded grid are dropped
    (propagator/src/injection.cu:46-48): the data are zero, Born forward records
    nothing and its adjoint injects nothing."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case("nsps")
    xs = [(g.NX - 1) * g.dx + 0.5] * 4
    off = p.traces(xs, [100.0] * 4, [0.0, 0.0, 12.0, 12.0], [0, 1, 1, 0])
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = to_dev(crandn(rng, (4, g.nw)))
    p.propagate(src, off, to_dev(wav), d, bd, bu)
    assert not to_host(d).any()
    ms = to_dev(crandn(rng, (g.nz, g.nw, g.ny, g.nx)))
    p.born(off, bd, bu, ms, ms, d)
    assert not to_host(d).any()
    r = to_dev(crandn(rng, (4, g.nw)))
    gs = to_dev(crandn(rng, (g.nz, g.nw, g.ny, g.nx)))
    gr = torch.empty_like(gs)
    p.born(off, bd, bu, gs, gr, r, adjoint=True)
    assert not to_host(gs).any() and not to_host(gr).any()


def test_no_receivers():
    """An empty receiver set (null data buffer allowed): modelling still fills
    the background wavefields, and the Born adjoint of no data is zero."""
    g, rng, st, acq, p, src, rec, wav, slow, den = _acq_case("pspi")
    _, bgd, bgu = wem.propagate(g, st, acq, slow, den, wav)
    none = p.traces([], [], [], [])
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((0, g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, none, to_dev(wav), d, bd, bu)
    assert rel(to_host(bd), np.stack(bgd)) < TOL
    assert rel(to_host(bu), np.stack(bgu)) < TOL
    gs = to_dev(crandn(rng, (g.nz, g.nw, g.ny, g.nx)))
    gr = torch.empty_like(gs)
    p.born(none, bd, bu, gs, gr, d, adjoint=True)
    assert not to_host(gs).any() and not to_host(gr).any()
