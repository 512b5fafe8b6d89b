"""Pins the CPU oracle against the reference's own known-answer and dot tests.

Sizes follow the reference tests where they are cheap and are reduced where the
pure-numpy oracle would take too long; each test names the reference test it
restates."""
import math

import numpy as np
import pytest

from oracle import wem
from tests.conftest import crandn, dot_err

TOL = 1e-10  # FP64 oracle: far tighter than the reference's 1e-5 (prop_unit_test.cpp:18)


# ---------------------------------------------------------------- FFT (operator/tests/operator_unit_test.cpp)

def test_fft_constant_signal_dc():
    """``constant_signal`` (:50-65): DC = n1*n2/sqrt(n1*n2), imag 0 everywhere."""
    n1, n2 = 100, 100
    x = np.ones((2, 3, n2, n1), dtype=np.complex128)
    y = wem.fft2(x)
    assert np.allclose(y[..., 0, 0].real, n1 * n2 / math.sqrt(n1 * n2), atol=1e-9)
    assert np.max(np.abs(y.imag)) < 1e-9
    y[..., 0, 0] = 0
    assert np.max(np.abs(y)) < 1e-9


def test_fft_mono_plane_wave():
    """``mono_plane_wave`` (:67-99): spike of height sqrt(n1*n2) at (k1, k2) = (10, 20)."""
    n1, n2, k1, k2 = 100, 100, 10, 20
    i1 = np.arange(n1)[None, :]
    i2 = np.arange(n2)[:, None]
    x = np.exp(1j * 2 * np.pi * (k1 * i1 / n1 + k2 * i2 / n2))[None, None]
    y = wem.fft2(x)
    assert abs(y[0, 0, k2, k1].real - n1 * n2 / math.sqrt(n1 * n2)) < 1e-9
    y[0, 0, k2, k1] = 0
    assert np.max(np.abs(y)) < 1e-9


def test_fft_forward_inverse(rng):
    """``forward_inverse`` (:36-48)."""
    x = 2 * crandn(rng, (2, 3, 20, 24))
    assert np.max(np.abs(wem.ifft2(wem.fft2(x)) - x)) < 1e-12


def test_fft_dot(rng):
    """``FFTTest.dotTest`` (:101-105): the inverse is the adjoint."""
    m = crandn(rng, (2, 3, 12, 10))
    d = crandn(rng, (2, 3, 12, 10))
    assert dot_err(m, wem.fft2(m), d, wem.ifft2(d)) < TOL


# ---------------------------------------------------------------- phase shift (propagator/tests/prop_unit_test.cpp:20-73)

def _ps_grid():
    n1, n2, n3 = 100, 100, 10   # hypercube(n1..n4) has o=0, d=1 on every axis
    kx, ky = wem.k_axis(n1, 1.0), wem.k_axis(n2, 1.0)
    w2 = wem.w2_axis(n3, 0.0, 1.0)
    sref = np.ones(n3, dtype=np.complex128)
    return kx, ky, w2, sref


def test_phase_shift_inverse_roundtrip():
    """``PS_Test.inv`` (:56-67): inverse(forward(x)) == x, rel. err <= 1e-7."""
    kx, ky, w2, sref = _ps_grid()
    x = np.ones((10, len(w2), 100, 100), dtype=np.complex128)
    P = wem.phase_forward_factor(w2, kx, ky, sref, 0.1, 0.0)
    Pi = wem.phase_inverse_factor(w2, kx, ky, sref, 0.1, 0.0)
    y = x * P[None]
    back = y * Pi[None]
    assert np.linalg.norm(back - x) / np.linalg.norm(x) <= 1e-7


def test_phase_shift_dot(rng):
    """``PS_Test.dotTest`` (:69-73) on a smaller batch."""
    kx, ky, w2, sref = _ps_grid()
    P = wem.phase_forward_factor(w2, kx, ky, sref, 0.1, 0.0)
    Q = wem.phase_adjoint_factor(w2, kx, ky, sref, 0.1, 0.0)
    m = crandn(rng, (2,) + P.shape)
    d = crandn(rng, (2,) + P.shape)
    assert dot_err(m, m * P[None], d, d * Q[None]) < TOL


def test_phase_shift_branches():
    """Evanescent waves decay; b>0 flips Re in the adjoint only
    (``propagator/src/phase_shift.cu:36-41`` vs ``:156-163``)."""
    kx = wem.k_axis(16, 1.0)
    ky = wem.k_axis(16, 1.0)
    w2 = np.array([1.0])
    P = wem.phase_forward_factor(w2, kx, ky, np.array([0.01 + 0.0j]), 1.0, 0.0)
    assert np.all(np.abs(P) <= 1.0 + 1e-15)
    assert abs(np.abs(P[0, 0, 0]) - 1.0) < 1e-15 and np.abs(P[0, 8, 8]) < 0.5
    sref = np.array([1.0 + 0.5j])  # b > 0
    Pf = wem.phase_forward_factor(w2, kx, ky, sref, 1.0, 0.0)
    Pa = wem.phase_adjoint_factor(w2, kx, ky, sref, 1.0, 0.0)
    assert not np.allclose(Pa, np.conj(Pf))


# ---------------------------------------------------------------- one step

def _small_grid(**kw):
    base = dict(nx=20, ny=16, nw=5, nz=4, dx=10.0, dy=10.0, dz=10.0, ow=2.0, dw=3.0,
                nref=3, eps=0.0, taperx=3, tapery=2)
    base.update(kw)
    return wem.Grid(**base)


def _refs(g, rng, nref=None):
    nref = nref or g.nref
    s = (1.0 / 1500.0) ** 2
    sref = np.empty((g.nz, nref, g.nw), dtype=np.complex128)
    for r in range(nref):
        sref[:, r, :] = s * (1.0 + 0.1 * r)
    labels = rng.integers(0, nref, size=(g.nz, g.nw, g.NY, g.NX))
    return sref, labels


def test_selector_dot(rng):
    """``Selector_Test.dotTest`` (prop_unit_test.cpp:187-197): self-adjoint mask."""
    labels = rng.integers(0, 3, size=(5, 10, 12))
    for v in range(3):
        m = crandn(rng, (2, 5, 10, 12))
        d = crandn(rng, (2, 5, 10, 12))
        assert dot_err(m, wem.select(labels, v, m), d, wem.select(labels, v, d)) < TOL


def test_pspi_dot_no_taper(rng):
    """``PSPI_Test.dotTest`` (prop_unit_test.cpp:147-151): the add-version pair is
    adjoint when the taper is off (the add-version adjoint has no taper,
    ``propagator/src/PSPI.cpp:26-44``)."""
    g = _small_grid(taperx=0, tapery=0)
    sref, labels = _refs(g, rng)
    m = crandn(rng, (2, g.nw, g.NY, g.NX))
    d = crandn(rng, (2, g.nw, g.NY, g.NX))
    Am = wem.pspi_forward(g, sref[1], labels[1], m)
    Atd = wem.pspi_adjoint(g, sref[1], labels[1], d)
    assert dot_err(m, Am, d, Atd) < TOL


def test_pspi_inplace_pair_dot_with_taper(rng):
    """The in-place pair (taper first / taper last, ``propagator/src/PSPI.cpp:66-103``)
    is adjoint with the taper on."""
    g = _small_grid()
    sref, labels = _refs(g, rng)
    m = crandn(rng, (2, g.nw, g.NY, g.NX))
    d = crandn(rng, (2, g.nw, g.NY, g.NX))
    Am = wem.pspi_forward(g, sref[2], labels[2], m, taper=True)
    Atd = wem.pspi_adjoint(g, sref[2], labels[2], d, taper=True)
    assert dot_err(m, Am, d, Atd) < TOL


def test_nsps_dot(rng):
    g = _small_grid()
    sref, labels = _refs(g, rng)
    m = crandn(rng, (3, g.nw, g.NY, g.NX))
    d = crandn(rng, (3, g.nw, g.NY, g.NX))
    Am = wem.nsps_forward(g, sref[0], labels[0], m)
    Atd = wem.nsps_adjoint(g, sref[0], labels[0], d)
    assert dot_err(m, Am, d, Atd) < TOL


def test_pspi_single_ref_is_phase_shift(rng):
    """With one reference and constant labels PSPI collapses to taper + FFT + phase
    shift + inverse FFT."""
    g = _small_grid(nref=1, taperx=0, tapery=0)
    sref, _ = _refs(g, rng, nref=1)
    labels = np.zeros((g.nz, g.nw, g.NY, g.NX), dtype=np.int64)
    m = crandn(rng, (1, g.nw, g.NY, g.NX))
    P = wem.phase_forward_factor(g.w2(), g.kx(), g.ky(), sref[0, 0], g.dz, g.eps)
    ref = wem.ifft2(P[None] * wem.fft2(m))
    assert np.allclose(wem.pspi_forward(g, sref[0], labels[0], m), ref, atol=1e-12)
    assert np.allclose(wem.nsps_forward(g, sref[0], labels[0], m), ref, atol=1e-12)


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_down_up_dot(rng, kind):
    """``UpDown_Test.down_dotTest`` / ``up_dotTest`` (prop_unit_test.cpp:314-340)."""
    g = _small_grid()
    sref, labels = _refs(g, rng)
    st = wem.Stepper(g, sref, labels, kind)
    m = crandn(rng, (2, g.nw, g.NY, g.NX))
    d = crandn(rng, (2, g.nw, g.NY, g.NX))
    if kind == "pspi":
        assert dot_err(m, wem.downward(st, g.nz, m), d, wem.downward_adjoint(st, g.nz, d)) < TOL
        assert dot_err(m, wem.upward(st, g.nz, m), d, wem.upward_adjoint(st, g.nz, d)) < TOL
    else:
        # NSPS in place has no taper and is adjoint step by step as well
        assert dot_err(m, wem.downward(st, g.nz, m), d, wem.downward_adjoint(st, g.nz, d)) < TOL


# ---------------------------------------------------------------- injection (prop_unit_test.cpp:199-262)

def _acq_grid(rng, g, ntrace=20, ns=5):
    cx = rng.uniform(g.ox + g.dx, (g.NX - 2) * g.dx, ntrace)
    cy = rng.uniform(g.oy + g.dy, (g.NY - 2) * g.dy, ntrace)
    cz = rng.uniform(g.oz + g.dz, (g.nz - 2) * g.dz, ntrace)
    ids = rng.integers(0, ns, ntrace)
    return cx, cy, cz, ids


def test_injection_dot(rng):
    g = _small_grid(nz=10)
    cx, cy, cz, ids = _acq_grid(rng, g)
    tr = wem.make_traces(cx, cy, cz, ids, g.ox, g.oy, g.dx, g.dy, g.oz, g.dz, g.NX, g.NY)
    for iz in range(g.nz):
        m = crandn(rng, (20, g.nw))
        d = crandn(rng, (5, g.nw, g.NY, g.NX))
        Am = wem.inject(tr, m, np.zeros_like(d), iz)
        Atd = wem.record(tr, d, np.zeros_like(m), iz)
        if not np.any(Am):
            assert not np.any(Atd)  # no trace touches this depth level
            continue
        assert dot_err(m, Am, d, Atd) < TOL


def test_injection_skip_and_weights():
    """Traces on the last row/column are dropped (``propagator/src/injection.cu:46-48``);
    on-node traces put weight lz on one node only."""
    g = _small_grid(nz=4)
    cx = [0.0, (g.NX - 1) * g.dx, 30.0]
    cy = [0.0, 0.0, (g.NY - 1) * g.dy]
    tr = wem.make_traces(cx, cy, [0.0] * 3, [0, 0, 0], g.ox, g.oy, g.dx, g.dy, g.oz, g.dz, g.NX, g.NY)
    assert list(tr.valid) == [True, False, False]
    wav = np.ones((3, g.nw), dtype=np.complex128)
    w = wem.inject(tr, wav, np.zeros((1, g.nw, g.NY, g.NX), dtype=np.complex128), 0)
    assert w[0, 0, 0, 0] == 1.0 and np.count_nonzero(w[0, 0]) == 1


# ---------------------------------------------------------------- reflection / scattering / imaging

def _model(g, rng, const=False):
    s = (1.0 / 1500.0) ** 2
    if const:
        slow = np.full((g.nz, g.nw, g.ny, g.nx), s, dtype=np.complex128)
    else:
        slow = s * (1 + 0.2 * rng.random((g.nz, g.nw, g.ny, g.nx))) + 0j
    den = 1.0 + 0.3 * rng.random((g.nz, g.nw, g.ny, g.nx)) + 0j
    return slow, den


def test_reflect_dot(rng):
    """``Reflect_Test.dot`` (prop_unit_test.cpp:393-401), padded wavefield."""
    g = _small_grid(padx=4, pady=3, nz=6)
    slow, den = _model(g, rng)
    for iz in range(g.nz - 1):
        m = crandn(rng, (2, g.nw, g.NY, g.NX))
        d = crandn(rng, (2, g.nw, g.NY, g.NX))
        Am = wem.reflect_forward(g, slow, den, iz, m, np.zeros_like(d))
        Atd = wem.reflect_adjoint(g, slow, den, iz, d, np.zeros_like(m))
        assert dot_err(m, Am, d, Atd) < TOL
    assert np.all(wem.reflect_coef(*wem.model_pair(slow, g.nz - 1), *wem.model_pair(den, g.nz - 1)) == 0)


def test_scatter_dot(rng):
    """``Scatter_Test.dotTest`` (born_unit_test.cpp:60-64)."""
    g = _small_grid(padx=3, pady=2, taylor=2)
    slow, _ = _model(g, rng)
    m = crandn(rng, (2, g.nw, g.NY, g.NX))
    d = crandn(rng, (2, g.nw, g.NY, g.NX))
    Am = wem.scatter_forward(g, slow[1], m)
    Atd = wem.scatter_adjoint(g, slow[1], d)
    assert dot_err(m, Am, d, Atd) < TOL


def test_ic_dot(rng):
    """``IC_Test.dotTest`` (born_unit_test.cpp:118-124)."""
    g = _small_grid(padx=2, pady=2)
    bg = crandn(rng, (3, g.nw, g.NY, g.NX))
    m = crandn(rng, (g.nw, g.ny, g.nx))
    d = crandn(rng, (3, g.nw, g.NY, g.NX))
    Am = wem.ic_forward(g, bg, m, np.zeros_like(d))
    Atd = wem.ic_adjoint(g, bg, d, np.zeros_like(m))
    assert dot_err(m, Am, d, Atd) < TOL


def test_lin_reflect_dot(rng):
    """``LinReflect_Test.dot`` (born_unit_test.cpp:181-185)."""
    g = _small_grid(nz=5)
    slow, den = _model(g, rng)
    for iz in (1, g.nz - 1):
        m = [crandn(rng, (g.nw, g.ny, g.nx)) for _ in range(4)]
        d = crandn(rng, (g.nw, g.ny, g.nx))
        Am = wem.lin_reflect_forward(slow, den, iz, m)
        Atd = wem.lin_reflect_adjoint(slow, den, iz, d)
        lhs = np.vdot(d.ravel(), Am.ravel())
        rhs = sum(np.vdot(b.ravel(), a.ravel()) for a, b in zip(m, Atd))
        assert abs((lhs / rhs).real - 1) < TOL


def _born_setup(rng, kind="pspi", padx=0, taper=2):
    g = _small_grid(nz=6, nx=16, ny=12, nw=3, padx=padx, pady=padx, taperx=taper, tapery=taper)
    sref, labels = _refs(g, rng)
    slow, den = _model(g, rng)
    slow[g.nz - 2:] *= 2.0
    st = wem.Stepper(g, sref, labels, kind)
    geom = dict(sx=[40.0, 90.0], sy=[50.0, 50.0], sz=[10.0, 10.0], s_ids=[7, 3],
                rx=list(np.linspace(10, 130, 8)), ry=[50.0] * 8, rz=[10.0] * 8,
                r_ids=[7, 3] * 4)
    acq = wem.make_acquisition(g, geom)
    wav = crandn(rng, (2, g.nw))
    data, bgd, bgu = wem.propagate(g, st, acq, slow, den, wav)
    return g, st, acq, slow, den, bgd, bgu, data


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_extended_born_dot(rng, kind):
    """``ExtendedBorn_Test.dotTest`` (born_unit_test.cpp:432-436; the operator's own
    dot test ``propagator/src/ExtendedBorn.h:61-128``) over all four sweeps, with the
    taper off as in that test (born_unit_test.cpp:392-393)."""
    g, st, acq, slow, den, bgd, bgu, data = _born_setup(rng, kind, padx=2, taper=0)
    assert np.linalg.norm(data) > 0
    ms = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
    mr = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
    d = crandn(rng, data.shape)
    Am = wem.born_forward(g, st, acq, slow, den, bgd, bgu, ms, mr)
    gs, gr = wem.born_adjoint(g, st, acq, slow, den, bgd, bgu, d)
    lhs = np.vdot(d.ravel(), Am.ravel())
    rhs = np.vdot(gs.ravel(), ms.ravel()) + np.vdot(gr.ravel(), mr.ravel())
    assert abs((lhs / rhs).real - 1) < 1e-9


def test_migrate_is_back_scattering_ic(rng):
    """The lockstep migration image equals sum_w Re of the back-scattering adjoint's
    imaging-condition output (``propagator/src/Scattering.cpp:104-111``)."""
    g, st, acq, slow, den, bgd, bgu, data = _born_setup(rng)
    img = wem.migrate(g, st, acq, crandn(np.random.default_rng(5), (2, g.nw)) * 0 + 1, data)
    assert img.shape == (g.nz, g.ny, g.nx) and np.isfinite(img).all()
    wav = np.ones((2, g.nw), dtype=np.complex128)
    _, bgd1, _ = wem.propagate(g, st, acq, slow, den, wav)
    bu = np.zeros_like(bgd1[0])
    for iz in range(g.nz):
        bu = wem.inject(acq.rec, data, bu, iz)
        I = wem.ic_adjoint(g, bgd1[iz], bu, np.zeros((g.nw, g.ny, g.nx), dtype=np.complex128))
        assert np.allclose(np.real(I).sum(0), img[iz], atol=1e-12)
        bu = st.adj(iz, bu)


def test_extended_born_taper_quirk(rng):
    """With a taper the reference's Born pair is not adjoint: the forward-scattering
    step uses the tapered PSPI forward (``propagator/src/PSPI.cpp:6-24``) but the
    untapered add-version adjoint (``propagator/src/PSPI.cpp:26-44``).  The oracle
    keeps that behaviour."""
    g, st, acq, slow, den, bgd, bgu, data = _born_setup(rng, "pspi", padx=2, taper=2)
    ms = crandn(rng, (g.nz, g.nw, g.ny, g.nx))
    mr = np.zeros_like(ms)
    d = crandn(rng, data.shape)
    Am = wem.born_forward(g, st, acq, slow, den, bgd, bgu, ms, mr)
    gs, gr = wem.born_adjoint(g, st, acq, slow, den, bgd, bgu, d)
    ratio = np.vdot(d.ravel(), Am.ravel()) / np.vdot(gs.ravel(), ms.ravel())
    assert abs(ratio.real - 1) > 1e-6


def test_smooth_step_dot_and_derivative(rng):
    g = wem.Grid(nx=16, ny=12, nw=3, nz=3, dx=10, dy=10, dz=10, ow=5, dw=4, padx=4, pady=4, nref=3, taperx=2,
                 tapery=2)
    s = 1 / 1800 * (1 + 0.1 * rng.random((g.nz, g.ny, g.nx)))
    refs = wem.smooth_refs(s, g.nref)
    sp = wem.pad_edge(g, s)
    x = crandn(rng, (2, g.nw, g.NY, g.NX))
    y = crandn(rng, x.shape)
    a = np.vdot(y, wem.smooth_forward(g, refs[1], sp[1], x))
    b = np.vdot(wem.smooth_adjoint(g, refs[1], sp[1], y), x)
    assert abs(a / b - 1) < 1e-12
    k = (1, 5, 7)
    h = 1e-7 * s[k]

    def step_with(v):
        ss = s.copy()
        ss[k] = v
        return wem.smooth_forward(g, refs[1], wem.pad_edge(g, ss)[1], x)
    fd = (step_with(s[k] + h) - step_with(s[k] - h)) / (2 * h)
    der = wem.smooth_deriv(g, refs[1], sp[1], x)
    assert np.abs(fd[:, :, 5, 7] - der[:, :, 5, 7]).max() < 1e-6 * np.abs(der[:, :, 5, 7]).max()


def test_smooth_gradient_matches_central_differences(rng):
    """The adjoint-state gradient of the FP64 oracle against central finite
    differences of its objective (references fixed), relative step 1e-6."""
    g = wem.Grid(nx=16, ny=12, nw=3, nz=4, dx=10, dy=10, dz=10, ow=5, dw=4, padx=4, pady=4, nref=3, taperx=2,
                 tapery=2)
    s = 1 / 1800 * (1 + 0.1 * rng.random((g.nz, g.ny, g.nx)))
    s[2:] *= 1.3
    refs = wem.smooth_refs(s, g.nref)
    geom = dict(sx=[70.0], sy=[50.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, 150, 10)), ry=[60.0] * 10,
                rz=[0.0] * 10, r_ids=[0] * 10)
    acq = wem.make_acquisition(g, geom)
    wav = crandn(rng, (1, g.nw))
    d_obs = wem.smooth_propagate(g, refs, s * 1.02, acq, wav)[0]
    J, grad = wem.smooth_gradient(g, refs, s, acq, wav, d_obs)
    cells = [(0, 3, 4), (1, 6, 7), (2, 11, 15), (2, 5, 5), (3, 8, 2), (1, 0, 15)]
    for k in cells:
        h = 1e-6 * s[k]
        sp_, sm_ = s.copy(), s.copy()
        sp_[k] += h
        sm_[k] -= h
        fd = (wem.smooth_objective(g, refs, sp_, acq, wav, d_obs) -
              wem.smooth_objective(g, refs, sm_, acq, wav, d_obs)) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(grad).max()), (k, grad[k], fd)
