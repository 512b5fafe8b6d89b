"""Parity of every CUDA operator of the path with the FP64 oracle (relative L2 on
the same seeded inputs).  Tolerances: 1e-5 for one operator application, as the
per-step bound of the reference tests (prop_unit_test.cpp:18)."""
import numpy as np
import pytest
import torch

from oracle import wem
from tests.conftest import crandn, dot_err
from tests.gpu_helpers import make_case, make_plan, oracle_labels, rel, to_dev, to_host, wavefield

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.mark.parametrize("NX,NY", [(16, 16), (20, 12), (100, 100), (128, 128), (192, 40), (320, 24),
                                   (384, 10), (512, 8), (1000, 4), (30, 1024), (1, 8), (96, 160), (160, 96),
                                   (640, 384), (384, 192), (64, 640), (20, 320)])
def test_fft2d(NX, NY):
    """cuFFT2d forward / adjoint (operator/src/FFT.cpp:36-55) and the FFT tests of
    operator/tests/operator_unit_test.cpp:36-99."""
    g, rng, sref, labels, _, _ = make_case(nx=NX, ny=NY, nw=3, nz=1, nref=1)
    p = make_plan(g, 2, sref, labels)
    x = wavefield(rng, 2, g)
    y = to_host(p.fft2d(to_dev(x), torch.empty(p.wshape, dtype=torch.complex64, device="cuda")))
    assert rel(y, wem.fft2(x)) < TOL
    z = to_host(p.fft2d(to_dev(x), torch.empty(p.wshape, dtype=torch.complex64, device="cuda"), inverse=True))
    assert rel(z, wem.ifft2(x)) < TOL
    # add semantics
    acc = to_dev(x)
    p.fft2d(to_dev(x), acc, add=True)
    assert rel(to_host(acc), x + wem.fft2(x)) < TOL


def test_fft_known_answers():
    """DC of a constant = sqrt(n1 n2); plane wave spike at (10, 20)
    (operator/tests/operator_unit_test.cpp:50-99)."""
    g, rng, sref, labels, _, _ = make_case(nx=100, ny=100, nw=2, nz=1, nref=1)
    p = make_plan(g, 1, sref, labels)
    ones = torch.ones(p.wshape, dtype=torch.complex64, device="cuda")
    y = to_host(p.fft2d(ones, torch.empty_like(ones)))
    assert abs(y[0, 0, 0, 0].real - 100.0) < 1e-4 and np.max(np.abs(y.imag)) < 1e-4
    i1 = np.arange(100)[None, :]
    i2 = np.arange(100)[:, None]
    pw = np.exp(1j * 2 * np.pi * (10 * i1 / 100 + 20 * i2 / 100))[None, None].repeat(2, axis=1)
    y = to_host(p.fft2d(to_dev(pw), torch.empty_like(ones)))
    assert abs(y[0, 0, 20, 10].real - 100.0) < 1e-3
    y[0, :, 20, 10] = 0
    assert np.max(np.abs(y)) < 1e-3


@pytest.mark.parametrize("complex_refs,eps", [(False, 0.0), (True, 0.0), (False, 0.05)])
def test_phase_shift(complex_refs, eps):
    g, rng, sref, labels, _, _ = make_case(nx=32, ny=24, nw=4, nz=1, nref=1, eps=eps, complex_refs=complex_refs)
    p = make_plan(g, 2, sref, labels)
    x = wavefield(rng, 2, g)
    s = sref[0, 0]
    kx, ky, w2 = g.kx(), g.ky(), g.w2()
    out = torch.empty(p.wshape, dtype=torch.complex64, device="cuda")
    for mode, fac in ((0, wem.phase_forward_factor), (1, wem.phase_adjoint_factor), (2, wem.phase_inverse_factor)):
        y = to_host(p.phase_shift(s, to_dev(x), out, mode=mode))
        assert rel(y, x * fac(w2, kx, ky, s, g.dz, g.eps)[None]) < TOL, mode


def test_phase_shift_inverse_roundtrip():
    """PS_Test.inv (propagator/tests/prop_unit_test.cpp:56-67) on the device."""
    from pyfwix_b200.plan import Plan
    p = Plan(nx=100, ny=100, nw=10, ns=3, nz=1, dx=1.0, dy=1.0, dz=0.1, ow=0.0, dw=1.0)
    ones = torch.ones(p.wshape, dtype=torch.complex64, device="cuda")
    s = np.ones(10, dtype=np.complex64)
    fw = p.phase_shift(s, ones, torch.empty_like(ones), mode=0)
    back = to_host(p.phase_shift(s, fw, torch.empty_like(ones), mode=2))
    assert rel(back, np.ones(p.wshape)) <= 1e-7


def test_select_and_taper():
    g, rng, sref, labels, _, _ = make_case(nx=24, ny=20, nw=4, nz=3, nref=3, padx=4, pady=4)
    p = make_plan(g, 2, sref, labels)
    x = wavefield(rng, 2, g)
    out = torch.empty(p.wshape, dtype=torch.complex64, device="cuda")
    for iz in range(g.nz):
        for v in range(3):
            y = to_host(p.select(iz, v, to_dev(x), out))
            assert np.array_equal(y, wem.select(labels[iz], v, x).astype(np.complex64))
    y = to_host(p.taper(to_dev(x), out))
    assert rel(y, g.taper()[None, None] * x) < 1e-6


STEP_CASES = [
    dict(nx=24, ny=20, padx=0, pady=0, eps=0.0, complex_refs=False, labels_per_w=True),
    dict(nx=192, ny=320, padx=0, pady=0, eps=0.0, complex_refs=False, labels_per_w=True),
    dict(nx=380, ny=100, padx=4, pady=0, eps=0.01, complex_refs=True, labels_per_w=False),
    dict(nx=32, ny=28, padx=8, pady=4, eps=0.02, complex_refs=True, labels_per_w=False),
    dict(nx=100, ny=60, padx=28, pady=4, eps=0.0, complex_refs=False, labels_per_w=False),
    dict(nx=256, ny=256, padx=0, pady=0, eps=0.0, complex_refs=False, labels_per_w=False),
    dict(nx=248, ny=252, padx=8, pady=4, eps=0.01, complex_refs=True, labels_per_w=True),
    dict(nx=380, ny=380, padx=4, pady=4, eps=0.0, complex_refs=False, labels_per_w=False),
    dict(nx=96, ny=160, padx=0, pady=0, eps=0.01, complex_refs=True, labels_per_w=True),
]


@pytest.mark.parametrize("case", STEP_CASES)
def test_pspi_step(case):
    """PSPI forward (PSPI.cpp:6-24, :66-83) and both adjoint forms (:26-44, :85-103)."""
    g, rng, sref, labels, _, _ = make_case(nw=4, nz=3, nref=4, **case)
    lab = oracle_labels(labels, g)
    p = make_plan(g, 2, sref, labels)
    x = wavefield(rng, 2, g)
    d0 = wavefield(rng, 2, g)
    for iz in range(g.nz):
        out = to_dev(d0)
        y = to_host(p.step(iz, to_dev(x), out, direction=0, add=True))
        assert rel(y, wem.pspi_forward(g, sref[iz], lab[iz], x, d0)) < TOL
        y = to_host(p.step(iz, to_dev(x), torch.empty_like(out), direction=1))
        assert rel(y, wem.pspi_adjoint(g, sref[iz], lab[iz], x)) < TOL
        y = to_host(p.step(iz, to_dev(x), torch.empty_like(out), direction=2))
        assert rel(y, wem.pspi_adjoint(g, sref[iz], lab[iz], x, taper=True)) < TOL
        xin = to_dev(x)
        y = to_host(p.step(iz, xin, xin, direction=0))  # in place
        assert rel(y, wem.pspi_forward(g, sref[iz], lab[iz], x)) < TOL


@pytest.mark.parametrize("case", STEP_CASES)
def test_nsps_step(case):
    """NSPS forward / adjoint (NSPS.cpp:6-45)."""
    g, rng, sref, labels, _, _ = make_case(nw=4, nz=2, nref=3, **case)
    lab = oracle_labels(labels, g)
    p = make_plan(g, 3, sref, labels, step="nsps")
    x = wavefield(rng, 3, g)
    d0 = wavefield(rng, 3, g)
    for iz in range(g.nz):
        y = to_host(p.step(iz, to_dev(x), to_dev(d0), direction=0, add=True))
        assert rel(y, wem.nsps_forward(g, sref[iz], lab[iz], x, d0)) < TOL
        y = to_host(p.step(iz, to_dev(x), to_dev(d0), direction=1, add=True))
        assert rel(y, wem.nsps_adjoint(g, sref[iz], lab[iz], x, d0)) < TOL


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_fused_step_matches_three_launch_step(kind, monkeypatch):
    """The 256 x 256 cluster step against the three-launch step on the same
    inputs (FWIX_FUSED=1 at plan creation selects the former), in place and
    with accumulation, every direction."""
    g, rng, sref, labels, _, _ = make_case(nx=256, ny=256, nw=3, nz=2, nref=4, padx=0, pady=0, eps=0.01,
                                           complex_refs=True, labels_per_w=False, taperx=20, tapery=20)
    p_three = make_plan(g, 2, sref, labels, step=kind)
    monkeypatch.setenv("FWIX_FUSED", "1")
    p_fused = make_plan(g, 2, sref, labels, step=kind)
    x = wavefield(rng, 2, g)
    d0 = wavefield(rng, 2, g)
    for direction in (0, 1, 2):
        a = to_host(p_fused.step(1, to_dev(x), to_dev(d0), direction=direction, add=True))
        b = to_host(p_three.step(1, to_dev(x), to_dev(d0), direction=direction, add=True))
        assert rel(a, b) < 1e-5, (direction, rel(a, b))
        xin = to_dev(x)
        a = to_host(p_fused.step(0, xin, xin, direction=direction))
        assert rel(a, to_host(p_three.step(0, to_dev(x), to_dev(d0), direction=direction))) < 1e-5


def test_step_dot_product():
    """Device dot tests of the in-place PSPI pair and the NSPS pair."""
    g, rng, sref, labels, _, _ = make_case(nx=48, ny=40, nw=3, nz=1, nref=4, padx=0)
    for kind, fwd, adj in (("pspi", 0, 2), ("nsps", 0, 1)):
        p = make_plan(g, 2, sref, labels, step=kind)
        m = wavefield(rng, 2, g)
        d = wavefield(rng, 2, g)
        Am = to_host(p.step(0, to_dev(m), torch.empty(p.wshape, dtype=torch.complex64, device="cuda"), direction=fwd))
        Atd = to_host(p.step(0, to_dev(d), torch.empty(p.wshape, dtype=torch.complex64, device="cuda"), direction=adj))
        assert dot_err(m, Am, d, Atd) < 1e-5


@pytest.mark.parametrize("taylor,pad,nx,ny", [(0, 0, 24, 20), (1, 0, 24, 20), (2, 8, 24, 20), (1, 0, 128, 64),
                                              (2, 8, 120, 60)])
def test_scatter(taylor, pad, nx, ny):
    """Scatter forward / adjoint (Scatter.cpp:76-102), padded slowness replicated
    into the pad (scatter.cu:240-277)."""
    g, rng, sref, labels, slow, den = make_case(nx=nx, ny=ny, nw=4, nz=3, padx=pad, pady=pad // 2, taylor=taylor)
    p = make_plan(g, 2, sref, labels, slow, den)
    x = wavefield(rng, 2, g)
    d0 = wavefield(rng, 2, g)
    for iz in (0, 2):
        y = to_host(p.scatter(iz, to_dev(x), to_dev(d0), add=True))
        assert rel(y, wem.scatter_forward(g, slow[iz], x, d0)) < TOL
        y = to_host(p.scatter(iz, to_dev(x), to_dev(d0), adjoint=True, add=True))
        assert rel(y, wem.scatter_adjoint(g, slow[iz], x, d0)) < TOL
        xin = to_dev(x)
        y = to_host(p.scatter(iz, xin, xin))  # in place (Scatter.cpp:104-116)
        assert rel(y, wem.scatter_forward(g, slow[iz], x)) < TOL


def test_reflect_ic_linreflect():
    g, rng, sref, labels, slow, den = make_case(nx=24, ny=20, nw=4, nz=4, padx=6, pady=4)
    p = make_plan(g, 2, sref, labels, slow, den)
    x = wavefield(rng, 2, g)
    d0 = wavefield(rng, 2, g)
    for iz in range(g.nz):
        y = to_host(p.reflect(iz, to_dev(x), to_dev(d0), add=True))
        assert rel(y, wem.reflect_forward(g, slow, den, iz, x, d0)) < TOL
        y = to_host(p.reflect(iz, to_dev(x), to_dev(d0), adjoint=True))
        assert rel(y, wem.reflect_adjoint(g, slow, den, iz, x, np.zeros_like(x))) < TOL
    bg = wavefield(rng, 2, g)
    img = crandn(rng, (g.nw, g.ny, g.nx))
    w = to_dev(d0)
    p.imaging(to_dev(bg), to_dev(img), w, add=True)
    assert rel(to_host(w), wem.ic_forward(g, bg, img, d0)) < TOL
    im = to_dev(img)
    p.imaging(to_dev(bg), im, to_dev(x), adjoint=True, add=True)
    assert rel(to_host(im), wem.ic_adjoint(g, bg, x, img)) < TOL
    dm = crandn(rng, (4, g.nw, g.ny, g.nx))
    for iz in (1, g.nz - 1):
        dr = torch.empty((g.nw, g.ny, g.nx), dtype=torch.complex64, device="cuda")
        p.lin_reflect(iz, to_dev(dm), dr)
        assert rel(to_host(dr), wem.lin_reflect_forward(slow, den, iz, list(dm))) < TOL
        r = crandn(rng, (g.nw, g.ny, g.nx))
        out = torch.zeros((4, g.nw, g.ny, g.nx), dtype=torch.complex64, device="cuda")
        p.lin_reflect(iz, out, to_dev(r), adjoint=True, add=True)
        assert rel(to_host(out), np.stack(wem.lin_reflect_adjoint(slow, den, iz, r))) < TOL


def test_injection_record():
    """Injection fwd / adj (injection.cu:7-188) with overlapping traces on one shot,
    traces on the skipped last row/column, and out-of-level traces."""
    g, rng, sref, labels, _, _ = make_case(nx=20, ny=16, nw=3, nz=6, padx=4, pady=2)
    p = make_plan(g, 3, sref, labels)
    n = 60
    cx = rng.uniform(0, (g.NX - 1) * g.dx, n)
    cy = rng.uniform(0, (g.NY - 1) * g.dy, n)
    cz = rng.uniform(0, (g.nz - 1) * g.dz, n)
    cx[:5] = (g.NX - 1) * g.dx  # dropped
    cx[5:15] = 30.0  # dense overlap
    cy[5:15] = 24.0
    ids = rng.integers(0, 3, n)
    ids[5:15] = 1
    tr_o = wem.make_traces(cx, cy, cz, ids, g.ox, g.oy, g.dx, g.dy, g.oz, g.dz, g.NX, g.NY)
    tr = p.traces(cx, cy, cz, ids)
    trace = crandn(rng, (n, g.nw))
    for iz in range(g.nz):
        w = torch.zeros(p.wshape, dtype=torch.complex64, device="cuda")
        p.inject(tr, iz, to_dev(trace), w)
        ref = wem.inject(tr_o, trace, np.zeros((3, g.nw, g.NY, g.NX), dtype=np.complex128), iz)
        assert np.linalg.norm(to_host(w) - ref) <= TOL * max(np.linalg.norm(ref), 1.0)
        wf = wavefield(rng, 3, g)
        d = torch.zeros((n, g.nw), dtype=torch.complex64, device="cuda")
        p.inject(tr, iz, d, to_dev(wf), adjoint=True)
        ref = wem.record(tr_o, wf, np.zeros_like(trace), iz)
        assert np.linalg.norm(to_host(d) - ref) <= TOL * max(np.linalg.norm(ref), 1.0)


@pytest.mark.parametrize("chunk", ["1", "3"])
def test_chunked_steps(monkeypatch, chunk):
    """Steps and the Born scatter run in chunks of slices whose intermediates stay in
    L2; forcing small chunks must not change the result."""
    monkeypatch.setenv("FWIX_CHUNK_SLICES", chunk)
    g, rng, sref, labels, slow, den = make_case(nx=64, ny=40, nw=4, nz=2, nref=3, padx=0, pady=0)
    lab = oracle_labels(labels, g)
    for kind in ("pspi", "nsps"):
        p = make_plan(g, 2, sref, labels, slow, den, step=kind)
        x = wavefield(rng, 2, g)
        fwd = wem.pspi_forward if kind == "pspi" else wem.nsps_forward
        y = to_host(p.step(1, to_dev(x), torch.empty(p.wshape, dtype=torch.complex64, device="cuda")))
        assert rel(y, fwd(g, sref[1], lab[1], x)) < TOL
        y = to_host(p.scatter(1, to_dev(x), torch.empty(p.wshape, dtype=torch.complex64, device="cuda"), adjoint=True))
        assert rel(y, wem.scatter_adjoint(g, slow[1], x)) < TOL
        y = to_host(p.fft2d(to_dev(x), torch.empty(p.wshape, dtype=torch.complex64, device="cuda"), inverse=True))
        assert rel(y, wem.ifft2(x)) < TOL


@pytest.mark.parametrize("complex_refs,eps", [(False, 0.0), (True, 0.03)])
def test_phase_cache_matches_inline(complex_refs, eps):
    """Steps read the cached factors when a phase cache is bound; results equal
    the in-kernel evaluation, including the adjoint's b > 0 branch."""
    g, rng, sref, labels, _, _ = make_case(nx=64, ny=64, nw=4, nz=3, nref=3, eps=eps, complex_refs=complex_refs)
    if complex_refs:
        sref = sref.copy()
        sref[:, 1, :] += 1j * abs(sref[:, 1, :]) * 0.3  # Im s2 > eps Re s2: b > 0 for this reference
    x = wavefield(rng, 2, g)
    outs = {}
    for cached in (False, True):
        for kind in ("pspi", "nsps"):
            p = make_plan(g, 2, sref, labels, step=kind)
            if not cached:
                p.disable_phase_cache()
            else:
                assert "pcache" in p._keep
            for d in (0, 1, 2):
                for iz in (2, 0, 2):
                    outs[(cached, kind, d, iz)] = to_host(p.step(iz, to_dev(x), torch.empty(p.wshape, dtype=torch.complex64,
                                                                                            device="cuda"), direction=d))
    for k, v in outs.items():
        if k[0]:
            assert rel(v, outs[(False,) + k[1:]]) < 1e-6, k

