"""The oracle against pyfwix's own CUDA kernels.

Every output of tests/golden/reference_kernels_<regime>.npz (phase shift fwd /
adj / inv, taper, select, PSPI fwd / add-adjoint / in-place adjoint, NSPS fwd /
adj, injection and recording, reflect, imaging condition, linearised
reflection, scatter fwd / adj) is recomputed by the FP64 oracle from the
fixture's inputs.

* ``real`` regime (real slowness, density and references, eps = 0: every
  benchmark configuration): the reference's float arithmetic is well
  conditioned, and the oracle must agree to 2e-6 relative L2 (float rounding).
* ``complex`` regime (complex slowness / references, eps = 0.01): the
  reference forms Re and Im of kz as sqrt((c +- a) / 2) (phase_shift.cu:38-41)
  and complex roots as sqrt((r +- a) / 2) (prop_kernels.cuh:89-102), which
  cancel in float when |b| << |a| (most of the spectrum is evanescent on this
  grid); its output then carries relative errors of 2e-5 (phase shift) to
  1.5e-4 (reflection), against 3e-7 for the same operators in the real
  regime.  The oracle must agree to 3e-4 there: a sign, branch or
  normalisation difference would show as an O(1) error."""

import numpy as np
import pytest

from oracle import wem
from tests.golden_case import REGIMES, c128, load

CASES = {r: load(r) for r in REGIMES}
TOL = {"real": 2e-6, "complex": 3e-4}


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def _case(regime):
    c = CASES[regime]
    if c is None:
        pytest.skip("golden fixture not generated")
    return c


@pytest.mark.parametrize("regime", REGIMES)
def test_phase_shift_modes(regime):
    g, gd, f = _case(regime)
    x = c128(f["x"])
    args = (g.w2(), g.kx(), g.ky(), c128(f["sref"][1]), g.dz, g.eps)
    assert rel(x * wem.phase_forward_factor(*args)[None], f["out_ps_fwd"]) < TOL[regime]
    assert rel(x * wem.phase_adjoint_factor(*args)[None], f["out_ps_adj"]) < TOL[regime]
    assert rel(x * wem.phase_inverse_factor(*args)[None], f["out_ps_inv"]) < TOL[regime]


@pytest.mark.parametrize("regime", REGIMES)
def test_taper_and_select(regime):
    g, gd, f = _case(regime)
    x = c128(f["x"])
    assert rel(x * g.taper()[None, None], f["out_taper"]) < 2e-6
    assert rel(wem.select(f["labels"], 1, x), f["out_select1"]) == 0.0


@pytest.mark.parametrize("regime", REGIMES)
def test_pspi_and_nsps(regime):
    g, gd, f = _case(regime)
    x, y = c128(f["x"]), c128(f["y"])
    sr, lab = c128(f["sref"]), f["labels"].astype(np.int64)
    tol = TOL[regime]
    assert rel(wem.pspi_forward(g, sr, lab, x, taper=True), f["out_pspi_fwd"]) < tol
    assert rel(wem.pspi_adjoint(g, sr, lab, y, taper=False), f["out_pspi_adj"]) < tol
    assert rel(wem.pspi_adjoint(g, sr, lab, y, taper=True), f["out_pspi_adj_inplace"]) < tol
    assert rel(wem.nsps_forward(g, sr, lab, x), f["out_nsps_fwd"]) < tol
    assert rel(wem.nsps_adjoint(g, sr, lab, y), f["out_nsps_adj"]) < tol


@pytest.mark.parametrize("regime", REGIMES)
@pytest.mark.parametrize("iz", [1, 2])
def test_injection_and_recording(regime, iz):
    g, gd, f = _case(regime)
    tr = wem.make_traces(f["cx"], f["cy"], f["cz"], f["ids"], g.ox, g.oy, g.dx, g.dy, g.oz, g.dz, g.NX, g.NY)
    inj = wem.inject(tr, c128(f["traces"]), np.zeros(f["x"].shape, np.complex128), iz)
    assert rel(inj, f[f"out_inject_z{iz}"]) < 2e-6
    rec = wem.record(tr, c128(f["y"]), np.zeros(f["traces"].shape, np.complex128), iz)
    assert rel(rec, f[f"out_record_z{iz}"]) < 2e-6


@pytest.mark.parametrize("regime", REGIMES)
def test_reflect_imaging_linreflect(regime):
    g, gd, f = _case(regime)
    x, y = c128(f["x"]), c128(f["y"])
    slow, den = c128(f["slow2"]), c128(f["den2"])          # levels z, z+1 as a 2-level model
    tol = TOL[regime]
    assert rel(wem.reflect_forward(g, slow, den, 0, x, np.zeros_like(x)), f["out_reflect_fwd"]) < tol
    assert rel(wem.reflect_adjoint(g, slow, den, 0, y, np.zeros_like(y)), f["out_reflect_adj"]) < tol
    img = c128(f["image"])
    assert rel(wem.ic_forward(g, x, img, np.zeros_like(x)), f["out_ic_fwd"]) < 2e-6
    assert rel(wem.ic_adjoint(g, x, y, np.zeros_like(img)), f["out_ic_adj"]) < 2e-6
    dm = c128(f["dm4"])
    assert rel(wem.lin_reflect_forward(slow, den, 0, dm), f["out_lin_reflect_fwd"]) < tol
    got = np.stack(wem.lin_reflect_adjoint(slow, den, 0, c128(f["dr_in"])))
    assert rel(got, f["out_lin_reflect_adj"]) < tol


@pytest.mark.parametrize("regime", REGIMES)
def test_scatter(regime):
    g, gd, f = _case(regime)
    s = c128(f["slow2"][0])
    assert rel(wem.scatter_forward(g, s, c128(f["x"])), f["out_scatter_fwd"]) < 2e-6
    assert rel(wem.scatter_adjoint(g, s, c128(f["y"])), f["out_scatter_adj"]) < 2e-6
