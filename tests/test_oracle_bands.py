"""The band-by-band oracle runs of ``tests/oracle_bands.py`` equal one run over all
frequencies: data and Born outputs concatenated over frequency, images,
gradients and the misfit summed."""
import numpy as np
import pytest

from oracle import wem
from tests import oracle_bands
from tests.conftest import crandn


def _setup(kind="pspi", nw=5):
    rng = np.random.default_rng(4)
    g = wem.Grid(nx=20, ny=16, nw=nw, nz=4, dx=10.0, dy=10.0, dz=10.0, ow=3.0, dw=2.0, padx=4, pady=2, nref=3,
                 taperx=2, tapery=2, taylor=1)
    s2 = (1 / 1800.0) ** 2 * (1 + 0.3 * rng.random((g.nz, g.ny, g.nx)))
    s2[2:] *= 1.5
    sref = np.repeat(((1 / 1800.0) ** 2 * np.array([1.0, 1.15, 1.4]))[None, :, None], g.nz, 0)
    sref = np.repeat(sref, g.nw, 2).astype(np.complex128)
    labels = rng.integers(0, 3, (g.nz, g.NY, g.NX))
    geom = dict(sx=[100.0], sy=[80.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, 190, 7)), ry=[70.0] * 7,
                rz=[0.0] * 7, r_ids=[0] * 7)
    args = dict(geom=geom, kind=kind, s2=s2, labels=labels, sref=sref, wavelet=crandn(rng, (1, g.nw)))
    return g, rng, args


def _serial(task, g, args):
    return oracle_bands._job(task, g, 0, g.nw, args)


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_banded_born_and_model_equal_one_run(kind):
    g, rng, a = _setup(kind)
    a = dict(a, ds=crandn(rng, (g.nz, g.ny, g.nx)) * 1e-8, dr=crandn(rng, (g.nz, g.ny, g.nx)) * 0.1,
             r=crandn(rng, (7, g.nw)))
    one = _serial("born", g, a)
    banded = oracle_bands.run("born", g, a, nband=3)
    for k in ("data", "born", "gs", "gr"):
        assert np.allclose(banded[k], one[k], rtol=1e-12, atol=1e-12 * np.abs(one[k]).max()), k
    m1, mb = _serial("model", g, a), oracle_bands.run("model", g, a, nband=2)
    assert np.allclose(mb["bgd"], m1["bgd"], rtol=1e-12, atol=1e-14)


def test_banded_migration_equals_one_run():
    g, rng, a = _setup()
    a = dict(a, data=crandn(rng, (7, g.nw)))
    one = _serial("migrate", g, a)
    banded = oracle_bands.run("migrate", g, a, nband=4)
    assert np.allclose(banded["image"], one["image"], rtol=1e-12, atol=1e-12 * np.abs(one["image"]).max())


def test_banded_smooth_gradient_equals_one_run():
    g, rng, a = _setup()
    s = np.sqrt(a["s2"])
    refs = wem.smooth_refs(s, g.nref)
    b = dict(geom=a["geom"], refs=refs, s_true=s * 1.01, s0=s, wavelet=a["wavelet"])
    d1, J1, g1, m1 = _serial("smooth", g, b)
    d2, J2, g2, m2 = oracle_bands.run("smooth", g, b, nband=3)
    assert np.allclose(d2, d1, rtol=1e-12, atol=1e-14) and np.allclose(m2, m1, rtol=1e-12, atol=1e-14)
    assert abs(J2 / J1 - 1) < 1e-12
    assert np.allclose(g2, g1, rtol=1e-10, atol=1e-12 * np.abs(g1).max())
