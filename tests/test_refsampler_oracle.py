"""Reference selector (``pyfwix_b200.refsampler``, the replacement of
``propagator/src/RefSampler.cpp:49-90``) against its numpy restatement
``oracle/refs.py``, and the k-means rule against OpenCV's ``cv::kmeans`` (the
library the reference calls) on inputs where k-means has one answer.  Runs on
the CPU (torch on the host), the same code as on the device."""
import numpy as np
import pytest
import torch

from oracle import refs as R


def _model(rng, nz=3, nw=4, ny=20, nx=24, complex_=False):
    s0 = (1 / 1800.0) ** 2
    s2 = s0 * (1 + 0.3 * rng.random((nz, nw, ny, nx)))
    if complex_:
        s2 = s2 + 1j * s0 * 0.01 * rng.standard_normal(s2.shape)
    return s2


def _sample_cpu(s2, nref, padx=0, pady=0, **kw):
    """refsampler.sample on a host tensor (it moves to the GPU when there is one)."""
    from pyfwix_b200 import refsampler
    sref, lab = refsampler.sample(torch.as_tensor(s2), nref, padx, pady, **kw)
    return sref.cpu().numpy(), lab.cpu().numpy()


@pytest.mark.parametrize("nref,padx,pady,complex_", [(4, 0, 0, False), (6, 8, 4, False), (3, 5, 0, True),
                                                     (1, 0, 3, False)])
def test_quantile_references_match_oracle(nref, padx, pady, complex_):
    rng = np.random.default_rng(11)
    s2 = _model(rng, complex_=complex_)
    sref, lab = _sample_cpu(s2, nref, padx, pady)
    sref_o, lab_o = R.sample(s2, nref, padx, pady)
    # the product returns complex64 references: equal to the oracle's to float rounding
    assert np.allclose(sref, sref_o, rtol=1e-6, atol=0)
    assert np.array_equal(lab.astype(np.int64), lab_o)
    # edge replication of the padded labels (RefSampler.cpp:70-86)
    if pady:
        assert np.array_equal(lab[:, :, -1], lab[:, :, s2.shape[2] - 1])
    if padx:
        assert np.array_equal(lab[..., -1], lab[..., s2.shape[3] - 1])


def test_quantile_rule_matches_bench_cpu_rule():
    """The CPU arm of the benchmark builds its references with np.quantile of the
    slowness at levels (2k+1)/(2 nref) and nearest labels in s^2: the same rule."""
    rng = np.random.default_rng(3)
    s2 = _model(rng, nz=2, nw=1)
    sref, lab = _sample_cpu(s2, 4)
    s = np.sqrt(s2[:, 0])
    for iz in range(2):
        c = np.quantile(s[iz], (np.arange(4) * 2 + 1) / 8) ** 2
        assert np.allclose(sref[iz, :, 0], c, rtol=1e-6)
        assert np.array_equal(lab[iz, 0], np.argmin(np.abs(s2[iz, 0][..., None] - c), axis=-1))


@pytest.mark.parametrize("complex_", [False, True])
def test_kmeans_references_match_oracle(complex_):
    rng = np.random.default_rng(5)
    s2 = _model(rng, nz=2, nw=3, complex_=complex_)
    sref, lab = _sample_cpu(s2, 4, method="kmeans")
    sref_o, lab_o = R.sample(s2, 4, method="kmeans")
    assert np.allclose(sref, sref_o, rtol=1e-6, atol=0)
    assert np.array_equal(lab.astype(np.int64), lab_o)


def test_kmeans_rows_stop_independently():
    """A row that converges early keeps its centres while another row of the same
    chunk still iterates (each row is its own cv::kmeans call in the reference)."""
    rng = np.random.default_rng(9)
    a = _model(rng, nz=1, nw=1)
    b = _model(np.random.default_rng(10), nz=1, nw=1)
    both = np.concatenate([a, b], axis=1)
    s_both, _ = _sample_cpu(both, 5, method="kmeans")
    s_a, _ = _sample_cpu(a, 5, method="kmeans")
    s_b, _ = _sample_cpu(b, 5, method="kmeans")
    assert np.allclose(s_both[:, :, 0], s_a[:, :, 0], rtol=1e-12, atol=0)
    assert np.allclose(s_both[:, :, 1], s_b[:, :, 0], rtol=1e-12, atol=0)


def test_kmeans_pinned_against_opencv():
    """Well separated clusters of s^2 (four velocities, +-0.2 % scatter each): the
    k-means centres are the cluster means whatever the seeding, so OpenCV's
    randomised cv::kmeans (KMEANS_PP_CENTERS, the reference's call) and the
    deterministic rule must agree, centres to float32 rounding and labels up to
    the order of the centres."""
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(21)
    vel = np.array([1500.0, 2100.0, 2900.0, 3800.0])
    npix = 24 * 20
    which = rng.integers(0, 4, npix)
    v = vel[which] * (1 + 0.002 * rng.standard_normal(npix))
    s2 = (1 / v ** 2).reshape(1, 1, 20, 24)
    sref, lab = _sample_cpu(s2, 4, method="kmeans")
    cv2.setRNGSeed(1234)
    pts = np.stack([s2.ravel().real, np.zeros(npix)], axis=1).astype(np.float32)
    crit = (cv2.TERM_CRITERIA_EPS + cv2.TERM_CRITERIA_MAX_ITER, 100, 1e-3)   # RefSampler.cpp:60
    _, cv_lab, cv_cent = cv2.kmeans(pts, 4, None, crit, 1, cv2.KMEANS_PP_CENTERS)
    order = np.argsort(cv_cent[:, 0])
    ours = np.sort(sref[0, :, 0].real)
    assert np.allclose(ours, cv_cent[order, 0], rtol=1e-5)
    # relabel OpenCV's clusters by ascending centre; ours come ascending (quantile start)
    rank = np.empty(4, np.int64)
    rank[order] = np.arange(4)
    assert np.array_equal(lab.ravel(), rank[cv_lab.ravel()])
    # and both are the true cluster membership (velocities ascending -> s^2 descending)
    assert np.array_equal(lab.ravel(), 3 - which)
