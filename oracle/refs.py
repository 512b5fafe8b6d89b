"""Reference slownesses and labels per (depth, frequency): CPU restatement.

TEST INFRASTRUCTURE ONLY.  The tests import this module as the checker of
``pyfwix_b200.refsampler``; the product never imports it.

The reference picks, for every (depth, frequency) row of the complex s^2 model,
nref k-means centres of the row's samples (``propagator/src/RefSampler.cpp:49-90``:
one ``cv::kmeans`` call per row, K = nref, KMEANS_PP_CENTERS seeding, stop after
100 iterations or a centre shift of at most 1e-3, one attempt), takes the centres
as the reference s^2 and each sample's cluster index as its label, and pads the
labels of a padded wavefield by edge replication (``:70-86``).  The seeding of
``cv::kmeans`` is random, so the library replaces it with a deterministic start;
this module restates those deterministic rules in numpy, row by row as the
reference calls ``cv::kmeans``:

* ``quantile_centers``: the reference slownesses are the quantiles
  (2k + 1) / (2 nref), k = 0 .. nref - 1, of the row's slowness sqrt(Re s^2)
  (linear interpolation between order statistics, numpy's default), squared;
* ``lloyd_centers``: Lloyd iterations on the complex s^2 started from those
  quantile centres (the objective of ``cv::kmeans``), at most ``iters`` of them,
  stopping when no centre moves by more than ``tol`` times the row's largest
  centre magnitude; an empty cluster keeps its centre;
* ``nearest``: the label of a sample is the index of the nearest centre in the
  complex plane (the first on a tie), as ``cv::kmeans`` assigns labels.
"""
from __future__ import annotations

import numpy as np


def quantile_levels(nref):
    return (2 * np.arange(nref) + 1) / (2.0 * nref)


def quantile_centers(rows, nref):
    """rows [R][npix] (real or complex s^2) -> centres [R][nref] complex128."""
    x = np.asarray(rows)
    s = np.sqrt(np.maximum(np.real(x).astype(np.float64), 0.0))
    q = np.quantile(s, quantile_levels(nref), axis=1).T          # [R][nref]
    return (q ** 2).astype(np.complex128)


def nearest(rows, centers):
    """Index of the nearest centre of each sample, [R][npix]."""
    x = np.asarray(rows).astype(np.complex128)
    d = np.abs(x[:, :, None] - np.asarray(centers)[:, None, :])
    return np.argmin(d, axis=2)


def lloyd_centers(rows, centers, iters=100, tol=1e-3):
    """Lloyd iterations on each row independently from the given centres."""
    x = np.asarray(rows).astype(np.complex128)
    out = np.array(centers, dtype=np.complex128, copy=True)
    for r in range(x.shape[0]):
        c = out[r]
        for _ in range(iters):
            lab = np.argmin(np.abs(x[r][:, None] - c[None, :]), axis=1)
            new = c.copy()
            for k in range(len(c)):
                m = lab == k
                if m.any():
                    new[k] = x[r][m].mean()
            shift = np.max(np.abs(new - c))
            c = new
            if shift <= tol * np.max(np.abs(c)):
                break
        out[r] = c
    return out


def sample(slow2, nref, padx=0, pady=0, method="quantile", iters=100, tol=1e-3):
    """slow2 [nz][nw][ny][nx] -> (sref [nz][nref][nw] complex128,
    labels [nz][nw][ny + pady][nx + padx] int64), labels edge-padded."""
    s = np.asarray(slow2)
    nz, nw, ny, nx = s.shape
    rows = s.reshape(nz * nw, ny * nx)
    c = quantile_centers(rows, nref)
    if method == "kmeans":
        c = lloyd_centers(rows, c, iters, tol)
    lab = nearest(rows, c).reshape(nz, nw, ny, nx)
    if padx or pady:
        lab = np.pad(lab, ((0, 0), (0, 0), (0, pady), (0, padx)), mode="edge")
    sref = c.reshape(nz, nw, nref).transpose(0, 2, 1)
    return sref, lab
