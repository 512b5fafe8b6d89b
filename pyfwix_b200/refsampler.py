"""Reference slownesses and labels per depth (the inputs of every PSPI / NSPS step).

The reference picks them with OpenCV k-means per (depth, frequency)
(``propagator/src/RefSampler.cpp:49-90``: ``cv::kmeans`` with K = nref,
KMEANS_PP_CENTERS, 100 iterations / eps 1e-3, one attempt) and pads the labels by
edge replication (``:75-86``).  cv::kmeans is randomised and unpinned, so here the
choice is deterministic:

* ``method="quantile"`` (default): reference slownesses are the quantiles
  (2k+1)/(2 nref) of the depth slice's slowness sqrt(Re s^2); the reference s^2
  is their square.
* ``method="kmeans"``: Lloyd iterations on s^2 started from those quantiles
  (the same objective as cv::kmeans, without the random seeding), each
  (depth, frequency) row stopped on its own.

Labels are the index of the nearest reference in s^2 (complex distance), padded
by edge replication.  Runs on the model's device with torch.
"""
from __future__ import annotations

import numpy as np
import torch


def _quantile_levels(nref, device):
    return (torch.arange(nref, device=device, dtype=torch.float64) * 2 + 1) / (2 * nref)


# Bytes of the [rows][ny*nx][nref] complex128 distance array one chunk of
# (depth, frequency) rows may take: a per-frequency model of 256 x 256 x 128
# frequencies x 200 depths would need 107 GB at once.
_CHUNK_BYTES = 1 << 28


def _nearest(x, centers):
    """Index of the nearest center (complex distance) per sample: [rows][npix]."""
    return torch.argmin(torch.abs(x[:, :, None] - centers[:, None, :]), dim=2)


def _quantile_centers(x, nref):
    """s^2 of the quantiles (2k+1)/(2 nref) of sqrt(Re s^2) per row (numpy's
    default linear interpolation)."""
    npix = x.shape[1]
    s = torch.sqrt(torch.clamp(x.real, min=0.0))
    q = _quantile_levels(nref, x.device)
    srt, _ = torch.sort(s, dim=1)
    pos = q * (npix - 1)
    lo = torch.floor(pos).long()
    hi = torch.clamp(lo + 1, max=npix - 1)
    frac = (pos - lo.to(pos.dtype))[None, :]
    sq = srt[:, lo] * (1 - frac) + srt[:, hi] * frac          # [rows, nref]
    return (sq ** 2).to(torch.complex128)


def _lloyd(x, centers, iters, tol):
    """Lloyd iterations on each row of x from the given centers.  Rows are
    independent, as the reference's one cv::kmeans call per (depth, frequency)
    row: a row stops, keeping the update that got it there, once none of its
    centers moved by more than tol times its largest center; an empty cluster
    keeps its center."""
    nref = centers.shape[1]
    active = torch.ones(centers.shape[0], dtype=torch.bool, device=x.device)
    for _ in range(iters):
        lab = _nearest(x, centers)
        new = centers.clone()
        for r in range(nref):
            m = (lab == r)
            cnt = m.sum(dim=1)
            ssum = torch.where(m, x, torch.zeros_like(x)).sum(dim=1)
            new[:, r] = torch.where(cnt > 0, ssum / torch.clamp(cnt, min=1), centers[:, r])
        shift = torch.abs(new - centers).amax(dim=1)
        centers = torch.where(active[:, None], new, centers)
        active = active & ~(shift <= tol * torch.abs(centers).amax(dim=1))
        if not bool(active.any()):
            break
    return centers


def sample(slow2, nref, padx=0, pady=0, method="quantile", iters=100, tol=1e-3, chunk_bytes=_CHUNK_BYTES):
    """slow2: complex or real s^2, [nz][nw or 1][ny][nx] (torch or numpy).

    Returns (sref [nz][nref][nw'] complex64, labels [nz][nw'][NY][NX] uint8) on
    slow2's device (CUDA if slow2 is numpy and a GPU is present), nw' = slow2's
    frequency extent.  The (depth, frequency) rows are independent and are
    processed in chunks of about ``chunk_bytes`` of distances each."""
    if method not in ("quantile", "kmeans"):
        raise ValueError(f"unknown reference method {method!r}")
    t = torch.as_tensor(slow2)
    if t.device.type == "cpu" and torch.cuda.is_available():
        t = t.to("cuda")
    if not t.is_complex():
        t = t.to(torch.float64).to(torch.complex128)
    else:
        t = t.to(torch.complex128)
    nz, nw, ny, nx = t.shape
    flat = t.reshape(nz * nw, ny * nx)
    rows = max(1, min(nz * nw, int(chunk_bytes) // max(1, ny * nx * nref * 16)))
    cs, ls = [], []
    for i in range(0, nz * nw, rows):
        x = flat[i:i + rows]
        c = _quantile_centers(x, nref)
        if method == "kmeans":
            c = _lloyd(x, c, iters, tol)
        cs.append(c)
        ls.append(_nearest(x, c).to(torch.uint8))
    centers = torch.cat(cs)
    lab = torch.cat(ls).reshape(nz, nw, ny, nx)
    if padx or pady:
        lab = torch.nn.functional.pad(lab.to(torch.float32), (0, padx, 0, pady), mode="replicate").to(torch.uint8)
    sref = centers.reshape(nz, nw, nref).permute(0, 2, 1).contiguous().to(torch.complex64)
    return sref, lab.contiguous()


def expand_refs(sref, nw):
    """[nz][nref][1] references for a frequency-invariant model -> [nz][nref][nw]."""
    sref = torch.as_tensor(sref)
    if sref.shape[2] == nw:
        return sref
    return sref.expand(sref.shape[0], sref.shape[1], nw).contiguous()
