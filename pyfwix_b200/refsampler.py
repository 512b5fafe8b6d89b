"""Reference slownesses and labels per depth (the inputs of every PSPI / NSPS step).

The reference picks them with OpenCV k-means per (depth, frequency)
(``propagator/src/RefSampler.cpp:49-90``: ``cv::kmeans`` with K = nref,
KMEANS_PP_CENTERS, 100 iterations / eps 1e-3, one attempt) and pads the labels by
edge replication (``:75-86``).  cv::kmeans is randomised and unpinned, so here the
choice is deterministic:

* ``method="quantile"`` (default): reference slownesses are the quantiles
  (2k+1)/(2 nref) of the depth slice's slowness sqrt(Re s^2); the reference s^2
  is their square.
* ``method="kmeans"``: Lloyd iterations on Re s^2 started from those quantiles
  (the same objective as cv::kmeans, without the random seeding).

Labels are the index of the nearest reference in s^2 (complex distance), padded
by edge replication.  Runs on the model's device with torch.
"""
from __future__ import annotations

import numpy as np
import torch


def _quantile_levels(nref, device):
    return (torch.arange(nref, device=device, dtype=torch.float64) * 2 + 1) / (2 * nref)


def sample(slow2, nref, padx=0, pady=0, method="quantile", iters=100, tol=1e-3):
    """slow2: complex or real s^2, [nz][nw or 1][ny][nx] (torch or numpy).

    Returns (sref [nz][nref][nw'] complex64, labels [nz][nw'][NY][NX] uint8) on
    slow2's device (CUDA if slow2 is numpy and a GPU is present), nw' = slow2's
    frequency extent."""
    t = torch.as_tensor(slow2)
    if t.device.type == "cpu" and torch.cuda.is_available():
        t = t.to("cuda")
    if not t.is_complex():
        t = t.to(torch.float64).to(torch.complex128)
    else:
        t = t.to(torch.complex128)
    nz, nw, ny, nx = t.shape
    dev = t.device
    flat = t.reshape(nz * nw, ny * nx)
    s = torch.sqrt(torch.clamp(flat.real, min=0.0))
    q = _quantile_levels(nref, dev)
    srt, _ = torch.sort(s, dim=1)
    # linear-interpolated quantiles (numpy's default "linear" method)
    pos = q * (ny * nx - 1)
    lo = torch.floor(pos).long()
    hi = torch.clamp(lo + 1, max=ny * nx - 1)
    frac = (pos - lo.to(pos.dtype))[None, :]
    sq = srt[:, lo] * (1 - frac) + srt[:, hi] * frac          # [nz*nw, nref]
    centers = (sq ** 2).to(torch.complex128)                  # reference s^2
    if method == "kmeans":
        x = flat
        for _ in range(iters):
            lab = torch.argmin(torch.abs(x[:, :, None] - centers[:, None, :]), dim=2)
            new = centers.clone()
            for r in range(nref):
                m = (lab == r)
                cnt = m.sum(dim=1)
                ssum = torch.where(m, x, torch.zeros_like(x)).sum(dim=1)
                new[:, r] = torch.where(cnt > 0, ssum / torch.clamp(cnt, min=1), centers[:, r])
            shift = torch.max(torch.abs(new - centers))
            centers = new
            if float(shift) <= tol * float(torch.max(torch.abs(centers))):
                break
    elif method != "quantile":
        raise ValueError(f"unknown reference method {method!r}")
    lab = torch.argmin(torch.abs(flat[:, :, None] - centers[:, None, :]), dim=2)
    lab = lab.reshape(nz, nw, ny, nx).to(torch.uint8)
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
