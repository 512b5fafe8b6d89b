"""The FP64 oracle run band by band over frequency in worker processes.

Every operator of the path acts on each frequency on its own -- the 2D
transforms, phase shifts, split-step factors and scattering weights are per
frequency, injection and recording move [ntrace][nw] traces to and from the
matching frequency slices, reflection and the imaging condition are pointwise
in frequency -- and the image, the FWI gradient and the misfit are sums over
frequency.  So an oracle run over nw frequencies equals the concatenation (or,
for the sums, the sum) of runs over bands of it, each band a Grid whose first
frequency is ow + i0 * dw.  The large parity cases use that to spread the
oracle over the host's cores.  Workers are started with the "spawn" method
(fresh interpreters: safe after the parent has initialised CUDA) and each uses
one FFT thread.

Inputs are the frequency-independent model (s^2 [nz][ny][nx], labels
[nz][NY][NX]) and the per-frequency arrays (references [nz][nref][nw], wavelet
[nsrc][nw], data [ntrace][nw]) that each job slices to its band.
"""
from __future__ import annotations

import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor
from dataclasses import replace

import numpy as np

_POOL = None


def workers():
    return max(1, min(16, os.cpu_count() or 1))


def pool():
    global _POOL
    if _POOL is None:
        _POOL = ProcessPoolExecutor(max_workers=workers(), mp_context=mp.get_context("spawn"))
    return _POOL


def bands(nw, n=None):
    n = max(1, min(nw, n or workers()))
    edges = np.linspace(0, nw, n + 1).round().astype(int)
    return [(int(a), int(b)) for a, b in zip(edges[:-1], edges[1:]) if b > a]


def _band_grid(g, i0, i1):
    return replace(g, ow=g.ow + i0 * g.dw, nw=i1 - i0, _cache={})


def _model(g, s2, labels, sref_band, kind):
    from oracle import wem
    shape = (g.nz, g.nw, g.ny, g.nx)
    slow = np.broadcast_to(np.asarray(s2, np.float64)[:, None].astype(np.complex128), shape)
    den = np.broadcast_to(np.complex128(1.0), shape)
    lab = np.broadcast_to(np.asarray(labels)[:, None], (g.nz, g.nw, g.NY, g.NX))
    st = wem.Stepper(g, np.asarray(sref_band, np.complex128), lab, kind)
    return slow, den, st


# frequency axis of each per-frequency input
_PER_W = {"sref": 2, "wavelet": 1, "data": 1, "r": 1}


def _band_args(a, i0, i1):
    out = dict(a)
    for k, ax in _PER_W.items():
        if out.get(k) is not None:
            sl = [slice(None)] * np.ndim(out[k])
            sl[ax] = slice(i0, i1)
            out[k] = np.ascontiguousarray(np.asarray(out[k])[tuple(sl)])
    return out


def _job(task, g, i0, i1, a):
    """One band [i0, i1) of ``task``; ``a`` holds that band's per-frequency arrays."""
    from oracle import wem
    wem.set_fft_workers(None)
    gb = _band_grid(g, i0, i1)
    acq = wem.make_acquisition(gb, a["geom"])
    if task == "smooth":
        wav = a["wavelet"]
        d_obs = wem.smooth_propagate(gb, a["refs"], a["s_true"], acq, wav)[0]
        J, grad = wem.smooth_gradient(gb, a["refs"], a["s0"], acq, wav, d_obs)
        data0 = wem.smooth_propagate(gb, a["refs"], a["s0"], acq, wav)[0]
        return d_obs, J, grad, data0
    slow, den, st = _model(gb, a["s2"], a["labels"], a["sref"], a["kind"])
    wav = a["wavelet"]
    data, bgd, bgu = wem.propagate(gb, st, acq, slow, den, wav)
    out = {"data": data}
    if task == "migrate":
        obs = a["data"] if a.get("data") is not None else data
        out["image"] = wem.migrate(gb, st, acq, wav, obs)
    if task == "born":
        shape = slow.shape
        ds = np.broadcast_to(np.asarray(a["ds"], np.complex128)[:, None], shape)
        dr = np.broadcast_to(np.asarray(a["dr"], np.complex128)[:, None], shape)
        out["born"] = wem.born_forward(gb, st, acq, slow, den, bgd, bgu, ds, dr)
        gs, gr = wem.born_adjoint(gb, st, acq, slow, den, bgd, bgu, np.asarray(a["r"], np.complex128))
        out["gs"], out["gr"] = gs.sum(axis=1), gr.sum(axis=1)
    if task == "model":
        out["bgd"] = None if bgd[0] is None else np.stack(bgd)
    return out


def run(task, g, args, nband=None):
    """Runs the oracle ``task`` over frequency bands in the worker pool and joins
    the results:

    * "model": Propagator::forward -> {"data" [ntr][nw], "bgd" [nz][ns][nw][NY][NX]};
    * "migrate": modelling, then the lockstep image of ``args["data"]`` (or of the
      modelled data) -> {"data", "image" [nz][ny][nx]};
    * "born": modelling, ExtendedBorn forward of (ds, dr) [nz][ny][nx] (one value
      per depth and cell for every frequency) and adjoint of ``args["r"]`` ->
      {"data", "born" [ntr][nw], "gs", "gr" [nz][ny][nx] summed over frequency};
    * "smooth": smooth-step modelling of s_true (d_obs) and the adjoint-state
      gradient at s0 -> (d_obs [ntr][nw], J, gradient [nz][ny][nx], data at s0
      [ntr][nw])."""
    parts = bands(g.nw, nband)
    futs = [pool().submit(_job, task, g, i0, i1, _band_args(args, i0, i1)) for i0, i1 in parts]
    res = [f.result() for f in futs]
    if task == "smooth":
        return (np.concatenate([r[0] for r in res], axis=1), sum(r[1] for r in res), sum(r[2] for r in res),
                np.concatenate([r[3] for r in res], axis=1))
    out = {"data": np.concatenate([r["data"] for r in res], axis=1)}
    if task == "migrate":
        out["image"] = sum(r["image"] for r in res)
    if task == "born":
        out["born"] = np.concatenate([r["born"] for r in res], axis=1)
        out["gs"] = sum(r["gs"] for r in res)
        out["gr"] = sum(r["gr"] for r in res)
    if task == "model" and res[0]["bgd"] is not None:
        out["bgd"] = np.concatenate([r["bgd"] for r in res], axis=2)
    return out
