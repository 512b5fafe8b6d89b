"""Shot and frequency batching with aperture windows: the drop-in for the
reference's ``StreamingPropagator`` / ``StreamingExtendedBorn``
(``propagator/src/StreamingPropagator.cpp:1-470``, the class the Python
``Propagator`` builds with ``nbatches``, ``fwix/CudaWEM.py:10-18``).

The shots are split into ``nbatches[0]`` groups and the frequencies into
``nbatches[1]`` bands.  Every (shot group, band) pair runs on a window of the
model: the bounding box of its sources and receivers widened by ``ginsu_x`` /
``ginsu_y`` (metres) and clipped to the model
(``StreamingPropagator.cpp:327-393``), so groups of different apertures run on
grids of different sizes.  Each pair has its own plan and its own CUDA stream;
the pairs are enqueued one after the other and overlap on the device.  Their
data are added into the global data at the pair's receivers and frequencies
(``:449-470``), their Born gradients into the global model at the window and
band.

Differences from the reference, stated: the windowed model is cut on the
device (the reference copies it on host threads, ``:396-418``), background
wavefields stay in device memory, a window's padding grows until the padded
size has no prime factor above 7 (the transform lengths of this library; cuFFT
takes any), and a pair's frequency band may also be chosen per shot group
(``bands``), which gives shot groups uneven bands.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import CudaWEM as _w
from .vectors import Axis, Hypercube, SuperVector, Vector


def _dev(*a, **k):
    return _w._dev(*a, **k)


def _get(*a, **k):
    return _w._get(*a, **k)


def _hyper(*a, **k):
    return _w._hyper(*a, **k)


def _model_pair(m):
    return _w._model_pair(m)


def _store(d, t):
    return _w._store(d, t)


def window_indices(xs, ys, axes_x, axes_y, ginsu_x=0.0, ginsu_y=0.0):
    """(min_ix, max_ix, min_iy, max_iy), inclusive, of the box around the points
    (xs, ys) widened by (ginsu_x, ginsu_y) and clipped to the axes
    (``StreamingPropagator.cpp:357-393``: floor for the low edge, ceil for the
    high edge, the whole axis when the box is degenerate)."""
    nx, ox, dx = axes_x
    ny, oy, dy = axes_y
    xs = np.asarray(xs, dtype=np.float64)
    ys = np.asarray(ys, dtype=np.float64)
    if xs.size == 0:
        return 0, nx - 1, 0, ny - 1
    min_x, max_x = float(xs.min()) - ginsu_x, float(xs.max()) + ginsu_x
    min_y, max_y = float(ys.min()) - ginsu_y, float(ys.max()) + ginsu_y
    min_ix = max(0, int(math.floor((min_x - ox) / dx)))
    max_ix = min(nx - 1, int(math.ceil((max_x - ox) / dx)))
    min_iy = max(0, int(math.floor((min_y - oy) / dy)))
    max_iy = min(ny - 1, int(math.ceil((max_y - oy) / dy)))
    if max_ix <= min_ix:
        min_ix, max_ix = 0, nx - 1
    if max_iy <= min_iy:
        min_iy, max_iy = 0, ny - 1
    return min_ix, max_ix, min_iy, max_iy


def next_fft_length(n):
    """Smallest m >= n whose prime factors are 2, 3, 5 and 7 (the transform
    lengths the passes support)."""
    m = max(1, int(n))
    while True:
        k = m
        for f in (2, 3, 5, 7):
            while k % f == 0:
                k //= f
        if k == 1:
            return m
        m += 1


def split_even(n, parts):
    """Sizes of ``parts`` contiguous chunks of n items, larger ones first."""
    parts = max(1, min(parts, n))
    base, extra = divmod(n, parts)
    return [base + (1 if i < extra else 0) for i in range(parts)]


class _Pair:
    """One (shot group, frequency band) pair: its window, band, traces and propagator."""

    def __init__(self, window, f0, nf, src_idx, rec_idx):
        self.window, self.f0, self.nf = window, f0, nf
        self.src_idx, self.rec_idx = src_idx, rec_idx
        self.prop = None
        self.stream = None


class StreamingPropagator:
    """Batched modelling over shot groups and frequency bands with aperture windows.

    Same arguments as ``CudaWEM.Propagator`` (``model`` the [s^2, density] pair with
    axes (x, y, w, z), ``data`` [ntrace][nw], ``wavelet`` [nsrc][nw], ``par``,
    ``geometry``) plus ``nbatches = (shot groups, frequency bands)``; ``par`` may
    hold ``ginsu_x`` / ``ginsu_y``.  ``bands`` optionally maps a shot-group index
    to (first frequency index, count) and replaces the uniform band split for
    that group."""

    def __init__(self, model, data, wavelet, par, geometry, nbatches=(1, 1), bands=None):
        s2, _ = _model_pair(model)
        self.par = par
        self.hyper = _hyper(s2, par, "model")
        ax = self.hyper.getAxes()
        self.ax = ax
        self.device = torch.device("cuda", torch.cuda.current_device())
        g = {k: np.asarray(v) for k, v in geometry.items()}
        self.g = g
        self.wavelet = _dev(wavelet, self.device)
        self.ntrace = len(g["rx"])
        dshape = tuple(np.shape(_w._raw(data))) if data is not None else (self.ntrace, None)
        self.nw = dshape[1] if dshape[1] is not None else ax[2].n
        if len(dshape) != 2 or dshape[0] != self.ntrace or ax[2].n not in (1, self.nw):
            raise RuntimeError("Error: data hypercube does not match the range")
        _w._remap_ids(g["s_ids"], g["r_ids"])  # every receiver belongs to a listed shot
        uniq = np.unique(g["s_ids"])
        groups = np.array_split(uniq, max(1, min(int(nbatches[0]), len(uniq))))
        fsizes = split_even(self.nw, int(nbatches[1]))
        fstarts = np.cumsum([0] + fsizes[:-1])
        gx, gy = float(_get(par, "ginsu_x", 0.0)), float(_get(par, "ginsu_y", 0.0))
        self.pairs = []
        for gi, grp in enumerate(groups):
            src_idx = np.nonzero(np.isin(g["s_ids"], grp))[0]
            rec_idx = np.nonzero(np.isin(g["r_ids"], grp))[0]
            win = window_indices(np.concatenate([g["sx"][src_idx], g["rx"][rec_idx]]),
                                 np.concatenate([g["sy"][src_idx], g["ry"][rec_idx]]),
                                 (ax[0].n, ax[0].o, ax[0].d), (ax[1].n, ax[1].o, ax[1].d), gx, gy)
            if bands is not None and gi in bands:
                blist = [tuple(bands[gi])]
            else:
                blist = list(zip(fstarts, fsizes))
            for f0, nf in blist:
                self.pairs.append(_Pair(win, int(f0), int(nf), src_idx, rec_idx))
        self._model_key = None

    def _window_hyper(self, p):
        ax = self.ax
        x0, x1, y0, y1 = p.window
        return Hypercube([Axis(x1 - x0 + 1, ax[0].o + x0 * ax[0].d, ax[0].d),
                          Axis(y1 - y0 + 1, ax[1].o + y0 * ax[1].d, ax[1].d),
                          Axis(p.nf, ax[2].o + p.f0 * ax[2].d, ax[2].d), ax[3]])

    def _window_model(self, p, model):
        """The pair's [s^2, density] window on the device (a frequency axis of length
        1 stays shared by every frequency)."""
        x0, x1, y0, y1 = p.window
        out = []
        for m in _model_pair(model):
            t = _dev(m, self.device)
            f = slice(0, 1) if t.shape[1] == 1 else slice(p.f0, p.f0 + p.nf)
            out.append(t[:, f, y0:y1 + 1, x0:x1 + 1].contiguous())
        h = self._window_hyper(p)
        if out[0].shape[1] == 1:
            ax = h.getAxes()
            h = Hypercube([ax[0], ax[1], Axis(1, ax[2].o, ax[2].d), ax[3]])
        return SuperVector(Vector(h, out[0]), Vector(h, out[1]))

    def _pair_geometry(self, p):
        g = self.g
        return dict(sx=g["sx"][p.src_idx], sy=g["sy"][p.src_idx], sz=g["sz"][p.src_idx],
                    s_ids=g["s_ids"][p.src_idx], rx=g["rx"][p.rec_idx], ry=g["ry"][p.rec_idx],
                    rz=g["rz"][p.rec_idx], r_ids=g["r_ids"][p.rec_idx])

    def _build(self, p, wmodel):
        if p.prop is None:
            data = torch.zeros((len(p.rec_idx), p.nf), dtype=torch.complex64, device=self.device)
            wav = self.wavelet[p.src_idx][:, p.f0:p.f0 + p.nf].contiguous()
            par = dict(self.par) if isinstance(self.par, dict) else {k: self.par.get(k) for k in self.par}
            # a window's padded size must be a supported transform length: the
            # padding grows to the next one (cuFFT in the reference takes any length)
            x0, x1, y0, y1 = p.window
            nxw, nyw = x1 - x0 + 1, y1 - y0 + 1
            par["padx"] = next_fft_length(nxw + int(_get(par, "padx", 0))) - nxw
            par["pady"] = next_fft_length(nyw + int(_get(par, "pady", 0))) - nyw
            if len(self.pairs) > 1 and _get(par, "run_id") is not None:
                # every pair keeps its checkpoint files in a run directory of its own
                par["run_id"] = f"{par['run_id']}_pair{self.pairs.index(p)}"
            p.prop = _w.WindowPropagator(wmodel, data, wav, par, self._pair_geometry(p))
            p.stream = torch.cuda.Stream(device=self.device)
        return p.prop

    def forward(self, add, model, data):
        out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
        main = torch.cuda.current_stream(self.device)
        results = []
        for p in self.pairs:
            wm = self._window_model(p, model)
            p.wm = wm  # the window the stored background wavefields belong to
            prop = self._build(p, wm)
            p.stream.wait_stream(main)
            with torch.cuda.stream(p.stream):
                d = torch.zeros((len(p.rec_idx), p.nf), dtype=torch.complex64, device=self.device)
                prop.forward(False, wm, d)
            results.append((p, d))
        for p, d in results:
            main.wait_stream(p.stream)
            rows = torch.as_tensor(p.rec_idx, device=self.device)
            out[rows, p.f0:p.f0 + p.nf] += d
        self._model_key = tuple(id(v) for v in _model_pair(model))
        _store(data, out)

    def load_backgrounds(self, model):
        """The backgrounds of ``model`` read back, for every (shot group, band)
        pair, from the checkpoint files of an earlier forward with the same
        geometry (``par`` keys ``wfld_path`` and ``run_id`` name them,
        ``pyfwix_b200.pool``) instead of modelling them again: a restart."""
        for p in self.pairs:
            wm = self._window_model(p, model)
            p.wm = wm
            self._build(p, wm).load_backgrounds(wm)
        self._model_key = tuple(id(v) for v in _model_pair(model))

    def get_compression_ratio(self):
        """Stored bytes ratio of the background wavefields (1 lossless; with
        compress_rate 8 that of the packed store), over the pairs built so far."""
        rs = [p.prop.get_compression_ratio() for p in self.pairs if p.prop is not None]
        return float(np.mean(rs)) if rs else 1.0


class StreamingExtendedBorn:
    """Extended Born over the pairs of a ``StreamingPropagator``: forward adds each
    pair's Born data into the global data, adjoint adds each pair's gradient
    into the global [ds^2, drho] at its window and band."""

    def __init__(self, model, data, slow_den, propagator):
        self.sp = propagator
        self.slow_den = slow_den
        self.borns = None

    def _ensure(self):
        sp = self.sp
        if sp._model_key != tuple(id(v) for v in _model_pair(self.slow_den)) or any(p.prop is None for p in sp.pairs):
            scratch = torch.zeros((sp.ntrace, sp.nw), dtype=torch.complex64, device=sp.device)
            sp.forward(False, self.slow_den, scratch)
        self.borns = [_w.WindowExtendedBorn(p.wm, None, p.wm, p.prop) for p in sp.pairs]

    def forward(self, add, model, data):
        sp = self.sp
        self._ensure()
        out = _dev(data, sp.device) if add else _dev(data, sp.device, zero=True)
        main = torch.cuda.current_stream(sp.device)
        results = []
        for p, born in zip(sp.pairs, self.borns):
            dm = sp._window_model(p, model)
            d = torch.zeros((len(p.rec_idx), p.nf), dtype=torch.complex64, device=sp.device)
            p.stream.wait_stream(main)
            with torch.cuda.stream(p.stream):
                born.forward(False, dm, d)
            results.append((p, d, dm))
        # sums in pair order on the caller's stream: the result does not depend on
        # which pair finishes first
        for p, d, _ in results:
            main.wait_stream(p.stream)
            rows = torch.as_tensor(p.rec_idx, device=sp.device)
            out[rows, p.f0:p.f0 + p.nf] += d
        _store(data, out)

    def adjoint(self, add, model, data):
        sp = self.sp
        self._ensure()
        ds_t, dr_t = (_dev(m, sp.device, zero=not add) for m in _model_pair(model))
        d_all = _dev(data, sp.device)
        main = torch.cuda.current_stream(sp.device)
        shared = ds_t.shape[1] == 1
        results = []
        for p, born in zip(sp.pairs, self.borns):
            x0, x1, y0, y1 = p.window
            nf = 1 if shared else p.nf
            gs = torch.zeros((ds_t.shape[0], nf, y1 - y0 + 1, x1 - x0 + 1), dtype=torch.complex64, device=sp.device)
            gr = torch.zeros_like(gs)
            d = d_all[torch.as_tensor(p.rec_idx, device=sp.device)][:, p.f0:p.f0 + p.nf].contiguous()
            p.stream.wait_stream(main)
            with torch.cuda.stream(p.stream):
                born.adjoint(False, [gs, gr], d)
            results.append((p, gs, gr, d))
        for p, gs, gr, _ in results:
            main.wait_stream(p.stream)
            x0, x1, y0, y1 = p.window
            f = slice(0, 1) if shared else slice(p.f0, p.f0 + p.nf)
            ds_t[:, f, y0:y1 + 1, x0:x1 + 1] += gs
            dr_t[:, f, y0:y1 + 1, x0:x1 + 1] += gr
        ds, dr = _model_pair(model)
        _store(ds, ds_t)
        _store(dr, dr_t)
