"""Drop-in for pyfwix's ``fwix.CudaWEM`` operator surface (``fwix/CudaWEM.py:7-157``).

Same class names, constructor arguments and methods as the reference:

=================  ==========================================================
``Propagator``     wavelet -> surface data through the down pass, reflection
                   and up pass (``propagator/src/Propagator.cpp:121-221``)
``ExtendedBorn``   linearised modelling and its adjoint, the FWI gradient
                   (``propagator/src/ExtendedBorn.cpp:80-150``)
``PhaseShift``     one phase shift of a spectrum (``propagator/src/PhaseShift.cpp``)
``RefSampler``     reference slownesses and labels per depth
``PSPI`` / ``NSPS``  one depth step (``propagator/src/PSPI.cpp``, ``NSPS.cpp``)
``Injection``      trilinear injection / recording at one depth
``Downward`` / ``Upward``  whole-depth sweeps (``propagator/src/OneWay.cpp:19-79``)
=================  ==========================================================

Arguments are :class:`~pyfwix_b200.vectors.Vector` / ``SuperVector`` objects (the
stand-ins for SEP vectors), torch tensors (CUDA or CPU) or numpy arrays, in the
reference layouts: model ``[nz][nw][ny][nx]`` complex s^2 and density, data
``[ntrace][nw]``, wavelet ``[nsrc][nw]``, wavefields ``[ns][nw][NY][NX]``.
``par`` is a dict (or any object with ``get``) with the reference's keys
(``nref, padx, pady, eps, taperx, tapery, eps_scat, taylor``); for bare arrays
it also carries the axes (``ox, dx, oy, dy, oz, dz, ow, dw``, frequencies in Hz).

``forward(add, model, data)`` writes ``data`` (adding to it when ``add``) and
``adjoint(add, model, data)`` writes ``model``, in place in whatever object the
caller passed.  Compute runs on the CUDA device of the first CUDA operand (the
current device otherwise); there is no CPU path.

Extensions over the reference, all opt-in through ``par``:
``step`` ("pspi" as in the reference's ``OneWay``, or "nsps"),
``ref_method`` ("quantile" or "kmeans"; the reference runs a randomised
OpenCV k-means), ``autotune`` (time the equivalent forms of the depth step
once per propagator and keep the fastest, ``fwix_plan_autotune``),
``background_store = "host"`` (with ``compress_rate`` 8 or 16: the packed
backgrounds in pinned host memory, read by the kernels over the host link, for
runs whose backgrounds do not fit in device memory), ``wfld_path`` / ``run_id``
(every forward also writes its stored backgrounds into the reference's
checkpoint-file layout, ``pyfwix_b200.pool``; ``load_backgrounds`` reads them
back), and a model whose frequency axis has length 1 (one s^2 for every
frequency).
"""
from __future__ import annotations

import warnings

import numpy as np
import torch

from . import _lib as L
from . import hostcopy, refsampler
from .plan import Plan
from .vectors import Axis, Hypercube, SuperVector, Vector

__all__ = ["Propagator", "ExtendedBorn", "PhaseShift", "RefSampler", "PSPI", "NSPS", "Injection",
           "Downward", "Upward", "WindowPropagator", "WindowExtendedBorn", "slowness_model"]


# ---------------------------------------------------------------------- helpers
def _get(par, key, default=None):
    if par is None:
        return default
    if hasattr(par, "get"):
        v = par.get(key, default)
    else:
        v = getattr(par, key, default)
    return default if v is None else v


def _device(*xs):
    for x in xs:
        t = x.arr if isinstance(x, Vector) else x
        if isinstance(t, torch.Tensor) and t.is_cuda:
            return t.device
    return torch.device("cuda", torch.cuda.current_device())


def _raw(x):
    return x.arr if isinstance(x, Vector) else x


def _hyper(x, par=None, kind=None):
    """Hypercube of an operand: its own, or built from ``par`` for bare arrays."""
    if isinstance(x, Vector):
        return x.getHyper()
    shape = tuple(np.shape(x) if not isinstance(x, torch.Tensor) else x.shape)
    if kind == "model" and len(shape) == 4:
        nz, nw, ny, nx = shape
        return Hypercube([Axis(nx, _get(par, "ox", 0.0), _get(par, "dx", 1.0)),
                          Axis(ny, _get(par, "oy", 0.0), _get(par, "dy", 1.0)),
                          Axis(nw, _get(par, "ow", 1.0), _get(par, "dw", 1.0)),
                          Axis(nz, _get(par, "oz", 0.0), _get(par, "dz", 1.0))])
    if kind == "wavefield" and len(shape) >= 3:
        ns = int(np.prod(shape[:-3])) if len(shape) > 3 else 1
        nw, ny, nx = shape[-3:]
        return Hypercube([Axis(nx, _get(par, "ox", 0.0), _get(par, "dx", 1.0)),
                          Axis(ny, _get(par, "oy", 0.0), _get(par, "dy", 1.0)),
                          Axis(nw, _get(par, "ow", 1.0), _get(par, "dw", 1.0)), Axis(ns)])
    return Hypercube.from_shape(shape)


def _dev(x, device, shape=None, zero=False):
    """Device complex64 contiguous view of an operand (the operand itself when it
    already is one, so kernels write into the caller's memory)."""
    t = _raw(x)
    if isinstance(t, torch.Tensor) and t.device == device and t.dtype == torch.complex64 and t.is_contiguous():
        if zero:
            t.zero_()
        return t
    if zero:
        return torch.zeros(tuple(np.shape(t)) if shape is None else shape, dtype=torch.complex64, device=device)
    h = hostcopy.host_view(t)
    if h is not None:
        return hostcopy.to_device(h, device)
    t = torch.as_tensor(t)
    if not t.is_complex():
        t = t.to(torch.float32)
    return t.to(device=device, dtype=torch.complex64).contiguous()


def _store(dst, t):
    """Copy a device result back into the caller's object when it is not the
    same memory."""
    raw = _raw(dst)
    h = hostcopy.host_view(raw) if t.is_cuda else None
    if h is not None and h.flags.writeable:
        hostcopy.to_host(t, h)                 # staged through pinned buffers
    elif isinstance(raw, torch.Tensor):
        if raw.data_ptr() != t.data_ptr() or raw.device != t.device:
            raw.copy_(t.reshape(raw.shape))
    elif isinstance(raw, np.ndarray):
        src = t.reshape(raw.shape)
        if raw.dtype == np.complex64 and raw.flags.c_contiguous and raw.flags.writeable:
            torch.from_numpy(raw).copy_(src)   # one device-to-host copy into the caller's array
        else:
            np.copyto(raw, src.cpu().numpy().astype(raw.dtype, copy=False))
    else:
        raise TypeError(f"cannot write a result into {type(dst).__name__}")


def _model_pair(model):
    if isinstance(model, SuperVector):
        return model.vecs[0], model.vecs[1]
    if isinstance(model, (list, tuple)) and len(model) == 2:
        return model[0], model[1]
    raise ValueError("model must be a [slowness^2, density] pair")


def _remap_ids(s_ids, r_ids):
    """Dense shot indices in sorted order of the source ids, receivers mapped
    with the same table (``propagator/src/Propagator.cpp:28-59``)."""
    s_ids = np.asarray(s_ids, dtype=np.int64)
    r_ids = np.asarray(r_ids, dtype=np.int64)
    uniq = np.unique(s_ids)
    s_new = np.searchsorted(uniq, s_ids).astype(np.int32)
    pos = np.searchsorted(uniq, r_ids)
    ok = (pos < len(uniq)) & (uniq[np.minimum(pos, len(uniq) - 1)] == r_ids)
    if not np.all(ok):
        raise RuntimeError("Error: Found a receiver associated with a Shot ID not present in the source list.")
    return s_new, pos.astype(np.int32), len(uniq)


def _grid_from_model(hyper):
    ax = hyper.getAxes()
    if len(ax) != 4:
        raise ValueError(f"slowness model must be 4-D (x, y, w, z), got {hyper}")
    return ax


def _pads(par):
    padx = int(_get(par, "padx", -1))
    pady = int(_get(par, "pady", -1))
    if padx < 0 or pady < 0:
        raise RuntimeError("Error: negative padx/pady values")
    return padx, pady


def _plan_from_slow(slow_hyper, par, ns, device, nz=None, padx=None, pady=None, nw=None):
    """Plan for a model hypercube (x, y, w, z); ``nw`` overrides the frequency count
    for a model whose frequency axis has length 1 (shared by every frequency)."""
    x, y, w, z = _grid_from_model(slow_hyper)
    if padx is None:
        padx, pady = _pads(par)
    if nw is not None and w.n not in (1, nw):
        raise RuntimeError("Error: model hypercube does not match the slow_hyper")
    return Plan(nx=x.n, ny=y.n, nw=w.n if nw is None else nw, ns=ns, nz=z.n if nz is None else nz,
                dx=x.d, dy=y.d, dz=z.d,
                ox=x.o, oy=y.o, oz=z.o, ow=w.o, dw=w.d, padx=padx, pady=pady,
                nref=int(_get(par, "nref", 1)), eps=float(_get(par, "eps", 0.0)),
                taperx=int(_get(par, "taperx", 0)), tapery=int(_get(par, "tapery", 0)),
                eps_scat=float(_get(par, "eps_scat", 0.04)), taylor=int(_get(par, "taylor", 1)),
                step=str(_get(par, "step", "pspi")), device=device)


def _refs(plan, slow2, par):
    """Reference s^2 and labels of every depth for a plan, from the model."""
    sref, labels = refsampler.sample(slow2, plan.nref, plan.NX - plan.nx, plan.NY - plan.ny,
                                     method=str(_get(par, "ref_method", "quantile")))
    sref = refsampler.expand_refs(sref, plan.nw)
    plan.set_refs(sref, labels, phase_cache=bool(_get(par, "phase_cache", True)))
    return sref, labels


# ---------------------------------------------------------------------- operators
class WindowPropagator:
    """Nonlinear modelling on one model window (the whole model it is given):
    wavelet -> recorded data for a [s^2, density] model.  ``Propagator`` runs one
    of these per (shot group, frequency band) pair.

    The background down- and up-going wavefields of the last ``forward`` stay in
    device memory for :class:`ExtendedBorn`: lossless by default, or, with the
    reference's ``compress_rate`` key set to 8, in this library's fixed-rate
    lossy format (8.5 bits per value, 3.76 x smaller; the reference keeps
    ZFP-compressed copies at that rate on disk, ``propagator/src/WavefieldPool.cpp``).
    ``nbatches`` is accepted for signature compatibility: every shot and
    frequency runs in one batch."""

    def __init__(self, model, data, wavelet, par, geometry, nbatches=(1, 1)):
        self.par = par
        s2, _ = _model_pair(model)
        self.slow_hyper = _hyper(s2, par, "model")
        self.range_shape = tuple(np.shape(_raw(data)))
        self.device = _device(s2, data, wavelet)
        self.nbatches = tuple(nbatches)
        g = geometry
        s_ids, r_ids, ns = _remap_ids(g["s_ids"], g["r_ids"])
        if len(self.range_shape) != 2 or self.range_shape[0] != len(np.asarray(g["rx"])):
            raise RuntimeError("Error: data hypercube does not match the range")
        self.plan = _plan_from_slow(self.slow_hyper, par, ns, self.device, nw=self.range_shape[1])
        self.src = self.plan.traces(g["sx"], g["sy"], g["sz"], s_ids)
        self.rec = self.plan.traces(g["rx"], g["ry"], g["rz"], r_ids)
        self.wavelet = _dev(wavelet, self.device)
        if tuple(self.wavelet.shape) != (self.src.ntrace, self.plan.nw):
            raise ValueError(f"wavelet must be [nsrc={self.src.ntrace}][nw={self.plan.nw}]")
        self.bg_down = self.bg_up = None
        self._bg_key = None
        rate = _get(par, "compress_rate")
        if rate is not None and float(rate) not in (8.0, 16.0):
            raise ValueError(f"compress_rate {rate} is not supported: the packed store has rates 8 and 16")
        self.packed = rate is not None
        self.rate = int(float(rate)) if self.packed else None
        if self.packed:
            self.plan.set_pack_rate(self.rate)
        where = str(_get(par, "background_store", "device"))
        if where not in ("device", "host"):
            raise ValueError(f"background_store must be 'device' or 'host', got {where!r}")
        if where == "host" and not self.packed:
            raise ValueError("background_store 'host' keeps the packed backgrounds: set compress_rate = 8 or 16")
        self.host_store = where == "host"
        self.pool = None

    def set_background_model(self, model):
        s2, den = _model_pair(model)
        if not _hyper(s2, self.par, "model").checkSame(self.slow_hyper):
            raise RuntimeError("Error: model hypercube does not match the slow_hyper")
        s2d, dend = self.plan.set_model(_raw(s2), _raw(den))
        _refs(self.plan, s2d, self.par)
        if bool(_get(self.par, "autotune", False)) and not getattr(self, "tuning", None):
            # par["autotune"]: time the equivalent forms of the depth step once
            # (synchronises the current stream) and keep the fastest
            self.tuning = self.plan.autotune()

    def _ensure_storage(self):
        if self.packed:
            if self.bg_down is None:
                self.bg_down = self.plan.packed(self.plan.nz, host=self.host_store)
                self.bg_up = self.plan.packed(self.plan.nz, host=self.host_store)
            return
        shape = (self.plan.nz,) + self.plan.wshape
        if self.bg_down is None or tuple(self.bg_down.shape) != shape:
            self.bg_down = torch.empty(shape, dtype=torch.complex64, device=self.device)
            self.bg_up = torch.empty(shape, dtype=torch.complex64, device=self.device)

    def forward(self, add, model, data):
        with torch.cuda.device(self.device):
            self.set_background_model(model)
            self._ensure_storage()
            out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
            if self.packed:
                self.plan.propagate_packed(self.src, self.rec, self.wavelet, out, self.bg_down, self.bg_up,
                                           add=bool(add))
            else:
                self.plan.propagate(self.src, self.rec, self.wavelet, out, self.bg_down, self.bg_up, add=bool(add))
            self._bg_key = tuple(id(v) for v in _model_pair(model))
            _store(data, out)
            if _get(self.par, "wfld_path") is not None:
                self._checkpoint()

    def _pool(self):
        if self.pool is None:
            from .pool import WavefieldPool
            import uuid
            run_id = str(_get(self.par, "run_id", "run_" + uuid.uuid4().hex[:12]))
            self.pool = WavefieldPool(self.plan, self.par, run_id, self.plan.nz)
        return self.pool

    def _checkpoint(self):
        """The stored backgrounds of the last forward, every depth, into the
        reference's checkpoint files (tags "down" and "up",
        ``propagator/src/OneWay.h:195-239``; file layout of
        ``propagator/src/WavefieldPool.cpp:78-100``)."""
        pool = self._pool()
        pool.store(self.bg_down, "down")
        pool.store(self.bg_up, "up")
        pool.wait_to_finish()

    def load_backgrounds(self, model):
        """Backgrounds of ``model`` read back from the checkpoint files of this
        propagator's pool (``par`` keys ``wfld_path`` and ``run_id`` name them),
        instead of modelling them again: the restart of a run whose forward was
        done earlier, with the same geometry."""
        with torch.cuda.device(self.device):
            self.set_background_model(model)
            pool = self._pool()
            self._ensure_storage()
            self.bg_down = pool.load("down", out=self.bg_down)
            self.bg_up = pool.load("up", out=self.bg_up)
            self._bg_key = tuple(id(v) for v in _model_pair(model))

    def born(self, dslow, dden, data, adjoint, add):
        """Extended Born on the stored backgrounds (packed or full)."""
        fn = self.plan.born_packed if self.packed else self.plan.born
        fn(self.rec, self.bg_down, self.bg_up, dslow, dden, data, adjoint=adjoint, add=add)

    def get_compression_ratio(self):
        """Bytes of a complex64 background wavefield over its stored bytes: 1
        uncompressed, 3.76 with compress_rate 8, 1.94 with compress_rate 16."""
        if not self.packed:
            return 1.0
        return 8.0 * float(np.prod(self.plan.wshape)) / self.plan.packed_bytes


class PackedGradientWarning(UserWarning):
    """The FWI gradient was computed on backgrounds kept in the lossy packed store."""


PACKED_GRADIENT_WARNING = (
    "compress_rate=8 keeps the background wavefields in the 8.5-bit packed store; the Born adjoint (the FWI "
    "gradient) on them differs from the lossless one by about 5e-3 relative L2 (measured on the 256 x 256 x 128 "
    "frequency workload), which is above the 1e-3 gradient tolerance of the lossless path.  Use compress_rate=16 "
    "(16.5 bits per value) or leave compress_rate unset for gradients that must meet it.")


class WindowExtendedBorn:
    """Extended Born modelling (domain [ds^2, drho], range data) about the
    background ``slow_den`` of a ``WindowPropagator``; ``adjoint`` is the FWI
    gradient (``fwix/workers.py:76``)."""

    def __init__(self, model, data, slow_den, propagator):
        self.prop = propagator
        self.slow_den = slow_den
        self.domain_shape = tuple(np.shape(_raw(_model_pair(model)[0])))

    def _background(self):
        p = self.prop
        if p._bg_key != tuple(id(v) for v in _model_pair(self.slow_den)) or p.bg_down is None:
            scratch = torch.zeros(p.range_shape, dtype=torch.complex64, device=p.device)
            p.forward(False, self.slow_den, scratch)

    def _model(self, model, zero):
        ds, dr = _model_pair(model)
        p = self.prop.plan
        shape = tuple(np.shape(_raw(ds)))
        if len(shape) != 4 or shape[0] != p.nz or shape[1] not in (1, p.nw) or shape[2:] != (p.ny, p.nx):
            raise ValueError(f"Born model must be [nz][nw or 1][ny][nx], got {shape}")
        return ds, dr, _dev(ds, self.prop.device, zero=zero), _dev(dr, self.prop.device, zero=zero)

    def forward(self, add, model, data):
        p = self.prop
        with torch.cuda.device(p.device):
            self._background()
            _, _, dsd, drd = self._model(model, zero=False)
            out = _dev(data, p.device) if add else _dev(data, p.device, zero=True)
            p.born(dsd, drd, out, adjoint=False, add=bool(add))
            _store(data, out)

    def adjoint(self, add, model, data):
        p = self.prop
        if p.packed and p.rate == 8:
            warnings.warn(PACKED_GRADIENT_WARNING, PackedGradientWarning, stacklevel=3)
        with torch.cuda.device(p.device):
            self._background()
            ds, dr, dsd, drd = self._model(model, zero=not add)
            d = _dev(data, p.device)
            p.born(dsd, drd, d, adjoint=True, add=bool(add))
            _store(ds, dsd)
            _store(dr, drd)


class PhaseShift:
    """``data (+)= P(s_ref) model`` on a spectrum [ns][nw][NY][NX] (``model`` and
    ``data`` share the hypercube; x and y axes give the wavenumbers, the third
    axis the frequencies in Hz)."""

    def __init__(self, model, data, dz, eps=0):
        h = _hyper(model, None, "wavefield")
        ax = h.getAxes()
        self.shape = h.shape
        self.device = _device(model, data)
        ns = int(np.prod([a.n for a in ax[3:]])) if len(ax) > 3 else 1
        self.plan = Plan(nx=ax[0].n, ny=ax[1].n, nw=ax[2].n, ns=ns, nz=1, dx=ax[0].d, dy=ax[1].d, dz=dz,
                         ow=ax[2].o, dw=ax[2].d, eps=eps, device=self.device)
        self.sref = None

    def set_slow(self, slow):
        """Reference s^2 of every frequency, [nw] complex."""
        s = _dev(slow, self.device).reshape(-1)
        if s.numel() != self.plan.nw:
            raise ValueError(f"set_slow expects {self.plan.nw} values")
        self.sref = s

    def _check(self):
        if self.sref is None:
            raise RuntimeError("PhaseShift: set_slow must be called first")

    def forward(self, add, model, data):
        self._check()
        with torch.cuda.device(self.device):
            out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
            self.plan.phase_shift(self.sref, _dev(model, self.device), out, L.PS_FWD, add=bool(add))
            _store(data, out)

    def adjoint(self, add, model, data):
        self._check()
        with torch.cuda.device(self.device):
            out = _dev(model, self.device) if add else _dev(model, self.device, zero=True)
            self.plan.phase_shift(self.sref, _dev(data, self.device), out, L.PS_ADJ, add=bool(add))
            _store(model, out)


class RefSampler:
    """Reference s^2 and labels of every depth of a slowness model
    (``propagator/src/RefSampler.cpp:49-90``), computed on the device once."""

    def __init__(self, slow, par):
        h = _hyper(slow, par, "model")
        _grid_from_model(h)
        padx, pady = int(_get(par, "padx", 0)), int(_get(par, "pady", 0))
        t = _raw(slow)
        dev = _device(slow)
        self.sref, self.labels = refsampler.sample(_dev(t, dev), int(_get(par, "nref", 1)), padx, pady,
                                                   method=str(_get(par, "ref_method", "quantile")))

    def get_ref_slow(self, iz, iref):
        return self.sref[iz, iref].cpu().numpy()

    def get_ref_labels(self, iz):
        return self.labels[iz].cpu().numpy().astype(np.int32)


class _OneStep:
    kind = "pspi"

    def __init__(self, model, data, slow, par):
        self.par = par
        wh = _hyper(model, par, "wavefield")
        sh = _hyper(slow, par, "model")
        x, y, w, z = _grid_from_model(sh)
        ax = wh.getAxes()
        padx, pady = ax[0].n - x.n, ax[1].n - y.n
        if padx < 0 or pady < 0 or ax[2].n != w.n:
            raise ValueError(f"wavefield {wh} does not match the slowness model {sh} plus padding")
        ns = int(np.prod([a.n for a in ax[3:]])) if len(ax) > 3 else 1
        self.device = _device(model, data, slow)
        par_kind = dict(par or {})
        par_kind["step"] = self.kind
        with torch.cuda.device(self.device):
            self.plan = _plan_from_slow(sh, par_kind, ns, self.device, padx=padx, pady=pady)
            _refs(self.plan, _dev(slow, self.device), par)
        self.iz = 0

    def set_depth(self, iz):
        if not 0 <= iz < self.plan.nz:
            raise RuntimeError(f"depth {iz} outside [0, {self.plan.nz})")
        self.iz = int(iz)

    def forward(self, add, model, data):
        with torch.cuda.device(self.device):
            out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
            self.plan.step(self.iz, _dev(model, self.device), out, direction=L.FWD, add=bool(add))
            _store(data, out)

    def adjoint(self, add, model, data):
        """Add-version adjoint: for PSPI it leaves out the taper, as the
        reference's ``PSPI::cu_adjoint(bool, ...)`` does (``propagator/src/PSPI.cpp:26-44``)."""
        with torch.cuda.device(self.device):
            out = _dev(model, self.device) if add else _dev(model, self.device, zero=True)
            self.plan.step(self.iz, _dev(data, self.device), out, direction=L.ADJ_ADD, add=bool(add))
            _store(model, out)


class PSPI(_OneStep):
    """PSPI depth step: taper, FFT, per reference phase shift and inverse FFT,
    select by label (``propagator/src/PSPI.cpp:6-103``)."""
    kind = "pspi"


class NSPS(_OneStep):
    """NSPS depth step: per reference select, FFT and phase shift, sum, one
    inverse FFT (``propagator/src/NSPS.cpp:6-45``)."""
    kind = "nsps"


class Injection:
    """Trilinear injection (forward: traces -> wavefield) and recording
    (adjoint) at the current depth (``propagator/src/injection.cu:7-188``).
    ``model`` is the traces [ntrace][nw], ``data`` the wavefield [ns][nw][NY][NX]
    whose x / y axes give the grid; ``oz``, ``dz`` the depth axis."""

    def __init__(self, model, data, oz, dz, cx, cy, cz, ids):
        wh = _hyper(data, None, "wavefield")
        ax = wh.getAxes()
        self.ax = ax
        self.ns = int(np.prod([a.n for a in ax[3:]])) if len(ax) > 3 else 1
        self.oz, self.dz = float(oz), float(dz)
        self.device = _device(model, data)
        self.iz = 0
        self.plan = None
        self.tr = None
        self.set_coords(cx, cy, cz, ids)

    def _build(self, nz):
        ax = self.ax
        self.plan = Plan(nx=ax[0].n, ny=ax[1].n, nw=ax[2].n, ns=self.ns, nz=nz, dx=ax[0].d, dy=ax[1].d,
                         dz=self.dz, ox=ax[0].o, oy=ax[1].o, oz=self.oz, ow=ax[2].o, dw=ax[2].d,
                         device=self.device)
        self.tr = self.plan.traces(self._coords[0], self._coords[1], self._coords[2], self._coords[3])

    def set_coords(self, cx, cy, cz, ids):
        cz_ = np.asarray(cz, dtype=np.float32)
        self._coords = (np.asarray(cx, np.float32), np.asarray(cy, np.float32), cz_, np.asarray(ids, np.int32))
        top = int(np.floor((float(cz_.max()) - self.oz) / self.dz)) + 2 if cz_.size else 1
        self._build(max(top, self.iz + 2, 2))

    def set_depth(self, iz):
        self.iz = int(iz)
        if self.iz + 1 >= self.plan.nz:
            self._build(self.iz + 2)

    def forward(self, add, model, data):
        with torch.cuda.device(self.device):
            out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
            self.plan.inject(self.tr, self.iz, _dev(model, self.device), out, adjoint=False, add=True)
            _store(data, out)

    def adjoint(self, add, model, data):
        with torch.cuda.device(self.device):
            out = _dev(model, self.device) if add else _dev(model, self.device, zero=True)
            self.plan.inject(self.tr, self.iz, out, _dev(data, self.device), adjoint=True, add=True)
            _store(model, out)


class _Sweep(_OneStep):
    """A whole-depth sweep.  ``forward(add, model, data)`` continues ``model``
    through every depth and adds the result to ``data``; ``forward(wfld)`` /
    ``adjoint(wfld)`` continue one wavefield in place, which is what the
    reference's Python classes end up exposing (their one-argument methods
    replace the three-argument ones, ``fwix/CudaWEM.py:131-141``)."""
    up = False

    def __init__(self, model, data, slow, par):
        par = dict(par or {})
        par.setdefault("step", "pspi")  # the reference's OneWay always runs PSPI
        self.kind = par["step"]
        super().__init__(model, data, slow, par)

    def _run(self, t, adjoint):
        (self.plan.upward if self.up else self.plan.downward)(t, adjoint=adjoint)

    def forward(self, *args):
        with torch.cuda.device(self.device):
            if len(args) == 1:
                t = _dev(args[0], self.device)
                self._run(t, False)
                _store(args[0], t)
                return
            add, model, data = args
            t = _dev(model, self.device).clone()
            self._run(t, False)
            out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
            out.add_(t)
            _store(data, out)

    def adjoint(self, *args):
        with torch.cuda.device(self.device):
            if len(args) == 1:
                t = _dev(args[0], self.device)
                self._run(t, True)
                _store(args[0], t)
                return
            add, model, data = args
            t = _dev(data, self.device).clone()
            self._run(t, True)
            out = _dev(model, self.device) if add else _dev(model, self.device, zero=True)
            out.add_(t)
            _store(model, out)


class Downward(_Sweep):
    """Depth 0 -> nz-1 continuation (``propagator/src/OneWay.cpp:19-48``)."""
    up = False


class Upward(_Sweep):
    """Depth nz-1 -> 0 continuation (``propagator/src/OneWay.cpp:50-79``)."""
    up = True


# The reference's Python Propagator always builds a StreamingPropagator
# (``fwix/CudaWEM.py:10-18``): shots and frequencies in ``nbatches`` groups, each
# on the window of the model its sources and receivers cover (plus ``ginsu_x`` /
# ``ginsu_y``).  These two keep that behaviour on top of the window classes.
from .streaming import StreamingExtendedBorn, StreamingPropagator  # noqa: E402


def slowness_model(s_real):
    """[s^2, density] model of a real slowness s [nz][ny][nx]: complex s^2 with a
    frequency axis of length 1 (shared by every frequency), density 1."""
    s = torch.as_tensor(s_real)
    if s.dim() != 3:
        raise ValueError(f"s_real must be [nz][ny][nx], got {tuple(s.shape)}")
    s2 = (s.double() ** 2)[:, None].to(torch.complex64).contiguous()
    return [s2, torch.ones_like(s2)]


class Propagator(StreamingPropagator):
    """Nonlinear modelling: wavelet -> recorded data for a [s^2, density] model,
    per (shot group, frequency band) on its acquisition window
    (``propagator/src/StreamingPropagator.cpp``, ``Propagator.cpp:121-221``).

    The background down- and up-going wavefields of the last ``forward`` stay in
    device memory (lossless, every depth) for :class:`ExtendedBorn`; the reference
    keeps ZFP-compressed copies on disk (``propagator/src/WavefieldPool.cpp``).

    Shortcuts beyond the reference's arguments: ``s_real`` (a real slowness
    [nz][ny][nx]) stands for the model [s^2, 1] (``model`` may then be None, in
    the constructor and in ``forward``; ``par`` carries the axes), and
    ``mode="smooth"`` models with the differentiable step (interpolation between
    the two bracketing references plus the split-step correction, density 1,
    the whole model in one batch) that ``fwi.FWIGradient`` differentiates;
    ``mode="parity"`` (default) is the reference's selection step."""

    def __init__(self, model, data, wavelet, par, geometry, nbatches=(1, 1), bands=None, mode="parity",
                 s_real=None):
        if mode not in ("parity", "smooth"):
            raise ValueError(f"mode must be 'parity' or 'smooth', got {mode!r}")
        self.mode = mode
        self.s_real = s_real
        self._s_model = None
        if s_real is not None:
            model = self._s_model = slowness_model(s_real)
        elif model is None:
            raise ValueError("Propagator needs a model or s_real")
        super().__init__(model, data, wavelet, par, geometry, nbatches, bands)
        self._smooth = None

    def _slowness_of(self, model):
        if model is None:
            if self.s_real is None:
                raise ValueError("forward needs a model (no s_real was given)")
            return torch.as_tensor(self.s_real)
        s2, _ = _model_pair(model)
        t = torch.as_tensor(_raw(s2))
        if t.dim() != 4 or t.shape[1] != 1:
            raise ValueError("mode='smooth' needs a frequency-independent model [nz][1][ny][nx] or s_real")
        return torch.sqrt(t[:, 0].real.double()).float()

    def forward(self, add, model, data):
        if self.mode == "parity":
            if model is None and self._s_model is None:
                raise ValueError("forward needs a model (no s_real was given)")
            return super().forward(add, model if model is not None else self._s_model, data)
        from .fwi import SmoothFWI
        s = self._slowness_of(model)
        if self._smooth is None:
            ax = self.ax
            par = {k: _get(self.par, k) for k in ("nref", "padx", "pady", "eps", "taperx", "tapery", "checkpoint",
                                                   "refs") if _get(self.par, k) is not None}
            par.update(ox=ax[0].o, dx=ax[0].d, oy=ax[1].o, dy=ax[1].d, ow=ax[2].o, dw=ax[2].d, oz=ax[3].o,
                       dz=ax[3].d)
            self._smooth = SmoothFWI(tuple(s.shape), {k: v for k, v in self.g.items()}, self.wavelet, par,
                                     device=self.device)
        d = self._smooth.model(s.to(self.device), keep=False)
        out = _dev(data, self.device) if add else _dev(data, self.device, zero=True)
        out += d
        _store(data, out)


class ExtendedBorn(StreamingExtendedBorn):
    """Extended Born modelling (domain [ds^2, drho], range data) about the
    background ``slow_den`` of ``propagator``; ``adjoint`` is the FWI gradient
    (``fwix/workers.py:76``, ``propagator/src/StreamingExtendedBorn.cpp``)."""
