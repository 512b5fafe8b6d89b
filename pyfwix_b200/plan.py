"""Plan object: owns a C-ABI plan, its workspace and the bound inputs.

Arrays are torch CUDA tensors in the reference layouts (complex64, x fastest):
wavefield [ns][nw][NY][NX], model [nz][nw][ny][nx], labels [nz][nw][NY][NX]
(uint8), refs [nz][nref][nw], traces [ntrace][nw].  Every call is enqueued on
torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L

STEP_KINDS = {"pspi": L.STEP_PSPI, "nsps": L.STEP_NSPS}


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _c64(t, device):
    t = torch.as_tensor(t)
    if not t.is_complex():
        t = t.to(torch.float32)
    return t.to(device=device, dtype=torch.complex64).contiguous()


class Plan:
    """One wavefield geometry (NX x NY x nw x ns) over nz depth levels plus the
    ``par`` keys of the path."""

    def __init__(self, nx, ny, nw, ns, nz, dx=1.0, dy=1.0, dz=1.0, ox=0.0, oy=0.0, oz=0.0,
                 ow=1.0, dw=1.0, padx=0, pady=0, nref=1, eps=0.0, taperx=0, tapery=0,
                 eps_scat=0.04, taylor=1, step="pspi", device=None):
        self.lib = L.load()
        self.device = torch.device(device if device is not None else "cuda")
        self.desc = L.FwixDesc(nx=nx, ny=ny, padx=padx, pady=pady, nw=nw, ns=ns, nz=nz,
                               ox=ox, oy=oy, oz=oz, dx=dx, dy=dy, dz=dz, ow=ow, dw=dw,
                               nref=nref, eps=eps, taperx=taperx, tapery=tapery,
                               eps_scat=eps_scat, taylor=taylor, step_kind=STEP_KINDS[step])
        self.nx, self.ny, self.nw, self.ns, self.nz = nx, ny, nw, ns, nz
        self.NX, self.NY = nx + padx, ny + pady
        self.nref, self.taylor, self.step_kind = nref, taylor, STEP_KINDS[step]
        self.pack_bits = 8
        self._h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            L.check(self.lib.fwix_plan_create(ctypes.byref(self.desc), ctypes.byref(self._h)))
        self._ws = None
        self._keep = {}

    # ------------------------------------------------------------------ shapes
    @property
    def wshape(self):
        return (self.ns, self.nw, self.NY, self.NX)

    @property
    def mshape(self):
        return (self.nz, self.nw, self.ny, self.nx)

    def wavefield(self, zero=True):
        f = torch.zeros if zero else torch.empty
        return f(self.wshape, dtype=torch.complex64, device=self.device)

    # ------------------------------------------------------------------ binding
    def ensure_workspace(self, cls=L.WS_STEP):
        need = int(self.lib.fwix_plan_workspace_bytes(self._h, cls))
        if self._ws is None or self._ws.numel() < need:
            self._ws = None
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
            L.check(self.lib.fwix_plan_set_workspace(self._h, _p(self._ws), need))
        return self._ws

    def enable_phase_cache(self, max_fraction=0.4, depths=None):
        """Bind a phase-factor cache (each depth's factors computed once and reused)
        of every depth, or of ``depths`` depths in rotation, when it fits in
        ``max_fraction`` of the device's free memory.  Returns whether the cache
        is on."""
        need = int(self.lib.fwix_plan_phase_cache_bytes(self._h))
        if depths is not None:
            need = need // self.nz * max(1, min(int(depths), self.nz))
        free, _ = torch.cuda.mem_get_info(self.device)
        # memory torch's allocator holds but does not use counts as free
        free += torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        if need == 0 or need > max_fraction * free:
            return False
        self._keep["pcache"] = torch.empty(need, dtype=torch.uint8, device=self.device)
        L.check(self.lib.fwix_plan_set_phase_cache(self._h, _p(self._keep["pcache"]), need))
        return True

    def disable_phase_cache(self):
        L.check(self.lib.fwix_plan_set_phase_cache(self._h, ctypes.c_void_p(0), 0))
        self._keep.pop("pcache", None)

    def set_refs(self, sref, labels, phase_cache=True):
        """sref [nz][nref][nw] complex; labels [nz][nw or 1][NY][NX] integer.  With
        ``phase_cache`` a phase-factor cache is bound: every depth when memory
        allows, else four depths in rotation."""
        sref = _c64(sref, self.device)
        if tuple(sref.shape) != (self.nz, self.nref, self.nw):
            raise ValueError(f"sref shape {tuple(sref.shape)} != {(self.nz, self.nref, self.nw)}")
        labels = torch.as_tensor(labels)
        if labels.dim() != 4 or tuple(labels.shape[2:]) != (self.NY, self.NX) or labels.shape[0] != self.nz \
                or labels.shape[1] not in (1, self.nw):
            raise ValueError(f"labels shape {tuple(labels.shape)} does not match [nz][nw|1][NY][NX]")
        if labels.numel() and (int(labels.min()) < 0 or int(labels.max()) > 255):
            raise ValueError("labels must lie in [0, 255]")
        labels = labels.to(device=self.device, dtype=torch.uint8).contiguous()
        wst = 0 if labels.shape[1] == 1 else self.NY * self.NX
        zst = labels.shape[1] * self.NY * self.NX
        L.check(self.lib.fwix_plan_set_refs(self._h, _p(sref), _p(labels), zst, wst))
        self._keep["sref"], self._keep["labels"] = sref, labels
        self._keep.pop("sm_ref_bound", None)  # the smooth references no longer match the bound ones
        if phase_cache and "pcache" not in self._keep and not self.enable_phase_cache():
            # no room for every depth: a few depths in rotation still spare the
            # column passes the per-sample factors (a migration level reuses its table)
            self.enable_phase_cache(depths=min(self.nz, 4))
        return sref, labels

    def set_model(self, slow, den):
        """Background s^2 and density, [nz][nw or 1][ny][nx] complex."""
        slow = _c64(slow, self.device)
        den = _c64(den, self.device)
        for t in (slow, den):
            if t.dim() != 4 or tuple(t.shape[2:]) != (self.ny, self.nx) or t.shape[0] != self.nz \
                    or t.shape[1] not in (1, self.nw):
                raise ValueError(f"model shape {tuple(t.shape)} does not match [nz][nw|1][ny][nx]")
        if slow.shape != den.shape:
            raise ValueError("slowness and density shapes differ")
        wst = 0 if slow.shape[1] == 1 else self.ny * self.nx
        zst = slow.shape[1] * self.ny * self.nx
        L.check(self.lib.fwix_plan_set_model(self._h, _p(slow), _p(den), zst, wst))
        self._keep["slow"], self._keep["den"] = slow, den
        return slow, den

    def set_smooth(self, slow_pad, sref_real):
        """Smooth step inputs: padded slowness [nz][NY][NX] and sorted real
        reference slownesses [nz][nref] (float).  Also binds the references'
        phase factors (s_r^2 for every frequency) through set_refs."""
        sp = torch.as_tensor(slow_pad).to(device=self.device, dtype=torch.float32).contiguous()
        sr = torch.as_tensor(sref_real).to(device=self.device, dtype=torch.float32).contiguous()
        if tuple(sp.shape) != (self.nz, self.NY, self.NX) or tuple(sr.shape) != (self.nz, self.nref):
            raise ValueError("smooth inputs must be [nz][NY][NX] and [nz][nref]")
        if self.nref > 1 and not bool(torch.all(sr[:, 1:] > sr[:, :-1])):
            raise ValueError("reference slownesses must increase strictly within each depth")
        prev = self._keep.get("sm_ref_bound")
        if prev is None or prev.shape != sr.shape or not torch.equal(prev, sr):
            # new references: their phase factors replace the cached ones; the same
            # references as bound keep the cache (the shots of one inversion step)
            sref2 = (sr.double() ** 2)[:, :, None].expand(self.nz, self.nref, self.nw).to(torch.complex64)
            labels = torch.zeros((self.nz, 1, self.NY, self.NX), dtype=torch.uint8, device=self.device)
            self.set_refs(sref2, labels)
            self._keep["sm_ref_bound"] = sr.clone()
        L.check(self.lib.fwix_plan_set_smooth(self._h, _p(sp), _p(sr)))
        self._keep["sm_s"], self._keep["sm_ref"] = sp, sr
        return sp, sr

    # ------------------------------------------------------------------ operators
    def smooth_step(self, iz, inp, out, mode=L.SMOOTH_FWD, add=False):
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_smooth_step(self._h, iz, mode, _p(inp), _p(out), int(add), _stream()))
        return out

    def autotune(self, iz=None, reps=3, kind=None):
        """Times the equivalent implementations of this plan's depth step (column
        tiles by cp.async or TMA, slices per launch, the one-launch cluster step at
        256 x 256) on a random wavefield at level ``iz`` (the middle one by
        default) and keeps the fastest (fwix_plan_autotune).  Synchronises the
        current stream.  Returns the choice as a dict."""
        self.ensure_workspace(L.WS_STEP)
        k = self.step_kind if kind is None else STEP_KINDS.get(kind, kind)
        iz = self.nz // 2 if iz is None else int(iz)
        x = torch.randn(self.wshape, dtype=torch.complex64, device=self.device)
        y = torch.empty_like(x)
        res = L.FwixTuning()
        L.check(self.lib.fwix_plan_autotune(self._h, k, iz, _p(x), _p(y), int(reps), _stream(), ctypes.byref(res)))
        return {"col_tma": bool(res.col_tma), "fused_cluster_step": bool(res.fused),
                "slices_per_launch": int(res.slices_per_launch), "streams": int(res.streams),
                "step_ms": float(res.ms), "candidates": int(res.candidates)}

    def set_tuning(self, choice):
        """Applies a choice ``autotune`` returned (the dict, for a plan of the same
        sizes) without timing anything (fwix_plan_set_tuning)."""
        t = L.FwixTuning()
        t.col_tma = int(bool(choice["col_tma"]))
        t.fused = int(bool(choice.get("fused_cluster_step", False)))
        t.slices_per_launch = int(choice["slices_per_launch"])
        t.streams = int(choice.get("streams", 1))
        L.check(self.lib.fwix_plan_set_tuning(self._h, ctypes.byref(t)))

    def smooth_step_pair(self, iz, inp, out, deriv, add=False):
        """out (+)= the smooth forward step of inp and deriv (+)= its slowness
        derivative, from one set of transforms."""
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_smooth_step_pair(self._h, iz, _p(inp), _p(out), _p(deriv), int(add), _stream()))
        return out, deriv

    def smooth_model_sweep(self, src, rec, wavelet, data, U, Ds, dSU=None):
        """Every-depth modelling sweep of the smooth step (fwix_smooth_model_sweep):
        data = recorded wavefield, Ds [nz] down fields (the recursion runs in
        them), dSU [nz-1] (or None) the up pass's step derivatives; U a working
        field."""
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_smooth_model_sweep(self._h, src._h, rec._h, _p(wavelet), _p(data), _p(U), _p(Ds),
                                                 _p(dSU), _stream()))

    def smooth_gradient_sweep(self, rec, res, Ds, dSU, mus, nu, G, gpad, crefl):
        """Every-depth gradient sweep (fwix_smooth_gradient_sweep): gpad [nz][NY][NX]
        and crefl [nz][ny][nx] (float) overwritten with the correlations; mus [nz]
        receives the mu fields (the recursion runs in them); nu, G working fields."""
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_smooth_gradient_sweep(self._h, rec._h, _p(res), _p(Ds), _p(dSU), _p(mus), _p(nu),
                                                    _p(G), _p(gpad), _p(crefl), _stream()))

    def correlate(self, a, b, out, add=False, padded=True):
        """out (+)= Re sum_{shots, w} conj(a) b, [NY][NX] (padded) or [ny][nx]."""
        L.check(self.lib.fwix_correlate(self._h, _p(a), _p(b), _p(out), int(add), int(padded), _stream()))
        return out

    def fft2d(self, inp, out, inverse=False, add=False):
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_fft2d(self._h, int(inverse), _p(inp), _p(out), int(add), _stream()))
        return out

    def phase_shift(self, sref_w, inp, out, mode=L.PS_FWD, add=False):
        sref_w = _c64(sref_w, self.device)
        L.check(self.lib.fwix_phase_shift(self._h, mode, _p(sref_w), _p(inp), _p(out), int(add), _stream()))
        return out

    def select(self, iz, value, inp, out, add=False):
        L.check(self.lib.fwix_select(self._h, iz, value, _p(inp), _p(out), int(add), _stream()))
        return out

    def taper(self, inp, out, add=False):
        L.check(self.lib.fwix_taper(self._h, _p(inp), _p(out), int(add), _stream()))
        return out

    def step(self, iz, inp, out, direction=L.FWD, add=False, kind=None):
        self.ensure_workspace(L.WS_STEP)
        k = self.step_kind if kind is None else STEP_KINDS.get(kind, kind)
        L.check(self.lib.fwix_step(self._h, k, iz, direction, _p(inp), _p(out), int(add), _stream()))
        return out

    def scatter(self, iz, inp, out, adjoint=False, add=False):
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_scatter(self._h, iz, int(adjoint), _p(inp), _p(out), int(add), _stream()))
        return out

    def reflect(self, iz, inp, out, adjoint=False, add=False):
        L.check(self.lib.fwix_reflect(self._h, iz, int(adjoint), _p(inp), _p(out), int(add), _stream()))
        return out

    def imaging(self, bg, image, wfld, adjoint=False, add=False):
        L.check(self.lib.fwix_imaging(self._h, int(adjoint), _p(bg), _p(image), _p(wfld), int(add), _stream()))

    def lin_reflect(self, iz, dmodel, dr, adjoint=False, add=False):
        L.check(self.lib.fwix_lin_reflect(self._h, iz, int(adjoint), _p(dmodel), _p(dr), int(add), _stream()))

    def traces(self, cx, cy, cz, ids):
        return Traces(self, cx, cy, cz, ids)

    def inject(self, tr, iz, traces, wfld, adjoint=False, add=True):
        L.check(self.lib.fwix_inject(self._h, tr._h, iz, int(adjoint), _p(traces), _p(wfld), int(add), _stream()))

    # ------------------------------------------------------------------ sweeps
    def downward(self, wfld, adjoint=False):
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_downward(self._h, int(adjoint), _p(wfld), _stream()))
        return wfld

    def upward(self, wfld, adjoint=False):
        self.ensure_workspace(L.WS_STEP)
        L.check(self.lib.fwix_upward(self._h, int(adjoint), _p(wfld), _stream()))
        return wfld

    def propagate(self, src, rec, wavelet, data, bg_down, bg_up=None, add=False):
        self.ensure_workspace(L.WS_SWEEP)
        L.check(self.lib.fwix_propagate(self._h, src._h, rec._h, _p(wavelet), _p(data), int(add),
                                        _p(bg_down), _p(bg_up), _stream()))
        return data

    def migrate(self, src, rec, wavelet, data, image, add=False):
        self.ensure_workspace(L.WS_SWEEP)
        L.check(self.lib.fwix_migrate(self._h, src._h, rec._h, _p(wavelet), _p(data), _p(image), int(add),
                                      _stream()))
        return image

    # -------------------------------------------------------------- packed store
    @property
    def packed_bytes(self):
        """Bytes of one packed wavefield at the plan's rate (8.5 or 16.5 bits per value)."""
        return int(self.lib.fwix_plan_packed_bytes(self._h))

    def set_pack_rate(self, bits):
        """Mantissa bits of the packed store, 8 (default) or 16."""
        L.check(self.lib.fwix_plan_set_pack_rate(self._h, int(bits)))
        self.pack_bits = int(bits)

    def packed(self, nfields=1, host=False):
        """Uninitialised storage for nfields packed wavefields (uint8 tensor), in
        device memory or, with ``host``, in pinned host memory: the packing and
        unpacking kernels then write and read it directly over the host link
        (pinned host memory is addressable from the device with the same
        pointer), which keeps the stored backgrounds out of device memory."""
        if host:
            return torch.empty((nfields, self.packed_bytes), dtype=torch.uint8, pin_memory=True)
        return torch.empty((nfields, self.packed_bytes), dtype=torch.uint8, device=self.device)

    def pack(self, wfld, packed):
        """One wavefield into packed storage at the plan's rate."""
        L.check(self.lib.fwix_pack_wavefield(self._h, _p(wfld), _p(packed), _stream()))
        return packed

    def unpack(self, packed, wfld):
        L.check(self.lib.fwix_unpack_wavefield(self._h, _p(packed), _p(wfld), _stream()))
        return wfld

    def propagate_packed(self, src, rec, wavelet, data, packed_down, packed_up=None, add=False):
        """Modelling with the down / up fields of every depth stored packed
        ([nz][packed_bytes] uint8 tensors)."""
        self.ensure_workspace(L.WS_SWEEP)
        L.check(self.lib.fwix_propagate_packed(self._h, src._h, rec._h, _p(wavelet), _p(data), int(add),
                                               _p(packed_down), _p(packed_up), _stream()))
        return data

    def born_packed(self, rec, packed_down, packed_up, dslow, dden, data, adjoint=False, add=False):
        """Extended Born on packed backgrounds (see born)."""
        self.ensure_workspace(L.WS_BORN_PACKED)
        nwm = dslow.shape[1] if dslow.dim() == 4 else self.nw
        if tuple(dslow.shape) != tuple(dden.shape) or nwm not in (1, self.nw):
            raise ValueError("dslow / dden must both be [nz][nw or 1][ny][nx]")
        mw = 0 if (nwm == 1 and self.nw > 1) else self.ny * self.nx
        L.check(self.lib.fwix_born_packed(self._h, int(adjoint), rec._h, _p(packed_down), _p(packed_up), _p(dslow),
                                          _p(dden), mw, _p(data), int(add), _stream()))

    def born(self, rec, bg_down, bg_up, dslow, dden, data, adjoint=False, add=False):
        """Extended Born.  dslow / dden are [nz][nw][ny][nx] (per frequency) or
        [nz][1][ny][nx] (one perturbation per depth for every frequency)."""
        self.ensure_workspace(L.WS_BORN)
        nwm = dslow.shape[1] if dslow.dim() == 4 else self.nw
        if tuple(dslow.shape) != tuple(dden.shape) or nwm not in (1, self.nw):
            raise ValueError("dslow / dden must both be [nz][nw or 1][ny][nx]")
        mw = 0 if (nwm == 1 and self.nw > 1) else self.ny * self.nx
        L.check(self.lib.fwix_born(self._h, int(adjoint), rec._h, _p(bg_down), _p(bg_up), _p(dslow), _p(dden),
                                   mw, _p(data), int(add), _stream()))

    def __del__(self):
        try:
            if self._h:
                self.lib.fwix_plan_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


class Traces:
    """Trace coordinates (host) turned into per-depth gather lists on the device
    (``propagator/src/injection.cu:33-71`` weights)."""

    def __init__(self, plan, cx, cy, cz, ids):
        self.plan = plan
        cx = np.ascontiguousarray(cx, dtype=np.float32)
        cy = np.ascontiguousarray(cy, dtype=np.float32)
        cz = np.ascontiguousarray(cz, dtype=np.float32)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        n = len(cx)
        if not (len(cy) == len(cz) == len(ids) == n):
            raise ValueError("coordinate and id arrays differ in length")
        self.ntrace = n
        self._h = ctypes.c_void_p()
        with torch.cuda.device(plan.device):
            L.check(plan.lib.fwix_traces_create(plan._h, n, cx.ctypes.data_as(ctypes.c_void_p),
                                                cy.ctypes.data_as(ctypes.c_void_p),
                                                cz.ctypes.data_as(ctypes.c_void_p),
                                                ids.ctypes.data_as(ctypes.c_void_p), ctypes.byref(self._h)))

    def __del__(self):
        try:
            if self._h:
                self.plan.lib.fwix_traces_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


def _addr(t):
    return t.data_ptr() if t is not None else None


def sweep(kind, instances, streams=()):
    """One batched sweep (``fwix_sweep``) over instances, each a dict with its
    ``plan`` and the arrays of that sweep kind (``src``, ``rec``: Traces;
    ``wavelet``, ``data``, ``wfld``, ``image``, ``bg_down``, ``bg_up``, ``dslow``,
    ``dden``: tensors; ``adjoint``, ``add``: flags).  Instances run on the given
    torch streams (largest first onto the least loaded), joined back into the
    current stream; no streams runs them one after the other on it."""
    n = len(instances)
    arr = (L.FwixInstance * max(n, 1))()
    for k, d in enumerate(instances):
        plan = d["plan"]
        plan.ensure_workspace(L.WS_BORN if kind in (L.SWEEP_BORN_FWD, L.SWEEP_BORN_ADJ) else
                              L.WS_SWEEP if kind in (L.SWEEP_MODEL, L.SWEEP_IMAGE) else L.WS_STEP)
        mw = 0
        if d.get("dslow") is not None:
            ds = d["dslow"]
            mw = 0 if (ds.shape[1] == 1 and plan.nw > 1) else plan.ny * plan.nx
        arr[k] = L.FwixInstance(
            plan=plan._h.value, src=d["src"]._h.value if d.get("src") is not None else None,
            rec=d["rec"]._h.value if d.get("rec") is not None else None,
            wavelet=_addr(d.get("wavelet")), data=_addr(d.get("data")), wfld=_addr(d.get("wfld")),
            image=_addr(d.get("image")), bg_down=_addr(d.get("bg_down")), bg_up=_addr(d.get("bg_up")),
            dslow=_addr(d.get("dslow")), dden=_addr(d.get("dden")), model_w_stride=mw,
            adjoint=int(d.get("adjoint", 0)), add=int(d.get("add", 0)))
    hs = (ctypes.c_void_p * max(len(streams), 1))(*[s.cuda_stream for s in streams])
    lib = L.load()
    L.check(lib.fwix_sweep(int(kind), arr, n, hs, len(streams), _stream()))
