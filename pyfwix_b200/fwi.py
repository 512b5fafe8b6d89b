"""FWI gradient with respect to slowness: modelling with the differentiable
("smooth") depth step and its adjoint-state gradient, behind a
``torch.autograd.Function``.

The reference's gradient is ``ExtendedBorn.adjoint`` of the data residual
(``fwix/workers.py:62-76``), a Born-linearised operator on s^2 per frequency.
Its modelling selects the nearest reference slowness per cell
(``propagator/src/selector.cu:29-35``), so the data depend on the slowness
only through piecewise-constant labels and cannot be differentiated cell by
cell.  Here the modelling keeps the reference's structure -- down pass with
source injection and recording, reflection, up pass with recording
(``propagator/src/Propagator.cpp:121-221``) -- with the smooth step
(``fwix_smooth_step``: interpolation between the two bracketing references
plus the split-step correction) so that J(s) = 1/2 |d(s) - d_obs|^2 has an exact
gradient:

  mu_iz = Rec_iz^H r + S_{iz-1}^H mu_{iz-1}                      (iz = 0 .. nz-1)
  nu_iz = Rec_iz^H r + conj(R_iz) mu_iz + S_iz^H nu_{iz+1}       (iz = nz-1 .. 0)
  dJ/ds = Re sum_{shots,w} [conj(mu_iz) dS_iz(U_{iz+1}) + conj(nu_{iz+1}) dS_iz(D_iz)]
          + dR/ds terms Re sum conj(mu_iz) D_iz

with D / U the down / up fields, R_iz = (s_iz - s_iz+1) / (s_iz + s_iz+1)
(density 1, ``propagator/src/reflect.cu:42-45``) and the reference
slownesses of each depth held fixed.  Every operator is a kernel of
libfwix_b200.so; this module only sequences them.

Storage: the down field, the up step's slowness derivative dS_iz(U_iz+1) (the
only use the gradient makes of U; the modelling's up pass takes it with the
paired step) and the mu field of every depth are kept in device memory
(``checkpoint=None``), or, with ``checkpoint=k``,
only every k-th down / up / mu field is kept and each k-level segment is
recomputed from its checkpoint when the backward sweeps reach it;
``checkpoint="auto"`` (the default) stores everything when it fits in device
memory and picks the interval otherwise.

With checkpoints the backward runs the mu recursion alone first (one adjoint
step per level, keeping mu at every segment start), then the nu recursion
segment by segment from the bottom, recomputing the segment's down fields, up
fields and mu fields and taking every gradient term there.  The down and up
recomputations use the paired step (``fwix_smooth_step_pair``: the step and its
slowness derivative from one set of transforms), so the derivative terms cost
little beyond the recomputation itself: about five steps per level for the
backward against three for the checkpointed forward.
"""
from __future__ import annotations

import collections
import hashlib
import weakref

import numpy as np
import torch

from . import _lib as L
from .plan import Plan

# Plans of recent SmoothFWI sizes, reused by later problems of the same sizes (the
# shots of one survey, the iterations of an inversion): a plan's tables, workspace
# and phase-factor cache are built once, and each problem rebinds its slowness,
# references and traces.  At most two are kept.
_PLAN_CACHE: "collections.OrderedDict[tuple, Plan]" = collections.OrderedDict()
_PLAN_CACHE_SIZE = 2


def _cached_plan(key, make):
    p = _PLAN_CACHE.get(key)
    if p is None:
        p = make()
        _PLAN_CACHE[key] = p
        while len(_PLAN_CACHE) > _PLAN_CACHE_SIZE:
            _PLAN_CACHE.popitem(last=False)
    else:
        _PLAN_CACHE.move_to_end(key)
    return p


def clear_plan_cache():
    """Releases the cached plans of earlier problems with their device memory:
    tables, workspace, phase-factor cache, the pooled stored-field blocks (tens
    of GB for a large every-depth gradient) and the trace lists."""
    _PLAN_CACHE.clear()


_TRACES_PER_PLAN = 16


def _traces(plan, cx, cy, cz, ids):
    """Gather lists of a trace set on ``plan``, kept while the plan lives (the
    last 16 sets): an FWI run visits the same shots every iteration, and the
    lists of a receiver on every surface node take a noticeable host time to
    build."""
    arrs = (np.ascontiguousarray(cx, np.float32), np.ascontiguousarray(cy, np.float32),
            np.ascontiguousarray(cz, np.float32), np.ascontiguousarray(ids, np.int32))
    h = hashlib.blake2b(digest_size=20)
    for a in arrs:
        h.update(np.int64(a.size).tobytes())
        h.update(a.tobytes())
    key = h.digest()
    cache = plan.__dict__.setdefault("_traces_cache", collections.OrderedDict())
    tr = cache.get(key)
    if tr is None:
        tr = plan.traces(*arrs)
        cache[key] = tr
        while len(cache) > _TRACES_PER_PLAN:
            cache.popitem(last=False)
    else:
        cache.move_to_end(key)
    return tr


def _pool(plan):
    """Stored-field blocks given back to a plan, keyed (family, fields)."""
    return plan.__dict__.setdefault("_fwi_blocks", {})


def smooth_refs(s, nref, spread=1e-3):
    """Reference slownesses per depth: nref values evenly spaced over the
    slice's [min, max] (slices narrower than spread * mean are widened)."""
    s = torch.as_tensor(s, dtype=torch.float64)
    lo = s.amin(dim=(1, 2))
    hi = s.amax(dim=(1, 2))
    mid, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
    half = torch.maximum(half, 0.5 * spread * mid)
    if nref == 1:
        return mid[:, None]
    return mid[:, None] + half[:, None] * torch.linspace(-1.0, 1.0, nref, dtype=torch.float64, device=s.device)


def pad_edge(s, padx, pady):
    """[nz][ny][nx] -> [nz][ny+pady][nx+padx], edge replicated."""
    if padx == 0 and pady == 0:
        return s
    return torch.nn.functional.pad(s[None], (0, padx, 0, pady), mode="replicate")[0]


def fold_edge(gp, ny, nx):
    """Transpose of pad_edge."""
    out = gp[:, :ny, :nx].clone()
    out[:, :, nx - 1] += gp[:, :ny, nx:].sum(dim=2)
    out[:, ny - 1, :] += gp[:, ny:, :nx].sum(dim=1)
    out[:, ny - 1, nx - 1] += gp[:, ny:, nx:].sum(dim=(1, 2))
    return out


def _get(par, key, default=None):
    v = par.get(key, default) if hasattr(par, "get") else getattr(par, key, default)
    return default if v is None else v


def _checkpoint_key(par):
    """``checkpoint`` of par: absent -> "auto"; None, 0 or 1 -> every depth
    stored; k -> every k-th level.  (A parameter object other than a dict cannot
    tell an absent key from None, and gives "auto" for both.)"""
    if isinstance(par, dict):
        return par.get("checkpoint", "auto")
    return _get(par, "checkpoint", "auto")


class SmoothFWI:
    """One shot batch: plan, acquisition and stored fields.

    ``par`` holds the grid axes (``ox, dx, oy, dy, oz, dz, ow, dw``; frequencies
    in Hz) and the step keys (``nref, padx, pady, eps, taperx, tapery``);
    optional ``refs`` ([nz][nref], fixed reference slownesses) and
    ``checkpoint`` (k, None for full storage, or "auto")."""

    def __init__(self, shape, geometry, wavelet, par, device=None):
        nz, ny, nx = shape
        wav = torch.as_tensor(wavelet)
        self.device = torch.device(device) if device is not None else (
            wav.device if wav.is_cuda else torch.device("cuda", torch.cuda.current_device()))
        self.par = par
        nw = wav.shape[1]
        from .CudaWEM import _remap_ids
        s_ids, r_ids, ns = _remap_ids(geometry["s_ids"], geometry["r_ids"])
        self.padx, self.pady = int(_get(par, "padx", 0)), int(_get(par, "pady", 0))
        kw = dict(nx=nx, ny=ny, nw=nw, ns=ns, nz=nz, dx=float(_get(par, "dx", 1.0)), dy=float(_get(par, "dy", 1.0)),
                  dz=float(_get(par, "dz", 1.0)), ox=float(_get(par, "ox", 0.0)), oy=float(_get(par, "oy", 0.0)),
                  oz=float(_get(par, "oz", 0.0)), ow=float(_get(par, "ow", 1.0)), dw=float(_get(par, "dw", 1.0)),
                  padx=self.padx, pady=self.pady, nref=int(_get(par, "nref", 2)), eps=float(_get(par, "eps", 0.0)),
                  taperx=int(_get(par, "taperx", 0)), tapery=int(_get(par, "tapery", 0)))
        key = (str(self.device),) + tuple(sorted(kw.items()))
        self.plan = _cached_plan(key, lambda: Plan(step="pspi", device=self.device, **kw))
        p = self.plan
        self.src = _traces(p, geometry["sx"], geometry["sy"], geometry["sz"], s_ids)
        self.rec = _traces(p, geometry["rx"], geometry["ry"], geometry["rz"], r_ids)
        self.wavelet = wav.to(self.device, torch.complex64).contiguous()
        self.ntrace = len(np.asarray(geometry["rx"]))
        # stored-field blocks in use; they go back to the plan's pool at the next
        # model() or when this problem is released
        self._held = {}
        weakref.finalize(self, _pool(p).update, self._held)
        self.Ds = self.dSU = self._blocks = None
        self.k = self._storage(_checkpoint_key(par))
        self.refs_fixed = _get(par, "refs", None)
        p.ensure_workspace(L.WS_STEP)

    def _storage(self, k):
        """None (every depth stored) or the checkpoint interval.  "auto" stores every
        depth when the down, up and mu fields of all depths fit in 60 % of the
        free device memory, else takes the smallest interval in 4, 8, ..., 256
        whose checkpoints plus segment buffers fit."""
        if k != "auto":
            return None if k in (None, 0, 1) else int(k)
        p = self.plan
        wb = p.ns * p.nw * p.NY * p.NX * 8
        free, _ = torch.cuda.mem_get_info(self.device)
        # memory torch's allocator holds but does not use (fields of an earlier shot)
        # is free for this shot's fields as well
        free += torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        # a reused plan's phase-factor cache belongs to the working set the budget
        # is for (a new plan allocates it after this decision)
        pc = p._keep.get("pcache") if hasattr(p, "_keep") else None
        if pc is not None:
            free += pc.numel() * pc.element_size()
        # and so are the stored-field blocks an earlier problem gave back to the plan
        for b in _pool(p).values():
            free += b.numel() * b.element_size()
        budget = 0.6 * free
        if 3 * p.nz * wb + 4 * wb <= budget:
            return None
        for k in (4, 8, 16, 32, 64, 128, 256):
            if self.checkpoint_fields(p.nz, k) * wb <= budget:
                return k
        return 256

    @staticmethod
    def checkpoint_fields(nz, k):
        """Wavefields held at once with checkpoints every k levels: the down, up
        and mu checkpoints, and one segment's down fields, their derivatives, the
        up derivatives and mu fields, plus working fields."""
        return 3 * (-(-nz // k)) + 4 * k + 6

    # ---------------------------------------------------------------- state
    def set_slowness(self, s):
        """Binds s [nz][ny][nx] (float): padded slowness, references, and s^2 /
        density 1 for the reflection coefficients."""
        p = self.plan
        s = torch.as_tensor(s).to(self.device, torch.float32).contiguous()
        self.s = s
        p._fwi_owner = weakref.ref(self)  # whose slowness the (possibly shared) plan holds
        refs = self.refs_fixed if self.refs_fixed is not None else smooth_refs(s, p.nref)
        self.refs = torch.as_tensor(refs).to(self.device, torch.float32)
        p.set_smooth(pad_edge(s, self.padx, self.pady), self.refs)
        s2 = (s.double() ** 2)[:, None].to(torch.complex64)
        p.set_model(s2, torch.ones_like(s2))

    def _field(self):
        return torch.zeros(self.plan.wshape, dtype=torch.complex64, device=self.device)

    # ---------------------------------------------------------------- modelling
    def _down_step(self, iz, D, data):
        """The checkpointed modelling's down step at iz (injection, recording, step)."""
        p = self.plan
        p.inject(self.src, iz, self.wavelet, D)
        p.inject(self.rec, iz, data, D, adjoint=True)
        p.smooth_step(iz, D, D)

    def _up_step(self, iz, U, Dz, data):
        """U_iz from U_iz+1 in place, with its reflection and recording."""
        p = self.plan
        p.smooth_step(iz, U, U)
        p.reflect(iz, Dz, U, add=True)
        p.inject(self.rec, iz, data, U, adjoint=True)

    def model(self, s, keep=True):
        """Data [ntrace][nw] for slowness s; with keep the fields the gradient
        needs are stored (all depths, or every k-th)."""
        self.set_slowness(s)
        self._give_back()  # the fields of an earlier model() are dead
        p, nz = self.plan, self.plan.nz
        data = torch.zeros((self.ntrace, p.nw), dtype=torch.complex64, device=self.device)
        if self.k is None:
            # one block per stored family (not nz fields), taken from the plan's pool:
            # the previous shot's block comes back whole, with no allocator traffic.
            # The up pass reflects every down field, so they are kept either way.
            # The gradient takes U only through dS_iz(U_iz+1): the up pass's paired
            # step stores that instead of U (one derivative step fewer per level in
            # the backward, the same memory).  Both passes run as one library call.
            dblk = self._take("D", nz)
            ublk = self._take("dSU", nz - 1) if keep and nz > 1 else None
            p.smooth_model_sweep(self.src, self.rec, self.wavelet, data, self._empty(), dblk, ublk)
            self.Ds = list(dblk)
            self.dSU = [ublk[iz] if ublk is not None and iz + 1 < nz else None for iz in range(nz)]
            self._blocks = (dblk, ublk)
            if not keep:
                self._give_back()
            return data
        k = self.k
        D = self._field()
        nck = -(-nz // k)
        dck, uck = self._take("Dck", nck), self._take("Uck", nck)
        self.Dck = {}
        for iz in range(nz):
            if iz % k == 0:
                dck[iz // k].copy_(D)   # the field before injection at iz
                self.Dck[iz] = dck[iz // k]
            self._down_step(iz, D, data)
        self.Uck = {nz: self._field()}
        U = self._field()
        bufs = dict(D=self._take("segD", k))
        for a in reversed(range(0, nz, k)):
            seg = self._segment_D(a, bufs)
            for iz in range(min(a + k, nz) - 1, a - 1, -1):
                self._up_step(iz, U, seg[iz - a], data)
            uck[a // k].copy_(U)
            self.Uck[a] = uck[a // k]
        if not keep:
            self._give_back()
        return data

    def _empty(self):
        return torch.empty(self.plan.wshape, dtype=torch.complex64, device=self.device)

    def _block(self, n):
        """n uninitialised fields in one allocation, [n][ns][nw][NY][NX]."""
        return torch.empty((n,) + tuple(self.plan.wshape), dtype=torch.complex64, device=self.device)

    def _take(self, name, n):
        """The block of n fields of the stored family ``name``, held until
        _give_back: the one the previous problem on this plan gave back (the same
        device memory, so a family of tens of GB is never carved up by smaller
        allocations or re-allocated behind a cache flush), else a new one."""
        b = self._held.get((name, n))
        if b is None:
            b = _pool(self.plan).pop((name, n), None)
        if b is None:
            b = self._block(n)
        self._held[(name, n)] = b
        return b

    def _give_back(self, families=None):
        """Returns held blocks (all, or those of ``families``) to the plan's pool
        once their fields are dead (later work on the same stream orders after the
        reads already enqueued)."""
        pool = _pool(self.plan)
        for key in [q for q in self._held if families is None or q[0] in families]:
            pool[key] = self._held.pop(key)
        if families is None:
            self.Ds = self.dSU = self._blocks = None
            self.Dck = self.Uck = None

    def _seg_buffers(self):
        """Fields of one checkpoint segment, taken once per sweep and reused by
        every segment: down fields, their derivatives, up derivatives, mu fields
        (k each) and two up fields for the walk."""
        k = self.k
        return dict(D=self._take("segD", k), dSD=self._take("segdSD", k), dSU=self._take("segdSU", k),
                    mu=self._take("segmu", k), U=self._take("segU", 2))

    def _segment_D(self, a, bufs, derivs=False):
        """Down fields D_a .. D_{a+k-1} (after injection) recomputed from the
        checkpoint at a, without recording; with ``derivs`` also dS_iz(D_iz) for
        every level of the segment above the bottom of the model.  Each step
        writes the next level's field (no copies); the fields live in ``bufs``."""
        p, nz = self.plan, self.plan.nz
        top = min(a + self.k, nz)
        Db, dDb = bufs["D"], bufs.get("dSD")
        D = Db[0]
        D.copy_(self.Dck[a])
        out, der = [], []
        for iz in range(a, top):
            p.inject(self.src, iz, self.wavelet, D)
            out.append(D)
            last = iz + 1 == top
            if derivs and iz + 1 < nz:
                d = dDb[iz - a]
                if last:
                    p.smooth_step(iz, D, d, mode=L.SMOOTH_DERIV)
                else:
                    nxt = Db[iz - a + 1]
                    p.smooth_step_pair(iz, D, nxt, d)
                    D = nxt
                der.append(d)
            elif not last:
                nxt = Db[iz - a + 1]
                p.smooth_step(iz, D, nxt)
                D = nxt
        return (out, der) if derivs else out

    def _segment_U_derivs(self, a, Dseg, bufs):
        """dS_iz(U_{iz+1}) for the levels iz of the segment above the bottom of the
        model, walking the up fields from the checkpoint U_{a+k} (which stays
        untouched) with the paired step; index iz - a."""
        p, nz = self.plan, self.plan.nz
        top = min(a + self.k, nz)
        der = [None] * (top - a)
        Ub, dUb = bufs["U"], bufs["dSU"]
        U = self.Uck[top]
        for j, iz in enumerate(range(top - 1, a - 1, -1)):
            nxt = Ub[j & 1]
            if iz + 1 < nz:
                d = dUb[iz - a]
                p.smooth_step_pair(iz, U, nxt, d)
                der[iz - a] = d
            else:
                nxt.zero_()   # the step of the zero field below the model
            if iz > a:
                p.reflect(iz, Dseg[iz - a], nxt, add=True)
                U = nxt
        return der

    def _segment_mu(self, a, bufs):
        """mu_a .. mu_{a+k-1} recomputed from mu_{a-1} (kept at a)."""
        p, nz = self.plan, self.plan.nz
        out = []
        m = self.Mck[a]
        Mb = bufs["mu"]
        for iz in range(a, min(a + self.k, nz)):
            nxt = Mb[iz - a]
            if iz > 0:
                p.smooth_step(iz - 1, m, nxt, mode=L.SMOOTH_ADJ)
            else:
                nxt.zero_()
            p.inject(self.rec, iz, self._res, nxt)
            out.append(nxt)
            m = nxt
        return out

    # ---------------------------------------------------------------- gradient
    def gradient(self, res):
        """dJ/ds [nz][ny][nx] (float32) for the residual res = d - d_obs, after
        model(s, keep=True)."""
        owner = getattr(self.plan, "_fwi_owner", None)
        if owner is None or owner() is not self:
            self.set_slowness(self.s)  # another problem rebound the shared plan since model()
        p, nz = self.plan, self.plan.nz
        res = torch.as_tensor(res).to(self.device, torch.complex64).contiguous()
        gpad = torch.zeros((nz, p.NY, p.NX), dtype=torch.float32, device=self.device)
        crefl = torch.zeros((nz, p.ny, p.nx), dtype=torch.float32, device=self.device)
        G = self._field()
        if self.k is None:
            if self.Ds is None:
                raise RuntimeError("gradient() needs model(s, keep=True) first")
            dblk, ublk = self._blocks
            mus = self._take("mu", nz)
            p.smooth_gradient_sweep(self.rec, res, dblk, ublk, mus, self._empty(), G, gpad, crefl)
        else:
            k = self.k
            self._res = res
            # mu recursion alone, keeping mu_{a-1} at every segment start a
            mu = self._field()
            mck = self._take("Mck", -(-nz // k))
            self.Mck = {}
            for iz in range(nz):
                if iz % k == 0:
                    mck[iz // k].copy_(mu)
                    self.Mck[iz] = mck[iz // k]
                if iz > 0:
                    p.smooth_step(iz - 1, mu, mu, mode=L.SMOOTH_ADJ)
                p.inject(self.rec, iz, res, mu)
            del mu
            # nu recursion segment by segment from the bottom, with every gradient term
            nu = self._field()
            bufs = self._seg_buffers()
            for a in reversed(range(0, nz, k)):
                Dseg, dSD = self._segment_D(a, bufs, derivs=True)
                dSU = self._segment_U_derivs(a, Dseg, bufs)
                mseg = self._segment_mu(a, bufs)
                for iz in range(min(a + k, nz) - 1, a - 1, -1):
                    j = iz - a
                    if iz + 1 < nz:
                        p.correlate(mseg[j], dSU[j], gpad[iz], add=True, padded=True)
                        p.correlate(mseg[j], Dseg[j], crefl[iz], add=True, padded=False)
                        p.correlate(nu, dSD[j], gpad[iz], add=True, padded=True)
                    p.smooth_step(iz, nu, nu, mode=L.SMOOTH_ADJ)
                    p.reflect(iz, mseg[j], nu, adjoint=True, add=True)
                    p.inject(self.rec, iz, res, nu)
                del Dseg, dSD, dSU, mseg
            self._res = None
            self.Mck = None
        # the gradient's own blocks; the modelling's stay for another gradient call
        self._give_back(("mu", "Mck", "segD", "segdSD", "segdSU", "segmu", "segU"))
        # reflection coefficients r_iz = (s_iz - s_iz+1) / (s_iz + s_iz+1)
        s = self.s
        grefl = torch.zeros_like(crefl)
        if nz > 1:
            s0, s1 = s[:-1], s[1:]
            den = (s0 + s1) ** 2
            grefl[:-1] += crefl[:-1] * (2 * s1 / den)
            grefl[1:] += crefl[:-1] * (-2 * s0 / den)
        return fold_edge(gpad, p.ny, p.nx) + grefl


class FWIGradient(torch.autograd.Function):
    """J = 1/2 |d(s) - d_obs|^2 for slowness s [nz][ny][nx] (float32, device);
    backward returns dJ/ds.  ``FWIGradient.apply(s, wavelet, geometry, d_obs, par)``."""

    last_storage = None  # "every depth" or the checkpoint interval of the last call

    @staticmethod
    def forward(ctx, s, wavelet, geometry, d_obs, par):
        prob = SmoothFWI(tuple(s.shape), geometry, wavelet, par, device=s.device if s.is_cuda else None)
        FWIGradient.last_storage = "every depth" if prob.k is None else prob.k
        data = prob.model(s.detach(), keep=True)
        res = data - torch.as_tensor(d_obs).to(prob.device, torch.complex64)
        ctx.prob, ctx.res = prob, res
        J = 0.5 * torch.sum(res.real.double() ** 2 + res.imag.double() ** 2)
        return J.to(s.dtype) if s.is_floating_point() else J

    @staticmethod
    def backward(ctx, gJ):
        g = ctx.prob.gradient(ctx.res)
        ctx.prob = ctx.res = None
        return (gJ * g).to(gJ.dtype), None, None, None, None


def shot_objective_and_gradient(s, shot_list, par, group=None, device=None):
    """J = 1/2 sum_i |d_i(s) - d_obs_i|^2 and dJ/ds over a list of shots, each
    rank of the process group running its share of the shots.

    This replaces the reference's shot loop and reduction: Dask workers each run
    a partition of the shots in micro-batches, accumulating the misfit and the
    ExtendedBorn adjoint of the residual (``fwix/workers.py:14-83``,
    ``_obj_grad_worker``), and the per-worker gradients are summed by a streaming
    Zarr reduction (``fwix/workers.py:154-177``, ``_reduce_vector``).  Here the
    shots are partitioned across the ranks by cost (longest first,
    ``pyfwix_b200.shots.partition``), each rank models and differentiates its
    own shots with no communication (the smooth-step modelling and
    adjoint-state gradient of ``SmoothFWI``), and one all-reduce sums J and the
    gradient (NCCL over NVLink between GPUs).  Without a process group it is the
    plain sum over all shots.

    ``s``: slowness [nz][ny][nx] (float32; its device is the one used unless
    ``device`` is given).  ``shot_list``: dicts with ``geometry`` (the
    reference's geometry dict), ``wavelet`` [nsrc][nw] and ``d_obs`` [ntrace][nw];
    a rank reads ``d_obs`` only for its own shots, so the other entries may hold
    None.  ``par`` as for ``SmoothFWI``; its ``refs`` (fixed reference slownesses)
    default to ``smooth_refs(s)`` on every rank alike.  Returns (J, gradient)
    identical on every rank."""
    from . import shots as _shots
    s = torch.as_tensor(s)
    dev = torch.device(device) if device is not None else s.device
    s = s.to(dev, torch.float32)
    nz, ny, nx = s.shape
    par = dict(par) if isinstance(par, dict) else {k: _get(par, k) for k in (
        "ox", "dx", "oy", "dy", "oz", "dz", "ow", "dw", "nref", "padx", "pady", "eps", "taperx", "tapery",
        "checkpoint", "refs") if _get(par, k) is not None}
    if par.get("refs") is None:
        par["refs"] = smooth_refs(s, int(par.get("nref", 2))).to(torch.float32)
    costs = [_shots.shot_cost(nx, ny, torch.as_tensor(sh["wavelet"]).shape[1], nz) for sh in shot_list]

    def work(i):
        sh = shot_list[i]
        prob = SmoothFWI(tuple(s.shape), sh["geometry"], torch.as_tensor(sh["wavelet"]).to(dev), par, device=dev)
        data = prob.model(s, keep=True)
        res = data - torch.as_tensor(sh["d_obs"]).to(dev, torch.complex64)
        J = 0.5 * float(torch.sum(res.real.double() ** 2 + res.imag.double() ** 2))
        return J, prob.gradient(res)

    return _shots.objective_and_gradient(costs, work, s, group)


class FWIShotsGradient(torch.autograd.Function):
    """J over many shots spread across the ranks of the process group
    (``shot_objective_and_gradient``); backward returns the summed dJ/ds.
    ``FWIShotsGradient.apply(s, shot_list, par)``.  The gradient is computed with
    the objective (each shot's stored fields are released before the next shot
    runs) and handed out by backward."""

    @staticmethod
    def forward(ctx, s, shot_list, par, group=None):
        J, g = shot_objective_and_gradient(s.detach(), shot_list, par, group=group)
        ctx.g = g
        out = torch.tensor(J, dtype=torch.float64, device=s.device)
        return out.to(s.dtype) if s.is_floating_point() else out

    @staticmethod
    def backward(ctx, gJ):
        g = ctx.g
        ctx.g = None
        return (gJ * g).to(gJ.dtype), None, None, None
