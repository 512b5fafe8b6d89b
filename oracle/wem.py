"""CPU restatement of pyfwix's one-way wave-equation depth-stepping path.

TEST INFRASTRUCTURE ONLY.  This module is the oracle: the parity tests, the
``smoke()`` check and the ``cpu_baseline`` leg of ``bench.py`` import it as the
checker.  The product path (``pyfwix_b200``) never imports it and never falls
back to it.

Everything here follows the reference's CUDA kernels and C++ drivers line for
line (citations are ``path:line`` inside the pyfwix project).  Arithmetic is
complex128 by default (the FP64 oracle); ``dtype=np.complex64`` turns the same
code into the FP32 CPU port that ``bench.py`` times (FFTs then go through
``scipy.fft`` with ``workers=N``).

Layouts (row-major, x fastest), as ``operator/src/complex_vector.h:10-20``:
  wavefield  [ns][nw][NY][NX]   complex      (NX = nx + padx, NY = ny + pady)
  model s^2  [nz][nw][ny][nx]   complex      (``fwix/utils.py:211``: 1/v^2)
  labels     [nz][nw][NY][NX]   int          (``propagator/src/RefSampler.cpp:27``)
  refs       [nz][nref][nw]     complex      (``propagator/src/RefSampler.cpp:28``)
  traces     [ntrace][nw]       complex      (``propagator/src/injection.cu:15-17``)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_FFT_WORKERS = None  # None -> numpy.fft; int -> scipy.fft with that many workers


def set_fft_workers(workers):
    """Route the unitary 2D FFTs through scipy.fft with ``workers`` threads
    (used by the FP32 CPU baseline); ``None`` restores numpy.fft."""
    global _FFT_WORKERS
    _FFT_WORKERS = workers


def fft2(x):
    """Unitary forward 2D DFT over the last two axes (e^{-i}, x 1/sqrt(nx*ny)).

    ``operator/src/FFT.cpp:22-28,36-44`` plans a rank-2 C2C transform over
    (ny, nx) for every (shot, frequency) and ``operator/src/fft_callback.cu:7-12``
    multiplies every stored output by rsqrt(nx*ny)."""
    if _FFT_WORKERS is not None:
        import scipy.fft as sfft
        return sfft.fft2(x, axes=(-2, -1), norm="ortho", workers=_FFT_WORKERS)
    return np.fft.fft2(x, axes=(-2, -1), norm="ortho")


def ifft2(x):
    """Unitary inverse 2D DFT (e^{+i}, x 1/sqrt(nx*ny)): ``CUFFT_INVERSE`` with the
    same store callback (``operator/src/FFT.cpp:47-55``)."""
    if _FFT_WORKERS is not None:
        import scipy.fft as sfft
        return sfft.ifft2(x, axes=(-2, -1), norm="ortho", workers=_FFT_WORKERS)
    return np.fft.ifft2(x, axes=(-2, -1), norm="ortho")


# --------------------------------------------------------------------------
# axes and tables
# --------------------------------------------------------------------------

def k_axis(n, d):
    """Wavenumbers ``2*pi*i/(n*d)`` for i <= n/2, ``2*pi*(i-n)/(n*d)`` above
    (``propagator/src/PhaseShift.h:47-57``; same table in
    ``propagator/src/Scatter.h:528-542``)."""
    i = np.arange(n, dtype=np.float64)
    half = n // 2
    i = np.where(i <= half, i, i - n)
    return 2.0 * np.pi * i / (d * n)


def w_axis(n, o, d):
    """Angular frequencies ``2*pi*(o + i*d)`` (``propagator/src/Scatter.h:544-556``)."""
    return 2.0 * np.pi * (o + d * np.arange(n, dtype=np.float64))


def w2_axis(n, o, d):
    """Squared angular frequencies (``propagator/src/PhaseShift.h:59-70``)."""
    return w_axis(n, o, d) ** 2


def taper_weights(n, tap):
    """1D raised-cosine weights of ``propagator/src/taper.cu:34-60``: low edge
    ``0.5*(1-cos(pi*i/tap))`` for i < tap, high edge
    ``0.5*(1+cos(pi*(i-n+tap)/tap))`` for i >= n-tap, else 1."""
    w = np.ones(n, dtype=np.float64)
    for i in range(n):
        if i < tap and tap > 0:
            w[i] = 0.5 * (1.0 - math.cos(math.pi * i / tap))
        elif i >= n - tap:
            w[i] = 0.5 * (1.0 + math.cos(math.pi * (i - n + tap) / tap))
    return w


def taper2d(NX, NY, tapx, tapy):
    """Separable 2D taper ``w_x * w_y`` (``propagator/src/taper.cu:62-63``)."""
    return taper_weights(NY, tapy)[:, None] * taper_weights(NX, tapx)[None, :]


# --------------------------------------------------------------------------
# phase shift
# --------------------------------------------------------------------------

def _kz_parts(w2, kx, ky, sref, eps):
    """The branch quantities a, b, c of ``propagator/src/phase_shift.cu:36-41``
    for every (w, ky, kx); ``sref`` is the per-frequency complex reference s^2."""
    sre = sref.real[:, None, None]
    sim = sref.imag[:, None, None]
    w2 = np.asarray(w2, dtype=np.float64)[:, None, None]
    a = w2 * sre - (kx[None, None, :] ** 2 + ky[None, :, None] ** 2)
    b = w2 * (sim - eps * sre)
    c = np.sqrt(a * a + b * b)
    return a, b, c


def phase_forward_factor(w2, kx, ky, sref, dz, eps):
    """Forward multiplier ``e^{Im dz} (cos(Re dz) - i sin(Re dz))`` with
    Re = sqrt((c+a)/2), Im = -sqrt((c-a)/2) and NO b>0 branch
    (``propagator/src/phase_shift.cu:36-55``)."""
    a, b, c = _kz_parts(w2, kx, ky, sref, eps)
    re = np.sqrt((c + a) / 2)
    im = -np.sqrt((c - a) / 2)
    re = np.broadcast_to(re, a.shape)
    return np.exp(im * dz) * np.exp(-1j * re * dz)


def phase_adjoint_factor(w2, kx, ky, sref, dz, eps):
    """Adjoint multiplier ``e^{Im dz} (cos(Re dz) + i sin(Re dz))`` where Re flips
    sign when b > 0 (``propagator/src/phase_shift.cu:153-178``)."""
    a, b, c = _kz_parts(w2, kx, ky, sref, eps)
    re = np.sqrt((c + a) / 2)
    re = np.where(np.broadcast_to(b, a.shape) > 0, -re, re)
    im = -np.sqrt((c - a) / 2)
    return np.exp(im * dz) * np.exp(1j * re * dz)


def phase_inverse_factor(w2, kx, ky, sref, dz, eps):
    """Inverse (growing) multiplier of ``propagator/src/phase_shift.cu:274-298``:
    Im = +sqrt((c-a)/2), Re flips sign when b > 0, factor e^{Im dz} e^{+i Re dz}."""
    a, b, c = _kz_parts(w2, kx, ky, sref, eps)
    re = np.sqrt((c + a) / 2)
    re = np.where(np.broadcast_to(b, a.shape) > 0, -re, re)
    im = np.sqrt((c - a) / 2)
    return np.exp(im * dz) * np.exp(1j * re * dz)


# --------------------------------------------------------------------------
# grid description
# --------------------------------------------------------------------------

@dataclass
class Grid:
    """Wavefield and model geometry plus the ``par`` keys of the path
    (``propagator/src/OneStep.h:212-219``, ``propagator/src/Taper.h:16-17``,
    ``propagator/src/Scatter.cpp:12-14``, ``propagator/src/Propagator.cpp:63-71``)."""
    nx: int
    ny: int
    nw: int
    nz: int
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0
    ox: float = 0.0
    oy: float = 0.0
    oz: float = 0.0
    ow: float = 1.0   # first frequency [Hz]
    dw: float = 1.0   # frequency step [Hz]
    padx: int = 0
    pady: int = 0
    nref: int = 1
    eps: float = 0.0
    taperx: int = 0
    tapery: int = 0
    eps_scat: float = 0.04
    taylor: int = 1
    dtype: type = np.complex128
    _cache: dict = field(default_factory=dict, repr=False)

    @property
    def NX(self):
        return self.nx + self.padx

    @property
    def NY(self):
        return self.ny + self.pady

    def kx(self):
        return k_axis(self.NX, self.dx)

    def ky(self):
        return k_axis(self.NY, self.dy)

    def w2(self):
        return w2_axis(self.nw, self.ow, self.dw)

    def w(self):
        return w_axis(self.nw, self.ow, self.dw)

    def taper(self):
        return taper2d(self.NX, self.NY, self.taperx, self.tapery)


# --------------------------------------------------------------------------
# selector / taper / one step
# --------------------------------------------------------------------------

def select(labels, value, x):
    """``labels == value`` mask applied to every shot (``propagator/src/selector.cu:7-37``;
    labels are [nw][NY][NX] and shared by all shots)."""
    return np.where(labels[None] == value, x, 0)


def _factors(g, sref_z, fn, factors, dtype):
    """Phase factors of every reference at one depth: the precomputed list when
    given (``Stepper`` keeps one per depth), else evaluated here."""
    if factors is not None:
        return [f.astype(dtype, copy=False) for f in factors]
    kx, ky, w2 = g.kx(), g.ky(), g.w2()
    return [fn(w2, kx, ky, sref_z[r], g.dz, g.eps).astype(dtype) for r in range(g.nref)]


def pspi_forward(g, sref_z, labels_z, m, d=None, taper=True, factors=None):
    """PSPI forward, add version (``propagator/src/PSPI.cpp:6-24``):
    d (+)= sum_r mask_r * F^-1( P_r * F(taper * m) ).  The in-place overload
    (``propagator/src/PSPI.cpp:66-83``) is the same map with d = 0."""
    Ps = _factors(g, sref_z, phase_forward_factor, factors, m.dtype)
    tap = g.taper().astype(m.real.dtype) if taper else 1.0
    mk = fft2(tap * m)
    out = np.zeros_like(m) if d is None else d.copy()
    for r in range(g.nref):
        P = Ps[r]
        ref = ifft2(mk * P[None])
        out += select(labels_z, r, ref)
    return out.astype(m.dtype, copy=False)


def pspi_adjoint(g, sref_z, labels_z, d, m=None, taper=False, factors=None):
    """PSPI adjoint.  Add version (``propagator/src/PSPI.cpp:26-44``):
    m (+)= F^-1( sum_r P_r^adj * F(mask_r * d) ) with NO taper; the in-place
    overload (``propagator/src/PSPI.cpp:85-103``) multiplies by the taper at the
    end (``taper=True``)."""
    Qs = _factors(g, sref_z, phase_adjoint_factor, factors, d.dtype)
    mk = np.zeros_like(d)
    for r in range(g.nref):
        Q = Qs[r]
        mk = mk + Q[None] * fft2(select(labels_z, r, d))
    x = ifft2(mk)
    if taper:
        x = g.taper().astype(d.real.dtype)[None, None] * x
    out = x if m is None else m + x
    return out.astype(d.dtype, copy=False)


def nsps_forward(g, sref_z, labels_z, m, d=None, factors=None):
    """NSPS forward (``propagator/src/NSPS.cpp:27-45``):
    d (+)= F^-1( sum_r P_r * F(mask_r * m) )."""
    Ps = _factors(g, sref_z, phase_forward_factor, factors, m.dtype)
    mk = np.zeros_like(m)
    for r in range(g.nref):
        P = Ps[r]
        mk = mk + P[None] * fft2(select(labels_z, r, m))
    x = ifft2(mk)
    out = x if d is None else d + x
    return out.astype(m.dtype, copy=False)


def nsps_adjoint(g, sref_z, labels_z, d, m=None, factors=None):
    """NSPS adjoint (``propagator/src/NSPS.cpp:6-25``):
    m (+)= sum_r mask_r * F^-1( P_r^adj * F(d) )."""
    Qs = _factors(g, sref_z, phase_adjoint_factor, factors, d.dtype)
    dk = fft2(d)
    out = np.zeros_like(d) if m is None else m.copy()
    for r in range(g.nref):
        Q = Qs[r]
        out += select(labels_z, r, ifft2(Q[None] * dk))
    return out.astype(d.dtype, copy=False)


class Stepper:
    """One depth step in place, the way ``OneWay::one_step_fwd/adj`` uses it
    (``propagator/src/OneWay.cpp:6-20``): PSPI in-place forward / adjoint.  The
    reference hard-wires PSPI there (``propagator/src/OneWay.h:24-25,39-40``);
    ``kind='nsps'`` swaps in NSPS for the NSPS-driven sweeps."""

    def __init__(self, g, sref, labels, kind="pspi", cache_factors=True, cache_bytes=4 << 30):
        self.g, self.sref, self.labels, self.kind = g, sref, labels, kind
        # the factors of a depth depend only on its references: evaluated once per
        # depth and direction and reused by later steps there (same values); the
        # most recent (depth, direction) pairs that fit in cache_bytes are kept
        self._cache = {} if cache_factors else None
        entry = 16 * g.nref * g.nw * g.NX * g.NY
        self._entries = max(1, int(cache_bytes) // max(entry, 1))

    def _f(self, iz, adjoint):
        if self._cache is None:
            return None
        key = (iz, adjoint)
        if key not in self._cache:
            g = self.g
            fn = phase_adjoint_factor if adjoint else phase_forward_factor
            while len(self._cache) >= self._entries:
                self._cache.pop(next(iter(self._cache)))
            self._cache[key] = [fn(g.w2(), g.kx(), g.ky(), self.sref[iz][r], g.dz, g.eps) for r in range(g.nref)]
        return self._cache[key]

    def fwd(self, iz, psi):
        if self.kind == "pspi":
            return pspi_forward(self.g, self.sref[iz], self.labels[iz], psi, taper=True, factors=self._f(iz, False))
        return nsps_forward(self.g, self.sref[iz], self.labels[iz], psi, factors=self._f(iz, False))

    def adj(self, iz, psi):
        if self.kind == "pspi":
            return pspi_adjoint(self.g, self.sref[iz], self.labels[iz], psi, taper=True, factors=self._f(iz, True))
        return nsps_adjoint(self.g, self.sref[iz], self.labels[iz], psi, factors=self._f(iz, True))

    def fwd_add(self, iz, m, d):
        """``prop->cu_forward(true, m, d)`` (``propagator/src/Scattering.cpp:50``)."""
        if self.kind == "pspi":
            return pspi_forward(self.g, self.sref[iz], self.labels[iz], m, d, taper=True, factors=self._f(iz, False))
        return nsps_forward(self.g, self.sref[iz], self.labels[iz], m, d, factors=self._f(iz, False))

    def adj_set(self, iz, d):
        """``prop->cu_adjoint(false, m, d)`` (``propagator/src/Scattering.cpp:58``)."""
        if self.kind == "pspi":
            return pspi_adjoint(self.g, self.sref[iz], self.labels[iz], d, None, taper=False,
                                factors=self._f(iz, True))
        return nsps_adjoint(self.g, self.sref[iz], self.labels[iz], d, factors=self._f(iz, True))


def downward(stepper, nz, psi):
    """``Downward::cu_forward`` (``propagator/src/OneWay.cpp:264-278``): for
    iz = 0..nz-1 step in place; returns the propagated field."""
    for iz in range(nz):
        psi = stepper.fwd(iz, psi)
    return psi


def downward_adjoint(stepper, nz, psi):
    """``Downward::cu_adjoint`` (``propagator/src/OneWay.cpp:280-293``)."""
    for iz in range(nz, 0, -1):
        psi = stepper.adj(iz - 1, psi)
    return psi


def upward(stepper, nz, psi):
    """``Upward::cu_forward`` (``propagator/src/OneWay.cpp:295-310``)."""
    for iz in range(nz, 0, -1):
        psi = stepper.fwd(iz - 1, psi)
    return psi


def upward_adjoint(stepper, nz, psi):
    """``Upward::cu_adjoint`` (``propagator/src/OneWay.cpp:312-323``)."""
    for iz in range(nz):
        psi = stepper.adj(iz, psi)
    return psi


# --------------------------------------------------------------------------
# injection / recording
# --------------------------------------------------------------------------

@dataclass
class Traces:
    """Per-trace interpolation data of ``propagator/src/injection.cu:33-53``,
    computed in float32 exactly as the kernel does (index selection is integer
    work and must match bit for bit)."""
    ix: np.ndarray
    iy: np.ndarray
    iz: np.ndarray
    lx: np.ndarray
    ly: np.ndarray
    lz: np.ndarray
    ids: np.ndarray
    valid: np.ndarray


def make_traces(cx, cy, cz, ids, ox, oy, dx, dy, oz, dz, NX, NY):
    f = np.float32
    cx, cy, cz = (np.asarray(v, dtype=f) for v in (cx, cy, cz))
    ox, oy, dx, dy, oz, dz = (f(v) for v in (ox, oy, dx, dy, oz, dz))
    iy = np.floor((cy - oy) / dy).astype(np.int64)
    ly = f(1) - (cy - (oy + iy.astype(f) * dy)) / dy
    ix = np.floor((cx - ox) / dx).astype(np.int64)
    lx = f(1) - (cx - (ox + ix.astype(f) * dx)) / dx
    iz = np.floor((cz - oz) / dz).astype(np.int64)
    lz = f(1) - (cz - (oz + iz.astype(f) * dz)) / dz
    valid = ~((ix < 0) | (ix >= NX - 1) | (iy < 0) | (iy >= NY - 1))
    return Traces(ix, iy, iz, lx.astype(np.float64), ly.astype(np.float64),
                  lz.astype(np.float64), np.asarray(ids, dtype=np.int64), valid)


def _level_weights(tr, iz_inj):
    """Active traces at depth level ``iz_inj`` and their four corner weights
    (``propagator/src/injection.cu:46-71``): lz on level iz, 1-lz on level iz+1."""
    on0 = tr.valid & (tr.iz == iz_inj)
    on1 = tr.valid & (tr.iz + 1 == iz_inj)
    act = np.nonzero(on0 | on1)[0]
    z = np.where(on0[act], tr.lz[act], 1.0 - tr.lz[act])
    lx, ly = tr.lx[act], tr.ly[act]
    w = np.stack([z * lx * ly, z * (1 - lx) * ly, z * lx * (1 - ly), z * (1 - lx) * (1 - ly)])
    return act, w


def inject(tr, traces, wfld, iz_inj):
    """``inj_forward`` (``propagator/src/injection.cu:7-96``): wfld += weights x trace
    at the 4 surrounding nodes of depth level ``iz_inj``."""
    out = wfld.copy()
    act, w = _level_weights(tr, iz_inj)
    if len(act) == 0:
        return out
    s, ix, iy = tr.ids[act], tr.ix[act], tr.iy[act]
    tv = traces[act]                                        # [na][nw]
    for k, (dy, dx) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
        np.add.at(out, (s[:, None], np.arange(out.shape[1])[None, :], (iy + dy)[:, None], (ix + dx)[:, None]),
                  w[k][:, None] * tv)
    return out


def record(tr, wfld, traces, iz_inj):
    """``inj_adjoint`` (``propagator/src/injection.cu:98-188``): traces += weighted
    gather of the 4 surrounding nodes."""
    out = traces.copy()
    act, w = _level_weights(tr, iz_inj)
    if len(act) == 0:
        return out
    s, ix, iy = tr.ids[act], tr.ix[act], tr.iy[act]
    acc = 0
    for k, (dy, dx) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
        acc = acc + w[k][:, None] * wfld[s, :, iy + dy, ix + dx]
    np.add.at(out, act, acc)
    return out


# --------------------------------------------------------------------------
# reflection, imaging condition, scattering, linearised reflection
# --------------------------------------------------------------------------

def model_pair(model, iz):
    """Slices (iz, iz+1) of a [nz][nw][ny][nx] model; the bottom slice is paired with
    itself so the coefficient vanishes (``propagator/src/Reflect.h:20-38``)."""
    nz = model.shape[0]
    return model[iz], model[iz + 1] if iz < nz - 1 else model[iz]


def reflect_coef(s0, s1, r0, r1):
    """``r = (rho1 sqrt(s0) - rho0 sqrt(s1)) / (rho1 sqrt(s0) + rho0 sqrt(s1))`` with
    principal complex square roots (``propagator/src/reflect.cu:42-45``,
    ``propagator/src/prop_kernels.cuh:89-102``)."""
    a = r1 * np.sqrt(s0.astype(np.complex128))
    b = r0 * np.sqrt(s1.astype(np.complex128))
    return (a - b) / (a + b)


def reflect_forward(g, slow, den, iz, down, up):
    """``refl_forward`` (``propagator/src/reflect.cu:8-52``): up += r * down over the
    unpadded (ny, nx) window of the padded wavefield."""
    s0, s1 = model_pair(slow, iz)
    r0, r1 = model_pair(den, iz)
    r = reflect_coef(s0, s1, r0, r1)
    out = up.copy()
    out[:, :, :g.ny, :g.nx] += down[:, :, :g.ny, :g.nx] * r[None]
    return out


def reflect_adjoint(g, slow, den, iz, up, down):
    """``refl_adjoint`` (``propagator/src/reflect.cu:54-97``): down += conj(r) * up."""
    s0, s1 = model_pair(slow, iz)
    r0, r1 = model_pair(den, iz)
    r = reflect_coef(s0, s1, r0, r1)
    out = down.copy()
    out[:, :, :g.ny, :g.nx] += up[:, :, :g.ny, :g.nx] * np.conj(r)[None]
    return out


def ic_forward(g, bg, image, wfld):
    """``ic_fwd`` (``propagator/src/imaging_condition.cu:9-55``):
    wfld[s,w,y,x] += bg[s,w,y,x] * image[w,y,x] on the unpadded window."""
    out = wfld.copy()
    out[:, :, :g.ny, :g.nx] += bg[:, :, :g.ny, :g.nx] * image[None]
    return out


def ic_adjoint(g, bg, wfld, image):
    """``ic_adj`` (``propagator/src/imaging_condition.cu:57-108``):
    image[w,y,x] += sum_s conj(bg) * wfld (per frequency, no sum over w)."""
    return image + np.sum(np.conj(bg[:, :, :g.ny, :g.nx]) * wfld[:, :, :g.ny, :g.nx], axis=0)


SCAT_COEF = (1.0, 1.0 / 2.0, 3.0 / 8.0, 5.0 / 16.0, 35.0 / 128.0)  # Scatter.h:526


def pad_slice(g, s):
    """Edge-replicating pad [nw][ny][nx] -> [nw][NY][NX] (``pad_fwd``,
    ``propagator/src/scatter.cu:240-277``)."""
    return np.pad(s, ((0, 0), (0, g.pady), (0, g.padx)), mode="edge")


def scatter_weights(g, slow_slice):
    """Per-cell weights W_n = (-i w dz/2) c_n s~^(-1/2-n) with
    s~ = Re s^2 + i (Im s^2 - eps_scat Re s^2) on the padded slice
    (``propagator/src/scatter.cu:61-106,155-195``; ``cuCpowf`` is the principal
    power, ``propagator/src/scatter.cu:6-21``)."""
    sp = pad_slice(g, slow_slice).astype(np.complex128)
    st = sp.real + 1j * (sp.imag - g.eps_scat * sp.real)
    w = g.w()[:, None, None]
    out = []
    for n in range(g.taylor + 1):
        out.append(-1j * (w * g.dz / 2.0) * SCAT_COEF[n] * np.power(st, -0.5 - n))
    return out


def scatter_kfilters(g):
    """Spectral multipliers Q_n = (|k|/w)^(2n) (``mult_kxky``,
    ``propagator/src/scatter.cu:23-59``)."""
    kx, ky, w = g.kx(), g.ky(), g.w()
    kk = np.sqrt(kx[None, None, :] ** 2 + ky[None, :, None] ** 2)
    return [np.power(kk / w[:, None, None], 2 * n) for n in range(g.taylor + 1)]


def scatter_forward(g, slow_slice, u, d=None):
    """``Scatter::cu_forward`` (``propagator/src/Scatter.cpp:76-88``; in place
    ``:104-116``): d (+)= sum_n W_n * F^-1(Q_n * F(u))."""
    W = [w.astype(u.dtype) for w in scatter_weights(g, slow_slice)]
    Q = [q.astype(u.real.dtype) for q in scatter_kfilters(g)]
    uk = fft2(u)
    out = np.zeros_like(u) if d is None else d.copy()
    for n in range(g.taylor + 1):
        out += W[n][None] * ifft2(Q[n][None] * uk)
    return out.astype(u.dtype, copy=False)


def scatter_adjoint(g, slow_slice, d, u=None):
    """``Scatter::cu_adjoint`` (``propagator/src/Scatter.cpp:91-102``; in place
    ``:118-133``): u (+)= sum_n F^-1(Q_n * F(conj(W_n) * d))."""
    W = [w.astype(d.dtype) for w in scatter_weights(g, slow_slice)]
    Q = [q.astype(d.real.dtype) for q in scatter_kfilters(g)]
    out = np.zeros_like(d) if u is None else u.copy()
    for n in range(g.taylor + 1):
        out += ifft2(Q[n][None] * fft2(np.conj(W[n])[None] * d))
    return out.astype(d.dtype, copy=False)


def _lin_refl_coefs(s0, s1, r0, r1):
    """Coefficients of ``drefl_forward`` (``propagator/src/lin_reflect.cu:48-92``)."""
    q0 = np.sqrt(s0.astype(np.complex128))
    q1 = np.sqrt(s1.astype(np.complex128))
    denom = r1 * q0 + r0 * q1
    inv2 = (1.0 / denom) ** 2
    s1s2sq = r0 * r1 * inv2
    r1r2sq = 2.0 * q0 * q1 * inv2
    sqrt_c = np.sqrt(q1 / q0)
    a_s = sqrt_c * s1s2sq
    b_s = s1s2sq / sqrt_c
    a_r = r0 * r1r2sq
    b_r = r1 * r1r2sq
    return a_s, b_s, a_r, b_r


def lin_reflect_forward(slow, den, iz, dm):
    """``drefl_forward``: dm = [ds2(iz), ds2(iz+1), drho(iz), drho(iz+1)] (each
    [nw][ny][nx]) -> dr[nw][ny][nx] = a_s ds0 - b_s ds1 + a_r drho1 - b_r drho0."""
    s0, s1 = model_pair(slow, iz)
    r0, r1 = model_pair(den, iz)
    a_s, b_s, a_r, b_r = _lin_refl_coefs(s0, s1, r0, r1)
    return a_s * dm[0] - b_s * dm[1] + a_r * dm[3] - b_r * dm[2]


def lin_reflect_adjoint(slow, den, iz, dr):
    """``drefl_adjoint`` (``propagator/src/lin_reflect.cu:97-184``)."""
    s0, s1 = model_pair(slow, iz)
    r0, r1 = model_pair(den, iz)
    a_s, b_s, a_r, b_r = _lin_refl_coefs(s0, s1, r0, r1)
    return [np.conj(a_s) * dr, -np.conj(b_s) * dr, -np.conj(b_r) * dr, np.conj(a_r) * dr]


# --------------------------------------------------------------------------
# drivers
# --------------------------------------------------------------------------

def remap_ids(s_ids, r_ids):
    """Dense shot ids (``propagator/src/Propagator.cpp:28-59``)."""
    uniq = sorted(set(int(i) for i in s_ids))
    m = {v: i for i, v in enumerate(uniq)}
    for r in r_ids:
        if int(r) not in m:
            raise RuntimeError("receiver associated with a shot id not present in the source list")
    return (np.array([m[int(i)] for i in s_ids], dtype=np.int64),
            np.array([m[int(i)] for i in r_ids], dtype=np.int64), len(uniq))


@dataclass
class Acquisition:
    src: Traces
    rec: Traces
    ns: int


def make_acquisition(g, geom):
    s_ids, r_ids, ns = remap_ids(geom["s_ids"], geom["r_ids"])
    src = make_traces(geom["sx"], geom["sy"], geom["sz"], s_ids, g.ox, g.oy, g.dx, g.dy,
                      g.oz, g.dz, g.NX, g.NY)
    rec = make_traces(geom["rx"], geom["ry"], geom["rz"], r_ids, g.ox, g.oy, g.dx, g.dy,
                      g.oz, g.dz, g.NX, g.NY)
    return Acquisition(src, rec, ns)


def propagate(g, stepper, acq, slow, den, wavelet, keep=True):
    """``Propagator::forward`` (``propagator/src/Propagator.cpp:121-221``).
    Returns (data, bg_down, bg_up) where bg_down[iz] is the down-going field
    stored before step iz and bg_up[iz] the up-going field after the step,
    reflection and recording at iz.  Checkpoints are kept losslessly (the
    reference stores them ZFP-compressed, ``propagator/src/WavefieldPool.cpp:52``)."""
    dt = g.dtype
    data = np.zeros((len(acq.rec.ix), g.nw), dtype=dt)
    wf = np.zeros((acq.ns, g.nw, g.NY, g.NX), dtype=dt)
    bg_down, bg_up = [None] * g.nz, [None] * g.nz
    for iz in range(g.nz):
        wf = inject(acq.src, wavelet, wf, iz)
        data = record(acq.rec, wf, data, iz)
        if keep:
            bg_down[iz] = wf.copy()
        wf = stepper.fwd(iz, wf)
    up = np.zeros_like(wf)
    for iz in range(g.nz - 1, -1, -1):
        up = stepper.fwd(iz, up)
        up = reflect_forward(g, slow, den, iz, bg_down[iz], up)
        data = record(acq.rec, up, data, iz)
        if keep:
            bg_up[iz] = up.copy()
    return data, bg_down, bg_up


def forward_scattering_fwd(g, stepper, iz_prop, slow, bg, image, target):
    """``ForwardScattering::cu_forward`` (``propagator/src/Scattering.cpp:43-52``):
    target += step_add( scatter( ic_fwd(image) ) )."""
    sc = ic_forward(g, bg, image, np.zeros_like(target))
    sc = scatter_forward(g, slow[iz_prop], sc)
    return stepper.fwd_add(iz_prop, sc, target)


def forward_scattering_adj(g, stepper, iz_prop, slow, bg, wfld):
    """``ForwardScattering::cu_adjoint`` (``propagator/src/Scattering.cpp:54-61``)."""
    sc = stepper.adj_set(iz_prop, wfld)
    sc = scatter_adjoint(g, slow[iz_prop], sc)
    return ic_adjoint(g, bg, sc, np.zeros((g.nw, g.ny, g.nx), dtype=wfld.dtype))


def _dm_pair(model_s, model_r, iz):
    s0, s1 = model_pair(model_s, iz)
    r0, r1 = model_pair(model_r, iz)
    return [s0, s1, r0, r1]


def born_forward(g, stepper, acq, slow, den, bg_down, bg_up, dslow, dden):
    """``ExtendedBorn::forward`` (``propagator/src/ExtendedBorn.cpp:80-118``): the four
    sweeps of ``:152-178`` (down scattering), ``:210-238`` (down-scattered field
    reflected up), ``:282-311`` (up scattering) and ``:352-389`` (back
    scattering), all recorded into one data array."""
    dt = g.dtype
    nrec = len(acq.rec.ix)
    data = np.zeros((nrec, g.nw), dtype=dt)
    shape = (acq.ns, g.nw, g.NY, g.NX)
    # 1. down scattering
    sd = np.zeros(shape, dtype=dt)
    born_down = [None] * g.nz
    for iz in range(g.nz):
        born_down[iz] = sd.copy()
        data = record(acq.rec, sd, data, iz)
        sd = stepper.fwd(iz, sd)
        sd = forward_scattering_fwd(g, stepper, iz, slow, bg_down[iz], dslow[iz], sd)
    # 2. down-scattered field reflected by the background, continued up
    su = np.zeros(shape, dtype=dt)
    for iz in range(g.nz - 1, -1, -1):
        su = stepper.fwd(iz, su)
        su = reflect_forward(g, slow, den, iz, born_down[iz], su)
        data = record(acq.rec, su, data, iz)
    # 3. up scattering of the up-going background
    uu = np.zeros(shape, dtype=dt)
    for iz in range(g.nz - 1, -1, -1):
        data = record(acq.rec, uu, data, iz)
        if iz > 0:
            uu = stepper.fwd(iz - 1, uu)
            uu = forward_scattering_fwd(g, stepper, iz - 1, slow, bg_up[iz], dslow[iz], uu)
    # 4. back scattering from the linearised reflection coefficient
    bu = np.zeros(shape, dtype=dt)
    for iz in range(g.nz - 1, -1, -1):
        bu = stepper.fwd(iz, bu)
        dr = lin_reflect_forward(slow, den, iz, _dm_pair(dslow, dden, iz))
        bu = ic_forward(g, bg_down[iz], dr, bu)
        data = record(acq.rec, bu, data, iz)
    return data


def born_adjoint(g, stepper, acq, slow, den, bg_down, bg_up, data):
    """``ExtendedBorn::adjoint`` (``propagator/src/ExtendedBorn.cpp:122-150``) with the
    sweeps of ``:313-349``, ``:240-280``, ``:180-208`` and ``:391-453``.  Returns
    (dslow, dden), each [nz][nw][ny][nx]."""
    dt = g.dtype
    shape = (acq.ns, g.nw, g.NY, g.NX)
    gs = np.zeros((g.nz, g.nw, g.ny, g.nx), dtype=dt)
    gr = np.zeros_like(gs)
    # up scattering adjoint; also stores the adjoint up-going field per depth
    uu = np.zeros(shape, dtype=dt)
    born_up = [None] * g.nz
    for iz in range(g.nz):
        if iz > 0:
            gs[iz] += forward_scattering_adj(g, stepper, iz - 1, slow, bg_up[iz], uu)
            uu = stepper.adj(iz - 1, uu)
        uu = inject(acq.rec, data, uu, iz)
        born_up[iz] = uu.copy()
    # reflected down-scattering adjoint
    sd = np.zeros(shape, dtype=dt)
    for iz in range(g.nz - 1, -1, -1):
        gs[iz] += forward_scattering_adj(g, stepper, iz, slow, bg_down[iz], sd)
        sd = stepper.adj(iz, sd)
        sd = reflect_adjoint(g, slow, den, iz, born_up[iz], sd)
    # direct down-scattering adjoint
    sd = np.zeros(shape, dtype=dt)
    for iz in range(g.nz - 1, -1, -1):
        gs[iz] += forward_scattering_adj(g, stepper, iz, slow, bg_down[iz], sd)
        sd = stepper.adj(iz, sd)
        sd = inject(acq.rec, data, sd, iz)
    # back scattering adjoint
    bu = np.zeros(shape, dtype=dt)
    for iz in range(g.nz):
        bu = inject(acq.rec, data, bu, iz)
        dr = ic_adjoint(g, bg_down[iz], bu, np.zeros((g.nw, g.ny, g.nx), dtype=dt))
        dm = lin_reflect_adjoint(slow, den, iz, dr)
        bu = stepper.adj(iz, bu)
        z1 = iz + 1 if iz < g.nz - 1 else iz
        gs[iz] += dm[0]
        gs[z1] += dm[1]
        gr[iz] += dm[2]
        gr[z1] += dm[3]
    return gs, gr


def migrate(g, stepper, acq, wavelet, data):
    """Cross-correlation image sum_w Re(sum_s conj(S) R) per depth.

    S is the down-going source field of ``propagator/src/Propagator.cpp:155-180``
    (inject, then step).  R is the receiver field of the back-scattering adjoint
    (``propagator/src/ExtendedBorn.cpp:396-408``: inject the data at iz, correlate,
    then continue down with the adjoint step), correlated by ``ic_adj``
    (``propagator/src/imaging_condition.cu:57-108``) and summed over frequency.
    Both fields move down in lockstep, so no checkpoint is needed.
    Returns the float image [nz][ny][nx]."""
    dt = g.dtype
    shape = (acq.ns, g.nw, g.NY, g.NX)
    S = np.zeros(shape, dtype=dt)
    R = np.zeros(shape, dtype=dt)
    img = np.zeros((g.nz, g.ny, g.nx), dtype=np.float64)
    for iz in range(g.nz):
        S = inject(acq.src, wavelet, S, iz)
        R = inject(acq.rec, data, R, iz)
        I = ic_adjoint(g, S, R, np.zeros((g.nw, g.ny, g.nx), dtype=dt))
        img[iz] = np.real(I).sum(axis=0)
        S = stepper.fwd(iz, S)
        R = stepper.adj(iz, R)
    return img


# --------------------------------------------------------------------------
# differentiable ("smooth") PSPI step and the adjoint-state FWI gradient.
# No reference counterpart: the reference's PSPI selects the nearest reference
# per cell (``propagator/src/selector.cu:29-35``), so its output is piecewise
# constant in the slowness.  The smooth step interpolates between the two
# references bracketing the local slowness s (hat functions on the sorted
# references, clamped at both ends) with the split-step correction
# exp(-i w (s - s_r) dz); the phase factors P_r are the reference's
# (``propagator/src/phase_shift.cu:7-61``) for s_r^2.  This section restates
# that definition in FP64 as the oracle of the B200 smooth step, and derives
# the gradient of J = 1/2 |d(s) - d_obs|^2 for the Propagator's modelling
# (down pass, reflection, up pass; ``propagator/src/Propagator.cpp:121-221``)
# with density 1 and the references held fixed.
# --------------------------------------------------------------------------

def hat_weights(s, refs):
    """Weights w_r(s) and derivatives w_r'(s), each [nref] + s.shape."""
    refs = np.asarray(refs, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    n = len(refs)
    w = np.zeros((n,) + s.shape)
    dw = np.zeros_like(w)
    if n == 1:
        w[0] = 1.0
        return w, dw
    lo, hi = s <= refs[0], s >= refs[-1]
    mid = ~(lo | hi)
    j = np.clip(np.searchsorted(refs, s, side="right") - 1, 0, n - 2)
    span = refs[j + 1] - refs[j]
    u = (s - refs[j]) / span
    for r in range(n):
        w[r] = np.where(mid & (j == r), 1 - u, 0.0) + np.where(mid & (j + 1 == r), u, 0.0)
        dw[r] = np.where(mid & (j == r), -1.0 / span, 0.0) + np.where(mid & (j + 1 == r), 1.0 / span, 0.0)
    w[0][lo] = 1.0
    w[n - 1][hi] = 1.0
    return w, dw


def _smooth_terms(g, refs_z, s_pad_z):
    """Per reference: phase factors P_r [nw][NY][NX] (s_r^2 for every frequency),
    split-step factors SS_r and hat weights / derivatives on the padded slice."""
    kx, ky, w2, w = g.kx(), g.ky(), g.w2(), g.w()
    wt, dwt = hat_weights(s_pad_z, refs_z)
    out = []
    for r, sr in enumerate(refs_z):
        sref_w = np.full(g.nw, float(sr) ** 2, dtype=np.complex128)
        P = phase_forward_factor(w2, kx, ky, sref_w, g.dz, g.eps)
        Pa = phase_adjoint_factor(w2, kx, ky, sref_w, g.dz, g.eps)
        SS = np.exp(-1j * w[:, None, None] * (s_pad_z[None] - sr) * g.dz)
        out.append((P, Pa, SS, wt[r][None], dwt[r][None]))
    return out


def smooth_forward(g, refs_z, s_pad_z, psi):
    """psi' = sum_r w_r SS_r F^-1(P_r F(taper psi))."""
    mk = fft2(psi * g.taper()[None, None])
    out = np.zeros_like(psi, dtype=np.complex128)
    for P, _, SS, wt, _ in _smooth_terms(g, refs_z, s_pad_z):
        out += (wt * SS)[None] * ifft2(P[None] * mk)
    return out


def smooth_adjoint(g, refs_z, s_pad_z, d):
    """Exact transpose of smooth_forward: taper F^-1(sum_r P_r^adj F(w_r conj(SS_r) d))."""
    mk = np.zeros_like(d, dtype=np.complex128)
    for _, Pa, SS, wt, _ in _smooth_terms(g, refs_z, s_pad_z):
        mk += Pa[None] * fft2((wt * np.conj(SS))[None] * d)
    return ifft2(mk) * g.taper()[None, None]


def smooth_deriv(g, refs_z, s_pad_z, psi):
    """Cell-wise derivative of smooth_forward with respect to s:
    sum_r (w_r' - i w dz w_r) SS_r F^-1(P_r F(taper psi))."""
    mk = fft2(psi * g.taper()[None, None])
    w = g.w()[:, None, None]
    out = np.zeros_like(psi, dtype=np.complex128)
    for P, _, SS, wt, dwt in _smooth_terms(g, refs_z, s_pad_z):
        out += ((dwt - 1j * w * g.dz * wt) * SS)[None] * ifft2(P[None] * mk)
    return out


def pad_edge(g, s):
    """[nz][ny][nx] -> [nz][NY][NX] by edge replication."""
    return np.pad(s, ((0, 0), (0, g.pady), (0, g.padx)), mode="edge")


def fold_edge(g, gp):
    """Transpose of pad_edge: padded-cell contributions summed into the edge cells."""
    out = gp[:, :g.ny, :g.nx].copy()
    out[:, :, g.nx - 1] += gp[:, :g.ny, g.nx:].sum(axis=2)
    out[:, g.ny - 1, :] += gp[:, g.ny:, :g.nx].sum(axis=1)
    out[:, g.ny - 1, g.nx - 1] += gp[:, g.ny:, g.nx:].sum(axis=(1, 2))
    return out


def smooth_refs(s, nref, spread=1e-3):
    """Reference slownesses per depth: nref values evenly spaced over the slice's
    [min, max] (a slice narrower than spread * mean is widened to that)."""
    s = np.asarray(s, dtype=np.float64)
    lo, hi = s.min(axis=(1, 2)), s.max(axis=(1, 2))
    mid, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
    half = np.maximum(half, 0.5 * spread * mid)
    if nref == 1:
        return mid[:, None]
    return mid[:, None] + half[:, None] * np.linspace(-1.0, 1.0, nref)[None, :]


def smooth_propagate(g, refs, s, acq, wavelet):
    """Modelling with the smooth step: the Propagator's down pass, reflection
    (density 1: r = (s0 - s1) / (s0 + s1), bottom r = 0) and up pass.  Returns
    (data, D, U): D[iz] the down field after injection at iz, U[iz] the up
    field after the step, reflection and recording at iz."""
    sp = pad_edge(g, s)
    s2 = np.repeat((np.asarray(s, np.float64) ** 2)[:, None].astype(np.complex128), g.nw, axis=1)
    den = np.ones_like(s2)
    data = np.zeros((len(acq.rec.ix), g.nw), dtype=np.complex128)
    D = np.zeros((acq.ns, g.nw, g.NY, g.NX), dtype=np.complex128)
    Ds, Us = [None] * g.nz, [None] * g.nz
    for iz in range(g.nz):
        D = inject(acq.src, wavelet, D, iz)
        data = record(acq.rec, D, data, iz)
        Ds[iz] = D.copy()
        D = smooth_forward(g, refs[iz], sp[iz], D)
    U = np.zeros_like(D)
    for iz in range(g.nz - 1, -1, -1):
        U = smooth_forward(g, refs[iz], sp[iz], U)
        U = reflect_forward(g, s2, den, iz, Ds[iz], U)
        data = record(acq.rec, U, data, iz)
        Us[iz] = U.copy()
    return data, Ds, Us


def smooth_objective(g, refs, s, acq, wavelet, d_obs):
    data, _, _ = smooth_propagate(g, refs, s, acq, wavelet)
    r = data - d_obs
    return 0.5 * float(np.real(np.vdot(r, r)))


def smooth_gradient(g, refs, s, acq, wavelet, d_obs):
    """(J, dJ/ds [nz][ny][nx]) by the adjoint-state method.

    mu_iz (adjoint of U_iz) = Rec_iz^H r + S_{iz-1}^H mu_{iz-1}, downward;
    nu_iz (adjoint of D_iz) = Rec_iz^H r + conj(R_iz) mu_iz + S_iz^H nu_{iz+1}, upward;
    dJ/ds collects Re<mu_iz, dS_iz(U_{iz+1})>, Re<nu_{iz+1}, dS_iz(D_iz)> and
    Re<mu_iz, dR_iz D_iz>, summed over shots and frequencies."""
    s = np.asarray(s, np.float64)
    data, Ds, Us = smooth_propagate(g, refs, s, acq, wavelet)
    res = data - d_obs
    J = 0.5 * float(np.real(np.vdot(res, res)))
    sp = pad_edge(g, s)
    s2 = np.repeat((s ** 2)[:, None].astype(np.complex128), g.nw, axis=1)
    den = np.ones_like(s2)
    gpad = np.zeros((g.nz, g.NY, g.NX))
    grefl = np.zeros((g.nz, g.ny, g.nx))
    corr = lambda a, b: np.real(np.sum(np.conj(a) * b, axis=(0, 1)))
    mus = [None] * g.nz
    mu = np.zeros_like(Ds[0])
    for iz in range(g.nz):
        if iz > 0:
            mu = smooth_adjoint(g, refs[iz - 1], sp[iz - 1], mu)
        mu = inject(acq.rec, res, mu, iz)
        mus[iz] = mu.copy()
        if iz + 1 < g.nz:
            gpad[iz] += corr(mu, smooth_deriv(g, refs[iz], sp[iz], Us[iz + 1]))
            c = corr(mu[:, :, :g.ny, :g.nx], Ds[iz][:, :, :g.ny, :g.nx])
            s0, s1 = s[iz], s[iz + 1]
            grefl[iz] += c * 2 * s1 / (s0 + s1) ** 2
            grefl[iz + 1] += c * (-2 * s0) / (s0 + s1) ** 2
    nu = np.zeros_like(Ds[0])
    for iz in range(g.nz - 1, -1, -1):
        if iz + 1 < g.nz:
            gpad[iz] += corr(nu, smooth_deriv(g, refs[iz], sp[iz], Ds[iz]))
        nu = smooth_adjoint(g, refs[iz], sp[iz], nu)
        nu = reflect_adjoint(g, s2, den, iz, mus[iz], nu)
        nu = inject(acq.rec, res, nu, iz)
    return J, fold_edge(g, gpad) + grefl
