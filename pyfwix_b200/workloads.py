"""Seeded synthetic workloads with the shapes, sizes and value distributions of the
benchmark configurations (there is no public dataset for this path).

config1: PSPI forward modelling + imaging, one shot, 128 x 128 x 100, nw = 64
         (2-30 Hz), v = 1500 + 0.5 z with a +10 % Gaussian anomaly (sigma 150 m at
         (640, 640, 500) m), nref = 4 quantile references, 15 Hz Ricker at the
         surface centre, receivers on every surface node, taper 20 cells.
config2: Born forward + adjoint with NSPS, one shot, 256 x 256 x 200, nw = 128
         (3-40 Hz), v = 1500 + 0.4 z times (1 + p), p = Gaussian-filtered white
         noise (sigma 5 cells) scaled to max |p| = 0.05; reflectivity = 5 flat
         layers at depths drawn from {10..189}, amplitudes U(-0.1, 0.1) relative to
         the background s^2.
config3: batched forward + imaging, 32 shots, each on its own grid: nx = ny drawn
         from {128, 192, 256, 320, 384}, nz = 200, d = 10 m, a band of 48-160
         frequencies (step 43/159 Hz) placed at random within 2-45 Hz; velocity of
         the config1 family (1500 + 0.5 z, +10 % Gaussian anomaly, sigma 150 m) with
         the anomaly centre drawn per shot over the middle half of the grid; PSPI,
         nref = 6; source at the grid centre, receivers on every surface node.
config4: FWI gradient, PSPI smooth step, 384 x 384 x 300, nw = 96 (3-30 Hz), nref 4,
         true model v = 1500 + 0.5 z times (1 + three Gaussian anomalies of +-8 %,
         sigma 150 m, at seeded centres), starting model the background; 8 sources
         at seeded surface positions (shot s uses source s), receivers on every
         surface node, depth checkpoints every 16 levels.
config5: large migration with gradient, one shot, 512 x 512 x 400, d = 12.5 m,
         nw = 200 (2-50 Hz), PSPI nref 8; 12 dipping layers of 1500-4500 m/s and a
         Gaussian body of 4500 m/s.

Seeds are ``numpy.random.default_rng(1000 + config_index)``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def ricker_spectrum(freqs, f0=15.0, dt=0.004, nt=512, t0=0.1):
    """Direct DTFT W(f) = sum_n r(n dt) exp(-2 pi i f n dt) of a Ricker wavelet."""
    t = np.arange(nt) * dt
    a = (np.pi * f0 * (t - t0)) ** 2
    r = (1 - 2 * a) * np.exp(-a)
    return np.exp(-2j * np.pi * np.outer(freqs, t)) @ r


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    nw: int
    ow: float
    dw: float
    nref: int
    step: str
    taperx: int = 20
    tapery: int = 20
    padx: int = 0
    pady: int = 0
    eps: float = 0.0
    eps_scat: float = 0.04
    taylor: int = 1
    ox: float = 0.0
    oy: float = 0.0
    oz: float = 0.0
    slow2: np.ndarray = None      # [nz][ny][nx] float32, s^2 = 1/v^2
    anomaly: tuple = None         # (cx, cy, cz) of the +10 % anomaly; slow2 then comes from slow2_on()
    layers: tuple = None          # config5's layers and body; slow2 then comes from slow2_on()
    geom: dict = field(default_factory=dict)
    wavelet: np.ndarray = None    # [nsrc][nw] complex64
    dslow: np.ndarray = None      # Born perturbation [nz][ny][nx] float32 (or None)

    @property
    def freqs(self):
        return self.ow + self.dw * np.arange(self.nw)

    @property
    def cells(self):
        """x*y*w*z cell-steps of one sweep over all shots."""
        ns = len(set(self.geom["s_ids"]))
        return ns * self.nx * self.ny * self.nw * self.nz

    def plan_kwargs(self):
        return dict(nx=self.nx, ny=self.ny, nw=self.nw, nz=self.nz, dx=self.dx, dy=self.dy,
                    dz=self.dz, ox=self.ox, oy=self.oy, oz=self.oz, ow=self.ow, dw=self.dw,
                    padx=self.padx, pady=self.pady, nref=self.nref, eps=self.eps,
                    taperx=self.taperx, tapery=self.tapery, eps_scat=self.eps_scat,
                    taylor=self.taylor, step=self.step)

    def surface_receivers(self, shot_id=0):
        gx, gy = np.meshgrid(self.ox + self.dx * np.arange(self.nx), self.oy + self.dy * np.arange(self.ny))
        n = gx.size
        return dict(rx=gx.ravel().astype(np.float32), ry=gy.ravel().astype(np.float32),
                    rz=np.full(n, self.oz, np.float32), r_ids=np.full(n, shot_id, np.int32))


def _coords(w):
    z = w.oz + w.dz * np.arange(w.nz)
    y = w.oy + w.dy * np.arange(w.ny)
    x = w.ox + w.dx * np.arange(w.nx)
    return np.meshgrid(z, y, x, indexing="ij")


def config1(nz=None, seed=1000):
    w = Workload(name="pspi-model-image-128x128x100-nw64", nx=128, ny=128, nz=nz or 100, dx=10.0, dy=10.0,
                 dz=10.0, nw=64, ow=2.0, dw=28.0 / 63.0, nref=4, step="pspi")
    Z, Y, X = _coords(w)
    v = (1500.0 + 0.5 * Z) * (1 + 0.10 * np.exp(-((X - 640) ** 2 + (Y - 640) ** 2 + (Z - 500) ** 2) / (2 * 150.0 ** 2)))
    w.slow2 = (1.0 / v ** 2).astype(np.float32)
    w.geom = dict(sx=np.array([640.0], np.float32), sy=np.array([640.0], np.float32),
                  sz=np.array([0.0], np.float32), s_ids=np.array([0], np.int32), **w.surface_receivers())
    w.wavelet = ricker_spectrum(w.freqs)[None, :].astype(np.complex64)
    return w


def config2(nz=None, nw=None, seed=1001):
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    nz_full = 200
    w = Workload(name="born-nsps-256x256x200-nw128", nx=256, ny=256, nz=nz or nz_full, dx=10.0, dy=10.0,
                 dz=10.0, nw=nw or 128, ow=3.0, dw=37.0 / 127.0, nref=4, step="nsps", taperx=20, tapery=20)
    p = gaussian_filter(rng.standard_normal((nz_full, w.ny, w.nx)), sigma=5)
    p *= 0.05 / np.max(np.abs(p))
    Z, Y, X = _coords(w)
    v = (1500.0 + 0.4 * Z) * (1 + p[: w.nz])
    w.slow2 = (1.0 / v ** 2).astype(np.float32)
    depths = rng.choice(np.arange(10, 190), size=5, replace=False)
    amps = rng.uniform(-0.1, 0.1, size=5)
    ds = np.zeros((w.nz, w.ny, w.nx), np.float32)
    for dpt, a in zip(depths, amps):
        if dpt < w.nz:
            ds[dpt] = a * w.slow2[dpt]
    w.dslow = ds
    w.geom = dict(sx=np.array([w.nx // 2 * w.dx], np.float32), sy=np.array([w.ny // 2 * w.dy], np.float32),
                  sz=np.array([0.0], np.float32), s_ids=np.array([0], np.int32), **w.surface_receivers())
    w.wavelet = ricker_spectrum(w.freqs)[None, :].astype(np.complex64)
    return w


def config4(nz=None, shot=0, seed=1003):
    """FWI gradient workload; returns (Workload with the starting model, true slowness
    s_true [nz][ny][nx] float32, starting slowness s0 [nz][ny][nx] float32)."""
    rng = np.random.default_rng(seed)
    nz_full = 300
    w = Workload(name="fwi-smooth-pspi-384x384x300-nw96", nx=384, ny=384, nz=nz or nz_full, dx=10.0, dy=10.0,
                 dz=10.0, nw=96, ow=3.0, dw=27.0 / 95.0, nref=4, step="pspi", taperx=20, tapery=20)
    Z, Y, X = _coords(w)
    v0 = 1500.0 + 0.5 * Z
    pert = np.zeros_like(v0)
    for _ in range(3):
        cx, cy = rng.uniform(0.25, 0.75, 2) * np.array([w.nx * w.dx, w.ny * w.dy])
        cz = rng.uniform(0.25, 0.75) * nz_full * w.dz
        amp = rng.choice([-0.08, 0.08])
        pert += amp * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2) / (2 * 150.0 ** 2))
    s_true = (1.0 / (v0 * (1 + pert))).astype(np.float32)
    s0 = (1.0 / v0).astype(np.float32)
    src = rng.uniform(0.1, 0.9, size=(8, 2)) * np.array([w.nx * w.dx, w.ny * w.dy])
    w.sources = src                      # the eight seeded source positions (x, y)
    w.geom = config4_geometry(w, shot)
    w.wavelet = ricker_spectrum(w.freqs)[None, :].astype(np.complex64)
    w.slow2 = s0 ** 2
    return w, s_true, s0


def config4_geometry(w, shot):
    """Geometry of shot ``shot`` (0-7) of the FWI workload: its source on the
    surface, receivers on every surface node."""
    sx, sy = w.sources[shot]
    return dict(sx=np.array([sx], np.float32), sy=np.array([sy], np.float32), sz=np.array([w.oz], np.float32),
                s_ids=np.array([0], np.int32), **w.surface_receivers())


def config3(nshots=32, nz=None, seed=1002):
    """Batched forward + imaging: a list of single-shot Workloads of uneven grid and
    band.  Their s^2 is generated on the device by ``slow2_on`` (the 32 models
    hold about 2 GB)."""
    rng = np.random.default_rng(seed)
    dw = 43.0 / 159.0
    out = []
    for i in range(nshots):
        n = int(rng.choice([128, 192, 256, 320, 384]))
        nw = int(rng.integers(48, 161))
        ow = 2.0 + float(rng.integers(0, 160 - nw + 1)) * dw
        w = Workload(name=f"shot{i}-{n}x{n}x{nz or 200}-nw{nw}", nx=n, ny=n, nz=nz or 200, dx=10.0, dy=10.0,
                     dz=10.0, nw=nw, ow=ow, dw=dw, nref=6, step="pspi", taperx=20, tapery=20)
        cx, cy = rng.uniform(0.25, 0.75, 2) * n * w.dx
        cz = float(rng.uniform(0.25, 0.75)) * 200 * w.dz
        w.anomaly = (float(cx), float(cy), cz)
        w.geom = dict(sx=np.array([n // 2 * w.dx], np.float32), sy=np.array([n // 2 * w.dy], np.float32),
                      sz=np.array([0.0], np.float32), s_ids=np.array([0], np.int32), **w.surface_receivers())
        w.wavelet = ricker_spectrum(w.freqs)[None, :].astype(np.complex64)
        out.append(w)
    return out


def slow2_on(w, device):
    """s^2 [nz][ny][nx] (float32, on ``device``) of a config1-family workload:
    v = (1500 + 0.5 z) (1 + 0.10 exp(-|r - c|^2 / (2 150^2)))."""
    import torch
    if getattr(w, "layers", None) is not None:
        return _slow2_layers(w, device)
    if w.anomaly is None:
        return torch.as_tensor(w.slow2).to(device)
    cx, cy, cz = w.anomaly
    z = (w.oz + w.dz * torch.arange(w.nz, device=device, dtype=torch.float64))[:, None, None]
    y = (w.oy + w.dy * torch.arange(w.ny, device=device, dtype=torch.float64))[None, :, None]
    x = (w.ox + w.dx * torch.arange(w.nx, device=device, dtype=torch.float64))[None, None, :]
    v = (1500.0 + 0.5 * z) * (1 + 0.10 * torch.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2)
                                                    / (2 * 150.0 ** 2)))
    return (1.0 / v ** 2).float().contiguous()


def config5(nz=None, seed=1004):
    """Large migration with gradient, one shot of 64: 512 x 512 x 400, d = 12.5 m,
    nw = 200 (2-50 Hz), PSPI with nref 8; 12 layers of 1500-4500 m/s whose
    interfaces dip by seeded angles within +-10 degrees, and a Gaussian body of
    4500 m/s; source at a seeded surface position, receivers on every surface node.
    s^2 comes from ``slow2_on`` (``w.layers`` holds the layer parameters)."""
    rng = np.random.default_rng(seed)
    nz_full = 400
    w = Workload(name="born-pspi-512x512x400-nw200", nx=512, ny=512, nz=nz or nz_full, dx=12.5, dy=12.5,
                 dz=12.5, nw=200, ow=2.0, dw=48.0 / 199.0, nref=8, step="pspi", taperx=20, tapery=20)
    depth = nz_full * w.dz
    tops = np.sort(rng.uniform(0.05, 0.95, 11)) * depth
    dips = np.deg2rad(rng.uniform(-10, 10, size=(11, 2)))
    vel = np.linspace(1500.0, 4500.0, 12)
    body = (float(rng.uniform(0.3, 0.7) * w.nx * w.dx), float(rng.uniform(0.3, 0.7) * w.ny * w.dy),
            float(rng.uniform(0.4, 0.7) * depth), 400.0)
    w.layers = (tops, dips, vel, body)
    sx, sy = rng.uniform(0.2, 0.8, 2) * np.array([w.nx * w.dx, w.ny * w.dy])
    w.geom = dict(sx=np.array([sx], np.float32), sy=np.array([sy], np.float32), sz=np.array([0.0], np.float32),
                  s_ids=np.array([0], np.int32), **w.surface_receivers())
    w.wavelet = ricker_spectrum(w.freqs)[None, :].astype(np.complex64)
    return w


def _slow2_layers(w, device):
    import torch
    tops, dips, vel, (bx, by, bz, br) = w.layers
    z = (w.oz + w.dz * torch.arange(w.nz, device=device, dtype=torch.float64))[:, None, None]
    y = (w.oy + w.dy * torch.arange(w.ny, device=device, dtype=torch.float64))[None, :, None]
    x = (w.ox + w.dx * torch.arange(w.nx, device=device, dtype=torch.float64))[None, None, :]
    cx, cy = w.nx * w.dx / 2, w.ny * w.dy / 2
    v = torch.full((w.nz, w.ny, w.nx), float(vel[0]), dtype=torch.float64, device=device)
    for i in range(len(tops)):
        surf = tops[i] + np.tan(dips[i, 0]) * (x - cx) + np.tan(dips[i, 1]) * (y - cy)
        v = torch.where(z >= surf, torch.full_like(v, float(vel[i + 1])), v)
    g = torch.exp(-((x - bx) ** 2 + (y - by) ** 2 + (z - bz) ** 2) / (2 * br ** 2))
    v = v + (4500.0 - v) * g
    return (1.0 / v ** 2).float().contiguous()


CONFIGS = {"config1": config1, "config2": config2}
