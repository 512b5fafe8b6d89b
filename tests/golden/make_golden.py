"""Generates the golden fixtures of this directory from pyfwix's OWN CUDA kernels.

Run on a machine with a GPU and the reference shim built
(``python -m oracle.refshim.build``, which compiles the reference's
``propagator/src/*.cu`` kernels into ``oracle/_ref/librefshim.so``):

    python tests/golden/make_golden.py [outdir]

Every fixture holds seeded inputs, the grid parameters and the output of the
reference's kernels composed the way the reference's C++ operators compose
them (each composition below cites the file:line it replays).  The 2D FFTs
between kernels are the unitary transforms of ``operator/src/FFT.cpp:36-69``
(cuFFT scaled by 1/sqrt(NX NY)), run here as ``torch.fft.fft2(norm="ortho")``.

One deviation, stated: the reference's NSPS add-adjoint
(``propagator/src/NSPS.cpp:6-25``) hands ``model_k`` and ``_wfld_ref`` to
``PhaseShift::cu_adjoint`` in swapped order, which zeroes the spectrum it just
computed; the fixture ``nsps`` records the transpose of the NSPS forward
instead (the same kernels in the order the forward implies), which is what the
operator's dot test requires.

Two regimes are written: ``reference_kernels_real.npz`` (real slowness and
density, real reference slownesses, eps = 0: the regime of every benchmark
configuration, where the reference's float arithmetic is well conditioned)
and ``reference_kernels_complex.npz`` (complex slowness and references,
eps = 0.01), where the reference's float square roots lose accuracy to
cancellation in the evanescent region (phase_shift.cu:38-41,
prop_kernels.cuh:89-102) and the tests bound the difference accordingly.

The fixtures pin the oracle (tests/test_golden.py, CPU) and the B200 kernels
(tests/test_gpu_golden.py).
"""
from __future__ import annotations

import ctypes
import math
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
SHIM = os.path.join(ROOT, "oracle", "_ref", "librefshim.so")

GRID = dict(nx=32, ny=32, padx=8, pady=4, nw=4, ns=2, nref=3, dx=10.0, dy=12.0, dz=10.0, ox=0.0, oy=0.0, oz=0.0,
            ow=10.0, dw=12.0, eps=0.01, taperx=4, tapery=3, eps_scat=0.04)


def _lib():
    lib = ctypes.CDLL(SHIM)
    for name in ("refshim_phase_shift", "refshim_select", "refshim_taper", "refshim_inject", "refshim_reflect",
                 "refshim_imaging", "refshim_lin_reflect", "refshim_mult_kxky", "refshim_slow_scale",
                 "refshim_scale_by_iw", "refshim_pad"):
        getattr(lib, name).restype = ctypes.c_int
    return lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _ok(st):
    if st != 0:
        raise RuntimeError(f"reference kernel failed with CUDA error {st}")


def _tables(g):
    """Wavenumbers and frequencies as the reference fills them on the host in
    float (``propagator/src/PhaseShift.h:43-70``, ``propagator/src/Scatter.h``)."""
    def k(n, d):
        dk = np.float32(2 * math.pi / (d * n))
        return np.array([(i if i <= n // 2 else i - n) * dk for i in range(n)], np.float32)
    NX, NY = g["nx"] + g["padx"], g["ny"] + g["pady"]
    f = np.array([g["ow"] + i * g["dw"] for i in range(g["nw"])], np.float32)
    w = (np.float32(2 * math.pi) * f).astype(np.float32)
    dev = lambda a: torch.as_tensor(a).cuda()
    return dev(k(NX, g["dx"])), dev(k(NY, g["dy"])), dev(w * w), dev(w)


def _c(a):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", torch.complex64)


def _fft(t):
    return torch.fft.fft2(t, norm="ortho").contiguous()


def _ifft(t):
    return torch.fft.ifft2(t, norm="ortho").contiguous()


def _crandn(rng, shape, scale=1.0):
    return (scale * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))).astype(np.complex64)


def make(outdir, regime):
    lib = _lib()
    g = dict(GRID)
    cplx = regime == "complex"
    if not cplx:
        g["eps"] = 0.0
    NX, NY, nw, ns, nref = g["nx"] + g["padx"], g["ny"] + g["pady"], g["nw"], g["ns"], g["nref"]
    kx, ky, w2, w = _tables(g)
    rng = np.random.default_rng(2024)
    s0 = (1.0 / 1800.0) ** 2
    sref = np.empty((nref, nw), np.complex64)
    for r in range(nref):
        sref[r] = s0 * (1 + 0.15 * r) * (1 + 0.02 * rng.random()) + 1j * cplx * s0 * 0.03 * rng.standard_normal(nw)
    labels = rng.integers(0, nref, size=(nw, NY, NX)).astype(np.int32)
    wshape = (ns, nw, NY, NX)
    x = _crandn(rng, wshape)
    y = _crandn(rng, wshape)
    dz, eps = g["dz"], g["eps"]
    out = {}
    lab_d = torch.as_tensor(labels).cuda()

    def ps(mode, sr, inp, acc):
        _ok(lib.refshim_phase_shift(mode, NX, NY, nw, ns, _p(w2), _p(kx), _p(ky), _p(sr), ctypes.c_float(dz),
                                    ctypes.c_float(eps), _p(inp), _p(acc)))

    def sel(value, inp, acc):
        _ok(lib.refshim_select(NX, NY, nw, ns, value, _p(lab_d), _p(inp), _p(acc)))

    def taper(inp, acc):
        _ok(lib.refshim_taper(NX, NY, nw, ns, g["taperx"], g["tapery"], _p(inp), _p(acc)))

    srefs = [_c(sref[r]) for r in range(nref)]
    xd, yd = _c(x), _c(y)

    # phase shift forward / adjoint / inverse of one reference (phase_shift.cu)
    for mode, name in ((0, "ps_fwd"), (1, "ps_adj"), (2, "ps_inv")):
        acc = torch.zeros_like(xd)
        ps(mode, srefs[1], xd, acc)
        out[name] = acc.cpu().numpy()

    # taper forward (taper.cu) and select (selector.cu)
    acc = torch.zeros_like(xd)
    taper(xd, acc)
    out["taper"] = acc.cpu().numpy()
    acc = torch.zeros_like(xd)
    sel(1, xd, acc)
    out["select1"] = acc.cpu().numpy()

    # PSPI add-forward (PSPI.cpp:6-24)
    mk = torch.zeros_like(xd)
    taper(xd, mk)
    mk = _fft(mk)
    data = torch.zeros_like(xd)
    for r in range(nref):
        wr = torch.zeros_like(xd)
        ps(0, srefs[r], mk, wr)
        wr = _ifft(wr)
        sel(r, wr, data)
    out["pspi_fwd"] = data.cpu().numpy()

    # PSPI add-adjoint, no taper (PSPI.cpp:26-44), and in-place adjoint (:85-103)
    mk = torch.zeros_like(yd)
    for r in range(nref):
        wr = torch.zeros_like(yd)
        sel(r, yd, wr)
        wr = _fft(wr)
        ps(1, srefs[r], wr, mk)
    m = _ifft(mk)
    out["pspi_adj"] = m.cpu().numpy()
    acc = torch.zeros_like(yd)
    taper(m, acc)
    out["pspi_adj_inplace"] = acc.cpu().numpy()

    # NSPS add-forward (NSPS.cpp:27-45)
    mk = torch.zeros_like(xd)
    for r in range(nref):
        wr = torch.zeros_like(xd)
        sel(r, xd, wr)
        wr = _fft(wr)
        ps(0, srefs[r], wr, mk)
    out["nsps_fwd"] = _ifft(mk).cpu().numpy()
    # NSPS adjoint as the transpose of the forward (see the module docstring)
    dk = _fft(yd)
    m = torch.zeros_like(yd)
    for r in range(nref):
        wr = torch.zeros_like(yd)
        ps(1, srefs[r], dk, wr)
        wr = _ifft(wr)
        sel(r, wr, m)
    out["nsps_adj"] = m.cpu().numpy()

    # Injection / recording at two levels (injection.cu)
    nt = 20
    cx = rng.uniform(-15, NX * g["dx"] + 5, nt).astype(np.float32)
    cy = rng.uniform(-15, NY * g["dy"] + 5, nt).astype(np.float32)
    cz = rng.uniform(0, 3.5 * dz, nt).astype(np.float32)
    ids = rng.integers(0, ns, nt).astype(np.int32)
    tr = _crandn(rng, (nt, nw))
    cxd, cyd, czd, idd = (torch.as_tensor(a).cuda() for a in (cx, cy, cz, ids))
    for iz in (1, 2):
        wf = torch.zeros_like(xd)
        trd = _c(tr)
        _ok(lib.refshim_inject(0, NX, NY, nw, ns, ctypes.c_float(g["ox"]), ctypes.c_float(g["oy"]),
                               ctypes.c_float(g["dx"]), ctypes.c_float(g["dy"]), nt, _p(cxd), _p(cyd), _p(czd),
                               _p(idd), ctypes.c_float(g["oz"]), ctypes.c_float(dz), iz, _p(trd), _p(wf)))
        out[f"inject_z{iz}"] = wf.cpu().numpy()
        rec = torch.zeros((nt, nw), dtype=torch.complex64, device="cuda")
        _ok(lib.refshim_inject(1, NX, NY, nw, ns, ctypes.c_float(g["ox"]), ctypes.c_float(g["oy"]),
                               ctypes.c_float(g["dx"]), ctypes.c_float(g["dy"]), nt, _p(cxd), _p(cyd), _p(czd),
                               _p(idd), ctypes.c_float(g["oz"]), ctypes.c_float(dz), iz, _p(rec), _p(yd)))
        out[f"record_z{iz}"] = rec.cpu().numpy()

    # Reflect / imaging / linearised reflection on one level (reflect.cu, imaging_condition.cu,
    # lin_reflect.cu); slow2 / den2 are the [2][nw][ny][nx] slices of levels z and z+1
    nx, ny = g["nx"], g["ny"]
    slow2 = (s0 * (1 + 0.3 * rng.random((2, nw, ny, nx)))
             + 1j * cplx * s0 * 0.01 * rng.standard_normal((2, nw, ny, nx))).astype(np.complex64)
    den2 = (1 + 0.4 * rng.random((2, nw, ny, nx)) + 0j).astype(np.complex64)
    sd, rd = _c(slow2), _c(den2)
    acc = torch.zeros_like(xd)
    _ok(lib.refshim_reflect(0, NX, NY, nx, ny, nw, ns, _p(sd), _p(rd), _p(xd), _p(acc)))
    out["reflect_fwd"] = acc.cpu().numpy()
    acc = torch.zeros_like(xd)
    _ok(lib.refshim_reflect(1, NX, NY, nx, ny, nw, ns, _p(sd), _p(rd), _p(acc), _p(yd)))
    out["reflect_adj"] = acc.cpu().numpy()
    image = _crandn(rng, (nw, ny, nx))
    imd = _c(image)
    acc = torch.zeros_like(xd)
    _ok(lib.refshim_imaging(0, NX, NY, nx, ny, nw, ns, _p(imd), _p(acc), _p(xd)))
    out["ic_fwd"] = acc.cpu().numpy()
    img = torch.zeros_like(imd)
    _ok(lib.refshim_imaging(1, NX, NY, nx, ny, nw, ns, _p(img), _p(yd), _p(xd)))
    out["ic_adj"] = img.cpu().numpy()
    dm4 = _crandn(rng, (4, nw, ny, nx))
    dmd = _c(dm4)
    dr = torch.zeros((nw, ny, nx), dtype=torch.complex64, device="cuda")
    _ok(lib.refshim_lin_reflect(0, nx, ny, nw, _p(dmd), _p(dr), _p(sd), _p(rd)))
    out["lin_reflect_fwd"] = dr.cpu().numpy()
    drin = _crandn(rng, (nw, ny, nx))
    dri = _c(drin)
    g4 = torch.zeros_like(dmd)
    _ok(lib.refshim_lin_reflect(1, nx, ny, nw, _p(g4), _p(dri), _p(sd), _p(rd)))
    out["lin_reflect_adj"] = g4.cpu().numpy()

    # Scatter forward / adjoint, taylor = 1 (Scatter.cpp:76-107); the slice is padded
    # by edge replication (scatter.cu pad_fwd); coefficients 1, 1/2 (Scatter.h)
    coef = [1.0, 0.5, 0.375, 0.3125, 0.2734375]
    taylor = 1
    sslice = _c(slow2[0])
    spad = torch.zeros((nw, NY, NX), dtype=torch.complex64, device="cuda")
    _ok(lib.refshim_pad(nx, ny, NX, NY, nw, _p(sslice), _p(spad)))
    wk = _fft(xd)
    data = torch.zeros_like(xd)
    for it in range(taylor + 1):
        sc = torch.zeros_like(xd)
        _ok(lib.refshim_mult_kxky(NX, NY, nw, ns, _p(w), _p(kx), _p(ky), it, _p(wk), _p(sc)))
        sc = _ifft(sc)
        _ok(lib.refshim_slow_scale(0, NX, NY, nw, ns, _p(spad), ctypes.c_float(coef[it]), it,
                                   ctypes.c_float(g["eps_scat"]), _p(sc), _p(sc)))
        _ok(lib.refshim_scale_by_iw(0, NX, NY, nw, ns, _p(w), ctypes.c_float(dz), _p(sc), _p(data)))
    out["scatter_fwd"] = data.cpu().numpy()
    model = torch.zeros_like(yd)
    for it in range(taylor + 1):
        sc = torch.zeros_like(yd)
        _ok(lib.refshim_scale_by_iw(1, NX, NY, nw, ns, _p(w), ctypes.c_float(dz), _p(sc), _p(yd)))
        _ok(lib.refshim_slow_scale(1, NX, NY, nw, ns, _p(spad), ctypes.c_float(coef[it]), it,
                                   ctypes.c_float(g["eps_scat"]), _p(sc), _p(sc)))
        sc = _fft(sc)
        wkk = torch.zeros_like(yd)
        _ok(lib.refshim_mult_kxky(NX, NY, nw, ns, _p(w), _p(kx), _p(ky), it, _p(sc), _p(wkk)))
        model += _ifft(wkk)
    out["scatter_adj"] = model.cpu().numpy()

    torch.cuda.synchronize()
    os.makedirs(outdir, exist_ok=True)
    path = os.path.join(outdir, f"reference_kernels_{regime}.npz")
    np.savez_compressed(path, grid=np.array(repr(g)), sref=sref, labels=labels.astype(np.uint8), x=x, y=y,
                        cx=cx, cy=cy, cz=cz, ids=ids, traces=tr, slow2=slow2, den2=den2, image=image,
                        dm4=dm4, dr_in=drin, taylor=np.int32(taylor), **{"out_" + k: v for k, v in out.items()})
    print("wrote", path, sum(v.nbytes for v in out.values()) // 1024, "KiB of outputs")
    return path


if __name__ == "__main__":
    for regime in ("real", "complex"):
        make(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)), regime)
