"""The B200 PSPI depth step against the reference's own GPU step at the
benchmark sizes: pyfwix's kernels (taper, phase shift, selector, compiled from
the reference sources into the oracle's shim) composed with cuFFT exactly as
PSPI::cu_forward composes them (propagator/src/PSPI.cpp:6-24).  Same inputs
on both sides; the outputs agree to the float tolerance of the parity tests
(the shim's cuFFT runs without the reference's 1/sqrt(NX NY) store callback,
so its output is divided by NX NY here), and the time per step of both is
printed (``pytest -s``) with the ratio.  The reference side is timed without
its per-depth host-to-device copies of labels and references, and without the
callback's work, so its time is a lower bound."""
import ctypes
import os

import numpy as np
import pytest
import torch

from tests.gpu_helpers import rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "librefshim.so")

# (NX = NY, nw, nref): the first, second and fourth benchmark configurations' slices
CASES = [(128, 64, 4), (256, 128, 4), (384, 96, 4)]


def _k_axis(n, d):
    i = np.arange(n)
    return (2 * np.pi * np.where(i <= n // 2, i, i - n) / (n * d)).astype(np.float32)


@pytest.mark.skipif(not os.path.exists(SHIM), reason="reference-kernel shim not built (reference sources absent)")
@pytest.mark.parametrize("n,nw,nref", CASES)
def test_pspi_step_against_reference_gpu_step(n, nw, nref):
    from pyfwix_b200.plan import Plan
    lib = ctypes.CDLL(SHIM)
    lib.refshim_pspi_forward_timed.restype = ctypes.c_int
    rng = np.random.default_rng(n)
    dx = dz = 10.0
    ow, dw = 3.0, 37.0 / max(nw - 1, 1)
    tap = 20
    s0 = (1 / 1500.0) ** 2
    sref = np.array([[s0 * (1 + 0.1 * r)] * nw for r in range(nref)], np.complex64)      # [nref][nw]
    labels = rng.integers(0, nref, size=(nw, n, n)).astype(np.int32)                       # [nw][NY][NX]
    p = Plan(nx=n, ny=n, nw=nw, ns=1, nz=1, dx=dx, dy=dx, dz=dz, ow=ow, dw=dw, nref=nref, taperx=tap, tapery=tap,
             step="pspi")
    p.set_refs(sref[None], labels[None].astype(np.uint8), phase_cache=False)
    p.ensure_workspace()
    x = torch.randn((1, nw, n, n), dtype=torch.complex64, device="cuda")
    dev = lambda a: torch.as_tensor(a).cuda()
    w2 = dev((2 * np.pi * (ow + dw * np.arange(nw))) ** 2).float()
    kx = dev(_k_axis(n, dx))
    sref_d, lab_d = dev(sref), dev(labels)
    out_ref, mk, wr = (torch.empty_like(x) for _ in range(3))
    ms = ctypes.c_float()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    reps = 10
    st = lib.refshim_pspi_forward_timed(n, n, nw, 1, nref, vp(w2), vp(kx), vp(kx), vp(sref_d), vp(lab_d),
                                        ctypes.c_float(dz), ctypes.c_float(0.0), tap, tap, vp(x), vp(out_ref), vp(mk),
                                        vp(wr), reps, ctypes.byref(ms))
    assert st == 0
    t_ref = ms.value

    def ours(cache):
        if cache:
            p.enable_phase_cache()
        else:
            p.disable_phase_cache()
        out = torch.empty_like(x)
        p.step(0, x, out)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            p.step(0, x, out)
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / reps

    out, t_ours = ours(False)
    out_c, t_cached = ours(True)
    want = (out_ref / (n * n)).cpu().numpy()
    assert rel(out.cpu().numpy(), want) < 1e-4
    assert rel(out_c.cpu().numpy(), want) < 1e-4
    cells = n * n * nw
    print(f"\nPSPI forward step {n}x{n}x{nw} nref {nref}: reference kernels + cuFFT {t_ref:.3f} ms "
          f"({cells / t_ref / 1e6:.2f} Gcell-steps/s); B200 step {t_ours:.3f} ms ({cells / t_ours / 1e6:.2f}), "
          f"{t_ref / t_ours:.1f}x; with the phase cache {t_cached:.3f} ms, {t_ref / t_cached:.1f}x")
    assert t_ours < t_ref
