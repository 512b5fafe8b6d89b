"""Whole-shot sweeps against the reference's own GPU path: pyfwix's kernels
(compiled from the reference sources into the oracle's shim) and cuFFT,
composed as the reference composes them (``refshim_shot_timed`` in
``oracle/refshim/shim.cu``: PSPI.cpp's in-place steps, Propagator.cpp's
modelling loop, the back-scattering adjoint's receiver field for the image).
That is the plain per-shot GPU path the batched B200 path is measured against.
The reference's injection kernel adds into the wavefield without atomics
(``propagator/src/injection.cu:89-92``), so with receivers on adjacent nodes its
launch loses some of the overlapping additions: the migration is timed with
that launch and compared with the same kernel launched one thread per
frequency (no race).

* First configuration, full size (128 x 128 x 100, 64 frequencies, nref 4):
  modelling and migration, outputs against the reference path's to 1e-4, times
  of both printed (``pytest -s``).
* Third configuration's batch (32 shots of 128-384 squared, 48-160 frequencies,
  nref 6) over its first ``NZ_BATCH`` levels (cell-steps grow in proportion to
  the depth count): the reference path shot after shot, and this library shot
  after shot, over streams and replayed from a CUDA graph; every image against
  the reference path's, and the throughputs printed with the ratio of the graph
  mode to the reference path.

The reference side runs without its ZFP compression and per-depth host copies
(see the shim), so its times are lower bounds."""
import ctypes
import os

import numpy as np
import pytest
import torch

from tests.gpu_helpers import rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "librefshim.so")
NZ_BATCH = 20

needs_shim = pytest.mark.skipif(not os.path.exists(SHIM), reason="reference-kernel shim not built")


def _k_axis(n, d):
    i = np.arange(n)
    return (2 * np.pi * np.where(i <= n // 2, i, i - n) / (n * d)).astype(np.float32)


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


class RefShot:
    """The reference path's inputs for one single-shot plan of this library (same
    references, labels, acquisition and model)."""

    def __init__(self, w, plan, src, rec, wav, s2=None):
        self.lib = ctypes.CDLL(SHIM)
        self.lib.refshim_shot_timed.restype = ctypes.c_int
        self.w, self.p = w, plan
        dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt)).cuda()
        self.w2 = dev((2 * np.pi * (w.ow + w.dw * np.arange(w.nw))) ** 2, np.float32)
        self.kx, self.ky = dev(_k_axis(plan.NX, w.dx), np.float32), dev(_k_axis(plan.NY, w.dy), np.float32)
        self.sref = plan._keep["sref"]
        lab = plan._keep["labels"]
        self.labels = lab[:, 0].to(torch.int32).contiguous()
        self.labw = torch.empty((w.nw, plan.NY, plan.NX), dtype=torch.int32, device="cuda")
        g = w.geom
        self.src = [dev(g[k], np.float32) for k in ("sx", "sy", "sz")] + [dev(np.zeros(len(g["sx"])), np.int32)]
        self.rec = [dev(g[k], np.float32) for k in ("rx", "ry", "rz")] + [dev(np.zeros(len(g["rx"])), np.int32)]
        self.wav = wav
        self.ws = [torch.empty(plan.wshape[1:], dtype=torch.complex64, device="cuda") for _ in range(4)]
        self.s2 = s2

    def run(self, task, data, reps=1):
        w, p = self.w, self.p
        ms = ctypes.c_float()
        keep = slow = den = None
        image = torch.zeros((w.nz, w.ny, w.nx), dtype=torch.float32, device="cuda")
        img_w = torch.empty((w.nw, w.ny, w.nx), dtype=torch.complex64, device="cuda")
        if task == 0:
            keep = torch.empty((w.nz, w.nw, p.NY, p.NX), dtype=torch.complex64, device="cuda")
            s2 = self.s2.to(torch.complex64)                                   # [nz][ny][nx]
            slow = torch.cat([s2, s2[-1:]])[:, None].expand(w.nz + 1, w.nw, w.ny, w.nx).contiguous()
            den = torch.ones_like(slow)
        st = self.lib.refshim_shot_timed(
            task, p.NX, p.NY, w.nw, w.nz, w.nref, _vp(self.w2), _vp(self.kx), _vp(self.ky), _vp(self.sref),
            _vp(self.labels), _vp(self.labw), ctypes.c_float(w.dz), ctypes.c_float(w.eps), w.taperx, w.tapery,
            ctypes.c_float(w.ox), ctypes.c_float(w.oy), ctypes.c_float(w.oz), ctypes.c_float(w.dx),
            ctypes.c_float(w.dy), len(w.geom["sx"]), *[_vp(t) for t in self.src], _vp(self.wav),
            len(w.geom["rx"]), *[_vp(t) for t in self.rec], _vp(data), _vp(slow), _vp(den), _vp(keep), _vp(image),
            _vp(img_w), *[_vp(t) for t in self.ws], reps, ctypes.byref(ms))
        assert st == 0, st
        return image, ms.value / 1e3


def _events(fn, reps=1):
    fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


@needs_shim
def test_config1_against_reference_gpu_path():
    from pyfwix_b200 import refsampler, workloads
    from pyfwix_b200.plan import Plan
    w = workloads.config1()
    p = Plan(ns=1, device="cuda", **w.plan_kwargs())
    s2 = torch.as_tensor(w.slow2).cuda()
    sref, labels = refsampler.sample(s2[:, None], w.nref)
    p.set_refs(refsampler.expand_refs(sref, w.nw), labels)
    s2c = s2[:, None].to(torch.complex64)
    p.set_model(s2c, torch.ones_like(s2c))
    g = w.geom
    src = p.traces(g["sx"], g["sy"], g["sz"], np.zeros(1, np.int32))
    rec = p.traces(g["rx"], g["ry"], g["rz"], np.zeros(len(g["rx"]), np.int32))
    wav = torch.as_tensor(w.wavelet).cuda()
    ref = RefShot(w, p, src, rec, wav, s2=s2)
    ntr = len(g["rx"])
    # modelling
    data_ref = torch.empty((ntr, w.nw), dtype=torch.complex64, device="cuda")
    _, t_ref_model = ref.run(0, data_ref, reps=3)
    bd = torch.empty((w.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    data = torch.empty_like(data_ref)
    t_model = _events(lambda: p.propagate(src, rec, wav, data, bd, None), reps=3)
    assert rel(data.cpu().numpy(), data_ref.cpu().numpy()) < 1e-4
    # migration of the same data: timed as the reference launches it, compared with
    # the receivers injected without that launch's race (task 2, see the shim)
    _, t_ref_image = ref.run(1, data, reps=3)
    img_ref, _ = ref.run(2, data, reps=0)
    img = torch.zeros((w.nz, w.ny, w.nx), dtype=torch.float32, device="cuda")
    t_image = _events(lambda: (img.zero_(), p.migrate(src, rec, wav, data, img)), reps=3)
    assert rel(img.cpu().numpy(), img_ref.cpu().numpy()) < 1e-4
    cells = 2 * w.nx * w.ny * w.nw * w.nz
    print(f"\nconfig1 {w.name}: modelling reference path {t_ref_model * 1e3:.1f} ms "
          f"({cells / t_ref_model / 1e9:.2f} Gcell-steps/s), B200 {t_model * 1e3:.1f} ms "
          f"({cells / t_model / 1e9:.2f}), {t_ref_model / t_model:.1f}x; imaging reference path "
          f"{t_ref_image * 1e3:.1f} ms ({cells / t_ref_image / 1e9:.2f}), B200 {t_image * 1e3:.1f} ms "
          f"({cells / t_image / 1e9:.2f}), {t_ref_image / t_image:.1f}x")
    assert t_model < t_ref_model and t_image < t_ref_image


@needs_shim
def test_config3_batch_against_reference_gpu_path():
    from pyfwix_b200 import workloads
    from pyfwix_b200.batch import MigrationBatch
    ws = workloads.config3(nshots=32, nz=NZ_BATCH)
    b = MigrationBatch(ws, nstreams=8)
    b.model_data()
    torch.cuda.synchronize()
    cells = 2 * b.cells
    t_plain = _events(b.run_plain)
    b.zero_images()
    b.run_plain()
    torch.cuda.synchronize()
    ours = [im.clone() for im in b.images()]
    t_streams = _events(b.run_streams)
    b.capture()
    t_graph = _events(b.run_graph)
    # the reference path, shot after shot, on the same instances and data
    t_ref = 0.0
    worst = 0.0
    for inst, im in zip(b.inst, ours):
        r = RefShot(inst.w, inst.plan, inst.src, inst.rec, inst.wavelet)
        _, t = r.run(1, inst.data, reps=1)
        img_ref, _ = r.run(2, inst.data, reps=0)
        t_ref += t
        worst = max(worst, rel(im.cpu().numpy(), img_ref.cpu().numpy()))
        del r
    assert worst < 1e-4, worst
    g = lambda t: cells / t / 1e9
    print(f"\nconfig3 batch, 32 shots, first {NZ_BATCH} levels ({cells} cell-steps): reference path shot "
          f"after shot {t_ref:.3f} s ({g(t_ref):.2f} Gcell-steps/s); B200 plain {t_plain:.3f} s ({g(t_plain):.2f}), "
          f"streams {t_streams:.3f} s ({g(t_streams):.2f}), graph {t_graph:.3f} s ({g(t_graph):.2f}); "
          f"graph over the reference path {t_ref / t_graph:.1f}x, plain over the reference path "
          f"{t_ref / t_plain:.1f}x; worst image difference {worst:.1e}")
    assert t_graph < t_ref
