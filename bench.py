#!/usr/bin/env python
"""Benchmark of the one-way WEM depth-stepping path on B200.

Workload (default, ``--config config2``): Born forward + adjoint (migration) with
NSPS on one shot, 256 x 256 x 200, 128 frequencies (3-40 Hz), seeded synthetic
model (see pyfwix_b200/workloads.py).  One step = ExtendedBorn forward of the
5-layer reflectivity (all four scattering sweeps) followed by ExtendedBorn
adjoint of the data it produced (the FWI/migration gradient), with the
background wavefields already computed and resident in HBM.

Metric: Gcell-steps/s, one cell-step = one (x, y, w) sample advanced one depth
level, counted once per operator application (Born forward and Born adjoint:
2 * nx*ny*nw*nz per step).

Under torchrun each rank runs its own shot (independent replicas, no collective
on the data path): value = cell-steps of all ranks / max-over-ranks time,
scaling "weak".

``--impl reference`` times the reference path's CPU restatement (the oracle in
complex64 with scipy.fft on all host threads) on a bounded slab of the same
workload; the reference itself has no CPU implementation of this path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-steps/s (x*y*w*z), Born forward + adjoint"
HBM_FALLBACK_GBS = 6650.0
ALG_BYTES_PER_CELL_STEP = 16  # one wavefield read + written once per depth step
TRAFFIC_PROFILE = "nsps_step_256x256x128.txt"  # DRAM bytes per step of the timed step's kernels (ncu)


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", default="config2")
    ap.add_argument("--nz", type=int, default=None, help="override depth count (quick runs only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-per-w", type=int, default=1,
                    help="also time e2e with the per-frequency model domain when host memory allows (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fwi", action="store_true", help="skip the FWI-gradient timing")
    ap.add_argument("--fwi-nz", type=int, default=None, help="depth levels of the FWI workload (quick runs)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched forward+imaging timing")
    ap.add_argument("--no-config1", action="store_true", help="skip the plain modelling + imaging timing")
    ap.add_argument("--no-autotune", action="store_true",
                    help="time the plan's default form of the depth step instead of the tuned one")
    ap.add_argument("--tuning", default=None,
                    help="apply this tuner choice instead of timing candidates: col_tma,slices_per_launch,streams"
                         "[,fused] (profiling runs, where the tuner would time under the profiler)")
    ap.add_argument("--no-packed", action="store_true", help="skip the packed-background Born timing")
    ap.add_argument("--large", action="store_true",
                    help="run only the 512 x 512 x 400 x 200 Born on packed storage and print its own line")
    ap.add_argument("--batched-nz", type=int, default=None, help="depth levels of the batched workload (quick runs)")
    ap.add_argument("--batched-shots", type=int, default=32)
    ap.add_argument("--batched-streams", type=int, default=8)
    ap.add_argument("--profile-n", type=int, default=None, help="lateral size of the profiled step (default: the workload's)")
    ap.add_argument("--profile-nw", type=int, default=96)
    ap.add_argument("--profile-nref", type=int, default=4)
    ap.add_argument("--profile-step", choices=["pspi", "nsps", "pspi-adj", "nsps-adj", "smooth", "smooth-adj"],
                    default=None,
                    help="run one depth step of the workload's wavefield and exit (for ncu captures)")
    return ap.parse_args()


# ----------------------------------------------------------------------------- helpers

def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def profiled_traffic(name):
    """Per-step DRAM bytes of the depth step from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_step:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------------------- B200 arm

def parse_tuning(text):
    """"col_tma,slices_per_launch,streams[,fused]" -> the dict Plan.set_tuning takes."""
    f = [int(v) for v in text.split(",")]
    return {"col_tma": bool(f[0]), "slices_per_launch": f[1], "streams": f[2],
            "fused_cluster_step": bool(f[3]) if len(f) > 3 else False}


def setup_born(w, device, autotune=True, tuning=None):
    import torch

    from pyfwix_b200 import refsampler
    from pyfwix_b200.plan import Plan

    plan = Plan(ns=1, device=device, **w.plan_kwargs())
    s2 = torch.as_tensor(w.slow2)[:, None].to(device)                    # [nz][1][ny][nx]
    sref, labels = refsampler.sample(s2, w.nref, w.padx, w.pady)
    plan.set_refs(refsampler.expand_refs(sref, w.nw), labels)
    s2c = s2.to(torch.complex64)
    plan.set_model(s2c, torch.ones_like(s2c))
    # the fastest equivalent form of this plan's depth step (else the plan's
    # defaults, or a choice given by the caller)
    if tuning is not None:
        plan.set_tuning(tuning)
        tuning = dict(tuning, applied_without_timing=True)
    else:
        tuning = plan.autotune() if autotune else None
    g = w.geom
    src = plan.traces(g["sx"], g["sy"], g["sz"], np.zeros(len(g["sx"]), np.int32))
    rec = plan.traces(g["rx"], g["ry"], g["rz"], np.zeros(len(g["rx"]), np.int32))
    wav = torch.as_tensor(w.wavelet).to(device)
    bd = torch.empty((w.nz,) + plan.wshape, dtype=torch.complex64, device=device)
    bu = torch.empty_like(bd)
    data = torch.empty((len(g["rx"]), w.nw), dtype=torch.complex64, device=device)
    plan.propagate(src, rec, wav, data, bd, bu)
    dslow = torch.as_tensor(w.dslow)[:, None].to(device).to(torch.complex64)
    dden = torch.zeros_like(dslow)
    gs = torch.empty_like(dslow)
    gr = torch.empty_like(dslow)
    plan.ensure_workspace(2)
    torch.cuda.synchronize()
    return dict(plan=plan, rec=rec, bd=bd, bu=bu, data=data, dslow=dslow, dden=dden, gs=gs, gr=gr, tuning=tuning)


def born_step(st):
    p = st["plan"]
    p.born(st["rec"], st["bd"], st["bu"], st["dslow"], st["dden"], st["data"])
    p.born(st["rec"], st["bd"], st["bu"], st["gs"], st["gr"], st["data"], adjoint=True)


def born_packed_timing(st, w, steps=2):
    """The same Born forward + adjoint step on backgrounds kept in the packed
    fixed-rate store, at 8.5 bits per value (top-level keys) and at 16.5 bits per
    value (``rate16``): Gcell-steps/s, the stored bytes of the backgrounds against
    complex64, and the gradient's relative difference from the lossless step's."""
    import torch
    p = st["plan"]
    gs_ref = st["gs"].clone()
    nref = float(torch.linalg.vector_norm(gs_ref))
    res = {}
    for bits in (8, 16):
        p.set_pack_rate(bits)
        pd, pu = p.packed(w.nz), p.packed(w.nz)
        for iz in range(w.nz):
            p.pack(st["bd"][iz], pd[iz])
            p.pack(st["bu"][iz], pu[iz])
        fn = lambda: (p.born_packed(st["rec"], pd, pu, st["dslow"], st["dden"], st["data"]),
                      p.born_packed(st["rec"], pd, pu, st["gs"], st["gr"], st["data"], adjoint=True))
        fn()
        t = time_steps(fn, steps, lambda: None)
        diff = float(torch.linalg.vector_norm(st["gs"] - gs_ref)) / nref if nref > 0 else None
        res[bits] = {"value": 2 * w.nx * w.ny * w.nw * w.nz * steps / t / 1e9, "unit": "Gcell-steps/s",
                     "ms_per_step": t / steps * 1e3,
                     "background_bytes_ratio": 8.0 * st["bd"][0].numel() / p.packed_bytes,
                     "gradient_rel_diff": diff}
        del pd, pu
        torch.cuda.empty_cache()
    p.set_pack_rate(8)
    out = dict(res[8])
    out["rate16"] = res[16]
    return out


def setup_surface(w, device, per_w=False, pinned=True):
    """The Born workload through the drop-in surface: ``pyfwix_b200.CudaWEM``'s
    ``Propagator`` and ``ExtendedBorn``, the classes and calls of
    ``fwix/workers.py:62-76`` (``prop.forward(False, model, res)``,
    ``born.forward / adjoint(False, model, data)``), with every caller array a
    numpy array in host memory (pinned, or pageable with ``pinned=False``).  The
    background model is frequency-independent ([nz][1][ny][nx], one value per
    cell for every frequency, as the configuration's model is); the Born model
    domain is that too, or with ``per_w`` the reference's per-frequency domain
    [nz][nw][ny][nx].  The backgrounds are modelled here, untimed."""
    import torch

    from pyfwix_b200 import CudaWEM

    def host(shape):
        if pinned:
            return torch.empty(shape, dtype=torch.complex64, pin_memory=True).numpy()
        return np.empty(shape, np.complex64)

    s2 = host((w.nz, 1, w.ny, w.nx))
    s2[...] = w.slow2[:, None]
    den = host(s2.shape)
    den[...] = 1.0
    g = w.geom
    ntr = len(g["rx"])
    data = host((ntr, w.nw))
    par = dict(nref=w.nref, padx=w.padx, pady=w.pady, taperx=w.taperx, tapery=w.tapery, eps=w.eps,
               eps_scat=w.eps_scat, taylor=w.taylor, step=w.step, ox=w.ox, dx=w.dx, oy=w.oy, dy=w.dy, oz=w.oz,
               dz=w.dz, ow=w.ow, dw=w.dw)
    model = [s2, den]
    prop = CudaWEM.Propagator(model, data, w.wavelet, par, g)
    prop.forward(False, model, data)
    nwm = w.nw if per_w else 1
    ds, dr = host((w.nz, nwm, w.ny, w.nx)), host((w.nz, nwm, w.ny, w.nx))
    ds[...] = w.dslow[:, None]
    dr[...] = 0.0
    gs, gr = host(ds.shape), host(ds.shape)
    born = CudaWEM.ExtendedBorn([ds, dr], data, model, prop)
    torch.cuda.synchronize()
    return dict(prop=prop, born=born, dm=[ds, dr], g=[gs, gr], data=data)


def born_step_e2e(su):
    """One Born forward + adjoint step through the surface with host arrays: the
    perturbation goes in, the Born data come back, go in again for the adjoint,
    and the gradient comes back (``fwix/workers.py:66-76``)."""
    su["born"].forward(False, su["dm"], su["data"])
    su["born"].adjoint(False, su["g"], su["data"])


def e2e_bytes(su):
    nb = lambda a: a.size * a.itemsize
    return {"h2d_bytes_per_step": nb(su["dm"][0]) + nb(su["dm"][1]) + nb(su["data"]),
            "d2h_bytes_per_step": nb(su["data"]) + nb(su["g"][0]) + nb(su["g"][1])}


def _host_available():
    try:
        import psutil
        return psutil.virtual_memory().available
    except Exception:
        return 0


def time_steps(fn, k, barrier):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(k):
        fn()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    return e0.elapsed_time(e1) / 1e3  # seconds


def step_roofline(st, w, reps=20):
    """Average duration of one NSPS depth step (row + column + row passes) on this
    workload's wavefield, timed with CUDA events on the launching stream."""
    import torch
    p = st["plan"]
    x = st["bd"][w.nz // 2].clone()
    for _ in range(3):
        p.step(w.nz // 2, x, x)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        p.step(w.nz // 2, x, x)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def fwi_gradient_timing(device, nz=None, checkpoint="auto"):
    """Seconds per shot of the autograd FWI gradient (FWIGradient forward =
    modelling + misfit, backward = adjoint-state gradient) on one shot of the
    384 x 384 x 300 workload, timed with CUDA events after one untimed shot; the
    observed data are modelled first in the true model (untimed)."""
    import torch

    from pyfwix_b200 import workloads
    from pyfwix_b200.fwi import FWIGradient, SmoothFWI
    w, s_true, s0 = workloads.config4(nz=nz)
    par = dict(nref=w.nref, padx=0, pady=0, taperx=w.taperx, tapery=w.tapery, eps=0.0, ox=w.ox, oy=w.oy,
               oz=w.oz, dx=w.dx, dy=w.dy, dz=w.dz, ow=w.ow, dw=w.dw, checkpoint=checkpoint)
    wav = torch.as_tensor(w.wavelet).to(device)
    prob = SmoothFWI(s_true.shape, w.geom, wav, dict(par, checkpoint=None), device=device)
    d_obs = prob.model(torch.as_tensor(s_true), keep=False)
    refs = prob.refs.clone()
    del prob
    torch.cuda.empty_cache()
    par["refs"] = refs
    # one untimed shot first (device memory of the stored fields comes from the
    # allocator's cache afterwards, as for every shot after the first of a job)
    sw = torch.as_tensor(s0, device=device).requires_grad_(True)
    FWIGradient.apply(sw, wav, w.geom, d_obs, par).backward()
    del sw
    s = torch.as_tensor(s0, device=device).requires_grad_(True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record()
    J = FWIGradient.apply(s, wav, w.geom, d_obs, par)
    ev[1].record()
    J.backward()
    ev[2].record()
    torch.cuda.synchronize()
    t_fwd, t_bwd = ev[0].elapsed_time(ev[1]) / 1e3, ev[1].elapsed_time(ev[2]) / 1e3
    assert torch.isfinite(s.grad).all()
    cells = w.nx * w.ny * w.nw * w.nz
    return {"workload": w.name + ("" if nz is None else f" (nz={w.nz})") + ", 1 shot of 8",
            "s_per_shot": t_fwd + t_bwd, "forward_s_per_shot": t_fwd, "gradient_s_per_shot": t_bwd,
            "grad_over_forward": (t_fwd + t_bwd) / t_fwd, "checkpoint": FWIGradient.last_storage,
            "forward_gcell_steps_per_s": 2 * cells / t_fwd / 1e9, "objective": float(J.detach())}


def fwi_shots_timing(device, ws, rank, barrier, nz=None):
    """The FWI objective and gradient over ``ws`` shots of the 384 x 384 x 300
    workload, one shot per rank, through the product's multi-shot entry point
    (``fwi.shot_objective_and_gradient``: shots partitioned across the ranks,
    each rank modelling and differentiating its own, one all-reduce of J and the
    gradient); each rank's observed data are modelled first in the true model
    (untimed).  Seconds for the whole call, max over ranks."""
    import torch

    from pyfwix_b200 import workloads
    from pyfwix_b200.fwi import SmoothFWI, shot_objective_and_gradient
    w, s_true, s0 = workloads.config4(nz=nz)
    par = dict(nref=w.nref, padx=0, pady=0, taperx=w.taperx, tapery=w.tapery, eps=0.0, ox=w.ox, oy=w.oy,
               oz=w.oz, dx=w.dx, dy=w.dy, dz=w.dz, ow=w.ow, dw=w.dw, checkpoint="auto")
    wav = torch.as_tensor(w.wavelet).to(device)
    shot_list = [dict(geometry=workloads.config4_geometry(w, r % 8), wavelet=wav, d_obs=None) for r in range(ws)]
    prob = SmoothFWI(s_true.shape, shot_list[rank]["geometry"], wav, dict(par, checkpoint=None), device=device)
    shot_list[rank]["d_obs"] = prob.model(torch.as_tensor(s_true), keep=False)
    par["refs"] = prob.refs.clone()
    del prob
    torch.cuda.empty_cache()
    s = torch.as_tensor(s0, device=device)
    shot_objective_and_gradient(s, shot_list, par)      # warm-up (allocator, plan tables)
    t = time_steps(lambda: shot_objective_and_gradient(s, shot_list, par), 1, barrier)
    return {"workload": w.name + ("" if nz is None else f" (nz={w.nz})") + f", {ws} shots, one per rank",
            "api": "pyfwix_b200.fwi.shot_objective_and_gradient (one all-reduce of J and dJ/ds)",
            "shots": ws, "s": t}


def config1_timing(device, reps=10, autotune=True):
    """Plain PSPI forward modelling + imaging of the first configuration (one shot,
    128 x 128 x 100, 64 frequencies 2-30 Hz, nref 4 quantile references, taper 20,
    15 Hz Ricker at the surface centre, receivers on every surface node):
    ``fwix_propagate`` (down pass with injection and recording, reflection, up
    pass with recording) and then ``fwix_migrate`` of the modelled data (source
    and receiver fields continued in lockstep, image summed over frequency at
    every level), each timed with CUDA events over ``reps`` runs after a warm-up
    run.  Cell-steps count both continued wavefields of each sweep."""
    import torch

    from pyfwix_b200 import refsampler, workloads
    from pyfwix_b200.plan import Plan
    w = workloads.config1()
    plan = Plan(ns=1, device=device, **w.plan_kwargs())
    s2 = torch.as_tensor(w.slow2)[:, None].to(device)
    sref, labels = refsampler.sample(s2, w.nref, w.padx, w.pady)
    plan.set_refs(refsampler.expand_refs(sref, w.nw), labels)
    s2c = s2.to(torch.complex64)
    plan.set_model(s2c, torch.ones_like(s2c))
    # the fastest equivalent form of this plan's depth step (else the plan's defaults)
    tuning = plan.autotune() if autotune else None
    g = w.geom
    src = plan.traces(g["sx"], g["sy"], g["sz"], np.zeros(len(g["sx"]), np.int32))
    rec = plan.traces(g["rx"], g["ry"], g["rz"], np.zeros(len(g["rx"]), np.int32))
    wav = torch.as_tensor(w.wavelet).to(device)
    bd = torch.empty((w.nz,) + plan.wshape, dtype=torch.complex64, device=device)
    data = torch.empty((len(g["rx"]), w.nw), dtype=torch.complex64, device=device)
    img = torch.zeros((w.nz, w.ny, w.nx), dtype=torch.float32, device=device)
    model = lambda: plan.propagate(src, rec, wav, data, bd, None)
    image = lambda: plan.migrate(src, rec, wav, data, img)
    model()
    image()
    t_model = time_steps(model, reps, lambda: None) / reps
    t_image = time_steps(image, reps, lambda: None) / reps
    cells = w.nx * w.ny * w.nw * w.nz
    return {"workload": w.name, "modelling_ms": t_model * 1e3, "imaging_ms": t_image * 1e3,
            "modelling_gcell_steps_per_s": 2 * cells / t_model / 1e9,
            "imaging_gcell_steps_per_s": 2 * cells / t_image / 1e9,
            "modelling_plus_imaging_gcell_steps_per_s": 4 * cells / (t_model + t_image) / 1e9,
            "tuning": tuning}


def batched_timing(device, nshots=32, nz=None, nstreams=8):
    """Batched forward + imaging (32 shots of uneven grid and band, each migrated:
    source and receiver wavefields continued in lockstep, image summed over
    frequency at every level) run three ways on the same instances -- shot after
    shot on one stream ("plain", the per-shot path), over CUDA streams, and
    replayed from one captured CUDA graph -- each timed with CUDA events over one
    pass after a warm-up pass.  Cell-steps count both continued wavefields."""
    import torch

    from pyfwix_b200 import workloads
    from pyfwix_b200.batch import MigrationBatch
    ws = workloads.config3(nshots=nshots, nz=nz)
    t0 = time.perf_counter()
    b = MigrationBatch(ws, device=device, nstreams=nstreams)
    b.model_data()
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    cells = 2 * b.cells
    out = {"workload": f"config3 batched forward+imaging, {nshots} shots, nx=ny in 128-384, nz={ws[0].nz}, "
                       f"48-160 frequencies each, PSPI nref 6",
           "cell_steps": cells, "nstreams": len(b.streams), "setup_s": setup_s}

    def once(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    b.run_plain()                      # warm-up
    t_plain = once(b.run_plain)
    t_streams = once(b.run_streams)
    t1 = time.perf_counter()
    b.capture()
    out["graph_capture_s"] = time.perf_counter() - t1
    b.run_graph()                      # warm-up (graph upload)
    t_graph = once(b.run_graph)
    for k, t in (("plain", t_plain), ("streams", t_streams), ("graph", t_graph)):
        out[k + "_gcell_steps_per_s"] = cells / t / 1e9
        out[k + "_s"] = t
    out["graph_over_plain"] = t_plain / t_graph
    del b
    torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------------------- CPU arm

class CpuBorn:
    """FP32 CPU restatement (the oracle in complex64, scipy.fft on all host threads)
    of one Born forward + adjoint on a slab of the workload: nz_s depth levels and
    nw_s frequencies at full lateral size."""

    def __init__(self, nz_s=2, nw_s=16):
        from oracle import wem
        from pyfwix_b200 import workloads

        self.wem = wem
        w = workloads.config2(nz=nz_s, nw=nw_s)
        self.w = w
        g = wem.Grid(nx=w.nx, ny=w.ny, nw=w.nw, nz=w.nz, dx=w.dx, dy=w.dy, dz=w.dz, ow=w.ow, dw=w.dw,
                     nref=w.nref, taperx=w.taperx, tapery=w.tapery, eps_scat=w.eps_scat, taylor=w.taylor,
                     dtype=np.complex64)
        s2 = w.slow2.astype(np.float64)
        s = np.sqrt(s2)
        q = (np.arange(w.nref) * 2 + 1) / (2 * w.nref)
        sref = np.empty((w.nz, w.nref, w.nw), np.complex64)
        labels = np.empty((w.nz, w.nw, w.ny, w.nx), np.int64)
        for iz in range(w.nz):
            c = np.quantile(s[iz], q) ** 2
            sref[iz] = c[:, None]
            labels[iz] = np.argmin(np.abs(s2[iz][..., None] - c), axis=-1)[None]
        self.slow = np.broadcast_to(s2[:, None], (w.nz, w.nw, w.ny, w.nx)).astype(np.complex64)
        self.den = np.ones_like(self.slow)
        self.g, self.st = g, wem.Stepper(g, sref, labels, w.step)
        self.acq = wem.make_acquisition(g, w.geom)
        self.cores = os.cpu_count() or 1
        wem.set_fft_workers(self.cores)
        try:
            _, self.bgd, self.bgu = wem.propagate(g, self.st, self.acq, self.slow, self.den, w.wavelet)
        finally:
            wem.set_fft_workers(None)
        self.ds = np.broadcast_to(w.dslow[:, None], self.slow.shape).astype(np.complex64)
        self.dr = np.zeros_like(self.ds)
        self.cells = 2 * w.nx * w.ny * w.nw * w.nz

    def step(self):
        wem = self.wem
        wem.set_fft_workers(self.cores)
        try:
            t0 = time.perf_counter()
            d = wem.born_forward(self.g, self.st, self.acq, self.slow, self.den, self.bgd, self.bgu, self.ds, self.dr)
            wem.born_adjoint(self.g, self.st, self.acq, self.slow, self.den, self.bgd, self.bgu,
                             d.astype(np.complex64))
            return time.perf_counter() - t0
        finally:
            wem.set_fft_workers(None)

    def describe(self, value):
        w = self.w
        return {"value": value, "unit": "Gcell-steps/s", "cores": self.cores, "kind": "port",
                "sample": f"Born fwd+adj on a {w.nz}-level x {w.nw}-frequency slab at {w.nx}x{w.ny} "
                          f"(complex64 oracle port, scipy.fft workers={self.cores})"}


def cpu_baseline():
    c = CpuBorn()
    t = c.step()
    return c.describe(c.cells / t / 1e9)


def run_reference(a):
    ws, rank, local = dist()
    if rank != 0:
        return
    c = CpuBorn(nz_s=2, nw_s=8)
    for _ in range(max(a.warmup, 0)):
        c.step()
    ts = [c.step() for _ in range(a.steps)]
    t = float(np.mean(ts))
    v = c.cells / t / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Gcell-steps/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded)",
            "config": {"workload": "born-nsps-256x256x200-nw128 (CPU sample: 2 levels x 8 frequencies)",
                       "global_batch": 1, "parallelism": "host threads"},
            "cpu_baseline": c.describe(v),
            "e2e": {"value": v, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- main

def profile_step(a):
    """One depth step on the workload's wavefield (random data), nothing else:
    the launch a kernel profiler captures."""
    import torch

    from pyfwix_b200 import _lib as L
    from pyfwix_b200 import refsampler, workloads
    from pyfwix_b200.plan import Plan
    torch.cuda.set_device(0)
    if a.profile_step.startswith("smooth"):
        # one differentiable step of the FWI workload (384 x 384 x 96, true model, depth 1)
        from pyfwix_b200.fwi import SmoothFWI
        w, s_true, _ = workloads.config4(nz=2)
        par = dict(nref=w.nref, padx=0, pady=0, taperx=w.taperx, tapery=w.tapery, eps=0.0, ox=w.ox, oy=w.oy,
                   oz=w.oz, dx=w.dx, dy=w.dy, dz=w.dz, ow=w.ow, dw=w.dw, checkpoint=None)
        prob = SmoothFWI(s_true.shape, w.geom, torch.as_tensor(w.wavelet).cuda(), par, device="cuda")
        prob.set_slowness(torch.as_tensor(s_true))
        x = torch.randn(prob.plan.wshape, dtype=torch.complex64, device="cuda")
        mode = {"smooth": L.SMOOTH_FWD, "smooth-adj": L.SMOOTH_ADJ}[a.profile_step]
        prob.plan.smooth_step(1, x, torch.empty_like(x), mode=mode)
        torch.cuda.synchronize()
        print(json.dumps({"profile_step": a.profile_step, "workload": w.name, "ok": True}))
        return
    if a.profile_n:
        # a step of another lateral size: config1-family velocity with 5 % seeded noise
        n, nw = a.profile_n, a.profile_nw
        w = workloads.Workload(name=f"step-{n}x{n}-nw{nw}-nref{a.profile_nref}", nx=n, ny=n, nz=2, dx=10.0,
                               dy=10.0, dz=10.0, nw=nw, ow=3.0, dw=27.0 / max(nw - 1, 1), nref=a.profile_nref,
                               step="pspi")
        rng = np.random.default_rng(1000 + n)
        v = (1500.0 + 0.5 * 10.0 * np.arange(2))[:, None, None] * (1 + 0.05 * rng.random((2, n, n)))
        w.slow2 = (1.0 / v ** 2).astype(np.float32)
    else:
        w = workloads.CONFIGS[a.config](nz=2)
    kind, adj = a.profile_step.split("-")[0], a.profile_step.endswith("-adj")
    kw = w.plan_kwargs()
    kw["step"] = kind
    plan = Plan(ns=1, device="cuda", **kw)
    s2 = torch.as_tensor(w.slow2)[:, None].cuda()
    sref, labels = refsampler.sample(s2, w.nref, w.padx, w.pady)
    plan.set_refs(refsampler.expand_refs(sref, w.nw), labels)
    x = torch.randn(plan.wshape, dtype=torch.complex64, device="cuda")
    plan.step(0, x, x, direction=L.ADJ_INPL if adj else L.FWD)
    torch.cuda.synchronize()
    print(json.dumps({"profile_step": a.profile_step, "workload": w.name, "ok": True}))


def large_born(a):
    """The fifth configuration's size on one GPU (512 x 512 x 400, 200 frequencies,
    PSPI nref 8, one shot): modelling and one Born forward + adjoint with the
    backgrounds and the per-level recursion fields in the packed store, which is
    what makes the shot fit (lossless storage would take three times 400
    wavefields of 419 MB).  Prints one JSON line with the times and the memory."""
    import torch

    from pyfwix_b200 import _lib as L
    from pyfwix_b200 import refsampler, workloads
    from pyfwix_b200.plan import Plan
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    w = workloads.config5(nz=a.nz)
    t0 = time.perf_counter()
    p = Plan(ns=1, device=dev, **w.plan_kwargs())
    s2 = workloads.slow2_on(w, dev)[:, None]
    sref, labels = refsampler.sample(s2, w.nref, w.padx, w.pady)
    p.set_refs(refsampler.expand_refs(sref, w.nw), labels)
    s2c = s2.to(torch.complex64)
    p.set_model(s2c, torch.ones_like(s2c))
    del s2, sref
    p.ensure_workspace(L.WS_BORN_PACKED)
    g = w.geom
    src = p.traces(g["sx"], g["sy"], g["sz"], np.zeros(1, np.int32))
    rec = p.traces(g["rx"], g["ry"], g["rz"], np.zeros(len(g["rx"]), np.int32))
    wav = torch.as_tensor(w.wavelet).to(dev)
    data = torch.empty((len(g["rx"]), w.nw), dtype=torch.complex64, device=dev)
    pd, pu = p.packed(w.nz), p.packed(w.nz)
    ds = torch.zeros((w.nz, 1, w.ny, w.nx), dtype=torch.complex64, device=dev)
    rng = np.random.default_rng(1004)
    levels = np.arange(min(10, w.nz // 4), max(w.nz - 10, w.nz // 4 + 1))
    for iz in rng.choice(levels, size=min(8, len(levels)), replace=False):
        ds[iz] = s2c[iz] * float(rng.uniform(-0.1, 0.1))
    dr = torch.zeros_like(ds)
    gs, gr = torch.empty_like(ds), torch.empty_like(ds)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    p.propagate_packed(src, rec, wav, data, pd, pu)
    ev[1].record()
    p.born_packed(rec, pd, pu, ds, dr, data)
    ev[2].record()
    p.born_packed(rec, pd, pu, gs, gr, data, adjoint=True)
    ev[3].record()
    torch.cuda.synchronize()
    t = [ev[i].elapsed_time(ev[i + 1]) / 1e3 for i in range(3)]
    cells = w.nx * w.ny * w.nw * w.nz
    wb = 8 * w.nx * w.ny * w.nw
    assert torch.isfinite(gs).all()
    print(json.dumps({"large_born": {
        "workload": w.name + ("" if a.nz is None else f" (nz={w.nz})"), "modelling_s": t[0], "born_forward_s": t[1],
        "born_adjoint_s": t[2], "born_gcell_steps_per_s": 2 * cells / (t[1] + t[2]) / 1e9,
        "modelling_gcell_steps_per_s": 2 * cells / t[0] / 1e9, "setup_s": setup_s,
        "peak_device_gb": torch.cuda.max_memory_allocated(dev) / 1e9,
        "stored_fields_gb": (2 * pd.numel() + w.nz * p.packed_bytes) / 1e9,
        "lossless_fields_gb": 3 * w.nz * wb / 1e9}}), flush=True)


def main():
    a = args_()
    if a.large:
        large_born(a)
        return
    if a.impl == "reference":
        run_reference(a)
        return
    if a.profile_step:
        profile_step(a)
        return
    import torch
    ws, rank, local = dist()
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        barrier = lambda: tdist.barrier(device_ids=[local])
    else:
        torch.cuda.set_device(0)
        barrier = lambda: None
    device = torch.device("cuda", torch.cuda.current_device())
    from pyfwix_b200 import workloads
    w = workloads.CONFIGS[a.config](nz=a.nz)
    st = setup_born(w, device, autotune=not a.no_autotune,
                    tuning=parse_tuning(a.tuning) if a.tuning else None)
    for _ in range(a.warmup):
        born_step(st)
    torch.cuda.synchronize()
    from pyfwix_b200 import _lib
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    n0 = _lib.load().fwix_launch_count()
    t = time_steps(lambda: born_step(st), a.steps, barrier)
    launches = int(_lib.load().fwix_launch_count() - n0)
    clk = clocks.stop()
    if ws > 1:
        tt = torch.tensor([t], device=device)
        tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
        t = float(tt.item())
    cells = 2 * w.nx * w.ny * w.nw * w.nz
    value = ws * cells * a.steps / t / 1e9
    # roofline of the depth step
    tstep = step_roofline(st, w)
    cells_step = w.nx * w.ny * w.nw
    peak, peak_kind = measured_peak()
    achieved = ALG_BYTES_PER_CELL_STEP * cells_step / tstep / 1e9
    traffic = profiled_traffic(TRAFFIC_PROFILE) if (w.nx, w.nw) == (256, 128) else None
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_kind,
            "traffic_source": ("profiles/" + TRAFFIC_PROFILE + ": ncu DRAM bytes of the same step's launches, "
                               "captured separately (a profiler cannot run inside the timed bench)")
            if traffic is not None else None,
            "kernel": "NSPS depth step (row pass + column pass + row pass), 256x256x128",
            "step_ms": tstep * 1e3, "alg_bytes_per_cell_step": ALG_BYTES_PER_CELL_STEP}
    # the FP32 arithmetic the same step needs (the bound that applies: nref + 1
    # complex 2D transforms of 5 log2(NX NY) flop per sample, and a complex
    # multiply-add of the phase factor per reference), against the FP32 issue rate
    # of 148 SMs x 128 lanes x 2 flop at the sampled SM clock
    flop = (w.nref + 1) * 5 * math.log2(w.nx * w.ny) + 8 * w.nref
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    fp32 = flop * cells_step / tstep / 1e12
    roof["fp32"] = {"flop_per_cell_step": flop, "achieved_tflops": fp32, "peak_tflops": fp32_peak,
                    "frac": fp32 / fp32_peak, "peak_source": f"nominal at the sampled {mhz:.0f} MHz"}
    bg_gb = st["bd"].numel() * 8 / 1e9
    tuning = st["tuning"]
    packed = born_packed_timing(st, w) if not a.no_packed else None
    fwi = batched = None
    del st
    torch.cuda.empty_cache()
    # end to end through the drop-in surface with host arrays
    e2e = None
    if not a.no_e2e:
        def reduce_max(te):
            if ws > 1:
                tt = torch.tensor([te], device=device)
                tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
                te = float(tt.item())
            return te
        su = setup_surface(w, device)
        born_step_e2e(su)
        te = reduce_max(time_steps(lambda: born_step_e2e(su), a.steps, barrier))
        e2e = {"value": ws * cells * a.steps / te / 1e9, "unit": "Gcell-steps/s", **e2e_bytes(su),
               "api": "pyfwix_b200.CudaWEM.ExtendedBorn forward + adjoint (False, model, data), numpy arrays "
                      "in pinned host memory",
               "model_layout": "[nz][1][ny][nx]: one perturbation per cell for every frequency (the "
                               "configuration's reflectivity is frequency-independent)"}
        del su
        torch.cuda.empty_cache()
        # the reference's per-frequency model domain [nz][nw][ny][nx] (13.4 GB per
        # component at this size), pageable numpy arrays as a caller passes them;
        # two steps, and only where the host has the memory for the four arrays
        need = 4 * w.nz * w.nw * w.ny * w.nx * 8
        if a.e2e_per_w and _host_available() > 2.5 * need:
            su = setup_surface(w, device, per_w=True, pinned=False)
            born_step_e2e(su)
            k = 2
            te = reduce_max(time_steps(lambda: born_step_e2e(su), k, barrier))
            e2e["per_frequency_model"] = {
                "value": ws * cells * k / te / 1e9, "unit": "Gcell-steps/s", "steps": k, **e2e_bytes(su),
                "model_layout": "[nz][nw][ny][nx] (the reference's ExtendedBorn domain), pageable numpy arrays"}
            del su
            torch.cuda.empty_cache()
        elif a.e2e_per_w:
            e2e["per_frequency_model"] = {"skipped": f"host memory: {_host_available() / 1e9:.0f} GB available, "
                                                     f"{2.5 * need / 1e9:.0f} GB wanted"}
    if not a.no_fwi:
        fwi = fwi_gradient_timing(device, nz=a.fwi_nz)
        # the configuration's depth checkpoints (every 16th level, segments recomputed)
        k16 = fwi_gradient_timing(device, nz=a.fwi_nz, checkpoint=16)
        fwi["checkpoint_16"] = {k: k16[k] for k in ("s_per_shot", "forward_s_per_shot", "gradient_s_per_shot",
                                                    "grad_over_forward", "checkpoint")}
        sh = fwi_shots_timing(device, ws, rank, barrier, nz=a.fwi_nz)
        if ws > 1:
            tt = torch.tensor([sh["s"]], device=device)
            tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
            sh["s"] = float(tt.item())
        sh["shots_per_s"] = ws / sh["s"]
        fwi["shots_across_ranks"] = sh
        from pyfwix_b200.fwi import clear_plan_cache
        clear_plan_cache()  # the FWI plan's phase cache is not needed by the timings below
        torch.cuda.empty_cache()
    config1 = config1_timing(device, autotune=not a.no_autotune) if not a.no_config1 else None
    if ws == 1 and not a.no_batched:
        batched = batched_timing(device, nshots=a.batched_shots, nz=a.batched_nz, nstreams=a.batched_streams)
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu:
        cpu = cpu_baseline()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Gcell-steps/s", "n_gpus": ws, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": t / a.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded)",
                "config": {"workload": w.name + ("" if a.nz is None else f" (nz={w.nz})"),
                           "global_batch": ws, "seq_len": None, "parallelism": f"shot replicas x{ws}",
                           "l2": "inputs larger than L2 (background wavefields 2 x %.1f GB)"
                                 % bg_gb},
                "gpu_launches": launches, "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
                "fwi_grad": fwi, "batched": batched, "born_packed_backgrounds": packed, "config1": config1,
                "tuning": tuning}
        print(json.dumps(line), flush=True)
    if ws > 1:
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
