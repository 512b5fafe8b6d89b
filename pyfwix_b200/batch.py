"""Many independent shots of uneven aperture and frequency band, forward-continued
and imaged together on one GPU.

Every shot is its own instance: its own grid (nx, ny), band (ow, dw, nw),
references and labels, plan and workspace -- the per-instance descriptor is the
plan.  The reference runs such a batch as ``StreamingPropagator`` instances on
TBB threads, one CUDA stream each (``propagator/src/StreamingPropagator.cpp``),
and images each shot with ``ExtendedBorn``'s imaging condition
(``propagator/src/imaging_condition.cu:9-108``).  Here the instances are
spread over a fixed set of CUDA streams by ``fwix_sweep`` (largest first, each
to the stream with the least work queued), so the kernels of small shots fill
the SMs that large ones leave idle, and the whole batch -- every instance's depth loop -- can be
captured once into one CUDA graph and replayed, which takes the host out of
the loop: one graph launch per batch instead of ~10 kernel launches per depth
and shot.

Per shot the work is ``fwix_migrate``: source and receiver wavefields
continued in lockstep over all depths and the image
I[z][y][x] += sum_w Re(conj(S) R) accumulated at every level.  The results do
not depend on the mode (plain, streams or graph): each instance's kernels run
in the same order on its own buffers.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from . import refsampler
from .plan import Plan, sweep


class Instance:
    """One shot: plan, traces, wavelet, recorded data and image."""

    def __init__(self, w, device, slow2, autotune=True):
        self.w = w
        self.plan = Plan(ns=1, device=device, **w.plan_kwargs())
        p = self.plan
        s2 = slow2[:, None]                                                  # [nz][1][ny][nx]
        sref, labels = refsampler.sample(s2, w.nref, w.padx, w.pady)
        p.set_refs(refsampler.expand_refs(sref, w.nw), labels, phase_cache=False)
        # one depth of phase factors, shared by the source and receiver steps of a level
        p.enable_phase_cache(depths=1)
        s2c = s2.to(torch.complex64)
        p.set_model(s2c, torch.ones_like(s2c))
        g = w.geom
        self.src = p.traces(g["sx"], g["sy"], g["sz"], np.zeros(len(g["sx"]), np.int32))
        self.rec = p.traces(g["rx"], g["ry"], g["rz"], np.zeros(len(g["rx"]), np.int32))
        self.wavelet = torch.as_tensor(w.wavelet).to(device)
        self.data = torch.zeros((len(g["rx"]), w.nw), dtype=torch.complex64, device=device)
        self.image = torch.zeros((w.nz, w.ny, w.nx), dtype=torch.float32, device=device)
        p.ensure_workspace(L.WS_SWEEP)
        # per instance, the fastest equivalent form of its depth step (column tile
        # movement, slices per launch) for its own grid and band
        self.tuning = p.autotune() if autotune else None

    @property
    def cells(self):
        w = self.w
        return w.nx * w.ny * w.nw * w.nz

    def model_data(self):
        """Recorded data of this shot (down pass, reflection, up pass).  The up pass
        reflects the down field of every depth, so the down fields are held for the
        duration of the call ([nz] wavefields, released afterwards)."""
        p = self.plan
        down = torch.empty((p.nz,) + p.wshape, dtype=torch.complex64, device=p.device)
        p.propagate(self.src, self.rec, self.wavelet, self.data, down, None)
        torch.cuda.current_stream(p.device).synchronize()
        del down

    def migrate(self):
        self.plan.migrate(self.src, self.rec, self.wavelet, self.data, self.image)


class MigrationBatch:
    """Forward + imaging of a list of single-shot workloads (``workloads.config3``)."""

    def __init__(self, workloads, device=None, nstreams=8, slow2_fn=None):
        self.device = torch.device(device if device is not None else "cuda")
        if slow2_fn is None:
            from .workloads import slow2_on as slow2_fn
        with torch.cuda.device(self.device):
            self.inst = [Instance(w, self.device, slow2_fn(w, self.device)) for w in workloads]
            self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, int(nstreams)))]
        self.graph = None

    @property
    def cells(self):
        """x*y*w*z cell-steps of one sweep over all shots."""
        return sum(i.cells for i in self.inst)

    def model_data(self):
        for i in self.inst:
            i.model_data()

    # -------------------------------------------------------------- execution
    def run_plain(self):
        """Shot after shot on the current stream (the per-shot path)."""
        for i in self.inst:
            i.migrate()

    def _enqueue_streams(self):
        # fwix_sweep assigns the instances (largest first onto the least loaded
        # stream) and forks / joins them on the caller's stream
        sweep(L.SWEEP_IMAGE, [dict(plan=i.plan, src=i.src, rec=i.rec, wavelet=i.wavelet, data=i.data,
                                   image=i.image) for i in self.inst], self.streams)

    def run_streams(self):
        """All shots at once over the streams, joined back into the current stream."""
        self._enqueue_streams()

    def capture(self):
        """Captures the streamed batch into one CUDA graph (each call records its
        kernels; nothing runs).  Returns the graph."""
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            self._enqueue_streams()
        torch.cuda.synchronize(self.device)
        self.graph = g
        return g

    def run_graph(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def zero_images(self):
        for i in self.inst:
            i.image.zero_()

    def images(self):
        return [i.image for i in self.inst]
