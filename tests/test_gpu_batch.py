"""Batched forward + imaging of shots with uneven grids and bands
(pyfwix_b200/batch.py): every instance's data and image against the FP64
oracle (Propagator.cpp:121-221 modelling, lockstep migration image), and the
three execution modes -- shot after shot, over CUDA streams, replayed from one
captured CUDA graph -- giving identical images."""
import numpy as np
import pytest
import torch

from oracle import wem
from tests.conftest import crandn
from tests.gpu_helpers import oracle_labels, rel

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _tiny_workloads():
    from pyfwix_b200 import workloads as W
    rng = np.random.default_rng(3)
    out = []
    for i, (n, nw, ow) in enumerate([(32, 4, 3.0), (48, 3, 5.0), (64, 5, 2.0), (40, 4, 4.0), (32, 3, 6.0)]):
        w = W.Workload(name=f"t{i}", nx=n, ny=n, nz=6, dx=10.0, dy=10.0, dz=10.0, nw=nw, ow=ow, dw=2.5, nref=3,
                       step="pspi", taperx=3, tapery=3)
        w.anomaly = (n * 5.0 + 7.0 * i, n * 4.0, 30.0)
        w.geom = dict(sx=np.array([n // 2 * w.dx], np.float32), sy=np.array([n // 3 * w.dy], np.float32),
                      sz=np.array([0.0], np.float32), s_ids=np.array([0], np.int32), **w.surface_receivers())
        w.wavelet = crandn(rng, (1, nw)).astype(np.complex64)
        out.append(w)
    return out


def _oracle(inst):
    w, p = inst.w, inst.plan
    g = wem.Grid(nx=w.nx, ny=w.ny, nw=w.nw, nz=w.nz, dx=w.dx, dy=w.dy, dz=w.dz, ow=w.ow, dw=w.dw, nref=w.nref,
                 taperx=w.taperx, tapery=w.tapery)
    sref = p._keep["sref"].cpu().numpy().astype(np.complex128)
    st = wem.Stepper(g, sref, oracle_labels(p._keep["labels"].cpu().numpy(), g), w.step)
    acq = wem.make_acquisition(g, w.geom)
    return g, st, acq


def test_batch_modes_and_oracle():
    from pyfwix_b200.batch import MigrationBatch
    from pyfwix_b200.workloads import slow2_on
    ws = _tiny_workloads()
    b = MigrationBatch(ws, nstreams=2)
    assert sorted(i for lane in b.assign for i in lane) == list(range(len(ws)))
    b.model_data()
    b.run_plain()
    torch.cuda.synchronize()
    plain = [im.clone() for im in b.images()]
    for inst, im in zip(b.inst, plain):
        g, st, acq = _oracle(inst)
        s2 = slow2_on(inst.w, "cpu").double().numpy()
        slow = np.repeat(s2[:, None], g.nw, axis=1).astype(np.complex128)
        data, _, _ = wem.propagate(g, st, acq, slow, np.ones_like(slow), inst.w.wavelet.astype(np.complex128))
        assert rel(inst.data.cpu().numpy(), data) < TOL
        img = wem.migrate(g, st, acq, inst.w.wavelet.astype(np.complex128), inst.data.cpu().numpy())
        assert rel(im.cpu().numpy(), img) < TOL
    for run in (b.run_streams, b.run_graph, b.run_graph):
        b.zero_images()
        run()
        torch.cuda.synchronize()
        for im, ref in zip(b.images(), plain):
            assert torch.equal(im, ref)
