"""Multi-rank shot distribution on CPU (gloo, world size 2): the cost-balanced
partition, and the objective / gradient summed by one all-reduce equals the
single-process sum over all shots.  The per-shot work is the FP64 oracle's
smooth-mode objective and gradient on a tiny grid (the sum over shots of the
per-shot gradients is the gradient of the total misfit)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from pyfwix_b200 import shots


def test_partition_balances_uneven_shots():
    costs = [shots.shot_cost(n, n, nw, 200) for n, nw in
             [(128, 48), (384, 160), (192, 96), (256, 64), (320, 120), (128, 160), (384, 48), (256, 100)]]
    parts = shots.partition(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert parts == shots.partition(costs, 3)             # deterministic
    assert shots.partition(costs, 1) == [list(range(len(costs)))]


def _shot_problem():
    from oracle import wem
    rng = np.random.default_rng(5)
    g = wem.Grid(nx=12, ny=10, nw=2, nz=3, dx=10, dy=10, dz=10, ow=6, dw=4, padx=4, pady=2, nref=2,
                 taperx=1, tapery=1)
    s = 1 / 1800 * (1 + 0.1 * rng.random((g.nz, g.ny, g.nx)))
    refs = wem.smooth_refs(s, g.nref)
    geoms, wavs, dobs = [], [], []
    for k in range(5):
        geom = dict(sx=[20.0 + 15 * k], sy=[40.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, 100, 6)),
                    ry=[50.0] * 6, rz=[0.0] * 6, r_ids=[0] * 6)
        acq = wem.make_acquisition(g, geom)
        wav = rng.standard_normal((1, g.nw)) + 1j * rng.standard_normal((1, g.nw))
        geoms.append(acq)
        wavs.append(wav)
        dobs.append(wem.smooth_propagate(g, refs, s * 1.03, acq, wav)[0])
    return g, s, refs, geoms, wavs, dobs


def _work_fn():
    from oracle import wem
    g, s, refs, acqs, wavs, dobs = _shot_problem()

    def work(i):
        J, grad = wem.smooth_gradient(g, refs, s, acqs[i], wavs[i], dobs[i])
        return J, torch.as_tensor(grad)
    return work, torch.zeros(s.shape, dtype=torch.float64)


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        work, like = _work_fn()
        J, g = shots.objective_and_gradient([1, 3, 2, 2, 1], work, like)
        out.put((rank, J, g.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_two_rank_gradient_equals_serial_sum():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    work, like = _work_fn()
    J_ref, g_ref = 0.0, np.zeros(like.shape)
    for i in range(5):
        Ji, gi = work(i)
        J_ref += Ji
        g_ref += gi.numpy()
    for rank, J, g in res:
        assert abs(J / J_ref - 1) < 1e-12
        assert np.allclose(g, g_ref, rtol=1e-12, atol=1e-300)


def _fwi_problem():
    """Five shots of a tiny smooth-mode FWI problem for the product entry point
    ``fwi.shot_objective_and_gradient``; the device plan is the oracle stand-in of
    ``tests/test_fwi_schedule.py`` (CPU, complex64 storage like the device)."""
    from oracle import wem
    g, s, refs, acqs, wavs, dobs = _shot_problem()
    shot_list = []
    for k in range(5):
        geom = dict(sx=[20.0 + 15 * k], sy=[40.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, 100, 6)),
                    ry=[50.0] * 6, rz=[0.0] * 6, r_ids=[0] * 6)
        shot_list.append(dict(geometry=geom, wavelet=torch.as_tensor(wavs[k]).to(torch.complex64),
                              d_obs=torch.as_tensor(dobs[k]).to(torch.complex64)))
    par = dict(nref=g.nref, padx=g.padx, pady=g.pady, taperx=g.taperx, tapery=g.tapery, eps=0.0, ox=0.0, oy=0.0,
               oz=0.0, dx=g.dx, dy=g.dy, dz=g.dz, ow=g.ow, dw=g.dw, checkpoint=None,
               refs=torch.as_tensor(refs, dtype=torch.float32))
    return torch.as_tensor(s, dtype=torch.float32), shot_list, par


def _fwi_rank(rank, world, port, out):
    import torch.distributed as dist
    from pyfwix_b200 import fwi
    from tests.test_fwi_schedule import OraclePlan
    fwi.Plan = OraclePlan
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s, shot_list, par = _fwi_problem()
        # this rank reads only its own shots' observed data
        mine = set(shots.partition([1] * len(shot_list), world)[rank])
        visible = [dict(sh, d_obs=sh["d_obs"] if i in mine else None) for i, sh in enumerate(shot_list)]
        J, g = fwi.shot_objective_and_gradient(s, visible, par, device="cpu")
        st = s.clone().requires_grad_(True)
        Ja = fwi.FWIShotsGradient.apply(st, visible, par)
        Ja.backward()
        out.put((rank, J, g.numpy(), float(Ja), st.grad.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_fwi_entry_point(monkeypatch):
    """The product's multi-shot FWI entry point on two gloo ranks: each rank runs
    its partition of the five shots and one all-reduce sums the objective and the
    gradient, equal to one process running every shot; the autograd wrapper gives
    the same gradient."""
    from pyfwix_b200 import fwi
    from tests.test_fwi_schedule import OraclePlan
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fwi_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    monkeypatch.setattr(fwi, "Plan", OraclePlan)
    s, shot_list, par = _fwi_problem()
    J_ref, g_ref = fwi.shot_objective_and_gradient(s, shot_list, par, device="cpu")
    assert J_ref > 0 and float(np.abs(g_ref.numpy()).max()) > 0
    for rank, J, g, Ja, ga in res:
        assert abs(J / J_ref - 1) < 1e-6
        assert np.allclose(g, g_ref.numpy(), rtol=1e-5, atol=1e-6 * np.abs(g_ref.numpy()).max())
        assert abs(Ja / J_ref - 1) < 1e-6
        assert np.allclose(ga, g_ref.numpy(), rtol=1e-5, atol=1e-6 * np.abs(g_ref.numpy()).max())
