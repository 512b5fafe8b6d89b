"""Column passes with TMA tiles (``pyfwix_b200/csrc/tma.cuh``: cp.async.bulk.tensor
loads into swizzled shared-memory tiles on bounded mbarrier waits, TMA stores of
the results) against the per-thread copies they replace, and the runtime
autotuner (``fwix_plan_autotune``).  Moving the tiles differently changes no
arithmetic, so the steps agree to the last bit; no bounded wait may run out."""
import numpy as np
import pytest
import torch

from oracle import wem
from tests.gpu_helpers import make_case, make_plan, oracle_labels, rel, to_dev, to_host, wavefield

pytestmark = pytest.mark.gpu


def _plans(monkeypatch, step, qtile=3, **kw):
    g, rng, sref, labels, slow, den = make_case(**kw)
    monkeypatch.setenv("FWIX_COL_TMA", "0")
    p0 = make_plan(g, 1, sref, labels, slow, den, step=step)
    monkeypatch.setenv("FWIX_COL_TMA", "1")
    monkeypatch.setenv("FWIX_QTILE", str(qtile))
    p1 = make_plan(g, 1, sref, labels, slow, den, step=step)
    monkeypatch.delenv("FWIX_COL_TMA")
    monkeypatch.delenv("FWIX_QTILE")
    return g, rng, sref, labels, slow, den, p0, p1


# plan lengths whose column passes take 16 columns per CTA (128 bytes per tile row,
# 128-byte swizzle: 128 - 320) or 8 (64 bytes, 64-byte swizzle: 384 - 640); qtile 3:
# the phase factors arrive as TMA tiles too (both column passes, lengths whose
# quarter-spectrum rows fit one box: up to 510), 0: per lane
@pytest.mark.parametrize("n,pad", [(124, 4), (192, 0), (256, 0), (316, 4), (380, 4), (512, 0), (640, 0)])
@pytest.mark.parametrize("step", ["pspi", "nsps"])
@pytest.mark.parametrize("qtile", [0, 3])
def test_tma_steps_equal_copy_steps(monkeypatch, n, pad, step, qtile):
    from pyfwix_b200 import _lib as L
    g, rng, sref, labels, slow, den, p0, p1 = _plans(monkeypatch, step, qtile, nx=n, ny=n, nw=6, nz=3, nref=4,
                                                     padx=pad, pady=pad, eps=0.01, complex_refs=True)
    lab = oracle_labels(labels, g)
    st = wem.Stepper(g, sref, lab, step)
    for d in (L.FWD, L.ADJ_ADD, L.ADJ_INPL):
        x = to_dev(wavefield(rng, 1, g))
        y0 = p0.step(1, x, torch.empty_like(x), direction=d)
        y1 = p1.step(1, x, torch.empty_like(x), direction=d)
        torch.cuda.synchronize()
        assert torch.equal(y0, y1), (step, d, rel(to_host(y1), to_host(y0)))
    # and against the oracle once (forward)
    x = wavefield(rng, 1, g)
    y = to_host(p1.step(1, to_dev(x), to_dev(np.zeros_like(x))))
    assert rel(y, st.fwd(1, x)) < 1e-5
    assert int(p1.lib.fwix_plan_wait_timeouts(p1._h)) == 0


def test_tma_born_equals_copy_born(monkeypatch):
    """Whole ExtendedBorn forward + adjoint (scatter passes included) at 256 x 256."""
    g, rng, sref, labels, slow, den, p0, p1 = _plans(monkeypatch, "nsps", nx=256, ny=256, nw=4, nz=4, nref=3)
    geom = dict(sx=[1280.0], sy=[1500.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, 2500, 16)),
                ry=[1200.0] * 16, rz=[0.0] * 16, r_ids=[0] * 16)
    outs = []
    for p in (p0, p1):
        src = p.traces(geom["sx"], geom["sy"], geom["sz"], [0])
        rec = p.traces(geom["rx"], geom["ry"], geom["rz"], [0] * 16)
        wav = torch.as_tensor(np.ones((1, g.nw), np.complex64)).cuda()
        bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
        bu = torch.empty_like(bd)
        d = torch.empty((16, g.nw), dtype=torch.complex64, device="cuda")
        p.propagate(src, rec, wav, d, bd, bu)
        ms = to_dev(np.random.default_rng(1).standard_normal((g.nz, g.nw, g.ny, g.nx)) * 1e-7)
        mr = torch.zeros_like(ms)
        out = torch.empty_like(d)
        p.born(rec, bd, bu, ms, mr, out)
        gs, gr = torch.empty_like(ms), torch.empty_like(ms)
        p.born(rec, bd, bu, gs, gr, out, adjoint=True)
        torch.cuda.synchronize()
        outs.append((out, gs, gr))
    for a, b in zip(*outs):
        assert torch.equal(a, b)


@pytest.mark.parametrize("n,step", [(256, "nsps"), (384, "pspi")])
def test_autotune_keeps_the_step(n, step):
    """The tuner times the candidates, keeps one, and the step it leaves gives the
    same output as before (all candidates are the same arithmetic)."""
    g, rng, sref, labels, slow, den = make_case(nx=n, ny=n, nw=8, nz=3, nref=4)
    p = make_plan(g, 1, sref, labels, slow, den, step=step)
    x = to_dev(wavefield(rng, 1, g))
    before = p.step(1, x, torch.empty_like(x))
    res = p.autotune(iz=1, reps=2)
    assert res["candidates"] >= 2 and res["step_ms"] > 0 and res["slices_per_launch"] >= 1
    after = p.step(1, x, torch.empty_like(x))
    torch.cuda.synchronize()
    assert rel(to_host(after), to_host(before)) < 1e-6
    assert int(p.lib.fwix_plan_wait_timeouts(p._h)) == 0


def test_set_tuning_applies_a_saved_choice():
    """fwix_plan_set_tuning: a second plan of the same sizes takes the first one's
    tuned choice without timing; its step equals the untuned step; out-of-range
    choices are refused."""
    from pyfwix_b200 import _lib as L
    g, rng, sref, labels, slow, den = make_case(nx=256, ny=256, nw=8, nz=3, nref=4)
    p = make_plan(g, 1, sref, labels, slow, den, step="nsps")
    q = make_plan(g, 1, sref, labels, slow, den, step="nsps")
    x = to_dev(wavefield(rng, 1, g))
    before = q.step(1, x, torch.empty_like(x))
    choice = p.autotune(iz=1, reps=2)
    q.set_tuning(choice)
    after = q.step(1, x, torch.empty_like(x))
    torch.cuda.synchronize()
    assert rel(to_host(after), to_host(before)) < 1e-6
    for bad in (dict(choice, slices_per_launch=0), dict(choice, streams=3),
                dict(choice, slices_per_launch=g.nw + 1)):
        with pytest.raises(RuntimeError):
            q.set_tuning(bad)
