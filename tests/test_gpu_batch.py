"""Batched forward + imaging of shots with uneven grids and bands
(pyfwix_b200/batch.py): every instance's data and image against the FP64
oracle (Propagator.cpp:121-221 modelling, lockstep migration image), and the
three execution modes -- shot after shot, over CUDA streams, replayed from one
captured CUDA graph -- giving the same images (to the rounding of their
frequency sums, which float atomics add in no fixed order)."""
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
            # images are summed over frequency by float atomics: order-dependent rounding
            assert rel(im.cpu().numpy(), ref.cpu().numpy()) < 1e-6


def _acq_plan(seed, nx, ny, nw, nz, kind, pad=4):
    from tests.gpu_helpers import make_case, make_plan
    g, rng, sref, labels, slow, den = make_case(seed=seed, nx=nx, ny=ny, nw=nw, nz=nz, nref=3, padx=pad, pady=pad)
    slow = slow.copy()
    slow[nz - 2:] *= 1.7
    p = make_plan(g, 1, sref, labels, slow, den, step=kind)
    geom = dict(sx=[nx * 5.0], sy=[ny * 6.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, (nx - 1) * 10.0, 9)),
                ry=[ny * 6.0] * 9, rz=[0.0] * 9, r_ids=[0] * 9)
    src = p.traces(geom["sx"], geom["sy"], geom["sz"], [0])
    rec = p.traces(geom["rx"], geom["ry"], geom["rz"], [0] * 9)
    wav = torch.as_tensor(crandn(rng, (1, nw)).astype(np.complex64)).cuda()
    return g, rng, p, src, rec, wav


def test_sweep_kinds_match_single_calls():
    """fwix_sweep over three instances of different sizes, on two streams, gives
    bit for bit what each instance's own sweep call gives, for every kind."""
    from pyfwix_b200 import _lib as L
    from pyfwix_b200.plan import sweep
    cases = [_acq_plan(1, 32, 24, 3, 5, "pspi"), _acq_plan(2, 44, 36, 4, 5, "nsps"), _acq_plan(3, 64, 64, 2, 5, "pspi", 0)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    # down / up, forward and adjoint, in place
    for kind, fn in ((L.SWEEP_DOWN, "downward"), (L.SWEEP_UP, "upward")):
        for adj in (0, 1):
            xs = [torch.as_tensor(crandn(rng, (1, g.nw, g.NY, g.NX)).astype(np.complex64)).cuda()
                  for g, rng, *_ in cases]
            ref = [getattr(p, fn)(x.clone(), adjoint=bool(adj)) for (g, rng, p, *_), x in zip(cases, xs)]
            sweep(kind, [dict(plan=c[2], wfld=x, adjoint=adj) for c, x in zip(cases, xs)], streams)
            torch.cuda.synchronize()
            for a, b in zip(xs, ref):
                assert torch.equal(a, b)
    # modelling with stored fields, then Born forward / adjoint and the image
    outs, refs = [], []
    for g, rng, p, src, rec, wav in cases:
        mk = lambda: dict(data=torch.zeros((9, g.nw), dtype=torch.complex64, device="cuda"),
                          bg_down=torch.zeros((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda"),
                          bg_up=torch.zeros((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda"))
        o, r = mk(), mk()
        p.propagate(src, rec, wav, r["data"], r["bg_down"], r["bg_up"])
        outs.append(dict(plan=p, src=src, rec=rec, wavelet=wav, **o))
        refs.append(r)
    sweep(L.SWEEP_MODEL, outs, streams)
    torch.cuda.synchronize()
    for o, r in zip(outs, refs):
        for k in ("data", "bg_down", "bg_up"):
            assert torch.equal(o[k], r[k])
    born_in, born_ref = [], []
    for (g, rng, p, src, rec, wav), o in zip(cases, outs):
        ds = torch.as_tensor(crandn(rng, (g.nz, g.nw, g.ny, g.nx)).astype(np.complex64)).cuda()
        dr = torch.as_tensor(crandn(rng, (g.nz, g.nw, g.ny, g.nx)).astype(np.complex64)).cuda()
        d = torch.empty((9, g.nw), dtype=torch.complex64, device="cuda")
        p.born(rec, o["bg_down"], o["bg_up"], ds, dr, d)
        born_ref.append(d)
        born_in.append(dict(plan=p, rec=rec, bg_down=o["bg_down"], bg_up=o["bg_up"], dslow=ds, dden=dr,
                            data=torch.empty_like(d)))
    sweep(L.SWEEP_BORN_FWD, born_in, streams)
    torch.cuda.synchronize()
    for b, r in zip(born_in, born_ref):
        assert torch.equal(b["data"], r)
    for b in born_in:
        gs, gr = torch.empty_like(b["dslow"]), torch.empty_like(b["dslow"])
        b["plan"].born(b["rec"], b["bg_down"], b["bg_up"], gs, gr, b["data"], adjoint=True)
        b["ref"] = (gs, gr)
        b["dslow"], b["dden"] = torch.empty_like(gs), torch.empty_like(gs)
    sweep(L.SWEEP_BORN_ADJ, born_in, streams)
    torch.cuda.synchronize()
    for b in born_in:
        assert torch.equal(b["dslow"], b["ref"][0]) and torch.equal(b["dden"], b["ref"][1])
    with pytest.raises(L.FwixError):
        sweep(L.SWEEP_DOWN, [dict(plan=cases[0][2], wfld=xs[0]), dict(plan=cases[0][2], wfld=xs[0])], streams)


def test_one_call_steps_and_image_accumulate():
    """fwix_pspi_step / fwix_nsps_step equal fwix_step with the same direction, and
    fwix_image_accumulate equals the frequency-summed correlation."""
    import ctypes
    from pyfwix_b200 import _lib as L
    lib = L.load()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for kind, fn in (("pspi", lib.fwix_pspi_step), ("nsps", lib.fwix_nsps_step)):
        g, rng, p, src, rec, wav = _acq_plan(4, 36, 28, 3, 3, kind)
        p.ensure_workspace(L.WS_STEP)
        x = torch.as_tensor(crandn(rng, p.wshape).astype(np.complex64)).cuda()
        for adj in (0, 1, 2):
            out = torch.empty_like(x)
            L.check(fn(p._h, 1, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), adj, s))
            ref = p.step(1, x, torch.empty_like(x), direction=adj)
            torch.cuda.synchronize()
            assert torch.equal(out, ref)
    y = torch.as_tensor(crandn(rng, p.wshape).astype(np.complex64)).cuda()
    img = torch.zeros((g.ny, g.nx), dtype=torch.float32, device="cuda")
    L.check(lib.fwix_image_accumulate(p._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                      ctypes.c_void_p(img.data_ptr()), 0, s))
    torch.cuda.synchronize()
    want = (x.conj() * y)[:, :, :g.ny, :g.nx].real.sum(dim=(0, 1))
    assert rel(img.cpu().numpy(), want.cpu().numpy()) < 1e-5
