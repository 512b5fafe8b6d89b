"""Background stores beyond device memory: packed backgrounds in pinned host
memory (read by the kernels over the host link), and the checkpoint files of
``pyfwix_b200.pool.WavefieldPool`` in the layout of the reference's
``WavefieldPool`` (``propagator/src/WavefieldPool.cpp:78-100``: one file per tag,
depth iz's fixed-size chunk at offset iz * chunk)."""
import os

import numpy as np
import pytest
import torch

from tests.conftest import crandn
from tests.gpu_helpers import make_case, make_plan, rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _setup(kind="pspi", nz=5):
    g, rng, sref, labels, slow, den = make_case(nx=32, ny=24, nw=4, nz=nz, nref=3, padx=4, pady=4)
    slow = slow.copy()
    slow[nz - 2:] *= 1.6
    p = make_plan(g, 1, sref, labels, slow, den, step=kind)
    geom = dict(sx=[150.0], sy=[120.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, 300, 12)), ry=[100.0] * 12,
                rz=[0.0] * 12, r_ids=[0] * 12)
    src = p.traces(geom["sx"], geom["sy"], geom["sz"], [0])
    rec = p.traces(geom["rx"], geom["ry"], geom["rz"], [0] * 12)
    wav = to_dev(crandn(rng, (1, g.nw)))
    return g, rng, p, src, rec, wav, slow, den, geom


def test_host_packed_backgrounds_equal_device_packed():
    g, rng, p, src, rec, wav, *_ = _setup()
    res = []
    for host in (False, True):
        pd, pu = p.packed(g.nz, host=host), p.packed(g.nz, host=host)
        assert pd.is_pinned() == host
        d = torch.empty((12, g.nw), dtype=torch.complex64, device="cuda")
        p.propagate_packed(src, rec, wav, d, pd, pu)
        ms = to_dev(np.random.default_rng(3).standard_normal((g.nz, g.nw, g.ny, g.nx)) * 1e-8)
        mr = torch.zeros_like(ms)
        out = torch.empty_like(d)
        p.born_packed(rec, pd, pu, ms, mr, out)
        gs, gr = torch.empty_like(ms), torch.empty_like(ms)
        p.born_packed(rec, pd, pu, gs, gr, out, adjoint=True)
        # the stored bytes (each field's zero tail up to 256 bytes included) and the fields they unpack to
        fields = torch.stack([p.unpack(pd[iz].cuda(), torch.empty(p.wshape, dtype=torch.complex64, device="cuda"))
                              for iz in range(g.nz)])
        torch.cuda.synchronize()
        res.append((d.clone(), pd.cpu(), fields, out.clone(), gs.clone(), gr.clone()))
    for a, b in zip(*res):
        assert torch.equal(a.cpu(), b.cpu())


@pytest.mark.parametrize("packed", [True, False])
def test_pool_files_in_the_reference_layout(tmp_path, packed):
    from pyfwix_b200.pool import WavefieldPool
    g, rng, p, src, rec, wav, *_ = _setup()
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((12, g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, wav, d, bd, bu)
    par = dict(wfld_path=str(tmp_path), wflds_to_store=2, **({"compress_rate": 8} if packed else {}))
    pool = WavefieldPool(p, par, "run0", g.nz)
    pool.store(bd, "down")
    pool.store(bu, "up")
    pool.wait_to_finish()
    chunk = p.packed_bytes if packed else bd[0].numel() * 8
    assert pool.chunk == chunk and pool.get_total_compressed_size() == 2 * g.nz * chunk
    f = os.path.join(str(tmp_path), "run0", "checkpoints_down.bin")
    assert os.path.getsize(f) == g.nz * chunk
    raw = np.fromfile(f, dtype=np.uint8)
    for iz in (0, g.nz - 1):
        want = p.pack(bd[iz], p.packed(1)[0]) if packed else bd[iz].reshape(-1).view(torch.uint8)
        assert np.array_equal(raw[iz * chunk:(iz + 1) * chunk], want.cpu().numpy())
    # read back: one depth, and every depth
    one = torch.empty(p.wshape, dtype=torch.complex64, device="cuda")
    pool.decompress_slice(2, "up", one)
    ref = p.unpack(p.pack(bu[2], p.packed(1)[0]), torch.empty_like(one)) if packed else bu[2]
    torch.cuda.synchronize()
    assert torch.equal(one, ref)
    allu = pool.load("up")
    if not packed:
        assert torch.equal(allu, bu)
    pool.close()


def test_surface_host_store_and_restart_from_files(tmp_path):
    """Propagator with compress_rate 8, the host store and checkpoint files; a
    second Propagator reads the files back (load_backgrounds) instead of
    modelling, and its ExtendedBorn adjoint equals the first one's."""
    from pyfwix_b200 import CudaWEM
    g, rng, p, src, rec, wav, slow, den, geom = _setup(nz=4)
    s2 = np.ascontiguousarray(slow[:, :1]).astype(np.complex64)
    dn = np.ascontiguousarray(den[:, :1]).astype(np.complex64)
    model = [s2, dn]
    base = dict(nref=g.nref, padx=g.padx, pady=g.pady, taperx=g.taperx, tapery=g.tapery, eps=0.0, ox=g.ox,
                dx=g.dx, oy=g.oy, dy=g.dy, oz=g.oz, dz=g.dz, ow=g.ow, dw=g.dw, compress_rate=8)
    wav_h = wav.cpu().numpy()
    d_dev = np.zeros((12, g.nw), np.complex64)
    CudaWEM.Propagator(model, d_dev, wav_h, dict(base), geom).forward(False, model, d_dev)
    par = dict(base, background_store="host", wfld_path=str(tmp_path), run_id="r1")
    d_host = np.zeros_like(d_dev)
    prop = CudaWEM.Propagator(model, d_host, wav_h, par, geom)
    prop.forward(False, model, d_host)
    assert np.abs(d_dev).max() > 0 and np.array_equal(d_host, d_dev)
    for tag in ("down", "up"):
        assert os.path.getsize(os.path.join(str(tmp_path), "r1", f"checkpoints_{tag}.bin")) > 0
    r = crandn(rng, d_host.shape).astype(np.complex64)
    dm = [np.zeros_like(s2), np.zeros_like(s2)]
    g1 = [np.zeros_like(s2), np.zeros_like(s2)]
    with pytest.warns(CudaWEM.PackedGradientWarning):
        CudaWEM.ExtendedBorn(dm, r, model, prop).adjoint(False, g1, r)
    prop2 = CudaWEM.Propagator(model, np.zeros_like(d_host), wav_h, par, geom)
    prop2.load_backgrounds(model)
    g2 = [np.zeros_like(s2), np.zeros_like(s2)]
    with pytest.warns(CudaWEM.PackedGradientWarning):
        CudaWEM.ExtendedBorn(dm, r, model, prop2).adjoint(False, g2, r)
    assert np.abs(g1[0]).max() > 0
    assert np.array_equal(g1[0], g2[0]) and np.array_equal(g1[1], g2[1])
