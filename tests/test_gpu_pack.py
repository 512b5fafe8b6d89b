"""Fixed-rate lossy store of wavefields on the device (pyfwix_b200/csrc/pack.cu):
packed bytes and unpacked values bit-exact against the oracle's restatement
(oracle/pack.py), with 16-byte aligned and unaligned buffers; modelling with
packed down / up fields against modelling with full ones; Born on packed
backgrounds (which also keeps its per-level recursion fields packed) within the
store's error of Born on the unpacked and on the exact backgrounds."""
import numpy as np
import pytest
import torch

from oracle import pack as opack
from tests.conftest import crandn
from tests.gpu_helpers import make_case, make_plan, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("nx,ny,nw,ns,pad", [(32, 24, 3, 1, 4), (60, 44, 5, 2, 4), (64, 64, 2, 1, 0)])
def test_pack_bits_against_oracle(nx, ny, nw, ns, pad, bits):
    g, rng, sref, labels, slow, den = make_case(nx=nx, ny=ny, nw=nw, nz=2, nref=2, padx=pad, pady=pad)
    p = make_plan(g, ns, sref, labels)
    p.set_pack_rate(bits)
    x = crandn(rng, p.wshape).astype(np.complex64)
    x *= np.float32(10.0) ** rng.integers(-5, 5, size=x.shape)
    x[0, 0, :2] = 0
    xd = torch.as_tensor(x).cuda()
    pk = p.packed(1)[0].fill_(0xAB)        # the pack writes every byte, its zero tail too
    p.pack(xd, pk)
    y = torch.empty_like(xd)
    p.unpack(pk, y)
    torch.cuda.synchronize()
    want = opack.pack(x, bits)
    assert pk.numel() == want.size == p.packed_bytes
    got = pk.cpu().numpy()
    assert np.array_equal(got, want)
    assert np.array_equal(y.cpu().numpy().view(np.float32), opack.unpack(want, x.shape, bits).view(np.float32))
    # buffers 8 bytes off a 16-byte boundary take the scalar path: same bytes
    xo = torch.zeros(x.size + 1, dtype=torch.complex64, device="cuda")[1:]
    xo.copy_(xd.ravel())
    po = torch.full((p.packed_bytes + 16,), 0xAB, dtype=torch.uint8, device="cuda")[4:4 + p.packed_bytes]
    import ctypes
    from pyfwix_b200 import _lib as L
    from pyfwix_b200.plan import _stream
    pack, unpack = ((L.load().fwix_pack_rate8, L.load().fwix_unpack_rate8) if bits == 8 else
                    (L.load().fwix_pack_wavefield, L.load().fwix_unpack_wavefield))
    L.check(pack(p._h, ctypes.c_void_p(xo.data_ptr()), ctypes.c_void_p(po.data_ptr()), _stream()))
    yo = torch.zeros(x.size + 1, dtype=torch.complex64, device="cuda")[1:]
    L.check(unpack(p._h, ctypes.c_void_p(po.data_ptr()), ctypes.c_void_p(yo.data_ptr()), _stream()))
    torch.cuda.synchronize()
    assert np.array_equal(po.cpu().numpy(), want)
    assert torch.equal(yo, y.ravel())


def _acq(g, p):
    geom = dict(sx=[80.0], sy=[96.0], sz=[0.0], s_ids=[0], rx=list(np.linspace(0, 300, 16)), ry=[100.0] * 16,
                rz=[0.0] * 16, r_ids=[0] * 16)
    src = p.traces(geom["sx"], geom["sy"], geom["sz"], [0])
    rec = p.traces(geom["rx"], geom["ry"], geom["rz"], [0] * 16)
    return src, rec


@pytest.mark.parametrize("kind,nx,ny,pad,nw", [("pspi", 32, 24, 4, 4), ("nsps", 64, 64, 0, 4),
                                               ("pspi", 27, 21, 0, 3)])
def test_packed_modelling_and_born(kind, nx, ny, pad, nw):
    """(27 x 21 x 3: an odd wavefield size, so the workspace fields sit 8 bytes off
    a 16-byte boundary and the packing kernels take their scalar path.)"""
    g, rng, sref, labels, slow, den = make_case(nx=nx, ny=ny, nw=nw, nz=6, nref=3, padx=pad, pady=pad)
    slow = slow.copy()
    slow[g.nz - 2:] *= 1.8
    p = make_plan(g, 1, sref, labels, slow, den, step=kind)
    src, rec = _acq(g, p)
    wav = torch.as_tensor(crandn(rng, (1, g.nw)).astype(np.complex64)).cuda()
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((16, g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, wav, d, bd, bu)
    pd, pu = p.packed(g.nz), p.packed(g.nz)
    dp = torch.empty_like(d)
    p.propagate_packed(src, rec, wav, dp, pd, pu)
    # the packed fields are the packed full fields, the up pass reflecting unpacked down fields
    ud, uu = torch.empty_like(bd), torch.empty_like(bu)
    for iz in range(g.nz):
        p.unpack(pd[iz], ud[iz])
        p.unpack(pu[iz], uu[iz])
    torch.cuda.synchronize()
    assert rel(ud.cpu().numpy(), bd.cpu().numpy()) < 1e-2
    assert rel(uu.cpu().numpy(), bu.cpu().numpy()) < 2e-2
    assert rel(dp.cpu().numpy(), d.cpu().numpy()) < 2e-2
    ms = torch.as_tensor(crandn(rng, (g.nz, g.nw, g.ny, g.nx)).astype(np.complex64)).cuda()
    mr = torch.as_tensor(crandn(rng, (g.nz, g.nw, g.ny, g.nx)).astype(np.complex64)).cuda()
    r = torch.as_tensor(crandn(rng, d.shape).astype(np.complex64)).cuda()
    for adjoint in (False, True):
        if not adjoint:
            o1, o2, o3 = (torch.empty_like(d) for _ in range(3))
            p.born_packed(rec, pd, pu, ms, mr, o1)
            p.born(rec, ud, uu, ms, mr, o2)
            p.born(rec, bd, bu, ms, mr, o3)
            outs = [(o1, o2, o3)]
        else:
            gp = [torch.empty_like(ms) for _ in range(6)]
            p.born_packed(rec, pd, pu, gp[0], gp[1], r, adjoint=True)
            p.born(rec, ud, uu, gp[2], gp[3], r, adjoint=True)
            p.born(rec, bd, bu, gp[4], gp[5], r, adjoint=True)
            outs = [(gp[0], gp[2], gp[4]), (gp[1], gp[3], gp[5])]
        torch.cuda.synchronize()
        for a, b, c in outs:
            assert rel(a.cpu().numpy(), b.cpu().numpy()) < 2e-2
            assert rel(a.cpu().numpy(), c.cpu().numpy()) < 3e-2
    n = int(np.prod(p.wshape))
    assert p.packed_bytes == opack.packed_bytes(2 * n)  # 17 bytes per 16 floats, padded to 256
    assert p.packed_bytes * 3.7 < 8 * n or n < 4096


@pytest.mark.parametrize("kind", ["pspi", "nsps"])
def test_rate16_born_within_gradient_tolerance(kind):
    """At 16 mantissa bits per value the packed backgrounds (and the packed
    per-level recursion fields) keep ExtendedBorn forward and adjoint within the
    1e-3 gradient bar of the lossless operator, where rate 8 does not."""
    g, rng, sref, labels, slow, den = make_case(nx=32, ny=24, nw=4, nz=6, nref=3, padx=4, pady=4)
    slow = slow.copy()
    slow[g.nz - 2:] *= 1.8
    p = make_plan(g, 1, sref, labels, slow, den, step=kind)
    src, rec = _acq(g, p)
    wav = torch.as_tensor(crandn(rng, (1, g.nw)).astype(np.complex64)).cuda()
    bd = torch.empty((g.nz,) + p.wshape, dtype=torch.complex64, device="cuda")
    bu = torch.empty_like(bd)
    d = torch.empty((16, g.nw), dtype=torch.complex64, device="cuda")
    p.propagate(src, rec, wav, d, bd, bu)
    r = torch.as_tensor(crandn(rng, d.shape).astype(np.complex64)).cuda()
    g_ref = [torch.empty((g.nz, g.nw, g.ny, g.nx), dtype=torch.complex64, device="cuda") for _ in range(2)]
    p.born(rec, bd, bu, g_ref[0], g_ref[1], r, adjoint=True)
    errs = {}
    for bits in (8, 16):
        p.set_pack_rate(bits)
        pd, pu = p.packed(g.nz), p.packed(g.nz)
        dp = torch.empty_like(d)
        p.propagate_packed(src, rec, wav, dp, pd, pu)
        gp = [torch.empty_like(g_ref[0]) for _ in range(2)]
        p.born_packed(rec, pd, pu, gp[0], gp[1], r, adjoint=True)
        torch.cuda.synchronize()
        errs[bits] = max(rel(gp[k].cpu().numpy(), g_ref[k].cpu().numpy()) for k in range(2))
        if bits == 16:
            assert rel(dp.cpu().numpy(), d.cpu().numpy()) < 1e-4
    assert errs[16] < 1e-3 < errs[8] * 10 and errs[16] < errs[8] / 50, errs
