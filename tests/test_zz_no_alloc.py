"""fwix_step_noalloc: the depth step for callers that cannot call cudaMalloc (for
example a host application that owns all device memory in its own pool).  The
entry point takes only caller-owned inputs and outputs and keeps its scratch in a
static device array, so it must give the same result as fwix_step, which uses a
caller-bound workspace.  Called twice in a row to show that the shared scratch
left by one call does not leak into the next.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import pytest
import torch

from tests.gpu_helpers import make_case, make_plan, rel, to_dev, to_host, wavefield

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(lib, plan, kind, iz, direction, sref, labels, inp, out, add):
    from pyfwix_b200 import _lib
    labels_t = plan._keep["labels"]
    wst = 0 if labels_t.shape[1] == 1 else plan.NY * plan.NX
    zst = labels_t.shape[1] * plan.NY * plan.NX
    st = lib.fwix_step_noalloc(ctypes.byref(plan.desc), kind, iz, direction, ctypes.c_void_p(sref.data_ptr()),
                               ctypes.c_void_p(labels_t.data_ptr()), zst, wst, ctypes.c_void_p(inp.data_ptr()),
                               ctypes.c_void_p(out.data_ptr()), int(add),
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)
    return out


# (nx, ny, pad, nw): a padded 48 x 40 grid takes the generic passes; 64 x 64 and
# 256 x 256 take the size-specialised register-resident passes that production
# grids use (256 x 256 x 16 frequencies: five wavefields of 8 MiB in the scratch).
SIZES = [(40, 36, (8, 4), 4), (56, 60, (8, 4), 4), (256, 256, (0, 0), 16)]


@pytest.mark.parametrize("size", SIZES, ids=["48x40", "64x64", "256x256"])
@pytest.mark.parametrize("kind,direction", [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)])
def test_noalloc_step_matches_workspace_step(kind, direction, size):
    from pyfwix_b200 import _lib
    lib = _lib.load()
    step = "pspi" if kind == 0 else "nsps"
    nx, ny, (padx, pady), nw = size
    ns = 2 if nx < 256 else 1
    g, rng, sref, labels, _, _ = make_case(nx=nx, ny=ny, nw=nw, nz=3, nref=4, padx=padx, pady=pady, eps=0.01,
                                           complex_refs=True, labels_per_w=False)
    p = make_plan(g, ns, sref, labels, step=step)
    sref_d = p._keep["sref"]
    for call in range(2):  # two calls in a row on the shared scratch
        x = wavefield(rng, ns, g)
        d0 = wavefield(rng, ns, g)
        iz = call + 1
        ref = to_host(p.step(iz, to_dev(x), to_dev(d0), direction=direction, add=True))
        got = to_host(_noalloc(lib, p, kind, iz, direction, sref_d, labels, to_dev(x), to_dev(d0), True))
        assert rel(got, ref) < TOL, (call, rel(got, ref))
        xin = to_dev(x)  # in place, add = 0
        ref2 = to_host(p.step(iz, to_dev(x), torch.empty_like(xin), direction=direction))
        got2 = to_host(_noalloc(lib, p, kind, iz, direction, sref_d, labels, xin, xin, False))
        assert rel(got2, ref2) < TOL


def test_noalloc_rejects_oversize_problem():
    from pyfwix_b200 import _lib
    lib = _lib.load()
    # 512 x 512 x 64 frequencies x 2 shots: (4 + 1) wavefields of 256 MiB exceed the scratch
    d = _lib.FwixDesc(nx=512, ny=512, nw=64, ns=2, nz=1, dx=10, dy=10, dz=10, ow=1, dw=1, nref=4)
    x = torch.zeros(8, dtype=torch.complex64, device="cuda")
    lab = torch.zeros(8, dtype=torch.uint8, device="cuda")
    st = lib.fwix_step_noalloc(ctypes.byref(d), 0, 0, 0, ctypes.c_void_p(x.data_ptr()),
                               ctypes.c_void_p(lab.data_ptr()), 0, 0, ctypes.c_void_p(x.data_ptr()),
                               ctypes.c_void_p(x.data_ptr()), 0, None)
    assert st == -2  # FWIX_ERR_UNSUPPORTED
    assert b"static scratch holds" in lib.fwix_last_error()
    # frequency and shot counts whose product with the slice size would wrap a
    # 64-bit byte count are refused the same way, before anything is launched
    big = _lib.FwixDesc(nx=1024, ny=1024, nw=2 ** 30, ns=2 ** 30, nz=1, dx=10, dy=10, dz=10, ow=1, dw=1, nref=255)
    st = lib.fwix_step_noalloc(ctypes.byref(big), 0, 0, 0, ctypes.c_void_p(x.data_ptr()),
                               ctypes.c_void_p(lab.data_ptr()), 0, 0, ctypes.c_void_p(x.data_ptr()),
                               ctypes.c_void_p(x.data_ptr()), 0, None)
    assert st == -2
    assert b"static scratch holds" in lib.fwix_last_error()
