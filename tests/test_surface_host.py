"""Host-side logic of the operator surface that needs no GPU: hypercube and
vector conventions (SEP axis order, conjugating dot product), shot-id
remapping and its error (``propagator/src/Propagator.cpp:28-59``), the
required padding keys (``propagator/src/Propagator.cpp:63-71``) and axes taken
from ``par`` for bare arrays."""
import numpy as np
import pytest
import torch

from pyfwix_b200 import CudaWEM, vectors


def test_hypercube_axis_order():
    h = vectors.Hypercube([vectors.Axis(8, 0, 10), vectors.Axis(6, 5, 12), vectors.Axis(3, 2, 0.5),
                           vectors.Axis(4, 0, 10)])
    assert h.shape == (4, 3, 6, 8)
    assert h.getAxis(1).n == 8 and h.getAxis(4).n == 4
    assert h.getN123() == 4 * 3 * 6 * 8 and h.getNdim() == 4
    assert h.checkSame(vectors.Hypercube(h.getAxes()))
    assert not h.checkSame(vectors.Hypercube.from_shape(h.shape))


def test_vector_ops():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((3, 4)) + 1j * rng.standard_normal((3, 4))
    b = rng.standard_normal((3, 4)) + 1j * rng.standard_normal((3, 4))
    va, vb = vectors.Vector(a), vectors.Vector(b)
    assert abs(va.dot(vb) - np.vdot(a, b)) < 1e-4 * abs(np.vdot(a, b))
    vc = va.clone().scaleAdd(vb, 2.0, -1.0)
    assert np.allclose(vc.arr.numpy(), 2 * a - b, atol=1e-5)
    assert va.cloneSpace().norm() == 0.0
    sv = vectors.SuperVector(va, vb)
    assert abs(sv.dot(sv) - (np.vdot(a, a) + np.vdot(b, b))) < 1e-3
    with pytest.raises(ValueError):
        vectors.Vector(vectors.Hypercube.from_shape((2, 2)), np.zeros((3, 3)))


def test_remap_ids_dense_sorted():
    s, r, ns = CudaWEM._remap_ids([10, 31, 21, 10], [21, 21, 10, 31])
    assert ns == 3
    assert list(s) == [0, 2, 1, 0] and list(r) == [1, 1, 0, 2]
    with pytest.raises(RuntimeError, match="Shot ID not present"):
        CudaWEM._remap_ids([1, 2], [1, 3])


def test_padding_keys_required():
    with pytest.raises(RuntimeError, match="negative padx/pady"):
        CudaWEM._pads({"nref": 2})
    assert CudaWEM._pads({"padx": 4, "pady": 0}) == (4, 0)


def test_axes_from_par_for_bare_arrays():
    par = dict(ox=1.0, dx=10.0, oy=2.0, dy=12.0, oz=0.0, dz=5.0, ow=3.0, dw=0.25)
    h = CudaWEM._hyper(np.zeros((7, 5, 6, 8), np.complex64), par, "model")
    x, y, w, z = h.getAxes()
    assert (x.n, x.o, x.d) == (8, 1.0, 10.0) and (y.n, y.d) == (6, 12.0)
    assert (w.n, w.o, w.d) == (5, 3.0, 0.25) and (z.n, z.d) == (7, 5.0)
    v = vectors.Vector(h, torch.zeros(h.shape, dtype=torch.complex64))
    assert CudaWEM._hyper(v) is h


def test_store_writes_back_into_numpy_and_tensors():
    t = torch.arange(6, dtype=torch.float32).to(torch.complex64)
    a = np.zeros(6, np.complex64)
    CudaWEM._store(a, t)
    assert np.array_equal(a, t.numpy())
    b = torch.zeros(2, 3, dtype=torch.complex64)
    CudaWEM._store(b, t)
    assert torch.equal(b.reshape(-1), t)


def test_window_indices_floor_ceil_clip_and_degenerate():
    """Acquisition window of a shot group (``propagator/src/StreamingPropagator.cpp:357-393``):
    floor of the low edge, ceil of the high edge, clipped to the axis, the whole
    axis when the box collapses to one sample."""
    from pyfwix_b200.streaming import window_indices
    ax = (100, 0.0, 10.0)
    ay = (50, 5.0, 20.0)
    # x in [123, 456] +- 30 -> [93, 486] m -> ix [9, 49]; y in [105, 305] +- 0 -> iy [5, 15]
    assert window_indices([123.0, 456.0], [105.0, 305.0], ax, ay, 30.0, 0.0) == (9, 49, 5, 15)
    # clipped at both ends
    assert window_indices([-50.0, 2000.0], [0.0, 2000.0], ax, ay, 0.0, 0.0) == (0, 99, 0, 49)
    # one point, no ginsu: the box is degenerate on both axes -> whole axes
    assert window_indices([200.0], [205.0], ax, ay) == (0, 99, 0, 49)
    # no points -> whole model
    assert window_indices([], [], ax, ay) == (0, 99, 0, 49)


def test_next_fft_length_and_even_split():
    from pyfwix_b200.streaming import next_fft_length, split_even
    assert [next_fft_length(n) for n in (1, 11, 13, 17, 23, 97, 256, 257)] == [1, 12, 14, 18, 24, 98, 256, 270]
    for n in range(1, 1100):
        m = next_fft_length(n)
        k = m
        for f in (2, 3, 5, 7):
            while k % f == 0:
                k //= f
        assert k == 1 and m >= n
    assert split_even(10, 3) == [4, 3, 3]
    assert split_even(2, 5) == [1, 1]
    assert sum(split_even(128, 7)) == 128


@pytest.mark.parametrize("method", ["quantile", "kmeans"])
def test_refsampler_chunks_rows_independently(method):
    """The (depth, frequency) rows of the reference sampler are independent: any
    chunking gives the same references and labels (Lloyd run to its fixed
    point, tol = 0), labels are the nearest reference and the pads replicate the
    last row / column (propagator/src/RefSampler.cpp:75-86)."""
    from pyfwix_b200 import refsampler
    rng = np.random.default_rng(3)
    shape = (3, 5, 20, 24)
    s2 = (1 / 1800.0) ** 2 * (1 + 0.5 * rng.random(shape)) + 1j * 1e-9 * rng.standard_normal(shape)
    whole = refsampler.sample(s2, 4, 3, 2, method=method, tol=0.0)
    for chunk in (20 * 24 * 4 * 16 * 2, 1):
        part = refsampler.sample(s2, 4, 3, 2, method=method, tol=0.0, chunk_bytes=chunk)
        assert torch.equal(part[0], whole[0]) and torch.equal(part[1], whole[1])
    sref, lab = whole
    assert sref.shape == (3, 4, 5) and lab.shape == (3, 5, 22, 27) and lab.dtype == torch.uint8
    refs = sref.numpy().astype(np.complex128)                        # [nz][nref][nw]
    near = np.argmin(np.abs(s2[:, None] - refs[:, :, :, None, None]), axis=1)
    assert np.mean(lab.numpy()[:, :, :20, :24] == near) > 0.999
    assert torch.equal(lab[:, :, 20:, :24], lab[:, :, 19:20, :24].expand(-1, -1, 2, -1))
    assert torch.equal(lab[:, :, :, 24:], lab[:, :, :, 23:24].expand(-1, -1, -1, 3))
    with pytest.raises(ValueError):
        refsampler.sample(s2, 4, method="median")
