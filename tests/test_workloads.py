"""The seeded synthetic workloads (pyfwix_b200/workloads.py) have the stated
shapes, bands and value ranges and are reproducible; CPU only."""
import numpy as np
import torch

from pyfwix_b200 import workloads


def test_config1_and_config2_shapes_and_ranges():
    w = workloads.config1(nz=20)
    assert w.slow2.shape == (20, 128, 128) and w.nw == 64
    assert abs(w.freqs[0] - 2.0) < 1e-9 and abs(w.freqs[-1] - 30.0) < 1e-9
    v = 1 / np.sqrt(w.slow2)
    assert v.min() >= 1500 - 1e-3 and v.max() <= (1500 + 0.5 * 190) * 1.1 + 1e-2
    assert len(w.geom["rx"]) == 128 * 128 and w.wavelet.shape == (1, 64)
    w2 = workloads.config2(nz=12, nw=8)
    assert w2.slow2.shape == (12, 256, 256) and w2.dslow.shape == (12, 256, 256) and w2.step == "nsps"
    v2 = 1 / np.sqrt(w2.slow2)
    base = 1500.0 + 0.4 * (w2.dz * np.arange(12))[:, None, None]
    assert np.max(np.abs(v2 / base - 1)) <= 0.05 + 1e-6
    again = workloads.config2(nz=12, nw=8)
    assert np.array_equal(again.slow2, w2.slow2) and np.array_equal(again.dslow, w2.dslow)


def test_config3_bands_and_grids():
    shots = workloads.config3(nshots=32, nz=4)
    assert len(shots) == 32
    for w in shots:
        assert w.nx == w.ny and w.nx in (128, 192, 256, 320, 384) and 48 <= w.nw <= 160
        assert w.freqs[0] >= 2.0 - 1e-9 and w.freqs[-1] <= 45.0 + 1e-9
        s2 = workloads.slow2_on(w, "cpu")
        assert tuple(s2.shape) == (4, w.ny, w.nx) and s2.dtype == torch.float32
    assert len({(w.nx, w.nw) for w in shots}) > 5  # uneven apertures and bands


def test_config4_and_config5_models():
    w, s_true, s0 = workloads.config4(nz=6)
    assert s_true.shape == s0.shape == (6, 384, 384) and w.nref == 4
    assert np.max(np.abs(s_true / s0 - 1)) < 0.09
    w5 = workloads.config5(nz=8)
    assert (w5.nx, w5.ny, w5.nw, w5.nref) == (512, 512, 200, 8)
    v = 1 / torch.sqrt(workloads.slow2_on(w5, "cpu").double())
    assert float(v.min()) >= 1500 - 1e-2 and float(v.max()) <= 4500 + 1e-2
