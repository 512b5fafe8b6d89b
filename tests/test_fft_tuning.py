"""The exchange placements committed in csrc/fast_<N>.cu are the ones the
model-based tuner (pyfwix_b200/tune_fft.py) picks for each plan's radix
stages, and each is a permutation of the line (CPU only)."""
import os
import re

import pytest

from pyfwix_b200 import tune_fft

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pyfwix_b200", "csrc")


def _committed(N):
    src = open(os.path.join(CSRC, f"fast_{N}.cu")).read()
    plans = re.findall(r"Plan<\s*(\d+),\s*(\d+),\s*fwix::fast::Radices<([\d,\s]+)>(?:,\s*(\d+))?"
                       r"(?:,\s*fwix::fast::XSw<([^;]*?)>)?>;", src)
    out = []
    for n, e, rad, sw, xs in plans:
        codes = []
        if xs:
            for m in re.finditer(r"xs\((\d+), (\d+), (\d+)\)|(-?\d+)", xs):
                codes.append(int(m.group(1)) | int(m.group(2)) << 4 | int(m.group(3)) << 8 if m.group(1)
                             else int(m.group(4)))
        out.append((int(n), int(e), tuple(int(r) for r in rad.split(",")), int(sw or 0), codes))
    return out


@pytest.mark.parametrize("N", sorted(tune_fft.PLANS))
def test_committed_placements_are_the_tuned_ones(N):
    E, rad = tune_fft.PLANS[N]
    plans = [p for p in _committed(N) if p[1] == E and p[2] == rad and p[3] == 0]
    assert len(plans) == 1, plans
    codes = plans[0][4]
    want, _, _ = tune_fft.best_placements(N, E, rad)
    if not codes:  # no XSw list: every exchange keeps the default placement
        assert want == [-1] * len(want)
    else:
        assert codes == want
    for c in codes:
        if c > 0:
            f = lambda p: p ^ (((p >> (c & 15)) * ((c >> 4) & 15)) & (c >> 8))
            assert sorted(f(p) for p in range(N)) == list(range(N))


def test_wavefront_model_known_cases():
    # 16 lanes on 16 distinct bank pairs: one wavefront per half-warp
    assert tune_fft.wavefronts(list(range(32))) == 2
    # stride 16 words: every lane of a half-warp on the same bank pair
    assert tune_fft.wavefronts([16 * i for i in range(32)]) == 32
    # the same word for all lanes is one wavefront (broadcast)
    assert tune_fft.wavefronts([5] * 32) == 2
