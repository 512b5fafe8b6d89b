"""Recipe for the oracle's reference-kernel shim (test infrastructure).

Compiles pyfwix's own CUDA kernels from the reference sources where they lie
(``propagator/src/{phase_shift,selector,taper,injection,reflect,scatter,
imaging_condition,lin_reflect}.cu``, headers from ``operator/src`` and
``propagator/src``) together with ``shim.cu`` and a stub ``hypercube.h`` into
``oracle/_ref/librefshim.so`` (git-ignored).  Nothing is copied out of the
reference tree.  The reference's full build (CMake, SEP-IO, OpenCV, zfp,
FFTW) is not used and cannot run here; the kernels need none of it.

``python -m oracle.refshim.build`` builds it; ``build_if_sources_present()`` is
what the package build calls (a no-op where the reference tree is absent).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_DIR = os.path.join(ORACLE, "_ref")
LIB = os.path.join(OUT_DIR, "librefshim.so")
# the reference tree: FWIX_REFERENCE_TREE, else a "reference" directory beside this repository
REF = os.environ.get("FWIX_REFERENCE_TREE",
                     os.path.normpath(os.path.join(os.path.dirname(ORACLE), os.pardir, "reference")))
KERNELS = ["phase_shift", "selector", "taper", "injection", "reflect", "scatter", "imaging_condition",
           "lin_reflect"]


def sources():
    return [os.path.join(REF, "propagator", "src", k + ".cu") for k in KERNELS]


def present():
    return all(os.path.exists(p) for p in sources())


def build(force=False):
    if not present():
        raise FileNotFoundError(f"reference sources not found under {REF}")
    deps = sources() + [os.path.join(HERE, "shim.cu"), os.path.join(HERE, "stub", "hypercube.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(p) <= os.path.getmtime(LIB) for p in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-w",
           "-I", os.path.join(HERE, "stub"), "-I", os.path.join(REF, "operator", "src"),
           "-I", os.path.join(REF, "propagator", "src"),
           os.path.join(HERE, "shim.cu")] + sources() + ["-lcufft", "-o", LIB + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("reference shim build failed:\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_if_sources_present():
    return build() if present() else None


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
