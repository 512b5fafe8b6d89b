"""Builds libfwix_b200.so in-tree with nvcc for sm_100a.

``python -m pyfwix_b200.build`` (or ``__graft_entry__.build()``) compiles the
CUDA sources under ``pyfwix_b200/csrc`` into ``pyfwix_b200/libfwix_b200.so``.
The library is rebuilt only when a source or header is newer than it.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libfwix_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-shared"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps += glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libfwix_b200.so")
    return exe


OBJDIR = os.path.join(ROOT, "_build")


def _compile(src, extra, verbose):
    obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
    cmd = [nvcc()] + ARCH + [f for f in FLAGS if f != "-shared"] + list(extra) + ["-I", INCLUDE, "-I", CSRC,
                                                                                    "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + res.stdout + res.stderr)
    return obj, (res.stdout + res.stderr) if verbose else ""


def build(force=False, verbose=False, extra=(), jobs=None):
    """Compile the library if needed (one object per source, in parallel) and
    return its path."""
    if not force and not _stale():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    jobs = jobs or max(1, min(len(sources()), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, verbose), sources()))
    for _, log in results:
        if log:
            print(log)
    cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC"] + [o for o, _ in results] + ["-o", LIB + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ())
