"""CPU checks of the drop-in boundary: the shared library loads, exports every
entry point include/fwix_b200.h declares, and rejects bad descriptors without a
GPU (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fwix_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(fwix_[a-z0-9_]+)\s*\(", src)))


def test_header_lists_entry_points():
    names = declared()
    assert "fwix_step" in names and "fwix_born" in names and len(names) >= 25


def test_library_exports_every_declared_symbol():
    from pyfwix_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from pyfwix_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared()


def test_invalid_descriptor_is_an_error_not_an_exit():
    from pyfwix_b200 import _lib
    lib = _lib.load()
    d = _lib.FwixDesc(nx=0, ny=4, nw=1, ns=1, nz=1, dx=1, dy=1, dz=1, nref=1)
    h = ctypes.c_void_p()
    st = lib.fwix_plan_create(ctypes.byref(d), ctypes.byref(h))
    assert st == -1 and not h.value
    assert b"positive" in lib.fwix_last_error()
    d = _lib.FwixDesc(nx=11 * 16, ny=4, nw=1, ns=1, nz=1, dx=1, dy=1, dz=1, nref=1)  # factor 11
    st = lib.fwix_plan_create(ctypes.byref(d), ctypes.byref(h))
    assert st == -2 and b"2^a 3^b 5^c" in lib.fwix_last_error()
    with pytest.raises(_lib.FwixError):
        _lib.check(-4)


def test_instance_struct_layout_matches_header(tmp_path):
    """The ctypes mirror of fwix_instance has the C struct's size and field
    offsets (compiled here with the system C compiler from the header)."""
    import shutil
    import subprocess
    from pyfwix_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = [f for f, _ in _lib.FwixInstance._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fwix_b200.h"\nint main(void) {\n'
                   '  printf("%zu", sizeof(fwix_instance));\n'
                   + "".join(f'  printf(" %zu", offsetof(fwix_instance, {f}));\n' for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.FwixInstance)] + [getattr(_lib.FwixInstance, f).offset for f in fields]
    assert got == want


def test_sweep_argument_checks_without_gpu():
    """fwix_sweep rejects a bad kind or a negative count before touching the GPU,
    and an empty batch with no streams is a no-op."""
    from pyfwix_b200 import _lib
    lib = _lib.load()
    assert lib.fwix_sweep(99, None, 0, None, 0, None) == -1
    assert b"kind" in lib.fwix_last_error()
    assert lib.fwix_sweep(_lib.SWEEP_IMAGE, None, -1, None, 0, None) == -1
    assert b"instance" in lib.fwix_last_error()
    assert lib.fwix_sweep(_lib.SWEEP_IMAGE, None, 0, None, 0, None) == 0


def test_null_plan_is_rejected_by_every_entry_point():
    """Every entry point that takes a plan (or trace set) first rejects a null one
    with FWIX_ERR_INVALID and a message, before any CUDA call; the destroy
    functions accept null like free()."""
    from pyfwix_b200 import _lib
    lib = _lib.load()
    sized = {"fwix_plan_workspace_bytes", "fwix_plan_phase_cache_bytes", "fwix_plan_packed_bytes",
             "fwix_plan_wait_timeouts"}
    for name, args in sorted(_lib.SIGNATURES.items()):
        if not args or args[0] is not _lib.P:
            continue
        zeros = [0 if a in (_lib.I, _lib.I64, ctypes.c_size_t) else None for a in args]
        st = getattr(lib, name)(*zeros)
        if name in sized:
            assert st == 0, name
        elif name in ("fwix_plan_destroy", "fwix_traces_destroy"):
            assert st == 0, name
        else:
            assert st == -1, (name, st)  # FWIX_ERR_INVALID
            assert lib.fwix_last_error(), name
    assert lib.fwix_plan_create(None, None) == -1
    st = lib.fwix_step_noalloc(None, 0, 0, 0, None, None, 0, 0, None, None, 0, None)
    assert st == -1 and lib.fwix_last_error()


def test_noalloc_descriptor_checks_without_gpu():
    """fwix_step_noalloc refuses, before any CUDA call, the descriptors that
    fwix_plan_create refuses (negative taper widths) and problems whose scratch
    size would wrap a 64-bit byte count.  The buffer pointers are never read on
    these paths."""
    from pyfwix_b200 import _lib
    lib = _lib.load()
    fake = ctypes.c_void_p(256)
    call = lambda d: lib.fwix_step_noalloc(ctypes.byref(d), 0, 0, 0, fake, fake, 0, 0, fake, fake, 0, None)
    d = _lib.FwixDesc(nx=64, ny=64, nw=1, ns=1, nz=1, dx=1, dy=1, dz=1, nref=1, taperx=-1)
    assert call(d) == -1 and b"taper" in lib.fwix_last_error()
    h = ctypes.c_void_p()
    assert lib.fwix_plan_create(ctypes.byref(d), ctypes.byref(h)) == -1
    big = _lib.FwixDesc(nx=1024, ny=1024, nw=2 ** 30, ns=2 ** 30, nz=1, dx=1, dy=1, dz=1, nref=255)
    assert call(big) == -2 and b"static scratch holds" in lib.fwix_last_error()
    wide = _lib.FwixDesc(nx=1000, ny=64, padx=100, nw=1, ns=1, nz=1, dx=1, dy=1, dz=1, nref=1)
    assert call(wide) == -2 and b"at most 1024" in lib.fwix_last_error()


def test_tuning_struct_layout_matches_header(tmp_path):
    """The ctypes mirror of fwix_tuning (fwix_plan_autotune's result) has the C
    struct's size and field offsets."""
    import shutil
    import subprocess
    from pyfwix_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = [f for f, _ in _lib.FwixTuning._fields_]
    src = tmp_path / "tuning.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fwix_b200.h"\nint main(void) {\n'
                   '  printf("%zu", sizeof(fwix_tuning));\n'
                   + "".join(f'  printf(" %zu", offsetof(fwix_tuning, {f}));\n' for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "tuning"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.FwixTuning)] + [getattr(_lib.FwixTuning, f).offset for f in fields]
    assert got == want
