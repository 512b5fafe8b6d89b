"""ctypes binding of libfwix_b200.so (the C ABI declared in include/fwix_b200.h).

The library is the product path: if it cannot be loaded the import fails with a
clear error.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfwix_b200.so")

FWIX_OK = 0
STATUS = {0: "FWIX_OK", -1: "FWIX_ERR_INVALID", -2: "FWIX_ERR_UNSUPPORTED", -3: "FWIX_ERR_CUDA",
          -4: "FWIX_ERR_STATE", -5: "FWIX_ERR_WORKSPACE"}

STEP_PSPI, STEP_NSPS = 0, 1
FWD, ADJ_ADD, ADJ_INPL = 0, 1, 2
PS_FWD, PS_ADJ, PS_INV = 0, 1, 2
SMOOTH_FWD, SMOOTH_ADJ, SMOOTH_DERIV = 0, 1, 2
WS_STEP, WS_SWEEP, WS_BORN, WS_BORN_PACKED = 0, 1, 2, 3


class FwixDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("padx", ctypes.c_int), ("pady", ctypes.c_int),
        ("nw", ctypes.c_int), ("ns", ctypes.c_int), ("nz", ctypes.c_int),
        ("ox", ctypes.c_float), ("oy", ctypes.c_float), ("oz", ctypes.c_float),
        ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
        ("ow", ctypes.c_float), ("dw", ctypes.c_float),
        ("nref", ctypes.c_int), ("eps", ctypes.c_float),
        ("taperx", ctypes.c_int), ("tapery", ctypes.c_int),
        ("eps_scat", ctypes.c_float), ("taylor", ctypes.c_int),
        ("step_kind", ctypes.c_int),
    ]


P = ctypes.c_void_p
I = ctypes.c_int
I64 = ctypes.c_int64


class FwixInstance(ctypes.Structure):
    """fwix_instance: one instance of a batched sweep (fwix_sweep)."""
    _fields_ = [
        ("plan", P), ("src", P), ("rec", P), ("wavelet", P), ("data", P), ("wfld", P), ("image", P),
        ("bg_down", P), ("bg_up", P), ("dslow", P), ("dden", P), ("model_w_stride", I64),
        ("adjoint", I), ("add", I),
    ]

class FwixTuning(ctypes.Structure):
    """fwix_tuning: the choice of fwix_plan_autotune."""
    _fields_ = [("col_tma", ctypes.c_int), ("fused", ctypes.c_int), ("slices_per_launch", ctypes.c_int64),
                ("ms", ctypes.c_float), ("candidates", ctypes.c_int), ("streams", ctypes.c_int)]


# name -> argtypes (all return fwix_status as int unless listed in _RET)
SIGNATURES = {
    "fwix_last_error": [],
    "fwix_version": [],
    "fwix_launch_count": [],
    "fwix_plan_create": [ctypes.POINTER(FwixDesc), ctypes.POINTER(P)],
    "fwix_plan_destroy": [P],
    "fwix_plan_workspace_bytes": [P, I],
    "fwix_plan_wait_timeouts": [P],
    "fwix_plan_set_workspace": [P, P, ctypes.c_size_t],
    "fwix_plan_set_refs": [P, P, P, I64, I64],
    "fwix_plan_phase_cache_bytes": [P],
    "fwix_plan_set_phase_cache": [P, P, ctypes.c_size_t],
    "fwix_plan_set_model": [P, P, P, I64, I64],
    "fwix_fft2d": [P, I, P, P, I, P],
    "fwix_phase_shift": [P, I, P, P, P, I, P],
    "fwix_select": [P, I, I, P, P, I, P],
    "fwix_taper": [P, P, P, I, P],
    "fwix_step": [P, I, I, I, P, P, I, P],
    "fwix_plan_set_smooth": [P, P, P],
    "fwix_smooth_step": [P, I, I, P, P, I, P],
    "fwix_smooth_step_pair": [P, I, P, P, P, I, P],
    "fwix_correlate": [P, P, P, P, I, I, P],
    "fwix_smooth_model_sweep": [P, P, P, P, P, P, P, P, P],
    "fwix_smooth_gradient_sweep": [P, P, P, P, P, P, P, P, P, P, P],
    "fwix_scatter": [P, I, I, P, P, I, P],
    "fwix_reflect": [P, I, I, P, P, I, P],
    "fwix_imaging": [P, I, P, P, P, I, P],
    "fwix_lin_reflect": [P, I, I, P, P, I, P],
    "fwix_traces_create": [P, I, P, P, P, P, ctypes.POINTER(P)],
    "fwix_traces_destroy": [P],
    "fwix_inject": [P, P, I, I, P, P, I, P],
    "fwix_downward": [P, I, P, P],
    "fwix_upward": [P, I, P, P],
    "fwix_propagate": [P, P, P, P, P, I, P, P, P],
    "fwix_migrate": [P, P, P, P, P, P, I, P],
    "fwix_born": [P, I, P, P, P, P, P, I64, P, I, P],
    "fwix_plan_autotune": [P, I, I, P, P, I, P, ctypes.POINTER(FwixTuning)],
    "fwix_plan_set_tuning": [P, ctypes.POINTER(FwixTuning)],
    "fwix_step_noalloc": [ctypes.POINTER(FwixDesc), I, I, I, P, P, I64, I64, P, P, I, P],
    "fwix_pspi_step": [P, I, P, P, I, P],
    "fwix_nsps_step": [P, I, P, P, I, P],
    "fwix_image_accumulate": [P, P, P, P, I, P],
    "fwix_sweep": [I, ctypes.POINTER(FwixInstance), I, ctypes.POINTER(P), I, P],
    "fwix_plan_packed_bytes": [P],
    "fwix_plan_set_pack_rate": [P, I],
    "fwix_pack_wavefield": [P, P, P, P],
    "fwix_unpack_wavefield": [P, P, P, P],
    "fwix_pack_rate8": [P, P, P, P],
    "fwix_unpack_rate8": [P, P, P, P],
    "fwix_propagate_packed": [P, P, P, P, P, I, P, P, P],
    "fwix_born_packed": [P, I, P, P, P, P, P, I64, P, I, P],
}
SWEEP_DOWN, SWEEP_UP, SWEEP_MODEL, SWEEP_IMAGE, SWEEP_BORN_FWD, SWEEP_BORN_ADJ = range(6)
_RET = {"fwix_last_error": ctypes.c_char_p, "fwix_version": I, "fwix_plan_workspace_bytes": ctypes.c_size_t,
        "fwix_plan_phase_cache_bytes": ctypes.c_size_t, "fwix_plan_packed_bytes": ctypes.c_size_t,
        "fwix_launch_count": ctypes.c_uint64, "fwix_plan_wait_timeouts": ctypes.c_uint64}

_lib = None


def load():
    """Load (once) and return the ctypes handle of libfwix_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m pyfwix_b200.build` "
            "(nvcc, sm_100a).  pyfwix_b200 has no CPU fallback.")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RET.get(name, I)
    _lib = lib
    return lib


class FwixError(RuntimeError):
    """Raised for a negative fwix_status; carries the status code."""

    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def check(status):
    if status != FWIX_OK:
        msg = load().fwix_last_error()
        raise FwixError(status, msg.decode() if msg else "")
    return status
