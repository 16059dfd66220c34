"""ctypes binding of libpfa_b200.so (declarations in include/pfa_b200.h).

Loading fails loudly: there is no CPU fallback.  ``load()`` raises ``PfaLibraryError`` when the
library is missing or cannot be opened.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(os.environ.get("PFA_B200_LIB", Path(__file__).resolve().parent / "lib" / "libpfa_b200.so"))

OK, BAD_CONFIG, BAD_DIMS, BAD_ARG, NOT_READY, CUDA, ALLOC, TIMEOUT, NO_DEVICE, TOO_LARGE = range(10)
MODE_FIXED, MODE_FLOAT32, MODE_MIXED = 0, 1, 2
LERP, SINC, CUBIC = 0, 1, 2
DETECT_ORDER_EMULATOR, DETECT_ORDER_FUSED = 0, 1
LAYOUT_CENTRED, LAYOUT_NATURAL = 0, 1
DETECT_MAG, DETECT_POWER, DETECT_COMPLEX = 0, 1, 2


class PfaLibraryError(RuntimeError):
    pass


class PfaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"pfa status {status}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("mode", C.c_int32), ("m", C.c_int32), ("n", C.c_int32), ("grid", C.c_int32),
                ("range_interp", C.c_int32), ("az_interp", C.c_int32), ("device", C.c_int32),
                ("fft_ept_cross", C.c_int32), ("fft_ept_range", C.c_int32), ("detect_order", C.c_int32),
                ("test_wait_polls", C.c_int32), ("reserved", C.c_int32 * 5)]


class FixedJob(C.Structure):
    _fields_ = [("f0", C.c_void_p), ("df", C.c_void_p), ("pr", C.c_void_p), ("tan_s", C.c_void_p),
                ("inv_order", C.c_void_p), ("kr_grid", C.c_void_p), ("kc_grid", C.c_void_p),
                ("ham_r", C.c_void_p), ("ham_c", C.c_void_p), ("twiddle", C.c_void_p),
                ("sinc_q15", C.c_void_p)]


class FloatJob(C.Structure):
    _fields_ = [("f0", C.c_void_p), ("df", C.c_void_p), ("f_last", C.c_void_p), ("pr", C.c_void_p),
                ("tan_s", C.c_void_p), ("order", C.c_void_p), ("kr_grid", C.c_void_p), ("kc_grid", C.c_void_p),
                ("ham_m", C.c_void_p), ("ham_n", C.c_void_p), ("sgn", C.c_int32), ("layout", C.c_int32)]


# name -> (restype, argtypes); every function declared in include/pfa_b200.h
SIGNATURES = {
    "pfa_plan_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "pfa_plan_destroy": (C.c_int, [C.c_void_p]),
    "pfa_plan_workspace_bytes": (C.c_size_t, [C.c_void_p]),
    "pfa_set_fixed_job": (C.c_int, [C.c_void_p, C.POINTER(FixedJob)]),
    "pfa_set_float_job": (C.c_int, [C.c_void_p, C.POINTER(FloatJob)]),
    "pfa_form_fixed": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pfa_form_fixed_iq16": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pfa_form_fixed_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "pfa_get_fixed_exponents": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pfa_form_fixed_noalloc": (C.c_int, [C.POINTER(Config), C.POINTER(FixedJob), C.c_void_p, C.c_void_p,
                                         C.c_void_p]),
    "pfa_form_float": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "pfa_form_float_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "pfa_form_fixed_host_frames": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "pfa_form_float_host_frames": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]),
    "pfa_autofocus_grad":(C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pfa_autofocus_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p]),
    "pfa_form_float_phase": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "pfa_display_workspace_bytes": (C.c_size_t, []),
    "pfa_display_u8": (C.c_int, [C.c_void_p, C.c_int64, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pfa_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "pfa_get_stage_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_char_p, C.c_size_t]),
    "pfa_status_string": (C.c_char_p, [C.c_int]),
    "pfa_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "pfa_version": (C.c_char_p, []),
}

_LIB = None


def load():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.is_file():
        raise PfaLibraryError(f"{LIB_PATH} not found: build it with mpfs250t-sar-ifp_b200/build.py")
    try:
        lib = C.CDLL(str(LIB_PATH))
    except OSError as e:
        raise PfaLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(status: int, plan=None):
    if status == OK:
        return
    lib = load()
    msg = lib.pfa_status_string(status).decode()
    if plan:
        buf = C.create_string_buffer(512)
        lib.pfa_last_error(plan, buf, 512)
        if buf.value:
            msg += ": " + buf.value.decode()
    raise PfaError(status, msg)
