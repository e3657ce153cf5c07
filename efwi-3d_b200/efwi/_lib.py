"""ctypes binding of libefwi.so (include/efwi.h).

The product path has no CPU fallback: if the CUDA library is missing or no
GPU is visible, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libefwi.so")

EFWI_OK = 0
EFWI_ERR_ARG = 1
EFWI_ERR_CUDA = 2
EFWI_ERR_CFL = 3
EFWI_ERR_STATE = 4
EFWI_ERR_NOMEM = 5
EFWI_ERR_TOO_LARGE = 6
NOALLOC_MAX_PARTIALS = 65536

MODE_REFERENCE = 0
MODE_EXACT = 1


class EfwiError(RuntimeError):
    """Error returned by the engine (the reference exits the process)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"efwi error {code}: {msg}")
        self.code = code


class CourantError(EfwiError):
    """Courant number above 1 (the reference prints it and exits)."""


class EfwiGrid(C.Structure):
    _fields_ = [("nz", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("npml", C.c_int),
                ("nt", C.c_int), ("dz", C.c_float), ("dx", C.c_float), ("dy", C.c_float),
                ("dt", C.c_float), ("f0", C.c_float)]


class EfwiShot(C.Structure):
    _fields_ = [("z_src", C.c_int), ("x_src", C.c_int), ("y_src", C.c_int), ("nrec", C.c_int),
                ("z_rec", C.POINTER(C.c_int)), ("x_rec", C.POINTER(C.c_int)),
                ("y_rec", C.POINTER(C.c_int)), ("win_start", C.POINTER(C.c_float)),
                ("win_end", C.POINTER(C.c_float)), ("weights", C.POINTER(C.c_float)),
                ("src_weight", C.c_float)]


class EfwiWindow(C.Structure):
    _fields_ = [("x0", C.c_int), ("y0", C.c_int), ("nx", C.c_int), ("ny", C.c_int)]


_lib = None
_lock = threading.Lock()

# name -> (restype, argtypes)
_SIGS = {
    "efwi_create": (C.c_int, [C.POINTER(EfwiGrid), C.POINTER(C.c_void_p)]),
    "efwi_destroy": (None, [C.c_void_p]),
    "efwi_last_error": (C.c_char_p, [C.c_void_p]),
    "efwi_version": (C.c_char_p, []),
    "efwi_set_options": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "efwi_set_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "efwi_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "efwi_set_tuning": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "efwi_set_nt_limit": (C.c_int, [C.c_void_p, C.c_int]),
    "efwi_set_lanes": (C.c_int, [C.c_void_p, C.c_int]),
    "efwi_set_model": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "efwi_set_survey": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(EfwiShot), C.POINTER(C.c_float)]),
    "efwi_forward": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_void_p]),
    "efwi_misfit": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                              C.POINTER(C.c_double), C.c_void_p]),
    "efwi_gradient": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_int,
                                C.POINTER(C.c_double), C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p]),
    "efwi_misfit_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_float, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]),
    "efwi_forward_windows": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                       C.c_void_p, C.c_int, C.c_void_p]),
    "efwi_gradient_windows": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                        C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]),
    "efwi_adjoint": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p]),
    "efwi_illumination": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]),
    "efwi_set_stf_gradient": (C.c_int, [C.c_void_p, C.c_void_p]),
    "efwi_set_scratch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "efwi_set_checkpoint_budget": (C.c_int, [C.c_void_p, C.c_longlong]),
    "efwi_state_bytes": (C.c_longlong, [C.c_void_p]),
    "efwi_checkpoint_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "efwi_checkpoint_plan": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.c_int]),
    "efwi_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "efwi_conv3d_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "efwi_conv3d_wgrad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                    C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "efwi_conv3d_set_kernel": (C.c_int, [C.c_int]),
    "efwi_conv3d_status": (C.c_int, [C.POINTER(C.c_int), C.c_void_p]),
    "efwi_conv3d_set_wgrad_kernel": (C.c_int, [C.c_int]),
    "efwi_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "efwi_profile_read": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_longlong),
                                    C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "efwi_kernel_name": (C.c_char_p, [C.c_int]),
    "efwi_kernel_count": (C.c_int, []),
}


def exported_symbols():
    return sorted(_SIGS)


def lib() -> C.CDLL:
    """Loads libefwi.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python efwi-3d_b200/csrc/build.py` "
                    "(there is no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(handle, rc: int) -> None:
    if rc == EFWI_OK:
        return
    msg = lib().efwi_last_error(handle)
    msg = msg.decode() if msg else ""
    if rc == EFWI_ERR_CFL:
        raise CourantError(rc, msg)
    raise EfwiError(rc, msg)


def kernel_names():
    L = lib()
    return [L.efwi_kernel_name(k).decode() for k in range(L.efwi_kernel_count())]


def checkpoint_plan(nt: int, slots: int, with_actions: bool = False) -> dict:
    """Binomial checkpoint schedule of the exact gradient (host only, no GPU):
    forward steps, slots used, repetition number and, optionally, the
    actions as (op, a, b) rows (op 0 advance a->b, 1 store slot a, 2 restore
    slot a (-1: zero state), 3 adjoint block a)."""
    L = lib()
    fs, su, rep = C.c_longlong(0), C.c_int(0), C.c_int(0)
    n = L.efwi_checkpoint_plan(nt, slots, C.byref(fs), C.byref(su), C.byref(rep), None, 0)
    if n < 0:
        raise ValueError(f"no checkpoint schedule for nt={nt}, slots={slots}")
    out = {"forward_steps": fs.value, "slots_used": su.value, "repetitions": rep.value,
           "actions": n}
    if with_actions:
        buf = (C.c_int * (3 * n))()
        L.efwi_checkpoint_plan(nt, slots, None, None, None, buf, n)
        out["actions"] = [tuple(buf[3 * k:3 * k + 3]) for k in range(n)]
    return out
