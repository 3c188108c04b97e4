"""ctypes binding of libsfb200.so (include/sfb200.h).

The library is loaded from this package directory. There is no fallback: if
the shared object is missing, importing this module raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsfb200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is not built; build it with `python -c 'import __graft_entry__ as g; g.build()'` "
        "from the repository root (nvcc for sm_100a is required)")

lib = C.CDLL(LIB_PATH)

SF_OK = 0
SF_ERR_ARG = 1
SF_ERR_CUDA = 2
SF_ERR_STATE = 3
SF_ERR_UNSUPPORTED = 4
SF_ERR_NOT_CONVERGED = 5
SF_ERR_NONFINITE = 6

SF_F64 = 0
SF_F32 = 1

SF_CG_F64 = 0
SF_CG_MIXED = 1
SF_CG_F64_PLAIN = 2

SF_MG_MIXED = 0
SF_MG_F64 = 1

vp = C.c_void_p
i32 = C.c_int
i64 = C.c_int64
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)

# name -> (restype, argtypes); this table is also the list of exported symbols
# that the header declares (checked by tests/test_abi.py).
SIGNATURES = {
    "sf_version": (i32, []),
    "sf_status_string": (C.c_char_p, [i32]),
    "sf_create": (i32, [C.POINTER(vp), i32, i32, i32, vp, vp, vp]),
    "sf_destroy": (i32, [vp]),
    "sf_last_error": (C.c_char_p, [vp]),
    "sf_get_dimensional_parameters": (i32, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]),
    "sf_set_cells": (i32, [vp, i64, vp, vp, i64]),
    "sf_set_structured": (i32, [vp, i32, i32, i32, vp]),
    "sf_set_cell_quantities": (i32, [vp, i32, vp, vp, vp]),
    "sf_set_coefficient": (i32, [vp, vp]),
    "sf_apply": (i32, [vp, i32, vp, vp, vp]),
    "sf_apply_multi": (i32, [vp, i32, i32, vp, i64, vp, i64, vp]),
    "sf_mul_host": (i32, [vp, vp, vp]),
    "sf_evaluate_cells": (i32, [vp, i32, i64, vp, vp, vp]),
    "sf_diagonal": (i32, [vp, i32, vp, vp]),
    "sf_cg": (i32, [vp, i32, vp, vp, C.c_double, i32, C.POINTER(i32), dp, vp]),
    "sf_set_option": (i32, [vp, C.c_char_p, C.c_double]),
    "sf_last_solve_info": (i32, [vp, C.POINTER(i32), C.POINTER(i32), dp]),
    "sf_get_info": (i32, [vp, C.c_char_p, dp]),
    "sf_cg_noalloc": (i32, [vp, i32, vp, vp, C.c_double, i32, C.POINTER(i32), dp, vp]),
    "sf_autotune": (i32, [vp, i32, vp]),
    "sf_set_coefficient_device": (i32, [vp, vp, vp]),
    "sf_kappa_vjp": (i32, [vp, i32, vp, vp, vp, vp]),
    "sf_batch_create": (i32, [C.POINTER(vp), i32, C.POINTER(vp), i32]),
    "sf_batch_destroy": (i32, [vp]),
    "sf_batch_last_error": (C.c_char_p, [vp]),
    "sf_batch_groups": (i32, [vp, C.POINTER(i32)]),
    "sf_batch_apply": (i32, [vp, i32, C.POINTER(vp), C.POINTER(vp), vp]),
    "sf_batch_autotune": (i32, [vp, i32, C.POINTER(vp), C.POINTER(vp), vp]),
    "sf_batch_group_kernel": (C.c_char_p, [vp, i32, i32]),
    "sf_kernel_name": (C.c_char_p, [vp, i32]),
    "sf_cg_kernel_name": (C.c_char_p, [vp]),
    "sf_set_structured_slab": (i32, [vp, i32, i32, i32, i32, i32, vp]),
    "sf_set_structured_numbering": (i32, [vp, i32, i32, i32, vp, vp]),
    "sf_rhs": (i32, [vp, vp, vp, vp]),
    "sf_cgd_start": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "sf_cgd_init": (i32, [vp, vp, C.c_double, vp]),
    "sf_cgd_apply": (i32, [vp, vp, vp, vp, vp]),
    "sf_cgd_update": (i32, [vp, vp, vp, vp, vp]),
    "sf_cgd_direction": (i32, [vp, vp, vp, vp, vp, vp]),
    "sf_mg_create": (i32, [C.POINTER(vp), vp, i32, C.POINTER(vp), C.POINTER(vp), vp]),
    "sf_mg_destroy": (i32, [vp]),
    "sf_mg_last_error": (C.c_char_p, [vp]),
    "sf_mg_set_option": (i32, [vp, C.c_char_p, C.c_double]),
    "sf_mg_get_info": (i32, [vp, C.c_char_p, dp]),
    "sf_mg_cg": (i32, [vp, i32, vp, vp, C.c_double, i32, C.POINTER(i32), dp, vp]),
    "sf_mg_refresh": (i32, [vp, vp]),
}

SF_NOALLOC_MAX_FREE = 262144

SF_CGD_SCALARS = 16
SF_CGD_RR = 3
SF_CGD_BB = 4
SF_CGD_DONE = 5
SF_CGD_ITERS = 6

for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class SumFacError(RuntimeError):
    """A failed library call; ``status`` is the SF_ERR_* code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int, handle=None, what: str = "") -> None:
    if status == SF_OK:
        return
    msg = ""
    if handle is not None:
        raw = lib.sf_last_error(handle)
        msg = raw.decode() if raw else ""
    text = lib.sf_status_string(status).decode()
    raise SumFacError(status, f"{what}: {text}" + (f" ({msg})" if msg else ""))
