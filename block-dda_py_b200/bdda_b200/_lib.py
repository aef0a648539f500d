"""ctypes binding of libbdda.so (the C ABI declared in include/bdda.h).

The library is built in-tree by ``block-dda_py_b200/csrc/build.py``.  There is
no fallback: if the shared object is missing, or no CUDA device is visible,
every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libbdda.so")

# status codes (include/bdda.h: enum bdda_status)
OK, NOT_CONVERGED, BREAKDOWN, BAD_ARG, NO_WORKSPACE, TIMEOUT, CUDA_ERROR = range(7)
# precisions (include/bdda.h: enum bdda_precision)
C128, C64 = 0, 1
# batched solve modes (include/bdda.h: enum bdda_batch_mode)
BATCH_C128, BATCH_C64, BATCH_MIXED = 0, 1, 2
# solvers (include/bdda.h: enum bdda_solver_kind)
BICGSTAB, COCG_RQ = 0, 1

_vp = C.c_void_p
_sz = C.c_size_t
_i = C.c_int
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pd = C.POINTER(C.c_double)

# name -> (restype, argtypes).  Every symbol of include/bdda.h is listed here;
# tests check the two lists against each other.
PROTOTYPES = {
    "bdda_status_string": (C.c_char_p, [_i]),
    "bdda_gre_occupancy_workspace_bytes": (_sz, [_i, _i, _i]),
    "bdda_dda_workspace_bytes": (_sz, [_vp, _i, _i, _i]),
    "bdda_dda_solve": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _d, _i, _i, _vp, _vp, _vp, _vp, _pi, _pd, _pd,
                            _vp, _sz, _vp]),
    "bdda_gre_occupancy": (_i, [_i, _i, _i, _vp, _vp, _vp, _i, _vp, _vp, _i, _i, _i, _d, _d, _d, _d, _d, _vp, _vp,
                                _vp, _sz, _vp]),
    "bdda_version": (_i, []),
    "bdda_tune_set": (_i, [_i, _i, _sz, _i]),
    "bdda_tune_get": (_i, [_i, _i, C.POINTER(_sz), _pi]),
    "bdda_tune_fixed": (_i, [_i]),
    "bdda_tune_pass": (_i, [_i, _i, _i, _i, _i, _i]),
    "bdda_batch_workspace_bytes": (_sz, [_vp, _i, _i, _i, _i]),
    "bdda_mixed_workspace_bytes": (_sz, [_vp, _i, _i]),
    "bdda_tune_mixed": (_i, [_d, _d, _d]),
    "bdda_tune_solver_graphs": (_i, [_i]),
    "bdda_tune_mixed_get": (_i, [_pd, _pd, _pd]),
    "bdda_fno_param_count": (_sz, [_vp]),
    "bdda_fno_offset": (_sz, [_vp, _i, _i]),
    "bdda_fno_workspace_bytes": (_sz, [_vp, _i, _pi]),
    "bdda_fno_buffer_offset": (_sz, [_vp, _i, _pi, _i]),
    "bdda_fno_features": (_i, [_vp, _pi, _i, _i, _vp, _vp, _vp, _pd, _vp, _vp, _sz, _vp]),
    "bdda_fno_forward": (_i, [_vp, _i, _pi, _vp, _i, _vp, _sz, _vp]),
    "bdda_fno_loss": (_i, [_vp, _i, _pi, _i, _vp, _vp, _vp, _vp, _vp, _pd, _vp, _sz, _vp]),
    "bdda_fno_backward": (_i, [_vp, _i, _pi, _vp, _vp, _vp, _vp, _sz, _vp]),
    "bdda_fno_adam": (_i, [_vp, _vp, _vp, _vp, _sz, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, _i, _vp]),
    "bdda_fno_warm_start": (_i, [_vp, _pi, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "bdda_mixed_solve": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _d, _i, _i, _vp, _pi, _pd, _pd,
                              _vp, _sz, _vp]),
    "bdda_batch_bicgstab": (_i, [_vp, _i, _i, _i, _d, _i, _i, _i, _pi, _pi, _pd, _pd, _vp, _sz, _vp]),
    "bdda_tune_pass_get": (_i, [_i, _i, _i, _i, _pi, _pi]),
    "bdda_tune_pass_variants": (_i, [_vp, _i, _i, _i, _i, _pi, _i, _pi]),
    "bdda_autotune": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _pd, _pd, _vp]),
    "bdda_plan_create": (_i, [_pi, _pi, C.POINTER(_vp)]),
    "bdda_plan_destroy": (None, [_vp]),
    "bdda_plan_grid": (_i, [_vp, _pi]),
    "bdda_plan_radices": (_i, [_vp, _i, _pi, _pi]),
    "bdda_plan_table_bytes": (_sz, [_vp]),
    "bdda_plan_attach_tables": (_i, [_vp, _vp, _vp]),
    "bdda_plan_wait_timeouts": (_i, [_vp, C.POINTER(C.c_uint), _vp]),
    "bdda_green_bytes": (_sz, [_vp, _i]),
    "bdda_green_build_workspace_bytes": (_sz, [_vp]),
    "bdda_green_build": (_i, [_vp, _d, _d, _vp, _vp, _vp]),
    "bdda_green_real": (_i, [_vp, _d, _d, _vp, _vp]),
    "bdda_green_convert": (_i, [_vp, _vp, _vp, _vp]),
    "bdda_green_export": (_i, [_vp, _vp, _vp, _vp]),
    "bdda_green_import": (_i, [_vp, _vp, _vp, _vp]),
    "bdda_mvp_workspace_bytes": (_sz, [_vp, _i, _i]),
    "bdda_occupancy_map": (_i, [_vp, _vp, _i, _vp, _vp]),
    "bdda_fft_mvp": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp]),
    "bdda_block_mvp": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bdda_block_mvp_noalloc_max_bytes": (_sz, []),
    "bdda_block_mvp_noalloc_fits": (_i, [_vp, _i, _i]),
    "bdda_block_mvp_noalloc": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bdda_solver_workspace_bytes": (_sz, [_vp, _i, _i, _i, _i]),
    "bdda_refine_workspace_bytes": (_sz, [_vp, _i, _i]),
    "bdda_refine_solve": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _d, _i, _d, _i, _vp, _pi,
                               C.POINTER(_d), C.POINTER(_d), _vp, _sz, _vp]),
    "bdda_polarizability": (_i, [_i, C.POINTER(_d), _d, _d, _d, _vp, _vp, _vp]),
    "bdda_incident_rhs": (_i, [_i, _i, _d, _vp, _vp, _vp, _vp, _vp]),
    "bdda_observables_workspace_bytes": (_sz, [_i]),
    "bdda_launch_count": (C.c_ulonglong, []),
    "bdda_profile_enable": (_i, [_i]),
    "bdda_profile_read": (_i, [_i, C.POINTER(_d), C.POINTER(C.c_longlong)]),
    "bdda_observables": (_i, [_i, _i, _d, _d, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bdda_solve": (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _d, _i, _vp, _pi,
                        C.POINTER(_d), C.POINTER(_d), _vp, _sz, _vp]),
    "bdda_bicgstab": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _d, _i, _vp, _pi,
                           C.POINTER(_d), C.POINTER(_d), _vp, _sz, _vp]),
    "bdda_cocg_rq": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _d, _i, _vp, _pi,
                          C.POINTER(_d), C.POINTER(_d), _vp, _sz, _vp]),
}


class BddaError(RuntimeError):
    """A libbdda call returned a failure status."""

    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__("%s: %s (status %d)" % (where, status_string(status), status))


_lock = threading.Lock()
_lib = None


def load() -> C.CDLL:
    """Load libbdda.so once and bind the prototypes; raise if it is absent."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    "libbdda.so not found at %s; build it with "
                    "`python block-dda_py_b200/csrc/build.py`" % LIB_PATH)
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in PROTOTYPES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def status_string(status: int) -> str:
    return load().bdda_status_string(status).decode()


def check(status: int, where: str) -> int:
    """Raise for any status other than OK / NOT_CONVERGED."""
    if status in (OK, NOT_CONVERGED):
        return status
    if status == BAD_ARG:
        raise ValueError("%s: %s" % (where, status_string(status)))
    if status == BREAKDOWN:
        raise np.linalg.LinAlgError("%s: %s" % (where, status_string(status)))
    raise BddaError(status, where)


def int3(values) -> C.Array:
    arr = (C.c_int * 3)()
    for i, v in enumerate(values):
        arr[i] = int(v)
    return arr
