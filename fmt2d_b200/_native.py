"""ctypes binding of the C ABI in include/fmt2d_gpu.h.

The shared library is built in-tree (fmt2d_b200/_lib/libfmt2d_b200.so) by
`fmt2d_b200.build.build()`.  There is no fallback: if the library is missing
or fails to load, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfmt2d_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "fmt2d_gpu.h")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class ModelDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("nzs", C.c_int), ("xpos", C.c_void_p), ("topo", C.c_void_p),
                ("zrel", C.c_void_p), ("vel", C.c_void_p), ("vwater", C.c_double),
                ("sed_z", C.c_void_p), ("moho_z", C.c_void_p), ("iface_inv", C.c_int)]


class LsqrParams(C.Structure):
    _fields_ = [("smooth_type", C.c_int), ("max_iter", C.c_int), ("wdv", C.c_double),
                ("wdv_iface", C.c_double), ("w_smooth", C.c_double),
                ("w_smooth_iface", C.c_double), ("eps_min", C.c_double)]


class Fmt2dError(RuntimeError):
    """A library call failed; `code` is its FMT2D_ERR_* status."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


class Fmt2dNotConverged(Fmt2dError):
    """fmt2d_forward returned FMT2D_ERR_CONVERGE: a time field did not reach
    its fixed point (nodes still moving after the last check, or the step cap
    reached)."""


ERR_CONVERGE = -5


def header_symbols() -> list[str]:
    """Every function the C header declares."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"FMT2D_API\s+int\s+(fmt2d_\w+)\s*\(", txt)))


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise Fmt2dError(f"native library not built: {LIB_PATH} (run fmt2d_b200.build.build())")
    L = C.CDLL(LIB_PATH)
    V = C.c_void_p
    P = C.POINTER
    L.fmt2d_ctx_create.argtypes = [P(V), C.c_int]
    L.fmt2d_ctx_destroy.argtypes = [V]
    L.fmt2d_last_error.argtypes = [V, C.c_char_p, C.c_int]
    L.fmt2d_upload_model.argtypes = [V, P(ModelDesc)]
    L.fmt2d_model_info.argtypes = [V, P(C.c_int), P(C.c_int), P(C.c_double), P(C.c_double)]
    L.fmt2d_region_nodes.argtypes = [V, C.c_int, P(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p]
    L.fmt2d_region_geometry.argtypes = [V, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fmt2d_inv_index.argtypes = [V, C.c_void_p, P(C.c_int), P(C.c_int)]
    L.fmt2d_forward.argtypes = [V, _dp, C.c_int, C.c_int]
    L.fmt2d_get_field.argtypes = [V, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fmt2d_stats.argtypes = [V, C.c_void_p, C.c_int]
    L.fmt2d_stream.argtypes = [V, P(V)]
    L.fmt2d_set_schedule.argtypes = [V, C.c_double, C.c_int, C.c_longlong]
    L.fmt2d_read_smesh.argtypes = [C.c_char_p, P(C.c_int), P(C.c_int), P(C.c_double),
                                   P(C.c_double)] + [C.c_void_p] * 4
    L.fmt2d_read_refl.argtypes = [C.c_char_p, P(C.c_int), C.c_void_p, C.c_void_p]
    L.fmt2d_read_geom.argtypes = [C.c_char_p, P(C.c_int), P(C.c_int)] + [C.c_void_p] * 8
    L.fmt2d_io_last_error.argtypes = [C.c_char_p, C.c_int]
    L.fmt2d_projection.argtypes = [V, C.c_int, C.c_int, C.c_int] + [P(C.c_int)] * 4 + \
        [C.c_void_p] * 4 + [P(C.c_longlong)]
    L.fmt2d_project_rows.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, P(C.c_longlong)]
    # npick, 7 input arrays, nparm, mvscale, crit_chi and 3 weights, 7 outputs
    L.fmt2d_select_data.argtypes = [C.c_int] + [C.c_void_p] * 7 + [C.c_int, C.c_void_p] + \
        [C.c_double] * 4 + [C.c_void_p] * 7
    L.fmt2d_gauss_smooth.argtypes = [V, C.c_int, C.c_double, C.c_double, C.c_double,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     P(C.c_longlong)]
    L.fmt2d_trace.argtypes = [V, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                              C.c_void_p, C.c_void_p, P(C.c_longlong)]
    L.fmt2d_frechet_rows.argtypes = [V, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    L.fmt2d_set_iface_window.argtypes = [V, C.c_double]
    L.fmt2d_trace_times.argtypes = [V, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p]
    L.fmt2d_set_frechet.argtypes = [V, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int]
    L.fmt2d_spmv.argtypes = [V, C.c_int, C.c_void_p, C.c_void_p]
    L.fmt2d_gtg_diag.argtypes = [V, C.c_void_p]
    L.fmt2d_lsqr.argtypes = [V, P(LsqrParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             P(C.c_int), P(C.c_double), P(C.c_double), P(C.c_double)]
    L.fmt2d_lsqr_noalloc.argtypes = [V, P(LsqrParams), C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, P(C.c_int), P(C.c_double), P(C.c_double),
                                     P(C.c_double)]
    L.fmt2d_lsqr_stats.argtypes = [V, P(C.c_double), P(C.c_int)]
    L.fmt2d_set_smoothing.argtypes = [V, C.c_double, C.c_double, C.c_double, C.c_void_p]
    L.fmt2d_model_velocity.argtypes = [V, C.c_void_p]
    L.fmt2d_model_interface.argtypes = [V, C.c_int, C.c_void_p]
    L.fmt2d_update_model.argtypes = [V, C.c_void_p, C.c_void_p]
    L.fmt2d_get_field_device.argtypes = [V, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fmt2d_forward_batch.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
    L.fmt2d_set_solve_threads.argtypes = [V, C.c_int]
    L.fmt2d_set_param_grid.argtypes = [V, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
    L.fmt2d_trace_entries.argtypes = [V, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fmt2d_misfit_gradient.argtypes = [V, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_int, P(C.c_double),
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]
    L.fmt2d_autotune.argtypes = [V, _dp, C.c_int, C.c_int, P(C.c_int), C.c_void_p]
    for name in header_symbols():
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
