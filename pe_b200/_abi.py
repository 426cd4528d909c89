"""ctypes binding of the C ABI in include/pe_b200.h (libpe_b200.so, built in-tree).

There is no fallback: if the shared library is missing or CUDA is unavailable, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpe_b200.so")

OK = 0
ERR_ARG, ERR_CAPACITY, ERR_NAN, ERR_TIMEOUT, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_UNSUPPORTED = range(1, 9)
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CAPACITY", 3: "ERR_NAN", 4: "ERR_TIMEOUT",
                5: "ERR_CUDA", 6: "ERR_STATE", 7: "ERR_NOMEM", 8: "ERR_UNSUPPORTED"}

DEM, HCSITS = 0, 1
FP64, MIXED = 0, 1
# pe's RelaxationModel (HardContactSemiImplicitTimesteppingSolvers.h:172-179)
INELASTIC_FRICTIONLESS, APPROX_INELASTIC_COULOMB_DECOUPLING = 0, 1
APPROX_INELASTIC_COULOMB_ORTHOGONAL_PROJECTIONS, INELASTIC_COULOMB_DECOUPLING = 2, 3
INELASTIC_COULOMB_ORTHOGONAL_PROJECTIONS, INELASTIC_GENERALIZED_MAX_DISSIPATION = 4, 5

# every symbol include/pe_b200.h declares
EXPORTS = ["pe_b200_default_params", "pe_b200_create", "pe_b200_destroy", "pe_b200_last_error",
           "pe_b200_set_gravity", "pe_b200_set_damping", "pe_b200_set_max_iterations",
           "pe_b200_set_relaxation_model", "pe_b200_set_error_reduction",
           "pe_b200_set_materials", "pe_b200_set_walls", "pe_b200_upload_bodies",
           "pe_b200_set_state", "pe_b200_set_orientations", "pe_b200_release_memory", "pe_b200_step", "pe_b200_download_bodies",
           "pe_b200_find_contacts", "pe_b200_last_step_stats", "pe_b200_set_residual",
           "pe_b200_kernel_launches", "pe_b200_stream", "pe_b200_set_profiling",
           "pe_b200_profile", "pe_b200_dem_step_static", "pe_b200_neighbor_list_stats",
           "pe_b200_adjoint_forward", "pe_b200_adjoint_backward", "pe_b200_set_graph_steps",
           "pe_b200_graph_active", "pe_b200_graph_stats", "pe_b200_get_tuning", "pe_b200_set_tuning",
           "pe_b200_autotune", "pe_b200_validate", "pe_b200_selftest_timeout",
           "pe_b200_upload_boxes", "pe_b200_download_boxes", "pe_b200_box_count"]

STATIC_MAX_SPHERES = 32768
STATIC_MAX_CELLS = 131072


class Params(C.Structure):
    _fields_ = [("solver", C.c_int32), ("precision", C.c_int32), ("relaxation_model", C.c_int32),
                ("max_iterations", C.c_int32), ("erp", C.c_double),
                ("gravity", C.c_double * 3), ("damping", C.c_double), ("device", C.c_int32),
                ("track_orientation", C.c_int32), ("max_contacts", C.c_int64),
                ("skin", C.c_double), ("neighbor_lists", C.c_int32), ("force_model", C.c_int32)]


class Material(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("density", "cor", "csf", "cdf", "poisson", "young",
                                          "stiffness", "dampingN", "dampingT")]


class Tuning(C.Structure):
    _fields_ = [("dem_variant", C.c_int32), ("rebuild_per_sm", C.c_int32), ("skin", C.c_double),
                ("ms_per_step", C.c_double), ("variants", C.c_int32), ("nbgs_sweeps", C.c_int32),
                ("dem_grid", C.c_int32), ("dem_split", C.c_int32)]


class PeB200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Loads libpe_b200.so; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pe_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dp = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    P = C.POINTER
    sig = {
        "pe_b200_default_params": (None, [P(Params)]),
        "pe_b200_create": (C.c_int, [P(Params), P(vp)]),
        "pe_b200_destroy": (C.c_int, [vp]),
        "pe_b200_last_error": (C.c_char_p, [vp]),
        "pe_b200_set_gravity": (C.c_int, [vp, P(dp)]),
        "pe_b200_set_damping": (C.c_int, [vp, dp]),
        "pe_b200_set_max_iterations": (C.c_int, [vp, i32]),
        "pe_b200_set_relaxation_model": (C.c_int, [vp, i32]),
        "pe_b200_set_error_reduction": (C.c_int, [vp, dp]),
        "pe_b200_set_materials": (C.c_int, [vp, i32, P(Material)]),
        "pe_b200_set_walls": (C.c_int, [vp, i32, i32, vp, vp, i32, vp, vp]),
        "pe_b200_upload_bodies": (C.c_int, [vp, i64, vp, vp, vp, vp, vp, vp, i32]),
        "pe_b200_set_state": (C.c_int, [vp, vp, vp, vp]),
        "pe_b200_set_orientations": (C.c_int, [vp, vp]),
        "pe_b200_release_memory": (C.c_int, [i32]),
        "pe_b200_step": (C.c_int, [vp, i32, dp]),
        "pe_b200_download_bodies": (C.c_int, [vp, vp, vp, vp, vp]),
        "pe_b200_find_contacts": (C.c_int, [vp, i64, vp, vp, P(i64)]),
        "pe_b200_last_step_stats": (C.c_int, [vp, P(i64), P(i32), P(dp), P(dp)]),
        "pe_b200_set_residual": (C.c_int, [vp, i32]),
        "pe_b200_kernel_launches": (i64, [vp]),
        "pe_b200_set_profiling": (C.c_int, [vp, i32]),
        "pe_b200_neighbor_list_stats": (C.c_int, [vp, P(i64), P(i64), P(i64), P(dp)]),
        "pe_b200_adjoint_forward": (C.c_int, [vp, i32, dp, i32]),
        "pe_b200_adjoint_backward": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "pe_b200_set_graph_steps": (C.c_int, [vp, i32]),
        "pe_b200_graph_active": (C.c_int, [vp]),
        "pe_b200_graph_stats": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "pe_b200_get_tuning": (C.c_int, [vp, P(Tuning)]),
        "pe_b200_set_tuning": (C.c_int, [vp, P(Tuning)]),
        "pe_b200_autotune": (C.c_int, [vp, dp, i32, P(Tuning)]),
        "pe_b200_validate": (C.c_int, [vp, P(i64)]),
        "pe_b200_upload_boxes": (C.c_int, [vp, i32, vp, vp, vp, vp, vp, vp, vp]),
        "pe_b200_download_boxes": (C.c_int, [vp, vp, vp, vp, vp]),
        "pe_b200_box_count": (i32, [vp]),
        "pe_b200_selftest_timeout": (C.c_int, [vp, i64]),
        "pe_b200_profile": (C.c_int, [vp, i32, P(C.c_char_p), P(dp), P(i64), P(i32)]),
        "pe_b200_stream": (vp, [vp]),
        "pe_b200_dem_step_static": (C.c_int, [i64, vp, vp, vp, vp, vp, i32, P(Material), i32, vp,
                                              vp, i32, vp, vp, P(dp), dp, dp, P(dp), P(dp), dp,
                                              vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def default_params() -> Params:
    p = Params()
    load().pe_b200_default_params(C.byref(p))
    return p
