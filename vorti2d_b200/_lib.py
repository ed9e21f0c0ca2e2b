"""ctypes binding of libvorti2d_b200.so (the C ABI in include/vorti2d_b200.h).

The shared library is built in-tree by ``vorti2d_b200.build``.  There is no
CPU fallback: if the library is missing or cannot be loaded, every entry point
raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libvorti2d_b200.so")

V2D_OK = 0
V2D_EARG = -1
V2D_ECAPACITY = -2
V2D_ECUDA = -3
V2D_ENONFINITE = -4
V2D_ENOTCONVERGED = -5
V2D_ETIMEOUT = -6
V2D_EBREAKDOWN = -7
V2D_ENOMEM = -8

PC_NONE, PC_BJACOBI, PC_LU = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_ll = ctypes.c_longlong


class KrylovParams(ctypes.Structure):
    _fields_ = [("restart", _i), ("max_it", _i), ("rtol", _d), ("atol", _d),
                ("precond", _i), ("precision", _i), ("inner_rtol", _d), ("dc_max_it", _i),
                ("lu_leaf", _i), ("lu_reuse_its", _i), ("lu_reuse_steps", _i),
                ("lu_solve", _i), ("lu_factor64", _i)]


class LinStats(ctypes.Structure):
    _fields_ = [("iterations", _i), ("restarts", _i), ("corrections", _i),
                ("converged", _i), ("res0", _d), ("res", _d)]


class SolverParams(ctypes.Structure):
    _fields_ = [("re", _d), ("invdtau", _d), ("inv2dt", _d), ("ca", _d), ("sa", _d),
                ("ff_bc", _i), ("krylov", KrylovParams)]


class NewtonInfo(ctypes.Structure):
    _fields_ = [("newton_iters", _i), ("krylov_iters", _i), ("corrections", _i),
                ("res", _d), ("lin_res_max", _d)]


class V2DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vorti2d_b200 error {code}: {msg}")
        self.code = code


class NotConvergedError(V2DError):
    pass


_SIGS = {
    "v2d_last_error": (ctypes.c_char_p, []),
    "v2d_version": (_i, []),
    "v2d_launch_count": (_ll, []),
    "v2d_node_neighbors": (_i, [_i, _i, _i, _ip]),
    "v2d_compute_metrics": (_i, [_i, _i, _d, _d, _dp, _dp] + [_dp] * 10),
    "v2d_compute_metrics_local": (_i, [_i, _i, _i, _i, _d, _d, _dp, _dp] + [_dp] * 10),
    "v2d_assemble_coo": (_i, [_i, _i] + [_d] * 6 + [_dp] * 14 + [_i] * 4 + [_d] * 2
                         + [_ip, _ip, _dp, _ip, _dp]),
    "v2d_assemble_coo_local": (_i, [_i] * 4 + [_d] * 6 + [_dp] * 14 + [_i, _i, _ip, _i, _i]
                               + [_d] * 2 + [_ip, _ip, _dp, _ip, _dp]),
    "v2d_compute_metrics_dev": (_i, [_i, _i, _d, _d, _vp, _vp, _vp, _vp]),
    "v2d_assemble_coo_noalloc": (_i, [_i, _i] + [_d] * 6 + [ctypes.POINTER(_vp)] + [_i] * 4
                                 + [_d] * 2 + [_vp, _vp, _vp, _ip, _vp, _vp]),
    "v2d_force_coeffs": (_i, [_i, _i, _d, _d, _d] + [_dp] * 7 + [_d, _d, _d, _dp]),
    "v2d_compute_velocity": (_i, [_i, _i, _d, _d] + [_dp] * 9),
    "v2d_solver_velocity": (_i, [_vp, _dp, _dp, _dp]),
    "v2d_solver_adjoint": (_i, [_vp, _d, _dp, _dp, _d, _i, _ip, _dp]),
    "v2d_solver_residual": (_i, [_vp, _d, _d, _d, _d, _d, _d, _dp]),
    "v2d_krylov_defaults": (None, [ctypes.POINTER(KrylovParams)]),
    "v2d_linsys_create": (_i, [_i, _i, ctypes.POINTER(KrylovParams), ctypes.POINTER(_vp)]),
    "v2d_linsys_assemble": (_i, [_vp, _ip, _ip, _dp, _ll, _dp]),
    "v2d_linsys_set_grid": (_i, [_vp, _i, _i]),
    "v2d_linsys_solve": (_i, [_vp, _dp, ctypes.POINTER(LinStats)]),
    "v2d_linsys_nnz": (_i, [_vp, ctypes.POINTER(_ll)]),
    "v2d_linsys_csr": (_i, [_vp, _ip, _ip, _dp]),
    "v2d_linsys_destroy": (_i, [_vp]),
    "v2d_solver_create": (_i, [_i, _i, _dp, _dp, ctypes.POINTER(SolverParams),
                               ctypes.POINTER(_vp)]),
    "v2d_solver_destroy": (_i, [_vp]),
    "v2d_solver_set_params": (_i, [_vp, ctypes.POINTER(SolverParams)]),
    "v2d_solver_set_state": (_i, [_vp, _dp, _dp, _dp, _dp]),
    "v2d_solver_get_state": (_i, [_vp, _dp, _dp, _dp, _dp]),
    "v2d_solver_get_metrics": (_i, [_vp, ctypes.POINTER(_dp)]),
    "v2d_solver_newton": (_i, [_vp, _d, _dp, ctypes.POINTER(LinStats)]),
    "v2d_solver_pseudo_solve": (_i, [_vp, _d, _d, _i, ctypes.POINTER(NewtonInfo)]),
    "v2d_solver_shift_history": (_i, [_vp]),
    "v2d_solver_step": (_i, [_vp, _d, _d, _i, _i, ctypes.POINTER(NewtonInfo)]),
    "v2d_solver_forces": (_i, [_vp, _d, _d, _d, _d, _dp]),
    "v2d_solver_nnz": (_i, [_vp, ctypes.POINTER(_ll)]),
    "v2d_solver_assemble": (_i, [_vp, _d]),
    "v2d_solver_export_system": (_i, [_vp, _ip, _ip, _dp, _dp]),
    "v2d_solver_state_ptrs": (_i, [_vp] + [ctypes.POINTER(_vp)] * 4),
    "v2d_solver_stream": (_i, [_vp, ctypes.POINTER(_vp)]),
    "v2d_batch_create": (_i, [_i, _ip, _ip, ctypes.POINTER(_dp), ctypes.POINTER(_dp),
                              ctypes.POINTER(SolverParams), ctypes.POINTER(_vp)]),
    "v2d_batch_destroy": (_i, [_vp]),
    "v2d_batch_set_active": (_i, [_vp, _ip]),
    "v2d_batch_newton": (_i, [_vp, _dp, _ip, ctypes.POINTER(LinStats)]),
    "v2d_batch_instance": (_i, [_vp, _i, ctypes.POINTER(_vp)]),
    "v2d_batch_factorizations": (_i, [_vp, ctypes.POINTER(_ll)]),
    "v2d_solver_time_spmv": (_i, [_vp, _i, _i, _ll, _dp]),
    "v2d_solver_phase_times": (_i, [_vp, _dp, _i]),
    "v2d_solver_time_kernel": (_i, [_vp, _i, _i, _ll, _dp]),
    "v2d_solver_time_lu_launches": (_i, [_vp, _i, _ll, _dp, _ip, _i, _ip]),
    "v2d_solver_time_lu_factor": (_i, [_vp, _i, _dp, _ip, _i, _ip]),
    "v2d_solver_lu_stats": (_i, [_vp, _dp]),
    "v2d_solver_lu_split": (_i, [_vp, _i, _ip]),
    "v2d_solver_residual_mesh": (_i, [_vp, _dp, _dp, _d, _d, _d, _d, _d, _d, _dp, _i, _dp]),
    "v2d_solver_trace_lu_apply": (_i, [_vp, ctypes.POINTER(ctypes.c_ulonglong), _ip, _i, _ip]),
    "v2d_solver_lu_flow_form": (_i, [_vp, _i, _ip]),
    "v2d_solver_lu_item_rows": (_i, [_vp, _ip, _i, _ip, _i, _ip]),
    "v2d_solver_shape_tangent": (_i, [_vp, _dp, _dp, _dp, _dp, _d, _d, _d, _d, _d, _d, _d, _d,
                                      _d, _dp, _dp]),
    "v2d_solver_shape_gradient": (_i, [_vp, _dp, _dp, _dp, _dp, _d, _d, _d, _d, _d, _d, _d, _d,
                                       _d, _d, _dp, _dp]),
    "v2d_solver_time_lu_apply": (_i, [_vp, _i, _ll, _dp, ctypes.POINTER(_ll)]),
    "v2d_lu_plan_info": (_i, [_i, _i, _ip, _ip, _i, ctypes.POINTER(_ll)]),
    "v2d_lu_solve_plan": (_i, [_i, _i, _ip, _ip, _i, _ip, _ip, _i, _ip, _i]),
    "v2d_lu_solve_plan_split": (_i, [_i, _i, _ip, _ip, _i, _ip, _i, _ip, _ip, _i, _ip, _i]),
}

_LIB = None


def lib():
    """Load the library once; raises RuntimeError if it is missing."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libvorti2d_b200.so not found at {LIB_PATH}; build it with "
                "`python -m vorti2d_b200.build` (CUDA toolkit, sm_100a). "
                "There is no CPU fallback.")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def exported_symbols():
    return list(_SIGS)


def last_error() -> str:
    return lib().v2d_last_error().decode(errors="replace")


def check(code: int, what: str = ""):
    if code == V2D_OK:
        return
    msg = last_error()
    if what:
        msg = f"{what}: {msg}"
    if code == V2D_EARG:
        raise ValueError(msg)
    if code == V2D_ENOTCONVERGED:
        raise NotConvergedError(code, msg)
    raise V2DError(code, msg)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def krylov_defaults() -> KrylovParams:
    p = KrylovParams()
    lib().v2d_krylov_defaults(ctypes.byref(p))
    return p
