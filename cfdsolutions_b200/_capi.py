"""ctypes binding of ``include/cfd_b200.h`` (the library's C ABI).

The shared library is the in-tree ``_lib/libcfd_b200.so`` built by
:mod:`cfdsolutions_b200.build`.  There is no fallback: if it is missing or
fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libcfd_b200.so"

CFD_OK = 0
ERRORS = {
    -1: "CFD_ERR_ARG", -2: "CFD_ERR_MESH", -3: "CFD_ERR_CUDA", -4: "CFD_ERR_IO", -5: "CFD_ERR_STATE",
    -6: "CFD_ERR_NUMERIC", -7: "CFD_ERR_NOT_CONVERGED", -8: "CFD_ERR_UNSUPPORTED", -9: "CFD_ERR_RANGE",
}
FLUX_ROE, FLUX_HLLC, FLUX_AUSM, FLUX_ROE_LMFIX, FLUX_ROE_PRECOND, FLUX_ROE_THORNBER, FLUX_VANLEER = 0, 1, 2, 3, 4, 5, 6
PRECOND_BTW, PRECOND_ERIKSSON, PRECOND_TURKEL = 2, 3, 5
PRECOND_LOCAL, PRECOND_GLOBAL, PRECOND_URLOCAL = 0, 1, 2
ORDER_FIRST, ORDER_SECOND = 0, 1
LIMITER_NONE, LIMITER_BJ, LIMITER_VENKAT = -1, 0, 1
GRAD_LSQ, GRAD_GG = 0, 1
PREC_FP64, PREC_FP32, PREC_BF16 = 0, 1, 2
PC_NONE, PC_BLOCK_JACOBI, PC_ILU0, PC_ILU0_MC = 0, 1, 2, 3
PREC_LOW_ONLY = 0x10
JAC_CENTRAL, JAC_FORWARD, JAC_BACKWARD, JAC_ALTERNATE = 0, 1, 2, 3
RMSFILE_EULER3D, RMSFILE_MPFLOW3D = 0, 1
VARS_CONSERVATIVE, VARS_RUP, VARS_PUT, VARS_RUT = 0, 1, 2, 3
BC_EULER_WALL, BC_FAR_FIELD, BC_INFLOW, BC_OUTFLOW = 0, 1, 2, 3
GS_STATIC_MAX_ROWS = 16384
PENDING = 1


class CfdError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("flux_scheme", C.c_int), ("order", C.c_int), ("limiter", C.c_int), ("limiter_order", C.c_int),
        ("limiter_smooth", C.c_int), ("gradient", C.c_int), ("ls_weight", C.c_int), ("entropy_fix", C.c_int),
        ("global_time", C.c_int), ("cfl_ramp", C.c_int), ("mach_ramp", C.c_int), ("zpg_iteration", C.c_int),
        ("gamma", C.c_double), ("mach", C.c_double), ("mach_min", C.c_double), ("alpha_deg", C.c_double),
        ("beta_deg", C.c_double), ("cfl_min", C.c_double), ("cfl_max", C.c_double), ("venkat_k", C.c_double),
        ("residual_kernel", C.c_int), ("pinf", C.c_double), ("precond_method", C.c_int), ("precond_type", C.c_int),
        ("precond_mach", C.c_double), ("outflow_pressure", C.c_double), ("variables", C.c_int),
    ]


class GmresOpts(C.Structure):
    _fields_ = [("restart", C.c_int), ("max_iters", C.c_int), ("rtol", C.c_double), ("precond", C.c_int),
                ("precision", C.c_int), ("refine", C.c_int), ("reuse_precond", C.c_int)]


class GmresStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("restarts", C.c_int), ("refinements", C.c_int),
                ("rel_residual", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("drop", C.c_double), ("include_diss", C.c_int),
                ("linear_solver", C.c_int), ("linear_iters", C.c_int), ("relax", C.c_double),
                ("gmres", GmresOpts), ("precond_update", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("rms_first", C.c_double), ("rms_last", C.c_double),
                ("linear_iterations", C.c_int), ("status", C.c_int)]


class UnsteadyOpts(C.Structure):
    _fields_ = [("dt", C.c_double), ("steps", C.c_int), ("inner_iterations", C.c_int), ("bdf2", C.c_int),
                ("include_diss", C.c_int), ("linear_solver", C.c_int), ("linear_iters", C.c_int),
                ("relax", C.c_double), ("gmres", GmresOpts)]


class UnsteadyStats(C.Structure):
    _fields_ = [("steps", C.c_int), ("inner_iterations", C.c_int), ("rms_last", C.c_double),
                ("linear_iterations", C.c_int), ("status", C.c_int)]


class ServeRequest(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("lx", C.c_double), ("ly", C.c_double),
                ("lz", C.c_double), ("jitter", C.c_double), ("mesh_seed", C.c_uint64), ("numbering", C.c_int),
                ("face_bc", C.c_int * 6), ("noise", C.c_double), ("state_seed", C.c_uint64), ("params", Params),
                ("opts", SolveOpts), ("keep_state", C.c_int)]


class ServeResult(C.Structure):
    _fields_ = [("status", C.c_int), ("stats", SolveStats), ("nnode", C.c_int), ("nghost", C.c_int),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_start_solve", C.c_double),
                ("t_done", C.c_double), ("bytes_estimate", C.c_double), ("message", C.c_char * 160)]


P = C.c_void_p
I = C.c_int
I64 = C.c_int64
D = C.c_double
dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

# name -> (restype, argtypes); every function declared in include/cfd_b200.h
SIGNATURES = {
    "cfd_abi_version": (I, []),
    "cfd_last_error": (C.c_char_p, []),
    "cfd_params_default": (None, [C.POINTER(Params)]),
    "cfd_create": (I, [I, C.POINTER(P)]),
    "cfd_destroy": (I, [P]),
    "cfd_set_stream": (I, [P, P]),
    "cfd_set_params": (I, [P, C.POINTER(Params)]),
    "cfd_synchronize": (I, [P]),
    "cfd_set_mesh": (I, [P, I, I, I, P, P, I, P, P, P, P, P, P, P]),
    "cfd_get_block_pattern": (I, [P, C.POINTER(I64), P, P, P]),
    "cfd_set_state": (I, [P, P]),
    "cfd_get_state": (I, [P, P]),
    "cfd_state_device_ptr": (I, [P, C.POINTER(P), C.POINTER(I64)]),
    "cfd_set_freestream": (I, [P]),
    "cfd_begin_iteration": (I, [P, I]),
    "cfd_apply_bc": (I, [P, I]),
    "cfd_gradient": (I, [P]),
    "cfd_limiter": (I, [P]),
    "cfd_residual": (I, [P, I]),
    "cfd_deltat": (I, [P, I]),
    "cfd_residual_rms": (I, [P, I, P]),
    "cfd_jacobian": (I, [P, I, I, I]),
    "cfd_block_gs": (I, [P, I, I, C.POINTER(D)]),
    "cfd_block_lusgs": (I, [P, I, C.POINTER(D)]),
    "cfd_jacobian_fd": (I, [P, I, I, I, I]),
    "cfd_block_gs_static": (I, [I, P, P, P, P, P, P, I, I, P, C.POINTER(D)]),
    "cfd_ilu_mc_order": (I, [P, P, C.POINTER(I)]),
    "cfd_gmres_default": (None, [C.POINTER(GmresOpts)]),
    "cfd_gmres": (I, [P, C.POINTER(GmresOpts), C.POINTER(GmresStats)]),
    "cfd_spmv": (I, [P, I, P, P]),
    "cfd_rms_file_open": (I, [C.c_char_p, I, I, I, C.POINTER(P)]),
    "cfd_rms_file_write": (I, [P, I, P, P, P]),
    "cfd_rms_file_write_ctx": (I, [P, P, I, I]),
    "cfd_rms_file_close": (I, [P]),
    "cfd_precond_apply": (I, [P, P, P]),
    "cfd_update": (I, [P, D]),
    "cfd_get_residual": (I, [P, P, P]),
    "cfd_get_deltat": (I, [P, P]),
    "cfd_get_extrema": (I, [P, P]),
    "cfd_get_farfield": (I, [P, P]),
    "cfd_set_farfield": (I, [P, P]),
    "cfd_get_gradients": (I, [P, P]),
    "cfd_get_limiters": (I, [P, P]),
    "cfd_get_system": (I, [P, P, P, P]),
    "cfd_set_system": (I, [P, P, P]),
    "cfd_residual_step": (I, [P, I, P, P, P]),
    "cfd_set_step_pipeline": (I, [P, I]),
    "cfd_solve_steady": (I, [P, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "cfd_solve_unsteady": (I, [P, C.POINTER(UnsteadyOpts), C.POINTER(UnsteadyStats)]),
    "cfd_vtk_write": (I, [C.c_char_p, I, P, C.c_int64, P, P, C.c_int64, P, C.POINTER(Params), P, C.c_int64]),
    "cfd_mesh_box": (I, [I, I, I, D, D, D, D, C.c_uint64, I, P, C.POINTER(P)]),
    "cfd_mesh_from_cells": (I, [I, P, I64, P, I64, P, P, C.POINTER(P)]),
    "cfd_mesh_sizes": (I, [P, P]),
    "cfd_mesh_export": (I, [P, P, P, P, P, P, P, P, P, P]),
    "cfd_mesh_export_cells": (I, [P, P, P, P]),
    "cfd_mesh_write_ugrid": (I, [P, C.c_char_p]),
    "cfd_mesh_read_ugrid": (I, [C.c_char_p, I, P, I, C.POINTER(P)]),
    "cfd_set_mesh_from": (I, [P, P]),
    "cfd_mesh_free": (None, [P]),
    "cfd_perturbed_freestream": (I, [P, D, D, D, D, D, C.c_uint64, P]),
    "cfd_initial_state": (I, [P, P, P, C.c_uint64, P]),
    "cfd_server_create": (I, [I, I, D, C.POINTER(P)]),
    "cfd_server_submit": (I, [P, C.POINTER(ServeRequest), C.POINTER(I64)]),
    "cfd_server_wait": (I, [P, I64, D, C.POINTER(ServeResult)]),
    "cfd_server_state": (I, [P, I64, P]),
    "cfd_server_release": (I, [P, I64]),
    "cfd_server_stats": (I, [P, P]),
    "cfd_server_set_batching": (I, [P, I, D]),
    "cfd_server_batch_stats": (I, [P, P]),
    "cfd_server_destroy": (I, [P]),
    "cfd_restart_write": (I, [C.c_char_p, I, I, I, P]),
    "cfd_restart_read": (I, [C.c_char_p, C.POINTER(I), I, I, P]),
}


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python cfdsolutions_b200/build.py`")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(code: int, where: str) -> None:
    if code != CFD_OK:
        raise CfdError(code, where, lib.cfd_last_error().decode(errors="replace"))


def ptr(a: np.ndarray | None):
    """Raw pointer of a C-contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays crossing the C ABI must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)
