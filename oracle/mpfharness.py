"""ctypes driver of the reference MPFLOW3D objects (``oracle/_ref/libmpflow3d_ref.so``).

Test infrastructure only (``tests/``): runs MPFLOW3D's own code on the same
mesh and state as the CUDA path.  Each session runs in a fresh ``spawn``-ed
process, because the reference keeps process-global and static state.

MPFLOW3D is run as its ideal-gas, non-dimensional configuration
(MATERIAL_TYPE_IDEALGAS, MATERIAL_COMP_TYPE_NDIM) with the freestream at the
reference pressure and temperature, which makes its non-dimensional
freestream rho = 1, p = 1, c = sqrt(1.4) (EOS/src/EOS_IdealGas.c:69-92,
MPFLOW3D/src/Material.cpp:196-245): the same scaling as the library's generic
non-dimensionalisation.  Its solution variables are VARIABLE_RUP
(rho, u, v, w, p); ``cons_to_rup`` / ``rup_to_cons`` convert states and
``jacobian_to_rup`` converts a conservative-variable Jacobian to its
RUP-variable form, so results compare field by field.

Parameter keys follow MPFLOW3D/src/SolverParameters.cpp:191-1050.
"""
from __future__ import annotations

import ctypes as C
import multiprocessing as mp
import os
import tempfile
import time
from pathlib import Path

import numpy as np

from oracle.refharness import _mesh_dict, _p, _quiet

HERE = Path(__file__).resolve().parent
MPF_LIB = HERE / "_ref" / "libmpflow3d_ref.so"
MPF_EXE = HERE / "_ref" / "mpflow3d"
GAMMA = 1.4  # MPFLOW3D hard-wires the ideal gas's gamma (MPFLOW3D/src/Material.cpp:130, EOS_IdealGas.c:73)

PRECOND = {None: "PRECOND_METHOD_NONE", 0: "PRECOND_METHOD_LMFIX", 1: "PRECOND_METHOD_THORNBER",
           2: "PRECOND_METHOD_BTW", 3: "PRECOND_METHOD_ERIKSSON", 5: "PRECOND_METHOD_TURKEL"}
PRECOND_TYPE = {0: "PRECOND_TYPE_LOCAL", 1: "PRECOND_TYPE_GLOBAL", 2: "PRECOND_TYPE_URLOCAL"}
LIMITER = {-1: "LIMITER_METHOD_NONE", 0: "LIMITER_METHOD_BERTH_JESPERSEN", 1: "LIMITER_METHOD_VENKATAKRISHNAN"}


def available() -> bool:
    return MPF_LIB.exists()


def precond_of(cfg: dict):
    """MPFLOW3D PRECOND_METHOD of a library configuration (flux_scheme as
    cfd_params: 0 Roe, 1 HLLC, 4 Turkel-family preconditioned Roe with
    precond_method, 5 Thornber)."""
    fs = cfg.get("flux_scheme", 0)
    if fs == 4:
        return cfg["precond_method"]
    if fs == 5:
        return 1
    return None


def param_text(cfg: dict) -> str:
    """MPFLOW3D parameter file for a library configuration ``cfg`` (keys of
    cfd_params).  REF/INF pressure and temperature are equal, so the
    non-dimensional freestream is rho = 1, p = 1 (module docstring)."""
    g = lambda k, d: cfg.get(k, d)  # noqa: E731
    mach = g("mach", 0.5)
    fs = g("flux_scheme", 0)
    lines = {
        "MESH_FILENAME": "none", "BC_FILENAME": "none", "SOLUTION_FILENAME": "none",
        "RESTART_INPUT_FILENAME": "none", "RESTART_OUTPUT_FILENAME": "none", "MESH_REORDER": "NO",
        "SOLVER_METHOD": "SOLVER_METHOD_STEADY",
        "SOLVER_SCHEME": "SOLVER_SCHEME_EXPLICIT" if g("scheme", "implicit") == "explicit" else
        "SOLVER_SCHEME_IMPLICIT",
        "FLUX_SCHEME": "FLUX_SCHEME_HLLC" if fs == 1 else "FLUX_SCHEME_ROE",
        "SOLVER_NITERATION": "1", "SOLVER_INNER_NITERATION": "1", "LINEAR_SOLVER_NITERATION": "10",
        "SOLVER_ORDER": "SOLVER_ORDER_SECOND" if g("order", 0) == 1 else "SOLVER_ORDER_FIRST",
        "TIME_INTEGRATION_METHOD": "TIME_INTEGRATION_METHOD_IMPLICIT_EULER",
        "TIME_INTEGRATION_TYPE": "TIME_INTEGRATION_TYPE_GLOBAL" if g("global_time", 0) else
        "TIME_INTEGRATION_TYPE_LOCAL",
        "PRECOND_METHOD": PRECOND[precond_of(cfg)],
        "PRECOND_TYPE": PRECOND_TYPE[g("precond_type", 1)], "PRECOND_SMOOTH": "NO",
        "BC_METHOD": "BC_METHOD_CHARCTERISTIC", "ZPG_ITERATION": str(g("zpg_iteration", 0)),
        "VARIABLE_TYPE": "VARIABLE_CON" if g("mpf_variable", "rup") == "con" else "VARIABLE_RUP", "ENTROPY_FIX": "YES" if g("entropy_fix", 0) else "NO",
        "JACOBIAN_METHOD": "JACOBIAN_METHOD_APPROX", "JACOBIAN_UPDATE": "1", "FIRST_ORDER_NITERATION": "0",
        "PHYSICAL_DELTA_TIME": "0.0", "SOLVER_RELAXATION": "1.0", "AVERAGE_TYPE": "AVERAGE_TYPE_ROE",
        "SOLUTION_SMOOTH": "NO", "SOLUTION_SMOOTH_NITERATION": "0", "SOLUTION_SMOOTH_RELAXATION": "0.5",
        "RESIDUAL_SMOOTH_METHOD": "RESIDUAL_SMOOTH_METHOD_NONE",
        "LIMITER_METHOD": LIMITER[g("limiter", -1)], "LIMITER_SMOOTH": "YES" if g("limiter_smooth", 0) else "NO",
        "LIMITER_ORDER": "LIMITER_ORDER_SECOND" if g("limiter_order", 0) == 1 else "LIMITER_ORDER_FIRST",
        "LIMITER_START_SOLVER_ITERATION": "0", "LIMITER_END_SOLVER_ITERATION": "1000000",
        "VENKAT_K_THRESHOLD": repr(float(g("venkat_k", 5.0))),
        "MATERIAL_TYPE": "MATERIAL_TYPE_IDEALGAS", "MATERIAL_NAME": "AIR",
        "MATERIAL_COMP_TYPE": "MATERIAL_COMP_TYPE_NDIM",
        "REF_PRESSURE": "101325.0", "REF_TEMPERATURE": "300.0", "REF_LENGTH": "1.0",
        "INF_PRESSURE": "101325.0", "INF_TEMPERATURE": "300.0",
        "INF_MACH": repr(float(mach)), "INF_MACH_RAMP": str(g("mach_ramp", 0)),
        "INF_MACH_MIN": repr(float(g("mach_min", mach))), "INF_MACH_MAX": repr(float(mach)),
        "INF_ALPHA": repr(float(g("alpha_deg", 2.0))), "INF_BETA": repr(float(g("beta_deg", 0.0))),
        # outflow pressure in Pa; the library's 0 means the freestream pressure
        "OUTFLOW_PRESSURE": repr(101325.0 * (g("outflow_pressure", 0.0) or 1.0)), "GUAGE_PRESSURE": "0.0",
        "CFL_RAMP": str(g("cfl_ramp", 0)), "CFL_MIN": repr(float(g("cfl_min", 10.0))),
        "CFL_MAX": repr(float(g("cfl_max", 10.0))),
        "RESTART_INPUT": "NO", "RESTART_OUTPUT": "NO",
    }
    return "".join(f"{k}={v}\n" for k, v in lines.items())


# ---------------------------------------------------------------- variables
def cons_to_rup(Q: np.ndarray, gamma: float = GAMMA, pinf: float = 0.0) -> np.ndarray:
    """Conservative SoA [5][n] -> (rho, u, v, w, p)."""
    r = Q[0]
    u, v, w = Q[1] / r, Q[2] / r, Q[3] / r
    p = (gamma - 1.0) * (Q[4] - 0.5 * r * (u * u + v * v + w * w)) - gamma * pinf
    return np.stack([r, u, v, w, p])


def rup_to_cons(R: np.ndarray, gamma: float = GAMMA, pinf: float = 0.0) -> np.ndarray:
    r, u, v, w, p = R
    return np.stack([r, r * u, r * v, r * w, (p + gamma * pinf) / (gamma - 1.0) + 0.5 * r * (u * u + v * v + w * w)])


def dcons_drup(R: np.ndarray, gamma: float = GAMMA) -> np.ndarray:
    """d(conservative)/d(rho,u,v,w,p) per node: [n][5][5]."""
    r, u, v, w, _ = R
    n = r.shape[0]
    M = np.zeros((n, 5, 5))
    M[:, 0, 0] = 1.0
    M[:, 1, 0], M[:, 1, 1] = u, r
    M[:, 2, 0], M[:, 2, 2] = v, r
    M[:, 3, 0], M[:, 3, 3] = w, r
    M[:, 4, 0] = 0.5 * (u * u + v * v + w * w)
    M[:, 4, 1], M[:, 4, 2], M[:, 4, 3] = r * u, r * v, r * w
    M[:, 4, 4] = 1.0 / (gamma - 1.0)
    return M


def jacobian_to_rup(A: np.ndarray, JA: np.ndarray, R: np.ndarray, gamma: float = GAMMA) -> np.ndarray:
    """Block-CRS Jacobian dRes/dQcons [nnzb][5][5] -> dRes/dQrup: each block of
    column j right-multiplied by d(cons)/d(rup) at node j."""
    M = dcons_drup(R, gamma)
    return np.einsum("bik,bkj->bij", A, M[JA])


# ------------------------------------------------------------------ session
def _load():
    lib = C.CDLL(str(MPF_LIB))
    P = C.c_void_p
    for name, args, res in [
        ("mpf_read_params", [C.c_char_p], None),
        ("mpf_setup_mesh", [C.c_int] * 3 + [P, P, C.c_int, P, P, P, P, P, P, P], None),
        ("mpf_set_state", [P], None), ("mpf_get_state", [P], None),
        ("mpf_begin_iteration", [C.c_int], None), ("mpf_gradient", [], None),
        ("mpf_apply_bc", [C.c_int], None), ("mpf_residual", [C.c_int], None),
        ("mpf_deltat", [C.c_int], None), ("mpf_rms", [C.c_int], C.c_double),
        ("mpf_jacobian", [C.c_int, C.c_int], None), ("mpf_lusgs", [C.c_int], C.c_double),
        ("mpf_block_gs", [C.c_int, C.c_int], C.c_double), ("mpf_update", [C.c_double], None),
        ("mpf_get_residual", [P, P], None), ("mpf_get_deltat", [P], None),
        ("mpf_get_extrema", [P], None), ("mpf_get_farfield", [P], None),
        ("mpf_nnz_blocks", [], C.c_int), ("mpf_get_crs", [P, P, P], None),
        ("mpf_get_matrix", [P, P, P], None), ("mpf_set_matrix", [P, P], None),
        ("mpf_transformation_matrix", [C.c_int, C.c_int, C.c_int, P], None),
        ("mpf_rms_write", [C.c_int, P, P, P, P], C.c_double), ("mpf_rms_close", [], None),
    ]:
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


def _session(mesh_arrays: dict, cfg: dict, R: np.ndarray | None, steps: list, quiet: bool = True) -> dict:
    if quiet:
        _quiet()
    os.chdir(tempfile.mkdtemp(prefix="cfdmpf_"))  # RMS_Writer writes Residual.res into the cwd
    lib = _load()
    pf = Path("param.txt")
    pf.write_text(param_text(cfg))
    lib.mpf_read_params(str(pf).encode())
    m = mesh_arrays
    nnode, nghost = m["nnode"], m["nghost"]
    arr = {k: np.ascontiguousarray(v) for k, v in m.items() if isinstance(v, np.ndarray)}
    lib.mpf_setup_mesh(nnode, nghost, arr["edge_nodes"].shape[0], _p(arr["edge_nodes"]), _p(arr["edge_areav"]),
                       arr["bedge_nodes"].shape[0], _p(arr["bedge_nodes"]), _p(arr["bedge_areav"]),
                       _p(arr["bedge_type"]), _p(arr["cvol"]), _p(arr["coords"]), _p(arr["n2n_ia"]),
                       _p(arr["n2n_ja"]))
    if R is not None:
        lib.mpf_set_state(_p(np.ascontiguousarray(R, np.float64)))
    out: dict = {"timings": {}}
    nnz = lib.mpf_nnz_blocks()
    for st in steps:
        op, args = st[0], st[1:]
        t0 = time.perf_counter()
        if op == "begin":
            lib.mpf_begin_iteration(*args)
        elif op == "gradient":
            lib.mpf_gradient()
        elif op == "bc":
            lib.mpf_apply_bc(*args)
        elif op == "residual":
            lib.mpf_residual(*args)
        elif op == "deltat":
            lib.mpf_deltat(*args)
        elif op == "rms":
            out.setdefault("rms", []).append(lib.mpf_rms(*args))
        elif op == "jacobian":
            lib.mpf_jacobian(*args)
        elif op == "lusgs":
            out.setdefault("lusgs_rms", []).append(lib.mpf_lusgs(*args))
        elif op == "gs":
            out.setdefault("gs_rms", []).append(lib.mpf_block_gs(*args))
        elif op == "update":
            lib.mpf_update(*args)
        elif op == "rms_write":
            it, conv, diss, ext8, sig2 = args
            out.setdefault("rms", []).append(lib.mpf_rms_write(
                int(it), _p(np.ascontiguousarray(conv, np.float64)), _p(np.ascontiguousarray(diss, np.float64)),
                _p(np.ascontiguousarray(ext8, np.float64)), _p(np.ascontiguousarray(sig2, np.float64))))
        elif op == "rms_close":
            lib.mpf_rms_close()
        elif op == "set_matrix":
            A, B = args
            lib.mpf_set_matrix(_p(np.ascontiguousarray(A, np.float64)), _p(np.ascontiguousarray(B, np.float64)))
        elif op == "get":
            what = args[0]
            if what == "residual":
                c = np.empty((5, nnode)); d = np.empty((5, nnode))
                lib.mpf_get_residual(_p(c), _p(d))
                out["conv"], out["diss"] = c, d
            elif what == "deltat":
                dt = np.empty(nnode); lib.mpf_get_deltat(_p(dt)); out["deltat"] = dt
            elif what == "extrema":
                e = np.empty(8); lib.mpf_get_extrema(_p(e)); out["extrema"] = e
            elif what == "farfield":
                e = np.empty(9); lib.mpf_get_farfield(_p(e)); out["farfield"] = e
            elif what == "state":
                q = np.empty((5, nnode + nghost)); lib.mpf_get_state(_p(q)); out["state"] = q
            elif what == "matrix":
                A = np.empty((nnz, 5, 5)); B = np.empty((nnode, 5)); X = np.empty((nnode, 5))
                lib.mpf_get_matrix(_p(A), _p(B), _p(X))
                out["A"], out["B"], out["X"] = A, B, X
            elif what == "crs":
                IA = np.empty(nnode + 1, np.int32); JA = np.empty(nnz, np.int32); IAU = np.empty(nnode, np.int32)
                lib.mpf_get_crs(_p(IA), _p(JA), _p(IAU))
                out["IA"], out["JA"], out["IAU"] = IA, JA, IAU
            elif what == "residual_file":
                out["residual_file"] = Path("Residual.res").read_bytes() if Path("Residual.res").exists() else b""
        else:
            raise ValueError(op)
        out["timings"].setdefault(op, []).append(time.perf_counter() - t0)
    return out


def run(mesh, cfg: dict, Q: np.ndarray | None, steps: list, quiet: bool = True, timeout: float = 600.0) -> dict:
    """Run ``steps`` on MPFLOW3D in a fresh spawned process.  ``Q`` is the
    library's conservative state [5][nnode+nghost].  With ``cfg["mpf_variable"]
    == "con"`` MPFLOW3D runs in conservative variables (VARIABLE_CON; its
    residual, BC and time step, not its implicit Jacobian, which needs RUP) and
    the state passes unchanged; otherwise it is handed to MPFLOW3D as RUP and a
    returned ``state`` is converted back to conservative variables
    (``state_rup`` keeps MPFLOW3D's own).  With ``cfg["variables"] == 1`` (the
    library's CFD_VARS_RUP) ``Q`` is already (rho, u, v, w, p) and passes
    unchanged both ways."""
    if not available():
        raise FileNotFoundError(f"{MPF_LIB} not built (make -C oracle ref)")
    con = cfg.get("mpf_variable", "rup") == "con"
    own = not con and cfg.get("variables", 0) == 1  # Q already holds (rho, u, v, w, p)
    R = None if Q is None else (np.asarray(Q, np.float64) if (con or own) else cons_to_rup(np.asarray(Q, np.float64)))
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        out = pool.apply_async(_session, (_mesh_dict(mesh), cfg, R, steps, quiet)).get(timeout)
    if "state" in out and not con:
        out["state_rup"] = out["state"]
        if not own:
            out["state"] = rup_to_cons(out["state"])
    return out
