"""ctypes driver of the reference Euler3D objects (``oracle/_ref/libeuler3d_ref.so``).

Test infrastructure only: used by ``tests/``, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` to run the *reference's own* code on the same
inputs as the CUDA path.  Each session runs in a fresh ``spawn``-ed process,
because the reference keeps process-global and static state (Roe scratch,
least-squares coefficients) that a second mesh in the same process would
reuse.

Parameter files follow Euler3D/src/SolverParameters.cpp:184-700 (KEY=VALUE).
"""
from __future__ import annotations

import ctypes as C
import multiprocessing as mp
import os
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libeuler3d_ref.so"
REF_EXE = HERE / "_ref" / "euler3d"

FLUX = {0: "FLUX_SCHEME_ROE", 1: "FLUX_SCHEME_HLLC", 2: "FLUX_SCHEME_AUSM", 3: "FLUX_SCHEME_ROE", 6: "FLUX_SCHEME_VANLEER"}
LIMITER = {-1: "LIMITER_METHOD_NONE", 0: "LIMITER_METHOD_BERTH_JESPERSEN", 1: "LIMITER_METHOD_VENKATAKRISHNAN"}


def available() -> bool:
    return REF_LIB.exists()


JACOBIAN = {0: "JACOBIAN_METHOD_CENTRAL", 1: "JACOBIAN_METHOD_FORWARD", 2: "JACOBIAN_METHOD_BACKWARD",
            3: "JACOBIAN_METHOD_ALTERNATE", 4: "JACOBIAN_METHOD_APPROX"}


def param_text(cfg: dict) -> str:
    """Reference parameter file for the options in ``cfg`` (same keys as cfd_params).

    Two keys only the reference has: ``e3d_precond`` selects one of Euler3D's own
    preconditioned Roe fluxes by its PRECOND_METHOD name, with ``e3d_precond_type``
    (PRECOND_TYPE_GLOBAL by default)."""
    g = lambda k, d: cfg.get(k, d)  # noqa: E731
    mach = g("mach", 0.5)
    lines = {
        "MESH_FILENAME": "none", "BC_FILENAME": "none", "SOLUTION_FILENAME": "none",
        "MESH_REORDER": "NO", "SOLVER_METHOD": "SOLVER_METHOD_STEADY",
        # explicit skips the reference's block-matrix allocation (one malloc per block row,
        # Euler3D/src/Solver.cpp:675-685) when only the residual is wanted
        "SOLVER_SCHEME": "SOLVER_SCHEME_EXPLICIT" if g("scheme", "implicit") == "explicit" else
        "SOLVER_SCHEME_IMPLICIT",
        "FLUX_SCHEME": FLUX[g("flux_scheme", 0)], "SOLVER_NITERATION": "1", "LINEAR_SOLVER_NITERATION": "10",
        "SOLVER_ORDER": "SOLVER_ORDER_SECOND" if g("order", 0) == 1 else "SOLVER_ORDER_FIRST",
        "TIME_INTEGRATION_METHOD": "TIME_INTEGRATION_METHOD_IMPLICIT_EULER",
        "TIME_INTEGRATION_TYPE": "TIME_INTEGRATION_TYPE_GLOBAL" if g("global_time", 0) else
        "TIME_INTEGRATION_TYPE_LOCAL",
        "PRECOND_METHOD": "PRECOND_METHOD_ROE_LMFIX" if g("flux_scheme", 0) == 3 else "PRECOND_METHOD_NONE",
        "BC_METHOD": "BC_METHOD_CHARCTERISTIC",
        "ZPG_ITERATION": str(g("zpg_iteration", 0)),
        "VARIABLE_TYPE": "VARIABLE_CONSERVATIVE", "ENTROPY_FIX": "YES" if g("entropy_fix", 0) else "NO",
        "JACOBIAN_METHOD": JACOBIAN[g("jacobian_method", 4)], "JACOBIAN_UPDATE": "1", "FIRST_ORDER_NITERATION": "0",
        "SOLVER_RELAXATION": "1.0", "RESIDUAL_SMOOTH_METHOD": "RESIDUAL_SMOOTH_METHOD_NONE",
        "LIMITER_METHOD": LIMITER[g("limiter", -1)], "LIMITER_SMOOTH": "YES" if g("limiter_smooth", 0) else "NO",
        "LIMITER_ORDER": "LIMITER_ORDER_SECOND" if g("limiter_order", 0) == 1 else "LIMITER_ORDER_FIRST",
        "LIMITER_START_SOLVER_ITERATION": "0", "LIMITER_END_SOLVER_ITERATION": "1000000",
        "VENKAT_K_THRESHOLD": repr(float(g("venkat_k", 5.0))),
        "NONDIMENSIONAL_METHOD": "NONDIMENSIONAL_METHOD_GENERIC", "GAMMA": repr(float(g("gamma", 1.4))),
        "REF_DENSITY": "1.0", "REF_MACH": repr(float(mach)), "REF_PRESSURE": "1.0",
        "REF_ALPHA": repr(float(g("alpha_deg", 2.0))), "REF_BETA": repr(float(g("beta_deg", 0.0))),
        "CFL_RAMP": str(g("cfl_ramp", 0)), "CFL_MIN": repr(float(g("cfl_min", 10.0))),
        "CFL_MAX": repr(float(g("cfl_max", 10.0))), "MACH_RAMP": str(g("mach_ramp", 0)),
        "MACH_MIN": repr(float(g("mach_min", mach))), "MACH_MAX": repr(float(mach)),
        "RESTART_INPUT": "NO", "RESTART_OUTPUT": "NO",
    }
    if "e3d_precond" in cfg:
        # Euler3D's own preconditioned Roe (FluxTest.cpp: Compute_Flux_Roe_Precondition_*),
        # e.g. "PRECOND_METHOD_ROE_BTW" with "PRECOND_TYPE_GLOBAL"
        lines["FLUX_SCHEME"] = "FLUX_SCHEME_ROE"
        lines["PRECOND_METHOD"] = cfg["e3d_precond"]
        lines["PRECOND_TYPE"] = cfg.get("e3d_precond_type", "PRECOND_TYPE_GLOBAL")
        lines["PRECOND_SMOOTH"] = "NO"
    return "".join(f"{k}={v}\n" for k, v in lines.items())


def _load():
    lib = C.CDLL(str(REF_LIB))
    P = C.c_void_p
    for name, args, res in [
        ("ref_read_params", [C.c_char_p], None),
        ("ref_setup_mesh", [C.c_int] * 3 + [P, P, C.c_int, P, P, P, P, P, P, P], None),
        ("ref_set_state", [P], None), ("ref_get_state", [P], None),
        ("ref_begin_iteration", [C.c_int], None), ("ref_gradient", [C.c_int], None),
        ("ref_limiter", [], None), ("ref_apply_bc", [C.c_int], None), ("ref_residual", [C.c_int], None),
        ("ref_deltat", [C.c_int], None), ("ref_jacobian", [C.c_int, C.c_int], None),
        ("ref_block_gs", [C.c_int, C.c_int], C.c_double), ("ref_lusgs", [C.c_int], C.c_double),
        ("ref_update", [C.c_double], None), ("ref_rhs_include_diss", [], C.c_double),
        ("ref_rms_write", [C.c_int, P, P, P], None), ("ref_rms_close", [], None),
        ("ref_get_residual", [P, P], None), ("ref_set_residual", [P, P], None),
        ("ref_get_deltat", [P], None), ("ref_set_deltat", [P], None),
        ("ref_get_extrema", [P], None), ("ref_get_farfield", [P], None),
        ("ref_nnz_blocks", [], C.c_int), ("ref_get_crs", [P, P, P], None),
        ("ref_get_matrix", [P, P, P], None), ("ref_set_matrix", [P, P], None),
        ("ref_get_gradients", [P], None), ("ref_set_gradients", [P], None), ("ref_get_limiters", [P], None),
        ("ref_mesh_from_ugrid", [C.c_char_p, C.c_int], None), ("ref_mesh_sizes", [P], None),
        ("ref_mesh_get", [P] * 9, None), ("ref_sizeof_edge3d", [], C.c_int),
    ]:
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _quiet():
    # the reference prints its whole parameter table and per-step info
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)


def _session(mesh_arrays: dict, cfg: dict, Q: np.ndarray | None, steps: list, quiet: bool = True) -> dict:
    if quiet:
        _quiet()
    os.chdir(tempfile.mkdtemp(prefix="cfdref_"))  # the reference writes Residual.res into the cwd
    lib = _load()
    with tempfile.TemporaryDirectory() as td:
        pf = Path(td) / "param.txt"
        pf.write_text(param_text(cfg))
        lib.ref_read_params(str(pf).encode())
    m = mesh_arrays
    nnode, nghost = m["nnode"], m["nghost"]
    arr = {k: np.ascontiguousarray(v) for k, v in m.items() if isinstance(v, np.ndarray)}
    lib.ref_setup_mesh(nnode, nghost, arr["edge_nodes"].shape[0], _p(arr["edge_nodes"]), _p(arr["edge_areav"]),
                       arr["bedge_nodes"].shape[0], _p(arr["bedge_nodes"]), _p(arr["bedge_areav"]),
                       _p(arr["bedge_type"]), _p(arr["cvol"]), _p(arr["coords"]), _p(arr["n2n_ia"]),
                       _p(arr["n2n_ja"]))
    if Q is not None:
        lib.ref_set_state(_p(np.ascontiguousarray(Q, np.float64)))
    out: dict = {"timings": {}}
    nnz = lib.ref_nnz_blocks()
    for st in steps:
        op, args = st[0], st[1:]
        t0 = time.perf_counter()
        if op == "begin":
            lib.ref_begin_iteration(*args)
        elif op == "bc":
            lib.ref_apply_bc(*args)
        elif op == "gradient":
            lib.ref_gradient(*args)
        elif op == "limiter":
            lib.ref_limiter()
        elif op == "residual":
            lib.ref_residual(*args)
        elif op == "deltat":
            lib.ref_deltat(*args)
        elif op == "jacobian":
            lib.ref_jacobian(*args)
        elif op == "gs":
            out.setdefault("gs_rms", []).append(lib.ref_block_gs(*args))
        elif op == "lusgs":
            out.setdefault("lusgs_rms", []).append(lib.ref_lusgs(*args))
        elif op == "update":
            lib.ref_update(*args)
        elif op == "rms_write":
            it, rms6, ext8, sig2 = args
            lib.ref_rms_write(int(it), _p(np.ascontiguousarray(rms6, np.float64)),
                              _p(np.ascontiguousarray(ext8, np.float64)), _p(np.ascontiguousarray(sig2, np.float64)))
        elif op == "rms_close":
            lib.ref_rms_close()
        elif op == "rhs_full":
            out.setdefault("rms_full", []).append(lib.ref_rhs_include_diss())
        elif op == "set_matrix":
            A, B = args
            lib.ref_set_matrix(_p(np.ascontiguousarray(A, np.float64)), _p(np.ascontiguousarray(B, np.float64)))
        elif op == "set_gradients":
            lib.ref_set_gradients(_p(np.ascontiguousarray(args[0], np.float64)))
        elif op == "set_residual":
            lib.ref_set_residual(_p(np.ascontiguousarray(args[0])), _p(np.ascontiguousarray(args[1])))
        elif op == "set_deltat":
            lib.ref_set_deltat(_p(np.ascontiguousarray(args[0])))
        elif op == "get":
            what = args[0]
            if what == "residual":
                c = np.empty((5, nnode)); d = np.empty((5, nnode))
                lib.ref_get_residual(_p(c), _p(d))
                out["conv"], out["diss"] = c, d
            elif what == "deltat":
                dt = np.empty(nnode); lib.ref_get_deltat(_p(dt)); out["deltat"] = dt
            elif what == "extrema":
                e = np.empty(8); lib.ref_get_extrema(_p(e)); out["extrema"] = e
            elif what == "farfield":
                e = np.empty(8); lib.ref_get_farfield(_p(e)); out["farfield"] = e
            elif what == "state":
                q = np.empty((5, nnode + nghost)); lib.ref_get_state(_p(q)); out["state"] = q
            elif what == "gradients":
                g = np.empty((15, nnode)); lib.ref_get_gradients(_p(g)); out["gradients"] = g
            elif what == "limiters":
                p = np.empty((5, nnode)); lib.ref_get_limiters(_p(p)); out["limiters"] = p
            elif what == "residual_file":
                out["residual_file"] = Path("Residual.res").read_bytes() if Path("Residual.res").exists() else b""
            elif what == "matrix":
                A = np.empty((nnz, 5, 5)); B = np.empty((nnode, 5)); X = np.empty((nnode, 5))
                lib.ref_get_matrix(_p(A), _p(B), _p(X))
                out["A"], out["B"], out["X"] = A, B, X
            elif what == "crs":
                IA = np.empty(nnode + 1, np.int32); JA = np.empty(nnz, np.int32); IAU = np.empty(nnode, np.int32)
                lib.ref_get_crs(_p(IA), _p(JA), _p(IAU))
                out["IA"], out["JA"], out["IAU"] = IA, JA, IAU
        else:
            raise ValueError(op)
        out["timings"].setdefault(op, []).append(time.perf_counter() - t0)
    return out


def _mesh_dict(mesh) -> dict:
    return {
        "nnode": mesh.nnode, "nghost": mesh.nghost, "edge_nodes": mesh.edge_nodes, "edge_areav": mesh.edge_areav,
        "bedge_nodes": mesh.bedge_nodes, "bedge_areav": mesh.bedge_areav, "bedge_type": mesh.bedge_type,
        "cvol": mesh.cvol, "coords": mesh.coords, "n2n_ia": mesh.n2n_ia, "n2n_ja": mesh.n2n_ja,
    }


def run(mesh, cfg: dict, Q: np.ndarray | None, steps: list, quiet: bool = True, timeout: float = 600.0) -> dict:
    """Run ``steps`` on the reference in a fresh spawned process; returns outputs."""
    if not available():
        raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        res = pool.apply_async(_session, (_mesh_dict(mesh), cfg, Q, steps, quiet))
        return res.get(timeout)


def _ugrid_session(path: str, reorder: int) -> dict:
    _quiet()
    os.chdir(tempfile.mkdtemp(prefix="cfdref_"))
    lib = _load()
    lib.ref_mesh_from_ugrid(path.encode(), reorder)
    sz = np.zeros(5, np.int32)
    lib.ref_mesh_sizes(_p(sz))
    nnode, nbnode, nedge, nbedge, nnz = (int(x) for x in sz)
    out = dict(nnode=nnode, nghost=nbnode, edge_nodes=np.empty((nedge, 2), np.int32), edge_areav=np.empty((nedge, 3)),
               bedge_nodes=np.empty((nbedge, 2), np.int32), bedge_areav=np.empty((nbedge, 3)),
               bedge_tag=np.empty(nbedge, np.int32), cvol=np.empty(nnode), coords=np.empty((nnode, 3)),
               n2n_ia=np.empty(nnode + 1, np.int32), n2n_ja=np.empty(nnz, np.int32))
    lib.ref_mesh_get(*(_p(out[k]) for k in ("edge_nodes", "edge_areav", "bedge_nodes", "bedge_areav", "bedge_tag",
                                            "cvol", "coords", "n2n_ia", "n2n_ja")))
    return out


def mesh_from_ugrid(path: str, reorder: int = 0, timeout: float = 600.0) -> dict:
    """The reference's own pre-processing (UGrid_Reader -> Create_Connectivity_Maps
    -> Calculate_Area_Volume) of a UGRID file; returns its mesh arrays."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply_async(_ugrid_session, (str(path), reorder)).get(timeout)


def run_many(mesh, cfg: dict, Q: np.ndarray | None, steps: list, procs: int, timeout: float = 1800.0) -> list:
    """The same reference session in ``procs`` concurrent spawned processes
    (independent single-threaded copies, one per host core)."""
    if not available():
        raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
    ctx = mp.get_context("spawn")
    md = _mesh_dict(mesh)
    with ctx.Pool(procs) as pool:
        rs = [pool.apply_async(_session, (md, cfg, Q, steps, True)) for _ in range(procs)]
        return [r.get(timeout) for r in rs]
