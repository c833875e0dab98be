"""ctypes wrapper of the oracle's C restatement (``oracle/_build/libcfd_oracle.so``).

Test infrastructure only (tests/, __graft_entry__.smoke, bench.py's CPU
baseline).  The library is built by ``make -C oracle``; if it is missing, it
is built here with the system C compiler (plain C, no GPU).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libcfd_oracle.so"


class Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("mach", C.c_double), ("alpha_deg", C.c_double), ("beta_deg", C.c_double),
                ("cfl", C.c_double), ("venkat_k", C.c_double), ("flux", C.c_int), ("order", C.c_int),
                ("limiter", C.c_int), ("limiter_order", C.c_int), ("limiter_smooth", C.c_int),
                ("entropy_fix", C.c_int), ("global_time", C.c_int), ("ls_weight", C.c_int), ("gradient", C.c_int),
                ("iteration", C.c_int), ("zpg_iteration", C.c_int), ("pinf", C.c_double),
                ("pc_method", C.c_int), ("pc_type", C.c_int), ("pc_mach", C.c_double), ("outflow_p", C.c_double),
                ("pc_avg", C.c_int), ("mpf_form", C.c_int), ("variables", C.c_int)]


class MeshC(C.Structure):
    _fields_ = [("nnode", C.c_int), ("nghost", C.c_int), ("nedge", C.c_int), ("nbedge", C.c_int),
                ("en", C.c_void_p), ("ea", C.c_void_p), ("bn", C.c_void_p), ("ba", C.c_void_p), ("bt", C.c_void_p),
                ("vol", C.c_void_p), ("xyz", C.c_void_p), ("ia", C.c_void_p), ("ja", C.c_void_p)]


def _lib():
    src = [HERE / "cfd_oracle.c", HERE / "cfd_oracle.h"]
    if not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in src):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    PP, PM = C.POINTER(Params), C.POINTER(MeshC)
    sig = {
        "orc_farfield": (None, [PP, P]), "orc_apply_bc": (None, [PM, PP, P]),
        "orc_gradient_lsq": (None, [PM, PP, P, P]), "orc_gradient_gg": (None, [PM, P, P]),
        "orc_limiter": (None, [PM, PP, P, P, P]), "orc_residual": (None, [PM, PP, P, P, P, P, P, P, P]),
        "orc_deltat": (None, [PM, PP, P, P]), "orc_block_pattern": (C.c_long, [PM, P, P, P]),
        "orc_jacobian": (None, [PM, PP, P, P, P, P, C.c_int, C.c_int, P, P, P, P, P]),
        "orc_block_gs": (C.c_double, [C.c_int, P, P, P, P, P, P, C.c_int, C.c_int]),
        "orc_block_lusgs": (C.c_double, [C.c_int, P, P, P, P, P, P, C.c_int]),
        "orc_ilu0": (C.c_int, [C.c_int, P, P, P, P, P]),
        "orc_gmres": (C.c_int, [C.c_int, P, P, P, P, P, P, C.c_int, C.c_int, C.c_double, C.c_int,
                                C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "orc_bspmv": (None, [C.c_int, P, P, P, P, P]),
        "orc_ilu0_apply": (None, [C.c_int, P, P, P, P, P, P]),
    }
    for k, (r, a) in sig.items():
        f = getattr(lib, k)
        f.restype, f.argtypes = r, a
    return lib


lib = _lib()


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Session:
    """Holds a mesh (and keeps its arrays alive) for restatement calls."""

    def __init__(self, mesh, cfg: dict, iteration: int = 0):
        self.mesh = mesh
        self.arrs = [np.ascontiguousarray(a) for a in (mesh.edge_nodes, mesh.edge_areav, mesh.bedge_nodes,
                                                      mesh.bedge_areav, mesh.bedge_type, mesh.cvol, mesh.coords,
                                                      mesh.n2n_ia, mesh.n2n_ja)]
        self.m = MeshC(mesh.nnode, mesh.nghost, mesh.nedge, mesh.nbedge, *(_p(a) for a in self.arrs))
        self.p = params(cfg, iteration)
        self.n = mesh.nnode
        nnz = lib.orc_block_pattern(C.byref(self.m), None, None, None)
        self.IA = np.zeros(self.n + 1, np.int32)
        self.JA = np.zeros(nnz, np.int32)
        self.IAU = np.zeros(self.n, np.int32)
        lib.orc_block_pattern(C.byref(self.m), _p(self.IA), _p(self.JA), _p(self.IAU))

    def apply_bc(self, Q):
        Q = np.ascontiguousarray(Q, np.float64).copy()
        lib.orc_apply_bc(C.byref(self.m), C.byref(self.p), _p(Q))
        return Q

    def gradient(self, Q, method=0):
        g = np.zeros((15, self.n))
        Q = np.ascontiguousarray(Q)
        if method == 1:
            lib.orc_gradient_gg(C.byref(self.m), _p(Q), _p(g))
        else:
            lib.orc_gradient_lsq(C.byref(self.m), C.byref(self.p), _p(Q), _p(g))
        return g

    def limiter(self, Q, grad):
        phi = np.zeros((5, self.n))
        lib.orc_limiter(C.byref(self.m), C.byref(self.p), _p(np.ascontiguousarray(Q)), _p(grad), _p(phi))
        return phi

    def residual(self, Q, grad=None, phi=None):
        conv = np.zeros((5, self.n)); diss = np.zeros((5, self.n)); dts = np.zeros(self.n); ext = np.zeros(6)
        lib.orc_residual(C.byref(self.m), C.byref(self.p), _p(np.ascontiguousarray(Q)), _p(grad), _p(phi),
                         _p(conv), _p(diss), _p(dts), _p(ext))
        return conv, diss, dts, ext

    def deltat(self, dtsum):
        dt = np.array(dtsum, dtype=np.float64, copy=True)
        ext = np.zeros(2)
        lib.orc_deltat(C.byref(self.m), C.byref(self.p), _p(dt), _p(ext))
        return dt, ext

    def jacobian(self, Q, dt, conv, diss, add_time=1, include_diss=0):
        A = np.zeros((len(self.JA), 5, 5)); B = np.zeros((self.n, 5))
        lib.orc_jacobian(C.byref(self.m), C.byref(self.p), _p(np.ascontiguousarray(Q)), _p(dt), _p(conv), _p(diss),
                         add_time, include_diss, _p(self.IA), _p(self.JA), _p(self.IAU), _p(A), _p(B))
        return A, B

    def block_gs(self, A, B, iters, direction=0):
        X = np.zeros((self.n, 5))
        rms = lib.orc_block_gs(self.n, _p(self.IA), _p(self.JA), _p(self.IAU), _p(np.ascontiguousarray(A)),
                               _p(np.ascontiguousarray(B)), _p(X), iters, direction)
        return X, rms

    def block_lusgs(self, A, B, iters):
        X = np.zeros((self.n, 5))
        rms = lib.orc_block_lusgs(self.n, _p(self.IA), _p(self.JA), _p(self.IAU), _p(np.ascontiguousarray(A)),
                                  _p(np.ascontiguousarray(B)), _p(X), iters)
        return X, rms

    def gmres(self, A, B, m=30, maxit=300, rtol=1e-6, precond=2):
        X = np.zeros((self.n, 5))
        it = C.c_int()
        rr = C.c_double()
        rc = lib.orc_gmres(self.n, _p(self.IA), _p(self.JA), _p(self.IAU), _p(np.ascontiguousarray(A)),
                           _p(np.ascontiguousarray(B)), _p(X), m, maxit, rtol, precond, C.byref(it), C.byref(rr))
        return X, rc, it.value, rr.value

    def ilu0(self, A):
        """ILU(0) factors in the block pattern (L unit-lower, U with inverted diagonal blocks)."""
        F = np.zeros((len(self.JA), 5, 5))
        rc = lib.orc_ilu0(self.n, _p(self.IA), _p(self.JA), _p(self.IAU), _p(np.ascontiguousarray(A)), _p(F))
        if rc:
            raise ArithmeticError("orc_ilu0: singular diagonal block")
        return F

    def ilu0_apply(self, F, r):
        z = np.zeros((self.n, 5))
        lib.orc_ilu0_apply(self.n, _p(self.IA), _p(self.JA), _p(self.IAU), _p(np.ascontiguousarray(F)),
                           _p(np.ascontiguousarray(r, np.float64)), _p(z))
        return z

    def spmv(self, A, x):
        y = np.zeros((self.n, 5))
        lib.orc_bspmv(self.n, _p(self.IA), _p(self.JA), _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(x)),
                      _p(y))
        return y


def params(cfg: dict, iteration: int = 0) -> Params:
    g = cfg.get
    cfl_min, cfl_max, ramp = g("cfl_min", 10.0), g("cfl_max", 10.0), g("cfl_ramp", 0)
    if ramp > 1 and cfl_max > cfl_min:
        cfl = cfl_min + (cfl_max - cfl_min) * (iteration / (ramp - 1)) if iteration < ramp else cfl_max
    else:
        cfl = cfl_max
    return Params(g("gamma", 1.4), g("mach", 0.5), g("alpha_deg", 2.0), g("beta_deg", 0.0), cfl, g("venkat_k", 5.0),
                  g("flux_scheme", 0), g("order", 0), g("limiter", -1), g("limiter_order", 0),
                  g("limiter_smooth", 0), g("entropy_fix", 0), g("global_time", 0), g("ls_weight", 0),
                  g("gradient", 0), iteration, g("zpg_iteration", 0), g("pinf", 0.0),
                  g("precond_method", 0), g("precond_type", 0), g("precond_mach", 0.0), g("outflow_pressure", 0.0),
                  g("precond_average", 0), g("mpf_form", 0), g("variables", 0))


def first_order_step(mesh, cfg: dict, Q: np.ndarray, gs_sweeps: int = 10) -> dict:
    """BC -> residual -> dt -> Jacobian -> block GS, as one Euler3D implicit iteration."""
    s = Session(mesh, cfg)
    Qb = s.apply_bc(Q)
    conv, diss, dts, ext = s.residual(Qb)
    dt, ext2 = s.deltat(dts)
    A, B = s.jacobian(Qb, dt, conv, diss)
    X, rms = s.block_gs(A, B, gs_sweeps)
    return dict(state=Qb, conv=conv, diss=diss, deltat=dt, extrema=np.r_[ext, ext2], A=A, B=B, X=X, gs_rms=rms,
                IA=s.IA, JA=s.JA, IAU=s.IAU)


def residual_pass(mesh, cfg: dict, Q: np.ndarray) -> dict:
    """BC -> (gradient -> limiter) -> residual -> dt (one residual evaluation)."""
    s = Session(mesh, cfg)
    Qb = s.apply_bc(Q)
    grad = phi = None
    if cfg.get("order", 0) == 1:
        grad = s.gradient(Qb, cfg.get("gradient", 0))
        if cfg.get("limiter", -1) != -1:
            phi = s.limiter(Qb, grad)
    conv, diss, dts, ext = s.residual(Qb, grad, phi)
    dt, ext2 = s.deltat(dts)
    return dict(state=Qb, grad=grad, phi=phi, conv=conv, diss=diss, deltat=dt, extrema=np.r_[ext, ext2])


def unsteady(mesh, cfg: dict, Q: np.ndarray, dt: float, steps: int, inner: int, bdf2: bool = True,
             include_diss: int = 1, rtol: float = 1e-13) -> np.ndarray:
    """Solver_Unsteady_Implicit (MPFLOW3D/src/Solver_Unsteady_Implicit.cpp:36-305) on the
    restatement: per inner iteration gradient/limiter, BC, residual, Jacobian without the
    pseudo-time term, the physical-time source and diagonal, a GMRES(30)+ILU(0) solve
    (tolerance rtol) and the update.  Returns the state [5, nnode+nghost]."""
    Q = np.array(Q, dtype=np.float64, copy=True)
    n = mesh.nnode
    qn = Q[:, :n].copy()
    qn1 = qn.copy()
    for t in range(steps):
        theta = 0.5 if (bdf2 and t > 0) else 0.0
        if bdf2:
            qn1 = qn.copy()
        qn = Q[:, :n].copy()
        if t == 0:
            qn1 = qn.copy()
        for it in range(inner):
            s = Session(mesh, cfg, iteration=it)
            g = phi = None
            if cfg.get("order", 0) == 1:
                g = s.gradient(Q, cfg.get("gradient", 0))
                if cfg.get("limiter", -1) != -1:
                    phi = s.limiter(Q, g)
            Q = s.apply_bc(Q)
            conv, diss, _, _ = s.residual(Q, g, phi)
            A, B = s.jacobian(Q, np.zeros(n), conv, diss, add_time=0, include_diss=include_diss)
            eta = mesh.cvol / dt
            src = eta * ((1.0 + theta) * (Q[:, :n] - qn) - theta * (qn - qn1))
            B -= src.T
            A[s.IAU] += (1.0 + theta) * eta[:, None, None] * np.eye(5)
            X, _, _, _ = s.gmres(A, B, m=30, maxit=3000, rtol=rtol, precond=2)
            Q[:, :n] += X.T
    return Q
