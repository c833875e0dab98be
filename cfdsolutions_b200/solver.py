"""Host-side mirror of the reference's hot-path entry points over the C ABI.

:class:`Euler3DGPU` keeps the reference's function names, argument meaning and
error behaviour (Euler3D/src/Solver_Steady_Implicit.cpp:35-184 calls them in
this order): ``Apply_Boundary_Condition``, ``Compute_Least_Square_Gradient``,
``Compute_Limiter``, ``Compute_Residual``, ``Compute_DeltaT``,
``Compute_Jacobian``, ``MC_Iterative_Block_LU_Jacobi_CRS``; the GMRES solve
that replaces the block sweeps is ``solve_gmres``.  All data stays resident on
the GPU between calls; ``get_*`` methods copy results back.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi
from .mesh import Mesh


def default_params(**kw) -> capi.Params:
    p = capi.Params()
    capi.lib.cfd_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


class Euler3DGPU:
    def __init__(self, mesh: Mesh, params: capi.Params | None = None, device: int = 0, stream: int | None = None):
        self.mesh = mesh
        self._h = C.c_void_p()
        capi.check(capi.lib.cfd_create(int(device), C.byref(self._h)), "cfd_create")
        if stream is not None:
            capi.check(capi.lib.cfd_set_stream(self._h, C.c_void_p(stream)), "cfd_set_stream")
        self.params = params if params is not None else default_params()
        capi.check(capi.lib.cfd_set_params(self._h, C.byref(self.params)), "cfd_set_params")
        m = mesh
        self._keep = [np.ascontiguousarray(a) for a in (
            m.edge_nodes, m.edge_areav, m.bedge_nodes, m.bedge_areav, m.bedge_type, m.cvol, m.coords, m.n2n_ia,
            m.n2n_ja)]
        capi.check(capi.lib.cfd_set_mesh(self._h, m.nnode, m.nghost, m.nedge, capi.ptr(self._keep[0]),
                                         capi.ptr(self._keep[1]), m.nbedge, capi.ptr(self._keep[2]),
                                         capi.ptr(self._keep[3]), capi.ptr(self._keep[4]), capi.ptr(self._keep[5]),
                                         capi.ptr(self._keep[6]), capi.ptr(self._keep[7]), capi.ptr(self._keep[8])),
                   "cfd_set_mesh")
        nnzb = C.c_int64()
        capi.check(capi.lib.cfd_get_block_pattern(self._h, C.byref(nnzb), None, None, None), "cfd_get_block_pattern")
        self.nnzb = int(nnzb.value)

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if self._h:
            capi.lib.cfd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_params(self, params: capi.Params):
        self.params = params
        capi.check(capi.lib.cfd_set_params(self._h, C.byref(params)), "cfd_set_params")

    def synchronize(self):
        capi.check(capi.lib.cfd_synchronize(self._h), "cfd_synchronize")

    # --------------------------------------------------------------- state
    def set_state(self, Q: np.ndarray):
        Q = np.ascontiguousarray(Q, np.float64)
        assert Q.shape == (5, self.mesh.nnode + self.mesh.nghost)
        capi.check(capi.lib.cfd_set_state(self._h, capi.ptr(Q)), "cfd_set_state")
        self.synchronize()

    def get_state(self) -> np.ndarray:
        Q = np.empty((5, self.mesh.nnode + self.mesh.nghost))
        capi.check(capi.lib.cfd_get_state(self._h, capi.ptr(Q)), "cfd_get_state")
        return Q

    # ------------------------------------------- reference-named hot path
    def begin_iteration(self, iteration: int):
        capi.check(capi.lib.cfd_begin_iteration(self._h, iteration), "cfd_begin_iteration")

    def Apply_Boundary_Condition(self, iteration: int):
        capi.check(capi.lib.cfd_apply_bc(self._h, iteration), "Apply_Boundary_Condition")

    def Compute_Least_Square_Gradient(self, weight_type: int = 0):
        if weight_type != self.params.ls_weight or self.params.gradient != capi.GRAD_LSQ:
            p = self.params
            p.ls_weight = weight_type
            p.gradient = capi.GRAD_LSQ
            self.set_params(p)
        capi.check(capi.lib.cfd_gradient(self._h), "Compute_Least_Square_Gradient")

    def Compute_Gradient(self):
        capi.check(capi.lib.cfd_gradient(self._h), "cfd_gradient")

    def Compute_Limiter(self):
        capi.check(capi.lib.cfd_limiter(self._h), "Compute_Limiter")

    def Compute_Residual(self, add_time: int = 1):
        capi.check(capi.lib.cfd_residual(self._h, int(add_time)), "Compute_Residual")

    def Compute_DeltaT(self, iteration: int):
        capi.check(capi.lib.cfd_deltat(self._h, iteration), "Compute_DeltaT")

    def Compute_Jacobian(self, add_time: int = 1, iteration: int = 0, include_diss: int = 0,
                         precision: int = capi.PREC_FP64):
        capi.check(capi.lib.cfd_jacobian(self._h, int(add_time), int(include_diss), int(precision)),
                   "Compute_Jacobian")

    def MC_Iterative_Block_LU_Jacobi_CRS(self, iterations: int, direction: int = 0) -> float:
        rms = C.c_double()
        code = capi.lib.cfd_block_gs(self._h, int(iterations), int(direction), C.byref(rms))
        if code == -6:  # numerical failure: NaN RMS, as the reference returns
            return float("nan")
        capi.check(code, "MC_Iterative_Block_LU_Jacobi_CRS")
        return rms.value

    def Compute_Jacobian_FiniteDifference(self, add_time: int = 1, iteration: int = 0,
                                          method: int = capi.JAC_CENTRAL, include_diss: int = 0):
        capi.check(capi.lib.cfd_jacobian_fd(self._h, int(add_time), int(include_diss), int(method), int(iteration)),
                   "Compute_Jacobian_FiniteDifference_Roe")

    def MC_Iterative_Block_LUSGS_CRS(self, iterations: int) -> float:
        rms = C.c_double()
        code = capi.lib.cfd_block_lusgs(self._h, int(iterations), C.byref(rms))
        if code == -6:  # numerical failure: NaN RMS, as the reference returns
            return float("nan")
        capi.check(code, "MC_Iterative_Block_LUSGS_CRS")
        return rms.value

    def solve_gmres(self, restart=30, max_iters=300, rtol=1e-6, precond=capi.PC_ILU0, precision=capi.PREC_FP64,
                    refine=1, allow_not_converged=False) -> capi.GmresStats:
        o = capi.GmresOpts(restart, max_iters, rtol, precond, precision, refine)
        st = capi.GmresStats()
        code = capi.lib.cfd_gmres(self._h, C.byref(o), C.byref(st))
        if not (allow_not_converged and code == -7):
            capi.check(code, "cfd_gmres")
        return st

    def spmv_device(self, x_ptr: int, y_ptr: int, precision: int = capi.PREC_FP64):
        """y = A x on device vectors [nnode][5] (raw device addresses)."""
        capi.check(capi.lib.cfd_spmv(self._h, int(precision), C.c_void_p(x_ptr), C.c_void_p(y_ptr)), "cfd_spmv")

    def precond_apply_device(self, r_ptr: int, z_ptr: int):
        """z = M^-1 r with the last cfd_gmres preconditioner, on device vectors."""
        capi.check(capi.lib.cfd_precond_apply(self._h, C.c_void_p(r_ptr), C.c_void_p(z_ptr)), "cfd_precond_apply")

    def update(self, relax: float = 1.0):
        capi.check(capi.lib.cfd_update(self._h, float(relax)), "cfd_update")

    def residual_rms(self, include_diss: bool = False) -> np.ndarray:
        out = np.zeros(6)
        capi.check(capi.lib.cfd_residual_rms(self._h, int(include_diss), capi.ptr(out)), "cfd_residual_rms")
        return out

    def residual_step(self, iteration: int = 0, Q: np.ndarray | None = None, want_residual: bool = False,
                      out: tuple | None = None):
        """One residual evaluation (cfd_residual_step).  With ``Q`` the state is
        copied in first; with ``want_residual`` or ``out=(conv, diss)`` the
        residuals are copied back (pass pinned arrays for full copy speed)."""
        conv = diss = None
        if out is not None:
            conv, diss = out
        elif want_residual:
            conv = np.empty((5, self.mesh.nnode))
            diss = np.empty((5, self.mesh.nnode))
        capi.check(capi.lib.cfd_residual_step(self._h, iteration, capi.ptr(Q), capi.ptr(conv), capi.ptr(diss)),
                   "cfd_residual_step")
        return conv, diss

    def set_step_pipeline(self, chunks: int = -1):
        """Chunks of the pipelined residual_step with host buffers (-1
        automatic, 0/1 off; cfd_set_step_pipeline)."""
        capi.check(capi.lib.cfd_set_step_pipeline(self._h, int(chunks)), "cfd_set_step_pipeline")

    def solve_steady(self, max_iterations=100, drop=1e-8, include_diss=1, linear_solver=1, linear_iters=10,
                     relax=1.0, gmres: capi.GmresOpts | None = None, precond_update: int = 1) -> capi.SolveStats:
        g = gmres if gmres is not None else capi.GmresOpts(30, 300, 1e-6, capi.PC_ILU0, capi.PREC_FP64, 1)
        o = capi.SolveOpts(max_iterations, drop, include_diss, linear_solver, linear_iters, relax, g,
                           int(precond_update))
        st = capi.SolveStats()
        capi.check(capi.lib.cfd_solve_steady(self._h, C.byref(o), C.byref(st)), "cfd_solve_steady")
        return st

    def solve_unsteady(self, dt, steps, inner_iterations=10, bdf2=True, include_diss=1, linear_solver=1,
                       linear_iters=10, relax=1.0, gmres: capi.GmresOpts | None = None) -> capi.UnsteadyStats:
        """Solver_Unsteady_Implicit (MPFLOW3D/src/Solver_Unsteady_Implicit.cpp:36-305)."""
        g = gmres if gmres is not None else capi.GmresOpts(30, 300, 1e-6, capi.PC_ILU0, capi.PREC_FP64, 1)
        o = capi.UnsteadyOpts(float(dt), int(steps), int(inner_iterations), int(bool(bdf2)), include_diss,
                              linear_solver, linear_iters, relax, g)
        st = capi.UnsteadyStats()
        capi.check(capi.lib.cfd_solve_unsteady(self._h, C.byref(o), C.byref(st)), "cfd_solve_unsteady")
        return st

    # ------------------------------------------------------------ readback
    def get_residual(self):
        conv = np.empty((5, self.mesh.nnode))
        diss = np.empty((5, self.mesh.nnode))
        capi.check(capi.lib.cfd_get_residual(self._h, capi.ptr(conv), capi.ptr(diss)), "cfd_get_residual")
        return conv, diss

    def get_deltat(self) -> np.ndarray:
        dt = np.empty(self.mesh.nnode)
        capi.check(capi.lib.cfd_get_deltat(self._h, capi.ptr(dt)), "cfd_get_deltat")
        return dt

    def get_extrema(self) -> np.ndarray:
        out = np.empty(8)
        capi.check(capi.lib.cfd_get_extrema(self._h, capi.ptr(out)), "cfd_get_extrema")
        return out

    def get_farfield(self) -> np.ndarray:
        out = np.empty(8)
        capi.check(capi.lib.cfd_get_farfield(self._h, capi.ptr(out)), "cfd_get_farfield")
        return out

    def get_gradients(self) -> np.ndarray:
        g = np.empty((15, self.mesh.nnode))
        capi.check(capi.lib.cfd_get_gradients(self._h, capi.ptr(g)), "cfd_get_gradients")
        return g

    def get_limiters(self) -> np.ndarray:
        phi = np.empty((5, self.mesh.nnode))
        capi.check(capi.lib.cfd_get_limiters(self._h, capi.ptr(phi)), "cfd_get_limiters")
        return phi

    def get_block_pattern(self):
        n = self.mesh.nnode
        IA = np.empty(n + 1, np.int32)
        JA = np.empty(self.nnzb, np.int32)
        IAU = np.empty(n, np.int32)
        capi.check(capi.lib.cfd_get_block_pattern(self._h, None, capi.ptr(IA), capi.ptr(JA), capi.ptr(IAU)),
                   "cfd_get_block_pattern")
        return IA, JA, IAU

    def get_system(self):
        A = np.empty((self.nnzb, 5, 5))
        B = np.empty((self.mesh.nnode, 5))
        X = np.empty((self.mesh.nnode, 5))
        capi.check(capi.lib.cfd_get_system(self._h, capi.ptr(A), capi.ptr(B), capi.ptr(X)), "cfd_get_system")
        return A, B, X

    def set_system(self, A: np.ndarray, B: np.ndarray):
        A = np.ascontiguousarray(A, np.float64)
        B = np.ascontiguousarray(B, np.float64)
        capi.check(capi.lib.cfd_set_system(self._h, capi.ptr(A), capi.ptr(B)), "cfd_set_system")
