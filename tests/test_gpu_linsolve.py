"""CUDA block-CRS linear solves against the oracle: GMRES(30) with ILU(0) /
block-Jacobi / no preconditioner, FP64 and mixed FP32/BF16 storage inside
FP64 iterative refinement, and the implicit steady driver.

The reference has no GMRES/ILU(0) on this path, so parity is against the
oracle's C restatement (pinned to a dense direct solve in
tests/test_oracle_pin.py) and against the reference's own block Gauss-Seidel
fixed point: every solver must reach the requested FP64 relative residual and
agree with the direct / restated solution to that accuracy."""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, capi
from oracle import restatement
from tests._util import make_case, params_from, relerr

pytestmark = pytest.mark.gpu


def _system(n=20, seed=11):
    m, cfg, Q = make_case(n=n, seed=seed)
    o = restatement.first_order_step(m, cfg, Q, gs_sweeps=1)
    return m, cfg, Q, o


def _residual(sess, A, B, X):
    return np.linalg.norm(B - sess.spmv(A, X)) / np.linalg.norm(B)


@pytest.mark.parametrize("precond", [capi.PC_ILU0, capi.PC_BLOCK_JACOBI, capi.PC_NONE])
def test_gmres_fp64_reaches_tolerance_and_matches_oracle(gpu_available, precond):
    m, cfg, Q, o = _system()
    rs = restatement.Session(m, cfg)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_system(o["A"].reshape(-1, 25), o["B"])
        st = s.solve_gmres(restart=30, max_iters=600, rtol=1e-8, precond=precond, precision=capi.PREC_FP64)
        _, _, X = s.get_system()
    assert st.rel_residual <= 1e-8
    assert _residual(rs, o["A"], o["B"], X) <= 1.1e-8
    Xr, rc, its, rr = rs.gmres(o["A"], o["B"], m=30, maxit=600, rtol=1e-10, precond=2)
    assert rc == 0
    assert relerr(X, Xr) <= 1e-6


def test_ilu0_iteration_count_matches_oracle(gpu_available):
    """Same natural-order block ILU(0): the GPU level-scheduled factorisation is
    the sequential one, so GMRES needs the same number of iterations (+-1)."""
    m, cfg, Q, o = _system(n=12)
    rs = restatement.Session(m, cfg)
    _, rc, its_ref, _ = rs.gmres(o["A"], o["B"], m=30, maxit=300, rtol=1e-6, precond=2)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_system(o["A"].reshape(-1, 25), o["B"])
        st = s.solve_gmres(restart=30, max_iters=300, rtol=1e-6, precond=capi.PC_ILU0)
    assert abs(st.iterations - its_ref) <= 1


@pytest.mark.parametrize("precision", [capi.PREC_FP32, capi.PREC_BF16])
def test_mixed_precision_refinement_reaches_fp64_tolerance(gpu_available, precision):
    m, cfg, Q = make_case(n=20, seed=11)
    rs = restatement.Session(m, cfg)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Apply_Boundary_Condition(0)
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        s.Compute_Jacobian(1, 0, 0, precision)
        A, B, _ = s.get_system()
        st = s.solve_gmres(restart=30, max_iters=600, rtol=1e-8, precond=capi.PC_ILU0, precision=precision,
                           refine=6)
        _, _, X = s.get_system()
    assert st.rel_residual <= 1e-8
    assert _residual(rs, A, B, X) <= 1.1e-8


def test_steady_solve_converges_and_matches_block_gs_path(gpu_available):
    """Implicit steady iterations with GMRES and with the reference's block GS
    reach the same converged state (both converge the same discrete equations)."""
    m, cfg, Q = make_case(n=6, seed=3)
    cfg = dict(cfg, cfl_min=10.0, cfl_max=1000.0, cfl_ramp=10)
    out = []
    for lin in (1, 0):
        with Euler3DGPU(m, params_from(cfg)) as s:
            s.set_state(Q)
            st = s.solve_steady(max_iterations=60, drop=1e-10, include_diss=1, linear_solver=lin, linear_iters=40,
                                gmres=capi.GmresOpts(30, 200, 1e-8, capi.PC_ILU0, capi.PREC_FP64, 1))
            out.append((st, s.get_state()))
    for st, _ in out:
        assert st.rms_last <= 1e-10 * st.rms_first, (st.rms_first, st.rms_last, st.iterations)
    k = m.nnode
    assert relerr(out[0][1][:, :k], out[1][1][:, :k]) <= 1e-8
