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


def _permuted_system(IA, JA, IAU, A, B, order):
    """Block-CRS system P A P^T, P B for the row order `order` (position -> row)."""
    n = len(order)
    pos = np.empty(n, np.int64)
    pos[order] = np.arange(n)
    IAp = np.zeros(n + 1, np.int32)
    rows = []
    for k, i in enumerate(order):
        cols = pos[JA[IA[i]:IA[i + 1]]]
        srt = np.argsort(cols)
        rows.append((cols[srt], np.arange(IA[i], IA[i + 1])[srt]))
        IAp[k + 1] = IAp[k] + len(cols)
    JAp = np.concatenate([r[0] for r in rows]).astype(np.int32)
    src = np.concatenate([r[1] for r in rows])
    IAUp = np.array([IAp[k] + int(np.nonzero(rows[k][0] == k)[0][0]) for k in range(n)], np.int32)
    return IAp, JAp, IAUp, np.ascontiguousarray(A[src]), np.ascontiguousarray(B[order]), pos


@pytest.mark.parametrize("n", [12, 20])
def test_ilu0_multicolour_is_ilu0_of_the_permuted_system(gpu_available, n):
    """CFD_PC_ILU0_MC is ILU(0) of P A P^T for the block multicolour order P
    the library reports: GMRES with it takes the iterations of the oracle's
    natural-order ILU(0) GMRES on the permuted system (+-1) and reaches the same
    solution."""
    import ctypes as C

    m, cfg, Q, o = _system(n=n)
    nn = m.nnode
    with Euler3DGPU(m, params_from(cfg)) as s:
        order = np.empty(nn, np.int32)
        ncol = C.c_int()
        capi.check(capi.lib.cfd_ilu_mc_order(s.handle, capi.ptr(order), C.byref(ncol)), "cfd_ilu_mc_order")
        IA, JA, IAU = s.get_block_pattern()
        s.set_system(o["A"].reshape(-1, 25), o["B"])
        st = s.solve_gmres(restart=30, max_iters=300, rtol=1e-6, precond=capi.PC_ILU0_MC)
        _, _, X = s.get_system()
    assert ncol.value >= 2 and sorted(order.tolist()) == list(range(nn))
    IAp, JAp, IAUp, Ap, Bp, pos = _permuted_system(IA, JA, IAU, o["A"], o["B"], order)
    Xp = np.zeros((nn, 5))
    it = C.c_int()
    rr = C.c_double()
    rc = restatement.lib.orc_gmres(nn, restatement._p(IAp), restatement._p(JAp), restatement._p(IAUp),
                                   restatement._p(Ap), restatement._p(Bp), restatement._p(Xp), 30, 300, 1e-6, 2,
                                   C.byref(it), C.byref(rr))
    assert rc == 0
    assert abs(st.iterations - it.value) <= 1, (st.iterations, it.value)
    assert relerr(X, Xp[pos]) <= 1e-5


@pytest.mark.parametrize("precision", [capi.PREC_FP32, capi.PREC_BF16])
def test_ilu0_multicolour_mixed_precision_reaches_fp64_tolerance(gpu_available, precision):
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
        st = s.solve_gmres(restart=30, max_iters=600, rtol=1e-8, precond=capi.PC_ILU0_MC, precision=precision,
                           refine=6)
        _, _, X = s.get_system()
    assert st.rel_residual <= 1e-8
    assert _residual(rs, A, B, X) <= 1.1e-8


@pytest.mark.parametrize("precision,tol", [(capi.PREC_FP32, 2e-6), (capi.PREC_BF16, 2e-2)])
def test_low_only_jacobian_is_the_fp64_jacobian_rounded(gpu_available, precision, tol):
    """CFD_PREC_LOW_ONLY keeps only the FP32/BF16 matrix; its blocks are the
    FP64 Jacobian's to storage precision (the diagonal is summed in FP64 from
    the stored off-diagonal blocks)."""
    m, cfg, Q = make_case(n=10, seed=5)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Apply_Boundary_Condition(0)
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        s.Compute_Jacobian(1, 0, 0, capi.PREC_FP64)
        A64, B64, _ = s.get_system()
        s.Compute_Jacobian(1, 0, 0, precision | capi.PREC_LOW_ONLY)
        Al, Bl, _ = s.get_system()
        with pytest.raises(capi.CfdError):  # the reference's block GS needs the FP64 system
            s.MC_Iterative_Block_LU_Jacobi_CRS(2, 0)
    np.testing.assert_array_equal(Bl, B64)
    scale = np.abs(A64).reshape(len(A64), -1).max(axis=1)
    err = np.abs(Al - A64).reshape(len(A64), -1).max(axis=1)
    assert np.all(err <= tol * np.maximum(scale, 1e-300))


@pytest.mark.parametrize("precision", [capi.PREC_FP32, capi.PREC_BF16])
def test_steady_solve_low_only_reaches_the_fp64_converged_state(gpu_available, precision):
    """Mixed precision (low-precision-only Jacobian and ILU(0) inside the FP64
    nonlinear defect correction) converges to the plain FP64 solution: the
    converged fields agree to 1e-8, relative to each field's magnitude or, for
    a field that vanishes in the converged flow (w-momentum at zero sideslip),
    to the momentum scale."""
    m, cfg, Q = make_case(n=8, seed=3)
    cfg = dict(cfg, cfl_min=10.0, cfl_max=1000.0, cfl_ramp=10)
    out = []
    for prec in (capi.PREC_FP64, precision | capi.PREC_LOW_ONLY):
        with Euler3DGPU(m, params_from(cfg)) as s:
            s.set_state(Q)
            st = s.solve_steady(max_iterations=200, drop=1e-11, include_diss=1, linear_solver=1,
                                gmres=capi.GmresOpts(30, 60, 1e-3, capi.PC_ILU0_MC, prec, 1))
            assert st.rms_last <= 1e-11 * st.rms_first, (st.iterations, st.rms_first, st.rms_last)
            out.append(s.get_state()[:, :m.nnode])
    mom = np.abs(out[0][1:4]).max()
    for v in range(5):
        scale = max(np.abs(out[0][v]).max(), mom if 1 <= v <= 3 else 0.0)
        assert np.abs(out[1][v] - out[0][v]).max() <= 1e-8 * scale


def test_steady_solve_with_lagged_preconditioner_reaches_the_same_state(gpu_available):
    """precond_update = 4: the ILU(0) factors are reused for 4 implicit
    iterations (the Jacobian is rebuilt every iteration); the converged state
    is the one of refactoring every iteration."""
    m, cfg, Q = make_case(n=8, seed=3)
    cfg = dict(cfg, cfl_min=10.0, cfl_max=1000.0, cfl_ramp=10)
    out = []
    for k in (1, 4):
        with Euler3DGPU(m, params_from(cfg)) as s:
            s.set_state(Q)
            st = s.solve_steady(max_iterations=300, drop=1e-11, include_diss=1, linear_solver=1,
                                gmres=capi.GmresOpts(30, 60, 1e-2, capi.PC_ILU0_MC, capi.PREC_FP64, 1, 0),
                                precond_update=k)
            assert st.rms_last <= 1e-11 * st.rms_first
            out.append(s.get_state()[:, :m.nnode])
    mom = np.abs(out[0][1:4]).max()
    for v in range(5):
        scale = max(np.abs(out[0][v]).max(), mom if 1 <= v <= 3 else 0.0)
        assert np.abs(out[1][v] - out[0][v]).max() <= 1e-8 * scale


def test_spmv_and_precond_apply_match_restatement(gpu_available):
    """cfd_spmv (FP64 and FP32 storage) against the restatement's block product
    on the same matrix, and cfd_precond_apply of the natural-order ILU(0)
    against the restatement's ILU(0) factors and triangular solves: the
    level-scheduled factorisation and solves compute the sequential algorithm,
    so the results agree to round-off (1e-12 normwise; products 1e-14)."""
    import torch
    m, cfg, Q, o = _system(n=10)
    rs = restatement.Session(m, cfg)
    x = np.random.default_rng(3).standard_normal((m.nnode, 5))
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Apply_Boundary_Condition(0)
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        s.Compute_Jacobian(1, 0, precision=capi.PREC_FP32)
        A, _, _ = s.get_system()
        xd = torch.from_numpy(x).cuda()
        yd = torch.empty_like(xd)
        out = {}
        for name, prec in (("fp64", capi.PREC_FP64), ("fp32", capi.PREC_FP32)):
            s.spmv_device(xd.data_ptr(), yd.data_ptr(), prec)
            s.synchronize()
            out[name] = yd.cpu().numpy()
        s.solve_gmres(restart=30, max_iters=300, rtol=1e-6, precond=capi.PC_ILU0, precision=capi.PREC_FP64)
        s.precond_apply_device(xd.data_ptr(), yd.data_ptr())
        s.synchronize()
        z = yd.cpu().numpy()
    assert relerr(out["fp64"], rs.spmv(A, x)) <= 1e-14
    assert relerr(out["fp32"], rs.spmv(A.astype(np.float32).astype(np.float64), x)) <= 1e-14
    assert relerr(z, rs.ilu0_apply(rs.ilu0(A), x)) <= 1e-12
