"""Parity of the CUDA path with the reference's own functions (the Euler3D
objects compiled into oracle/_ref, run on the same mesh arrays and state).

Tolerances: residuals within 1e-12 relative in FP64 (normwise
per equation, max |gpu - ref| / max |ref|); the same bound for ghost states,
time steps, gradients, limiters and Jacobian blocks.  Block Gauss-Seidel on an
identical system is bit-exact (level scheduling preserves the sequential
row order and the kernel avoids fused multiply-adds).
"""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU
from oracle import refharness
from tests._util import CFG1, low_pressure_spots, make_case, params_from, relerr, relerr_rows

TOL = 1e-12

pytestmark = pytest.mark.gpu


def _first_order_steps():
    return [("begin", 0), ("bc", 0), ("get", "state"), ("residual", 1), ("get", "residual"), ("get", "extrema"),
            ("deltat", 0), ("get", "deltat"), ("get", "extrema"), ("get", "farfield"), ("jacobian", 1, 0),
            ("get", "matrix"), ("gs", 10, 0), ("get", "matrix")]


def _gpu_first_order(s: Euler3DGPU):
    out = {}
    s.begin_iteration(0)
    s.Apply_Boundary_Condition(0)
    out["state"] = s.get_state()
    s.Compute_Residual(1)
    out["conv"], out["diss"] = s.get_residual()
    out["extrema_res"] = s.get_extrema()
    s.Compute_DeltaT(0)
    out["deltat"] = s.get_deltat()
    out["extrema"] = s.get_extrema()
    out["farfield"] = s.get_farfield()
    s.Compute_Jacobian(1, 0)
    out["A"], out["B"], _ = s.get_system()
    out["gs_rms"] = s.MC_Iterative_Block_LU_Jacobi_CRS(10, 0)
    _, _, out["X"] = s.get_system()
    return out


@pytest.mark.parametrize("n,rcm", [(6, False), (20, False), (12, True)])
def test_first_order_roe_step_matches_reference(gpu_available, ref_available, n, rcm):
    m, cfg, Q = make_case(n=n, seed=11 + n, rcm=rcm)
    ref = refharness.run(m, cfg, Q, _first_order_steps())
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        g = _gpu_first_order(s)
        IA, JA, IAU = s.get_block_pattern()
    # far field, ghost states
    np.testing.assert_allclose(g["farfield"], ref["farfield"], rtol=1e-15, atol=0)
    assert relerr_rows(g["state"], ref["state"]) <= 1e-13
    # residuals (convective and dissipative kept separate, as Euler3D)
    assert relerr_rows(g["conv"], ref["conv"]) <= TOL
    assert relerr_rows(g["diss"], ref["diss"]) <= TOL
    # time step and eigenvalue / time-step extrema
    assert relerr(g["deltat"], ref["deltat"]) <= TOL
    np.testing.assert_allclose(g["extrema"], ref["extrema"], rtol=1e-13, atol=0)
    # Jacobian blocks and right-hand side, same block-CRS pattern
    assert relerr(g["A"], ref["A"]) <= TOL
    assert relerr(g["B"], ref["B"]) <= TOL
    # block Gauss-Seidel: X within round-off of the reference solve of (almost) the same system
    assert relerr(g["X"], ref["X"]) <= 1e-9
    assert abs(g["gs_rms"] - ref["gs_rms"][0]) <= 1e-9 * abs(ref["gs_rms"][0])


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_block_gauss_seidel_bit_exact(gpu_available, ref_available, direction):
    m, cfg, Q = make_case(n=8, seed=5)
    ref0 = refharness.run(m, cfg, Q, [("begin", 0), ("bc", 0), ("residual", 1), ("deltat", 0), ("jacobian", 1, 0),
                                      ("get", "matrix")])
    A, B = ref0["A"], ref0["B"]
    ref = refharness.run(m, cfg, Q, [("set_matrix", A, B), ("gs", 7, direction), ("get", "matrix")])
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_system(A.reshape(-1, 25), B)
        rms = s.MC_Iterative_Block_LU_Jacobi_CRS(7, direction)
        _, _, X = s.get_system()
    np.testing.assert_array_equal(X, ref["X"])
    assert abs(rms - ref["gs_rms"][0]) <= 1e-13 * abs(ref["gs_rms"][0])


@pytest.mark.parametrize("flux", [0, 1])
@pytest.mark.parametrize("limiter", [-1, 1])
def test_second_order_lsq_residual_matches_reference(gpu_available, ref_available, flux, limiter):
    cfg = dict(CFG1, flux_scheme=flux, order=1, limiter=limiter, limiter_order=1, venkat_k=5.0, mach=0.8,
               mach_min=0.8, alpha_deg=1.25)
    m, cfg, Q = make_case(n=10, seed=21, cfg=cfg)
    steps = [("begin", 0), ("gradient", 0)]
    if limiter != -1:
        steps.append(("limiter",))
    steps += [("bc", 0), ("residual", 1), ("get", "residual"), ("get", "gradients"), ("deltat", 0),
              ("get", "deltat")]
    if limiter != -1:
        steps.append(("get", "limiters"))
    ref = refharness.run(m, cfg, Q, steps)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Compute_Least_Square_Gradient(0)
        if limiter != -1:
            s.Compute_Limiter()
        s.Apply_Boundary_Condition(0)
        s.Compute_Residual(1)
        conv, diss = s.get_residual()
        grad = s.get_gradients()
        s.Compute_DeltaT(0)
        dt = s.get_deltat()
        phi = s.get_limiters() if limiter != -1 else None
    assert relerr_rows(grad, ref["gradients"]) <= TOL
    if limiter != -1:
        assert np.abs(phi - ref["limiters"]).max() <= 1e-10
    assert relerr_rows(conv, ref["conv"]) <= TOL
    if flux == 0:
        assert relerr_rows(diss, ref["diss"]) <= TOL
    else:
        assert np.abs(diss).max() == 0.0 and np.abs(ref["diss"]).max() == 0.0
    assert relerr(dt, ref["deltat"]) <= TOL


def test_hllc_first_order_and_entropy_fix(gpu_available, ref_available):
    for cfg in (dict(CFG1, flux_scheme=1), dict(CFG1, entropy_fix=1)):
        m, cfg, Q = make_case(n=8, seed=31, cfg=cfg)
        ref = refharness.run(m, cfg, Q, [("begin", 0), ("bc", 0), ("residual", 1), ("get", "residual"),
                                         ("deltat", 0), ("get", "deltat"), ("get", "extrema")])
        with Euler3DGPU(m, params_from(cfg)) as s:
            s.set_state(Q)
            s.begin_iteration(0)
            s.Apply_Boundary_Condition(0)
            s.Compute_Residual(1)
            conv, diss = s.get_residual()
            s.Compute_DeltaT(0)
            dt = s.get_deltat()
            ext = s.get_extrema()
        assert relerr_rows(conv, ref["conv"]) <= TOL
        assert relerr_rows(diss, ref["diss"]) <= TOL if np.abs(ref["diss"]).max() > 0 else np.abs(diss).max() == 0
        assert relerr(dt, ref["deltat"]) <= TOL
        np.testing.assert_allclose(ext, ref["extrema"], rtol=1e-13)


def test_implicit_iterations_track_reference(gpu_available, ref_available):
    """Three implicit Euler3D iterations (BC, residual, dt, Jacobian, 10 block-GS
    sweeps, update) on the device against the reference loop."""
    m, cfg, Q = make_case(n=8, seed=41)
    steps = []
    for it in range(3):
        steps += [("begin", it), ("bc", it), ("residual", 1), ("deltat", it), ("jacobian", 1, it), ("gs", 10, 0),
                  ("update", 1.0)]
    steps.append(("get", "state"))
    ref = refharness.run(m, cfg, Q, steps)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        for it in range(3):
            s.begin_iteration(it)
            s.Apply_Boundary_Condition(it)
            s.Compute_Residual(1)
            s.Compute_DeltaT(it)
            s.Compute_Jacobian(1, it)
            s.MC_Iterative_Block_LU_Jacobi_CRS(10, 0)
            s.update(1.0)
        Qg = s.get_state()
    k = m.nnode
    assert relerr_rows(Qg[:, :k], ref["state"][:, :k]) <= 1e-10


@pytest.mark.parametrize("iters", [1, 5])
def test_block_lusgs_bit_exact(gpu_available, ref_available, iters):
    """LU-SGS on the GPU (level-scheduled forward and backward sweeps, pivoted
    diagonal solves) equals the reference's MC_Iterative_Block_LUSGS_CRS bit
    for bit, including its returned RMS."""
    m, cfg, Q = make_case(n=8, seed=6)
    ref0 = refharness.run(m, cfg, Q, [("begin", 0), ("bc", 0), ("residual", 1), ("deltat", 0), ("jacobian", 1, 0),
                                      ("get", "matrix")])
    A, B = ref0["A"], ref0["B"]
    ref = refharness.run(m, cfg, Q, [("set_matrix", A, B), ("lusgs", iters), ("get", "matrix")])
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_system(A.reshape(-1, 25), B)
        rms = s.MC_Iterative_Block_LUSGS_CRS(iters)
        _, _, X = s.get_system()
    np.testing.assert_array_equal(X, ref["X"])
    assert rms == ref["lusgs_rms"][0]


@pytest.mark.parametrize("method,iteration,flux", [(0, 0, 0), (1, 0, 0), (2, 0, 0), (3, 1, 0), (0, 0, 3), (3, 1, 3)])
def test_finite_difference_jacobian_matches_reference(gpu_available, ref_available, method, iteration, flux):
    """Finite-difference Roe Jacobian (JACOBIAN_METHOD_CENTRAL / FORWARD /
    BACKWARD / ALTERNATE) from the reference's own state after its boundary
    update: the off-diagonal blocks (interior-edge difference quotients of
    the matrix-form Roe flux) equal the reference's bit for bit; the diagonal
    blocks, summed per row in another order, to 1e-13 of the row scale.
    Through this library's own boundary update the ghost states differ from
    the reference's in the last bits, which the 1e-8 difference quotient of
    the boundary blocks amplifies by up to 1e8: the diagonal agrees to 1e-8.
    Flux 3 differences Compute_RoeFlux's low-Mach-fix branch (M 0.1)."""
    m, cfg, Q = make_case(n=5, seed=4, cfg=dict(CFG1, flux_scheme=flux, mach=0.1 if flux == 3 else 0.5,
                                                mach_min=0.1 if flux == 3 else 0.5))
    cfg = dict(cfg, jacobian_method=method)
    ref = refharness.run(m, cfg, Q, [("begin", iteration), ("bc", iteration), ("get", "state"), ("residual", 1),
                                     ("deltat", iteration), ("jacobian", 1, iteration), ("get", "matrix"),
                                     ("get", "crs")])
    gpu_cfg = {k: v for k, v in cfg.items() if k != "jacobian_method"}  # a call argument here
    out = []
    for own_bc in (False, True):
        with Euler3DGPU(m, params_from(gpu_cfg)) as s:
            s.set_state(Q if own_bc else ref["state"])
            s.begin_iteration(iteration)
            if own_bc:
                s.Apply_Boundary_Condition(iteration)
            s.Compute_Residual(1)
            s.Compute_DeltaT(iteration)
            s.Compute_Jacobian_FiniteDifference(1, iteration, method)
            A, B, _ = s.get_system()
            IA, JA, IAU = s.get_block_pattern()
        out.append((A, B))
    np.testing.assert_array_equal(IA, ref["IA"])
    np.testing.assert_array_equal(JA, ref["JA"])
    diag = np.zeros(len(JA), bool)
    diag[IAU] = True
    scale = np.abs(ref["A"][diag]).reshape(len(IAU), -1).max(axis=1)
    for (A, B), tol in zip(out, (1e-13, 1e-8)):
        if tol == 1e-13:
            np.testing.assert_array_equal(A[~diag], ref["A"][~diag])
        err = np.abs(A[diag] - ref["A"][diag]).reshape(len(IAU), -1).max(axis=1)
        assert np.all(err <= tol * scale), (tol, float((err / scale).max()))
        np.testing.assert_allclose(B, ref["B"], rtol=0, atol=1e-12 * np.abs(ref["B"]).max())


@pytest.mark.parametrize("face_bc,mach", [((1, 1, 1, 1, 1, 1), 0.1), ((2, 3, 0, 0, 0, 0), 0.2)])
def test_low_mach_fix_residual_and_ghosts_match_reference(gpu_available, ref_available, face_bc, mach):
    """Roe with the low-Mach fix (PRECOND_METHOD_ROE_LMFIX): second-order
    residual (Compute_Flux_Roe_LMFIX) and the ghost states of the
    preconditioned characteristic BC, on an all-far-field cube and on a
    channel (inflow at x = 0, outflow at x = 1, walls elsewhere)."""
    from cfdsolutions_b200 import box_mesh
    cfg = dict(CFG1, flux_scheme=3, order=1, limiter=1, limiter_order=1, venkat_k=5.0, mach=mach, mach_min=mach,
               alpha_deg=0.0 if face_bc[0] == 2 else 2.0)
    m = box_mesh(8, jitter=0.15, seed=41, face_bc=face_bc)
    _, cfg, Q = make_case(cfg=cfg, mesh=m, seed=41)
    ref = refharness.run(m, cfg, Q, [("begin", 0), ("gradient", 0), ("limiter",), ("bc", 0), ("get", "state"),
                                     ("residual", 1), ("get", "residual"), ("deltat", 0), ("get", "deltat")])
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Compute_Least_Square_Gradient(0)
        s.Compute_Limiter()
        s.Apply_Boundary_Condition(0)
        state = s.get_state()
        s.Compute_Residual(1)
        conv, diss = s.get_residual()
        s.Compute_DeltaT(0)
        dt = s.get_deltat()
    assert relerr_rows(state, ref["state"]) <= TOL
    assert relerr_rows(conv, ref["conv"]) <= TOL
    assert relerr_rows(diss, ref["diss"]) <= TOL
    assert relerr(dt, ref["deltat"]) <= TOL


@pytest.mark.parametrize("spots", [False, True], ids=["smooth", "limiter-fix"])
@pytest.mark.parametrize("lorder", [0, 1])
def test_second_order_extrema_match_reference(gpu_available, ref_available, spots, lorder):
    """Eigenvalue extrema of a second-order Roe residual (LSQ + Venkatakrishnan)
    against the reference, also on states with low-pressure spots, where the
    limiter's pressure corrections fire: the reference evaluates the residual
    once with the corrected limiters, so the GPU's first pass (before the
    fixes) must not count (1e-13)."""
    cfg = dict(CFG1, order=1, limiter=1, limiter_order=lorder, venkat_k=5.0, mach=0.8, mach_min=0.8,
               alpha_deg=1.25)
    m, cfg, Q = make_case(n=8, seed=9, cfg=cfg, noise=0.02)
    if spots:
        Q = low_pressure_spots(Q, m.nnode, cfg["gamma"], seed=9)
    ref = refharness.run(m, cfg, Q, [("begin", 0), ("gradient", 0), ("limiter",), ("bc", 0), ("residual", 1),
                                     ("deltat", 0), ("get", "extrema"), ("get", "limiters"), ("get", "residual")])
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Compute_Least_Square_Gradient(0)
        s.Compute_Limiter()
        s.Apply_Boundary_Condition(0)
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        ext = s.get_extrema()
        conv, _ = s.get_residual()
    if spots:
        assert (ref["limiters"] == 0).all(axis=0).sum() >= 3  # the corrections fired
    assert relerr_rows(conv, ref["conv"]) <= TOL
    assert np.abs(ext - ref["extrema"]).max() <= 1e-13 * np.abs(ref["extrema"]).max()
