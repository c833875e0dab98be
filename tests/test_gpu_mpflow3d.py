"""The CUDA path against MPFLOW3D compiled from its own sources.

Same cases as tests/test_oracle_pin_mpflow3d.py (listed, with the
differences that are by design, in tests/_mpf.py), with the GPU in place of
the restatement: MPFLOW3D's preconditioned Roe family with its
preconditioned characteristic BC, its Thornber, HLLC and Roe edge loops,
first and second order (LSQ + Venkatakrishnan / Barth-Jespersen), and the
implicit path's pseudo-time term and right-hand side B = -(Res_Conv +
Res_Diss).  Tolerances: ghost states and time steps 1e-13 (observed a few
1e-16), residuals and Jacobian blocks 1e-12 normwise.
"""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU
from oracle import restatement
from tests import _mpf
from tests._util import params_from, relerr_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mpf_available():
    from oracle import mpfharness
    if not mpfharness.available():
        pytest.skip("MPFLOW3D oracle not built (make -C oracle ref)")
    return True


def _gpu_pass(m, cfg, Q, apply_bc=True):
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        if cfg.get("order", 0) == 1:
            s.Compute_Gradient()
            if cfg.get("limiter", -1) != -1:
                s.Compute_Limiter()
        if apply_bc:
            s.Apply_Boundary_Condition(0)
        out = {"state": s.get_state()}
        s.Compute_Residual(1)
        out["conv"], out["diss"] = s.get_residual()
        s.Compute_DeltaT(0)
        out["deltat"] = s.get_deltat()
        out["extrema"] = s.get_extrema()
    return out


@pytest.mark.parametrize("name,cfg,face_bc", _mpf.PRECOND_CASES, ids=[c[0] for c in _mpf.PRECOND_CASES])
def test_gpu_preconditioned_pass_matches_mpflow3d(gpu_available, mpf_available, name, cfg, face_bc):
    m, cfg, Q = _mpf.case(cfg, face_bc)
    ref = _mpf.mpf_pass(m, cfg, Q)
    g = _gpu_pass(m, cfg, Q)
    assert _mpf.rel(g["state"][:, m.nnode:], ref["state"][:, m.nnode:]) <= 1e-13
    assert relerr_rows(g["conv"], ref["conv"]) <= 1e-12
    assert relerr_rows(g["diss"], ref["diss"]) <= 1e-12
    assert _mpf.rel(g["deltat"], ref["deltat"]) <= 1e-13
    assert _mpf.rel(g["extrema"], ref["extrema"]) <= 1e-13


@pytest.mark.parametrize("name,cfg", _mpf.EDGE_CASES, ids=[c[0] for c in _mpf.EDGE_CASES])
def test_gpu_edge_loop_matches_mpflow3d_on_its_ghost_states(gpu_available, mpf_available, name, cfg):
    """Convective residual, time step and extrema straight against MPFLOW3D;
    the Roe dissipation through the chain GPU = closed form = MPFLOW3D's
    matrix with the nz entry, MPFLOW3D's matrix as written = MPFLOW3D."""
    m, cfg, Q = _mpf.case(cfg)
    ref = _mpf.mpf_pass(m, cfg, Q)
    g = _gpu_pass(m, cfg, ref["state"], apply_bc=False)
    assert relerr_rows(g["conv"], ref["conv"]) <= 1e-12
    assert _mpf.rel(g["deltat"], ref["deltat"]) <= 1e-13
    if cfg["flux_scheme"] == 1:
        assert np.abs(g["diss"]).max() == 0.0 and np.abs(ref["diss"]).max() == 0.0
        return
    assert _mpf.rel(g["extrema"], ref["extrema"]) <= 1e-13
    s_fixed = restatement.Session(m, dict(cfg, mpf_form=2))
    s_written = restatement.Session(m, dict(cfg, mpf_form=1))
    for s, target, tol in ((s_fixed, g["diss"], 1e-12), (s_written, ref["diss"], 1e-12)):
        grad = phi = None
        if cfg.get("order", 0) == 1:
            grad = s.gradient(ref["state"], 0)
            phi = s.limiter(ref["state"], grad)
        _, diss, _, _ = s.residual(ref["state"], grad, phi)
        assert relerr_rows(target, diss) <= tol


@pytest.mark.parametrize("name,cfg", _mpf.JAC_CASES, ids=[c[0] for c in _mpf.JAC_CASES])
def test_gpu_pseudo_time_term_and_rhs_match_mpflow3d(gpu_available, mpf_available, name, cfg):
    m, cfg, Q = _mpf.case(cfg)
    Qb, R, A, B = _mpf.mpf_jacobians(m, cfg, Q)
    mats = {}
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Qb)
        s.begin_iteration(0)
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        for add_time in (0, 1):
            s.Compute_Jacobian(add_time, 0, include_diss=1)
            mats[add_time] = s.get_system()[:2]
        IA, JA, IAU = s.get_block_pattern()
    mine = _mpf.pseudo_time_blocks(mats[1][0], mats[0][0], JA, IAU, R)
    assert _mpf.rel(mine, (A[1] - A[0])[IAU]) <= 1e-12
    if cfg["flux_scheme"] == 4:  # (the Roe case's B carries MPFLOW3D's dissipation matrix)
        assert _mpf.rel(mats[1][1], B) <= 1e-12
