"""The restatement against MPFLOW3D compiled from its own sources.

Every case runs MPFLOW3D's own functions (oracle/_ref/libmpflow3d_ref.so,
one spawned process per session) and the restatement (oracle/cfd_oracle.c)
on the same mesh and state; tests/_mpf.py lists the cases and the
differences that are by design.  Tolerances: ghost states and time steps
1e-13, residuals 1e-12 normwise (observed <= 1e-13), Jacobian blocks 1e-12.
"""
import numpy as np
import pytest

from oracle import restatement
from tests import _mpf
from tests._util import relerr_rows


@pytest.fixture(scope="module")
def mpf_available():
    from oracle import mpfharness
    if not mpfharness.available():
        pytest.skip("MPFLOW3D oracle not built (make -C oracle ref)")
    return True


def _restatement_pass(m, cfg, Q, apply_bc=True):
    s = restatement.Session(m, cfg)
    Qb = s.apply_bc(Q) if apply_bc else np.array(Q, copy=True)
    grad = phi = None
    if cfg.get("order", 0) == 1:
        grad = s.gradient(Qb, cfg.get("gradient", 0))
        if cfg.get("limiter", -1) != -1:
            phi = s.limiter(Qb, grad)
    conv, diss, dts, ext = s.residual(Qb, grad, phi)
    dt, ext2 = s.deltat(dts)
    return dict(state=Qb, conv=conv, diss=diss, deltat=dt, extrema=np.r_[ext, ext2])


@pytest.mark.parametrize("name,cfg,face_bc", _mpf.PRECOND_CASES, ids=[c[0] for c in _mpf.PRECOND_CASES])
def test_preconditioned_pass_matches_mpflow3d(mpf_available, name, cfg, face_bc):
    """Turkel / Eriksson / BTW preconditioned Roe (Roe_Fluxes.cpp:2043) with
    local, global and unrestricted-local beta, the preconditioned
    characteristic BC (BC.cpp:113) on far field and on inflow/outflow/slip
    walls, first and second order (LSQ + Venkatakrishnan)."""
    m, cfg, Q = _mpf.case(cfg, face_bc)
    ref = _mpf.mpf_pass(m, cfg, Q)
    o = _restatement_pass(m, cfg, Q)
    assert _mpf.rel(o["state"][:, m.nnode:], ref["state"][:, m.nnode:]) <= 1e-13
    assert relerr_rows(o["conv"], ref["conv"]) <= 1e-12
    assert relerr_rows(o["diss"], ref["diss"]) <= 1e-12
    assert _mpf.rel(o["deltat"], ref["deltat"]) <= 1e-13
    assert _mpf.rel(o["extrema"], ref["extrema"]) <= 1e-13


@pytest.mark.parametrize("name,cfg", _mpf.EDGE_CASES, ids=[c[0] for c in _mpf.EDGE_CASES])
def test_edge_loop_matches_mpflow3d_on_its_ghost_states(mpf_available, name, cfg):
    """Roe (MPFLOW3D's matrix-form dissipation, ``mpf_form=1``), HLLC
    (HLLC_Fluxes.cpp:1610) and Thornber (Roe_Fluxes.cpp:1081), first and
    second order, from MPFLOW3D's own post-BC state."""
    m, cfg, Q = _mpf.case(cfg)
    ref = _mpf.mpf_pass(m, cfg, Q)
    o = _restatement_pass(m, dict(cfg, mpf_form=1), ref["state"], apply_bc=False)
    assert relerr_rows(o["conv"], ref["conv"]) <= 1e-12
    assert relerr_rows(o["diss"], ref["diss"]) <= 1e-12
    assert _mpf.rel(o["deltat"], ref["deltat"]) <= 1e-13
    if cfg["flux_scheme"] != 1:
        assert _mpf.rel(o["extrema"], ref["extrema"]) <= 1e-13


@pytest.mark.parametrize("name,cfg", [c for c in _mpf.EDGE_CASES if c[1]["flux_scheme"] in (0, 5)],
                         ids=[c[0] for c in _mpf.EDGE_CASES if c[1]["flux_scheme"] in (0, 5)])
def test_mpflow3d_roe_matrix_differs_from_closed_form_only_in_its_w_entry(name, cfg):
    """With the w-momentum diagonal written E1 (1 - nz^2), MPFLOW3D's matrix
    form equals the closed form the library uses (FluxTest.cpp:3143-3200) to
    round-off; as written (E1 (1 - ny^2)) it does not."""
    m, cfg, Q = _mpf.case(cfg)
    closed = _restatement_pass(m, cfg, Q)
    fixed = _restatement_pass(m, dict(cfg, mpf_form=2), Q)
    as_written = _restatement_pass(m, dict(cfg, mpf_form=1), Q)
    assert relerr_rows(fixed["conv"], closed["conv"]) == 0.0
    assert relerr_rows(fixed["diss"], closed["diss"]) <= 1e-13
    assert relerr_rows(as_written["diss"], closed["diss"]) > 1e-6


@pytest.mark.parametrize("name,cfg", _mpf.JAC_CASES, ids=[c[0] for c in _mpf.JAC_CASES])
def test_pseudo_time_term_and_rhs_match_mpflow3d(mpf_available, name, cfg):
    """MPFLOW3D's implicit path (RUP variables): the Jacobian's pseudo-time
    term (V/dt) Mop Kinv (Roe_Jacobian.cpp:241-264) and B = -(Res_Conv +
    Res_Diss) (:237-241), against the restatement's conservative-variable
    Jacobian through the chain rule, from MPFLOW3D's post-BC state."""
    m, cfg, Q = _mpf.case(cfg)
    Qb, R, A, B = _mpf.mpf_jacobians(m, cfg, Q)
    s = restatement.Session(m, dict(cfg, mpf_form=1))
    conv, diss, dts, _ = s.residual(Qb)
    dt, _ = s.deltat(dts)
    A1, B1 = s.jacobian(Qb, dt, conv, diss, add_time=1, include_diss=1)
    A0, _ = s.jacobian(Qb, dt, conv, diss, add_time=0, include_diss=1)
    mine = _mpf.pseudo_time_blocks(A1, A0, s.JA, s.IAU, R)
    theirs = (A[1] - A[0])[s.IAU]
    assert _mpf.rel(mine, theirs) <= 1e-12
    assert _mpf.rel(B1, B) <= 1e-12


# ---------------------------------------------------------------- RUP variables
@pytest.mark.parametrize("name,cfg,face_bc", _mpf.RUP_PASS_CASES, ids=[c[0] for c in _mpf.RUP_PASS_CASES])
def test_rup_preconditioned_pass_matches_mpflow3d(mpf_available, name, cfg, face_bc):
    """The restatement with (rho, u, v, w, p) states against MPFLOW3D's
    VARIABLE_RUP: ghost states of the preconditioned characteristic BC written
    in RUP, gradients and limiters of the RUP variables, faces reconstructed in
    them (HigherOrderReconstructQ.cpp:21-72), residual and time step."""
    m, cfg, R = _mpf.rup_case(cfg, face_bc)
    ref = _mpf.mpf_pass_rup(m, cfg, R)
    o = _restatement_pass(m, cfg, R)
    assert _mpf.rel(o["state"][:, m.nnode:], ref["state"][:, m.nnode:]) <= 1e-13
    assert relerr_rows(o["conv"], ref["conv"]) <= 1e-12
    assert relerr_rows(o["diss"], ref["diss"]) <= 1e-12
    assert _mpf.rel(o["deltat"], ref["deltat"]) <= 1e-13
    assert _mpf.rel(o["extrema"], ref["extrema"]) <= 1e-13


@pytest.mark.parametrize("name,cfg", _mpf.RUP_EDGE_CASES, ids=[c[0] for c in _mpf.RUP_EDGE_CASES])
def test_rup_edge_loop_matches_mpflow3d_on_its_ghost_states(mpf_available, name, cfg):
    """Roe (MPFLOW3D's matrix form as written, ``mpf_form=1``), HLLC and
    Thornber (velocities blended at fixed rho and p) on RUP states, first and
    second order, from MPFLOW3D's own post-BC state."""
    m, cfg, R = _mpf.rup_case(cfg)
    ref = _mpf.mpf_pass_rup(m, cfg, R)
    o = _restatement_pass(m, dict(cfg, mpf_form=1), ref["state"], apply_bc=False)
    assert relerr_rows(o["conv"], ref["conv"]) <= 1e-12
    assert relerr_rows(o["diss"], ref["diss"]) <= 1e-12
    assert _mpf.rel(o["deltat"], ref["deltat"]) <= 1e-13
    if cfg["flux_scheme"] != 1:
        assert _mpf.rel(o["extrema"], ref["extrema"]) <= 1e-13


@pytest.mark.parametrize("name,cfg", _mpf.RUP_JAC_CASES, ids=[c[0] for c in _mpf.RUP_JAC_CASES])
def test_rup_jacobian_matches_mpflow3d(mpf_available, name, cfg):
    """MPFLOW3D's whole implicit system in (rho, u, v, w, p) columns: the
    convective blocks dF/dW at the nodes (CompressibleUtils.cpp:85-186), the
    dissipation Mop |A| at the Roe state (Roe_Fluxes.cpp:3009-3203, its
    w-momentum entry as written, ``mpf_form=1``; Turkel family :3440-3810), the
    pseudo-time term (V/dt) Mop [Kinv] (Roe_Jacobian.cpp:241-264) and
    B = -(Res_Conv + Res_Diss), from MPFLOW3D's post-BC state."""
    m, cfg, R = _mpf.rup_case(cfg)
    Rb, A, B = _mpf.mpf_jacobian_rup(m, cfg, R)
    s = restatement.Session(m, dict(cfg, mpf_form=1))
    grad = phi = None
    if cfg.get("order", 0) == 1:
        grad = s.gradient(Rb, cfg.get("gradient", 0))
        phi = s.limiter(Rb, grad)
    conv, diss, dts, _ = s.residual(Rb, grad, phi)
    dt, _ = s.deltat(dts)
    A1, B1 = s.jacobian(Rb, dt, conv, diss, add_time=1, include_diss=1)
    assert _mpf.rel(A1, A) <= 1e-12
    assert _mpf.rel(B1, B) <= 1e-12
