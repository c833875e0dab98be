"""The CUDA path with (rho, u, v, w, p) states (cfd_params.variables = CFD_VARS_RUP).

MPFLOW3D's implicit formulation (VARIABLE_RUP): gradients, limiters and the
second-order faces act on the stored (rho, u, v, w, p), ghost states are
written in them, and the Jacobian's columns and the update refer to them.
Compared with the restatement in the same variables (itself pinned to
MPFLOW3D's own functions in tests/test_oracle_pin_mpflow3d.py), and where the
library and MPFLOW3D agree by design (the preconditioned family, whose BC the
library follows) with MPFLOW3D directly, including three implicit iterations.
Tolerances: ghost states and time steps 1e-13, residuals and Jacobian blocks
1e-12 normwise, iterates 1e-10 (as the Euler3D loop's).
"""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, box_mesh, to_conservative, to_rup
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
        s.Compute_Jacobian(1, 0, include_diss=1)
        out["A"], out["B"], _ = s.get_system()
    return out


def _oracle_pass(m, cfg, Q, apply_bc=True):
    s = restatement.Session(m, cfg)
    Qb = s.apply_bc(Q) if apply_bc else np.array(Q, copy=True)
    grad = phi = None
    if cfg.get("order", 0) == 1:
        grad = s.gradient(Qb, cfg.get("gradient", 0))
        if cfg.get("limiter", -1) != -1:
            phi = s.limiter(Qb, grad)
    conv, diss, dts, ext = s.residual(Qb, grad, phi)
    dt, ext2 = s.deltat(dts)
    A, B = s.jacobian(Qb, dt, conv, diss, add_time=1, include_diss=1)
    return dict(state=Qb, conv=conv, diss=diss, deltat=dt, extrema=np.r_[ext, ext2], A=A, B=B)


def _check(g, o, nnode, extrema=True):
    assert _mpf.rel(g["state"][:, nnode:], o["state"][:, nnode:]) <= 1e-13
    assert relerr_rows(g["conv"], o["conv"]) <= 1e-12
    assert relerr_rows(g["diss"], o["diss"]) <= 1e-12
    assert _mpf.rel(g["deltat"], o["deltat"]) <= 1e-13
    if extrema:
        assert _mpf.rel(g["extrema"], o["extrema"]) <= 1e-13
    assert _mpf.rel(g["A"].reshape(-1), np.asarray(o["A"]).reshape(-1)) <= 1e-12
    assert _mpf.rel(g["B"], o["B"]) <= 1e-12


@pytest.mark.parametrize("name,cfg,face_bc", _mpf.RUP_PASS_CASES, ids=[c[0] for c in _mpf.RUP_PASS_CASES])
def test_gpu_rup_preconditioned_pass_and_jacobian_match_mpflow3d(gpu_available, mpf_available, name, cfg,
                                                                 face_bc):
    """Turkel / Eriksson / BTW with the preconditioned characteristic BC on
    RUP states: ghost states, residual, time step, extrema, the whole
    Jacobian in (rho,u,v,w,p) columns and B, against MPFLOW3D itself and
    against the restatement."""
    m, cfg, R = _mpf.rup_case(cfg, face_bc)
    g = _gpu_pass(m, cfg, R)
    _check(g, _oracle_pass(m, cfg, R), m.nnode)
    ref = _mpf.mpf_pass_rup(m, cfg, R)
    assert _mpf.rel(g["state"][:, m.nnode:], ref["state"][:, m.nnode:]) <= 1e-13
    assert relerr_rows(g["conv"], ref["conv"]) <= 1e-12
    assert relerr_rows(g["diss"], ref["diss"]) <= 1e-12
    assert _mpf.rel(g["deltat"], ref["deltat"]) <= 1e-13
    if cfg.get("order", 0) == 0:
        Rb, A, B = _mpf.mpf_jacobian_rup(m, cfg, R)
        assert _mpf.rel(g["A"].reshape(-1), A.reshape(-1)) <= 1e-12
        assert _mpf.rel(g["B"], B) <= 1e-12


@pytest.mark.parametrize("name,cfg", _mpf.RUP_EDGE_CASES, ids=[c[0] for c in _mpf.RUP_EDGE_CASES])
def test_gpu_rup_edge_loop_and_jacobian_match_restatement(gpu_available, mpf_available, name, cfg):
    """Roe (closed-form dissipation), HLLC and Thornber on RUP states from
    MPFLOW3D's own post-BC state, with the Jacobian; the restatement's Roe in
    MPFLOW3D's matrix form as written is the pinned one, its closed form (the
    library's) differs from it only in MPFLOW3D's w-momentum entry."""
    m, cfg, R = _mpf.rup_case(cfg)
    Rb = _mpf.mpf_pass_rup(m, cfg, R)["state"]
    _check(_gpu_pass(m, cfg, Rb, apply_bc=False), _oracle_pass(m, cfg, Rb, apply_bc=False), m.nnode,
           extrema=cfg["flux_scheme"] != 1)


@pytest.mark.parametrize("name,cfg", [("roe", dict(_mpf.CFG1, variables=1)),
                                      ("roe_o2", dict(_mpf.CFG1, **_mpf.SECOND, variables=1)),
                                      ("hllc", dict(_mpf.CFG1, flux_scheme=1, variables=1)),
                                      ("stiffened", dict(_mpf.CFG1, pinf=30.0, variables=1))])
def test_gpu_rup_full_pass_matches_restatement(gpu_available, name, cfg):
    """The library's own characteristic BC (Euler3D's, written in RUP), the
    residual, time step and Jacobian on RUP states, ideal and stiffened gas."""
    m, cfg, Q = _mpf.case(cfg)
    R = to_rup(Q, cfg["gamma"], cfg.get("pinf", 0.0))
    _check(_gpu_pass(m, cfg, R), _oracle_pass(m, cfg, R), m.nnode, extrema=cfg["flux_scheme"] != 1)


def test_gpu_rup_first_order_residual_equals_conservative(gpu_available):
    """At first order the faces are the node states, so on the same states
    (ghosts included) the residual and time step of the RUP formulation equal
    the conservative ones to round-off.  (The characteristic BC averages the
    interior and ghost states in the stored variables, as MPFLOW3D does,
    BC.cpp:171, so the ghost states it writes differ between the two.)"""
    cfg = dict(_mpf.CFG1)
    m, cfg, Q = _mpf.case(cfg)
    c = _gpu_pass(m, cfg, Q, apply_bc=False)
    r = _gpu_pass(m, dict(cfg, variables=1), to_rup(Q, cfg["gamma"]), apply_bc=False)
    assert relerr_rows(r["conv"], c["conv"]) <= 1e-12
    assert relerr_rows(r["diss"], c["diss"]) <= 1e-12
    assert _mpf.rel(r["deltat"], c["deltat"]) <= 1e-13
    assert _mpf.rel(to_conservative(r["state"], cfg["gamma"]), c["state"]) <= 1e-15


def test_gpu_rup_implicit_iterations_track_mpflow3d(gpu_available, mpf_available):
    """Three implicit MPFLOW3D iterations in RUP (Turkel, local beta: BC,
    residual, time step, Jacobian, 10 block-GS sweeps, Q += X) on the device
    against MPFLOW3D's own loop (Solver_Steady_Implicit.cpp:111-184)."""
    m, cfg, R = _mpf.rup_case(_mpf.precond(5, 0, variables=1))
    steps = []
    for it in range(3):
        steps += [("begin", it), ("bc", it), ("residual", 1), ("deltat", it), ("jacobian", 1, it), ("gs", 10, 0),
                  ("update", 1.0)]
    steps.append(("get", "state"))
    from oracle import mpfharness
    ref = mpfharness.run(m, cfg, R, steps)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(R)
        for it in range(3):
            s.begin_iteration(it)
            s.Apply_Boundary_Condition(it)
            s.Compute_Residual(1)
            s.Compute_DeltaT(it)
            s.Compute_Jacobian(1, it, include_diss=1)
            s.MC_Iterative_Block_LU_Jacobi_CRS(10, 0)
            s.update(1.0)
        Rg = s.get_state()
    k = m.nnode
    assert relerr_rows(Rg[:, :k], ref["state"][:, :k]) <= 1e-10
    assert relerr_rows(Rg[:, :k], R[:, :k]) > 1e-6  # the iterations moved the state


def _water_channel_drop(variables, drop, max_iterations=400):
    """Drop reached by the steady solve of a small stiffened-gas water channel
    (Turkel-preconditioned Roe, second order, inflow/outflow and slip walls)."""
    from cfdsolutions_b200 import capi, default_params
    water = dict(gamma=4.4, pinf=6000.0, mach=0.0062, mach_min=0.0062)
    cfg = dict(_mpf.CFG1, **water, flux_scheme=4, precond_method=5, precond_type=0, precond_mach=0.0062, order=1,
               limiter=1, venkat_k=5.0, alpha_deg=0.0, cfl_min=10.0, cfl_max=1e4, cfl_ramp=20)
    m = box_mesh((16, 4, 4), lengths=(4.0, 1.0, 1.0), jitter=0.1, seed=7, face_bc=_mpf.CHANNEL_BC, rcm=True)
    _, cfg, Q = _mpf.make_case(mesh=m, cfg=cfg, seed=7, noise=(0.0, 0.02, 0.0))
    state = Q if variables == 0 else to_rup(Q, cfg["gamma"], cfg["pinf"])
    with Euler3DGPU(m, default_params(**dict(cfg, variables=variables))) as s:
        s.set_state(state)
        capi.check(capi.lib.cfd_ilu_mc_order(s.handle, None, None), "cfd_ilu_mc_order")
        g = capi.GmresOpts(30, 30, 0.1, capi.PC_ILU0_MC, capi.PREC_FP64, 1)
        st = s.solve_steady(max_iterations=max_iterations, drop=drop, include_diss=1, linear_solver=1, gmres=g)
        return st.rms_last / st.rms_first, st.iterations


def test_gpu_rup_stiffened_steady_solve_goes_below_the_conservative_floor(gpu_available):
    """Water as a stiffened gas (gamma pinf = 26,400 times the pressure):
    in conservative variables the pressure is a difference of numbers of
    that size and the implicit solve stalls near a 1e-10 drop; stored as
    (rho, u, v, w, p) the same solve goes on to a 1e-12 drop."""
    drop, its = _water_channel_drop(1, 1e-12)
    assert drop <= 1e-12, (drop, its)


def test_gpu_rup_option_checks(gpu_available):
    """variables other than CFD_VARS_CONSERVATIVE / CFD_VARS_RUP is
    CFD_ERR_ARG; the finite-difference Jacobian and the physical-time driver,
    written for conservative states, return CFD_ERR_UNSUPPORTED on a RUP
    context and leave it usable."""
    from cfdsolutions_b200 import capi, default_params
    m, cfg, Q = _mpf.case(dict(_mpf.CFG1))
    with Euler3DGPU(m, params_from(cfg)) as s:
        with pytest.raises(capi.CfdError) as e:
            s.set_params(default_params(**dict(cfg, variables=2)))
        assert e.value.code == -1  # CFD_ERR_ARG
        s.set_params(default_params(**dict(cfg, variables=1)))
        s.set_state(to_rup(Q, cfg["gamma"]))
        s.begin_iteration(0)
        s.Apply_Boundary_Condition(0)
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        with pytest.raises(capi.CfdError) as e:
            s.Compute_Jacobian_FiniteDifference(1, 0)
        assert e.value.code == -8  # CFD_ERR_UNSUPPORTED
        with pytest.raises(capi.CfdError) as e:
            s.solve_unsteady(0.1, 1)
        assert e.value.code == -8
        s.Compute_Jacobian(1, 0, include_diss=1)
        _, B, _ = s.get_system()
        assert np.isfinite(B).all()
