"""Stiffened-gas EOS (p = (gamma - 1) rho e - gamma pinf) on the GPU against
the oracle's restatement, which carries the same EOS; the reference itself is
ideal-gas only, so pinf = 0 stays pinned to it by the parity tests and the
restatement's stiffened-gas algebra is pinned by the property tests of the
oracle (supersonic upwinding of every flux family, freestream preservation).

Tolerance.  In conservative variables the pressure is the difference
(gamma - 1) rho e - gamma pinf of two numbers of size gamma pinf, so two
correct FP64 evaluations differ by about eps * gamma * pinf in p (the GPU
forms it with one fused multiply-add, the restatement with two roundings).
Residuals are compared at 1e-12 * (1 + gamma * pinf) relative (p = 1 is
the reference pressure), the conditioning of the EOS itself; Jacobian blocks,
which hold no such difference, at 1e-12.
"""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, box_mesh
from oracle import restatement
from tests._util import CFG1, make_case, params_from, relerr, relerr_rows
from tests.test_gpu_kernels import gpu_pass

pytestmark = pytest.mark.gpu

WATER = dict(gamma=4.4, pinf=6000.0, mach=0.0062, mach_min=0.0062)  # 1000 kg/m^3, 1 bar, pinf 6e8 Pa, ~10 m/s
CHANNEL_BC = (2, 3, 0, 0, 0, 0)  # inflow at x = 0, outflow at x = lx, slip walls
# MPFLOW3D's Turkel preconditioning, local beta with the freestream Mach as reference
PRECOND = dict(flux_scheme=4, precond_method=5, precond_type=0, precond_mach=0.0062)


def tol(cfg):
    return 1e-12 * (1.0 + cfg["gamma"] * cfg.get("pinf", 0.0))


CASES = [
    ("roe1_far", dict(CFG1, gamma=4.4, pinf=3.0), (1, 1, 1, 1, 1, 1)),
    ("roe2_far", dict(CFG1, gamma=4.4, pinf=3.0, order=1, gradient=1, limiter=1, venkat_k=5.0), (1,) * 6),
    ("hllc2_far", dict(CFG1, gamma=4.4, pinf=3.0, flux_scheme=1, order=1, gradient=1, limiter=1), (1,) * 6),
    ("ausm2_far", dict(CFG1, gamma=4.4, pinf=3.0, flux_scheme=2, order=1, gradient=1, limiter=1), (1,) * 6),
    ("lmfix2_far", dict(CFG1, gamma=4.4, pinf=3.0, flux_scheme=3, order=1, limiter=1, limiter_order=1), (1,) * 6),
    ("lmfix2_water_channel", dict(CFG1, **WATER, flux_scheme=3, order=1, limiter=1, limiter_order=1,
                                  alpha_deg=0.0), CHANNEL_BC),
    ("roe2_water_channel", dict(CFG1, **WATER, order=1, gradient=1, limiter=1, alpha_deg=0.0), CHANNEL_BC),
    ("turkel2_water_channel", dict(CFG1, **WATER, **PRECOND, order=1, limiter=1, alpha_deg=0.0), CHANNEL_BC),
    # (small inflow angles, so that no momentum residual is round-off only)
    ("turkel1_water_channel", dict(CFG1, **WATER, **PRECOND, alpha_deg=1.0, beta_deg=1.0), CHANNEL_BC),
    ("eriksson2_far", dict(CFG1, gamma=4.4, pinf=3.0, flux_scheme=4, precond_method=3, precond_type=1,
                           precond_mach=0.2, order=1, gradient=1, limiter=1, mach=0.1, mach_min=0.1), (1,) * 6),
    ("btw1_far_urlocal", dict(CFG1, flux_scheme=4, precond_method=2, precond_type=2, mach=0.2, mach_min=0.2),
     (1,) * 6),
    ("thornber2_far", dict(CFG1, flux_scheme=5, order=1, gradient=1, limiter=1, mach=0.2, mach_min=0.2), (1,) * 6),
    ("thornber1_water_channel", dict(CFG1, **WATER, flux_scheme=5, alpha_deg=1.0, beta_deg=1.0), CHANNEL_BC),
]


@pytest.mark.parametrize("name,cfg,face_bc", CASES, ids=[c[0] for c in CASES])
def test_stiffened_residual_matches_restatement(gpu_available, name, cfg, face_bc):
    m = box_mesh((12, 6, 6), lengths=(2.0, 1.0, 1.0), jitter=0.1, seed=23, face_bc=face_bc)
    noise = (0.0, 0.02, 0.0) if cfg.get("pinf", 0.0) > 100 else 0.02
    _, cfg, Q = make_case(mesh=m, cfg=cfg, seed=23, noise=noise)
    o = restatement.residual_pass(m, cfg, Q)
    g = gpu_pass(m, cfg, Q)
    t = tol(cfg)
    if "grad" in g:
        assert relerr_rows(g["grad"], o["grad"]) <= t
    if "phi" in g:
        assert np.abs(g["phi"] - o["phi"]).max() <= 1e-12
    assert relerr_rows(g["conv"], o["conv"]) <= t
    if np.abs(o["diss"]).max() > 0:
        assert relerr_rows(g["diss"], o["diss"]) <= t
    assert relerr(g["deltat"], o["deltat"]) <= 1e-12


@pytest.mark.parametrize("flux", [0, 3, 4, 5])
def test_stiffened_jacobian_and_ghosts_match_restatement(gpu_available, flux):
    """Ghost states, approximate Jacobian (for flux 4 with the preconditioned
    dissipation and pseudo-time term) and right-hand side on the water channel."""
    cfg = dict(CFG1, **WATER, **PRECOND, alpha_deg=0.0)
    cfg["flux_scheme"] = flux
    m = box_mesh((10, 5, 5), lengths=(2.0, 1.0, 1.0), jitter=0.1, seed=31, face_bc=CHANNEL_BC)
    _, cfg, Q = make_case(mesh=m, cfg=cfg, seed=31, noise=(0.0, 0.02, 0.0))
    o = restatement.first_order_step(m, cfg, Q, gs_sweeps=1)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Apply_Boundary_Condition(0)
        state = s.get_state()
        farfield = s.get_farfield()
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        s.Compute_Jacobian(1, 0)
        A, B, _ = s.get_system()
    # freestream of the stiffened gas: c^2 = gamma (p + pinf) / rho with rho = p = 1
    assert abs(farfield[6] - np.sqrt(4.4 * 6001.0)) <= 1e-13 * farfield[6]
    # ghost states carry the pressure difference through dp / c^2 and dp / (rho c)
    assert relerr_rows(state, o["state"]) <= 1e-12
    assert relerr(A, o["A"]) <= 1e-12
    assert relerr(B, o["B"]) <= tol(cfg)


def test_low_mach_water_channel_steady_solve(gpu_available):
    """A small water channel (stiffened gas, Turkel-preconditioned Roe, second
    order, inflow/outflow and slip walls, +-2 % velocity noise) reaches a 1e-8
    residual drop with the FP32 Jacobian/ILU(0) as with FP64, to the same
    state (both continued to the round-off floor of the stiffened EOS)."""
    from cfdsolutions_b200 import capi, default_params
    cfg = dict(CFG1, **WATER, **PRECOND, order=1, limiter=1, venkat_k=5.0, alpha_deg=0.0,
               cfl_min=10.0, cfl_max=1e4, cfl_ramp=20)
    m = box_mesh((16, 4, 4), lengths=(4.0, 1.0, 1.0), jitter=0.1, seed=7, face_bc=CHANNEL_BC, rcm=True)
    _, cfg, Q = make_case(mesh=m, cfg=cfg, seed=7, noise=(0.0, 0.02, 0.0))
    states = {}
    for name, prec in (("fp64", capi.PREC_FP64), ("fp32", capi.PREC_FP32 | capi.PREC_LOW_ONLY)):
        with Euler3DGPU(m, default_params(**cfg)) as s:
            s.set_state(Q)
            capi.check(capi.lib.cfd_ilu_mc_order(s.handle, None, None), "cfd_ilu_mc_order")
            g = capi.GmresOpts(30, 30, 0.1, capi.PC_ILU0_MC, prec, 1)
            st = s.solve_steady(max_iterations=400, drop=1e-8, include_diss=1, linear_solver=1, gmres=g)
            assert st.rms_last <= 1e-8 * st.rms_first, (name, st.iterations, st.rms_last / st.rms_first)
            s.set_params(default_params(**dict(cfg, cfl_min=cfg["cfl_max"], cfl_ramp=0)))
            s.solve_steady(max_iterations=60, drop=1e-3, include_diss=1, linear_solver=1, gmres=g)
            states[name] = s.get_state()[:, :m.nnode]
    a, b = states["fp32"], states["fp64"]
    for v in range(5):
        scale = np.abs(b[v]).max() if v in (0, 4) else np.abs(b[1:4]).max()
        assert np.abs(a[v] - b[v]).max() <= 1e-8 * scale, (v, np.abs(a[v] - b[v]).max() / scale)
