"""Cases and runners shared by the MPFLOW3D pins (restatement and GPU).

MPFLOW3D is compiled from its own sources into oracle/_ref (oracle/Makefile)
and driven one function at a time by oracle/mpf_harness.cpp.  Two of its
variable sets are used:

* VARIABLE_CON (``mpf_variable="con"``): MPFLOW3D's residual, boundary update
  and time step in conservative variables, the library's formulation.  Run
  with the implicit scheme, so that the explicit scheme's residual
  preconditioning (MPFLOW3D/src/Roe_Fluxes.cpp:3962-3990) stays off; its
  Jacobian is never called (it needs RUP, CompressibleUtils.cpp:85-186).
* VARIABLE_RUP (the implicit path of MPFLOW3D): the Jacobian and right-hand
  side, compared through the chain rule d/d(rho,u,v,w,p) = d/dQ . dQ/d(rho,u,v,w,p).

Where MPFLOW3D and the library differ by design, the cases say so:

* MPFLOW3D's non-preconditioned characteristic BC (BC.cpp:33-100) is not
  Euler3D's, which the library follows, so the Roe, HLLC and Thornber cases
  take MPFLOW3D's own ghost states as input and compare the edge loop.
* MPFLOW3D forms the Roe dissipation as Mop P dW (Roe_Fluxes.cpp:1605-1683)
  with E1 (1 - ny^2) on the w-momentum diagonal, where the closed form has
  E1 (1 - nz^2).  The restatement's ``mpf_form=1`` writes that matrix as
  MPFLOW3D does and is pinned to it; ``mpf_form=2`` (the same matrix with
  nz) equals the library's closed form.
* MPFLOW3D's HLLC records the eigenvalue extrema, Euler3D's (the library's)
  does not; HLLC extrema are not compared.
"""
from __future__ import annotations

import numpy as np

from cfdsolutions_b200 import box_mesh
from tests._util import CFG1, make_case

CHANNEL_BC = (2, 3, 0, 0, 0, 0)  # inflow at x = 0, outflow at x = lx, slip walls


def precond(method, ptype, **kw):
    return dict(CFG1, flux_scheme=4, precond_method=method, precond_type=ptype, precond_mach=0.2, mach=0.2,
                mach_min=0.2, **kw)


SECOND = dict(order=1, gradient=0, limiter=1, venkat_k=5.0)

# The preconditioned family with MPFLOW3D's preconditioned characteristic BC:
# the whole pass (BC, gradient, limiter, residual, time step) is compared.
PRECOND_CASES = [
    ("turkel_local", precond(5, 0), None),
    ("turkel_global", precond(5, 1), None),
    ("turkel_urlocal", precond(5, 2), None),
    ("eriksson_local", precond(3, 0), None),
    ("eriksson_global", precond(3, 1), None),
    ("btw_global", precond(2, 1), None),
    ("btw_urlocal", precond(2, 2), None),
    ("turkel_local_o2", precond(5, 0, **SECOND), None),
    ("turkel_channel", precond(5, 0, alpha_deg=1.0, beta_deg=1.0), CHANNEL_BC),
    ("turkel_channel_o2", precond(5, 0, alpha_deg=1.0, beta_deg=1.0, **SECOND), CHANNEL_BC),
]

# Flux families whose BC differs by design: MPFLOW3D's ghost states are the input.
EDGE_CASES = [
    ("roe", dict(CFG1)),
    ("roe_entropy_fix", dict(CFG1, entropy_fix=1)),
    ("roe_o2_venkat", dict(CFG1, **SECOND)),
    ("roe_o2_bj_smooth", dict(CFG1, **dict(SECOND, limiter=0), limiter_smooth=1)),
    ("roe_o2_limiter_order2", dict(CFG1, **SECOND, limiter_order=1)),
    ("hllc", dict(CFG1, flux_scheme=1)),
    ("hllc_o2", dict(CFG1, flux_scheme=1, **SECOND)),
    ("thornber", dict(CFG1, flux_scheme=5, mach=0.2, mach_min=0.2)),
    ("thornber_o2", dict(CFG1, flux_scheme=5, mach=0.2, mach_min=0.2, **SECOND)),
]

# Jacobian pseudo-time term and B = -(Res_Conv + Res_Diss), MPFLOW3D's implicit (RUP) path.
JAC_CASES = [
    ("roe", dict(CFG1)),
    ("turkel_local", precond(5, 0)),
    ("eriksson_global", precond(3, 1)),
    ("btw_urlocal", precond(2, 2)),
]


# The library's RUP formulation (cfd_params.variables = CFD_VARS_RUP) against
# MPFLOW3D's own (VARIABLE_RUP): the same state handed over unchanged.
RUP = dict(variables=1)
RUP_PASS_CASES = [(n, dict(c, **RUP), bc) for n, c, bc in PRECOND_CASES
                  if n in ("turkel_local", "eriksson_global", "btw_urlocal", "turkel_local_o2", "turkel_channel_o2")]
RUP_EDGE_CASES = [(n, dict(c, **RUP)) for n, c in EDGE_CASES
                  if n in ("roe", "roe_o2_venkat", "roe_o2_bj_smooth", "hllc", "hllc_o2", "thornber", "thornber_o2")]
# the whole Jacobian in (rho,u,v,w,p) columns, with the pseudo-time term, and B
RUP_JAC_CASES = [(n, dict(c, **RUP)) for n, c in JAC_CASES] + [("roe_o2_venkat", dict(CFG1, **SECOND, **RUP))]


def mesh_for(face_bc):
    if face_bc is None:
        return box_mesh(5, jitter=0.15, seed=11)
    return box_mesh((8, 4, 4), lengths=(2.0, 1.0, 1.0), jitter=0.1, seed=23, face_bc=face_bc)


def case(cfg, face_bc=None):
    m = mesh_for(face_bc)
    return make_case(mesh=m, cfg=cfg, seed=23 if face_bc else 11, noise=0.02)


PASS_STEPS = [("begin", 0), ("gradient",), ("bc", 0), ("get", "state"), ("residual", 1), ("deltat", 0),
              ("get", "residual"), ("get", "deltat"), ("get", "extrema")]


def mpf_pass(m, cfg, Q):
    """MPFLOW3D (conservative variables): gradient + limiter, BC, residual, time step."""
    from oracle import mpfharness
    return mpfharness.run(m, dict(cfg, mpf_variable="con"), Q, PASS_STEPS)


def rup_case(cfg, face_bc=None):
    """A case's mesh, configuration and state in (rho, u, v, w, p)."""
    from cfdsolutions_b200 import to_rup
    m, cfg, Q = case(cfg, face_bc)
    return m, cfg, to_rup(Q, cfg.get("gamma", 1.4), cfg.get("pinf", 0.0))


def mpf_pass_rup(m, cfg, R):
    """MPFLOW3D in its RUP variables: gradient + limiter, BC, residual, time step."""
    from oracle import mpfharness
    return mpfharness.run(m, cfg, R, PASS_STEPS)


def mpf_jacobian_rup(m, cfg, R):
    """MPFLOW3D's implicit path on a RUP state: the pass, then the Jacobian
    with the pseudo-time term.  Returns (post-BC state, A, B)."""
    from oracle import mpfharness
    out = mpfharness.run(m, cfg, R, PASS_STEPS + [("jacobian", 1, 0), ("get", "matrix")])
    return out["state"], out["A"], out["B"]


def mpf_jacobians(m, cfg, Q):
    """MPFLOW3D's implicit path (RUP): first-order pass, then the Jacobian
    without and with the pseudo-time term.  Returns (post-BC state, {0: A, 1: A}, B)."""
    from oracle import mpfharness
    out = {}
    for add_time in (0, 1):
        steps = PASS_STEPS + [("jacobian", add_time, 0), ("get", "matrix")]
        out[add_time] = mpfharness.run(m, cfg, Q, steps)
    return out[1]["state"], out[1]["state_rup"], {k: v["A"] for k, v in out.items()}, out[1]["B"]


def pseudo_time_blocks(A1, A0, JA, IAU, R):
    """Diagonal pseudo-time blocks of a conservative-variable Jacobian pair,
    in (rho, u, v, w, p) columns (right-multiplied by dQ/d(rho,u,v,w,p))."""
    from oracle import mpfharness
    return mpfharness.jacobian_to_rup(A1 - A0, JA, R)[IAU]


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
