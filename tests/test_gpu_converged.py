"""Converged steady states against the reference's own converged state.

The reference (Euler3D compiled from its sources, oracle/_ref) runs its
implicit loop -- characteristic BCs, least-squares gradient, Venkatakrishnan
limiter, Roe residual, local time step with the CFL ramp, approximate Roe
Jacobian, 10 block Gauss-Seidel sweeps, update
(Euler3D/src/Solver_Steady_Implicit.cpp:35-184) -- with the right-hand side
B = -(Res + Res_Diss) of MPFLOW3D's driver (MPFLOW3D/src/Roe_Jacobian.cpp:237-241;
Euler3D's own B = -Res leaves the dissipation out), until the residual stops
falling (its round-off floor).  The GPU solves the same steady problem with
GMRES(30) + block-multicolour ILU(0) and FP64, FP32 or BF16 storage of the
Jacobian.  Both are fixed points of the same discrete residual, so the
converged density, momentum and energy must agree to 1e-8
(relative to each field's largest magnitude); observed: FP64 and FP32 about
1e-11, BF16 the same after its slightly different path.
"""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, capi, default_params
from oracle import refharness
from tests._util import CFG1, make_case

pytestmark = pytest.mark.gpu

CFG = dict(CFG1, order=1, gradient=0, limiter=1, venkat_k=5.0, mach=0.8, mach_min=0.8, alpha_deg=1.25,
           cfl_min=10.0, cfl_max=1000.0, cfl_ramp=20)


def reference_converged(m, cfg, Q, iterations=120, sweeps=10):
    steps = []
    for it in range(iterations):
        steps += [("begin", it), ("gradient", 0), ("limiter",), ("bc", it), ("residual", 1), ("deltat", it),
                  ("jacobian", 1, it), ("rhs_full",), ("gs", sweeps, 0), ("update", 1.0)]
    steps.append(("get", "state"))
    out = refharness.run(m, cfg, Q, steps)
    return out["state"], np.asarray(out["rms_full"])


def field_errors(a, b, nnode):
    """max |a - b| per field (rho, momentum, energy) over that field's largest |b|."""
    a, b = a[:, :nnode], b[:, :nnode]
    mom = np.abs(b[1:4]).max()
    return (float(np.abs(a[0] - b[0]).max() / np.abs(b[0]).max()), float(np.abs(a[1:4] - b[1:4]).max() / mom),
            float(np.abs(a[4] - b[4]).max() / np.abs(b[4]).max()))


@pytest.fixture(scope="module")
def converged_case(ref_available):
    m, cfg, Q = make_case(n=8, seed=13, cfg=CFG, noise=0.01)
    Qref, rms = reference_converged(m, cfg, Q)
    assert rms[-1] <= 1e-10 * rms[0]  # the reference reached its round-off floor
    return m, cfg, Q, Qref


@pytest.mark.parametrize("name,prec", [("fp64", capi.PREC_FP64), ("fp32", capi.PREC_FP32 | capi.PREC_LOW_ONLY),
                                       ("bf16", capi.PREC_BF16 | capi.PREC_LOW_ONLY)])
def test_converged_state_matches_reference_solve(gpu_available, converged_case, name, prec):
    m, cfg, Q, Qref = converged_case
    with Euler3DGPU(m, default_params(**cfg)) as s:
        s.set_state(Q)
        capi.check(capi.lib.cfd_ilu_mc_order(s.handle, None, None), "cfd_ilu_mc_order")
        g = capi.GmresOpts(30, 60, 1e-3, capi.PC_ILU0_MC, prec, 1)
        st = s.solve_steady(max_iterations=200, drop=1e-11, include_diss=1, linear_solver=1, gmres=g)
        assert st.rms_last <= 1e-10 * st.rms_first, (name, st.iterations, st.rms_last / st.rms_first)
        Qg = s.get_state()
    errs = field_errors(Qg, Qref, m.nnode)
    assert max(errs) <= 1e-8, (name, errs)
