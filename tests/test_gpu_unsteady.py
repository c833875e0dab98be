"""Physical-time implicit solve (MPFLOW3D's Solver_Unsteady_Implicit) on the
GPU against the same loop on the oracle's restatement, and the freestream as
a solution of every physical step."""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, box_mesh, capi
from oracle import restatement
from tests._util import CFG1, make_case, params_from, relerr_rows

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bdf2,order", [(False, 0), (True, 0), (True, 1)])
def test_unsteady_matches_restatement(gpu_available, bdf2, order):
    cfg = dict(CFG1, order=order, limiter=1 if order else -1, venkat_k=5.0)
    m = box_mesh(6, jitter=0.15, seed=19)
    _, cfg, Q = make_case(cfg=cfg, mesh=m, seed=19, noise=0.02)
    dt, steps, inner = 0.05, 3, 3
    ref = restatement.unsteady(m, cfg, Q, dt, steps, inner, bdf2=bdf2)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        g = capi.GmresOpts(30, 3000, 1e-13, capi.PC_ILU0, capi.PREC_FP64, 1)
        st = s.solve_unsteady(dt, steps, inner, bdf2=bdf2, gmres=g)
        out = s.get_state()
    assert st.steps == steps and st.inner_iterations == steps * inner
    n = m.nnode
    # both solve each Newton system to 1e-13; the states agree to its conditioning
    assert relerr_rows(out[:, :n], ref[:, :n]) <= 1e-10


def test_unsteady_keeps_a_freestream(gpu_available):
    m, cfg, Q = make_case(n=5, seed=3, noise=0.0)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        st = s.solve_unsteady(0.1, 4, 2, bdf2=True, linear_solver=0, linear_iters=10)
        out = s.get_state()
    assert st.rms_last < 1e-12
    np.testing.assert_allclose(out[:, :m.nnode], Q[:, :m.nnode], rtol=1e-12, atol=1e-14)
