"""The CUDA hot path on a mixed-element mesh (tetrahedra, pyramids, prisms and
hexahedra read from UGRID by cfd_mesh_read_ugrid) against the reference's
own functions on the same median dual: ghost states, first- and second-order
Roe residuals (LSQ + Venkatakrishnan), time steps and the Jacobian's
right-hand side to 1e-12 normwise; the dual is pinned to the reference's
pre-processing in tests/test_mesh_mixed.py."""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU
from cfdsolutions_b200.mesh import read_ugrid
from oracle import refharness
from tests import _mixed
from tests._util import CFG1, make_case, params_from, relerr, relerr_rows

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [0, 1])
def test_mixed_mesh_residual_matches_reference(gpu_available, ref_available, tmp_path, order):
    path = tmp_path / "mixed.ugrid"
    _mixed.write_ugrid(path, *_mixed.mixed_box((4, 3, 3), jitter=0.1, seed=2))
    m = read_ugrid(str(path))
    cfg = dict(CFG1, order=order, limiter=1 if order else -1, venkat_k=5.0, mach=0.8, mach_min=0.8,
               alpha_deg=1.25)
    _, cfg, Q = make_case(mesh=m, cfg=cfg, seed=4, noise=0.02)
    steps = [("begin", 0)]
    if order:
        steps += [("gradient", 0), ("limiter",)]
    steps += [("bc", 0), ("get", "state"), ("residual", 1), ("get", "residual"), ("deltat", 0), ("get", "deltat")]
    ref = refharness.run(m, cfg, Q, steps)
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        if order:
            s.Compute_Least_Square_Gradient(0)
            s.Compute_Limiter()
        s.Apply_Boundary_Condition(0)
        state = s.get_state()
        s.Compute_Residual(1)
        conv, diss = s.get_residual()
        s.Compute_DeltaT(0)
        dt = s.get_deltat()
    assert relerr_rows(state, ref["state"]) <= 1e-13
    assert relerr_rows(conv, ref["conv"]) <= 1e-12
    assert relerr_rows(diss, ref["diss"]) <= 1e-12
    assert relerr(dt, ref["deltat"]) <= 1e-12
