"""The pipelined end-to-end residual step against the unpipelined one.

cfd_residual_step with a host state in and both residuals out copies the
state up and the residuals down in node chunks while other chunks are
computed.  Every kernel computes a node exactly as the whole-mesh launch
does, so the residuals, time steps, extrema, gradients and limiters must be
bit-identical to the step run as one call after the other, including when the
limiter's pressure fixes fire (the residuals are then evaluated again after
the chunks went down, and copied again).
"""
import numpy as np
import pytest
import torch

from cfdsolutions_b200 import Euler3DGPU, box_mesh, default_params, perturbed_freestream
from cfdsolutions_b200.mesh import NUMBERING_PATCH_RCM
from tests._util import low_pressure_spots

BASE = dict(order=1, limiter=1, limiter_order=0, gradient=1, venkat_k=5.0, gamma=1.4, mach=0.8, mach_min=0.8,
            alpha_deg=1.25, cfl_min=10.0, cfl_max=10.0)


def _steps(m, params, Q, chunks, iterations=3):
    stream = torch.cuda.Stream()
    conv = torch.empty((5, m.nnode), dtype=torch.float64).pin_memory().numpy()
    diss = torch.empty((5, m.nnode), dtype=torch.float64).pin_memory().numpy()
    qh = torch.from_numpy(np.ascontiguousarray(Q)).pin_memory().numpy()
    out = []
    with Euler3DGPU(m, params, stream=stream.cuda_stream) as s:
        s.set_step_pipeline(chunks)
        for it in range(iterations):
            s.residual_step(it, qh, out=(conv, diss))
            out.append((conv.copy(), diss.copy(), s.get_deltat(), s.get_extrema(), s.get_gradients(),
                        s.get_limiters()))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["roe", "hllc", "roe_fixes", "roe_limiter_order1"])
def test_pipelined_step_is_bit_identical(gpu_available, case):
    m = box_mesh(40, jitter=0.15, seed=11, rcm=NUMBERING_PATCH_RCM)
    cfg = dict(BASE)
    if case == "hllc":
        cfg["flux_scheme"] = 1
    if case == "roe_limiter_order1":
        cfg["limiter_order"] = 1
    Q = perturbed_freestream(m, 1.4, 0.8, 1.25, noise=0.01, seed=12)
    if case == "roe_fixes":
        Q = low_pressure_spots(Q, m.nnode, 1.4)
    p = default_params(**cfg)
    serial = _steps(m, p, Q, chunks=0)
    for chunks in (3, 7):
        piped = _steps(m, p, Q, chunks=chunks)
        for a, b in zip(serial, piped):
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y)
