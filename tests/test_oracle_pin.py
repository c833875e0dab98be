"""Pins the oracle's C restatement (oracle/cfd_oracle.c) against the reference
itself: the Euler3D objects compiled from the reference sources into
oracle/_ref, run on identical mesh arrays and states.  The restatement then
serves as the checker of the CUDA path at every size it finishes in seconds.

Also pins the parts the reference lacks (Green-Gauss, AUSM+, ILU(0)-GMRES) by
properties: linear exactness, freestream preservation, conservation and
agreement with a dense direct solve.
"""
import numpy as np
import pytest

from oracle import refharness, restatement
from tests._util import CFG1, make_case, relerr, relerr_rows

TOL = 1e-13


@pytest.mark.parametrize("n,rcm", [(6, False), (20, False), (10, True)])
def test_first_order_step_matches_reference(ref_available, n, rcm):
    m, cfg, Q = make_case(n=n, seed=100 + n, rcm=rcm)
    ref = refharness.run(m, cfg, Q, [("begin", 0), ("bc", 0), ("get", "state"), ("residual", 1),
                                     ("get", "residual"), ("deltat", 0), ("get", "deltat"), ("get", "extrema"),
                                     ("jacobian", 1, 0), ("get", "crs"), ("gs", 10, 0), ("get", "matrix")])
    o = restatement.first_order_step(m, cfg, Q, gs_sweeps=10)
    assert relerr_rows(o["state"], ref["state"]) == 0.0
    assert relerr_rows(o["conv"], ref["conv"]) <= TOL
    assert relerr_rows(o["diss"], ref["diss"]) <= TOL
    assert relerr(o["deltat"], ref["deltat"]) <= TOL
    np.testing.assert_allclose(o["extrema"], ref["extrema"], rtol=1e-14)
    np.testing.assert_array_equal(o["IA"], ref["IA"])
    np.testing.assert_array_equal(o["JA"], ref["JA"])
    np.testing.assert_array_equal(o["IAU"], ref["IAU"])
    assert relerr(o["A"], ref["A"]) <= TOL
    assert relerr(o["B"], ref["B"]) <= TOL
    assert relerr(o["X"], ref["X"]) <= 1e-11
    assert abs(o["gs_rms"] - ref["gs_rms"][0]) <= 1e-11 * ref["gs_rms"][0]


@pytest.mark.parametrize("flux,limiter,lorder,smooth", [(0, -1, 0, 0), (0, 1, 1, 0), (1, 1, 1, 1), (0, 0, 1, 0),
                                                        (1, -1, 1, 0)])
def test_second_order_matches_reference(ref_available, flux, limiter, lorder, smooth):
    cfg = dict(CFG1, flux_scheme=flux, order=1, limiter=limiter, limiter_order=lorder, limiter_smooth=smooth,
               venkat_k=5.0, mach=0.8, mach_min=0.8, alpha_deg=1.25)
    m, cfg, Q = make_case(n=8, seed=7, cfg=cfg, noise=0.02)
    steps = [("begin", 0), ("gradient", 0)] + ([("limiter",)] if limiter != -1 else [])
    steps += [("bc", 0), ("residual", 1), ("get", "residual"), ("get", "gradients"), ("deltat", 0),
              ("get", "deltat")] + ([("get", "limiters")] if limiter != -1 else [])
    ref = refharness.run(m, cfg, Q, steps)
    s = restatement.Session(m, cfg)
    # the reference computes gradients and limiters before the ghost update
    g = s.gradient(Q)
    phi = s.limiter(Q, g) if limiter != -1 else None
    Qb = s.apply_bc(Q)
    conv, diss, dts, _ = s.residual(Qb, g, phi)
    dt, _ = s.deltat(dts)
    assert relerr_rows(g, ref["gradients"]) <= TOL
    if limiter != -1:
        assert np.abs(phi - ref["limiters"]).max() <= 1e-13
    assert relerr_rows(conv, ref["conv"]) <= TOL
    assert np.abs(diss - ref["diss"]).max() <= TOL * max(np.abs(ref["diss"]).max(), 1.0)
    assert relerr(dt, ref["deltat"]) <= TOL


def test_entropy_fix_and_global_time_match_reference(ref_available):
    for extra in (dict(entropy_fix=1), dict(global_time=1), dict(cfl_ramp=5, cfl_min=2.0, cfl_max=50.0)):
        cfg = dict(CFG1, **extra)
        m, cfg, Q = make_case(n=6, seed=3, cfg=cfg)
        it = 2
        ref = refharness.run(m, cfg, Q, [("begin", it), ("bc", it), ("residual", 1), ("get", "residual"),
                                         ("deltat", it), ("get", "deltat")])
        s = restatement.Session(m, cfg, iteration=it)
        Qb = s.apply_bc(Q)
        conv, diss, dts, _ = s.residual(Qb)
        dt, _ = s.deltat(dts)
        assert relerr_rows(diss, ref["diss"]) <= TOL
        assert relerr(dt, ref["deltat"]) <= TOL


def test_wall_and_outflow_ghost_states_match_reference(ref_available):
    from cfdsolutions_b200 import box_mesh
    m = box_mesh((8, 4, 4), lengths=(2.0, 1.0, 1.0), jitter=0.1, seed=9, face_bc=(2, 3, 0, 0, 0, 0))
    _, cfg, Q = make_case(mesh=m, cfg=dict(CFG1, mach=0.3, mach_min=0.3, alpha_deg=0.0))
    ref = refharness.run(m, cfg, Q, [("begin", 0), ("bc", 0), ("get", "state")])
    o = restatement.Session(m, cfg).apply_bc(Q)
    assert relerr_rows(o, ref["state"]) <= 1e-15


def test_green_gauss_exact_for_linear_fields_interior():
    m, cfg, _ = make_case(n=6, seed=2)
    x, y, z = m.coords.T
    n = m.nnode + m.nghost
    Q = np.zeros((5, n))
    coef = np.array([[1.0, 0.2, -0.3, 0.5], [0.3, 1.0, 0.7, -0.2], [0.1, -0.5, 0.4, 0.9], [2.0, 0.0, 0.0, 1.0],
                     [-1.0, 0.3, 0.3, 0.3]])
    for v in range(5):
        Q[v, :m.nnode] = coef[v, 0] + coef[v, 1] * x + coef[v, 2] * y + coef[v, 3] * z
    s = restatement.Session(m, cfg)
    g = s.gradient(Q, method=1)
    interior = np.ones(m.nnode, bool)
    interior[m.bedge_nodes[:, 0]] = False
    for v in range(5):
        for d in range(3):
            assert np.abs(g[3 * v + d, interior] - coef[v, d + 1]).max() < 1e-12
    g2 = s.gradient(Q, method=0)  # least squares: exact everywhere
    for v in range(5):
        for d in range(3):
            assert np.abs(g2[3 * v + d] - coef[v, d + 1]).max() < 1e-11


@pytest.mark.parametrize("flux", [0, 1, 2])
def test_freestream_preservation_and_conservation(flux):
    cfg = dict(CFG1, flux_scheme=flux)
    m, cfg, Q0 = make_case(n=5, seed=4, noise=0.0)
    s = restatement.Session(m, cfg)
    Qb = s.apply_bc(Q0)
    conv, diss, _, _ = s.residual(Qb)
    scale = np.abs(Qb).max() * np.abs(m.edge_areav).max()
    assert np.abs(conv + diss).max() < 1e-13 * scale * 20
    # conservation: interior fluxes cancel, sum of residuals = sum of boundary fluxes
    _, _, Q = make_case(mesh=m, cfg=cfg, noise=0.05)
    Qb = s.apply_bc(Q)
    conv, diss, _, _ = s.residual(Qb)
    mb = restatement.Session(m, cfg)
    m2 = type(m)(**{**m.__dict__, "edge_nodes": m.edge_nodes[:0], "edge_areav": m.edge_areav[:0]})
    sb = restatement.Session(m2, cfg)
    cb, db, _, _ = sb.residual(Qb)
    assert np.abs((conv + diss).sum(1) - (cb + db).sum(1)).max() < 1e-12 * np.abs(cb).sum()
    del mb


def test_ilu_gmres_agrees_with_dense_solve():
    m, cfg, Q = make_case(n=4, seed=8)
    o = restatement.first_order_step(m, cfg, Q, gs_sweeps=1)
    s = restatement.Session(m, cfg)
    n = m.nnode
    dense = np.zeros((5 * n, 5 * n))
    for i in range(n):
        for k in range(s.IA[i], s.IA[i + 1]):
            j = s.JA[k]
            dense[5 * i:5 * i + 5, 5 * j:5 * j + 5] = o["A"][k]
    x_ref = np.linalg.solve(dense, o["B"].ravel()).reshape(n, 5)
    for pc in (0, 1, 2):
        X, rc, its, rr = s.gmres(o["A"], o["B"], m=30, maxit=500, rtol=1e-10, precond=pc)
        assert rc == 0 and rr <= 1e-10
        assert relerr(X, x_ref) <= 1e-8
    # ILU(0) preconditioning needs fewer iterations than none
    it_none = s.gmres(o["A"], o["B"], rtol=1e-8, precond=0)[2]
    it_ilu = s.gmres(o["A"], o["B"], rtol=1e-8, precond=2)[2]
    assert it_ilu < it_none


def test_block_lusgs_restatement_is_the_reference(ref_available):
    """LU-SGS (MC_Iterative_Block_LUSGS_CRS): the restatement's sweeps,
    pivoted diagonal solves and returned RMS equal the reference's bit for bit."""
    m, cfg, Q = make_case(n=7, seed=9)
    ref0 = refharness.run(m, cfg, Q, [("begin", 0), ("bc", 0), ("residual", 1), ("deltat", 0), ("jacobian", 1, 0),
                                      ("get", "matrix")])
    A, B = ref0["A"], ref0["B"]
    ref = refharness.run(m, cfg, Q, [("set_matrix", A, B), ("lusgs", 4), ("get", "matrix")])
    X, rms = restatement.Session(m, cfg).block_lusgs(A, B, 4)
    np.testing.assert_array_equal(X, ref["X"])
    assert rms == ref["lusgs_rms"][0]
