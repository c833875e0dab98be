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
from tests._util import CFG1, low_pressure_spots, make_case, relerr, relerr_rows

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


@pytest.mark.parametrize("flux,limiter,lorder", [(0, 1, 0), (1, 1, 1), (0, 1, 1), (1, 1, 0)])
def test_limiter_pressure_corrections_match_reference(ref_available, flux, limiter, lorder):
    """States with low-pressure spots, where the limiter's reconstructed-pressure
    correction (Limiters.cpp:273-304) and, for Roe, the sequential Roe-average
    fix (:61-110) fire: the restatement zeroes the reference's limiters and
    gives its residual."""
    cfg = dict(CFG1, flux_scheme=flux, order=1, limiter=limiter, limiter_order=lorder, venkat_k=5.0, mach=0.8,
               mach_min=0.8, alpha_deg=1.25)
    m, cfg, Q = make_case(n=8, seed=9, cfg=cfg, noise=0.02)
    Q = low_pressure_spots(Q, m.nnode, cfg["gamma"], seed=9)
    ref = refharness.run(m, cfg, Q, [("begin", 0), ("gradient", 0), ("limiter",), ("bc", 0), ("residual", 1),
                                     ("get", "residual"), ("get", "limiters")])
    s = restatement.Session(m, cfg)
    g = s.gradient(Q)
    phi = s.limiter(Q, g)
    conv, diss, _, _ = s.residual(s.apply_bc(Q), g, phi)
    assert (ref["limiters"] == 0).all(axis=0).sum() >= 3  # the corrections fired
    np.testing.assert_array_equal(phi == 0, ref["limiters"] == 0)
    assert np.abs(phi - ref["limiters"]).max() <= 1e-13
    assert relerr_rows(conv, ref["conv"]) <= TOL
    assert np.abs(diss - ref["diss"]).max() <= TOL * max(np.abs(ref["diss"]).max(), 1.0)


@pytest.mark.parametrize("method,e3d,average,ptype", [(2, "PRECOND_METHOD_ROE_BTW", 1, 1),
                                                       (3, "PRECOND_METHOD_ROE_ERIKSSON", 0, 1),
                                                       (3, "PRECOND_METHOD_ROE_ERIKSSON", 0, 0)],
                         ids=["btw-global", "eriksson-global", "eriksson-local"])
@pytest.mark.parametrize("order", [0, 1])
def test_preconditioned_roe_matches_euler3d(ref_available, method, e3d, average, ptype, order):
    """The restatement's preconditioned Roe (flux 4, written after MPFLOW3D with
    closed-form eigenvectors of K A) against Euler3D's own BTW and Eriksson
    fluxes (FluxTest.cpp:3842-4238, 4238-4628), compiled from the reference,
    with the global beta = min(1, M_ref)^2 and, for Eriksson, the local beta of
    the face and its two ends (FluxTest.cpp:4405-4412, no smoothing).  Euler3D's BTW takes the simple mean
    of the face states (FluxTest.cpp:3917-3940, precond_average 1), its
    Eriksson the Roe average.  Compared at the nodes without boundary edges:
    the reference's preconditioned boundary condition is not on this path, so
    the ghost update is not run."""
    mach = 0.1
    base = dict(CFG1, order=order, gradient=0, limiter=1 if order else -1, venkat_k=5.0, mach=mach, mach_min=mach,
                alpha_deg=1.25)
    cfg = dict(base, flux_scheme=4, precond_method=method, precond_type=ptype, precond_mach=mach,
               precond_average=average)
    m, cfg, Q = make_case(n=8, seed=41, cfg=cfg, noise=0.02)
    steps = [("begin", 0)] + ([("gradient", 0), ("limiter",)] if order else []) + \
            [("residual", 1), ("get", "residual"), ("deltat", 0), ("get", "deltat")]
    ref = refharness.run(m, dict(base, flux_scheme=0, e3d_precond=e3d,
                                 e3d_precond_type="PRECOND_TYPE_GLOBAL" if ptype == 1 else "PRECOND_TYPE_LOCAL"),
                         Q, steps)
    s = restatement.Session(m, cfg)
    g = s.gradient(Q) if order else None
    phi = s.limiter(Q, g) if order else None
    conv, diss, dts, _ = s.residual(Q, g, phi)
    dt, _ = s.deltat(dts)
    inner = np.setdiff1d(np.arange(m.nnode), m.bedge_nodes.reshape(-1, 2)[:, 0])
    assert len(inner) > 300
    assert relerr_rows(conv[:, inner], ref["conv"][:, inner]) <= TOL
    assert relerr_rows(diss[:, inner], ref["diss"][:, inner]) <= 1e-13
    assert relerr(dt[inner], ref["deltat"][inner]) <= TOL


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


@pytest.mark.parametrize("face_bc,mach", [((1, 1, 1, 1, 1, 1), 0.1), ((2, 3, 0, 0, 0, 0), 0.2)])
def test_low_mach_fix_restatement_matches_reference(ref_available, face_bc, mach):
    """Flux 3 of the restatement (Roe with the low-Mach fix and the
    preconditioned characteristic BC) against Compute_Flux_Roe_LMFIX and
    Compute_Precondition_Characteristic_BoundaryCondition of the reference,
    second order with the Venkatakrishnan limiter."""
    from cfdsolutions_b200 import box_mesh
    cfg = dict(CFG1, flux_scheme=3, order=1, limiter=1, limiter_order=1, venkat_k=5.0, mach=mach, mach_min=mach,
               alpha_deg=0.0 if face_bc[0] == 2 else 2.0)
    m = box_mesh(8, jitter=0.15, seed=41, face_bc=face_bc)
    _, cfg, Q = make_case(cfg=cfg, mesh=m, seed=41)
    ref = refharness.run(m, cfg, Q, [("begin", 0), ("gradient", 0), ("limiter",), ("bc", 0), ("get", "state"),
                                     ("residual", 1), ("get", "residual"), ("get", "limiters"), ("deltat", 0),
                                     ("get", "deltat")])
    s = restatement.Session(m, cfg)
    g = s.gradient(Q)
    phi = s.limiter(Q, g)
    Qb = s.apply_bc(Q)
    conv, diss, dts, _ = s.residual(Qb, g, phi)
    dt, _ = s.deltat(dts)
    assert np.abs(phi - ref["limiters"]).max() <= 1e-13
    assert relerr_rows(Qb, ref["state"]) <= 1e-15
    assert relerr_rows(conv, ref["conv"]) <= TOL
    assert relerr_rows(diss, ref["diss"]) <= TOL
    assert relerr(dt, ref["deltat"]) <= TOL


def _two_node_mesh(areav):
    """One interior edge 0 -> 1 with area vector ``areav``, no boundary."""
    from cfdsolutions_b200.mesh import Mesh
    z2, zb = np.zeros((0, 2), np.int32), np.zeros((0, 3))
    return Mesh(nnode=2, nghost=0, edge_nodes=np.array([[0, 1]], np.int32), edge_areav=np.array([areav], float),
                bedge_nodes=z2, bedge_areav=zb, bedge_type=np.zeros(0, np.int32), cvol=np.ones(2),
                coords=np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]]), n2n_ia=np.array([0, 1, 2], np.int32),
                n2n_ja=np.array([1, 0], np.int32))


def _stiffened_flux(q, a, gamma, pinf):
    """F(q).a of the Euler equations with p = (gamma - 1)(rho et - rho q^2 / 2) - gamma pinf."""
    rho, u = q[0], q[1:4] / q[0]
    p = (gamma - 1.0) * (q[4] - 0.5 * rho * (u @ u)) - gamma * pinf
    un = u @ a
    return np.r_[rho * un, rho * u * un + p * a, (q[4] + p) * un]


@pytest.mark.parametrize("flux", [0, 1, 2, 3])
@pytest.mark.parametrize("pinf", [0.0, 3.0, 6000.0])
def test_stiffened_gas_fluxes_upwind_when_supersonic(flux, pinf):
    """Stiffened-gas algebra of every flux family, with no reference to pin
    it: when all waves run one way the Roe flux (the Roe property A dQ = dF
    must hold for the stiffened-gas averages), HLLC and AUSM+ all reduce to
    the upwind state's exact flux F(q).a."""
    gamma = 4.4
    a = np.array([0.3, -0.2, 0.25])
    n = a / np.linalg.norm(a)
    c_ref = np.sqrt(gamma * (1.0 + pinf))

    def state(rho, p, vel):
        return np.r_[rho, rho * vel, (p + gamma * pinf) / (gamma - 1.0) + 0.5 * rho * (vel @ vel)]

    t = np.cross(n, [0.0, 0.0, 1.0])
    qa = state(1.0, 1.0, 3.0 * c_ref * n + 0.1 * c_ref * t)
    qb = state(1.1, 1.3, 2.6 * c_ref * n - 0.2 * c_ref * t)
    cfg = dict(CFG1, flux_scheme=flux, gamma=gamma, pinf=pinf)
    for sign in (1.0, -1.0):
        m = _two_node_mesh(sign * a)
        Q = np.stack([qa, qb], axis=1)
        conv, diss, _, _ = restatement.Session(m, cfg).residual(Q)
        F = conv[:, 0] + diss[:, 0]
        # with the area vector reversed both states move against it: node 1 is upwind
        up = qa if sign > 0 else qb
        exact = _stiffened_flux(up, sign * a, gamma, pinf)
        # round-off scale: the flux plus the pressure cancellation (gamma pinf) in p
        scale = np.abs(exact).max() + gamma * pinf * np.abs(a).max()
        assert np.abs(F - exact).max() <= 1e-13 * scale, (F, exact)
        np.testing.assert_allclose(conv[:, 1] + diss[:, 1], -F, rtol=0, atol=0)


@pytest.mark.parametrize("face_bc,flux", [((1, 1, 1, 1, 1, 1), 0), ((1, 1, 1, 1, 1, 1), 1), ((1, 1, 1, 1, 1, 1), 2),
                                          ((1, 1, 1, 1, 1, 1), 3), ((2, 3, 0, 0, 0, 0), 3),
                                          ((1, 1, 1, 1, 1, 1), 4), ((2, 3, 0, 0, 0, 0), 4)])
def test_stiffened_gas_freestream_preserved(face_bc, flux):
    """A uniform stiffened-gas freestream (gamma 4.4, pinf 6000, u ~ c/160)
    is a steady state: ghost states are the freestream and the residual
    vanishes to round-off of the energy flux scale.  The channel (inflow,
    outflow, slip walls) uses the low-Mach fix, whose outflow keeps the
    freestream (without it the subsonic outflow imposes 0.935 p), or the
    preconditioned Roe, whose outflow imposes the freestream pressure."""
    from cfdsolutions_b200 import box_mesh
    m = box_mesh((8, 4, 4), lengths=(2.0, 1.0, 1.0), jitter=0.1, seed=5, face_bc=face_bc)
    cfg = dict(CFG1, flux_scheme=flux, gamma=4.4, pinf=6000.0, mach=0.0062, mach_min=0.0062,
               alpha_deg=0.0 if face_bc[0] == 2 else 2.0, precond_method=5, precond_type=0, precond_mach=0.0062)
    _, cfg, Q0 = make_case(mesh=m, cfg=cfg, noise=0.0)
    s = restatement.Session(m, cfg)
    Qb = s.apply_bc(Q0)
    np.testing.assert_allclose(Qb, Q0, rtol=1e-14, atol=0)
    conv, diss, _, _ = s.residual(Qb)
    amax = np.abs(m.edge_areav).max()
    for v in range(5):
        # each equation against its own flux scale: rho u, rho u^2 + p, (rho et + p) u
        fscale = np.abs(Qb[v]).max() * np.abs(Qb[1]).max() / Qb[0].min() + (1.0 if 1 <= v <= 3 else 0.0)
        assert np.abs(conv[v] + diss[v]).max() <= 1e-12 * fscale * amax * 20


def _precond_expected(qa, qb, a, gamma, pinf, method, ptype, pmach):
    """-1/2 |a| Mop Kinv |K A| Mpr (qb - qa) with |K A| from numpy's
    eigendecomposition: the preconditioned Roe dissipation written from its
    definition, independent of the closed-form eigenvectors under test."""
    def prim(q):
        rho, u = q[0], q[1:4] / q[0]
        p = (gamma - 1.0) * (q[4] - 0.5 * rho * (u @ u)) - gamma * pinf
        return rho, u, p, (q[4] + p) / rho, np.sqrt(gamma * (p + pinf) / rho)
    rl, ul, _, hl, cl = prim(qa)
    rr, ur, _, hr, cr = prim(qb)
    rho = np.sqrt(rl * rr)
    s = rho / (rl + rho)
    u = ul + s * (ur - ul)
    ht = hl + s * (hr - hl)
    c = np.sqrt((gamma - 1.0) * (ht - 0.5 * u @ u))
    n = a / np.linalg.norm(a)
    mach, mmax = np.linalg.norm(u) / c, max(np.linalg.norm(ul) / cl, np.linalg.norm(ur) / cr)
    if ptype == 0:
        M, G = max(mach, mmax), pmach
        b = (0.5 * M * M / (G * G) - M / G + 1.0) if M < G else 0.5
        b = min(1.0, b * (np.sqrt(M * G) + M))
    elif ptype == 2:
        b = min(1.0, mach)
    else:
        b = min(1.0, pmach)
    beta = b * b
    alpha = 0.4 if method == 5 else 0.0
    delta = 1.0 if method == 2 else beta
    un = u @ n
    A = np.zeros((5, 5))
    A[0, 0] = A[1, 1] = A[2, 2] = A[3, 3] = A[4, 4] = un
    A[0, 1:4] = rho * n
    A[1:4, 4] = n / rho
    A[4, 1:4] = rho * c * c * n
    K = np.eye(5)
    K[0, 4] = (delta - 1.0) / (c * c)
    K[1:4, 4] = -alpha * u / (rho * c * c)
    K[4, 4] = beta
    lam, V = np.linalg.eig(K @ A)
    absKA = (V @ np.diag(np.abs(lam.real)) @ np.linalg.inv(V)).real
    q2 = u @ u
    g1 = gamma - 1.0
    Mpr = np.array([[1, 0, 0, 0, 0], [-u[0] / rho, 1 / rho, 0, 0, 0], [-u[1] / rho, 0, 1 / rho, 0, 0],
                    [-u[2] / rho, 0, 0, 1 / rho, 0], [0.5 * g1 * q2, -g1 * u[0], -g1 * u[1], -g1 * u[2], g1]])
    Mop = np.linalg.inv(Mpr)
    return -0.5 * np.linalg.norm(a) * (Mop @ np.linalg.inv(K) @ absKA @ Mpr @ (qb - qa)), np.abs(lam.real).max()


@pytest.mark.parametrize("method", [2, 3, 5])
@pytest.mark.parametrize("ptype", [0, 1, 2])
@pytest.mark.parametrize("pinf", [0.0, 6000.0])
def test_preconditioned_roe_dissipation_matches_its_definition(method, ptype, pinf):
    """Flux 4 (the Turkel-family preconditioned Roe of MPFLOW3D, restated;
    the compiled reference is Euler3D, which lacks it): the closed-form
    eigenvectors give Mop Kinv |K A| Mpr dQ, and the time-step eigenvalue is
    the spectral radius of K A."""
    gamma = 4.4
    a = np.array([0.3, -0.2, 0.25])
    c0 = np.sqrt(gamma * (1.0 + pinf))

    def state(rho, p, vel):
        return np.r_[rho, rho * vel, (p + gamma * pinf) / (gamma - 1.0) + 0.5 * rho * (vel @ vel)]

    qa = state(1.0, 1.0, c0 * np.array([0.05, 0.01, -0.02]))
    qb = state(1.02, 1.0 + 1e-3 * c0 * c0, c0 * np.array([0.045, 0.015, -0.01]))
    cfg = dict(CFG1, flux_scheme=4, gamma=gamma, pinf=pinf, precond_method=method, precond_type=ptype,
               precond_mach=0.1)
    conv, diss, dts, _ = restatement.Session(_two_node_mesh(a), cfg).residual(np.stack([qa, qb], axis=1))
    exp, lmax = _precond_expected(qa, qb, a, gamma, pinf, method, ptype, 0.1)
    assert np.abs(diss[:, 0] - exp).max() <= 1e-9 * np.abs(exp).max(), (diss[:, 0], exp)
    assert abs(dts[0] - np.linalg.norm(a) * lmax) <= 1e-12 * dts[0]


def test_preconditioned_roe_without_preconditioning_is_roe():
    """beta = 1 with BTW (K = I): flux 4 reduces to the Roe flux (on the same
    ghost states; the two families have their own characteristic BCs)."""
    m, cfg, Q = make_case(n=5, seed=12, noise=0.02)
    s0 = restatement.Session(m, dict(cfg, flux_scheme=0))
    s4 = restatement.Session(m, dict(cfg, flux_scheme=4, precond_method=2, precond_type=1, precond_mach=1.0))
    Qb = s0.apply_bc(Q)
    c0, d0, t0, _ = s0.residual(Qb)
    c4, d4, t4, _ = s4.residual(Qb)
    np.testing.assert_allclose(c4, c0, rtol=0, atol=1e-12 * np.abs(c0).max())
    np.testing.assert_allclose(d4, d0, rtol=0, atol=1e-12 * np.abs(d0).max())
    np.testing.assert_allclose(t4, t0, rtol=1e-13)


def test_thornber_is_roe_above_mach_one_and_blends_velocities_below():
    """Flux 5 (MPFLOW3D's Thornber modification, restated): at max(M_L, M_R)
    >= 1 it is the Roe flux; below, the Roe flux of states whose velocities are
    blended toward each other by (1 - z)/2, density and energy kept."""
    a = np.array([0.3, -0.2, 0.25])
    g = 1.4

    def state(rho, p, vel):
        return np.r_[rho, rho * vel, p / (g - 1.0) + 0.5 * rho * (vel @ vel)]

    def flux(qa, qb, f):
        conv, diss, _, _ = restatement.Session(_two_node_mesh(a), dict(CFG1, flux_scheme=f)).residual(
            np.stack([qa, qb], axis=1))
        return conv[:, 0] + diss[:, 0]

    c = np.sqrt(g)
    qa, qb = state(1.0, 1.0, c * np.array([1.2, 0.1, 0.0])), state(1.1, 1.2, c * np.array([0.9, -0.1, 0.2]))
    np.testing.assert_allclose(flux(qa, qb, 5), flux(qa, qb, 0), rtol=0, atol=1e-14)
    va, vb = c * np.array([0.1, 0.02, -0.01]), c * np.array([0.08, -0.03, 0.02])
    qa, qb = state(1.0, 1.0, va), state(1.02, 1.01, vb)
    z = max(np.linalg.norm(va) / np.sqrt(g * 1.0 / 1.0), np.linalg.norm(vb) / np.sqrt(g * 1.01 / 1.02))
    ma, mb = qa.copy(), qb.copy()
    ma[1:4] = qa[0] * 0.5 * ((1 + z) * va + (1 - z) * vb)
    mb[1:4] = qb[0] * 0.5 * ((1 + z) * vb + (1 - z) * va)
    np.testing.assert_allclose(flux(qa, qb, 5), flux(ma, mb, 0), rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("order", [0, 1])
def test_vanleer_matches_reference(ref_available, order):
    """Flux 6 (FLUX_SCHEME_VANLEER, Compute_VanLeerFlux) of the restatement
    against the compiled reference: residual and time step, first and second
    order (LSQ + Venkatakrishnan)."""
    cfg = dict(CFG1, flux_scheme=6, order=order, limiter=1 if order else -1, venkat_k=5.0, mach=0.8, mach_min=0.8,
               alpha_deg=1.25)
    m, cfg, Q = make_case(n=7, seed=21, cfg=cfg, noise=0.02)
    steps = [("begin", 0)] + ([("gradient", 0), ("limiter",)] if order else [])
    steps += [("bc", 0), ("residual", 1), ("get", "residual"), ("deltat", 0), ("get", "deltat")]
    ref = refharness.run(m, cfg, Q, steps)
    s = restatement.Session(m, cfg)
    g = phi = None
    if order:
        g = s.gradient(Q)
        phi = s.limiter(Q, g)
    Qb = s.apply_bc(Q)
    conv, diss, dts, _ = s.residual(Qb, g, phi)
    dt, _ = s.deltat(dts)
    assert relerr_rows(conv, ref["conv"]) <= TOL
    assert np.abs(diss).max() == 0.0 and np.abs(ref["diss"]).max() == 0.0
    assert relerr(dt, ref["deltat"]) <= TOL
