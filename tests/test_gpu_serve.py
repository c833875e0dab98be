"""Serving loop (cfd_server_*): steady-solve requests admitted against a
device-memory budget and run concurrently, one host thread and CUDA stream per
worker.  Every kernel of the solve is deterministic, so a request's converged
state must be the same when it runs alone and when it runs beside others, and
the same as the plain API's solve of the same inputs."""
import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, capi, default_params
from cfdsolutions_b200.mesh import box_mesh
from cfdsolutions_b200.serve import Server, initial_state, request, steady_opts

pytestmark = pytest.mark.gpu

BASE = dict(flux_scheme=0, order=1, limiter=1, gradient=1, venkat_k=5.0, gamma=1.4, cfl_min=10.0, cfl_max=1000.0,
            cfl_ramp=10)
CASES = [(6, 0.5, 2.0), (8, 0.8, -3.0), (5, 0.3, 7.0), (9, 0.65, 0.0), (7, 0.85, 10.0), (6, 0.4, -5.0)]


def _requests(precision=capi.PREC_FP32 | capi.PREC_LOW_ONLY):
    out = []
    for k, (n, mach, alpha) in enumerate(CASES):
        p = default_params(**dict(BASE, mach=mach, mach_min=mach, alpha_deg=alpha))
        out.append(request(n, p, steady_opts(max_iterations=400, drop=1e-10, rtol=0.1, precision=precision),
                           mesh_seed=100 + k, state_seed=200 + k, keep_state=True))
    return out


def _run(reqs, workers, budget=20e9, batching=True, window_us=50.0):
    with Server(device=0, workers=workers, budget_bytes=budget, batching=batching, window_us=window_us) as srv:
        ids = [srv.submit(r) for r in reqs]
        res = [srv.wait(i) for i in ids]
        for r in res:
            assert r.status == 0, (r.status, r.message)
        states = [srv.state(i, r) for i, r in zip(ids, res)]
        stats = srv.stats()
        stats.update(srv.batch_stats())
    return res, states, stats


def test_served_result_is_the_same_alone_and_in_the_mix(gpu_available):
    reqs = _requests()
    mixed, s_mixed, _ = _run(reqs, workers=4)
    alone = []
    for r in reqs:
        res, st, _ = _run([r], workers=1)
        alone.append((res[0], st[0]))
    for m, sm, (a, sa) in zip(mixed, s_mixed, alone):
        assert m.status == 0 and a.status == 0
        assert m.rms_last <= 1e-10 * m.rms_first
        assert m.iterations == a.iterations and m.linear_iterations == a.linear_iterations
        np.testing.assert_array_equal(sm, sa)


def test_served_result_matches_the_plain_api(gpu_available):
    """The server's solve is the library's cfd_solve_steady on the same mesh
    and initial state (cfd_perturbed_freestream)."""
    req = _requests()[1]
    res, states, _ = _run([req], workers=2)
    m = box_mesh(req.nx, jitter=req.jitter, seed=req.mesh_seed, rcm=req.numbering)
    Q0 = initial_state(req)
    with Euler3DGPU(m, req.params) as s:
        s.set_state(Q0)
        st = s.solve_steady(max_iterations=req.opts.max_iterations, drop=req.opts.drop, include_diss=1,
                            linear_solver=1, gmres=req.opts.gmres)
        Q = s.get_state()
    assert st.iterations == res[0].iterations
    assert np.abs(Q - states[0]).max() <= 1e-12 * np.abs(Q).max()


def test_admission_keeps_reserved_memory_within_the_budget(gpu_available):
    reqs = _requests()[:3]
    first, _, _ = _run(reqs, workers=3)
    budget = 1.5 * max(r.bytes_estimate for r in first)  # room for one request at a time
    res, _, stats = _run(reqs, workers=3, budget=budget)
    assert all(r.status == 0 for r in res)
    assert stats["peak_reserved_bytes"] <= budget
    order = sorted(res, key=lambda r: r.t_admit)
    for a, b in zip(order, order[1:]):
        assert b.t_admit >= a.t_done - 1e-6  # admitted only after the previous one released its memory
    with Server(device=0, workers=1, budget_bytes=budget) as srv:
        big = request(48, reqs[0].params, reqs[0].opts)
        with pytest.raises(capi.CfdError) as e:
            srv.submit(big)
        assert e.value.code == -9  # CFD_ERR_RANGE


def test_fused_launches_change_nothing(gpu_available):
    """With the requests' interior residuals and GMRES SpMVs fused into
    launches over a request table (a wide window, so that several requests
    share launches) every request takes the same implicit and GMRES
    iterations as in the unfused server and ends in the same state to
    round-off: 1e-13 absolute on fields of size 1 (the fused and the
    request's own kernel run the same per-node code, but the compiler may
    contract a multiply-add differently in each)."""
    reqs = _requests()
    fused, s_fused, st = _run(reqs, workers=6, window_us=500.0)
    plain, s_plain, st0 = _run(reqs, workers=6, batching=False)
    for kind in ("residual", "spmv"):
        assert st[kind]["jobs"] > st[kind]["launches"] > 0  # some launches carried several requests
        assert st0[kind]["jobs"] == 0
    for a, b, sa, sb in zip(fused, plain, s_fused, s_plain):
        assert a.iterations == b.iterations and a.linear_iterations == b.linear_iterations
        np.testing.assert_allclose(sa, sb, rtol=0, atol=1e-13)


def test_autotuner_picks_a_measured_schedule(gpu_available):
    """autotune() times each refresh period on the sample's median request of
    each size bucket and each server schedule on the whole sample, and returns
    the fastest of the candidates it timed; every timed request converges."""
    from cfdsolutions_b200.serve import autotune, size_bucket

    sides = [6, 7, 9, 8]
    p = default_params(**dict(BASE, mach=0.6, mach_min=0.6))

    def make(k, pu):
        return request(sides[k], p, steady_opts(max_iterations=400, drop=1e-8, rtol=0.1, precond_update=pu),
                       mesh_seed=300 + k, state_seed=400 + k)

    cands = ((2, True, 0.0), (2, False, 0.0))
    tune = autotune(make, range(len(sides)), server_candidates=cands, refresh_candidates=(1, 4))
    assert tune["server"] in cands
    assert set(tune["precond_update"]) == {size_bucket(n) for n in sides}
    assert all(v in (1, 4) for v in tune["precond_update"].values())
    assert len(tune["timings"]["server"]) == len(cands)
    assert all(rate > 0 for rate in tune["timings"]["server"].values())


def test_fused_launches_keep_precisions_apart(gpu_available):
    """Requests with FP32 and BF16 Jacobians in one server: their SpMVs are
    fused only with jobs of the same storage type (one kernel instantiation per
    launch), and every request takes the unfused server's iterations and ends
    in its state to round-off (1e-13 absolute, as above)."""
    reqs = _requests()[:3] + _requests(capi.PREC_BF16 | capi.PREC_LOW_ONLY)[3:]
    fused, s_fused, st = _run(reqs, workers=6, window_us=500.0)
    plain, s_plain, _ = _run(reqs, workers=6, batching=False)
    assert st["spmv"]["jobs"] > st["spmv"]["launches"] > 0
    for a, b, sa, sb in zip(fused, plain, s_fused, s_plain):
        assert a.iterations == b.iterations and a.linear_iterations == b.linear_iterations
        np.testing.assert_allclose(sa, sb, rtol=0, atol=1e-13)
