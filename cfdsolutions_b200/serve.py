"""Serving loop binding: steady-solve requests run concurrently on one GPU.

Wraps ``cfd_server_*`` (``include/cfd_b200.h``): a native server with a FIFO
of requests, admission against a device-memory budget, and one host thread
and CUDA stream per worker.  Each request is a tet-split box mesh, flow
conditions, a seeded initial perturbation and implicit steady-solve options.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi as capi
from .solver import default_params


def steady_opts(max_iterations=800, drop=1e-8, include_diss=1, linear_solver=1, linear_iters=10, relax=1.0,
                restart=30, gmres_iters=30, rtol=0.1, precond=capi.PC_ILU0_MC,
                precision=capi.PREC_FP32 | capi.PREC_LOW_ONLY, precond_update=1) -> capi.SolveOpts:
    g = capi.GmresOpts(restart, gmres_iters, rtol, precond, precision, 1, 0)
    return capi.SolveOpts(max_iterations, drop, include_diss, linear_solver, linear_iters, relax, g, precond_update)


def request(n, params: capi.Params, opts: capi.SolveOpts, lengths=(1.0, 1.0, 1.0), jitter=0.15, mesh_seed=1,
            numbering=2, face_bc=(1, 1, 1, 1, 1, 1), noise=0.01, state_seed=2, keep_state=False) -> capi.ServeRequest:
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    r = capi.ServeRequest()
    r.nx, r.ny, r.nz = nx, ny, nz
    r.lx, r.ly, r.lz = (float(x) for x in lengths)
    r.jitter, r.mesh_seed, r.numbering = float(jitter), int(mesh_seed), int(numbering)
    for k in range(6):
        r.face_bc[k] = int(face_bc[k])
    r.noise, r.state_seed = float(noise), int(state_seed)
    r.params, r.opts, r.keep_state = params, opts, int(keep_state)
    return r


def initial_state(req: capi.ServeRequest) -> np.ndarray:
    """The initial state the server gives ``req`` (cfd_initial_state on the
    same mesh), for running the same solve through the plain API."""
    fb = np.array(list(req.face_bc), np.int32)
    h = C.c_void_p()
    capi.check(capi.lib.cfd_mesh_box(req.nx, req.ny, req.nz, req.lx, req.ly, req.lz, req.jitter, req.mesh_seed,
                                     req.numbering, capi.ptr(fb), C.byref(h)), "cfd_mesh_box")
    try:
        sizes = np.zeros(7, np.int64)
        capi.check(capi.lib.cfd_mesh_sizes(h, capi.ptr(sizes)), "cfd_mesh_sizes")
        Q = np.empty((5, int(sizes[0] + sizes[1])))
        noise = np.full(3, req.noise)
        capi.check(capi.lib.cfd_initial_state(h, C.byref(req.params), capi.ptr(noise), req.state_seed, capi.ptr(Q)),
                   "cfd_initial_state")
        return Q
    finally:
        capi.lib.cfd_mesh_free(h)


@dataclass
class Result:
    status: int
    iterations: int
    linear_iterations: int
    rms_first: float
    rms_last: float
    nnode: int
    nghost: int
    t_submit: float
    t_admit: float
    t_start_solve: float
    t_done: float
    bytes_estimate: float
    message: str = ""

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    def __init__(self, device: int = 0, workers: int = 8, budget_bytes: float = 150e9, batching: bool = True,
                 window_us: float = 50.0):
        self._h = C.c_void_p()
        capi.check(capi.lib.cfd_server_create(int(device), int(workers), float(budget_bytes), C.byref(self._h)),
                   "cfd_server_create")
        capi.check(capi.lib.cfd_server_set_batching(self._h, int(bool(batching)), float(window_us)),
                   "cfd_server_set_batching")

    def batch_stats(self) -> dict:
        """Fused launches so far and the jobs they carried, per kernel kind."""
        o = np.zeros(4)
        capi.check(capi.lib.cfd_server_batch_stats(self._h, capi.ptr(o)), "cfd_server_batch_stats")
        return {"residual": {"launches": int(o[0]), "jobs": int(o[1])},
                "spmv": {"launches": int(o[2]), "jobs": int(o[3])}}

    def submit(self, req: capi.ServeRequest) -> int:
        i = C.c_int64()
        capi.check(capi.lib.cfd_server_submit(self._h, C.byref(req), C.byref(i)), "cfd_server_submit")
        return i.value

    def wait(self, rid: int, timeout: float = -1.0) -> Result | None:
        r = capi.ServeResult()
        code = capi.lib.cfd_server_wait(self._h, int(rid), float(timeout), C.byref(r))
        if code == capi.PENDING:
            return None
        capi.check(code, "cfd_server_wait")
        return Result(r.status, r.stats.iterations, r.stats.linear_iterations, r.stats.rms_first, r.stats.rms_last,
                      r.nnode, r.nghost, r.t_submit, r.t_admit, r.t_start_solve, r.t_done, r.bytes_estimate,
                      r.message.decode(errors="replace"))

    def state(self, rid: int, res: Result) -> np.ndarray:
        Q = np.empty((5, res.nnode + res.nghost))
        capi.check(capi.lib.cfd_server_state(self._h, int(rid), capi.ptr(Q)), "cfd_server_state")
        return Q

    def release(self, rid: int):
        capi.check(capi.lib.cfd_server_release(self._h, int(rid)), "cfd_server_release")

    def stats(self) -> dict:
        o = np.zeros(5)
        capi.check(capi.lib.cfd_server_stats(self._h, capi.ptr(o)), "cfd_server_stats")
        return {"active": int(o[0]), "queued": int(o[1]), "reserved_bytes": o[2], "peak_reserved_bytes": o[3],
                "clock_s": o[4]}

    def close(self):
        if self._h:
            capi.lib.cfd_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ autotuner
SIZE_BUCKETS = ((16, 32), (32, 64), (64, 1 << 30))  # cube sides [lo, hi)


def size_bucket(n: int) -> int:
    for k, (lo, hi) in enumerate(SIZE_BUCKETS):
        if lo <= n < hi:
            return k
    return 0 if n < SIZE_BUCKETS[0][0] else len(SIZE_BUCKETS) - 1


def autotune(make_request, sample, device: int = 0, budget_bytes: float = 150e9,
             server_candidates=((16, True, 0.0), (16, True, 50.0), (16, True, 500.0), (16, False, 0.0),
                                (12, True, 50.0)),
             refresh_candidates=(5, 10, 20)) -> dict:
    """Measured choice of the serving schedule for a request mix.

    ``make_request(k, precond_update)`` builds request k of the mix with the
    given preconditioner refresh period; ``sample`` lists the request indices
    to calibrate on.  Two searches, each timed on the GPU:

    * per cube-size bucket (``SIZE_BUCKETS``), the implicit solve's ILU(0)
      refresh period (``precond_update``): the bucket's median request of the
      sample is solved alone under each candidate and the fastest wins;
    * for the server, the worker count and the fusion of the requests'
      residual and SpMV launches (on/off and the batcher's window): the
      whole sample, submitted at once with the chosen refresh periods, runs
      under each candidate and the highest solves per second wins.

    Returns {"precond_update": {bucket: period}, "server": (workers,
    batching, window_us), "timings": ...}.  The results of every request are
    the same under every schedule up to the refresh period, which changes the
    preconditioner and so the iterates (not the converged state)."""
    import time

    timings = {"refresh": {}, "server": {}}
    by_bucket = {}
    for k in sample:
        by_bucket.setdefault(size_bucket(int(make_request(k, 1).nx)), []).append(k)
    refresh = {}
    with Server(device=device, workers=1, budget_bytes=budget_bytes) as srv:
        for b, ks in sorted(by_bucket.items()):
            ks = sorted(ks, key=lambda k: make_request(k, 1).nx)
            k = ks[len(ks) // 2]
            best = None
            for pu in refresh_candidates:
                t0 = time.perf_counter()
                r = srv.wait(srv.submit(make_request(k, pu)))
                dt = time.perf_counter() - t0
                timings["refresh"][f"bucket{b}_n{make_request(k, 1).nx}_pu{pu}"] = dt
                if r.status == 0 and (best is None or dt < best[0]):
                    best = (dt, pu)
            refresh[b] = best[1] if best else refresh_candidates[0]
    pick = lambda k: refresh.get(size_bucket(int(make_request(k, 1).nx)), refresh_candidates[0])  # noqa: E731
    best = None
    for workers, batching, window in server_candidates:
        with Server(device=device, workers=workers, budget_bytes=budget_bytes, batching=batching,
                    window_us=window) as srv:
            t0 = time.perf_counter()
            ids = [srv.submit(make_request(k, pick(k))) for k in sample]
            res = [srv.wait(i) for i in ids]
            dt = time.perf_counter() - t0
        rate = len(sample) / dt
        timings["server"][f"w{workers}_{'fused' if batching else 'unfused'}_{window:g}us"] = rate
        if all(r.status == 0 for r in res) and (best is None or rate > best[0]):
            best = (rate, (workers, batching, window))
    return {"precond_update": refresh, "server": best[1] if best else server_candidates[0], "timings": timings}


__all__ = ["Server", "Result", "request", "steady_opts", "initial_state", "default_params", "autotune",
           "size_bucket", "SIZE_BUCKETS"]
