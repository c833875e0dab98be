"""Benchmark of the hot path: second-order residual evaluation on the
128^3-hex tet cube (2.15 M nodes, 14.8 M edges), RCM order, Green-Gauss
gradients, Venkatakrishnan limiter (K = 5), Roe flux, M = 0.8, alpha = 1.25,
gamma = 1.4, +-1 % seeded noise.  One step = one residual evaluation of the
hot path: far-field reset, characteristic ghost update, gradients, limiter,
flux residual, local time step.  HLLC and AUSM+ steps are timed beside it.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

value  = whole-job GEdges/s = (interior + boundary edges) x steps x ranks / max-over-ranks time,
         state resident in HBM, CUDA events on the library's stream.
e2e    = the same through the C ABI call cfd_residual_step with pinned host
         buffers: state H2D and residuals D2H inside the timed region.
--impl reference: the reference's own CPU code (Euler3D objects compiled from
         its sources) on a bounded sample of the workload, one single-threaded
         process per host core (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "residual GEdges/s (%HBM peak)"
UNIT = "GEdges/s"
CFG = dict(flux_scheme=0, order=1, limiter=1, limiter_order=0, gradient=1, venkat_k=5.0, gamma=1.4, mach=0.8,
           mach_min=0.8, alpha_deg=1.25, cfl_min=10.0, cfl_max=10.0)
FLUX_NAMES = {0: "roe", 1: "hllc", 2: "ausm+"}
# begin, bc, Green-Gauss + limiter, residual (interior + boundary edges), limiter-fix apply, gated Roe-fix
# pass, gated residual (interior + boundary), dt
KERNELS_PER_STEP = 10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128, help="hexes per side of the cube")
    ap.add_argument("--cpu-sample-n", type=int, default=48, help="hexes per side of the CPU baseline sample")
    ap.add_argument("--cpu-procs", type=int, default=0, help="reference processes (0 = one per core, max 16)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--side-rcm", action="store_true", help="also time the plain node-level RCM numbering")
    ap.add_argument("--no-steady", action="store_true", help="skip the time-to-steady-state solves")
    ap.add_argument("--no-serve", action="store_true", help="skip the served batch")
    ap.add_argument("--no-lowmach", action="store_true", help="skip the low-Mach liquid channel solves")
    ap.add_argument("--no-linear", action="store_true", help="skip the linear-algebra kernel rooflines")
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-nmax", type=int, default=96, help="largest cube side of the served mix")
    ap.add_argument("--serve-rate", type=float, default=4.0,
                    help="Poisson arrival rate of the whole mix, requests per second (the latency run takes every "
                         "other request, so it sees half the rate)")
    ap.add_argument("--serve-calibration", type=int, default=24, help="requests the autotuner calibrates on")
    ap.add_argument("--serve-sequential", type=int, default=24,
                    help="requests of the mix solved one at a time for the sequential FP64 baseline")
    ap.add_argument("--profile-linear", action="store_true",
                    help="small linear-solve case for ncu captures (Jacobian + one GMRES(30) call per precision)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling case for ncu: two residual steps per kernel variant, no timing, no output line")
    ap.add_argument("--profile-steady", type=int, default=0, metavar="ITERS",
                    help="run the first ITERS implicit iterations of the steady solve on an --n cube (launch lists)")
    ap.add_argument("--profile-lowmach", type=int, default=0, metavar="ITERS",
                    help="ncu case: ITERS implicit iterations of the low-Mach channel (FP32 Jacobian), no output line")
    return ap.parse_args()


def algorithmic_bytes(nnode, nedge, nghost):
    """Compulsory traffic of one second-order residual launch: edge nodes +
    area (32 B/edge), node Q read + residual write + spectral radius (88 B/node),
    boundary edge + ghost state (72 B/ghost), plus gradients, limiter and
    coordinates read per node (184 B/node)."""
    return 32 * nedge + 88 * nnode + 72 * nghost + 184 * nnode


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_figure(key):
    """A `key: value` figure of the committed ncu summary of the residual kernel
    (None if not captured)."""
    p = ROOT / "profiles" / "residual_roe2_128.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith(key + ":"):
            return float(line.split(":")[1])
    return None


def traffic_from_profile():
    """DRAM bytes per residual launch from the committed ncu summary, scaled
    per edge (None if not captured)."""
    p = ROOT / "profiles" / "residual_roe2_128.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_edge:"):
            return float(line.split(":")[1])
    return None


class Clocks:
    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = Path(tempfile.gettempdir()) / f"cfd_b200_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "reasons": reasons}


def reference_throughput(sample_n, procs, warmup, steps):
    """Reference CPU residual passes (LSQ gradient + Venkatakrishnan + Roe
    residual + dt, its own second-order path) on a sample_n^3 cube, one
    single-threaded reference process per core; returns (GEdges/s, details)."""
    # the sample mesh comes from the oracle's numpy builder, so this leg maps
    # no library of this repository: only the reference's own objects run
    from oracle import boxmesh, refharness

    m = boxmesh.box_mesh(sample_n, jitter=0.15, seed=1234, rcm=True)
    Q = boxmesh.perturbed_freestream(m, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
    cfg = dict(CFG, gradient=0, scheme="explicit")
    one = [("begin", 0), ("gradient", 0), ("limiter",), ("bc", 0), ("residual", 1), ("deltat", 0)]
    steps_all = one * (warmup + steps)
    outs = refharness.run_many(m, cfg, Q, steps_all, procs)
    units = m.nedge + m.nbedge
    rates, per_pass = [], []
    for o in outs:
        t = o["timings"]
        tot = [sum(x) for x in zip(*(t[k] for k in ("begin", "gradient", "limiter", "bc", "residual", "deltat")))]
        timed = tot[warmup:]
        per_pass.append(statistics.mean(timed))
        rates.append(units / statistics.mean(timed) / 1e9)
    sample = (f"{sample_n}^3-hex tet cube ({m.nnode} nodes, {units} edges), {warmup}+{steps} passes of "
              f"LSQ gradient + Venkatakrishnan + Roe residual + dt per process, {procs} concurrent "
              f"single-threaded reference processes")
    return sum(rates), dict(per_pass_s=statistics.mean(per_pass), procs=procs, sample=sample,
                            per_process_gedges=statistics.mean(rates))


STEADY = dict(CFG, cfl_min=10.0, cfl_max=1000.0, cfl_ramp=20)
STEADY_DROP = 1e-8
STEADY_RTOL = 0.1  # inner GMRES tolerance of each implicit iteration
# factor the ILU(0) preconditioner every 15 implicit iterations: at 128^3 (FP64 / FP32 seconds to
# the 1e-8 drop) 5: 10.65 / 8.41, 10: 10.04 / 7.96, 15: 9.85 / 7.84, 20: 9.79 / 7.81, 30: 10.14 / 8.14,
# 50: 11.91 / 8.87, always 286 implicit iterations (GMRES iterations 1423 at 5, 1445 at 15)
STEADY_PC_UPDATE = 15
LOWMACH_PC_UPDATE = 5  # the preconditioned low-Mach channel: ~17 GMRES iterations per implicit one


def steady_config(n):
    return {"workload": f"implicit steady solve to a {STEADY_DROP:g} L2 residual drop, {n}^3-hex tet cube, "
                        "second-order Roe residual (Green-Gauss + Venkatakrishnan K=5), approximate first-order Roe "
                        "Jacobian, CFL 10->1000 over 20 iterations, B = -(Res + Res_Diss)",
            "linear": f"GMRES(30), inner rtol {STEADY_RTOL}, ILU(0) in block multicolour order (32-row patches), "
                      f"refactored every {STEADY_PC_UPDATE} implicit iterations (Jacobian every iteration)",
            "mixed": "fp32/bf16: Jacobian and ILU(0) stored in FP32 (BF16 Jacobian), FP64 residual, Arnoldi with "
                     "compensated FP64 dots, FP64 nonlinear update; no FP64 copy of the Jacobian"}


def steady_solves(mesh, Q, dev, stream, timed_once):
    """Time to the steady residual drop, plain FP64 and mixed precision, on the
    bench mesh; the converged mixed-precision states are compared with FP64."""
    from cfdsolutions_b200 import Euler3DGPU, capi, default_params

    out, states = {}, {}
    for name, prec in (("fp64", capi.PREC_FP64), ("fp32", capi.PREC_FP32 | capi.PREC_LOW_ONLY),
                       ("bf16", capi.PREC_BF16 | capi.PREC_LOW_ONLY)):
        t0 = time.perf_counter()
        with Euler3DGPU(mesh, default_params(**STEADY), device=dev, stream=stream.cuda_stream) as ss:
            ss.set_state(Q)
            ss.synchronize()
            t1 = time.perf_counter()
            capi.check(capi.lib.cfd_ilu_mc_order(ss.handle, None, None), "cfd_ilu_mc_order")  # mesh setup
            ss.synchronize()
            if name == "fp64":  # host set-up before the first solve (context, device layouts, ILU ordering)
                out["setup_s"] = {"context_and_layouts": t1 - t0, "ilu_ordering": time.perf_counter() - t1}
            g = capi.GmresOpts(30, 30, STEADY_RTOL, capi.PC_ILU0_MC, prec, 1)
            box = {}

            def run():
                box["st"] = ss.solve_steady(max_iterations=800, drop=STEADY_DROP, include_diss=1, linear_solver=1,
                                            gmres=g, precond_update=STEADY_PC_UPDATE)

            ms = timed_once(run)
            st = box["st"]
            out[name] = {"seconds": ms / 1e3, "newton_iterations": st.iterations,
                         "gmres_iterations": st.linear_iterations, "rms_drop": st.rms_last / st.rms_first,
                         "converged": bool(st.rms_last <= STEADY_DROP * st.rms_first)}
            # untimed: continue at the final CFL to a 1e-11 drop, so the
            # precisions are compared at convergence, not at the stopping point
            ss.set_params(default_params(**dict(STEADY, cfl_min=STEADY["cfl_max"], cfl_ramp=0)))
            st2 = ss.solve_steady(max_iterations=400, drop=1e-11 * st.rms_first / max(st.rms_last, 1e-300),
                                  include_diss=1, linear_solver=1, gmres=g, precond_update=STEADY_PC_UPDATE)
            out[name]["rms_drop_compared"] = st2.rms_last / st.rms_first
            states[name] = ss.get_state()[:, :mesh.nnode]
    ref = states["fp64"]
    mom = float(np.abs(ref[1:4]).max())
    for name in ("fp32", "bf16"):
        err = 0.0
        for v in range(5):
            scale = max(float(np.abs(ref[v]).max()), mom if 1 <= v <= 3 else 0.0)
            err = max(err, float(np.abs(states[name][v] - ref[v]).max()) / scale)
        out[name]["max_rel_err_vs_fp64"] = err  # converged fields (1e-11 drop), per-field scale
        out[name]["speedup_vs_fp64"] = out["fp64"]["seconds"] / out[name]["seconds"]
    return out


def reference_converged_errors(dev, stream, n=12, iterations=120):
    """Converged fields against the reference's own converged solve, on an
    n^3 sample of the steady workload with the reference's least-squares
    gradient: the reference's implicit loop (compiled Euler3D: BCs, LSQ +
    Venkatakrishnan, Roe residual, dt with the CFL ramp, approximate Jacobian,
    10 block Gauss-Seidel sweeps, update) with B = -(Res + Res_Diss), run to
    its round-off floor on the host; the GPU's FP64 / FP32 / BF16 steady
    solves of the same problem to a 1e-11 drop.  Returns the per-field
    relative error of each GPU state (max over rho, momentum, energy of
    max |diff| / max |reference field|)."""
    from cfdsolutions_b200 import Euler3DGPU, box_mesh, capi, default_params, perturbed_freestream
    from oracle import refharness

    cfg = dict(STEADY, gradient=0)
    m = box_mesh(n, jitter=0.15, seed=1234, rcm=True)
    Q = perturbed_freestream(m, cfg["gamma"], cfg["mach"], cfg["alpha_deg"], noise=0.01, seed=1235)
    steps = []
    for it in range(iterations):
        steps += [("begin", it), ("gradient", 0), ("limiter",), ("bc", it), ("residual", 1), ("deltat", it),
                  ("jacobian", 1, it), ("rhs_full",), ("gs", 10, 0), ("update", 1.0)]
    steps.append(("get", "state"))
    ref = refharness.run(m, cfg, Q, steps)
    Qr = ref["state"][:, :m.nnode]
    mom = float(np.abs(Qr[1:4]).max())
    out = {"sample": f"{n}^3-hex tet cube ({m.nnode} nodes), LSQ gradient; reference: {iterations} implicit "
                     f"iterations of compiled Euler3D with B = -(Res + Res_Diss), residual drop "
                     f"{ref['rms_full'][-1] / ref['rms_full'][0]:.2e}; GPU: GMRES(30) + multicolour ILU(0) "
                     f"to a 1e-11 drop"}
    for name, prec in (("fp64", capi.PREC_FP64), ("fp32", capi.PREC_FP32 | capi.PREC_LOW_ONLY),
                       ("bf16", capi.PREC_BF16 | capi.PREC_LOW_ONLY)):
        with Euler3DGPU(m, default_params(**cfg), device=dev, stream=stream.cuda_stream) as ss:
            ss.set_state(Q)
            capi.check(capi.lib.cfd_ilu_mc_order(ss.handle, None, None), "cfd_ilu_mc_order")
            g = capi.GmresOpts(30, 60, 1e-3, capi.PC_ILU0_MC, prec, 1)
            ss.solve_steady(max_iterations=200, drop=1e-11, include_diss=1, linear_solver=1, gmres=g)
            Qg = ss.get_state()[:, :m.nnode]
        errs = [float(np.abs(Qg[0] - Qr[0]).max() / np.abs(Qr[0]).max()),
                float(np.abs(Qg[1:4] - Qr[1:4]).max() / mom),
                float(np.abs(Qg[4] - Qr[4]).max() / np.abs(Qr[4]).max())]
        out[name] = max(errs)
    return out


# The low-Mach liquid channel: stiffened-gas water (gamma 4.4, pinf 6e8 Pa over
# a 1 bar reference pressure, rho 1000 kg/m^3), u = 10 m/s (c = 1625 m/s,
# M = 0.0062) with +-2 % seeded velocity noise, inflow / outflow / slip walls,
# Turkel-preconditioned Roe (local beta, reference Mach = freestream Mach).
LOWMACH_MESH = (192, 48, 48)
LOWMACH = dict(flux_scheme=4, precond_method=5, precond_type=0, precond_mach=0.0062, order=1, gradient=0,
               limiter=1, venkat_k=5.0, gamma=4.4, pinf=6000.0, mach=0.0062, mach_min=0.0062, alpha_deg=0.0,
               cfl_min=10.0, cfl_max=1e4, cfl_ramp=20)


def lowmach_case(size):
    from cfdsolutions_b200 import box_mesh, perturbed_freestream
    from cfdsolutions_b200.mesh import NUMBERING_PATCH_RCM
    m = box_mesh(size, lengths=(4.0, 1.0, 1.0), jitter=0.1, seed=4242, rcm=NUMBERING_PATCH_RCM,
                 face_bc=(2, 3, 0, 0, 0, 0))
    Q = perturbed_freestream(m, LOWMACH["gamma"], LOWMACH["mach"], 0.0, noise=(0.0, 0.02, 0.0), seed=4243,
                             pinf=LOWMACH["pinf"])
    return m, Q


def lowmach_config(m):
    nx, ny, nz = LOWMACH_MESH
    return {"workload": f"implicit steady solve to a {STEADY_DROP:g} L2 residual drop, 4x1x1 channel of {nx}x{ny}x{nz} "
                        f"hexes split into tets ({m.nnode} nodes), jitter 0.1h, inflow / outflow / slip walls",
            "physics": "stiffened-gas water: gamma 4.4, pinf 6e8 Pa (6000 over the 1 bar reference pressure), "
                       "rho 1000 kg/m^3, u 10 m/s (c 1625 m/s, M 0.0062), +-2 % seeded velocity noise; "
                       "Turkel-preconditioned Roe (MPFLOW3D PRECOND_METHOD_TURKEL, PRECOND_TYPE_LOCAL, reference "
                       "Mach 0.0062), second order (LSQ gradient + Venkatakrishnan K=5), preconditioned "
                       "characteristic BCs, CFL 10->1e4 over 20 iterations",
            "linear": f"GMRES(30), inner rtol {STEADY_RTOL}, block-multicolour ILU(0) refactored every "
                      f"{LOWMACH_PC_UPDATE} iterations",
            "mixed": "fp32: Jacobian and ILU(0) stored in FP32 only, FP64 residual and Arnoldi"}


def lowmach_solves(dev, stream, timed_once):
    """Config of the low-Mach liquid channel: time to the residual drop, plain
    FP64 and FP32 Jacobian/ILU(0); the converged states (continued untimed at
    the final CFL to the round-off floor of the stiffened EOS) compared."""
    from cfdsolutions_b200 import Euler3DGPU, capi, default_params, to_rup

    m, Q = lowmach_case(LOWMACH_MESH)
    out, states = {"config": lowmach_config(m)}, {}
    # fp64_rup: the FP64 solve with the state stored as (rho, u, v, w, p) (MPFLOW3D's VARIABLE_RUP)
    for name, prec, variables in (("fp64", capi.PREC_FP64, 0), ("fp32", capi.PREC_FP32 | capi.PREC_LOW_ONLY, 0),
                                  ("fp64_rup", capi.PREC_FP64, 1)):
        cfg = dict(LOWMACH, variables=variables)
        with Euler3DGPU(m, default_params(**cfg), device=dev, stream=stream.cuda_stream) as ss:
            ss.set_state(Q if variables == 0 else to_rup(Q, LOWMACH["gamma"], LOWMACH["pinf"]))
            capi.check(capi.lib.cfd_ilu_mc_order(ss.handle, None, None), "cfd_ilu_mc_order")
            g = capi.GmresOpts(30, 30, STEADY_RTOL, capi.PC_ILU0_MC, prec, 1)
            box = {}

            def run():
                box["st"] = ss.solve_steady(max_iterations=800, drop=STEADY_DROP, include_diss=1, linear_solver=1,
                                            gmres=g, precond_update=LOWMACH_PC_UPDATE)

            ms = timed_once(run)
            st = box["st"]
            out[name] = {"seconds": ms / 1e3, "newton_iterations": st.iterations,
                         "gmres_iterations": st.linear_iterations, "rms_drop": st.rms_last / st.rms_first,
                         "converged": bool(st.rms_last <= STEADY_DROP * st.rms_first)}
            ss.set_params(default_params(**dict(cfg, cfl_min=LOWMACH["cfl_max"], cfl_ramp=0)))
            st2 = ss.solve_steady(max_iterations=100, drop=1e-4, include_diss=1, linear_solver=1, gmres=g,
                                  precond_update=LOWMACH_PC_UPDATE)
            out[name]["rms_drop_compared"] = st2.rms_last / st.rms_first
            if variables == 0:
                states[name] = ss.get_state()[:, :m.nnode]
    ref = states["fp64"]
    mom = float(np.abs(ref[1:4]).max())
    err = 0.0
    for v in range(5):
        scale = max(float(np.abs(ref[v]).max()), mom if 1 <= v <= 3 else 0.0)
        err = max(err, float(np.abs(states["fp32"][v] - ref[v]).max()) / scale)
    out["fp32"]["max_rel_err_vs_fp64"] = err
    out["fp32"]["speedup_vs_fp64"] = out["fp64"]["seconds"] / out["fp32"]["seconds"]
    out["fp64_rup"]["note"] = ("state stored as (rho, u, v, w, p): the pressure carries no gamma pinf "
                               "cancellation, so rms_drop_compared (the continued solve) falls below the "
                               "conservative floor")
    return m, out


def lowmach_port_rate(size, iters):
    """The oracle's restatement of the same implicit iteration (single
    threaded) on a smaller channel: node-iterations per second."""
    import time as _t
    from oracle import restatement
    m, Q = lowmach_case(size)
    n = m.nnode
    per = []
    for it in range(iters + 1):
        t0 = _t.perf_counter()
        s = restatement.Session(m, LOWMACH, iteration=it)
        Qb = s.apply_bc(Q)
        gr = s.gradient(Qb, 0)
        phi = s.limiter(Qb, gr)
        conv, diss, dts, _ = s.residual(Qb, gr, phi)
        dt, _ = s.deltat(dts)
        A, B = s.jacobian(Qb, dt, conv, diss, include_diss=1)
        X, _, _, _ = s.gmres(A, B, m=30, maxit=30, rtol=STEADY_RTOL, precond=2)
        Q = Qb.copy()
        Q[:, :n] += X.T
        per.append(_t.perf_counter() - t0)
    per_it = statistics.mean(per[1:])
    sample = (f"{size[0]}x{size[1]}x{size[2]}-hex channel ({n} nodes), 1+{iters} implicit iterations of the "
              "oracle's C restatement (BC, LSQ gradient, Venkatakrishnan, preconditioned Roe residual, dt, "
              "preconditioned Jacobian, GMRES(30)+ILU(0) to rtol 0.1, update), one thread")
    return n / per_it, per_it, sample


def reference_implicit_rate(sample_n, procs, iters):
    """The reference's own implicit iteration (second-order residual, Jacobian,
    10 block Gauss-Seidel sweeps, update) on a sample_n^3 cube, one
    single-threaded process per core; returns node-iterations per second."""
    from cfdsolutions_b200 import box_mesh, perturbed_freestream
    from oracle import refharness

    m = box_mesh(sample_n, jitter=0.15, seed=1234, rcm=True)
    Q = perturbed_freestream(m, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
    cfg = dict(STEADY, gradient=0)
    one = [("begin", 0), ("gradient", 0), ("limiter",), ("bc", 0), ("residual", 1), ("deltat", 0),
           ("jacobian", 1, 0), ("gs", 10, 0), ("update", 1.0)]
    outs = refharness.run_many(m, cfg, Q, one * (iters + 1), procs)
    per_it = []
    for o in outs:
        t = o["timings"]
        tot = [sum(x) for x in zip(*(t[k] for k in ("begin", "gradient", "limiter", "bc", "residual", "deltat",
                                                     "jacobian", "gs", "update")))]
        per_it.append(statistics.mean(tot[1:]))
    rate = sum(m.nnode / x for x in per_it)
    sample = (f"{sample_n}^3-hex tet cube ({m.nnode} nodes), 1+{iters} implicit iterations of the reference "
              f"(LSQ gradient, Venkatakrishnan, Roe residual, dt, approximate Roe Jacobian, 10 block Gauss-Seidel "
              f"sweeps, update) per process, {procs} concurrent single-threaded processes")
    return rate, statistics.mean(per_it), sample


def serve_requests(count, nmax, rate, seed=7):
    """Seeded request mix of the served batch: cube side log-uniform in
    [16, nmax] hexes, Mach U[0.3, 0.85], alpha U[-5, 10] deg, Poisson arrivals
    at `rate` per second (arrival offsets in seconds)."""
    rng = np.random.default_rng(seed)
    ns = np.round(np.exp(rng.uniform(np.log(16), np.log(nmax), count))).astype(int)
    machs = rng.uniform(0.3, 0.85, count)
    alphas = rng.uniform(-5.0, 10.0, count)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
    return ns, machs, alphas, arrivals - arrivals[0]


def serve_request_builder(ns, machs, alphas, precision):
    """make_request(k, precond_update) of the seeded mix: request k with the
    steady workload's physics and tolerances."""
    from cfdsolutions_b200 import default_params
    from cfdsolutions_b200.serve import request, steady_opts

    def make(k, pu):
        p = default_params(**dict(STEADY, mach=float(machs[k]), mach_min=float(machs[k]), alpha_deg=float(alphas[k])))
        return request(int(ns[k]), p, steady_opts(drop=STEADY_DROP, rtol=STEADY_RTOL, precision=precision,
                                                  precond_update=int(pu)),
                       mesh_seed=1000 + k, state_seed=2000 + k)
    return make


def serve_run(make, ks, refresh, arrivals, schedule, dev):
    """Submits requests ks (request k with refresh(k) as its preconditioner
    refresh period) at their arrival times to a server with the given
    (workers, batching, window_us) schedule -- all at once when arrivals are
    zeros, one at a time (waiting for each) when arrivals is None -- and waits
    for all; returns the results, the wall time from the first submission,
    the peak reservation and the fused-launch counts."""
    from cfdsolutions_b200.serve import Server

    workers, batching, window = schedule
    reqs = [make(k, refresh(k)) for k in ks]
    with Server(device=dev, workers=workers, budget_bytes=150e9, batching=batching, window_us=window) as srv:
        t0 = time.perf_counter()
        if arrivals is None:  # sequential: one request at a time
            res = []
            for r in reqs:
                res.append(srv.wait(srv.submit(r)))
        else:
            ids = []
            for k, r in enumerate(reqs):
                dt = arrivals[k] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                ids.append(srv.submit(r))
            res = [srv.wait(i) for i in ids]
        wall = time.perf_counter() - t0
        peak = srv.stats()["peak_reserved_bytes"]
        fused = srv.batch_stats()
    return res, wall, peak, fused


def cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def max_over_ranks(x, world, device=None):
    """The largest value of x over all ranks of the process group (x itself
    on one rank): every multi-GPU time here is the slowest rank's."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, seconds, world):
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank in at most `seconds` (the max over ranks)."""
    return units_per_rank * world / seconds


def reference_sample_config(sample_n):
    """The workload the reference arm times: the headline's flow and limiter on
    a sample_n^3 cube with the reference's own gradient (least squares; the
    reference has no Green-Gauss) and plain RCM numbering."""
    return {"workload": f"second-order residual evaluation, {sample_n}^3-hex tet cube (6 tets/hex), RCM, jitter "
                        "0.15h, least-squares gradient + Venkatakrishnan K=5 + Roe, M=0.8, alpha=1.25, +-1% noise",
            "sample_of": "the headline workload at 128^3 (Green-Gauss), which the reference cannot run",
            "numbering": "reverse Cuthill-McKee", "flux": "roe", "gradient": "least-squares",
            "limiter": "venkatakrishnan", "venkat_k": 5.0, "mach": 0.8, "alpha_deg": 1.25, "precision": "fp64"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    procs = args.cpu_procs or min(16, cpu_count())
    val, d = reference_throughput(args.cpu_sample_n, procs, max(1, min(args.warmup, 3)), max(1, args.steps))
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": d["per_pass_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": reference_sample_config(args.cpu_sample_n),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": procs, "kind": "reference", "sample": d["sample"]},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def linear_rooflines(s, mesh, stream, timed, args, peak):
    """Jacobian assembly (FP32 blocks, low-precision-only system, the steady
    solve's form), block SpMV with the FP32 matrix and one block-multicolour
    ILU(0) apply with FP32 factors, each timed alone with CUDA events over
    repeated calls on the library's stream, against the measured HBM copy
    bandwidth.  Algorithmic bytes (compulsory traffic per call):
      SpMV:     100 nnzb (FP32 blocks) + 4 nnzb (JA) + 4 (N+1) (IA) + 40 N (x) + 40 N (y)
      ILU apply: the same on the L+U factors (forward and backward solve together)
      Jacobian: 100 nnzb + 4 nnzb + 4 (N+1), plus Q (40 (N+G)), dt (8 N), residuals
                (80 N) read and B (40 N) written."""
    import torch
    from cfdsolutions_b200 import capi

    n, g = mesh.nnode, mesh.nghost
    for i in range(2):
        s.residual_step(i)
    prec = capi.PREC_FP32 | capi.PREC_LOW_ONLY
    jac = lambda i: s.Compute_Jacobian(1, 0, include_diss=1, precision=prec)  # noqa: E731
    k = max(5, args.steps // 30)
    ms_jac = timed(jac, k, 2) / k
    nnzb = s.nnzb
    capi.check(capi.lib.cfd_ilu_mc_order(s.handle, None, None), "cfd_ilu_mc_order")
    s.solve_gmres(restart=30, max_iters=2, rtol=1e-12, precond=capi.PC_ILU0_MC, precision=prec,
                  allow_not_converged=True)
    dev = torch.cuda.current_device()
    x = torch.randn((n, 5), dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    k2 = max(10, args.steps // 6)
    ms_spmv = timed(lambda i: s.spmv_device(x.data_ptr(), y.data_ptr(), capi.PREC_FP32), k2, 3) / k2
    ms_ilu = timed(lambda i: s.precond_apply_device(x.data_ptr(), y.data_ptr()), k, 2) / k
    b_mat = 100 * nnzb + 4 * nnzb + 4 * (n + 1)
    out = {"system": f"128^3 tet cube: {n} block rows, {nnzb} blocks; FP32 blocks (low-precision-only system)"}
    for name, ms, b, kern in (
            ("spmv", ms_spmv, b_mat + 80 * n, "k_bspmv<float> (five lanes per block row, two blocks in flight)"),
            ("ilu_apply", ms_ilu, b_mat + 80 * n, "k_mc_fwd + k_mc_bwd (block-multicolour ILU(0), FP32 factors)"),
            ("jacobian", ms_jac, b_mat + 40 * (n + g) + 128 * n, "k_jac_edges + k_jac_rows (FP32 blocks)")):
        ach = b / (ms / 1e3) / 1e9
        out[name] = {"bound": "hbm", "kernel": kern, "ms": ms, "algorithmic_bytes": b, "achieved": ach,
                     "peak": peak, "unit": "GB/s", "frac": ach / peak}
    return out


def profile_case(n):
    """Small fixed case for ncu captures (`--profile --n 64`): the bench
    workload on an n^3 cube, two residual steps with the node-gather kernel then
    two with the patch kernel."""
    from cfdsolutions_b200 import Euler3DGPU, box_mesh, default_params, perturbed_freestream
    from cfdsolutions_b200.mesh import NUMBERING_PATCH_RCM

    m = box_mesh(n, jitter=0.15, seed=1234, rcm=NUMBERING_PATCH_RCM)
    Q = perturbed_freestream(m, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
    for kern in (0, 1):
        with Euler3DGPU(m, default_params(**dict(CFG, residual_kernel=kern))) as s:
            s.set_state(Q)
            for i in range(2):
                s.residual_step(i)
            s.synchronize()


def profile_lowmach_case(iters):
    """`--profile-lowmach ITERS`: the low-Mach channel's first ITERS implicit
    iterations with the FP32 low-precision-only system, for launch lists."""
    from cfdsolutions_b200 import Euler3DGPU, capi, default_params
    m, Q = lowmach_case(LOWMACH_MESH)
    with Euler3DGPU(m, default_params(**LOWMACH)) as ss:
        ss.set_state(Q)
        capi.check(capi.lib.cfd_ilu_mc_order(ss.handle, None, None), "cfd_ilu_mc_order")
        g = capi.GmresOpts(30, 30, STEADY_RTOL, capi.PC_ILU0_MC, capi.PREC_FP32 | capi.PREC_LOW_ONLY, 1)
        ss.solve_steady(max_iterations=iters, drop=STEADY_DROP, include_diss=1, linear_solver=1, gmres=g,
                        precond_update=LOWMACH_PC_UPDATE)
        ss.synchronize()


def profile_steady_case(n, iters):
    """`--profile-steady ITERS --n N`: the first ITERS implicit iterations of
    the steady workload on an N^3 cube, FP64 then the FP32
    low-precision-only system, for launch lists."""
    from cfdsolutions_b200 import Euler3DGPU, box_mesh, capi, default_params, perturbed_freestream
    from cfdsolutions_b200.mesh import NUMBERING_PATCH_RCM

    m = box_mesh(n, jitter=0.15, seed=1234, rcm=NUMBERING_PATCH_RCM)
    Q = perturbed_freestream(m, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
    for prec in (capi.PREC_FP64, capi.PREC_FP32 | capi.PREC_LOW_ONLY):
        with Euler3DGPU(m, default_params(**STEADY)) as ss:
            ss.set_state(Q)
            capi.check(capi.lib.cfd_ilu_mc_order(ss.handle, None, None), "cfd_ilu_mc_order")
            g = capi.GmresOpts(30, 30, STEADY_RTOL, capi.PC_ILU0_MC, prec, 1)
            ss.synchronize()
            t0 = time.perf_counter()
            ss.solve_steady(max_iterations=iters, drop=STEADY_DROP, include_diss=1, linear_solver=1, gmres=g,
                            precond_update=STEADY_PC_UPDATE)
            ss.synchronize()
            print(f"profile-steady precision {prec}: {iters} implicit iterations in "
                  f"{time.perf_counter() - t0:.3f} s", flush=True)


def profile_linear_case(n):
    """Small fixed case for ncu captures of the linear solver
    (`--profile-linear --n 64`): the steady workload's Jacobian at CFL 1000 on
    an n^3 cube, then GMRES(30) with the block multicolour ILU(0): once with
    the FP64 system, once with the FP32 low-precision-only system."""
    from cfdsolutions_b200 import Euler3DGPU, box_mesh, capi, default_params, perturbed_freestream
    from cfdsolutions_b200.mesh import NUMBERING_PATCH_RCM

    m = box_mesh(n, jitter=0.15, seed=1234, rcm=NUMBERING_PATCH_RCM)
    Q = perturbed_freestream(m, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
    with Euler3DGPU(m, default_params(**dict(STEADY, cfl_min=1000.0))) as s:
        s.set_state(Q)
        s.residual_step(0)
        for prec in (capi.PREC_FP64, capi.PREC_FP32 | capi.PREC_LOW_ONLY):
            s.Compute_Jacobian(1, 0, 1, prec)
            s.solve_gmres(30, 30, 1e-12, capi.PC_ILU0_MC, prec, 1, allow_not_converged=True)
        s.synchronize()


def workload_config(n, mesh=None):
    c = {"workload": f"second-order residual evaluation, {n}^3-hex tet cube (6 tets/hex), RCM, jitter 0.15h, "
                     "Green-Gauss + Venkatakrishnan K=5 + Roe, M=0.8, alpha=1.25, +-1% noise",
         "numbering": "blocked RCM: reverse Cuthill-McKee over 128-node coordinate-bisection patches",
         "flux": "roe", "gradient": "green-gauss", "limiter": "venkatakrishnan", "venkat_k": 5.0, "mach": 0.8,
         "alpha_deg": 1.25, "precision": "fp64", "parallelism": "replicas (one mesh per GPU)",
         "l2": "inputs larger than L2 (resident working set > 126 MB)"}
    if mesh is not None:
        c.update(nodes=mesh.nnode, edges=mesh.nedge, ghosts=mesh.nghost)
    return c


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.profile:
        profile_case(args.n)
        return
    if args.profile_lowmach:
        profile_lowmach_case(args.profile_lowmach)
        return
    if args.profile_steady:
        profile_steady_case(args.n, args.profile_steady)
        return
    if args.profile_linear:
        profile_linear_case(args.n)
        return

    import torch
    import torch.distributed as dist

    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    dev = local
    torch.cuda.set_device(dev)

    from cfdsolutions_b200 import Euler3DGPU, box_mesh, default_params, perturbed_freestream
    from cfdsolutions_b200.mesh import NUMBERING_PATCH_RCM, NUMBERING_RCM

    t0 = time.time()
    mesh = box_mesh(args.n, jitter=0.15, seed=1234, rcm=NUMBERING_PATCH_RCM)
    Q = perturbed_freestream(mesh, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
    setup_s = time.time() - t0
    units = mesh.nedge + mesh.nbedge
    stream = torch.cuda.Stream(device=dev)
    s = Euler3DGPU(mesh, default_params(**CFG), device=dev, stream=stream.cuda_stream)
    s.set_state(Q)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    def timed(fn, k, w):
        for i in range(w):
            fn(i)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for i in range(k):
            fn(w + i)
        ev1.record(stream)
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1), world, f"cuda:{dev}")

    # ---- headline: resident residual steps (Roe)
    with Clocks(dev) as clk:
        ms = timed(lambda i: s.residual_step(i), args.steps, args.warmup)
    clocks = clk.summary()
    ms_step = ms / args.steps
    value = aggregate_rate(units * args.steps, ms / 1e3, world) / 1e9

    # ---- per-kernel breakdown of one step (events between calls)
    names = ["begin", "bc", "gradient", "limiter", "residual", "deltat"]
    calls = [lambda: s.begin_iteration(0), lambda: s.Apply_Boundary_Condition(0), s.Compute_Gradient,
             s.Compute_Limiter, lambda: s.Compute_Residual(1), lambda: s.Compute_DeltaT(0)]
    reps = max(3, args.steps // 2)
    acc = {n: 0.0 for n in names}
    for _ in range(reps):
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(calls) + 1)]
        evs[0].record(stream)
        for c, e in zip(calls, evs[1:]):
            c()
            e.record(stream)
        torch.cuda.synchronize(dev)
        for j, n in enumerate(names):
            acc[n] += evs[j].elapsed_time(evs[j + 1])
    breakdown = {n: acc[n] / reps for n in names}

    # ---- roofline of the dominant kernel (flux residual): its call inside the
    # steps above (events around each call), i.e. right after the fused
    # Green-Gauss + limiter pass, whose limited gradients it reads
    ms_res = breakdown["residual"]
    peak, peak_kind = measured_peak()
    abytes = algorithmic_bytes(mesh.nnode, mesh.nedge, mesh.nghost)
    achieved = abytes / (ms_res / 1e3) / 1e9
    tpe = traffic_from_profile()
    # one cfd_residual: k_residual_gather<ROE,SECOND,limited gradients> (interior edges),
    # k_residual_bnd<ROE> (boundary edges) and the gated limiter-fix passes
    roofline = {"bound": "hbm", "kernel": "k_residual_gather<ROE,SECOND> + k_residual_bnd<ROE>", "achieved": achieved,
                "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic_bytes_per_launch": abytes, "launch_ms": ms_res,
                "traffic": (tpe * units) if tpe else None,
                # the kernel is bound by FP64 issue, not HBM (ncu, profiles/residual_roe2_128.md)
                "fp64_pipe_active_pct": profile_figure("fp64_pipe_active_pct"),
                "issue_active_pct": profile_figure("issue_active_pct")}

    # ---- other flux families (HLLC, AUSM+)
    per_flux = {"roe": {"gedges_per_s": value / world, "ms_per_step": ms_step}}
    for fl in (1, 2):
        s.set_params(default_params(**dict(CFG, flux_scheme=fl)))
        msf = timed(lambda i: s.residual_step(i), args.steps, args.warmup)
        per_flux[FLUX_NAMES[fl]] = {"gedges_per_s": units * args.steps / (msf / 1e3) / 1e9,
                                    "ms_per_step": msf / args.steps}
    s.set_params(default_params(**CFG))

    # ---- the same step with the shared-memory patch kernel, and on the plain node-level RCM numbering
    side = {}
    s.set_params(default_params(**dict(CFG, residual_kernel=1)))
    msg = timed(lambda i: s.residual_step(i), args.steps, args.warmup)
    side["patch_kernel_gedges_per_s"] = units * args.steps / (msg / 1e3) / 1e9
    s.set_params(default_params(**CFG))
    # the headline mesh with the reference's least-squares gradient
    s.set_params(default_params(**dict(CFG, gradient=0)))
    msg = timed(lambda i: s.residual_step(i), args.steps, args.warmup)
    side["lsq_gradient_gedges_per_s"] = units * args.steps / (msg / 1e3) / 1e9
    s.set_params(default_params(**CFG))
    # the reference arm's own sample (same mesh builder, numbering and options),
    # for a like-for-like ratio beside the headline
    ms_ = args.cpu_sample_n
    m3 = box_mesh(ms_, jitter=0.15, seed=1234, rcm=NUMBERING_RCM)
    q3 = perturbed_freestream(m3, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
    with Euler3DGPU(m3, default_params(**dict(CFG, gradient=0)), device=dev, stream=stream.cuda_stream) as s3:
        s3.set_state(q3)
        ms3 = timed(lambda i: s3.residual_step(i), args.steps, args.warmup)
    side["reference_sample_on_gpu"] = {"config": reference_sample_config(ms_),
                                       "gedges_per_s": (m3.nedge + m3.nbedge) * args.steps / (ms3 / 1e3) / 1e9,
                                       "ms_per_step": ms3 / args.steps}
    del m3, q3
    if args.side_rcm:
        m2 = box_mesh(args.n, jitter=0.15, seed=1234, rcm=NUMBERING_RCM)
        q2 = perturbed_freestream(m2, CFG["gamma"], CFG["mach"], CFG["alpha_deg"], noise=0.01, seed=1235)
        with Euler3DGPU(m2, default_params(**CFG), device=dev, stream=stream.cuda_stream) as s2:
            s2.set_state(q2)
            ms2 = timed(lambda i: s2.residual_step(i), args.steps, args.warmup)
        side["plain_rcm_numbering_gedges_per_s"] = units * args.steps / (ms2 / 1e3) / 1e9
        del m2, q2

    # ---- end to end through the C ABI with pinned host buffers
    qh = torch.from_numpy(np.ascontiguousarray(Q)).pin_memory()
    conv = torch.empty((5, mesh.nnode), dtype=torch.float64).pin_memory()
    diss = torch.empty((5, mesh.nnode), dtype=torch.float64).pin_memory()
    qn, cn, dn = qh.numpy(), conv.numpy(), diss.numpy()
    k_e2e = max(args.warmup + 3, args.steps // 3)
    s.set_step_pipeline(0)  # the calls one after the other: copy in, kernels, copy out
    ms_serial = timed(lambda i: s.residual_step(i, qn, out=(cn, dn)), k_e2e, args.warmup)
    s.set_step_pipeline(-1)  # copies overlapped with the kernels in node chunks (the default)
    ms_e2e = timed(lambda i: s.residual_step(i, qn, out=(cn, dn)), k_e2e, args.warmup)
    e2e = {"value": units * k_e2e * world / (ms_e2e / 1e3) / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": int(qn.nbytes), "d2h_bytes_per_step": int(cn.nbytes + dn.nbytes),
           "ms_per_step": ms_e2e / k_e2e, "steps": k_e2e,
           "pcie_gbs": (qn.nbytes + cn.nbytes + dn.nbytes) / (ms_e2e / k_e2e / 1e3) / 1e9,
           "unpipelined": {"value": units * k_e2e * world / (ms_serial / 1e3) / 1e9, "ms_per_step": ms_serial / k_e2e}}

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import refharness
        if refharness.available():
            procs = args.cpu_procs or min(16, cpu_count())
            val, d = reference_throughput(args.cpu_sample_n, procs, 1, 2)
            cpu = {"value": val, "unit": UNIT, "cores": procs, "kind": "reference", "sample": d["sample"],
                   "per_core_value": d["per_process_gedges"]}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": "reference oracle library not built"}

    # ---- the implicit step's linear-algebra kernels on the same 128^3 system
    linear = None if args.no_linear else linear_rooflines(s, mesh, stream, timed, args, peak)
    s.close()

    # ---- time to the steady residual drop (plain FP64 and mixed precision)
    def timed_once(fn):
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        fn()
        ev1.record(stream)
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1), world, f"cuda:{dev}")

    steady = None
    if not args.no_steady:
        steady = {"metric": "time to steady residual drop", "unit": "s", "higher_is_better": False,
                  "config": steady_config(args.n)}
        steady.update(steady_solves(mesh, Q, dev, stream, timed_once))
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            from oracle import refharness
            if refharness.available():
                procs = args.cpu_procs or min(16, cpu_count())
                rate, per_it, sample = reference_implicit_rate(32, procs, 2)
                gpu_rate = mesh.nnode * steady["fp64"]["newton_iterations"] / steady["fp64"]["seconds"]
                steady["cpu_baseline"] = {"value": rate, "unit": "node-iterations/s", "cores": procs,
                                          "kind": "reference", "sample": sample, "seconds_per_iteration": per_it,
                                          "gpu_fp64_value": gpu_rate}
                errs = reference_converged_errors(dev, stream)
                steady["vs_reference_cpu_solve"] = errs
                for name in ("fp64", "fp32", "bf16"):
                    steady[name]["max_rel_err_vs_reference_cpu_solve"] = errs[name]

    # ---- the low-Mach liquid channel (stiffened gas, preconditioned Roe)
    lowmach = None
    if not args.no_lowmach:
        lm_mesh, lowmach = lowmach_solves(dev, stream, timed_once)
        lowmach.update({"metric": "time to steady residual drop", "unit": "s", "higher_is_better": False})
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            rate, per_it, sample = lowmach_port_rate((96, 24, 24), 3)
            gpu_rate = lm_mesh.nnode * lowmach["fp64"]["newton_iterations"] / lowmach["fp64"]["seconds"]
            lowmach["cpu_baseline"] = {"value": rate, "unit": "node-iterations/s", "cores": 1, "kind": "port",
                                       "sample": sample, "seconds_per_iteration": per_it, "gpu_fp64_value": gpu_rate}

    # ---- served batch (config 5: continuous admission, fused residual launches,
    # autotuned schedule) vs sequential plain FP64 solves
    serve = None
    if not args.no_serve:
        from cfdsolutions_b200 import capi
        from cfdsolutions_b200.serve import SIZE_BUCKETS, autotune, size_bucket
        ns, machs, alphas, arr = serve_requests(args.serve_requests, args.serve_nmax, args.serve_rate)
        mixed = capi.PREC_FP32 | capi.PREC_LOW_ONLY
        make = serve_request_builder(ns, machs, alphas, mixed)
        make64 = serve_request_builder(ns, machs, alphas, capi.PREC_FP64)
        calib = list(range(0, len(ns), max(1, len(ns) // args.serve_calibration)))[:args.serve_calibration]
        barrier()
        tune = autotune(make, calib, device=dev)
        refresh = lambda k: tune["precond_update"].get(size_bucket(int(ns[k])), STEADY_PC_UPDATE)  # noqa: E731
        sched = tune["server"]
        every = list(range(len(ns)))
        barrier()
        # latency at the stated rate: every other request of the mix, arriving at their Poisson offsets
        at_rate = every[::2]
        res, wall, peak, fused = serve_run(make, at_rate, refresh, arr[::2], sched, dev)
        barrier()
        sat, sat_wall, sat_peak, sat_fused = serve_run(make, every, refresh, np.zeros(len(ns)), sched, dev)
        barrier()
        # sequential plain FP64 on a subsample of the same mix spread evenly over its sizes (the
        # smallest and the largest included); the whole mix's sequential time is each request's
        # time interpolated in cube side between the sampled ones (log-log), since solve time
        # grows ~ n^3 and a small sample's mean is dominated by where its largest member falls
        by_size = sorted(every, key=lambda k: (int(ns[k]), k))
        seq_ks = [by_size[i] for i in sorted(set(np.linspace(0, len(ns) - 1, args.serve_sequential).round()
                                                   .astype(int).tolist()))]
        seq, seq_wall, _, _ = serve_run(make64, seq_ks, lambda k: STEADY_PC_UPDATE, None, (1, False, 0.0), dev)
        side_t = {}
        for k, r in zip(seq_ks, seq):
            side_t.setdefault(int(ns[k]), []).append(r.latency)
        xs = np.log(np.array(sorted(side_t)))
        ys = np.log(np.array([np.mean(side_t[n]) for n in sorted(side_t)]))
        seq_mix_s = float(np.exp(np.interp(np.log(ns.astype(float)), xs, ys)).sum())
        # host wall clocks of the replicas' servers: the slowest rank sets each rate
        wall, sat_wall, seq_wall, seq_mix_s = (max_over_ranks(w, world, f"cuda:{dev}")
                                               for w in (wall, sat_wall, seq_wall, seq_mix_s))
        lat = np.array([r.latency for r in res])
        sat_lat = np.array([r.latency for r in sat])
        conv = lambda rs: sum(r.status == 0 and r.rms_last <= STEADY_DROP * r.rms_first for r in rs)  # noqa: E731
        ok, ok_seq = conv(res) + conv(sat), conv(seq)
        serve = {
            "metric": "served steady solves", "unit": "solves/s",
            "config": {"requests": args.serve_requests, "cube_side": f"log-uniform in [16, {args.serve_nmax}] hexes",
                       "mach": "U[0.3, 0.85]", "alpha_deg": "U[-5, 10]",
                       "arrivals": f"capacity: all {len(ns)} at once; latency: every other request of the mix "
                                   f"({len(at_rate)}) at Poisson arrivals of {args.serve_rate / 2:g}/s",
                       "budget_gb": 150.0, "physics": "as steady",
                       "served_precision": "fp32 low-precision-only Jacobian + ILU(0)",
                       "sequential": f"plain fp64 solves one at a time through the same server (1 worker, no "
                                     f"fusion) on {len(seq_ks)} requests of the mix spread evenly over its cube "
                                     f"sides; value = requests / the mix's time, each request's time interpolated "
                                     f"(log-log in cube side) between the sampled ones"},
            "autotuner": {"calibration_requests": len(calib), "workers": sched[0], "fused_residual_and_spmv_launches": sched[1],
                          "window_us": sched[2],
                          "precond_update_by_cube_side": {f"[{SIZE_BUCKETS[b][0]}, {min(SIZE_BUCKETS[b][1], 97)})": v
                                                          for b, v in tune["precond_update"].items()},
                          "timings": tune["timings"]},
            # launches over a request table in the saturated run, and the requests' jobs they carried
            "fused_launches": sat_fused,
            # capacity: all requests submitted at once; latency: at the stated arrival rate
            "value": aggregate_rate(len(sat), sat_wall, world), "wall_s": sat_wall,
            "saturated_p50_s": float(np.percentile(sat_lat, 50)), "saturated_p99_s": float(np.percentile(sat_lat, 99)),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "at_rate_solves_per_s": aggregate_rate(len(res), wall, world), "converged": ok, "requests_run": len(res) + len(sat),
            "peak_reserved_gb": max(peak, sat_peak) / 1e9,
            "sequential_fp64": {"value": aggregate_rate(len(ns), seq_mix_s, world), "mix_seconds": seq_mix_s,
                                "sample_solves_per_s": aggregate_rate(len(seq), seq_wall, world),
                                "sample_wall_s": seq_wall, "sample_requests": len(seq), "converged": ok_seq,
                                "p50_solve_s": float(np.percentile([r.t_done - r.t_admit for r in seq], 50))},
        }
        serve["speedup_vs_sequential_fp64"] = serve["value"] / serve["sequential_fp64"]["value"]

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded tet-split cube, seeded +-1% state noise)",
            "config": workload_config(args.n, mesh), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": KERNELS_PER_STEP * args.steps, "clocks": clocks, "per_flux": per_flux,
            "breakdown_ms": breakdown, "variants": side, "setup_s": setup_s, "linear": linear, "steady": steady,
            "lowmach": lowmach,
            "serve": serve,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
