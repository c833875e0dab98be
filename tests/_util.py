"""Helpers shared by the tests: configurations, error norms."""
import numpy as np

from cfdsolutions_b200 import box_mesh, default_params, perturbed_freestream

# Config 1 of the hot path: 20^3 hexes -> 6 tets each, jitter 0.15h, far field,
# gamma 1.4, M 0.5, alpha 2 deg, +-1 % seeded noise, first-order Roe, CFL 10.
CFG1 = dict(flux_scheme=0, order=0, limiter=-1, gamma=1.4, mach=0.5, mach_min=0.5, alpha_deg=2.0,
            cfl_min=10.0, cfl_max=10.0)


def make_case(n=20, seed=11, rcm=False, cfg=None, noise=0.01, mesh=None):
    cfg = dict(CFG1 if cfg is None else cfg)
    m = mesh if mesh is not None else box_mesh(n, jitter=0.15, seed=seed, rcm=rcm)
    Q = perturbed_freestream(m, cfg.get("gamma", 1.4), cfg.get("mach", 0.5), cfg.get("alpha_deg", 2.0),
                             cfg.get("beta_deg", 0.0), noise=noise, seed=seed + 1, pinf=cfg.get("pinf", 0.0))
    return m, cfg, Q


def params_from(cfg):
    return default_params(**cfg)


def relerr(a, b):
    """max |a-b| / max |b| over the whole field (normwise, per call)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def relerr_rows(a, b):
    """max over components of normwise relative error (rows = equations)."""
    return max(relerr(x, y) for x, y in zip(a, b))


def low_pressure_spots(Q, nnode, gamma, scale=0.02, seed=5, share=0.03):
    """Q with the pressure of a seeded 3 % of the nodes scaled by `scale`
    (momentum kept): the reconstructed pressure of those nodes' neighbours goes
    negative, so the limiter's pressure correction fires."""
    rng = np.random.default_rng(seed)
    Q = Q.copy()
    idx = rng.choice(nnode, size=max(1, int(share * nnode)), replace=False)
    ke = 0.5 * (Q[1:4, idx] ** 2).sum(0) / Q[0, idx]
    Q[4, idx] = scale * (Q[4, idx] - ke) + ke
    return Q
