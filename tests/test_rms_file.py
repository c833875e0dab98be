"""The library's residual history file against the reference's own writers.

Euler3D's RMS_Writer (Euler3D/src/RMSIO.cpp:21-97) and MPFLOW3D's
(MPFLOW3D/src/RMSIO.cpp:21-154), compiled from their sources, write
Residual.res from values the harness sets; cfd_rms_file_* writes the same
values and the two files must be byte-identical: header, column names, rule
lines, number formats and MPFLOW3D's normalisation over its first five
writes.  MPFLOW3D computes its RMS from the residual arrays itself; the values
handed to the library are the same sums in the same order.
"""
import ctypes as C
import math

import numpy as np
import pytest

from cfdsolutions_b200 import box_mesh, capi
from tests._util import CFG1, make_case


def _library_file(tmp_path, layout, variables, precond, lines):
    path = tmp_path / f"lib_{layout}_{variables}_{precond}.res"
    h = C.c_void_p()
    capi.check(capi.lib.cfd_rms_file_open(str(path).encode(), layout, variables, precond, C.byref(h)),
               "cfd_rms_file_open")
    for it, rms, ext, sig in lines:
        r = np.ascontiguousarray(rms, np.float64)
        e = np.ascontiguousarray(ext, np.float64)
        s = np.ascontiguousarray(sig, np.float64)
        capi.check(capi.lib.cfd_rms_file_write(h, it, capi.ptr(r), capi.ptr(e), capi.ptr(s)), "cfd_rms_file_write")
    capi.check(capi.lib.cfd_rms_file_close(h), "cfd_rms_file_close")
    return path.read_bytes()


def _lines(seed, count=7):
    rng = np.random.default_rng(seed)
    out = []
    for it in range(count):
        rms = 10.0 ** rng.uniform(-9, -2, 6)
        ext = np.sort(10.0 ** rng.uniform(-4, 1, 8).reshape(4, 2), axis=1).ravel()
        sig = np.sort(rng.uniform(0.01, 1.0, 2))
        out.append((it, rms, ext, sig))
    return out


@pytest.mark.parametrize("precond", [0, 1])
def test_euler3d_residual_file_is_byte_identical(ref_available, tmp_path, precond):
    from oracle import refharness
    cfg = dict(CFG1, flux_scheme=3 if precond else 0)  # PRECOND_METHOD_ROE_LMFIX turns the sigma columns on
    m, cfg, Q = make_case(n=3, seed=5, cfg=cfg)
    lines = _lines(3 + precond)
    steps = [("rms_write", it, rms, ext, sig) for it, rms, ext, sig in lines] + [("rms_close",),
                                                                                ("get", "residual_file")]
    ref = refharness.run(m, cfg, Q, steps)["residual_file"]
    mine = _library_file(tmp_path, capi.RMSFILE_EULER3D, 0, precond, lines)
    assert len(ref) > 0
    assert mine == ref


def _mpf_rms(conv, diss):
    """MPFLOW3D's RMS (RMSIO.cpp:106-118): sums of squares in node order."""
    n = conv.shape[1]
    s = [0.0] * 5
    for i in range(n):
        for k in range(5):
            r = conv[k, i] + diss[k, i]
            s[k] += r * r
    tot = s[0] + s[1] + s[2] + s[3] + s[4]
    return [math.sqrt(x / n) for x in s] + [math.sqrt(tot / (5.0 * n))]


@pytest.mark.parametrize("precond", [0, 1])
def test_mpflow3d_residual_file_is_byte_identical(tmp_path, precond):
    from oracle import mpfharness
    if not mpfharness.available():
        pytest.skip("MPFLOW3D oracle not built (make -C oracle ref)")
    cfg = dict(CFG1, mpf_variable="con")
    if precond:
        cfg.update(flux_scheme=4, precond_method=5, precond_type=1, precond_mach=0.2)
    m = box_mesh(3, jitter=0.1, seed=5)
    _, cfg, Q = make_case(mesh=m, cfg=cfg, seed=5)
    rng = np.random.default_rng(11 + precond)
    steps, lines = [], []
    for it, _, ext, sig in _lines(7 + precond, count=8):
        conv = rng.standard_normal((5, m.nnode)) * 10.0 ** (-it)
        diss = rng.standard_normal((5, m.nnode)) * 10.0 ** (-it - 1)
        steps.append(("rms_write", it, conv, diss, ext, sig))
        lines.append((it, _mpf_rms(conv, diss), ext, sig))
    steps += [("rms_close",), ("get", "residual_file")]
    ref = mpfharness.run(m, cfg, Q, steps)["residual_file"]
    mine = _library_file(tmp_path, capi.RMSFILE_MPFLOW3D, capi.VARS_CONSERVATIVE,
                         precond, lines)
    assert len(ref) > 0
    assert mine == ref
