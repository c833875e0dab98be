"""The C ABI: the library loads without a GPU and exports every function
declared in include/cfd_b200.h; the host-side entry points that need no GPU
(mesh builder, restart files, option defaults) work on CPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from cfdsolutions_b200 import _capi as capi
from cfdsolutions_b200 import box_mesh

HEADER = Path(__file__).resolve().parents[1] / "include" / "cfd_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(cfd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) > 30
    for n in names:
        assert hasattr(capi.lib, n), f"{n} declared in cfd_b200.h but not exported"
        assert n in capi.SIGNATURES, f"{n} has no ctypes signature"


def test_abi_version_and_defaults():
    assert capi.lib.cfd_abi_version() == 6
    p = capi.Params()
    capi.lib.cfd_params_default(C.byref(p))
    assert p.gamma == 1.4 and p.flux_scheme == capi.FLUX_ROE and p.limiter == capi.LIMITER_NONE
    o = capi.GmresOpts()
    capi.lib.cfd_gmres_default(C.byref(o))
    assert o.restart == 30 and o.precond == capi.PC_ILU0


def test_null_context_is_an_error_not_a_crash():
    assert capi.lib.cfd_residual(None, 1) == -1
    assert capi.lib.cfd_gmres(None, None, None) == -5
    assert "NULL" in capi.lib.cfd_last_error().decode() or capi.lib.cfd_last_error() is not None


def test_restart_roundtrip(tmp_path):
    n, g = 7, 3
    Q = np.random.default_rng(0).standard_normal((5, n + g))
    p = str(tmp_path / "r.bin").encode()
    capi.check(capi.lib.cfd_restart_write(p, 12, n, g, capi.ptr(Q)), "write")
    raw = (tmp_path / "r.bin").read_bytes()
    # Restart_Writer layout (Euler3D/src/RestartIO.cpp:45-109): 4 int32 then rows of 5 doubles
    hdr = np.frombuffer(raw[:16], np.int32)
    assert hdr.tolist() == [12, n, g, 5]
    rows = np.frombuffer(raw[16:], np.float64).reshape(n + g, 5)
    np.testing.assert_array_equal(rows.T, Q)
    Q2 = np.zeros_like(Q)
    it = C.c_int()
    capi.check(capi.lib.cfd_restart_read(p, C.byref(it), n, g, capi.ptr(Q2)), "read")
    assert it.value == 12
    np.testing.assert_array_equal(Q2, Q)
    assert capi.lib.cfd_restart_read(p, C.byref(it), n + 1, g, capi.ptr(Q2)) == -4


def test_mesh_counts_match_closed_forms():
    # tet-split cube of n^3 hexes: E = 3n(n+1)^2 + 3n^2(n+1) + n^3, G = 36 n^2
    for n in (2, 5, 20):
        m = box_mesh(n, jitter=0.15, seed=3)
        assert m.nnode == (n + 1) ** 3
        assert m.nedge == 3 * n * (n + 1) ** 2 + 3 * n * n * (n + 1) + n ** 3
        assert m.nbedge == m.nghost == 36 * n * n
        assert abs(m.cvol.sum() - 1.0) < 1e-12


def test_mesh_dual_closure():
    # every dual cell is closed: sum of outward area vectors = 0 (Area_Volume.cpp:861-899)
    m = box_mesh(6, jitter=0.15, seed=5, rcm=True)
    acc = np.zeros((m.nnode, 3))
    np.add.at(acc, m.edge_nodes[:, 0], m.edge_areav)
    np.add.at(acc, m.edge_nodes[:, 1], -m.edge_areav)
    np.add.at(acc, m.bedge_nodes[:, 0], m.bedge_areav)
    assert np.abs(acc).max() < 1e-15
    # orientation: area vector points from L to R
    d = m.coords[m.edge_nodes[:, 1]] - m.coords[m.edge_nodes[:, 0]]
    assert (np.einsum("ij,ij->i", d, m.edge_areav) > 0).all()


def test_rcm_reduces_bandwidth():
    m0 = box_mesh(8, jitter=0.1, seed=1, rcm=False)
    m1 = box_mesh(8, jitter=0.1, seed=1, rcm=True)
    bw = lambda m: int(np.abs(m.edge_nodes[:, 1] - m.edge_nodes[:, 0]).max())  # noqa: E731
    assert bw(m1) <= bw(m0)
    assert abs(m1.cvol.sum() - m0.cvol.sum()) < 1e-12


def test_mesh_rejects_bad_cells():
    coords = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    tets = np.array([[0, 2, 1, 3]], np.int32)  # negative orientation
    with pytest.raises(capi.CfdError):
        from cfdsolutions_b200 import from_cells
        from_cells(coords, tets, np.zeros((0, 3), np.int32), np.zeros(0, np.int32))


def test_perturbed_freestream_matches_the_freestream_without_noise():
    """cfd_perturbed_freestream (host code, the serving loop's initial state)
    is the generic freestream at noise 0, and stays within +-noise of it."""
    import ctypes as C

    from cfdsolutions_b200.mesh import perturbed_freestream
    from cfdsolutions_b200 import box_mesh

    fb = np.ones(6, np.int32)
    h = C.c_void_p()
    capi.check(capi.lib.cfd_mesh_box(4, 4, 4, 1.0, 1.0, 1.0, 0.1, 3, 0, capi.ptr(fb), C.byref(h)), "cfd_mesh_box")
    try:
        m = box_mesh(4, jitter=0.1, seed=3)
        n = m.nnode + m.nghost
        Q0 = np.empty((5, n))
        capi.check(capi.lib.cfd_perturbed_freestream(h, 1.4, 0.7, 3.0, 1.0, 0.0, 9, capi.ptr(Q0)), "pf")
        np.testing.assert_allclose(Q0, perturbed_freestream(m, 1.4, 0.7, 3.0, 1.0, noise=0.0), rtol=1e-15, atol=1e-15)
        Q1 = np.empty((5, n))
        capi.check(capi.lib.cfd_perturbed_freestream(h, 1.4, 0.7, 3.0, 1.0, 0.02, 9, capi.ptr(Q1)), "pf")
        rho = Q1[0, :m.nnode]
        assert np.all(np.abs(rho - 1.0) <= 0.02) and np.std(rho) > 0.005
        np.testing.assert_array_equal(Q1[:, m.nnode:], Q0[:, m.nnode:])
        Q2 = np.empty((5, n))
        capi.check(capi.lib.cfd_perturbed_freestream(h, 1.4, 0.7, 3.0, 1.0, 0.02, 9, capi.ptr(Q2)), "pf")
        np.testing.assert_array_equal(Q1, Q2)
    finally:
        capi.lib.cfd_mesh_free(h)


def test_initial_state_in_rup_variables():
    """cfd_initial_state with variables = CFD_VARS_RUP writes the same
    perturbed freestream as (rho, u, v, w, p); to_rup / to_conservative
    convert between the two to round-off, ideal and stiffened gas."""
    from cfdsolutions_b200 import default_params, to_conservative, to_rup

    fb = np.ones(6, np.int32)
    h = C.c_void_p()
    capi.check(capi.lib.cfd_mesh_box(4, 4, 4, 1.0, 1.0, 1.0, 0.1, 3, 0, capi.ptr(fb), C.byref(h)), "cfd_mesh_box")
    try:
        m = box_mesh(4, jitter=0.1, seed=3)
        n = m.nnode + m.nghost
        noise = np.array([0.02, 0.03, 0.01])
        for gamma, pinf in ((1.4, 0.0), (4.4, 6000.0)):
            p = default_params(gamma=gamma, pinf=pinf, mach=0.3)
            Qc, Qr = np.empty((5, n)), np.empty((5, n))
            capi.check(capi.lib.cfd_initial_state(h, C.byref(p), capi.ptr(noise), 5, capi.ptr(Qc)), "is")
            p.variables = 1
            capi.check(capi.lib.cfd_initial_state(h, C.byref(p), capi.ptr(noise), 5, capi.ptr(Qr)), "is")
            np.testing.assert_allclose(to_rup(Qc, gamma, pinf), Qr, rtol=1e-9 if pinf else 1e-14, atol=1e-14)
            np.testing.assert_allclose(to_conservative(Qr, gamma, pinf), Qc, rtol=1e-14, atol=1e-14)
            assert np.all(Qr[4] > 0.98) and np.all(Qr[4] < 1.02)  # the pressure itself, not rho et
    finally:
        capi.lib.cfd_mesh_free(h)
