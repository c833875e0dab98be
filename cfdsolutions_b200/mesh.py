"""Median-dual meshes in the reference's array layout, built by the library's
O(N+E) host builder (``cfd_mesh_box`` / ``cfd_mesh_from_cells``).

Array conventions follow the reference (Euler3D/include/Commons.h:97-105):
``edge_nodes[e] = (L, R)`` with ``L < R`` and ``edge_areav[e]`` pointing from
``L`` to ``R``; boundary edge ``b`` joins physical node ``bedge_nodes[b,0]`` to
its private ghost node ``nnode + b`` with the outward area vector.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi as capi


@dataclass
class Mesh:
    nnode: int
    nghost: int
    edge_nodes: np.ndarray   # int32 [nedge, 2]
    edge_areav: np.ndarray   # float64 [nedge, 3]
    bedge_nodes: np.ndarray  # int32 [nbedge, 2]
    bedge_areav: np.ndarray  # float64 [nbedge, 3]
    bedge_type: np.ndarray   # int32 [nbedge]
    cvol: np.ndarray         # float64 [nnode]
    coords: np.ndarray       # float64 [nnode, 3]
    n2n_ia: np.ndarray       # int32 [nnode+1]
    n2n_ja: np.ndarray       # int32 [2*nedge]
    tets: np.ndarray | None = None
    tris: np.ndarray | None = None
    tri_bc: np.ndarray | None = None

    @property
    def nedge(self) -> int:
        return int(self.edge_nodes.shape[0])

    @property
    def nbedge(self) -> int:
        return int(self.bedge_nodes.shape[0])


def _export(handle, with_cells: bool) -> Mesh:
    sizes = np.zeros(7, np.int64)
    capi.check(capi.lib.cfd_mesh_sizes(handle, capi.ptr(sizes)), "cfd_mesh_sizes")
    nnode, nghost, nedge, nbedge, ntet, ntri, nnz = (int(x) for x in sizes)
    m = Mesh(
        nnode=nnode, nghost=nghost,
        edge_nodes=np.zeros((nedge, 2), np.int32), edge_areav=np.zeros((nedge, 3)),
        bedge_nodes=np.zeros((nbedge, 2), np.int32), bedge_areav=np.zeros((nbedge, 3)),
        bedge_type=np.zeros(nbedge, np.int32), cvol=np.zeros(nnode), coords=np.zeros((nnode, 3)),
        n2n_ia=np.zeros(nnode + 1, np.int32), n2n_ja=np.zeros(nnz, np.int32),
    )
    capi.check(capi.lib.cfd_mesh_export(handle, *(capi.ptr(a) for a in (
        m.edge_nodes, m.edge_areav, m.bedge_nodes, m.bedge_areav, m.bedge_type, m.cvol, m.coords, m.n2n_ia,
        m.n2n_ja))), "cfd_mesh_export")
    if with_cells:
        m.tets = np.zeros((ntet, 4), np.int32)
        m.tris = np.zeros((ntri, 3), np.int32)
        m.tri_bc = np.zeros(ntri, np.int32)
        capi.check(capi.lib.cfd_mesh_export_cells(handle, capi.ptr(m.tets), capi.ptr(m.tris), capi.ptr(m.tri_bc)),
                   "cfd_mesh_export_cells")
    return m


NUMBERING_NATURAL, NUMBERING_RCM, NUMBERING_PATCH_RCM = 0, 1, 2
PATCH_NODES = 128


def box_mesh(n: int | tuple[int, int, int], lengths=(1.0, 1.0, 1.0), jitter: float = 0.15, seed: int = 1,
             rcm: bool | int = False, face_bc=(1, 1, 1, 1, 1, 1), with_cells: bool = False,
             ugrid_path: str | None = None) -> Mesh:
    """Tet-split box (6 tets per hex), interior nodes jittered by U(+-jitter*h).

    ``rcm``: False/0 natural numbering, True/1 reverse Cuthill-McKee,
    2 blocked RCM over 128-node coordinate-bisection patches."""
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    fb = np.ascontiguousarray(face_bc, dtype=np.int32)
    h = C.c_void_p()
    capi.check(capi.lib.cfd_mesh_box(nx, ny, nz, float(lengths[0]), float(lengths[1]), float(lengths[2]),
                                     float(jitter), int(seed), int(rcm), capi.ptr(fb), C.byref(h)),
               "cfd_mesh_box")
    try:
        if ugrid_path is not None:
            capi.check(capi.lib.cfd_mesh_write_ugrid(h, ugrid_path.encode()), "cfd_mesh_write_ugrid")
        return _export(h, with_cells)
    finally:
        capi.lib.cfd_mesh_free(h)


def read_ugrid(path: str, bc_types=None, numbering: int = 0) -> Mesh:
    """Mixed-element UGRID mesh (tets, pyramids, prisms, hexahedra; boundary
    triangles and quadrilaterals) and its median dual (``cfd_mesh_read_ugrid``).
    ``bc_types[t-1]`` is the BC type of boundary tag t (None: far field)."""
    h = C.c_void_p()
    tb = None if bc_types is None else np.ascontiguousarray(bc_types, np.int32)
    capi.check(capi.lib.cfd_mesh_read_ugrid(str(path).encode(), 0 if tb is None else tb.size,
                                            None if tb is None else capi.ptr(tb), int(numbering), C.byref(h)),
               "cfd_mesh_read_ugrid")
    try:
        return _export(h, False)
    finally:
        capi.lib.cfd_mesh_free(h)


def from_cells(coords: np.ndarray, tets: np.ndarray, tris: np.ndarray, tri_bc: np.ndarray) -> Mesh:
    coords = np.ascontiguousarray(coords, np.float64)
    tets = np.ascontiguousarray(tets, np.int32)
    tris = np.ascontiguousarray(tris, np.int32)
    tri_bc = np.ascontiguousarray(tri_bc, np.int32)
    h = C.c_void_p()
    capi.check(capi.lib.cfd_mesh_from_cells(coords.shape[0], capi.ptr(coords), tets.shape[0], capi.ptr(tets),
                                            tris.shape[0], capi.ptr(tris), capi.ptr(tri_bc), C.byref(h)),
               "cfd_mesh_from_cells")
    try:
        return _export(h, True)
    finally:
        capi.lib.cfd_mesh_free(h)


def perturbed_freestream(mesh: Mesh, gamma: float, mach: float, alpha_deg: float, beta_deg: float = 0.0,
                         noise=0.01, seed: int = 2, pinf: float = 0.0) -> np.ndarray:
    """Conservative state SoA [5, nnode+nghost]: freestream of the generic
    non-dimensionalisation (rho=1, p=1, c=sqrt(gamma); Euler3D/src/Material.cpp:119-124,
    :185-210), or of the stiffened gas with constant ``pinf`` (c = sqrt(gamma (1 + pinf))),
    with density, velocity and pressure of physical nodes multiplied by
    (1 + U(+-noise)) from ``seed``; ``noise`` is one amplitude or a
    (density, velocity, pressure) triple."""
    nr, nv, npr = (noise, noise, noise) if np.isscalar(noise) else tuple(noise)
    n = mesh.nnode + mesh.nghost
    c = np.sqrt(gamma * (1.0 + pinf))
    a, b = np.deg2rad(alpha_deg), np.deg2rad(beta_deg)
    u = mach * c * np.cos(a) * np.cos(b)
    v = mach * c * np.sin(a)
    w = mach * c * np.sin(b) * np.cos(a)
    rho = np.ones(n)
    vel = np.tile(np.array([u, v, w])[:, None], (1, n))
    p = np.ones(n)
    rng = np.random.default_rng(seed)
    k = mesh.nnode
    rho[:k] *= 1.0 + nr * rng.uniform(-1, 1, k)
    vel[:, :k] *= 1.0 + nv * rng.uniform(-1, 1, (3, k))
    p[:k] *= 1.0 + npr * rng.uniform(-1, 1, k)
    et = (p + gamma * pinf) / ((gamma - 1.0) * rho) + 0.5 * (vel ** 2).sum(0)
    Q = np.empty((5, n))
    Q[0] = rho
    Q[1:4] = rho * vel
    Q[4] = rho * et
    return Q


def write_vtk(mesh: Mesh, path: str, params, Q: np.ndarray, tri_tag: np.ndarray | None = None) -> None:
    """VTK legacy solution file of the reference's VTK_Writer (Euler3D/src/MeshIO.cpp:219)
    for a mesh built with its cells (``with_cells=True``) and a state Q [5, nnode+nghost]."""
    if mesh.tets is None or mesh.tris is None:
        raise ValueError("write_vtk needs the mesh's cells (build it with with_cells=True)")
    Q = np.ascontiguousarray(Q, np.float64)
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    tris = np.ascontiguousarray(mesh.tris, np.int32)
    tets = np.ascontiguousarray(mesh.tets, np.int32)
    tag = None if tri_tag is None else np.ascontiguousarray(tri_tag, np.int32)
    capi.check(capi.lib.cfd_vtk_write(str(path).encode(), mesh.nnode, capi.ptr(coords), tris.shape[0], capi.ptr(tris),
                                      None if tag is None else capi.ptr(tag), tets.shape[0], capi.ptr(tets),
                                      C.byref(params), capi.ptr(Q), Q.shape[1]), "cfd_vtk_write")


def to_rup(Q: np.ndarray, gamma: float, pinf: float = 0.0) -> np.ndarray:
    """Conservative state SoA [5, n] -> (rho, u, v, w, p) (CFD_VARS_RUP;
    MPFLOW3D Material_Transformations, VARIABLE_CON -> VARIABLE_RUP), with
    p = (gamma - 1)(rho et - rho q^2 / 2) - gamma pinf."""
    Q = np.asarray(Q, np.float64)
    r = Q[0]
    u, v, w = Q[1] / r, Q[2] / r, Q[3] / r
    p = (gamma - 1.0) * (Q[4] - 0.5 * r * (u * u + v * v + w * w)) - gamma * pinf
    return np.stack([r, u, v, w, p])


def to_conservative(R: np.ndarray, gamma: float, pinf: float = 0.0) -> np.ndarray:
    """(rho, u, v, w, p) SoA [5, n] -> conservative, rho et = (p + gamma pinf) / (gamma - 1) + rho q^2 / 2."""
    r, u, v, w, p = np.asarray(R, np.float64)
    return np.stack([r, r * u, r * v, r * w, (p + gamma * pinf) / (gamma - 1.0) + 0.5 * r * (u * u + v * v + w * w)])
