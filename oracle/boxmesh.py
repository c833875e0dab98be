"""Tet-split box meshes and their median dual in numpy (test infrastructure).

Builds the same meshes as the library's ``cfd_mesh_box`` (Freudenthal split
of every hex into 6 positive tets sharing the v000 -> v111 diagonal, two
boundary triangles per face quad split through the quad's lowest corner) and
their median-dual metrics the way the reference's pre-processing defines them
(``Euler3D/src/Area_Volume.cpp``: per tet edge the two triangles mid-edge ->
face centroid -> tet centroid, oriented from the lower to the higher node
index; a quarter of each tet's volume per vertex; per boundary-triangle vertex
one boundary edge to a private ghost node with a third of the triangle's area
vector, the vertices in the reversed winding the reference's UGRID reader
gives, ``Euler3D/src/MeshIO.cpp:22-45``).  Vectorised over tets, so a 48^3
cube (663,552 tets) takes seconds.

It exists so that the reference arm of ``bench.py`` can build its sample mesh
without loading the CUDA library; ``tests/test_boxmesh.py`` checks it against
the library's builder.  The jitter draws its own numpy random numbers, so a
jittered mesh is the library's mesh only when the coordinates are passed in.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
_PAIRS = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
_OTHERS = ((2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1))


def _grid(n):
    return (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)


def box_cells(n, lengths=(1.0, 1.0, 1.0), jitter=0.0, seed=0, coords=None, face_bc=(1, 1, 1, 1, 1, 1)):
    """Coordinates [nnode, 3], tets [ntet, 4], boundary triangles [ntri, 3]
    (outward right-hand normals) and their BC types, in natural numbering."""
    nx, ny, nz = _grid(n)
    px, py, pz = nx + 1, ny + 1, nz + 1
    k, j, i = np.meshgrid(np.arange(pz), np.arange(py), np.arange(px), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    h = np.array([lengths[0] / nx, lengths[1] / ny, lengths[2] / nz])
    if coords is None:
        xyz = np.stack([i * h[0], j * h[1], k * h[2]], axis=1).astype(np.float64)
        interior = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
        rng = np.random.default_rng(seed)
        xyz[interior] += jitter * h * rng.uniform(-1.0, 1.0, (int(interior.sum()), 3))
    else:
        xyz = np.asarray(coords, np.float64).reshape(-1, 3)

    def nid(a, b, c):
        return a + px * (b + py * c)

    hk, hj, hi = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()
    tets = np.empty((hi.size, 6, 4), np.int64)
    for p, perm in enumerate(_PERMS):
        o = np.zeros((hi.size, 3), np.int64)
        tets[:, p, 0] = nid(hi, hj, hk)
        for s in range(3):
            o[:, perm[s]] = 1
            tets[:, p, s + 1] = nid(hi + o[:, 0], hj + o[:, 1], hk + o[:, 2])
        if p in (1, 2, 5):  # odd permutation: swap the last two for a positive volume
            tets[:, p, [2, 3]] = tets[:, p, [3, 2]]
    tets = tets.reshape(-1, 4)

    # boundary quads, per face position the low face's quad then the high
    # face's (the library's loop order), each split through its lowest corner
    parts = []
    fk, fj = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    fk, fj = fk.ravel(), fj.ravel()
    z0 = np.zeros_like(fj)
    parts.append(_face_pairs(
        np.stack([nid(z0, fj, fk), nid(z0, fj, fk + 1), nid(z0, fj + 1, fk + 1), nid(z0, fj + 1, fk)], 1),
        np.stack([nid(z0 + nx, fj, fk), nid(z0 + nx, fj + 1, fk), nid(z0 + nx, fj + 1, fk + 1),
                  nid(z0 + nx, fj, fk + 1)], 1), face_bc[0], face_bc[1]))
    fk, fi = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    fk, fi = fk.ravel(), fi.ravel()
    z0 = np.zeros_like(fi)
    parts.append(_face_pairs(
        np.stack([nid(fi, z0, fk), nid(fi + 1, z0, fk), nid(fi + 1, z0, fk + 1), nid(fi, z0, fk + 1)], 1),
        np.stack([nid(fi, z0 + ny, fk), nid(fi, z0 + ny, fk + 1), nid(fi + 1, z0 + ny, fk + 1),
                  nid(fi + 1, z0 + ny, fk)], 1), face_bc[2], face_bc[3]))
    fj, fi = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    fj, fi = fj.ravel(), fi.ravel()
    z0 = np.zeros_like(fi)
    parts.append(_face_pairs(
        np.stack([nid(fi, fj, z0), nid(fi, fj + 1, z0), nid(fi + 1, fj + 1, z0), nid(fi + 1, fj, z0)], 1),
        np.stack([nid(fi, fj, z0 + nz), nid(fi + 1, fj, z0 + nz), nid(fi + 1, fj + 1, z0 + nz),
                  nid(fi, fj + 1, z0 + nz)], 1), face_bc[4], face_bc[5]))
    tris = np.concatenate([t for t, _ in parts])
    tri_bc = np.concatenate([b for _, b in parts])
    return xyz, tets, tris, tri_bc


def _face_pairs(qa, qb, bca, bcb):
    """Triangles and BC types of two opposite faces' quads, interleaved
    (quad a-b-c-d counter-clockwise from outside -> a-b-c, a-c-d)."""
    m = qa.shape[0]
    q = np.empty((2 * m, 4), np.int64)
    q[0::2], q[1::2] = qa, qb
    bc = np.empty(2 * m, np.int32)
    bc[0::2], bc[1::2] = bca, bcb
    t = np.empty((2 * m, 2, 3), np.int64)
    t[:, 0] = q[:, [0, 1, 2]]
    t[:, 1] = q[:, [0, 2, 3]]
    return t.reshape(-1, 3), np.repeat(bc, 2)


def median_dual(xyz, tets, tris, tri_bc):
    """Median-dual metrics of a tet mesh: the arrays the reference keeps in
    intEdge / bndEdge / cVolume / coordXYZ / crs_*_Node2Node."""
    nnode = xyz.shape[0]
    pairs = np.array(_PAIRS)
    others = np.array(_OTHERS)
    a = tets[:, pairs[:, 0]]
    b = tets[:, pairs[:, 1]]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    keys = (lo * nnode + hi).ravel()
    ukeys = np.unique(keys)
    edge_nodes = np.stack([ukeys // nnode, ukeys % nnode], axis=1).astype(np.int32)
    eidx = np.searchsorted(ukeys, keys).reshape(-1, 6)
    x = xyz[tets]  # [ntet, 4, 3]
    g = x.mean(axis=1)
    vol = np.einsum("ij,ij->i", x[:, 1] - x[:, 0], np.cross(x[:, 2] - x[:, 0], x[:, 3] - x[:, 0])) / 6.0
    if not (vol > 0).all():
        raise ValueError("tetrahedra with non-positive volume")
    cvol = np.zeros(nnode)
    np.add.at(cvol, tets.ravel(), np.repeat(0.25 * np.abs(vol), 4))
    areav = np.zeros((ukeys.size, 3))
    for p in range(6):
        ia, ib = pairs[p]
        ic, id_ = others[p]
        mid = 0.5 * (x[:, ia] + x[:, ib])
        f1 = (x[:, ia] + x[:, ib] + x[:, ic]) / 3.0
        f2 = (x[:, ia] + x[:, ib] + x[:, id_]) / 3.0
        rg = g - mid
        S = 0.5 * (np.cross(f1 - mid, rg) + np.cross(rg, f2 - mid))
        ab = xyz[hi[:, p]] - xyz[lo[:, p]]
        sgn = np.where(np.einsum("ij,ij->i", S, ab) >= 0.0, 1.0, -1.0)
        np.add.at(areav, eidx[:, p], sgn[:, None] * S)
    # node graph (no diagonal), rows sorted
    both = np.concatenate([edge_nodes, edge_nodes[:, ::-1]])
    order = np.lexsort((both[:, 1], both[:, 0]))
    both = both[order]
    n2n_ia = np.zeros(nnode + 1, np.int32)
    np.add.at(n2n_ia, both[:, 0] + 1, 1)
    n2n_ia = np.cumsum(n2n_ia).astype(np.int32)
    n2n_ja = both[:, 1].astype(np.int32)
    # boundary edges: per triangle vertex (reversed winding), one ghost each
    e1 = xyz[tris[:, 1]] - xyz[tris[:, 0]]
    e2 = xyz[tris[:, 2]] - xyz[tris[:, 0]]
    nrm = np.cross(e1, e2) / 6.0
    ntri = tris.shape[0]
    nbedge = 3 * ntri
    bedge_nodes = np.empty((nbedge, 2), np.int32)
    bedge_nodes[:, 0] = tris[:, ::-1].ravel()
    bedge_nodes[:, 1] = nnode + np.arange(nbedge)
    bedge_areav = np.repeat(nrm, 3, axis=0)
    bedge_type = np.repeat(tri_bc, 3).astype(np.int32)
    return SimpleNamespace(nnode=nnode, nghost=nbedge, nedge=edge_nodes.shape[0], nbedge=nbedge,
                           edge_nodes=edge_nodes, edge_areav=areav, bedge_nodes=bedge_nodes,
                           bedge_areav=bedge_areav, bedge_type=bedge_type, cvol=cvol, coords=xyz.copy(),
                           n2n_ia=n2n_ia, n2n_ja=n2n_ja)


def box_mesh(n, lengths=(1.0, 1.0, 1.0), jitter=0.0, seed=0, rcm=False, coords=None,
             face_bc=(1, 1, 1, 1, 1, 1)):
    """Tet-split box and its median dual; ``rcm`` renumbers the nodes by
    reverse Cuthill-McKee (scipy's) before the dual is built."""
    xyz, tets, tris, tri_bc = box_cells(n, lengths, jitter, seed, coords, face_bc)
    if rcm:
        from scipy.sparse import coo_matrix
        from scipy.sparse.csgraph import reverse_cuthill_mckee
        nnode = xyz.shape[0]
        pairs = np.array(_PAIRS)
        r = tets[:, pairs[:, 0]].ravel()
        c = tets[:, pairs[:, 1]].ravel()
        g = coo_matrix((np.ones(r.size), (r, c)), shape=(nnode, nnode)).tocsr()
        g = (g + g.T).tocsr()
        perm = reverse_cuthill_mckee(g, symmetric_mode=True)  # perm[new] = old
        inv = np.empty(nnode, np.int64)
        inv[perm] = np.arange(nnode)
        xyz, tets, tris = xyz[perm], inv[tets], inv[tris]
    return median_dual(xyz, tets, tris, tri_bc)


def perturbed_freestream(mesh, gamma, mach, alpha_deg, beta_deg=0.0, noise=0.01, seed=0):
    """Conservative SoA state [5][nnode + nghost] of the generic
    non-dimensional freestream (rho = 1, p = 1, c = sqrt(gamma)) with every
    physical node's components scaled by (1 + U(-noise, noise))."""
    a, b = np.radians(alpha_deg), np.radians(beta_deg)
    c = np.sqrt(gamma)
    u = mach * c * np.cos(a) * np.cos(b)
    v = mach * c * np.sin(a) * np.cos(b)
    w = mach * c * np.sin(b)
    et = 1.0 / (gamma - 1.0) + 0.5 * (u * u + v * v + w * w)
    q = np.array([1.0, u, v, w, et])
    n = mesh.nnode + mesh.nghost
    Q = np.repeat(q[:, None], n, axis=1)
    rng = np.random.default_rng(seed)
    Q[:, :mesh.nnode] *= 1.0 + rng.uniform(-noise, noise, (5, mesh.nnode))
    return Q
