"""Mixed-element test meshes written as UGRID files.

A box of nx*ny*nz hexahedra, interior nodes jittered, each hex kept or split
by a pattern: a hexahedron; two prisms (split through the vertical diagonal
plane (i,j)-(i+1,j+1)); six pyramids on the hex faces with a new apex at the
hex centre; six tetrahedra (the Freudenthal split of the box meshes).  Hexes
and pyramid-split hexes keep their quadrilateral faces, so a mesh of those two
kinds is conforming; prisms and tets put diagonals on their faces, which a
neighbouring quadrilateral does not have (the median dual is still defined
cell by cell, which is what the pin against the reference compares).
Boundary faces: the box faces of each boundary cell, as that cell's split
leaves them (quadrilaterals, or two triangles), outward right-hand normal.
"""
from __future__ import annotations

import numpy as np

HEX, PRISMS, PYRAMIDS, TETS = 0, 1, 2, 3


def mixed_box(n=(3, 3, 3), jitter=0.15, seed=3, kinds=(HEX, PRISMS, PYRAMIDS, TETS)):
    nx, ny, nz = n
    px, py, pz = nx + 1, ny + 1, nz + 1
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(pz), np.arange(py), np.arange(px), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    h = np.array([1.0 / nx, 1.0 / ny, 1.0 / nz])
    xyz = np.stack([i * h[0], j * h[1], k * h[2]], 1).astype(np.float64)
    inner = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    xyz[inner] += jitter * h * rng.uniform(-1, 1, (int(inner.sum()), 3))
    coords = list(map(tuple, xyz))

    def nid(a, b, c):
        return a + px * (b + py * c)

    tets, pyrs, prisms, hexes, tris, quads = [], [], [], [], [], []
    perms = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
    for c in range(nz):
        for b in range(ny):
            for a in range(nx):
                kind = kinds[(a + 2 * b + 3 * c) % len(kinds)]
                v = [nid(a, b, c), nid(a + 1, b, c), nid(a + 1, b + 1, c), nid(a, b + 1, c),
                     nid(a, b, c + 1), nid(a + 1, b, c + 1), nid(a + 1, b + 1, c + 1), nid(a, b + 1, c + 1)]
                # outward faces of the hex (counter-clockwise seen from outside)
                faces = {"z0": (v[0], v[3], v[2], v[1]), "z1": (v[4], v[5], v[6], v[7]),
                         "y0": (v[0], v[1], v[5], v[4]), "y1": (v[2], v[3], v[7], v[6]),
                         "x0": (v[3], v[0], v[4], v[7]), "x1": (v[1], v[2], v[6], v[5])}
                on = {"x0": a == 0, "x1": a == nx - 1, "y0": b == 0, "y1": b == ny - 1, "z0": c == 0,
                      "z1": c == nz - 1}
                if kind == HEX:
                    hexes.append(v)
                elif kind == PRISMS:
                    prisms.append([v[0], v[1], v[2], v[4], v[5], v[6]])
                    prisms.append([v[0], v[2], v[3], v[4], v[6], v[7]])
                elif kind == PYRAMIDS:
                    g = tuple(np.mean([coords[t] for t in v], axis=0))
                    coords.append(g)
                    apex = len(coords) - 1
                    for f in faces.values():
                        pyrs.append([f[3], f[2], f[1], f[0], apex])  # base normal towards the apex
                else:
                    for p, perm in enumerate(perms):
                        o = [0, 0, 0]
                        t = [nid(a, b, c)]
                        for s in range(3):
                            o[perm[s]] = 1
                            t.append(nid(a + o[0], b + o[1], c + o[2]))
                        if p in (1, 2, 5):
                            t[2], t[3] = t[3], t[2]
                        tets.append(t)
                for name, f in faces.items():
                    if not on[name]:
                        continue
                    if kind == TETS or (kind == PRISMS and name in ("z0", "z1")):
                        # split through the face's lowest node (tets) / along the prisms' diagonal
                        lo = int(np.argmin(f)) if kind == TETS else f.index(v[0] if name == "z0" else v[4])
                        q = f[lo:] + f[:lo]
                        tris += [[q[0], q[1], q[2]], [q[0], q[2], q[3]]]
                    else:
                        quads.append(list(f))
    return (np.array(coords), np.array(tets, int).reshape(-1, 4), np.array(pyrs, int).reshape(-1, 5),
            np.array(prisms, int).reshape(-1, 6), np.array(hexes, int).reshape(-1, 8),
            np.array(tris, int).reshape(-1, 3), np.array(quads, int).reshape(-1, 4))


_PYR_TO_FILE = (0, 3, 4, 1, 2)  # file[k] = internal[_PYR_TO_FILE[k]] (the reader's translation inverted)


def write_ugrid(path, coords, tets, pyrs, prisms, hexes, tris, quads, tri_tag=None, quad_tag=None):
    with open(path, "w") as f:
        f.write(f"{len(coords)} {len(tris)} {len(quads)} {len(tets)} {len(pyrs)} {len(prisms)} {len(hexes)}\n")
        for x in coords:
            f.write("%.17g %.17g %.17g\n" % (x[0], x[1], x[2]))
        for t in tris:
            f.write(" ".join(str(v + 1) for v in t) + "\n")
        for q in quads:
            f.write(" ".join(str(v + 1) for v in q) + "\n")
        for k in range(len(tris)):
            f.write(f"{1 if tri_tag is None else tri_tag[k]}\n")
        for k in range(len(quads)):
            f.write(f"{1 if quad_tag is None else quad_tag[k]}\n")
        for t in tets:
            f.write(" ".join(str(v + 1) for v in t) + "\n")
        for p in pyrs:
            f.write(" ".join(str(p[_PYR_TO_FILE[k]] + 1) for k in range(5)) + "\n")
        for p in prisms:
            f.write(" ".join(str(v + 1) for v in p) + "\n")
        for hx in hexes:
            f.write(" ".join(str(v + 1) for v in hx) + "\n")
