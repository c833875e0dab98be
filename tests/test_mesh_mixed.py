"""Mixed-element meshes: the library's UGRID reader and median-dual builder
(cfd_mesh_read_ugrid) against the reference's own pre-processing
(UGrid_Reader -> Create_Connectivity_Maps -> Calculate_Area_Volume,
Euler3D/main.cpp:121-128, compiled from its sources) on meshes of
tetrahedra, pyramids, prisms and hexahedra with boundary triangles and
quadrilaterals: the same edges, area vectors and control volumes to
round-off, the same boundary edges in the same order, the same node graph."""
import numpy as np
import pytest

from cfdsolutions_b200.mesh import read_ugrid
from oracle import refharness
from tests import _mixed


def _compare(m, r):
    assert r["nnode"] == m.nnode and r["nghost"] == m.nghost
    mine = {tuple(e): a for e, a in zip(m.edge_nodes.reshape(-1, 2).tolist(), m.edge_areav.reshape(-1, 3))}
    ref = {tuple(e): a for e, a in zip(r["edge_nodes"].tolist(), r["edge_areav"])}
    assert set(mine) == set(ref)
    scale = np.abs(m.edge_areav).max()
    assert max(np.abs(mine[k] - ref[k]).max() for k in mine) <= 1e-13 * scale
    np.testing.assert_allclose(m.cvol, r["cvol"], rtol=1e-13, atol=0)
    np.testing.assert_array_equal(m.bedge_nodes.reshape(-1, 2), r["bedge_nodes"])
    np.testing.assert_allclose(m.bedge_areav.reshape(-1, 3), r["bedge_areav"], rtol=0,
                               atol=1e-13 * np.abs(r["bedge_areav"]).max())
    for i in range(m.nnode):
        assert set(m.n2n_ja[m.n2n_ia[i]:m.n2n_ia[i + 1]].tolist()) == \
            set(r["n2n_ja"][r["n2n_ia"][i]:r["n2n_ia"][i + 1]].tolist())


@pytest.mark.parametrize("kinds", [(_mixed.HEX,), (_mixed.PRISMS,), (_mixed.PYRAMIDS,), (_mixed.TETS,),
                                   (_mixed.HEX, _mixed.PRISMS, _mixed.PYRAMIDS, _mixed.TETS)],
                         ids=["hex", "prism", "pyramid", "tet", "all"])
def test_mixed_mesh_matches_reference_preprocessing(tmp_path, ref_available, kinds):
    cells = _mixed.mixed_box((3, 3, 2), jitter=0.15, seed=5, kinds=kinds)
    path = tmp_path / "mixed.ugrid"
    _mixed.write_ugrid(path, *cells)
    m = read_ugrid(str(path))
    r = refharness.mesh_from_ugrid(str(path))
    _compare(m, r)


def test_conforming_hex_pyramid_mesh_closes_every_dual_cell(tmp_path):
    """Hexahedra and pyramid-split hexahedra keep their quadrilateral faces:
    every dual cell's faces sum to zero and the volumes add up to the box."""
    cells = _mixed.mixed_box((4, 3, 3), jitter=0.15, seed=8, kinds=(_mixed.HEX, _mixed.PYRAMIDS))
    path = tmp_path / "hexpyr.ugrid"
    _mixed.write_ugrid(path, *cells)
    m = read_ugrid(str(path))
    en, ea = m.edge_nodes.reshape(-1, 2), m.edge_areav.reshape(-1, 3)
    bn, ba = m.bedge_nodes.reshape(-1, 2), m.bedge_areav.reshape(-1, 3)
    s = np.zeros((m.nnode, 3))
    np.add.at(s, en[:, 0], ea)
    np.add.at(s, en[:, 1], -ea)
    np.add.at(s, bn[:, 0], ba)
    assert np.abs(s).max() <= 1e-14
    assert abs(m.cvol.sum() - 1.0) <= 1e-13
    assert (m.cvol > 0).all()


def test_ugrid_boundary_tags_map_to_bc_types(tmp_path):
    cells = _mixed.mixed_box((2, 2, 2), jitter=0.1, seed=1, kinds=(_mixed.HEX,))
    coords, tets, pyrs, prisms, hexes, tris, quads = cells
    tags = 1 + (np.arange(len(quads)) % 3)
    path = tmp_path / "tags.ugrid"
    _mixed.write_ugrid(path, *cells, quad_tag=tags)
    m = read_ugrid(str(path), bc_types=[1, 2, 3])
    np.testing.assert_array_equal(m.bedge_type, np.repeat(tags, 4))
