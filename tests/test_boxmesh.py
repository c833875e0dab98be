"""The oracle's numpy box-mesh builder (oracle/boxmesh.py, used by the
reference arm of bench.py so that it needs no CUDA library) builds the
library's meshes: same edges, boundary edges and node graph, area vectors
and control volumes to round-off."""
import numpy as np
import pytest

from cfdsolutions_b200 import box_mesh
from oracle import boxmesh


@pytest.mark.parametrize("n", [3, (4, 3, 2), 6])
def test_numpy_box_mesh_equals_library_mesh(n):
    m = box_mesh(n, jitter=0.15, seed=5)
    o = boxmesh.box_mesh(n, coords=m.coords)
    assert (o.nnode, o.nedge, o.nbedge, o.nghost) == (m.nnode, m.nedge, m.nbedge, m.nghost)
    assert np.array_equal(o.edge_nodes, m.edge_nodes.reshape(-1, 2))
    assert np.abs(o.edge_areav - m.edge_areav.reshape(-1, 3)).max() <= 1e-15
    assert np.abs(o.cvol - m.cvol).max() <= 1e-15
    assert np.array_equal(o.bedge_nodes, m.bedge_nodes.reshape(-1, 2))
    assert np.abs(o.bedge_areav - m.bedge_areav.reshape(-1, 3)).max() <= 1e-15
    assert np.array_equal(o.bedge_type, m.bedge_type)
    assert np.array_equal(o.n2n_ia, m.n2n_ia) and np.array_equal(o.n2n_ja, m.n2n_ja)


def test_numpy_box_mesh_closes_every_dual_cell():
    """Each dual cell's faces sum to zero (Area_Volume.cpp:861-899), with RCM
    numbering and jitter; volumes add up to the box."""
    o = boxmesh.box_mesh(5, jitter=0.15, seed=2, rcm=True)
    s = np.zeros((o.nnode, 3))
    np.add.at(s, o.edge_nodes[:, 0], o.edge_areav)
    np.add.at(s, o.edge_nodes[:, 1], -o.edge_areav)
    np.add.at(s, o.bedge_nodes[:, 0], o.bedge_areav)
    assert np.abs(s).max() <= 1e-14
    assert abs(o.cvol.sum() - 1.0) <= 1e-13
