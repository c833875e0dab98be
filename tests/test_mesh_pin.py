"""Pins the project's median-dual builder against the reference's own
pre-processing: the mesh is written as UGRID, read back by the reference's
UGrid_Reader -> Create_Connectivity_Maps -> Calculate_Area_Volume
(Euler3D/main.cpp:121-128), and every array is compared."""
import numpy as np
import pytest

from cfdsolutions_b200 import box_mesh
from oracle import refharness


@pytest.mark.parametrize("n,seed", [(3, 7), (6, 9)])
def test_builder_matches_reference_preprocessing(tmp_path, ref_available, n, seed):
    path = tmp_path / f"box{n}.ugrid"
    m = box_mesh(n, jitter=0.15, seed=seed, ugrid_path=str(path))
    r = refharness.mesh_from_ugrid(str(path))
    assert r["nnode"] == m.nnode and r["nghost"] == m.nghost
    mine = {tuple(e): a for e, a in zip(m.edge_nodes.tolist(), m.edge_areav)}
    ref = {tuple(e): a for e, a in zip(r["edge_nodes"].tolist(), r["edge_areav"])}
    assert set(mine) == set(ref)
    scale = np.abs(m.edge_areav).max()
    assert max(np.abs(mine[k] - ref[k]).max() for k in mine) <= 1e-13 * scale
    np.testing.assert_allclose(m.cvol, r["cvol"], rtol=1e-13, atol=0)
    np.testing.assert_array_equal(m.bedge_nodes, r["bedge_nodes"])
    np.testing.assert_allclose(m.bedge_areav, r["bedge_areav"], rtol=0, atol=1e-13 * np.abs(m.bedge_areav).max())
    for i in range(m.nnode):
        a = set(m.n2n_ja[m.n2n_ia[i]:m.n2n_ia[i + 1]].tolist())
        b = set(r["n2n_ja"][r["n2n_ia"][i]:r["n2n_ia"][i + 1]].tolist())
        assert a == b
