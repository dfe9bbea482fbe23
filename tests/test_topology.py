"""Vectorised host topology (emerge_b200.mesh) against the loop restatement
of Mesh3D._pre_update / Nedelec2 (mesh3d.py:706-776, nedelec2.py:61-79)."""
import numpy as np
import pytest

from emerge_b200.mesh import Nedelec2Field, TetMesh, structured_box, tet_signed_volumes
from oracle.oracle import topology_loops


@pytest.mark.parametrize("n,seed", [((1, 1, 1), 0), ((2, 3, 2), 1), ((3, 2, 4), 2)])
def test_topology_matches_reference_rules(n, seed):
    nodes, tets = structured_box(*n, jitter=0.1, seed=seed)
    rng = np.random.default_rng(seed)
    tets = tets[:, rng.permutation(tets.shape[1])]  # arbitrary tet order
    m = TetMesh(nodes, tets)
    f = Nedelec2Field(m)
    edges, tris, t2e, t2t, t2f = topology_loops(tets)
    assert np.array_equal(m.edges, edges) and np.array_equal(m.tris, tris)
    assert np.array_equal(m.tet_to_edge, t2e) and np.array_equal(m.tet_to_tri, t2t)
    assert np.array_equal(f.get_tet_to_field(), t2f)
    assert f.n_field == 2 * edges.shape[1] + 2 * tris.shape[1]


def test_config0_sizes_and_orientation():
    nodes, tets = structured_box(12, 6, 30)
    m = TetMesh(nodes, tets)
    assert (m.n_nodes, m.n_tets, m.n_edges, m.n_tris) == (2821, 12960, 17004, 27144)
    assert Nedelec2Field(m).n_field == 88296
    assert (tet_signed_volumes(nodes, tets) > 0).all()


def test_bad_input_rejected():
    nodes, tets = structured_box(1, 1, 1)
    bad = tets.copy()
    bad[0, 0] = nodes.shape[1]
    with pytest.raises(ValueError):
        TetMesh(nodes, bad)
    with pytest.raises(ValueError):
        TetMesh(nodes[:2], tets)
