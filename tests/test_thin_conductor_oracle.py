"""ThinConductor (partitioned field) host side, against the fixture the
reference's own Nedelec2.partition_dof and assembler chain made
(tests/golden/make_golden_thin.py):

* the DoF split restated in ``Nedelec2Field.partition_dof`` equals the
  reference's (n_field, tet_to_field, tri_to_field_os, edge_to_field_os, and
  get_tet_to_field() keeps the unsplit map);
* ``TetMesh.tri_to_tet`` follows the reference's rule;
* the oracle chain (volume + Robin + opposite-side generate_csc) equals the
  reference's final K;
* ``OppositeSideTerm.pairs`` spans the reference's other-side pattern.
"""
import numpy as np
import pytest

from emerge_b200.mesh import MISSING_ID, DoFSplitError, Nedelec2Field, TetMesh, grid_level_tris
from emerge_b200.thin_conductor import OppositeSideTerm
from oracle import oracle as O
from tests.golden_util import load_npz

G = load_npz("thin.npz")


def _field():
    f = Nedelec2Field(TetMesh(G["nodes"], G["tets"]))
    f.partition_dof([(G["strip0"], G["normal0"]), (G["strip1"], G["normal1"])])
    return f


def test_partition_matches_reference():
    f = _field()
    assert f.n_field == int(G["n_field"]) > int(G["n_field0"])
    assert np.array_equal(f.tet_to_field, G["tet_to_field"])
    assert np.array_equal(f.tri_to_field_os, G["tri_to_field_os"])
    assert np.array_equal(f.edge_to_field_os, G["edge_to_field_os"])
    assert np.array_equal(f.get_tet_to_field(), G["tet_to_field_orig"])
    # the split moved some tets, and a second call changes nothing
    assert not np.array_equal(f.tet_to_field, f.get_tet_to_field())
    n = f.n_field
    f.partition_dof([(G["strip0"], G["normal0"])])
    assert f.n_field == n


def test_tri_to_tet_rule():
    m = TetMesh(G["nodes"], G["tets"])
    t2t = m.tri_to_tet
    want = np.full((2, m.n_tris), MISSING_ID)
    for tet in range(m.n_tets):
        for tri in m.tet_to_tri[:, tet]:
            want[0 if want[0, tri] == MISSING_ID else 1, tri] = tet
    assert np.array_equal(t2t, want)
    assert np.all(t2t[0] >= 0) and np.all((t2t[1] == MISSING_ID) | (t2t[1] > t2t[0]))


def test_exterior_surface_refused():
    f = Nedelec2Field(TetMesh(G["nodes"], G["tets"]))
    with pytest.raises(DoFSplitError):
        f.partition_dof([(G["port"], np.array([0.0, 0.0, 1.0]))])


def test_edge_split_rule_and_numbering():
    f = _field()
    m = f.mesh
    E, F, n0 = m.n_edges, m.n_tris, int(G["n_field0"])
    se, st = f.split_edges, f.split_tris
    # an edge splits when exactly two triangles of one strip hold it
    want = set()
    for s in (G["strip0"], G["strip1"]):
        c = np.bincount(m.tri_to_edge[:, s].ravel(), minlength=E)
        want |= set(np.flatnonzero(c == 2).tolist())
    assert set(se.tolist()) == want
    assert np.array_equal(st, np.unique(np.concatenate([G["strip0"], G["strip1"]])))
    # new numbers follow the old ones: edges (both DoFs), then faces
    ne, nf = se.size, st.size
    assert np.array_equal(f.edge_to_field_os[0, se], n0 + np.arange(ne))
    assert np.array_equal(f.edge_to_field_os[1, se], n0 + ne + np.arange(ne))
    assert np.array_equal(f.tri_to_field_os[6, st], n0 + 2 * ne + np.arange(nf))
    assert np.array_equal(f.tri_to_field_os[7, st], n0 + 2 * ne + nf + np.arange(nf))
    assert f.n_field == n0 + 2 * ne + 2 * nf and n0 == 2 * E + 2 * F


def _oracle_K(f):
    k0 = float(G["k0"])
    dE, dB, pat = O.tet_mass_stiffness_matrices(f, G["er"], G["ur"], np.zeros(0, np.int64))
    assert pat.N == f.n_field
    K = pat.to_csc(dE - dB * k0 ** 2)
    B1 = O.robin_entries(f, G["port"], complex(G["g_port"]))
    B2 = np.zeros_like(B1)
    for s, g in zip((G["strip0"], G["strip1"]), G["g_tc"]):
        B1 = O.robin_entries(f, s, complex(g), B1)
        B2 = O.robin_entries(f, s, complex(g), B2)
    K = K + O.generate_csc(f, B1)
    OS = O.generate_csc(f, B2, O.tri_rowcol(f, other_side=True))
    return (K + OS).tocsc(), OS.tocsc()


def test_oracle_chain_matches_reference_K():
    f = _field()
    K, OS = _oracle_K(f)
    for got, pre in ((K, "K"), (OS, "os")):
        assert np.array_equal(got.indptr, G[f"{pre}_indptr"])
        assert np.array_equal(got.indices, G[f"{pre}_indices"])
        want = G[f"{pre}_data"]
        err = np.abs(got.data - want).max() / np.abs(want).max()
        assert err <= 1e-12, (pre, err)


def test_opposite_pairs_span_reference_pattern():
    f = _field()
    T0, T1 = OppositeSideTerm(f, G["strip0"]), OppositeSideTerm(f, G["strip1"])
    pairs = set()
    for T in (T0, T1):
        r, c = T.pairs()
        pairs |= set(zip(c.tolist(), r.tolist()))
    ip, ix = G["os_indptr"], G["os_indices"]
    ref = {(c, int(ix[p])) for c in range(ip.size - 1) for p in range(ip[c], ip[c + 1])}
    assert ref <= pairs  # generate_csc drops exact zeros only
    # the new DoFs appear only in the other-side term
    n0 = int(G["n_field0"])
    assert any(c >= n0 for c, _ in ref) and any(r >= n0 for _, r in ref)


def test_opposite_term_needs_partitioned_field():
    f = Nedelec2Field(TetMesh(G["nodes"], G["tets"]))
    with pytest.raises(ValueError, match="partition_dof"):
        OppositeSideTerm(f, G["strip0"])
    m = f.mesh
    assert np.array_equal(grid_level_tris(m, tuple(G["dims"]), 2, 2, (0, 0, 0), (3, 2, 5)), G["strip0"])
