"""Oracle restatement of the heat-conduction Lagrange-2 assembly (stiffness
and mass element matrices, COO layout, CSC pattern) against the golden
fixture made by the reference's own code (tests/golden/make_golden_heat.py).
Tolerance 1e-12 relative (max entry); pattern bit-exact."""
import numpy as np

from emerge_b200.mesh import TetMesh, structured_box
from oracle import oracle as O
from tests.golden_util import load_npz, rel_err


def heat_mesh():
    nodes, tets = structured_box(6, 4, 10, jitter=0.1, seed=13)
    m = TetMesh(nodes, tets)
    return m, np.concatenate([m.tets, m.tet_to_edge + m.n_nodes])


def test_leg2_values_and_pattern_match_reference():
    g = load_npz("heat.npz")
    m, t2f = heat_mesh()
    rows, cols = O.leg2_rowcol(t2f)
    assert np.array_equal(rows, g["rows"]) and np.array_equal(cols, g["cols"])
    K = O.leg2_values(m, g["cond"], "stiff")
    M = O.leg2_values(m, g["rho_cp"], "mass")
    for mine, ref in ((K, g["K"]), (M, g["M"])):
        fro, mx = rel_err(mine, ref)
        assert fro <= 1e-12 and mx <= 1e-12, (fro, mx)
    pat = O.CSCPattern.from_rowcol(rows, cols, int(g["N"]))
    assert np.array_equal(pat.indptr, g["indptr"]) and np.array_equal(pat.indices, g["indices"])
    fro, mx = rel_err(pat.values(K.astype(np.complex128)).real, g["Kdata"])
    assert fro <= 1e-12 and mx <= 1e-12
    assert np.array_equal(pat.values_f8(K), pat.values(K.astype(np.complex128)).real)
