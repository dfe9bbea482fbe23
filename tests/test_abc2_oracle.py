"""Oracle restatement of the second-order absorbing boundary correction
(robin_abc_order2.py) against the reference's own output
(tests/golden/abc2.npz, made by tests/golden/make_golden_abc2.py): single
triangles of mixed scales and orientations, and the matrix builder over three
faces of the 12x6x30 WR-90 box. Tolerance 1e-12 relative (max entry)."""
import numpy as np

from emerge_b200 import workloads as W
from oracle import oracle as O
from tests.golden_util import load_npz


def test_single_triangles_match_reference():
    g = load_npz("abc2.npz")
    for X, cf, B in zip(g["tri_X"], g["tri_cf"], g["tri_B"]):
        mine = O.abc2_block(X, cf)
        assert np.abs(mine - B).max() <= 1e-12 * np.abs(B).max()
        assert np.array_equal(mine, mine.T)  # products commute: bitwise symmetric


def test_matrix_builder_matches_reference():
    g = load_npz("abc2.npz")
    wl = W.wr90_air()
    f = wl.field
    Mat = O.abc2_entries(f, g["abc_ids"], complex(g["abc_cf"]))
    mine = Mat.reshape(-1, 64)[g["abc_ids"]]
    assert np.abs(mine - g["abc_B"]).max() <= 1e-12 * np.abs(g["abc_B"]).max()
    # a triangle listed twice counts twice, like the reference's +=
    ids2 = np.concatenate([g["abc_ids"][:5], g["abc_ids"][:5]])
    M2 = O.abc2_entries(f, ids2, 1.0).reshape(-1, 64)
    M1 = O.abc2_entries(f, g["abc_ids"][:5], 1.0).reshape(-1, 64)
    assert np.array_equal(M2, 2 * M1)
