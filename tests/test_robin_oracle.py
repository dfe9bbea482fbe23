"""Oracle restatement of the Robin (port) boundary term against the golden
fixture made by the reference's own code (tests/golden/make_golden_robin.py),
and the host-side surface selection. Tolerance 1e-13 relative (max entry)."""
import numpy as np

from emerge_b200 import workloads as W
from oracle import oracle as O
from tests.golden_util import load_npz

TOL = 1e-13


def test_single_triangles_match_reference():
    g = load_npz("robin.npz")
    for X, gam, B in zip(g["tri_X"], g["tri_gamma"], g["tri_B"]):
        mine = O.tri_stiff(X, gam)
        assert np.abs(mine - B).max() <= TOL * np.abs(B).max()
        assert np.array_equal(mine, mine.T)  # the reference's blocks are exactly symmetric too
        assert np.array_equal(B, B.T)


def test_port_faces_match_reference():
    g = load_npz("robin.npz")
    wl = W.wr90_air()
    ids = W.port_tris(wl)
    assert np.array_equal(ids, g["port_ids"])
    assert abs(W.rect_port_gamma(wl.freq) - complex(g["port_gamma"])) <= 1e-12 * abs(complex(g["port_gamma"]))
    Bmat = O.robin_entries(wl.field, ids, complex(g["port_gamma"]))
    mine = Bmat.reshape(-1, 64)[ids]
    assert np.abs(mine - g["port_B"]).max() <= TOL * np.abs(g["port_B"]).max()
    # every other tri slot stays zero
    others = np.setdiff1d(np.arange(wl.field.mesh.n_tris), ids)
    assert not np.any(Bmat.reshape(-1, 64)[others])


def test_robin_csc_lies_in_the_volume_pattern():
    """Every port DoF pair shares a tet, so K + Robin keeps A's pattern."""
    wl = W.wr90_air(n=(6, 4, 10))
    f = wl.field
    ids = W.port_tris(wl)
    R = O.generate_csc(f, O.robin_entries(f, ids, W.rect_port_gamma(wl.freq)))
    _, _, cmap = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    from scipy.sparse import csc_matrix

    A = csc_matrix((np.ones(cmap.nnz), cmap.indices, cmap.indptr), shape=(f.n_field, f.n_field))
    S = (A + abs(R)).tocsc()
    S.sum_duplicates()
    assert S.nnz == cmap.nnz
    assert R.nnz > 0 and np.array_equal(np.sort(ids), np.unique(ids))


def test_force_single_triangles_match_reference():
    g = load_npz("robin.npz")
    for X, U, fref in zip(g["tri_X"], g["tri_U"], g["tri_f"]):
        mine = O.tri_force(X, U)
        assert np.abs(mine - fref).max() <= TOL * np.abs(fref).max()


def test_force_on_port_faces_matches_reference():
    g = load_npz("robin.npz")
    wl = W.wr90_air()
    ids = g["port_ids"]
    pts = O.tri_points(wl.field, ids)
    assert np.abs(pts - g["port_pts"]).max() <= 1e-15 * np.abs(pts).max()
    U = np.zeros(pts.shape, np.complex128)
    U[1] = (1 + 0.5j) * np.sin(np.pi * g["port_pts"][0] / W.WR90[0])
    b = O.force_entries(wl.field, ids, U)
    ref = g["port_b"]
    assert np.abs(b - ref).max() <= TOL * np.abs(ref).max()
    assert np.count_nonzero(ref) > 0
