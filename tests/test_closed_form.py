"""The closed-form element tables (emerge_b200/csrc/gen_tables.py) reproduce
the reference's 11-point KEAST4 element matrices, checked against the golden
fixtures of the reference's ned2_tet_stiff_mass (through _matrix_builder)."""
import os
import sys

import numpy as np
import pytest

from tests.golden_util import field_from, load_npz

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "emerge_b200", "csrc"))
import gen_tables as gt  # noqa: E402

IDSET1 = [(0, 1), (0, 2), (0, 3), (1, 2), (3, 1), (2, 3)]
IDSET2 = [(0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 2, 3)]
MASS, STIFF = gt.tables()


def matinv(M):
    off = [M[0, 1], M[0, 2], M[1, 0], M[1, 2], M[2, 0], M[2, 1]]
    if all(v == 0 for v in off):
        return np.diag([1 / M[0, 0], 1 / M[1, 1], 1 / M[2, 2]])
    return np.linalg.inv(M)


def closed_form(X, gid, Ms, Mm):
    order = np.argsort(gid)
    rank = np.argsort(order)
    Jo = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=1)
    det = np.linalg.det(Jo)
    gl = np.zeros((4, 3))
    gl[1:] = np.linalg.inv(Jo)
    gl[0] = -gl[1:].sum(0)
    g = gl[order]
    sig, V = np.sign(det), abs(det) / 6
    Xc = [np.cross(g[a], g[b]) for a, b in gt.EDGES]
    G = np.array([[(Mm @ g[m]) @ g[n] for n in range(4)] for m in range(4)])
    H = np.array([[(Ms @ Xc[p]) @ Xc[q] for q in range(6)] for p in range(6)])
    kap = [gt.EDGES.index(tuple(sorted([rank[u], rank[v]]))) for u, v in IDSET1]
    kap = kap + [6 + k for k in kap]
    kf = [gt.FACES.index(tuple(sorted(rank[list(t)]))) for t in IDSET2]
    kap += [12 + k for k in kf] + [16 + k for k in kf]
    K = np.zeros((20, 20), complex)
    M = np.zeros((20, 20), complex)
    for a in range(20):
        for b in range(a, 20):
            x, y = kap[a], kap[b]
            s = (sig if gt.ODD[x] else 1) * (sig if gt.ODD[y] else 1)
            K[a, b] = K[b, a] = V * s * sum(float(c) * H[p][q] for p, q, c in STIFF[(x, y)])
            M[a, b] = M[b, a] = V * s * sum(float(c) * G[m][n] for m, n, c in MASS[(x, y)])
    return K, M


@pytest.mark.parametrize("name", ["tiny.npz", "small_diag.npz"])
def test_closed_form_equals_reference_quadrature(name):
    g = load_npz(name)
    f = field_from(g["nodes"], g["tets"])
    nT = g["tets"].shape[1]
    assy = np.delete(np.arange(nT), g["conductor_tets"]) if g["conductor_tets"].size else np.arange(nT)
    dE = g["dataE"].reshape(-1, 20, 20)
    dB = g["dataB"].reshape(-1, 20, 20)
    for ia, it in enumerate(assy):
        v = f.mesh.tets[:, it]
        K, M = closed_form(f.mesh.nodes[:, v], v, matinv(g["ur"][:, :, it]), g["er"][:, :, it])
        assert np.abs(K - dE[ia]).max() <= 1e-12 * np.abs(dE[ia]).max()
        assert np.abs(M - dB[ia]).max() <= 1e-12 * np.abs(dB[ia]).max()


def test_table_structure():
    # every ordered pair has at most 4 mass and 9 stiffness terms; M symmetric in (x, y) transposition
    assert max(len(v) for v in MASS.values()) <= 4
    assert max(len(v) for v in STIFF.values()) <= 9
    for (x, y), terms in MASS.items():
        assert sorted((n, m, c) for m, n, c in terms) == MASS[(y, x)]


def test_generated_header_is_current(tmp_path):
    out = tmp_path / "t.cuh"
    gt.emit_header(str(out))
    committed = os.path.join(os.path.dirname(gt.__file__), "nedelec_tables.cuh")
    assert out.read_text() == open(committed).read()
