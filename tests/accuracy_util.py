"""80-bit (long double) evaluation of the Nedelec-2 element integrals, used as
the near-exact yardstick for accuracy checks: exact closed-form integrals
(gen_tables) on edge-vector geometry, 64-bit mantissa arithmetic."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "emerge_b200", "csrc"))
import gen_tables as gt  # noqa: E402

IDSET1 = [(0, 1), (0, 2), (0, 3), (1, 2), (3, 1), (2, 3)]
IDSET2 = [(0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 2, 3)]
_MASS, _STIFF = gt.tables()
_LD = {}


def _c(c):
    if c not in _LD:
        _LD[c] = np.longdouble(c.numerator) / np.longdouble(c.denominator)
    return _LD[c]


def matinv(M):
    off = [M[0, 1], M[0, 2], M[1, 0], M[1, 2], M[2, 0], M[2, 1]]
    if all(v == 0 for v in off):
        return np.diag([1 / M[0, 0], 1 / M[1, 1], 1 / M[2, 2]])
    return np.linalg.inv(M)


def element_ld(X, gid, Ms, Mm):
    """(K, M) 20x20 in the reference DoF order, clongdouble."""
    X = np.asarray(X).astype(np.longdouble)
    order = np.argsort(gid)
    rank = np.argsort(order)
    e = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=1)
    c23, c31, c12 = np.cross(e[:, 1], e[:, 2]), np.cross(e[:, 2], e[:, 0]), np.cross(e[:, 0], e[:, 1])
    det = e[:, 0] @ c23
    gl = np.zeros((4, 3), dtype=np.longdouble)
    gl[1], gl[2], gl[3] = c23 / det, c31 / det, c12 / det
    gl[0] = -(gl[1] + gl[2] + gl[3])
    sig = 1 if det > 0 else -1
    V = abs(det) / 6
    g = gl[order]
    Xc = [np.cross(g[a], g[b]) for a, b in gt.EDGES]
    Mm = np.asarray(Mm).astype(np.clongdouble)
    Ms = np.asarray(Ms).astype(np.clongdouble)
    G = np.array([[(Mm @ g[m]) @ g[n] for n in range(4)] for m in range(4)])
    H = np.array([[(Ms @ Xc[p]) @ Xc[q] for q in range(6)] for p in range(6)])
    kap = [gt.EDGES.index(tuple(sorted([rank[u], rank[v]]))) for u, v in IDSET1]
    kap = kap + [6 + k for k in kap]
    kf = [gt.FACES.index(tuple(sorted(rank[list(t)]))) for t in IDSET2]
    kap += [12 + k for k in kf] + [16 + k for k in kf]
    K = np.zeros((20, 20), np.clongdouble)
    M = np.zeros((20, 20), np.clongdouble)
    for a in range(20):
        for b in range(a, 20):
            x, y = kap[a], kap[b]
            s = (sig if gt.ODD[x] else 1) * (sig if gt.ODD[y] else 1)
            K[a, b] = K[b, a] = V * s * sum(_c(c) * H[p][q] for p, q, c in _STIFF[(x, y)])
            M[a, b] = M[b, a] = V * s * sum(_c(c) * G[m][n] for m, n, c in _MASS[(x, y)])
    return K, M


def per_tet_errors(vals, ref_ld):
    """max-entry error of each 20x20 block relative to that block's max."""
    out = []
    for v, r in zip(vals, ref_ld):
        s = float(np.abs(r).max())
        out.append(float(np.abs(v.astype(np.clongdouble) - r).max()) / s)
    return np.array(out)
