"""Generate the post-processing golden fixture by running the reference's own
numba code (compiled/base/interp.py ``ned2_tet_interp`` :286-387,
mth/integrals.py ``surface_integral`` :64-103 with ``gaus_quad_tri``),
imported from the EMerge source tree with oracle/ref_loader.py:

    python tests/golden/make_golden_interp.py

Writes tests/golden/interp.npz for the 12x6x30 WR-90 air box (12,960 tets):
* x (N,): a seeded complex solution vector;
* pts (3, 2000), tet_of (2000,): random points inside random tets; E (3, 2000)
  from ned2_tet_interp;
* port_ids (nb,), port_tets (nb,): the z = 0 port triangles and the tet on
  each; rule5 (4, nq): gaus_quad_tri(5); U5 (3, nq, nb): the TE10-shaped
  field (0, (1 + 0.5j) sin(pi x / a), 0) at the rule's points;
  overlap_active / overlap_passive: surface_integral of
  (E - Q U) . conj(U) with Q = 1 / 0 (sparam_field_power's integrand times 2 Z0).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from emerge_b200 import workloads as W  # noqa: E402
from emerge_b200.mesh import plane_tris  # noqa: E402
from oracle.ref_loader import load_reference  # noqa: E402


def main():
    R = load_reference()
    wl = W.wr90_air()
    f = wl.field
    m = f.mesh
    rng = np.random.default_rng(21)
    x = rng.normal(size=f.n_field) + 1j * rng.normal(size=f.n_field)
    n = 2000
    tet_of = rng.integers(0, m.n_tets, n)
    bary = rng.dirichlet(np.ones(4), n)
    pts = np.einsum("dvn,nv->dn", m.nodes[:, m.tets[:, tet_of]], bary)
    args = (np.ascontiguousarray(m.tets), np.ascontiguousarray(m.tris), np.ascontiguousarray(m.edges),
            np.ascontiguousarray(m.nodes), np.ascontiguousarray(f.tet_to_field), np.ascontiguousarray(m.tet_to_edge),
            np.ascontiguousarray(m.tet_to_tri))
    dof = np.asarray(f.dofcodes3d, dtype=np.int64)

    def interp(points, mapping):
        return np.array(R.interp.ned2_tet_interp(np.ascontiguousarray(points), x, *args,
                                                 np.unique(mapping).astype(np.int64), mapping.astype(np.int64), dof))

    E = interp(pts, tet_of)
    ids = plane_tris(m, 2, float(m.nodes[2].min()))
    tets_of_tri = np.array([int(np.flatnonzero((m.tet_to_tri == t).any(axis=0))[0]) for t in ids])
    rule = np.array(R.integrals.gaus_quad_tri(5))
    nq = rule.shape[1]
    xf, yf, zf, shape = R.integrals.generate_int_points_tri(np.ascontiguousarray(m.nodes),
                                                           np.ascontiguousarray(m.tris[:, ids]), rule)
    P = np.stack([xf, yf, zf])
    mapping = np.tile(tets_of_tri, nq)  # point k * nb + i lies on tri i
    U = np.zeros((3, P.shape[1]), np.complex128)
    U[1] = (1 + 0.5j) * np.sin(np.pi * P[0] / W.WR90[0])
    Ef = interp(P, mapping)
    out = {}
    for name, Q in (("overlap_active", 1.0), ("overlap_passive", 0.0)):
        def integrand(xx, yy, zz, Q=Q):
            e = Ef - Q * U
            return e[0] * np.conj(U[0]) + e[1] * np.conj(U[1]) + e[2] * np.conj(U[2])
        out[name] = R.integrals.surface_integral(np.ascontiguousarray(m.nodes), np.ascontiguousarray(m.tris[:, ids]),
                                                 integrand, None, gq_order=5)
    np.savez_compressed(os.path.join(HERE, "interp.npz"), x=x, pts=pts, tet_of=tet_of, E=E, port_ids=ids,
                        port_tets=tets_of_tri, rule5=rule, U5=U.reshape(3, nq, ids.size),
                        overlap_active=np.complex128(out["overlap_active"]),
                        overlap_passive=np.complex128(out["overlap_passive"]))
    print("points", n, "port tris", ids.size, "nq", nq, out)


if __name__ == "__main__":
    main()
