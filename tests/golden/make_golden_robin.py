"""Generate the Robin (port) boundary-term golden fixture by running the
reference's own numba code (robinbc.py ``ned2_tri_stiff`` :316-378 and
``compute_bc_entries`` :381-402), imported from the EMerge source tree with
oracle/ref_loader.py. Run in a container that has the reference tree:

    python tests/golden/make_golden_robin.py

Writes tests/golden/robin.npz:
* tri_X (16, 3, 3), tri_gamma (16,), tri_B (16, 8, 8): single triangles of
  mixed scales, offsets and orientations, complex gamma;
* port_ids (nb,), port_gamma, port_B (nb, 64): compute_bc_entries over the
  two port faces (z = 0 and z = 50 mm) of the 12x6x30 WR-90 air box at 10 GHz
  with the TE10 gamma = j beta (port_bcs.py:963-983);
* tri_U (16, 3, 6), tri_f (16, 8): ned2_tri_force (:220-277) of the same
  single triangles with random complex fields;
* port_pts (3, 6, nb) from generate_points_3d (:104-135) and port_b (N,):
  compute_force_entries (:280-313) over the port faces with the field
  U = (0, (1 + 0.5j) sin(pi x / a), 0).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from emerge_b200 import workloads as W  # noqa: E402
from oracle.ref_loader import load_reference  # noqa: E402

DOFCODES_2D = np.array([64, 64, 64, 66, 66, 66, 128, 129], dtype=np.int64)


def main():
    R = load_reference()
    rng = np.random.default_rng(11)
    Xs, gs, Bs = [], [], []
    for i in range(16):
        scale = 10.0 ** rng.uniform(-4, 0)
        off = rng.uniform(-1, 1, 3) * 10.0 ** rng.uniform(-3, 0)
        X = (rng.normal(size=(3, 3)) * scale + off[:, None]).astype(np.float64)
        g = complex(rng.normal(), rng.normal())
        Xs.append(X)
        gs.append(g)
        Bs.append(np.asarray(R.robinbc.ned2_tri_stiff(np.ascontiguousarray(X), g, DOFCODES_2D)))
    wl = W.wr90_air()
    m = wl.field.mesh
    ids = W.port_tris(wl)
    gamma = W.rect_port_gamma(wl.freq)
    Bmat = np.zeros(m.n_tris * 64, np.complex128)
    Bmat = R.robinbc.compute_bc_entries(np.ascontiguousarray(m.nodes), np.ascontiguousarray(m.tris), Bmat, ids,
                                        complex(gamma), DOFCODES_2D)
    port_B = Bmat.reshape(m.n_tris, 64)[ids]
    Us = [rng.normal(size=(3, 6)) + 1j * rng.normal(size=(3, 6)) for _ in Xs]
    fs = [np.asarray(R.robinbc.ned2_tri_force(np.ascontiguousarray(X), np.ascontiguousarray(U), DOFCODES_2D))
          for X, U in zip(Xs, Us)]
    D = np.ascontiguousarray(R.robinbc.DPTS)
    xf, yf, zf = R.robinbc.generate_points_3d(np.ascontiguousarray(m.nodes), np.ascontiguousarray(m.tris), D, ids)
    pts = np.stack([xf, yf, zf]).reshape(3, D.shape[1], ids.size)
    U = np.zeros((3, D.shape[1], ids.size), np.complex128)
    U[1] = (1 + 0.5j) * np.sin(np.pi * pts[0] / W.WR90[0])
    tri_to_field = np.ascontiguousarray(wl.field.tri_to_field)
    b = R.robinbc.compute_force_entries(np.ascontiguousarray(m.nodes), np.ascontiguousarray(m.tris),
                                        np.zeros(wl.field.n_field, np.complex128), ids, U, tri_to_field,
                                        DOFCODES_2D)
    np.savez_compressed(os.path.join(HERE, "robin.npz"), tri_X=np.array(Xs), tri_gamma=np.array(gs),
                        tri_B=np.array(Bs), port_ids=ids, port_gamma=np.complex128(gamma), port_B=port_B,
                        tri_U=np.array(Us), tri_f=np.array(fs), port_pts=pts, port_b=b)
    print("tris", len(Xs), "port tris", ids.size, "gamma", gamma)


if __name__ == "__main__":
    main()
