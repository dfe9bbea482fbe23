"""Generate the second-order absorbing boundary (ABC) golden fixture by
running the reference's own numba code (robin_abc_order2.py
``_abc_order_2_terms`` :143-217 and ``_matrix_builder`` :225-251), imported
from the EMerge source tree with oracle/ref_loader.py:

    python tests/golden/make_golden_abc2.py

Writes tests/golden/abc2.npz:
* tri_X (16, 3, 3), tri_cf (16,), tri_B (16, 8, 8): single triangles of mixed
  scales, offsets and orientations with a complex coefficient;
* abc_ids (nb,), abc_cf, abc_B (nb, 64): the matrix builder over the x = 0,
  x = a and z = max faces of the 12x6x30 WR-90 air box (each triangle's block
  at its own 64 slots of the [F][64] COO array).
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

DOFCODES_2D = np.array([64, 64, 64, 66, 66, 66, 128, 129], dtype=np.int64)


def main():
    R = load_reference()
    rng = np.random.default_rng(23)
    Xs, cfs, Bs = [], [], []
    for _ in range(16):
        scale = 10.0 ** rng.uniform(-4, 0)
        off = rng.uniform(-1, 1, 3) * 10.0 ** rng.uniform(-3, 0)
        X = (rng.normal(size=(3, 3)) * scale + off[:, None]).astype(np.float64)
        cf = complex(rng.normal(), rng.normal())
        Xs.append(X)
        cfs.append(cf)
        Bs.append(np.asarray(R.abc2._abc_order_2_terms(np.ascontiguousarray(X), cf, DOFCODES_2D)))
    wl = W.wr90_air()
    f = wl.field
    m = f.mesh
    ids = np.concatenate([plane_tris(m, 0, 0.0), plane_tris(m, 0, float(m.nodes[0].max())),
                          plane_tris(m, 2, float(m.nodes[2].max()))]).astype(np.int64)
    cf = complex(0.013, -0.42)
    Mat = R.abc2._matrix_builder(np.ascontiguousarray(m.nodes), np.ascontiguousarray(m.tris).astype(np.int64),
                                 np.ascontiguousarray(m.edges).astype(np.int64),
                                 np.ascontiguousarray(f.tri_to_field).astype(np.int64), ids, cf, DOFCODES_2D)
    abc_B = np.asarray(Mat).reshape(m.n_tris, 64)[ids]
    np.savez_compressed(os.path.join(HERE, "abc2.npz"), tri_X=np.array(Xs), tri_cf=np.array(cfs),
                        tri_B=np.array(Bs), abc_ids=ids, abc_cf=np.complex128(cf), abc_B=abc_B)
    print("tris", len(Xs), "abc tris", ids.size, "max |B|", np.abs(abc_B).max())


if __name__ == "__main__":
    main()
