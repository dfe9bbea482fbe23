"""Generate the heat-conduction golden fixture by running the reference's own
numba code (physics/heatconduction/assembly/grad.py: ``_stiff_matrix_builder``,
``_mass_matrix_builder``, ``tet_stiffness_matrix`` with its CSCMapping),
imported from the EMerge source tree with oracle/ref_loader.py:

    python tests/golden/make_golden_heat.py

Writes tests/golden/heat.npz for a 6x4x10-hex jittered box (1,440 tets) with a
Lagrange-2 field (tet_to_field = [tets; tet_to_edge + n_nodes]): random
symmetric positive-definite conductivity tensors and rho_cp per tet; the COO
values of both builders, their rows/cols, and the stiffness CSC arrays.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from emerge_b200.mesh import TetMesh, structured_box  # noqa: E402
from oracle.ref_loader import load_reference  # noqa: E402


def main():
    R = load_reference()
    nodes, tets = structured_box(6, 4, 10, jitter=0.1, seed=13)
    m = TetMesh(nodes, tets)
    t2f = np.concatenate([m.tets, m.tet_to_edge + m.n_nodes]).astype(np.int64)
    N = m.n_nodes + m.n_edges
    rng = np.random.default_rng(5)
    Q = rng.normal(size=(m.n_tets, 3, 3))
    cond = np.einsum("nij,nkj->ikn", Q, Q) + 0.5 * np.eye(3)[:, :, None]  # [3, 3, nT], SPD
    rho_cp = rng.uniform(1e6, 4e6, m.n_tets)
    K, rows, cols = R.heat._stiff_matrix_builder(np.ascontiguousarray(m.nodes), np.ascontiguousarray(m.tets),
                                                 np.ascontiguousarray(t2f), np.ascontiguousarray(cond))
    M, mrows, mcols = R.heat._mass_matrix_builder(np.ascontiguousarray(m.nodes), np.ascontiguousarray(m.tets),
                                                  np.ascontiguousarray(t2f), rho_cp)
    cm = R.csc_cast.CSCMapping.from_rowcol(rows, cols, N)
    Kc = cm.to_csc(K)
    np.savez_compressed(os.path.join(HERE, "heat.npz"), cond=cond, rho_cp=rho_cp, K=K, M=M, rows=rows, cols=cols,
                        indptr=Kc.indptr, indices=Kc.indices, Kdata=Kc.data, N=N)
    print("tets", m.n_tets, "N", N, "nnz", Kc.nnz)


if __name__ == "__main__":
    main()
