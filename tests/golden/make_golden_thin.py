"""Generate the ThinConductor (partitioned field) golden fixture by running the
reference's own code, imported from the EMerge source tree with
oracle/ref_loader.py:

    python tests/golden/make_golden_thin.py

* ``Nedelec2.__init__`` and ``Nedelec2.partition_dof`` (elements/nedelec2.py:
  36-245) over two internal strips of a jittered 4x3x5-hex box (360 tets),
  given to it through a small stand-in for the mesh object (the attributes
  and the three helpers ``partition_dof`` reads: get_triangles, get_edges,
  get_normal, the last as in mesh3d.py:1220-1240);
* the microwave assembly of assembler.py:485-494 and :576-639 on that field:
  ``tet_mass_stiffness_matrices`` (curlcurl.py:222-270) with its CSCMapping,
  ``K = to_csc(E - k0^2 B)``, a port Robin term on the z = 0 face and both
  strips as ThinConductors (``assemble_robin_bc`` into B_robin and B_robin_2),
  ``K += generate_csc(B_robin)``, ``K += generate_csc(B_robin_2,
  empty_tri_rowcol(other_side=True))`` (femdata.py:75-118).

Writes tests/golden/thin.npz: the mesh, strips, materials and gammas; the
partition (n_field, tet_to_field, tri_to_field_os, edge_to_field_os); the
other-side matrix alone and the final K (CSC arrays).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from emerge_b200.mesh import MISSING_ID, TetMesh, grid_level_tris, structured_box  # noqa: E402
from oracle.ref_loader import load_nedelec2, load_reference  # noqa: E402

DIMS = (4, 3, 5)
STRIPS = ((2, 2, (0, 0, 0), (3, 2, 5)), (2, 4, (1, 1, 0), (4, 3, 5)))  # (axis, level, lo, hi)


class _MeshStandIn:
    """The mesh attributes Nedelec2 and partition_dof read (mesh3d.py)."""

    _MISSING_ID = MISSING_ID

    def __init__(self, m: TetMesh, tags: dict, normals: dict):
        self.nodes, self.tets, self.tris, self.edges = m.nodes, m.tets, m.tris, m.edges
        self.tet_to_edge, self.tet_to_tri, self.tri_to_edge = m.tet_to_edge, m.tet_to_tri, m.tri_to_edge
        self.n_nodes, self.n_tets, self.n_edges, self.n_tris = m.n_nodes, m.n_tets, m.n_edges, m.n_tris
        # tri -> (lower tet, higher tet), written out plainly
        t2t = np.full((2, m.n_tris), MISSING_ID, dtype=int)
        for tet in range(m.n_tets):
            for tri in m.tet_to_tri[:, tet]:
                t2t[0 if t2t[0, tri] == MISSING_ID else 1, tri] = tet
        self.tri_to_tet = t2t
        self.centers = m.nodes[:, m.tets].mean(axis=1)
        self.tri_centers = m.nodes[:, m.tris].mean(axis=1)
        self._tags = tags
        self.ftag_to_normal = normals
        self.ftag_to_edge = {t: sorted(set(m.tri_to_edge[:, ids].ravel().tolist())) for t, ids in tags.items()}
        zc = self.centers[2]
        cut = np.median(zc)
        self.vtag_to_tet = {1: np.flatnonzero(zc < cut), 2: np.flatnonzero(zc >= cut)}

    def get_triangles(self, tags):
        tags = [tags] if isinstance(tags, int) else tags
        return np.concatenate([self._tags[t] for t in tags]).astype(int)

    def get_edges(self, tags):
        tags = [tags] if isinstance(tags, int) else tags
        return np.array(sorted(set(sum((self.ftag_to_edge[t] for t in tags), []))))

    def get_normal(self, itri):
        i1, i2, i3 = self.tris[:, itri]
        p0, p1, p2 = self.nodes[:, i1], self.nodes[:, i2], self.nodes[:, i3]
        n = np.cross(p1 - p0, p2 - p0)
        return n / np.linalg.norm(n)


def main():
    R = load_reference()
    NE = load_nedelec2()
    nodes, tets = structured_box(*DIMS, jitter=0.08, seed=21)
    m = TetMesh(nodes, tets)
    strips = [grid_level_tris(m, DIMS, a, lev, lo, hi) for a, lev, lo, hi in STRIPS]
    normals = [np.array([0.0, 0.0, 1.0]), np.array([0.0, 0.0, -1.0])]
    tags = {11: strips[0], 12: strips[1]}
    mesh = _MeshStandIn(m, tags, {11: normals[0], 12: normals[1]})
    field = NE.nedelec2.Nedelec2(mesh, NE.dofsets.ElementSpace.SECOND_MIXED_VOLAKIS.get_set())
    n0 = field.n_field
    field.partition_dof([[11], [12]])

    rng = np.random.default_rng(8)
    nT = m.n_tets
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = rng.uniform(1, 6, nT) * (1 - 1j * rng.uniform(1e-3, 1e-2, nT))
        ur[d, d] = rng.uniform(1, 2, nT)
    k0 = 2 * np.pi * 10e9 / 299792458.0
    dataE, dataB, cmap = R.curlcurl.tet_mass_stiffness_matrices(field, er, ur, np.zeros(0, dtype=int))
    K = cmap.to_csc(dataE - dataB * k0 ** 2)

    port = grid_level_tris(m, DIMS, 2, 0)
    g_port = 1j * 158.0
    g_tc = [(2.0 + 3.0j) * 1e2, (0.5 - 1.5j) * 1e2]
    B1 = field.empty_tri_matrix()
    B2 = B1.copy().astype(np.complex128)
    B1 = R.robinbc.assemble_robin_bc(field, B1, port, g_port)
    for ids, g in zip(strips, g_tc):
        B1 = R.robinbc.assemble_robin_bc(field, B1, ids, g)
        B2 = R.robinbc.assemble_robin_bc(field, B2, ids, g)
    K += field.generate_csc(B1)
    rows, cols = field.empty_tri_rowcol(other_side=True)
    OS = field.generate_csc(B2, (rows, cols))
    K += OS
    K = K.tocsc()
    OS = OS.tocsc()
    np.savez_compressed(
        os.path.join(HERE, "thin.npz"), nodes=nodes, tets=tets, dims=np.array(DIMS), strip0=strips[0],
        strip1=strips[1], normal0=normals[0], normal1=normals[1], port=port, g_port=np.complex128(g_port),
        g_tc=np.array(g_tc), er=er, ur=ur, k0=np.float64(k0), n_field0=np.int64(n0), n_field=np.int64(field.n_field),
        tet_to_field=field.tet_to_field, tet_to_field_orig=field.get_tet_to_field(),
        tri_to_field_os=field.tri_to_field_os, edge_to_field_os=field.edge_to_field_os,
        os_indptr=OS.indptr, os_indices=OS.indices, os_data=OS.data,
        K_indptr=K.indptr, K_indices=K.indices, K_data=K.data)
    print("tets", nT, "n_field", n0, "->", field.n_field, "strip tris", [s.size for s in strips],
          "K nnz", K.nnz, "OS nnz", OS.nnz)


if __name__ == "__main__":
    main()
