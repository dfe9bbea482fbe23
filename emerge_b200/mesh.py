"""Tetrahedral mesh topology and the Nedelec-2 DoF numbering (host side).

This is the input definition of the assembly path. EMerge builds it from a
gmsh mesh in ``Mesh3D._pre_update`` (mesh3d.py:706-776) and ``Nedelec2.__init__``
(elements/nedelec2.py:44, 61-79). The rules restated here, vectorised with numpy:

* edges = unique sorted node pairs, sorted lexicographically   (mesh3d.py:706-732)
* tris  = unique sorted node triples, sorted lexicographically (mesh3d.py:706-732)
* tet_to_edge[6, nT] with local pairs (1,2),(1,3),(1,4),(2,3),(4,2),(3,4) and
  tet_to_tri[4, nT] with (1,2,3),(1,3,4),(1,4,2),(2,3,4) (1-based, in the tet's
  own vertex order)                                             (mesh3d.py:760-776)
* Nedelec2 (SECOND_MIXED_VOLAKIS, dofsets.py:114-115): n_field = 2E + 2F and
  tet_to_field rows 0-5 = tet_to_edge, 6-11 = tet_to_edge + E,
  12-15 = tet_to_tri + 2E, 16-19 = tet_to_tri + 2E + F   (nedelec2.py:65-79)

Also here: the seeded structured box generator used for the synthetic
workloads (Kuhn split of each hex into 6 tets, jittered interior vertices,
every tet oriented to det > 0).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# local (0-based) vertex pairs/triples of the reference's edge/face slots
EDGE_SLOTS = np.array([(0, 1), (0, 2), (0, 3), (1, 2), (3, 1), (2, 3)], dtype=np.int64)
FACE_SLOTS = np.array([(0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 2, 3)], dtype=np.int64)
# dofcodes of SECOND_MIXED_VOLAKIS: edge ids [0, 2], face ids [0, 1] (dofsets.py:39,114-115)
VOLAKIS_DOFCODES = np.array([64] * 6 + [66] * 6 + [128] * 4 + [129] * 4, dtype=np.int64)
VOLAKIS_DOFCODES_2D = np.array([64] * 3 + [66] * 3 + [128, 129], dtype=np.int64)


def _unique_rows(keys: np.ndarray):
    """Lexicographically sorted unique rows of an int64 (n, k) array and the
    inverse index of every input row."""
    n, k = keys.shape
    order = np.lexsort(keys.T[::-1])
    sk = keys[order]
    new = np.ones(n, dtype=bool)
    new[1:] = np.any(sk[1:] != sk[:-1], axis=1)
    uid = np.cumsum(new) - 1
    inv = np.empty(n, dtype=np.int64)
    inv[order] = uid
    return sk[new], inv


@dataclass
class TetMesh:
    """Mesh topology in the reference's layout (``Mesh3D``): nodes f8[3,nN],
    tets i8[4,nT], edges i8[2,E], tris i8[3,F], tet_to_edge i8[6,nT],
    tet_to_tri i8[4,nT], tri_to_edge i8[3,F]."""

    nodes: np.ndarray
    tets: np.ndarray
    edges: np.ndarray = field(init=False)
    tris: np.ndarray = field(init=False)
    tet_to_edge: np.ndarray = field(init=False)
    tet_to_tri: np.ndarray = field(init=False)
    tri_to_edge: np.ndarray = field(init=False)

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(self.nodes, dtype=np.float64)
        self.tets = np.ascontiguousarray(self.tets, dtype=np.int64)
        if self.nodes.ndim != 2 or self.nodes.shape[0] != 3:
            raise ValueError("nodes must have shape (3, nN)")
        if self.tets.ndim != 2 or self.tets.shape[0] != 4:
            raise ValueError("tets must have shape (4, nT)")
        nT = self.tets.shape[1]
        if nT and (self.tets.min() < 0 or self.tets.max() >= self.nodes.shape[1]):
            raise ValueError("tet node index out of range")
        t = self.tets.T  # (nT, 4)
        ev = np.sort(np.stack([t[:, EDGE_SLOTS[:, 0]], t[:, EDGE_SLOTS[:, 1]]], axis=-1), axis=-1)
        edges, einv = _unique_rows(ev.reshape(-1, 2))
        fv = np.sort(np.stack([t[:, FACE_SLOTS[:, 0]], t[:, FACE_SLOTS[:, 1]], t[:, FACE_SLOTS[:, 2]]], axis=-1), axis=-1)
        tris, finv = _unique_rows(fv.reshape(-1, 3))
        self.edges = np.ascontiguousarray(edges.T)
        self.tris = np.ascontiguousarray(tris.T)
        self.tet_to_edge = np.ascontiguousarray(einv.reshape(nT, 6).T)
        self.tet_to_tri = np.ascontiguousarray(finv.reshape(nT, 4).T)
        # tri_to_edge[3, F]: edges (v0,v1), (v1,v2), (v0,v2) of each sorted tri (mesh3d.py:836-839)
        nN = self.nodes.shape[1]
        ekey = self.edges[0] * nN + self.edges[1]
        tr = self.tris
        self.tri_to_edge = np.ascontiguousarray(np.stack([
            np.searchsorted(ekey, tr[0] * nN + tr[1]), np.searchsorted(ekey, tr[1] * nN + tr[2]),
            np.searchsorted(ekey, tr[0] * nN + tr[2])]).astype(np.int64))

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[1]

    @property
    def n_tets(self) -> int:
        return self.tets.shape[1]

    @property
    def n_edges(self) -> int:
        return self.edges.shape[1]

    @property
    def n_tris(self) -> int:
        return self.tris.shape[1]

    @property
    def tri_to_tet(self) -> np.ndarray:
        """i8[2, F]: the two tets of every triangle, the lower tet index first,
        MISSING_ID where a boundary triangle has one (mesh3d.py:781-795: a
        stable sort of the tets' face slots by triangle)."""
        t2t = getattr(self, "_tri_to_tet", None)
        if t2t is None:
            nT, F = self.n_tets, self.n_tris
            flat = self.tet_to_tri.ravel(order="F")
            order = np.argsort(flat, kind="stable")
            st, stet = flat[order], np.repeat(np.arange(nT, dtype=np.int64), 4)[order]
            t2t = np.full((2, F), MISSING_ID, dtype=np.int64)
            _, first, counts = np.unique(st, return_index=True, return_counts=True)
            t2t[0, st[first]] = stet[first]
            two = counts == 2
            t2t[1, st[first[two]]] = stet[first[two] + 1]
            self._tri_to_tet = t2t
        return t2t

    def tri_normals(self, tri_ids: np.ndarray) -> np.ndarray:
        """f8[3, n]: the unit normal (v1 - v0) x (v2 - v0) of each triangle in
        its sorted vertex order (mesh3d.py:1220-1240)."""
        v = self.nodes[:, self.tris[:, tri_ids]]  # (3, 3 vertices, n)
        n = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], axis=0)
        return n / np.linalg.norm(n, axis=0)


MISSING_ID = -1234  # mesh3d.py:29: the missing second tet of a boundary triangle


class DoFSplitError(ValueError):
    """A surface given to ``partition_dof`` lies on the domain's exterior
    (the reference's DoFSplitException, nedelec2.py:32, :190-195)."""


class Nedelec2Field:
    """The parts of the reference ``Nedelec2`` (elements/nedelec2.py:36-101)
    that the assembly path reads: ``mesh``, ``n_field``, ``dofcodes3d``,
    ``get_tet_to_field()``, ``ntets``. Only SECOND_MIXED_VOLAKIS is built."""

    def __init__(self, mesh: TetMesh):
        self.mesh = mesh
        E, F = mesh.n_edges, mesh.n_tris
        self.nedges, self.ntris, self.ntets = E, F, mesh.n_tets
        self.n_field = 2 * E + 2 * F
        self.dofcodes3d = VOLAKIS_DOFCODES.copy()
        t2f = np.empty((20, mesh.n_tets), dtype=np.int64)
        t2f[0:6] = mesh.tet_to_edge
        t2f[6:12] = mesh.tet_to_edge + E
        t2f[12:16] = mesh.tet_to_tri + 2 * E
        t2f[16:20] = mesh.tet_to_tri + 2 * E + F
        self.tet_to_field = t2f
        # triangle DoFs (nedelec2.py:69-79): 3 ne0 edges, 3 ne2 edges, nf0, nf1
        self.dofcodes2d = VOLAKIS_DOFCODES_2D.copy()
        tf = np.empty((8, F), dtype=np.int64)
        tf[0:3] = mesh.tri_to_edge
        tf[3:6] = mesh.tri_to_edge + E
        tf[6] = np.arange(F) + 2 * E
        tf[7] = np.arange(F) + 2 * E + F
        self.tri_to_field = tf
        self.edge_to_field = np.stack([np.arange(E), np.arange(E) + E]).astype(np.int64)
        # set by partition_dof (nedelec2.py:82-95)
        self.tri_to_field_os: np.ndarray | None = None
        self.edge_to_field_os: np.ndarray | None = None
        self._tet_to_field_orig: np.ndarray | None = None
        self._partitioned = False
        self.split_edges = np.zeros(0, np.int64)
        self.split_tris = np.zeros(0, np.int64)

    def get_tet_to_field(self) -> np.ndarray:
        """The DoF map the curl-curl volume assembly uses: the map from before
        ``partition_dof`` once the field is partitioned (nedelec2.py:104-107)."""
        if self._tet_to_field_orig is not None:
            return self._tet_to_field_orig
        return self.tet_to_field

    def partition_dof(self, surfaces) -> None:
        """Split the DoFs of internal surfaces between their two sides
        (``Nedelec2.partition_dof`` and ``_partition_dof_face``,
        nedelec2.py:114-245), the set-up of a ThinConductor.

        ``surfaces``: a list of (tri_ids, base_normal) pairs, one per face tag
        of the reference (``mesh.get_triangles([tag])`` and
        ``mesh.ftag_to_normal[tag]``). Per surface: every triangle is split;
        an edge is split when exactly two of the surface's triangles hold it;
        each triangle's moved tet is ``tri_to_tet[1]`` when its normal
        (``TetMesh.tri_normals``) has a positive dot product with the base
        normal, else ``tri_to_tet[0]``. Over all surfaces the split edges and
        triangles are sorted and numbered after the existing DoFs: edge DoF
        ``e + i*E`` of the k-th split edge becomes ``n + k + i*nE``, face DoF
        ``2E + t + i*F`` of the k-th split triangle ``n + 2nE + k + i*nF``
        (n the DoF count before, nE / nF the split counts); ``n_field`` grows
        by ``2nE + 2nF``. The moved tets' ``tet_to_field`` columns and the
        split triangles' ``tri_to_field_os`` columns (and ``edge_to_field_os``)
        take the new numbers; ``get_tet_to_field()`` keeps the map from
        before. A second call does nothing, as in the reference."""
        if self._partitioned:
            return
        m = self.mesh
        E, F = m.n_edges, m.n_tris
        if self.tri_to_field_os is None:
            self.tri_to_field_os = self.tri_to_field.copy()
            self.edge_to_field_os = self.edge_to_field.copy()
            self._tet_to_field_orig = self.tet_to_field.copy()
        t2t = m.tri_to_tet
        tets, edges, tris = [], [], []
        for tri_ids, normal in surfaces:
            ids = np.asarray(tri_ids, dtype=np.int64).ravel()
            linked = t2t[:, ids]
            if np.any(linked == MISSING_ID):
                raise DoFSplitError("cannot split the DoFs of a surface on the exterior of the domain")
            count = np.bincount(m.tri_to_edge[:, ids].ravel(), minlength=E)
            edges.append(np.flatnonzero(count == 2))
            tris.append(ids)
            dot = np.sum(m.tri_normals(ids) * np.asarray(normal, dtype=np.float64).reshape(3, 1), axis=0)
            tets.append(np.where(dot > 0, linked[1], linked[0]))
        se = np.unique(np.concatenate(edges)) if edges else np.zeros(0, np.int64)
        st = np.unique(np.concatenate(tris)) if tris else np.zeros(0, np.int64)
        n0, ne, nf = self.n_field, se.size, st.size
        remap = np.arange(n0, dtype=np.int64)
        for i in range(2):
            remap[se + i * E] = n0 + np.arange(ne) + i * ne
            remap[st + 2 * E + i * F] = n0 + 2 * ne + np.arange(nf) + i * nf
        self.n_field = n0 + 2 * ne + 2 * nf
        moved = np.unique(np.concatenate(tets)) if tets else np.zeros(0, np.int64)
        self.tet_to_field[:, moved] = remap[self.tet_to_field[:, moved]]
        self.tri_to_field_os[:, st] = remap[self.tri_to_field[:, st]]
        self.edge_to_field_os[:, se] = remap[self.edge_to_field[:, se]]
        self.split_edges, self.split_tris = se, st
        self._partitioned = True

    @property
    def n_tets(self) -> int:
        return self.ntets


def tet_signed_volumes(nodes: np.ndarray, tets: np.ndarray) -> np.ndarray:
    p = nodes[:, tets]  # (3, 4, nT)
    a, b, c = p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]
    return np.einsum("in,in->n", a, np.cross(b, c, axis=0)) / 6.0


def orient_positive(nodes: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """Swap the last two vertices of every tet whose determinant is negative
    (gmsh emits positively oriented tets; the reference's element matrices
    depend on the orientation, curlcurl.py:142-167)."""
    tets = tets.copy()
    neg = tet_signed_volumes(nodes, tets) < 0
    tets[2, neg], tets[3, neg] = tets[3, neg].copy(), tets[2, neg].copy()
    return tets


# Kuhn split of the unit cube along the main diagonal (corner 0 -> corner 7);
# corner bit 0 = +x, bit 1 = +y, bit 2 = +z.
_KUHN = np.array([[0, 1, 3, 7], [0, 1, 5, 7], [0, 2, 3, 7], [0, 2, 6, 7], [0, 4, 5, 7], [0, 4, 6, 7]],
                 dtype=np.int64)


def structured_box(nx: int, ny: int, nz: int, size=(22.86e-3, 10.16e-3, 50e-3), jitter: float = 0.05,
                   seed: int = 0, origin=(0.0, 0.0, 0.0)):
    """Seeded jittered structured tet box: nx*ny*nz hexes, 6 Kuhn tets each.

    Interior vertices move uniformly in [-jitter, +jitter] * cell size per axis;
    boundary vertices keep the coordinate of the face they lie on. Node id
    ``i + (nx+1)*(j + (ny+1)*k)``. Returns (nodes f8[3,nN], tets i8[4,nT]) with
    every tet positively oriented."""
    rng = np.random.default_rng(seed)
    hx, hy, hz = size[0] / nx, size[1] / ny, size[2] / nz
    i = np.arange(nx + 1)
    j = np.arange(ny + 1)
    k = np.arange(nz + 1)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    x = origin[0] + I * hx
    y = origin[1] + J * hy
    z = origin[2] + K * hz
    if jitter:
        d = rng.uniform(-jitter, jitter, size=(3, I.size))
        x = x + np.where((I > 0) & (I < nx), d[0] * hx, 0.0)
        y = y + np.where((J > 0) & (J < ny), d[1] * hy, 0.0)
        z = z + np.where((K > 0) & (K < nz), d[2] * hz, 0.0)
    nodes = np.stack([x, y, z]).astype(np.float64)
    hi, hj, hk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    hi, hj, hk = hi.transpose(2, 1, 0).ravel(), hj.transpose(2, 1, 0).ravel(), hk.transpose(2, 1, 0).ravel()
    corners = np.empty((8, hi.size), dtype=np.int64)
    for c in range(8):
        ci, cj, ck = hi + (c & 1), hj + ((c >> 1) & 1), hk + ((c >> 2) & 1)
        corners[c] = ci + (nx + 1) * (cj + (ny + 1) * ck)
    tets = corners[_KUHN.T.reshape(-1)].reshape(4, 6, hi.size).transpose(0, 2, 1).reshape(4, -1)
    tets = orient_positive(nodes, tets)
    return nodes, np.ascontiguousarray(tets)


def plane_tris(mesh: TetMesh, axis: int, value: float, rtol: float = 1e-9) -> np.ndarray:
    """Ids of the triangles whose three vertices lie on the plane
    x[axis] = value (to rtol times the mesh extent along that axis): the
    surface a port or an absorbing boundary is applied to (the reference
    selects them by the face's physical tag, mesh3d ``get_triangles``)."""
    x = mesh.nodes[axis]
    tol = rtol * max(float(x.max() - x.min()), 1e-300)
    on = np.abs(x - value) <= tol
    return np.flatnonzero(on[mesh.tris].all(axis=0)).astype(np.int64)


def grid_level_tris(mesh: TetMesh, dims, axis: int, level: int, lo=(0, 0, 0), hi=None) -> np.ndarray:
    """Ids of the triangles of a ``structured_box(*dims)`` mesh whose three
    vertices have grid index ``level`` along ``axis`` and grid indices within
    [lo, hi] along the other axes: a (jittered) grid surface, e.g. the strip
    of a ThinConductor inside the box (the reference takes it from a face
    tag, mesh3d ``get_triangles``)."""
    nx, ny, nz = dims
    hi = (nx, ny, nz) if hi is None else hi
    ids = np.arange(mesh.n_nodes)
    g = np.stack([ids % (nx + 1), (ids // (nx + 1)) % (ny + 1), ids // ((nx + 1) * (ny + 1))])
    ok = g[axis] == level
    for a in range(3):
        if a != axis:
            ok &= (g[a] >= lo[a]) & (g[a] <= hi[a])
    return np.flatnonzero(ok[mesh.tris].all(axis=0)).astype(np.int64)
