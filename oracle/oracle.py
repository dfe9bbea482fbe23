"""CPU ORACLE wrapper -- test infrastructure, not product code.

Loads ``oracle/libemoracle.so`` (plain-C restatement of the reference path,
``oracle/nedelec_oracle.c``) with ctypes and exposes the reference's call
surface on numpy arrays:

* ``matrix_builder``   -> curlcurl.py:387-456 ``_matrix_builder``
* ``CSCPattern``       -> csc_cast.py:29-63   ``CSCMapping`` (from_rowcol / to_csc)
* ``tet_mass_stiffness_matrices`` -> curlcurl.py:222-270
* ``tri_stiff``, ``robin_entries``, ``tri_rowcol``, ``generate_csc``
                       -> robinbc.py:316-402 (``ned2_tri_stiff``,
                          ``compute_bc_entries``), femdata.py:52-56,75-92,104-118
* ``leg2_values``, ``leg2_rowcol`` -> physics/heatconduction/assembly/grad.py:
                          199-400 (Lagrange-2 heat stiffness / mass, COO)
* ``ned2_interp``, ``port_overlap`` -> compiled/base/interp.py:286-387,
                          mth/integrals.py:13-24,64-103, sparam.py:62-97
* ``tri_force``, ``force_entries``, ``tri_points`` -> robinbc.py:104-135,220-313
                          (``generate_points_3d``, ``ned2_tri_force``,
                          ``compute_force_entries``)
* ``ChunkedAssembly``  -> _matrix_builder + to_csc(E - k0^2 B) (curlcurl.py:387-456,
                          csc_cast.py:55-177, assembler.py:494) over all tets of a
                          mesh too large for its full COO, in chunks of tets, equal
                          bit for bit to the one-piece scatter (chunked_oracle.c)
* ``topology_loops``   -> mesh3d.py:706-776 and nedelec2.py:61-79 restated as
  plain Python loops (small meshes only; checks the vectorised host topology)

Parity status: pinned. ``tests/test_oracle_golden.py`` checks it against the
fixtures that ``tests/golden/make_golden.py`` produced by running the
reference's own numba functions.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
from scipy.sparse import csc_matrix

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libemoracle.so")
_lib = None

_p = ctypes.c_void_p
_i64 = ctypes.c_int64


def build() -> str:
    """Compile the C oracle (``make -C oracle``)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_matrix_builder.restype = ctypes.c_int
        L.oracle_matrix_builder.argtypes = [_p, _i64, _p, _i64, _p, _i64, _p, _i64, _p, _p, _p, _p, _p, _p, _i64,
                                            _p, _p, _p, _p, ctypes.c_int]
        L.oracle_csc_pattern.restype = _i64
        L.oracle_csc_pattern.argtypes = [_p, _p, _i64, _i64, _p, _p, _p, _p, ctypes.c_int]
        L.oracle_csc_indices.restype = None
        L.oracle_csc_indices.argtypes = [_p, _p, _p, _i64, _p]
        L.oracle_scatter_f8.restype = None
        L.oracle_scatter_f8.argtypes = [_p, _p, _p, _p, _i64, _p, ctypes.c_int]
        L.oracle_scatter_c16.restype = None
        L.oracle_scatter_c16.argtypes = [_p, _p, _p, _p, _i64, _p, ctypes.c_int]
        L.oracle_scatter_lincomb_c16.restype = None
        L.oracle_scatter_lincomb_c16.argtypes = [_p, _p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_double, _p, _p, _p, _i64, _p, ctypes.c_int]
        L.oracle_num_threads.restype = ctypes.c_int
        L.oracle_tri_stiff.restype = None
        L.oracle_tri_stiff.argtypes = [_p, ctypes.c_double, ctypes.c_double, _p]
        L.oracle_abc2_block.restype = None
        L.oracle_abc2_block.argtypes = [_p, ctypes.c_double, ctypes.c_double, _p]
        L.oracle_abc2_entries.restype = ctypes.c_int
        L.oracle_abc2_entries.argtypes = [_p, _i64, _p, _i64, _p, _i64, ctypes.c_double, ctypes.c_double, _p]
        L.oracle_robin_entries.restype = ctypes.c_int
        L.oracle_robin_entries.argtypes = [_p, _i64, _p, _i64, _p, _i64, ctypes.c_double, ctypes.c_double, _p]
        L.oracle_tri_force.restype = None
        L.oracle_tri_force.argtypes = [_p, _p, _p]
        L.oracle_leg2_builder.restype = ctypes.c_int
        L.oracle_leg2_builder.argtypes = [_p, _i64, _p, _i64, _p, ctypes.c_int, _p]
        L.oracle_ned2_interp.restype = None
        L.oracle_ned2_interp.argtypes = [_p, _i64, _p, _i64, _p, _i64, _p, _i64, _p, _p, _p, _p, _i64, _p, _p]
        L.oracle_port_overlap.restype = None
        L.oracle_port_overlap.argtypes = [_p, _i64, _p, _i64, _p, _i64, _p, _i64, _p, _p, _p, _p, _p, _i64, _p,
                                          ctypes.c_int, _p, ctypes.c_double, _p, _p]
        L.oracle_dof_incidence.restype = ctypes.c_int
        L.oracle_dof_incidence.argtypes = [_p, _i64, _p, _i64, _i64, _p, _p]
        L.oracle_pattern_rows.restype = _i64
        L.oracle_pattern_rows.argtypes = [_p, _i64, _p, _p, _p, _i64, _i64, _p, _p, ctypes.c_int]
        L.oracle_chunk_order.restype = ctypes.c_int
        L.oracle_chunk_order.argtypes = [_p, _i64, _p, _i64, _i64, _p, _p, _i64, _p, _p, _p, ctypes.c_int,
                                         ctypes.c_int]
        L.oracle_chunk_scatter.restype = None
        L.oracle_chunk_scatter.argtypes = [_p, _p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, _p, _p, _p, ctypes.c_int, _p, ctypes.c_int]
        L.oracle_force_entries.restype = ctypes.c_int
        L.oracle_force_entries.argtypes = [_p, _i64, _p, _i64, _p, _p, _i64, _p, _i64, _p]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def num_threads() -> int:
    return lib().oracle_num_threads()


def matrix_builder(nodes, tets, tris, edges, tet_to_field, tet_to_edge, tet_to_tri, ur, er, tetids,
                   nthreads: int = 0):
    """``_matrix_builder`` (curlcurl.py:387-456): returns (dataE, dataB, rows, cols)."""
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    tets = np.ascontiguousarray(tets, dtype=np.int64)
    tris = np.ascontiguousarray(tris, dtype=np.int64)
    edges = np.ascontiguousarray(edges, dtype=np.int64)
    t2f = np.ascontiguousarray(tet_to_field, dtype=np.int64)
    t2e = np.ascontiguousarray(tet_to_edge, dtype=np.int64)
    t2t = np.ascontiguousarray(tet_to_tri, dtype=np.int64)
    ur = np.ascontiguousarray(ur, dtype=np.complex128)
    er = np.ascontiguousarray(er, dtype=np.complex128)
    tetids = np.ascontiguousarray(tetids, dtype=np.int64)
    nA = tetids.shape[0]
    dataE = np.empty(400 * nA, dtype=np.complex128)
    dataB = np.empty(400 * nA, dtype=np.complex128)
    rows = np.empty(400 * nA, dtype=np.int64)
    cols = np.empty(400 * nA, dtype=np.int64)
    rc = lib().oracle_matrix_builder(_ptr(nodes), nodes.shape[1], _ptr(tets), tets.shape[1], _ptr(tris),
                                     tris.shape[1], _ptr(edges), edges.shape[1], _ptr(t2f), _ptr(t2e), _ptr(t2t),
                                     _ptr(ur), _ptr(er), _ptr(tetids), nA, _ptr(dataE), _ptr(dataB), _ptr(rows),
                                     _ptr(cols), int(nthreads))
    if rc != 0:
        raise ValueError("tet id out of range")
    return dataE, dataB, rows, cols


def matrix_builder_into(mesh_arrays, tetids, out, nthreads: int = 0):
    """``_matrix_builder`` (curlcurl.py:387-456) into preallocated arrays:
    mesh_arrays = (nodes, tets, tris, edges, t2f, t2e, t2t, ur, er) already
    contiguous in the oracle's dtypes, out = (dataE, dataB, rows, cols) of at
    least 400 * len(tetids) entries."""
    nodes, tets, tris, edges, t2f, t2e, t2t, ur, er = mesh_arrays
    dataE, dataB, rows, cols = out
    nA = tetids.shape[0]
    rc = lib().oracle_matrix_builder(_ptr(nodes), nodes.shape[1], _ptr(tets), tets.shape[1], _ptr(tris),
                                     tris.shape[1], _ptr(edges), edges.shape[1], _ptr(t2f), _ptr(t2e), _ptr(t2t),
                                     _ptr(ur), _ptr(er), _ptr(tetids), nA, _ptr(dataE), _ptr(dataB), _ptr(rows),
                                     _ptr(cols), int(nthreads))
    if rc != 0:
        raise ValueError("tet id out of range")


class ChunkedAssembly:
    """The reference's cached-pattern assembly of A = E - k0^2 B over every
    assembled tet of a mesh whose full COO arrays (19.2 KB per tet) would not
    fit in host memory: ``_matrix_builder`` on chunks of consecutive tetids,
    each chunk scattered into the one CSC value array in the order of the
    reference's ``to_csc`` (column, row, slot), so the result equals the
    one-piece ``CSCPattern.values_lincomb`` bit for bit (chunked_oracle.c).
    The pattern and each chunk's scatter order are built once (the reference
    caches its CSCMapping); ``step`` is the per-frequency work."""

    def __init__(self, field, er, ur, conductor_tets, chunk_tets: int = 100_000, nthreads: int = 0):
        mesh = field.mesh
        self.nthreads = int(nthreads) if nthreads else num_threads()
        nT = mesh.tets.shape[1]
        tet_assy = np.arange(nT, dtype=np.int64)
        conductor_tets = np.asarray(conductor_tets, dtype=np.int64)
        if conductor_tets.size:
            tet_assy = np.delete(tet_assy, conductor_tets)
        self.tetids = np.ascontiguousarray(tet_assy)
        self.nA = nA = self.tetids.shape[0]
        self.N = N = int(field.n_field)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        i64 = lambda a: np.ascontiguousarray(a, dtype=np.int64)
        c16 = lambda a: np.ascontiguousarray(a, dtype=np.complex128)
        self.mesh_arrays = (f64(mesh.nodes), i64(mesh.tets), i64(mesh.tris), i64(mesh.edges),
                            i64(field.get_tet_to_field()), i64(mesh.tet_to_edge), i64(mesh.tet_to_tri), c16(ur),
                            c16(er))
        t2f = self.mesh_arrays[4]
        L = lib()
        dptr = np.empty(N + 1, np.int64)
        dtet = np.empty(20 * nA, np.int32)
        if L.oracle_dof_incidence(_ptr(t2f), nT, _ptr(self.tetids), nA, N, _ptr(dptr), _ptr(dtet)) != 0:
            raise ValueError("DoF index out of range")
        max_deg = int(np.diff(dptr).max()) if N else 0
        self.indptr = np.empty(N + 1, np.int64)
        nnz = L.oracle_pattern_rows(_ptr(t2f), nT, _ptr(self.tetids), _ptr(dptr), _ptr(dtet), N, max_deg,
                                    _ptr(self.indptr), None, self.nthreads)
        if nnz < 0:
            raise MemoryError("pattern rows")
        self.nnz = int(nnz)
        self.indices = np.empty(self.nnz, np.int32)
        L.oracle_pattern_rows(_ptr(t2f), nT, _ptr(self.tetids), _ptr(dptr), _ptr(dtet), N, max_deg,
                              _ptr(self.indptr), _ptr(self.indices), self.nthreads)
        del dptr, dtet
        self.chunk_tets = int(chunk_tets)
        self.chunks = []
        nsplit = 4 * self.nthreads
        for a0 in range(0, nA, self.chunk_tets):
            a1 = min(nA, a0 + self.chunk_tets)
            S = 400 * (a1 - a0)
            perm = np.empty(S, np.int32)
            tgt = np.empty(S, np.int32)
            splits = np.empty(nsplit + 1, np.int64)
            rc = L.oracle_chunk_order(_ptr(t2f), nT, _ptr(self.tetids), a0, a1, _ptr(self.indptr),
                                      _ptr(self.indices), N, _ptr(perm), _ptr(tgt), _ptr(splits), nsplit,
                                      self.nthreads)
            if rc != 0:
                raise ValueError(f"chunk order failed ({rc})")
            self.chunks.append((a0, a1, perm, tgt, splits))
        n = min(self.chunk_tets, nA) if nA else 1
        self.buf = (np.empty(400 * n, np.complex128), np.empty(400 * n, np.complex128), np.empty(400 * n, np.int64),
                    np.empty(400 * n, np.int64))

    def step(self, alpha, beta, out: np.ndarray | None = None) -> np.ndarray:
        """A's values (complex128 [nnz], CSC order): alpha*E + beta*B over all
        assembled tets, chunk by chunk."""
        a, b = complex(alpha), complex(beta)
        if out is None:
            out = np.zeros(self.nnz, np.complex128)
        else:
            out[:] = 0
        L = lib()
        dE, dB = self.buf[0], self.buf[1]
        for a0, a1, perm, tgt, splits in self.chunks:
            matrix_builder_into(self.mesh_arrays, self.tetids[a0:a1], self.buf, self.nthreads)
            L.oracle_chunk_scatter(_ptr(dE), _ptr(dB), a.real, a.imag, b.real, b.imag, _ptr(perm), _ptr(tgt),
                                   _ptr(splits), splits.shape[0] - 1, _ptr(out), self.nthreads)
        return out


class CSCPattern:
    """``CSCMapping`` (csc_cast.py:29-63): pattern + COO-slot map."""

    def __init__(self, indptr, indices, target, col_offsets, perm, N):
        self.indptr, self.indices, self.target = indptr, indices, target
        self.col_offsets, self.perm, self.N = col_offsets, perm, N
        self.nnz = int(indices.shape[0])

    @staticmethod
    def from_rowcol(rows, cols, N, nthreads: int = 0) -> "CSCPattern":
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        S = rows.shape[0]
        col_offsets = np.empty(N + 1, dtype=np.int64)
        perm = np.empty(S, dtype=np.int64)
        indptr = np.empty(N + 1, dtype=np.int64)
        target = np.empty(S, dtype=np.int64)
        nnz = lib().oracle_csc_pattern(_ptr(rows), _ptr(cols), S, N, _ptr(col_offsets), _ptr(perm), _ptr(indptr),
                                       _ptr(target), int(nthreads))
        if nnz < 0:
            raise MemoryError("oracle pattern allocation failed")
        indices = np.empty(nnz, dtype=np.int64)
        lib().oracle_csc_indices(_ptr(rows), _ptr(perm), _ptr(target), S, _ptr(indices))
        return CSCPattern(indptr, indices, target, col_offsets, perm, N)

    def values_f8(self, data, nthreads: int = 0) -> np.ndarray:
        """``scatter_to_csc_f8`` (csc_cast.py:150-177): real data."""
        data = np.ascontiguousarray(data, dtype=np.float64)
        out = np.zeros(self.nnz, dtype=np.float64)
        lib().oracle_scatter_f8(_ptr(data), _ptr(self.perm), _ptr(self.target), _ptr(self.col_offsets), self.N,
                                _ptr(out), int(nthreads))
        return out

    def values(self, data, nthreads: int = 0) -> np.ndarray:
        data = np.ascontiguousarray(data, dtype=np.complex128)
        out = np.zeros(self.nnz, dtype=np.complex128)
        lib().oracle_scatter_c16(_ptr(data), _ptr(self.perm), _ptr(self.target), _ptr(self.col_offsets), self.N,
                                 _ptr(out), int(nthreads))
        return out

    def values_lincomb(self, dataE, dataB, alpha, beta, nthreads: int = 0) -> np.ndarray:
        """scatter of alpha*dataE + beta*dataB (the caller's E - k0^2 B,
        assembler.py:494) without materialising the combination."""
        out = np.zeros(self.nnz, dtype=np.complex128)
        a, b = complex(alpha), complex(beta)
        lib().oracle_scatter_lincomb_c16(_ptr(dataE), _ptr(dataB), a.real, a.imag, b.real, b.imag, _ptr(self.perm),
                                         _ptr(self.target),
                                         _ptr(self.col_offsets), self.N, _ptr(out), int(nthreads))
        return out

    def to_csc(self, data, nthreads: int = 0) -> csc_matrix:
        return csc_matrix((self.values(data, nthreads), self.indices, self.indptr), shape=(self.N, self.N))


def tet_mass_stiffness_matrices(field, er, ur, conductor_tets, cscmap=None, nthreads: int = 0):
    """``tet_mass_stiffness_matrices`` (curlcurl.py:222-270) on the oracle."""
    mesh = field.mesh
    tet_assy = np.arange(mesh.tets.shape[1])
    conductor_tets = np.asarray(conductor_tets, dtype=np.int64)
    if conductor_tets.shape[0] > 0:
        tet_assy = np.delete(tet_assy, conductor_tets)
    dataE, dataB, rows, cols = matrix_builder(mesh.nodes, mesh.tets, mesh.tris, mesh.edges,
                                              field.get_tet_to_field(), mesh.tet_to_edge, mesh.tet_to_tri, ur, er,
                                              tet_assy, nthreads)
    if cscmap is None:
        cscmap = CSCPattern.from_rowcol(rows, cols, field.n_field, nthreads)
    return dataE, dataB, cscmap


def topology_loops(tets: np.ndarray):
    """Mesh3D._pre_update edge/tri extraction and tet->edge/tri maps
    (mesh3d.py:706-776), plus Nedelec2 tet_to_field (nedelec2.py:65-79),
    restated with the reference's own Python loops. Small meshes only."""
    edgeset, triset = set(), set()
    for itet in range(tets.shape[1]):
        i1, i2, i3, i4 = sorted(int(v) for v in tets[:, itet])
        edgeset.update({(i1, i2), (i1, i3), (i1, i4), (i2, i3), (i2, i4), (i3, i4)})
        triset.update({(i1, i2, i3), (i1, i2, i4), (i1, i3, i4), (i2, i3, i4)})
    edges = np.array(sorted(edgeset)).T
    tris = np.array(sorted(triset)).T
    inv_edges = {tuple(edges[:, i].tolist()): i for i in range(edges.shape[1])}
    inv_tris = {tuple(tris[:, i].tolist()): i for i in range(tris.shape[1])}
    idset1 = ((1, 2), (1, 3), (1, 4), (2, 3), (4, 2), (3, 4))
    idset2 = ((1, 2, 3), (1, 3, 4), (1, 4, 2), (2, 3, 4))
    nT = tets.shape[1]
    t2e = np.zeros((6, nT), dtype=np.int64)
    t2t = np.zeros((4, nT), dtype=np.int64)
    for itet in range(nT):
        t = tets[:, itet]
        t2e[:, itet] = [inv_edges[tuple(sorted((int(t[i - 1]), int(t[j - 1]))))] for i, j in idset1]
        t2t[:, itet] = [inv_tris[tuple(sorted((int(t[i - 1]), int(t[j - 1]), int(t[k - 1]))))] for i, j, k in idset2]
    E, F = edges.shape[1], tris.shape[1]
    t2f = np.zeros((20, nT), dtype=np.int64)
    for i in range(2):  # nedof = 2 (edge ids [0, 2])
        t2f[6 * i:6 * (i + 1)] = t2e + i * E
    for i in range(2):  # nfdof = 2 (face ids [0, 1])
        t2f[12 + 4 * i:12 + 4 * (i + 1)] = t2t + i * F + 2 * E
    return edges, tris, t2e, t2t, t2f


# ---------------------------------------------------------------- Robin boundary term
def tri_stiff(X: np.ndarray, gamma: complex) -> np.ndarray:
    """``ned2_tri_stiff`` (robinbc.py:316-378): X f8[3, 3] = the triangle's
    vertex coordinates (column v = vertex v) -> c16[8, 8]."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.empty(64, np.complex128)
    g = complex(gamma)
    lib().oracle_tri_stiff(_ptr(X), g.real, g.imag, _ptr(out))
    return out.reshape(8, 8)


def abc2_block(X: np.ndarray, cf: complex) -> np.ndarray:
    """``_abc_order_2_terms`` (robin_abc_order2.py:143-217): X f8[3, 3] ->
    c16[8, 8], cf times the area-weighted curl-curl block."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.empty(64, np.complex128)
    c = complex(cf)
    lib().oracle_abc2_block(_ptr(X), c.real, c.imag, _ptr(out))
    return out.reshape(8, 8)


def abc2_entries(field, tri_ids, cf: complex, Mat: np.ndarray | None = None) -> np.ndarray:
    """``abc_order_2_matrix`` / ``_matrix_builder`` (robin_abc_order2.py:225-281):
    every listed tri's block added into the tri COO array c16[F*64]."""
    m = field.mesh
    F = m.tris.shape[1]
    if Mat is None:
        Mat = np.zeros(F * 64, np.complex128)
    nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
    tris = np.ascontiguousarray(m.tris, dtype=np.int64)
    ids = np.ascontiguousarray(tri_ids, dtype=np.int64)
    c = complex(cf)
    if lib().oracle_abc2_entries(_ptr(nodes), nodes.shape[1], _ptr(tris), F, _ptr(ids), ids.shape[0], c.real, c.imag,
                                 _ptr(Mat)) != 0:
        raise IndexError("triangle or node index out of range")
    return Mat


def robin_entries(field, tri_ids, gamma: complex, Bmat: np.ndarray | None = None) -> np.ndarray:
    """``assemble_robin_bc`` / ``compute_bc_entries`` (robinbc.py:381-451):
    adds every listed tri's 8x8 block into the tri COO array Bmat c16[F*64]
    (``empty_tri_matrix``, femdata.py:52-56) at itri*64."""
    m = field.mesh
    F = m.tris.shape[1]
    if Bmat is None:
        Bmat = np.zeros(F * 64, np.complex128)
    nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
    tris = np.ascontiguousarray(m.tris, dtype=np.int64)
    ids = np.ascontiguousarray(tri_ids, dtype=np.int64)
    g = complex(gamma)
    rc = lib().oracle_robin_entries(_ptr(nodes), nodes.shape[1], _ptr(tris), F, _ptr(ids), ids.shape[0], g.real,
                                    g.imag, _ptr(Bmat))
    if rc != 0:
        raise IndexError("tri id or vertex index out of range")
    return Bmat


def tri_rowcol(field, other_side: bool = False):
    """``empty_tri_rowcol`` (femdata.py:75-92): per tri 64 slots,
    rows[p + 8*ii + jj] = t2f[ii], cols[...] = t2f[jj] over ``tri_to_field``,
    or over ``tri_to_field_os`` (the split DoFs of a partitioned field) with
    ``other_side``."""
    t2f = field.tri_to_field_os if other_side else field.tri_to_field  # (8, F)
    F = t2f.shape[1]
    rows = np.repeat(t2f.T[:, :, None], 8, axis=2).reshape(F * 64)
    cols = np.repeat(t2f.T[:, None, :], 8, axis=1).reshape(F * 64)
    return rows, cols


def generate_csc(field, data: np.ndarray, rowcol=None) -> csc_matrix:
    """``generate_csc`` (femdata.py:104-118) with the tri row/col arrays
    (``tri_rowcol(field)`` unless given): the nonzero slots only, duplicates
    summed by scipy, shape (n_field, n_field)."""
    rows, cols = tri_rowcol(field) if rowcol is None else rowcol
    ids = np.argwhere(data != 0)[:, 0]
    return csc_matrix((data[ids], (rows[ids], cols[ids])), shape=(field.n_field, field.n_field))


def tri_force(X: np.ndarray, U: np.ndarray) -> np.ndarray:
    """``ned2_tri_force`` (robinbc.py:220-277): X f8[3, 3] vertex coordinates,
    U c16[3, 6] the incident field at the 6 points -> c16[8]."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    U = np.ascontiguousarray(U, dtype=np.complex128)
    out = np.empty(8, np.complex128)
    lib().oracle_tri_force(_ptr(X), _ptr(U), _ptr(out))
    return out


def tri_points(field, tri_ids) -> np.ndarray:
    """``generate_points_3d`` (robinbc.py:104-135) as loops: the 6 quadrature
    points of every listed tri, f8[3, 6, nb]."""
    m = field.mesh
    D = np.array([[0.81684757298045896, 0.09157621350977101, 0.09157621350977101, 0.10810301816807000,
                   0.44594849091596500, 0.44594849091596500],
                  [0.09157621350977101, 0.81684757298045896, 0.09157621350977101, 0.44594849091596500,
                   0.10810301816807000, 0.44594849091596500],
                  [0.09157621350977004, 0.09157621350977008, 0.81684757298045807, 0.44594849091596500,
                   0.44594849091596500, 0.10810301816807000]])
    ids = np.asarray(tri_ids, dtype=np.int64)
    out = np.empty((3, 6, ids.size))
    for i, t in enumerate(ids):
        v = m.tris[:, t]
        for d in range(3):
            x1, x2, x3 = m.nodes[d, v]
            out[d, :, i] = x1 * D[0] + x2 * D[1] + x3 * D[2]
    return out


def force_entries(field, tri_ids, U: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    """``assemble_robin_bc_bvec`` / ``compute_force_entries`` (robinbc.py:280-313,
    405-433): b[tri_to_field[:, t]] += ned2_tri_force(t) for every listed tri,
    U c16[3, 6, nb] the incident field at ``tri_points``."""
    m = field.mesh
    N = int(field.n_field)
    if b is None:
        b = np.zeros(N, np.complex128)
    ids = np.ascontiguousarray(tri_ids, dtype=np.int64)
    U = np.ascontiguousarray(U, dtype=np.complex128)
    if U.shape != (3, 6, ids.size):
        raise ValueError("U must have shape (3, 6, n_tris)")
    nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
    tris = np.ascontiguousarray(m.tris, dtype=np.int64)
    t2f = np.ascontiguousarray(field.tri_to_field, dtype=np.int64)
    rc = lib().oracle_force_entries(_ptr(nodes), nodes.shape[1], _ptr(tris), tris.shape[1], _ptr(t2f), _ptr(ids),
                                    ids.size, _ptr(U), N, _ptr(b))
    if rc != 0:
        raise IndexError("tri id or index out of range")
    return b


# ---------------------------------------------------------------- post-processing
def _mesh_args(field):
    m = field.mesh
    c = np.ascontiguousarray
    return (c(m.nodes, dtype=np.float64), m.n_nodes, c(m.tets, dtype=np.int64), m.n_tets, c(m.edges, dtype=np.int64),
            m.n_edges, c(m.tris, dtype=np.int64), m.n_tris, c(m.tet_to_edge, dtype=np.int64),
            c(m.tet_to_tri, dtype=np.int64))


def ned2_interp(field, x, points, tet_of) -> np.ndarray:
    """``ned2_tet_interp`` (interp.py:286-387): the solution x (c16[N]) at
    points f8[3, n] inside tets tet_of (i8[n], -1 = outside -> NaN) ->
    c16[3, n]."""
    a = _mesh_args(field)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    pts = np.ascontiguousarray(points, dtype=np.float64)
    t = np.ascontiguousarray(tet_of, dtype=np.int64)
    out = np.empty((3, pts.shape[1]), np.complex128)
    lib().oracle_ned2_interp(*[(_ptr(v) if isinstance(v, np.ndarray) else v) for v in a], _ptr(x), _ptr(pts),
                             pts.shape[1], _ptr(t), _ptr(out))
    return out


def port_overlap(field, x, tri_ids, tri_tets, rule, U, q: float):
    """sum over tris of area * sum_k w_k (E - q U) . conj(U) at the rule's
    points (surface_integral with unit constants of sparam_field_power's
    integrand times 2 Z0); rule f8[4, nq] (weights, L1, L2, L3), U
    c16[3, nq, nb]. Returns (total, per-tri c16[nb])."""
    a = _mesh_args(field)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    ids = np.ascontiguousarray(tri_ids, dtype=np.int64)
    tt = np.ascontiguousarray(tri_tets, dtype=np.int64)
    rule = np.ascontiguousarray(rule, dtype=np.float64)
    U = np.ascontiguousarray(U, dtype=np.complex128)
    per = np.empty(ids.size, np.complex128)
    tot = np.zeros(1, np.complex128)
    lib().oracle_port_overlap(*[(_ptr(v) if isinstance(v, np.ndarray) else v) for v in a], _ptr(x), _ptr(ids),
                              _ptr(tt), ids.size, _ptr(rule), rule.shape[1], _ptr(U), float(q), _ptr(per), _ptr(tot))
    return complex(tot[0]), per


# ---------------------------------------------------------------- heat conduction (Lagrange-2)
def leg2_values(mesh, coef, kind: str) -> np.ndarray:
    """``_stiff_matrix_builder`` (kind 'stiff', coef = conductivity f8[3, 3, nT])
    or ``_mass_matrix_builder`` (kind 'mass', coef = rho_cp f8[nT]),
    grad.py:333-400: the COO values f8[100 nT]."""
    nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64)
    tets = np.ascontiguousarray(mesh.tets, dtype=np.int64)
    c = np.ascontiguousarray(coef, dtype=np.float64)
    out = np.empty(100 * tets.shape[1])
    lib().oracle_leg2_builder(_ptr(nodes), nodes.shape[1], _ptr(tets), tets.shape[1], _ptr(c),
                              0 if kind == "stiff" else 1, _ptr(out))
    return out


def leg2_rowcol(tet_to_field: np.ndarray):
    """COO rows/cols of grad.py:350-354: per tet 100 slots, rows[p + 10 ii +
    jj] = t2f[ii], cols[p + 10 ii + jj] = t2f[jj]."""
    t = np.asarray(tet_to_field).T  # (nT, 10)
    nT = t.shape[0]
    rows = np.repeat(t[:, :, None], 10, axis=2).reshape(nT * 100)
    cols = np.repeat(t[:, None, :], 10, axis=1).reshape(nT * 100)
    return rows, cols
