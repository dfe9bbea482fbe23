"""Column sharding of one assembly across ranks (one process per GPU).

The global system A (CSC, N = 2E + 2F columns) is split by ENTITY: rank r
owns the edges and faces whose lowest global node id lies in its node range
[node_lo, node_hi). Edges and faces are sorted lexicographically by node ids
(mesh3d.py:706-732), so a rank owns one contiguous edge range [e0, e1) and
one contiguous face range [f0, f1), i.e. four contiguous column ranges of A:

    [e0, e1), [E + e0, E + e1), [2E + f0, 2E + f1), [2E + F + f0, 2E + F + f1)

(the two DoFs of an edge/face, nedelec2.py:65-79). Node ranges are cut so
that the estimated nonzeros per rank balance.

Each rank assembles every tet that touches one of its entities (the halo
tets are recomputed on both sides; no exchange step), builds the pattern of
that tet subset and keeps its four column ranges. An owned column receives
contributions from exactly the tets that touch its entity, all of which the
rank assembles, in the same relative order as the full assembly, so the
owned columns are identical to the corresponding columns of the full A
(pattern and values). The column blocks of all ranks, concatenated per
group in rank order, are the full A.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Shard:
    rank: int
    world: int
    node_lo: int
    node_hi: int
    edge_lo: int
    edge_hi: int
    face_lo: int
    face_hi: int
    n_edges: int
    n_tris: int
    n_tets: int
    tetids: np.ndarray  # ascending global ids of the tets this rank assembles
    est_nnz: int

    def column_ranges(self) -> list:
        E, F = self.n_edges, self.n_tris
        e0, e1, f0, f1 = self.edge_lo, self.edge_hi, self.face_lo, self.face_hi
        return [(e0, e1), (E + e0, E + e1), (2 * E + f0, 2 * E + f1), (2 * E + F + f0, 2 * E + F + f1)]

    def excluded_tets(self) -> np.ndarray:
        """Tets this rank does not assemble, in the reference's conductor_tets
        form (curlcurl.py:248-250): passing it to tet_mass_stiffness_matrices
        assembles exactly ``tetids``."""
        keep = np.zeros(self.n_tets, bool)
        keep[self.tetids] = True
        return np.flatnonzero(~keep).astype(np.int64)


def entity_weights(mesh, assembled: np.ndarray | None = None):
    """Estimated nonzeros of the two columns of each edge and face: an
    interior edge in k tets touches 1 + 3k edges and 3k faces, a face in k
    tets touches 3 + 3k edges and 1 + 3k faces; each column holds two rows per
    adjacent entity. Returns (w_edge i64[E], w_face i64[F])."""
    t2e, t2t = mesh.tet_to_edge, mesh.tet_to_tri
    if assembled is not None:
        t2e, t2t = t2e[:, assembled], t2t[:, assembled]
    ke = np.bincount(t2e.ravel(), minlength=mesh.n_edges)
    kf = np.bincount(t2t.ravel(), minlength=mesh.n_tris)
    return 4 + 24 * ke, 16 + 24 * kf


def partition(mesh, world: int, conductor_tets=None) -> list:
    """Shards of all ranks (see module docstring)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    nT, nN = mesh.n_tets, mesh.n_nodes
    assembled = np.ones(nT, bool)
    if conductor_tets is not None and len(conductor_tets):
        assembled[np.asarray(conductor_tets, dtype=np.int64)] = False
    ids = np.flatnonzero(assembled)
    we, wf = entity_weights(mesh, ids)
    first_e, first_f = mesh.edges[0], mesh.tris[0]  # nondecreasing: lexicographic order
    per_node = np.bincount(first_e, weights=we, minlength=nN) + np.bincount(first_f, weights=wf, minlength=nN)
    cum = np.concatenate([[0.0], np.cumsum(per_node)])
    total = cum[-1]
    cuts = [0] + [int(np.searchsorted(cum, total * r / world, side="left")) for r in range(1, world)] + [nN]
    cuts = np.maximum.accumulate(np.clip(cuts, 0, nN))
    shards = []
    for r in range(world):
        n0, n1 = int(cuts[r]), int(cuts[r + 1])
        e0, e1 = (int(x) for x in np.searchsorted(first_e, [n0, n1], side="left"))
        f0, f1 = (int(x) for x in np.searchsorted(first_f, [n0, n1], side="left"))
        own = (((mesh.tet_to_edge >= e0) & (mesh.tet_to_edge < e1)).any(axis=0)
               | ((mesh.tet_to_tri >= f0) & (mesh.tet_to_tri < f1)).any(axis=0))
        tetids = np.flatnonzero(own & assembled).astype(np.int64)
        est = int(we[e0:e1].sum() + wf[f0:f1].sum())
        shards.append(Shard(r, world, n0, n1, e0, e1, f0, f1, mesh.n_edges, mesh.n_tris, nT, tetids, est))
    return shards


def shard_of(mesh, rank: int, world: int, conductor_tets=None) -> Shard:
    return partition(mesh, world, conductor_tets)[rank]


@dataclass
class ColumnBlock:
    """The owned columns of one rank: per column range (c0, c1) the CSC
    pointers relative to the range's first nonzero, the row indices and the
    values."""

    ranges: list
    indptr: list  # int64 [c1 - c0 + 1] each, starting at 0
    indices: list
    values: list


def extract_block(shard: Shard, indptr: np.ndarray, indices: np.ndarray, values: np.ndarray) -> ColumnBlock:
    """Owned columns out of a rank's local CSC arrays (pattern of its tet
    subset, global column numbering)."""
    ip, ix, vs = [], [], []
    for c0, c1 in shard.column_ranges():
        lo, hi = int(indptr[c0]), int(indptr[c1])
        ip.append(np.asarray(indptr[c0:c1 + 1], dtype=np.int64) - lo)
        ix.append(np.asarray(indices[lo:hi]))
        vs.append(np.asarray(values[lo:hi]))
    return ColumnBlock(shard.column_ranges(), ip, ix, vs)


def merge_blocks(blocks: list, N: int):
    """Full CSC arrays (indptr i64[N+1], indices, values) from the column
    blocks of all ranks (ordered by rank)."""
    col_len = np.zeros(N, np.int64)
    pieces_i, pieces_v = [], []
    for g in range(4):
        for b in blocks:
            c0, c1 = b.ranges[g]
            col_len[c0:c1] = np.diff(b.indptr[g])
            pieces_i.append(b.indices[g])
            pieces_v.append(b.values[g])
    indptr = np.concatenate([[0], np.cumsum(col_len)])
    return indptr, np.concatenate(pieces_i), np.concatenate(pieces_v)


class ShardedAssembly:
    """One rank's shard on its GPU, through the drop-in: the rank's tet subset
    is assembled (``tet_mass_stiffness_matrices`` with the complement as the
    excluded set) and the owned column ranges are views into the local A."""

    def __init__(self, field, er, ur, shard: Shard, precision: str = "fp64", device=None):
        import torch

        from .assembly import DeviceMaterial, DeviceMesh, GpuCSCMapping, _Job, _prec

        self.shard = shard
        self.dmesh = DeviceMesh(field, shard.excluded_tets(), device)
        self.cmap = GpuCSCMapping(self.dmesh)
        self.job = _Job(self.dmesh, DeviceMaterial(er, ur, self.dmesh.n_tets, self.dmesh.device), _prec(precision))
        cols = torch.tensor([c for r in shard.column_ranges() for c in r], dtype=torch.int64,
                            device=self.dmesh.device)
        b = self.cmap.d_indptr.index_select(0, cols).cpu().numpy().astype(np.int64)
        self.bounds = [(int(b[2 * g]), int(b[2 * g + 1])) for g in range(4)]
        self.own_nnz = sum(hi - lo for lo, hi in self.bounds)

    def assemble(self, alpha: complex, beta: complex, out=None) -> list:
        """alpha*K + beta*M of the owned columns: four device views (complex128),
        one per column range, stream-ordered."""
        out = self.cmap.assemble_device(self.job, alpha, beta, out)
        return [out[lo:hi] for lo, hi in self.bounds]

    def block(self, alpha: complex, beta: complex) -> ColumnBlock:
        """Host copy of the owned column block."""
        vals = self.cmap.assemble_device(self.job, alpha, beta)[: self.cmap.nnz]
        self.dmesh.check_status()
        return extract_block(self.shard, self.cmap.indptr, self.cmap.indices, vals.cpu().numpy())
