"""ThinConductor's opposite-side boundary term on the GPU, and the grown
pattern it needs.

Reference (physics/microwave/assembly/assembler.py:576-639)::

    B_matrix_robin_2 = B_matrix_robin.copy()          # when a ThinConductor exists
    for bc in robin_bcs:
        B_matrix_robin = assemble_robin_bc(field, B_matrix_robin, tri_ids, gamma)
        if isinstance(bc, ThinConductor):
            B_matrix_robin_2 = assemble_robin_bc(field, B_matrix_robin_2, tri_ids, gamma)
    K += field.generate_csc(B_matrix_robin)
    rows, cols = field.empty_tri_rowcol(other_side=True)
    K += field.generate_csc(B_matrix_robin_2, (rows, cols))

Before that the field was partitioned over the ThinConductor surfaces
(microwave_3d.py:639-642, nedelec2.py:114-172): each split triangle and each
edge inside a surface got a second set of DoFs, numbered after the first,
and ``tri_to_field_os`` maps the split triangles to them. The volume assembly
keeps the unsplit map (curlcurl.py:244), so A's columns of the new DoFs are
empty, and the second matrix puts the same 8x8 triangle blocks on the
other-side DoFs. Its pairs lie partly outside A's pattern; scipy's ``+=``
returns the union of both patterns.

Here::

    R = RobinTerm(field, tc_tris, cscmap)            # this side, on A's pattern
    T = OppositeSideTerm(field, tc_tris)             # the other side
    X = ExtendedCSCMapping(cscmap, [T])              # A's pattern + T's pairs, built once
    K = X.to_csc(Evec - Bvec * k0**2 + R * gamma + T * gamma)

``ExtendedCSCMapping`` lays out the union once (emg_csc_lookup); every
assembly forms A on its own pattern, moves its values to their union
positions in one pass with the new entries zeroed (emg_csc_shift), then
adds the opposite-side blocks (emg_robin_build_dofs / emg_robin_apply). The
union keeps explicit zeros where the reference's scipy sum drops entries
that cancel; the matrix is the same.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.sparse import csc_matrix

from . import _lib as L
from .assembly import ElemValues, GpuCSCMapping, LinComb, _to_dev

__all__ = ["OppositeSideTerm", "ExtendedCSCMapping"]


class OppositeSideTerm:
    """The Robin blocks of ``tri_ids`` on the other-side DoFs of a
    partitioned field (``field.tri_to_field_os``): the term of
    ``generate_csc(B2, empty_tri_rowcol(other_side=True))``. ``gamma * T``
    joins a combination for ``ExtendedCSCMapping.to_csc`` / ``to_device``;
    the device blocks are built when an ExtendedCSCMapping takes the term."""

    _is_opposite_term = True

    def __init__(self, field, tri_ids):
        t2f_os = getattr(field, "tri_to_field_os", None)
        if t2f_os is None:
            raise ValueError("the field has no other side: call field.partition_dof(...) first")
        m = field.mesh
        ids = np.asarray(tri_ids, dtype=np.int64).ravel()
        if ids.size and (ids.min() < 0 or ids.max() >= m.n_tris):
            raise IndexError("triangle id out of range")
        self.dofs = np.ascontiguousarray(np.asarray(t2f_os)[:, ids].T.astype(np.int64))  # (nb, 8)
        if self.dofs.size and (self.dofs.min() < 0 or self.dofs.max() >= int(field.n_field)):
            raise IndexError("other-side DoF outside [0, n_field)")
        self._field, self._ids = field, ids
        self.n_btris = int(ids.size)
        self.xmap = None

    def pairs(self) -> tuple[np.ndarray, np.ndarray]:
        """(rows, cols) of the 64 slots of every triangle, slot 8r + c at
        (dofs[r], dofs[c]) (femdata.py:80-104)."""
        d = self.dofs
        rows = np.repeat(d, 8, axis=1).reshape(-1)
        cols = np.tile(d, (1, 8)).reshape(-1)
        return rows, cols

    def _bind(self, xmap: "ExtendedCSCMapping") -> None:
        if self.xmap is not None and self.xmap is not xmap:
            raise ValueError("the opposite-side term already belongs to another extended mapping")
        self.xmap = xmap
        dev = xmap.device
        m = self._field.mesh
        r = L.Robin()
        L.check(L.lib().emg_robin_init(self.n_btris, L.ctypes.byref(r)))
        self.desc = r
        self.d_keys = torch.empty(max(r.n_keys, 1), dtype=torch.int64, device=dev)
        self.d_vals = torch.empty(max(r.n_slots, 1), dtype=torch.complex128, device=dev)
        if not self.n_btris:
            return
        nodes = _to_dev(m.nodes, torch.float64, dev)
        tris = _to_dev(m.tris, torch.int32, dev)
        t2e = _to_dev(m.tri_to_edge, torch.int32, dev)
        btris = _to_dev(self._ids, torch.int32, dev)
        dofs = _to_dev(self.dofs, torch.int32, dev)
        status = torch.zeros(2, dtype=torch.int64, device=dev)
        st = L.stream_handle(dev)
        L.check(L.lib().emg_robin_build_dofs(L.ctypes.byref(r), L.ptr(nodes), m.n_nodes, L.ptr(tris), L.ptr(t2e),
                                             m.n_tris, m.n_edges, L.ptr(btris), L.ptr(dofs), L.ptr(xmap.d_indptr),
                                             L.ptr(xmap.d_indices), xmap.N, L.ptr(self.d_keys), L.ptr(self.d_vals),
                                             L.ptr(status), st))
        f, i = L.ctypes.c_int64(), L.ctypes.c_int64()
        L.check(L.lib().emg_status_read(L.ptr(status), L.ctypes.byref(f), L.ctypes.byref(i), st))
        if f.value:
            t = int(self._ids[i.value]) if 0 <= i.value < self._ids.size else i.value
            raise L.EmgMeshError(L.EMG_EMESH, f"opposite-side triangle {t}: "
                                 + ("pair outside the grown pattern" if f.value & L.EMG_ST_INDEX
                                    else "degenerate triangle"))

    def apply(self, U: torch.Tensor, gamma: complex) -> torch.Tensor:
        """U[p] += gamma * (the term at p) on the extended mapping's values."""
        x = self.xmap
        if x is None:
            raise ValueError("the opposite-side term is not part of an ExtendedCSCMapping yet")
        if U.dtype != torch.complex128 or U.numel() < x.nnz:
            raise ValueError("U must be complex128 with the extended mapping's nnz values")
        g = complex(gamma)
        L.check(L.lib().emg_robin_apply(L.ctypes.byref(self.desc), L.ptr(self.d_keys), L.ptr(self.d_vals), g.real,
                                        g.imag, L.ptr(U), x.nnz, L.stream_handle(x.device)))
        return U

    def _lc(self) -> LinComb:
        return LinComb(None, {self: 1.0 + 0.0j})

    def __mul__(self, c):
        return self._lc() * c

    __rmul__ = __mul__

    def __neg__(self):
        return self._lc() * -1.0

    def __add__(self, o):
        return self._lc() + o

    __radd__ = __add__

    def __sub__(self, o):
        return self._lc() - o

    def __rsub__(self, o):
        return (-self._lc()) + o


class ExtendedCSCMapping:
    """A's pattern (``cscmap``) grown by the pairs of opposite-side terms:
    the pattern of the reference's ``K += generate_csc(B2, other-side
    rowcol)``. Same surface as ``GpuCSCMapping`` for callers (``N``, ``nnz``,
    ``indptr``/``indices``, ``d_indptr``/``d_indices``, ``to_device``,
    ``to_csc``, ``host_buffer``), so a ``SolveSubmatrix`` can take it."""

    def __init__(self, cscmap: GpuCSCMapping, terms):
        self.base = cscmap
        self.device = cscmap.device
        self.N = N = cscmap.N
        self.terms = list(terms)
        for t in self.terms:
            if not getattr(t, "_is_opposite_term", False):
                raise TypeError("ExtendedCSCMapping takes OppositeSideTerm objects")
            if int(t._field.n_field) != N:
                raise ValueError("an opposite-side term belongs to another field")
        dev, st = self.device, L.stream_handle(self.device)
        pr = [t.pairs() for t in self.terms]
        rows = np.concatenate([p[0] for p in pr]) if pr else np.zeros(0, np.int64)
        cols = np.concatenate([p[1] for p in pr]) if pr else np.zeros(0, np.int64)
        key = np.unique(cols * N + rows)  # column-major order of the distinct pairs
        uc, ur = key // N, key % N
        pos = torch.empty(max(key.size, 1), dtype=torch.int64, device=dev)
        if key.size:
            # both inputs held until the lookup has run (a freed block would be reused at once)
            d_uc, d_ur = _to_dev(uc, torch.int64, dev), _to_dev(ur, torch.int64, dev)
            L.check(L.lib().emg_csc_lookup(L.ptr(cscmap.d_indptr), L.ptr(cscmap.d_indices), N, L.ptr(d_uc),
                                           L.ptr(d_ur), key.size, L.ptr(pos), st))
        pos = pos[: key.size].cpu().numpy()
        if np.any(pos == np.iinfo(np.int64).min):
            raise IndexError("opposite-side pair outside [0, N)")
        new = pos < 0
        xc, xr = uc[new], ur[new]
        ins = -(pos[new] + 1)  # insertion points in A, non-decreasing
        n_x = int(xc.size)
        self.n_extra = n_x
        self.nnz = cscmap.nnz + n_x
        if self.nnz >= (1 << 31):
            raise ValueError("the grown pattern exceeds int32 indices")
        # an entry p of A moves by the number of new entries inserted at or
        # before it; the e-th new entry (column-major) lands at ins[e] + e
        starts = np.unique(ins)
        seg_start = np.concatenate([[0], starts]) if (starts.size == 0 or starts[0] != 0) else starts
        seg_shift = np.searchsorted(ins, seg_start, side="right").astype(np.int64)
        xpos = ins + np.arange(n_x, dtype=np.int64)
        self._seg_start = _to_dev(seg_start.astype(np.int64), torch.int64, dev)
        self._seg_shift = _to_dev(seg_shift, torch.int64, dev)
        self._n_seg = int(seg_start.size)
        self._xpos = _to_dev(xpos, torch.int64, dev) if n_x else torch.zeros(1, dtype=torch.int64, device=dev)
        counts = np.bincount(xc, minlength=N) if n_x else np.zeros(N, np.int64)
        indptr = cscmap.indptr.astype(np.int64) + np.concatenate([[0], np.cumsum(counts)])
        self._indptr = indptr.astype(np.int32)
        self.d_indptr = _to_dev(self._indptr, torch.int32, dev)
        self.d_indices = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        xrow = _to_dev(xr.astype(np.int32), torch.int32, dev) if n_x else None
        L.check(L.lib().emg_csc_shift(L.ptr(cscmap.d_indices), cscmap.nnz, 4, L.ptr(self._seg_start),
                                      L.ptr(self._seg_shift), self._n_seg, L.ptr(self._xpos),
                                      L.ptr(xrow) if xrow is not None else None, n_x, L.ptr(self.d_indices),
                                      self.nnz, st))
        self._indices = None
        for t in self.terms:
            t._bind(self)

    @property
    def indptr(self) -> np.ndarray:
        return self._indptr

    @property
    def indices(self) -> np.ndarray:
        if self._indices is None:
            self._indices = self.d_indices[: self.nnz].cpu().numpy()
        return self._indices

    def grow(self, A: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """A's values (complex128 [base nnz], device) at their union positions,
        the new entries zero."""
        b = self.base
        if A.dtype != torch.complex128 or A.numel() < b.nnz:
            raise ValueError("A must be complex128 with the base mapping's nnz values")
        if out is None:
            out = torch.empty(max(self.nnz, 1), dtype=torch.complex128, device=self.device)
        L.check(L.lib().emg_csc_shift(L.ptr(A), b.nnz, 16, L.ptr(self._seg_start), L.ptr(self._seg_shift),
                                      self._n_seg, L.ptr(self._xpos), None, self.n_extra, L.ptr(out), self.nnz,
                                      L.stream_handle(self.device)))
        return out

    def to_device(self, data) -> torch.Tensor:
        """Values of to_csc(data) kept on the device (complex128 [nnz])."""
        if isinstance(data, ElemValues) or getattr(data, "_is_robin_term", False) \
                or getattr(data, "_is_opposite_term", False):
            data = data._lc()
        if not isinstance(data, LinComb):
            return self.grow(self.base.to_device(data))[: self.nnz]
        ops = data.opposite_terms
        for t, _ in ops:
            if t.xmap is not self:
                raise ValueError("an opposite-side term of the combination belongs to another mapping")
        U = self.grow(self.base.to_device(data.without_opposite()))
        for t, g in ops:
            t.apply(U, g)
        return U[: self.nnz]

    def host_buffer(self) -> np.ndarray:
        return torch.empty(max(self.nnz, 1), dtype=torch.complex128, pin_memory=True).numpy()[: self.nnz]

    def to_csc(self, data, out: np.ndarray | None = None) -> csc_matrix:
        """The reference's K after ``K += generate_csc(B2, other-side rowcol)``
        as a scipy csc_matrix (shape (N, N), the union pattern)."""
        d = self.to_device(data)
        if out is None:
            host = torch.empty(d.shape, dtype=torch.complex128, pin_memory=True)
            host.copy_(d)
            vals = host.numpy()
        else:
            if out.dtype != np.complex128 or out.shape != (self.nnz,) or not out.flags["C_CONTIGUOUS"]:
                raise ValueError(f"out must be a contiguous complex128 array of {self.nnz} values")
            torch.from_numpy(out).copy_(d)
            vals = out
        return csc_matrix((vals, self.indices, self.indptr), shape=(self.N, self.N))
