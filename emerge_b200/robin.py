"""Robin (third-kind) boundary term on the GPU: ports, absorbing boundaries
and surface impedances on boundary triangles.

Reference (physics/microwave/assembly/assembler.py:576-630)::

    B_matrix_robin = field.empty_tri_matrix()
    B_matrix_robin = assemble_robin_bc(field, B_matrix_robin, tri_ids, gamma)
    K += field.generate_csc(B_matrix_robin)

Here the term is a lazy object that joins the caller's combination of
element values::

    R = RobinTerm(field, tri_ids, cscmap)           # built once per surface
    A = cscmap.to_csc(Evec - Bvec * k0**2 + R * gamma)

``RobinTerm`` builds each triangle's 8x8 block once for gamma = 1 (the block
is linear in gamma, robinbc.py:316-378) and the position in A of each of its
64 DoF pairs; every assembly then adds gamma times the blocks into A's values
on the device, summing each position in a fixed order. Every DoF pair of a
triangle shares a tet with it, so A's pattern does not change.

``RobinTerm(..., kind="abc2")`` is the second-order absorbing boundary
correction on the same triangles and positions (abc_order_2_matrix,
robin_abc_order2.py:143-281): the block A sum_q w_q c_a c_b of the scalar
2-D curls, scaled by the coefficient the assembler passes
(assembler.py:626-632)::

    R2 = RobinTerm(field, abc_tri_ids, cscmap, kind="abc2")
    A = cscmap.to_csc(Evec - Bvec * k0**2 + R * gamma + R2 * c2)
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.sparse import csc_matrix

from . import _lib as L
from .assembly import GpuCSCMapping, LinComb, _to_dev

__all__ = ["RobinTerm", "assemble_robin_bc", "abc_order_2_matrix"]

# barycentric rows L1..L3 of the 6-point triangle rule (robinbc.py:189-196)
_TRI_L = np.array([
    [0.81684757298045896, 0.09157621350977101, 0.09157621350977101, 0.10810301816807000, 0.44594849091596500,
     0.44594849091596500],
    [0.09157621350977101, 0.81684757298045896, 0.09157621350977101, 0.44594849091596500, 0.10810301816807000,
     0.44594849091596500],
    [0.09157621350977004, 0.09157621350977008, 0.81684757298045807, 0.44594849091596500, 0.44594849091596500,
     0.10810301816807000]])


class RobinTerm:
    """The boundary term of the triangles ``tri_ids`` (int, into
    ``field.mesh.tris``) on the pattern of ``cscmap``; ``gamma * term`` is a
    lazy combination for ``cscmap.to_csc`` / ``to_device``. A triangle listed
    twice counts twice, as in the reference."""

    _is_robin_term = True

    def __init__(self, field, tri_ids, cscmap: GpuCSCMapping, kind: str = "robin"):
        if kind not in ("robin", "abc2"):
            raise ValueError("kind must be 'robin' (the Robin / port term) or 'abc2' (second-order ABC correction)")
        self.kind = kind
        m = field.mesh
        ids = np.asarray(tri_ids, dtype=np.int64).ravel()
        if ids.size and (ids.min() < 0 or ids.max() >= m.n_tris):
            raise IndexError("triangle id out of range")
        if int(field.n_field) != cscmap.N:
            raise ValueError("the mapping belongs to another field")
        self.cmap = cscmap
        self.n_btris = int(ids.size)
        dev = cscmap.device
        r = L.Robin()
        L.check(L.lib().emg_robin_init(self.n_btris, L.ctypes.byref(r)))
        self.desc = r
        self.d_keys = torch.empty(max(r.n_keys, 1), dtype=torch.int64, device=dev)
        self.d_vals = torch.empty(max(r.n_slots, 1), dtype=torch.complex128, device=dev)
        self._field, self._ids = field, ids
        if self.n_btris:
            self._nodes = _to_dev(m.nodes, torch.float64, dev)
            self._tris = _to_dev(m.tris, torch.int32, dev)
            self._t2e = _to_dev(m.tri_to_edge, torch.int32, dev)
            self._btris = _to_dev(ids, torch.int32, dev)
            self._status = torch.zeros(2, dtype=torch.int64, device=dev)
            build = L.lib().emg_abc2_build if kind == "abc2" else L.lib().emg_robin_build
            L.check(build(L.ctypes.byref(r), L.ptr(self._nodes), m.n_nodes, L.ptr(self._tris),
                                            L.ptr(self._t2e), m.n_tris, m.n_edges, L.ptr(self._btris),
                                            L.ptr(cscmap.d_indptr), L.ptr(cscmap.d_indices), cscmap.N,
                                            L.ptr(self.d_keys), L.ptr(self.d_vals), L.ptr(self._status),
                                            L.stream_handle(dev)))
            self._check("outside the assembled pattern or bad index")

    def _check(self, what: str) -> None:
        st = L.stream_handle(self.cmap.device)
        f, i = L.ctypes.c_int64(), L.ctypes.c_int64()
        L.check(L.lib().emg_status_read(L.ptr(self._status), L.ctypes.byref(f), L.ctypes.byref(i), st))
        if f.value:
            t = int(self._ids[i.value]) if 0 <= i.value < self._ids.size else i.value
            raise L.EmgMeshError(L.EMG_EMESH, f"boundary triangle {t}: "
                                 + (what if f.value & L.EMG_ST_INDEX else "degenerate triangle"))

    def quadrature_points(self) -> np.ndarray:
        """The 6 quadrature points of every listed triangle, f8[3, 6, n_btris]
        (generate_points_3d, robinbc.py:104-135): where the caller evaluates
        the incident field for ``force``."""
        m = self._field.mesh
        v = m.nodes[:, m.tris[:, self._ids]]  # (3, 3 vertices, nb)
        return np.einsum("dvn,vq->dqn", v, _TRI_L)

    def force(self, U, b: torch.Tensor | None = None) -> torch.Tensor:
        """Port forcing vector (assemble_robin_bc_bvec, robinbc.py:405-433):
        b (complex128 [N], device) += the triangles' entries for the incident
        field U (complex [3, 6, n_btris] at ``quadrature_points``)."""
        if self.kind != "robin":
            raise ValueError("only the Robin / port term has a forcing vector")
        dev = self.cmap.device
        if b is None:
            b = torch.zeros(self.cmap.N, dtype=torch.complex128, device=dev)
        if b.dtype != torch.complex128 or b.numel() != self.cmap.N:
            raise ValueError("b must be complex128 with N values")
        if not self.n_btris:
            return b
        if isinstance(U, torch.Tensor):
            Ud = U.to(device=dev, dtype=torch.complex128).contiguous()
        else:
            Ud = _to_dev(np.asarray(U, dtype=np.complex128), torch.complex128, dev)
        if tuple(Ud.shape) != (3, 6, self.n_btris):
            raise ValueError(f"U must have shape (3, 6, {self.n_btris})")
        r = self.desc
        fkeys = torch.empty(max(r.n_fkeys, 1), dtype=torch.int64, device=dev)
        fvals = torch.empty(max(r.n_fslots, 1), dtype=torch.complex128, device=dev)
        m = self._field.mesh
        self._status.zero_()
        L.check(L.lib().emg_robin_force(L.ctypes.byref(r), L.ptr(self._nodes), m.n_nodes, L.ptr(self._tris),
                                        L.ptr(self._t2e), m.n_tris, m.n_edges, L.ptr(self._btris), L.ptr(Ud),
                                        L.ptr(fkeys), L.ptr(fvals), L.ptr(b), self.cmap.N, L.ptr(self._status),
                                        L.stream_handle(dev)))
        self._check("bad index")
        return b

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

    def apply(self, A: torch.Tensor, gamma: complex, cscmap: GpuCSCMapping | None = None) -> torch.Tensor:
        """A[p] += gamma * (the term at p) on A's device values (complex128
        [nnz]); stream-ordered."""
        if cscmap is not None and cscmap is not self.cmap:
            raise ValueError("the boundary term was built on another mapping")
        if A.dtype != torch.complex128 or A.numel() < self.cmap.nnz:
            raise ValueError("A must be complex128 with nnz values")
        g = complex(gamma)
        L.check(L.lib().emg_robin_apply(L.ctypes.byref(self.desc), L.ptr(self.d_keys), L.ptr(self.d_vals), g.real,
                                        g.imag, L.ptr(A), self.cmap.nnz, L.stream_handle(self.cmap.device)))
        return A

    def to_device(self, gamma: complex = 1.0) -> torch.Tensor:
        """gamma times the term on A's pattern (complex128 [nnz], zeros off the
        boundary), e.g. the P of a frequency sweep."""
        out = torch.zeros(max(self.cmap.nnz, 1), dtype=torch.complex128, device=self.cmap.device)
        return self.apply(out, gamma)[: self.cmap.nnz]

    def to_csc(self, gamma: complex = 1.0) -> csc_matrix:
        """The term alone as a csc_matrix on A's pattern (explicit zeros off the
        boundary; the reference's generate_csc stores only the nonzeros)."""
        return self.cmap.to_csc(self * gamma)


def abc_order_2_matrix(field, tri_ids, coeff: complex, cscmap: GpuCSCMapping) -> LinComb:
    """``coeff`` times the second-order absorbing boundary correction of
    ``tri_ids`` as a lazy combination (the reference's abc_order_2_matrix,
    robin_abc_order2.py:259-281, added into its tri matrix and generate_csc'd,
    assembler.py:626-640), to be added to the element-value combination."""
    return RobinTerm(field, tri_ids, cscmap, kind="abc2") * coeff


def assemble_robin_bc(field, tri_ids, gamma: complex, cscmap: GpuCSCMapping) -> LinComb:
    """``gamma`` times the boundary term of ``tri_ids`` as a lazy combination
    (the reference's assemble_robin_bc + generate_csc, robinbc.py:436-451,
    femdata.py:104-118), to be added to the element-value combination."""
    return RobinTerm(field, tri_ids, cscmap) * gamma
