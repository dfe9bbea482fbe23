"""Post-processing on the device: the Nedelec-2 solution at points and the
port overlap integrals of the S-parameters.

Reference: ``ned2_tet_interp`` (compiled/base/interp.py:286-387) evaluates the
solution at points whose tets are known; the S-parameters integrate
(E - Q U) . conj(U) / (2 Z0) over each port face (physics/microwave/sparam.py:
62-97, mth/integrals.py:64-103), with E interpolated at the points of a
triangle rule and U the port mode. Here both run as kernels on the solution
vector in HBM (``emg_ned2_interp``, ``emg_port_overlap``); only the points,
the mode values and the scalar results cross to the host.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from .assembly import _device, _to_dev

__all__ = ["FieldOnDevice", "PortOverlap", "TRI_RULE_6"]

# The 6-point triangle rule (weights, L1, L2, L3) that the reference's
# surface integrals use at gq_order 5 and its Robin terms use throughout
# (robinbc.py:189-196).
TRI_RULE_6 = np.array([
    [0.10995174365532200, 0.10995174365532200, 0.10995174365532200, 0.22338158967801100, 0.22338158967801100,
     0.22338158967801100],
    [0.81684757298045896, 0.09157621350977101, 0.09157621350977101, 0.10810301816807000, 0.44594849091596500,
     0.44594849091596500],
    [0.09157621350977101, 0.81684757298045896, 0.09157621350977101, 0.44594849091596500, 0.10810301816807000,
     0.44594849091596500],
    [0.09157621350977004, 0.09157621350977008, 0.81684757298045807, 0.44594849091596500, 0.44594849091596500,
     0.10810301816807000]])


class FieldOnDevice:
    """The mesh arrays interpolation needs, on the device, for one field."""

    def __init__(self, field, device=None):
        m = field.mesh
        self.field = field
        self.device = _device(device)
        dev = self.device
        self.nodes = _to_dev(m.nodes, torch.float64, dev)
        self.tets = _to_dev(m.tets, torch.int32, dev)
        self.t2e = _to_dev(m.tet_to_edge, torch.int32, dev)
        self.t2t = _to_dev(m.tet_to_tri, torch.int32, dev)
        self.tris = _to_dev(m.tris, torch.int32, dev)
        self.n_nodes, self.n_tets, self.n_edges, self.n_tris = m.n_nodes, m.n_tets, m.n_edges, m.n_tris
        self.N = int(field.n_field)

    def _x(self, x) -> torch.Tensor:
        t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128))
        t = t.to(device=self.device, dtype=torch.complex128).contiguous()
        if t.numel() != self.N:
            raise ValueError(f"solution must have {self.N} values")
        return t

    def interpolate(self, x, points, tet_of) -> torch.Tensor:
        """The solution x at points f8[3, n] inside tets tet_of (int, -1 =
        outside -> NaN): complex128 [3, n] on the device."""
        xd = self._x(x)
        pts = _to_dev(np.asarray(points, dtype=np.float64), torch.float64, self.device)
        tt = _to_dev(np.asarray(tet_of, dtype=np.int64), torch.int32, self.device)
        n = int(pts.shape[1])
        out = torch.empty((3, n), dtype=torch.complex128, device=self.device)
        L.check(L.lib().emg_ned2_interp(L.ptr(self.nodes), self.n_nodes, L.ptr(self.tets), self.n_tets,
                                        L.ptr(self.t2e), L.ptr(self.t2t), self.n_edges, self.n_tris, L.ptr(xd),
                                        L.ptr(pts), n, L.ptr(tt), L.ptr(out), L.stream_handle(self.device)))
        return out


class PortOverlap:
    """Overlap integrals of a port face: for triangles ``tri_ids`` (each on
    the face of one tet) and a triangle rule, ``(x, U, q)`` gives
    sum over triangles of area * sum_k w_k (E - q U) . conj(U), E the solution
    x at the rule's points and U the port mode there (complex [3, nq, nb] at
    ``quadrature_points``). Dividing by 2 Z0 gives sparam_field_power."""

    def __init__(self, fod: FieldOnDevice, tri_ids, rule: np.ndarray = TRI_RULE_6):
        m = fod.field.mesh
        ids = np.asarray(tri_ids, dtype=np.int64).ravel()
        if ids.size and (ids.min() < 0 or ids.max() >= m.n_tris):
            raise IndexError("triangle id out of range")
        # the (lowest-numbered) tet each triangle is a face of
        owner = np.full(m.n_tris, m.n_tets, dtype=np.int64)
        np.minimum.at(owner, m.tet_to_tri.ravel(), np.tile(np.arange(m.n_tets), 4))
        self.tri_tets = owner[ids]
        if ids.size and self.tri_tets.max() >= m.n_tets:
            raise ValueError("a port triangle belongs to no tet")
        self.fod, self.ids = fod, ids
        self.rule = np.ascontiguousarray(rule, dtype=np.float64)
        if self.rule.ndim != 2 or self.rule.shape[0] != 4 or not 1 <= self.rule.shape[1] <= 16:
            raise ValueError("rule must be f8[4, nq] with 1 <= nq <= 16")
        dev = fod.device
        self.d_ids = _to_dev(ids, torch.int32, dev)
        self.d_tets = _to_dev(self.tri_tets, torch.int32, dev)
        self.status = torch.zeros(2, dtype=torch.int64, device=dev)

    @property
    def nq(self) -> int:
        return int(self.rule.shape[1])

    def quadrature_points(self) -> np.ndarray:
        """f8[3, nq, nb]: x = v1 L1 + v2 L2 + v3 L3 (generate_int_points_tri)."""
        m = self.fod.field.mesh
        v = m.nodes[:, m.tris[:, self.ids]]  # (3, 3, nb)
        return (v[:, 0][:, None, :] * self.rule[1][None, :, None] + v[:, 1][:, None, :] * self.rule[2][None, :, None]
                + v[:, 2][:, None, :] * self.rule[3][None, :, None])

    def __call__(self, x, U, q: float = 0.0):
        """(total complex, per-triangle complex128 [nb] on the device)."""
        fod = self.fod
        dev = fod.device
        nb = self.ids.size
        xd = fod._x(x)
        Ud = U if isinstance(U, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(U, dtype=np.complex128))
        Ud = Ud.to(device=dev, dtype=torch.complex128).contiguous()
        if tuple(Ud.shape) != (3, self.nq, nb):
            raise ValueError(f"U must have shape (3, {self.nq}, {nb})")
        per = torch.empty(max(nb, 1), dtype=torch.complex128, device=dev)
        tot = torch.empty(1, dtype=torch.complex128, device=dev)
        self.status.zero_()
        L.check(L.lib().emg_port_overlap(L.ptr(fod.nodes), fod.n_nodes, L.ptr(fod.tets), fod.n_tets, L.ptr(fod.t2e),
                                         L.ptr(fod.t2t), L.ptr(fod.tris), fod.n_edges, fod.n_tris, L.ptr(xd),
                                         L.ptr(self.d_ids), L.ptr(self.d_tets), nb,
                                         self.rule.ctypes.data_as(L.ctypes.POINTER(L.ctypes.c_double)), self.nq,
                                         L.ptr(Ud), float(q), L.ptr(per), L.ptr(tot), L.ptr(self.status),
                                         L.stream_handle(dev)))
        f, i = L.ctypes.c_int64(), L.ctypes.c_int64()
        L.check(L.lib().emg_status_read(L.ptr(self.status), L.ctypes.byref(f), L.ctypes.byref(i),
                                        L.stream_handle(dev)))
        if f.value:
            raise L.EmgMeshError(L.EMG_EMESH, f"port triangle index {i.value}: bad index")
        return complex(tot.cpu()[0]), per[:nb]
