"""Heat-conduction (Lagrange-2) assembly on the GPU: the drop-in for
physics/heatconduction/assembly/grad.py:403-462 as its assembler calls it
(physics/heatconduction/assembly/assembler.py:123-130)::

    Amat_coo, cscmap = tet_stiffness_matrix(field, cond_thermal)
    Amat = cscmap.to_csc(Amat_coo)
    Bmat_coo, cscmap = tet_mass_matrix(field, density * specific_heat)
    Bmat = cscmap.to_csc(Bmat_coo)

``field`` is anything with ``mesh`` (nodes f8[3, nN], tets [4, nT]),
``tet_to_field`` (int [10, nT]: 4 node DoFs then 6 edge DoFs; a partitioned
field may renumber them) and ``n_field``, such as the reference's Legrange2
or ``Legrange2`` below. The COO values stay on the device (``CooValues``,
100 per tet in the reference's row-major slot order); the mapping is a general
COO -> CSC one (``GpuCOOMapping``), also usable for any other slot list.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.sparse import csc_matrix

from . import _lib as L
from .assembly import _device, _prec, _to_dev

__all__ = ["Legrange2", "CooValues", "GpuCOOMapping", "tet_stiffness_matrix", "tet_mass_matrix"]


class Legrange2:
    """The Lagrange-2 DoF numbering of elements/leg2.py:48-73: node DoFs
    0..nN-1, then edge DoFs nN + edge index."""

    def __init__(self, mesh):
        self.mesh = mesh
        self.n_field = int(mesh.n_nodes + mesh.n_edges)
        self.tet_to_field = np.concatenate([np.asarray(mesh.tets), np.asarray(mesh.tet_to_edge) + mesh.n_nodes]
                                           ).astype(np.int64)


class CooValues:
    """COO slot values on the device (f8 or c16): 100 per tet, either in the
    reference's row-major blocks or (``transposed``, as the element kernels
    write them for the gather) with each tet's block transposed. ``np.asarray``
    gives the reference layout; arithmetic stays on the device."""

    def __init__(self, values: torch.Tensor, layout, transposed: bool = False):
        self.values = values
        self.layout = layout
        self.transposed = bool(transposed)

    def __len__(self):
        return int(self.values.numel())

    def _wrap(self, v):
        return CooValues(v, self.layout, self.transposed)

    def _flip(self, v: torch.Tensor) -> torch.Tensor:
        return v.view(-1, 10, 10).transpose(1, 2).reshape(-1)

    def reference_layout(self) -> torch.Tensor:
        """The values in the reference's slot order (device)."""
        return self._flip(self.values) if self.transposed else self.values

    def _other(self, o):
        if isinstance(o, CooValues):
            if o.layout is not self.layout:
                raise ValueError("COO values of different slot layouts")
            if o.transposed == self.transposed:
                return o.values
            return self._flip(o.values)
        if isinstance(o, (np.ndarray, torch.Tensor)) and np.ndim(o) > 0:
            t = o if isinstance(o, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(o))
            t = t.to(self.values.device).reshape(-1)
            if t.numel() != self.values.numel():
                raise ValueError("COO arrays differ in length")
            return self._flip(t) if self.transposed else t
        return o

    def __add__(self, o):
        return self._wrap(self.values + self._other(o))

    __radd__ = __add__

    def __sub__(self, o):
        return self._wrap(self.values - self._other(o))

    def __rsub__(self, o):
        return self._wrap(self._other(o) - self.values)

    def __mul__(self, c):
        if isinstance(c, CooValues) or np.ndim(c) > 0:
            raise TypeError("only scalar multiples of COO values")
        return self._wrap(self.values * c)

    __rmul__ = __mul__

    def __truediv__(self, c):
        return self._wrap(self.values / c)

    def __neg__(self):
        return self._wrap(-self.values)

    def __array__(self, dtype=None, copy=None):
        a = self.reference_layout().cpu().numpy()
        return a if dtype is None else a.astype(dtype)


class GpuCOOMapping:
    """``CSCMapping.from_rowcol(rows, cols, N)`` (mth/csc_cast.py:51-177) on
    the device. Entries are the distinct (row, col) pairs, rows ascending in
    each column; an entry's value is the sum of its slots in slot order.
    ``indptr``/``indices`` are int32 as the reference's csc_matrix holds
    them."""

    def __init__(self, d_rows: torch.Tensor, d_cols: torch.Tensor, N: int, device=None):
        dev = d_rows.device
        self.device = dev
        self.N = int(N)
        S = int(d_rows.numel())
        if d_cols.numel() != S:
            raise ValueError("rows and cols differ in length")
        self.block_dofs = 0  # 10 when the slots are 10x10 blocks per tet (from_tet_to_field)
        m = L.CooMap()
        L.check(L.lib().emg_coo_init(S, self.N, L.ctypes.byref(m)))
        self.desc = m
        self.S = S
        self._rows = d_rows.to(torch.int32).contiguous()
        cols = d_cols.to(torch.int32).contiguous()
        self.d_perm = torch.empty(m.perm_bytes // 4, dtype=torch.int32, device=dev)
        ws = torch.empty(max(m.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        self.d_indptr = torch.empty(self.N + 1, dtype=torch.int32, device=dev)
        status = torch.zeros(2, dtype=torch.int64, device=dev)
        st = L.stream_handle(dev)
        L.check(L.lib().emg_coo_build(L.ctypes.byref(m), L.ptr(self._rows), L.ptr(cols), L.ptr(self.d_perm),
                                      L.ptr(ws), L.ptr(self.d_indptr), L.ptr(status), st))
        self.nnz = int(m.nnz)
        self.d_indices = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        self.d_run = torch.empty(self.nnz + 1, dtype=torch.int32, device=dev)
        L.check(L.lib().emg_coo_finish(L.ctypes.byref(m), L.ptr(self._rows), L.ptr(self.d_perm), L.ptr(ws),
                                       L.ptr(self.d_indptr), L.ptr(self.d_indices), L.ptr(self.d_run), st))
        self._rows = None  # the rows live on in d_indices
        self._indptr = self._indices = None

    @staticmethod
    def from_rowcol(rows, cols, N: int, device=None) -> "GpuCOOMapping":
        """The mapping of a slot list (int rows, cols in [0, N); numpy arrays
        or device tensors). Indices are checked before they are narrowed to
        int32, so none can wrap into range."""
        dev = _device(device)
        out = []
        for a in (rows, cols):
            if isinstance(a, torch.Tensor):
                if a.numel() and (int(a.min()) < 0 or int(a.max()) >= N):
                    raise L.EmgMeshError(L.EMG_EMESH, "COO index outside [0, N)")
                out.append(a.to(device=dev, dtype=torch.int32))
            else:
                h = np.asarray(a)
                if h.size and (h.min() < 0 or h.max() >= N):
                    raise L.EmgMeshError(L.EMG_EMESH, "COO index outside [0, N)")
                out.append(_to_dev(h, torch.int32, dev))
        return GpuCOOMapping(out[0], out[1], N)

    @staticmethod
    def from_tet_to_field(tet_to_field, N: int, device=None) -> "GpuCOOMapping":
        """The slots of ``D x D`` element blocks: slot D^2 t + D i + j has row
        t2f[i, t] and column t2f[j, t] (grad.py:350-354)."""
        dev = _device(device)
        t2f = np.asarray(tet_to_field)
        D, nT = t2f.shape
        if t2f.size and (t2f.min() < 0 or t2f.max() >= N):
            raise IndexError("tet_to_field entry outside [0, N)")
        d_t2f = _to_dev(t2f, torch.int32, dev)
        S = D * D * nT
        rows = torch.empty(max(S, 1), dtype=torch.int32, device=dev)
        cols = torch.empty(max(S, 1), dtype=torch.int32, device=dev)
        L.check(L.lib().emg_coo_rowcol(L.ptr(d_t2f), int(D), int(nT), L.ptr(rows), L.ptr(cols),
                                       L.stream_handle(dev)))
        cm = GpuCOOMapping(rows[:S], cols[:S], N)
        cm.block_dofs = int(D)
        return cm

    @property
    def indptr(self) -> np.ndarray:
        if self._indptr is None:
            self._indptr = self.d_indptr.cpu().numpy()
        return self._indptr

    @property
    def indices(self) -> np.ndarray:
        if self._indices is None:
            self._indices = self.d_indices[: self.nnz].cpu().numpy()
        return self._indices

    def to_device(self, data) -> torch.Tensor:
        """CSC values on the device (f8, or c16 for complex slot values)."""
        block = 0
        if isinstance(data, CooValues):
            v = data.values
            if data.transposed:
                if self.block_dofs != 10:
                    raise ValueError("transposed block values need a mapping of 10x10 element blocks")
                block = 10
        elif isinstance(data, torch.Tensor):
            v = data
        else:
            a = np.asarray(data)
            v = _to_dev(a, torch.complex128 if np.iscomplexobj(a) else torch.float64, self.device)
        v = v.to(self.device)
        cplx = v.is_complex()
        v = v.to(torch.complex128 if cplx else torch.float64).contiguous()
        if v.numel() != self.S:
            raise ValueError(f"{v.numel()} slot values for a mapping of {self.S} slots")
        out = torch.empty(max(self.nnz, 1), dtype=v.dtype, device=self.device)
        L.check(L.lib().emg_coo_gather(L.ctypes.byref(self.desc), L.ptr(self.d_perm), L.ptr(self.d_run),
                                       1 if cplx else 0, block, L.ptr(v), L.ptr(out),
                                       L.stream_handle(self.device)))
        return out[: self.nnz]

    def to_csc(self, data, out: np.ndarray | None = None) -> csc_matrix:
        """``CSCMapping.to_csc`` (csc_cast.py:55-63); ``out``: an optional
        host array (f8 or c16 [nnz], matching the values) to receive them, as
        ``GpuCSCMapping.to_csc``."""
        d = self.to_device(data)
        if out is None:
            host = torch.empty(d.shape, dtype=d.dtype, pin_memory=True)
            host.copy_(d)
            vals = host.numpy()
        else:
            want = np.complex128 if d.is_complex() else np.float64
            if out.dtype != want or out.shape != (self.nnz,) or not out.flags["C_CONTIGUOUS"]:
                raise ValueError(f"out must be a contiguous {np.dtype(want).name} array of {self.nnz} values")
            torch.from_numpy(out).copy_(d)
            vals = out
        return csc_matrix((vals, self.indices, self.indptr), shape=(self.N, self.N))


class _HeatMesh:
    """Nodes, tets and the COO mapping of one field, kept on the device and
    reused by the stiffness and mass calls of that field."""

    def __init__(self, field, device):
        m = field.mesh
        t2f = np.asarray(field.tet_to_field)
        if t2f.ndim != 2 or t2f.shape[0] != 10:
            raise ValueError("tet_to_field must be [10, n_tets]")
        self.n_nodes, self.n_tets = int(m.n_nodes), int(np.asarray(m.tets).shape[1])
        if t2f.shape[1] != self.n_tets:
            raise ValueError("tet_to_field and mesh.tets differ in tet count")
        self.nodes = _to_dev(np.asarray(m.nodes, dtype=np.float64), torch.float64, device)
        t = np.asarray(m.tets)
        if t.size and (t.min() < 0 or t.max() >= self.n_nodes):  # before narrowing to int32
            raise IndexError("tet node index outside [0, n_nodes)")
        self.tets = _to_dev(t, torch.int32, device)
        self.cmap = GpuCOOMapping.from_tet_to_field(t2f, int(field.n_field), device)
        self.key = (id(m.nodes), id(m.tets), id(field.tet_to_field), int(field.n_field))


_CACHE: dict = {}


def _heat_mesh(field, device) -> _HeatMesh:
    dev = _device(device)
    h = _CACHE.get(id(field))
    key = (id(field.mesh.nodes), id(field.mesh.tets), id(field.tet_to_field), int(field.n_field))
    if h is None or h[0] is not field or h[1].key != key or h[1].nodes.device != dev:
        _CACHE.clear()  # one field resident at a time
        h = (field, _HeatMesh(field, dev))
        _CACHE[id(field)] = h
    return h[1]


def _element(field, coef: np.ndarray, kind: int, precision: str, device) -> tuple[CooValues, GpuCOOMapping]:
    prec = _prec(precision)
    if prec == L.EMG_MIXED:
        raise ValueError("the heat elements come in 'fp64' (the reference's quadrature loop) and 'exact' (moments)")
    hm = _heat_mesh(field, device)
    dev = hm.nodes.device
    d_coef = _to_dev(np.ascontiguousarray(coef, dtype=np.float64), torch.float64, dev)
    vals = torch.empty(max(100 * hm.n_tets, 1), dtype=torch.float64, device=dev)
    status = torch.zeros(2, dtype=torch.int64, device=dev)
    st = L.stream_handle(dev)
    L.check(L.lib().emg_leg2_element(L.ptr(hm.nodes), hm.n_nodes, L.ptr(hm.tets), hm.n_tets, L.ptr(d_coef), kind,
                                     prec, L.EMG_LAYOUT_COO_T, L.ptr(vals), L.ptr(status), st))
    f, i = L.ctypes.c_int64(), L.ctypes.c_int64()
    L.check(L.lib().emg_status_read(L.ptr(status), L.ctypes.byref(f), L.ctypes.byref(i), st))
    if f.value:
        raise L.EmgMeshError(L.EMG_EMESH, f"tet {i.value}: "
                             + ("bad node index" if f.value & L.EMG_ST_INDEX else "degenerate tet"))
    return CooValues(vals[: 100 * hm.n_tets], hm.cmap, transposed=True), hm.cmap


def tet_stiffness_matrix(field, cond_termal: np.ndarray, *, precision: str = "fp64",
                         device=None) -> tuple[CooValues, GpuCOOMapping]:
    """Drop-in for grad.py:403-437: the stiffness COO values
    K_ij = V sum_q w_q (k grad N_i) . grad N_j per tet (conductivity
    f8[3, 3, n_tets]) and the COO -> CSC mapping. ``precision``: 'fp64' runs
    the reference's quadrature loop in its operation order; 'exact' folds the
    same rule into 16 gradient products per tet (translation invariant; about
    30x fewer operations)."""
    c = np.asarray(cond_termal, dtype=np.float64)
    nT = np.asarray(field.mesh.tets).shape[1]
    if c.shape != (3, 3, nT):
        raise ValueError(f"cond_termal must be (3, 3, {nT})")
    return _element(field, c, 0, precision, device)


def tet_mass_matrix(field, rho_cp: np.ndarray, *, precision: str = "fp64",
                    device=None) -> tuple[CooValues, GpuCOOMapping]:
    """Drop-in for grad.py:440-462: the capacity COO values
    M_ij = rho_cp V sum_q w_q N_i N_j per tet and the COO -> CSC mapping
    ('exact': rho_cp V times the rule's constant 10x10 block)."""
    r = np.asarray(rho_cp, dtype=np.float64).ravel()
    nT = np.asarray(field.mesh.tets).shape[1]
    if r.shape != (nT,):
        raise ValueError(f"rho_cp must have {nT} values")
    return _element(field, r, 1, precision, device)
