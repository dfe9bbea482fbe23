"""Drop-in for EMerge's Nedelec-2 volume assembly on a B200.

Reference call site (physics/microwave/assembly/assembler.py:485-494)::

    Evec, Bvec, cscmap = tet_mass_stiffness_matrices(field, er, ur, conductor_tets, self.cached_cscmap)
    K = self.cached_cscmap.to_csc(Evec - Bvec * (K0**2))

``tet_mass_stiffness_matrices`` here has the same signature and meaning as
curlcurl.py:222-270. It returns two lazy, device-backed element-value objects
(the reference's COO arrays ``dataE`` = K and ``dataB`` = M) and a
``GpuCSCMapping`` (the reference's ``CSCMapping``, csc_cast.py:29-63). The
caller's ``Evec - Bvec * k0**2`` builds a lazy combination; ``to_csc`` runs
the fused element kernel + column gather on the GPU and returns a
``scipy.sparse.csc_matrix`` with the reference's indptr/indices (int32) and
complex128 data. ``np.asarray(Evec)`` materialises the reference COO layout.

Differences from the reference, on purpose:
* a zero-volume, non-finite or index-invalid tet raises ``EmgMeshError``
  (the reference silently produces inf/NaN entries);
* ``precision="fp64"`` (default) reproduces the reference's own FP64
  arithmetic; ``"mixed"`` keeps the geometry in FP64 and contracts the
  quadrature's (exact, precomputed) sums of basis products with the tet's
  tensors in FP32 (relative error <= 1e-6 against FP64, and closer than
  FP64 to the exact integrals on sliver tets); ``"exact"`` evaluates the element integrals
  in closed form, free of the reference's absolute-coordinate cancellation
  (it then differs from the reference by the reference's rounding error).
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.sparse import csc_matrix

from . import _lib as L

__all__ = ["tet_mass_stiffness_matrices", "GpuCSCMapping", "ElemValues", "LinComb", "DeviceMesh", "DeviceMaterial",
           "classify_material"]


def _device(device) -> torch.device:
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("emerge_b200 needs a CUDA device (there is no CPU fallback)")
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError("emerge_b200 runs on CUDA devices only")
    return d


_NP = {torch.float64: np.float64, torch.int32: np.int32, torch.int64: np.int64, torch.complex128: np.complex128,
       torch.complex64: np.complex64, torch.uint8: np.uint8}


def _empty(numel: int, dtype: torch.dtype, dev: torch.device, alloc=None) -> torch.Tensor:
    """Device tensor of numel elements: from ``alloc(numel, dtype)`` when the
    caller manages device memory itself (e.g. a serving arena), else torch."""
    if alloc is not None:
        return alloc(int(numel), dtype)
    return torch.empty(int(numel), dtype=dtype, device=dev)


def _to_dev(a: np.ndarray, dtype: torch.dtype, dev: torch.device, alloc=None) -> torch.Tensor:
    if alloc is None:
        return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dtype, non_blocking=False)
    h = np.ascontiguousarray(a, dtype=_NP[dtype])
    t = alloc(int(h.size), dtype)
    t.copy_(torch.from_numpy(h.reshape(-1)))
    return t.view(h.shape)


def _prec(precision: str) -> int:
    p = {"fp64": L.EMG_FP64, "plain": L.EMG_FP64, "mixed": L.EMG_MIXED,
         "exact": L.EMG_EXACT}.get(str(precision).lower())
    if p is None:
        raise ValueError(f"precision must be 'fp64', 'mixed' or 'exact', got {precision!r}")
    return p


class DeviceMesh:
    """Device copies of the mesh arrays the path reads (int32 SoA)."""

    def __init__(self, field, conductor_tets=None, device=None, alloc=None, reuse: "DeviceMesh | None" = None):
        dev = _device(device)
        mesh = field.mesh
        self.device = dev
        self.alloc = alloc
        self.n_nodes = int(mesh.nodes.shape[1])
        self.n_tets = int(mesh.tets.shape[1])
        self.n_edges = int(mesh.edges.shape[1])
        self.n_tris = int(mesh.tris.shape[1])
        self.N = int(field.n_field)
        self.N_volume = 2 * self.n_edges + 2 * self.n_tris
        if self.N < self.N_volume:
            raise ValueError("only the SECOND_MIXED_VOLAKIS space (n_field = 2E + 2F) is supported")
        if self.N > self.N_volume:
            # a partitioned field (ThinConductor, nedelec2.py:114-172): the
            # volume assembly keeps the map from before the split
            # (curlcurl.py:244) and the pattern's extra columns stay empty
            _check_volume_map(field, mesh)
        dc = np.asarray(field.dofcodes3d)
        if dc.shape != (20,) or not np.array_equal(dc, [64] * 6 + [66] * 6 + [128] * 4 + [129] * 4):
            raise ValueError(f"unsupported dofcodes {dc.tolist()} (expected SECOND_MIXED_VOLAKIS)")
        self.nodes = _to_dev(mesh.nodes, torch.float64, dev, alloc)
        # the device tets of ``reuse`` (a mapping's own mesh) when the caller
        # passes the very same tet array again, as the reference does with its
        # cached CSCMapping on every frequency; coordinates are always copied
        if (reuse is not None and reuse._field.mesh.tets is mesh.tets and reuse.device == dev
                and reuse.n_tets == self.n_tets):
            self.tets = reuse.tets
        else:
            t = np.asarray(mesh.tets)
            if t.size and (t.min() < 0 or t.max() >= self.n_nodes):  # before narrowing to int32
                raise IndexError("tet node index outside [0, n_nodes)")
            self.tets = _to_dev(t, torch.int32, dev, alloc)
        self.tetids_host = _tet_assy(self.n_tets, conductor_tets)
        self.n_assy = int(self.tetids_host.shape[0]) if self.tetids_host is not None else self.n_tets
        self.tetids = _to_dev(self.tetids_host, torch.int32, dev, alloc) if self.tetids_host is not None else None
        self._field = field
        self.status = _empty(2, torch.int64, dev, alloc)
        self.status.zero_()

    def topology(self):
        mesh = self._field.mesh
        return (_to_dev(mesh.tet_to_edge, torch.int32, self.device, self.alloc),
                _to_dev(mesh.tet_to_tri, torch.int32, self.device, self.alloc))

    def check_status(self, stream=None):
        f, i = L.ctypes.c_int64(), L.ctypes.c_int64()
        L.check(L.lib().emg_status_read(L.ptr(self.status), L.ctypes.byref(f), L.ctypes.byref(i),
                                        stream or L.stream_handle(self.device)))
        if f.value:
            what = []
            if f.value & L.EMG_ST_INDEX:
                what.append("index out of range")
            if f.value & L.EMG_ST_DEGENERATE:
                what.append("degenerate (zero-volume / repeated-vertex / non-finite) tet")
            if f.value & L.EMG_ST_CAPACITY:
                what.append("capacity exceeded")
            raise L.EmgMeshError(L.EMG_EMESH, f"{', '.join(what)} at assembled index {i.value}")

    def reset_status(self):
        L.check(L.lib().emg_status_reset(L.ptr(self.status), L.stream_handle(self.device)))


def _check_volume_map(field, mesh) -> None:
    """get_tet_to_field() of a partitioned field must be the unsplit map
    (rows: tet_to_edge, + E, tet_to_tri + 2E, + 2E + F)."""
    t2f = np.asarray(field.get_tet_to_field())
    E, F = int(mesh.edges.shape[1]), int(mesh.tris.shape[1])
    t2e, t2t = np.asarray(mesh.tet_to_edge), np.asarray(mesh.tet_to_tri)
    ok = (t2f.shape == (20, t2e.shape[1]) and np.array_equal(t2f[0:6], t2e) and np.array_equal(t2f[6:12], t2e + E)
          and np.array_equal(t2f[12:16], t2t + 2 * E) and np.array_equal(t2f[16:20], t2t + 2 * E + F))
    if not ok:
        raise ValueError("a partitioned field must keep its unsplit tet_to_field for the volume assembly")


def _tet_assy(nT: int, conductor_tets):
    """tet_assy of curlcurl.py:248-250 (None = all tets)."""
    if conductor_tets is None:
        return None
    c = np.asarray(conductor_tets, dtype=np.int64).ravel()
    if c.size == 0:
        return None
    if c.min() < 0 or c.max() >= nT:
        raise IndexError("conductor tet index out of range")
    return np.delete(np.arange(nT, dtype=np.int64), c).astype(np.int32)


def classify_material(t: np.ndarray) -> int:
    """EMG_MAT_ISO / DIAG / FULL for a c16[3,3,nT] tensor array."""
    off = [(0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)]
    if any(np.any(t[i, j] != 0) for i, j in off):
        return L.EMG_MAT_FULL
    if np.array_equal(t[0, 0], t[1, 1]) and np.array_equal(t[1, 1], t[2, 2]):
        return L.EMG_MAT_ISO
    return L.EMG_MAT_DIAG


def _is_identity(t: np.ndarray) -> bool:
    off = [(0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)]
    return (all(not np.any(t[i, j] != 0) for i, j in off) and all(np.all(t[d, d] == 1) for d in range(3)))


def material_kind(t: np.ndarray) -> tuple:
    """(``classify_material(t)``, ``_is_identity(t)``) in one multi-threaded
    native pass (emg_material_classify); t is c16[3, 3, nT]."""
    a = np.ascontiguousarray(t, dtype=np.complex128)
    k, i = L.ctypes.c_int(), L.ctypes.c_int()
    L.check(L.lib().emg_material_classify(a.ctypes.data_as(L.ctypes.c_void_p), int(a.shape[2]), 0,
                                          L.ctypes.byref(k), L.ctypes.byref(i)))
    return int(k.value), bool(i.value)


class DeviceMaterial:
    """Per-tet er, ur in the compact layout of their kind (see emg_material).

    er, ur: the reference's c16[3, 3, nT] tensors, or (for callers that hold
    isotropic materials only, such as a serving request) er as c16[nT]
    scalars with ur None (mu_r = 1) or c16[nT]."""

    def __init__(self, er: np.ndarray, ur: np.ndarray | None, n_tets: int, device, alloc=None):
        er = np.asarray(er)
        if er.ndim == 1:
            if er.shape != (n_tets,) or (ur is not None and np.shape(ur) != (n_tets,)):
                raise ValueError(f"scalar er/ur must have shape ({n_tets},)")
            self.kind = L.EMG_MAT_ISO
            self.er = _to_dev(er.astype(np.complex128, copy=False), torch.complex128, device, alloc)
            self.ur = (None if ur is None
                       else _to_dev(np.asarray(ur).astype(np.complex128, copy=False), torch.complex128, device, alloc))
            self.h2d_bytes = self.er.numel() * 16 + (self.ur.numel() * 16 if self.ur is not None else 0)
            return
        ur = np.asarray(ur)
        if er.shape != (3, 3, n_tets) or ur.shape != (3, 3, n_tets):
            raise ValueError(f"er/ur must have shape (3, 3, {n_tets})")
        kind, _ = material_kind(er)
        ur_kind, ur_id = material_kind(ur)
        if not ur_id:
            kind = max(kind, ur_kind)
        self.kind = kind

        def pack(t):
            if kind == L.EMG_MAT_ISO:
                return _to_dev(t[0, 0].astype(np.complex128, copy=False), torch.complex128, device, alloc)
            if kind == L.EMG_MAT_DIAG:
                return _to_dev(np.stack([t[0, 0], t[1, 1], t[2, 2]]).astype(np.complex128, copy=False),
                               torch.complex128, device, alloc)
            return _to_dev(t.astype(np.complex128, copy=False), torch.complex128, device, alloc)

        self.er = pack(er)
        self.ur = None if ur_id else pack(ur)
        self.h2d_bytes = self.er.numel() * 16 + (self.ur.numel() * 16 if self.ur is not None else 0)

    def struct(self) -> L.Material:
        return L.Material(self.kind, self.er.data_ptr(), self.ur.data_ptr() if self.ur is not None else None)


class _Job:
    """Mesh + materials + precision of one tet_mass_stiffness_matrices call."""

    def __init__(self, dmesh: DeviceMesh, dmat: DeviceMaterial, precision: int):
        self.mesh, self.mat, self.precision = dmesh, dmat, precision


class ElemValues:
    """Lazy element values in the reference COO layout (curlcurl.py:449-455):
    ``which`` = 'K' (the reference's dataE) or 'M' (dataB)."""

    def __init__(self, job: _Job, which: str):
        self.job, self.which = job, which
        self.shape = (400 * job.mesh.n_assy,)
        self.dtype = np.dtype(np.complex128)

    def __len__(self):
        return self.shape[0]

    def _lc(self) -> "LinComb":
        return LinComb(self.job, {self.which: 1.0 + 0.0j})

    def __mul__(self, c):
        return self._lc() * c

    __rmul__ = __mul__

    def __truediv__(self, c):
        return self._lc() * (1.0 / c)

    def __neg__(self):
        return self._lc() * -1.0

    def __add__(self, o):
        return self._lc() + o

    __radd__ = __add__

    def __sub__(self, o):
        return self._lc() - o

    def __rsub__(self, o):
        return (-self) + o

    def to_device(self) -> torch.Tensor:
        """Element values on the device, complex128 [400*nA] (complex64 for
        the mixed form)."""
        job = self.job
        m = job.mesh
        dt = torch.complex64 if job.precision == L.EMG_MIXED else torch.complex128
        out = torch.empty(400 * m.n_assy, dtype=dt, device=m.device)
        mat = job.mat.struct()
        m.reset_status()
        L.check(L.lib().emg_element_values(
            L.ptr(m.nodes), m.n_nodes, L.ptr(m.tets), m.n_tets, L.ptr(m.tetids), m.n_assy, L.ctypes.byref(mat),
            job.precision, L.EMG_OUT_K if self.which == "K" else L.EMG_OUT_M, L.EMG_LAYOUT_COO, 0.0, 0.0, 0.0, 0.0,
            L.ptr(out), L.ptr(m.status), L.stream_handle(m.device)))
        m.check_status()
        return out

    def __array__(self, dtype=None, copy=None):
        a = self.to_device().to(torch.complex128).cpu().numpy()
        return a if dtype is None else a.astype(dtype)


class LinComb:
    """alpha*K + beta*M built lazily by the caller's arithmetic."""

    def __init__(self, job: _Job, coef: dict):
        self.job, self.coef = job, dict(coef)

    def _other(self, o):
        """(job, coef) of the other operand, or NotImplemented."""
        if isinstance(o, ElemValues) or getattr(o, "_is_robin_term", False) or getattr(o, "_is_opposite_term", False):
            o = o._lc()
        if not isinstance(o, LinComb):
            return NotImplemented
        if self.job is not None and o.job is not None and o.job is not self.job:
            raise ValueError("element values of different assemblies cannot be combined")
        return (self.job if self.job is not None else o.job), o.coef

    def __add__(self, o):
        r = self._other(o)
        if r is NotImplemented:
            return NotImplemented
        job, oc = r
        c = dict(self.coef)
        for k, v in oc.items():
            c[k] = c.get(k, 0) + v
        return LinComb(job, c)

    __radd__ = __add__

    def __sub__(self, o):
        r = self._other(o)
        if r is NotImplemented:
            return NotImplemented
        job, oc = r
        c = dict(self.coef)
        for k, v in oc.items():
            c[k] = c.get(k, 0) - v
        return LinComb(job, c)

    def __rsub__(self, o):
        return (-self) + o

    def __mul__(self, s):
        if not np.isscalar(s):
            return NotImplemented
        return LinComb(self.job, {k: v * complex(s) for k, v in self.coef.items()})

    __rmul__ = __mul__

    def __neg__(self):
        return self * -1.0

    @property
    def alpha(self) -> complex:
        return complex(self.coef.get("K", 0.0))

    @property
    def beta(self) -> complex:
        return complex(self.coef.get("M", 0.0))

    @property
    def robin_terms(self) -> list:
        """(RobinTerm, gamma) pairs of the combination."""
        return [(k, complex(v)) for k, v in self.coef.items() if getattr(k, "_is_robin_term", False)]

    @property
    def opposite_terms(self) -> list:
        """(OppositeSideTerm, gamma) pairs of the combination."""
        return [(k, complex(v)) for k, v in self.coef.items() if getattr(k, "_is_opposite_term", False)]

    def without_opposite(self) -> "LinComb":
        return LinComb(self.job, {k: v for k, v in self.coef.items() if not getattr(k, "_is_opposite_term", False)})

    def __array__(self, dtype=None, copy=None):
        if self.robin_terms or self.opposite_terms:
            raise TypeError("a combination with a boundary term has no tet COO layout; use cscmap.to_csc")
        K = np.asarray(ElemValues(self.job, "K"))
        M = np.asarray(ElemValues(self.job, "M"))
        a = self.alpha * K + self.beta * M
        return a if dtype is None else a.astype(dtype)


class GpuCSCMapping:
    """The reference's ``CSCMapping`` (csc_cast.py:29-63) on the GPU: the
    sparsity pattern (indptr, indices: bit-identical to the reference's) and
    the column-gather plan, built once per mesh and assembled-tet set.

    ``value_layout``: the element values the assembly writes and gathers --
    ``"block"`` (default: per tet the 2x2 blocks of its 55 entity pairs, one
    4-byte record and one contiguous read per four entries of A) or
    ``"packed"`` (the canonical upper triangle, one record per two entries,
    ``record_bytes`` 8 or 4). A is bit for bit the same in both."""

    def __init__(self, dmesh: DeviceMesh, chunk_order: str = "morton", record_bytes: int = 8,
                 value_layout: str = "block"):
        if chunk_order not in ("morton", "interleave"):
            raise ValueError(f"chunk_order must be 'morton' or 'interleave', got {chunk_order!r}")
        if value_layout not in ("packed", "block"):
            raise ValueError(f"value_layout must be 'packed' or 'block', got {value_layout!r}")
        lib = L.lib()
        m = dmesh
        self.device = m.device
        self.N = m.N
        self.n_assy = m.n_assy
        self._mesh_key = (m.n_nodes, m.n_tets, m.n_edges, m.n_tris,
                          None if m.tetids_host is None else hash(m.tetids_host.tobytes()))
        plan = L.Plan()
        L.check(lib.emg_plan_init(m.n_tets, m.n_assy, m.n_edges, m.n_tris, L.ctypes.byref(plan)))
        if record_bytes == 4 and m.n_assy * 210 >= (1 << 31):
            record_bytes = 8  # too many tets for the compact record
        L.check(lib.emg_plan_set_record_width(L.ctypes.byref(plan), int(record_bytes)))
        if value_layout == "block":
            L.check(lib.emg_plan_set_value_layout(L.ctypes.byref(plan), L.EMG_LAYOUT_BLOCK))
        self.value_layout = value_layout
        self.plan = plan
        self.alloc = m.alloc
        self.d_plan = _empty(max(plan.plan_bytes, 1), torch.uint8, m.device, m.alloc)
        ws = _empty(max(plan.workspace_bytes, 1), torch.uint8, m.device, m.alloc)
        self.d_indptr = _empty(self.N + 1, torch.int32, m.device, m.alloc)
        t2e, t2t = m.topology()
        st = L.stream_handle(m.device)
        L.check(lib.emg_plan_build(L.ctypes.byref(plan), L.ptr(m.tets), L.ptr(t2e), L.ptr(t2t), L.ptr(m.tetids),
                                   L.ptr(self.d_plan), L.ptr(ws), L.ptr(self.d_indptr), L.ptr(m.status), st))
        self.nnz = int(plan.nnz)
        if self.N > m.N_volume:  # the split DoFs' columns of a partitioned field are empty
            self.d_indptr[m.N_volume + 1:].fill_(self.nnz)
        self.d_indices = _empty(max(self.nnz, 1), torch.int32, m.device, m.alloc)
        L.check(lib.emg_plan_finish(L.ctypes.byref(plan), L.ptr(t2e), L.ptr(t2t), L.ptr(m.tetids),
                                    L.ptr(self.d_plan), L.ptr(self.d_indptr), L.ptr(self.d_indices),
                                    L.ptr(m.status), st))
        if chunk_order == "morton":
            L.check(lib.emg_plan_order(L.ctypes.byref(plan), L.ptr(self.d_plan), L.ptr(m.nodes), m.n_nodes,
                                       L.ptr(m.tets), L.ptr(m.tetids), L.ptr(ws), st))
        del ws
        m.check_status()
        self._indptr = self._indices = None
        self.dmesh = m  # its device tets are shared with later calls on the same tet array
        self._ws = None
        self._ws_prec = None

    @property
    def indptr(self) -> np.ndarray:
        """Host copy of the CSC column pointers (int32 [N+1]), made on first use."""
        if self._indptr is None:
            self._indptr = self.d_indptr.cpu().numpy()
        return self._indptr

    @property
    def indices(self) -> np.ndarray:
        """Host copy of the CSC row indices (int32 [nnz]), made on first use."""
        if self._indices is None:
            self._indices = self.d_indices[: self.nnz].cpu().numpy()
        return self._indices

    @staticmethod
    def from_field(field, conductor_tets=None, device=None) -> "GpuCSCMapping":
        return GpuCSCMapping(DeviceMesh(field, conductor_tets, device))

    def _check_job(self, job: _Job):
        m = job.mesh
        key = (m.n_nodes, m.n_tets, m.n_edges, m.n_tris,
               None if m.tetids_host is None else hash(m.tetids_host.tobytes()))
        if key != self._mesh_key:
            raise ValueError("element values belong to a different mesh / conductor set than this mapping")

    def workspace(self, precision: int) -> torch.Tensor:
        need = L.lib().emg_assemble_workspace_size(self.n_assy, precision)
        if self._ws is None or self._ws.numel() < need:
            self._ws = _empty(max(need, 1), torch.uint8, self.device, self.alloc)
        return self._ws

    def assemble_device(self, job: _Job, alpha: complex, beta: complex, out: torch.Tensor | None = None):
        """A = alpha*K + beta*M values (complex128, CSC order) on the device;
        stream-ordered, no synchronisation."""
        self._check_job(job)
        m = job.mesh
        if out is None:
            out = _empty(max(self.nnz, 1), torch.complex128, self.device, self.alloc)
        ws = self.workspace(job.precision)
        mat = job.mat.struct()
        m.reset_status()
        L.check(L.lib().emg_assemble(
            L.ctypes.byref(self.plan), L.ptr(self.d_plan), L.ptr(self.d_indptr), L.ptr(m.nodes), m.n_nodes,
            L.ptr(m.tets), L.ptr(m.tetids), L.ctypes.byref(mat), job.precision, alpha.real, alpha.imag, beta.real,
            beta.imag, L.ptr(ws), ws.numel(), L.ptr(out), L.ptr(m.status), L.stream_handle(m.device)))
        return out

    def gather_device(self, values: torch.Tensor, precision: int = L.EMG_FP64, out: torch.Tensor | None = None):
        """Column gather of element values already on the device (reference
        COO layout [nA][20][20])."""
        if values.numel() != 400 * self.n_assy:
            raise ValueError(f"expected {400 * self.n_assy} element values, got {values.numel()}")
        if out is None:
            out = torch.empty(max(self.nnz, 1), dtype=torch.complex128, device=self.device)
        L.check(L.lib().emg_gather(L.ctypes.byref(self.plan), L.ptr(self.d_plan), L.ptr(self.d_indptr), L.ptr(values),
                                   None, precision, L.EMG_LAYOUT_COO, 1.0, 0.0, 0.0, 0.0, L.ptr(out), None,
                                   L.stream_handle(self.device)))
        return out

    def to_device(self, data) -> torch.Tensor:
        """Values of to_csc(data) kept on the device (complex128 [nnz])."""
        if isinstance(data, ElemValues):
            data = data._lc()
        if getattr(data, "_is_robin_term", False) or getattr(data, "_is_opposite_term", False):
            data = data._lc()
        if isinstance(data, LinComb):
            if data.opposite_terms:
                raise ValueError("an opposite-side term grows the pattern: assemble through its ExtendedCSCMapping")
            if data.job is not None:
                out = self.assemble_device(data.job, data.alpha, data.beta)
                data.job.mesh.check_status()
            else:
                out = torch.zeros(max(self.nnz, 1), dtype=torch.complex128, device=self.device)
            for term, gamma in data.robin_terms:
                term.apply(out, gamma, self)
            return out[: self.nnz]
        arr = np.asarray(data)
        if not np.iscomplexobj(arr):
            arr = arr.astype(np.complex128)
        v = _to_dev(arr.astype(np.complex128, copy=False), torch.complex128, self.device)
        return self.gather_device(v)[: self.nnz]

    def host_buffer(self) -> np.ndarray:
        """A page-locked complex128 [nnz] host array for ``to_csc(..., out=)``.
        Page-locking costs about 0.8 s per GB once; a caller that keeps
        earlier results alive can reuse a few such buffers instead of having
        every call lock fresh memory."""
        return torch.empty(max(self.nnz, 1), dtype=torch.complex128, pin_memory=True).numpy()[: self.nnz]

    def to_csc(self, data, out: np.ndarray | None = None) -> csc_matrix:
        """``CSCMapping.to_csc`` (csc_cast.py:55-63): data is an element-value
        object / combination of this assembly or a host COO array in the
        reference layout. The values land in ``out`` (complex128 [nnz], host;
        page-locked from ``host_buffer`` for full copy speed) or in a
        page-locked array from torch's host allocator, which recycles it once
        the returned matrix is gone."""
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


def tet_mass_stiffness_matrices(field, er: np.ndarray, ur: np.ndarray, conductor_tets: np.ndarray,
                                cscmap: GpuCSCMapping | None = None, *, precision: str = "fp64", device=None):
    """Drop-in for curlcurl.py:222-270. Returns (dataE, dataB, cscmap) where
    dataE (stiffness) and dataB (mass) are lazy device-backed element values
    and cscmap is a ``GpuCSCMapping`` (built on first use, reused after)."""
    dmesh = DeviceMesh(field, conductor_tets, device, reuse=getattr(cscmap, "dmesh", None))
    dmat = DeviceMaterial(er, ur, dmesh.n_tets, dmesh.device)
    job = _Job(dmesh, dmat, _prec(precision))
    if cscmap is None:
        cscmap = GpuCSCMapping(dmesh)
    return ElemValues(job, "K"), ElemValues(job, "M"), cscmap
