"""The solve-DoF submatrix on the device.

Before every solve the reference slices the assembled system to the DoFs that
are not fixed by PEC conditions (solver.py:2071)::

    Asel = A[:, solve_ids][solve_ids, :]
    bsel = b[solve_ids]

``SolveSubmatrix(cscmap, solve_ids)`` builds the reduced pattern once (rows
renumbered and ascending, as scipy's slicing gives them) and a map from each
kept entry to its position in A; per frequency ``values(A)`` gathers the
reduced values on the device, so a GPU solver never needs A on the host;
``solve`` hands them to a sparse direct solver on the device (cuSOLVER's
sparse QR through emg_sparse_solve: the reference's cuDSS is not part of
this toolkit) and ``expand`` puts the solution back on all N DoFs.
"""
from __future__ import annotations

import warnings

import numpy as np
import torch
from scipy.sparse import csc_matrix

from . import _lib as L
from .assembly import GpuCSCMapping, _to_dev

__all__ = ["SolveSubmatrix", "superlu_like_reference"]


def superlu_like_reference(A: csc_matrix, b: np.ndarray) -> np.ndarray:
    """Solve A x = b on the host with scipy's SuperLU under the reference's
    SolverSuperLU settings without scikit-sparse (solver.py:869-975):
    MMD_AT_PLUS_A column ordering, relax 0, diagonal pivot threshold 0.001,
    SymmetricMode, no equilibration, single iterative refinement -- for
    comparing a GPU-assembled system with the reference's own solve."""
    from scipy.sparse.linalg import splu

    lu = splu(csc_matrix(A), permc_spec="MMD_AT_PLUS_A", relax=0, diag_pivot_thresh=0.001,
              options=dict(SymmetricMode=True, Equil=False, IterRefine="SINGLE"))
    return lu.solve(np.asarray(b))


class SolveSubmatrix:
    """A[:, solve_ids][solve_ids, :] of the pattern of ``cscmap``;
    ``solve_ids`` are DoF numbers (any order, duplicates ignored)."""

    def __init__(self, cscmap: GpuCSCMapping, solve_ids):
        self.cmap = cscmap
        dev = cscmap.device
        N = cscmap.N
        ids = np.unique(np.asarray(solve_ids, dtype=np.int64).ravel())
        if ids.size and (ids[0] < 0 or ids[-1] >= N):
            raise IndexError("solve id out of range")
        self.solve_ids = ids
        keep = np.zeros(N, np.uint8)
        keep[ids] = 1
        d_keep = _to_dev(keep, torch.uint8, dev)
        sel = L.Select()
        L.check(L.lib().emg_select_init(N, L.ctypes.byref(sel)))
        ws = torch.empty(max(sel.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        self.d_indptr = torch.empty(N + 1, dtype=torch.int32, device=dev)
        status = torch.zeros(2, dtype=torch.int64, device=dev)
        st = L.stream_handle(dev)
        L.check(L.lib().emg_select_build(L.ctypes.byref(sel), L.ptr(cscmap.d_indptr), L.ptr(cscmap.d_indices),
                                         L.ptr(d_keep), L.ptr(ws), L.ptr(self.d_indptr), L.ptr(status), st))
        self.M, self.nnz = int(sel.M), int(sel.nnz_sel)
        self.d_indices = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        self.d_take = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        L.check(L.lib().emg_select_finish(L.ctypes.byref(sel), L.ptr(cscmap.d_indptr), L.ptr(cscmap.d_indices),
                                          L.ptr(d_keep), L.ptr(ws), L.ptr(self.d_indptr), L.ptr(self.d_indices),
                                          L.ptr(self.d_take), st))
        self.sel = sel
        self.d_ids = _to_dev(ids, torch.int64, dev)

    def values(self, A: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """Asel's values (complex128 [nnz_sel], device) from A's (complex128
        [nnz], device); stream-ordered."""
        if A.dtype != torch.complex128 or A.numel() < self.cmap.nnz:
            raise ValueError("A must be complex128 with nnz values")
        if out is None:
            out = torch.empty(max(self.nnz, 1), dtype=torch.complex128, device=self.cmap.device)
        L.check(L.lib().emg_select_values(L.ctypes.byref(self.sel), L.ptr(self.d_take), L.ptr(A), self.cmap.nnz,
                                          L.ptr(out), L.stream_handle(self.cmap.device)))
        return out[: self.nnz]

    def rhs(self, b: torch.Tensor) -> torch.Tensor:
        """b[solve_ids] on the device."""
        return b.index_select(0, self.d_ids)

    def to_csc(self, data) -> csc_matrix:
        """Asel as a host csc_matrix; data: anything ``cscmap.to_device``
        takes (element-value combinations, boundary terms) or A's device values."""
        A = data if isinstance(data, torch.Tensor) else self.cmap.to_device(data)
        v = self.values(A).cpu().numpy()
        return csc_matrix((v, self.d_indices[: self.nnz].cpu().numpy(), self.d_indptr[: self.M + 1].cpu().numpy()),
                          shape=(self.M, self.M))

    _REORDER = {"none": 0, "symrcm": 1, "symamd": 2, "metis": 3}

    def solve(self, values: torch.Tensor, b: torch.Tensor, *, symmetric: bool = True, tol: float = 1e-12,
              reorder: str = "symrcm") -> torch.Tensor:
        """x (complex128 [M], device) with Asel x = b: ``values`` are Asel's
        (``values(A)``), ``b`` the reduced right-hand side (``rhs``). With
        ``symmetric`` (Asel = Asel^T, as for every system this library
        assembles, port terms included) the CSC arrays are passed as CSR;
        otherwise they are converted on the device first. Raises
        np.linalg.LinAlgError if the solver finds Asel singular."""
        dev = self.cmap.device
        if self.M == 0:
            return torch.zeros(0, dtype=torch.complex128, device=dev)
        v = values.to(device=dev, dtype=torch.complex128).contiguous()[: self.nnz]
        rhs = b.to(device=dev, dtype=torch.complex128).contiguous()
        if v.numel() != self.nnz or rhs.numel() != self.M:
            raise ValueError(f"values need {self.nnz} and b {self.M} entries")
        if reorder not in self._REORDER:
            raise ValueError(f"reorder must be one of {sorted(self._REORDER)}")
        ptr, ind = self.d_indptr[: self.M + 1], self.d_indices[: self.nnz]
        if not symmetric:  # CSC of Asel -> CSR of Asel (arrays from emg_select_*: valid by construction)
            with warnings.catch_warnings():
                warnings.simplefilter("ignore", UserWarning)
                csr = torch.sparse_csc_tensor(ptr.to(torch.int64), ind.to(torch.int64), v, size=(self.M, self.M),
                                              check_invariants=False).to_sparse_csr()
            ptr = csr.crow_indices().to(torch.int32).contiguous()
            ind = csr.col_indices().to(torch.int32).contiguous()
            v = csr.values().contiguous()
        x = torch.empty(self.M, dtype=torch.complex128, device=dev)
        sing = L.ctypes.c_int64(-1)
        L.check(L.lib().emg_sparse_solve(self.M, self.nnz, L.ptr(ptr), L.ptr(ind), L.ptr(v), L.ptr(rhs), L.ptr(x),
                                         float(tol), self._REORDER[reorder], L.ctypes.byref(sing),
                                         L.stream_handle(dev)))
        if sing.value >= 0:
            raise np.linalg.LinAlgError(f"the reduced system is singular (row {sing.value})")
        return x

    def expand(self, x: torch.Tensor) -> torch.Tensor:
        """The solution on all N DoFs (complex128, device): x at solve_ids,
        zero at the fixed (PEC) DoFs, as the reference's solution vector."""
        full = torch.zeros(self.cmap.N, dtype=torch.complex128, device=self.cmap.device)
        full[self.d_ids] = x.to(torch.complex128)
        return full
