"""Frequency sweep on a resident mesh (the cached multi-frequency path of
assembler.py:455-494).

The reference caches the COO arrays Evec (K) and Bvec (M) when no material is
frequency dependent and, per frequency, runs ``to_csc(Evec - Bvec * k0**2)``.
Here K and M are gathered once into CSC values that stay in HBM, and
``emg_form_sweep`` forms A_f = a_f*K + b_f*M (+ c_f*P) for a batch of
frequencies, reading K, M (and P) once per batch. Port and absorbing
boundaries (``RobinTerm``, the reference's assemble_robin_bc per frequency,
assembler.py:576-630) are added as gamma_f times their term, touching only
the boundary positions.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
from scipy.sparse import csc_matrix

from . import _lib as L
from .assembly import ElemValues, GpuCSCMapping

C0 = 299792458.0
EPS0 = 8.854187818814e-12  # const.py:23 of the reference


class FrequencySweep:
    """K and M of one assembly resident on the device; A(f) on demand."""

    def __init__(self, E: ElemValues, B: ElemValues, cscmap: GpuCSCMapping, P: torch.Tensor | None = None,
                 robin=None):
        if E.job is not B.job:
            raise ValueError("E and B must come from the same tet_mass_stiffness_matrices call")
        self.cscmap = cscmap
        self.K = cscmap.to_device(E)
        self.M = cscmap.to_device(B)
        self.P = P
        if P is not None and (P.dtype != torch.complex128 or P.numel() != cscmap.nnz):
            raise ValueError("P must be complex128 values in the mapping's CSC order")
        self.nnz = cscmap.nnz
        self.robin = [] if robin is None else (list(robin) if isinstance(robin, (list, tuple)) else [robin])
        for r in self.robin:
            if r.cmap is not cscmap:
                raise ValueError("a boundary term was built on another mapping")

    @classmethod
    def with_conductivity(cls, field, er: np.ndarray, tand: np.ndarray, cond: np.ndarray, ur: np.ndarray,
                          conductor_tets: np.ndarray, cscmap: GpuCSCMapping | None = None, *,
                          precision: str = "fp64", device=None, robin=None) -> "FrequencySweep":
        """A sweep over materials with a conductivity, which the reference
        cannot cache: it forms er(w) = er (1 - j tand) - j cond / (w eps0)
        and reassembles every frequency (assembler.py:439-456). The mass
        matrix is linear in er, so with M1 = M[er (1 - j tand)] and
        P = M[-j cond / eps0], all assembled once here,
            A(w) = K - k0^2 M1 - (k0^2 / w) P,
        which ``form(conductive_coefficients(freqs))`` produces per frequency
        from the three resident matrices (arrays c16[3, 3, n_tets] as the
        reference's). The excluded conductor tets are the caller's, as in
        the reference (cond above its PEC limit)."""
        from .assembly import tet_mass_stiffness_matrices

        er = np.asarray(er, dtype=np.complex128)
        er1 = er * (1 - 1j * np.asarray(tand, dtype=np.complex128))
        E, B, cmap = tet_mass_stiffness_matrices(field, er1, ur, conductor_tets, cscmap, precision=precision,
                                                 device=device)
        es = -1j * np.asarray(cond, dtype=np.complex128) / EPS0
        _, Bs, _ = tet_mass_stiffness_matrices(field, es, ur, conductor_tets, cmap, precision=precision, device=device)
        P = cmap.to_device(Bs).clone()
        return cls(E, B, cmap, P=P, robin=robin)

    @staticmethod
    def conductive_coefficients(freqs) -> np.ndarray:
        """Coefficient rows of K - k0^2 M1 - (k0^2 / w) P (``with_conductivity``)."""
        f = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
        w = 2 * np.pi * f
        k0 = w / C0
        return FrequencySweep.coefficients(f, gamma=-(k0 ** 2) / w)

    @staticmethod
    def coefficients(freqs, gamma=None) -> np.ndarray:
        """(nf, 6) coefficients (a, b, c) of A_f = K - k0^2 M + gamma_f P."""
        f = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
        k0 = 2 * np.pi * f / C0
        c = np.zeros((f.size, 6))
        c[:, 0] = 1.0
        c[:, 2] = -(k0 ** 2)
        if gamma is not None:
            g = np.broadcast_to(np.asarray(gamma, dtype=np.complex128), f.shape)
            c[:, 4], c[:, 5] = g.real, g.imag
        return c

    def form(self, coef: np.ndarray, out: torch.Tensor | None = None, robin_gamma=None) -> torch.Tensor:
        """A values for each row of ``coef`` (nf x 6), into out[nf, nnz]
        (complex128, device), plus robin_gamma[f, j] times boundary term j
        (robin_gamma: (nf,) for one term or (nf, n_terms)); stream-ordered."""
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        nf = coef.shape[0]
        if out is None:
            out = torch.empty((nf, self.nnz), dtype=torch.complex128, device=self.K.device)
        if out.shape != (nf, self.nnz) or not out.is_contiguous():
            raise ValueError("out must be a contiguous (nf, nnz) complex128 tensor")
        L.check(L.lib().emg_form_sweep(L.ptr(self.K), L.ptr(self.M), L.ptr(self.P), self.nnz,
                                       coef.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nf, L.ptr(out), self.nnz,
                                       L.stream_handle(self.K.device)))
        if self.robin:
            if robin_gamma is None:
                raise ValueError("the sweep has boundary terms: pass robin_gamma")
            g = np.asarray(robin_gamma, dtype=np.complex128).reshape(nf, -1)
            if g.shape[1] != len(self.robin):
                raise ValueError(f"robin_gamma needs {len(self.robin)} column(s)")
            for i in range(nf):
                for j, r in enumerate(self.robin):
                    r.apply(out[i], complex(g[i, j]))
        elif robin_gamma is not None:
            raise ValueError("robin_gamma given but the sweep has no boundary term")
        return out

    def to_csc(self, freq: float, gamma=None, robin_gamma=None) -> csc_matrix:
        a = self.form(self.coefficients([freq], gamma), robin_gamma=None if robin_gamma is None
                      else np.reshape(np.asarray(robin_gamma, dtype=np.complex128), (1, -1)))[0]
        host = torch.empty(a.shape, dtype=torch.complex128, pin_memory=True)
        host.copy_(a)
        m = self.cscmap
        return csc_matrix((host.numpy(), m.indices, m.indptr), shape=(m.N, m.N))
