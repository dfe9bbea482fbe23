"""Resident frequency sweep: A(f) formed from K and M kept on the device
equals the per-frequency assembly (and the oracle) within the plain-FP64
tolerance, 1e-12 relative."""
import numpy as np
import pytest
import torch

from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.sweep import FrequencySweep
from emerge_b200 import workloads as W
from emerge_b200.workloads import wr90_dielectric
from oracle import oracle as O
from tests.golden_util import rel_err

pytestmark = pytest.mark.gpu


def test_sweep_matches_per_frequency_assembly():
    wl = wr90_dielectric(n=(8, 5, 12))
    f = wl.field
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets)
    sw = FrequencySweep(E, B, cmap)
    freqs = np.linspace(8e9, 12e9, 37)
    A = sw.form(FrequencySweep.coefficients(freqs))
    dE, dB, ocmap = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, wl.conductor_tets)
    for i in (0, 17, 36):
        k0 = 2 * np.pi * freqs[i] / 299792458.0
        direct = cmap.to_csc(E - B * k0 ** 2).data
        got = A[i].cpu().numpy()
        assert rel_err(got, direct)[0] < 1e-13
        assert max(rel_err(got, ocmap.values_lincomb(dE, dB, 1.0, -k0 ** 2))) < 1e-12
    # a port-like term P with its own coefficient
    P = torch.zeros(cmap.nnz, dtype=torch.complex128, device=A.device)
    P[::97] = 1.0 + 0.5j
    sw2 = FrequencySweep(E, B, cmap, P)
    g = 1j * np.linspace(100.0, 200.0, freqs.size)
    A2 = sw2.form(FrequencySweep.coefficients(freqs, g))
    ref = A + torch.from_numpy(g).to(A.device)[:, None] * P[None, :]
    assert torch.allclose(A2, ref, rtol=1e-14, atol=0)
    csc = sw2.to_csc(freqs[5], g[5])
    assert np.array_equal(csc.indptr, cmap.indptr) and np.allclose(csc.data, A2[5].cpu().numpy(), rtol=0, atol=0)


def test_conductive_sweep_matches_per_frequency_assembly():
    """Materials with a conductivity: the resident three-matrix sweep
    (FrequencySweep.with_conductivity) against assembling er(w) = er (1 - j
    tand) - j cond / (w eps0) from scratch at each frequency, as the
    reference does; 1e-12 relative (Frobenius and max entry)."""
    from emerge_b200.sweep import EPS0

    wl = W.wr90_dielectric(n=(8, 5, 12), seed=3)
    f = wl.field
    nT = f.ntets
    rng = np.random.default_rng(4)
    tand = np.zeros((3, 3, nT), np.complex128)
    cond = np.zeros((3, 3, nT), np.complex128)
    sig = rng.choice([0.0, 0.5, 20.0], size=nT)
    for d in range(3):
        tand[d, d] = rng.uniform(0.0, 0.02, nT)
        cond[d, d] = sig
    none = np.zeros(0, np.int64)
    sw = FrequencySweep.with_conductivity(f, wl.er, tand, cond, wl.ur, none)
    freqs = np.array([1e9, 5e9, 12e9])
    A = sw.form(FrequencySweep.conductive_coefficients(freqs))
    for i, fr in enumerate(freqs):
        w = 2 * np.pi * fr
        er_w = wl.er * (1 - 1j * tand) - 1j * cond / (w * EPS0)
        E, B, _ = tet_mass_stiffness_matrices(f, er_w, wl.ur, none, sw.cscmap)
        direct = sw.cscmap.to_device(E - B * (w / W.C0) ** 2).cpu().numpy()
        fro, mx = rel_err(A[i].cpu().numpy(), direct)
        assert fro <= 1e-12 and mx <= 1e-12, (fr, fro, mx)
