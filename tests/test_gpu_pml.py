"""Anisotropic lossy PML shell + 2% slivers (the 84x50x40 construction on a
20x12x10 box): plain FP64 parity with the reference (oracle) on every entry,
and the mixed form's error against FP64 per tensor component.

Tolerances: FP64 vs oracle <= 1e-12 relative (Frobenius and max-entry) for
K, M, A, and <= 1e-13 per tet (max-entry relative to that block's max);
mixed vs FP64 <= 1e-6 relative for K, M, A."""
import numpy as np
import pytest

from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.workloads import wr90_pml_slivers
from oracle import oracle as O
from tests.golden_util import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pml():
    return wr90_pml_slivers(n=(20, 12, 10))


def test_pml_slivers_fp64_parity(pml):
    f, er, ur, k0 = pml.field, pml.er, pml.ur, pml.k0
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, pml.conductor_tets)
    dE, dB, ocmap = O.tet_mass_stiffness_matrices(f, er, ur, pml.conductor_tets)
    assert np.array_equal(cmap.indptr, ocmap.indptr) and np.array_equal(cmap.indices, ocmap.indices)
    for mine, ref in ((np.asarray(E), dE), (np.asarray(B), dB)):
        a, r = mine.reshape(-1, 400), ref.reshape(-1, 400)
        per = np.abs(a - r).max(axis=1) / np.abs(r).max(axis=1)
        assert per.max() <= 1e-13, per.max()
    for key, mine, ref in (("K", cmap.to_csc(E).data, ocmap.values(dE)), ("M", cmap.to_csc(B).data, ocmap.values(dB)),
                           ("A", cmap.to_csc(E - B * k0 ** 2).data, ocmap.values_lincomb(dE, dB, 1.0, -k0 ** 2))):
        fro, mx = rel_err(mine, ref)
        assert fro <= 1e-12 and mx <= 1e-12, (key, fro, mx)


def _component(t, c):
    """PML tensor with only diagonal component c kept; the others set to 1."""
    out = np.zeros_like(t)
    for d in range(3):
        out[d, d] = t[d, d] if d == c else 1.0
    return out


@pytest.mark.parametrize("comp", [0, 1, 2, "full"])
def test_pml_slivers_mixed_error_per_component(pml, comp):
    f, k0 = pml.field, pml.k0
    er = pml.er if comp == "full" else _component(pml.er, comp)
    ur = pml.ur if comp == "full" else _component(pml.ur, comp)
    E64, B64, cmap = tet_mass_stiffness_matrices(f, er, ur, pml.conductor_tets)
    E32, B32, _ = tet_mass_stiffness_matrices(f, er, ur, pml.conductor_tets, cmap, precision="mixed")
    errs = {}
    for key, a, b in (("K", E32, E64), ("M", B32, B64), ("A", E32 - B32 * k0 ** 2, E64 - B64 * k0 ** 2)):
        errs[key] = rel_err(cmap.to_csc(a).data, cmap.to_csc(b).data)
    print(f"component {comp}: " + ", ".join(f"{k} fro {v[0]:.2e} max {v[1]:.2e}" for k, v in errs.items()))
    for key, (fro, mx) in errs.items():
        assert fro <= 1e-6 and mx <= 1e-6, (comp, key, fro, mx)
