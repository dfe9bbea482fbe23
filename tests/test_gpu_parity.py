"""GPU path (libemgpu through the drop-in) against the golden fixtures of the
reference and against the CPU oracle.

Tolerances (relative, Frobenius and max-entry, per K, M and A):
  plain FP64 <= 1e-12; mixed (FP32 contraction) <= 1e-6.
Pattern (indptr, indices) must be bit-exact.
"""
import hashlib

import numpy as np
import pytest

from emerge_b200.assembly import tet_mass_stiffness_matrices
from oracle import oracle as O
from tests.golden_util import config0_inputs, dielectric_inputs, field_from, load_json, load_npz, rel_err

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-12
TOL_MIXED = 1e-6


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _assert_close(x, ref, tol, what=""):
    fro, mx = rel_err(x, ref)
    assert fro <= tol and mx <= tol, (what, fro, mx)


@pytest.mark.parametrize("name", ["tiny.npz", "small_diag.npz"])
def test_full_fixture_fp64(name):
    g = load_npz(name)
    f = field_from(g["nodes"], g["tets"])
    E, B, cmap = tet_mass_stiffness_matrices(f, g["er"], g["ur"], g["conductor_tets"])
    _assert_close(np.asarray(E), g["dataE"], TOL_FP64, "dataE")
    _assert_close(np.asarray(B), g["dataB"], TOL_FP64, "dataB")
    assert np.array_equal(cmap.indptr, g["indptr"]) and cmap.indptr.dtype == np.int32
    assert np.array_equal(cmap.indices, g["indices"]) and cmap.indices.dtype == np.int32
    k0 = float(g["k0"])
    A = cmap.to_csc(E - B * k0 ** 2)
    assert np.array_equal(A.indptr, g["indptr"]) and np.array_equal(A.indices, g["indices"])
    _assert_close(A.data, g["A"], TOL_FP64, "A")
    _assert_close(cmap.to_csc(E).data, g["K"], TOL_FP64, "K")
    _assert_close(cmap.to_csc(B).data, g["M"], TOL_FP64, "M")
    # a host COO array in the reference layout goes through the same gather
    _assert_close(cmap.to_csc(g["dataE"] - g["dataB"] * k0 ** 2).data, g["A"], TOL_FP64, "A(host COO)")


@pytest.mark.parametrize("name", ["tiny.npz", "small_diag.npz"])
def test_full_fixture_mixed(name):
    g = load_npz(name)
    f = field_from(g["nodes"], g["tets"])
    E, B, cmap = tet_mass_stiffness_matrices(f, g["er"], g["ur"], g["conductor_tets"], precision="mixed")
    k0 = float(g["k0"])
    _assert_close(cmap.to_csc(E - B * k0 ** 2).data, g["A"], TOL_MIXED, "A")
    _assert_close(cmap.to_csc(E).data, g["K"], TOL_MIXED, "K")
    _assert_close(cmap.to_csc(B).data, g["M"], TOL_MIXED, "M")


def _summary_case(g, nodes, tets, er, ur, precision, tol):
    f = field_from(nodes, tets)
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64), precision=precision)
    assert cmap.nnz == g["nnz"] and cmap.N == g["NF"]
    assert _sha(cmap.indptr.astype(np.int64)) == g["indptr_sha256_i64"]
    assert _sha(cmap.indices.astype(np.int64)) == g["indices_sha256_i64"]
    k0 = g["k0"]
    ids = np.array(g["sample_nnz"])
    for key, data in (("K", E), ("M", B), ("A", E - B * k0 ** 2)):
        v = cmap.to_csc(data).data
        assert abs(np.linalg.norm(v) - g[f"{key}_fro"]) <= tol * g[f"{key}_fro"], key
        ref = np.array(g[f"{key}_sample_re"]) + 1j * np.array(g[f"{key}_sample_im"])
        assert np.abs(v[ids] - ref).max() <= tol * g[f"{key}_max"], key
    return f, E, B, cmap


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_config0_golden_and_oracle(precision, tol):
    g = load_json("config0.json")
    nodes, tets, er, ur = config0_inputs()
    f, E, B, cmap = _summary_case(g, nodes, tets, er, ur, precision, tol)
    # full comparison against the oracle on every entry
    dE, dB, ocmap = O.tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    k0 = g["k0"]
    ref = ocmap.values_lincomb(dE, dB, 1.0, -k0 ** 2)
    _assert_close(cmap.to_csc(E - B * k0 ** 2).data, ref, tol, "A vs oracle")
    if precision == "fp64":
        _assert_close(np.asarray(E), dE, tol, "dataE vs oracle")
        _assert_close(np.asarray(B), dB, tol, "dataB vs oracle")


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_dielectric_golden(precision, tol):
    g = load_json("dielectric.json")
    nodes, tets, er, ur, _ = dielectric_inputs(g)
    _summary_case(g, nodes, tets, er, ur, precision, tol)


def test_element_values_fp64_match_reference_per_tet():
    """Plain form reproduces the reference's arithmetic: per-tet max-entry
    relative difference to the oracle (the reference restated) <= 1e-13 on
    the config-0 box, whose absolute-coordinate rounding is ~1e-12."""
    nodes, tets, er, ur = config0_inputs()
    f = field_from(nodes, tets)
    E, B, _ = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    dE, dB, _ = O.tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    for mine, ref in ((np.asarray(E), dE), (np.asarray(B), dB)):
        a = mine.reshape(-1, 400)
        r = ref.reshape(-1, 400)
        per = np.abs(a - r).max(axis=1) / np.abs(r).max(axis=1)
        assert per.max() <= 1e-13, per.max()


def test_exact_form_against_80bit_evaluation():
    """The exact form is within 1e-13 (per tet, max-entry) of an 80-bit
    evaluation of the exact integrals on a finer grid where the reference's
    own rounding reaches ~1e-11."""
    from emerge_b200 import workloads as W
    from tests.accuracy_util import element_ld, matinv, per_tet_errors

    wl = W.wr90_dielectric(n=(50, 25, 34))
    f = wl.field
    m = f.mesh
    E, B, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64), precision="exact")
    ids = np.sort(np.random.default_rng(2).choice(f.ntets, 60, replace=False))
    Ed = np.asarray(E).reshape(-1, 20, 20)[ids]
    Bd = np.asarray(B).reshape(-1, 20, 20)[ids]
    ref = [element_ld(m.nodes[:, m.tets[:, it]], m.tets[:, it], matinv(wl.ur[:, :, it]), wl.er[:, :, it]) for it in ids]
    assert per_tet_errors(Ed, [r[0] for r in ref]).max() <= 1e-13
    assert per_tet_errors(Bd, [r[1] for r in ref]).max() <= 1e-13
