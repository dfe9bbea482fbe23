"""The CPU oracle (C restatement of the reference path) against the golden
fixtures produced by the reference's own numba code."""
import hashlib

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden_util import config0_inputs, dielectric_inputs, field_from, load_json, load_npz, rel_err


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["tiny.npz", "small_diag.npz"])
def test_oracle_full_fixture(name):
    g = load_npz(name)
    f = field_from(g["nodes"], g["tets"])
    dataE, dataB, cmap = O.tet_mass_stiffness_matrices(f, g["er"], g["ur"], g["conductor_tets"])
    # COO layout and values (curlcurl.py:449-455)
    assert np.array_equal(f.mesh.edges, g["edges"]) and np.array_equal(f.mesh.tris, g["tris"])
    for mine, ref in ((dataE, g["dataE"]), (dataB, g["dataB"])):
        fro, mx = rel_err(mine, ref)
        assert fro < 1e-12 and mx < 1e-12, (fro, mx)
    # pattern bit-exact (csc_cast.py:65-160)
    assert np.array_equal(cmap.indptr, g["indptr"].astype(np.int64))
    assert np.array_equal(cmap.indices, g["indices"].astype(np.int64))
    k0 = float(g["k0"])
    for key, vals in (("K", cmap.values(dataE)), ("M", cmap.values(dataB)),
                      ("A", cmap.values(dataE - dataB * k0 ** 2))):
        fro, mx = rel_err(vals, g[key])
        assert fro < 1e-12 and mx < 1e-12, (key, fro, mx)
    lc = cmap.values_lincomb(dataE, dataB, 1.0, -k0 ** 2)
    assert rel_err(lc, g["A"])[0] < 1e-12


def _check_summary(g, nodes, tets, er, ur):
    assert _sha(nodes) == g["nodes_sha256"] and _sha(tets) == g["tets_sha256"]
    f = field_from(nodes, tets)
    dataE, dataB, cmap = O.tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    assert cmap.nnz == g["nnz"] and f.n_field == g["NF"] and dataE.shape[0] == g["S"]
    assert _sha(cmap.indptr.astype(np.int64)) == g["indptr_sha256_i64"]
    assert _sha(cmap.indices.astype(np.int64)) == g["indices_sha256_i64"]
    k0 = g["k0"]
    ids = np.array(g["sample_nnz"])
    vals = {"K": cmap.values(dataE), "M": cmap.values(dataB), "A": cmap.values_lincomb(dataE, dataB, 1.0, -k0 ** 2)}
    for key, v in vals.items():
        assert abs(np.linalg.norm(v) - g[f"{key}_fro"]) <= 1e-12 * g[f"{key}_fro"]
        ref = np.array(g[f"{key}_sample_re"]) + 1j * np.array(g[f"{key}_sample_im"])
        assert np.abs(v[ids] - ref).max() <= 1e-12 * g[f"{key}_max"], key
    sl = np.array(g["sample_slot"])
    for key, v in (("dataE", dataE), ("dataB", dataB)):
        ref = np.array(g[f"{key}_sample_re"]) + 1j * np.array(g[f"{key}_sample_im"])
        assert np.abs(v[sl] - ref).max() <= 1e-12 * np.abs(v).max(), key
    return f, cmap


def test_oracle_config0_summary():
    g = load_json("config0.json")
    _check_summary(g, *config0_inputs())


def test_oracle_dielectric_summary():
    g = load_json("dielectric.json")
    nodes, tets, er, ur, blk = dielectric_inputs(g)
    assert _sha(blk) == g["block_of_tet_sha256"]
    _check_summary(g, nodes, tets, er, ur)
