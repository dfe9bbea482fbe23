"""Oracle parity at scale on the headline workload's construction (WR-90 box,
+-15% jitter, eps_r ~ U[1,10] (1 - j U[1e-3,1e-2]) per 8x8x8-cell block,
10 GHz):

* the full A (and K, M) of the 24x12x60-hex box (103,680 tets, 28.8M
  nonzeros) against the oracle's one-piece to_csc: pattern bit-exact, values
  within 1e-12 (plain FP64) / 1e-6 (mixed), relative Frobenius and max entry;
* at the full 100x50x67-hex size (2,010,000 tets, 557.8M nonzeros), the
  complete columns of 1,200 sampled entities (800 edges, 400 faces; 2,400
  columns): the oracle runs on exactly the tets that touch a sampled entity,
  so each sampled column holds all of its contributions and must equal the
  GPU's column -- its rows bit-exact, its values within the same tolerances.
"""
import numpy as np
import pytest
import torch

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices
from oracle import oracle as O
from tests.golden_util import rel_err

pytestmark = pytest.mark.gpu

NONE = np.zeros(0, np.int64)


def test_full_A_config1_construction_24x12x60():
    wl = W.wr90_dielectric(n=(24, 12, 60))
    f = wl.field
    assert f.ntets == 103_680
    k2 = wl.k0 ** 2
    dE, dB, pat = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, NONE)
    ref = {"K": pat.values_lincomb(dE, dB, 1.0, 0.0), "M": pat.values_lincomb(dE, dB, 0.0, 1.0),
           "A": pat.values_lincomb(dE, dB, 1.0, -k2)}
    del dE, dB
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-6)):
        E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, NONE, precision=precision)
        assert np.array_equal(cmap.indptr, pat.indptr) and np.array_equal(cmap.indices, pat.indices)
        for key, comb in (("K", E * 1.0), ("M", B * 1.0), ("A", E - B * k2)):
            got = cmap.to_device(comb).cpu().numpy()
            fro, mx = rel_err(got, ref[key])
            assert fro <= tol and mx <= tol, (precision, key, fro, mx)


def _entity_columns(x, E, F):
    """The two CSC columns of entity x (edges 0..E-1, faces E..E+F-1)."""
    return (x, x + E) if x < E else (E + x, E + F + x)


def test_sampled_complete_columns_full_size():
    wl = W.wr90_dielectric()
    f = wl.field
    m = f.mesh
    assert f.ntets == 2_010_000
    E, F = m.n_edges, m.n_tris
    rng = np.random.default_rng(2024)
    ents = np.concatenate([rng.choice(E, 800, replace=False), E + rng.choice(F, 400, replace=False)])
    # every tet touching a sampled entity
    edge_s = np.zeros(E, bool)
    face_s = np.zeros(F, bool)
    edge_s[ents[ents < E]] = True
    face_s[ents[ents >= E] - E] = True
    touch = edge_s[m.tet_to_edge].any(axis=0) | face_s[m.tet_to_tri].any(axis=0)
    tetids = np.flatnonzero(touch).astype(np.int64)
    dE, dB, rows, cols = O.matrix_builder(m.nodes, m.tets, m.tris, m.edges, f.get_tet_to_field(), m.tet_to_edge,
                                          m.tet_to_tri, wl.ur, wl.er, tetids)
    pat = O.CSCPattern.from_rowcol(rows, cols, f.n_field)
    k2 = wl.k0 ** 2
    ref = pat.values_lincomb(dE, dB, 1.0, -k2)
    cols_s = np.array([c for x in ents for c in _entity_columns(int(x), E, F)], np.int64)
    E_, B_, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, NONE)
    lo, hi = cmap.indptr[cols_s].astype(np.int64), cmap.indptr[cols_s + 1].astype(np.int64)
    idx = np.concatenate([np.arange(a, b) for a, b in zip(lo, hi)])
    # the oracle's rows of each sampled column are the GPU's rows
    ref_idx = np.concatenate([np.arange(pat.indptr[c], pat.indptr[c + 1]) for c in cols_s])
    assert np.array_equal(cmap.indices[idx], pat.indices[ref_idx])
    want = ref[ref_idx]
    sel = torch.from_numpy(idx).to(cmap.device)
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-6)):
        E_, B_, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, NONE, cmap, precision=precision)
        got = cmap.to_device(E_ - B_ * k2)[sel].cpu().numpy()
        fro, mx = rel_err(got, want)
        assert fro <= tol and mx <= tol, (precision, fro, mx)
    assert len(cols_s) == 2400 and want.size > 50_000
