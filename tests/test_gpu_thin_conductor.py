"""ThinConductor's opposite-side term on the GPU (ExtendedCSCMapping,
OppositeSideTerm): against the reference-generated fixture (thin.npz), against
the oracle chain on a 24x12x60-hex box with two strips, and at the
2,010,000-tet size through properties of the grown pattern."""
import numpy as np
import pytest
import torch
from scipy.sparse import csc_matrix

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.mesh import Nedelec2Field, TetMesh, grid_level_tris
from emerge_b200.robin import RobinTerm
from emerge_b200.solve_dofs import SolveSubmatrix
from emerge_b200.thin_conductor import ExtendedCSCMapping, OppositeSideTerm
from oracle import oracle as O
from tests.golden_util import load_npz

pytestmark = pytest.mark.gpu

NONE = np.zeros(0, np.int64)


def _close(got: csc_matrix, want: csc_matrix, tol: float):
    """Same matrix: every stored entry of ``want`` is in ``got`` and the
    difference is within tol of the largest entry (``got`` may hold explicit
    zeros where scipy's sum dropped a cancelled entry)."""
    assert got.shape == want.shape
    d = (got - want).tocsc()
    scale = np.abs(want.data).max()
    assert (np.abs(d.data).max() if d.nnz else 0.0) <= tol * scale
    g = got.tocsc()
    g.sort_indices()
    gi = set(zip(np.repeat(np.arange(g.shape[1]), np.diff(g.indptr)).tolist(), g.indices.tolist()))
    w = want.tocsc()
    wi = set(zip(np.repeat(np.arange(w.shape[1]), np.diff(w.indptr)).tolist(), w.indices.tolist()))
    assert wi <= gi


def _fixture_case():
    G = load_npz("thin.npz")
    f = Nedelec2Field(TetMesh(G["nodes"], G["tets"]))
    strips = (G["strip0"], G["strip1"])
    f.partition_dof([(strips[0], G["normal0"]), (strips[1], G["normal1"])])
    return G, f, strips


def test_fixture_final_K_and_other_side_alone():
    G, f, strips = _fixture_case()
    k0 = float(G["k0"])
    E, B, cmap = tet_mass_stiffness_matrices(f, G["er"], G["ur"], NONE)
    assert cmap.N == f.n_field and cmap.indptr.size == f.n_field + 1
    Rp = RobinTerm(f, G["port"], cmap)
    Rs = [RobinTerm(f, s, cmap) for s in strips]
    Ts = [OppositeSideTerm(f, s) for s in strips]
    X = ExtendedCSCMapping(cmap, Ts)
    assert X.n_extra > 0 and X.nnz == cmap.nnz + X.n_extra
    g = [complex(x) for x in G["g_tc"]]
    comb = E - B * k0 ** 2 + Rp * complex(G["g_port"]) + Rs[0] * g[0] + Rs[1] * g[1] + Ts[0] * g[0] + Ts[1] * g[1]
    K = X.to_csc(comb)
    ref = csc_matrix((G["K_data"], G["K_indices"], G["K_indptr"]), shape=K.shape)
    _close(K, ref, 1e-12)
    # the grown pattern is the reference's here (nothing cancels)
    assert np.array_equal(K.indptr, ref.indptr) and np.array_equal(K.indices, ref.indices)
    OSr = csc_matrix((G["os_data"], G["os_indices"], G["os_indptr"]), shape=K.shape)
    _close(X.to_csc(Ts[0] * g[0] + Ts[1] * g[1]), OSr, 1e-13)
    # without the other side the base mapping is A's pattern, and mixing is refused
    with pytest.raises(ValueError, match="ExtendedCSCMapping"):
        cmap.to_device(E + Ts[0])


def test_solve_submatrix_takes_extended_mapping():
    G, f, strips = _fixture_case()
    k0 = float(G["k0"])
    E, B, cmap = tet_mass_stiffness_matrices(f, G["er"], G["ur"], NONE)
    Ts = [OppositeSideTerm(f, s) for s in strips]
    X = ExtendedCSCMapping(cmap, Ts)
    comb = E - B * k0 ** 2 + Ts[0] * 3.0 + Ts[1] * (1 - 2j)
    full = X.to_csc(comb)
    keep = np.ones(f.n_field, bool)
    keep[np.random.default_rng(3).choice(f.n_field, 200, replace=False)] = False
    ids = np.flatnonzero(keep)
    sub = SolveSubmatrix(X, ids)
    got = sub.to_csc(comb)
    want = full[:, ids][ids, :].tocsc()
    want.sort_indices()
    assert np.array_equal(got.indptr, want.indptr) and np.array_equal(got.indices, want.indices)
    assert np.array_equal(got.data, want.data)


def _strip_case(n, strips_spec):
    wl = W.wr90_dielectric(n=n)
    f = wl.field
    m = f.mesh
    strips = [grid_level_tris(m, n, 2, lev, lo, hi) for lev, lo, hi in strips_spec]
    f.partition_dof([(s, np.array([0.0, 0.0, 1.0])) for s in strips])
    return wl, f, strips


def test_two_strips_24x12x60_against_oracle():
    n = (24, 12, 60)
    wl, f, strips = _strip_case(n, [(20, (4, 2, 0), (20, 10, 60)), (41, (0, 0, 0), (12, 12, 60))])
    assert f.ntets == 103_680 and f.n_field > 2 * f.mesh.n_edges + 2 * f.mesh.n_tris
    k2 = wl.k0 ** 2
    g = [(3.0 + 1.0j) * 50, (0.2 - 2.0j) * 50]
    dE, dB, pat = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, NONE)
    ref = pat.to_csc(dE - dB * k2)
    del dE, dB
    B1 = np.zeros(f.mesh.n_tris * 64, np.complex128)
    B2 = np.zeros_like(B1)
    for s, gg in zip(strips, g):
        B1 = O.robin_entries(f, s, gg, B1)
        B2 = O.robin_entries(f, s, gg, B2)
    ref = (ref + O.generate_csc(f, B1) + O.generate_csc(f, B2, O.tri_rowcol(f, other_side=True))).tocsc()
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, NONE)
    Rs = [RobinTerm(f, s, cmap) for s in strips]
    Ts = [OppositeSideTerm(f, s) for s in strips]
    X = ExtendedCSCMapping(cmap, Ts)
    K = X.to_csc(E - B * k2 + Rs[0] * g[0] + Rs[1] * g[1] + Ts[0] * g[0] + Ts[1] * g[1])
    _close(K, ref, 1e-12)
    assert np.array_equal(K.indptr, ref.indptr) and np.array_equal(K.indices, ref.indices)


def test_full_size_grown_pattern_properties():
    """2,010,000 tets, one 80x40-hex strip at mid height: A's entries keep
    their values at their new positions, the new entries hold the other side
    alone, and the union is sorted CSC."""
    wl, f, strips = _strip_case((100, 50, 67), [(33, (10, 5, 0), (90, 45, 67))])
    assert f.ntets == 2_010_000
    k2 = wl.k0 ** 2
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, NONE)
    T = OppositeSideTerm(f, strips[0])
    X = ExtendedCSCMapping(cmap, [T])
    A = cmap.to_device(E - B * k2)
    U = X.grow(A)
    dev = A.device
    ip_b = cmap.d_indptr[: cmap.N + 1].to(torch.int64)
    ip_x = X.d_indptr[: X.N + 1].to(torch.int64)
    # per column: the base entries first (their rows are below the split DoFs), then the new ones
    col_b = torch.repeat_interleave(torch.arange(cmap.N, device=dev), ip_b[1:] - ip_b[:-1])
    pos_base = ip_x[col_b] + (torch.arange(cmap.nnz, device=dev) - ip_b[col_b])
    assert torch.equal(U[pos_base], A[: cmap.nnz])
    assert torch.equal(X.d_indices[pos_base], cmap.d_indices[: cmap.nnz])
    extra = torch.ones(X.nnz, dtype=torch.bool, device=dev)
    extra[pos_base] = False
    assert int(extra.sum()) == X.n_extra > 0
    assert not bool((U[extra] != 0).any())
    g = 7.0 - 3.0j
    V = X.to_device(E - B * k2 + T * g)
    os_col = torch.zeros(cmap.N, dtype=torch.bool, device=dev)
    os_col[torch.from_numpy(T.dofs.ravel()).to(dev)] = True
    keep = ~os_col[col_b]  # columns the other side does not touch keep A's values bit for bit
    assert torch.equal(V[pos_base[keep]], A[: cmap.nnz][keep])
    osv = X.to_device(T * g)
    assert torch.equal(V[extra], osv[extra])
    # sorted rows in every column of the union
    idx = X.d_indices[: X.nnz].to(torch.int64)
    col_x = torch.repeat_interleave(torch.arange(X.N, device=dev), ip_x[1:] - ip_x[:-1])
    assert bool(((idx[1:] > idx[:-1]) | (col_x[1:] != col_x[:-1])).all())
