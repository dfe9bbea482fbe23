"""Heat-conduction Lagrange-2 assembly and the general COO -> CSC mapping on
the GPU, against the reference's own output (tests/golden/heat.npz) and the
oracle. Tolerance 1e-12 relative (Frobenius and max entry) for values; the
CSC pattern is bit-exact. At larger sizes: K annihilates constants (the
Lagrange basis sums to one) and the entries of M sum to the quadrature's
integral of rho_cp."""
import numpy as np
import pytest
import torch
from scipy.sparse import coo_matrix

from emerge_b200 import _lib as L
from emerge_b200.heat import GpuCOOMapping, Legrange2, tet_mass_matrix, tet_stiffness_matrix
from emerge_b200.mesh import TetMesh, structured_box
from oracle import oracle as O
from tests.golden_util import load_npz, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12


def heat_field():
    nodes, tets = structured_box(6, 4, 10, jitter=0.1, seed=13)
    return Legrange2(TetMesh(nodes, tets))


@pytest.mark.parametrize("precision", ["fp64", "exact"])
def test_heat_matrices_match_reference_golden(precision):
    g = load_npz("heat.npz")
    f = heat_field()
    assert f.n_field == int(g["N"])
    K, cmap = tet_stiffness_matrix(f, g["cond"], precision=precision)
    M, cmap2 = tet_mass_matrix(f, g["rho_cp"], precision=precision)
    assert cmap2 is cmap  # one resident mapping per field
    for mine, ref in ((np.asarray(K), g["K"]), (np.asarray(M), g["M"])):
        fro, mx = rel_err(mine, ref)
        assert fro <= TOL and mx <= TOL, (fro, mx)
    A = cmap.to_csc(K)
    assert A.dtype == np.float64
    assert np.array_equal(A.indptr, g["indptr"]) and np.array_equal(A.indices, g["indices"])
    fro, mx = rel_err(A.data, g["Kdata"])
    assert fro <= TOL and mx <= TOL, (fro, mx)
    # the host COO array in the reference layout gives the same CSC values
    assert np.array_equal(cmap.to_csc(g["K"]).indices, A.indices)
    assert rel_err(cmap.to_csc(g["K"]).data, g["Kdata"])[1] <= 1e-15


def test_transient_combination_and_oracle_mass():
    g = load_npz("heat.npz")
    f = heat_field()
    K, cmap = tet_stiffness_matrix(f, g["cond"])
    M, _ = tet_mass_matrix(f, g["rho_cp"])
    dt = 0.25
    A = cmap.to_csc(K + M / dt)
    B = (cmap.to_csc(K) + cmap.to_csc(M) / dt).tocsc()
    assert rel_err(A.data, B.data)[1] <= 1e-15
    rows, cols = O.leg2_rowcol(f.tet_to_field)
    pat = O.CSCPattern.from_rowcol(rows, cols, f.n_field)
    ref = pat.values(O.leg2_values(f.mesh, g["rho_cp"], "mass").astype(np.complex128)).real
    fro, mx = rel_err(cmap.to_csc(M).data, ref)
    assert fro <= TOL and mx <= TOL, (fro, mx)


def test_layouts_and_oracle_arithmetic():
    """Through the C ABI: the row-major (reference) and transposed element
    layouts hold the same values, and gathering either (block_dofs 0 / 10)
    gives bit-identical CSC values. The fp64 form repeats the reference's
    operations: it agrees with the oracle's C restatement to rounding."""
    g = load_npz("heat.npz")
    f = heat_field()
    K, cmap = tet_stiffness_matrix(f, g["cond"])
    M, _ = tet_mass_matrix(f, g["rho_cp"])
    from emerge_b200.heat import _heat_mesh

    hm = _heat_mesh(f, cmap.device)
    st = L.stream_handle(cmap.device)
    status = torch.zeros(2, dtype=torch.int64, device=cmap.device)
    for kind, coef, vals in ((0, g["cond"], K), (1, g["rho_cp"], M)):
        d_coef = torch.from_numpy(np.ascontiguousarray(coef)).cuda()
        row = torch.empty(100 * hm.n_tets, dtype=torch.float64, device=cmap.device)
        L.check(L.lib().emg_leg2_element(L.ptr(hm.nodes), hm.n_nodes, L.ptr(hm.tets), hm.n_tets, L.ptr(d_coef), kind,
                                         L.EMG_FP64, L.EMG_LAYOUT_COO, L.ptr(row), L.ptr(status), st))
        assert torch.equal(row, vals.reference_layout())
        a = torch.empty(cmap.nnz, dtype=torch.float64, device=cmap.device)
        L.check(L.lib().emg_coo_gather(L.ctypes.byref(cmap.desc), L.ptr(cmap.d_perm), L.ptr(cmap.d_run), 0, 0,
                                       L.ptr(row), L.ptr(a), st))
        assert torch.equal(a, cmap.to_device(vals))
        ref = O.leg2_values(f.mesh, coef, "stiff" if kind == 0 else "mass")
        assert rel_err(row.cpu().numpy(), ref)[1] <= 1e-14
    assert int(status[0]) == 0
    # mixing layouts: a host array in the reference layout joins device values
    A = cmap.to_csc(K + g["M"])
    assert rel_err(A.data, cmap.to_csc(K).data + cmap.to_csc(M).data)[1] <= 1e-14


@pytest.mark.parametrize("cplx", [False, True])
def test_general_coo_mapping_matches_scipy(cplx):
    """Random slots with repeats, empty columns and unsorted input: the
    pattern is scipy's summed-duplicate CSC with sorted rows, bit for bit; the
    values agree to rounding (scipy sums in another order)."""
    rng = np.random.default_rng(3)
    N, S = 700, 20000
    rows = rng.integers(0, N, S)
    cols = rng.integers(0, N // 2, S) * 2  # odd columns stay empty
    v = rng.normal(size=S) + (1j * rng.normal(size=S) if cplx else 0)
    cm = GpuCOOMapping.from_rowcol(rows, cols, N, device="cuda")
    A = cm.to_csc(v)
    ref = coo_matrix((v, (rows, cols)), shape=(N, N)).tocsc()
    ref.sum_duplicates()
    ref.sort_indices()
    assert np.array_equal(A.indptr, ref.indptr) and np.array_equal(A.indices, ref.indices)
    assert A.dtype == (np.complex128 if cplx else np.float64)
    assert rel_err(A.data, ref.data)[1] <= 1e-14
    # deterministic: the slot order fixes the sum order
    assert np.array_equal(cm.to_csc(v).data, A.data)


def test_empty_and_out_of_range_slots():
    cm = GpuCOOMapping.from_rowcol(np.zeros(0, np.int64), np.zeros(0, np.int64), 5, device="cuda")
    A = cm.to_csc(np.zeros(0))
    assert A.nnz == 0 and np.array_equal(A.indptr, np.zeros(6, np.int32))
    with pytest.raises(L.EmgMeshError):
        GpuCOOMapping.from_rowcol(np.array([0, 1]), np.array([0, 5]), 5, device="cuda")
    with pytest.raises(L.EmgMeshError):
        GpuCOOMapping.from_rowcol(np.array([0, -1]), np.array([0, 1]), 5, device="cuda")
    with pytest.raises(L.EmgMeshError):  # would wrap to 5 in int32
        GpuCOOMapping.from_rowcol(np.array([0, 2 ** 32 + 1]), np.array([0, 1]), 5, device="cuda")
    with pytest.raises(L.EmgMeshError):
        GpuCOOMapping.from_rowcol(torch.tensor([0, 1]), torch.tensor([0, 2 ** 32 + 1]), 5, device="cuda")


def test_partitioned_numbering_matches_oracle():
    """A renumbered tet_to_field (as partition_dof leaves it): the pattern
    follows the given numbering."""
    g = load_npz("heat.npz")
    f = heat_field()
    perm = np.random.default_rng(1).permutation(f.n_field)
    f.tet_to_field = perm[f.tet_to_field]
    K, cmap = tet_stiffness_matrix(f, g["cond"])
    rows, cols = O.leg2_rowcol(f.tet_to_field)
    pat = O.CSCPattern.from_rowcol(rows, cols, f.n_field)
    A = cmap.to_csc(K)
    assert np.array_equal(A.indptr, pat.indptr) and np.array_equal(A.indices, pat.indices)
    fro, mx = rel_err(A.data, pat.values(g["K"].astype(np.complex128)).real)
    assert fro <= TOL and mx <= TOL, (fro, mx)


def test_degenerate_tet_raises():
    f = heat_field()
    m = f.mesh
    tets = m.tets.copy()
    tets[3, 7] = tets[0, 7]  # repeated vertex: zero volume
    bad = Legrange2.__new__(Legrange2)
    bad.mesh = type("M", (), {"nodes": m.nodes, "tets": tets, "n_nodes": m.n_nodes, "n_edges": m.n_edges})()
    bad.tet_to_field, bad.n_field = f.tet_to_field, f.n_field
    for precision in ("fp64", "exact"):
        with pytest.raises(L.EmgMeshError, match="degenerate"):
            tet_mass_matrix(bad, np.ones(m.n_tets), precision=precision)
        with pytest.raises(L.EmgMeshError, match="degenerate"):
            tet_stiffness_matrix(bad, np.ones((3, 3, m.n_tets)), precision=precision)


def test_exact_form_is_translation_invariant():
    """The moment form does not depend on where the mesh sits: shifting the
    box by 1e3 of its own size changes its values by rounding only, while the
    two forms still agree to 1e-12 at the origin."""
    g = load_npz("heat.npz")
    f = heat_field()
    K0 = np.asarray(tet_stiffness_matrix(f, g["cond"], precision="exact")[0])
    Kf = np.asarray(tet_stiffness_matrix(f, g["cond"], precision="fp64")[0])
    assert rel_err(K0, Kf)[1] <= 1e-12
    shifted = Legrange2(TetMesh(f.mesh.nodes + 50.0, f.mesh.tets))
    K1 = np.asarray(tet_stiffness_matrix(shifted, g["cond"], precision="exact")[0])
    assert rel_err(K1, K0)[1] <= 1e-11
    with pytest.raises(ValueError):
        tet_mass_matrix(f, g["rho_cp"], precision="mixed")


@pytest.mark.parametrize("precision", ["fp64", "exact"])
def test_properties_at_size(precision):
    """A 192k-tet box: K @ 1 = 0 (gradients of a constant vanish) and the
    entries of M sum to sum_q w_q * sum_t rho_cp V_t (the basis is a
    partition of unity; the reference's 8-digit weights sum to 1.0000003, not
    1); the pattern has one column per DoF with the diagonal in it."""
    nodes, tets = structured_box(40, 20, 40, jitter=0.15, seed=4)
    m = TetMesh(nodes, tets)
    f = Legrange2(m)
    rng = np.random.default_rng(8)
    Q = rng.normal(size=(m.n_tets, 3, 3))
    cond = np.einsum("nij,nkj->ikn", Q, Q) + 0.5 * np.eye(3)[:, :, None]
    rho = rng.uniform(1.0, 3.0, m.n_tets)
    K, cmap = tet_stiffness_matrix(f, cond, precision=precision)
    M, _ = tet_mass_matrix(f, rho, precision=precision)
    A = cmap.to_csc(K)
    one = np.ones(f.n_field)
    assert np.abs(A @ one).max() <= 1e-9 * np.abs(A.data).max()
    X = m.nodes[:, m.tets]  # (3, 4, nT)
    V = np.abs(np.einsum("it,it->t", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0], axis=0))) / 6
    Mc = cmap.to_device(M)
    wsum = -0.078933 + 4 * 0.04573333 + 6 * 0.14933333
    expect = wsum * float((rho * V).sum())
    assert abs(float(Mc.sum()) - expect) <= 1e-10 * expect
    assert np.all(np.diff(A.indptr) > 0)
    d = A.diagonal()
    assert np.all(d > 0)
    assert torch.cuda.is_available()
