"""Size-independent properties of the GPU path at larger sizes, plus error
behaviour. Tolerances: FP64 <= 1e-12 relative unless stated; bitwise where the
design guarantees it (pattern, determinism, symmetry)."""
import numpy as np
import pytest
import torch

from emerge_b200 import _lib as L
from emerge_b200.assembly import GpuCSCMapping, tet_mass_stiffness_matrices
from emerge_b200.mesh import Nedelec2Field, TetMesh, structured_box
from oracle import oracle as O
from tests.golden_util import rel_err

pytestmark = pytest.mark.gpu


def _blocky(nT, rng, n_blocks=37):
    blk = rng.integers(0, n_blocks, nT)
    eps = rng.uniform(1, 10, n_blocks) * (1 - 1j * rng.uniform(1e-3, 1e-2, n_blocks))
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = eps[blk]
        ur[d, d] = 1.0
    return er, ur


@pytest.fixture(scope="module")
def mid_case():
    # 40 x 20 x 27 hexes = 129,600 tets (config-1 construction, +-15% jitter)
    nodes, tets = structured_box(40, 20, 27, jitter=0.15, seed=3)
    f = Nedelec2Field(TetMesh(nodes, tets))
    er, ur = _blocky(f.ntets, np.random.default_rng(3))
    return f, er, ur


def test_pattern_size_formula_symmetry_and_determinism(mid_case):
    f, er, ur = mid_case
    m = f.mesh
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    assert cmap.nnz == 4 * m.n_edges + 52 * m.n_tris + 168 * m.n_tets
    k0 = 2 * np.pi * 10e9 / 299792458.0
    A1 = cmap.to_csc(E - B * k0 ** 2)
    A2 = cmap.to_csc(E - B * k0 ** 2)
    assert np.array_equal(A1.data, A2.data)  # bitwise run-to-run
    At = A1.T.tocsc()
    At.sort_indices()
    assert np.array_equal(At.indptr, A1.indptr) and np.array_equal(At.indices, A1.indices)
    assert np.array_equal(At.data, A1.data)  # bitwise complex-symmetric
    # linearity: A = K - k0^2 M from separately gathered K and M
    K = cmap.to_csc(E).data
    M = cmap.to_csc(B).data
    fro, _ = rel_err(A1.data, K - k0 ** 2 * M)
    assert fro < 1e-13


def test_sampled_tets_against_oracle(mid_case):
    f, er, ur = mid_case
    m = f.mesh
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    rng = np.random.default_rng(9)
    sample = np.sort(rng.choice(m.n_tets, 3000, replace=False))
    dE, dB, _, _ = O.matrix_builder(m.nodes, m.tets, m.tris, m.edges, f.get_tet_to_field(), m.tet_to_edge,
                                    m.tet_to_tri, ur, er, sample)
    Ed = E.to_device().view(-1, 400)[torch.from_numpy(sample).to(E.to_device().device)]
    Bd = B.to_device().view(-1, 400)[torch.from_numpy(sample).to(Ed.device)]
    for mine, ref in ((Ed, dE), (Bd, dB)):
        fro, mx = rel_err(mine.cpu().numpy().ravel(), ref)
        assert fro < 1e-12 and mx < 1e-12


def test_checksum_of_slots_equals_sum_of_values(mid_case):
    f, er, ur = mid_case
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    a = cmap.to_device(E - B * 7.0)
    slots = E.to_device() - 7.0 * B.to_device()
    s1 = complex(a.sum().item())
    s2 = complex(slots.sum().item())
    assert abs(s1 - s2) <= 1e-12 * float(slots.abs().sum().item())


def test_tet_order_invariance():
    nodes, tets = structured_box(6, 5, 7, jitter=0.1, seed=4)
    perm = np.random.default_rng(4).permutation(tets.shape[1])
    f1 = Nedelec2Field(TetMesh(nodes, tets))
    f2 = Nedelec2Field(TetMesh(nodes, tets[:, perm]))
    er, ur = _blocky(tets.shape[1], np.random.default_rng(5))
    E1, B1, c1 = tet_mass_stiffness_matrices(f1, er, ur, np.zeros(0, np.int64))
    E2, B2, c2 = tet_mass_stiffness_matrices(f2, er[:, :, perm], ur[:, :, perm], np.zeros(0, np.int64))
    A1, A2 = c1.to_csc(E1 - 3.0 * B1), c2.to_csc(E2 - 3.0 * B2)
    assert np.array_equal(A1.indptr, A2.indptr) and np.array_equal(A1.indices, A2.indices)
    assert rel_err(A1.data, A2.data)[0] < 1e-14


def test_conductor_exclusion_and_empty():
    nodes, tets = structured_box(3, 2, 2, jitter=0.1, seed=6)
    f = Nedelec2Field(TetMesh(nodes, tets))
    nT = f.ntets
    er, ur = _blocky(nT, np.random.default_rng(6))
    cond = np.array([0, 5, 17, 30], np.int64)
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, cond)
    dE, dB, ocmap = O.tet_mass_stiffness_matrices(f, er, ur, cond)
    assert np.array_equal(cmap.indptr, ocmap.indptr) and np.array_equal(cmap.indices, ocmap.indices)
    assert rel_err(cmap.to_csc(E - B).data, ocmap.values_lincomb(dE, dB, 1.0, -1.0))[0] < 1e-12
    # every tet a conductor: empty pattern, like the reference
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.arange(nT))
    assert cmap.nnz == 0 and np.all(cmap.indptr == 0)
    assert cmap.to_csc(E - B).nnz == 0


def test_degenerate_tet_raises():
    nodes, tets = structured_box(2, 2, 2, jitter=0.0, seed=0)
    nodes = nodes.copy()
    t = tets[:, 5]
    nodes[:, t[3]] = nodes[:, t[0]]  # collapse a tet: zero volume
    f = Nedelec2Field(TetMesh(nodes, tets))
    er, ur = _blocky(f.ntets, np.random.default_rng(0))
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    with pytest.raises(L.EmgMeshError):
        cmap.to_csc(E - B)


def test_mapping_rejects_other_mesh():
    n1, t1 = structured_box(2, 2, 2, seed=1)
    n2, t2 = structured_box(2, 2, 3, seed=1)
    f1, f2 = Nedelec2Field(TetMesh(n1, t1)), Nedelec2Field(TetMesh(n2, t2))
    er1, ur1 = _blocky(f1.ntets, np.random.default_rng(1))
    er2, ur2 = _blocky(f2.ntets, np.random.default_rng(1))
    _, _, c1 = tet_mass_stiffness_matrices(f1, er1, ur1, np.zeros(0, np.int64))
    E2, B2, _ = tet_mass_stiffness_matrices(f2, er2, ur2, np.zeros(0, np.int64))
    with pytest.raises(ValueError):
        c1.to_csc(E2 - B2)
    assert isinstance(c1, GpuCSCMapping)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chunk_order_changes_no_value(mid_case, precision):
    """The Morton processing order of the gather's entity chunks and the
    default interleave, in the block layout and in the packed one with 8- or
    4-byte contribution records, give bitwise identical A (same sums, other
    warps)."""
    f, er, ur = mid_case[0], mid_case[1], mid_case[2]
    from emerge_b200.assembly import DeviceMaterial, DeviceMesh, _Job, _prec

    dm = DeviceMesh(f, np.zeros(0, np.int64))
    job = _Job(dm, DeviceMaterial(er, ur, dm.n_tets, dm.device), _prec(precision))
    outs = []
    for order, width, layout in (("interleave", 8, "block"), ("morton", 8, "block"), ("morton", 8, "packed"),
                                 ("interleave", 8, "packed"), ("morton", 4, "packed"), ("interleave", 4, "packed")):
        cm = GpuCSCMapping(dm, chunk_order=order, record_bytes=width, value_layout=layout)
        outs.append(cm.assemble_device(job, 1.0 + 0j, -2345.5 + 1.25j)[: cm.nnz].cpu().numpy())
        dm.check_status()
    for o in outs[1:]:
        assert np.array_equal(outs[0], o)
    with pytest.raises(ValueError):
        GpuCSCMapping(dm, chunk_order="hilbert")


def test_repeat_calls_share_device_tets_and_see_moved_nodes():
    """A call that passes the mapping back with the same tet array reuses the
    mapping's device tets (the reference's cached-CSCMapping call pattern);
    node coordinates are copied every call, so moving nodes in place changes
    the values exactly as a fresh assembly does."""
    nodes, tets = structured_box(6, 4, 5, jitter=0.1, seed=2)
    f = Nedelec2Field(TetMesh(nodes, tets))
    er, ur = _blocky(f.ntets, np.random.default_rng(2))
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    A1 = cmap.to_csc(E - B * 3.0).data
    E2, B2, cmap2 = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64), cmap)
    assert cmap2 is cmap and E2.job.mesh.tets.data_ptr() == cmap.dmesh.tets.data_ptr()
    assert np.array_equal(cmap.to_csc(E2 - B2 * 3.0).data, A1)
    f.mesh.nodes[:, :] *= 1.5  # same topology, new geometry
    E3, B3, _ = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64), cmap)
    E4, B4, c4 = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    A3, A4 = cmap.to_csc(E3 - B3 * 3.0).data, c4.to_csc(E4 - B4 * 3.0).data
    assert np.array_equal(A3, A4) and not np.array_equal(A3, A1)


def test_to_csc_into_a_caller_buffer():
    """to_csc(..., out=) writes the values into the caller's array (reused
    across calls) with the same result as the default path; a wrong buffer
    is refused."""
    nodes, tets = structured_box(4, 3, 5, jitter=0.1, seed=6)
    f = Nedelec2Field(TetMesh(nodes, tets))
    er, ur = _blocky(f.ntets, np.random.default_rng(6))
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, np.zeros(0, np.int64))
    buf = cmap.host_buffer()
    for k2 in (1.0, 7.5):
        A = cmap.to_csc(E - B * k2, out=buf)
        assert np.shares_memory(A.data, buf)
        assert np.array_equal(A.data, cmap.to_csc(E - B * k2).data)
    with pytest.raises(ValueError):
        cmap.to_csc(E, out=np.zeros(cmap.nnz, np.float64))
    from emerge_b200.heat import Legrange2, tet_stiffness_matrix

    hf = Legrange2(TetMesh(nodes, tets))
    cond = np.zeros((3, 3, hf.mesh.n_tets))
    for d in range(3):
        cond[d, d] = 2.0
    K, hmap = tet_stiffness_matrix(hf, cond)
    hb = np.empty(hmap.nnz, np.float64)
    H = hmap.to_csc(K, out=hb)
    assert np.shares_memory(H.data, hb) and np.array_equal(H.data, hmap.to_csc(K).data)


def _orient(nodes, tets):
    """Reorder each tet to a positive determinant (the reference's meshes
    come that way from gmsh)."""
    tets = tets.copy()
    X = nodes[:, tets]
    det = np.einsum("it,it->t", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0], axis=0))
    flip = det < 0
    tets[1, flip], tets[2, flip] = tets[2, flip].copy(), tets[1, flip].copy()
    return tets


@pytest.mark.parametrize("n_tets", [1, 2])
def test_one_and_two_tet_meshes_full_tensors(n_tets):
    """The smallest meshes: one tet (A is its dense 20x20 block, nnz 400) and
    two tets sharing a face, with full (non-diagonal) complex er and ur, in
    both forms against the oracle."""
    rng = np.random.default_rng(40 + n_tets)
    base = np.array([[0.0, 1.0, 0.0, 0.0, 0.9], [0.0, 0.0, 1.0, 0.0, 0.8], [0.0, 0.0, 0.0, 1.0, 0.7]]) * 1e-3
    nodes = base + rng.uniform(-0.1e-3, 0.1e-3, base.shape)
    tets = np.array([[0, 1], [1, 2], [2, 3], [3, 4]], np.int64)[:, :n_tets]
    if n_tets == 1:
        nodes = nodes[:, :4]
    tets = _orient(nodes, tets)
    f = Nedelec2Field(TetMesh(nodes, tets))
    er = rng.uniform(1, 4, (3, 3, n_tets)) + 1j * rng.uniform(-0.2, 0.2, (3, 3, n_tets))
    ur = rng.uniform(-0.3, 0.3, (3, 3, n_tets)) + 1j * rng.uniform(-0.1, 0.1, (3, 3, n_tets))
    for d in range(3):
        ur[d, d] += 2.0
    none = np.zeros(0, np.int64)
    m = f.mesh
    E, B, cmap = tet_mass_stiffness_matrices(f, er, ur, none)
    dE, dB, ocmap = O.tet_mass_stiffness_matrices(f, er, ur, none)
    assert cmap.nnz == 4 * m.n_edges + 52 * m.n_tris + 168 * n_tets
    assert np.array_equal(cmap.indptr, ocmap.indptr) and np.array_equal(cmap.indices, ocmap.indices)
    if n_tets == 1:
        assert cmap.nnz == 400 and np.all(np.diff(cmap.indptr) == 20)
    k2 = (2 * np.pi * 10e9 / 299792458.0) ** 2
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-6)):
        E, B, _ = tet_mass_stiffness_matrices(f, er, ur, none, cmap, precision=precision)
        for a, (ra, rb) in ((E * 1.0, (1.0, 0.0)), (B * 1.0, (0.0, 1.0)), (E - B * k2, (1.0, -k2))):
            got = cmap.to_csc(a).data
            want = ocmap.values_lincomb(dE, dB, ra, rb)
            fro, mx = rel_err(got, want)
            assert fro <= tol and mx <= tol, (precision, ra, rb, fro, mx)
