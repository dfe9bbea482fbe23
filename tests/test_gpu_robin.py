"""Robin (port) boundary term on the GPU against the reference's own output
(tests/golden/robin.npz) and the oracle. Tolerances: 1e-12 relative
(Frobenius and max entry) for the term alone and for A + term; the pattern is
A's, bit-exact."""
import numpy as np
import pytest

from emerge_b200 import _lib as L
from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.robin import RobinTerm, assemble_robin_bc
from emerge_b200.sweep import FrequencySweep
from oracle import oracle as O
from tests.golden_util import load_npz, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _sparse_rel(mine, ref):
    d = (mine - ref).tocsc()
    d.sum_duplicates()
    nref = np.sqrt((abs(ref.data) ** 2).sum())
    fro = np.sqrt((abs(d.data) ** 2).sum()) / nref
    mx = (abs(d.data).max() if d.nnz else 0.0) / abs(ref.data).max()
    return fro, mx


def test_port_term_matches_reference_golden():
    g = load_npz("robin.npz")
    wl = W.wr90_air()
    f = wl.field
    ids = g["port_ids"]
    gamma = complex(g["port_gamma"])
    Bmat = np.zeros(f.mesh.n_tris * 64, np.complex128)
    Bmat.reshape(-1, 64)[ids] = g["port_B"]
    ref = O.generate_csc(f, Bmat)
    _, _, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R = RobinTerm(f, ids, cmap)
    mine = R.to_csc(gamma)
    assert np.array_equal(mine.indptr, cmap.indptr) and np.array_equal(mine.indices, cmap.indices)
    fro, mx = _sparse_rel(mine, ref)
    assert fro <= TOL and mx <= TOL, (fro, mx)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_system_with_ports_matches_oracle(precision, tol):
    """A = K - k0^2 M + gamma R (drop-in combination) against the oracle's
    K - k0^2 M plus generate_csc of its Robin entries, on a lossy box."""
    wl = W.wr90_dielectric(n=(10, 6, 16), seed=5)
    f = wl.field
    ids = W.port_tris(wl)
    k0 = wl.k0
    gamma = W.rect_port_gamma(wl.freq)
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64), precision=precision)
    R = RobinTerm(f, ids, cmap)
    A = cmap.to_csc(E - B * k0 ** 2 + R * gamma)
    A2 = cmap.to_csc(E - B * k0 ** 2 + assemble_robin_bc(f, ids, gamma, cmap))
    assert np.array_equal(A.data, A2.data)
    dE, dB, ocmap = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    from scipy.sparse import csc_matrix

    K = csc_matrix((ocmap.values_lincomb(dE, dB, 1.0, -k0 ** 2), ocmap.indices, ocmap.indptr), shape=A.shape)
    ref = (K + O.generate_csc(f, O.robin_entries(f, ids, gamma))).tocsc()
    ref.sort_indices()
    assert np.array_equal(ref.indptr, A.indptr) and np.array_equal(ref.indices, A.indices)
    fro, mx = rel_err(A.data, ref.data)
    assert fro <= tol and mx <= tol, (fro, mx)


def test_repeated_triangles_count_twice_and_apply_is_linear():
    wl = W.wr90_air(n=(6, 4, 10))
    f = wl.field
    ids = W.port_tris(wl)
    _, _, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R1 = RobinTerm(f, ids, cmap).to_device(1.0).cpu().numpy()
    R2 = RobinTerm(f, np.concatenate([ids, ids]), cmap).to_device(1.0).cpu().numpy()
    assert np.allclose(R2, 2 * R1, rtol=1e-15, atol=0)
    g = 0.3 - 2.5j
    Rg = RobinTerm(f, ids, cmap).to_device(g).cpu().numpy()
    assert np.allclose(Rg, g * R1, rtol=1e-15, atol=0)
    assert np.count_nonzero(R1) > 0 and np.count_nonzero(R1) < cmap.nnz


def test_triangle_outside_the_assembled_pattern_raises():
    wl = W.wr90_air(n=(4, 3, 5))
    f = wl.field
    m = f.mesh
    ids = W.port_tris(wl)[:1]
    t = int(ids[0])
    touching = np.flatnonzero((m.tet_to_tri == t).any(axis=0))
    _, _, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, touching)  # the tri's tet is a conductor
    with pytest.raises(L.EmgMeshError):
        RobinTerm(f, ids, cmap)
    with pytest.raises(IndexError):
        RobinTerm(f, np.array([m.n_tris]), cmap)


def test_sweep_with_port_terms():
    wl = W.wr90_dielectric(n=(8, 5, 12), seed=2)
    f = wl.field
    z = f.mesh.nodes[2]
    from emerge_b200.mesh import plane_tris

    p1 = plane_tris(f.mesh, 2, float(z.min()))
    p2 = plane_tris(f.mesh, 2, float(z.max()))
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R1, R2 = RobinTerm(f, p1, cmap), RobinTerm(f, p2, cmap)
    sw = FrequencySweep(E, B, cmap, robin=[R1, R2])
    freqs = np.linspace(8e9, 12e9, 9)
    gam = np.array([W.rect_port_gamma(x) for x in freqs])
    A = sw.form(FrequencySweep.coefficients(freqs), robin_gamma=np.stack([gam, gam], axis=1))
    for i in (0, 4, 8):
        k0 = 2 * np.pi * freqs[i] / W.C0
        direct = cmap.to_csc(E - B * k0 ** 2 + R1 * gam[i] + R2 * gam[i]).data
        assert rel_err(A[i].cpu().numpy(), direct)[0] < 1e-13
    with pytest.raises(ValueError):
        sw.form(FrequencySweep.coefficients(freqs))


def test_port_force_matches_reference_golden():
    g = load_npz("robin.npz")
    wl = W.wr90_air()
    f = wl.field
    _, _, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R = RobinTerm(f, g["port_ids"], cmap)
    pts = R.quadrature_points()
    assert np.abs(pts - g["port_pts"]).max() <= 1e-15 * np.abs(pts).max()
    U = np.zeros(pts.shape, np.complex128)
    U[1] = (1 + 0.5j) * np.sin(np.pi * pts[0] / W.WR90[0])
    b = R.force(U).cpu().numpy()
    ref = g["port_b"]
    fro, mx = rel_err(b, ref)
    assert fro <= TOL and mx <= TOL, (fro, mx)
    b2 = R.force(U, R.force(U)).cpu().numpy()  # accumulates
    assert np.allclose(b2, 2 * b, rtol=1e-15, atol=0)


def test_driven_guide_solution_matches_oracle_system():
    """End to end: the system of a WR-90 section with two TE10 ports and a
    port-1 excitation, assembled on the GPU (A through the drop-in with the
    Robin terms, b through the forcing vector) and by the oracle, solved with
    scipy's SuperLU: the solutions agree to 1e-9 (the 1e-12 assembly parity
    times the conditioning of this small system)."""
    from scipy.sparse import csc_matrix
    from scipy.sparse.linalg import splu

    from emerge_b200.mesh import plane_tris

    wl = W.wr90_dielectric(n=(6, 3, 12), seed=9)
    f = wl.field
    m = f.mesh
    z = m.nodes[2]
    p1, p2 = plane_tris(m, 2, float(z.min())), plane_tris(m, 2, float(z.max()))
    k0, gamma = wl.k0, W.rect_port_gamma(wl.freq)
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R1, R2 = RobinTerm(f, p1, cmap), RobinTerm(f, p2, cmap)
    A = cmap.to_csc(E - B * k0 ** 2 + R1 * gamma + R2 * gamma)
    pts = R1.quadrature_points()
    U = np.zeros(pts.shape, np.complex128)
    U[1] = -2j * abs(gamma) * np.sin(np.pi * pts[0] / W.WR90[0])
    b = R1.force(U).cpu().numpy()
    dE, dB, oc = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    Aref = (csc_matrix((oc.values_lincomb(dE, dB, 1.0, -k0 ** 2), oc.indices, oc.indptr), shape=A.shape)
            + O.generate_csc(f, O.robin_entries(f, np.concatenate([p1, p2]), gamma))).tocsc()
    bref = O.force_entries(f, p1, U)
    assert rel_err(b, bref)[0] <= TOL
    x = splu(A).solve(b)
    xref = splu(Aref).solve(bref)
    assert np.linalg.norm(x - xref) <= 1e-9 * np.linalg.norm(xref)
    assert np.linalg.norm(Aref @ x - bref) <= 1e-9 * np.linalg.norm(bref)


def test_abc2_term_matches_reference_golden():
    """The second-order ABC correction (kind="abc2") over three faces of the
    12x6x30 box against the reference's abc_order_2_matrix output; the
    pattern is A's."""
    g = load_npz("abc2.npz")
    wl = W.wr90_air()
    f = wl.field
    ids = g["abc_ids"]
    cf = complex(g["abc_cf"])
    Mat = np.zeros(f.mesh.n_tris * 64, np.complex128)
    Mat.reshape(-1, 64)[ids] = g["abc_B"]
    ref = O.generate_csc(f, Mat)
    _, _, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    R2 = RobinTerm(f, ids, cmap, kind="abc2")
    mine = R2.to_csc(cf)
    assert np.array_equal(mine.indptr, cmap.indptr) and np.array_equal(mine.indices, cmap.indices)
    fro, mx = _sparse_rel(mine, ref)
    assert fro <= TOL and mx <= TOL, (fro, mx)
    with pytest.raises(ValueError):
        R2.force(np.zeros((3, 6, ids.size), np.complex128))
    with pytest.raises(ValueError):
        RobinTerm(f, ids, cmap, kind="abc3")


def test_system_with_ports_and_abc2_matches_oracle():
    """A = K - k0^2 M + gamma R_ports + c2 R_abc2 through the drop-in
    combination against the oracle's pieces, FP64, on a lossy box."""
    from scipy.sparse import csc_matrix

    from emerge_b200.mesh import plane_tris
    from emerge_b200.robin import abc_order_2_matrix

    wl = W.wr90_dielectric(n=(10, 6, 16), seed=7)
    f = wl.field
    m = f.mesh
    ports = W.port_tris(wl)
    sides = np.concatenate([plane_tris(m, 0, float(m.nodes[0].min())), plane_tris(m, 1, float(m.nodes[1].max()))])
    k0, gamma, c2 = wl.k0, W.rect_port_gamma(wl.freq), complex(0.02, -0.3)
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    A = cmap.to_csc(E - B * k0 ** 2 + RobinTerm(f, ports, cmap) * gamma + abc_order_2_matrix(f, sides, c2, cmap))
    dE, dB, oc = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    K = csc_matrix((oc.values_lincomb(dE, dB, 1.0, -k0 ** 2), oc.indices, oc.indptr), shape=A.shape)
    ref = (K + O.generate_csc(f, O.robin_entries(f, ports, gamma)) + O.generate_csc(f, O.abc2_entries(f, sides, c2)))
    ref = ref.tocsc()
    ref.sort_indices()
    assert np.array_equal(ref.indptr, A.indptr) and np.array_equal(ref.indices, A.indices)
    fro, mx = rel_err(A.data, ref.data)
    assert fro <= 1e-12 and mx <= 1e-12, (fro, mx)
