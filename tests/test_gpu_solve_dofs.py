"""Solve-DoF submatrix on the device against scipy's slicing of the same A,
A[:, ids][ids, :] (solver.py:2071): pattern and values bit-exact."""
import numpy as np
import pytest
import torch

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.mesh import plane_tris
from emerge_b200.robin import RobinTerm
from emerge_b200.solve_dofs import SolveSubmatrix

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("keep_frac", [1.0, 0.83, 0.3, 0.0])
def test_submatrix_matches_scipy_slicing(keep_frac):
    wl = W.wr90_dielectric(n=(8, 5, 12), seed=11)
    f = wl.field
    m = f.mesh
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    z = m.nodes[2]
    R = RobinTerm(f, plane_tris(m, 2, float(z.min())), cmap)
    data = E - B * wl.k0 ** 2 + R * W.rect_port_gamma(wl.freq)
    A = cmap.to_csc(data)
    rng = np.random.default_rng(3)
    ids = np.flatnonzero(rng.random(f.n_field) < keep_frac)
    sub = SolveSubmatrix(cmap, rng.permutation(np.concatenate([ids, ids[:7]])))  # order and repeats do not matter
    ref = A[:, ids][ids, :]
    mine = sub.to_csc(data)
    assert mine.shape == ref.shape and sub.M == ids.size
    assert np.array_equal(mine.indptr, ref.indptr) and np.array_equal(mine.indices, ref.indices)
    assert np.array_equal(mine.data, ref.data)
    b = torch.arange(f.n_field, dtype=torch.float64, device=cmap.device).to(torch.complex128)
    assert np.array_equal(sub.rhs(b).cpu().numpy(), np.arange(f.n_field)[ids].astype(np.complex128))


def test_pec_walls_removed():
    """The usual use: every DoF on the box's side walls (x and y faces) is a
    PEC DoF; the reduced system keeps the rest."""
    wl = W.wr90_air(n=(6, 4, 10))
    f = wl.field
    m = f.mesh
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    walls = np.concatenate([plane_tris(m, a, float(v)) for a in (0, 1) for v in (m.nodes[a].min(), m.nodes[a].max())])
    pec = np.unique(f.tri_to_field[:, walls])
    solve = np.setdiff1d(np.arange(f.n_field), pec)
    sub = SolveSubmatrix(cmap, solve)
    A = cmap.to_csc(E - B * wl.k0 ** 2)
    ref = A[:, solve][solve, :]
    mine = sub.to_csc(cmap.to_device(E - B * wl.k0 ** 2))
    assert np.array_equal(mine.indptr, ref.indptr) and np.array_equal(mine.indices, ref.indices)
    assert np.array_equal(mine.data, ref.data)
    with pytest.raises(IndexError):
        SolveSubmatrix(cmap, [f.n_field])


@pytest.mark.parametrize("reorder", ["none", "symrcm", "symamd", "metis"])
def test_device_solve_matches_superlu(reorder):
    """The reduced system of a lossy guide with a port term and PEC walls,
    solved on the device (emg_sparse_solve) and by scipy's SuperLU on the
    host: same solution to 1e-9 relative (two factorizations of a system of
    moderate condition), residual below 1e-10; the CSR conversion path for a
    non-symmetric caller agrees."""
    from scipy.sparse.linalg import splu

    wl = W.wr90_dielectric(n=(6, 3, 10), seed=4)
    f = wl.field
    m = f.mesh
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    z = m.nodes[2]
    R = RobinTerm(f, plane_tris(m, 2, float(z.min())), cmap)
    walls = np.concatenate([plane_tris(m, a, float(v)) for a in (0, 1) for v in (m.nodes[a].min(), m.nodes[a].max())])
    solve = np.setdiff1d(np.arange(f.n_field), np.unique(f.tri_to_field[:, walls]))
    sub = SolveSubmatrix(cmap, solve)
    A = cmap.to_device(E - B * wl.k0 ** 2 + R * W.rect_port_gamma(wl.freq))
    vals = sub.values(A)
    rng = np.random.default_rng(5)
    b = rng.normal(size=sub.M) + 1j * rng.normal(size=sub.M)
    x = sub.solve(vals, torch.from_numpy(b), reorder=reorder).cpu().numpy()
    Asel = sub.to_csc(A)
    xr = splu(Asel).solve(b)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)
    assert np.linalg.norm(Asel @ x - b) <= 1e-10 * np.linalg.norm(b)
    x2 = sub.solve(vals, torch.from_numpy(b), symmetric=False, reorder=reorder).cpu().numpy()
    assert np.linalg.norm(x2 - x) <= 1e-12 * np.linalg.norm(x)
    full = sub.expand(torch.from_numpy(x).to(cmap.device)).cpu().numpy()
    assert np.array_equal(full[solve], x) and not np.any(np.delete(full, solve))


def test_device_solve_reports_a_singular_system():
    wl = W.wr90_air(n=(3, 2, 3))
    f = wl.field
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, np.zeros(0, np.int64))
    sub = SolveSubmatrix(cmap, np.arange(f.n_field))
    Z = torch.zeros(sub.nnz, dtype=torch.complex128, device=cmap.device)  # every pivot exactly zero
    with pytest.raises(np.linalg.LinAlgError):
        sub.solve(Z, torch.ones(sub.M, dtype=torch.complex128))
    with pytest.raises(ValueError):
        sub.solve(Z, torch.ones(sub.M + 1, dtype=torch.complex128))
