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
