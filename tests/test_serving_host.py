"""Host-side pieces of the serving engine that need no GPU: the closed-form
nonzero count used for admission, checked against the oracle's CSC pattern,
and the footprint estimate's bounds."""
import numpy as np

from emerge_b200 import workloads as W
from emerge_b200.serving import AssemblyJob, nnz_of
from oracle import oracle as O


def test_nnz_closed_form_matches_oracle_pattern():
    for wl in (W.wr90_air(n=(6, 4, 10)), W.wr90_dielectric(n=(8, 5, 9), seed=3), W.wr90_pml_slivers(n=(10, 6, 6))):
        m = wl.field.mesh
        _, _, cmap = O.tet_mass_stiffness_matrices(wl.field, wl.er, wl.ur, np.zeros(0, np.int64))
        assert nnz_of(m.n_tets, m.n_edges, m.n_tris) == cmap.indices.size


def test_footprint_covers_resident_arrays():
    wl = W.wr90_air(n=(12, 6, 30))
    m = wl.field.mesh
    j = AssemblyJob(wl.field, wl.er, wl.ur, np.array([10e9]))
    nnz = nnz_of(m.n_tets, m.n_edges, m.n_tris)
    fp64, mixed = j.footprint(0, 4), j.footprint(1, 4)
    # K, M and 4 output slots (complex128) plus the packed element values
    assert fp64 >= 6 * 16 * nnz + 210 * 16 * m.n_tets
    assert fp64 - mixed == 210 * 8 * m.n_tets
