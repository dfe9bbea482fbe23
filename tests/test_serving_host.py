"""Host-side pieces of the serving engine that need no GPU: the closed-form
nonzero count used for admission, checked against the oracle's CSC pattern,
and the footprint estimate's bounds."""
import numpy as np
import pytest

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
    # K, M and 4 output slots (complex128) plus the packed element values of K and of M
    assert fp64 >= 6 * 16 * nnz + 2 * 220 * 16 * m.n_tets  # workspaces sized for either value layout
    assert abs((fp64 - mixed) - 2 * 220 * 8 * m.n_tets) <= 512
    # the cold-cache footprint is the mesh entry's plus the job's own
    assert fp64 == j.mesh_footprint() + j.job_footprint(0, 4)
    assert j.mesh_key == AssemblyJob(wl.field, wl.er, wl.ur, np.array([9e9])).mesh_key


def test_arena_first_fit_coalescing_and_block_bounds():
    import torch

    from emerge_b200.serving import ARENA_ALIGN, DeviceArena

    a = DeviceArena(10 * ARENA_ALIGN, "cpu")
    b1, b2, b3 = a.reserve(3 * ARENA_ALIGN), a.reserve(ARENA_ALIGN + 1), a.reserve(3 * ARENA_ALIGN)
    assert (b1.off, b2.off, b3.off) == (0, 3 * ARENA_ALIGN, 5 * ARENA_ALIGN) and a.in_use == 8 * ARENA_ALIGN
    assert a.reserve(3 * ARENA_ALIGN) is None  # 2 blocks left
    a.release(b2)
    a.release(b1)  # coalesces with b2's space: 5 free blocks at 0
    b4 = a.reserve(5 * ARENA_ALIGN)
    assert b4.off == 0
    a.release(b3)
    a.release(b4)
    assert a._free == [(0, 10 * ARENA_ALIGN)] and a.in_use == 0 and a.peak == 8 * ARENA_ALIGN
    blk = a.reserve(2 * ARENA_ALIGN)
    x = blk(16, torch.complex128)  # 256 B
    y = blk(3, torch.int32)
    assert x.numel() == 16 and y.numel() == 3 and y.data_ptr() - x.data_ptr() == ARENA_ALIGN
    with pytest.raises(MemoryError):
        blk(1, torch.uint8)
