"""Column sharding on the GPU: the shards of 1, 2 and 3 ranks, assembled one
after another on this GPU (they never wait on one another), merge into a
matrix bitwise equal to the unsharded GPU assembly."""
import numpy as np
import pytest

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.partition import ShardedAssembly, merge_blocks, partition

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_shards_merge_to_full(precision):
    wl = W.wr90_dielectric(n=(16, 8, 30), seed=6)
    f = wl.field
    cond = np.arange(5, f.ntets, 67)
    k0 = wl.k0
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, cond, precision=precision)
    ref = cmap.to_csc(E - B * k0 ** 2)
    for world in (1, 2, 3):
        blocks = [ShardedAssembly(f, wl.er, wl.ur, s, precision).block(1.0 + 0j, complex(-k0 ** 2))
                  for s in partition(f.mesh, world, cond)]
        ip, ix, vv = merge_blocks(blocks, f.n_field)
        assert np.array_equal(ip, ref.indptr) and np.array_equal(ix, ref.indices), world
        assert np.array_equal(vv, ref.data), world
