"""The chunked CPU reference (oracle/chunked_oracle.c), which times the
reference's assembly over a whole mesh too large for its full COO arrays:
the same pattern as the reference's CSCMapping and, chunk size whatever it
is, the same A bit for bit as the one-piece scatter (each nonzero sums its
slots in the same order)."""
import numpy as np
import pytest

from emerge_b200.mesh import Nedelec2Field, TetMesh, structured_box
from oracle import oracle as O

K2 = (2 * np.pi * 10e9 / 299792458.0) ** 2


def _case(conductors):
    nodes, tets = structured_box(7, 5, 6, jitter=0.12, seed=5)
    f = Nedelec2Field(TetMesh(nodes, tets))
    nT = f.ntets
    rng = np.random.default_rng(2)
    er = np.zeros((3, 3, nT), np.complex128)
    ur = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        er[d, d] = rng.uniform(1, 10, nT) - 1j * rng.uniform(0, 0.1, nT)
        ur[d, d] = 1.0
    cond = np.sort(rng.choice(nT, nT // 9, replace=False)) if conductors else np.zeros(0, np.int64)
    return f, er, ur, cond


@pytest.mark.parametrize("conductors", [False, True])
@pytest.mark.parametrize("chunk", [1, 37, 1000, 10 ** 6])
def test_chunked_equals_one_piece(conductors, chunk):
    f, er, ur, cond = _case(conductors)
    dE, dB, pat = O.tet_mass_stiffness_matrices(f, er, ur, cond, nthreads=4)
    want = pat.values_lincomb(dE, dB, 1.0, -K2, nthreads=4)
    ch = O.ChunkedAssembly(f, er, ur, cond, chunk_tets=chunk, nthreads=4)
    assert np.array_equal(ch.indptr, pat.indptr) and np.array_equal(ch.indices, pat.indices)
    got = ch.step(1.0, -K2)
    assert np.array_equal(got.view(np.float64), want.view(np.float64))
    # a second step reuses the buffers and gives the same values
    assert np.array_equal(ch.step(1.0, -K2).view(np.float64), want.view(np.float64))
