"""Size-independent properties at the full size of the headline workload
(100x50x67 hexes, 2,010,000 tets, 557.8M nonzeros), where no oracle run fits
a test: the exact nonzero count 4E + 52F + 168T, the sum of A's values equal
to the sum of all element-slot values (every slot lands in exactly one
nonzero; FP64, 1e-12 of the absolute sum), bitwise determinism, linearity in
the combination's coefficients (1e-13), and the mixed form within 1e-6 of
FP64 (relative Frobenius and max entry) for A."""
import numpy as np
import pytest
import torch

from emerge_b200 import workloads as W
from emerge_b200.assembly import tet_mass_stiffness_matrices

pytestmark = pytest.mark.gpu


def test_full_size_properties():
    wl = W.wr90_dielectric()
    f = wl.field
    m = f.mesh
    none = np.zeros(0, np.int64)
    E, B, cmap = tet_mass_stiffness_matrices(f, wl.er, wl.ur, none)
    assert f.ntets == 2_010_000
    assert cmap.nnz == 4 * m.n_edges + 52 * m.n_tris + 168 * f.ntets
    assert np.array_equal(np.diff(cmap.indptr) > 0, np.ones(cmap.N, bool))
    k2 = wl.k0 ** 2
    A = cmap.to_device(E - B * k2).clone()
    # every element slot lands in exactly one nonzero
    slots = E.to_device() - k2 * B.to_device()
    s_slots = complex(slots.sum().item())
    scale = float(slots.abs().sum().item())
    del slots
    assert abs(complex(A.sum().item()) - s_slots) <= 1e-12 * scale
    # bitwise determinism
    assert torch.equal(cmap.to_device(E - B * k2), A)
    # linearity: 2K - 3M from the combination equals 2 K - 3 M formed apart
    K = cmap.to_device(E * 1.0).clone()
    M = cmap.to_device(B * 1.0).clone()
    L2 = cmap.to_device(E * 2.0 - B * 3.0)
    d = L2 - (2.0 * K - 3.0 * M)
    assert float(d.abs().max()) <= 1e-13 * float(L2.abs().max())
    del K, M, L2, d
    torch.cuda.empty_cache()
    # the mixed form within its stated tolerance
    E2, B2, _ = tet_mass_stiffness_matrices(f, wl.er, wl.ur, none, cmap, precision="mixed")
    A32 = cmap.to_device(E2 - B2 * k2)
    diff = A32 - A
    fro = float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(A))
    mx = float(diff.abs().max() / A.abs().max())
    assert fro <= 1e-6 and mx <= 1e-6, (fro, mx)
