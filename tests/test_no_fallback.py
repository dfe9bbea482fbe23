"""The product path has no CPU fallback: without a CUDA device the drop-in
calls raise instead of computing on the host, and a missing library is a
loud error naming the build step. Host-only."""
import numpy as np
import pytest
import torch

from emerge_b200 import _lib as L
from emerge_b200 import heat
from emerge_b200.assembly import tet_mass_stiffness_matrices
from emerge_b200.mesh import Nedelec2Field, TetMesh, structured_box


@pytest.mark.skipif(torch.cuda.is_available(), reason="a CUDA device is present")
def test_drop_in_calls_refuse_to_run_without_a_gpu():
    nodes, tets = structured_box(2, 2, 2, seed=1)
    f = Nedelec2Field(TetMesh(nodes, tets))
    er = np.zeros((3, 3, f.ntets), complex)
    for d in range(3):
        er[d, d] = 1.0
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        tet_mass_stiffness_matrices(f, er, er.copy(), np.zeros(0, np.int64))
    hf = heat.Legrange2(TetMesh(nodes, tets))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        heat.tet_mass_matrix(hf, np.ones(hf.mesh.n_tets))


def test_missing_library_is_a_loud_error(monkeypatch, tmp_path):
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "libemgpu.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        L.lib()
