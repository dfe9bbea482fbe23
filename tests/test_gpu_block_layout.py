"""The entity-pair block layout (EMG_LAYOUT_BLOCK) against the packed
triangle: the same A bit for bit in every form and material kind, the same
pattern, the COO gather still served by a block plan, and the plan's guards."""
import ctypes

import numpy as np
import pytest
import torch

from emerge_b200 import _lib as L
from emerge_b200.assembly import DeviceMaterial, DeviceMesh, GpuCSCMapping, _Job, _prec
from emerge_b200.mesh import Nedelec2Field, TetMesh, structured_box

pytestmark = pytest.mark.gpu


def _tensors(kind, nT, rng):
    t = np.zeros((3, 3, nT), np.complex128)
    u = np.zeros((3, 3, nT), np.complex128)
    for d in range(3):
        base = rng.uniform(1, 8, nT) * (1 - 1j * rng.uniform(1e-3, 1e-2, nT))
        t[d, d] = base if kind == "iso" else base * rng.uniform(0.5, 1.5, nT)
        u[d, d] = 1.0 if kind == "iso" else rng.uniform(1, 2, nT)
    if kind == "full":
        for r in range(3):
            for c in range(3):
                if r != c:
                    t[r, c] = rng.uniform(-0.3, 0.3, nT) + 0.05j * rng.uniform(-1, 1, nT)
                    u[r, c] = rng.uniform(-0.1, 0.1, nT)
    return t, u


@pytest.mark.parametrize("kind", ["iso", "diag", "full"])
@pytest.mark.parametrize("precision", ["fp64", "mixed", "exact"])
def test_block_layout_equals_packed_bitwise(kind, precision):
    nodes, tets = structured_box(9, 6, 7, jitter=0.15, seed=4)
    f = Nedelec2Field(TetMesh(nodes, tets))
    er, ur = _tensors(kind, f.ntets, np.random.default_rng(7))
    dm = DeviceMesh(f, np.array([3, 17, 100], np.int64))
    job = _Job(dm, DeviceMaterial(er, ur, dm.n_tets, dm.device), _prec(precision))
    cp = GpuCSCMapping(dm, value_layout="packed")
    cb = GpuCSCMapping(dm, value_layout="block")
    assert cb.plan.value_layout == L.EMG_LAYOUT_BLOCK and cp.plan.value_layout == L.EMG_LAYOUT_PACKED
    assert torch.equal(cp.d_indptr, cb.d_indptr) and torch.equal(cp.d_indices[: cp.nnz], cb.d_indices[: cb.nnz])
    a, b = 1.0 + 0.25j, -2345.5 + 1.25j
    Ap = cp.assemble_device(job, a, b)[: cp.nnz]
    Ab = cb.assemble_device(job, a, b)[: cb.nnz]
    dm.check_status()
    assert torch.equal(Ap, Ab)
    assert torch.count_nonzero(Ab) > 0


def test_block_plan_serves_the_coo_gather():
    nodes, tets = structured_box(5, 4, 6, jitter=0.1, seed=3)
    f = Nedelec2Field(TetMesh(nodes, tets))
    dm = DeviceMesh(f, None)
    rng = np.random.default_rng(1)
    coo = rng.normal(size=(f.ntets, 20, 20)) + 1j * rng.normal(size=(f.ntets, 20, 20))
    coo = coo + coo.transpose(0, 2, 1)
    v = torch.from_numpy(coo.reshape(-1)).to(dm.device)
    cp = GpuCSCMapping(dm, value_layout="packed")
    cb = GpuCSCMapping(dm, value_layout="block")
    assert torch.equal(cp.gather_device(v)[: cp.nnz], cb.gather_device(v)[: cb.nnz])


def test_layout_guards():
    lib = L.lib()
    p = L.Plan()
    L.check(lib.emg_plan_init(1000, 1000, 1500, 2500, ctypes.byref(p)))
    packed_bytes = p.plan_bytes
    assert lib.emg_plan_set_value_layout(ctypes.byref(p), 7) == L.EMG_EINVAL
    L.check(lib.emg_plan_set_value_layout(ctypes.byref(p), L.EMG_LAYOUT_BLOCK))
    assert p.value_layout == L.EMG_LAYOUT_BLOCK and p.plan_bytes < packed_bytes
    # a packed gather on a block plan (and the reverse) is refused before any launch
    assert lib.emg_gather(ctypes.byref(p), ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None,
                          L.EMG_FP64, L.EMG_LAYOUT_PACKED, 1.0, 0.0, 0.0, 0.0, ctypes.c_void_p(16), None,
                          None) == L.EMG_EINVAL
