"""emg_assemble_batch: several independent jobs (different meshes, plans,
materials, coefficients, conductor sets) assembled by one element launch and
one gather launch over a job table give each job's A bit for bit as
emg_assemble gives it alone, in every precision and material kind."""
import ctypes

import numpy as np
import pytest
import torch

from emerge_b200 import _lib as L
from emerge_b200 import workloads as W
from emerge_b200.assembly import DeviceMaterial, DeviceMesh, GpuCSCMapping, _Job

pytestmark = pytest.mark.gpu


def _cases():
    a = W.wr90_air(n=(6, 4, 10))
    b = W.wr90_dielectric(n=(8, 5, 9), seed=3)
    d = W.wr90_air(n=(12, 6, 30), seed=5)
    cond = np.arange(0, d.n_tets, 97, dtype=np.int64)
    c = W.wr90_pml_slivers(n=(10, 6, 6))  # diagonal tensors
    return [(a, None), (b, None), (d, cond)], [(c, None)]


def _setup(cases, dev, layout="block"):
    out = []
    for wl, cond in cases:
        dm = DeviceMesh(wl.field, cond, dev)
        cm = GpuCSCMapping(dm, value_layout=layout)
        mat = DeviceMaterial(wl.er, wl.ur, wl.n_tets, dev)
        out.append((wl, dm, cm, mat))
    return out


def _run_batch(items, precision, coefs, dev):
    descs = (L.AssemblyJobDesc * len(items))()
    keep = []
    for i, ((wl, dm, cm, mat), (a, b)) in enumerate(zip(items, coefs)):
        ws = torch.empty(max(L.lib().emg_assemble_workspace_size(cm.n_assy, precision), 1), dtype=torch.uint8,
                         device=dev)
        A = torch.full((cm.nnz,), complex("nan"), dtype=torch.complex128, device=dev)
        st = torch.zeros(2, dtype=torch.int64, device=dev)
        keep.append((ws, A, st))
        d = descs[i]
        d.plan = ctypes.pointer(cm.plan)
        d.d_plan, d.d_indptr = cm.d_plan.data_ptr(), cm.d_indptr.data_ptr()
        d.d_nodes, d.n_nodes, d.d_tets = dm.nodes.data_ptr(), dm.n_nodes, dm.tets.data_ptr()
        d.d_tetids = dm.tetids.data_ptr() if dm.tetids is not None else None
        d.mat = mat.struct()
        d.alpha_re, d.alpha_im, d.beta_re, d.beta_im = a.real, a.imag, b.real, b.imag
        d.d_values, d.d_A, d.d_status = ws.data_ptr(), A.data_ptr(), st.data_ptr()
    nb = int(L.lib().emg_assemble_batch_table_bytes(len(items)))
    h_tab = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
    d_tab = torch.empty(nb, dtype=torch.uint8, device=dev)
    L.check(L.lib().emg_assemble_batch(descs, len(items), precision, L.ptr(h_tab), L.ptr(d_tab), nb,
                                       L.stream_handle(dev)))
    torch.cuda.synchronize()
    for _, _, st in keep:
        assert int(st[0]) == 0
    return [A for _, A, _ in keep]


@pytest.mark.parametrize("layout", ["block", "packed"])
@pytest.mark.parametrize("precision", [L.EMG_FP64, L.EMG_MIXED, L.EMG_EXACT])
def test_batch_equals_single_jobs(precision, layout):
    dev = torch.device("cuda", 0)
    iso, diag = _cases()
    for group in (iso, diag):
        items = _setup(group, dev, layout)
        coefs = [(1.0 + 0.5j, -(3.0 + 0.25j) * (k + 1)) for k in range(len(items))]
        got = _run_batch(items, precision, coefs, dev)
        for (wl, dm, cm, mat), (a, b), A in zip(items, coefs, got):
            ref = cm.assemble_device(_Job(dm, mat, precision), a, b)[: cm.nnz]
            dm.check_status()
            assert torch.equal(A, ref)


def test_batch_rejects_mixed_kinds_and_small_tables():
    dev = torch.device("cuda", 0)
    iso, diag = _cases()
    items = _setup([iso[0], diag[0]], dev)
    with pytest.raises(L.EmgError, match="material kind"):
        _run_batch(items, L.EMG_FP64, [(1.0, 0.0)] * 2, dev)
    mixed_layouts = _setup([iso[0]], dev, "block") + _setup([iso[1]], dev, "packed")
    with pytest.raises(L.EmgError, match="value layout"):
        _run_batch(mixed_layouts, L.EMG_FP64, [(1.0, 0.0)] * 2, dev)
    descs = (L.AssemblyJobDesc * 1)()
    small = torch.empty(8, dtype=torch.uint8, pin_memory=True)
    assert L.lib().emg_assemble_batch(descs, 1, L.EMG_FP64, L.ptr(small), L.ptr(small), 8,
                                      L.stream_handle(dev)) == L.EMG_EINVAL
