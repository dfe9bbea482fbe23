"""emg_assemble_noalloc: the assembly entry point for callers that cannot
allocate device memory at the call site (its element-value scratch is a
96 MiB file-scope device array). Called through the C ABI twice in a row, it
must reproduce emg_assemble (same plan, inputs and precision) within the
plain-FP64 tolerance of the parity tests (1e-12 relative) and reject plans
larger than its scratch. Collected last on purpose; it must also pass alone
in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

from emerge_b200 import _lib as L
from emerge_b200.assembly import DeviceMaterial, DeviceMesh, GpuCSCMapping
from emerge_b200.workloads import wr90_air, wr90_dielectric

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _call_both(wl, precision):
    dev = torch.device("cuda", torch.cuda.current_device())
    dmesh = DeviceMesh(wl.field, wl.conductor_tets, dev)
    cmap = GpuCSCMapping(dmesh)
    dmat = DeviceMaterial(wl.er, wl.ur, wl.n_tets, dev)
    mat = dmat.struct()
    lib = L.lib()
    st = L.stream_handle(dev)
    a, b = 1.0 + 0j, complex(-wl.k0 ** 2)
    status = torch.zeros(2, dtype=torch.int64, device=dev)

    def run(fn_noalloc):
        out = torch.full((cmap.nnz,), float("nan"), dtype=torch.complex128, device=dev)
        L.check(lib.emg_status_reset(L.ptr(status), st))
        common = (ctypes.byref(cmap.plan), L.ptr(cmap.d_plan), L.ptr(cmap.d_indptr), L.ptr(dmesh.nodes),
                  dmesh.n_nodes, L.ptr(dmesh.tets), L.ptr(dmesh.tetids), ctypes.byref(mat), precision, a.real, a.imag,
                  b.real, b.imag)
        if fn_noalloc:
            L.check(lib.emg_assemble_noalloc(*common, L.ptr(out), L.ptr(status), st))
        else:
            ws = torch.empty(lib.emg_assemble_workspace_size(dmesh.n_assy, precision), dtype=torch.uint8, device=dev)
            L.check(lib.emg_assemble(*common, L.ptr(ws), ws.numel(), L.ptr(out), L.ptr(status), st))
        f, i = ctypes.c_int64(), ctypes.c_int64()
        L.check(lib.emg_status_read(L.ptr(status), ctypes.byref(f), ctypes.byref(i), st))
        assert f.value == 0
        return out.cpu().numpy()

    ref = run(False)
    first = run(True)
    second = run(True)
    return ref, first, second


@pytest.mark.parametrize("precision", [L.EMG_FP64, L.EMG_MIXED])
def test_noalloc_matches_workspace_entry_point_twice(precision):
    ref, first, second = _call_both(wr90_air(), precision)
    for got in (first, second):
        assert np.isfinite(got).all()
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        mx = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= TOL and mx <= TOL, (err, mx)


def test_noalloc_second_mesh_after_first():
    # a different (smaller) plan after a larger one: the shared array's stale
    # contents must not leak into the result
    _call_both(wr90_air(), L.EMG_FP64)
    ref, first, second = _call_both(wr90_dielectric(n=(6, 4, 8)), L.EMG_FP64)
    assert np.abs(first - ref).max() <= TOL * np.abs(ref).max()
    assert np.abs(second - ref).max() <= TOL * np.abs(ref).max()


def test_noalloc_rejects_plans_beyond_its_scratch():
    lib = L.lib()
    plan = L.Plan()
    L.check(lib.emg_plan_init(40000, 40000, 48000, 80000, ctypes.byref(plan)))  # 40,000 tets > 28,597
    mat = L.Material(L.EMG_MAT_ISO, None, None)
    rc = lib.emg_assemble_noalloc(ctypes.byref(plan), None, None, None, 0, None, None, ctypes.byref(mat), L.EMG_FP64,
                                  1.0, 0.0, 0.0, 0.0, None, None, None)
    assert rc == L.EMG_ERANGE
    assert b"static scratch" in lib.emg_last_error()
