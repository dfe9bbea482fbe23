"""libemgpu.so builds for sm_100a, loads without a GPU and exports every
symbol include/emgpu.h declares (no compute calls here)."""
import ctypes
import os
import re

from emerge_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "emgpu.h")).read()
    return sorted(set(re.findall(r"\b(emg_[a-z0-9_]+)\s*\(", src)))


def test_header_matches_binding_list():
    assert declared_symbols() == sorted(L.EXPORTS)


def test_library_loads_and_exports_all():
    lib = L.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.emg_version() >= 1


def test_host_only_entry_points():
    lib = L.lib()
    p = L.Plan()
    assert lib.emg_plan_init(12960, 12960, 17004, 27144, ctypes.byref(p)) == 0
    assert p.N == 88296 and p.n_items == 129600 and p.plan_bytes > 0 and p.workspace_bytes > 0
    assert lib.emg_plan_init(-1, 0, 0, 0, ctypes.byref(p)) == L.EMG_EINVAL
    assert b"negative" in lib.emg_last_error()
    assert p.record_bytes == 8
    wide = p.plan_bytes
    assert lib.emg_plan_set_record_width(ctypes.byref(p), 4) == 0 and p.record_bytes == 4
    assert p.plan_bytes < wide
    assert lib.emg_plan_set_record_width(ctypes.byref(p), 3) == L.EMG_EINVAL
    # enough for either element-value layout (210 packed / 220 block values per tet)
    assert lib.emg_assemble_workspace_size(10, L.EMG_FP64) == 10 * 220 * 16
    assert lib.emg_assemble_workspace_size(10, L.EMG_MIXED) == 10 * 220 * 8
    assert p.value_layout == L.EMG_LAYOUT_PACKED
    packed = p.plan_bytes
    assert lib.emg_plan_set_value_layout(ctypes.byref(p), L.EMG_LAYOUT_BLOCK) == 0
    assert p.value_layout == L.EMG_LAYOUT_BLOCK and p.plan_bytes < packed
    assert lib.emg_plan_set_value_layout(ctypes.byref(p), L.EMG_LAYOUT_COO) == L.EMG_EINVAL


def test_size_limits_are_range_errors():
    """Meshes beyond 32-bit indexing are refused on the host, before any
    device work: 400 slots per assembled tet must fit int32 (the reference
    COO slot index), and so must the DoF count 2(E + F)."""
    lib = L.lib()
    p = L.Plan()
    top = (2 ** 31 - 1) // 400
    assert lib.emg_plan_init(top, top, 100, 100, ctypes.byref(p)) == 0
    assert lib.emg_plan_init(top + 1, top + 1, 100, 100, ctypes.byref(p)) == L.EMG_ERANGE
    assert b"too large" in lib.emg_last_error()
    assert lib.emg_plan_init(10, 10, 2 ** 29, 2 ** 29, ctypes.byref(p)) == L.EMG_ERANGE
    assert lib.emg_plan_init(10, 11, 100, 100, ctypes.byref(p)) == L.EMG_EINVAL
