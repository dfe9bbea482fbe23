"""ctypes binding of ``libemgpu.so`` (the C ABI declared in include/emgpu.h).

The library is built in-tree (``python -m emerge_b200.build``). There is no
CPU fallback: if the shared library or a CUDA device is missing, every entry
point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libemgpu.so")

EMG_OK, EMG_EINVAL, EMG_ECUDA, EMG_EMESH, EMG_ERANGE, EMG_EDEVICE = 0, -1, -2, -3, -4, -5
EMG_ST_INDEX, EMG_ST_DEGENERATE, EMG_ST_CAPACITY = 1, 2, 4
EMG_MAT_ISO, EMG_MAT_DIAG, EMG_MAT_FULL = 0, 1, 2
EMG_FP64, EMG_MIXED, EMG_EXACT = 0, 1, 2
EMG_OUT_LINCOMB, EMG_OUT_K, EMG_OUT_M = 0, 1, 2
EMG_LAYOUT_COO, EMG_LAYOUT_PACKED, EMG_LAYOUT_COO_T, EMG_LAYOUT_BLOCK = 0, 1, 2, 3

# every symbol include/emgpu.h declares
EXPORTS = (
    "emg_version", "emg_last_error", "emg_device_check", "emg_material_classify", "emg_status_reset", "emg_status_read", "emg_plan_init",
    "emg_plan_build", "emg_plan_finish", "emg_element_values", "emg_gather", "emg_assemble_workspace_size",
    "emg_assemble", "emg_form_sweep", "emg_assemble_noalloc", "emg_form_batch", "emg_plan_order",
    "emg_plan_set_record_width", "emg_plan_set_value_layout", "emg_assemble_batch_table_bytes", "emg_assemble_batch",
    "emg_robin_init", "emg_robin_build", "emg_abc2_build", "emg_robin_apply", "emg_robin_force",
    "emg_robin_build_dofs", "emg_csc_lookup", "emg_csc_shift",
    "emg_select_init", "emg_select_build", "emg_select_finish", "emg_select_values", "emg_ned2_interp",
    "emg_port_overlap", "emg_sparse_solve", "emg_coo_init", "emg_coo_rowcol", "emg_coo_build", "emg_coo_finish", "emg_coo_gather",
    "emg_leg2_element",
)


class EmgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"emgpu error {code}: {msg}")
        self.code = code


class EmgMeshError(EmgError, ValueError):
    """The device status word reported a bad index, a degenerate tet or a
    capacity overflow."""


class Plan(ctypes.Structure):
    _fields_ = [
        ("n_tets", ctypes.c_int64), ("n_assy", ctypes.c_int64), ("n_edges", ctypes.c_int64),
        ("n_tris", ctypes.c_int64), ("n_ent", ctypes.c_int64), ("n_items", ctypes.c_int64), ("N", ctypes.c_int64),
        ("nnz", ctypes.c_int64), ("max_col", ctypes.c_int64), ("off_ent_ptr", ctypes.c_size_t),
        ("off_item", ctypes.c_size_t), ("off_item_pos", ctypes.c_size_t), ("off_ent_cnt", ctypes.c_size_t),
        ("off_contrib", ctypes.c_size_t), ("off_posoff", ctypes.c_size_t), ("off_pidx", ctypes.c_size_t),
        ("off_order", ctypes.c_size_t),
        ("plan_bytes", ctypes.c_size_t),
        ("workspace_bytes", ctypes.c_size_t),
        ("record_bytes", ctypes.c_int32),
        ("value_layout", ctypes.c_int32),
        ("off_hoff", ctypes.c_size_t),
    ]


class Robin(ctypes.Structure):
    _fields_ = [("n_btris", ctypes.c_int64), ("n_slots", ctypes.c_int64), ("n_keys", ctypes.c_int64),
                ("keys_bytes", ctypes.c_size_t), ("values_bytes", ctypes.c_size_t), ("n_fslots", ctypes.c_int64),
                ("n_fkeys", ctypes.c_int64), ("fkeys_bytes", ctypes.c_size_t), ("fvalues_bytes", ctypes.c_size_t)]


class Select(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int64), ("M", ctypes.c_int64), ("nnz_sel", ctypes.c_int64),
                ("workspace_bytes", ctypes.c_size_t)]


class CooMap(ctypes.Structure):
    _fields_ = [("S", ctypes.c_int64), ("N", ctypes.c_int64), ("nnz", ctypes.c_int64), ("perm_bytes", ctypes.c_size_t),
                ("run_bytes", ctypes.c_size_t), ("workspace_bytes", ctypes.c_size_t)]


class FormItem(ctypes.Structure):
    _fields_ = [("K", ctypes.c_void_p), ("M", ctypes.c_void_p), ("P", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("nnz", ctypes.c_int64), ("group", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("coef", ctypes.c_double * 6)]


FORM_TILE = 32768


class Material(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("d_er", ctypes.c_void_p), ("d_ur", ctypes.c_void_p)]


class AssemblyJobDesc(ctypes.Structure):
    """emg_assembly_job: one job of emg_assemble_batch."""
    _fields_ = [("plan", ctypes.POINTER(Plan)), ("d_plan", ctypes.c_void_p), ("d_indptr", ctypes.c_void_p),
                ("d_nodes", ctypes.c_void_p), ("n_nodes", ctypes.c_int64), ("d_tets", ctypes.c_void_p),
                ("d_tetids", ctypes.c_void_p), ("mat", Material), ("alpha_re", ctypes.c_double),
                ("alpha_im", ctypes.c_double), ("beta_re", ctypes.c_double), ("beta_im", ctypes.c_double),
                ("d_values", ctypes.c_void_p), ("d_A", ctypes.c_void_p), ("d_status", ctypes.c_void_p)]


_lib = None
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double


def lib():
    """Load libemgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m emerge_b200.build` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.emg_version.restype = ctypes.c_int
    L.emg_last_error.restype = ctypes.c_char_p
    L.emg_device_check.argtypes = [ctypes.c_int]
    L.emg_status_reset.argtypes = [_P, _P]
    L.emg_material_classify.argtypes = [_P, _I64, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]
    L.emg_status_read.argtypes = [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), _P]
    L.emg_plan_init.argtypes = [_I64, _I64, _I64, _I64, ctypes.POINTER(Plan)]
    L.emg_plan_build.argtypes = [ctypes.POINTER(Plan), _P, _P, _P, _P, _P, _P, _P, _P, _P]
    L.emg_plan_finish.argtypes = [ctypes.POINTER(Plan), _P, _P, _P, _P, _P, _P, _P, _P]
    L.emg_element_values.argtypes = [_P, _I64, _P, _I64, _P, _I64, ctypes.POINTER(Material), ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _P, _P, _P]
    L.emg_gather.argtypes = [ctypes.POINTER(Plan), _P, _P, _P, _P, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _P,
                             _P, _P]
    L.emg_assemble_workspace_size.argtypes = [_I64, ctypes.c_int]
    L.emg_assemble_workspace_size.restype = ctypes.c_size_t
    L.emg_assemble.argtypes = [ctypes.POINTER(Plan), _P, _P, _P, _I64, _P, _P, ctypes.POINTER(Material),
                               ctypes.c_int, _D, _D, _D, _D, _P, ctypes.c_size_t, _P, _P, _P]
    L.emg_assemble_batch_table_bytes.argtypes = [ctypes.c_int]
    L.emg_assemble_batch_table_bytes.restype = ctypes.c_size_t
    L.emg_assemble_batch.argtypes = [ctypes.POINTER(AssemblyJobDesc), ctypes.c_int, ctypes.c_int, _P, _P,
                                     ctypes.c_size_t, _P]
    L.emg_form_sweep.argtypes = [_P, _P, _P, _I64, ctypes.POINTER(_D), ctypes.c_int, _P, _I64, _P]
    L.emg_form_batch.argtypes = [_P, _P, _P, ctypes.c_int, _P]
    L.emg_plan_set_record_width.argtypes = [ctypes.POINTER(Plan), ctypes.c_int]
    L.emg_plan_set_value_layout.argtypes = [ctypes.POINTER(Plan), ctypes.c_int]
    L.emg_plan_order.argtypes = [ctypes.POINTER(Plan), _P, _P, _I64, _P, _P, _P, _P]
    L.emg_robin_init.argtypes = [_I64, ctypes.POINTER(Robin)]
    L.emg_abc2_build.argtypes = [ctypes.POINTER(Robin), _P, _I64, _P, _P, _I64, _I64, _P, _P, _P, _I64, _P, _P, _P,
                                 _P]
    L.emg_robin_build.argtypes = [ctypes.POINTER(Robin), _P, _I64, _P, _P, _I64, _I64, _P, _P, _P, _I64, _P, _P, _P,
                                  _P]
    L.emg_robin_apply.argtypes = [ctypes.POINTER(Robin), _P, _P, _D, _D, _P, _I64, _P]
    L.emg_robin_build_dofs.argtypes = [ctypes.POINTER(Robin), _P, _I64, _P, _P, _I64, _I64, _P, _P, _P, _P, _I64, _P,
                                       _P, _P, _P]
    L.emg_csc_lookup.argtypes = [_P, _P, _I64, _P, _P, _I64, _P, _P]
    L.emg_csc_shift.argtypes = [_P, _I64, ctypes.c_int, _P, _P, ctypes.c_int, _P, _P, _I64, _P, _I64, _P]
    L.emg_select_init.argtypes = [_I64, ctypes.POINTER(Select)]
    L.emg_select_build.argtypes = [ctypes.POINTER(Select), _P, _P, _P, _P, _P, _P, _P]
    L.emg_select_finish.argtypes = [ctypes.POINTER(Select), _P, _P, _P, _P, _P, _P, _P, _P]
    L.emg_select_values.argtypes = [ctypes.POINTER(Select), _P, _P, _I64, _P, _P]
    L.emg_ned2_interp.argtypes = [_P, _I64, _P, _I64, _P, _P, _I64, _I64, _P, _P, _I64, _P, _P, _P]
    L.emg_port_overlap.argtypes = [_P, _I64, _P, _I64, _P, _P, _P, _I64, _I64, _P, _P, _P, _I64, _P, ctypes.c_int, _P,
                                   _D, _P, _P, _P, _P]
    L.emg_sparse_solve.argtypes = [_I64, _I64, _P, _P, _P, _P, _P, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_I64),
                                   _P]
    L.emg_coo_init.argtypes = [_I64, _I64, ctypes.POINTER(CooMap)]
    L.emg_coo_rowcol.argtypes = [_P, ctypes.c_int, _I64, _P, _P, _P]
    L.emg_coo_build.argtypes = [ctypes.POINTER(CooMap), _P, _P, _P, _P, _P, _P, _P]
    L.emg_coo_finish.argtypes = [ctypes.POINTER(CooMap), _P, _P, _P, _P, _P, _P, _P]
    L.emg_coo_gather.argtypes = [ctypes.POINTER(CooMap), _P, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P]
    L.emg_leg2_element.argtypes = [_P, _I64, _P, _I64, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P]
    L.emg_robin_force.argtypes = [ctypes.POINTER(Robin), _P, _I64, _P, _P, _I64, _I64, _P, _P, _P, _P, _P, _I64, _P,
                                  _P]
    L.emg_assemble_noalloc.argtypes = [ctypes.POINTER(Plan), _P, _P, _P, _I64, _P, _P, ctypes.POINTER(Material),
                                       ctypes.c_int, _D, _D, _D, _D, _P, _P, _P]
    for name in ("emg_device_check", "emg_material_classify", "emg_status_reset", "emg_status_read", "emg_plan_init", "emg_plan_build",
                 "emg_plan_finish", "emg_element_values", "emg_gather", "emg_assemble", "emg_form_sweep",
                 "emg_assemble_noalloc", "emg_form_batch", "emg_plan_order", "emg_plan_set_record_width", "emg_assemble_batch",
                 "emg_robin_init", "emg_robin_build", "emg_abc2_build",
                 "emg_robin_apply", "emg_robin_force", "emg_select_init", "emg_select_build", "emg_select_finish",
                 "emg_select_values", "emg_ned2_interp", "emg_port_overlap", "emg_sparse_solve", "emg_coo_init", "emg_coo_rowcol",
                 "emg_coo_build", "emg_coo_finish", "emg_coo_gather", "emg_leg2_element", "emg_plan_set_value_layout",
                 "emg_robin_build_dofs", "emg_csc_lookup", "emg_csc_shift"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != EMG_OK:
        msg = lib().emg_last_error().decode(errors="replace")
        if rc == EMG_EMESH:
            raise EmgMeshError(rc, msg)
        raise EmgError(rc, msg)


def ptr(t) -> ctypes.c_void_p:
    """Raw device/host pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return ctypes.c_void_p(0)
    return ctypes.c_void_p(t.data_ptr())


def stream_handle(device=None) -> ctypes.c_void_p:
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
