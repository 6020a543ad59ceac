"""Loader for the in-tree CUDA engine ``libcqgpu.so`` (C ABI declared in include/cqgpu.h).

The library is built in-tree by ``__graft_entry__.build()`` (or ``python -m
chronusq_public_b200.build``).  There is no CPU fallback: when the shared library is
missing or no CUDA device is present, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcqgpu.so")

_lib = None


class CqgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("cqgpu error %d (%s): %s" % (status, STATUS.get(status, "?"), msg))
        self.status = status


STATUS = {0: "ok", 1: "bad argument", 2: "out of device memory", 3: "CUDA error",
          4: "device wait timed out", 5: "non-finite input", 6: "invalid call order",
          7: "unsupported input"}

EXPORTED = [
    "cqg_version", "cqg_status_string", "cqg_create", "cqg_destroy", "cqg_last_error",
    "cqg_set_basis", "cqg_set_threshold", "cqg_set_precision", "cqg_get_schwarz",
    "cqg_get_sizes", "cqg_twoe_contract_direct", "cqg_form_pt", "cqg_get_stats",
    "cqg_set_timing", "cqg_class_name", "cqg_probe_fma_peak", "cqg_one_e", "cqg_set_list_budget",
    "cqg_set_basis_batch", "cqg_get_batch_layout", "cqg_twoe_contract_direct_batch", "cqg_one_e_batch",
    "cqg_set_graph_mode", "cqg_graph_status", "cqg_autotune_next", "cqg_get_launch_shapes", "cqg_set_active",
    "cqg_mlp_gemm_bf16", "cqg_mlp_silu_bwd", "cqg_mlp_to_bf16", "cqg_mlp_colsum", "cqg_mlp_mse", "cqg_mlp_adam",
    "cqg_one_e_noalloc", "cqg_dipole", "cqg_get_schedule", "cqg_set_schedule",
    "cqg_set_fusion", "cqg_get_fusion", "cqg_mlp_adam_dev", "cqg_set_siblings", "cqg_get_siblings",
    "cqg_schedule_lists", "cqg_list_class", "cqg_set_sibling_min",
]


class CqgStats(ctypes.Structure):
    _fields_ = [
        ("quartets", ctypes.c_longlong),
        ("quartets_fp32", ctypes.c_longlong),
        ("prim_quartets", ctypes.c_longlong),
        ("model_flops", ctypes.c_double),
        ("model_flops_fp32", ctypes.c_double),
        ("ms_screen", ctypes.c_double),
        ("ms_eri", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("launches", ctypes.c_longlong),
        ("chunks", ctypes.c_longlong),
        ("class_quartets", ctypes.c_longlong * 55),
        ("class_ms", ctypes.c_double * 55),
        ("ms_fused", ctypes.c_double),
        ("fused_tier", ctypes.c_int),
        ("list_entries", ctypes.c_longlong),
        ("sibling_classes", ctypes.c_longlong),
    ]


def load(path: str = LIB_PATH):
    """Load the shared library and declare argument types (no GPU needed)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libcqgpu.so is not built (expected at %s); run __graft_entry__.build()" % path)
    L = ctypes.CDLL(path)
    vp, d, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.cqg_version.restype = ctypes.c_char_p
    L.cqg_status_string.restype = ctypes.c_char_p
    L.cqg_status_string.argtypes = [ctypes.c_int]
    L.cqg_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int]
    L.cqg_destroy.argtypes = [vp]
    L.cqg_last_error.argtypes = [vp]
    L.cqg_last_error.restype = ctypes.c_char_p
    L.cqg_set_basis.argtypes = [vp, ctypes.c_int, i, i, i, d, d, d]
    L.cqg_set_threshold.argtypes = [vp, ctypes.c_double]
    L.cqg_set_precision.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.cqg_get_schwarz.argtypes = [vp, d]
    L.cqg_get_sizes.argtypes = [vp, i, i, i]
    L.cqg_twoe_contract_direct.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(vp), i, d,
                                           ctypes.c_int, ctypes.c_int, vp]
    L.cqg_form_pt.argtypes = [vp, ctypes.c_int, ctypes.c_double, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp]
    L.cqg_get_stats.argtypes = [vp, ctypes.POINTER(CqgStats)]
    L.cqg_set_timing.argtypes = [vp, ctypes.c_int]
    L.cqg_set_list_budget.argtypes = [vp, ctypes.c_longlong]
    L.cqg_set_basis_batch.argtypes = [vp, ctypes.c_int, i, i, i, i, d, d, d]
    L.cqg_get_batch_layout.argtypes = [vp, i, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.cqg_twoe_contract_direct_batch.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(vp), i, d,
                                                 ctypes.c_char_p, vp]
    L.cqg_one_e_batch.argtypes = [vp, i, d, d, vp, vp, vp, vp]
    L.cqg_set_graph_mode.argtypes = [vp, ctypes.c_longlong, ctypes.c_int]
    L.cqg_graph_status.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), i, i, i]
    L.cqg_autotune_next.argtypes = [vp]
    L.cqg_get_launch_shapes.argtypes = [vp, i, i]
    L.cqg_get_schedule.argtypes = [vp, i, i, i, i]
    L.cqg_set_schedule.argtypes = [vp, i, i, i, i]
    L.cqg_set_fusion.argtypes = [vp, ctypes.c_int]
    L.cqg_get_fusion.argtypes = [vp, i, d]
    L.cqg_set_siblings.argtypes = [vp, ctypes.c_int]
    L.cqg_get_siblings.argtypes = [vp, i]
    L.cqg_schedule_lists.argtypes = []
    L.cqg_list_class.argtypes = [ctypes.c_int]
    L.cqg_set_sibling_min.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.cqg_set_active.argtypes = [vp, ctypes.c_char_p]
    ll, f, fp = ctypes.c_longlong, ctypes.c_float, ctypes.POINTER(ctypes.c_float)
    L.cqg_mlp_gemm_bf16.argtypes = [vp, ll, ll, vp, ll, ll, vp, ll, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                    vp, ll, ctypes.c_int, ctypes.c_int, vp]
    L.cqg_mlp_silu_bwd.argtypes = [vp, vp, vp, ll, vp]
    L.cqg_mlp_to_bf16.argtypes = [vp, vp, ll, vp]
    L.cqg_mlp_colsum.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
    L.cqg_mlp_mse.argtypes = [vp, vp, vp, ll, f, vp, vp, vp]
    L.cqg_mlp_adam.argtypes = [vp, vp, vp, vp, ll, f, f, f, f, ctypes.c_int, f, vp, vp]
    L.cqg_mlp_adam_dev.argtypes = [vp, vp, vp, vp, ll, vp, f, f, f, f, vp, vp]
    L.cqg_class_name.argtypes = [ctypes.c_int]
    L.cqg_class_name.restype = ctypes.c_char_p
    L.cqg_probe_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, d]
    L.cqg_one_e.argtypes = [vp, ctypes.c_int, d, d, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp]
    L.cqg_one_e_noalloc.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int, vp]
    L.cqg_dipole.argtypes = [vp, d, vp, ctypes.c_int, ctypes.c_int, vp]
    for name in ["cqg_create", "cqg_destroy", "cqg_set_basis", "cqg_set_threshold", "cqg_set_precision",
                 "cqg_get_schwarz", "cqg_get_sizes", "cqg_twoe_contract_direct", "cqg_form_pt",
                 "cqg_get_stats", "cqg_set_timing", "cqg_probe_fma_peak", "cqg_one_e",
                 "cqg_set_list_budget", "cqg_set_basis_batch", "cqg_get_batch_layout",
                 "cqg_twoe_contract_direct_batch", "cqg_one_e_batch", "cqg_set_graph_mode",
                 "cqg_graph_status", "cqg_autotune_next", "cqg_get_launch_shapes", "cqg_set_active",
                 "cqg_mlp_gemm_bf16", "cqg_mlp_silu_bwd", "cqg_mlp_to_bf16", "cqg_mlp_colsum", "cqg_mlp_mse",
                 "cqg_mlp_adam", "cqg_one_e_noalloc", "cqg_dipole", "cqg_get_schedule", "cqg_set_schedule", "cqg_set_fusion", "cqg_get_fusion", "cqg_mlp_adam_dev",
                 "cqg_set_siblings", "cqg_get_siblings", "cqg_schedule_lists", "cqg_list_class",
                 "cqg_set_sibling_min"]:
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def lib():
    return load()


def check(status: int, ctx=None):
    if status != 0:
        msg = ""
        if ctx:
            msg = (lib().cqg_last_error(ctx) or b"").decode()
        raise CqgError(status, msg)


def schedule_lists():
    """Names of the schedule's work lists, in cqg_get_schedule order: the FP64 then the FP32
    pair-entry lists of the quartet classes, then their FP64 and FP32 sibling-entry lists
    ("(ss|ss) siblings")."""
    L = lib()
    names = class_names()
    n = int(L.cqg_schedule_lists())
    out = []
    for b in range(n):
        k = int(L.cqg_list_class(b))
        out.append(names[k] + (" siblings" if b >= n // 2 else ""))
    return out


def class_names():
    L = lib()
    out = []
    k = 0
    while True:
        s = L.cqg_class_name(k)
        if s is None:
            break
        out.append(s.decode())
        k += 1
    return out
