"""Loader and ctypes signatures of the native library libhodlr_b200.so.

The library is the product: every solve runs in its CUDA kernels.  There is no
Python or CPU fallback; if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhodlr_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "hodlr_gpu.h")

HODLR_OK = 0
ERR_CUDA = -1000
ERR_NOMEM = -1001
ERR_STATE = -1002
ERR_NOCONV = -1003
ERR_TIMEOUT = -1004
ERR_UNSUPPORTED = -1005
ERR_IO = -1006
PREC_FP64 = 0
PREC_MIXED = 1

PHASES = ["getrf", "getrs", "reduce", "node_factor", "node_apply", "broadcast", "matvec",
          "convert", "leaf_panel", "leaf_update", "leaf_trsm", "sweep_levels"]
NODE_FIELDS = ["nrow", "ncol", "row_beg", "col_beg", "lchild", "rchild", "parent", "depth",
               "vncol", "is_leaf"]


class HodlrError(RuntimeError):
    def __init__(self, fn: str, status: int, text: str):
        super().__init__(f"{fn} failed: status {status} ({text})")
        self.status = status
        self.fn = fn


if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python -m fastsolver_b200.build` "
        "(the solver has no non-CUDA implementation)")

lib = ctypes.CDLL(LIB_PATH)

_i, _d, _ll, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)

_SIGS = {
    "hodlr_leaf_solve": [_i, _i, _vp, _i, _vp, _i, _vp, _vp, _vp],
    "hodlr_gemm_reduce": [_d, _i, _i, _i, _vp, _i, _vp, _i, _i, _vp, _i, _vp],
    "hodlr_gemm_reduce_noalloc": [_d, _i, _i, _i, _vp, _i, _vp, _i, _i, _vp, _i, _vp],
    "hodlr_node_lu_solve": [_i, _i, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _vp],
    "hodlr_node_schur2_solve": [_i, _i, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _vp],
    "hodlr_gemm_broadcast": [_d, _d, _i, _i, _i, _vp, _i, _i, _vp, _i, _i, _vp],
    "hodlr_leaf_solve_batched": [_i, _vp, _i, _i, _vp, _vp],
    "hodlr_build_tree": [_i, _i, _i, _i, _ip, _i],
    "hodlr_gemm_f32": [_i, _i, _i, _i, ctypes.c_float, _vp, _i, _vp, _i, ctypes.c_float, _vp, _i,
                       _i, _vp],
    "hodlr_create": [ctypes.POINTER(_vp), _i, _i, _i, _i],
    "hodlr_destroy": [_vp],
    "hodlr_tree_info": [_vp, _ip, _ip, _ip, _ip, _ip],
    "hodlr_tree_nodes": [_vp, _ip, _i],
    "hodlr_set_matrix": [_vp, _vp, _ll, _vp, _ll, _vp, _ll, _i, _vp],
    "hodlr_set_rhs": [_vp, _vp, _ll, _i, _vp],
    "hodlr_get_matrix": [_vp, _vp, _ll, _vp, _ll, _vp, _ll, _vp, _ll, _i, _vp],
    "hodlr_init_circulant": [_vp, _d, _vp],
    "hodlr_init_rhs_drand48": [_vp, ctypes.c_long, _vp],
    "hodlr_init_gaussian": [_vp, ctypes.c_ulonglong, _d, _vp],
    "hodlr_solve_fused": [_vp, _i, _i, _vp],
    "hodlr_factor": [_vp, _i, _vp],
    "hodlr_solve": [_vp, _vp],
    "hodlr_solve_refined": [_vp, _i, _d, _i, _ip, _dp, _vp],
    "hodlr_solve_refined_host": [_vp, _vp, _ll, _vp, _ll, _vp, _ll, _vp, _ll, _vp, _ll, _i, _d,
                                 _i, _ip, _dp, _vp],
    "hodlr_matvec": [_vp, _vp, _ll, _vp, _ll, _i, _vp],
    "hodlr_relres": [_vp, _dp, _vp],
    "hodlr_get_solution": [_vp, _vp, _ll, _i, _vp],
    "hodlr_set_profiling": [_vp, _i],
    "hodlr_phase_times": [_vp, _dp, ctypes.POINTER(ctypes.c_longlong), _i],
    "hodlr_batch_create": [ctypes.POINTER(_vp), ctypes.POINTER(_vp), _i],
    "hodlr_batch_destroy": [_vp],
    "hodlr_batch_solve_refined": [_vp, _d, _i, _ip, _dp, _dp, _ip, _vp],
    "hodlr_batch_set_profiling": [_vp, _i],
    "hodlr_batch_phase_times": [_vp, _dp, ctypes.POINTER(ctypes.c_longlong), _i],
    "hodlr_get_schedule": [_vp, _vp],
    "hodlr_set_schedule": [_vp, _vp],
    "hodlr_autotune": [_vp, _i, _d, _i, _vp, _dp, _vp, _i, _ip],
    "hodlr_batch_autotune": [_vp, _d, _i, _vp, _dp, _vp, _i, _ip],
    "hodlr_launch_count": [],
    "hodlr_reset_launch_count": [],
    "hodlr_status_string": [_i],
    "hodlr_debug_tc_wait_hook": [_ll, _i],
    "hodlr_debug_sweep_barrier_hook": [_ll, _i],
    "hodlr_set_leaf_size": [_vp, _i],
    "hodlr_get_num_leaf": [_vp],
    "hodlr_legion_leaves": [_vp, _ip, _i],
    "hodlr_text_write": [ctypes.c_char_p, _vp, _ll, _i, _i, _i, ctypes.c_long, _i],
    "hodlr_text_read": [ctypes.c_char_p, _vp, _ll, _i, _i, _i, _ip,
                        ctypes.POINTER(ctypes.c_long)],
    "hodlr_save_rhs": [_vp, ctypes.c_char_p, ctypes.c_long],
    "hodlr_save_solution": [_vp, ctypes.c_char_p],
    "hodlr_load_rhs": [_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)],
}


class Schedule(ctypes.Structure):
    """hodlr_schedule (include/hodlr_gpu.h)."""
    _fields_ = [("leaf_nb", ctypes.c_int), ("leaf_ob32", ctypes.c_int),
                ("leaf_ob64", ctypes.c_int), ("reduce_rows", ctypes.c_int),
                ("bcast_rows", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}

    @classmethod
    def from_dict(cls, d: dict) -> "Schedule":
        return cls(**{k: int(d[k]) for k, _ in cls._fields_})


class TuneTrial(ctypes.Structure):
    """hodlr_tune_trial (include/hodlr_gpu.h)."""
    _fields_ = [("schedule", Schedule), ("ms", ctypes.c_double)]


for _name, _args in _SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _i
lib.hodlr_launch_count.restype = ctypes.c_longlong
lib.hodlr_reset_launch_count.restype = None
lib.hodlr_status_string.restype = ctypes.c_char_p


def status_text(status: int) -> str:
    return lib.hodlr_status_string(int(status)).decode()


def check(fn: str, status: int, ok=(0,)) -> int:
    """Raise HodlrError for a status outside `ok`."""
    if status not in ok:
        raise HodlrError(fn, status, status_text(status))
    return status


def call(fn: str, *args, ok=(0,)) -> int:
    return check(fn, getattr(lib, fn)(*args), ok)


def launch_count() -> int:
    return int(lib.hodlr_launch_count())


def reset_launch_count() -> None:
    lib.hodlr_reset_launch_count()
