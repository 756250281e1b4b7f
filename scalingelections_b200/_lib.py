"""ctypes binding of libse.so, the C ABI declared in include/se.h.

The library must have been built (``python -m scalingelections_b200.build`` or
``__graft_entry__.build()``); there is deliberately no fallback: importing a compute entry
point without the CUDA library raises.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libse.so"

SE_OK = 0
SE_ERR_INVALID = 1
SE_ERR_CUDA = 2
SE_ERR_UNSUPPORTED = 3
SE_ERR_DEVICE = 4
SE_ERR_OVERFLOW = 5
SE_ERR_WORKSPACE = 6
SE_ERR_HOST = 7

LANES_AUTO = 0
LANES_U16 = 16
LANES_U32 = 32

_c_i64 = ctypes.c_int64
_c_int = ctypes.c_int
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

# name -> (restype, argtypes); every symbol include/se.h declares.
SIGNATURES: dict[str, tuple] = {
    "se_last_error": (ctypes.c_char_p, []),
    "se_version": (_c_int, []),
    "se_device_count": (_c_int, [_ip]),
    "se_device_info": (_c_int, [_c_int, ctypes.c_char_p, _c_int, _ip, _dp, _ip, _ip]),
    "se_closure_workspace_bytes": (_c_i64, [_c_int, _c_int, _c_int]),
    "se_closure": (_c_int, [_vp, _c_i64, _c_int, _vp, _c_i64, _c_int, _c_int, _vp, _c_i64, _vp]),
    "se_closure_profiled": (_c_int, [_vp, _c_i64, _c_int, _vp, _c_i64, _c_int, _c_int, _vp, _c_i64, _vp, _dp, _ip]),
    "se_closure_enqueue": (_c_int, [_vp, _c_i64, _c_int, _vp, _c_i64, _c_int, ctypes.c_uint32, _vp, _c_i64, _vp]),
    "se_closure_check": (_c_int, [_vp, _vp]),
    "se_closure_launch_count": (_c_int, [_c_int]),
    "se_closure_workspace_bytes_flow": (_c_i64, [_c_int, _c_int, _c_int]),
    "se_closure_set_mode": (_c_int, [_c_int]),
    "se_closure_set_variant_table": (_c_int, [_vp, _vp, _c_int]),
    "se_closure_schedule": (_c_int, [_c_int, _c_int, _c_i64]),
    "se_closure_flow_task": (_c_int, [ctypes.c_uint32, _c_int, _ip, _ip, _ip, _ip]),
    "se_closure_noalloc": (_c_int, [_vp, _c_i64, _c_int, _vp, _c_i64, _c_int, _vp]),
    "se_batch_workspace_bytes": (_c_i64, [_c_int, _vp]),
    "se_batch_prepare": (_c_int, [_c_int, _vp, _vp, _c_i64, _c_int, _c_int, _vp]),
    "se_batch_run": (_c_int, [_vp, _vp]),
    "se_batch_graph_build": (_c_int, [_vp]),
    "se_batch_graph_launch": (_c_int, [_vp, _vp]),
    "se_batch_release": (_c_int, [_vp]),
    "se_batch_check": (_c_int, [_vp, _vp]),
    "se_batch_set_wait_limit": (_c_int, [_vp, ctypes.c_uint64]),
    "se_batch_task_count": (_c_i64, [_vp, _c_int]),
    "se_batch_profile": (_c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_int64), _dp, _vp]),
    "se_engine_workspace_bytes": (_c_i64, [_c_int]),
    "se_engine_create": (_c_int, [_vp, _c_i64, _c_int, _c_int, _c_int, _vp]),
    "se_engine_request_scratch_bytes": (_c_i64, [_c_i64, _c_int]),
    "se_engine_request_positions_bytes": (_c_i64, [_c_i64, _c_int]),
    "se_engine_poll_tallied": (_c_int, [_vp, _ip, _c_int, _ip]),
    "se_engine_submit": (_c_int, [_vp, _vp, _vp, _ip, ctypes.POINTER(ctypes.c_uint32)]),
    "se_engine_poll": (_c_int, [_vp, _ip, ctypes.POINTER(ctypes.c_uint32), _c_int, _ip]),
    "se_engine_stats": (_c_int, [_vp, ctypes.POINTER(ctypes.c_int64), _ip, _ip, _dp, ctypes.POINTER(ctypes.c_int64), _dp]),
    "se_engine_stop": (_c_int, [_vp]),
    "se_engine_destroy": (_c_int, [_vp]),
    "se_shard_workspace_bytes": (_c_i64, [_c_int, _c_int, _c_int, _c_int]),
    "se_shard_create": (_c_int, [_c_int, _c_int, _c_int, _c_int, ctypes.c_uint32, _vp, _c_i64, _vp]),
    "se_shard_destroy": (_c_int, [_vp]),
    "se_shard_init": (_c_int, [_vp, _vp, _c_i64, _vp]),
    "se_shard_pivot": (_c_int, [_vp, _c_int, _vp]),
    "se_shard_panel_offset": (_c_i64, [_vp, _c_int]),
    "se_shard_panel_bytes": (_c_i64, [_vp]),
    "se_shard_update": (_c_int, [_vp, _c_int, _vp]),
    "se_shard_update_part": (_c_int, [_vp, _c_int, _c_int, _vp]),
    "se_shard_finalize": (_c_int, [_vp, _vp, _c_i64, _vp]),
    "se_shard_check": (_c_int, [_vp, _vp]),
    "se_tally_workspace_bytes": (_c_i64, [_c_i64, _c_int]),
    "se_tally": (_c_int, [_vp, _vp, _c_i64, _c_int, _vp, _c_i64, _vp, _c_i64, _vp]),
    "se_tally_enqueue": (_c_int, [_vp, _vp, _c_i64, _c_int, _vp, _c_i64, _vp, _c_i64, _vp]),
    "se_random_preferences": (_c_int, [_c_int, ctypes.c_uint32, ctypes.c_uint64, _vp, _c_i64, _vp]),
    "se_tally_ex": (_c_int, [_vp, _c_int, _vp, _c_i64, _c_i64, _c_int, ctypes.c_uint, _vp, _c_i64, _vp, _c_i64, _vp]),
    "se_rank": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp]),
    "se_mallows_workspace_bytes": (_c_i64, [_c_i64, _c_int]),
    "se_mallows_ballots": (_c_int, [_c_i64, _c_int, ctypes.c_double, ctypes.c_uint64, _vp, _vp, _vp, _c_i64, _vp]),
    "se_minmax_peak": (_c_int, [_c_int, _c_int, _dp, _dp, _dp, _dp]),
}

class Election(ctypes.Structure):
    """se_election_t"""
    _fields_ = [("d_pref", ctypes.c_void_p), ("ld_pref", ctypes.c_int64), ("d_out", ctypes.c_void_p),
                ("ld_out", ctypes.c_int64), ("d_wins", ctypes.c_void_p), ("d_ranking", ctypes.c_void_p),
                ("C", ctypes.c_int32), ("lane_bits", ctypes.c_int32), ("value_offset", ctypes.c_uint32),
                ("micro_tile", ctypes.c_int32)]


class Request(ctypes.Structure):
    """se_request_t"""
    _fields_ = [("d_ids", ctypes.c_void_p), ("d_offsets", ctypes.c_void_p), ("V", ctypes.c_int64),
                ("C", ctypes.c_int32), ("value_offset", ctypes.c_uint32), ("d_prefs", ctypes.c_void_p),
                ("d_out", ctypes.c_void_p), ("d_wins", ctypes.c_void_p), ("d_ranking", ctypes.c_void_p),
                ("d_scratch", ctypes.c_void_p), ("scratch_bytes", ctypes.c_int64),
                ("d_positions", ctypes.c_void_p), ("positions_bytes", ctypes.c_int64)]


class BatchPlan(ctypes.Structure):
    """se_batch_plan_t (opaque)"""
    _fields_ = [("opaque", ctypes.c_int64 * 40)]


_lib: ctypes.CDLL | None = None
_lock = threading.Lock()


class SchulzeError(RuntimeError):
    """A failed libse call. Subclasses RuntimeError, which is what the reference's native
    module raises for every failure (scaling_elections.cu:868-931)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not LIB_PATH.exists():
                    raise ImportError(
                        f"{LIB_PATH} is missing: build the CUDA library first "
                        "(python -m scalingelections_b200.build)")
                L = ctypes.CDLL(str(LIB_PATH))
                for name, (res, args) in SIGNATURES.items():
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def last_error() -> str:
    msg = lib().se_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    if status != SE_OK:
        raise SchulzeError(status, last_error() or f"libse error {status}")
