"""ctypes bindings of libhl.so (the C ABI in include/hl.h and include/hl_debug.h).

The library is the only compute path: if it is missing this module raises at
import time instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhl.so")

HL_OK = 0
HL_ERR_INVALID_INPUT = 1
HL_ERR_CUDA = 2
HL_ERR_OUT_OF_MEMORY = 3
HL_ERR_TIMEOUT = 4
HL_ERR_UNSUPPORTED = 5
STATUS_NAMES = {0: "Ok", 1: "InvalidInput", 2: "Backend", 3: "OutOfMemory", 4: "Timeout",
                5: "Unsupported"}

HL_MODE_DETERMINISTIC = 0
HL_MODE_THROUGHPUT = 1
HL_MAP_COMMUNITY, HL_MAP_REFINED, HL_MAP_SUB_PREVIOUS, HL_MAP_SUB_CURRENT = 0, 1, 2, 3
HL_FLAG_KEEP_SELF_LOOPS = 1 << 0
HL_FLAG_BATCH_MODULARITY = 1 << 1
HL_FLAG_KERNEL_TIMING = 1 << 2
HL_FLAG_NO_AUTOTUNE = 1 << 3
HL_FLAG_NO_SMALL_ROUNDS = 1 << 4
HL_NOALLOC_MAX_ELEMS = 1 << 28


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_uint64), ("total_ms", C.c_double),
                ("bytes", C.c_uint64), ("items", C.c_uint64)]


class Config(C.Structure):
    _fields_ = [("resolution", C.c_double), ("mode", C.c_uint32), ("max_levels", C.c_uint32),
                ("max_rounds", C.c_uint32), ("flags", C.c_uint32), ("hbm_budget", C.c_uint64),
                ("device", C.c_int32)]


class BatchStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("levels", C.c_uint32), ("moves", C.c_uint64),
                ("candidates", C.c_uint64), ("traversed", C.c_uint64), ("splits", C.c_uint64),
                ("merges", C.c_uint64), ("changed", C.c_uint64), ("refined", C.c_uint64),
                ("edges", C.c_uint64), ("modularity", C.c_double), ("device_ms", C.c_double),
                ("launches", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RequestDone(C.Structure):
    """hl_request_done: completion record of one served request."""
    _fields_ = [("request_id", C.c_uint64), ("batch_id", C.c_uint64), ("batch_seq", C.c_uint64),
                ("edges", C.c_uint64), ("batch_edges", C.c_uint64), ("changed", C.c_uint64),
                ("modularity", C.c_double), ("queue_ms", C.c_double), ("service_ms", C.c_double),
                ("latency_ms", C.c_double), ("graph", C.c_uint32), ("batch_requests", C.c_uint32),
                ("status", C.c_int32), ("pad_", C.c_uint32), ("level0_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


# hl_level_fn / hl_server_level_fn (per-level output callbacks)
LEVEL_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_uint64, C.POINTER(C.c_uint32),
                       C.POINTER(C.c_uint32))
SERVER_LEVEL_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint64,
                              C.POINTER(C.c_uint32), C.POINTER(C.c_uint32))


class HitLeidenError(RuntimeError):
    """Error raised by the library; ``kind`` mirrors HitLeidenError's variants
    (src/core/error.rs:19-27) plus the device-side statuses."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.kind = STATUS_NAMES.get(status, "Backend")
        super().__init__(f"{self.kind}: {message}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with hit-leiden_b200/build.py "
                          "(the CUDA library is the only compute path)")
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    st = C.c_int
    p32 = C.POINTER(C.c_uint32)
    sig = {
        "hl_config_default": (st, [C.POINTER(Config)]),
        "hl_create": (st, [C.POINTER(Config), C.c_uint32, vp, vp, vp, C.c_uint64, C.POINTER(vp)]),
        "hl_create_device": (st, [C.POINTER(Config), C.c_uint32, vp, vp, vp, C.c_uint64,
                                  C.POINTER(vp)]),
        "hl_apply_batch": (st, [vp, vp, vp, vp, C.c_uint64, C.POINTER(BatchStats)]),
        "hl_apply_batch_device": (st, [vp, vp, vp, vp, C.c_uint64, C.POINTER(BatchStats)]),
        "hl_set_resolution": (st, [vp, C.c_double]),
        "hl_set_mode": (st, [vp, C.c_uint32]),
        "hl_kernel_stats": (st, [vp, vp, C.c_uint32, p32]),
        "hl_reset_kernel_stats": (st, [vp]),
        "hl_num_nodes": (st, [vp, p32]),
        "hl_num_levels": (st, [vp, p32]),
        "hl_level_size": (st, [vp, C.c_uint32, p32]),
        "hl_num_edges": (st, [vp, C.c_uint32, C.POINTER(C.c_uint64)]),
        "hl_get_partition": (st, [vp, vp]),
        "hl_get_map": (st, [vp, C.c_uint32, C.c_uint32, vp]),
        "hl_get_csr": (st, [vp, C.c_uint32, vp, vp, vp]),
        "hl_modularity": (st, [vp, C.POINTER(C.c_double)]),
        "hl_modularity_of": (st, [vp, vp, C.POINTER(C.c_double)]),
        "hl_canonicalize": (st, [C.c_int32, vp, C.c_uint64]),
        "hl_destroy": (None, [vp]),
        "hl_device_bytes": (st, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "hl_apply_batches": (st, [vp, vp, vp, vp, vp, C.c_uint32, C.c_uint32, vp,
                                  C.POINTER(BatchStats)]),
        "hl_server_create": (st, [C.c_uint32, C.c_uint64, C.POINTER(vp)]),
        "hl_server_add_graph": (st, [vp, vp, p32]),
        "hl_server_set_edge_estimate": (st, [vp, C.c_uint64]),
        "hl_server_set_coalescing": (st, [vp, C.c_uint32]),
        "hl_server_submit": (st, [vp, C.c_uint32, vp, vp, vp, C.c_uint64,
                                  C.POINTER(C.c_uint64)]),
        "hl_server_poll": (st, [vp, C.POINTER(RequestDone), C.c_uint32, p32, C.c_int32]),
        "hl_server_drain": (st, [vp]),
        "hl_server_set_level_callback": (st, [vp, SERVER_LEVEL_FN, vp]),
        "hl_set_level_callback": (st, [vp, LEVEL_FN, vp]),
        "hl_server_destroy": (None, [vp]),
        "hl_last_error": (C.c_char_p, []),
        "hl_version": (C.c_char_p, []),
        "hl_dbg_move_eval": (st, [C.c_int32, C.c_uint32, vp, vp, vp, vp, vp, C.c_uint64, vp,
                                  C.c_double, C.c_double, vp, C.c_uint64, vp, vp]),
        "hl_dbg_select_decoupled": (st, [C.c_int32, vp, vp, vp, vp, C.c_uint64, vp,
                                         C.POINTER(C.c_uint64)]),
        "hl_dbg_apply_delta": (st, [C.c_int32, C.c_uint32, vp, vp, vp, C.c_uint32, vp, vp, vp,
                                    C.c_uint64, C.c_int32, vp, vp, vp, C.c_uint64,
                                    C.POINTER(C.c_uint64)]),
        "hl_dbg_inc_movement": (st, [C.c_int32, C.c_uint32, vp, vp, vp, vp, vp, vp, C.c_uint64,
                                     vp, vp, C.c_double, C.c_uint32, C.c_int32, vp, vp, p32]),
        "hl_dbg_inc_refinement": (st, [C.c_int32, C.c_uint32, vp, vp, vp, vp, vp, vp, C.c_double,
                                       C.c_int32, vp]),
        "hl_dbg_inc_aggregation": (st, [C.c_int32, C.c_uint32, vp, vp, vp, vp, vp, vp,
                                        C.c_uint64, vp, vp, vp, C.c_int32, C.c_int32, vp, p32, vp,
                                        vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]),
        "hl_dbg_tree_sum": (st, [C.c_int32, vp, C.c_uint64, C.POINTER(C.c_double)]),
        "hl_dbg_seq_sums": (st, [C.c_int32, C.c_uint32, vp, vp, C.c_double, C.c_int32, vp]),
        "hl_dbg_set_exact_tfilter": (st, [C.c_int32]),
        "hl_dbg_set_mode": (st, [C.c_uint32]),
        "hl_dbg_set_bucket_slots": (st, [C.c_uint32]),
        "hl_dbg_set_hub_defer": (st, [C.c_uint32]),
        "hl_dbg_set_pb_round": (st, [C.c_uint64]),
        "hl_dbg_set_bins": (st, [C.c_uint32, C.c_uint32]),
        "hl_autotune_info": (st, [vp, p32, p32, p32, p32]),
        "hl_tree_sum_noalloc": (st, [vp, C.c_uint64, vp, vp]),
        "hl_dbg_modularity": (st, [C.c_int32, C.c_uint32, vp, vp, vp, vp,
                                   C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != HL_OK:
        msg = lib.hl_last_error().decode(errors="replace")
        raise HitLeidenError(status, msg)


def ptr(a) -> C.c_void_p:
    """Host pointer of a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    return C.c_void_p(a.ctypes.data)


def u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)
