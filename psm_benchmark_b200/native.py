"""ctypes binding of libpsm_b200.so (the C ABI in include/psm_b200.h).

There is no fallback: if the library is missing or cannot reach an sm_100
device, calls raise PsmError.
"""
from __future__ import annotations

import ctypes as C
import os
from functools import lru_cache
from pathlib import Path

_PKG = Path(__file__).resolve().parent
# PSM_LIB selects another build of the library (A/B timing of kernel variants).
LIB_PATH = Path(os.environ["PSM_LIB"]) if os.environ.get("PSM_LIB") else _PKG / "libpsm_b200.so"

PSM_OK, PSM_ERR_ARG, PSM_ERR_OOM, PSM_ERR_TIMEOUT, PSM_ERR_CUDA, PSM_ERR_IO, PSM_ERR_INTERNAL = 0, 1, 2, 3, 4, 5, 9
FILTERS = {"NLF": 0, "GQL": 1, "CFL": 2}
ORDERS = {"GQL": 0, "CFL": 1}
ENGINES = {"LFTJ": 0, "GQL": 1, "EXPLORE": 2}

EXPORTS = [
    "psm_status_string", "psm_last_error", "psm_version",
    "psm_graph_from_csr", "psm_graph_load", "psm_graph_info", "psm_graph_free",
    "psm_context_create", "psm_context_free",
    "psm_match", "psm_run_create", "psm_run_candidates", "psm_run_table", "psm_run_order",
    "psm_run_embeddings", "psm_run_free", "psm_match_batch", "psm_run_recount_noalloc",
    "psm_context_set_batch_tuning", "psm_context_get_batch_tuning", "psm_autotune_batch",
    "psm_match_join", "psm_query_decompose", "psm_hash_join", "psm_match_join_ex", "psm_query_decompose_ex",
    "psm_server_create", "psm_server_submit", "psm_server_poll", "psm_server_pending", "psm_server_estimate",
    "psm_server_clock_ns", "psm_server_destroy", "psm_server_set_batch_tuning",
    "psm_graph_load_binary", "psm_graph_store_binary", "psm_graph_convert", "psm_graph_convert_edgelist",
    "psm_intersect_check",
]
MAX_UNITS = 32


class PsmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"psm error {code}: {msg}")
        self.code = code


class QueryDesc(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("num_edges", C.c_uint32),
                ("labels", C.POINTER(C.c_uint32)), ("edges", C.POINTER(C.c_uint32))]


class Options(C.Structure):
    _fields_ = [("filter", C.c_uint32), ("order", C.c_uint32), ("engine", C.c_uint32), ("emit", C.c_uint32),
                ("cap", C.c_uint64), ("time_limit_s", C.c_double), ("emit_capacity", C.c_uint64)]


class Result(C.Structure):
    _fields_ = [("count", C.c_uint64), ("calls", C.c_uint64), ("memory_bytes", C.c_uint64),
                ("table_entries", C.c_uint64), ("alg_bytes", C.c_uint64), ("donations", C.c_uint64),
                ("overtime", C.c_uint32), ("filter_ok", C.c_uint32), ("status", C.c_uint32),
                ("reserved", C.c_uint32), ("prep_ms", C.c_double), ("enum_ms", C.c_double),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("tasks", C.c_uint64),
                ("idle_polls", C.c_uint64), ("count_internal", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ServerConfig(C.Structure):
    _fields_ = [("lanes", C.c_uint32), ("max_batch", C.c_uint32), ("lane_arena_bytes", C.c_uint64),
                ("full_gpu_lanes", C.c_uint32), ("reserved", C.c_uint32)]


class RequestResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("count", C.c_uint64), ("status", C.c_uint32), ("overtime", C.c_uint32),
                ("submit_ns", C.c_uint64), ("start_ns", C.c_uint64), ("done_ns", C.c_uint64),
                ("batch_size", C.c_uint32), ("lane", C.c_uint32), ("prep_ms", C.c_double), ("enum_ms", C.c_double)]


TEAMS = {"RULE": 0, "BLOCK": 1, "CLUSTER": 2}
INTERSECTS = {"BINARY": 0, "AUTO": 1, "MERGE": 2}


class BatchTuning(C.Structure):
    _fields_ = [("team", C.c_uint32), ("grabs_per_warp", C.c_uint32), ("enum_quarters", C.c_uint32),
                ("intersect", C.c_uint32), ("ms", C.c_double)]

    def as_dict(self):
        team = {v: k for k, v in TEAMS.items()}[self.team]
        isect = {v: k for k, v in INTERSECTS.items()}[self.intersect]
        return {"team": team, "grabs_per_warp": self.grabs_per_warp, "enum_quarters": self.enum_quarters,
                "intersect": isect, "ms": self.ms}


SPLIT_PATTERNS = {"BOUNDED": 0, "STAR": 1, "TWINTWIG": 2, "SEED": 3, "SKETCHTREE": 4, "COST": 5}
JOIN_METHODS = {"LEFTDEEP": 0, "BUSHY": 1}


class JoinOptions(C.Structure):
    _fields_ = [("pattern", C.c_uint32), ("join_method", C.c_uint32), ("max_unit", C.c_uint32),
                ("reserved", C.c_uint32)]


class JoinResult(C.Structure):
    _fields_ = [("count", C.c_uint64), ("units", C.c_uint32), ("status", C.c_uint32),
                ("unit_mask", C.c_uint32 * MAX_UNITS), ("unit_rows", C.c_uint64 * MAX_UNITS),
                ("join_rows", C.c_uint64 * MAX_UNITS), ("prep_ms", C.c_double), ("enum_ms", C.c_double),
                ("join_ms", C.c_double), ("work_bytes", C.c_uint64), ("memory_bytes", C.c_uint64)]


@lru_cache(maxsize=1)
def lib():
    if not LIB_PATH.exists():
        raise PsmError(PSM_ERR_CUDA, f"{LIB_PATH} is not built (python -m psm_benchmark_b200.build)")
    L = C.CDLL(str(LIB_PATH))
    u32p = C.POINTER(C.c_uint32)
    vp = C.c_void_p
    sig = {
        "psm_status_string": ([C.c_int], C.c_char_p),
        "psm_last_error": ([], C.c_char_p),
        "psm_version": ([], C.c_char_p),
        "psm_graph_from_csr": ([u32p, u32p, u32p, C.c_uint32, C.POINTER(vp)], C.c_int),
        "psm_graph_load": ([C.c_char_p, C.POINTER(vp)], C.c_int),
        "psm_graph_load_binary": ([C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(vp)], C.c_int),
        "psm_graph_store_binary": ([u32p, u32p, u32p, C.c_uint32, C.c_char_p, C.c_char_p, C.c_char_p], C.c_int),
        "psm_graph_convert": ([C.c_char_p, C.c_char_p], C.c_int),
        "psm_graph_convert_edgelist": ([C.c_char_p, C.c_char_p, C.c_uint32, C.c_uint64], C.c_int),
        "psm_graph_info": ([vp, u32p, C.POINTER(C.c_uint64), u32p, u32p, u32p], C.c_int),
        "psm_graph_free": ([vp], None),
        "psm_context_create": ([C.c_int, C.c_uint64, C.POINTER(vp)], C.c_int),
        "psm_context_free": ([vp], None),
        "psm_match": ([vp, vp, C.POINTER(QueryDesc), C.POINTER(Options), C.POINTER(Result)], C.c_int),
        "psm_run_create": ([vp, vp, C.POINTER(QueryDesc), C.POINTER(Options), C.POINTER(vp), C.POINTER(Result)],
                           C.c_int),
        "psm_run_candidates": ([vp, C.c_uint32, u32p, C.c_uint32, u32p], C.c_int),
        "psm_run_table": ([vp, C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32, u32p, u32p], C.c_int),
        "psm_run_order": ([vp, u32p, u32p], C.c_int),
        "psm_run_embeddings": ([vp, u32p, C.c_uint64, C.POINTER(C.c_uint64)], C.c_int),
        "psm_run_free": ([vp], None),
        "psm_context_set_batch_tuning": ([vp, C.POINTER(BatchTuning)], C.c_int),
        "psm_context_get_batch_tuning": ([vp, C.POINTER(BatchTuning)], C.c_int),
        "psm_autotune_batch": ([vp, vp, C.POINTER(QueryDesc), C.c_uint32, C.POINTER(Options), C.c_uint32,
                                C.POINTER(BatchTuning), C.POINTER(BatchTuning), C.c_uint32, u32p], C.c_int),
        "psm_match_batch": ([vp, vp, C.POINTER(QueryDesc), C.c_uint32, C.POINTER(Options), C.POINTER(Result)],
                            C.c_int),
        "psm_run_recount_noalloc": ([vp, C.c_uint64, C.c_double, C.POINTER(C.c_uint64), u32p], C.c_int),
        "psm_match_join": ([vp, vp, C.POINTER(QueryDesc), C.POINTER(Options), C.c_uint32, C.POINTER(JoinResult)],
                           C.c_int),
        "psm_query_decompose": ([C.POINTER(QueryDesc), C.c_uint32, u32p, u32p], C.c_int),
        "psm_match_join_ex": ([vp, vp, C.POINTER(QueryDesc), C.POINTER(Options), C.POINTER(JoinOptions),
                               C.POINTER(JoinResult)], C.c_int),
        "psm_query_decompose_ex": ([C.POINTER(QueryDesc), C.POINTER(JoinOptions), C.c_double, C.c_double, u32p, u32p,
                                    u32p, u32p], C.c_int),
        "psm_server_create": ([C.c_int, vp, C.POINTER(Options), C.POINTER(ServerConfig), C.POINTER(vp)], C.c_int),
        "psm_server_submit": ([vp, C.POINTER(QueryDesc), C.POINTER(C.c_uint64)], C.c_int),
        "psm_server_poll": ([vp, C.POINTER(RequestResult), C.c_uint32, u32p, C.c_double], C.c_int),
        "psm_server_pending": ([vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
        "psm_server_estimate": ([vp, C.POINTER(QueryDesc), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
        "psm_server_clock_ns": ([], C.c_uint64),
        "psm_server_destroy": ([vp], None),
        "psm_server_set_batch_tuning": ([vp, C.POINTER(BatchTuning)], C.c_int),
        "psm_hash_join": ([vp, u32p, C.c_uint64, C.c_uint32, u32p, u32p, C.c_uint64, C.c_uint32, u32p, u32p, u32p,
                           C.c_uint64, u32p, u32p, C.POINTER(C.c_uint64)], C.c_int),
        "psm_intersect_check": ([u32p, C.c_uint32, u32p, C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


def check(rc: int, allow=()):
    if rc != PSM_OK and rc not in allow:
        raise PsmError(rc, lib().psm_last_error().decode())
    return rc


def parse_method(method: str):
    """'CFL_CFL_EXPLORE' -> (filter, order, engine) codes (-BackMethods triple,
    matching/StudyPerformance.cpp:1013-1030)."""
    parts = method.split("_")
    if len(parts) != 3:
        raise PsmError(PSM_ERR_ARG, f"method must be FILTER_ORDER_ENGINE, got {method!r}")
    f, o, e = parts
    if f not in FILTERS or o not in ORDERS or e not in ENGINES:
        raise PsmError(PSM_ERR_ARG, f"unsupported method {method!r} (filters NLF/GQL/CFL, orders GQL/CFL, "
                                    "engines GQL/EXPLORE/LFTJ)")
    return FILTERS[f], ORDERS[o], ENGINES[e]
