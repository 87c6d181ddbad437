"""ctypes bindings of include/gmapf_c.h (the library's C ABI).

The shared library is built in-tree (gmapf_b200/libgmapf_b200.so).  When it
is missing it is built on first import if nvcc is available; there is no
other implementation to fall back to.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgmapf_b200.so"


class Config(C.Structure):
    """include/gmapf/Config.h:5-18, same layout."""
    _fields_ = [
        ("AgentsMaxCount", C.c_int32),
        ("AgentRadius", C.c_float),
        ("AgentSpeed", C.c_float),
        ("PathFinderParallelAgents", C.c_int32),
        ("PathFinderThreadsPerAgents", C.c_int32),
        ("PathFinderQueueCapacity", C.c_int32),
        ("PathFinderHeuristicK", C.c_float),
        ("IsDebug", C.c_uint8),
        ("IsProfiler", C.c_uint8),
    ]


class V2(C.Structure):
    _fields_ = [("X", C.c_float), ("Y", C.c_float)]


class Node(C.Structure):
    """include/gmapf/misc/CuNodesMap.h:14-21 (48 bytes)."""
    _fields_ = [
        ("P1", V2), ("P2", V2), ("P3", V2), ("PCenter", V2),
        ("NeibsIdx", C.c_int32 * 3), ("_pad", C.c_int32),
    ]


class Options(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("mode", C.c_int32),
        ("block_threads", C.c_int32),
        ("autotune", C.c_int32),
        ("search_mem_budget", C.c_int64),
        ("order_by_estimate", C.c_int32),
        ("visited_mode", C.c_int32),
        ("path_smoothing", C.c_int32),
        ("round_limit", C.c_int32),
        ("promote_rounds", C.c_int32),
        ("_reserved", C.c_int32 * 1),
    ]


class ServeStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64), ("found", C.c_int64),
        ("applied", C.c_int64), ("superseded", C.c_int64), ("waiting", C.c_int64), ("in_flight", C.c_int64),
        ("launches", C.c_int64), ("latency_samples", C.c_int64), ("capacity", C.c_int32), ("slots", C.c_int32),
        ("latency_p50_ms", C.c_float), ("latency_p99_ms", C.c_float), ("latency_mean_ms", C.c_float),
        ("latency_max_ms", C.c_float),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StepStats(C.Structure):
    _fields_ = [
        ("requests", C.c_int64), ("found", C.c_int64), ("expansions", C.c_int64),
        ("rounds", C.c_int64), ("deg_sum", C.c_int64), ("claims", C.c_int64),
        ("path_nodes", C.c_int64), ("moving", C.c_int64),
        ("ms_step_wall", C.c_float), ("ms_search", C.c_float), ("ms_mover", C.c_float),
        ("ms_total_device", C.c_float), ("neighbours", C.c_int64), ("promoted", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


MODE_BATCHED = 0
MODE_PLAIN = 1
STATUS_NAMES = {
    0: "GMAPF_OK", 1: "GMAPF_E_STATE", 2: "GMAPF_E_INVALID_POS", 3: "GMAPF_E_CUDA",
    4: "GMAPF_E_CAPACITY", 5: "GMAPF_E_DEVICE_TIMEOUT", 6: "GMAPF_E_INVALID_ARG",
    7: "GMAPF_E_UNSUPPORTED", 8: "GMAPF_E_DEVICE",
}

P = C.c_void_p
I32P = C.POINTER(C.c_int32)
V2P = C.POINTER(V2)

# name -> (restype, argtypes); the complete list of exported entry points
SIGNATURES = {
    "gmapf_create": (C.c_int, [C.POINTER(P)]),
    "gmapf_destroy": (C.c_int, [P]),
    "gmapf_last_error": (C.c_char_p, []),
    "gmapf_init": (C.c_int, [P, C.POINTER(Config)]),
    "gmapf_set_options": (C.c_int, [P, C.POINTER(Options)]),
    "gmapf_get_options": (C.c_int, [P, C.POINTER(Options)]),
    "gmapf_fill_map_start": (C.c_int, [P, C.c_float, C.c_float]),
    "gmapf_fill_map_obstacle": (C.c_int, [P, V2P, C.c_int32]),
    "gmapf_fill_map_end": (C.c_int, [P]),
    "gmapf_fill_map_manually": (C.c_int, [P, C.POINTER(Node), C.c_int32]),
    "gmapf_add_agent": (C.c_int, [P, C.c_float, C.c_float, I32P]),
    "gmapf_set_agent_targ_pos": (C.c_int, [P, C.c_int32, C.c_float, C.c_float]),
    "gmapf_set_agent_targ_pos_bulk": (C.c_int, [P, I32P, V2P, C.c_int32]),
    "gmapf_set_agent_targ_pos_device": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_int32]),
    "gmapf_manual_start": (C.c_int, [P]),
    "gmapf_async_step": (C.c_int, [P, C.c_float]),
    "gmapf_wait_step_end": (C.c_int, [P]),
    "gmapf_get_agent_pos": (C.c_int, [P, C.c_int32, V2P]),
    "gmapf_get_agent_state": (C.c_int, [P, C.c_int32, I32P]),
    "gmapf_agent_pos_view": (V2P, [P]),
    "gmapf_get_agents": (C.c_int, [P, V2P, I32P, C.c_int32]),
    "gmapf_agent_count": (C.c_int32, [P]),
    "gmapf_profiler_dump": (C.c_int, [P]),
    "gmapf_map_count": (C.c_int32, [P]),
    "gmapf_get_map_nodes": (C.c_int, [P, C.POINTER(Node), C.c_int32]),
    "gmapf_locate_points": (C.c_int, [P, V2P, C.c_int32, I32P]),
    "gmapf_debug_get_agents": (C.c_int, [P, V2P, I32P, I32P, I32P, I32P, I32P, V2P, I32P]),
    "gmapf_debug_get_path": (C.c_int, [P, C.c_int32, I32P, C.c_int32, I32P]),
    "gmapf_last_step_stats": (C.c_int, [P, C.POINTER(StepStats)]),
    "gmapf_step_time_percentile": (C.c_int, [P, C.c_float, C.POINTER(C.c_float)]),
    "gmapf_reset_profiler": (C.c_int, [P]),
    "gmapf_kernel_launches": (C.c_int64, [P]),
    "gmapf_search_shape": (C.c_int, [P, I32P, I32P, I32P, I32P, I32P]),
    "gmapf_set_tune_cache": (C.c_int, [P, C.c_char_p]),
    "gmapf_tune_source": (C.c_int, [P, I32P]),
    "gmapf_set_search_timeline": (C.c_int, [P, C.c_void_p, C.c_int32]),
    "gmapf_stream_handle": (C.c_void_p, [P]),
    "gmapf_search_batch_host": (C.c_int, [P, I32P, I32P, C.c_int32, I32P, I32P, I32P, C.c_int32,
                                          C.POINTER(StepStats)]),
    "gmapf_search_batch_device": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(StepStats)]),
    "gmapf_last_search_ms": (C.c_int, [P, C.POINTER(C.c_float)]),
    "gmapf_map_save": (C.c_int, [P, C.c_char_p]),
    "gmapf_map_load": (C.c_int, [P, C.c_char_p]),
    "gmapf_fill_map_end_cached": (C.c_int, [P, C.c_char_p, I32P]),
    "gmapf_step_ready": (C.c_int32, [P]),
    "gmapf_serve_start": (C.c_int, [P, C.c_int32]),
    "gmapf_serve_submit": (C.c_int, [P, I32P, V2P, C.c_int32, C.POINTER(C.c_int64)]),
    "gmapf_serve_poll": (C.c_int, [P]),
    "gmapf_serve_drain": (C.c_int, [P, C.c_float]),
    "gmapf_serve_get_stats": (C.c_int, [P, C.POINTER(ServeStats), C.c_int32]),
    "gmapf_serve_result": (C.c_int, [P, C.c_int32, I32P, I32P, I32P, C.c_int32]),
    "gmapf_serve_stop": (C.c_int, [P]),
    "gmapf_clock_ns": (C.c_int64, []),
    "gmapf_batch_create": (C.c_int, [C.POINTER(P), C.c_int32, C.POINTER(Options), C.POINTER(P)]),
    "gmapf_batch_destroy": (C.c_int, [P]),
    "gmapf_batch_world": (P, [P]),
    "gmapf_batch_scene_base": (C.c_int, [P, C.c_int32, I32P, I32P]),
    "gmapf_search_batch_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                             C.c_int32, C.c_float, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_int32, C.c_void_p]),
}

_lib = None


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load the in-tree library (building it first when possible)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and os.environ.get("GMAPF_NO_BUILD") != "1":
        try:
            from . import build as _build
            # a library built with the navmesh builder (CDT headers) is not
            # replaced by one built without them on a machine that lacks them
            if _build.needs_build(LIB_PATH, _build._sources()) and os.path.exists(_build.NVCC) and \
                    (_build.cdt_dir() or not LIB_PATH.exists()):
                _build.build_library()
        except Exception:
            if not LIB_PATH.exists():
                raise
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with python gmapf_b200/build.py")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
