"""Python mirror of the reference's gmapf::GMAPF (include/gmapf/GMAPF.h:30-98)
over the library's C ABI, plus numpy helpers for bulk access.

Method names, argument meaning and the lifecycle rules follow the
reference (src/GMAPF.cu); its `throw std::exception(msg)` becomes
GMAPFError (a RuntimeError) carrying the C status code.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum

import numpy as np

from . import _lib
from ._lib import Config, Node, Options, StepStats, V2, MODE_BATCHED, MODE_PLAIN


class EAgentState(IntEnum):
    """include/gmapf/Agent.h:7-12"""
    Idle = 0
    Search = 1
    Move = 2


class GMAPFError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = _lib.STATUS_NAMES.get(status, str(status))
        super().__init__(f"[gmapf] {self.status_name}: {message}")


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a: np.ndarray, t=C.c_int32):
    return a.ctypes.data_as(C.POINTER(t))


NODE_DTYPE = np.dtype([("P1", "<f4", 2), ("P2", "<f4", 2), ("P3", "<f4", 2), ("PCenter", "<f4", 2),
                       ("NeibsIdx", "<i4", 3), ("_pad", "<i4")])
assert NODE_DTYPE.itemsize == C.sizeof(Node) == 48


def make_config(agents_max: int, radius: float, speed: float, parallel_agents: int, threads_per_agent: int,
                queue_capacity: int, heuristic_k: float = 1.0, is_debug: bool = False,
                is_profiler: bool = False) -> Config:
    c = Config()
    c.AgentsMaxCount = agents_max
    c.AgentRadius = radius
    c.AgentSpeed = speed
    c.PathFinderParallelAgents = parallel_agents
    c.PathFinderThreadsPerAgents = threads_per_agent
    c.PathFinderQueueCapacity = queue_capacity
    c.PathFinderHeuristicK = heuristic_k
    c.IsDebug = 1 if is_debug else 0
    c.IsProfiler = 1 if is_profiler else 0
    return c


def make_options(mode: int = MODE_BATCHED, device: int = 0, block_threads: int = 0, autotune: bool = False,
                 search_mem_budget: int = 0, order_by_estimate: bool = True, visited_mode: int = 0,
                 path_smoothing: int = 0, round_limit: int = 0, promote_rounds: int = 0) -> Options:
    """path_smoothing: 0 / False off, 1 / True funnel corners, 2 corners one
    agent radius off the walls."""
    o = Options()
    o.round_limit = round_limit
    o.promote_rounds = promote_rounds
    o.path_smoothing = int(path_smoothing)
    o.device = device
    o.mode = mode
    o.block_threads = block_threads
    o.autotune = 1 if autotune else 0
    o.search_mem_budget = search_mem_budget
    o.order_by_estimate = 1 if order_by_estimate else 0
    o.visited_mode = visited_mode
    return o


class GMAPF:
    """gmapf::GMAPF with the same lifecycle: Init -> FillMap* -> AddAgent ->
    (SetAgentTargPos) -> [ManualStart] -> AsyncStep/WaitStepEnd ..."""

    def __init__(self):
        self._lib = _lib.load()
        h = C.c_void_p()
        self._check(self._lib.gmapf_create(C.byref(h)))
        self._h = h
        self._owned = True

    @classmethod
    def _view(cls, handle) -> "GMAPF":
        """A non-owning wrapper (a scene batch's world)."""
        g = cls.__new__(cls)
        g._lib = _lib.load()
        g._h = C.c_void_p(handle)
        g._owned = False
        return g

    # -- plumbing --------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = self._lib.gmapf_last_error()
            raise GMAPFError(rc, msg.decode() if msg else "")

    def close(self) -> None:
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                self._lib.gmapf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- reference API (GMAPF.h:39-57) -------------------------------------
    def Init(self, config: Config) -> None:
        self._check(self._lib.gmapf_init(self._h, C.byref(config)))

    def ManualStart(self) -> None:
        self._check(self._lib.gmapf_manual_start(self._h))

    def AddAgent(self, pos) -> int:
        out = C.c_int32()
        self._check(self._lib.gmapf_add_agent(self._h, float(pos[0]), float(pos[1]), C.byref(out)))
        return out.value

    def SetAgentTargPos(self, agent_id: int, pos) -> None:
        self._check(self._lib.gmapf_set_agent_targ_pos(self._h, int(agent_id), float(pos[0]), float(pos[1])))

    SetAgentTargetPos = SetAgentTargPos  # README.md:78 spelling

    def FillMapStart(self, size) -> None:
        self._check(self._lib.gmapf_fill_map_start(self._h, float(size[0]), float(size[1])))

    def FillMapObstacle(self, vertices) -> None:
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 2)
        self._check(self._lib.gmapf_fill_map_obstacle(self._h, v.ctypes.data_as(C.POINTER(V2)), len(v)))

    def FillMapEnd(self) -> None:
        self._check(self._lib.gmapf_fill_map_end(self._h))

    def FillMapManually(self, nodes: np.ndarray) -> None:
        arr = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
        self._check(self._lib.gmapf_fill_map_manually(self._h, arr.ctypes.data_as(C.POINTER(Node)), len(arr)))

    # -- navmesh files -----------------------------------------------------
    def map_save(self, path) -> None:
        self._check(self._lib.gmapf_map_save(self._h, str(path).encode()))

    def map_load(self, path) -> None:
        self._check(self._lib.gmapf_map_load(self._h, str(path).encode()))

    def FillMapEndCached(self, path) -> bool:
        """FillMapEnd through a cache file; True when the cached navmesh was used."""
        hit = C.c_int32()
        self._check(self._lib.gmapf_fill_map_end_cached(self._h, str(path).encode(), C.byref(hit)))
        return bool(hit.value)

    def AsyncStep(self, delta_time: float) -> None:
        self._check(self._lib.gmapf_async_step(self._h, float(delta_time)))

    def step_ready(self) -> bool:
        """True when no step runs or its device work is done (WaitStepEnd will not block)."""
        return bool(self._lib.gmapf_step_ready(self._h))

    def WaitStepEnd(self) -> None:
        self._check(self._lib.gmapf_wait_step_end(self._h))

    def GetAgentPos(self, agent_id: int):
        v = V2()
        self._check(self._lib.gmapf_get_agent_pos(self._h, int(agent_id), C.byref(v)))
        return (v.X, v.Y)

    def GetAgentState(self, agent_id: int) -> EAgentState:
        s = C.c_int32()
        self._check(self._lib.gmapf_get_agent_state(self._h, int(agent_id), C.byref(s)))
        return EAgentState(s.value)

    def ProfilerDump(self) -> None:
        self._check(self._lib.gmapf_profiler_dump(self._h))

    # -- extras ------------------------------------------------------------
    def set_options(self, **kw) -> None:
        """mode, device, block_threads, autotune, search_mem_budget,
        order_by_estimate, visited_mode, path_smoothing, round_limit,
        promote_rounds (see gmapf_options)."""
        o = make_options(**kw)
        self._check(self._lib.gmapf_set_options(self._h, C.byref(o)))

    def options(self) -> dict:
        o = Options()
        self._check(self._lib.gmapf_get_options(self._h, C.byref(o)))
        return {k: getattr(o, k) for k, _ in o._fields_ if k != "_reserved"}

    @property
    def agent_count(self) -> int:
        return self._lib.gmapf_agent_count(self._h)

    @property
    def node_count(self) -> int:
        return self._lib.gmapf_map_count(self._h)

    def map_nodes(self) -> np.ndarray:
        n = self.node_count
        out = np.zeros(n, dtype=NODE_DTYPE)
        self._check(self._lib.gmapf_get_map_nodes(self._h, out.ctypes.data_as(C.POINTER(Node)), n))
        return out

    def locate(self, pts) -> np.ndarray:
        p = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 2)
        out = np.empty(len(p), dtype=np.int32)
        self._check(self._lib.gmapf_locate_points(self._h, p.ctypes.data_as(C.POINTER(V2)), len(p), _ptr(out)))
        return out

    def set_targets(self, ids, pos) -> None:
        ids = _i32(ids)
        p = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 2)
        self._check(self._lib.gmapf_set_agent_targ_pos_bulk(self._h, _ptr(ids), p.ctypes.data_as(C.POINTER(V2)),
                                                             len(ids)))

    # -- serving (gmapf_serve_*) ---------------------------------------------
    def serve_start(self, max_in_flight: int = 0) -> None:
        self._check(self._lib.gmapf_serve_start(self._h, int(max_in_flight)))

    def serve_submit(self, ids, pos, arrival_ns=None) -> None:
        ids = _i32(ids)
        p = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 2)
        arr = None
        if arrival_ns is not None:
            arr = np.ascontiguousarray(arrival_ns, dtype=np.int64)
            arr = arr.ctypes.data_as(C.POINTER(C.c_int64))
        self._check(self._lib.gmapf_serve_submit(self._h, _ptr(ids), p.ctypes.data_as(C.POINTER(V2)), len(ids), arr))

    def serve_poll(self) -> None:
        self._check(self._lib.gmapf_serve_poll(self._h))

    def serve_drain(self, timeout_s: float = 60.0) -> None:
        self._check(self._lib.gmapf_serve_drain(self._h, float(timeout_s)))

    def serve_stats(self, reset: bool = False) -> dict:
        st = _lib.ServeStats()
        self._check(self._lib.gmapf_serve_get_stats(self._h, C.byref(st), 1 if reset else 0))
        return st.as_dict()

    def serve_result(self, agent: int):
        """(found, length, path) of the agent's finished query not yet installed by a frame."""
        f, L = C.c_int32(), C.c_int32()
        out = np.empty(max(1, self.node_count), np.int32)
        self._check(self._lib.gmapf_serve_result(self._h, int(agent), C.byref(f), C.byref(L), _ptr(out), len(out)))
        return f.value, L.value, out[:max(0, min(L.value, len(out)))].copy()

    def serve_stop(self) -> None:
        self._check(self._lib.gmapf_serve_stop(self._h))

    def set_targets_device(self, d_ids: int, d_pos: int, n: int) -> None:
        """Retarget n agents from device-resident ids (int32) and positions
        (float32 pairs); raw device addresses, enqueued before the next step."""
        self._check(self._lib.gmapf_set_agent_targ_pos_device(self._h, d_ids, d_pos, int(n)))

    def agents(self):
        n = self.agent_count
        pos = np.empty((n, 2), dtype=np.float32)
        st = np.empty(n, dtype=np.int32)
        self._check(self._lib.gmapf_get_agents(self._h, pos.ctypes.data_as(C.POINTER(V2)), _ptr(st), n))
        return pos, st

    def debug_agents(self) -> dict:
        n = self.agent_count
        d = {
            "pos": np.empty((n, 2), np.float32), "state": np.empty(n, np.int32), "cur_node": np.empty(n, np.int32),
            "targ_node": np.empty(n, np.int32), "step_idx": np.empty(n, np.int32),
            "step_node": np.empty(n, np.int32), "step_pos": np.empty((n, 2), np.float32),
            "path_len": np.empty(n, np.int32),
        }
        v2 = lambda a: a.ctypes.data_as(C.POINTER(V2))
        self._check(self._lib.gmapf_debug_get_agents(
            self._h, v2(d["pos"]), _ptr(d["state"]), _ptr(d["cur_node"]), _ptr(d["targ_node"]),
            _ptr(d["step_idx"]), _ptr(d["step_node"]), v2(d["step_pos"]), _ptr(d["path_len"])))
        return d

    def path(self, agent_id: int, cap: int | None = None) -> np.ndarray:
        cap = cap if cap is not None else max(1, self.node_count)
        out = np.empty(cap, dtype=np.int32)
        L = C.c_int32()
        self._check(self._lib.gmapf_debug_get_path(self._h, int(agent_id), _ptr(out), cap, C.byref(L)))
        return out[:min(L.value, cap)].copy()

    def last_stats(self) -> dict:
        s = StepStats()
        self._check(self._lib.gmapf_last_step_stats(self._h, C.byref(s)))
        return s.as_dict()

    def step_percentile(self, q: float) -> float:
        v = C.c_float()
        self._check(self._lib.gmapf_step_time_percentile(self._h, float(q), C.byref(v)))
        return v.value

    def reset_profiler(self) -> None:
        self._check(self._lib.gmapf_reset_profiler(self._h))

    @property
    def kernel_launches(self) -> int:
        return self._lib.gmapf_kernel_launches(self._h)

    @property
    def stream_handle(self) -> int:
        """cudaStream_t of the library (0 before the start)."""
        return self._lib.gmapf_stream_handle(self._h) or 0

    def set_tune_cache(self, path) -> None:
        """Autotuner cache file (before the start); None turns it off."""
        self._check(self._lib.gmapf_set_tune_cache(self._h, None if path is None else str(path).encode()))

    def set_search_timeline(self, d_timeline: int, rows: int) -> None:
        """Device buffer (raw address) of 2 x rows uint64 for the batch searches'
        per-request start and end times (GPU global timer, ns); 0 turns it off."""
        self._check(self._lib.gmapf_set_search_timeline(self._h, d_timeline or None, int(rows)))

    def tune_source(self) -> int:
        """0: the Config's shape, 1: tuned at the start, 2: from the autotuner cache."""
        v = C.c_int32()
        self._check(self._lib.gmapf_tune_source(self._h, C.byref(v)))
        return v.value

    def search_shape(self) -> dict:
        v = [C.c_int32() for _ in range(5)]
        self._check(self._lib.gmapf_search_shape(self._h, *[C.byref(x) for x in v]))
        return dict(zip(["T", "C", "block_threads", "visited_mode", "slots"], [x.value for x in v]))

    def search_batch(self, starts, targets, path_stride: int, check: bool = True):
        """Independent searches on host buffers (copies inside the call).
        check=False returns the outputs and statistics of a call that reported
        a device-side check (a path longer than its row, say) instead of
        raising; the status is then in the statistics' "status"."""
        s = _i32(starts)
        t = _i32(targets)
        n = len(s)
        found = np.empty(n, np.int32)
        lens = np.empty(n, np.int32)
        paths = np.full((n, path_stride), -1, np.int32)
        st = StepStats()
        rc = self._lib.gmapf_search_batch_host(self._h, _ptr(s), _ptr(t), n, _ptr(found), _ptr(lens), _ptr(paths),
                                               path_stride, C.byref(st))
        if check or rc not in (0, 8):  # 8: GMAPF_E_DEVICE
            self._check(rc)
        d = st.as_dict()
        d["status"] = rc
        return found, lens, paths, d

    def search_batch_device(self, d_starts: int, d_targets: int, n: int, d_found: int, d_lens: int, d_paths: int,
                            path_stride: int) -> dict:
        """Searches on device pointers already resident in HBM (raw addresses)."""
        st = StepStats()
        self._check(self._lib.gmapf_search_batch_device(self._h, d_starts, d_targets, n, d_found, d_lens, d_paths,
                                                         path_stride, C.byref(st)))
        return st.as_dict()

    def last_search_ms(self) -> float:
        v = C.c_float()
        self._check(self._lib.gmapf_last_search_ms(self._h, C.byref(v)))
        return v.value


class SceneBatch:
    """Several scenes stepped as one (gmapf_batch_*): each scene is a GMAPF
    that was initialised, filled and given its agents; after binding, the
    scenes keep their per-agent calls (SetAgentTargPos, GetAgentPos, ...)
    with their own ids, and frames run on the batch (one compaction, one
    persistent search launch and one mover pass for all scenes).  `world` is
    the merged context (global agent and triangle ids) for statistics,
    device-resident retargets and the stream handle."""

    def __init__(self, scenes, **options):
        self._lib = _lib.load()
        self.scenes = list(scenes)
        arr = (C.c_void_p * len(self.scenes))(*[g._h.value for g in self.scenes])
        h = C.c_void_p()
        o = make_options(**options) if options else None
        rc = self._lib.gmapf_batch_create(arr, len(self.scenes), C.byref(o) if o is not None else None, C.byref(h))
        if rc != 0:
            msg = self._lib.gmapf_last_error()
            raise GMAPFError(rc, msg.decode() if msg else "")
        self._h = h
        self.world = GMAPF._view(self._lib.gmapf_batch_world(h))

    def scene_base(self, scene: int):
        """(first global agent id, first global triangle id) of a scene."""
        a, n = C.c_int32(), C.c_int32()
        self.world._check(self._lib.gmapf_batch_scene_base(self._h, int(scene), C.byref(a), C.byref(n)))
        return a.value, n.value

    def ManualStart(self) -> None:
        self.world.ManualStart()

    def AsyncStep(self, dt: float) -> None:
        self.world.AsyncStep(dt)

    def WaitStepEnd(self) -> None:
        self.world.WaitStepEnd()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.world._h = None
            self._lib.gmapf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def clock_ns() -> int:
    """The host clock serving arrival times are measured in (steady clock, ns)."""
    return int(_lib.load().gmapf_clock_ns())
