"""ctypes front-end of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class SearchStats(C.Structure):
    _fields_ = [("rounds", C.c_longlong), ("expansions", C.c_longlong), ("claims", C.c_longlong),
                ("deg_sum", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
I = C.POINTER(C.c_int)
F = C.POINTER(C.c_float)


def _p(a, t=C.c_int):
    return a.ctypes.data_as(C.POINTER(t))


def load():
    global _lib
    if _lib is not None:
        return _lib
    src = [HERE / "gmapf_oracle.cpp", HERE / "gmapf_oracle.h", HERE / "navmesh_oracle.cpp", HERE / "Makefile"]
    if (not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in src)) and \
            os.environ.get("GMAPF_NO_BUILD") != "1":
        sys.path.insert(0, str(HERE.parent))
        from gmapf_b200 import build as _build  # the build recipe only (where the CDT headers are)
        cdt = _build.cdt_dir()
        # a library built with the CDT headers is not replaced by one built
        # without them (a machine without the reference tree keeps the first)
        if cdt or not LIB.exists():
            subprocess.run(["make", "-s", "-C", str(HERE)] + ([f"CDT_DIR={cdt}"] if cdt else []), check=True)
    lib = C.CDLL(str(LIB))
    sig = {
        "orc_map_create": (C.c_void_p, [F, I, C.c_int]),
        "orc_map_destroy": (None, [C.c_void_p]),
        "orc_map_count": (C.c_int, [C.c_void_p]),
        "orc_map_centroids": (None, [C.c_void_p, F]),
        "orc_locate_linear": (C.c_int, [C.c_void_p, C.c_float, C.c_float]),
        "orc_locate": (C.c_int, [C.c_void_p, C.c_float, C.c_float]),
        "orc_locate_batch": (None, [C.c_void_p, F, C.c_int, I]),
        "orc_navmesh_build": (C.c_int, [C.c_float, C.c_float, F, I, C.c_int, F, I, C.c_int]),
        "orc_in_node": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_int]),
        "orc_dist_sqr": (C.c_float, [C.c_void_p, C.c_int, C.c_int]),
        "orc_search": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, I, C.c_int, I,
                                 C.POINTER(SearchStats)]),
        "orc_search_batch": (C.c_int, [C.c_void_p, I, I, C.c_int, C.c_int, C.c_int, C.c_float, I, I, I, C.c_int,
                                       C.POINTER(SearchStats), C.c_int]),
        "orc_queue_sim": (C.c_int, [F, I, I, C.c_int, I, C.c_int, C.c_int, I, I]),
        "orc_search_batch_order": (C.c_int, [C.c_void_p, I, I, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int,
                                             C.c_ulonglong, I, I, I, C.c_int, C.POINTER(SearchStats), C.c_int]),
        "orc_queue_sim_order": (C.c_int, [F, I, I, C.c_int, I, C.c_int, C.c_int, C.c_int, I, I]),
        "orc_bfs_hops": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "orc_dijkstra_len": (C.c_double, [C.c_void_p, C.c_int, C.c_int]),
        "orc_world_set_smoothing": (None, [C.c_void_p, C.c_int]),
        "orc_path_len": (C.c_double, [C.c_void_p, C.c_int, I, C.c_int]),
        "orc_world_create": (C.c_void_p, [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                          C.c_float]),
        "orc_world_destroy": (None, [C.c_void_p]),
        "orc_world_add_agent": (C.c_int, [C.c_void_p, C.c_float, C.c_float]),
        "orc_world_set_target": (C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_float]),
        "orc_world_step": (None, [C.c_void_p, C.c_float, C.c_int]),
        "orc_world_count": (C.c_int, [C.c_void_p]),
        "orc_world_get": (None, [C.c_void_p, F, I, I, I, I, I, F, I]),
        "orc_world_get_path": (C.c_int, [C.c_void_p, C.c_int, I, C.c_int]),
        "orc_world_last_stats": (None, [C.c_void_p, C.POINTER(C.c_longlong)]),
        "orc_world_set": (None, [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float,
                                 C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, I, C.c_int]),
    }
    for k, (r, a) in sig.items():
        f = getattr(lib, k)
        f.restype = r
        f.argtypes = a
    _lib = lib
    return lib


def navmesh(size, obstacles):
    """(tri, nbr) of the navmesh FillMapStart(size), FillMapObstacle(o) for
    each obstacle and FillMapEnd() build (the reference's CDT call sequence,
    oracle/navmesh_oracle.cpp)."""
    lib = load()
    xy = np.ascontiguousarray(np.concatenate([np.asarray(o, np.float32).reshape(-1, 2) for o in obstacles])
                              if obstacles else np.zeros((0, 2), np.float32), np.float32)
    counts = np.ascontiguousarray([len(o) for o in obstacles], np.int32)
    cap = 4 * (len(xy) + 4) + 64
    tri = np.empty((cap, 6), np.float32)
    nbr = np.empty((cap, 3), np.int32)
    n = lib.orc_navmesh_build(float(size[0]), float(size[1]), _p(xy, C.c_float), _p(counts), len(counts),
                              _p(tri, C.c_float), _p(nbr), cap)
    if n < 0:
        raise RuntimeError({-1: "navmesh larger than expected", -2: "oracle built without the CDT headers",
                            -3: "CDT failed"}.get(n, str(n)))
    return tri[:n].copy(), nbr[:n].copy()


def nodes_to_arrays(nodes):
    """gmapf_node records (NODE_DTYPE) -> (tri float32 [n,6], nbr int32 [n,3])."""
    tri = np.ascontiguousarray(np.concatenate([nodes["P1"], nodes["P2"], nodes["P3"]], 1), np.float32)
    nbr = np.ascontiguousarray(nodes["NeibsIdx"], np.int32)
    return tri, nbr


class OMap:
    def __init__(self, nodes=None, tri=None, nbr=None):
        self.lib = load()
        if nodes is not None:
            tri, nbr = nodes_to_arrays(nodes)
        self.tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 6)
        self.nbr = np.ascontiguousarray(nbr, np.int32).reshape(-1, 3)
        self.h = self.lib.orc_map_create(_p(self.tri, C.c_float), _p(self.nbr), len(self.tri))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_map_destroy(self.h)
            self.h = None

    @property
    def n(self):
        return len(self.tri)

    def centroids(self):
        out = np.empty((self.n, 2), np.float32)
        self.lib.orc_map_centroids(self.h, _p(out, C.c_float))
        return out

    def locate(self, x, y, linear=False):
        f = self.lib.orc_locate_linear if linear else self.lib.orc_locate
        return f(self.h, float(x), float(y))

    def locate_batch(self, pts):
        """orc_locate for an (n, 2) array of points."""
        p = np.ascontiguousarray(pts, np.float32).reshape(-1, 2)
        out = np.empty(len(p), np.int32)
        self.lib.orc_locate_batch(self.h, _p(p, C.c_float), len(p), _p(out))
        return out

    def free_points(self, size, n, rng):
        """n points uniform over [0, W) x [0, H), kept when inside a triangle
        (the rule of gmapf_b200.scenarios.free_points, located here)."""
        W, H = size
        out = np.empty((0, 2), np.float32)
        while len(out) < n:
            k = max(64, 2 * (n - len(out)))
            p = np.stack([rng.uniform(0, W, k), rng.uniform(0, H, k)], 1).astype(np.float32)
            out = np.concatenate([out, p[self.locate_batch(p) >= 0]])
        return out[:n]

    def search(self, s, t, T, Cap, K=1.0):
        path = np.empty(max(1, self.n), np.int32)
        L = C.c_int()
        st = SearchStats()
        f = self.lib.orc_search(self.h, int(s), int(t), int(T), int(Cap), float(K), _p(path), len(path), C.byref(L),
                                C.byref(st))
        return f, path[:L.value].copy(), st.as_dict()

    def search_batch(self, starts, targets, T, Cap, K=1.0, threads=None, path_stride=None, order=None):
        """path_stride=0: lengths and counters only, no path rows.  order=(fifo,
        seed) emulates the reference's own orders (orc_search_batch_order):
        fifo=1 its queue key, F alone with equal F first in first out; seed != 0
        the lanes of each neighbour slot of a round in a seeded random order."""
        s = np.ascontiguousarray(starts, np.int32)
        t = np.ascontiguousarray(targets, np.int32)
        n = len(s)
        stride = max(1, self.n) if path_stride is None else path_stride
        found = np.empty(n, np.int32)
        lens = np.empty(n, np.int32)
        paths = np.full((n, stride), -1, np.int32) if stride > 0 else None
        st = SearchStats()
        nthr = int(threads or os.cpu_count() or 1)
        if order is None:
            rc = self.lib.orc_search_batch(self.h, _p(s), _p(t), n, int(T), int(Cap), float(K), _p(found), _p(lens),
                                           _p(paths) if paths is not None else None, stride, C.byref(st), nthr)
        else:
            rc = self.lib.orc_search_batch_order(self.h, _p(s), _p(t), n, int(T), int(Cap), float(K), int(order[0]),
                                                 int(order[1]), _p(found), _p(lens),
                                                 _p(paths) if paths is not None else None, stride, C.byref(st), nthr)
        if rc != 0:
            raise RuntimeError("oracle path row too small")
        return found, lens, paths, st.as_dict()

    def bfs_hops(self, s, t):
        return self.lib.orc_bfs_hops(self.h, int(s), int(t))

    def dijkstra_len(self, s, t):
        return self.lib.orc_dijkstra_len(self.h, int(s), int(t))

    def path_len(self, s, path):
        p = np.ascontiguousarray(path, np.int32)
        return self.lib.orc_path_len(self.h, int(s), _p(p), len(p))


def queue_sim(F_, G_, ids, ops, cap, fifo=False):
    lib = load()
    F_ = np.ascontiguousarray(F_, np.float32)
    G_ = np.ascontiguousarray(G_, np.int32)
    ids = np.ascontiguousarray(ids, np.int32)
    ops = np.ascontiguousarray(ops, np.int32)
    popped = np.full(len(ops), -2, np.int32)
    final = np.full(max(1, cap), -2, np.int32)
    if fifo:
        k = lib.orc_queue_sim_order(_p(F_, C.c_float), _p(G_), _p(ids), len(F_), _p(ops), len(ops), int(cap), 1,
                                    _p(popped), _p(final))
    else:
        k = lib.orc_queue_sim(_p(F_, C.c_float), _p(G_), _p(ids), len(F_), _p(ops), len(ops), int(cap), _p(popped),
                              _p(final))
    npop = int((np.asarray(ops) == 0).sum())
    return popped[:npop].copy(), final[:k].copy()


class OWorld:
    def __init__(self, omap: OMap, agents_max, radius, speed, parallel_agents, T, Cap, K=1.0):
        self.lib = load()
        self.map = omap
        self.h = self.lib.orc_world_create(omap.h, agents_max, radius, speed, parallel_agents, T, Cap, K)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_world_destroy(self.h)
            self.h = None

    def set_smoothing(self, mode):
        """0 / False off, 1 / True funnel corners, 2 corners one agent radius off the walls."""
        self.lib.orc_world_set_smoothing(self.h, int(mode))

    def add_agent(self, x, y):
        return self.lib.orc_world_add_agent(self.h, float(x), float(y))

    def set_target(self, i, x, y):
        return self.lib.orc_world_set_target(self.h, int(i), float(x), float(y))

    def step(self, dt, threads=None):
        self.lib.orc_world_step(self.h, float(dt), int(threads or os.cpu_count() or 1))

    @property
    def count(self):
        return self.lib.orc_world_count(self.h)

    def get(self):
        n = self.count
        d = {"pos": np.empty((n, 2), np.float32), "state": np.empty(n, np.int32), "cur_node": np.empty(n, np.int32),
             "targ_node": np.empty(n, np.int32), "step_idx": np.empty(n, np.int32),
             "step_node": np.empty(n, np.int32), "step_pos": np.empty((n, 2), np.float32),
             "path_len": np.empty(n, np.int32)}
        self.lib.orc_world_get(self.h, _p(d["pos"], C.c_float), _p(d["state"]), _p(d["cur_node"]),
                               _p(d["targ_node"]), _p(d["step_idx"]), _p(d["step_node"]),
                               _p(d["step_pos"], C.c_float), _p(d["path_len"]))
        return d

    def path(self, i):
        out = np.empty(max(1, self.map.n), np.int32)
        L = self.lib.orc_world_get_path(self.h, int(i), _p(out), len(out))
        return out[:L].copy()

    def last_stats(self):
        a = (C.c_longlong * 6)()
        self.lib.orc_world_last_stats(self.h, a)
        return dict(zip(["requests", "found", "expansions", "rounds", "moving", "collided"], list(a)))
