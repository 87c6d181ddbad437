"""Seeded synthetic scenarios with the shapes of the reference's benchmark
configurations (no dataset ships with the reference; these stand in for it).

  cfg1  100x100 map, 4 rectangles (sides U[10,30]), 256 agents, r=2, T=4, C=16
  cfg2  1000x1000 map, 200 rectangles (sides U[10,60]), 2048 agents, T=8, C=32,
        every agent retargeted every 100 steps
  cfg3  4000x4000 maze from a randomized-DFS maze of cells x cells (walls 4 wide),
        16384 agents, r=2, all retargeted in the same frame
  cfg4  64 independent scenes of random sizes, obstacles, agent counts and radii
        (a scene batch), retargets with probability 0.02 per agent per step
  zigzag  the reference driver's map (main.cpp:152-175) with its agent layout
        (main.cpp:14-43)

Obstacles are axis-aligned rectangles placed without overlap (gap >= 1 and
>= 1 from the border); maze walls are non-overlapping wall segments plus
corner pillars.  Free points are drawn uniformly over the map and kept when
they lie in a navmesh triangle.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .api import GMAPF, make_config, MODE_BATCHED


@dataclass
class Scenario:
    name: str
    size: tuple
    obstacles: list  # list of (k,2) float32 vertex arrays
    agents: int
    radius: float
    speed: float
    parallel_agents: int
    threads_per_agent: int
    queue_capacity: int
    heuristic_k: float = 1.0
    dt: float = 1.0 / 60.0
    steps: int = 200
    retarget_every: int = 0
    seed: int = 0
    meta: dict = field(default_factory=dict)


def _rect(x0, y0, x1, y1):
    # the reference's obstacle vertex order (main.cpp:167-170)
    return np.array([[x0, y0], [x0, y1], [x1, y1], [x1, y0]], dtype=np.float32)


def random_rects(rng, W, H, n, lo, hi, max_tries=200000):
    out = []
    tries = 0
    while len(out) < n and tries < max_tries:
        tries += 1
        w, h = rng.uniform(lo, hi, size=2)
        if w + 2 >= W or h + 2 >= H:
            continue
        x = rng.uniform(1.0, W - w - 1.0)
        y = rng.uniform(1.0, H - h - 1.0)
        r = (np.float32(x), np.float32(y), np.float32(x + w), np.float32(y + h))
        ok = True
        for o in out:
            if not (r[2] + 1 < o[0] or o[2] + 1 < r[0] or r[3] + 1 < o[1] or o[3] + 1 < r[1]):
                ok = False
                break
        if ok:
            out.append(r)
    return [_rect(*r) for r in out]


def maze_walls(cells: int, side: float = 4000.0, thick: float = 4.0, seed: int = 3):
    """Randomized-DFS perfect maze; walls as non-overlapping segments + pillars."""
    rng = np.random.default_rng(seed)
    N = cells
    C = side / N
    t = thick / 2
    vis = np.zeros(N * N, bool)
    right = np.ones(N * N, bool)
    bottom = np.ones(N * N, bool)
    stack = [0]
    vis[0] = True
    while stack:
        c = stack[-1]
        x, y = c % N, c // N
        nb = []
        if x > 0 and not vis[c - 1]:
            nb.append(c - 1)
        if x < N - 1 and not vis[c + 1]:
            nb.append(c + 1)
        if y > 0 and not vis[c - N]:
            nb.append(c - N)
        if y < N - 1 and not vis[c + N]:
            nb.append(c + N)
        if not nb:
            stack.pop()
            continue
        n = nb[int(rng.integers(len(nb)))]
        if n == c + 1:
            right[c] = False
        elif n == c - 1:
            right[n] = False
        elif n == c + N:
            bottom[c] = False
        else:
            bottom[n] = False
        vis[n] = True
        stack.append(n)
    rects = []
    for y in range(N):
        for x in range(N):
            c = y * N + x
            if x < N - 1 and right[c]:
                rects.append(((x + 1) * C - t, y * C + t, (x + 1) * C + t, (y + 1) * C - t))
            if y < N - 1 and bottom[c]:
                rects.append((x * C + t, (y + 1) * C - t, (x + 1) * C - t, (y + 1) * C + t))
            if x < N - 1 and y < N - 1:
                rects.append(((x + 1) * C - t, (y + 1) * C - t, (x + 1) * C + t, (y + 1) * C + t))
    return [_rect(*r) for r in rects]


def cfg1(seed: int = 1) -> Scenario:
    rng = np.random.default_rng(seed)
    return Scenario("cfg1", (100.0, 100.0), random_rects(rng, 100, 100, 4, 10, 30), agents=256, radius=2.0,
                    speed=1.0, parallel_agents=256, threads_per_agent=4, queue_capacity=16, steps=200, seed=seed)


def cfg2(seed: int = 2) -> Scenario:
    rng = np.random.default_rng(seed)
    return Scenario("cfg2", (1000.0, 1000.0), random_rects(rng, 1000, 1000, 200, 10, 60), agents=2048, radius=2.0,
                    speed=1.0, parallel_agents=2048, threads_per_agent=8, queue_capacity=32, steps=1000,
                    retarget_every=100, seed=seed)


def cfg3(cells: int = 160, seed: int = 3, agents: int = 16384, threads_per_agent: int = 8,
         queue_capacity: int = 32) -> Scenario:
    return Scenario(f"cfg3-maze{cells}", (4000.0, 4000.0), maze_walls(cells, 4000.0, 4.0, seed), agents=agents,
                    radius=2.0, speed=1.0, parallel_agents=agents, threads_per_agent=threads_per_agent,
                    queue_capacity=queue_capacity, steps=1, seed=seed, meta={"cells": cells})


def cfg4(n_scenes: int = 64, seed: int = 4, agents_range=(64, 1024), threads_per_agent: int = 8,
         queue_capacity: int = 32) -> list:
    """The multi-scene configuration: n_scenes independent scenes, each with a
    map side U[200, 2000], U[10, 500] rectangles with sides U[10, 60] (as many
    as fit without overlap), U[agents_range] agents of radius U[1, 3] and speed
    1, and random retargets with probability 0.02 per agent per step."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        side = float(rng.uniform(200, 2000))
        nrect = int(rng.integers(10, 501))
        A = int(rng.integers(agents_range[0], agents_range[1] + 1))
        r = float(np.float32(rng.uniform(1, 3)))
        sub = np.random.default_rng(int(rng.integers(1 << 30)))
        out.append(Scenario(f"cfg4-scene{k}", (side, side), random_rects(sub, side, side, nrect, 10, 60, 20000),
                            agents=A, radius=r, speed=1.0, parallel_agents=A, threads_per_agent=threads_per_agent,
                            queue_capacity=queue_capacity, steps=500, seed=seed * 1000 + k,
                            meta={"retarget_p": 0.02}))
    return out


def zigzag() -> Scenario:
    obs = []
    for i in range(2, 9):  # main.cpp:152-175
        y0 = i * 100.0
        x0, x1 = (100.0, 1000.0) if i % 2 == 0 else (0.0, 100.0)
        obs.append(_rect(x0, y0, x1, y0 + 10))
    return Scenario("zigzag", (1000.0, 1000.0), obs, agents=2048, radius=2.0, speed=1.0, parallel_agents=2048,
                    threads_per_agent=2, queue_capacity=16, steps=1, seed=0)


def build_map(g: GMAPF, scn: Scenario) -> None:
    g.FillMapStart(scn.size)
    for o in scn.obstacles:
        g.FillMapObstacle(o)
    g.FillMapEnd()


def free_points(g: GMAPF, scn: Scenario, n: int, rng) -> np.ndarray:
    W, H = scn.size
    out = np.empty((0, 2), np.float32)
    while len(out) < n:
        k = max(64, 2 * (n - len(out)))
        p = np.stack([rng.uniform(0, W, k), rng.uniform(0, H, k)], 1).astype(np.float32)
        ok = g.locate(p) >= 0
        out = np.concatenate([out, p[ok]])
    return out[:n]


def make_world(scn: Scenario, mode: int = MODE_BATCHED, profiler: bool = False, block_threads: int = 0,
               threads_per_agent: int | None = None, queue_capacity: int | None = None, agents: int | None = None,
               parallel_agents: int | None = None, search_mem_budget: int = 0, visited_mode: int = 0,
               autotune: bool = False, path_smoothing: int = 0, device: int = 0, promote_rounds: int = 0):
    """Build a GMAPF for the scenario on CUDA device `device`; returns (g, starts, rng)."""
    A = scn.agents if agents is None else agents
    g = GMAPF()
    P = parallel_agents if parallel_agents is not None else (scn.parallel_agents if agents is None else A)
    g.Init(make_config(A, scn.radius, scn.speed, P, threads_per_agent or scn.threads_per_agent,
                       queue_capacity or scn.queue_capacity, scn.heuristic_k, is_profiler=profiler))
    g.set_options(mode=mode, block_threads=block_threads, search_mem_budget=search_mem_budget,
                  visited_mode=visited_mode, autotune=autotune, path_smoothing=path_smoothing, device=device,
                  promote_rounds=promote_rounds)
    build_map(g, scn)
    rng = np.random.default_rng(1000 + scn.seed)
    if scn.name == "zigzag":
        starts = np.array([[i / 5.0, 0.0] for i in range(A)], np.float32)  # main.cpp:28-32
    else:
        starts = free_points(g, scn, A, rng)
    for p in starts:
        g.AddAgent(p)
    return g, starts, rng
