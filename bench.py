#!/usr/bin/env python
"""bench.py -- the G-MAPF per-frame step on B200.

Workload (one "step" = one frame with every agent retargeted, the
batched-uneven-queries configuration): a 4000x4000 maze built by seeded
randomized DFS over cells x cells (walls 4 wide) and triangulated by CDT on
the host, 16,384 agents of radius 2 and speed 1, every agent given a fresh
uniform free-space target before each frame, threads/agent T and queue
capacity C.  One frame = request compaction, the searches (path queries),
path writes, mover (move, grid collisions, path progress) and the copy of
positions and states back to the host mirror.

  value  path queries/s with the targets already resident in device memory
         (device-side retarget + frame, CUDA events on the library's stream,
         summed over the timed frames; L2 flushed between frames)
  e2e    the same through the reference-facing API with host buffers:
         SetAgentTargPos (bulk) -> AsyncStep -> WaitStepEnd, host wall time
  plain  the plain per-agent form (one static launch per request chunk, host
         read-back of counts), same arithmetic, same frames

`--impl reference` times the reference's own CPU implementation of the path:
the reference has none, so it is the C++ restatement in oracle/ (the
deterministic port of the reference's step), multithreaded over all host
cores, on a bounded sample of each frame's requests.

Multi-GPU (torchrun): every rank runs its own scene (weak scaling, no data
path collective); the timed region is bracketed by a barrier and the time
is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import tempfile
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "p99 step ms & path queries/s at 16k agents, batched vs plain, on 1 B200"


VISITED = {1: "shared-memory bitmap", 2: "query-stamped global records", 3: "global bitmap (L2-resident)",
           4: "global bitmap, moved into shared memory by a search still running at the batch's tail"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------- helpers --

def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return ws, rank, local


def init_dist(ws, local, use_cuda=True):
    if ws <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist
    backend = "nccl" if use_cuda and torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def reduce_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        # the raw samples (GMAPF_CLOCKS_DIR, else the temp directory); the line carries the summary
        self.path = Path(os.environ.get("GMAPF_CLOCKS_DIR", tempfile.gettempdir())) / f"gmapf_clocks_rank{gpu_index}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def search_counters(T: int, C: int, vm: int):
    """The search kernel's per-unit counters for this shape from the committed
    ncu capture (profiles/search_counters.json): DRAM bytes per claimed node
    and warp instructions per round, measured on a small case (the 64x64-cell
    maze, one 16,384-query launch) and applied to the timed frames' own
    claims and rounds.  None when no capture matches the shape."""
    p = ROOT / "profiles" / "search_counters.json"
    if not p.exists():
        return None
    return json.loads(p.read_text()).get(f"T{T}_C{C}_vm{vm}")


def measured_traffic(T: int, C: int, vm: int, claims_per_step: float):
    """DRAM bytes per search launch: the capture's bytes per claimed node
    times this frame's claims (record writes dominate and grow with claims)."""
    d = search_counters(T, C, vm)
    if not d:
        return None, None
    return d["dram_bytes_per_claim"] * claims_per_step, d["source"]


def search_side_counters(T: int, C: int, vm: int, rounds: int, search_ms: float) -> dict:
    """L2 traffic rate (the capture's L2 bytes per round x the timed frames'
    rounds over their search time), threads per warp instruction and the
    share of branches whose targets were uniform across the warp, from the
    same capture; empty when none matches the shape."""
    d = search_counters(T, C, vm)
    if not d or not search_ms:
        return {}
    out = {"l2_gbs": d["l2_bytes_per_round"] * rounds / (search_ms / 1e3) / 1e9} if "l2_bytes_per_round" in d else {}
    for k in ("threads_per_warp_instruction", "branch_targets_uniform_pct"):
        if k in d:
            out[k] = d[k]
    return out


def measured_inst_per_round(T: int, C: int, vm: int):
    """Warp instructions per search round from the capture, or None."""
    d = search_counters(T, C, vm)
    if not d:
        return None, None
    return d["inst_per_round"], d["source"]


def issue_roofline(rounds: int, search_ms: float, ipr, src, sm_mhz, sms: int):
    """The search kernel against the schedulers' issue rate: instructions
    (rounds x instructions per round) per second over 4 schedulers x SMs x SM
    clock (one warp instruction per scheduler per cycle)."""
    if ipr is None or not search_ms:
        return None
    mhz = sm_mhz or 1965.0
    achieved = rounds * ipr / (search_ms / 1e3) / 1e9
    peak = 4 * sms * mhz / 1e3
    return {"bound": "issue", "kernel": "k_search", "achieved": achieved, "peak": peak,
            "unit": "G warp instructions/s", "frac": achieved / peak, "inst_per_round": ipr,
            "inst_source": src, "peak_basis": f"4 schedulers x {sms} SMs x {mhz:.0f} MHz (sampled SM clock)"}


def algorithmic_bytes(st: dict, n_nodes: int) -> float:
    """Search bytes by the fixed per-unit definitions: per expansion 12 B of
    adjacency plus 24 B per neighbour (centroid, visited word, record); per
    query N/4 B of visited bitmap, 16 B of request and 4 B per path node."""
    return (12.0 * st["expansions"] + 24.0 * st["deg_sum"] + st["requests"] * (n_nodes / 4.0 + 16.0)
            + 4.0 * st["path_nodes"])


# ----------------------------------------------------- multi-scene (cfg4) --

def multi_scene(steps: int, warmup: int, n_scenes: int = 64):
    """64 independent scenes (random sides, obstacles, agent counts and radii),
    retargets with probability 0.02 per agent per step through each scene's
    host API.  One scene batch (one compaction, one persistent search launch
    and one mover pass per frame) against the same scenes as separate
    contexts stepped in turn -- how the reference runs several maps (one map
    per GMAPF instance).  Host wall time per frame, retargets included."""
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S
    scns = S.cfg4(n_scenes, seed=4)

    def scene(scn):
        g = G.GMAPF()
        g.Init(G.make_config(scn.agents, scn.radius, scn.speed, scn.agents, scn.threads_per_agent,
                             scn.queue_capacity, scn.heuristic_k))
        S.build_map(g, scn)
        for p in S.free_points(g, scn, scn.agents, np.random.default_rng(scn.seed)):
            g.AddAgent(p)
        return g

    # the same retargets for both forms: per step, per scene (ids, points)
    probe = [scene(scn) for scn in scns]
    total = warmup + steps
    plan = []
    for k in range(total):
        row = []
        for scn, g in zip(scns, probe):
            rng = np.random.default_rng((scn.seed, k))
            ids = np.arange(scn.agents) if k == 0 else np.nonzero(rng.random(scn.agents) < 0.02)[0]
            row.append((ids.astype(np.int32), S.free_points(g, scn, len(ids), rng) if len(ids) else None))
        plan.append(row)
    for g in probe:
        g.close()
    A = sum(s.agents for s in scns)
    out = {"workload": f"{n_scenes} scenes: sides U[200,2000], U[10,500] rectangles (sides U[10,60]), "
                       f"U[64,1024] agents of radius U[1,3], retarget p=0.02 per agent per step",
           "agents": A, "steps": steps, "warmup": warmup}

    def timed(step_fn, scenes):
        wall = []
        for k in range(total):
            t0 = time.perf_counter()
            for g, (ids, pts) in zip(scenes, plan[k]):
                if pts is not None:
                    g.set_targets(ids, pts)
            step_fn()
            if k >= warmup:
                wall.append((time.perf_counter() - t0) * 1e3)
        return wall

    # one scene batch
    scenes = [scene(scn) for scn in scns]
    out["triangles"] = sum(g.node_count for g in scenes)
    batch = G.SceneBatch(scenes)
    batch.ManualStart()

    def step_batch():
        batch.AsyncStep(1.0 / 60.0)
        batch.WaitStepEnd()

    wb = timed(step_batch, scenes)
    launches = batch.world.kernel_launches
    batch.close()
    for g in scenes:
        g.close()
    # separate contexts, stepped in turn
    seps = [scene(scn) for scn in scns]
    for g in seps:
        g.ManualStart()

    def step_sep():
        for g in seps:
            g.AsyncStep(1.0 / 60.0)
            g.WaitStepEnd()

    ws = timed(step_sep, seps)
    for g in seps:
        g.close()
    for name, w in (("batch", wb), ("separate_in_turn", ws)):
        out[name] = {"ms_per_step": statistics.mean(w), "p50_step_ms": pct(w, 50), "p99_step_ms": pct(w, 99),
                     "steps_per_s": 1e3 / statistics.mean(w), "agent_steps_per_s": A * 1e3 / statistics.mean(w)}
    out["batch_over_separate"] = out["batch"]["steps_per_s"] / out["separate_in_turn"]["steps_per_s"]
    out["batch_kernel_launches"] = launches
    return out


# --------------------------------------------------------- serving (cfg5) --

def serving(rates, duration_s: float, n_scenes: int = 8, agents: int = 8192):
    """Serving loop: n_scenes resident scenes of the 1000x1000, 200-rectangle
    type (different seeds), `agents` agents each, one scene batch.  Retargets
    of uniformly chosen agents to uniform free points arrive as a Poisson
    process at each rate for duration_s; frames (movement and collision
    avoidance for every agent) run every 1/60 s.  Latency: arrival (the
    Poisson time) to the query's device completion timestamp."""
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S
    from gmapf_b200.api import clock_ns
    scns = [S.cfg2(seed=21 + k) for k in range(n_scenes)]
    scenes = []
    for scn in scns:
        g = G.GMAPF()
        g.Init(G.make_config(agents, scn.radius, scn.speed, agents, scn.threads_per_agent, scn.queue_capacity,
                             scn.heuristic_k))
        S.build_map(g, scn)
        for p in S.free_points(g, scn, agents, np.random.default_rng(scn.seed)):
            g.AddAgent(p)
        scenes.append(g)
    # targets: a pool of free points per scene
    pools = [S.free_points(g, scn, 65536, np.random.default_rng(scn.seed + 500)) for g, scn in zip(scenes, scns)]
    batch = G.SceneBatch(scenes)
    w = batch.world
    w.serve_start()
    A = n_scenes * agents
    frame_ns = int(1e9 / 60)
    out = {"workload": f"{n_scenes} resident scenes (1000x1000, 200 rectangles, seeds 21..{20 + n_scenes}), "
                       f"{agents} agents each ({A} total); Poisson retargets of uniform agents to uniform free "
                       f"points; frames every 1/60 s", "agents": A, "triangles": w.node_count,
           "duration_s": duration_s, "rates": []}
    rng = np.random.default_rng(99)
    for rate in rates:
        n = int(rate * duration_s)
        arr = np.cumsum(rng.exponential(1.0 / rate, n))
        arr = arr[arr < duration_s]
        ids = rng.integers(0, A, len(arr)).astype(np.int32)
        sc = ids // agents
        pos = np.stack([pools[s][rng.integers(0, 65536)] for s in sc]) if len(ids) else np.zeros((0, 2), np.float32)
        w.serve_drain()
        w.serve_stats(reset=True)
        steps = []
        t0 = clock_ns()
        arr_ns = (t0 + arr * 1e9).astype(np.int64)
        nxt, k = t0, 0
        end = t0 + int(duration_s * 1e9)
        while True:
            now = clock_ns()
            if now >= end and k >= len(arr_ns):
                break
            j = int(np.searchsorted(arr_ns, now, side="right"))
            if j > k:
                w.serve_submit(ids[k:j], pos[k:j], arr_ns[k:j])
                k = j
            w.serve_poll()
            if now >= nxt:
                f0 = clock_ns()
                w.AsyncStep(1.0 / 60.0)
                while not w.step_ready():  # keep admitting while the frame runs
                    now = clock_ns()
                    j = int(np.searchsorted(arr_ns, now, side="right"))
                    if j > k:
                        w.serve_submit(ids[k:j], pos[k:j], arr_ns[k:j])
                        k = j
                    w.serve_poll()
                w.WaitStepEnd()
                steps.append((clock_ns() - f0) * 1e-6)
                nxt += frame_ns
        w.serve_drain()
        st = w.serve_stats()
        out["rates"].append({
            "offered_qps": rate, "submitted": int(st["submitted"]), "completed": int(st["completed"]),
            "found": int(st["found"]), "served_qps": st["completed"] / duration_s,
            "latency_p50_ms": st["latency_p50_ms"], "latency_p99_ms": st["latency_p99_ms"],
            "latency_mean_ms": st["latency_mean_ms"], "latency_max_ms": st["latency_max_ms"],
            "batch_launches": int(st["launches"]), "ring_capacity": int(st["capacity"]),
            "frames": len(steps), "step_p50_ms": pct(steps, 50), "step_p99_ms": pct(steps, 99)})
    w.serve_stop()
    batch.close()
    for g in scenes:
        g.close()
    return out


# ------------------------------------------------------- shared definitions --

# Search shape (threads per agent, queue capacity) of the headline frames:
# the shape the autotuner picks for these maps on B200 (T=32, C=16 on both
# mazes).  Both arms run it: the GPU arm autotunes at the start and reports
# its pick; should the pick differ, its headline still runs this shape (the
# line says so), so the two arms always time the same method.
TUNED_SHAPE = {160: (32, 16), 64: (32, 16)}


def headline_shape(args):
    if args.shape:
        T, C = (int(x) for x in args.shape.split(","))
        return T, C
    return TUNED_SHAPE.get(args.cells, (args.threads_per_agent, args.queue_capacity))


def workload_config(args, triangles, A, T, C):
    """The `config` both arms print for the headline workload."""
    return {"workload": f"maze {args.cells}x{args.cells} cells on 4000x4000, {A} agents, all retargeted every "
                        f"frame", "triangles": triangles, "agents": A, "threads_per_agent": T, "queue_capacity": C}


# --------------------------------------------------------------- b200 arm --

def make_scene(cells, seed, T, C, mode, agents, profiler=True, autotune=False):
    """The maze scene on this rank's GPU (LOCAL_RANK): the library context and
    the device-resident targets the frames hand it share that device."""
    import torch
    from gmapf_b200 import scenarios as S
    scn = S.cfg3(cells=cells, seed=seed, agents=agents, threads_per_agent=T, queue_capacity=C)
    g, starts, rng = S.make_world(scn, mode=mode, profiler=profiler, autotune=autotune,
                                  device=torch.cuda.current_device())
    t0 = time.perf_counter()
    g.ManualStart()  # device upload, landmarks and (batched) the autotuner
    g.startup_s = time.perf_counter() - t0
    return scn, g, rng


def target_sets(g, scn, rng, k, A):
    from gmapf_b200 import scenarios as S
    return [S.free_points(g, scn, A, rng) for _ in range(k)]


def run_frames_device(g, sets, warmup, steps, torch, flush):
    """value: device-resident retargets; per-frame device time on the library's stream."""
    A = sets[0].shape[0]
    dev_ids = torch.arange(A, dtype=torch.int32, device="cuda")
    dev_sets = [torch.from_numpy(s).cuda() for s in sets]
    ext = torch.cuda.ExternalStream(g.stream_handle)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    stats, ms = [], []
    launches0 = None
    for k in range(warmup + steps):
        flush.zero_()  # L2 flush (larger than the 126 MB L2), outside the timed window
        torch.cuda.synchronize()
        if k == warmup:
            launches0 = g.kernel_launches
        tk = k - warmup
        if tk >= 0:
            ev[tk][0].record(ext)
        g.set_targets_device(dev_ids.data_ptr(), dev_sets[k].data_ptr(), A)
        g.AsyncStep(1.0 / 60.0)
        if tk >= 0:
            ev[tk][1].record(ext)
        g.WaitStepEnd()
        if tk >= 0:
            stats.append(g.last_stats())
    torch.cuda.synchronize()
    launches = g.kernel_launches - launches0
    ms = [a.elapsed_time(b) for a, b in ev]
    return ms, stats, launches


def run_frames_host(g, sets, warmup, steps, overlap=False):
    """e2e: host buffers through the reference-facing API.  Per frame the host
    wall time of each call (bulk SetAgentTargPos, AsyncStep, WaitStepEnd) and
    the frame's device time (CUDA events inside the frame) are kept, so the
    end-to-end tail can be attributed.  overlap=False: retarget, AsyncStep,
    WaitStepEnd in turn (the reference's usage).  overlap=True: the next
    frame's targets are set while this frame runs (after AsyncStep, before
    WaitStepEnd; the library applies them at the next AsyncStep), so the
    point location and the host work of a retarget hide behind the frame.
    Either way every timed frame includes one full retarget's copies.
    Returns (wall per frame, statistics, parts); parts["step"] is the
    AsyncStep -> WaitStepEnd time."""
    A = sets[0].shape[0]
    ids = np.arange(A, dtype=np.int32)
    wall, stats = [], []
    parts = {"retarget": [], "async_step": [], "wait_step_end": [], "step": [], "device": []}
    total = warmup + steps
    if overlap:
        g.set_targets(ids, sets[0])
    for k in range(total):
        t0 = time.perf_counter()
        if not overlap:
            g.set_targets(ids, sets[k])
        t1 = time.perf_counter()
        g.AsyncStep(1.0 / 60.0)
        t2 = time.perf_counter()
        if overlap and k + 1 < len(sets):
            g.set_targets(ids, sets[k + 1])
        t3 = time.perf_counter()
        g.WaitStepEnd()
        t4 = time.perf_counter()
        if k >= warmup:
            wall.append((t4 - t0) * 1e3)
            st = g.last_stats()
            stats.append(st)
            parts["retarget"].append((t1 - t0 + t3 - t2) * 1e3)
            parts["async_step"].append((t2 - t1) * 1e3)
            parts["wait_step_end"].append((t4 - t3) * 1e3)
            parts["step"].append((t4 - t1) * 1e3)
            parts["device"].append(st["ms_total_device"])
    return wall, stats, parts


def attribution(wall, parts):
    """p50/p99 of each part of the host-API frame time (ms)."""
    out = {"frames": len(wall), "total": {"p50": pct(wall, 50), "p99": pct(wall, 99)}}
    for k, v in parts.items():
        out[k] = {"p50": pct(v, 50), "p99": pct(v, 99), "mean": statistics.mean(v) if v else None}
    out["host_over_device"] = {"p50": pct(wall, 50) - pct(parts["device"], 50),
                               "p99": pct(wall, 99) - pct(parts["device"], 99)}
    return out


def path_quality(g, sample):
    """Hop count over the BFS optimum and centroid polyline length over the
    FP64 Dijkstra optimum, for a sample of the last frame's agents (their
    start is the current triangle: nobody moves in a full-retarget frame)."""
    from gmapf_b200 import path_quality as PQ
    d = g.debug_agents()
    ids = np.random.default_rng(5).choice(len(d["cur_node"]), size=min(sample, len(d["cur_node"])), replace=False)
    ids.sort()
    paths = [g.path(int(i)) for i in ids]
    q = PQ.summary(g.map_nodes(), d["cur_node"][ids], d["targ_node"][ids], d["path_len"][ids], paths)
    q["sample"] = f"{len(ids)} agents of the last timed frame (found paths with start != target)"
    return q


def pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q, method="higher")) if len(v) else None


def cpu_baseline(g, scn, sets, T, C, sample, threads):
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    om = O.OMap(g.map_nodes())
    d = g.debug_agents()
    starts = d["cur_node"][:sample]
    targets = g.locate(sets[0][:sample])
    t0 = time.perf_counter()
    found, lens, _, st = om.search_batch(starts, targets, T, C, threads=threads, path_stride=0)
    dt = time.perf_counter() - t0
    return {"value": sample / dt, "unit": "path queries/s", "cores": threads, "kind": "port",
            "sample": f"{sample} of the frame's {len(sets[0])} queries (same map, T={T}, C={C}), "
                      f"oracle/ C++ restatement, {threads} host threads"}


def longest_query(g, starts, targets, torch):
    """The frame's slowest search: found with the search timeline on a
    frame-sized batch of the frame's queries (each request's start and end on
    the GPU global timer), then timed alone (one-query batch, CUDA events,
    best of 3).  Its time alone bounds any schedule of the frame from below."""
    n = len(starts)
    tl = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
    g.set_search_timeline(tl.data_ptr(), n)
    g.search_batch(starts, targets, 2, check=False)  # 2-entry rows: long paths raise the path-capacity flag
    batch_ms = g.last_search_ms()
    g.set_search_timeline(0, 0)
    x = tl.cpu().numpy().reshape(n, 2)
    dur = (x[:, 1] - x[:, 0]) / 1e6
    i = int(np.argmax(dur))
    alone = []
    for _ in range(3):
        st = g.search_batch(starts[i:i + 1], targets[i:i + 1], 2, check=False)[3]
        alone.append(g.last_search_ms())
    return {"query": i, "rounds": int(st["rounds"]), "path_len": int(st["path_nodes"]),
            "alone_ms": min(alone), "in_batch_ms": float(dur[i]), "batch_ms": batch_ms,
            "us_per_round_alone": 1e3 * min(alone) / max(1, st["rounds"]),
            "us_per_round_in_batch": 1e3 * float(dur[i]) / max(1, st["rounds"])}


def mover_roofline(stats, A, peak, peak_kind):
    """The mover phase (k_move_bin, k_cell_scan, k_scatter, k_collide_progress)
    against HBM: per agent per frame 64 + 16 B plus 8 B per agent read from
    the 3x3 grid cells (the `neighbours` counter), over the mover's CUDA-event
    time of the frames in which agents moved."""
    fr = [s for s in stats if s["moving"] > 0 and s["ms_mover"] > 0]
    if not fr:
        return None
    byt = sum(80.0 * A + 8.0 * s["neighbours"] for s in fr)
    ms = sum(s["ms_mover"] for s in fr)
    achieved = byt / (ms / 1e3) / 1e9
    return {"bound": "hbm", "kernels": "k_move_bin + k_cell_scan + k_scatter + k_collide_progress",
            "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
            "algorithmic_bytes_per_frame": byt / len(fr), "mover_ms_per_frame": ms / len(fr),
            "neighbours_per_agent": sum(s["neighbours"] for s in fr) / (len(fr) * A), "frames": len(fr)}


def mover_cfg2(steps, peak, peak_kind):
    """The reference's headline-scale configuration as specified (its TestFull
    driver, main.cpp:45-86): 1000x1000 map with 200 rectangles, 2,048 agents
    of radius 2 and speed 1, every agent retargeted to a fresh free point
    every 100 steps, T=8, C=32, `steps` frames of 1/60 s through the host API."""
    from gmapf_b200 import scenarios as S
    import gmapf_b200 as G
    scn = S.cfg2()
    A = scn.agents
    g, starts, rng = S.make_world(scn, agents=A, profiler=True)
    g.ManualStart()
    ids = np.arange(A, dtype=np.int32)
    wall, stats = [], []
    for k in range(steps):
        t0 = time.perf_counter()
        if k % scn.retarget_every == 0:
            g.set_targets(ids, S.free_points(g, scn, A, rng))
        t1 = time.perf_counter()
        g.AsyncStep(scn.dt)
        g.WaitStepEnd()
        wall.append((time.perf_counter() - t1) * 1e3)
        stats.append(g.last_stats())
    out = {"workload": "1000x1000, 200 rectangles (sides 10-60), 2048 agents r=2 speed 1, all retargeted every "
                       f"100 steps, T=8, C=32, {steps} steps", "triangles": g.node_count, "agents": A,
           "steps": steps, "p50_step_ms": pct(wall, 50), "p99_step_ms": pct(wall, 99),
           "agent_steps_per_s": A * steps / (sum(wall) / 1e3),
           "device_ms_per_step": statistics.mean(s["ms_total_device"] for s in stats),
           "moving_per_step": statistics.mean(s["moving"] for s in stats),
           "roofline": mover_roofline(stats, A, peak, peak_kind)}
    g.close()
    return out


def mover_frames(g, frames, torch, flush, peak, peak_kind):
    """Frames with no retargets after the full-retarget frames: every agent
    walks its path (and collides).  Host wall per frame, the frame's and the
    mover's CUDA-event device time; L2 flushed between frames."""
    A = g.agent_count
    wall, stats = [], []
    for k in range(frames):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.AsyncStep(1.0 / 60.0)
        g.WaitStepEnd()
        wall.append((time.perf_counter() - t0) * 1e3)
        stats.append(g.last_stats())
    mv = [s["ms_mover"] for s in stats]
    return {"frames": frames, "agents": A, "p50_step_ms": pct(wall, 50), "p99_step_ms": pct(wall, 99),
            "device_ms_per_step": {"p50": pct([s["ms_total_device"] for s in stats], 50),
                                   "p99": pct([s["ms_total_device"] for s in stats], 99)},
            "mover_ms_per_step": {"p50": pct(mv, 50), "p99": pct(mv, 99)},
            "moving_per_step": statistics.mean(s["moving"] for s in stats),
            "agent_steps_per_s": A * frames / (sum(wall) / 1e3),
            "agent_steps_per_s_device": A * frames / (sum(s["ms_total_device"] for s in stats) / 1e3),
            "roofline": mover_roofline(stats, A, peak, peak_kind)}


def bench_b200(args):
    import torch
    ws, rank, local = dist_env()
    dist = init_dist(ws, local)
    torch.cuda.set_device(local)
    import gmapf_b200 as G

    A = args.agents
    Tc, Cc = args.threads_per_agent, args.queue_capacity  # the Config's shape (the plain form's)
    Th, Ch = headline_shape(args)  # the headline shape, shared with the reference arm
    seed = 3 + rank
    autotune = not args.no_autotune
    scn, g, rng = make_scene(args.cells, seed, Tc, Cc, G.MODE_BATCHED, A, autotune=autotune)
    shape = g.search_shape()
    pick = (shape["T"], shape["C"])
    shape_source = "autotuned per map" if autotune else "fixed"
    if pick != (Th, Ch):
        g.close()
        scn, g, rng = make_scene(args.cells, seed, Th, Ch, G.MODE_BATCHED, A)
        shape = g.search_shape()
        shape_source = (f"the headline shape shared with the reference arm (the autotuner picked T={pick[0]}, "
                        f"C={pick[1]})" if autotune else "fixed")
    n_nodes = g.node_count
    K, W = args.steps, args.warmup
    sets = target_sets(g, scn, rng, W + K, A)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")  # 256 MB > L2
    peak, peak_kind = measured_peaks()

    barrier(dist)
    with ClockSampler(local) as clk:
        ms, dstats, launches = run_frames_device(g, sets, W, K, torch, flush)
    barrier(dist)
    dev_total_ms = reduce_max(dist, float(sum(ms)))
    queries = float(sum(s["requests"] for s in dstats))
    all_queries = reduce_sum(dist, queries)
    value = all_queries / (dev_total_ms / 1e3)

    # The extras below belong to the one-GPU line: a multi-GPU line carries
    # the scaled metric only, so the GPUs of a scaling run are not held for them.
    extras = ws == 1

    # path quality of the last device-timed frame (sample; outside the timing)
    quality = None
    if extras and args.quality_sample > 0:
        quality = path_quality(g, args.quality_sample)

    # the frame's slowest search, alone (its time bounds the frame from below)
    longest = None
    if extras and args.longest:
        d = g.debug_agents()
        longest = longest_query(g, d["cur_node"].astype(np.int32), g.locate(sets[-1]).astype(np.int32), torch)

    # p99 over many full-retarget frames through the host API (fresh targets
    # each): the next frame's targets set while a frame runs, and, for the
    # attribution of the end-to-end tail, the reference's usage in turn
    p99_long = None
    if extras and args.p99_frames > 0:
        p99_long = {"frames": args.p99_frames}
        for name, ov in (("overlapped", True), ("sequential", False)):
            wl, _, pl = run_frames_host(g, target_sets(g, scn, rng, 3 + args.p99_frames, A), 3, args.p99_frames,
                                        overlap=ov)
            p99_long[name] = {"p50_step_ms": pct(pl["step"], 50), "p99_step_ms": pct(pl["step"], 99),
                              "max_step_ms": max(pl["step"]), "p99_frame_wall_ms": pct(wl, 99),
                              "attribution": attribution(wl, pl)}

    # e2e through the host API (fresh targets, same scene): the headline form
    # sets each frame's targets while the previous frame runs
    sets_e2e = target_sets(g, scn, rng, W + K, A)
    g.reset_profiler()
    barrier(dist)
    wall, hstats, parts = run_frames_host(g, sets_e2e, W, K, overlap=True)
    barrier(dist)
    e2e_total = reduce_max(dist, float(sum(wall)))
    e2e_q = reduce_sum(dist, float(sum(s["requests"] for s in hstats)))
    e2e_value = e2e_q / (e2e_total / 1e3)
    e2e_seq = None
    if extras:
        wall_s, hst_s, parts_s = run_frames_host(g, sets_e2e, W, K, overlap=False)
        e2e_seq = {"value": sum(s["requests"] for s in hst_s) / (sum(wall_s) / 1e3), "unit": "path queries/s",
                   "p50_step_ms": pct(parts_s["step"], 50), "p99_step_ms": pct(parts_s["step"], 99),
                   "attribution": attribution(wall_s, parts_s)}

    # roofline of the dominant kernel (search), from the profiler's CUDA events
    search_ms = [s["ms_search"] for s in dstats]
    ab = [algorithmic_bytes(s, n_nodes) for s in dstats]
    achieved = sum(ab) / (sum(search_ms) / 1e3) / 1e9
    traffic, traffic_src = measured_traffic(shape["T"], shape["C"], shape["visited_mode"],
                                            sum(s["claims"] for s in dstats) / max(1, K))
    ipr, ipr_src = measured_inst_per_round(shape["T"], shape["C"], shape["visited_mode"])
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count

    # frames in which every agent walks its path (the mover at the maze scale)
    moving = None
    if extras and args.mover_frames > 0:
        moving = mover_frames(g, args.mover_frames, torch, flush, peak, peak_kind)
        moving["workload"] = (f"maze {args.cells}x{args.cells}, {A} agents walking the paths of the last "
                              f"full-retarget frame, no retargets")

    # batched form at the Config's own shape (same arithmetic as the plain form)
    fixed = None
    if extras and (Th, Ch) != (Tc, Cc) and not args.no_plain:
        scn_f, gf, rng_f = make_scene(args.cells, seed, Tc, Cc, G.MODE_BATCHED, A)
        msf, stf, _ = run_frames_device(gf, sets, W, K, torch, flush)
        wf, hf, _ = run_frames_host(gf, sets_e2e, W, K)
        fixed = {"threads_per_agent": Tc, "queue_capacity": Cc, "unit": "path queries/s",
                 "value": sum(s["requests"] for s in stf) / (sum(msf) / 1e3),
                 "e2e_value": sum(s["requests"] for s in hf) / (sum(wf) / 1e3),
                 "device_ms_per_step": {"mean": statistics.mean(msf), "p99": pct(msf, 99)},
                 "found_rate": sum(s["found"] for s in stf) / max(1, sum(s["requests"] for s in stf))}
        gf.close()

    # plain per-agent form on the same frames, at both shapes
    plain = {}
    if extras and not args.no_plain:
        for (T, C) in sorted({(Th, Ch), (Tc, Cc)}):
            scn_p, gp, rng_p = make_scene(args.cells, seed, T, C, G.MODE_PLAIN, A)
            pk = max(2, min(K, 5))
            wall_p, pst, _ = run_frames_host(gp, sets_e2e[:1 + pk], 1, pk)
            plain[f"T{T}_C{C}"] = {"threads_per_agent": T, "queue_capacity": C,
                                   "value": sum(s["requests"] for s in pst) / (sum(wall_p) / 1e3),
                                   "unit": "path queries/s", "p99_step_ms": pct(wall_p, 99),
                                   "ms_per_step": statistics.mean(wall_p), "steps": pk}
            gp.close()
    batched_over_plain = None
    if plain:
        batched_over_plain = {f"T{Th}_C{Ch}": e2e_value / plain[f"T{Th}_C{Ch}"]["value"]}
        if fixed:
            batched_over_plain[f"T{Tc}_C{Cc}"] = fixed["e2e_value"] / plain[f"T{Tc}_C{Cc}"]["value"]
        batched_over_plain["note"] = ("host-API path queries/s of the batched form over the plain form at the "
                                      "same threads per agent and queue capacity (the same searches)")

    cpu = None
    if extras and not args.no_cpu:  # on rank 0 at N=1 only
        cpu = cpu_baseline(g, scn, sets, shape["T"], shape["C"], args.cpu_sample, os.cpu_count() or 1)

    # the reference's headline-scale configuration, as specified (mover at scale)
    cfg2 = mover_cfg2(args.cfg2_steps, peak, peak_kind) if extras and args.cfg2_steps > 0 else None

    # the multi-scene configuration (scene batch against separate contexts)
    multi = None
    if extras and args.multi_scene_steps > 0:
        multi = multi_scene(args.multi_scene_steps, 3)

    # the serving configuration (Poisson retargets, frames every 1/60 s)
    serve = None
    if extras and args.serve_seconds > 0:
        serve = serving([50000, 150000, 500000], args.serve_seconds)

    # secondary workload: the 64x64-cell maze of the configuration text
    secondary = None
    if extras and args.secondary_cells and args.secondary_cells != args.cells:
        scn2, g2, rng2 = make_scene(args.secondary_cells, 3, Tc, Cc, G.MODE_BATCHED, A, autotune=autotune)
        sh2 = g2.search_shape()
        sets2 = target_sets(g2, scn2, rng2, W + K, A)
        ms2, st2, _ = run_frames_device(g2, sets2, W, K, torch, flush)
        wall2, _, parts2 = run_frames_host(g2, target_sets(g2, scn2, rng2, W + args.p99_frames_secondary,
                                                           A), W, args.p99_frames_secondary)
        d2 = g2.debug_agents()
        lq2 = longest_query(g2, d2["cur_node"].astype(np.int32), g2.locate(sets2[-1]).astype(np.int32),
                            torch) if args.longest else None
        secondary = {"workload": f"maze {args.secondary_cells}x{args.secondary_cells} cells",
                     "triangles": g2.node_count, "threads_per_agent": sh2["T"],
                     "queue_capacity": sh2["C"], "block_threads": sh2["block_threads"],
                     "value": sum(s["requests"] for s in st2) / (sum(ms2) / 1e3),
                     "e2e_value": A * len(wall2) / (sum(wall2) / 1e3), "p99_step_ms": pct(wall2, 99),
                     "p50_step_ms": pct(wall2, 50), "ms_per_step_device": statistics.mean(ms2),
                     "device_ms_per_step": {"p50": pct(ms2, 50), "p99": pct(ms2, 99)},
                     "attribution": attribution(wall2, parts2), "longest_query": lq2}
        g2.close()

    if rank == 0:
        st_sum = {k: sum(s[k] for s in dstats) for k in ["requests", "found", "expansions", "rounds", "claims",
                                                          "promoted"]}
        clocks = clk.summary()
        cfg = workload_config(args, n_nodes, A, shape["T"], shape["C"])
        cfg.update({"l2": "flushed between frames (256 MB write); per-frame search records exceed L2",
                    "parallelism": f"{ws} independent scenes (one per GPU)"})
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "path queries/s",
            "n_gpus": ws,
            "steps": K,
            "warmup": W,
            "ms_per_step": dev_total_ms / K,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+i32",
            "data": "synthetic: seeded randomized-DFS maze, uniform free-space starts and targets",
            "config": cfg,
            "setup": {"block_threads": shape["block_threads"], "shape_source": shape_source,
                      "autotuner_pick": {"threads_per_agent": pick[0], "queue_capacity": pick[1]},
                      "start_s": round(g.startup_s, 2), "config_threads_per_agent": Tc,
                      "config_queue_capacity": Cc, "visited_mode": VISITED[shape["visited_mode"]],
                      "slots": shape["slots"], "form": "batched (persistent search, CUDA graph)",
                      # visited placement 4: searches per frame that moved their visited
                      # bitmap into the shared memory of their block's finished warps
                      "moved_to_shared_per_frame": st_sum["promoted"] / max(1, K)},
            "p99_step_ms": pct(parts["step"], 99),
            "p50_step_ms": pct(parts["step"], 50),
            "device_ms_per_step": {"mean": statistics.mean(ms), "p50": pct(ms, 50), "p99": pct(ms, 99),
                                   "max": max(ms)},
            "found_rate": st_sum["found"] / max(1, st_sum["requests"]),
            "expansions_per_s": st_sum["expansions"] / (sum(ms) / 1e3),
            "longest_query": longest,
            "plain": plain or None,
            "batched_config_shape": fixed,
            "batched_over_plain": batched_over_plain,
            "path_quality": quality,
            "reference_cuda_build": "not run: its claim race can feed a stale record to KernelBuildPath, whose "
                                    "device asserts and unbounded parent walk can trap or hang a shared GPU; path "
                                    "costs are reported against the BFS and FP64 Dijkstra optima instead, and "
                                    "against its own queue and claim orders emulated on the CPU "
                                    "(oracle/reference_order_paths.py)",
            "e2e_step_ms_over_many_frames": p99_long,
            "e2e_attribution": attribution(wall, parts),
            "e2e_sequential": e2e_seq,
            "roofline": {"bound": "hbm", "kernel": "k_search", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": traffic_src,
                         "search_ms_per_step": statistics.mean(search_ms),
                         "algorithmic_bytes_per_step": statistics.mean(ab),
                         **search_side_counters(shape["T"], shape["C"], shape["visited_mode"], st_sum["rounds"],
                                                sum(search_ms))},
            "roofline_issue": issue_roofline(st_sum["rounds"], sum(search_ms), ipr, ipr_src, clocks.get("sm_mhz"),
                                             sms),
            "mover": {"maze_frames": moving, "cfg2": cfg2},
            "cpu_baseline": cpu,
            # per frame: target points to the device point location (8 B) and
            # the located triangles back (4 B), dirty target records (16 B)
            # and dt up; positions (8 B) and states (4 B), counters and
            # statistics back
            "e2e": {"value": e2e_value, "unit": "path queries/s", "h2d_bytes_per_step": 24 * A + 4,
                    "d2h_bytes_per_step": 16 * A + 64 + 8 * 9, "p99_step_ms": pct(parts["step"], 99),
                    "p50_step_ms": pct(parts["step"], 50),
                    "form": "each frame's targets set (bulk SetAgentTargPos) while the previous frame runs"},
            "gpu_launches": launches,
            "clocks": clocks,
            "secondary": secondary,
            "multi_scene": multi,
            "serving": serve,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------- reference arm --

def bench_reference(args):
    """The reference has no CPU implementation of the step (PathFinderCPU.h is
    unused and a different algorithm), so this arm times its C++ restatement
    in oracle/ on all host cores, on the GPU arm's workload and search shape.
    Nothing here loads the product library: the navmesh comes from the
    oracle's own build (the reference's CDT call sequence) and points are
    located by the oracle."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    from gmapf_b200 import scenarios as S  # the seeded scenario generator only (pure numpy)
    A = args.agents
    T, C = headline_shape(args)
    seed = 3
    scn = S.cfg3(cells=args.cells, seed=seed, agents=A, threads_per_agent=T, queue_capacity=C)
    tri, nbr = O.navmesh(scn.size, scn.obstacles)
    om = O.OMap(tri=tri, nbr=nbr)
    # the GPU arm's frames: agents at seeded free points, every frame a fresh
    # set of free-point targets from the same generator
    rng = np.random.default_rng(1000 + scn.seed)
    starts = om.locate_batch(om.free_points(scn.size, A, rng))
    threads = os.cpu_count() or 1
    sample = min(args.ref_sample, A)
    times, qs = [], []
    for k in range(args.warmup + args.steps):
        targets = om.locate_batch(om.free_points(scn.size, A, rng))
        t0 = time.perf_counter()
        om.search_batch(starts[:sample], targets[:sample], T, C, threads=threads, path_stride=0)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
            qs.append(sample)
    value = sum(qs) / sum(times)
    desc = (f"the first {sample} agents' queries of each {A}-agent full-retarget frame (same maze, starts and "
            f"targets as the GPU arm's frames, T={T}, C={C}); the reference has no CPU step, so this is its C++ "
            f"restatement in oracle/, {threads} host threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "path queries/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+i32",
            "data": "synthetic: seeded randomized-DFS maze, uniform free-space starts and targets",
            "config": workload_config(args, len(tri), A, T, C),
            "cpu_baseline": {"value": value, "unit": "path queries/s", "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": "path queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------- profiling runs --

def timeline_summary(tl: np.ndarray, slots: int) -> dict:
    """tl: (n, 2) start/end in ns of one batch; times in ms from the first start."""
    t0 = int(tl[:, 0].min())
    st = (tl[:, 0].astype(np.int64) - t0) / 1e6
    en = (tl[:, 1].astype(np.int64) - t0) / 1e6
    total = float(en.max())
    grid = np.linspace(0.0, total, 11)
    active = [int(((st <= x) & (en > x)).sum()) for x in grid]
    # the first moment after the ramp at which fewer than 90% of the slots are busy
    busy = [x for x, a in zip(grid, active) if x > 0 and a < 0.9 * min(slots, len(tl))]
    dur = en - st
    i = int(np.argmax(dur))
    return {"launch_ms": round(total, 3),
            "all_slots_busy_until_ms": round(float(busy[0]), 3) if busy else round(total, 3),
            "last_start_ms": round(float(st.max()), 3),
            "done_90_99_ms": [round(float(np.percentile(en, q)), 3) for q in (90, 99)],
            "slowest": {"request": i, "start_ms": round(float(st[i]), 3), "ms": round(float(dur[i]), 3)},
            "running_at": [[round(float(x), 2), a] for x, a in zip(grid, active)]}


def profile_search(spec: str, budget_mb: int, timeline: bool):
    """One batch search on a seeded maze, for profilers (ncu -k k_search):
    spec = "CELLS,T,C,VISITED_MODE,QUERIES".  Builds the CELLS x CELLS maze of
    the batched-uneven-queries configuration, draws QUERIES seeded free-space
    start/target pairs (numpy default_rng(7), starts then targets) and runs
    gmapf_search_batch_host once with threads per agent T, queue capacity C
    and visited mode 1 (shared-memory bitmap), 2 (global records), 3
    (global bitmap) or 4 (global bitmap, moved into shared memory by a search
    still running at the batch's tail); budget_mb caps the search state (and so the resident
    slots) to keep a capture small.  Paths are not kept (2-entry rows: long
    paths raise the path-capacity flag, which is expected).  With timeline,
    each request's start and end on the GPU global timer are recorded
    (gmapf_set_search_timeline) and summarised."""
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S
    cells, T, C, vm, nq = (int(x) for x in spec.split(","))
    scn = S.cfg3(cells=cells)
    g = G.GMAPF()
    g.Init(G.make_config(4, scn.radius, scn.speed, 4, T, C, scn.heuristic_k))
    g.set_options(visited_mode=vm, search_mem_budget=budget_mb << 20)
    S.build_map(g, scn)
    rng = np.random.default_rng(7)
    s = g.locate(S.free_points(g, scn, nq, rng)).astype(np.int32)
    t = g.locate(S.free_points(g, scn, nq, rng)).astype(np.int32)
    buf = None
    if timeline:
        import torch
        buf = torch.zeros(2 * nq, dtype=torch.int64, device="cuda")
        g.set_search_timeline(buf.data_ptr(), nq)
    st = g.search_batch(s, t, 2, check=False)[3]  # long paths overflow the 2-entry rows: expected
    out = {"search_ms": g.last_search_ms(), "shape": g.search_shape()}
    out["stats"] = {k: st[k] for k in ("requests", "found", "rounds", "expansions", "claims", "deg_sum",
                                       "path_nodes", "promoted")}
    if timeline:
        out["timeline"] = timeline_summary(buf.cpu().numpy().reshape(nq, 2), g.search_shape()["slots"])
    print(json.dumps(out), flush=True)
    g.close()


def profile_frames(workload: str, frames: int):
    """Frames for profilers (ncu -k on the mover kernels), no bench line.
    workload "cfg2": the 2,048-agent configuration, all agents retargeted at
    frame 0 and walking after; "maze64": the 64x64-cell maze with 16,384
    agents, all retargeted at frame 0 and walking after.  Frame 0 carries the
    searches; frames 1.. move and collide every agent."""
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S
    if workload == "cfg2":
        scn, A = S.cfg2(), 2048
    else:
        scn, A = S.cfg3(cells=int(workload[4:])), 16384
    g, starts, rng = S.make_world(scn, agents=A, threads_per_agent=8, queue_capacity=32, profiler=True)
    g.ManualStart()
    g.set_targets(np.arange(A, dtype=np.int32), S.free_points(g, scn, A, rng))
    st = []
    for k in range(frames):
        g.AsyncStep(1.0 / 60.0)
        g.WaitStepEnd()
        st.append(g.last_stats())
    print(json.dumps({"workload": workload, "agents": A, "frames": frames,
                      "moving": [s["moving"] for s in st], "ms_mover": [round(s["ms_mover"], 4) for s in st]}))
    g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cells", type=int, default=160, help="maze cells per side (160: ~100k triangles)")
    ap.add_argument("--secondary-cells", type=int, default=64, help="also report this maze (0: off)")
    ap.add_argument("--p99-frames", type=int, default=100,
                    help="extra full-retarget frames through the host API for the step p50/p99 (0: off)")
    ap.add_argument("--serve-seconds", type=float, default=1.0,
                    help="seconds per arrival rate of the serving configuration (0: off)")
    ap.add_argument("--multi-scene-steps", type=int, default=100,
                    help="frames of the 64-scene configuration, batch vs separate contexts (0: off)")
    ap.add_argument("--agents", type=int, default=16384)
    ap.add_argument("--threads-per-agent", type=int, default=8)
    ap.add_argument("--queue-capacity", type=int, default=32)
    ap.add_argument("--cpu-sample", type=int, default=2048)
    ap.add_argument("--ref-sample", type=int, default=2048)
    ap.add_argument("--shape", default="", metavar="T,C",
                    help="headline search shape of both arms (default: the autotuner's pick for the maze)")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--quality-sample", type=int, default=128, help="agents whose paths are compared with BFS/Dijkstra")
    ap.add_argument("--no-autotune", action="store_true", help="batched form at the Config's T and C")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-longest", dest="longest", action="store_false",
                    help="skip timing the frame's slowest search alone")
    ap.add_argument("--mover-frames", type=int, default=30,
                    help="frames with every agent walking its path after the full-retarget frames (0: off)")
    ap.add_argument("--cfg2-steps", type=int, default=1000,
                    help="steps of the 2,048-agent configuration, retargets every 100 (0: off)")
    ap.add_argument("--p99-frames-secondary", type=int, default=30,
                    help="host-API frames of the secondary maze for its p50/p99")
    ap.add_argument("--profile-search", default="", metavar="CELLS,T,C,VM,QUERIES",
                    help="profiling run: one batch search on the CELLS maze (no bench line)")
    ap.add_argument("--profile-budget-mb", type=int, default=0, help="search-state cap of --profile-search")
    ap.add_argument("--profile-timeline", action="store_true", help="--profile-search: per-request timeline")
    ap.add_argument("--profile-frames", default="", metavar="cfg2|mazeN",
                    help="profiling run: frames of the mover workload (no bench line)")
    args = ap.parse_args()
    if args.profile_frames:
        profile_frames(args.profile_frames, max(2, args.steps))
        return
    if args.profile_search:
        profile_search(args.profile_search, args.profile_budget_mb, args.profile_timeline)
        return
    if args.warmup < 3:
        log("warmup raised to 3 (timing rule)")
        args.warmup = 3
    if args.impl == "reference":
        bench_reference(args)
    else:
        bench_b200(args)


if __name__ == "__main__":
    main()
