"""One batch search on a seeded maze, for profilers.

    python -m gmapf_b200.profile_search CELLS T C VISITED_MODE QUERIES [BUDGET_MB] [--timeline]

builds the CELLS x CELLS maze of the batched-uneven-queries configuration,
draws QUERIES seeded free-space start/target pairs (numpy default_rng(7),
starts then targets) and runs gmapf_search_batch_host once with threads per
agent T, queue capacity C and visited mode 1 (shared-memory bitmap), 2
(global records) or 3 (global bitmap); BUDGET_MB caps the search state
(and so the number of resident slots) to keep a profiler capture small.  Paths are not kept (a 2-entry row is passed, so long
paths raise the path-capacity flag, which is expected); the kernel time is
printed.  With --timeline each request's start and end on the GPU global
timer are recorded (gmapf_set_search_timeline) and the batch's timeline is
summarised: how long every slot stays busy, when the last request starts,
when 90% / 99% / all are done, the slowest request, and how many run at
eleven points of the launch.
"""
from __future__ import annotations

import sys

import numpy as np

from . import scenarios as S
from .api import GMAPF, GMAPFError, make_config


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
    return {"launch_ms": round(total, 3), "all_slots_busy_until_ms": round(float(busy[0]), 3) if busy else round(total, 3),
            "last_start_ms": round(float(st.max()), 3),
            "done_90_99_ms": [round(float(np.percentile(en, q)), 3) for q in (90, 99)],
            "slowest": {"request": i, "start_ms": round(float(st[i]), 3), "ms": round(float(dur[i]), 3)},
            "running_at": [[round(float(x), 2), a] for x, a in zip(grid, active)]}


def main(argv: list[str]) -> None:
    timeline = "--timeline" in argv
    argv = [a for a in argv if a != "--timeline"]
    cells, T, C, vm, nq = (int(a) for a in argv[:5])
    budget = int(argv[5]) << 20 if len(argv) > 5 else 0
    scn = S.cfg3(cells=cells)
    g = GMAPF()
    g.Init(make_config(4, scn.radius, scn.speed, 4, T, C, scn.heuristic_k))
    g.set_options(visited_mode=vm, search_mem_budget=budget)
    S.build_map(g, scn)
    rng = np.random.default_rng(7)
    s = g.locate(S.free_points(g, scn, nq, rng)).astype(np.int32)
    t = g.locate(S.free_points(g, scn, nq, rng)).astype(np.int32)
    buf = None
    if timeline:
        import torch
        buf = torch.zeros(2 * nq, dtype=torch.int64, device="cuda")
        g.set_search_timeline(buf.data_ptr(), nq)
    try:
        g.search_batch(s, t, 2)
    except GMAPFError:
        pass
    print("ms", g.last_search_ms(), g.search_shape())
    if timeline:
        print("timeline", timeline_summary(buf.cpu().numpy().reshape(nq, 2), g.search_shape()["slots"]))


if __name__ == "__main__":
    main(sys.argv[1:])
