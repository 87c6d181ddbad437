"""One batch search on a seeded maze, for profilers.

    python -m gmapf_b200.profile_search CELLS T C VISITED_MODE QUERIES [BUDGET_MB]

builds the CELLS x CELLS maze of the batched-uneven-queries configuration,
draws QUERIES seeded free-space start/target pairs (numpy default_rng(7),
starts then targets) and runs gmapf_search_batch_host once with threads per
agent T, queue capacity C and visited mode 1 (shared-memory bitmap), 2
(global records) or 3 (global bitmap); BUDGET_MB caps the search state
(and so the number of resident slots) to keep a profiler capture small.  Paths are not kept (a 2-entry row is passed, so long
paths raise the path-capacity flag, which is expected); the kernel time is
printed.
"""
from __future__ import annotations

import sys

import numpy as np

from . import scenarios as S
from .api import GMAPF, GMAPFError, make_config


def main(argv: list[str]) -> None:
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
    try:
        g.search_batch(s, t, 2)
    except GMAPFError:
        pass
    print("ms", g.last_search_ms(), g.search_shape())


if __name__ == "__main__":
    main(sys.argv[1:])
