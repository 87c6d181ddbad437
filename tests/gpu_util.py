"""Helpers shared by the GPU parity tests."""
import numpy as np

import gmapf_b200 as G
from gmapf_b200 import scenarios as S


def map_world(scn, T=None, Cap=None, mode=G.MODE_BATCHED, agents=4, block_threads=0, visited_mode=0,
              order=True, promote_rounds=None):
    """promote_rounds: with visited placement 4 a search moves its bitmap into
    its block's shared memory once it has run that many rounds and the block's
    other warps have left; by default these tests let it move from its first
    round on."""
    g = G.GMAPF()
    g.Init(G.make_config(agents, scn.radius, scn.speed, agents, T or scn.threads_per_agent,
                         Cap or scn.queue_capacity, scn.heuristic_k))
    if promote_rounds is None:
        promote_rounds = 1 if visited_mode == 4 else 0
    g.set_options(mode=mode, block_threads=block_threads, visited_mode=visited_mode, order_by_estimate=order,
                  promote_rounds=promote_rounds)
    S.build_map(g, scn)
    return g


def random_queries(g, scn, n, seed):
    rng = np.random.default_rng(seed)
    a = g.locate(S.free_points(g, scn, n, rng))
    b = g.locate(S.free_points(g, scn, n, rng))
    return a.astype(np.int32), b.astype(np.int32)


def close_rel(a, b, rtol=1e-4):
    """|a-b| <= rtol * max(|b|, 1), NaN == NaN."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    ok = np.abs(a - b) <= rtol * np.maximum(np.abs(b), 1.0)
    return bool(np.all(ok | both_nan)), float(np.nanmax(np.abs(a - b))) if a.size else 0.0
