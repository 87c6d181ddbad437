"""Path-cost references: the BFS hop optimum and the FP64 Dijkstra polyline
optimum (gmapf_b200.path_quality, scipy) against the oracle's own BFS and
Dijkstra, and the search's paths against both optima."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import path_quality as PQ
from gmapf_b200 import scenarios as S


def world(scn):
    g = G.GMAPF()
    g.Init(G.make_config(4, scn.radius, scn.speed, 4, 8, 32, scn.heuristic_k))
    S.build_map(g, scn)
    return g


def pairs(g, scn, n, seed):
    rng = np.random.default_rng(seed)
    a = g.locate(S.free_points(g, scn, n, rng)).astype(np.int32)
    b = g.locate(S.free_points(g, scn, n, rng)).astype(np.int32)
    return a, b


@pytest.mark.parametrize("scn", [S.cfg2(), S.cfg3(cells=24)], ids=["cfg2", "maze24"])
def test_optima_match_oracle(oracle_mod, scn):
    g = world(scn)
    nodes = g.map_nodes()
    om = oracle_mod.OMap(nodes)
    s, t = pairs(g, scn, 60, seed=21)
    hops, lens = PQ.optima(nodes, s, t)
    for i in range(len(s)):
        assert hops[i] == om.bfs_hops(s[i], t[i])
        ref = om.dijkstra_len(s[i], t[i])
        assert abs(lens[i] - ref) <= 1e-9 * max(1.0, ref)


def test_disconnected_optimum_is_unreachable(oracle_mod):
    nodes = np.zeros(4, G.NODE_DTYPE)
    nodes["P1"] = [[0, 0], [1, 0], [10, 0], [11, 0]]
    nodes["P2"] = [[1, 0], [1, 1], [11, 0], [11, 1]]
    nodes["P3"] = [[0, 1], [0, 1], [10, 1], [10, 1]]
    nodes["PCenter"] = (nodes["P1"] + nodes["P2"] + nodes["P3"]) / 3
    nodes["NeibsIdx"] = [[1, -1, -1], [0, -1, -1], [3, -1, -1], [2, -1, -1]]
    hops, lens = PQ.optima(nodes, [0, 0], [1, 3])
    assert hops.tolist() == [1, -1] and lens[1] == -1.0
    om = oracle_mod.OMap(nodes)
    assert om.bfs_hops(0, 3) == -1 and om.dijkstra_len(0, 3) == -1.0


@pytest.mark.parametrize("T,Cap", [(8, 32), (2, 16), (32, 16)])
def test_search_paths_against_optima(oracle_mod, T, Cap):
    scn = S.cfg3(cells=24)
    g = world(scn)
    nodes = g.map_nodes()
    om = oracle_mod.OMap(nodes)
    s, t = pairs(g, scn, 200, seed=22)
    stride = om.n
    f, l, p, _ = om.search_batch(s, t, T, Cap, 1.0, path_stride=stride)
    hops, lens = PQ.optima(nodes, s, t)
    cen = nodes["PCenter"].astype(np.float64)
    for i in range(len(s)):
        if not f[i] or s[i] == t[i]:
            continue
        assert l[i] >= hops[i]  # never shorter than the hop optimum
        assert PQ.polyline_length(cen, s[i], p[i, :l[i]]) >= lens[i] * (1 - 1e-12)
    q = PQ.summary(nodes, s, t, l, [p[i, :l[i]] for i in range(len(s))])
    assert q["queries"] > 150 and q["hops_over_bfs"]["mean"] >= 1.0


def test_exhaustive_queues_find_every_reachable_pair(oracle_mod):
    # queues large enough never evict, so found == reachable
    scn = S.cfg2()
    g = world(scn)
    nodes = g.map_nodes()
    om = oracle_mod.OMap(nodes)
    s, t = pairs(g, scn, 300, seed=23)
    f, l, p, _ = om.search_batch(s, t, 8, 512, 1.0, path_stride=om.n)
    hops, _ = PQ.optima(nodes, s, t)
    assert np.array_equal(f.astype(bool), hops >= 0)
