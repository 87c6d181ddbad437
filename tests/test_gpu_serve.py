"""Serving form (gmapf_serve_*): retargets admitted continuously into a
device ring, drained by a persistent search launch while the host keeps
appending, installed into agents at frame boundaries.  Results are exact
against the batch search and the oracle, and the same alone and in a mix."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S

pytestmark = pytest.mark.gpu


def world(scn, agents, T=8, Cap=32, vm=0):
    # visited placement 4: searches may move into shared memory from their first round on
    g, starts, rng = S.make_world(scn, agents=agents, threads_per_agent=T, queue_capacity=Cap, visited_mode=vm,
                                  promote_rounds=1 if vm == 4 else 0)
    g.ManualStart()
    return g, starts, rng


def oracle_check(oracle_mod, g, T, Cap, starts, targets, results):
    om = oracle_mod.OMap(g.map_nodes())
    f, l, p, _ = om.search_batch(np.asarray(starts, np.int32), np.asarray(targets, np.int32), T, Cap, 1.0,
                                 path_stride=om.n)
    for i, (rf, rl, rp) in enumerate(results):
        assert rf == f[i] and rl == l[i], f"query {i}: ({rf}, {rl}) vs oracle ({f[i]}, {l[i]})"
        if rf:
            assert np.array_equal(rp, p[i, :l[i]]), f"query {i}: path differs"


@pytest.mark.parametrize("vm", [1, 3, 4])
def test_serve_matches_oracle_and_installs_paths(oracle_mod, vm):
    scn = S.cfg2()
    g, starts, rng = world(scn, 600, vm=vm)
    g.serve_start()
    ids = np.arange(0, 600, 2, dtype=np.int32)
    tp = S.free_points(g, scn, len(ids), rng)
    g.serve_submit(ids, tp)
    g.serve_drain()
    st = g.serve_stats()
    assert st["completed"] == len(ids) and st["in_flight"] == 0 and st["waiting"] == 0
    s_nodes = g.locate(starts[ids])
    t_nodes = g.locate(tp)
    res = [g.serve_result(int(a)) for a in ids]
    oracle_check(oracle_mod, g, 8, 32, s_nodes, t_nodes, res)
    # the next frame installs them
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    d = g.debug_agents()
    for a, (f, L, p) in zip(ids, res):
        assert d["targ_node"][a] == t_nodes[list(ids).index(a)]
        assert d["path_len"][a] == (L if f else 0)
        if f and L > 0:
            assert np.array_equal(g.path(int(a)), p)
    untouched = np.setdiff1d(np.arange(600), ids)
    assert np.all(d["state"][untouched] == G.EAgentState.Idle)


def test_same_alone_and_in_the_mix(oracle_mod):
    scn = S.cfg2()
    g, starts, rng = world(scn, 1200)
    g.serve_start()
    a_ids = np.arange(100, dtype=np.int32)
    a_tp = S.free_points(g, scn, len(a_ids), rng)
    g.serve_submit(a_ids, a_tp)
    g.serve_drain()
    alone = {int(a): g.serve_result(int(a)) for a in a_ids}
    g.serve_stop()
    # the same queries spread over a stream of others, submitted in small
    # groups while earlier groups are still running
    g2, _, _ = world(scn, 1200)
    g2.serve_start(max_in_flight=256)
    b_ids = np.arange(100, 1200, dtype=np.int32)
    b_tp = S.free_points(g2, scn, len(b_ids), np.random.default_rng(77))
    order = np.random.default_rng(78).permutation(len(a_ids) + len(b_ids))
    all_ids = np.concatenate([a_ids, b_ids])
    all_tp = np.concatenate([a_tp, b_tp])
    for k in range(0, len(order), 37):
        sel = order[k:k + 37]
        g2.serve_submit(all_ids[sel], all_tp[sel])
        g2.serve_poll()
    g2.serve_drain()
    st = g2.serve_stats()
    assert st["completed"] == len(all_ids) and st["launches"] >= 1
    for a in a_ids:
        f, L, p = g2.serve_result(int(a))
        fa, La, pa = alone[int(a)]
        assert (f, L) == (fa, La) and np.array_equal(p, pa), f"agent {a}: mixed result differs from alone"


def test_admission_waits_for_free_entries():
    scn = S.cfg2()
    g, starts, rng = world(scn, 800)
    g.serve_start(max_in_flight=16)
    ids = np.arange(800, dtype=np.int32)
    g.serve_submit(ids, S.free_points(g, scn, len(ids), rng))
    st = g.serve_stats()
    assert st["capacity"] == 16 and st["admitted"] <= 16 and st["waiting"] >= 800 - 16
    g.serve_drain()
    st = g.serve_stats()
    assert st["completed"] == 800 and st["waiting"] == 0
    assert st["latency_samples"] == 800 and 0 < st["latency_p50_ms"] <= st["latency_p99_ms"]


def test_newer_query_supersedes_older():
    scn = S.cfg2()
    g, starts, rng = world(scn, 50)
    g.serve_start()
    tp = S.free_points(g, scn, 2, rng)
    g.serve_submit([7], tp[:1])
    g.serve_submit([7], tp[1:])
    g.serve_drain()
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    d = g.debug_agents()
    assert d["targ_node"][7] == g.locate(tp[1:])[0]
    st = g.serve_stats()
    assert st["completed"] == 2 and st["applied"] + st["superseded"] == 2 and st["superseded"] >= 1


def test_serving_while_frames_run():
    # queries submitted between and during frames; every installed path is a
    # chain of neighbours that ends at the agent's target
    scn = S.cfg2()
    g, starts, rng = world(scn, 1000)
    g.serve_start()
    nb = g.map_nodes()["NeibsIdx"]
    for k in range(40):
        ids = np.nonzero(rng.random(1000) < 0.05)[0].astype(np.int32)
        if len(ids):
            g.serve_submit(ids, S.free_points(g, scn, len(ids), rng))
        g.AsyncStep(scn.dt)
        g.serve_poll()
        g.WaitStepEnd()
    g.serve_drain()
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    d = g.debug_agents()
    checked = 0
    for a in np.nonzero(d["path_len"] > 0)[0][:200]:
        p = g.path(int(a))
        assert p[-1] == d["targ_node"][a]
        for x, y in zip(p[:-1], p[1:]):
            assert y in nb[x]
        checked += 1
    assert checked > 50


def test_scene_batch_serving(oracle_mod):
    scns = S.cfg4(3, seed=12, agents_range=(60, 120))
    scenes = []
    for scn in scns:
        g = G.GMAPF()
        g.Init(G.make_config(scn.agents, scn.radius, scn.speed, scn.agents, 8, 32, 1.0))
        S.build_map(g, scn)
        for p in S.free_points(g, scn, scn.agents, np.random.default_rng(scn.seed)):
            g.AddAgent(p)
        scenes.append(g)
    b = G.SceneBatch(scenes)
    b.world.serve_start()
    subs = []
    for s, (scn, g) in enumerate(zip(scns, scenes)):
        ids = np.arange(0, g.agent_count, 3, dtype=np.int32)
        tp = S.free_points(g, scn, len(ids), np.random.default_rng(100 + s))
        g.serve_submit(ids, tp)  # scene-local ids
        subs.append((ids, tp))
    b.world.serve_drain()
    for s, (g, (ids, tp)) in enumerate(zip(scenes, subs)):
        ab, nb0 = b.scene_base(s)
        pos, _ = g.agents()
        res = []
        for a in ids:
            f, L, p = b.world.serve_result(int(a) + ab)
            res.append((f, L, p - nb0))
        oracle_check(oracle_mod, g, 8, 32, g.locate(pos[ids]), g.locate(tp), res)
    b.close()


def test_serving_configuration_scale(oracle_mod):
    # the serving configuration's size: 8 resident scenes of the 1000x1000,
    # 200-rectangle type with 8,192 agents each (one scene batch), 32,768
    # retargets submitted in one burst and drained; a sample of the results
    # against the oracle
    scns = [S.cfg2(seed=21 + k) for k in range(8)]
    scenes = []
    for scn in scns:
        g = G.GMAPF()
        g.Init(G.make_config(8192, scn.radius, scn.speed, 8192, 8, 32, scn.heuristic_k))
        S.build_map(g, scn)
        for p in S.free_points(g, scn, 8192, np.random.default_rng(scn.seed)):
            g.AddAgent(p)
        scenes.append(g)
    b = G.SceneBatch(scenes)
    b.world.serve_start()
    subs = []
    for s, (scn, g) in enumerate(zip(scns, scenes)):
        rng = np.random.default_rng(300 + s)
        ids = np.sort(rng.choice(8192, 4096, replace=False)).astype(np.int32)
        tp = S.free_points(g, scn, len(ids), rng)
        g.serve_submit(ids, tp)
        subs.append((ids, tp))
    b.world.serve_drain()
    st = b.world.serve_stats()
    assert st["completed"] == 8 * 4096 and st["in_flight"] == 0 and st["waiting"] == 0
    for s, (g, (ids, tp)) in enumerate(zip(scenes, subs)):
        ab, nb0 = b.scene_base(s)
        pos, _ = g.agents()
        pick = np.arange(0, len(ids), 64)
        res = []
        for k in pick:
            f, L, p = b.world.serve_result(int(ids[k]) + ab)
            res.append((f, L, p - nb0))
        oracle_check(oracle_mod, g, 8, 32, g.locate(pos[ids[pick]]), g.locate(tp[pick]), res)
    b.close()
