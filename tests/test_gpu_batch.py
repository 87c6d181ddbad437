"""Scene batches on the GPU: every scene of a batch, stepped together with the
others (one compaction, one persistent search launch, one mover pass), against
that scene alone in the oracle world; paths and states exact, positions within
1e-4 relative."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S
from gpu_util import close_rel

pytestmark = pytest.mark.gpu


def build(oracle_mod, scns, P_div=1, T=8, Cap=32):
    scenes, worlds, pts = [], [], []
    for scn in scns:
        A = scn.agents
        P = max(1, A // P_div)
        g = G.GMAPF()
        g.Init(G.make_config(A, scn.radius, scn.speed, P, T, Cap, scn.heuristic_k))
        S.build_map(g, scn)
        rng = np.random.default_rng(scn.seed)
        start = S.free_points(g, scn, A, rng)
        ow = oracle_mod.OWorld(oracle_mod.OMap(g.map_nodes()), A, scn.radius, scn.speed, P, T, Cap, scn.heuristic_k)
        for p in start:
            g.AddAgent(p)
            assert ow.add_agent(p[0], p[1]) >= 0
        scenes.append(g)
        worlds.append(ow)
        pts.append(rng)
    return scenes, worlds, pts


def compare(g, ow, tag):
    d = g.debug_agents()
    o = ow.get()
    for k in ["state", "cur_node", "targ_node", "step_idx", "step_node", "path_len"]:
        assert np.array_equal(d[k], o[k]), f"{k} differs ({tag})"
    ok, mx = close_rel(d["pos"], o["pos"])
    assert ok, f"positions differ ({tag}, max abs diff {mx})"
    ok, mx = close_rel(d["step_pos"], o["step_pos"])
    assert ok, f"step targets differ ({tag})"
    return d


def run(scns, scenes, worlds, rngs, batch, steps, p_retarget=0.02, check_every=20, device_world=False):
    import torch
    for k in range(steps):
        dev_ids, dev_pos = [], []
        for s, (scn, g, ow, rng) in enumerate(zip(scns, scenes, worlds, rngs)):
            A = g.agent_count
            ids = np.arange(A) if k == 0 else np.nonzero(rng.random(A) < p_retarget)[0]
            if len(ids) == 0:
                continue
            tp = S.free_points(g, scn, len(ids), rng)
            if device_world:
                dev_ids.append(ids + batch.scene_base(s)[0])
                dev_pos.append(tp)
            else:
                g.set_targets(ids.astype(np.int32), tp)
            for i, p in zip(ids, tp):
                assert ow.set_target(int(i), p[0], p[1]) == 0
        if device_world and dev_ids:
            ids_t = torch.from_numpy(np.concatenate(dev_ids).astype(np.int32)).cuda()
            pos_t = torch.from_numpy(np.concatenate(dev_pos).astype(np.float32)).cuda()
            batch.world.set_targets_device(ids_t.data_ptr(), pos_t.data_ptr(), len(ids_t))
            torch.cuda.synchronize()
        batch.AsyncStep(scns[0].dt)
        batch.WaitStepEnd()
        for ow in worlds:
            ow.step(scns[0].dt, 8)
        if (k + 1) % check_every == 0 or k == steps - 1:
            for s, (g, ow) in enumerate(zip(scenes, worlds)):
                compare(g, ow, f"scene {s}, step {k}")


@pytest.mark.parametrize("vm", [0, 3, 4])
def test_batch_matches_scenes_alone(oracle_mod, vm):
    # visited placement 4: searches may move into shared memory from their first round on
    scns = S.cfg4(6, seed=9, agents_range=(40, 160))
    scenes, worlds, rngs = build(oracle_mod, scns)
    batch = G.SceneBatch(scenes, visited_mode=vm, promote_rounds=1 if vm == 4 else 0)
    run(scns, scenes, worlds, rngs, batch, 80)
    # paths, in each scene's own triangle ids
    for g, ow in zip(scenes, worlds):
        d = g.debug_agents()
        for i in np.nonzero(d["path_len"] > 0)[0][:40]:
            assert np.array_equal(g.path(int(i)), ow.path(int(i)))
    # host mirrors follow the device
    for g in scenes:
        pos, st = g.agents()
        assert np.array_equal(st, g.debug_agents()["state"])
    batch.close()


def test_cfg4_full_run(oracle_mod):
    # the configuration as specified: 64 scenes (sides 200..2000, 10..500
    # rectangles, 64..1024 agents of radius 1..3), retargets with probability
    # 0.02 per agent per step, 500 steps, one scene batch
    scns = S.cfg4()
    scenes, worlds, rngs = build(oracle_mod, scns)
    batch = G.SceneBatch(scenes)
    run(scns, scenes, worlds, rngs, batch, 500, check_every=50)
    batch.close()


def test_batch_per_scene_request_limits(oracle_mod):
    # PathFinderParallelAgents below the agent count: each scene defers its own overflow
    scns = S.cfg4(4, seed=10, agents_range=(60, 120))
    scenes, worlds, rngs = build(oracle_mod, scns, P_div=3)
    batch = G.SceneBatch(scenes)
    run(scns, scenes, worlds, rngs, batch, 40, check_every=5)
    batch.close()


def test_batch_device_retargets_and_plain_form(oracle_mod):
    scns = S.cfg4(4, seed=11, agents_range=(40, 100))
    scenes, worlds, rngs = build(oracle_mod, scns)
    batch = G.SceneBatch(scenes, mode=G.MODE_PLAIN)
    batch.ManualStart()
    run(scns, scenes, worlds, rngs, batch, 40, device_world=True)
    batch.close()
