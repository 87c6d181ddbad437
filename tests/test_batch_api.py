"""Scene batches (gmapf_batch_*): binding rules and per-scene forwarding that
need no GPU (creation is host-side; the device work starts at the first step)."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S


def scene(scn, agents, T=8, Cap=32, K=1.0, P=None):
    g = G.GMAPF()
    g.Init(G.make_config(agents, scn.radius, scn.speed, P or agents, T, Cap, K))
    S.build_map(g, scn)
    rng = np.random.default_rng(scn.seed)
    pts = S.free_points(g, scn, agents, rng)
    for p in pts:
        g.AddAgent(p)
    return g, pts


def small_scenes(n=3, agents=20):
    return [scene(s, agents) for s in S.cfg4(n, seed=7)]


def status(e):
    return e.value.status_name


def test_bases_and_forwarded_getters():
    sc = small_scenes(3, 20)
    b = G.SceneBatch([g for g, _ in sc])
    base_a, base_n = 0, 0
    for k, (g, pts) in enumerate(sc):
        assert b.scene_base(k) == (base_a, base_n)
        base_a += g.agent_count
        base_n += g.node_count
        # positions and states come from the world's mirror, in scene ids
        assert np.allclose(g.GetAgentPos(3), pts[3])
        assert g.GetAgentState(3) == G.EAgentState.Idle
    assert b.world.agent_count == base_a and b.world.node_count == base_n
    # a target set on a scene shows up in that scene only
    g1, pts1 = sc[1]
    g1.SetAgentTargPos(2, pts1[5])
    assert g1.GetAgentState(2) == G.EAgentState.Search
    assert sc[0][0].GetAgentState(2) == G.EAgentState.Idle
    b.close()


def test_bound_scenes_refuse_map_agent_and_step_calls():
    sc = small_scenes(2, 8)
    b = G.SceneBatch([g for g, _ in sc])
    g, pts = sc[0]
    for call in [lambda: g.AddAgent(pts[0]), lambda: g.AsyncStep(0.1), lambda: g.ManualStart(),
                 lambda: g.set_options(visited_mode=2), lambda: g.FillMapEnd()]:
        with pytest.raises(G.GMAPFError) as e:
            call()
        assert status(e) == "GMAPF_E_STATE"
    # the world takes no agents and locates nothing itself
    with pytest.raises(G.GMAPFError) as e:
        b.world.AddAgent(pts[0])
    assert status(e) == "GMAPF_E_STATE"
    with pytest.raises(G.GMAPFError) as e:
        b.world.SetAgentTargPos(0, pts[0])
    assert status(e) == "GMAPF_E_STATE"
    # out-of-range scene ids stay out of range (not wrapped into a neighbour)
    with pytest.raises(G.GMAPFError) as e:
        g.SetAgentTargPos(g.agent_count, pts[0])
    assert status(e) == "GMAPF_E_INVALID_ARG"
    b.close()


def test_create_checks_scenes():
    (g0, _), (g1, _) = small_scenes(2, 8)
    with pytest.raises(G.GMAPFError) as e:
        G.SceneBatch([g0, g0])
    assert status(e) == "GMAPF_E_INVALID_ARG"
    other = scene(S.cfg4(1, seed=8)[0], 8, T=16)[0]
    with pytest.raises(G.GMAPFError) as e:
        G.SceneBatch([g0, other])
    assert status(e) == "GMAPF_E_INVALID_ARG"
    empty = G.GMAPF()
    empty.Init(G.make_config(4, 1, 1, 4, 8, 32))
    with pytest.raises(G.GMAPFError) as e:
        G.SceneBatch([g0, empty])
    assert status(e) == "GMAPF_E_STATE"
    b = G.SceneBatch([g0, g1])
    with pytest.raises(G.GMAPFError) as e:
        G.SceneBatch([g1])
    assert status(e) == "GMAPF_E_STATE"
    b.close()
    # after the batch is gone the scenes only answer E_STATE to agent calls
    with pytest.raises(G.GMAPFError) as e:
        g0.GetAgentPos(0)
    assert status(e) == "GMAPF_E_STATE"
    g0.close()
    g1.close()


def test_scene_destroyed_before_batch():
    sc = small_scenes(2, 8)
    b = G.SceneBatch([g for g, _ in sc])
    sc[0][0].close()
    assert sc[1][0].GetAgentState(0) == G.EAgentState.Idle
    b.close()
