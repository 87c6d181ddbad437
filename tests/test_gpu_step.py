"""Full per-frame step parity: AsyncStep/WaitStepEnd through the C ABI against
the oracle world; paths and states exact, positions within 1e-4 relative."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S
from gpu_util import close_rel

pytestmark = pytest.mark.gpu


def make_pair(oracle_mod, scn, agents, mode=G.MODE_BATCHED, T=None, Cap=None, P=None, vm=0, smoothing=False,
              promote_rounds=None):
    # visited placement 4: by default a search may move its bitmap into its
    # block's shared memory from its first round on
    if promote_rounds is None:
        promote_rounds = 1 if vm == 4 else 0
    g, starts, rng = S.make_world(scn, mode=mode, agents=agents, threads_per_agent=T, queue_capacity=Cap,
                                  parallel_agents=P, visited_mode=vm, path_smoothing=smoothing,
                                  promote_rounds=promote_rounds)
    om = oracle_mod.OMap(g.map_nodes())
    ow = oracle_mod.OWorld(om, agents, scn.radius, scn.speed, P or agents, T or scn.threads_per_agent,
                           Cap or scn.queue_capacity, scn.heuristic_k)
    ow.set_smoothing(smoothing)
    for p in starts:
        assert ow.add_agent(p[0], p[1]) >= 0
    return g, ow, rng


def retarget(g, ow, scn, ids, rng):
    tp = S.free_points(g, scn, len(ids), rng)
    g.set_targets(ids, tp)
    for i, p in zip(ids, tp):
        assert ow.set_target(int(i), p[0], p[1]) == 0


def compare(g, ow, step):
    d = g.debug_agents()
    o = ow.get()
    for k in ["state", "cur_node", "targ_node", "step_idx", "step_node", "path_len"]:
        assert np.array_equal(d[k], o[k]), f"{k} differs at step {step}"
    ok, mx = close_rel(d["pos"], o["pos"])
    assert ok, f"positions differ at step {step} (max abs diff {mx})"
    ok, mx = close_rel(d["step_pos"], o["step_pos"])
    assert ok, f"step targets differ at step {step}"
    return d


def run(g, ow, scn, steps, rng, retarget_every=0, check_every=10, threads=8):
    A = g.agent_count
    for k in range(steps):
        if retarget_every and k % retarget_every == 0:
            retarget(g, ow, scn, np.arange(A), rng)
        g.AsyncStep(scn.dt)
        g.WaitStepEnd()
        ow.step(scn.dt, threads)
        if (k + 1) % check_every == 0 or k == steps - 1:
            d = compare(g, ow, k)
    return d


def test_cfg1_200_steps(oracle_mod):
    scn = S.cfg1()
    g, ow, rng = make_pair(oracle_mod, scn, scn.agents)
    retarget(g, ow, scn, np.arange(scn.agents), rng)
    d = run(g, ow, scn, 200, rng)
    # paths identical for every agent that has one
    for i in range(scn.agents):
        if d["path_len"][i] > 0:
            assert np.array_equal(g.path(i), ow.path(i))
    # host mirror equals the device state after WaitStepEnd
    pos, st = g.agents()
    assert np.array_equal(st, d["state"])
    assert np.array_equal(pos, d["pos"], equal_nan=True)


@pytest.mark.parametrize("vm", [1, 2, 3, 4])
def test_cfg2_retargets(oracle_mod, vm):
    scn = S.cfg2()
    g, ow, rng = make_pair(oracle_mod, scn, 512, vm=vm)
    run(g, ow, scn, 250, rng, retarget_every=100, check_every=25)


@pytest.mark.parametrize("vm", [2, 3])
def test_cfg2_full_run(oracle_mod, vm):
    # the configuration as specified: 2,048 agents on the 1000x1000 map with
    # 200 rectangles, every agent retargeted every 100 steps, 1,000 steps
    scn = S.cfg2()
    g, ow, rng = make_pair(oracle_mod, scn, 2048, vm=vm)
    d = run(g, ow, scn, 1000, rng, retarget_every=100, check_every=50)
    for i in range(0, 2048, 97):
        if d["path_len"][i] > 0:
            assert np.array_equal(g.path(i), ow.path(i))


def test_plain_mode_step(oracle_mod):
    scn = S.cfg1()
    g, ow, rng = make_pair(oracle_mod, scn, 128, mode=G.MODE_PLAIN)
    retarget(g, ow, scn, np.arange(128), rng)
    run(g, ow, scn, 120, rng, check_every=30)


def test_request_capacity_defers(oracle_mod):
    # PathFinderParallelAgents below the number of searching agents: the rest
    # stay in Search for later frames (PathFinder.h:97-102)
    scn = S.cfg1()
    g, ow, rng = make_pair(oracle_mod, scn, 200, P=64)
    retarget(g, ow, scn, np.arange(200), rng)
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    ow.step(scn.dt)
    st = g.last_stats()
    assert st["requests"] == 64
    compare(g, ow, 0)
    run(g, ow, scn, 30, rng, check_every=5)


def test_zigzag_reference_driver(oracle_mod):
    # main.cpp TestFull layout: agents at (i/5, 0) heading to (i/5, 950)
    scn = S.zigzag()
    A = 1024
    g, ow, rng = make_pair(oracle_mod, scn, A, T=2, Cap=16)
    tp = np.array([[i / 5.0, 950.0] for i in range(A)], np.float32)
    g.set_targets(np.arange(A), tp)
    for i, p in enumerate(tp):
        ow.set_target(i, p[0], p[1])
    run(g, ow, scn, 60, rng, check_every=20)


@pytest.mark.parametrize("smoothing", [1, 2])
@pytest.mark.parametrize("mode", [G.MODE_BATCHED, G.MODE_PLAIN])
def test_path_smoothing_against_oracle(oracle_mod, mode, smoothing):
    # opt-in funnel corners instead of centroids: same triangle paths, agents
    # steer to the corners; device and oracle funnels agree exactly.  With
    # smoothing 2 the portals are narrowed by the agent radius at both ends.
    scn = S.cfg2()
    g, ow, rng = make_pair(oracle_mod, scn, 512, mode=mode, smoothing=smoothing)
    d = run(g, ow, scn, 250, rng, retarget_every=100, check_every=25)
    tri = g.map_nodes()
    moving = np.nonzero(d["state"] == G.EAgentState.Move)[0]
    assert len(moving) > 50
    # steering points of steps before the last (the last step steers to the target)
    inner = moving[d["step_idx"][moving] < d["path_len"][moving]]
    sp = np.asarray(d["step_pos"], np.float32)[inner]
    assert len(inner) > 20
    if smoothing == 1:
        # steering points lie on corridor vertices or at the target
        verts = {tuple(np.float32(v)) for t in tri for v in (t["P1"], t["P2"], t["P3"])}
        assert sum(tuple(p) in verts for p in sp) > 0
    else:
        # corners keep about one radius from every vertex (a portal narrower
        # than two radii gives its midpoint, at least as far from its ends)
        verts = np.unique(np.concatenate([tri["P1"], tri["P2"], tri["P3"]]).astype(np.float64), axis=0)
        dmin = np.sqrt(((sp[:, None, :].astype(np.float64) - verts[None]) ** 2).sum(-1)).min(1)
        assert (dmin >= 0.999 * scn.radius).mean() > 0.5
        assert (dmin > 0).all()  # none on a wall vertex


def test_path_smoothing_shortens_routes(oracle_mod):
    # agents that steer through funnel corners arrive no later than agents
    # that walk centroid to centroid (same targets, no other agents nearby)
    scn = S.cfg2()
    times = {}
    for smooth in (False, True):
        g, starts, rng = S.make_world(scn, agents=16, path_smoothing=smooth)
        tp = S.free_points(g, scn, 16, np.random.default_rng(41))
        g.set_targets(np.arange(16), tp)
        done = np.full(16, -1)
        for k in range(60 * 120):
            g.AsyncStep(1.0)
            g.WaitStepEnd()
            _, st = g.agents()
            newly = (st == G.EAgentState.Idle) & (done < 0) & (k > 0)
            done[newly] = k
            if (done >= 0).all():
                break
        times[smooth] = done
    assert (times[True] >= 0).all() and (times[False] >= 0).all()
    assert times[True].sum() <= times[False].sum()


def test_step_ready_tracks_the_running_step(oracle_mod):
    import time
    scn = S.cfg2()
    g, ow, rng = make_pair(oracle_mod, scn, 512)
    assert g.step_ready()  # nothing running
    retarget(g, ow, scn, np.arange(512), rng)
    g.AsyncStep(scn.dt)
    t_end = time.time() + 20
    while not g.step_ready():
        assert time.time() < t_end
    g.WaitStepEnd()
    assert g.step_ready()
    ow.step(scn.dt, 8)
    compare(g, ow, 0)


def test_collision_neighbour_counter(oracle_mod):
    """The step statistics count the agents read from the 3x3 grid cells by
    the collision pass (the mover's per-agent traffic in the bench's
    roofline): every agent reads at least its own cell's agents, itself
    included, when anybody moves; nothing is read when nobody moves."""
    scn = S.cfg2()
    A = 512
    g, ow, rng = make_pair(oracle_mod, scn, A)
    retarget(g, ow, scn, np.arange(A), rng)
    g.AsyncStep(scn.dt)  # searches: nobody is moving yet
    g.WaitStepEnd()
    st = g.last_stats()
    assert st["moving"] == 0 and st["neighbours"] == 0
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    st = g.last_stats()
    assert st["moving"] > 0
    assert A <= st["neighbours"] <= A * A


@pytest.mark.parametrize("speed,mode,smoothing", [(300.0, G.MODE_BATCHED, 0), (300.0, G.MODE_PLAIN, 0),
                                                  (60.0, G.MODE_BATCHED, 2)])
def test_fast_crowded_walks(oracle_mod, speed, mode, smoothing):
    # agents that cross several triangles per frame, snap onto shared
    # centroids and collide head on (coincident agents push by 0/0 = NaN, as
    # the reference's AgentsMover.h:108 does); a fifth retargeted every 10
    # frames; compared with the oracle world every frame for 100 frames
    import dataclasses
    scn = dataclasses.replace(S.cfg2(), speed=speed)
    A = 2048
    g, ow, rng = make_pair(oracle_mod, scn, A, mode=mode, smoothing=smoothing)
    retarget(g, ow, scn, np.arange(A), rng)
    for f in range(100):
        if f and f % 10 == 0:
            retarget(g, ow, scn, np.sort(rng.choice(A, A // 5, replace=False)), rng)
        g.AsyncStep(scn.dt)
        g.WaitStepEnd()
        ow.step(scn.dt, 8)
        compare(g, ow, f)
