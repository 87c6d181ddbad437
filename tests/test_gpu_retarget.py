"""Large host retargets after start locate their points on the device
(gmapf_set_agent_targ_pos_bulk): the same triangles as the host rule, and the
same stop at the first invalid point as one call per item."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S

pytestmark = pytest.mark.gpu


def hard_points(g):
    """Triangle vertices, edge midpoints and centroids: points on shared edges
    and corners, where the first containing triangle in ascending id decides."""
    nd = g.map_nodes()
    v = [nd[k].astype(np.float32) for k in ("P1", "P2", "P3")]
    mids = [(v[0] + v[1]) / 2, (v[1] + v[2]) / 2, (v[2] + v[0]) / 2]
    cen = (v[0] + v[1] + v[2]) / 3
    return np.concatenate(v + mids + [cen]).astype(np.float32)


def test_device_located_targets_equal_the_host_rule():
    scn = S.cfg3(cells=24)
    A = 6000
    g, starts, rng = S.make_world(scn, agents=A)
    g.ManualStart()
    pts = np.concatenate([hard_points(g), S.free_points(g, scn, A, rng)])
    pts = pts[np.random.default_rng(5).permutation(len(pts))]
    want_all = g.locate(pts)  # host rule (grid, first containing triangle in ascending id)
    pts = pts[want_all >= 0][:A]
    assert len(pts) == A
    want = want_all[want_all >= 0][:A]
    g.set_targets(np.arange(A), pts)  # n >= 2048 after start: device point location
    st = np.array([int(g.GetAgentState(i)) for i in range(A)])
    assert np.all(st == int(G.EAgentState.Search))
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    d = g.debug_agents()
    assert np.array_equal(d["targ_node"], want)


def test_device_located_bulk_stops_at_the_first_invalid_point():
    scn = S.cfg2()
    g, starts, rng = S.make_world(scn, agents=5000)
    g.ManualStart()
    tp = S.free_points(g, scn, 5000, rng)
    tp[3000] = [-10.0, -10.0]
    with pytest.raises(G.GMAPFError) as e:
        g.set_targets(np.arange(5000), tp)
    assert e.value.status_name == "GMAPF_E_INVALID_POS"
    st = np.array([int(g.GetAgentState(i)) for i in range(5000)])
    assert np.all(st[:3000] == int(G.EAgentState.Search)) and np.all(st[3000:] == int(G.EAgentState.Idle))
    # the applied part steps like any retarget
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    d = g.debug_agents()
    assert np.array_equal(d["targ_node"][:3000], g.locate(tp[:3000]))


def test_bulk_retarget_while_a_step_runs():
    # the device point location has its own stream: it does not wait for the
    # running frame, and the targets apply at the next step
    scn = S.cfg2()
    g, starts, rng = S.make_world(scn, agents=4096)
    g.ManualStart()
    g.set_targets(np.arange(4096), S.free_points(g, scn, 4096, rng))
    g.AsyncStep(scn.dt)
    tp = S.free_points(g, scn, 4096, rng)
    g.set_targets(np.arange(4096), tp)
    g.WaitStepEnd()
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()
    d = g.debug_agents()
    assert np.array_equal(d["targ_node"], g.locate(tp))


def test_device_retarget_refuses_host_memory():
    scn = S.cfg2()
    g, starts, rng = S.make_world(scn, agents=64)
    g.ManualStart()
    ids = np.arange(64, dtype=np.int32)
    tp = S.free_points(g, scn, 64, rng).astype(np.float32)
    with pytest.raises(G.GMAPFError) as e:
        g.set_targets_device(ids.ctypes.data, tp.ctypes.data, 64)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    g.AsyncStep(scn.dt)  # nothing was applied; the context steps on
    g.WaitStepEnd()
    assert np.all(g.debug_agents()["state"] == int(G.EAgentState.Idle))
