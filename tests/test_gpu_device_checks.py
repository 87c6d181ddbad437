"""Device-side checks made to fire on purpose, without faulting anything:
the round limit (gmapf_options.round_limit, the bound that stands in for a
wait limit in the search), a path longer than its output row, and the
serving drain timeout.  Each call reports its status through the C ABI and
the context stays usable: the next call or frame is clean.  Reference
behaviour for comparison: the reference stops a search when its queues run
dry (PathFinder.h:97-102, :268-274) and has no bound on its rounds."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S
from gpu_util import map_world, random_queries

pytestmark = pytest.mark.gpu


def oracle_rounds(oracle_mod, nodes, s, t, T, Cap):
    om = oracle_mod.OMap(nodes)
    r = np.array([om.search(a, b, T, Cap)[2]["rounds"] for a, b in zip(s, t)])
    f, l, p, _ = om.search_batch(s, t, T, Cap, path_stride=om.n)
    return r, f, l, p


def test_round_limit_in_a_batch_search(oracle_mod):
    T, Cap = 8, 32
    scn = S.cfg3(cells=24)
    g = map_world(scn, T=T, Cap=Cap)
    g2 = G.GMAPF()  # options are fixed at the start: the limit goes on a second context
    g2.Init(G.make_config(4, scn.radius, scn.speed, 4, T, Cap))
    s, t = random_queries(g, scn, 300, seed=3)
    r, of, ol, op = oracle_rounds(oracle_mod, g.map_nodes(), s, t, T, Cap)
    limit = int(np.median(r))
    g2.set_options(round_limit=limit)
    S.build_map(g2, scn)
    with pytest.raises(G.GMAPFError) as e:
        g2.search_batch(s, t, g2.node_count)
    assert e.value.status_name == "GMAPF_E_DEVICE" and "round limit" in str(e.value)
    # searches that end within the limit are exact; the context stays usable
    short = r <= limit
    f, l, p, _ = g2.search_batch(s[short], t[short], g2.node_count)
    assert np.array_equal(f, of[short]) and np.array_equal(l, ol[short])
    for i in range(int(short.sum())):
        assert np.array_equal(p[i, :l[i]], op[short][i, :l[i]])


def test_round_limit_in_a_step_then_a_clean_frame(oracle_mod):
    T, Cap = 8, 32
    scn = S.cfg3(cells=24)
    A = 128
    g, starts, rng = S.make_world(scn, agents=A, threads_per_agent=T, queue_capacity=Cap)
    nodes = g.map_nodes()
    tp = S.free_points(g, scn, A, rng)
    s, t = g.locate(starts).astype(np.int32), g.locate(tp).astype(np.int32)
    r, of, ol, op = oracle_rounds(oracle_mod, nodes, s, t, T, Cap)
    g.close()
    limit = int(np.median(r[s != t]))
    g, starts2, _ = S.make_world(scn, agents=A, threads_per_agent=T, queue_capacity=Cap)
    assert np.array_equal(starts2, starts)
    g.set_options(round_limit=limit)
    g.ManualStart()
    g.set_targets(np.arange(A), tp)
    g.AsyncStep(scn.dt)
    with pytest.raises(G.GMAPFError) as e:
        g.WaitStepEnd()
    assert e.value.status_name == "GMAPF_E_DEVICE" and "round limit" in str(e.value)
    d = g.debug_agents()
    cut = (r > limit) & (s != t)
    assert cut.sum() > 0
    assert np.all(d["state"][cut] == int(G.EAgentState.Idle)) and np.all(d["path_len"][cut] == 0)
    ok = ~cut & (s != t)
    assert np.array_equal(d["path_len"][ok], ol[ok])
    # the next frame has no new requests from the cut agents: it is clean
    g.AsyncStep(scn.dt)
    g.WaitStepEnd()


def test_path_longer_than_its_row(oracle_mod):
    import torch
    T, Cap = 8, 32
    scn = S.cfg3(cells=24)
    g = map_world(scn, T=T, Cap=Cap)
    s, t = random_queries(g, scn, 200, seed=4)
    om = oracle_mod.OMap(g.map_nodes())
    of, ol, op, _ = om.search_batch(s, t, T, Cap, path_stride=om.n)
    stride = 4
    assert (ol > stride).sum() > 0
    dev = torch.device("cuda")
    d_s, d_t = torch.from_numpy(s).to(dev), torch.from_numpy(t).to(dev)
    f = torch.full((len(s),), -7, dtype=torch.int32, device=dev)
    l = torch.full((len(s),), -7, dtype=torch.int32, device=dev)
    p = torch.full((len(s), stride), -7, dtype=torch.int32, device=dev)
    with pytest.raises(G.GMAPFError) as e:
        g.search_batch_device(d_s.data_ptr(), d_t.data_ptr(), len(s), f.data_ptr(), l.data_ptr(), p.data_ptr(),
                              stride)
    assert e.value.status_name == "GMAPF_E_DEVICE" and "did not fit" in str(e.value)
    assert np.array_equal(f.cpu().numpy(), of) and np.array_equal(l.cpu().numpy(), ol)
    ph = p.cpu().numpy()
    long_rows = ol > stride
    assert np.all(ph[long_rows] == -7)
    for i in np.nonzero(~long_rows)[0]:
        assert np.array_equal(ph[i, :ol[i]], op[i, :ol[i]])
    # a wide enough row: clean
    fw, lw, pw, _ = g.search_batch(s, t, g.node_count)
    assert np.array_equal(lw, ol)


def test_serve_drain_timeout_then_complete():
    scn = S.cfg3(cells=64)
    A = 4096
    g, starts, rng = S.make_world(scn, agents=A, threads_per_agent=8, queue_capacity=32)
    g.ManualStart()
    g.serve_start()
    g.serve_submit(np.arange(A, dtype=np.int32), S.free_points(g, scn, A, rng))
    with pytest.raises(G.GMAPFError) as e:
        g.serve_drain(timeout_s=-1.0)  # a deadline already past: the queries are still running
    assert e.value.status_name == "GMAPF_E_DEVICE_TIMEOUT"
    g.serve_drain(timeout_s=120.0)
    st = g.serve_stats()
    assert st["completed"] == A and st["in_flight"] == 0 and st["waiting"] == 0
