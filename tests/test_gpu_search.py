"""Search parity: the CUDA search (through the C ABI) against the oracle, bit-exact
on found flags, path lengths, triangle sequences and search counters."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S
from gpu_util import map_world, random_queries

pytestmark = pytest.mark.gpu


def check_batch(oracle_mod, g, starts, targets, T, Cap, K=1.0):
    nodes = g.map_nodes()
    om = oracle_mod.OMap(nodes)
    stride = max(1, om.n)
    f, l, p, st = g.search_batch(starts, targets, stride)
    of, ol, op, ost = om.search_batch(starts, targets, T, Cap, K, path_stride=stride)
    assert np.array_equal(f, of), "found flags differ"
    assert np.array_equal(l, ol), "path lengths differ"
    for i in range(len(starts)):
        if f[i]:
            assert np.array_equal(p[i, :l[i]], op[i, :ol[i]]), f"path {i} differs"
    assert st["expansions"] == ost["expansions"]
    assert st["rounds"] == ost["rounds"]
    assert st["claims"] == ost["claims"]
    assert st["deg_sum"] == ost["deg_sum"]
    return f, l, p, st


@pytest.mark.parametrize("vm", [1, 2, 3, 4])
@pytest.mark.parametrize("T,Cap", [(2, 1), (2, 16), (4, 16), (8, 2), (32, 64)])
def test_cfg1_all_pairs(oracle_mod, T, Cap, vm):
    scn = S.cfg1()
    g = map_world(scn, T=T, Cap=Cap, visited_mode=vm)
    n = g.node_count
    s, t = np.meshgrid(np.arange(n), np.arange(n))
    f, l, p, st = check_batch(oracle_mod, g, s.ravel().astype(np.int32), t.ravel().astype(np.int32), T, Cap)
    assert f.mean() > 0.5


@pytest.mark.parametrize("vm", [1, 2, 3, 4])
@pytest.mark.parametrize("T,Cap", [(8, 32), (4, 16), (16, 8)])
def test_cfg2_random(oracle_mod, T, Cap, vm):
    scn = S.cfg2()
    g = map_world(scn, T=T, Cap=Cap, visited_mode=vm)
    s, t = random_queries(g, scn, 2048, seed=11)
    check_batch(oracle_mod, g, s, t, T, Cap)


@pytest.mark.parametrize("vm", [1, 2, 3, 4])
@pytest.mark.parametrize("T,Cap", [(8, 32), (32, 64), (2, 256), (16, 16)])
def test_maze64_random(oracle_mod, T, Cap, vm):
    scn = S.cfg3(cells=64)
    g = map_world(scn, T=T, Cap=Cap, visited_mode=vm)
    s, t = random_queries(g, scn, 512, seed=12)
    f, l, p, st = check_batch(oracle_mod, g, s, t, T, Cap)
    # path validity: consecutive triangles are neighbours and the path ends at the target
    nb = g.map_nodes()["NeibsIdx"]
    for i in range(len(s)):
        if f[i] and l[i] > 0:
            seq = [s[i]] + list(p[i, :l[i]])
            assert seq[-1] == t[i]
            for a, b in zip(seq[:-1], seq[1:]):
                assert b in nb[a]


@pytest.mark.parametrize("T,Cap", [(32, 16), (8, 32), (4, 16)])
def test_alone_search_moves_to_shared_memory(oracle_mod, T, Cap):
    # visited placement 4: a search still running once the other warps of its
    # block have left moves its queues and visited bitmap into the block's
    # shared memory and finishes there; batches of three queries leave most
    # searches alone in their blocks, so both kinds of rounds and the move
    # between them are compared with the oracle
    scn = S.cfg3(cells=64)
    g = map_world(scn, T=T, Cap=Cap, visited_mode=4, promote_rounds=1)
    s, t = random_queries(g, scn, 24, seed=41)
    moved = 0
    for k in range(0, 24, 3):
        moved += check_batch(oracle_mod, g, s[k:k + 3], t[k:k + 3], T, Cap)[3]["promoted"]
    assert moved > 0


@pytest.mark.parametrize("vm", [1, 2, 3, 4])
def test_plain_equals_batched(oracle_mod, vm):
    scn = S.cfg2()
    gb = map_world(scn, T=8, Cap=32, mode=G.MODE_BATCHED, visited_mode=vm)
    gp = map_world(scn, T=8, Cap=32, mode=G.MODE_PLAIN, visited_mode=vm % 3 + 1)
    s, t = random_queries(gb, scn, 1500, seed=13)
    fb, lb, pb, _ = gb.search_batch(s, t, gb.node_count)
    fp, lp, pp, _ = gp.search_batch(s, t, gp.node_count)
    assert np.array_equal(fb, fp) and np.array_equal(lb, lp) and np.array_equal(pb, pp)


def test_autotune_picks_a_shape_and_stays_exact(oracle_mod):
    scn = S.cfg3(cells=24)
    g = G.GMAPF()
    g.Init(G.make_config(4, scn.radius, scn.speed, 4, 8, 32, scn.heuristic_k))
    g.set_options(autotune=True)
    S.build_map(g, scn)
    g.ManualStart()
    sh = g.search_shape()
    assert sh["T"] in (2, 4, 8, 16, 32) and sh["C"] in (8, 16, 32, 64, 128, 256)
    assert sh["visited_mode"] in (1, 2, 3, 4) and sh["block_threads"] in (32, 64, 128, 256, 384, 512, 768)
    s, t = random_queries(g, scn, 1000, seed=17)
    check_batch(oracle_mod, g, s, t, sh["T"], sh["C"])


def test_autotune_keeps_fixed_options(oracle_mod):
    scn = S.cfg2()
    g = G.GMAPF()
    g.Init(G.make_config(4, scn.radius, scn.speed, 4, 8, 32, scn.heuristic_k))
    g.set_options(autotune=True, visited_mode=2, block_threads=64)
    S.build_map(g, scn)
    g.ManualStart()
    sh = g.search_shape()
    assert sh["visited_mode"] == 2 and sh["block_threads"] == 64
    s, t = random_queries(g, scn, 600, seed=18)
    check_batch(oracle_mod, g, s, t, sh["T"], sh["C"])


def test_autotune_cache_reuses_the_shape(oracle_mod, tmp_path):
    path = tmp_path / "tune.txt"

    def started(scn):
        g = G.GMAPF()
        g.Init(G.make_config(4, scn.radius, scn.speed, 4, 8, 32, scn.heuristic_k))
        g.set_options(autotune=True)
        g.set_tune_cache(path)
        S.build_map(g, scn)
        g.ManualStart()
        return g

    shape = lambda g: {k: v for k, v in g.search_shape().items() if k != "slots"}
    scn = S.cfg3(cells=24)
    g1 = started(scn)
    assert g1.tune_source() == 1
    assert len(path.read_text().splitlines()) == 1
    s, t = random_queries(g1, scn, 800, seed=21)
    r1 = g1.search_batch(s, t, g1.node_count)
    sh1 = shape(g1)
    g1.close()
    path.write_text("not a cache line\n" + path.read_text())  # foreign lines are skipped
    g2 = started(scn)
    assert g2.tune_source() == 2 and shape(g2) == sh1
    r2 = g2.search_batch(s, t, g2.node_count)
    assert all(np.array_equal(x, y) for x, y in zip(r1[:3], r2[:3]))
    check_batch(oracle_mod, g2, s, t, sh1["T"], sh1["C"])
    g2.close()
    g3 = started(S.cfg3(cells=24, seed=4))  # another map: tuned, a line of its own
    assert g3.tune_source() == 1
    assert len(path.read_text().splitlines()) == 3


def test_search_timeline():
    import torch
    scn = S.cfg3(cells=32)
    g = map_world(scn, T=8, Cap=16)
    s, t = random_queries(g, scn, 1000, seed=40)
    a = g.search_batch(s, t, g.node_count)
    buf = torch.zeros(2 * 1000, dtype=torch.int64, device="cuda")
    g.set_search_timeline(buf.data_ptr(), 1000)
    b = g.search_batch(s, t, g.node_count)  # recording changes no result
    assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))
    tl = buf.cpu().numpy().reshape(-1, 2)
    assert np.all(tl[:, 0] > 0) and np.all(tl[:, 1] >= tl[:, 0])
    s2, t2 = np.concatenate([s, s]), np.concatenate([t, t])
    with pytest.raises(G.GMAPFError) as e:  # more requests than the buffer holds
        g.search_batch(s2, t2, g.node_count)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    g.set_search_timeline(0, 0)
    g.search_batch(s2, t2, g.node_count)


def test_device_entry_points_refuse_host_memory():
    # pageable host buffers handed to the *_device entry points are refused
    # before any launch (GMAPF_E_INVALID_ARG), not read by a kernel
    scn = S.cfg2()
    g = map_world(scn, T=8, Cap=32)
    s, t = random_queries(g, scn, 64, seed=41)
    found, lens = np.zeros(64, np.int32), np.zeros(64, np.int32)
    paths = np.zeros((64, 8), np.int32)
    with pytest.raises(G.GMAPFError) as e:
        g.search_batch_device(s.ctypes.data, t.ctypes.data, 64, found.ctypes.data, lens.ctypes.data,
                              paths.ctypes.data, 8)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    tl = np.zeros(128, np.uint64)
    with pytest.raises(G.GMAPFError) as e:
        g.set_search_timeline(tl.ctypes.data, 64)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    f, ln, p, st = g.search_batch(s, t, g.node_count)  # the context is unharmed
    assert st["requests"] == 64


def test_longest_first_order_does_not_change_results(oracle_mod):
    scn = S.cfg3(cells=32)
    go = map_world(scn, T=8, Cap=16, order=True)
    gu = map_world(scn, T=8, Cap=16, order=False)
    s, t = random_queries(go, scn, 3000, seed=15)
    a = go.search_batch(s, t, go.node_count)
    b = gu.search_batch(s, t, gu.node_count)
    assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))
    assert a[3]["expansions"] == b[3]["expansions"]


@pytest.mark.parametrize("bt", [32, 64, 256])
def test_block_shape_does_not_change_results(oracle_mod, bt):
    scn = S.cfg2()
    g = map_world(scn, T=4, Cap=16, block_threads=bt)
    s, t = random_queries(g, scn, 700, seed=14)
    check_batch(oracle_mod, g, s, t, 4, 16)


@pytest.mark.parametrize("vm", [1, 2, 3, 4])
def test_edge_cases(oracle_mod, vm):
    scn = S.cfg1()
    g = map_world(scn, T=4, Cap=16, visited_mode=vm)
    n = g.node_count
    # empty batch
    f, l, p, st = g.search_batch(np.zeros(0, np.int32), np.zeros(0, np.int32), n)
    assert len(f) == 0
    # start == target: found, empty path
    f, l, p, st = g.search_batch(np.array([3], np.int32), np.array([3], np.int32), n)
    assert f[0] == 1 and l[0] == 0
    # out-of-range node ids are rejected on the host
    with pytest.raises(G.GMAPFError) as e:
        g.search_batch(np.array([n], np.int32), np.array([0], np.int32), n)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    # the same batch twice gives the same answer (slot epochs, no clearing)
    s = np.arange(n, dtype=np.int32)
    t = s[::-1].copy()
    a = g.search_batch(s, t, n)
    b = g.search_batch(s, t, n)
    assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))


@pytest.mark.parametrize("vm", [1, 2, 3, 4])
def test_disconnected_map_not_found(oracle_mod, vm):
    # two separate triangles: searches between them exhaust both queues
    g = G.GMAPF()
    g.Init(G.make_config(4, 1, 1, 4, 4, 16))
    g.set_options(visited_mode=vm, promote_rounds=1 if vm == 4 else 0)
    nodes = np.zeros(4, G.NODE_DTYPE)
    nodes["P1"] = [[0, 0], [1, 0], [10, 0], [11, 0]]
    nodes["P2"] = [[1, 0], [1, 1], [11, 0], [11, 1]]
    nodes["P3"] = [[0, 1], [0, 1], [10, 1], [10, 1]]
    nodes["NeibsIdx"] = [[1, -1, -1], [0, -1, -1], [3, -1, -1], [2, -1, -1]]
    g.FillMapManually(nodes)
    f, l, p, st = g.search_batch(np.array([0, 0, 2], np.int32), np.array([3, 1, 3], np.int32), 4)
    assert f.tolist() == [0, 1, 1]
    assert l.tolist() == [0, 1, 1]


def test_live_contexts_with_different_shapes(oracle_mod):
    # the kernel's shared-memory limit is shared by every context in the process:
    # a context started later for a smaller map must not break a larger one
    big_scn, small_scn = S.cfg3(cells=24), S.cfg1()
    big = map_world(big_scn, T=8, Cap=32, visited_mode=1)
    s1, t1 = random_queries(big, big_scn, 300, seed=31)
    check_batch(oracle_mod, big, s1, t1, 8, 32)
    small = map_world(small_scn, T=8, Cap=4, visited_mode=1)
    s2, t2 = random_queries(small, small_scn, 300, seed=32)
    check_batch(oracle_mod, small, s2, t2, 8, 4)
    check_batch(oracle_mod, big, s1, t1, 8, 32)
