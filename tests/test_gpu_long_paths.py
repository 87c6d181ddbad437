"""Long paths against the oracle, element by element: a corridor of triangles
whose searches meet in the middle, with sides of 0 to ~2,500 hops, so that
the path walk crosses its 256-hop checkpoints on both sides (and stops one
hop before, at, and one hop after them).  Path layout as in the reference's
KernelBuildPath (PathFinder.h:253-307): the nodes after the start up to and
including the target."""
import numpy as np
import pytest

import gmapf_b200 as G

pytestmark = pytest.mark.gpu

N = 6000


def corridor(n):
    """A strip of n triangles between y=0 and y=1; triangle i touches i-1 and i+1."""
    nodes = np.zeros(n, G.NODE_DTYPE)
    for i in range(n):
        x = i // 2
        if i % 2 == 0:
            nodes["P1"][i], nodes["P2"][i], nodes["P3"][i] = (x, 0), (x + 1, 0), (x, 1)
        else:
            nodes["P1"][i], nodes["P2"][i], nodes["P3"][i] = (x + 1, 0), (x + 1, 1), (x, 1)
        nb = [j for j in (i - 1, i + 1) if 0 <= j < n]
        nodes["NeibsIdx"][i] = nb + [-1] * (3 - len(nb))
    return nodes


def queries():
    s, t = [], []
    # path lengths L = gS + gT + 1 around twice each checkpoint depth
    for L in (1, 2, 3, 4, 7, 12, 13, 510, 511, 512, 513, 514, 515, 516, 1022, 1023, 1024, 1025, 1026, 1027,
              1535, 1536, 1537, 4000, 5001, N - 1):
        a = 100 if L + 100 < N else 0
        s.append(a)
        t.append(a + L)
        s.append(a + L)  # the other direction
        t.append(a)
    rng = np.random.default_rng(11)
    for _ in range(40):
        a, b = rng.integers(0, N, 2)
        if a == b:
            continue
        s.append(int(a))
        t.append(int(b))
    return np.array(s, np.int32), np.array(t, np.int32)


@pytest.mark.parametrize("T,Cap", [(32, 16), (16, 16), (8, 32)])
@pytest.mark.parametrize("vm", [1, 2, 3, 4])
def test_long_corridor_paths(oracle_mod, T, Cap, vm):
    nodes = corridor(N)
    g = G.GMAPF()
    g.Init(G.make_config(4, 0.1, 1.0, 4, T, Cap))
    g.set_options(visited_mode=vm, promote_rounds=300 if vm == 4 else 0)  # 4: searches move after 300 rounds
    g.FillMapManually(nodes)
    g.ManualStart()
    s, t = queries()
    f, l, p, st = g.search_batch(s, t, N)
    om = oracle_mod.OMap(g.map_nodes())
    of, ol, op, ost = om.search_batch(s, t, T, Cap, path_stride=N)
    assert np.array_equal(f, of) and np.array_equal(l, ol)
    assert f.all()
    for i in range(len(s)):
        assert np.array_equal(p[i, :l[i]], op[i, :l[i]]), (i, s[i], t[i], l[i])
        # the corridor's path is the run of ids between the ends
        step = 1 if t[i] > s[i] else -1
        assert np.array_equal(p[i, :l[i]], np.arange(s[i] + step, t[i] + step, step))
    for k in ("expansions", "rounds", "claims", "deg_sum"):
        assert st[k] == ost[k], k
    g.close()
