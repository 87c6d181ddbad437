"""The oracle's emulation of the reference's own search orders (test and
analysis infrastructure, never what the kernels do): its queue key, F alone
with equal F first in first out (CuQueue.h:39-63), and the lanes of each
neighbour slot of a round taken in a random order, as the reference's
threads race inside each claim and frontier append (PathFinder.h:198-231).  Paths found under it
are valid paths of the method: chains of neighbours from the start to the
target, never shorter than the BFS optimum."""
import numpy as np
import pytest

from gmapf_b200 import scenarios as S


@pytest.fixture(scope="module")
def maze(oracle_mod):
    scn = S.cfg3(cells=24)
    tri, nbr = oracle_mod.navmesh(scn.size, scn.obstacles)
    om = oracle_mod.OMap(tri=tri, nbr=nbr)
    rng = np.random.default_rng(5)
    s = om.locate_batch(om.free_points(scn.size, 300, rng)).astype(np.int32)
    t = om.locate_batch(om.free_points(scn.size, 300, rng)).astype(np.int32)
    return om, nbr, s, t


@pytest.mark.parametrize("T,Cap", [(32, 16), (8, 32)])
def test_default_order_is_the_oracle(maze, T, Cap):
    om, _, s, t = maze
    a = om.search_batch(s, t, T, Cap)
    b = om.search_batch(s, t, T, Cap, order=(0, 0))
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert a[3] == b[3]


@pytest.mark.parametrize("T,Cap", [(32, 16), (8, 32)])
def test_reference_orders_give_valid_paths(maze, T, Cap):
    om, nbr, s, t = maze
    base = om.search_batch(s, t, T, Cap)
    changed = 0
    for order in [(1, 0), (1, 1), (1, 2), (0, 3)]:
        f, l, p, st = om.search_batch(s, t, T, Cap, order=order)
        for i in range(len(s)):
            if s[i] == t[i] or not f[i]:
                continue
            path = p[i, :l[i]]
            assert path[-1] == t[i]
            prev = s[i]
            for x in path:
                assert x in nbr[prev], (order, i)
                prev = x
            assert l[i] >= om.bfs_hops(s[i], t[i])
        changed += int(sum(not np.array_equal(p[i, :l[i]], base[2][i, :base[1][i]]) for i in range(len(s))))
    assert changed > 0  # the emulated orders do change paths
