"""Navmesh files: save/load round trip, the FillMapEnd cache keyed by the
FillMap* input, and rejection of damaged files (host only, no GPU)."""
import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S


def fresh():
    g = G.GMAPF()
    g.Init(G.make_config(4, 2, 1, 4, 8, 32))
    return g


def fill_input(g, scn):
    g.FillMapStart(scn.size)
    for o in scn.obstacles:
        g.FillMapObstacle(o)


def test_save_load_round_trip(tmp_path):
    scn = S.cfg2()
    a = fresh()
    S.build_map(a, scn)
    a.map_save(tmp_path / "m.nav")
    b = fresh()
    b.map_load(tmp_path / "m.nav")
    assert np.array_equal(a.map_nodes(), b.map_nodes())
    pts = np.random.default_rng(3).uniform(0, 1000, (500, 2)).astype(np.float32)
    assert np.array_equal(a.locate(pts), b.locate(pts))


def test_cached_fill_hits_only_for_the_same_input(tmp_path):
    scn = S.cfg2()
    path = tmp_path / "cache.nav"
    a = fresh()
    fill_input(a, scn)
    assert a.FillMapEndCached(path) is False  # built and written
    b = fresh()
    fill_input(b, scn)
    assert b.FillMapEndCached(path) is True  # loaded
    assert np.array_equal(a.map_nodes(), b.map_nodes())
    ref = fresh()
    S.build_map(ref, scn)
    assert np.array_equal(ref.map_nodes(), b.map_nodes())
    # another obstacle set: rebuilt, cache replaced
    c = fresh()
    fill_input(c, S.cfg2(seed=5))
    assert c.FillMapEndCached(path) is False
    d = fresh()
    fill_input(d, S.cfg2(seed=5))
    assert d.FillMapEndCached(path) is True


def test_damaged_files_are_rejected_or_rebuilt(tmp_path):
    scn = S.cfg1()
    a = fresh()
    S.build_map(a, scn)
    path = tmp_path / "m.nav"
    a.map_save(path)
    raw = bytearray(path.read_bytes())
    raw[-7] ^= 0x40  # flip a bit inside the records
    bad = tmp_path / "bad.nav"
    bad.write_bytes(bytes(raw))
    with pytest.raises(G.GMAPFError) as e:
        fresh().map_load(bad)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    (tmp_path / "short.nav").write_bytes(bytes(raw[:40]))
    with pytest.raises(G.GMAPFError):
        fresh().map_load(tmp_path / "short.nav")
    # the cached fill rebuilds over a damaged cache
    g = fresh()
    fill_input(g, scn)
    assert g.FillMapEndCached(bad) is False
    assert np.array_equal(g.map_nodes(), a.map_nodes())
    h = fresh()
    fill_input(h, scn)
    assert h.FillMapEndCached(bad) is True


def test_load_respects_lifecycle(tmp_path):
    a = fresh()
    S.build_map(a, S.cfg1())
    a.map_save(tmp_path / "m.nav")
    with pytest.raises(G.GMAPFError) as e:
        a.map_load(tmp_path / "m.nav")  # map already filled
    assert e.value.status_name == "GMAPF_E_STATE"
