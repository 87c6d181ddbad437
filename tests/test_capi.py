"""C ABI: the library loads, exports every declared entry point, and keeps the
reference's lifecycle and error rules (host-only checks, no GPU)."""
import re
from pathlib import Path

import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S

HDR = Path(__file__).resolve().parents[1] / "include" / "gmapf_c.h"


def declared_functions():
    txt = HDR.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gmapf_[a-z0-9_]+)\s*\(", txt)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    from gmapf_b200._lib import SIGNATURES
    assert set(SIGNATURES) == set(names)


def test_config_layout_matches_reference():
    import ctypes as C
    from gmapf_b200._lib import Config, Node
    assert C.sizeof(Config) == 32  # 7 x 4-byte fields + 2 bools, padded (Config.h)
    assert C.sizeof(Node) == 48    # CuNodesMap::Node, __align__(16)
    assert Node.NeibsIdx.offset == 32


def test_ctypes_mirrors_match_the_c_header(tmp_path):
    # every struct the Python binding passes through the C ABI has the C
    # header's size and field offsets (a C program built against
    # include/gmapf_c.h prints them)
    import ctypes as C
    import shutil
    import subprocess
    from gmapf_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = {"gmapf_config": _lib.Config, "gmapf_v2": _lib.V2, "gmapf_node": _lib.Node,
               "gmapf_options": _lib.Options, "gmapf_step_stats": _lib.StepStats,
               "gmapf_serve_stats": _lib.ServeStats}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "gmapf_c.h"', "int main(void) {"]
    for name, cls in mirrors.items():
        lines.append(f'printf("{name} sizeof %zu\\n", sizeof({name}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", str(HDR.parent), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for name, cls in mirrors.items():
        assert got[(name, "sizeof")] == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert got[(name, f)] == getattr(cls, f).offset, (name, f)


def test_lifecycle_rules():
    g = G.GMAPF()
    with pytest.raises(G.GMAPFError) as e:
        g.FillMapEnd()
    assert e.value.status_name == "GMAPF_E_STATE"
    with pytest.raises(G.GMAPFError):
        g.AddAgent((1, 1))
    g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    with pytest.raises(G.GMAPFError) as e:
        g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    assert "already initialized" in str(e.value)
    with pytest.raises(G.GMAPFError):
        g.AddAgent((1, 1))  # map not filled
    g.FillMapStart((100, 100))
    g.FillMapObstacle([(30, 40), (30, 60), (60, 60), (60, 40)])
    g.FillMapEnd()
    with pytest.raises(G.GMAPFError) as e:
        g.FillMapEnd()
    assert "already filled" in str(e.value)
    with pytest.raises(G.GMAPFError) as e:
        g.AddAgent((45, 50))  # inside the obstacle
    assert e.value.status_name == "GMAPF_E_INVALID_POS"
    ids = [g.AddAgent((5, 5 + i)) for i in range(4)]
    assert ids == [0, 1, 2, 3]
    with pytest.raises(G.GMAPFError) as e:
        g.AddAgent((5, 50))
    assert e.value.status_name == "GMAPF_E_CAPACITY"
    g.SetAgentTargetPos(1, (90, 90))
    assert g.GetAgentState(1) == G.EAgentState.Search
    assert g.GetAgentState(0) == G.EAgentState.Idle
    assert g.GetAgentPos(2) == (5.0, 7.0)
    with pytest.raises(G.GMAPFError):
        g.SetAgentTargPos(9, (1, 1))
    with pytest.raises(G.GMAPFError) as e:
        g.ProfilerDump()
    assert "profiler disabled" in str(e.value)
    g.WaitStepEnd()  # no step running: no-op (GMAPF.cu:293-294)
    g.close()


def test_bad_config_rejected():
    g = G.GMAPF()
    with pytest.raises(G.GMAPFError):
        g.Init(G.make_config(4, 2, 1, 4, 3, 16))  # T must be 2,4,8,16,32
    g2 = G.GMAPF()
    with pytest.raises(G.GMAPFError):
        g2.Init(G.make_config(4, 2, 1, 4, 4, 0))


def test_set_options_validates_ranges():
    g = G.GMAPF()
    g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    for bad in [dict(visited_mode=5), dict(visited_mode=-1), dict(block_threads=48), dict(block_threads=800),
                dict(mode=7), dict(round_limit=-1), dict(promote_rounds=-1)]:
        with pytest.raises(G.GMAPFError) as e:
            g.set_options(**bad)
        assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    for vm in (0, 1, 2, 3, 4):
        g.set_options(visited_mode=vm)
    g.set_options(visited_mode=4, block_threads=128, promote_rounds=100)
    assert g.options()["promote_rounds"] == 100
    g.set_options(round_limit=500)
    assert g.options()["round_limit"] == 500
    for sm in (0, 1, 2):
        g.set_options(path_smoothing=sm)
    with pytest.raises(G.GMAPFError) as e:
        g.set_options(path_smoothing=3)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"


def test_fill_map_manually_checks_neighbours():
    g = G.GMAPF()
    g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    nodes = np.zeros(2, G.NODE_DTYPE)
    nodes["P1"] = [[0, 0], [1, 0]]
    nodes["P2"] = [[1, 0], [1, 1]]
    nodes["P3"] = [[0, 1], [0, 1]]
    nodes["NeibsIdx"] = [[1, -1, -1], [5, -1, -1]]
    with pytest.raises(G.GMAPFError) as e:
        g.FillMapManually(nodes)
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    nodes["NeibsIdx"] = [[1, -1, -1], [0, -1, -1]]
    g.FillMapManually(nodes)
    out = g.map_nodes()
    assert np.allclose(out["PCenter"][0], [1 / 3, 1 / 3])  # recomputed on ingest (GMAPF.cu:215)


def test_host_locate_matches_oracle_linear_scan(oracle_mod):
    scn = S.cfg2()
    g = G.GMAPF()
    g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    S.build_map(g, scn)
    nodes = g.map_nodes()
    om = oracle_mod.OMap(nodes)
    rng = np.random.default_rng(5)
    pts = rng.uniform(-10, 1010, size=(3000, 2)).astype(np.float32)
    tri = np.concatenate([nodes["P1"], nodes["P2"], nodes["P3"]], 1).reshape(-1, 2)
    pts = np.concatenate([pts, tri[rng.integers(0, len(tri), 500)]]).astype(np.float32)
    got = g.locate(pts)
    want = np.array([om.locate(x, y, linear=True) for x, y in pts])
    assert np.array_equal(got, want)


def test_navmesh_sizes():
    # triangle counts of the seeded scenarios (CDT on the host)
    for scn, lo, hi in [(S.cfg1(), 10, 200), (S.cfg2(), 800, 4000), (S.zigzag(), 10, 200)]:
        g = G.GMAPF()
        g.Init(G.make_config(4, 2, 1, 4, 4, 16))
        S.build_map(g, scn)
        assert lo <= g.node_count <= hi, (scn.name, g.node_count)
        nodes = g.map_nodes()
        nb = nodes["NeibsIdx"]
        # neighbour lists are symmetric
        for i in range(len(nb)):
            for j in nb[i]:
                if j >= 0:
                    assert i in nb[j]


def test_tune_cache_is_set_before_the_start(tmp_path):
    scn = S.cfg1()
    g, starts, rng = S.make_world(scn, agents=4)
    g.set_tune_cache(tmp_path / "tune.txt")
    g.set_tune_cache(None)
    with pytest.raises(G.GMAPFError) as e:
        g.tune_source()
    assert e.value.status_name == "GMAPF_E_STATE"


def test_search_timeline_arguments():
    scn = S.cfg1()
    g, starts, rng = S.make_world(scn, agents=4)
    with pytest.raises(G.GMAPFError) as e:
        g.set_search_timeline(0x1000, 0)  # a buffer needs a positive row count
    assert e.value.status_name == "GMAPF_E_INVALID_ARG"
    g.set_search_timeline(0, 0)


def test_bulk_retarget_stops_at_the_first_invalid_point():
    # large bulks locate in parallel; the items before the first invalid one
    # are applied, the rest are not (as one call per item would do)
    scn = S.cfg2()
    g, starts, rng = S.make_world(scn, agents=5000)
    tp = S.free_points(g, scn, 5000, rng)
    tp[3000] = [-10.0, -10.0]
    with pytest.raises(G.GMAPFError) as e:
        g.set_targets(np.arange(5000), tp)
    assert e.value.status_name == "GMAPF_E_INVALID_POS"
    st = np.array([int(g.GetAgentState(i)) for i in range(5000)])
    assert np.all(st[:3000] == int(G.EAgentState.Search)) and np.all(st[3000:] == int(G.EAgentState.Idle))
