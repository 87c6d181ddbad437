"""bench.py's roofline helpers (no GPU): the committed ncu tables are found
for the bench's shape, and the roofline objects carry consistent fractions."""
import importlib.util
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_and_instruction_tables_cover_the_bench_shape(bench):
    # the shape the autotuner picks for the 160x160-cell maze
    traffic, src = bench.measured_traffic(32, 16, 3, 363e6)  # a maze160 frame claims ~363 M nodes
    assert traffic is not None and (ROOT / src).exists()
    assert 5e9 < traffic < 40e9  # bytes per frame launch of 16,384 searches
    ipr, src = bench.measured_inst_per_round(32, 16, 3)
    assert ipr is not None and (ROOT / src).exists() and 100 < ipr < 1000
    # a shape with no capture reports none rather than a borrowed figure
    assert bench.measured_traffic(8, 32, 3, 1e6) == (None, None)
    assert bench.measured_inst_per_round(2, 8, 1) == (None, None)


def test_issue_roofline_arithmetic(bench):
    r = bench.issue_roofline(rounds=35_208_375, search_ms=30.0, ipr=358.2, src="x", sm_mhz=1965.0, sms=148)
    assert r["bound"] == "issue"
    assert r["peak"] == pytest.approx(4 * 148 * 1.965)
    assert r["achieved"] == pytest.approx(35_208_375 * 358.2 / 0.030 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert bench.issue_roofline(1, 1.0, None, None, 1965.0, 148) is None


def test_algorithmic_bytes_definition(bench):
    st = {"expansions": 10, "deg_sum": 20, "requests": 2, "path_nodes": 7}
    n = 400
    assert bench.algorithmic_bytes(st, n) == 12 * 10 + 24 * 20 + 2 * (n / 4 + 16) + 4 * 7


def test_mover_roofline_definition(bench):
    stats = [{"moving": 10, "ms_mover": 0.5, "neighbours": 1000},
             {"moving": 0, "ms_mover": 0.01, "neighbours": 0},  # nobody moved: not a mover frame
             {"moving": 12, "ms_mover": 0.5, "neighbours": 3000}]
    r = bench.mover_roofline(stats, 100, 6000.0, "measured")
    byt = 2 * 80.0 * 100 + 8.0 * 4000
    assert r["frames"] == 2
    assert r["achieved"] == pytest.approx(byt / 1e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6000.0)
    assert bench.mover_roofline([{"moving": 0, "ms_mover": 0.0, "neighbours": 0}], 10, 1.0, "x") is None


def test_attribution_parts(bench):
    wall = [10.0, 11.0, 30.0]
    parts = {"retarget": [1.0, 1.0, 2.0], "async_step": [0.1, 0.1, 0.1], "wait_step_end": [8.9, 9.9, 27.9],
             "device": [8.5, 9.5, 27.0]}
    a = bench.attribution(wall, parts)
    assert a["total"]["p99"] == 30.0 and a["device"]["p50"] == 9.5
    assert a["host_over_device"]["p99"] == pytest.approx(3.0)


def test_both_arms_share_the_headline_config(bench):
    class Args:
        cells, shape, threads_per_agent, queue_capacity = 160, "", 8, 32
    T, C = bench.headline_shape(Args)
    assert (T, C) == bench.TUNED_SHAPE[160]
    a = bench.workload_config(Args, 101698, 16384, T, C)
    assert a == bench.workload_config(Args, 101698, 16384, T, C)
    assert a["threads_per_agent"] == T and a["queue_capacity"] == C
    Args.shape = "8,32"
    assert bench.headline_shape(Args) == (8, 32)


def test_reference_arm_runs_without_the_product_library():
    """bench.py --impl reference times the oracle on the GPU arm's workload and
    shape; it never loads libgmapf_b200 (the navmesh and the point location
    come from the oracle)."""
    import json
    import subprocess
    import sys
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--cells', '24', '--agents', '256', "
            "'--ref-sample', '64', '--steps', '1', '--warmup', '3']; sys.path.insert(0, %r); import bench; "
            "bench.main(); maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'product': 'libgmapf_b200' in maps, 'oracle': 'liboracle' in maps}))" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    line, libs = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["threads_per_agent"] == 8 and line["config"]["queue_capacity"] == 32  # no tuned shape at 24
    assert libs == {"product": False, "oracle": True}


def test_oracle_navmesh_equals_fill_map_end(oracle_mod):
    """The oracle's own navmesh build (the reference's CDT call sequence) gives
    the library's FillMapEnd triangles and neighbour lists bit for bit."""
    import numpy as np
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S
    for scn in (S.cfg1(), S.cfg2(), S.cfg3(cells=24)):
        tri, nbr = oracle_mod.navmesh(scn.size, scn.obstacles)
        g = G.GMAPF()
        g.Init(G.make_config(4, 2, 1, 4, 8, 32))
        S.build_map(g, scn)
        t2, n2 = oracle_mod.nodes_to_arrays(g.map_nodes())
        assert np.array_equal(tri, t2) and np.array_equal(nbr, n2), scn.name
        pts = np.random.default_rng(3).uniform(0, scn.size[0], (2000, 2)).astype(np.float32)
        assert np.array_equal(oracle_mod.OMap(tri=tri, nbr=nbr).locate_batch(pts), g.locate(pts))


def test_search_side_counters(bench):
    d = bench.search_side_counters(32, 16, 3, rounds=35_000_000, search_ms=30.0)
    assert 100 < d["l2_gbs"] < 20000 and 0 < d["threads_per_warp_instruction"] <= 32
    assert bench.search_side_counters(2, 8, 1, 1, 1.0) == {}


def test_every_visited_placement_has_a_name(bench):
    # the bench line names the visited placement the library picked; every
    # placement gmapf_options.visited_mode accepts (1..4) has a name
    assert set(bench.VISITED) == {1, 2, 3, 4}
