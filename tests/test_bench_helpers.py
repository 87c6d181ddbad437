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
    traffic, src = bench.measured_traffic(160, 32, 16, 3, 16384)
    assert traffic is not None and (ROOT / src).exists()
    assert 10e9 < traffic < 40e9  # bytes per frame launch of 16,384 searches
    ipr, src = bench.measured_inst_per_round(160, 32, 16, 3)
    assert ipr is not None and (ROOT / src).exists() and 100 < ipr < 1000
    # a shape with no capture reports none rather than a borrowed figure
    assert bench.measured_traffic(160, 8, 32, 3, 16384) == (None, None)
    assert bench.measured_inst_per_round(64, 2, 8, 1) == (None, None)


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
