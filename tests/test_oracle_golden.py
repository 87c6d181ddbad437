"""The oracle against the reference's own code (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref/ref_harness)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32).tolist()


@pytest.fixture(scope="module")
def queue_cases():
    return json.loads((GOLD / "ref_queue.json").read_text())["cases"]


@pytest.fixture(scope="module")
def geo_maps():
    return json.loads((GOLD / "ref_geometry.json").read_text())["maps"]


def test_queue_matches_reference_cuqueue(oracle_mod, queue_cases):
    assert len(queue_cases) >= 40
    for c in queue_cases:
        popped, final = oracle_mod.queue_sim(c["F"], np.zeros(len(c["F"])), c["ids"], c["ops"], c["cap"])
        assert popped.tolist() == c["popped"], c["cap"]
        assert final.tolist() == c["final"]


def test_centroids_match_reference(oracle_mod, geo_maps):
    for m in geo_maps:
        om = oracle_mod.OMap(tri=m["tri"], nbr=m["nbr"])
        assert sum(bits(om.centroids().reshape(-1)) != np.array(m["centroid_bits"])) == 0, m["name"]


def test_point_location_matches_reference(oracle_mod, geo_maps):
    for m in geo_maps:
        om = oracle_mod.OMap(tri=m["tri"], nbr=m["nbr"])
        for p, want in zip(m["points"], m["locate"]):
            assert om.locate(p[0], p[1], linear=True) == want
            assert om.locate(p[0], p[1]) == want  # grid-accelerated, same answer


def test_in_node_and_dist_match_reference(oracle_mod, geo_maps):
    for m in geo_maps:
        om = oracle_mod.OMap(tri=m["tri"], nbr=m["nbr"])
        lib = om.lib
        for p, q, want in zip(m["points"], m["in_node_q"], m["in_node"]):
            assert lib.orc_in_node(om.h, p[0], p[1], q) == want
        got = [lib.orc_dist_sqr(om.h, a, b) for a, b in m["pairs"]]
        assert bits(got) == m["dist_sqr_bits"]


def test_rotation_constants_match_reference(geo_maps):
    # V2Float::GetRotated(10) computes cos/sin of the float angle; the oracle
    # and the kernels use cos/sin of 10 degrees taken in double and rounded.
    cs = np.float32(math.cos(10 * math.pi / 180))
    sn = np.float32(math.sin(10 * math.pi / 180))
    for m in geo_maps:
        v = np.asarray(m["vectors"], np.float32)
        rx = v[:, 0] * cs - v[:, 1] * sn
        ry = v[:, 0] * sn + v[:, 1] * cs
        ref = np.asarray(m["rotated_bits"], np.uint32).view(np.float32).reshape(-1, 2)
        ulp = np.spacing(np.abs(ref).max(axis=1, keepdims=True).astype(np.float32))
        assert np.all(np.abs(np.stack([rx, ry], 1) - ref) <= 2 * ulp)
