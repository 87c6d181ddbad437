"""Path costs under the reference's own search orders, emulated on the CPU.

Analysis infrastructure beside the oracle (never imported by the library).
The reference's CUDA search cannot be run here (its claim race can feed a
stale record to KernelBuildPath, PathFinder.h:253-307, whose device asserts
and unbounded parent walk can trap or hang a shared GPU), and its order is
not one order: its queue breaks F ties first in first out (CuQueue.h:39-63)
and its threads race for claims, meets and frontier positions
(PathFinder.h:198-231).  This script runs the oracle's deterministic order
(the one the kernels follow, bit for bit) beside emulations of those orders
(orc_search_batch_order: the F-only first-in-first-out queue key, alone and
with the lanes of each neighbour slot of a round in seeded random orders) on
the same queries, and compares path costs: hops over the BFS optimum and centroid
polyline length over the FP64 Dijkstra optimum.

    python oracle/reference_order_paths.py [--cells 160] [--queries 2048] [--seeds 4]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from gmapf_b200 import scenarios as S  # noqa: E402


def costs(om, s, t, f, l, p, bfs, dij):
    """Per-query hops/BFS and length/Dijkstra of the found, non-trivial paths."""
    hops, length = [], []
    for i in range(len(s)):
        if not f[i] or s[i] == t[i] or bfs[i] <= 0:
            continue
        hops.append(l[i] / bfs[i])
        length.append(om.path_len(s[i], p[i, :l[i]]) / dij[i])
    return np.array(hops), np.array(length)


def summary(x):
    return {"mean": round(float(x.mean()), 4), "p50": round(float(np.median(x)), 4),
            "p95": round(float(np.quantile(x, 0.95)), 4), "max": round(float(x.max()), 4)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=160)
    ap.add_argument("--queries", type=int, default=2048)
    ap.add_argument("--seeds", type=int, default=4)
    ap.add_argument("--shapes", default="32x16,8x32")
    a = ap.parse_args()
    scn = S.cfg3(cells=a.cells)
    tri, nbr = O.navmesh(scn.size, scn.obstacles)
    om = O.OMap(tri=tri, nbr=nbr)
    rng = np.random.default_rng(7)
    s = om.locate_batch(om.free_points(scn.size, a.queries, rng)).astype(np.int32)
    t = om.locate_batch(om.free_points(scn.size, a.queries, rng)).astype(np.int32)
    t0 = time.time()
    bfs = np.array([om.bfs_hops(x, y) for x, y in zip(s, t)])
    dij = np.array([om.dijkstra_len(x, y) for x, y in zip(s, t)])
    out = {"map": f"maze {a.cells}x{a.cells} cells, {om.n} triangles", "queries": a.queries,
           "optima_s": round(time.time() - t0, 1), "shapes": {}}
    for shape in a.shapes.split(","):
        T, C = (int(v) for v in shape.split("x"))
        base = om.search_batch(s, t, T, C)
        bh, bl = costs(om, s, t, *base[:3], bfs, dij)
        res = {"deterministic (the kernels' order)": {"found": int(base[0].sum()), "hops_over_bfs": summary(bh),
                                                      "length_over_dijkstra": summary(bl),
                                                      "rounds": base[3]["rounds"]}}
        orders = [("first-in-first-out ties", (1, 0))] + [
            (f"first-in-first-out ties, racing lanes (seed {k})", (1, k)) for k in range(1, a.seeds + 1)]
        for name, order in orders:
            f, l, p, st = om.search_batch(s, t, T, C, order=order)
            h, ln = costs(om, s, t, f, l, p, bfs, dij)
            same = sum(bool(f[i] == base[0][i] and l[i] == base[1][i]
                            and np.array_equal(p[i, :l[i]], base[2][i, :l[i]])) for i in range(len(s)))
            res[name] = {"found": int(f.sum()), "hops_over_bfs": summary(h), "length_over_dijkstra": summary(ln),
                         "rounds": st["rounds"], "paths_equal_to_deterministic": round(same / len(s), 4)}
        out["shapes"][f"T={T}, C={C}"] = res
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
