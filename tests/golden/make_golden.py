"""Generates the golden fixtures that pin the oracle to the reference's own code.

Runs oracle/_ref/ref_harness (the reference's CuQueue, CuNodesMap and V2Float,
compiled for the host from the reference sources by oracle/ref/build_ref.sh)
on seeded inputs and stores inputs and outputs as JSON next to this script:

  ref_queue.json     bounded-queue push/pop sequences (CuQueue.h:33-70)
  ref_queue_ties.json  the same with many equal F keys (and distinct G and
                     ids): the reference orders equal F first-in first-out,
                     the oracle by (G, id); these cases record the
                     reference's own order where the two differ
  ref_geometry.json  centroids (src/GMAPF.cu:215), TryGetNodeIdx, IsInNode,
                     GetDistSqr (CuNodesMap.h) and GetRotated(10) (V2Float.h:39-47)
                     on the cfg1, zigzag and a cfg2-shaped navmesh

In ref_queue.json the queue keys are distinct, so the reference's FIFO order
for equal F and the oracle's (F, G, id) order cannot differ on them;
ref_queue_ties.json is where they can.  Needs the reference tree
(this script is run where it is mounted; the JSON files travel instead).
"""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"


def f32s(x):
    return [float(np.float32(v)) for v in x]


def run(inp: str) -> list[str]:
    r = subprocess.run([str(HARNESS)], input=inp, capture_output=True, text=True, check=True)
    return r.stdout.strip().splitlines()


def queue_cases(rng):
    cases = []
    for k in range(48):
        cap = int(rng.choice([1, 2, 3, 4, 5, 8, 16, 32]))
        nops = int(rng.integers(5, 120))
        pushes = int(nops * 0.7) + 1
        F = rng.permutation(np.linspace(0.5, 5000.0, pushes * 3).astype(np.float32))[:pushes]
        ids = rng.permutation(100000)[:pushes].astype(np.int32)
        ops, pi = [], 0
        for _ in range(nops):
            if pi < pushes and rng.random() < 0.65:
                ops.append(1)
                pi += 1
            else:
                ops.append(0)
        lines = [f"Q {cap} {len(ops)}"]
        j = 0
        for o in ops:
            if o == 1:
                lines.append(f"u {float(F[j]):.9g} {int(ids[j])}")
                j += 1
            else:
                lines.append("o")
        out = run("\n".join(lines) + "\n")[0]
        popped, final = out[1:].split("|")
        cases.append({"cap": cap, "ops": ops, "F": f32s(F[:j]), "ids": ids[:j].tolist(),
                      "popped": [int(v) for v in popped.split()], "final": [int(v) for v in final.split()]})
    return cases


def queue_tie_cases(rng):
    """F drawn from a handful of values, so most pushes tie with queued items;
    G and ids distinct.  The reference's Push ignores G (it compares F only)."""
    cases = []
    for k in range(40):
        cap = int(rng.choice([2, 3, 4, 6, 8, 16]))
        nops = int(rng.integers(10, 90))
        pushes = int(nops * 0.7) + 1
        F = rng.choice(np.float32([1.5, 2.0, 2.5, 7.0, 9.25])[:int(rng.integers(2, 6))], pushes).astype(np.float32)
        G = rng.permutation(1000)[:pushes].astype(np.int32)
        ids = rng.permutation(100000)[:pushes].astype(np.int32)
        ops, pi = [], 0
        for _ in range(nops):
            if pi < pushes and rng.random() < 0.65:
                ops.append(1)
                pi += 1
            else:
                ops.append(0)
        lines = [f"Q {cap} {len(ops)}"]
        j = 0
        for o in ops:
            if o == 1:
                lines.append(f"u {float(F[j]):.9g} {int(ids[j])}")
                j += 1
            else:
                lines.append("o")
        out = run("\n".join(lines) + "\n")[0]
        popped, final = out[1:].split("|")
        cases.append({"cap": cap, "ops": ops, "F": f32s(F[:j]), "G": G[:j].tolist(), "ids": ids[:j].tolist(),
                      "popped": [int(v) for v in popped.split()], "final": [int(v) for v in final.split()]})
    return cases


def geometry_case(name, nodes, rng):
    tri = np.concatenate([nodes["P1"], nodes["P2"], nodes["P3"]], 1).astype(np.float32)
    nbr = nodes["NeibsIdx"].astype(np.int32)
    n = len(tri)
    lines = [f"M {n}"] + [" ".join(f"{float(v):.9g}" for v in tri[i]) + " " + " ".join(str(int(v)) for v in nbr[i])
                          for i in range(n)]
    lines.append("C")
    lo, hi = tri.min(), tri.max()
    pts = list(rng.uniform(lo - 5, hi + 5, size=(300, 2)).astype(np.float32))
    verts = tri.reshape(-1, 2)
    pts += list(verts[rng.integers(0, len(verts), 60)])                       # vertices
    a = tri[:, 0:2]
    b = tri[:, 2:4]
    pts += list(((a + b) / np.float32(2))[rng.integers(0, n, 60)].astype(np.float32))  # edge midpoints
    pts = np.array(pts, np.float32)
    lines.append(f"P {len(pts)}")
    lines += [f"{float(p[0]):.9g} {float(p[1]):.9g}" for p in pts]
    qi = rng.integers(0, n, len(pts))
    lines.append(f"I {len(pts)}")
    lines += [f"{float(p[0]):.9g} {float(p[1]):.9g} {int(k)}" for p, k in zip(pts, qi)]
    pairs = rng.integers(0, n, size=(200, 2))
    lines.append(f"D {len(pairs)}")
    lines += [f"{int(x)} {int(y)}" for x, y in pairs]
    vecs = rng.normal(0, 3, size=(100, 2)).astype(np.float32)
    lines.append(f"R {len(vecs)}")
    lines += [f"{float(v[0]):.9g} {float(v[1]):.9g}" for v in vecs]
    out = run("\n".join(lines) + "\n")
    cen = [int(v, 16) for v in out[0].split()[1:]]
    loc = [int(v) for v in out[1].split()[1:]]
    inn = [int(v) for v in out[2].split()[1:]]
    dsq = [int(v, 16) for v in out[3].split()[1:]]
    rot = [int(v, 16) for v in out[4].split()[1:]]
    return {"name": name, "tri": tri.tolist(), "nbr": nbr.tolist(), "centroid_bits": cen,
            "points": pts.tolist(), "locate": loc, "in_node_q": qi.tolist(), "in_node": inn,
            "pairs": pairs.tolist(), "dist_sqr_bits": dsq, "vectors": vecs.tolist(), "rotated_bits": rot}


def main():
    if not HARNESS.exists():
        sys.exit(f"{HARNESS} missing: run oracle/ref/build_ref.sh first")
    from gmapf_b200 import scenarios as S
    from gmapf_b200 import GMAPF, make_config
    rng = np.random.default_rng(20261203)
    (HERE / "ref_queue.json").write_text(json.dumps({"cases": queue_cases(rng)}))
    # drawn from their own generator, so that the files above stay as they were
    (HERE / "ref_queue_ties.json").write_text(json.dumps({"cases": queue_tie_cases(np.random.default_rng(77))}))
    geo = []
    for scn in [S.cfg1(), S.zigzag(), S.cfg2()]:
        g = GMAPF()
        g.Init(make_config(4, 2.0, 1.0, 4, 4, 16))
        S.build_map(g, scn)
        nodes = g.map_nodes()
        if len(nodes) > 400:
            nodes = nodes[:400].copy()
            nb = nodes["NeibsIdx"]
            nb[nb >= 400] = -1
            # re-pack so that every list stays "valid entries first"
            for i in range(len(nb)):
                v = [x for x in nb[i] if x >= 0]
                nb[i] = v + [-1] * (3 - len(v))
        geo.append(geometry_case(scn.name, nodes, rng))
    (HERE / "ref_geometry.json").write_text(json.dumps({"maps": geo}))
    print("wrote", HERE / "ref_queue.json", HERE / "ref_geometry.json")


if __name__ == "__main__":
    main()
