"""Path cost against the optimum, for reporting search quality.

The search is bounded (queues of capacity C, first claim wins, nodes never
reopened), so its paths are not shortest.  Two references, both over the
navmesh's triangle graph:

  - hop count (the search's own cost G, PathFinder.h:210) against the BFS
    optimum;
  - centroid polyline length (the route agents walk, AgentsMover.h:143-175)
    against the FP64 Dijkstra optimum on centroid-distance edge weights.

Both optima come from scipy's compiled graph routines on a CSR matrix built
from the map's neighbour lists.
"""
from __future__ import annotations

import numpy as np


def graph(nodes: np.ndarray):
    """CSR adjacency (unweighted, and FP64 centroid-distance weighted) of the map."""
    from scipy.sparse import csr_matrix
    n = len(nodes)
    nb = nodes["NeibsIdx"].astype(np.int64)
    rows = np.repeat(np.arange(n), 3)
    cols = nb.ravel()
    ok = cols >= 0
    rows, cols = rows[ok], cols[ok]
    cen = nodes["PCenter"].astype(np.float64)
    w = np.sqrt(((cen[rows] - cen[cols]) ** 2).sum(1))
    w = np.maximum(w, 1e-300)  # csgraph treats explicit zeros as missing edges
    return csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n)), csr_matrix((w, (rows, cols)), shape=(n, n)), cen


def polyline_length(cen: np.ndarray, start: int, path: np.ndarray) -> float:
    """Centroid-to-centroid length of start followed by the path (start excluded
    from the path, target last, as the search writes it)."""
    seq = np.concatenate([[start], np.asarray(path, np.int64)])
    if len(seq) < 2:
        return 0.0
    d = cen[seq[1:]] - cen[seq[:-1]]
    return float(np.sqrt((d * d).sum(1)).sum())


def optima(nodes: np.ndarray, starts, targets):
    """(bfs_hops, dijkstra_len) per (start, target); -1 where unreachable."""
    from scipy.sparse.csgraph import dijkstra
    gu, gw, _ = graph(nodes)
    starts = np.asarray(starts, np.int64)
    targets = np.asarray(targets, np.int64)
    hops = np.full(len(starts), -1, np.int64)
    lens = np.full(len(starts), -1.0)
    uniq, inv = np.unique(starts, return_inverse=True)
    du = dijkstra(gu, directed=True, indices=uniq, unweighted=True)
    dw = dijkstra(gw, directed=True, indices=uniq)
    for i in range(len(starts)):
        h, l = du[inv[i], targets[i]], dw[inv[i], targets[i]]
        if np.isfinite(h):
            hops[i] = int(round(h))
            lens[i] = float(l)
    return hops, lens


def summary(nodes: np.ndarray, starts, targets, lens_found, paths) -> dict:
    """Ratios of found paths' hop counts and polyline lengths to the optima.

    lens_found: path length per query (0 for start == target); paths: list of
    int arrays (the path rows).  Queries whose start equals the target are
    skipped."""
    hops_opt, len_opt = optima(nodes, starts, targets)
    cen = nodes["PCenter"].astype(np.float64)
    hr, lr = [], []
    for s, L, p, ho, lo in zip(starts, lens_found, paths, hops_opt, len_opt):
        if L <= 0 or ho <= 0:
            continue
        hr.append(L / ho)
        lr.append(polyline_length(cen, int(s), p) / max(lo, 1e-12))
    hr, lr = np.asarray(hr), np.asarray(lr)
    if not len(hr):
        return {"queries": 0}

    def stats(v):
        return {"mean": float(v.mean()), "p50": float(np.percentile(v, 50)), "p95": float(np.percentile(v, 95)),
                "max": float(v.max())}

    return {"queries": int(len(hr)), "hops_over_bfs": stats(hr), "length_over_dijkstra_fp64": stats(lr)}
