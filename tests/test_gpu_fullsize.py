"""The bench frame's size and shape: the ~100k-triangle maze (160x160 cells,
101,698 triangles), 16,384 searches in one batch, 32 threads per agent and
queue capacity 16 (the shape the autotuner picks for this map), visited
bitmap in global memory (placement 3) or in global memory and then, for a
search still running at the batch's tail, in shared memory (placement 4, the default
pick).  Checked through properties that do not depend on
size: two runs agree bit for bit, a sample agrees with the oracle exactly,
paths are connected chains of neighbours that end at their targets, and no
path is shorter than the BFS optimum.  The per-frame step at the same size
(16,384 agents) is compared with the oracle world frame by frame."""
import os

import numpy as np
import pytest
import torch

from gmapf_b200 import path_quality as PQ
from gmapf_b200 import scenarios as S
from gpu_util import map_world, random_queries
from test_gpu_step import make_pair, retarget, run as run_steps

pytestmark = pytest.mark.gpu

T, CAP, N_QUERIES, STRIDE = 32, 16, 16384, 16384


def run(g, s, t):
    n = len(s)
    ds, dt = torch.from_numpy(s).cuda(), torch.from_numpy(t).cuda()
    f = torch.zeros(n, dtype=torch.int32, device="cuda")
    ln = torch.zeros(n, dtype=torch.int32, device="cuda")
    p = torch.full((n, STRIDE), -1, dtype=torch.int32, device="cuda")
    st = g.search_batch_device(ds.data_ptr(), dt.data_ptr(), n, f.data_ptr(), ln.data_ptr(), p.data_ptr(), STRIDE)
    torch.cuda.synchronize()
    return f, ln, p, st


@pytest.mark.parametrize("vm", [3, 4])
def test_full_frame_batch(oracle_mod, vm):
    # placement 4 at its default: searches may move from their 512th round on
    scn = S.cfg3(cells=160)
    g = map_world(scn, T=T, Cap=CAP, visited_mode=vm, promote_rounds=0)
    assert g.node_count > 100_000
    s, t = random_queries(g, scn, N_QUERIES, seed=31)
    f1, l1, p1, st1 = run(g, s, t)
    f2, l2, p2, st2 = run(g, s, t)
    assert torch.equal(f1, f2) and torch.equal(l1, l2) and torch.equal(p1, p2)
    assert st1["rounds"] == st2["rounds"] and st1["expansions"] == st2["expansions"]
    if vm == 4:
        assert st1["promoted"] > 0 and st2["promoted"] > 0  # the long searches moved
    f, ln = f1.cpu().numpy(), l1.cpu().numpy()
    assert f.sum() >= 0.99 * N_QUERIES  # the maze is connected; losses come only from bounded queues

    rng = np.random.default_rng(32)
    nodes = g.map_nodes()
    # exact parity with the oracle on a sample (a search's result depends only
    # on its own start and target, not on the rest of the batch)
    idx = np.sort(rng.choice(N_QUERIES, 256, replace=False))
    om = oracle_mod.OMap(nodes)
    of, ol, op, _ = om.search_batch(s[idx], t[idx], T, CAP, scn.heuristic_k, path_stride=STRIDE)
    sample = p1[torch.from_numpy(idx).cuda()].cpu().numpy()
    assert np.array_equal(f[idx], of) and np.array_equal(ln[idx], ol)
    for k in range(len(idx)):
        if of[k]:
            assert np.array_equal(sample[k, :ol[k]], op[k, :ol[k]]), f"query {idx[k]} differs from the oracle"

    # connected chains of neighbours ending at the target (start excluded)
    idx = np.sort(rng.choice(np.flatnonzero((f == 1) & (ln > 0)), 2048, replace=False))
    rows = p1[torch.from_numpy(idx).cuda()].cpu().numpy()
    nb = nodes["NeibsIdx"]
    for k, i in enumerate(idx):
        seq = np.concatenate([[s[i]], rows[k, :ln[i]]])
        assert seq[-1] == t[i]
        assert np.all((nb[seq[:-1]] == seq[1:, None]).any(axis=1)), f"query {i}: not a chain of neighbours"

    # never shorter than the BFS optimum
    idx = rng.choice(np.flatnonzero(f == 1), 128, replace=False)
    hops, _ = PQ.optima(nodes, s[idx], t[idx])
    assert np.all(ln[idx] >= hops)


@pytest.mark.parametrize("vm", [3, 4])
def test_full_frame_steps(oracle_mod, vm):
    # the step itself at this size: 16,384 agents all retargeted in one frame
    # (compaction, search, path rows), then two frames of movement and
    # collisions, each compared with the oracle world (states, nodes, path
    # steps exactly; positions within 1e-4 relative)
    scn = S.cfg3(cells=160)
    A = 16384
    g, ow, rng = make_pair(oracle_mod, scn, A, T=T, Cap=CAP, vm=vm, promote_rounds=0)
    retarget(g, ow, scn, np.arange(A), rng)
    d = run_steps(g, ow, scn, 3, rng, check_every=1, threads=os.cpu_count() or 8)
    assert (d["path_len"] > 0).sum() >= 0.99 * A
    for i in range(0, A, 509):
        if d["path_len"][i] > 0:
            assert np.array_equal(g.path(i), ow.path(i))


def test_full_frames_walking_with_partial_retargets(oracle_mod):
    # 16,384 agents on the maze over 40 frames: a full retarget, then every 8
    # frames 2,048 random agents get new targets while the others walk their
    # long paths through each other (speed 300, so that agents cross several
    # triangles and meet); compared with the oracle world every 4 frames
    # (states, nodes, path steps exactly; positions within 1e-4 relative)
    import dataclasses
    scn = dataclasses.replace(S.cfg3(cells=160), speed=300.0)
    A = 16384
    g, ow, rng = make_pair(oracle_mod, scn, A, T=T, Cap=CAP, vm=3)
    retarget(g, ow, scn, np.arange(A), rng)
    threads = os.cpu_count() or 8
    for block in range(5):
        if block:
            retarget(g, ow, scn, np.sort(rng.choice(A, 2048, replace=False)), rng)
        d = run_steps(g, ow, scn, 8, rng, check_every=4, threads=threads)
    moving = d["state"] == 2
    assert moving.sum() > 0.5 * A
    assert (d["step_idx"][moving] > 3).sum() > 0.5 * moving.sum()  # the walkers went through several triangles
