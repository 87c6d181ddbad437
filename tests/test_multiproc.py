"""Multi-rank host logic on CPU (gloo, world size 2): the benchmark's
max-over-ranks timing and summed throughput, per-rank independent scenes
(weak scaling, no data-path collective), and the reference arm under
torchrun (rank 0 alone prints one line, the others exit 0)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import bench
    import numpy as np
    import oracle as O
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S

    dist = bench.init_dist(ws, rank, use_cuda=False)
    # each rank: its own scene (seed = 3 + rank), its own queries, no exchange
    scn = S.cfg3(cells=12, seed=3 + rank, agents=64, threads_per_agent=4, queue_capacity=16)
    g = G.GMAPF()
    g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    S.build_map(g, scn)
    om = O.OMap(g.map_nodes())
    rng = np.random.default_rng(rank)
    s = g.locate(S.free_points(g, scn, 64, rng))
    t = g.locate(S.free_points(g, scn, 64, rng))
    f, l, _, st = om.search_batch(s, t, 4, 16, threads=1, path_stride=0)
    local_ms = 10.0 * (rank + 1)
    bench.barrier(dist)
    mx = bench.reduce_max(dist, local_ms)
    tot = bench.reduce_sum(dist, float(len(s)))
    q.put((rank, mx, tot, int(f.sum()), g.node_count))
    dist.destroy_process_group()


def test_two_rank_reductions_and_independent_scenes():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=240)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, mx, tot, found, nodes in res:
        assert mx == 20.0       # max over ranks
        assert tot == 128.0     # queries summed over ranks
        assert found > 0
    assert res[0][4] != res[1][4] or res[0][3] != res[1][3]  # different scenes per rank


def test_reference_arm_under_torchrun():
    port = free_port()
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--cells", "12",
                        "--ref-sample", "64"], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
