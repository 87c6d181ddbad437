"""gmapf_search_batch_noalloc: the search entry point for callers that may not
allocate device memory (an engine owning every GPU allocation, memory fully
reserved).  Called through the C ABI twice in a row, it must give exactly
the results of the allocating entry point (gmapf_search_batch_device) and of
the CPU oracle on the same navmesh, queries, threads per agent and queue
capacity.  The buffers below are this test's own; the entry point allocates
nothing.  The other cases pin the rest of its contract: found = -1 for ids
outside the navmesh, rows longer than path_stride left untouched, found = -2
when a search reaches the round limit, pageable host memory refused.

This file sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S
from gpu_util import map_world, random_queries

pytestmark = pytest.mark.gpu

FILL = -7


def call_noalloc(lib, d_nodes, n, d_s, d_t, nq, T, Cap, f, l, p, stride, round_limit=0):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.gmapf_search_batch_noalloc(d_nodes, n, d_s, d_t, nq, T, Cap, C.c_float(1.0), round_limit, f, l, p,
                                        stride, C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc


def setup(cells, T, Cap, nq, seed=31):
    import torch
    scn = S.cfg3(cells=cells)
    g = map_world(scn, T=T, Cap=Cap)
    nodes = g.map_nodes()
    s, t = random_queries(g, scn, nq, seed=seed)
    dev = torch.device("cuda")
    d_nodes = torch.from_numpy(nodes.view(np.uint8).copy()).to(dev)
    return g, nodes, s, t, d_nodes


def outputs(nq, stride):
    import torch
    dev = torch.device("cuda")
    return (torch.full((nq,), FILL, dtype=torch.int32, device=dev),
            torch.full((nq,), FILL, dtype=torch.int32, device=dev),
            torch.full((nq, stride), FILL, dtype=torch.int32, device=dev))


def rows_equal(p_gpu, L, p_ref, stride):
    """Rows of paths that fit the stride are equal; longer rows stay untouched."""
    p_gpu = p_gpu.cpu().numpy()
    for i, n in enumerate(L):
        if n <= stride:
            if not np.array_equal(p_gpu[i, :n], p_ref[i, :n]):
                return False, i
        elif not np.all(p_gpu[i] == FILL):
            return False, i
    return True, -1


@pytest.mark.parametrize("cells,T,Cap,nq", [(64, 8, 32, 3000), (24, 32, 16, 1500), (24, 2, 4, 800),
                                            (24, 4, 16, 1000), (24, 16, 8, 1000)])
def test_noalloc_matches_allocating_entry_point_and_oracle(oracle_mod, cells, T, Cap, nq):
    import torch
    g, nodes, s, t, d_nodes = setup(cells, T, Cap, nq)
    n = len(nodes)
    s[:3] = t[:3]  # start == target: found, empty path
    stride = 4096 if cells <= 24 else 8192
    dev = torch.device("cuda")
    d_s = torch.from_numpy(s).to(dev)
    d_t = torch.from_numpy(t).to(dev)

    # allocating entry point (context-owned working memory)
    f0, l0, p0 = outputs(nq, stride)
    torch.cuda.synchronize()
    g.search_batch_device(d_s.data_ptr(), d_t.data_ptr(), nq, f0.data_ptr(), l0.data_ptr(), p0.data_ptr(), stride)
    # the oracle
    of, ol, op, _ = oracle_mod.OMap(nodes).search_batch(s, t, T, Cap, path_stride=stride)
    assert np.array_equal(f0.cpu().numpy(), of) and np.array_equal(l0.cpu().numpy(), ol)

    lib = G._lib.load()
    for call in range(2):  # two calls in a row share the built-in scratch array
        f1, l1, p1 = outputs(nq, stride)
        torch.cuda.synchronize()
        rc = call_noalloc(lib, d_nodes.data_ptr(), n, d_s.data_ptr(), d_t.data_ptr(), nq, T, Cap, f1.data_ptr(),
                          l1.data_ptr(), p1.data_ptr(), stride)
        assert rc == 0, lib.gmapf_last_error()
        assert torch.equal(f1, f0), f"found flags differ from the allocating entry point on call {call}"
        assert torch.equal(l1, l0), f"path lengths differ from the allocating entry point on call {call}"
        assert np.array_equal(f1.cpu().numpy(), of), f"found flags differ from the oracle on call {call}"
        assert np.array_equal(l1.cpu().numpy(), ol), f"path lengths differ from the oracle on call {call}"
        ok, i = rows_equal(p1, ol, op, stride)
        assert ok, f"path row {i} differs from the oracle on call {call}"
        L = l0.cpu().numpy()
        mask = torch.from_numpy(np.arange(stride)[None, :] < np.where(L <= stride, L, 0)[:, None]).to(dev)
        assert torch.equal(torch.where(mask, p1, -1), torch.where(mask, p0, -1)), f"paths differ on call {call}"
    assert int(f0[:3].sum()) == 3 and int(l0[:3].sum()) == 0


def test_noalloc_ids_outside_the_navmesh_and_short_rows(oracle_mod):
    """found = -1 (length 0) for an id outside the navmesh; a path longer than
    path_stride keeps its length and leaves its row untouched."""
    import torch
    T, Cap = 8, 32
    g, nodes, s, t, d_nodes = setup(24, T, Cap, 600, seed=5)
    n = len(nodes)
    s[0], t[1], s[2], t[3] = -1, n, n + 5, -3
    stride = 8
    of, ol, op, _ = oracle_mod.OMap(nodes).search_batch(np.clip(s, 0, n - 1), np.clip(t, 0, n - 1), T, Cap,
                                                        path_stride=n)
    dev = torch.device("cuda")
    d_s, d_t = torch.from_numpy(s).to(dev), torch.from_numpy(t).to(dev)
    f, l, p = outputs(len(s), stride)
    lib = G._lib.load()
    rc = call_noalloc(lib, d_nodes.data_ptr(), n, d_s.data_ptr(), d_t.data_ptr(), len(s), T, Cap, f.data_ptr(),
                      l.data_ptr(), p.data_ptr(), stride)
    assert rc == 0, lib.gmapf_last_error()
    fh, lh = f.cpu().numpy(), l.cpu().numpy()
    assert np.all(fh[:4] == -1) and np.all(lh[:4] == 0)
    assert np.array_equal(fh[4:], of[4:]) and np.array_equal(lh[4:], ol[4:])
    assert (lh > stride).sum() > 10, "the case needs paths longer than the stride"
    ok, i = rows_equal(p[4:], lh[4:], op[4:], stride)
    assert ok, f"row {i + 4}"
    assert np.all(p[:4].cpu().numpy() == FILL)


def test_noalloc_round_limit_reports_minus_two(oracle_mod):
    """A search still running after round_limit rounds ends with found = -2;
    searches that end sooner are exact, and the next call without a limit is
    exact for all (the shared scratch carries nothing over)."""
    import torch
    T, Cap = 8, 32
    g, nodes, s, t, d_nodes = setup(24, T, Cap, 400, seed=9)
    n = len(nodes)
    om = oracle_mod.OMap(nodes)
    rounds = np.array([om.search(a, b, T, Cap)[2]["rounds"] for a, b in zip(s, t)])
    of, ol, op, _ = om.search_batch(s, t, T, Cap, path_stride=n)
    limit = int(np.median(rounds))
    dev = torch.device("cuda")
    d_s, d_t = torch.from_numpy(s).to(dev), torch.from_numpy(t).to(dev)
    lib = G._lib.load()
    f, l, p = outputs(len(s), n)
    rc = call_noalloc(lib, d_nodes.data_ptr(), n, d_s.data_ptr(), d_t.data_ptr(), len(s), T, Cap, f.data_ptr(),
                      l.data_ptr(), p.data_ptr(), n, round_limit=limit)
    assert rc == 0, lib.gmapf_last_error()
    fh, lh = f.cpu().numpy(), l.cpu().numpy()
    ended = rounds <= limit  # a search that ends in its last allowed round is not cut
    assert np.all(fh[~ended] == -2) and np.all(lh[~ended] == 0) and (~ended).sum() > 0
    assert np.array_equal(fh[ended], of[ended]) and np.array_equal(lh[ended], ol[ended])
    f, l, p = outputs(len(s), n)
    rc = call_noalloc(lib, d_nodes.data_ptr(), n, d_s.data_ptr(), d_t.data_ptr(), len(s), T, Cap, f.data_ptr(),
                      l.data_ptr(), p.data_ptr(), n)
    assert rc == 0, lib.gmapf_last_error()
    assert np.array_equal(f.cpu().numpy(), of) and np.array_equal(l.cpu().numpy(), ol)
    ok, i = rows_equal(p, ol, op, n)
    assert ok, f"row {i}"


def test_noalloc_refuses_host_memory():
    """Pageable host buffers are refused before anything runs (a kernel given
    them would fault)."""
    import torch
    T, Cap = 8, 32
    g, nodes, s, t, d_nodes = setup(24, T, Cap, 16, seed=2)
    n = len(nodes)
    dev = torch.device("cuda")
    d_s, d_t = torch.from_numpy(s).to(dev), torch.from_numpy(t).to(dev)
    f, l, p = outputs(len(s), 64)
    host_out = np.zeros(len(s), np.int32)
    lib = G._lib.load()
    for args in [(nodes.ctypes.data, d_s.data_ptr(), f.data_ptr()),
                 (d_nodes.data_ptr(), s.ctypes.data, f.data_ptr()),
                 (d_nodes.data_ptr(), d_s.data_ptr(), host_out.ctypes.data)]:
        rc = call_noalloc(lib, args[0], n, args[1], d_t.data_ptr(), len(s), T, Cap, args[2], l.data_ptr(),
                          p.data_ptr(), 64)
        assert rc == 6, "pageable host memory must be refused (GMAPF_E_INVALID_ARG)"
        assert b"reach" in lib.gmapf_last_error()
    assert np.all(f.cpu().numpy() == FILL)  # nothing ran


def test_noalloc_rejects_oversized_and_bad_arguments():
    lib = G._lib.load()
    null = C.c_void_p(0)
    rc = lib.gmapf_search_batch_noalloc(null, 3_000_000, null, null, 1, 8, 32, C.c_float(1.0), 0, null, null, null,
                                        16, null)
    assert rc == 4  # GMAPF_E_CAPACITY
    assert b"64 MiB" in lib.gmapf_last_error()
    rc = lib.gmapf_search_batch_noalloc(null, 10, null, null, 1, 3, 32, C.c_float(1.0), 0, null, null, null, 16,
                                        null)
    assert rc == 6  # GMAPF_E_INVALID_ARG
    rc = lib.gmapf_search_batch_noalloc(null, 10, null, null, 1, 8, 32, C.c_float(1.0), -1, null, null, null, 16,
                                        null)
    assert rc == 6  # negative round limit
