"""gmapf_search_batch_noalloc: the search entry point for callers that may not
allocate device memory (an engine owning every GPU allocation, memory fully
reserved).  Called through the C ABI twice in a row, it must give exactly
the results of the allocating entry point (gmapf_search_batch_device) on the
same navmesh, queries, threads per agent and queue capacity.  The buffers
below are this test's own; the entry point allocates nothing.

This file sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

import gmapf_b200 as G
from gmapf_b200 import scenarios as S
from gpu_util import map_world, random_queries

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cells,T,Cap,nq", [(64, 8, 32, 3000), (24, 32, 16, 1500), (24, 2, 4, 800)])
def test_noalloc_matches_allocating_entry_point(cells, T, Cap, nq):
    import torch

    scn = S.cfg3(cells=cells)
    g = map_world(scn, T=T, Cap=Cap)
    nodes = g.map_nodes()
    n = len(nodes)
    s, t = random_queries(g, scn, nq, seed=31)
    s[:3] = t[:3]  # start == target: found, empty path
    stride = 4096 if cells <= 24 else 8192

    dev = torch.device("cuda")
    d_nodes = torch.from_numpy(nodes.view(np.uint8).copy()).to(dev)
    d_s = torch.from_numpy(s).to(dev)
    d_t = torch.from_numpy(t).to(dev)

    def outputs():
        return (torch.full((nq,), -7, dtype=torch.int32, device=dev),
                torch.full((nq,), -7, dtype=torch.int32, device=dev),
                torch.full((nq, stride), -1, dtype=torch.int32, device=dev))

    # allocating entry point (context-owned working memory)
    f0, l0, p0 = outputs()
    torch.cuda.synchronize()
    g.search_batch_device(d_s.data_ptr(), d_t.data_ptr(), nq, f0.data_ptr(), l0.data_ptr(), p0.data_ptr(), stride)

    lib = G._lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row share the built-in scratch array
        f1, l1, p1 = outputs()
        torch.cuda.synchronize()
        rc = lib.gmapf_search_batch_noalloc(d_nodes.data_ptr(), n, d_s.data_ptr(), d_t.data_ptr(), nq, T, Cap,
                                            C.c_float(1.0), f1.data_ptr(), l1.data_ptr(), p1.data_ptr(), stride,
                                            C.c_void_p(stream))
        assert rc == 0, lib.gmapf_last_error()
        torch.cuda.synchronize()
        assert torch.equal(f1, f0), f"found flags differ on call {call}"
        assert torch.equal(l1, l0), f"path lengths differ on call {call}"
        L = l0.cpu().numpy()
        ok = L <= stride
        mask = torch.from_numpy(np.arange(stride)[None, :] < np.where(ok, L, 0)[:, None]).to(dev)
        assert torch.equal(torch.where(mask, p1, -1), torch.where(mask, p0, -1)), f"paths differ on call {call}"
    assert int(f0[:3].sum()) == 3 and int(l0[:3].sum()) == 0


def test_noalloc_rejects_oversized_and_bad_arguments():
    lib = G._lib.load()
    null = C.c_void_p(0)
    rc = lib.gmapf_search_batch_noalloc(null, 3_000_000, null, null, 1, 8, 32, C.c_float(1.0), null, null, null,
                                        16, null)
    assert rc == 4  # GMAPF_E_CAPACITY
    assert b"64 MiB" in lib.gmapf_last_error()
    rc = lib.gmapf_search_batch_noalloc(null, 10, null, null, 1, 3, 32, C.c_float(1.0), null, null, null, 16, null)
    assert rc == 6  # GMAPF_E_INVALID_ARG
