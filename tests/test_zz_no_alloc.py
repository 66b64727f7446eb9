"""The allocation-free BFS entry point (trav_bfs_csr_noalloc) agrees with trav_bfs.

Some callers cannot allocate device memory -- their device memory is owned by another allocator, or their
path cannot take the synchronisation of cudaMalloc -- so this entry point runs on a CSR they already hold and
takes its scratch from a static device array.  This file is collected last: a failure here leaves every
other test already run.  It passes alone in a fresh process and after the rest of the suite.
"""
import numpy as np
import pytest

import oracle as O
import pytrav as T

pytestmark = pytest.mark.gpu


def _csr_on_device(torch, V, s, d, w):
    off, adj, _ = O.csr(V, s, d, w)
    return (torch.from_numpy(off.astype(np.int32)).cuda(), torch.from_numpy(adj[: len(s)].copy()).cuda())


def test_noalloc_bfs_matches_trav_bfs_on_two_calls_in_a_row():
    import torch

    s, d, w = O.rmat(14, 8, seed=77)
    V = 1 << 14
    off_t, adj_t = _csr_on_device(torch, V, s, d, w)
    g = T.Graph.from_edges(V, s, d, w)
    out = torch.full((V,), 12345, dtype=torch.int32, device="cuda")
    hub = int(np.bincount(s, minlength=V).argmax())
    for src in (hub, 4097):  # two calls in a row share the static scratch
        T.bfs_csr_noalloc(off_t, adj_t, V, len(s), src, out)
        torch.cuda.synchronize()
        want = g.bfs([src])[0]
        assert np.array_equal(out.cpu().numpy(), want), src  # bit-exact, as every BFS test here


def test_noalloc_limits_and_bad_csr_are_rejected():
    import torch

    V = 8
    off = torch.tensor([0, 1, 2, 2, 2, 2, 2, 2, 2], dtype=torch.int32, device="cuda")
    adj = torch.tensor([1, 9], dtype=torch.int32, device="cuda")  # 9 is out of range
    out = torch.empty(V, dtype=torch.int32, device="cuda")
    with pytest.raises(T.TravError) as e:
        T.bfs_csr_noalloc(off, adj, V, 2, 0, out)
    assert e.value.code == T.TRAV_ERR_BAD_ARG
    with pytest.raises(T.TravError) as e:
        T.bfs_csr_noalloc(off, adj, (1 << 18) + 1, 2, 0, out)
    assert e.value.code == T.TRAV_ERR_BAD_ARG and "262144" in str(e.value)
