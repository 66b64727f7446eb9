"""The allocation-free BFS entry point (trav_bfs_csr_noalloc) against the oracle and trav_bfs.

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


def _csr_on_device(torch, V, s, d):
    off, adj, _ = O.csr(V, s, d, np.zeros(len(s), np.float32))
    return off, adj, (torch.from_numpy(off.astype(np.int32)).cuda(), torch.from_numpy(adj[: len(s)].copy()).cuda())


def test_noalloc_bfs_matches_oracle_and_trav_bfs_on_two_calls_in_a_row():
    import torch

    s, d, w = O.rmat(14, 8, seed=77)
    V = 1 << 14
    off, adj, (off_t, adj_t) = _csr_on_device(torch, V, s, d)
    g = T.Graph.from_edges(V, s, d, w)
    out = torch.full((V,), 12345, dtype=torch.int32, device="cuda")
    hub = int(np.bincount(s, minlength=V).argmax())
    for src in (hub, 4097):  # two calls in a row share the static scratch
        T.bfs_csr_noalloc(off_t, adj_t, V, len(s), src, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got, O.bfs_levels(V, s, d, src, csr_arrays=(off, adj))), src  # bit-exact
        assert np.array_equal(got, g.bfs([src])[0]), src
    g.free()


def test_noalloc_bfs_at_its_size_limits_on_a_side_stream():
    """V = 262144 and E = 2^24, the largest graph the static scratch takes, run on a non-default stream."""
    import torch

    s, d, _ = O.rmat(18, 64, seed=5, drop_self_loops=False)
    V, E = 1 << 18, len(s)
    assert E == 1 << 24
    off, adj, (off_t, adj_t) = _csr_on_device(torch, V, s, d)
    out = torch.full((V,), 777, dtype=torch.int32, device="cuda")
    st = torch.cuda.Stream()
    hub = int(np.bincount(s, minlength=V).argmax())
    for src in (hub, int(s[12345])):
        with torch.cuda.stream(st):
            T.bfs_csr_noalloc(off_t, adj_t, V, E, src, out, stream=st)
        st.synchronize()
        assert np.array_equal(out.cpu().numpy(), O.bfs_levels(V, s, d, src, csr_arrays=(off, adj))), src


def test_noalloc_limits_bad_csr_and_host_pointers_are_rejected():
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
    # host memory is refused before anything is launched on it
    host_off = np.array([0, 1, 1, 1, 1, 1, 1, 1, 1], np.int32)
    with pytest.raises(T.TravError) as e:
        T.bfs_csr_noalloc(host_off, adj, V, 1, 0, out)
    assert e.value.code == T.TRAV_ERR_BAD_ARG and "device" in str(e.value)
    # the entry point still works after the rejected calls
    good_adj = torch.tensor([1, 2], dtype=torch.int32, device="cuda")
    off2 = torch.tensor([0, 1, 2, 2, 2, 2, 2, 2, 2], dtype=torch.int32, device="cuda")
    T.bfs_csr_noalloc(off2, good_adj, V, 2, 0, out)
    assert out.cpu().tolist() == [0, 1, 2, -1, -1, -1, -1, -1]
