"""The SCC forward-backward reachability sweep (forward_backward.cu's bfs(), :139-170) on the library's BFS
kernels, through the C ABI (trav_reach_el_masked), against the oracle's restatement of the reference's edge
sweeps (orc_reach_masked): forward and backward, several tree labelings, bit for bit."""
import numpy as np
import pytest

import oracle as O
import pytrav as T

pytestmark = pytest.mark.gpu


def _sweep(torch, V, s, d, pivot, trees):
    dev = torch.device("cuda")
    ts, td = torch.from_numpy(s).to(dev), torch.from_numpy(d).to(dev)
    tp = torch.tensor([pivot], dtype=torch.int32, device=dev)
    tt = torch.from_numpy(trees.astype(np.int32)).to(dev)
    vis = torch.full((V,), 9, dtype=torch.uint8, device=dev)
    T._check(T.lib().trav_reach_el_masked(ts.data_ptr(), td.data_ptr(), V, len(s), tp.data_ptr(), tt.data_ptr(),
                                          vis.data_ptr()))
    return vis.cpu().numpy()


@pytest.mark.parametrize("ntrees", [1, 2, 4, 64])
def test_masked_sweep_matches_the_reference_restatement(ntrees):
    import torch

    V = 1 << 12
    s, d, _ = O.rmat(12, 8, seed=21, drop_self_loops=False)
    rng = np.random.default_rng(ntrees)
    trees = rng.integers(0, ntrees, V).astype(np.int32)
    deg = np.bincount(s, minlength=V)
    for pivot in (int(deg.argmax()), int(np.flatnonzero(deg > 0)[17])):
        for a, b in ((s, d), (d, s)):  # the forward sweep, then the backward one on the reversed edges
            got = _sweep(torch, V, a, b, pivot, trees)
            assert np.array_equal(got, O.reach_masked(V, a, b, pivot, trees)), (ntrees, pivot)
    if ntrees == 1:  # one tree: plain reachability
        assert np.array_equal(got, (O.bfs_levels(V, d, s, pivot) >= 0).astype(np.uint8))


def test_masked_sweep_of_a_lone_tree_reaches_only_the_pivot():
    import torch

    V = 1 << 10
    s, d, _ = O.rmat(10, 8, seed=4, drop_self_loops=False)
    trees = np.zeros(V, np.int32)
    pivot = int(np.bincount(s, minlength=V).argmax())
    trees[pivot] = 7
    got = _sweep(torch, V, s, d, pivot, trees)
    assert got[pivot] == 1 and int(got.sum()) == 1
