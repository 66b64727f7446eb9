"""Failure paths, made to happen without faulting the GPU.

* A step budget that runs out, and a grid-barrier wait limit that runs out: the persistent kernel records the
  error on the device and returns, the host reports TRAV_ERR_TIMEOUT, and the handle still answers the next
  query correctly.  (The reference's only guard is the V-iteration cap of bellman_ford_wrapper,
  algorithm/sssp/gpu/bellman_ford.cu:126; its BFS loop has none, algorithm/bfs/gpu/bfs.cu:69.)
* An allocation failure, injected on the host in place of cudaMalloc's: TRAV_ERR_OOM, nothing leaked into the
  next call.
"""
import numpy as np
import pytest

import oracle as O
import pytrav as T
from pytrav import learn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grid():
    """A 128 x 128 grid: hundreds of BFS levels and SSSP rounds, so every limit is reached."""
    V, s, d, w = learn.grid_graph(128, seed=3)
    g = T.Graph.from_edges(V, s, d, w)
    yield g, V, s, d, w
    g.free()


def test_step_budget_runs_out_then_the_handle_still_works(grid):
    g, V, s, d, w = grid
    src = 0
    g.set_limits(max_steps=3)
    for call in (lambda: g.bfs([src]), lambda: g.sssp([src], delta=1.0), lambda: g.sssp([src], delta=0.0)):
        with pytest.raises(T.TravError) as e:
            call()
        assert e.value.code == T.TRAV_ERR_TIMEOUT and "step budget" in str(e.value)
    g.set_limits()
    assert np.array_equal(g.bfs([src])[0], O.bfs_levels(V, s, d, src))
    want = O.dijkstra(V, s, d, w, src).view(np.uint32)
    assert np.array_equal(g.sssp([src], delta=1.0)[0].view(np.uint32), want)


def test_grid_barrier_wait_limit_runs_out_then_the_handle_still_works(grid):
    g, V, s, d, w = grid
    src = 5
    g.set_limits(timeout_ns=1)  # any barrier wait at all exceeds 1 ns
    for call in (lambda: g.bfs([src]), lambda: g.sssp([src], delta=2.0)):
        with pytest.raises(T.TravError) as e:
            call()
        assert e.value.code == T.TRAV_ERR_TIMEOUT and "timed out" in str(e.value)
    g.set_limits()
    assert np.array_equal(g.bfs([src])[0], O.bfs_levels(V, s, d, src))
    want = O.dijkstra(V, s, d, w, src).view(np.uint32)
    assert np.array_equal(g.sssp([src], delta=2.0)[0].view(np.uint32), want)


@pytest.mark.parametrize("where,after", [("build", 0), ("build", 1), ("build", 5), ("build", 11), ("query", 0),
                                         ("batch", 0), ("batch", 2)])
def test_injected_allocation_failure_is_reported_as_oom(where, after):
    import torch

    s, d, w = O.rmat(10, 8, seed=2)
    V = 1 << 10
    src = int(s[0])
    want = O.bellman_ford(V, s, d, w, src).view(np.uint32)
    g = None if where == "build" else T.Graph.from_edges(V, s, d, w)
    out = torch.empty(V, dtype=torch.float32, device="cuda")
    T.inject_alloc_failure(after)
    try:
        with pytest.raises(T.TravError) as e:
            if where == "build":
                T.Graph.from_edges(V, s, d, w)
            elif where == "query":
                g.sssp([src, src, src], delta=0.1)  # three control blocks: the workspace grows
            else:
                b = T.Batch([g])
                b.run([(0, 1, src, 0.1, T.SCHEDULE_PLAIN, out)])
        assert e.value.code == T.TRAV_ERR_OOM, str(e.value)
    finally:
        T.inject_alloc_failure(-1)
    # nothing of the failed call is left behind: the graph builds and answers correctly
    g = g or T.Graph.from_edges(V, s, d, w)
    assert np.array_equal(g.sssp([src], delta=0.1)[0].view(np.uint32), want)
    b = T.Batch([g])
    b.run([(0, 1, src, 0.1, T.SCHEDULE_PLAIN, out)])
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
    b.close()
    g.free()
