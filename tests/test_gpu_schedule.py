"""The schedule changes only the path a traversal takes, never its results.

Forced decision plans and MLPs with arbitrary weights drive the direction of each BFS step and the width of
each SSSP bucket; levels and distances must stay bit-identical to the oracle.  Also checks the decision and
phase logs the trace collector relies on.
"""
import numpy as np
import pytest

import oracle as O
import pytrav as T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph():
    import torch

    assert torch.cuda.is_available()
    s, d, w = O.rmat(14, 16, seed=61)
    V = 1 << 14
    g = T.Graph.from_edges(V, s, d, w)
    src = int(np.bincount(s, minlength=V).argmax())
    csr = O.csr(V, s, d, w)
    want_lv = O.bfs_levels(V, s, d, src, csr_arrays=csr)
    want_d = O.dijkstra(V, s, d, w, src, csr_arrays=csr).view(np.uint32)
    return g, src, want_lv, want_d


def test_forced_bfs_plans_keep_levels(graph):
    g, src, want_lv, _ = graph
    rng = np.random.default_rng(0)
    for _ in range(12):
        plan = rng.integers(0, 2, 16).astype(np.uint8)
        g.set_plan(0, plan)
        assert np.array_equal(g.bfs([src])[0], want_lv), plan
        x, ch, ph, _, _ = g.last_decisions()
        n = len(ch)
        assert np.array_equal(ch, plan[:n]) and n == want_lv.max() + 1
        assert np.all(np.diff(ph) >= 1)  # each decision opens a later phase
    g.set_plan(0, None)


def test_forced_sssp_widths_keep_distances(graph):
    g, src, _, want_d = graph
    rng = np.random.default_rng(1)
    for _ in range(12):
        plan = rng.integers(0, 6, 64).astype(np.uint8)
        g.set_plan(1, plan)
        got = g.sssp([src], delta=0.05)[0]
        assert np.array_equal(got.view(np.uint32), want_d)
        x, ch, ph, lo, hi = g.last_decisions()
        assert np.array_equal(ch, plan[: len(ch)])
        assert np.all(hi > lo) and np.all(np.diff(lo) > 0)  # buckets advance
    g.set_plan(1, None)


def test_arbitrary_mlp_schedules_keep_results(graph):
    g, src, want_lv, want_d = graph
    for seed in range(4):
        rng = np.random.default_rng(seed)
        g.set_mlp(0, rng.normal(scale=2.0, size=T.mlp_param_count(0)))
        g.set_mlp(1, rng.normal(scale=2.0, size=T.mlp_param_count(1)))
        assert np.array_equal(g.bfs([src], schedule=T.SCHEDULE_LEARNED)[0], want_lv)
        got = g.sssp([src], delta=0.05, schedule=T.SCHEDULE_LEARNED)[0]
        assert np.array_equal(got.view(np.uint32), want_d)


def test_phase_log_is_consistent(graph):
    g, src, want_lv, _ = graph
    g.bfs([src])
    kind, size, end, edges = g.last_phase_log()
    dirs, frontier = g.last_bfs_trace()
    assert np.all(np.diff(end) >= 0) and np.all(np.diff(edges) >= 0)
    assert [k for k in kind if k in (0, 1)] == dirs.tolist()  # one top-down / bottom-up phase per step
    assert frontier.tolist() == [int((want_lv == i).sum()) for i in range(len(frontier))]


def test_grid_size_keeps_results(graph):
    g, src, want_lv, want_d = graph
    most, most_s = g.set_grid(0), g.set_grid(1)
    assert min(most, most_s) >= 148
    for ctas in (1, 3, 37, most // 2, most):
        g.set_grid(0, ctas)
        g.set_grid(1, min(ctas, most_s))
        assert np.array_equal(g.bfs([src])[0], want_lv), ctas
        got = g.sssp([src], delta=0.05)[0]
        assert np.array_equal(got.view(np.uint32), want_d), ctas
    with pytest.raises(T.TravError):
        g.set_grid(0, most + 1)
    g.set_grid(0, 0)
    g.set_grid(1, 0)


def test_cuda_graph_capture_replays_same_results(graph):
    import torch

    g, src, want_lv, want_d = graph
    srcs = [src, (src + 17) % g.V, (src + 101) % g.V]
    ref_lv = g.bfs(srcs)
    ref_d = g.sssp(srcs, delta=0.05)
    lv = torch.empty((len(srcs), g.V), dtype=torch.int32, device="cuda")
    di = torch.empty((len(srcs), g.V), dtype=torch.float32, device="cuda")
    g.set_capture(True)
    try:
        for delta in (0.05, 0.05, 0.2, 0.05):  # record, replay, record anew, record anew
            lv.fill_(7)
            di.fill_(7)
            g.bfs(srcs, out=lv)
            g.sssp(srcs, out=di, delta=delta)
            assert np.array_equal(lv.cpu().numpy(), ref_lv)
            if delta == 0.05:
                assert np.array_equal(di.cpu().numpy().view(np.uint32), ref_d.view(np.uint32))
            assert len(g.last_batch_ms()) == len(srcs)
        # an uncaptured call with another delta after a replay still counts its own light prefixes
        g.set_capture(False)
        assert np.array_equal(g.sssp([src], delta=0.3)[0].view(np.uint32), want_d)
        assert np.array_equal(g.sssp(srcs, delta=0.05).view(np.uint32), ref_d.view(np.uint32))
    finally:
        g.set_capture(False)
