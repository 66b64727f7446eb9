"""Batched queries: many BFS / SSSP queries over graphs of uneven sizes in one persistent launch.

Every result of a batch must equal the oracle's (levels, and fp32 distances bit for bit), whatever the launch
shape the batch runs with; the autotuner may only pick among shapes that all give those results.
"""
import numpy as np
import pytest

import oracle as O
import pytrav as T

pytestmark = pytest.mark.gpu

# (scale, edge factor, seed): uneven sizes, like the batched workload's RMAT mix
GRAPHS = [(8, 8, 3), (12, 16, 4), (10, 32, 5), (13, 8, 6), (9, 24, 7)]


@pytest.fixture(scope="module")
def batch_case():
    import torch

    assert torch.cuda.is_available()
    graphs, want = [], []
    queries = []
    rng = np.random.default_rng(11)
    for gi, (scale, ef, seed) in enumerate(GRAPHS):
        s, d, w = O.rmat(scale, ef, seed=seed)
        V = 1 << scale
        g = T.Graph.from_edges(V, s, d, w)
        graphs.append(g)
        csr = O.csr(V, s, d, w)
        deg = np.bincount(s, minlength=V)
        srcs = rng.choice(np.flatnonzero(deg > 0), 4, replace=False)
        for k, src in enumerate(srcs):
            kind = k % 2
            delta = [0.1, 0.0][(k // 2) % 2] if kind == 1 else 0.0
            if kind == 0:
                ref = O.bfs_levels(V, s, d, int(src), csr_arrays=csr)
                out = torch.empty(V, dtype=torch.int32, device="cuda")
            else:
                ref = O.dijkstra(V, s, d, w, int(src), csr_arrays=csr)
                out = torch.empty(V, dtype=torch.float32, device="cuda")
            queries.append((gi, kind, int(src), delta, T.SCHEDULE_PLAIN, out))
            want.append(ref)
    return graphs, queries, want


def _check(queries, want):
    for (gi, kind, src, delta, _, out), ref in zip(queries, want):
        got = out.cpu().numpy()
        if kind == 0:
            assert np.array_equal(got, ref), (gi, src)
        else:
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (gi, src, delta)


def _clear(queries):
    for q in queries:
        q[5].fill_(7)


def test_batch_matches_oracle(batch_case):
    graphs, queries, want = batch_case
    b = T.Batch(graphs)
    _clear(queries)
    ms = b.run(queries)
    assert ms > 0
    _check(queries, want)
    b.close()


@pytest.mark.parametrize("shape", [(1, 32, 256), (3, 8, 64), (37, 64, 1024), (16, 0, 128), (5, 1024, 8192)])
def test_batch_shapes_keep_results(batch_case, shape):
    graphs, queries, want = batch_case
    b = T.Batch(graphs)
    b.shape = shape
    assert b.shape == shape
    _clear(queries)
    b.run(queries)
    _check(queries, want)
    b.close()


def test_batch_whole_grid_team_and_repeat(batch_case):
    graphs, queries, want = batch_case
    b = T.Batch(graphs)
    most = graphs[0].set_grid(1)  # the batch kernel has the SSSP kernel's occupancy
    b.shape = (most, 32, 256)
    for _ in range(2):
        _clear(queries)
        b.run(queries)
        _check(queries, want)
    b.close()


def test_batch_autotune_picks_a_valid_shape(batch_case):
    graphs, queries, want = batch_case
    b = T.Batch(graphs)
    best = b.autotune(queries, reps=1)
    assert b.shape == best
    assert best[0] >= 1 and 0 <= best[1] <= 1024 and 64 <= best[2] <= 8192
    _clear(queries)
    b.run(queries)
    _check(queries, want)
    b.close()
    # the tuned shape went into the table: a new batch of the same kind takes it without timing
    b2 = T.Batch(graphs)
    b2.shape = (1, 8, 1024)
    assert b2.autotune(queries, reps=0) == best
    b2.close()


def test_batch_equals_single_query_api(batch_case):
    graphs, queries, _ = batch_case
    b = T.Batch(graphs)
    _clear(queries)
    b.run(queries)
    for gi, kind, src, delta, _, out in queries:
        g = graphs[gi]
        single = g.bfs([src])[0] if kind == 0 else g.sssp([src], delta=delta)[0]
        assert np.array_equal(out.cpu().numpy().view(np.uint32), single.view(np.uint32))
    b.close()


def test_batch_errors(batch_case):
    import torch

    graphs, queries, _ = batch_case
    b = T.Batch(graphs)
    out = torch.empty(graphs[0].V, dtype=torch.int32, device="cuda")
    with pytest.raises(T.TravError):
        b.run([(len(graphs), 0, 0, 0.0, T.SCHEDULE_PLAIN, out)])
    with pytest.raises(T.TravError):
        b.run([(0, 0, graphs[0].V, 0.0, T.SCHEDULE_PLAIN, out)])
    with pytest.raises(T.TravError):
        b.run([(0, 2, 0, 0.0, T.SCHEDULE_PLAIN, out)])
    with pytest.raises(T.TravError):
        b.run([(0, 0, 0, 0.0, T.SCHEDULE_LEARNED, out)])  # no network installed
    with pytest.raises(T.TravError):
        b.shape = (0, 32, 256)
    with pytest.raises(T.TravError):
        b.shape = (4, 32, 32)
    assert b.run([]) == 0.0
    b.close()


@pytest.mark.parametrize("parts", [1, 3, 4])
def test_host_output_batch_equals_device_output_batch(parts):
    """trav_batch_run_host (host output arrays; per-query copies started by the kernel's completion flags while
    the launch runs; one or several launches) gives the results of trav_batch_run, and the oracle's."""
    import torch

    s, d, w = O.rmat(12, 16, seed=31)
    V = 1 << 12
    g = T.Graph.from_edges(V, s, d, w)
    deg = np.bincount(s, minlength=V)
    srcs = [int(x) for x in np.flatnonzero(deg > 0)[[0, 5, 77, 301, 902]]]
    dev_q, host_q, host_out = [], [], []
    for src in srcs:
        for kind in (1, 0):
            dt = torch.float32 if kind == 1 else torch.int32
            dev_q.append((0, kind, src, 0.1, T.SCHEDULE_PLAIN, torch.empty(V, dtype=dt, device="cuda")))
            h = torch.full((V,), 3, dtype=dt).pin_memory() if parts != 3 else np.full(V, 3, np.float32 if kind else np.int32)
            host_out.append(h)
            host_q.append((0, kind, src, 0.1, T.SCHEDULE_PLAIN, h))
    b = T.Batch([g])
    b.run(dev_q)
    ms = b.run_host(host_q, parts=parts)
    assert ms > 0
    for (gi, kind, src, _, _, dv), h in zip(dev_q, host_out):
        got = h.numpy() if hasattr(h, "numpy") else h
        assert np.array_equal(got.view(np.uint32), dv.cpu().numpy().view(np.uint32)), (kind, src)
        if kind == 1:
            assert np.array_equal(got.view(np.uint32), O.bellman_ford(V, s, d, w, src).view(np.uint32))
        else:
            assert np.array_equal(got, O.bfs_levels(V, s, d, src))
    # a device output array is refused by the library itself
    import ctypes as C
    arr = (T.Query * 1)(T.Query(0, 1, srcs[0], 0.1, T.SCHEDULE_PLAIN, dev_q[0][5].data_ptr()))
    ms_out = C.c_float()
    assert T.lib().trav_batch_run_host(b._h, arr, 1, 2, C.byref(ms_out)) == T.TRAV_ERR_BAD_ARG
    b.close()
    g.free()


def test_host_output_batch_interleaves_cheap_queries_and_stays_exact():
    """A host-output batch with few teams spreads its cheap (BFS) queries among the expensive (SSSP) ones and
    keeps two per team for the end; the results are still the device-output batch's and the oracle's."""
    import torch

    s, d, w = O.rmat(13, 16, seed=37)
    V = 1 << 13
    g = T.Graph.from_edges(V, s, d, w)
    deg = np.bincount(s, minlength=V)
    srcs = [int(x) for x in np.flatnonzero(deg > 0)[::97][:20]]
    dev_q, host_q, host_out = [], [], []
    for src in srcs:
        for kind in (1, 0):
            dt = torch.float32 if kind == 1 else torch.int32
            dev_q.append((0, kind, src, 0.1, T.SCHEDULE_PLAIN, torch.empty(V, dtype=dt, device="cuda")))
            h = torch.full((V,), 7, dtype=dt).pin_memory()
            host_out.append(h)
            host_q.append((0, kind, src, 0.1, T.SCHEDULE_PLAIN, h))
    b = T.Batch([g])
    b.shape = (148, 32, 256)  # four teams: 40 queries, the last 8 BFS, 12 BFS spread among 20 SSSP
    b.run(dev_q)
    b.run_host(host_q, parts=1)
    for (gi, kind, src, _, _, dv), h in zip(dev_q, host_out):
        assert np.array_equal(h.numpy().view(np.uint32), dv.cpu().numpy().view(np.uint32)), (kind, src)
        if kind == 1:
            assert np.array_equal(h.numpy().view(np.uint32), O.bellman_ford(V, s, d, w, src).view(np.uint32))
        else:
            assert np.array_equal(h.numpy(), O.bfs_levels(V, s, d, src))
    b.close()
    g.free()
