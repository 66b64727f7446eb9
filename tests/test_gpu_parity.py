"""Parity of the CUDA path (through the C ABI) with the oracle and the reference's golden vectors.

Bar: bit-exact for everything -- RMAT edges, the device CSR layout, BFS
levels and fp32 SSSP distances (compared as uint32 bit patterns).
"""
import numpy as np
import pytest

import oracle as O
import pytrav as T
from conftest import case_edges

pytestmark = pytest.mark.gpu

DELTAS = [0.0, float("inf"), 0.1, 0.013, 1.0, 7.5]


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    assert _t.cuda.is_available(), "GPU tests need a CUDA device"
    return _t


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def test_device_rmat_is_bit_exact_with_oracle(torch):
    for scale, avg, seed, drop in [(8, 8, 0, False), (12, 16, 1, True), (16, 16, 1, True), (17, 4, 99, False)]:
        V = 1 << scale
        E = V * avg
        s = torch.empty(E, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        w = torch.empty(E, dtype=torch.float32, device="cuda")
        g = T.Graph.rmat(scale, avg, seed=seed, drop_self_loops=drop, edges_out=(s, d, w))
        n = g.generated_edges
        os_, od, ow = O.rmat(scale, avg, seed=seed, drop_self_loops=drop)
        assert n == len(os_)
        assert np.array_equal(s[:n].cpu().numpy(), os_) and np.array_equal(d[:n].cpu().numpy(), od)
        assert np.array_equal(bits(w[:n].cpu().numpy()), bits(ow))
        assert g.V == V and g.E == n


def test_device_layout_equals_oracle_layout(torch):
    for scale, avg, seed in [(6, 4, 1), (10, 8, 2), (13, 16, 5)]:
        s, d, w = O.rmat(scale, avg, seed=seed)
        V = 1 << scale
        g = T.Graph.from_edges(V, s, d, w)
        got = g.export_layout()
        want = O.device_layout(V, s, d, w)
        for k in ("new_of_old", "old_of_new", "out_adj", "in_adj"):
            assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(got["out_off"].astype(np.int64), want["out_off"])
        assert np.array_equal(got["in_off"].astype(np.int64), want["in_off"])
        assert np.array_equal(bits(got["out_w"]), bits(want["out_w"]))
        assert g.max_out_degree == int(np.bincount(s, minlength=V).max())


def test_device_in_edge_weights_follow_the_in_rows(torch):
    # The CSC is one stable sort of the edges by (new target, new source), so its weights are the edge-list
    # weights (-0.0 read as +0.0) in that order; the layout's in_adj pins the order itself.
    for scale, avg, seed in [(6, 4, 1), (10, 8, 2), (13, 16, 5)]:
        s, d, w = O.rmat(scale, avg, seed=seed)
        w = w.copy()
        w[::7] = -0.0
        V = 1 << scale
        g = T.Graph.from_edges(V, s, d, w)
        want = O.device_layout(V, s, d, w)
        n2o = want["new_of_old"]
        ns, nd = n2o[s], n2o[d]
        order = np.lexsort((ns, nd))
        assert np.array_equal(ns[order], want["in_adj"])
        w0 = np.where(w == 0.0, np.float32(0.0), w).astype(np.float32)
        assert np.array_equal(bits(g.export_in_w()), bits(w0[order]))
        g.free()


def test_golden_cases_bfs_levels(golden, torch):
    meta, arrays = golden
    for name, c in meta["cases"].items():
        V, s, d, w = case_edges(name, meta, arrays)
        g = T.Graph.from_edges(V, s, d, w)
        vis = arrays[f"{name}/visited"]
        for force in (-1, 0, 1):
            lv = g.bfs(c["sources"], force_direction=force)
            for i, src in enumerate(c["sources"]):
                want = O.bfs_levels(V, s, d, src)
                assert np.array_equal(lv[i], want), (name, src, force)
                assert np.array_equal(lv[i] >= 0, vis[i].astype(bool)), (name, src, force)


def test_golden_cases_sssp_distances(golden, torch):
    meta, arrays = golden
    for name, c in meta["cases"].items():
        V, s, d, w = case_edges(name, meta, arrays)
        g = T.Graph.from_edges(V, s, d, w)
        want = arrays[f"{name}/dist"]
        for delta in DELTAS:
            got = g.sssp(c["sources"], delta=delta)
            assert np.array_equal(bits(got), bits(want)), (name, delta)


def test_config1_rmat_s16_ef16_bellman_ford(torch):
    # RMAT s16 ef16, a/b/c/d 57/19/19/5, seed 1, loops dropped, max out-degree source
    s, d, w = O.rmat(16, 16, seed=1)
    V = 1 << 16
    deg = np.bincount(s, minlength=V)
    src = int(np.flatnonzero(deg == deg.max())[0])
    g = T.Graph.rmat(16, 16, seed=1)
    assert g.E == len(s)
    want = O.bellman_ford(V, s, d, w, src)
    for delta in (0.0, 0.1):
        assert np.array_equal(bits(g.sssp([src], delta=delta)[0]), bits(want)), delta
    lv = g.bfs([src])[0]
    assert np.array_equal(lv, O.bfs_levels(V, s, d, src))
    st = g.last_stats()
    assert st.reached == int((lv >= 0).sum())


def test_many_sources_and_device_outputs(torch):
    s, d, w = O.rmat(14, 8, seed=21)
    V = 1 << 14
    g = T.Graph.from_edges(V, s, d, w)
    rng = np.random.default_rng(0)
    srcs = rng.integers(0, V, 24).astype(np.int32)
    csr = O.csr(V, s, d, w)
    lv_dev = torch.empty((len(srcs), V), dtype=torch.int32, device="cuda")
    g.bfs(srcs, out=lv_dev)
    di_dev = torch.empty((len(srcs), V), dtype=torch.float32, device="cuda")
    g.sssp(srcs, out=di_dev, delta=0.05)
    lv = lv_dev.cpu().numpy()
    di = di_dev.cpu().numpy()
    for i, x in enumerate(srcs):
        assert np.array_equal(lv[i], O.bfs_levels(V, s, d, int(x), csr_arrays=csr))
        assert np.array_equal(bits(di[i]), bits(O.dijkstra(V, s, d, w, int(x), csr_arrays=csr)))


def test_high_diameter_grid_and_uniform(torch):
    # 4-neighbour grid with integer weights in [1,100): a long, thin frontier
    n = 96
    idx = np.arange(n * n).reshape(n, n)
    pairs = [(idx[:, :-1], idx[:, 1:]), (idx[:, 1:], idx[:, :-1]), (idx[:-1, :], idx[1:, :]), (idx[1:, :], idx[:-1, :])]
    s = np.concatenate([a.ravel() for a, _ in pairs]).astype(np.int32)
    d = np.concatenate([b.ravel() for _, b in pairs]).astype(np.int32)
    rng = np.random.default_rng(5)
    w = rng.integers(1, 100, len(s)).astype(np.float32)
    V = n * n
    g = T.Graph.from_edges(V, s, d, w)
    for src in (0, V // 2 + n // 2):
        want = O.dijkstra(V, s, d, w, src)
        for delta in (0.0, 1.0, 50.0, 300.0):
            assert np.array_equal(bits(g.sssp([src], delta=delta)[0]), bits(want)), delta
        assert np.array_equal(g.bfs([src])[0], O.bfs_levels(V, s, d, src))
    # uniform random graph
    V = 1 << 14
    s = rng.integers(0, V, 16 * V).astype(np.int32)
    d = rng.integers(0, V, 16 * V).astype(np.int32)
    w = rng.random(16 * V).astype(np.float32)
    g = T.Graph.from_edges(V, s, d, w)
    want = O.dijkstra(V, s, d, w, 3)
    for delta in (0.0, 0.1, 0.02):
        assert np.array_equal(bits(g.sssp([3], delta=delta)[0]), bits(want))
    assert np.array_equal(g.bfs([3])[0], O.bfs_levels(V, s, d, 3))


def test_unweighted_graph_defaults_to_unit_weights(torch):
    s, d, _ = O.rmat(10, 8, seed=8)
    V = 1 << 10
    g = T.Graph.from_edges(V, s, d, None)
    lv = g.bfs([0])[0]
    dist = g.sssp([0])[0]
    assert np.array_equal(np.where(lv >= 0, lv.astype(np.float32), O.FLT_MAX), dist)


def test_reference_wrappers_on_device_edge_lists(torch):
    s, d, w = O.rmat(12, 8, seed=31)
    V, E = 1 << 12, len(s)
    ts, td, tw = (torch.from_numpy(x).cuda() for x in (s, d, w))
    dist = torch.empty(V, dtype=torch.float32, device="cuda")
    T.init_distances(dist, V, 77)
    h = dist.cpu().numpy()
    assert h[77] == 0 and np.all(np.delete(h, 77) == O.FLT_MAX)
    T.bellman_ford_wrapper(ts, td, tw, V, E, 77, dist)
    assert np.array_equal(bits(dist.cpu().numpy()), bits(O.bellman_ford(V, s, d, w, 77)))
    vis = torch.zeros(V, dtype=torch.uint8, device="cuda")
    T.bfs_wrapper(ts, td, V, E, vis, 77)
    assert np.array_equal(vis.cpu().numpy().astype(bool), O.bfs_levels(V, s, d, 77) >= 0)


def test_bellman_ford_wrapper_continues_from_given_distances(torch):
    # the reference's wrapper relaxes whatever the array holds (two seeds here)
    s, d, w = O.rmat(10, 8, seed=32)
    V, E = 1 << 10, len(s)
    init = np.full(V, O.FLT_MAX, np.float32)
    init[[5, 900]] = [0.0, 0.25]
    want = init.copy()
    changed = True
    while changed:  # the reference's sweep (sssp.hpp:47-61), vectorised per edge order
        changed = False
        for e in range(E):
            c = np.float32(want[s[e]] + w[e])
            if want[d[e]] > c:
                want[d[e]] = c
                changed = True
    dist = torch.from_numpy(init).cuda()
    T.bellman_ford_wrapper(*(torch.from_numpy(x).cuda() for x in (s, d, w)), V, E, 0, dist)
    assert np.array_equal(bits(dist.cpu().numpy()), bits(want))


def test_algorithmic_bytes_match_oracle(torch):
    s, d, w = O.rmat(13, 16, seed=41)
    V = 1 << 13
    g = T.Graph.from_edges(V, s, d, w)
    layout = O.device_layout(V, s, d, w)
    src = int(np.bincount(s, minlength=V).argmax())
    for force in (-1, 0, 1):
        lv = g.bfs([src], force_direction=force)[0]
        dirs, frontier = g.last_bfs_trace()
        st = g.last_stats()
        lv_new = lv[layout["old_of_new"]]
        assert st.algorithmic_bytes == O.bfs_bytes(V, layout, lv_new, dirs), force
        assert st.steps == len(dirs) == lv.max() + 1
        assert frontier[0] == 1
    dist = g.sssp([src], delta=0.1)[0]
    st = g.last_stats()
    assert st.algorithmic_bytes == O.sssp_bytes(V, layout["out_off"], dist[layout["old_of_new"]])


def test_beamer_switches_direction_on_rmat(torch):
    g = T.Graph.rmat(16, 16, seed=1)
    g.bfs([0])
    dirs, _ = g.last_bfs_trace()
    assert dirs[0] == 0 and 1 in dirs.tolist(), dirs


@pytest.mark.parametrize("bad", ["source", "neg_weight", "id_range", "learned_without_mlp", "nan_delta"])
def test_errors_are_reported(torch, bad):
    s = np.array([0, 1, 2], np.int32)
    d = np.array([1, 2, 0], np.int32)
    w = np.array([1.0, 1.0, 1.0], np.float32)
    with pytest.raises(T.TravError) as e:
        if bad == "source":
            T.Graph.from_edges(3, s, d, w).bfs([3])
        elif bad == "neg_weight":
            T.Graph.from_edges(3, s, d, np.array([1.0, -1.0, 1.0], np.float32))
        elif bad == "id_range":
            T.Graph.from_edges(2, s, d, w)
        elif bad == "learned_without_mlp":
            T.Graph.from_edges(3, s, d, w).bfs([0], schedule=T.SCHEDULE_LEARNED)
        else:
            T.Graph.from_edges(3, s, d, w).sssp([0], delta=float("nan"))
    assert e.value.code == T.TRAV_ERR_BAD_ARG
