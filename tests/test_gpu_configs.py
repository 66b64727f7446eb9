"""The benchmark configurations at their full sizes, checked against the reference and the oracle.

* C2, RMAT s23 ef32 seed 1 (the bench's graph, built on the device): for three of the bench's seeded sources the
  SSSP distances (delta 0.1, plain and learned schedules) equal the reference's own cpu_bellman_ford bit for bit,
  BFS reachability equals its cpu_parallel_bfs, and BFS levels equal the oracle's queue BFS (oracle/_ref is the
  reference compiled from its sources; the oracle is pinned to it in tests/test_oracle.py).
* C3, the 4096 x 4096 grid (integer weights 1..99) and the uniform graph of 2^24 vertices and degree 16: one
  source each, distances equal the oracle's Dijkstra (the same fixpoint as cpu_bellman_ford: the property test
  of the oracle shows any relaxation order gives Dijkstra's bits), levels equal its queue BFS, for the plain and
  the learned schedules.
* C5, RMAT s26 ef16 (1.07 B edges, built on the device): too large for the CPU in a test, so its results are
  checked on the GPU through the properties that pin them exactly (tests/test_gpu_fullsize.py explains them).
"""
import os

import numpy as np
import pytest

import oracle as O
import pytrav as T
from pytrav import learn

pytestmark = pytest.mark.gpu

ABCD = (57, 19, 19, 5)


def _threads():
    return max(1, os.cpu_count() or 1)


def test_c2_rmat_s23_matches_the_reference_bit_for_bit():
    import bench

    if not O.ref_available():
        pytest.skip("oracle/_ref is not built")
    scale, ef, seed = 23, 32, 1
    V = 1 << scale
    g = T.Graph.rmat(scale, ef, ABCD, seed=seed, drop_self_loops=True)
    have = learn.install(g)
    s, d, w = O.rmat(scale, ef, ABCD, seed=seed, drop_self_loops=True, threads=_threads())
    assert g.E == len(s)
    sources = bench.pick_sources(np.bincount(s, minlength=V), 64, seed)[[0, 21, 63]]
    assert np.array_equal(sources, bench.pick_sources(g.out_degrees(), 64, seed)[[0, 21, 63]])
    gel = O.RefGraph.edges_list(V, s, d, w)
    off, adj, wt = O.csr(V, s, d, w)
    del s, d, w
    gcsr = O.RefGraph.csr(V, off, adj, wt)
    try:
        for src in sources.tolist():
            want = gel.bellman_ford(src, threads=_threads()).view(np.uint32)
            reach = gcsr.parallel_bfs(src, threads=_threads()).astype(bool)
            lv_want = O.bfs_levels(V, None, None, src, csr_arrays=(off, adj))
            for sched in ([T.SCHEDULE_PLAIN] + ([T.SCHEDULE_LEARNED] if have else [])):
                got = g.sssp([src], delta=0.1, schedule=sched)[0]
                assert np.array_equal(got.view(np.uint32), want), (src, sched)
                lv = g.bfs([src], schedule=sched)[0]
                assert np.array_equal(lv, lv_want), (src, sched)
                assert np.array_equal(lv >= 0, reach), (src, sched)
    finally:
        gel.free()
        gcsr.free()
        g.free()


@pytest.mark.parametrize("which", ["grid4096", "uniform24"])
def test_c3_inputs_match_the_oracle(which):
    if which == "grid4096":
        V, s, d, w = learn.grid_graph(4096, seed=11)
        delta = learn.plain_delta(50.0, 4)
    else:
        V, s, d, w = learn.uniform_graph(24, 16, seed=12)
        delta = learn.FIXED_DELTA
    g = T.Graph.from_edges(V, s, d, w)
    have = learn.install(g)
    src = int(np.flatnonzero(np.bincount(s, minlength=V) > 0)[V // 3 % 1000 + 17])
    off, adj, wt = O.csr(V, s, d, w)
    del s, d, w
    want = O.dijkstra(V, None, None, None, src, csr_arrays=(off, adj, wt)).view(np.uint32)
    lv_want = O.bfs_levels(V, None, None, src, csr_arrays=(off, adj))
    try:
        for sched in ([T.SCHEDULE_PLAIN] + ([T.SCHEDULE_LEARNED] if have else [])):
            assert np.array_equal(g.sssp([src], delta=delta, schedule=sched)[0].view(np.uint32), want), sched
            assert np.array_equal(g.bfs([src], schedule=sched)[0], lv_want), sched
    finally:
        g.free()


def test_c5_rmat_s26_properties_on_the_gpu():
    """d[s] = 0; no edge relaxes (fixpoint); every reached vertex has an in-edge that gives its distance; BFS
    levels: no edge skips a level and every reached vertex has a parent one level up.  Evaluated over all
    1.07 B edges in chunks on the GPU; the learned and plain schedules agree bit for bit."""
    import torch

    g = T.Graph.rmat(26, 16, ABCD, seed=1, drop_self_loops=True)
    have = learn.install(g)
    V, E = g.V, g.E
    src = int(np.flatnonzero(g.out_degrees() > 0)[123457])
    dev = torch.device("cuda")
    di = torch.empty((1, V), dtype=torch.float32, device=dev)
    lv = torch.empty((1, V), dtype=torch.int32, device=dev)
    g.sssp([src], out=di, delta=0.1)
    g.bfs([src], out=lv)
    if have:
        di2 = torch.empty_like(di)
        lv2 = torch.empty_like(lv)
        g.sssp([src], out=di2, delta=0.1, schedule=T.SCHEDULE_LEARNED)
        g.bfs([src], out=lv2, schedule=T.SCHEDULE_LEARNED)
        assert torch.equal(di.view(torch.int32), di2.view(torch.int32)) and torch.equal(lv, lv2)
        del di2, lv2
    L = g.export_layout()
    old_of_new = torch.from_numpy(L["old_of_new"]).to(dev).long()
    D = di[0][old_of_new]                # results in the layout's ids
    Lv = lv[0].long()[old_of_new]
    s_new = int(torch.nonzero(old_of_new == src)[0])
    fmax = torch.finfo(torch.float32).max
    assert float(D[s_new]) == 0.0 and int(Lv[s_new]) == 0
    off = torch.from_numpy(L["out_off"]).to(dev).long()
    adj_all = torch.from_numpy(L["out_adj"])
    w_all = torch.from_numpy(L["out_w"])
    justd = torch.zeros(V, dtype=torch.bool, device=dev)
    justl = torch.zeros(V, dtype=torch.bool, device=dev)
    chunk = 1 << 27
    for e0 in range(0, E, chunk):
        e1 = min(E, e0 + chunk)
        dst = adj_all[e0:e1].to(dev).long()
        w = w_all[e0:e1].to(dev)
        srcv = torch.searchsorted(off, torch.arange(e0, e1, device=dev), right=True) - 1
        du, dv = D[srcv], D[dst]
        reached = du < fmax
        relax = du + w  # one round-to-nearest fp32 add, as the kernels
        assert bool(((dv <= relax) | ~reached).all())
        justd[dst[reached & (relax == dv)]] = True
        lu, lvv = Lv[srcv], Lv[dst]
        rl = lu >= 0
        assert bool(((lvv >= 0) | ~rl).all()) and bool(((lvv <= lu + 1) | ~rl).all())
        justl[dst[rl & (lvv == lu + 1)]] = True
        del dst, w, srcv, du, dv, relax, lu, lvv
    need = torch.arange(V, device=dev) != s_new
    assert bool((justd | ~((D < fmax) & need)).all())
    assert bool((justl | ~((Lv > 0) & need)).all())
    g.free()
