"""The CPU oracle pinned against the reference's golden vectors (and the live reference build when present)."""
import ctypes
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, case_edges


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_rand_r_matches_libc():
    libc = ctypes.CDLL(None)
    libc.rand_r.argtypes = [ctypes.POINTER(ctypes.c_uint)]
    for seed in (0, 1, 12345, 0xDEADBEEF):
        st = ctypes.c_uint(seed)
        want = [libc.rand_r(ctypes.byref(st)) for _ in range(2000)]
        assert O.rand_r_stream(seed, 2000).tolist() == want


def test_lcg_skip_equals_stepping():
    L = O.lib()
    for seed in (0, 7, 2**31 + 5):
        st = ctypes.c_uint32(seed)
        for n in range(1, 50):
            L.orc_rand_r(ctypes.byref(st))
            assert L.orc_lcg_skip(seed, 3 * n) == st.value


def test_rmat_seed0_equals_reference_rmat_parallel():
    ref = np.load(f"{GOLDEN}/rmat_ref_s8_ef8.npz")
    s, d, w = O.rmat(8, 8, seed=0, drop_self_loops=False, threads=3)
    assert np.array_equal(s, ref["src"]) and np.array_equal(d, ref["dst"])
    assert np.array_equal(w.view(np.uint32), ref["w"].view(np.uint32))


def test_rmat_digests_of_larger_reference_runs(golden):
    meta, _ = golden
    for key, ent in meta["rmat_ref"].items():
        scale, avg = int(key.split("_")[0][1:]), int(key.split("_")[1][2:])
        s, d, w = O.rmat(scale, avg, seed=0, drop_self_loops=False)
        assert len(s) == ent["edges"]
        assert _sha(s, d, w) == ent["sha256"], key


def test_rmat_independent_of_threads():
    a = O.rmat(12, 8, seed=5, threads=1)
    b = O.rmat(12, 8, seed=5, threads=7)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_rmat_drops_only_self_loops():
    s0, d0, w0 = O.rmat(10, 16, seed=2, drop_self_loops=False)
    s1, d1, w1 = O.rmat(10, 16, seed=2, drop_self_loops=True)
    keep = s0 != d0
    assert np.array_equal(s1, s0[keep]) and np.array_equal(d1, d0[keep]) and np.array_equal(w1, w0[keep])


def test_bellman_ford_and_dijkstra_match_reference_golden(golden):
    meta, arrays = golden
    for name, c in meta["cases"].items():
        V, s, d, w = case_edges(name, meta, arrays)
        want = arrays[f"{name}/dist"]
        for i, src in enumerate(c["sources"]):
            got = O.bellman_ford(V, s, d, w, src)
            assert np.array_equal(got.view(np.uint32), want[i].view(np.uint32)), (name, src)
            dj = O.dijkstra(V, s, d, w, src)
            assert np.array_equal(dj.view(np.uint32), want[i].view(np.uint32)), (name, src, "dijkstra")


def test_bfs_levels_reachability_matches_reference_golden(golden):
    meta, arrays = golden
    for name, c in meta["cases"].items():
        V, s, d, w = case_edges(name, meta, arrays)
        vis = arrays[f"{name}/visited"]
        for i, src in enumerate(c["sources"]):
            lv = O.bfs_levels(V, s, d, src)
            assert np.array_equal(lv >= 0, vis[i].astype(bool)), (name, src)
            assert lv[src] == 0


def test_bfs_levels_are_hop_distances():
    # unit-weight SSSP equals BFS levels: an independent check of the restatement
    s, d, w = O.rmat(11, 8, seed=4)
    V = 1 << 11
    src = int(np.bincount(s, minlength=V).argmax())
    lv = O.bfs_levels(V, s, d, src)
    dist = O.dijkstra(V, s, d, np.ones(len(s), np.float32), src)
    hop = np.where(dist < O.FLT_MAX, dist, -1).astype(np.int64)
    assert np.array_equal(lv, hop)


def test_csr_order_matches_reference_conversion():
    if not O.ref_available():
        pytest.skip("reference build not present")
    s, d, w = O.rmat(11, 8, seed=9)
    V = 1 << 11
    g = O.RefGraph.csr_via_reference(V, s, d, w)
    ro, ra, rw = g.export_csr()
    oo, oa, ow = O.csr(V, s, d, w)
    assert np.array_equal(ro, oo) and np.array_equal(ra, oa) and np.array_equal(rw, ow)


def test_live_reference_agrees_on_fresh_graphs():
    if not O.ref_available():
        pytest.skip("reference build not present")
    for scale, avg, seed in [(9, 4, 11), (13, 8, 12)]:
        s, d, w = O.rmat(scale, avg, seed=seed)
        V = 1 << scale
        src = int(np.bincount(s, minlength=V).argmax())
        gel = O.RefGraph.edges_list(V, s, d, w)
        want = gel.bellman_ford(src, threads=4)
        assert np.array_equal(O.bellman_ford(V, s, d, w, src).view(np.uint32), want.view(np.uint32))
        gc = O.RefGraph.csr_via_reference(V, s, d, w)
        assert np.array_equal(O.bfs_levels(V, s, d, src) >= 0, gc.parallel_bfs(src, 4).astype(bool))


def test_device_layout_restatement_is_consistent():
    s, d, w = O.rmat(9, 8, seed=3)
    V = 1 << 9
    L = O.device_layout(V, s, d, w)
    deg = np.bincount(s, minlength=V)
    o2n = L["old_of_new"]
    assert np.all(np.diff(deg[o2n]) <= 0)  # degree descending
    assert np.array_equal(L["new_of_old"][o2n], np.arange(V))
    # same multiset of relabelled edges, rows sorted
    n = L["new_of_old"]
    got = sorted(zip(np.repeat(np.arange(V), np.diff(L["out_off"])), L["out_adj"], L["out_w"].view(np.uint32)))
    want = sorted(zip(n[s], n[d], w.view(np.uint32)))
    assert got == want
    for v in range(V):
        row_w = L["out_w"][L["out_off"][v]:L["out_off"][v + 1]]
        assert np.all(np.diff(row_w) >= 0)  # out rows by weight: a light prefix for any delta
        row_in = L["in_adj"][L["in_off"][v]:L["in_off"][v + 1]]
        assert np.all(np.diff(row_in) >= 0)


def test_algorithmic_bytes_formulae():
    s, d, w = O.rmat(9, 8, seed=3)
    V = 1 << 9
    L = O.device_layout(V, s, d, w)
    src_new = 0
    n2o = L["old_of_new"]
    dist_old = O.dijkstra(V, s, d, w, int(n2o[src_new]))
    dist_new = dist_old[n2o]
    reached = dist_new < O.FLT_MAX
    deg = np.diff(L["out_off"])
    assert O.sssp_bytes(V, L["out_off"], dist_new) == 4 * V + 12 * reached.sum() + 12 * deg[reached].sum()
    lv_old = O.bfs_levels(V, s, d, int(n2o[src_new]))
    lv_new = lv_old[n2o]
    nsteps = lv_new.max() + 1
    td = O.bfs_bytes(V, L, lv_new, np.zeros(nsteps, np.uint8))
    # all top-down: 4V + 12 per reached + 8 per out-edge of reached + 8 per discovered
    assert td == 4 * V + 12 * (lv_new >= 0).sum() + 8 * deg[lv_new >= 0].sum() + 8 * ((lv_new >= 1).sum())


def test_el_file_bytes_layout():
    with open(f"{GOLDEN}/el_small.bin", "rb") as f:
        b = f.read()
    assert len(b) == 13 + 12 * 6 and b[0] == 1
    V = int.from_bytes(b[1:5], "little")
    E = int.from_bytes(b[5:13], "little")
    assert (V, E) == (6, 6)


def test_el_optimize_matches_reference_fixture(golden):
    """The optimisation pass restatement against the reference's optimize_graph_for_CPU output (fixture)."""
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "el_optimize.npz"))
    meta = golden[0]["optimize"]
    seg = meta["segment"]
    s, d, w = O.el_optimize(f["src"], f["dst"], f["w"], segment=seg)
    assert len(s) == meta["E_after"] == len(f["ref_src"])
    # same arcs and weights (the reference's std::sort leaves the order inside a segment pair open)
    mine = sorted(zip(s.tolist(), d.tolist(), w.tolist()))
    ref = sorted(zip(f["ref_src"].tolist(), f["ref_dst"].tolist(), f["ref_w"].tolist()))
    assert mine == ref
    # both orders group edges by (src // segment, dst // segment)
    for a, b in ((s, d), (f["ref_src"], f["ref_dst"])):
        key = (a // seg).astype(np.int64) * (1 << 20) + (b // seg)
        assert np.all(np.diff(key) >= 0)
    # inside a group, the restatement keeps (src, dst, w) order
    key = (s // seg).astype(np.int64) * (1 << 20) + (d // seg)
    order = np.lexsort((w, d, s, key))
    assert np.array_equal(order, np.arange(len(s)))
    assert len(set(zip(s.tolist(), d.tolist()))) == len(s) and not np.any(s == d)


def test_gpu_transactions_matches_reference_fixture(golden):
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "el_optimize.npz"))
    meta = golden[0]["optimize"]
    for k, want in meta["transactions_before"].items():
        assert O.gpu_transactions(f["src"], f["dst"], int(k)) == want
    for k, want in meta["transactions_after_reference_order"].items():
        assert O.gpu_transactions(f["ref_src"], f["ref_dst"], int(k)) == want


def test_el_optimize_live_reference_small_segments():
    if not O.ref_available():
        pytest.skip("reference build not present")
    rng = np.random.default_rng(5)
    for V, E in ((70000, 3001), (140000, 9000), (10, 40), (5, 31)):
        s = rng.integers(0, V, E).astype(np.int32)
        d = rng.integers(0, V, E).astype(np.int32)
        w = (rng.integers(0, 3, E) / 2).astype(np.float32)
        g = O.RefGraph.edges_list(V, s, d, w)
        assert O.gpu_transactions(s, d, 4) == g.gpu_transactions(4)
        n = g.optimize_for_cpu(4)
        rs, rd, rw = g.export_el()
        ms, md, mw = O.el_optimize(s, d, w, segment=65536)
        assert n == len(ms)
        assert sorted(zip(ms.tolist(), md.tolist(), mw.tolist())) == sorted(zip(rs.tolist(), rd.tolist(), rw.tolist()))
        g.free()


def test_masked_reach_restatement_is_reachability_inside_the_pivots_tree():
    """orc_reach_masked (the SCC sweep) equals a queue BFS over the edges whose ends share the pivot's tree."""
    import collections

    V = 1 << 9
    s, d, _ = O.rmat(9, 8, seed=6, drop_self_loops=False)
    trees = np.random.default_rng(1).integers(0, 3, V).astype(np.int32)
    adj = collections.defaultdict(list)
    for a, b in zip(s.tolist(), d.tolist()):
        if trees[a] == trees[b]:
            adj[a].append(b)
    for pivot in (0, int(np.bincount(s, minlength=V).argmax())):
        want = np.zeros(V, np.uint8)
        want[pivot] = 1
        q = collections.deque([pivot])
        while q:
            u = q.popleft()
            for v in adj[u]:
                if not want[v]:
                    want[v] = 1
                    q.append(v)
        assert np.array_equal(O.reach_masked(V, s, d, pivot, trees), want)
