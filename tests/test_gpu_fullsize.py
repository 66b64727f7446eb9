"""Full-size workload (RMAT s23 ef32, the benchmark's graph): results checked through size-independent properties.

The oracle cannot finish Dijkstra or BFS at this size in seconds, so the GPU results are checked against the
properties that characterise them exactly, evaluated on the GPU over every edge of the exported layout:

* BFS levels: level[s] = 0; no edge u -> v with u reached has level[v] > level[u] + 1 (or v unreached); every
  reached v != s has an in-edge from a vertex at level[v] - 1.
* SSSP distances: d[s] = 0; no edge u -> v with u reached has fl(d[u] + w) < d[v] (the relaxation fixpoint);
  every reached v != s has an in-edge with fl(d[u] + w) == d[v] (the distance is the length of a path).
  Weights are > 0 except on the rare edges whose rand_r draw was 0, so justifying edges form no cycle and
  the two conditions pin the distances to the exact minimum over paths of the left-folded fp32 sums.
* The learned and plain schedules, delta 0.1 and Bellman-Ford give the same bits.
"""
import numpy as np
import pytest

import pytrav as T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    import torch

    assert torch.cuda.is_available()
    g = T.Graph.rmat(23, 32, (57, 19, 19, 5), seed=1, drop_self_loops=True)
    L = g.export_layout()
    dev = torch.device("cuda")
    E = g.E
    off = torch.from_numpy(L["out_off"]).to(dev).long()
    src = torch.repeat_interleave(torch.arange(g.V, device=dev), off[1:] - off[:-1], output_size=E)
    lay = dict(src=src, dst=torch.from_numpy(L["out_adj"]).to(dev).long(), w=torch.from_numpy(L["out_w"]).to(dev),
               old_of_new=torch.from_numpy(L["old_of_new"]).to(dev).long())
    deg = g.out_degrees()
    rng = np.random.default_rng(5)
    sources = rng.choice(np.flatnonzero(deg > 0), 2, replace=False).astype(np.int32)
    yield g, lay, sources
    g.free()


def _in_new_ids(x, lay):
    """Per-vertex results indexed by original id -> indexed by the layout's (new) ids."""
    return x[lay["old_of_new"]]


def test_bfs_levels_properties(big):
    import torch

    g, lay, sources = big
    lv = torch.empty((len(sources), g.V), dtype=torch.int32, device="cuda")
    g.bfs(sources, out=lv)
    for q, s in enumerate(sources):
        L = _in_new_ids(lv[q].long(), lay)
        s_new = int(torch.nonzero(lay["old_of_new"] == int(s))[0])
        assert int(L[s_new]) == 0 and int((L == 0).sum()) == 1
        lu, lvv = L[lay["src"]], L[lay["dst"]]
        reached_u = lu >= 0
        assert bool(((lvv >= 0) | ~reached_u).all())                      # no reached -> unreached edge
        assert bool(((lvv <= lu + 1) | ~reached_u).all())                  # no shortcut
        just = torch.zeros(g.V, dtype=torch.bool, device="cuda")
        just[lay["dst"][reached_u & (lvv == lu + 1)]] = True               # a parent one level up
        need = (L > 0)
        assert bool((just | ~need).all())


def test_sssp_distances_properties(big):
    import torch

    g, lay, sources = big
    di = torch.empty((len(sources), g.V), dtype=torch.float32, device="cuda")
    g.sssp(sources, out=di, delta=0.1)
    fmax = torch.finfo(torch.float32).max
    for q, s in enumerate(sources):
        D = _in_new_ids(di[q], lay)
        s_new = int(torch.nonzero(lay["old_of_new"] == int(s))[0])
        assert float(D[s_new]) == 0.0
        du, dv = D[lay["src"]], D[lay["dst"]]
        reached_u = du < fmax
        relax = du + lay["w"]  # one round-to-nearest fp32 add, as the kernels
        assert bool(((dv <= relax) | ~reached_u).all())                    # fixpoint
        just = torch.zeros(g.V, dtype=torch.bool, device="cuda")
        just[lay["dst"][reached_u & (relax == dv)]] = True
        need = (D < fmax) & (torch.arange(g.V, device="cuda") != s_new)
        assert bool((just | ~need).all())                                  # every distance is a path length


def test_schedules_and_widths_agree_at_full_size(big):
    import torch

    from pytrav import learn

    g, _, sources = big
    base = g.sssp(sources, delta=0.1).view(np.uint32)
    assert np.array_equal(g.sssp(sources, delta=0.0).view(np.uint32), base)   # Bellman-Ford
    assert np.array_equal(g.sssp(sources, delta=0.4).view(np.uint32), base)
    lv = g.bfs(sources)
    if learn.install(g):
        assert np.array_equal(g.sssp(sources, delta=0.1, schedule=T.SCHEDULE_LEARNED).view(np.uint32), base)
        assert np.array_equal(g.bfs(sources, schedule=T.SCHEDULE_LEARNED), lv)
    assert np.array_equal(g.bfs(sources, force_direction=0), lv)              # top-down only
    del torch
