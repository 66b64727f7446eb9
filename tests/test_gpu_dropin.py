"""The drop-in boundary exercised by the reference's own, unchanged GPU callers.

oracle/_ref/libtrav_dropin.so is the reference's SingleSourceShortestPaths::gpu_bellman_ford (sssp.hpp:219-277),
BFS::gpu_bfs (bfs.hpp:212-254) and TransitiveClosure's GPU reachability (transitive_closure.hpp:20-70) compiled
from its headers and linked against libtrav_b200.so in place of bellman_ford.cu / bfs.cu (oracle/build_dropin.sh).
Their results are compared bit for bit with the reference's own CPU implementations (oracle/_ref/libtrav_ref.so):
cpu_bellman_ford distances and cpu_parallel_bfs reachability.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(O.HERE, "_ref", "libtrav_dropin.so")


@pytest.fixture(scope="module")
def dropin():
    if not (os.path.exists(DROPIN) and O.ref_available()):
        pytest.skip("oracle/_ref is not built (oracle/build_dropin.sh needs the reference sources)")
    import pytrav as T

    T.lib()  # the product library first, so the harness binds to the same copy
    L = C.CDLL(DROPIN)
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
    L.dropin_gpu_bellman_ford.argtypes = [C.c_int, C.c_longlong, i32p, i32p, f32p, C.c_int, f32p]
    L.dropin_gpu_bellman_ford.restype = C.c_double
    L.dropin_gpu_bfs.argtypes = [C.c_int, C.c_longlong, i32p, i32p, C.c_int, u8p]
    L.dropin_tc_gpu_bfs.argtypes = [C.c_int, C.c_longlong, i32p, i32p, i32p, C.c_int, u8p]
    return L


def _reference_results(V, s, d, w, sources):
    gel = O.RefGraph.edges_list(V, s, d, w)
    gcsr = O.RefGraph.csr_via_reference(V, s, d, w)
    try:
        dist = [gel.bellman_ford(int(x), threads=4) for x in sources]
        reach = [gcsr.parallel_bfs(int(x), threads=4) for x in sources]
    finally:
        gel.free()
        gcsr.free()
    return dist, reach


@pytest.mark.parametrize("scale,ef,seed,loops", [(12, 8, 3, False), (16, 16, 1, True)])
def test_reference_gpu_bellman_ford_and_gpu_bfs_run_on_the_library(dropin, scale, ef, seed, loops):
    """(16, 16, 1, loops dropped) is the C1 configuration, from its max-out-degree source."""
    V = 1 << scale
    s, d, w = O.rmat(scale, ef, seed=seed, drop_self_loops=loops)
    deg = np.bincount(s, minlength=V)
    sources = [int(deg.argmax()), int(np.flatnonzero(deg > 0)[len(s) % 97])]
    want_d, want_r = _reference_results(V, s, d, w, sources)
    for k, src in enumerate(sources):
        dist = np.empty(V, np.float32)
        mteps = dropin.dropin_gpu_bellman_ford(V, len(s), s, d, w, src, dist)
        assert mteps > 0, "gpu_bellman_ford threw"
        assert np.array_equal(dist.view(np.uint32), want_d[k].view(np.uint32)), src
        vis = np.full(V, 7, np.uint8)
        assert dropin.dropin_gpu_bfs(V, len(s), s, d, src, vis) == 0
        assert np.array_equal(vis, want_r[k].astype(np.uint8)), src


def test_transitive_closure_gpu_reachability_runs_on_the_library(dropin):
    V = 1 << 11
    s, d, w = O.rmat(11, 4, seed=9, drop_self_loops=False)
    deg = np.bincount(s, minlength=V)
    sources = np.array([int(deg.argmax()), 5, 1000, int(np.flatnonzero(deg == 0)[0])], np.int32)
    _, want_r = _reference_results(V, s, d, w, sources)
    vis = np.full(len(sources) * V, 3, np.uint8)
    assert dropin.dropin_tc_gpu_bfs(V, len(s), s, d, sources, len(sources), vis) == 0
    for k in range(len(sources)):
        assert np.array_equal(vis[k * V:(k + 1) * V], want_r[k].astype(np.uint8)), sources[k]
