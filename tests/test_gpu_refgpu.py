"""The reference's own GPU path (bellman_ford.cu / bfs.cu built unchanged for sm_100a, oracle/_ref) gives the
same results as this library: the secondary baseline the bench times is doing the same work.  Its BF relaxes
without atomics (bellman_ford.cu:62-99) and iterates until a sweep changes nothing, which still ends at the
unique fixpoint, so the distance bits must be equal."""
import numpy as np
import pytest

import oracle as O
import pytrav as T

pytestmark = pytest.mark.gpu


def test_reference_gpu_path_matches_the_library():
    if not O.refgpu_available():
        pytest.skip("oracle/_ref/libtrav_refgpu.so is not built (oracle/build_refgpu.sh needs the reference sources)")
    V = 1 << 14
    s, d, w = O.rmat(14, 16, seed=8)
    g = T.Graph.from_edges(V, s, d, w)
    L = O.refgpu()
    assert L.refgpu_upload(V, len(s), s, d, w) == 0
    try:
        deg = np.bincount(s, minlength=V)
        for src in (int(deg.argmax()), int(np.flatnonzero(deg > 0)[99])):
            dist = np.empty(V, np.float32)
            vis = np.empty(V, np.uint8)
            with O.quiet_stdout():
                t_s = L.refgpu_sssp(src, dist)
                t_b = L.refgpu_bfs(src, vis)
            assert t_s > 0 and t_b > 0
            assert np.array_equal(dist.view(np.uint32), g.sssp([src], delta=0.1)[0].view(np.uint32))
            assert np.array_equal(vis.astype(bool), g.bfs([src])[0] >= 0)
    finally:
        L.refgpu_free()
        g.free()
