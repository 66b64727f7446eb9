"""Order independence of the fp32 SSSP fixpoint, on the host.

The kernels' bit-exactness rests on one property: every relaxation is the single rounded add fl(d[u] + w), which
is monotone in d[u] and never below d[u] for w >= 0, so any order of relaxations that reaches a fixpoint reaches
the same one (the minimum over paths of the left-folded sums).  Push rounds, pull rounds, deferred atomics and
wide buckets are all such orders.  Here the oracle's Bellman-Ford sweep runs over random permutations of random
edge lists -- zero and negative-zero weights, repeated arcs, self-loops, unreachable vertices, weights far apart in
magnitude -- and must give Dijkstra's bits every time.
"""
import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

import oracle as O

WEIGHT_KINDS = ["unit", "tiny", "integers", "mixed"]


def _weights(rng, kind, E):
    if kind == "unit":
        w = rng.random(E, dtype=np.float32)
    elif kind == "tiny":
        w = (rng.random(E) * 1e-6).astype(np.float32)
    elif kind == "integers":
        w = rng.integers(1, 100, E).astype(np.float32)
    else:
        w = (rng.random(E) * 10.0 ** rng.integers(-8, 8, E)).astype(np.float32)
    w[rng.random(E) < 0.1] = 0.0
    w[rng.random(E) < 0.05] = -0.0
    return w


@settings(max_examples=60, deadline=None)
@given(V=st.integers(1, 48), E=st.integers(0, 240), seed=st.integers(0, 2**31 - 1),
       kind=st.sampled_from(WEIGHT_KINDS))
def test_relaxation_order_does_not_change_the_bits(V, E, seed, kind):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, V, E).astype(np.int32)
    d = rng.integers(0, V, E).astype(np.int32)
    w = _weights(rng, kind, E)
    if E > 4:
        s[:2], d[:2] = d[:2], s[:2]  # some reverse arcs
        s[2] = d[2]  # a self-loop
        s[3], d[3], w[3] = s[4], d[4], w[4] * 2  # a heavier repeated arc
    src = int(rng.integers(0, V))
    want = O.dijkstra(V, s, d, w, src).view(np.uint32)
    for _ in range(3):
        p = rng.permutation(E)
        got = O.bellman_ford(V, s[p], d[p], w[p], src).view(np.uint32)
        assert np.array_equal(got, want)
