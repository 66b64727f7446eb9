"""SSSP pull rounds: a heavy round that scans the in-rows of the vertices a heavy edge could still improve.

On a skewed RMAT graph the first bucket settles the hubs, whose heavy out-rows hold most of the edges, so the
heavy round after it pulls (phase kind 7 in the query's log, after the check phase, kind 6).  The distances must
equal the oracle's bit for bit: with the plain schedule, with wide forced buckets (a heavy edge can then land inside
the bucket it left, so the pull set must reach below the bucket bound), and in a batch launch.
"""
import numpy as np
import pytest

import oracle as O
import pytrav as T

pytestmark = pytest.mark.gpu

PULL_CHECK, PULL = 6, 7


@pytest.fixture(scope="module")
def skewed():
    import torch

    assert torch.cuda.is_available()
    scale, ef = 13, 32
    s, d, w = O.rmat(scale, ef, seed=4)
    V = 1 << scale
    g = T.Graph.from_edges(V, s, d, w)
    csr = O.csr(V, s, d, w)
    deg = np.bincount(s, minlength=V)
    order = np.argsort(-deg, kind="stable")
    nz = np.flatnonzero(deg > 0)
    sources = [int(order[0]), int(order[5]), int(nz[np.argmin(deg[nz])])]
    want = {src: O.dijkstra(V, s, d, w, src, csr_arrays=csr) for src in sources}
    yield g, sources, want
    g.free()


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def test_pull_round_runs_and_matches_oracle(skewed):
    g, sources, want = skewed
    pulled = 0
    for src in sources:
        got = g.sssp([src], delta=0.1)[0]
        assert np.array_equal(_bits(got), _bits(want[src])), src
        kinds = g.last_phase_log()[0]
        pulled += int(np.sum(kinds == PULL))
        assert np.sum(kinds == PULL) <= np.sum(kinds == PULL_CHECK)  # every pull follows a check
    assert pulled > 0, "no heavy round pulled on the skewed graph"


@pytest.mark.parametrize("option", [1, 2, 5])
def test_pull_with_wide_buckets_matches_oracle(skewed, option):
    g, sources, want = skewed
    g.set_plan(1, np.full(64, option, np.uint8))
    try:
        for src in sources:
            got = g.sssp([src], delta=0.1)[0]
            assert np.array_equal(_bits(got), _bits(want[src])), (src, option)
    finally:
        g.set_plan(1, None)


def test_pull_in_batch_matches_oracle(skewed):
    import torch

    g, sources, want = skewed
    outs = [torch.full((g.V,), 7.0, dtype=torch.float32, device="cuda") for _ in sources]
    b = T.Batch([g])
    b.run([(0, 1, src, 0.1, T.SCHEDULE_PLAIN, out) for src, out in zip(sources, outs)])
    for src, out in zip(sources, outs):
        assert np.array_equal(_bits(out.cpu().numpy()), _bits(want[src])), src
    b.close()
