"""What the shipped schedule networks gain over the plain schedule on a graph they were not trained on.

RMAT s21 ef32 with seed 777 (the training graphs use seeds 101-106, the evaluation graphs others): 6 sources,
device time of BFS and SSSP (delta 0.1) under the plain schedule (Beamer alpha 15 / beta 18, fixed delta) and the
learned one, best of three runs each.  The results must be identical, and the learned schedule must not be slower
overall; the measured ratios are printed (pytest -s) and attached to the test report.
"""
import numpy as np
import pytest

import pytrav as T
from pytrav import learn

pytestmark = pytest.mark.gpu


def test_learned_schedule_gain_on_a_held_out_graph(record_property):
    import torch

    g = T.Graph.rmat(21, 32, (57, 19, 19, 5), seed=777, drop_self_loops=True)
    if not learn.install(g):
        pytest.skip("no trained schedule networks in parallel-task1_b200/weights")
    src = learn.sources_of(g, 6, seed=5)
    n = len(src)
    out = {k: (torch.empty((n, g.V), dtype=torch.int32, device="cuda"),
               torch.empty((n, g.V), dtype=torch.float32, device="cuda")) for k in ("plain", "learned")}
    ms = {}
    for name, sched in (("plain", T.SCHEDULE_PLAIN), ("learned", T.SCHEDULE_LEARNED)):
        lv, di = out[name]
        tb, ts = [], []
        for _ in range(3):
            g.bfs(src, out=lv, schedule=sched)
            tb.append(float(np.sum(g.last_batch_ms())))
            g.sssp(src, out=di, delta=0.1, schedule=sched)
            ts.append(float(np.sum(g.last_batch_ms())))
        ms[name] = (min(tb), min(ts))
    assert torch.equal(out["plain"][0], out["learned"][0])
    assert torch.equal(out["plain"][1].view(torch.int32), out["learned"][1].view(torch.int32))
    bfs_gain = ms["plain"][0] / ms["learned"][0]
    sssp_gain = ms["plain"][1] / ms["learned"][1]
    total_gain = sum(ms["plain"]) / sum(ms["learned"])
    for k, v in (("bfs_gain", bfs_gain), ("sssp_gain", sssp_gain), ("total_gain", total_gain)):
        record_property(k, round(v, 4))
    print(f"\nlearned schedule on held-out RMAT s21 ef32: BFS x{bfs_gain:.3f}, SSSP x{sssp_gain:.3f}, "
          f"total x{total_gain:.3f} (plain {ms['plain']}, learned {ms['learned']} ms)")
    assert total_gain >= 1.0, ms
    g.free()
