"""A small, fixed traversal workload to put under a profiler: the bench's RMAT graph (a/b/c/d 57/19/19/5
percent, seed 1, self loops dropped) at a chosen scale, n seeded sources picked as the bench picks them, and the
learned schedule.

    python -m pytrav.profile_case --scale 22 --sources 8 --mode batch

Modes:
  batch  two launches of one batch_persistent kernel over the n BFS and n SSSP queries, at a fixed launch shape
         (so no autotuner trials run first); capture the second with `-k regex:batch_persistent -s 1 -c 1`;
  sssp   the n SSSP queries twice as single-query sssp_persistent launches (capture with `-s <2n> -c 1`);
  bfs    the same for bfs_persistent.

The graph, its light rows and the outputs are all the device holds: about 2.5 GB at scale 22 and 5 GB at 23."""
import argparse
import os
import sys

import numpy as np

ABCD = (57, 19, 19, 5)  # integer percents, as the reference generator takes them


def pick_sources(deg, n, seed):
    """n distinct seeded sources among vertices of nonzero out-degree, sorted (the bench's rule)."""
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(deg > 0)
    return np.sort(rng.choice(cand, size=min(n, len(cand)), replace=False)).astype(np.int32)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--ef", type=int, default=32)
    ap.add_argument("--sources", type=int, default=8)
    ap.add_argument("--delta", type=float, default=0.1)
    ap.add_argument("--mode", choices=["batch", "sssp", "bfs"], default="batch")
    ap.add_argument("--shape", default="74,64,256", help="batch launch shape: CTAs per team, small degree, item")
    a = ap.parse_args(argv)

    import torch

    import pytrav as T
    from pytrav import learn

    g = T.Graph.rmat(a.scale, a.ef, ABCD, seed=1, drop_self_loops=True)
    srcs = [int(s) for s in pick_sources(g.out_degrees(), a.sources, 1)]
    if not learn.install(g, delta=a.delta):
        sys.exit("schedule weights missing")
    n, V = len(srcs), g.V
    lv = torch.empty((n, V), dtype=torch.int32, device="cuda")
    di = torch.empty((n, V), dtype=torch.float32, device="cuda")
    # algorithmic bytes of the queries (one single-query launch each; the count is the same however a query runs)
    alg = 0
    for i, s in enumerate(srcs):
        if a.mode in ("batch", "bfs"):
            g.bfs([s], out=lv[i:i + 1], schedule=T.SCHEDULE_LEARNED)
            alg += g.last_stats().algorithmic_bytes
        if a.mode in ("batch", "sssp"):
            g.sssp([s], out=di[i:i + 1], delta=a.delta, schedule=T.SCHEDULE_LEARNED)
            alg += g.last_stats().algorithmic_bytes
    print(f"algorithmic bytes of the {a.mode} queries: {alg}")
    if a.mode == "batch":
        b = T.Batch([g])
        b.shape = tuple(int(x) for x in a.shape.split(","))
        q = [(0, 1, s, a.delta, T.SCHEDULE_LEARNED, di[i]) for i, s in enumerate(srcs)] + \
            [(0, 0, s, 0.0, T.SCHEDULE_LEARNED, lv[i]) for i, s in enumerate(srcs)]
        for _ in range(2):
            ms = b.run(q)
        print(f"batch_persistent s{a.scale} ef{a.ef}: {2 * n} queries in {ms:.3f} ms")
        b.close()
    else:
        for _ in range(2):
            if a.mode == "sssp":
                g.sssp(srcs, out=di, delta=a.delta, schedule=T.SCHEDULE_LEARNED)
            else:
                g.bfs(srcs, out=lv, schedule=T.SCHEDULE_LEARNED)
        print(f"{a.mode}_persistent s{a.scale} ef{a.ef}: {n} queries in {np.sum(g.last_batch_ms()):.3f} ms")
    torch.cuda.synchronize()
    g.free()


if __name__ == "__main__":
    main()
