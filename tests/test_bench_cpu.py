"""The bench's host-side legs without a GPU: the reference arm's bounded sample, its parity record and config."""
import argparse

import pytest

import bench
import oracle as O


def test_reference_arm_sample_runs_on_host():
    if not O.ref_available():
        pytest.skip("oracle/_ref is not built")
    a = argparse.Namespace(scale=10, ef=8, seed=1, sources=4)
    ref = bench.CpuReference(a, threads=2)
    try:
        v, desc = ref.sample(0.2)
    finally:
        ref.free()
    assert ref.E > 0 and v > 0
    assert "cpu_parallel_bfs" in desc and "cpu_bellman_ford" in desc


def test_cpu_baseline_parity_record_compares_bits():
    """The CPU-baseline leg compares the reference's results with the GPU step's: here the step's results are
    stood in for by the oracle's (equal), then by the oracle's with one distance bit flipped (not equal)."""
    if not O.ref_available():
        pytest.skip("oracle/_ref is not built")
    import numpy as np

    a = argparse.Namespace(scale=10, ef=8, seed=1, sources=3)
    V = 1 << a.scale
    s, d, w = O.rmat(a.scale, a.ef, (57, 19, 19, 5), seed=a.seed, drop_self_loops=True)
    srcs = bench.pick_sources(np.bincount(s, minlength=V), a.sources, a.seed)
    lv = np.stack([O.bfs_levels(V, s, d, int(x)) for x in srcs])
    di = np.stack([O.dijkstra(V, s, d, w, int(x)) for x in srcs])
    _, _, _, _, parity = bench.cpu_reference_run(a, 0.05, levels=lv, dist=di)
    assert parity["sources"] >= 1 and parity["equal"] is True
    bad = di.copy()
    bad[:, np.flatnonzero(lv[0] > 0)[0]] = np.nextafter(bad[:, np.flatnonzero(lv[0] > 0)[0]], np.float32(2))
    _, _, _, _, parity = bench.cpu_reference_run(a, 0.05, levels=lv, dist=bad)
    assert parity["sources"] >= 1 and parity["equal"] is False


def test_both_arms_print_the_same_config():
    a = argparse.Namespace(scale=23, ef=32, seed=1, sources=64, delta=0.1)
    c = bench.bench_config(a, 1 << 23, 268431728, 1)
    assert c == bench.bench_config(a, 1 << 23, 268431728, 1)
    assert "delta 0.1" in c["workload"] and "delta-stepping" not in c["workload"]
    assert set(bench.host_cpu()) == {"cpu_model", "physical_cores", "logical_cpus"}


def test_committed_traffic_is_read_for_its_own_workload_only():
    """roofline.traffic comes from profiles/traffic.txt: a per-query capture on the bench graph is scaled to the
    launch's queries, and a workload without a capture gets none (not another graph's figure)."""
    per_query = bench.ncu_traffic("batch_persistent", queries=1, workload="rmat_s23_ef32")
    assert per_query and per_query > 1e9
    assert bench.ncu_traffic("batch_persistent", queries=128, workload="rmat_s23_ef32") == pytest.approx(128 * per_query)
    assert bench.ncu_traffic("batch_persistent", queries=32, workload="rmat_s26_ef16") is None
    assert bench.ncu_traffic("no_such_kernel", queries=1, workload="rmat_s23_ef32") is None
