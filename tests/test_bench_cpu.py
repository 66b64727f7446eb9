"""The bench's host-side legs without a GPU: the reference arm's bounded sample and the e2e part boundaries."""
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


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 8, 16, 63, 64, 100])
def test_e2e_parts_cover_the_sources_in_order(n):
    cut = bench.e2e_cuts(n)
    assert cut[0] == 0 and cut[-1] == n
    assert all(b > a for a, b in zip(cut, cut[1:]))  # no empty part
    assert len(cut) - 1 <= 4
    if n == 64:
        assert cut == [0, 24, 44, 58, 64]
