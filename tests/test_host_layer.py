"""The C++ host layer (host/trav_library.hpp) compiled and run: its file APIs on CPU, its graph, SSSP and BFS
classes through the sample programs on the GPU."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import pytrav as T
from conftest import GOLDEN, PKG, ROOT

SAMPLES = os.path.join(PKG, "sample")


def _compile_check(tmp_path):
    exe = str(tmp_path / "host_layer_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", PKG,
                    os.path.join(ROOT, "tests", "host_layer_check.cpp"), "-o", exe, "-L", PKG, "-ltrav_b200",
                    "-Wl,-rpath," + PKG], check=True, capture_output=True)
    return exe


def test_host_layer_file_apis(tmp_path):
    exe = _compile_check(tmp_path)
    el = os.path.join(GOLDEN, "el_small.bin")
    adj = os.path.join(GOLDEN, "adj_small.bin")
    r = subprocess.run([exe, "files", el, adj, str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines() if " " in line)
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))["files"]
    want = " ".join(f"{s}>{d}:{np.float32(w):.9g}" for s, d, w in zip(meta["src"], meta["dst"], meta["w"]))
    assert lines["el"] == f"V={meta['V']} E={len(meta['src'])} directed=1 " + want
    assert lines["adj"] == f"V={meta['V']} E={len(meta['src'])} directed=1 " + want
    # the edge list saved again is byte-identical to the reference writer's
    assert open(tmp_path / "el_again.bin", "rb").read() == open(el, "rb").read()
    # the adjacency list written from the edge list reads back as the same rows
    ids, values, off, dst, w, V, _ = T.read_adjacency_list(str(tmp_path / "adj_from_el.bin"))
    src, d, wt = T.adjacency_to_edges(ids, off, dst, w)
    assert src.tolist() == meta["src"] and d.tolist() == meta["dst"] and np.all(values == 0)
    # pairs of the 13 + 72-byte fixture: 85 // 12 = 7 pairs
    assert "pairs V=8 E=7" in r.stdout
    assert "missing=0" in r.stdout


@pytest.mark.gpu
def test_bfs_sample_matches_oracle():
    """sample/bfs <scale> [seed]: R_MAT_parallel(2^scale, 16, 45/20/20/15) from vertex 0, as the reference's
    sample generates (sample/bfs.cpp:138); reached count and level count checked against the oracle."""
    scale, seed = 12, 0
    r = subprocess.run([os.path.join(SAMPLES, "bfs"), str(scale), str(seed)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"reached (\d+) of (\d+) vertices in (\d+) levels", r.stdout)
    assert m, r.stdout
    s, d, _ = O.rmat(scale, 16, (45, 20, 20, 15), seed=seed, drop_self_loops=False)
    lv = O.bfs_levels(1 << scale, s, d, 0)
    assert int(m.group(1)) == int((lv >= 0).sum())
    assert int(m.group(2)) == 1 << scale
    assert int(m.group(3)) == int(lv.max()) + 1
    assert "GPU perfomance" in r.stdout


@pytest.mark.gpu
def test_sssp_sample_on_a_reference_format_file(tmp_path):
    """sample/sssp <graph.el> [runs] [delta] [out]: the graph is written in the reference's edge-list format,
    the sample's distances (Bellman-Ford and delta-stepping) are checked bit for bit against the oracle."""
    V = 1 << 11
    s, d, w = O.rmat(11, 8, seed=4)
    el = str(tmp_path / "g.el")
    T.write_edges_list(el, V, s, d, w)
    for delta in ("0", "0.1"):
        out = tmp_path / f"dist_{delta}.bin"
        r = subprocess.run([os.path.join(SAMPLES, "sssp"), el, "3", delta, str(out)], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.count("GPU-only perfomance") == 3
        raw = out.read_bytes()
        rec = 4 + 4 * V
        assert len(raw) == 3 * rec
        for k in range(3):
            src = int(np.frombuffer(raw[k * rec:k * rec + 4], np.int32)[0])
            got = np.frombuffer(raw[k * rec + 4:(k + 1) * rec], np.float32)
            assert np.array_equal(got.view(np.uint32), O.bellman_ford(V, s, d, w, src).view(np.uint32)), (delta, k)
