"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference library's own CPU implementations, compiled from its
sources by oracle/build_ref.sh into oracle/_ref/libtrav_ref.so:

* R_MAT_parallel with one thread (seed 0 by construction of the reference)
  -> ``rmat_ref_s8_ef8.npz`` (the full edge list) and SHA-256 digests of
  larger runs in ``golden.json``;
* cpu_bellman_ford distances and cpu_sequential_bfs / cpu_parallel_bfs
  reachability on hand-made edge cases and seeded RMAT graphs
  -> ``cases.npz`` + ``golden.json``;
* save_to_edges_list_bin_file / save_to_adjacency_list_bin_file bytes of a
  small graph -> ``el_small.bin``, ``adj_small.bin``.

The seeded RMAT graphs are produced by the oracle's restatement of the
generator, whose seed-0 output is itself pinned to the reference above.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

F32MAX = np.finfo(np.float32).max


def hand_cases():
    """(name, V, src, dst, w, sources) edge cases the reference handles."""
    cases = []
    # chain 0->1->...->9
    cases.append(("chain", 10, np.arange(9), np.arange(1, 10), np.full(9, 0.5), [0, 5, 9]))
    # star out of 0 plus a back edge
    cases.append(("star", 8, np.zeros(7, int), np.arange(1, 8), np.linspace(0.1, 0.7, 7), [0, 3]))
    # two components
    cases.append(("disconnected", 8, np.array([0, 1, 2, 4, 5, 6]), np.array([1, 2, 3, 5, 6, 7]),
                  np.array([1, 2, 3, 1, 2, 3], float), [0, 4, 7]))
    # duplicate edges with different weights, self-loops, zero weights
    cases.append(("dups_loops_zero", 6, np.array([0, 0, 0, 1, 1, 2, 3, 3, 4, 4, 5]),
                  np.array([1, 1, 1, 1, 2, 3, 3, 4, 5, 0, 5]),
                  np.array([0.9, 0.3, 0.6, 0.0, 0.0, 0.25, 0.0, 1.0, 0.5, 0.125, 0.0]), [0, 3]))
    # weights near FLT_MAX: sums overflow to +inf and must never relax
    cases.append(("flt_max_boundary", 5, np.array([0, 1, 0, 2, 3]), np.array([1, 2, 2, 3, 4]),
                  np.array([3.0e38, 3.0e38, 1.0, F32MAX, 1.0e-45]), [0, 1]))
    # rounding: many paths whose left-folded sums differ in the last bit
    rng = np.random.default_rng(7)
    V = 64
    s = rng.integers(0, V, 2048)
    d = rng.integers(0, V, 2048)
    w = rng.random(2048).astype(np.float32) * np.float32(1e-3) + np.float32(1.0)
    cases.append(("rounding_dense", V, s, d, w, [0, 17, 63]))
    # single vertex, no edges
    cases.append(("single_vertex", 1, np.array([], int), np.array([], int), np.array([], float), [0]))
    return cases


def rmat_cases():
    out = []
    for scale, avg, seed, nsrc in [(10, 8, 1, 4), (12, 16, 1, 4), (14, 8, 3, 2)]:
        s, d, w = O.rmat(scale, avg, seed=seed, drop_self_loops=True)
        V = 1 << scale
        deg = np.bincount(s, minlength=V)
        rng = np.random.default_rng(seed)
        srcs = [int(deg.argmax())] + [int(x) for x in rng.choice(np.flatnonzero(deg), nsrc - 1, replace=False)]
        out.append((f"rmat_s{scale}_ef{avg}_seed{seed}", V, s, d, w, srcs))
    return out


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def optimize_fixture():
    """An edge list with loops, repeated arcs (some with equal weights), zero weights and ids spread over four
    of the reference's CPU cache segments (65,536 vertices at elem_size 4); the reference's
    optimize_graph_for_CPU result and check_gpu_memory_transactions_count before and after."""
    rng = np.random.default_rng(17)
    V, E = 250000, 20011
    s = rng.integers(0, V, E).astype(np.int32)
    d = rng.integers(0, V, E).astype(np.int32)
    w = (rng.integers(0, 8, E) / 8).astype(np.float32)
    s[:300] = d[:300]                          # loops
    s[300:1300], d[300:1300] = s[1300:2300], d[1300:2300]  # repeated arcs
    g = O.RefGraph.edges_list(V, s, d, w)
    before = {str(k): g.gpu_transactions(k) for k in (4, 8)}
    n = g.optimize_for_cpu(4)
    os_, od, ow = g.export_el()
    after = {str(k): g.gpu_transactions(k) for k in (4, 8)}
    g.free()
    np.savez_compressed(os.path.join(HERE, "el_optimize.npz"), src=s, dst=d, w=w, ref_src=os_, ref_dst=od, ref_w=ow)
    return {"V": V, "E": E, "E_after": int(n), "segment": 262144 // 4, "transactions_before": before,
            "transactions_after_reference_order": after}


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libtrav_ref.so is missing: run oracle/build_ref.sh first")
    meta = {"rmat_ref": {}, "cases": {}}
    arrays = {}

    # --- reference RMAT, one thread
    s, d, w = O.ref_rmat(256, 8, threads=1)
    np.savez_compressed(os.path.join(HERE, "rmat_ref_s8_ef8.npz"), src=s, dst=d, w=w)
    for scale, avg in [(12, 16), (16, 16)]:
        s, d, w = O.ref_rmat(1 << scale, avg, threads=1)
        meta["rmat_ref"][f"s{scale}_ef{avg}"] = {"edges": int(len(s)), "sha256": digest(s, d, w)}

    # --- traversal results from the reference
    for name, V, s, d, w, sources in hand_cases() + rmat_cases():
        s = np.asarray(s, np.int32)
        d = np.asarray(d, np.int32)
        w = np.asarray(w, np.float32)
        gel = O.RefGraph.edges_list(V, s, d, w)
        gcsr = O.RefGraph.csr_via_reference(V, s, d, w)
        entry = {"V": V, "E": int(len(s)), "sources": sources, "el_sha256": digest(s, d, w)}
        small = len(s) <= 20000
        if small:
            arrays[f"{name}/src"], arrays[f"{name}/dst"], arrays[f"{name}/w"] = s, d, w
        dist = np.stack([gel.bellman_ford(x, threads=1) for x in sources])
        vis = np.stack([gcsr.sequential_bfs(x) for x in sources])
        visp = np.stack([gcsr.parallel_bfs(x, threads=4) for x in sources])
        assert np.array_equal(vis, visp), name
        arrays[f"{name}/dist"] = dist
        arrays[f"{name}/visited"] = vis
        entry["stored_edges"] = small
        meta["cases"][name] = entry
        gel.free()
        gcsr.free()
    np.savez_compressed(os.path.join(HERE, "cases.npz"), **arrays)

    # --- file formats written by the reference
    V = 6
    s = np.array([0, 0, 1, 2, 3, 5], np.int32)
    d = np.array([1, 2, 3, 3, 4, 0], np.int32)
    w = np.array([0.5, 1.5, 0.25, 2.0, 0.125, 3.0], np.float32)
    g = O.RefGraph.edges_list(V, s, d, w)
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "el.bin")
        assert O.ref().ref_save_edges_list(g.h, p.encode()) == 0
        with open(p, "rb") as f:
            el = f.read()
    gc = O.RefGraph.csr_via_reference(V, s, d, w)
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "adj.bin")
        assert O.ref().ref_save_adjacency_list(gc.h, p.encode()) == 0
        with open(p, "rb") as f:
            adj = f.read()
    with open(os.path.join(HERE, "el_small.bin"), "wb") as f:
        f.write(el)
    with open(os.path.join(HERE, "adj_small.bin"), "wb") as f:
        f.write(adj)
    meta["files"] = {"V": V, "src": s.tolist(), "dst": d.tolist(), "w": w.tolist()}

    # --- graph optimisation pass: the reference's optimize_graph_for_CPU and its transaction count
    meta["optimize"] = optimize_fixture()
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote golden fixtures:", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
