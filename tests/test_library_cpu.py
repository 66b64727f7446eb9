"""The C-ABI library loads, exports every symbol include/trav.h declares, and its host-only parts work without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import pytrav as T
from conftest import GOLDEN, ROOT


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "trav.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(trav_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    declared = _declared_functions()
    assert declared, "no functions parsed from include/trav.h"
    out = subprocess.run(["nm", "-D", "--defined-only", T.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (trav_[a-z0-9_]+)$", out, flags=re.M))
    missing = [f for f in declared if f not in exported]
    assert not missing, f"declared but not exported: {missing}"
    assert sorted(T.EXPORTS) == declared


def test_reference_cxx_wrappers_exported():
    # the reference's C++ template wrappers, so its sssp.hpp / bfs.hpp link unchanged
    out = subprocess.run(["nm", "-DC", "--defined-only", T.LIB_PATH], capture_output=True, text=True, check=True).stdout
    for sig in ("init_distances_wrapper<float>(float*, int, int)",
                "init_distances_wrapper<double>(double*, int, int)",
                "bellman_ford_wrapper<float>(int*, int*, float*, int, long long, int, float*)",
                "bellman_ford_wrapper<double>(int*, int*, double*, int, long long, int, double*)",
                "bfs_wrapper(int*, int*, int, long long, bool*, int)"):
        assert sig in out, sig


def test_version_and_param_counts():
    assert b"sm_100a" in T.lib().trav_version()
    assert T.mlp_param_count(0) == 32 * 10 + 32 + 32 * 32 + 32 + 2 * 32 + 2
    assert T.mlp_param_count(1) == 32 * 10 + 32 + 32 * 32 + 32 + 6 * 32 + 6
    assert T.mlp_param_count(7) == -1


def test_reads_reference_written_edge_list():
    import json
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))["files"]
    src, dst, w, V, directed = T.read_edges_list(os.path.join(GOLDEN, "el_small.bin"))
    assert V == meta["V"] and directed
    assert src.tolist() == meta["src"] and dst.tolist() == meta["dst"]
    assert np.array_equal(w, np.array(meta["w"], np.float32))


def test_writes_identical_bytes(tmp_path):
    import json
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))["files"]
    p = str(tmp_path / "el.bin")
    T.write_edges_list(p, meta["V"], meta["src"], meta["dst"], meta["w"])
    assert open(p, "rb").read() == open(os.path.join(GOLDEN, "el_small.bin"), "rb").read()


def test_unweighted_records(tmp_path):
    p = tmp_path / "uw.bin"
    hdr = bytes([1]) + (4).to_bytes(4, "little") + (3).to_bytes(8, "little")
    recs = np.array([[0, 1], [1, 2], [2, 3]], np.int32).tobytes()
    p.write_bytes(hdr + recs)
    src, dst, w, V, _ = T.read_edges_list(str(p), unweighted=True)
    assert V == 4 and src.tolist() == [0, 1, 2] and dst.tolist() == [1, 2, 3] and np.all(w == 1.0)


@pytest.mark.parametrize("mutate", ["truncate", "extra", "header_mismatch", "missing"])
def test_corrupt_edge_list_files_rejected(tmp_path, mutate):
    good = open(os.path.join(GOLDEN, "el_small.bin"), "rb").read()
    p = tmp_path / "bad.bin"
    if mutate == "truncate":
        p.write_bytes(good[:-5])
    elif mutate == "extra":
        p.write_bytes(good + b"\0" * 3)
    elif mutate == "header_mismatch":
        p.write_bytes(good[:5] + (7).to_bytes(8, "little") + good[13:])
    else:
        p = tmp_path / "nope.bin"
    with pytest.raises(T.TravError) as e:
        T.read_edges_list(str(p))
    assert e.value.code == T.TRAV_ERR_IO


def test_no_device_is_a_clean_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(T.TravError) as e:
        T.Graph.from_edges(4, np.array([0, 1]), np.array([1, 2]), np.array([1.0, 1.0]))
    assert e.value.code == T.TRAV_ERR_NO_DEVICE


def test_overflow_int32_is_rejected_before_any_device_access():
    """Graphs of 2^31 or more edges do not fit the device CSR's int32 offsets: rejected from the sizes alone,
    with pointers that are never dereferenced (the reference's bfs_kernel would index them with an int)."""
    import ctypes as C

    L = T.lib()
    h = C.c_void_p()
    dummy = C.c_void_p(16)  # never read: the size check comes first
    rc = L.trav_graph_from_edges(4, 1 << 31, dummy, dummy, dummy, T.MEM_HOST, C.byref(h))
    assert rc == T.TRAV_ERR_OVERFLOW_INT32 and not h.value
    assert b"2^31" in L.trav_last_error()
    e = C.c_int64()
    rc = L.trav_graph_rmat(26, 32, 57, 19, 19, 5, 1, 1, None, None, None, C.byref(e), C.byref(h))
    assert rc == T.TRAV_ERR_OVERFLOW_INT32 and not h.value


def test_noalloc_bfs_refuses_host_pointers_without_launching():
    """The allocation-free BFS checks that its arrays are device memory before its CSR check runs on the GPU."""
    off = np.array([0, 1, 1], np.int32)
    adj = np.array([1], np.int32)
    lv = np.empty(2, np.int32)
    with pytest.raises(T.TravError) as e:
        T.bfs_csr_noalloc(off, adj, 2, 1, 0, lv)
    assert e.value.code == T.TRAV_ERR_BAD_ARG and "device" in str(e.value)


def test_tune_table_round_trip_and_rejects_malformed_files(tmp_path):
    """The autotuner's persisted shape table is host-only: load merges, save writes the same lines back."""
    good = tmp_path / "shapes.txt"
    good.write_text("# comment\nctas592_v23_e28_g0_q7_s4_l8 74 64 256\nctas592_v18_e23_g6_q9_s4_l0 8 32 128\n")
    assert T.tune_table_load(str(good)) >= 2
    out = tmp_path / "again.txt"
    T.tune_table_save(str(out))
    lines = [line for line in out.read_text().splitlines() if not line.startswith("#")]
    assert "ctas592_v23_e28_g0_q7_s4_l8 74 64 256" in lines and "ctas592_v18_e23_g6_q9_s4_l0 8 32 128" in lines
    for bad in ("key 74 64\n", "key 0 32 128\n", "key 8 32 99999\n"):
        p = tmp_path / "bad.txt"
        p.write_text(bad)
        with pytest.raises(T.TravError) as e:
            T.tune_table_load(str(p))
        assert e.value.code == T.TRAV_ERR_IO
    with pytest.raises(T.TravError):
        T.tune_table_load(str(tmp_path / "missing.txt"))
