"""The reference's other graph files: the adjacency-list binary (read and write) and the headerless pair files of
the BFS sample.  Host code only, no GPU: the reference-written fixture is read byte for byte, round-tripped, and
compared with the reference's own loader where oracle/_ref is built."""
import json
import os

import numpy as np
import pytest

import oracle as O
import pytrav as T
from conftest import GOLDEN


def test_reads_reference_written_adjacency_list():
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))["files"]
    ids, values, off, dst, w, V, directed = T.read_adjacency_list(os.path.join(GOLDEN, "adj_small.bin"))
    assert V == meta["V"] and directed
    assert ids.tolist() == list(range(V))
    assert off.tolist() == [0, 2, 3, 4, 5, 5, 6]
    src, d, wt = T.adjacency_to_edges(ids, off, dst, w)
    # the fixture was written from the golden edge list, already grouped by source
    assert src.tolist() == meta["src"] and d.tolist() == meta["dst"]
    assert np.array_equal(wt, np.array(meta["w"], np.float32))
    # vertex values are whatever the reference's Vertex<int> records held; they are carried, not interpreted
    assert len(values) == V


def test_adjacency_list_round_trip_is_byte_identical(tmp_path):
    path = os.path.join(GOLDEN, "adj_small.bin")
    ids, values, off, dst, w, V, directed = T.read_adjacency_list(path)
    out = str(tmp_path / "adj.bin")
    T.write_adjacency_list(out, ids, values, off, dst, w, directed=directed)
    assert open(out, "rb").read() == open(path, "rb").read()


def test_adjacency_list_of_an_rmat_graph_matches_the_reference_loader(tmp_path):
    if not O.ref_available():
        pytest.skip("oracle/_ref is not built")
    V = 1 << 9
    s, d, w = O.rmat(9, 8, seed=3, drop_self_loops=True)
    gc = O.RefGraph.csr_via_reference(V, s, d, w)
    p = str(tmp_path / "rmat_adj.bin")
    assert O.ref().ref_save_adjacency_list(gc.h, p.encode()) == 0
    gc.free()
    ids, values, off, dst, w2, V2, _ = T.read_adjacency_list(p)
    assert V2 == V and off[-1] == len(s)
    ref = O.RefGraph.load_adjacency_list_as_el(p)
    rs, rd, rw = ref.export_el()
    ref.free()
    src, dd, ww = T.adjacency_to_edges(ids, off, dst, w2)
    assert np.array_equal(src, rs) and np.array_equal(dd, rd) and np.array_equal(ww.view(np.uint32), rw.view(np.uint32))
    out = str(tmp_path / "again.bin")
    T.write_adjacency_list(out, ids, values, off, dst, w2)
    assert open(out, "rb").read() == open(p, "rb").read()


@pytest.mark.parametrize("mutate", ["truncate_header", "truncate_edges", "extra", "count_mismatch", "negative"])
def test_corrupt_adjacency_list_files_rejected(tmp_path, mutate):
    good = open(os.path.join(GOLDEN, "adj_small.bin"), "rb").read()
    if mutate == "truncate_header":
        data = good[:10]
    elif mutate == "truncate_edges":
        data = good[:-3]
    elif mutate == "extra":
        data = good + b"\0" * 4
    elif mutate == "count_mismatch":
        data = good[:5] + (7).to_bytes(8, "little") + good[13:]
    else:
        data = good[:13 + 8] + (-1).to_bytes(4, "little", signed=True) + good[13 + 12:]
    p = tmp_path / "bad.bin"
    p.write_bytes(data)
    with pytest.raises(T.TravError) as e:
        T.read_adjacency_list(str(p))
    assert e.value.code == T.TRAV_ERR_IO


def test_pairs_file_keeps_the_reference_edge_count(tmp_path):
    """sample/bfs.cpp:84-114 counts file_size / 12 edges and reads 8-byte pairs: 12 pairs (96 bytes) give 8
    edges, the first 8 pairs, each of weight 1.0, over 2^pow vertices."""
    pairs = np.arange(24, dtype=np.int32).reshape(12, 2) % 16
    p = tmp_path / "pairs.bin"
    p.write_bytes(pairs.tobytes())
    src, dst, w, V = T.read_pairs(str(p), 4)
    assert V == 16 and len(src) == 8
    assert src.tolist() == pairs[:8, 0].tolist() and dst.tolist() == pairs[:8, 1].tolist()
    assert np.all(w == 1.0)
    q = tmp_path / "odd.bin"
    q.write_bytes(pairs.tobytes()[:23])  # 23 bytes: one edge
    src, dst, w, V = T.read_pairs(str(q), 3)
    assert V == 8 and src.tolist() == [0] and dst.tolist() == [1]
    e = tmp_path / "empty.bin"
    e.write_bytes(b"")
    assert len(T.read_pairs(str(e), 2)[0]) == 0
    with pytest.raises(T.TravError) as ex:
        T.read_pairs(str(tmp_path / "missing.bin"), 2)
    assert ex.value.code == T.TRAV_ERR_IO
