"""Test infrastructure, not product code: numpy front end of the CPU oracle.

Loads ``oracle/liborc.so`` (the C restatement in ``trav_oracle.c``) and, when
it was built, ``oracle/_ref/libtrav_ref.so`` (the reference library's own CPU
implementations compiled from its sources).  Only tests/, ``__graft_entry__``'s
smoke check and bench.py's CPU-baseline leg import this module, and only to
check or to time the CPU side; the product path never calls it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FLT_MAX = np.float32(np.finfo(np.float32).max)

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

_orc = None
_ref = None


def lib():
    global _orc
    if _orc is None:
        path = os.path.join(HERE, "liborc.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run oracle/build.sh)")
        L = C.CDLL(path)
        L.orc_rand_r.argtypes = [C.POINTER(C.c_uint32)]
        L.orc_rand_r.restype = C.c_int
        L.orc_lcg_skip.argtypes = [C.c_uint32, C.c_uint64]
        L.orc_lcg_skip.restype = C.c_uint32
        L.orc_rmat.argtypes = [C.c_int] * 6 + [C.c_uint32, C.c_int, _i32p, _i32p, _f32p]
        L.orc_rmat.restype = None
        L.orc_drop_self_loops.argtypes = [C.c_int64, _i32p, _i32p, _f32p]
        L.orc_drop_self_loops.restype = C.c_int64
        L.orc_bellman_ford.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _f32p, C.c_int32, _f32p]
        L.orc_bellman_ford.restype = C.c_int
        L.orc_reach_masked.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, C.c_int32, _i32p, _u8p]
        L.orc_reach_masked.restype = C.c_int
        L.orc_dijkstra.argtypes = [C.c_int32, _i64p, _i32p, _f32p, C.c_int32, _f32p]
        L.orc_dijkstra.restype = None
        L.orc_build_csr.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _f32p, _i64p, _i32p, _f32p]
        L.orc_build_csr.restype = None
        L.orc_bfs_levels.argtypes = [C.c_int32, _i64p, _i32p, C.c_int32, _i32p]
        L.orc_bfs_levels.restype = C.c_int
        L.orc_device_layout.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _f32p, _i32p, _i32p,
                                        _i64p, _i32p, _f32p, _i64p, _i32p]
        L.orc_device_layout.restype = None
        L.orc_sssp_bytes.argtypes = [C.c_int32, _i64p, _f32p]
        L.orc_sssp_bytes.restype = C.c_int64
        L.orc_bfs_bytes.argtypes = [C.c_int32, _i64p, _i64p, _i32p, _i32p, _u8p, C.c_int]
        L.orc_bfs_bytes.restype = C.c_int64
        L.orc_mlp_loss_grad.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, C.c_int, _f64p, _i32p, C.c_void_p]
        L.orc_el_optimize.argtypes = [C.c_int64, _i32p, _i32p, _f32p, C.c_int32, _i32p, _i32p, _f32p]
        L.orc_el_optimize.restype = C.c_int64
        L.orc_gpu_transactions.argtypes = [C.c_int64, _i32p, _i32p, C.c_int32]
        L.orc_gpu_transactions.restype = C.c_int64
        L.orc_mlp_loss_grad.restype = C.c_double
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libtrav_ref.so"))


def ref():
    """The reference library's own CPU path (oracle/_ref/libtrav_ref.so)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libtrav_ref.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference build missing: {path} (run oracle/build_ref.sh where the reference is)")
        L = C.CDLL(path)
        vp = C.c_void_p
        L.ref_graph_el.argtypes = [C.c_int, C.c_longlong, _i32p, _i32p, _f32p]
        L.ref_graph_el.restype = vp
        L.ref_graph_csr_via_reference.argtypes = [C.c_int, C.c_longlong, _i32p, _i32p, _f32p]
        L.ref_graph_csr_via_reference.restype = vp
        L.ref_graph_csr.argtypes = [C.c_int, C.c_longlong, _i64p, _i32p, _f32p]
        L.ref_graph_csr.restype = vp
        L.ref_graph_export_csr.argtypes = [vp, _i64p, _i32p, _f32p]
        L.ref_graph_export_el.argtypes = [vp, _i32p, _i32p, _f32p]
        L.ref_graph_vertices.argtypes = [vp]
        L.ref_graph_edges.argtypes = [vp]
        L.ref_graph_edges.restype = C.c_longlong
        L.ref_graph_free.argtypes = [vp]
        L.ref_graph_free.restype = None
        L.ref_cpu_bellman_ford.argtypes = [vp, C.c_int, _f32p, C.c_int]
        L.ref_cpu_sequential_bfs.argtypes = [vp, C.c_int, _u8p]
        L.ref_cpu_parallel_bfs.argtypes = [vp, C.c_int, _u8p, C.c_int]
        L.ref_rmat_parallel.argtypes = [C.c_int] * 7 + [_i32p, _i32p, _f32p]
        L.ref_save_edges_list.argtypes = [vp, C.c_char_p]
        L.ref_save_adjacency_list.argtypes = [vp, C.c_char_p]
        L.ref_load_edges_list.argtypes = [C.c_char_p]
        L.ref_optimize_for_cpu.argtypes = [vp, C.c_int]
        L.ref_optimize_for_cpu.restype = C.c_longlong
        L.ref_gpu_transactions.argtypes = [vp, C.c_int]
        L.ref_gpu_transactions.restype = C.c_longlong
        L.ref_load_edges_list.restype = vp
        L.ref_load_adjacency_list_as_el.argtypes = [C.c_char_p]
        L.ref_load_adjacency_list_as_el.restype = vp
        L.ref_graph_vertices.restype = C.c_int
        L.ref_wtime.restype = C.c_double
        _ref = L
    return _ref


# ---------------------------------------------------------------- generators
def rmat(scale: int, avg: int, abcd=(57, 19, 19, 5), seed: int = 1, drop_self_loops: bool = True,
         threads: int = 0):
    """Seeded RMAT edge list (restatement of R_MAT_parallel); returns (src, dst, w)."""
    V = 1 << scale
    E = V * avg
    src = np.empty(E, np.int32)
    dst = np.empty(E, np.int32)
    w = np.empty(E, np.float32)
    lib().orc_rmat(scale, avg, *abcd, seed & 0xFFFFFFFF, threads or (os.cpu_count() or 1), src, dst, w)
    if drop_self_loops:
        n = lib().orc_drop_self_loops(E, src, dst, w)
        src, dst, w = src[:n].copy(), dst[:n].copy(), w[:n].copy()
    return src, dst, w


def rand_r_stream(seed: int, n: int):
    st = C.c_uint32(seed & 0xFFFFFFFF)
    return np.array([lib().orc_rand_r(C.byref(st)) for _ in range(n)], np.int64)


# ---------------------------------------------------------------- algorithms
def bellman_ford(V, src, dst, w, source):
    dist = np.empty(V, np.float32)
    lib().orc_bellman_ford(V, len(src), _c(src, np.int32), _c(dst, np.int32), _c(w, np.float32), source, dist)
    return dist


def csr(V, src, dst, w):
    off = np.empty(V + 1, np.int64)
    adj = np.empty(max(len(src), 1), np.int32)
    wt = np.empty(max(len(src), 1), np.float32)
    lib().orc_build_csr(V, len(src), _c(src, np.int32), _c(dst, np.int32), _c(w, np.float32), off, adj, wt)
    return off, adj, wt


def reach_masked(V, src, dst, pivot, trees):
    """The SCC forward-backward reachability sweep from pivot within its tree (uint8 visited)."""
    vis = np.empty(V, np.uint8)
    lib().orc_reach_masked(V, len(src), _c(src, np.int32), _c(dst, np.int32), int(pivot), _c(trees, np.int32), vis)
    return vis


def dijkstra(V, src, dst, w, source, csr_arrays=None):
    off, adj, wt = csr_arrays if csr_arrays is not None else csr(V, src, dst, w)
    dist = np.empty(V, np.float32)
    lib().orc_dijkstra(V, off, adj, wt, source, dist)
    return dist


def bfs_levels(V, src, dst, source, csr_arrays=None):
    if csr_arrays is None:
        off, adj, _ = csr(V, src, dst, np.zeros(len(src), np.float32))
    else:
        off, adj = csr_arrays[0], csr_arrays[1]
    lv = np.empty(V, np.int32)
    lib().orc_bfs_levels(V, off, adj, source, lv)
    return lv


def device_layout(V, src, dst, w):
    E = len(src)
    n2o = np.empty(V, np.int32)
    o2n = np.empty(V, np.int32)
    oo = np.empty(V + 1, np.int64)
    oa = np.empty(max(E, 1), np.int32)
    ow = np.empty(max(E, 1), np.float32)
    io = np.empty(V + 1, np.int64)
    ia = np.empty(max(E, 1), np.int32)
    lib().orc_device_layout(V, E, _c(src, np.int32), _c(dst, np.int32), _c(w, np.float32), n2o, o2n, oo, oa, ow, io, ia)
    return dict(new_of_old=n2o, old_of_new=o2n, out_off=oo, out_adj=oa[:E], out_w=ow[:E], in_off=io, in_adj=ia[:E])


def sssp_bytes(V, offsets, dist):
    return int(lib().orc_sssp_bytes(V, _c(offsets, np.int64), _c(dist, np.float32)))


def bfs_bytes(V, layout, levels_new, dirs):
    dirs = np.ascontiguousarray(dirs, np.uint8)
    return int(lib().orc_bfs_bytes(V, layout["out_off"], layout["in_off"], _c(layout["in_adj"], np.int32),
                                   _c(levels_new, np.int32), dirs, len(dirs)))


def el_optimize(src, dst, w, segment=0):
    """Graph optimisation pass: (src, dst, w) sorted by (src, dst, w) without loops and repeated arcs, then
    grouped by (src // segment, dst // segment) when segment > 0."""
    E = len(src)
    s, d, ww = _c(src, np.int32), _c(dst, np.int32), _c(w, np.float32)
    os_, od, ow = np.empty(max(E, 1), np.int32), np.empty(max(E, 1), np.int32), np.empty(max(E, 1), np.float32)
    n = lib().orc_el_optimize(E, s, d, ww, segment, os_, od, ow)
    return os_[:n].copy(), od[:n].copy(), ow[:n].copy()


def gpu_transactions(src, dst, elem_size=4):
    """Distinct 128-byte segments per warp of 32 consecutive edges, summed (the last warp excluded)."""
    return int(lib().orc_gpu_transactions(len(src), _c(src, np.int32), _c(dst, np.int32), elem_size))


def mlp_loss_grad(F, H, O, params, x, labels, want_grad=True):
    params = _c(params, np.float64)
    x = _c(x, np.float64)
    labels = _c(labels, np.int32)
    g = np.zeros_like(params) if want_grad else None
    loss = lib().orc_mlp_loss_grad(F, H, O, params, len(labels), x, labels,
                                   g.ctypes.data if g is not None else None)
    return loss, g


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------- reference wrappers
class RefGraph:
    """Handle on a reference ``Graph<int,float>`` built by the harness."""

    def __init__(self, handle, V, E):
        self.h, self.V, self.E = handle, V, E

    @classmethod
    def edges_list(cls, V, src, dst, w):
        return cls(ref().ref_graph_el(V, len(src), _c(src, np.int32), _c(dst, np.int32), _c(w, np.float32)), V, len(src))

    @classmethod
    def csr_via_reference(cls, V, src, dst, w):
        h = ref().ref_graph_csr_via_reference(V, len(src), _c(src, np.int32), _c(dst, np.int32), _c(w, np.float32))
        return cls(h, V, len(src))

    @classmethod
    def csr(cls, V, offsets, adj, w):
        return cls(ref().ref_graph_csr(V, int(offsets[-1]), _c(offsets, np.int64), _c(adj, np.int32),
                                       _c(w, np.float32)), V, int(offsets[-1]))

    @classmethod
    def load_adjacency_list_as_el(cls, path):
        """The reference's adjacency-list loader, then its conversion to an edge list."""
        h = ref().ref_load_adjacency_list_as_el(path.encode())
        assert h, f"reference loader refused {path}"
        return cls(h, ref().ref_graph_vertices(h), ref().ref_graph_edges(h))

    def export_csr(self):
        off = np.empty(self.V + 1, np.int64)
        adj = np.empty(max(self.E, 1), np.int32)
        w = np.empty(max(self.E, 1), np.float32)
        assert ref().ref_graph_export_csr(self.h, off, adj, w) == 0
        return off, adj[: self.E], w[: self.E]

    def bellman_ford(self, source, threads=1):
        d = np.empty(self.V, np.float32)
        assert ref().ref_cpu_bellman_ford(self.h, source, d, threads) == 0
        return d

    def sequential_bfs(self, source):
        r = np.empty(self.V, np.uint8)
        assert ref().ref_cpu_sequential_bfs(self.h, source, r) == 0
        return r

    def optimize_for_cpu(self, elem_size=4):
        """The reference's optimize_graph_for_CPU on this edge-list graph (in place); returns the new edge count."""
        self.E = int(ref().ref_optimize_for_cpu(self.h, elem_size))
        return self.E

    def gpu_transactions(self, elem_size=4):
        return int(ref().ref_gpu_transactions(self.h, elem_size))

    def export_el(self):
        s, d, w = np.empty(max(self.E, 1), np.int32), np.empty(max(self.E, 1), np.int32), np.empty(max(self.E, 1), np.float32)
        ref().ref_graph_export_el(self.h, s, d, w)
        return s[:self.E], d[:self.E], w[:self.E]

    def parallel_bfs(self, source, threads=0):
        r = np.empty(self.V, np.uint8)
        assert ref().ref_cpu_parallel_bfs(self.h, source, r, threads) == 0
        return r

    def free(self):
        if self.h:
            ref().ref_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def ref_rmat(V, avg, abcd=(57, 19, 19, 5), threads=1):
    E = V * avg
    src = np.empty(E, np.int32)
    dst = np.empty(E, np.int32)
    w = np.empty(E, np.float32)
    ref().ref_rmat_parallel(V, avg, *abcd, threads, src, dst, w)
    return src, dst, w


# ------------------------------------------------- the reference's GPU path
_refgpu = None


def refgpu_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libtrav_refgpu.so"))


def refgpu():
    """The reference's own bellman_ford.cu / bfs.cu built for sm_100a (oracle/_ref/libtrav_refgpu.so)."""
    global _refgpu
    if _refgpu is None:
        path = os.path.join(HERE, "_ref", "libtrav_refgpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference GPU build missing: {path} (run oracle/build_refgpu.sh where the reference is)")
        L = C.CDLL(path)
        L.refgpu_upload.argtypes = [C.c_int, C.c_longlong, _i32p, _i32p, _f32p]
        L.refgpu_upload.restype = C.c_int
        L.refgpu_sssp.argtypes = [C.c_int, _f32p]
        L.refgpu_sssp.restype = C.c_double
        L.refgpu_bfs.argtypes = [C.c_int, _u8p]
        L.refgpu_bfs.restype = C.c_double
        L.refgpu_free.argtypes = []
        L.refgpu_free.restype = None
        _refgpu = L
    return _refgpu


class quiet_stdout:
    """Send file descriptor 1 to /dev/null for a block (the reference's wrappers print with cout/printf)."""

    def __enter__(self):
        import sys

        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False
