"""Python binding of the B200 traversal library (ctypes over include/trav.h).

Mirrors the reference's operator surface for the traversal path:

* ``Graph`` -- a device graph built from an edge list (``from_edges``), a
  reference-format edge-list file (``load_edges_list``) or the seeded device
  RMAT generator (``rmat``, restating ``GraphGenerationAPI::R_MAT_parallel``,
  include/test/generation/graph_generation_API.hpp:403-484).
* ``Graph.bfs`` / ``Graph.sssp`` -- ``BFS::gpu_bfs`` (algorithm/bfs/bfs.hpp:
  212-254) and ``SingleSourceShortestPaths::gpu_bellman_ford`` (algorithm/sssp/
  sssp.hpp:219-277), batched over sources, returning levels / fp32 distances in
  the caller's vertex ids.
* ``init_distances``, ``bellman_ford_wrapper``, ``bfs_wrapper`` -- the
  reference's device-pointer wrappers (algorithm/sssp/gpu/bellman_ford.cu:
  38-144, algorithm/bfs/gpu/bfs.cu:43-81).

Errors raise ``TravError`` carrying the library's status code and message;
there is no CPU fallback: without the compiled library or a GPU the calls fail.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "libtrav_b200.so")

TRAV_OK = 0
TRAV_ERR_BAD_ARG = -1
TRAV_ERR_OOM = -2
TRAV_ERR_OVERFLOW_INT32 = -3
TRAV_ERR_TIMEOUT = -4
TRAV_ERR_CUDA = -5
TRAV_ERR_NO_DEVICE = -6
TRAV_ERR_IO = -7
MEM_HOST, MEM_DEVICE = 0, 1
SCHEDULE_PLAIN, SCHEDULE_LEARNED = 0, 1
MLP_OUTPUTS = (2, 6)  # schedule network outputs: BFS direction, SSSP bucket width delta * 4^k
FLT_MAX = np.float32(np.finfo(np.float32).max)

# Every symbol include/trav.h declares (checked by the CPU test suite).
EXPORTS = [
    "trav_graph_from_edges", "trav_graph_rmat", "trav_graph_free", "trav_graph_info", "trav_graph_export",
    "trav_graph_export_in_w",
    "trav_bfs", "trav_sssp", "trav_last_stats", "trav_last_bfs_trace", "trav_init_distances_f32",
    "trav_bellman_ford_el_f32", "trav_bfs_el", "trav_el_file_read", "trav_el_file_write", "trav_mlp_set",
    "trav_mlp_param_count", "trav_last_error", "trav_version", "trav_last_batch_ms", "trav_graph_set_stream",
    "trav_bfs_csr_noalloc", "trav_last_phase_log", "trav_mlp_loss_grad", "trav_mlp_train", "trav_set_plan",
    "trav_last_decisions", "trav_set_grid", "trav_batch_create", "trav_batch_free", "trav_batch_run",
    "trav_batch_autotune", "trav_batch_set_shape", "trav_batch_get_shape", "trav_graph_set_capture",
    "trav_el_optimize", "trav_el_gpu_transactions", "trav_adj_file_read", "trav_adj_file_write",
    "trav_pairs_file_read", "trav_set_limits", "trav_inject_alloc_failure", "trav_reach_el_masked",
    "trav_mlp_set_margin", "trav_batch_run_host", "trav_tune_table_save", "trav_tune_table_load",
    "trav_set_sssp_split", "trav_graph_mean_weight",
]


class TravError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"trav error {code}: {msg}")
        self.code = code


class BfsOpts(C.Structure):
    _fields_ = [("schedule", C.c_int32), ("alpha", C.c_float), ("beta", C.c_float), ("force_direction", C.c_int32)]


class SsspOpts(C.Structure):
    _fields_ = [("schedule", C.c_int32), ("delta", C.c_float)]


class Query(C.Structure):
    _fields_ = [("graph", C.c_int32), ("kind", C.c_int32), ("source", C.c_int32), ("delta", C.c_float),
                ("schedule", C.c_int32), ("out", C.c_void_p)]


class BatchShape(C.Structure):
    _fields_ = [("team_ctas", C.c_int32), ("small_deg", C.c_int32), ("item", C.c_int32)]

    def as_tuple(self):
        return (self.team_ctas, self.small_deg, self.item)


class QueryStats(C.Structure):
    _fields_ = [("kind", C.c_int32), ("steps", C.c_int32), ("buckets", C.c_int32), ("bottom_up_steps", C.c_int32),
                ("reached", C.c_int64), ("reached_edges", C.c_int64), ("algorithmic_bytes", C.c_int64),
                ("kernel_ms", C.c_float), ("edges_scanned", C.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python parallel-task1_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, f32 = C.c_void_p, C.c_int32, C.c_int64, C.c_float
        L.trav_last_error.restype = C.c_char_p
        L.trav_version.restype = C.c_char_p
        L.trav_graph_from_edges.argtypes = [i32, i64, vp, vp, vp, i32, C.POINTER(vp)]
        L.trav_graph_rmat.argtypes = [i32] * 6 + [C.c_uint32, i32, vp, vp, vp, C.POINTER(i64), C.POINTER(vp)]
        L.trav_graph_free.argtypes = [vp]
        L.trav_graph_info.argtypes = [vp, C.POINTER(i32), C.POINTER(i64), C.POINTER(i32)]
        L.trav_graph_export.argtypes = [vp] * 8
        L.trav_graph_export_in_w.argtypes = [vp, vp]
        L.trav_bfs.argtypes = [vp, vp, i32, C.POINTER(BfsOpts), vp, i32]
        L.trav_sssp.argtypes = [vp, vp, i32, C.POINTER(SsspOpts), vp, i32]
        L.trav_last_stats.argtypes = [vp, C.POINTER(QueryStats)]
        L.trav_last_bfs_trace.argtypes = [vp, vp, vp, i32, C.POINTER(i32)]
        L.trav_init_distances_f32.argtypes = [vp, i32, i32]
        L.trav_bellman_ford_el_f32.argtypes = [vp, vp, vp, i32, i64, i32, vp]
        L.trav_bfs_el.argtypes = [vp, vp, i32, i64, vp, i32]
        L.trav_reach_el_masked.argtypes = [vp, vp, i32, i64, vp, vp, vp]
        L.trav_el_file_read.argtypes = [C.c_char_p, i32, C.POINTER(i32), C.POINTER(i64), C.POINTER(i32), vp, vp, vp]
        L.trav_el_file_write.argtypes = [C.c_char_p, i32, i32, i64, vp, vp, vp]
        L.trav_adj_file_read.argtypes = [C.c_char_p, C.POINTER(i32), C.POINTER(i64), C.POINTER(i32)] + [vp] * 5
        L.trav_adj_file_write.argtypes = [C.c_char_p, i32, i32, i64] + [vp] * 5
        L.trav_pairs_file_read.argtypes = [C.c_char_p, i32, C.POINTER(i32), C.POINTER(i64), vp, vp, vp]
        L.trav_mlp_set.argtypes = [vp, i32, vp, i32]
        L.trav_mlp_set_margin.argtypes = [vp, i32, f32]
        L.trav_set_sssp_split.argtypes = [vp, f32]
        L.trav_graph_mean_weight.argtypes = [vp, C.POINTER(f32)]
        L.trav_set_grid.argtypes = [vp, i32, i32, C.POINTER(i32)]
        L.trav_graph_set_capture.argtypes = [vp, i32]
        L.trav_el_optimize.argtypes = [vp, vp, vp, i32, i64, i32, i32, C.POINTER(i64)]
        L.trav_el_gpu_transactions.argtypes = [vp, vp, i32, i64, i32, i32, C.POINTER(i64)]
        L.trav_batch_create.argtypes = [C.POINTER(vp), i32, C.POINTER(vp)]
        L.trav_batch_free.argtypes = [vp]
        L.trav_batch_free.restype = None
        L.trav_batch_run.argtypes = [vp, C.POINTER(Query), i32, C.POINTER(f32)]
        L.trav_batch_run_host.argtypes = [vp, C.POINTER(Query), i32, i32, C.POINTER(f32)]
        L.trav_batch_autotune.argtypes = [vp, C.POINTER(Query), i32, i32, C.POINTER(BatchShape)]
        L.trav_tune_table_save.argtypes = [C.c_char_p]
        L.trav_tune_table_load.argtypes = [C.c_char_p, C.POINTER(i32)]
        L.trav_batch_set_shape.argtypes = [vp, C.POINTER(BatchShape)]
        L.trav_batch_get_shape.argtypes = [vp, C.POINTER(BatchShape)]
        L.trav_mlp_param_count.argtypes = [i32]
        L.trav_mlp_param_count.restype = i32
        L.trav_last_batch_ms.argtypes = [vp, vp, i32, C.POINTER(i32)]
        L.trav_graph_set_stream.argtypes = [vp, vp]
        L.trav_bfs_csr_noalloc.argtypes = [vp, vp, i32, i64, i32, vp, vp]
        L.trav_last_phase_log.argtypes = [vp, vp, vp, vp, vp, i32, C.POINTER(i32)]
        L.trav_mlp_loss_grad.argtypes = [i32, vp, vp, vp, i32, vp, C.POINTER(f32)]
        L.trav_mlp_train.argtypes = [i32, vp, vp, vp, i32, i32, f32, C.POINTER(f32)]
        L.trav_set_plan.argtypes = [vp, i32, vp, i32]
        L.trav_set_limits.argtypes = [vp, i32, C.c_uint64]
        L.trav_inject_alloc_failure.argtypes = [i32]
        L.trav_last_decisions.argtypes = [vp, vp, vp, vp, vp, vp, i32, C.POINTER(i32)]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != TRAV_OK:
        raise TravError(rc, lib().trav_last_error().decode())


def _ptr(a):
    """Data pointer of a numpy array or a torch tensor (host or CUDA)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _is_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


@dataclass
class Stats:
    kind: str
    steps: int
    buckets: int
    bottom_up_steps: int
    reached: int
    reached_edges: int
    algorithmic_bytes: int
    kernel_ms: float
    edges_scanned: int


class Graph:
    """A graph resident on the current CUDA device."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        V, E, md = C.c_int32(), C.c_int64(), C.c_int32()
        _check(lib().trav_graph_info(self._h, C.byref(V), C.byref(E), C.byref(md)))
        self.V, self.E, self.max_out_degree = V.value, E.value, md.value

    # -------------------------------------------------------------- builders
    @classmethod
    def from_edges(cls, V: int, src, dst, w=None):
        """Edge list as numpy arrays (host) or CUDA tensors (device)."""
        mem = MEM_DEVICE if _is_cuda(src) else MEM_HOST
        if mem == MEM_HOST:
            src = np.ascontiguousarray(src, np.int32)
            dst = np.ascontiguousarray(dst, np.int32)
            w = None if w is None else np.ascontiguousarray(w, np.float32)
        h = C.c_void_p()
        _check(lib().trav_graph_from_edges(V, len(src), _ptr(src), _ptr(dst), _ptr(w), mem, C.byref(h)))
        return cls(h.value)

    @classmethod
    def rmat(cls, scale: int, avg: int, abcd=(57, 19, 19, 5), seed: int = 1, drop_self_loops: bool = True,
             edges_out=None):
        """Seeded device RMAT; edges_out=(src, dst, w) CUDA tensors of V*avg entries receive the edge list."""
        h = C.c_void_p()
        E = C.c_int64()
        s, d, w = edges_out if edges_out is not None else (None, None, None)
        _check(lib().trav_graph_rmat(scale, avg, *abcd, seed & 0xFFFFFFFF, int(drop_self_loops), _ptr(s), _ptr(d),
                                     _ptr(w), C.byref(E), C.byref(h)))
        g = cls(h.value)
        g.generated_edges = E.value
        return g

    @classmethod
    def load_edges_list(cls, path: str, unweighted: bool = False):
        src, dst, w, V, _directed = read_edges_list(path, unweighted)
        return cls.from_edges(V, src, dst, w)

    def free(self):
        if self._h is not None and self._h.value:
            lib().trav_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # --------------------------------------------------------------- queries
    def bfs(self, sources, out=None, schedule=SCHEDULE_PLAIN, alpha=15.0, beta=18.0, force_direction=-1):
        """Levels [n, V] (int32, -1 unreachable).  out: numpy (host) or CUDA tensor (device)."""
        src = np.ascontiguousarray(np.atleast_1d(sources), np.int32)
        if out is None:
            out = np.empty((len(src), self.V), np.int32)
        mem = MEM_DEVICE if _is_cuda(out) else MEM_HOST
        o = BfsOpts(schedule, alpha, beta, force_direction)
        _check(lib().trav_bfs(self._h, src.ctypes.data, len(src), C.byref(o), _ptr(out), mem))
        return out

    def sssp(self, sources, out=None, delta=0.0, schedule=SCHEDULE_PLAIN):
        """Distances [n, V] (fp32, FLT_MAX unreachable).  delta <= 0 or inf: Bellman-Ford."""
        src = np.ascontiguousarray(np.atleast_1d(sources), np.int32)
        if out is None:
            out = np.empty((len(src), self.V), np.float32)
        mem = MEM_DEVICE if _is_cuda(out) else MEM_HOST
        o = SsspOpts(schedule, delta)
        _check(lib().trav_sssp(self._h, src.ctypes.data, len(src), C.byref(o), _ptr(out), mem))
        return out

    def last_stats(self) -> Stats:
        s = QueryStats()
        _check(lib().trav_last_stats(self._h, C.byref(s)))
        return Stats("bfs" if s.kind == 0 else "sssp", s.steps, s.buckets, s.bottom_up_steps, s.reached,
                     s.reached_edges, s.algorithmic_bytes, s.kernel_ms, s.edges_scanned)

    def last_bfs_trace(self):
        cap = 4096
        dirs = np.zeros(cap, np.uint8)
        fr = np.zeros(cap, np.int64)
        n = C.c_int32()
        _check(lib().trav_last_bfs_trace(self._h, dirs.ctypes.data, fr.ctypes.data, cap, C.byref(n)))
        k = min(n.value, cap)
        return dirs[:k].copy(), fr[:k].copy()

    def last_batch_ms(self):
        """Device time (ms) of each launch of the last batch."""
        n = C.c_int32()
        _check(lib().trav_last_batch_ms(self._h, None, 0, C.byref(n)))
        ms = np.zeros(max(n.value, 1), np.float32)
        _check(lib().trav_last_batch_ms(self._h, ms.ctypes.data, n.value, C.byref(n)))
        return ms[: n.value]

    def set_stream(self, stream):
        """Run queries on a CUDA stream (int handle or torch.cuda.Stream); None = the handle's own."""
        h = getattr(stream, "cuda_stream", stream)
        _check(lib().trav_graph_set_stream(self._h, C.c_void_p(h) if h else None))

    def last_phase_log(self):
        """Per-phase log of the last query: (kind, frontier size, end time us, cumulative edges expanded)."""
        cap = 4096
        kind = np.zeros(cap, np.uint8)
        size = np.zeros(cap, np.int64)
        end = np.zeros(cap, np.float64)
        edges = np.zeros(cap, np.int64)
        n = C.c_int32()
        _check(lib().trav_last_phase_log(self._h, kind.ctypes.data, size.ctypes.data, end.ctypes.data,
                                         edges.ctypes.data, cap, C.byref(n)))
        k = min(n.value, cap)
        return kind[:k].copy(), size[:k].copy(), end[:k].copy(), edges[:k].copy()

    def set_capture(self, on: bool = True):
        """Record calls with device outputs into CUDA graphs and replay them while their arguments repeat."""
        _check(lib().trav_graph_set_capture(self._h, 1 if on else 0))

    def set_grid(self, kind: int, ctas: int = 0) -> int:
        """CTAs of later `kind` launches (0 = as many as fit); returns that maximum."""
        most = C.c_int32(0)
        _check(lib().trav_set_grid(self._h, kind, ctas, C.byref(most)))
        return most.value

    def set_limits(self, max_steps: int = 0, timeout_ns: int = 0):
        """Step budget and grid-barrier wait limit of later queries (0 = the defaults)."""
        _check(lib().trav_set_limits(self._h, max_steps, timeout_ns))

    def set_plan(self, kind: int, plan=None):
        """Force decisions of later queries of `kind` (0 BFS, 1 SSSP); entries of 255 follow the schedule."""
        p = np.ascontiguousarray(plan if plan is not None else [], np.uint8)
        _check(lib().trav_set_plan(self._h, kind, p.ctypes.data if len(p) else None, len(p)))

    def last_decisions(self):
        """Decisions of the last query: (features [n,10], choice, phase index, lo, hi)."""
        cap = 1024
        x = np.zeros((cap, 10), np.float32)
        ch = np.zeros(cap, np.uint8)
        ph = np.zeros(cap, np.int32)
        lo = np.zeros(cap, np.float32)
        hi = np.zeros(cap, np.float32)
        n = C.c_int32()
        _check(lib().trav_last_decisions(self._h, x.ctypes.data, ch.ctypes.data, ph.ctypes.data, lo.ctypes.data,
                                         hi.ctypes.data, cap, C.byref(n)))
        k = min(n.value, cap)
        return x[:k].copy(), ch[:k].copy(), ph[:k].copy(), lo[:k].copy(), hi[:k].copy()

    def set_mlp(self, kind: int, params):
        p = np.ascontiguousarray(params, np.float32)
        _check(lib().trav_mlp_set(self._h, kind, p.ctypes.data, len(p)))

    def set_sssp_split(self, scale: float):
        """Learned SSSP queries on this graph run with delta x scale (the learned split; 1 = the caller's delta)."""
        _check(lib().trav_set_sssp_split(self._h, float(scale)))

    @property
    def mean_weight(self) -> float:
        w = C.c_float(0.0)
        _check(lib().trav_graph_mean_weight(self._h, C.byref(w)))
        return w.value

    def set_mlp_margin(self, kind: int, margin: float):
        """Logit margin the kind's network needs to leave the plain option (0 = plain argmax)."""
        _check(lib().trav_mlp_set_margin(self._h, kind, float(margin)))

    def out_degrees(self):
        """Out-degree of every vertex in the caller's ids."""
        n2o = np.empty(self.V, np.int32)
        oo = np.empty(self.V + 1, np.int32)
        _check(lib().trav_graph_export(self._h, n2o.ctypes.data, None, oo.ctypes.data, None, None, None, None))
        return np.diff(oo)[n2o]

    def export_layout(self):
        V, E = self.V, self.E
        n2o = np.empty(V, np.int32)
        o2n = np.empty(V, np.int32)
        oo = np.empty(V + 1, np.int32)
        oa = np.empty(max(E, 1), np.int32)
        ow = np.empty(max(E, 1), np.float32)
        io = np.empty(V + 1, np.int32)
        ia = np.empty(max(E, 1), np.int32)
        _check(lib().trav_graph_export(self._h, *(x.ctypes.data for x in (n2o, o2n, oo, oa, ow, io, ia))))
        return dict(new_of_old=n2o, old_of_new=o2n, out_off=oo, out_adj=oa[:E], out_w=ow[:E], in_off=io,
                    in_adj=ia[:E])

    def export_in_w(self):
        """Weight of every in-edge, in the order of the exported in_adj."""
        iw = np.empty(max(self.E, 1), np.float32)
        _check(lib().trav_graph_export_in_w(self._h, iw.ctypes.data))
        return iw[: self.E]


def mlp_param_count(kind: int) -> int:
    return int(lib().trav_mlp_param_count(kind))


MLP_FEATURES = 10


def mlp_loss_grad(kind: int, params, x, labels):
    """(loss, gradient) of the schedule MLP on the GPU training kernels."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_FEATURES)
    y = np.ascontiguousarray(labels, np.int32)
    g = np.empty_like(p)
    loss = C.c_float()
    _check(lib().trav_mlp_loss_grad(kind, p.ctypes.data, x.ctypes.data, y.ctypes.data, len(y), g.ctypes.data,
                                    C.byref(loss)))
    return float(loss.value), g


def mlp_train(kind: int, params, x, labels, epochs: int = 500, lr: float = 1e-2):
    """Train in place with full-batch Adam on the GPU; returns (params, final loss)."""
    p = np.array(params, np.float32)
    x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_FEATURES)
    y = np.ascontiguousarray(labels, np.int32)
    loss = C.c_float()
    _check(lib().trav_mlp_train(kind, p.ctypes.data, x.ctypes.data, y.ctypes.data, len(y), epochs, lr, C.byref(loss)))
    return p, float(loss.value)


def mlp_init(kind: int, seed: int = 0):
    """Glorot-uniform weights, zero biases, in the packed layout."""
    rng = np.random.default_rng(seed)
    F, H, O = MLP_FEATURES, 32, MLP_OUTPUTS[kind]
    parts = []
    for fan_in, fan_out in ((F, H), (H, H), (H, O)):
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        parts.append(rng.uniform(-lim, lim, fan_in * fan_out))
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts).astype(np.float32)


# ----------------------------------------------- reference-shaped wrappers
def init_distances(d, V: int, source: int):
    """init_distances_wrapper<float> on a CUDA float tensor."""
    _check(lib().trav_init_distances_f32(_ptr(d), V, source))


def bellman_ford_wrapper(src, dst, w, V: int, E: int, source: int, d):
    """bellman_ford_wrapper<float> on CUDA tensors; relaxes d in place."""
    _check(lib().trav_bellman_ford_el_f32(_ptr(src), _ptr(dst), _ptr(w), V, E, source, _ptr(d)))


def bfs_wrapper(src, dst, V: int, E: int, visited, source: int):
    """bfs_wrapper on CUDA tensors; visited is a uint8/bool CUDA tensor of V entries."""
    _check(lib().trav_bfs_el(_ptr(src), _ptr(dst), V, E, _ptr(visited), source))


def inject_alloc_failure(after: int):
    """Test hook: the allocation after `after` more successful ones fails (TRAV_ERR_OOM), once; -1 disarms."""
    _check(lib().trav_inject_alloc_failure(after))


def bfs_csr_noalloc(row_offsets, adj, V: int, E: int, source: int, levels, stream=None):
    """Top-down BFS over a device CSR (CUDA int32 tensors) into `levels`, allocating nothing.

    For callers that cannot allocate device memory (memory owned by another allocator, or paths that cannot
    take cudaMalloc's synchronisation); scratch comes from the library's static 8 MiB device array, so
    V <= 262144 and E <= 16777216.  Overlapping calls race on that array.
    """
    h = getattr(stream, "cuda_stream", stream)
    _check(lib().trav_bfs_csr_noalloc(_ptr(row_offsets), _ptr(adj), V, E, source, _ptr(levels),
                                      C.c_void_p(h) if h else None))


# --------------------------------------------------------------- files
def read_edges_list(path: str, unweighted: bool = False):
    V, E, D = C.c_int32(), C.c_int64(), C.c_int32()
    p = path.encode()
    _check(lib().trav_el_file_read(p, int(unweighted), C.byref(V), C.byref(E), C.byref(D), None, None, None))
    src = np.empty(E.value, np.int32)
    dst = np.empty(E.value, np.int32)
    w = np.empty(E.value, np.float32)
    _check(lib().trav_el_file_read(p, int(unweighted), C.byref(V), C.byref(E), C.byref(D), src.ctypes.data,
                                   dst.ctypes.data, w.ctypes.data))
    return src, dst, w, V.value, bool(D.value)


def write_edges_list(path: str, V: int, src, dst, w, directed: bool = True):
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    _check(lib().trav_el_file_write(path.encode(), int(directed), V, len(src), src.ctypes.data, dst.ctypes.data,
                                    w.ctypes.data))


def read_adjacency_list(path: str):
    """The reference's adjacency-list binary: (ids, values, offsets, dst, w, V, directed); row v's edges are
    dst/w[offsets[v]:offsets[v+1]] in file order and its source vertex is ids[v]."""
    V, E, D = C.c_int32(), C.c_int64(), C.c_int32()
    p = path.encode()
    _check(lib().trav_adj_file_read(p, C.byref(V), C.byref(E), C.byref(D), None, None, None, None, None))
    ids = np.empty(V.value, np.int32)
    values = np.empty(V.value, np.int32)
    off = np.empty(V.value + 1, np.int64)
    dst = np.empty(max(E.value, 1), np.int32)
    w = np.empty(max(E.value, 1), np.float32)
    _check(lib().trav_adj_file_read(p, C.byref(V), C.byref(E), C.byref(D), ids.ctypes.data, values.ctypes.data,
                                    off.ctypes.data, dst.ctypes.data, w.ctypes.data))
    return ids, values, off, dst[: E.value], w[: E.value], V.value, bool(D.value)


def write_adjacency_list(path: str, ids, values, offsets, dst, w, directed: bool = True):
    ids = np.ascontiguousarray(ids, np.int32)
    values = np.ascontiguousarray(values, np.int32)
    offsets = np.ascontiguousarray(offsets, np.int64)
    dst = np.ascontiguousarray(dst, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    _check(lib().trav_adj_file_write(path.encode(), int(directed), len(ids), int(offsets[-1]), ids.ctypes.data,
                                     values.ctypes.data, offsets.ctypes.data, dst.ctypes.data, w.ctypes.data))


def adjacency_to_edges(ids, offsets, dst, w):
    """Edge list (src, dst, w) of an adjacency list, rows in file order."""
    src = np.repeat(np.asarray(ids, np.int32), np.diff(np.asarray(offsets, np.int64)))
    return src, np.asarray(dst, np.int32), np.asarray(w, np.float32)


def read_pairs(path: str, vertices_pow: int):
    """Headerless {int32 src, int32 dst} pairs as the reference's BFS sample reads them: (src, dst, w, V) with
    V = 2^vertices_pow, the first file_size / 12 pairs and every weight 1.0."""
    V, E = C.c_int32(), C.c_int64()
    p = path.encode()
    _check(lib().trav_pairs_file_read(p, vertices_pow, C.byref(V), C.byref(E), None, None, None))
    src = np.empty(max(E.value, 1), np.int32)
    dst = np.empty(max(E.value, 1), np.int32)
    w = np.empty(max(E.value, 1), np.float32)
    _check(lib().trav_pairs_file_read(p, vertices_pow, C.byref(V), C.byref(E), src.ctypes.data, dst.ctypes.data,
                                      w.ctypes.data))
    return src[: E.value], dst[: E.value], w[: E.value], V.value


class Batch:
    """Many BFS / SSSP queries over several graphs in one persistent launch.

    queries: iterable of (graph index, kind 0 BFS / 1 SSSP, source, delta,
    schedule, out) with `out` a CUDA tensor of the graph's V results (int32
    levels or float32 distances).
    """

    def __init__(self, graphs):
        self.graphs = list(graphs)  # kept alive while the batch exists
        hs = (C.c_void_p * len(self.graphs))(*[g._h.value for g in self.graphs])
        h = C.c_void_p()
        _check(lib().trav_batch_create(hs, len(self.graphs), C.byref(h)))
        self._h = h

    def close(self):
        if self._h is not None and self._h.value:
            lib().trav_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _queries(queries, host=False):
        qs = list(queries)
        arr = (Query * max(1, len(qs)))()
        for i, (gi, kind, src, delta, sched, out) in enumerate(qs):
            assert _is_cuda(out) != host, "batch results must be " + ("host arrays" if host else "CUDA tensors")
            arr[i] = Query(gi, kind, int(src), float(delta), sched, _ptr(out))
        return arr, len(qs)

    def run(self, queries) -> float:
        """Run the queries in one launch; returns its device time in ms."""
        arr, n = self._queries(queries)
        ms = C.c_float(0.0)
        _check(lib().trav_batch_run(self._h, arr, n, C.byref(ms)))
        return ms.value

    def run_host(self, queries, parts: int = 1) -> float:
        """Run queries whose `out` is host memory (pinned tensors or numpy arrays; pinned memory lets the copies
        overlap the work).  Each query's results are copied back as soon as the kernel flags it done, while the
        launch runs on; `parts` > 1 cuts the queries into that many shrinking launches.  Returns the summed
        device time in ms."""
        arr, n = self._queries(queries, host=True)
        ms = C.c_float(0.0)
        _check(lib().trav_batch_run_host(self._h, arr, n, parts, C.byref(ms)))
        return ms.value

    def autotune(self, queries, reps: int = 2):
        """Time candidate launch shapes on these queries; keeps and returns the fastest (team_ctas, small_deg, item).
        reps=0 takes the tuning table's shape for this kind of batch when it has one."""
        arr, n = self._queries(queries)
        best = BatchShape()
        _check(lib().trav_batch_autotune(self._h, arr, n, reps, C.byref(best)))
        return best.as_tuple()

    @property
    def shape(self):
        s = BatchShape()
        _check(lib().trav_batch_get_shape(self._h, C.byref(s)))
        return s.as_tuple()

    @shape.setter
    def shape(self, value):
        s = BatchShape(*value)
        _check(lib().trav_batch_set_shape(self._h, C.byref(s)))


def el_optimize(src, dst, w, vertices: int, segment: int = 0):
    """The optimisation pass, in place on int32 src / dst and float32 w (numpy arrays or CUDA tensors); returns
    the new edge count (the first that many entries hold the result)."""
    n = C.c_int64(0)
    mem = MEM_DEVICE if _is_cuda(src) else MEM_HOST
    _check(lib().trav_el_optimize(_ptr(src), _ptr(dst), _ptr(w), vertices, len(src), segment, mem, C.byref(n)))
    return n.value


def el_gpu_transactions(src, dst, vertices: int, elem_size: int = 4) -> int:
    """Memory transactions of an edge-per-thread sweep over src / dst (numpy arrays or CUDA tensors)."""
    n = C.c_int64(0)
    mem = MEM_DEVICE if _is_cuda(src) else MEM_HOST
    _check(lib().trav_el_gpu_transactions(_ptr(src), _ptr(dst), vertices, len(src), elem_size, mem, C.byref(n)))
    return n.value


# ------------------------------------------------------- launch-shape table
TUNE_TABLE = os.path.join(PKG, "weights", "batch_shapes.txt")


def tune_table_save(path: str = TUNE_TABLE):
    """Write the process's table of autotuned batch launch shapes."""
    _check(lib().trav_tune_table_save(path.encode()))


def tune_table_load(path: str = TUNE_TABLE) -> int:
    """Merge a saved table of batch launch shapes into the process's; returns the table's size."""
    n = C.c_int32(0)
    _check(lib().trav_tune_table_load(path.encode(), C.byref(n)))
    return n.value
