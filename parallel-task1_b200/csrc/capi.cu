// C ABI of the traversal library (declared in include/trav.h).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "trav_internal.cuh"
#include "mlp_device.cuh"

#include "handle.cuh"

namespace trav {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

int cuda_fail(cudaError_t e, const char *what)
{
    g_err = std::string("CUDA error: ") + cudaGetErrorString(e) + " at " + what;
    if (e == cudaErrorMemoryAllocation) return TRAV_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return TRAV_ERR_NO_DEVICE;
    return TRAV_ERR_CUDA;
}

// Allocations left before the injected failure (-1: none armed).
static std::atomic<int64_t> g_alloc_fail_after{-1};

cudaError_t dev_malloc_bytes(void **p, size_t bytes)
{
    int64_t left = g_alloc_fail_after.load();
    while (left >= 0) {
        if (g_alloc_fail_after.compare_exchange_weak(left, left - 1)) {
            if (left == 0) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;  // fires once, then the injection is disarmed
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
}

bool is_device_ptr(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace trav

using namespace trav;

#define TRY_CUDA(expr)                                      \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

#define TRY(expr)                  \
    do {                           \
        int _rc = (expr);          \
        if (_rc != TRAV_OK) return _rc; \
    } while (0)

namespace {

int bad(const char *msg)
{
    set_error(msg);
    return TRAV_ERR_BAD_ARG;
}

int check_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error("no CUDA device available");
        return TRAV_ERR_NO_DEVICE;
    }
    return TRAV_OK;
}

// Finish a new handle from a built device graph.
int finish_handle(trav_graph *h)
{
    h->new_of_old.resize((size_t)h->g.V);
    if (h->g.V > 0)
        TRY_CUDA(cudaMemcpy(h->new_of_old.data(), h->g.new_of_old, sizeof(int32_t) * (size_t)h->g.V,
                            cudaMemcpyDeviceToHost));
    TRY(workspace_ensure(&h->ws, h->g, 1, h->st));
    for (int b = 0; b < 2; b++) {
        TRY_CUDA(dev_malloc(&h->staging[b], sizeof(float) * (size_t)(h->g.V > 0 ? h->g.V : 1)));
        TRY_CUDA(cudaEventCreateWithFlags(&h->done[b], cudaEventDisableTiming));
        TRY_CUDA(cudaEventCreateWithFlags(&h->copied[b], cudaEventDisableTiming));
    }
    TRY_CUDA(cudaStreamCreateWithFlags(&h->cst, cudaStreamNonBlocking));
    TRY_CUDA(cudaStreamSynchronize(h->st));
    return TRAV_OK;
}

void destroy(trav_graph *h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->cst) cudaStreamSynchronize(h->cst);
    free_graph(&h->g);
    workspace_free(&h->ws);
    for (int b = 0; b < 2; b++) {
        cudaFree(h->staging[b]);
        if (h->done[b]) cudaEventDestroy(h->done[b]);
        if (h->copied[b]) cudaEventDestroy(h->copied[b]);
    }
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    for (auto &c : h->cap)
        if (c.exec) cudaGraphExecDestroy(c.exec);
    cudaFree(h->mlp[0]);
    cudaFree(h->mlp[1]);
    if (h->cst) cudaStreamDestroy(h->cst);
    if (h->own_st) cudaStreamDestroy(h->own_st);
    delete h;
}

int new_handle(trav_graph **out)
{
    TRY(check_device());
    trav_graph *h = new (std::nothrow) trav_graph();
    if (!h) {
        set_error("host allocation failed");
        return TRAV_ERR_OOM;
    }
    cudaGetDevice(&h->device);
    cudaError_t e = cudaStreamCreateWithFlags(&h->own_st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    h->st = h->own_st;
    *out = h;
    return TRAV_OK;
}

template <class T>
void put(std::vector<unsigned char> &k, const T &v)
{
    const unsigned char *p = reinterpret_cast<const unsigned char *>(&v);
    k.insert(k.end(), p, p + sizeof(T));
}

// Everything a captured call's launches depend on besides the graph itself.
std::vector<unsigned char> capture_key(const trav_graph *g, int kind, const int32_t *sources, int32_t n,
                                       const trav_bfs_opts *bo, float delta, const float *mlp, const void *out)
{
    std::vector<unsigned char> k;
    put(k, kind);
    put(k, n);
    for (int32_t i = 0; i < n; i++) put(k, sources[i]);
    put(k, out);
    put(k, mlp);
    put(k, delta);
    if (bo) put(k, *bo);
    put(k, g->ws.grid[kind]);
    put(k, g->ws.small_deg);
    put(k, g->ws.item);
    put(k, g->ws.plan[kind]);
    put(k, g->ws.plan_len[kind]);
    put(k, g->ws.max_steps);
    put(k, g->ws.split_scale);
    put(k, g->ws.light.nlight);
    put(k, g->ws.light.loff);
    put(k, g->ws.light.ledge);
    put(k, g->ws.timeout_ns);
    put(k, g->st);
    put(k, g->ws.ctl);
    return k;
}

// Run n queries of one kind.  Device outputs go straight to out + q*V; host
// outputs are written to a double-buffered device staging area and copied on
// a second stream, so the copy of query q overlaps the traversal of q+1
// (fully when `out` is pinned host memory).  With capture on, a call with
// device outputs is recorded into a CUDA graph the first time and replayed
// while its arguments repeat.
int run_batch(trav_graph *g, int kind, const int32_t *sources, int32_t n, const trav_bfs_opts *bo, float delta,
              const float *mlp, void *out, int32_t mem)
{
    TRY_CUDA(cudaSetDevice(g->device));
    TRY(workspace_ensure(&g->ws, g->g, n, g->st));
    while ((int)g->ev.size() < 2 * n) {
        cudaEvent_t e;
        TRY_CUDA(cudaEventCreate(&e));
        g->ev.push_back(e);
    }
    const size_t V = (size_t)g->g.V;
    unsigned char *base = static_cast<unsigned char *>(out);
    auto enqueue = [&]() -> int {
        for (int32_t q = 0; q < n; q++) {
            const int32_t s_new = g->new_of_old[(size_t)sources[q]];
            void *dst;
            const int b = q & 1;
            if (mem == TRAV_MEM_DEVICE) {
                dst = base + 4 * V * (size_t)q;
            } else {
                if (q >= 2) TRY_CUDA(cudaStreamWaitEvent(g->st, g->copied[b], 0));
                dst = g->staging[b];
            }
            if (kind == 0) TRY(launch_bfs(g->g, &g->ws, q, s_new, *bo, mlp, dst, 0, g->st, g->ev[2 * q], g->ev[2 * q + 1]));
            else TRY(launch_sssp(g->g, &g->ws, q, s_new, delta, mlp, dst, 1, g->st, g->ev[2 * q], g->ev[2 * q + 1]));
            if (mem == TRAV_MEM_HOST) {
                TRY_CUDA(cudaEventRecord(g->done[b], g->st));
                TRY_CUDA(cudaStreamWaitEvent(g->cst, g->done[b], 0));
                TRY_CUDA(cudaMemcpyAsync(base + 4 * V * (size_t)q, dst, 4 * V, cudaMemcpyDeviceToHost, g->cst));
                TRY_CUDA(cudaEventRecord(g->copied[b], g->cst));
            }
        }
        return TRAV_OK;
    };
    if (g->capture && mem == TRAV_MEM_DEVICE) {
        trav_graph::Captured &c = g->cap[kind];
        // the light rows of delta are built before the capture (it allocates
        // and synchronises); the graph bakes in their addresses, which are part
        // of the key, so a rebuild for another delta records a new graph
        if (kind == 1 && delta > 0.0f && std::isfinite(delta))
            TRY(light_rows_build(g->g, mlp ? delta * g->ws.split_scale : delta, &g->ws.light, g->st));
        std::vector<unsigned char> key = capture_key(g, kind, sources, n, bo, delta, mlp, out);
        if (!c.exec || c.key != key) {
            if (c.exec) cudaGraphExecDestroy(c.exec);
            c.exec = nullptr;
            c.key.clear();
            TRY_CUDA(cudaStreamBeginCapture(g->st, cudaStreamCaptureModeThreadLocal));
            const int rc = enqueue();
            cudaGraph_t graph = nullptr;
            const cudaError_t e = cudaStreamEndCapture(g->st, &graph);
            if (rc != TRAV_OK) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            const cudaError_t ei = cudaGraphInstantiate(&c.exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
            c.key = std::move(key);
        }
        TRY_CUDA(cudaGraphLaunch(c.exec, g->st));
    } else {
        TRY(enqueue());
    }
    TRY_CUDA(cudaStreamSynchronize(g->st));
    TRY_CUDA(cudaStreamSynchronize(g->cst));
    g->last_kind = kind;
    g->last_n = n;
    TRY(check_queries(&g->ws, n, kind == 0 ? "bfs" : "sssp"));
    g->batch_ms.assign((size_t)n, 0.0f);
    for (int32_t q = 0; q < n; q++) TRY_CUDA(cudaEventElapsedTime(&g->batch_ms[(size_t)q], g->ev[2 * q], g->ev[2 * q + 1]));
    return TRAV_OK;
}

template <class T>
struct DevTmp {
    T *p = nullptr;
    ~DevTmp() { if (p) cudaFree(p); }
};

int check_sources(const trav_graph *h, const int32_t *sources, int32_t n)
{
    if (!sources || n < 0) return bad("sources must be a host array of n >= 0 vertex ids");
    for (int32_t i = 0; i < n; i++)
        if (sources[i] < 0 || sources[i] >= h->g.V) return bad("source vertex out of range [0, V)");
    return TRAV_OK;
}

}  // namespace

extern "C" {

const char *trav_last_error(void) { return g_err.c_str(); }

const char *trav_version(void) { return "trav-b200 0.1 (sm_100a)"; }

int trav_inject_alloc_failure(int32_t after)
{
    if (after < -1) return bad("after must be >= -1");
    g_alloc_fail_after.store(after);
    return TRAV_OK;
}

int trav_graph_from_edges(int32_t vertices, int64_t edges, const int32_t *src, const int32_t *dst, const float *w,
                          int32_t mem, trav_graph **out)
{
    if (!out) return bad("out must not be NULL");
    *out = nullptr;
    if (vertices < 1) return bad("vertices must be >= 1");
    if (edges < 0) return bad("edges must be >= 0");
    if (edges >= (int64_t)INT32_MAX) {
        set_error("graph has 2^31 or more edges; the device CSR uses int32 offsets");
        return TRAV_ERR_OVERFLOW_INT32;
    }
    if (edges > 0 && (!src || !dst)) return bad("src and dst must not be NULL");
    if (mem != TRAV_MEM_HOST && mem != TRAV_MEM_DEVICE) return bad("mem must be TRAV_MEM_HOST or TRAV_MEM_DEVICE");
    trav_graph *h = nullptr;
    TRY(new_handle(&h));
    std::unique_ptr<trav_graph, void (*)(trav_graph *)> guard(h, destroy);
    DevTmp<int32_t> ds, dd;
    DevTmp<float> dw;
    const int32_t *ps = src, *pd = dst;
    const float *pw = w;
    if (mem == TRAV_MEM_HOST && edges > 0) {
        TRY_CUDA(dev_malloc(&ds.p, sizeof(int32_t) * (size_t)edges));
        TRY_CUDA(dev_malloc(&dd.p, sizeof(int32_t) * (size_t)edges));
        TRY_CUDA(cudaMemcpyAsync(ds.p, src, sizeof(int32_t) * (size_t)edges, cudaMemcpyHostToDevice, h->st));
        TRY_CUDA(cudaMemcpyAsync(dd.p, dst, sizeof(int32_t) * (size_t)edges, cudaMemcpyHostToDevice, h->st));
        if (w) {
            TRY_CUDA(dev_malloc(&dw.p, sizeof(float) * (size_t)edges));
            TRY_CUDA(cudaMemcpyAsync(dw.p, w, sizeof(float) * (size_t)edges, cudaMemcpyHostToDevice, h->st));
        }
        ps = ds.p;
        pd = dd.p;
        pw = dw.p;
    }
    TRY(build_graph_device(vertices, edges, ps, pd, pw, h->st, &h->g));
    TRY(finish_handle(h));
    *out = guard.release();
    return TRAV_OK;
}

int trav_graph_rmat(int32_t scale, int32_t avg, int32_t a, int32_t b, int32_t c, int32_t d, uint32_t seed,
                    int32_t drop_self_loops, int32_t *src, int32_t *dst, float *w, int64_t *edges_out,
                    trav_graph **out)
{
    if (scale < 1 || scale > 30) return bad("scale must be in [1, 30]");
    if (avg < 1) return bad("avg must be >= 1");
    const int64_t E = ((int64_t)1 << scale) * avg;
    if (E >= (int64_t)INT32_MAX) {
        set_error("graph has 2^31 or more edges; the device CSR uses int32 offsets");
        return TRAV_ERR_OVERFLOW_INT32;
    }
    if ((src || dst || w) && !(src && dst && w)) return bad("src, dst and w must be all NULL or all device buffers");
    if (src && !(is_device_ptr(src) && is_device_ptr(dst) && is_device_ptr(w)))
        return bad("src, dst and w must be device buffers");
    trav_graph *h = nullptr;
    TRY(new_handle(&h));
    std::unique_ptr<trav_graph, void (*)(trav_graph *)> guard(h, destroy);
    DevTmp<int32_t> ds, dd;
    DevTmp<float> dw;
    int32_t *ps = src, *pd = dst;
    float *pw = w;
    if (!src) {
        TRY_CUDA(dev_malloc(&ds.p, sizeof(int32_t) * (size_t)E));
        TRY_CUDA(dev_malloc(&dd.p, sizeof(int32_t) * (size_t)E));
        TRY_CUDA(dev_malloc(&dw.p, sizeof(float) * (size_t)E));
        ps = ds.p;
        pd = dd.p;
        pw = dw.p;
    }
    int64_t En = 0;
    TRY(rmat_device(scale, avg, a, b, c, d, seed, drop_self_loops, ps, pd, pw, &En, h->st));
    if (edges_out) *edges_out = En;
    if (!out) return TRAV_OK;  // generation only
    TRY(build_graph_device((int32_t)1 << scale, En, ps, pd, pw, h->st, &h->g));
    TRY(finish_handle(h));
    *out = guard.release();
    return TRAV_OK;
}

int trav_graph_free(trav_graph *g)
{
    destroy(g);
    return TRAV_OK;
}

int trav_graph_info(const trav_graph *g, int32_t *vertices, int64_t *edges, int32_t *max_out_degree)
{
    if (!g) return bad("graph handle is NULL");
    if (vertices) *vertices = g->g.V;
    if (edges) *edges = g->g.E;
    if (max_out_degree) *max_out_degree = g->g.max_out_degree;
    return TRAV_OK;
}

int trav_graph_mean_weight(const trav_graph *g, float *mean_weight)
{
    if (!g || !mean_weight) return bad("graph handle and mean_weight must not be NULL");
    *mean_weight = g->g.mean_w;
    return TRAV_OK;
}

int trav_set_sssp_split(trav_graph *g, float scale)
{
    if (!g) return bad("graph handle is NULL");
    if (!(scale > 0.0f) || !std::isfinite(scale)) return bad("scale must be finite and > 0");
    TRY_CUDA(cudaSetDevice(g->device));
    TRY_CUDA(cudaStreamSynchronize(g->st));
    g->ws.split_scale = scale;
    return TRAV_OK;
}

int trav_graph_export(const trav_graph *g, int32_t *new_of_old, int32_t *old_of_new, int32_t *out_off,
                      int32_t *out_adj, float *out_w, int32_t *in_off, int32_t *in_adj)
{
    if (!g) return bad("graph handle is NULL");
    TRY_CUDA(cudaSetDevice(g->device));
    const size_t V = (size_t)g->g.V, E = (size_t)g->g.E;
    if (new_of_old) TRY_CUDA(cudaMemcpy(new_of_old, g->g.new_of_old, 4 * V, cudaMemcpyDeviceToHost));
    if (old_of_new) TRY_CUDA(cudaMemcpy(old_of_new, g->g.old_of_new, 4 * V, cudaMemcpyDeviceToHost));
    if (out_off) TRY_CUDA(cudaMemcpy(out_off, g->g.out_off, 4 * (V + 1), cudaMemcpyDeviceToHost));
    if (in_off) TRY_CUDA(cudaMemcpy(in_off, g->g.in_off, 4 * (V + 1), cudaMemcpyDeviceToHost));
    if (E) {
        if (out_adj) TRY_CUDA(cudaMemcpy(out_adj, g->g.out_adj, 4 * E, cudaMemcpyDeviceToHost));
        if (out_w) TRY_CUDA(cudaMemcpy(out_w, g->g.out_w, 4 * E, cudaMemcpyDeviceToHost));
        if (in_adj) TRY_CUDA(cudaMemcpy(in_adj, g->g.in_adj, 4 * E, cudaMemcpyDeviceToHost));
    }
    return TRAV_OK;
}

int trav_graph_export_in_w(const trav_graph *g, float *in_w)
{
    if (!g) return bad("graph handle is NULL");
    if (!in_w && g->g.E > 0) return bad("in_w must not be NULL");
    TRY_CUDA(cudaSetDevice(g->device));
    if (g->g.E > 0) TRY_CUDA(cudaMemcpy(in_w, g->g.in_w, 4 * (size_t)g->g.E, cudaMemcpyDeviceToHost));
    return TRAV_OK;
}

int trav_bfs(trav_graph *g, const int32_t *sources, int32_t n, const trav_bfs_opts *opts, int32_t *levels,
             int32_t mem)
{
    if (!g) return bad("graph handle is NULL");
    if (!levels && n > 0) return bad("levels must not be NULL");
    if (mem != TRAV_MEM_HOST && mem != TRAV_MEM_DEVICE) return bad("mem must be TRAV_MEM_HOST or TRAV_MEM_DEVICE");
    TRY(check_sources(g, sources, n));
    trav_bfs_opts o{TRAV_SCHEDULE_PLAIN, 15.0f, 18.0f, -1};
    if (opts) o = *opts;
    if (!(o.alpha > 0.0f) || !(o.beta > 0.0f)) return bad("alpha and beta must be > 0");
    if (o.force_direction < -1 || o.force_direction > 1) return bad("force_direction must be -1, 0 or 1");
    const float *mlp = nullptr;
    if (o.schedule == TRAV_SCHEDULE_LEARNED) {
        if (!g->mlp[0]) return bad("learned BFS schedule requested but no BFS MLP is loaded (trav_mlp_set)");
        mlp = g->mlp[0];
    } else if (o.schedule != TRAV_SCHEDULE_PLAIN) {
        return bad("schedule must be TRAV_SCHEDULE_PLAIN or TRAV_SCHEDULE_LEARNED");
    }
    if (n == 0) return TRAV_OK;
    return run_batch(g, 0, sources, n, &o, 0.0f, mlp, levels, mem);
}

int trav_sssp(trav_graph *g, const int32_t *sources, int32_t n, const trav_sssp_opts *opts, float *dist,
              int32_t mem)
{
    if (!g) return bad("graph handle is NULL");
    if (!dist && n > 0) return bad("dist must not be NULL");
    if (mem != TRAV_MEM_HOST && mem != TRAV_MEM_DEVICE) return bad("mem must be TRAV_MEM_HOST or TRAV_MEM_DEVICE");
    TRY(check_sources(g, sources, n));
    trav_sssp_opts o{TRAV_SCHEDULE_PLAIN, 0.0f};
    if (opts) o = *opts;
    if (std::isnan(o.delta)) return bad("delta must not be NaN");
    const float *mlp = nullptr;
    if (o.schedule == TRAV_SCHEDULE_LEARNED) {
        if (!g->mlp[1]) return bad("learned SSSP schedule requested but no SSSP MLP is loaded (trav_mlp_set)");
        if (!(o.delta > 0.0f) || std::isinf(o.delta)) return bad("the learned SSSP schedule needs a finite delta > 0");
        mlp = g->mlp[1];
    } else if (o.schedule != TRAV_SCHEDULE_PLAIN) {
        return bad("schedule must be TRAV_SCHEDULE_PLAIN or TRAV_SCHEDULE_LEARNED");
    }
    if (n == 0) return TRAV_OK;
    return run_batch(g, 1, sources, n, nullptr, o.delta, mlp, dist, mem);
}

int trav_last_stats(trav_graph *g, trav_query_stats *out)
{
    if (!g || !out) return bad("graph handle and out must not be NULL");
    if (g->last_kind < 0 || g->last_n < 1) return bad("no query has run on this handle");
    TRY_CUDA(cudaSetDevice(g->device));
    const int q = g->last_n - 1;
    Ctl h;
    TRY_CUDA(cudaMemcpy(&h, g->ws.ctl + q, offsetof(Ctl, dirs), cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof(*out));
    out->kind = g->last_kind;
    out->steps = h.steps;
    out->buckets = h.buckets;
    out->bottom_up_steps = h.bottom_up_steps;
    out->kernel_ms = g->batch_ms[(size_t)q];
    out->edges_scanned = (int64_t)h.edges_scanned;
    TRY(query_bytes(g->g, &g->ws, q, g->last_kind, &out->algorithmic_bytes, &out->reached, &out->reached_edges, g->st));
    return TRAV_OK;
}

int trav_last_batch_ms(trav_graph *g, float *ms, int32_t cap, int32_t *n)
{
    if (!g || !n) return bad("graph handle and n must not be NULL");
    *n = g->last_n;
    for (int32_t i = 0; ms && i < cap && i < g->last_n; i++) ms[i] = g->batch_ms[(size_t)i];
    return TRAV_OK;
}

int trav_graph_set_stream(trav_graph *g, void *stream)
{
    if (!g) return bad("graph handle is NULL");
    TRY_CUDA(cudaSetDevice(g->device));
    TRY_CUDA(cudaStreamSynchronize(g->st));
    g->st = stream ? static_cast<cudaStream_t>(stream) : g->own_st;
    return TRAV_OK;
}

int trav_el_optimize(int32_t *src, int32_t *dst, float *w, int32_t vertices, int64_t edges, int32_t segment,
                     int32_t mem, int64_t *edges_out)
{
    TRY(check_device());
    if (!edges_out) return bad("edges_out must not be NULL");
    *edges_out = 0;
    if (vertices < 1 || edges < 0) return bad("need vertices >= 1 and edges >= 0");
    if (edges >= (int64_t)INT32_MAX) {
        set_error("edge lists of 2^31 or more edges are not supported");
        return TRAV_ERR_OVERFLOW_INT32;
    }
    if (segment < 0) return bad("segment must be >= 0");
    if (mem != TRAV_MEM_HOST && mem != TRAV_MEM_DEVICE) return bad("mem must be TRAV_MEM_HOST or TRAV_MEM_DEVICE");
    if (edges == 0) return TRAV_OK;
    if (!src || !dst || !w) return bad("src, dst and w must hold `edges` entries");
    if (mem == TRAV_MEM_DEVICE && (!is_device_ptr(src) || !is_device_ptr(dst) || !is_device_ptr(w)))
        return bad("src, dst and w must be device arrays (mem = TRAV_MEM_DEVICE)");
    TRY_CUDA(cudaDeviceSynchronize());
    DevTmp<int32_t> ds, dd;
    DevTmp<float> dw;
    int32_t *s = src, *d = dst;
    float *ww = w;
    const size_t bi = sizeof(int32_t) * (size_t)edges, bf = sizeof(float) * (size_t)edges;
    if (mem == TRAV_MEM_HOST) {
        TRY_CUDA(dev_malloc(&ds.p, bi));
        TRY_CUDA(dev_malloc(&dd.p, bi));
        TRY_CUDA(dev_malloc(&dw.p, bf));
        TRY_CUDA(cudaMemcpy(ds.p, src, bi, cudaMemcpyHostToDevice));
        TRY_CUDA(cudaMemcpy(dd.p, dst, bi, cudaMemcpyHostToDevice));
        TRY_CUDA(cudaMemcpy(dw.p, w, bf, cudaMemcpyHostToDevice));
        s = ds.p, d = dd.p, ww = dw.p;
    }
    TRY(validate_edges(vertices, edges, s, d, ww, 0));
    TRY(el_optimize_device(s, d, ww, edges, segment, edges_out, 0));
    if (mem == TRAV_MEM_HOST && *edges_out > 0) {
        const size_t n = (size_t)*edges_out;
        TRY_CUDA(cudaMemcpy(src, s, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        TRY_CUDA(cudaMemcpy(dst, d, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        TRY_CUDA(cudaMemcpy(w, ww, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    return TRAV_OK;
}

int trav_el_gpu_transactions(const int32_t *src, const int32_t *dst, int32_t vertices, int64_t edges,
                             int32_t elem_size, int32_t mem, int64_t *count)
{
    TRY(check_device());
    if (!count) return bad("count must not be NULL");
    *count = 0;
    if (vertices < 1 || edges < 0 || elem_size < 1) return bad("need vertices >= 1, edges >= 0 and elem_size >= 1");
    if (mem != TRAV_MEM_HOST && mem != TRAV_MEM_DEVICE) return bad("mem must be TRAV_MEM_HOST or TRAV_MEM_DEVICE");
    if (edges == 0) return TRAV_OK;
    if (!src || !dst) return bad("src and dst must hold `edges` entries");
    if (mem == TRAV_MEM_DEVICE && (!is_device_ptr(src) || !is_device_ptr(dst)))
        return bad("src and dst must be device arrays (mem = TRAV_MEM_DEVICE)");
    TRY_CUDA(cudaDeviceSynchronize());
    DevTmp<int32_t> ds, dd;
    const int32_t *s = src, *d = dst;
    if (mem == TRAV_MEM_HOST) {
        const size_t bi = sizeof(int32_t) * (size_t)edges;
        TRY_CUDA(dev_malloc(&ds.p, bi));
        TRY_CUDA(dev_malloc(&dd.p, bi));
        TRY_CUDA(cudaMemcpy(ds.p, src, bi, cudaMemcpyHostToDevice));
        TRY_CUDA(cudaMemcpy(dd.p, dst, bi, cudaMemcpyHostToDevice));
        s = ds.p, d = dd.p;
    }
    TRY(validate_edges(vertices, edges, s, d, nullptr, 0));
    return el_transactions_device(s, d, edges, elem_size, count, 0);
}

int trav_graph_set_capture(trav_graph *g, int32_t on)
{
    if (!g) return bad("graph handle is NULL");
    TRY_CUDA(cudaSetDevice(g->device));
    TRY_CUDA(cudaStreamSynchronize(g->st));
    g->capture = on != 0;
    for (auto &c : g->cap) {
        if (c.exec) cudaGraphExecDestroy(c.exec);
        c.exec = nullptr;
        c.key.clear();
    }
    return TRAV_OK;
}

int trav_set_grid(trav_graph *g, int32_t kind, int32_t ctas, int32_t *max_ctas)
{
    if (!g) return bad("graph handle is NULL");
    if (kind != 0 && kind != 1) return bad("kind must be 0 (BFS) or 1 (SSSP)");
    TRY_CUDA(cudaSetDevice(g->device));
    const int most = persistent_grid_size(kind);
    if (most <= 0) return TRAV_ERR_CUDA;
    if (max_ctas) *max_ctas = most;
    if (ctas < 0 || ctas > most) return bad("ctas must lie in [0, the co-resident maximum]");
    TRY_CUDA(cudaStreamSynchronize(g->st));
    g->ws.grid[kind] = ctas;
    return TRAV_OK;
}

int trav_set_limits(trav_graph *g, int32_t max_steps, uint64_t timeout_ns)
{
    if (!g) return bad("graph handle is NULL");
    if (max_steps < 0) return bad("max_steps must be >= 0 (0 = the default budget)");
    TRY_CUDA(cudaSetDevice(g->device));
    TRY_CUDA(cudaStreamSynchronize(g->st));
    g->ws.max_steps = max_steps;
    g->ws.timeout_ns = timeout_ns;
    return TRAV_OK;
}

int trav_set_plan(trav_graph *g, int32_t kind, const uint8_t *plan, int32_t n)
{
    if (!g) return bad("graph handle is NULL");
    if (kind != 0 && kind != 1) return bad("kind must be 0 (BFS) or 1 (SSSP)");
    if (n < 0 || (n > 0 && !plan)) return bad("plan must hold n >= 0 entries");
    TRY_CUDA(cudaSetDevice(g->device));
    TRY_CUDA(cudaStreamSynchronize(g->st));
    cudaFree(g->ws.plan[kind]);
    g->ws.plan[kind] = nullptr;
    g->ws.plan_len[kind] = 0;
    if (n == 0) return TRAV_OK;
    TRY_CUDA(dev_malloc(&g->ws.plan[kind], (size_t)n));
    TRY_CUDA(cudaMemcpy(g->ws.plan[kind], plan, (size_t)n, cudaMemcpyHostToDevice));
    g->ws.plan_len[kind] = n;
    return TRAV_OK;
}

int trav_last_decisions(trav_graph *g, float *x, uint8_t *choice, int32_t *phase, float *lo, float *hi, int32_t cap,
                        int32_t *n)
{
    if (!g || !n) return bad("graph handle and n must not be NULL");
    if (g->last_n < 1) return bad("no query has run on this handle");
    TRY_CUDA(cudaSetDevice(g->device));
    std::unique_ptr<Ctl> h(new Ctl);
    TRY_CUDA(cudaMemcpy(h.get(), g->ws.ctl + (g->last_n - 1), sizeof(Ctl), cudaMemcpyDeviceToHost));
    *n = h->ndec;
    int m = h->ndec < cap ? h->ndec : cap;
    if (m > kMaxDec) m = kMaxDec;
    for (int i = 0; i < m; i++) {
        if (x)
            for (int k = 0; k < kDecFeat; k++) x[i * kDecFeat + k] = h->dec_x[i][k];
        if (choice) choice[i] = h->dec_choice[i];
        if (phase) phase[i] = h->dec_phase[i];
        if (lo) lo[i] = h->dec_lo[i];
        if (hi) hi[i] = h->dec_hi[i];
    }
    return TRAV_OK;
}

int trav_last_phase_log(trav_graph *g, uint8_t *kind, int64_t *size, double *end_us, int64_t *edges, int32_t cap,
                        int32_t *n)
{
    if (!g || !n) return bad("graph handle and n must not be NULL");
    if (g->last_n < 1) return bad("no query has run on this handle");
    TRY_CUDA(cudaSetDevice(g->device));
    std::unique_ptr<Ctl> h(new Ctl);
    TRY_CUDA(cudaMemcpy(h.get(), g->ws.ctl + (g->last_n - 1), sizeof(Ctl), cudaMemcpyDeviceToHost));
    *n = h->nphase;
    int m = h->nphase < cap ? h->nphase : cap;
    if (m > kMaxTrace) m = kMaxTrace;
    for (int i = 0; i < m; i++) {
        if (kind) kind[i] = h->ph_kind[i];
        if (size) size[i] = h->ph_size[i];
        if (end_us) end_us[i] = (double)(long long)(h->ph_end_ns[i] - h->t0_ns) * 1e-3;
        if (edges) edges[i] = (int64_t)h->ph_scanned[i];
    }
    return TRAV_OK;
}

int trav_last_bfs_trace(trav_graph *g, uint8_t *dirs, int64_t *frontier, int32_t cap, int32_t *nsteps)
{
    if (!g || !nsteps) return bad("graph handle and nsteps must not be NULL");
    if (g->last_kind != 0 || g->last_n < 1) return bad("the last query on this handle was not a BFS");
    TRY_CUDA(cudaSetDevice(g->device));
    const Ctl *c = g->ws.ctl + (g->last_n - 1);
    int steps = 0;
    TRY_CUDA(cudaMemcpy(&steps, &c->steps, sizeof(int), cudaMemcpyDeviceToHost));
    *nsteps = steps;
    int n = steps < cap ? steps : cap;
    if (n > kMaxTrace) n = kMaxTrace;
    if (n > 0 && dirs) TRY_CUDA(cudaMemcpy(dirs, c->dirs, (size_t)n, cudaMemcpyDeviceToHost));
    if (n > 0 && frontier) {
        std::vector<unsigned> f((size_t)n);
        TRY_CUDA(cudaMemcpy(f.data(), c->frontier, 4 * (size_t)n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++) frontier[i] = f[(size_t)i];
    }
    return TRAV_OK;
}

int32_t trav_mlp_param_count(int32_t kind)
{
    if (kind == 0) return mlp_param_count(kBfsOut);
    if (kind == 1) return mlp_param_count(kSsspOut);
    return -1;
}

int trav_mlp_set(trav_graph *g, int32_t kind, const float *params, int32_t count)
{
    if (!g) return bad("graph handle is NULL");
    if (kind != 0 && kind != 1) return bad("kind must be 0 (BFS) or 1 (SSSP)");
    if (!params || count != trav_mlp_param_count(kind)) return bad("params must hold trav_mlp_param_count(kind) floats");
    for (int32_t i = 0; i < count; i++)
        if (!std::isfinite(params[i])) return bad("MLP parameters must be finite");
    TRY_CUDA(cudaSetDevice(g->device));
    if (!g->mlp[kind]) TRY_CUDA(dev_malloc(&g->mlp[kind], sizeof(float) * (size_t)count));
    TRY_CUDA(cudaMemcpy(g->mlp[kind], params, sizeof(float) * (size_t)count, cudaMemcpyHostToDevice));
    return TRAV_OK;
}

int trav_mlp_set_margin(trav_graph *g, int32_t kind, float margin)
{
    if (!g) return bad("graph handle is NULL");
    if (kind != 0 && kind != 1) return bad("kind must be 0 (BFS) or 1 (SSSP)");
    if (!(margin >= 0.0f) || !std::isfinite(margin)) return bad("margin must be finite and >= 0");
    TRY_CUDA(cudaSetDevice(g->device));
    TRY_CUDA(cudaStreamSynchronize(g->st));
    g->ws.mlp_margin[kind] = margin;
    return TRAV_OK;
}

// ------------------------------------------------ reference-shaped entry points

static __global__ void init_distances_kernel(float *d, int32_t V, int32_t s)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x)
        d[i] = i == s ? 0.0f : FLT_MAX;
}

static __global__ void gather_bits_kernel(unsigned *value, const float *d, const int32_t *old_of_new, int32_t V)
{
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < V; r += gridDim.x * blockDim.x)
        value[r] = __float_as_uint(d[old_of_new[r]]);
}

int trav_init_distances_f32(float *d, int32_t vertices, int32_t source)
{
    TRY(check_device());
    if (!d || vertices < 1 || !is_device_ptr(d)) return bad("d must be a device array of vertices >= 1 floats");
    if (source < 0 || source >= vertices) return bad("source vertex out of range [0, V)");
    init_distances_kernel<<<(vertices + 255) / 256 < 4096 ? (vertices + 255) / 256 : 4096, 256>>>(d, vertices, source);
    TRY_CUDA(cudaGetLastError());
    TRY_CUDA(cudaDeviceSynchronize());
    return TRAV_OK;
}

int trav_bellman_ford_el_f32(const int32_t *src, const int32_t *dst, const float *w, int32_t vertices, int64_t edges,
                             int32_t source, float *d)
{
    TRY(check_device());
    if (!d || vertices < 1) return bad("d must be a device array of vertices >= 1 floats");
    if (source < 0 || source >= vertices) return bad("source vertex out of range [0, V)");
    if (edges < 0 || (edges > 0 && (!src || !dst || !w))) return bad("edge arrays must be device arrays of `edges` entries");
    if (!is_device_ptr(d) || (edges > 0 && !(is_device_ptr(src) && is_device_ptr(dst) && is_device_ptr(w))))
        return bad("src, dst, w and d must be device memory (the reference wrappers take device arrays)");
    if (edges >= (int64_t)INT32_MAX) {
        set_error("graph has 2^31 or more edges; the device CSR uses int32 offsets");
        return TRAV_ERR_OVERFLOW_INT32;
    }
    TRY_CUDA(cudaDeviceSynchronize());
    trav_graph *h = nullptr;
    TRY(new_handle(&h));
    std::unique_ptr<trav_graph, void (*)(trav_graph *)> guard(h, destroy);
    TRY(build_graph_device(vertices, edges, src, dst, w, h->st, &h->g));
    TRY(workspace_ensure(&h->ws, h->g, 1, h->st));
    gather_bits_kernel<<<(vertices + 255) / 256 < 4096 ? (vertices + 255) / 256 : 4096, 256, 0, h->st>>>(
        reinterpret_cast<unsigned *>(h->ws.queue[1]), d, h->g.old_of_new, vertices);
    TRY_CUDA(cudaGetLastError());
    TRY(launch_sssp(h->g, &h->ws, 0, -1, INFINITY, nullptr, d, 1, h->st, nullptr, nullptr));
    TRY_CUDA(cudaStreamSynchronize(h->st));
    return check_queries(&h->ws, 1, "bellman_ford_wrapper");
}

int trav_bfs_el(const int32_t *src, const int32_t *dst, int32_t vertices, int64_t edges, uint8_t *visited,
                int32_t source)
{
    TRY(check_device());
    if (!visited || vertices < 1) return bad("visited must be a device array of vertices >= 1 bytes");
    if (source < 0 || source >= vertices) return bad("source vertex out of range [0, V)");
    if (edges < 0 || (edges > 0 && (!src || !dst))) return bad("edge arrays must be device arrays of `edges` entries");
    if (!is_device_ptr(visited) || (edges > 0 && !(is_device_ptr(src) && is_device_ptr(dst))))
        return bad("src, dst and visited must be device memory (the reference wrapper takes device arrays)");
    if (edges >= (int64_t)INT32_MAX) {
        set_error("graph has 2^31 or more edges; the device CSR uses int32 offsets");
        return TRAV_ERR_OVERFLOW_INT32;
    }
    TRY_CUDA(cudaDeviceSynchronize());
    trav_graph *h = nullptr;
    TRY(new_handle(&h));
    std::unique_ptr<trav_graph, void (*)(trav_graph *)> guard(h, destroy);
    TRY(build_graph_device(vertices, edges, src, dst, nullptr, h->st, &h->g));
    TRY(workspace_ensure(&h->ws, h->g, 1, h->st));
    trav_bfs_opts o{TRAV_SCHEDULE_PLAIN, 15.0f, 18.0f, -1};
    int32_t s_new = 0;
    TRY_CUDA(cudaMemcpy(&s_new, h->g.new_of_old + source, sizeof(int32_t), cudaMemcpyDeviceToHost));
    TRY(launch_bfs(h->g, &h->ws, 0, s_new, o, nullptr, visited, 2, h->st, nullptr, nullptr));
    TRY_CUDA(cudaStreamSynchronize(h->st));
    return check_queries(&h->ws, 1, "bfs_wrapper");
}

static __global__ void permute_color_kernel(int32_t *color_new, const int32_t *color, const int32_t *old_of_new,
                                            int32_t V)
{
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < V; r += gridDim.x * blockDim.x)
        color_new[r] = color[old_of_new[r]];
}

int trav_reach_el_masked(const int32_t *src, const int32_t *dst, int32_t vertices, int64_t edges,
                         const int32_t *pivot, const int32_t *trees, uint8_t *visited)
{
    TRY(check_device());
    if (!visited || !pivot || !trees || vertices < 1)
        return bad("pivot, trees and visited must be device arrays (trees and visited of vertices >= 1 entries)");
    if (edges < 0 || (edges > 0 && (!src || !dst))) return bad("edge arrays must be device arrays of `edges` entries");
    if (!is_device_ptr(visited) || !is_device_ptr(pivot) || !is_device_ptr(trees) ||
        (edges > 0 && !(is_device_ptr(src) && is_device_ptr(dst))))
        return bad("src, dst, pivot, trees and visited must be device memory (the reference's sweep takes device arrays)");
    if (edges >= (int64_t)INT32_MAX) {
        set_error("graph has 2^31 or more edges; the device CSR uses int32 offsets");
        return TRAV_ERR_OVERFLOW_INT32;
    }
    TRY_CUDA(cudaDeviceSynchronize());
    int32_t p = 0;
    TRY_CUDA(cudaMemcpy(&p, pivot, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (p < 0 || p >= vertices) return bad("the pivot vertex lies outside [0, V)");
    int32_t want = 0;
    TRY_CUDA(cudaMemcpy(&want, trees + p, sizeof(int32_t), cudaMemcpyDeviceToHost));
    trav_graph *h = nullptr;
    TRY(new_handle(&h));
    std::unique_ptr<trav_graph, void (*)(trav_graph *)> guard(h, destroy);
    TRY(build_graph_device(vertices, edges, src, dst, nullptr, h->st, &h->g));
    TRY(workspace_ensure(&h->ws, h->g, 1, h->st));
    DevTmp<int32_t> color;
    TRY_CUDA(dev_malloc(&color.p, sizeof(int32_t) * (size_t)vertices));
    permute_color_kernel<<<(vertices + 255) / 256 < 4096 ? (vertices + 255) / 256 : 4096, 256, 0, h->st>>>(
        color.p, trees, h->g.old_of_new, vertices);
    TRY_CUDA(cudaGetLastError());
    trav_bfs_opts o{TRAV_SCHEDULE_PLAIN, 15.0f, 18.0f, -1};
    int32_t p_new = 0;
    TRY_CUDA(cudaMemcpy(&p_new, h->g.new_of_old + p, sizeof(int32_t), cudaMemcpyDeviceToHost));
    TRY(launch_bfs(h->g, &h->ws, 0, p_new, o, nullptr, visited, 2, h->st, nullptr, nullptr, color.p, want));
    TRY_CUDA(cudaStreamSynchronize(h->st));
    return check_queries(&h->ws, 1, "trav_reach_el_masked");
}

// ----------------------------------------------------------- graph files

int trav_el_file_read(const char *path, int32_t unweighted, int32_t *vertices, int64_t *edges, int32_t *directed,
                      int32_t *src, int32_t *dst, float *w)
{
    if (!path || !vertices || !edges) return bad("path, vertices and edges must not be NULL");
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error(std::string("cannot open ") + path);
        return TRAV_ERR_IO;
    }
    std::unique_ptr<FILE, int (*)(FILE *)> guard(f, fclose);
    unsigned char hdr[13];
    if (fread(hdr, 1, 13, f) != 13) {
        set_error("edge-list file shorter than its 13-byte header");
        return TRAV_ERR_IO;
    }
    int32_t V;
    int64_t E;
    memcpy(&V, hdr + 1, 4);
    memcpy(&E, hdr + 5, 8);
    const int rec = unweighted ? 8 : 12;
    if (V < 0 || E < 0) {
        set_error("edge-list header holds a negative vertex or edge count");
        return TRAV_ERR_IO;
    }
    fseek(f, 0, SEEK_END);
    long long size = ftell(f);
    if (size != 13 + (long long)rec * E) {
        set_error("edge-list file size does not match its header (" + std::to_string(size) + " bytes for E=" +
                  std::to_string(E) + ")");
        return TRAV_ERR_IO;
    }
    *vertices = V;
    *edges = E;
    if (directed) *directed = hdr[0] ? 1 : 0;
    if (!src) return TRAV_OK;
    if (!dst || (!w && !unweighted)) return bad("dst and w must not be NULL when src is given");
    fseek(f, 13, SEEK_SET);
    const int64_t kBatch = 1 << 20;
    std::vector<unsigned char> buf((size_t)(kBatch * rec));
    for (int64_t e0 = 0; e0 < E; e0 += kBatch) {
        int64_t n = E - e0 < kBatch ? E - e0 : kBatch;
        if (fread(buf.data(), (size_t)rec, (size_t)n, f) != (size_t)n) {
            set_error("short read in edge-list file");
            return TRAV_ERR_IO;
        }
        for (int64_t i = 0; i < n; i++) {
            const unsigned char *r = buf.data() + i * rec;
            memcpy(&src[e0 + i], r, 4);
            memcpy(&dst[e0 + i], r + 4, 4);
            if (unweighted) {
                if (w) w[e0 + i] = 1.0f;
            } else {
                memcpy(&w[e0 + i], r + 8, 4);
            }
        }
    }
    return TRAV_OK;
}

int trav_el_file_write(const char *path, int32_t directed, int32_t vertices, int64_t edges, const int32_t *src,
                       const int32_t *dst, const float *w)
{
    if (!path || vertices < 0 || edges < 0 || (edges > 0 && (!src || !dst || !w)))
        return bad("path, counts and arrays must be valid");
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error(std::string("cannot create ") + path);
        return TRAV_ERR_IO;
    }
    std::unique_ptr<FILE, int (*)(FILE *)> guard(f, fclose);
    unsigned char hdr[13];
    hdr[0] = directed ? 1 : 0;
    memcpy(hdr + 1, &vertices, 4);
    memcpy(hdr + 5, &edges, 8);
    if (fwrite(hdr, 1, 13, f) != 13) {
        set_error("write failed");
        return TRAV_ERR_IO;
    }
    const int64_t kBatch = 1 << 20;
    std::vector<unsigned char> buf((size_t)(kBatch * 12));
    for (int64_t e0 = 0; e0 < edges; e0 += kBatch) {
        int64_t n = edges - e0 < kBatch ? edges - e0 : kBatch;
        for (int64_t i = 0; i < n; i++) {
            unsigned char *r = buf.data() + i * 12;
            memcpy(r, &src[e0 + i], 4);
            memcpy(r + 4, &dst[e0 + i], 4);
            memcpy(r + 8, &w[e0 + i], 4);
        }
        if (fwrite(buf.data(), 12, (size_t)n, f) != (size_t)n) {
            set_error("write failed");
            return TRAV_ERR_IO;
        }
    }
    return TRAV_OK;
}

}  // extern "C"
