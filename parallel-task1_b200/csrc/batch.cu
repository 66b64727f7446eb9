// Batches: many BFS / SSSP queries over several graphs in one persistent
// launch (C ABI declared in include/trav.h).  The device side is
// batch_persistent in traverse.cu; this file builds the query descriptors,
// owns the teams' scratch and runs the autotuner over launch shapes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "handle.cuh"
#include "trav_internal.cuh"

using namespace trav;

#define TRY_CUDA(expr)                                      \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

#define TRY(expr)                       \
    do {                                \
        int _rc = (expr);               \
        if (_rc != TRAV_OK) return _rc; \
    } while (0)

struct trav_batch {
    std::vector<trav_graph *> graphs;
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int32_t vmax = 1, wmax = 1;
    int64_t emax = 0, chunk_cap = 1;
    // scratch of the teams (grown on demand)
    int teams_alloc = 0;
    unsigned char *team_mem = nullptr;
    size_t team_bytes = 0;
    TeamWs *d_teams = nullptr;
    Ctl *ctl = nullptr;
    // query descriptors of the last run
    BatchQuery *d_q = nullptr;
    int q_cap = 0;
    unsigned *d_next = nullptr;
    std::map<std::pair<int, float>, LightRows> light;  // light rows per (graph, delta)
    // host-output runs: device staging of the results and the copy stream
    unsigned char *staging = nullptr;
    size_t staging_bytes = 0;
    cudaStream_t cst = nullptr;
    unsigned *done = nullptr;  // per-query completion flags, mapped host memory
    int done_cap = 0;
    trav_batch_shape shape{16, kSmallDeg, kItem};
};

namespace {

int bad(const char *msg)
{
    set_error(msg);
    return TRAV_ERR_BAD_ARG;
}

size_t round_up(size_t x) { return (x + 255) & ~size_t(255); }

// Byte layout of one team's scratch (every array 256-byte aligned).
struct TeamLayout {
    size_t value, rcls, visited, front0, front1, q[6], chunks[4], total;
};

TeamLayout team_layout(const trav_batch *b)
{
    TeamLayout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += round_up(bytes);
        return at;
    };
    L.value = take(sizeof(unsigned long long) * (size_t)b->vmax);
    L.rcls = take(sizeof(unsigned char) * (size_t)b->vmax);
    L.visited = take(sizeof(unsigned) * (size_t)b->wmax);
    L.front0 = take(sizeof(unsigned) * (size_t)b->wmax);
    L.front1 = take(sizeof(unsigned) * (size_t)b->wmax);
    for (int i = 0; i < 6; i++) L.q[i] = take(sizeof(int32_t) * (size_t)b->vmax);
    for (int i = 0; i < 4; i++) L.chunks[i] = take(sizeof(int2) * (size_t)b->chunk_cap);
    L.total = o;
    return L;
}

// Free the team scratch (run_launch allocates it again, sized to what is free).
int release_teams(trav_batch *b)
{
    TRY_CUDA(cudaStreamSynchronize(b->st));
    cudaFree(b->team_mem);
    cudaFree(b->d_teams);
    cudaFree(b->ctl);
    b->team_mem = nullptr;
    b->d_teams = nullptr;
    b->ctl = nullptr;
    b->teams_alloc = 0;
    return TRAV_OK;
}

int ensure_teams(trav_batch *b, int teams)
{
    if (teams <= b->teams_alloc) return TRAV_OK;
    TRY(release_teams(b));
    const TeamLayout L = team_layout(b);
    b->team_bytes = L.total;
    TRY_CUDA(dev_malloc(&b->team_mem, L.total * (size_t)teams));
    TRY_CUDA(dev_malloc(&b->d_teams, sizeof(TeamWs) * (size_t)teams));
    TRY_CUDA(dev_malloc(&b->ctl, sizeof(Ctl) * (size_t)teams));
    std::vector<TeamWs> h((size_t)teams);
    for (int t = 0; t < teams; t++) {
        unsigned char *m = b->team_mem + L.total * (size_t)t;
        TeamWs &w = h[(size_t)t];
        w.value = reinterpret_cast<unsigned *>(m + L.value);
        w.rcls = m + L.rcls;
        w.visited = reinterpret_cast<unsigned *>(m + L.visited);
        w.front0 = reinterpret_cast<unsigned *>(m + L.front0);
        w.front1 = reinterpret_cast<unsigned *>(m + L.front1);
        int32_t *q[6];
        for (int i = 0; i < 6; i++) q[i] = reinterpret_cast<int32_t *>(m + L.q[i]);
        w.q0 = q[0];
        w.q1 = q[1];
        w.far0 = q[2];
        w.far1 = q[3];
        w.hq0 = q[4];
        w.hq1 = q[5];
        int2 *c[4];
        for (int i = 0; i < 4; i++) c[i] = reinterpret_cast<int2 *>(m + L.chunks[i]);
        w.chunks0 = c[0];
        w.chunks1 = c[1];
        w.hch0 = c[2];
        w.hch1 = c[3];
        w.ctl = b->ctl + t;
    }
    TRY_CUDA(cudaMemcpy(b->d_teams, h.data(), sizeof(TeamWs) * (size_t)teams, cudaMemcpyHostToDevice));
    b->teams_alloc = teams;
    return TRAV_OK;
}

int shape_ok(const trav_batch_shape &s, int most)
{
    if (s.team_ctas < 1 || s.team_ctas > most) return bad("team_ctas must lie in [1, the co-resident CTAs]");
    if (s.small_deg < 0 || s.small_deg > kMaxSmallDeg) return bad("small_deg must lie in [0, 1024]");
    if (s.item < kMinItem || s.item > kMaxItem) return bad("item must lie in [64, 8192]");
    return TRAV_OK;
}

bool finite_delta(float d) { return d > 0.0f && std::isfinite(d); }

constexpr int kBusy = 1;  // a run_launch poll's "keep calling me" (TRAV_OK and the errors are <= 0)
#ifndef TRAV_SMOOTH_ORDER
#define TRAV_SMOOTH_ORDER 1
#endif
constexpr bool kSmoothOrder = TRAV_SMOOTH_ORDER;  // host-output runs spread the cheap queries (build_queries)

// Descriptors in dispatch order: the most edges first (an SSSP query counts
// as four BFS queries), so the long queries start while the short ones fill
// the gaps.
//
// With smooth_tail > 0 (host-output runs) the results also have to cross to
// the host as the queries finish.  Largest first ends with a burst of short
// queries whose results arrive faster than the copy engine takes them (at RMAT
// s23: 64 BFS results, 2.1 GB, in the last 24 ms against 57 GB/s).  So the
// cheaper queries are spread among the expensive ones in proportion, keeping
// only the smooth_tail cheapest for the end (two per team), where short
// queries still even out the teams' finishing times.
int build_queries(trav_batch *b, const trav_query *qs, int32_t n, std::vector<BatchQuery> *out, int smooth_tail = 0)
{
    std::vector<int32_t> order((size_t)n);
    std::iota(order.begin(), order.end(), 0);
    auto cost = [&](int32_t i) {
        const trav_graph *g = b->graphs[(size_t)qs[i].graph];
        return (double)(g->g.E + g->g.V) * (qs[i].kind == 1 ? 4.0 : 1.0);
    };
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return cost(x) > cost(y); });
    if (smooth_tail > 0 && n > 0) {
        double mean = 0.0;
        for (int32_t i : order) mean += cost(i) / n;
        std::vector<int32_t> big, small;  // both still most expensive first
        for (int32_t i : order) (cost(i) > mean ? big : small).push_back(i);
        const size_t t = std::min(small.size(), (size_t)smooth_tail);
        const std::vector<int32_t> tail(small.end() - (std::ptrdiff_t)t, small.end());
        small.resize(small.size() - t);
        const double per = big.empty() ? 0.0 : (double)small.size() / (double)big.size();
        double owed = 0.0;
        size_t si = 0;
        order.clear();
        for (int32_t i : big) {
            order.push_back(i);
            for (owed += per; si < small.size() && owed >= 1.0; owed -= 1.0) order.push_back(small[si++]);
        }
        while (si < small.size()) order.push_back(small[si++]);
        order.insert(order.end(), tail.begin(), tail.end());
    }
    out->clear();
    for (int32_t i : order) {
        const trav_query &q = qs[i];
        trav_graph *g = b->graphs[(size_t)q.graph];
        BatchQuery d{};
        d.out_off = g->g.out_off;
        d.out_adj = g->g.out_adj;
        d.out_w = g->g.out_w;
        d.in_off = g->g.in_off;
        d.in_adj = g->g.in_adj;
        d.in_w = g->g.in_w;
        d.new_of_old = g->g.new_of_old;
        d.V = g->g.V;
        d.E = g->g.E;
        d.mean_w = g->g.mean_w;
        d.max_deg = g->g.max_out_degree;
        d.kind = q.kind;
        d.id = i;
        d.source = g->new_of_old[(size_t)q.source];
        d.out = q.out;
        d.mlp = q.schedule == TRAV_SCHEDULE_LEARNED ? g->mlp[q.kind] : nullptr;
        d.mlp_margin = g->ws.mlp_margin[q.kind];
        d.delta = INFINITY;
        d.nlight = nullptr;
        d.loff = nullptr;
        d.ledge = nullptr;
        if (q.kind == 1 && finite_delta(q.delta)) {
            // the learned schedule also picks the query's delta (the graph's learned split)
            d.delta = d.mlp ? q.delta * g->ws.split_scale : q.delta;
            // light rows once per (graph, delta) for the batch's lifetime
            LightRows &lr = b->light[std::make_pair(q.graph, d.delta)];
            TRY(light_rows_build(g->g, d.delta, &lr, b->st));
            d.nlight = lr.nlight;
            d.loff = lr.loff;
            d.ledge = lr.ledge;
        }
        out->push_back(d);
    }
    return TRAV_OK;
}

int check_queries_host(const trav_batch *b, const trav_query *qs, int32_t n)
{
    if (n < 0 || (n > 0 && !qs)) return bad("queries must be a host array of n >= 0 entries");
    for (int32_t i = 0; i < n; i++) {
        const trav_query &q = qs[i];
        if (q.graph < 0 || q.graph >= (int32_t)b->graphs.size()) return bad("query graph index out of range");
        if (q.kind != 0 && q.kind != 1) return bad("query kind must be 0 (BFS) or 1 (SSSP)");
        const trav_graph *g = b->graphs[(size_t)q.graph];
        if (q.source < 0 || q.source >= g->g.V) return bad("query source out of range [0, V)");
        if (!q.out) return bad("query out must be a device array of V results");
        if (q.schedule != TRAV_SCHEDULE_PLAIN && q.schedule != TRAV_SCHEDULE_LEARNED)
            return bad("query schedule must be TRAV_SCHEDULE_PLAIN or TRAV_SCHEDULE_LEARNED");
        if (q.schedule == TRAV_SCHEDULE_LEARNED && !g->mlp[q.kind])
            return bad("learned schedule asked for a graph without a network (trav_mlp_set)");
    }
    return TRAV_OK;
}

}  // namespace

namespace {

// One launch of the queries already in b->d_q; *ms receives its device time.
// `done` (mapped host flags, may be nullptr) is passed to the kernel; while the
// launch runs, `poll` (may be empty) is called until it returns something other
// than kBusy or the launch has ended.
int run_launch(trav_batch *b, int32_t n, const trav_batch_shape &s, float *ms, unsigned *done = nullptr,
               const std::function<int(bool ended)> &poll = {})
{
    const int most = persistent_grid_size(2);
    if (most <= 0) return TRAV_ERR_CUDA;
    TRY(shape_ok(s, most));
    int teams = std::max(1, std::min(most / s.team_ctas, (int)n));
    if (teams > b->teams_alloc) {
        // every team needs scratch for the batch's largest graph: run fewer
        // teams (each still of team_ctas CTAs) when the device cannot hold them
        size_t free_b = 0, total_b = 0;
        TRY_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t have = (size_t)b->teams_alloc * b->team_bytes + free_b;
        const size_t spare = (size_t)1 << 30;  // left for the caller
        const size_t per = team_layout(b).total + sizeof(Ctl) + sizeof(TeamWs);
        const size_t fit = have > spare ? (have - spare) / per : 0;
        if (fit < 1) {
            set_error("batch: not enough device memory for one team's scratch");
            return TRAV_ERR_OOM;
        }
        teams = (int)std::min<size_t>((size_t)teams, fit);
    }
    TRY(ensure_teams(b, teams));
    for (int t = 0; t < teams; t++) TRY_CUDA(cudaMemsetAsync(b->ctl + t, 0, offsetof(Ctl, dirs), b->st));
    BatchArgs a{};
    a.queries = b->d_q;
    a.nq = n;
    a.next = b->d_next;
    a.teams = b->d_teams;
    a.team_ctas = s.team_ctas;
    a.small_deg = s.small_deg;
    a.item = s.item;
    a.timeout_ns = 10ull * 1000000000ull;
    a.done = done;
    TRY(launch_batch(a, teams, b->st, b->ev0, b->ev1));
    int prc = TRAV_OK;
    if (poll) {
        // the kernel's own barrier waits are bounded, so the launch ends and so does this loop
        for (;;) {
            const bool ended = cudaStreamQuery(b->st) != cudaErrorNotReady;
            prc = poll(ended);
            if (prc != kBusy || ended) break;
            std::this_thread::yield();
        }
    }
    TRY_CUDA(cudaStreamSynchronize(b->st));
    TRY(check_ctls(b->ctl, teams, "batch"));
    if (prc != TRAV_OK && prc != kBusy) return prc;
    float t = 0.0f;
    TRY_CUDA(cudaEventElapsedTime(&t, b->ev0, b->ev1));
    if (ms) *ms = t;
    return TRAV_OK;
}

int upload_queries(trav_batch *b, const trav_query *qs, int32_t n, int smooth_tail = 0)
{
    TRY(check_queries_host(b, qs, n));
    std::vector<BatchQuery> d;
    TRY(build_queries(b, qs, n, &d, smooth_tail));
    if (n > b->q_cap) {
        TRY_CUDA(cudaStreamSynchronize(b->st));
        cudaFree(b->d_q);
        b->d_q = nullptr;
        b->q_cap = 0;
        TRY_CUDA(dev_malloc(&b->d_q, sizeof(BatchQuery) * (size_t)n));
        b->q_cap = n;
    }
    if (n > 0) TRY_CUDA(cudaMemcpyAsync(b->d_q, d.data(), sizeof(BatchQuery) * (size_t)n, cudaMemcpyHostToDevice, b->st));
    TRY_CUDA(cudaStreamSynchronize(b->st));  // the host vector goes out of scope
    return TRAV_OK;
}

// Launch shapes the autotuner found, process-wide, by kind of batch
// (trav_tune_table_save / _load persist them).
std::map<std::string, trav_batch_shape> g_tune_table;
std::mutex g_tune_mu;

int ceil_log2(int64_t x)
{
    int k = 0;
    while (k < 62 && ((int64_t)1 << k) < x) k++;
    return k;
}

// What the best launch shape depends on: the device (its co-resident CTAs),
// the size of the largest graph queried, the number of graphs and queries,
// and the shares of SSSP and learned-schedule queries (in eighths).
std::string tune_key(const trav_batch *b, const trav_query *qs, int32_t n, int most)
{
    int64_t vmax = 1, emax = 1;
    int sssp = 0, learned = 0;
    std::vector<char> used(b->graphs.size(), 0);
    for (int32_t i = 0; i < n; i++) {
        const trav_graph *g = b->graphs[(size_t)qs[i].graph];
        used[(size_t)qs[i].graph] = 1;
        vmax = std::max<int64_t>(vmax, g->g.V);
        emax = std::max<int64_t>(emax, g->g.E);
        sssp += qs[i].kind == 1;
        learned += qs[i].schedule == TRAV_SCHEDULE_LEARNED;
    }
    const int graphs = (int)std::count(used.begin(), used.end(), 1);
    const int nn = std::max(n, 1);
    return "ctas" + std::to_string(most) + "_v" + std::to_string(ceil_log2(vmax)) + "_e" +
           std::to_string(ceil_log2(emax)) + "_g" + std::to_string(ceil_log2(graphs)) + "_q" +
           std::to_string(ceil_log2(nn)) + "_s" + std::to_string(8 * sssp / nn) + "_l" +
           std::to_string(8 * learned / nn);
}

}  // namespace

extern "C" {

int trav_batch_create(trav_graph *const *graphs, int32_t n, trav_batch **out)
{
    if (!out) return bad("out must not be NULL");
    *out = nullptr;
    if (!graphs || n < 1) return bad("graphs must hold n >= 1 graph handles");
    for (int32_t i = 0; i < n; i++)
        if (!graphs[i]) return bad("graph handle is NULL");
    for (int32_t i = 1; i < n; i++)
        if (graphs[i]->device != graphs[0]->device) return bad("the graphs of a batch must live on one device");
    trav_batch *b = new (std::nothrow) trav_batch();
    if (!b) {
        set_error("host allocation failed");
        return TRAV_ERR_OOM;
    }
    b->graphs.assign(graphs, graphs + n);
    b->device = graphs[0]->device;
    for (const trav_graph *g : b->graphs) {
        b->vmax = std::max(b->vmax, g->g.V);
        b->emax = std::max(b->emax, g->g.E);
    }
    b->wmax = (b->vmax + 31) / 32;
    b->chunk_cap = (int64_t)b->vmax + b->emax / kMinItem + 1;
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e == cudaSuccess) e = dev_malloc(&b->d_next, sizeof(unsigned));
    if (e != cudaSuccess) {
        trav_batch_free(b);
        return cuda_fail(e, "trav_batch_create");
    }
    *out = b;
    return TRAV_OK;
}

void trav_batch_free(trav_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    cudaFree(b->team_mem);
    cudaFree(b->d_teams);
    cudaFree(b->ctl);
    cudaFree(b->d_q);
    cudaFree(b->d_next);
    for (auto &kv : b->light) light_rows_free(&kv.second);
    if (b->cst) cudaStreamSynchronize(b->cst);
    cudaFree(b->staging);
    cudaFreeHost(b->done);
    if (b->cst) cudaStreamDestroy(b->cst);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

int trav_batch_run(trav_batch *b, const trav_query *queries, int32_t n, float *device_ms)
{
    if (!b) return bad("batch handle is NULL");
    TRY_CUDA(cudaSetDevice(b->device));
    // the graphs' own streams may still be writing them
    for (trav_graph *g : b->graphs) TRY_CUDA(cudaStreamSynchronize(g->st));
    TRY(upload_queries(b, queries, n));
    if (n == 0) {
        if (device_ms) *device_ms = 0.0f;
        return TRAV_OK;
    }
    return run_launch(b, n, b->shape, device_ms);
}

int trav_batch_run_host(trav_batch *b, const trav_query *queries, int32_t n, int32_t parts, float *device_ms)
{
    if (!b) return bad("batch handle is NULL");
    if (parts < 1) return bad("parts must be >= 1");
    TRY_CUDA(cudaSetDevice(b->device));
    for (trav_graph *g : b->graphs) TRY_CUDA(cudaStreamSynchronize(g->st));
    TRY(check_queries_host(b, queries, n));
    for (int32_t i = 0; i < n; i++)
        if (is_device_ptr(queries[i].out)) return bad("trav_batch_run_host takes host output arrays (use trav_batch_run)");
    if (device_ms) *device_ms = 0.0f;
    if (n == 0) return TRAV_OK;
    // every query's results get a slot in one device staging area
    std::vector<size_t> at((size_t)n + 1, 0);
    for (int32_t i = 0; i < n; i++)
        at[(size_t)i + 1] = at[(size_t)i] + 4 * (size_t)b->graphs[(size_t)queries[i].graph]->g.V;
    if (at[(size_t)n] > b->staging_bytes) {
        if (b->cst) TRY_CUDA(cudaStreamSynchronize(b->cst));
        cudaFree(b->staging);
        b->staging = nullptr;
        b->staging_bytes = 0;
        // Team scratch is sized to the free memory when it is allocated, so on
        // a large graph it may have left too little for the staging area:
        // place the staging first and let the launches size the teams again.
        TRY(release_teams(b));
        TRY_CUDA(dev_malloc(&b->staging, at[(size_t)n]));
        b->staging_bytes = at[(size_t)n];
    }
    if (!b->cst) TRY_CUDA(cudaStreamCreateWithFlags(&b->cst, cudaStreamNonBlocking));
    if (n > b->done_cap) {
        cudaFreeHost(b->done);
        b->done = nullptr;
        b->done_cap = 0;
        TRY_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&b->done), sizeof(unsigned) * (size_t)n, cudaHostAllocMapped));
        b->done_cap = n;
    }
    unsigned *done_dev = nullptr;
    TRY_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&done_dev), b->done, 0));
    std::vector<trav_query> dq(queries, queries + n);
    for (int32_t i = 0; i < n; i++) dq[(size_t)i].out = b->staging + at[(size_t)i];
    // Part p holds a share of the queries proportional to 2 (parts - p) + 1.
    // Within a part, each query's results go to the host as soon as its team
    // has written them: the kernel raises the query's flag in mapped host
    // memory, and this thread, polling the flags while the launch runs, queues
    // the copy on a second stream.  Only the last queries' copies follow the
    // launch, so parts = 1 (one launch) is normally best.
    std::vector<int32_t> cut((size_t)parts + 1, 0);
    double wsum = 0.0;
    for (int p = 0; p < parts; p++) wsum += 2.0 * (parts - p) + 1.0;
    double acc = 0.0;
    for (int p = 0; p < parts; p++) {
        acc += 2.0 * (parts - p) + 1.0;
        cut[(size_t)p + 1] = (int32_t)std::lround(n * acc / wsum);
    }
    cut[(size_t)parts] = n;
    volatile unsigned *flag = b->done;
    std::vector<char> sent((size_t)n, 0);
    auto send = [&](int32_t i) -> int {
        sent[(size_t)i] = 1;
        TRY_CUDA(cudaMemcpyAsync(queries[i].out, b->staging + at[(size_t)i], at[(size_t)i + 1] - at[(size_t)i],
                                 cudaMemcpyDeviceToHost, b->cst));
        return TRAV_OK;
    };
    float total = 0.0f;
    // Copies may be queued when a launch fails: whatever happens, the call
    // returns only once none of them can still write the caller's arrays.
    const int rc = [&]() -> int {
        for (int p = 0; p < parts; p++) {
            const int32_t q0 = cut[(size_t)p], q1 = cut[(size_t)p + 1];
            if (q1 <= q0) continue;
            const int most = persistent_grid_size(2);
            const int teams = std::max(1, std::min(most > 0 ? most / std::max(1, b->shape.team_ctas) : 1, q1 - q0));
            TRY(upload_queries(b, dq.data() + q0, q1 - q0, kSmoothOrder ? 2 * teams : 0));
            std::memset(b->done, 0, sizeof(unsigned) * (size_t)(q1 - q0));
            int32_t left = q1 - q0;
            auto poll = [&](bool) -> int {
                for (int32_t i = q0; i < q1 && left > 0; i++)
                    if (!sent[(size_t)i] && flag[i - q0]) {
                        TRY(send(i));
                        left--;
                    }
                return left > 0 ? kBusy : TRAV_OK;
            };
            float ms = 0.0f;
            TRY(run_launch(b, q1 - q0, b->shape, &ms, done_dev, poll));
            total += ms;
            // the launch has ended: whatever was not copied yet goes now
            for (int32_t i = q0; i < q1; i++)
                if (!sent[(size_t)i]) TRY(send(i));
        }
        return TRAV_OK;
    }();
    const cudaError_t ce = cudaStreamSynchronize(b->cst);
    if (rc != TRAV_OK) return rc;
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamSynchronize(b->cst)");
    if (device_ms) *device_ms = total;
    return TRAV_OK;
}

int trav_batch_autotune(trav_batch *b, const trav_query *queries, int32_t n, int32_t reps, trav_batch_shape *best)
{
    if (!b) return bad("batch handle is NULL");
    if (reps < 0) return bad("reps must be >= 0");
    TRY_CUDA(cudaSetDevice(b->device));
    for (trav_graph *g : b->graphs) TRY_CUDA(cudaStreamSynchronize(g->st));
    TRY(check_queries_host(b, queries, n));
    const int most = persistent_grid_size(2);
    if (most <= 0) return TRAV_ERR_CUDA;
    const std::string key = tune_key(b, queries, n, most);
    if (reps == 0 && n > 0) {
        // a shape tuned earlier for this kind of batch on this kind of device
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_table.find(key);
        if (it != g_tune_table.end() && shape_ok(it->second, most) == TRAV_OK) {
            b->shape = it->second;
            if (best) *best = b->shape;
            return TRAV_OK;
        }
    }
    if (reps == 0) reps = 1;
    TRY(upload_queries(b, queries, n));
    if (n > 0) {
        auto time_of = [&](const trav_batch_shape &s, float *t) {
            float m = INFINITY;
            for (int r = 0; r < reps; r++) {
                float x = 0.0f;
                TRY(run_launch(b, n, s, &x));
                m = std::min(m, x);
            }
            *t = m;
            return TRAV_OK;
        };
        // coordinate descent: team size, then tile threshold, then item size, twice
        std::vector<int> team_opts;
        for (int c : {1, 2, 4, 8, 16, 37, 74, 148, 296})
            if (c < most) team_opts.push_back(c);
        team_opts.push_back(most);
        const int deg_opts[] = {8, 16, 32, 64};
        const int item_opts[] = {128, 256, 512, 1024};
        trav_batch_shape cur = b->shape;
        cur.team_ctas = std::min(cur.team_ctas, most);
        float cur_t = 0.0f;
        TRY(time_of(cur, &cur_t));
        auto consider = [&](trav_batch_shape s) {
            float t = 0.0f;
            TRY(time_of(s, &t));
            if (t < cur_t) {
                cur = s;
                cur_t = t;
            }
            return TRAV_OK;
        };
        for (int pass = 0; pass < 2; pass++) {
            for (int c : team_opts) {
                trav_batch_shape s = cur;
                s.team_ctas = c;
                TRY(consider(s));
            }
            for (int d : deg_opts) {
                trav_batch_shape s = cur;
                s.small_deg = d;
                TRY(consider(s));
            }
            for (int it : item_opts) {
                trav_batch_shape s = cur;
                s.item = it;
                TRY(consider(s));
            }
        }
        b->shape = cur;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_table[key] = cur;
    }
    if (best) *best = b->shape;
    return TRAV_OK;
}

int trav_tune_table_save(const char *path)
{
    if (!path) return bad("path must not be NULL");
    std::lock_guard<std::mutex> lock(g_tune_mu);
    FILE *f = fopen(path, "w");
    if (!f) {
        set_error(std::string("cannot create ") + path);
        return TRAV_ERR_IO;
    }
    fprintf(f, "# trav-b200 batch launch shapes: key team_ctas small_deg item\n");
    for (const auto &kv : g_tune_table)
        fprintf(f, "%s %d %d %d\n", kv.first.c_str(), kv.second.team_ctas, kv.second.small_deg, kv.second.item);
    const bool ok = fclose(f) == 0;
    if (!ok) {
        set_error(std::string("write failed: ") + path);
        return TRAV_ERR_IO;
    }
    return TRAV_OK;
}

int trav_tune_table_load(const char *path, int32_t *entries)
{
    if (!path) return bad("path must not be NULL");
    FILE *f = fopen(path, "r");
    if (!f) {
        set_error(std::string("cannot open ") + path);
        return TRAV_ERR_IO;
    }
    std::map<std::string, trav_batch_shape> got;
    char line[512];
    int lineno = 0;
    while (fgets(line, sizeof line, f)) {
        lineno++;
        if (line[0] == '#' || line[0] == '\n') continue;
        char key[256];
        trav_batch_shape s{};
        if (sscanf(line, "%255s %d %d %d", key, &s.team_ctas, &s.small_deg, &s.item) != 4 || s.team_ctas < 1 ||
            s.small_deg < 0 || s.small_deg > kMaxSmallDeg || s.item < kMinItem || s.item > kMaxItem) {
            fclose(f);
            set_error(std::string("malformed tuning table line ") + std::to_string(lineno) + " in " + path);
            return TRAV_ERR_IO;
        }
        got[key] = s;
    }
    fclose(f);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (const auto &kv : got) g_tune_table[kv.first] = kv.second;
    if (entries) *entries = (int32_t)g_tune_table.size();
    return TRAV_OK;
}

int trav_batch_set_shape(trav_batch *b, const trav_batch_shape *shape)
{
    if (!b || !shape) return bad("batch handle and shape must not be NULL");
    TRY_CUDA(cudaSetDevice(b->device));
    const int most = persistent_grid_size(2);
    if (most <= 0) return TRAV_ERR_CUDA;
    TRY(shape_ok(*shape, most));
    b->shape = *shape;
    return TRAV_OK;
}

int trav_batch_get_shape(const trav_batch *b, trav_batch_shape *shape)
{
    if (!b || !shape) return bad("batch handle and shape must not be NULL");
    *shape = b->shape;
    return TRAV_OK;
}

}  // extern "C"
