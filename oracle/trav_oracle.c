/* Test infrastructure, not product code: CPU oracle for the traversal path.
 * See trav_oracle.h for the contract of each function and the reference
 * file:line it restates.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load this library, and only as the checker.
 */
#include "trav_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LCG_A 1103515245u
#define LCG_C 12345u

/* glibc rand_r: three steps of next = next * 1103515245 + 12345, taking 11,
 * 10 and 10 bits of next / 65536. */
int orc_rand_r(uint32_t *state)
{
    uint32_t next = *state;
    int result;
    next = next * LCG_A + LCG_C;
    result = (int)((next / 65536u) % 2048u);
    next = next * LCG_A + LCG_C;
    result <<= 10;
    result ^= (int)((next / 65536u) % 1024u);
    next = next * LCG_A + LCG_C;
    result <<= 10;
    result ^= (int)((next / 65536u) % 1024u);
    *state = next;
    return result;
}

/* Affine-map exponentiation: x -> A x + C applied `steps` times. */
uint32_t orc_lcg_skip(uint32_t state, uint64_t steps)
{
    uint32_t acc_a = 1u, acc_c = 0u; /* accumulated map */
    uint32_t cur_a = LCG_A, cur_c = LCG_C;
    while (steps) {
        if (steps & 1u) {
            acc_a = acc_a * cur_a;
            acc_c = acc_c * cur_a + cur_c;
        }
        cur_c = cur_c * cur_a + cur_c;
        cur_a = cur_a * cur_a;
        steps >>= 1;
    }
    return acc_a * state + acc_c;
}

/* One RMAT edge (graph_generation_API.hpp:435-470): descend scale-1 quadrant
 * levels from the midpoint with integer-percent probabilities, then two
 * coin-flip decrements, then a weight rand_r / RAND_MAX in float. */
static void rmat_edge(int scale, int a, int b, int c, int d, uint32_t *st,
                      int32_t *from, int32_t *to, float *wt)
{
    int V = 1 << scale;
    int x = V / 2, y = V / 2;
    for (int i = 1; i < scale; i++) {
        int step = 1 << (scale - (i + 1));
        int p = orc_rand_r(st) % 100;
        if (p < a) { x -= step; y -= step; }
        else if (p < a + b) { x -= step; y += step; }
        else if (p < a + b + c) { x += step; y -= step; }
        else if (p < a + b + c + d) { x += step; y += step; }
    }
    if (orc_rand_r(st) % 2 == 0) x--;
    if (orc_rand_r(st) % 2 == 0) y--;
    *from = x;
    *to = y;
    *wt = (float)orc_rand_r(st) / (float)RAND_MAX;
}

void orc_rmat(int scale, int avg, int a, int b, int c, int d, uint32_t seed, int threads,
              int32_t *src, int32_t *dst, float *w)
{
    int64_t E = (int64_t)(1 << scale) * avg;
    uint64_t steps_per_edge = 3ull * (uint64_t)(scale + 2);
    if (threads < 1) threads = 1;
#pragma omp parallel num_threads(threads)
    {
        int nt = 1, t = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        t = omp_get_thread_num();
#endif
        int64_t lo = E * t / nt, hi = E * (t + 1) / nt;
        uint32_t st = orc_lcg_skip(seed, steps_per_edge * (uint64_t)lo);
        for (int64_t e = lo; e < hi; e++)
            rmat_edge(scale, a, b, c, d, &st, &src[e], &dst[e], &w[e]);
    }
}

int64_t orc_drop_self_loops(int64_t E, int32_t *src, int32_t *dst, float *w)
{
    int64_t k = 0;
    for (int64_t e = 0; e < E; e++) {
        if (src[e] == dst[e]) continue;
        src[k] = src[e];
        dst[k] = dst[e];
        w[k] = w[e];
        k++;
    }
    return k;
}

/* sssp.hpp:21-62: FLT_MAX init, source 0, repeat full sweeps relaxing
 * d[dst] > d[src] + w with one float add until nothing changes. */
int orc_bellman_ford(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, const float *w,
                     int32_t source, float *dist)
{
    for (int32_t i = 0; i < V; i++) dist[i] = FLT_MAX;
    dist[source] = 0.0f;
    int sweeps = 0, changes = 1;
    while (changes) {
        sweeps++;
        changes = 0;
        for (int64_t e = 0; e < E; e++) {
            volatile float cand = dist[src[e]] + w[e]; /* one rounded fp32 add */
            if (dist[dst[e]] > cand) {
                dist[dst[e]] = cand;
                changes = 1;
            }
        }
    }
    return sweeps;
}

/* algorithm/scc/gpu/forward_backward.cu:71-99 and 139-170 (init_visited,
 * bfs_kernel, bfs): visited = pivot only, then repeat edge sweeps marking dst
 * when src is visited, src and dst lie in the same tree and dst is not yet
 * visited, until a sweep marks nothing.  Returns the sweep count. */
int orc_reach_masked(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, int32_t pivot,
                     const int32_t *trees, uint8_t *visited)
{
    for (int32_t i = 0; i < V; i++) visited[i] = 0;
    visited[pivot] = 1;
    int sweeps = 0, changes = 1;
    while (changes) {
        sweeps++;
        changes = 0;
        for (int64_t e = 0; e < E; e++) {
            const int32_t s = src[e], t = dst[e];
            if (visited[s] && trees[s] == trees[t] && !visited[t]) {
                visited[t] = 1;
                changes = 1;
            }
        }
    }
    return sweeps;
}

/* ---- binary heap keyed by float distance ---- */
typedef struct { float key; int32_t v; } heap_item;

static void heap_push(heap_item *h, int64_t *n, float key, int32_t v)
{
    int64_t i = (*n)++;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (h[p].key <= key) break;
        h[i] = h[p];
        i = p;
    }
    h[i].key = key;
    h[i].v = v;
}

static heap_item heap_pop(heap_item *h, int64_t *n)
{
    heap_item top = h[0];
    heap_item last = h[--(*n)];
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        float mk = last.key;
        if (l < *n && h[l].key < mk) { m = l; mk = h[l].key; }
        if (r < *n && h[r].key < mk) { m = r; }
        if (m == i) break;
        h[i] = h[m];
        i = m;
    }
    if (*n > 0) h[i] = last;
    return top;
}

void orc_dijkstra(int32_t V, const int64_t *offsets, const int32_t *adj, const float *w,
                  int32_t source, float *dist)
{
    for (int32_t i = 0; i < V; i++) dist[i] = FLT_MAX;
    dist[source] = 0.0f;
    int64_t cap = offsets[V] + 1, n = 0;
    heap_item *h = (heap_item *)malloc(sizeof(heap_item) * (size_t)cap);
    heap_push(h, &n, 0.0f, source);
    while (n > 0) {
        heap_item it = heap_pop(h, &n);
        if (it.key != dist[it.v]) continue; /* stale */
        for (int64_t k = offsets[it.v]; k < offsets[it.v + 1]; k++) {
            volatile float cand = it.key + w[k];
            if (cand < dist[adj[k]]) {
                dist[adj[k]] = cand;
                heap_push(h, &n, cand, adj[k]);
            }
        }
    }
    free(h);
}

void orc_build_csr(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, const float *w,
                   int64_t *offsets, int32_t *adj, float *wt)
{
    memset(offsets, 0, sizeof(int64_t) * ((size_t)V + 1));
    for (int64_t e = 0; e < E; e++) offsets[src[e] + 1]++;
    for (int32_t v = 0; v < V; v++) offsets[v + 1] += offsets[v];
    int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * ((size_t)V + 1));
    memcpy(cur, offsets, sizeof(int64_t) * ((size_t)V + 1));
    for (int64_t e = 0; e < E; e++) {
        int64_t k = cur[src[e]]++;
        adj[k] = dst[e];
        if (wt) wt[k] = w[e];
    }
    free(cur);
}

/* bfs.hpp:3-46 with level[dst] = level[cur] + 1 recorded at push. */
int orc_bfs_levels(int32_t V, const int64_t *offsets, const int32_t *adj, int32_t source, int32_t *levels)
{
    for (int32_t i = 0; i < V; i++) levels[i] = -1;
    int32_t *queue = (int32_t *)malloc(sizeof(int32_t) * (size_t)(V > 0 ? V : 1));
    int64_t head = 0, tail = 0;
    queue[tail++] = source;
    levels[source] = 0;
    int maxl = 0;
    while (head < tail) {
        int32_t u = queue[head++];
        for (int64_t k = offsets[u]; k < offsets[u + 1]; k++) {
            int32_t v = adj[k];
            if (levels[v] < 0) {
                levels[v] = levels[u] + 1;
                if (levels[v] > maxl) maxl = levels[v];
                queue[tail++] = v;
            }
        }
    }
    free(queue);
    return maxl + 1;
}

/* ---- device layout ---- */
static const int32_t *g_sort_deg;
static int cmp_deg_desc(const void *pa, const void *pb)
{
    int32_t a = *(const int32_t *)pa, b = *(const int32_t *)pb;
    if (g_sort_deg[a] != g_sort_deg[b]) return g_sort_deg[a] > g_sort_deg[b] ? -1 : 1;
    return a < b ? -1 : (a > b);
}

typedef struct { uint32_t key; int64_t e; } row_item;
static int cmp_row_item(const void *pa, const void *pb)
{
    const row_item *a = (const row_item *)pa, *b = (const row_item *)pb;
    if (a->key != b->key) return a->key < b->key ? -1 : 1;
    return a->e < b->e ? -1 : (a->e > b->e);
}

/* Weight sort key: the bit pattern of a non-negative float orders like its
 * value; -0.0 is taken as +0.0. */
static uint32_t weight_key(float w)
{
    uint32_t u;
    if (w == 0.0f) w = 0.0f;
    memcpy(&u, &w, 4);
    return u;
}

void orc_device_layout(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, const float *w,
                       int32_t *new_of_old, int32_t *old_of_new,
                       int64_t *out_off, int32_t *out_adj, float *out_w,
                       int64_t *in_off, int32_t *in_adj)
{
    int32_t *deg = (int32_t *)calloc((size_t)V + 1, sizeof(int32_t));
    for (int64_t e = 0; e < E; e++) deg[src[e]]++;
    for (int32_t v = 0; v < V; v++) old_of_new[v] = v;
    g_sort_deg = deg;
    qsort(old_of_new, (size_t)V, sizeof(int32_t), cmp_deg_desc);
    for (int32_t r = 0; r < V; r++) new_of_old[old_of_new[r]] = r;

    /* out rows: key = weight, tie by edge order; in rows: key = new src, tie by edge order */
    int64_t *ecount = (int64_t *)calloc((size_t)V + 1, sizeof(int64_t));
    int64_t *icount = (int64_t *)calloc((size_t)V + 1, sizeof(int64_t));
    for (int64_t e = 0; e < E; e++) {
        ecount[new_of_old[src[e]] + 1]++;
        icount[new_of_old[dst[e]] + 1]++;
    }
    for (int32_t v = 0; v < V; v++) {
        ecount[v + 1] += ecount[v];
        icount[v + 1] += icount[v];
    }
    memcpy(out_off, ecount, sizeof(int64_t) * ((size_t)V + 1));
    memcpy(in_off, icount, sizeof(int64_t) * ((size_t)V + 1));
    row_item *oitems = (row_item *)malloc(sizeof(row_item) * (size_t)(E > 0 ? E : 1));
    row_item *iitems = (row_item *)malloc(sizeof(row_item) * (size_t)(E > 0 ? E : 1));
    for (int64_t e = 0; e < E; e++) {
        int32_t s = new_of_old[src[e]], t = new_of_old[dst[e]];
        int64_t k = ecount[s]++;
        oitems[k].key = weight_key(w[e]);
        oitems[k].e = e;
        int64_t j = icount[t]++;
        iitems[j].key = (uint32_t)s;
        iitems[j].e = e;
    }
    for (int32_t v = 0; v < V; v++) {
        qsort(oitems + out_off[v], (size_t)(out_off[v + 1] - out_off[v]), sizeof(row_item), cmp_row_item);
        qsort(iitems + in_off[v], (size_t)(in_off[v + 1] - in_off[v]), sizeof(row_item), cmp_row_item);
    }
    for (int64_t k = 0; k < E; k++) {
        const int64_t e = oitems[k].e;
        out_adj[k] = new_of_old[dst[e]];
        out_w[k] = w[e] == 0.0f ? 0.0f : w[e];
        in_adj[k] = (int32_t)iitems[k].key;
    }
    free(oitems);
    free(iitems);
    free(ecount);
    free(icount);
    free(deg);
}

int64_t orc_sssp_bytes(int32_t V, const int64_t *offsets, const float *dist)
{
    int64_t b = 4 * (int64_t)V;
    for (int32_t v = 0; v < V; v++)
        if (dist[v] < FLT_MAX) b += 12 + 12 * (offsets[v + 1] - offsets[v]);
    return b;
}

int64_t orc_bfs_bytes(int32_t V, const int64_t *out_off, const int64_t *in_off, const int32_t *in_adj,
                      const int32_t *levels_new, const uint8_t *dirs, int nsteps)
{
    int64_t b = 4 * (int64_t)V;
    for (int s = 0; s < nsteps; s++) {
        if (dirs[s] == 0) {
            for (int32_t v = 0; v < V; v++) {
                if (levels_new[v] == s) b += 12 + 8 * (out_off[v + 1] - out_off[v]);
                if (levels_new[v] == s + 1) b += 8;
            }
        } else {
            for (int32_t v = 0; v < V; v++) {
                int32_t lv = levels_new[v];
                if (lv >= 0 && lv <= s) continue; /* already visited */
                b += 12;
                int64_t k = in_off[v];
                for (; k < in_off[v + 1]; k++) {
                    b += 8;
                    if (levels_new[in_adj[k]] == s) break;
                }
                if (lv == s + 1) b += 4;
            }
        }
    }
    return b;
}

double orc_mlp_loss_grad(int F, int H, int O, const double *params, int n, const double *x,
                         const int32_t *label, double *grad)
{
    const double *W1 = params, *b1 = W1 + H * F, *W2 = b1 + H, *b2 = W2 + H * H, *W3 = b2 + H, *b3 = W3 + O * H;
    int np = H * F + H + H * H + H + O * H + O;
    double *gW1 = grad, *gb1 = gW1 + H * F, *gW2 = gb1 + H, *gb2 = gW2 + H * H, *gW3 = gb2 + H, *gb3 = gW3 + O * H;
    if (grad) memset(grad, 0, sizeof(double) * (size_t)np);
    double *h1 = (double *)malloc(sizeof(double) * (size_t)H), *h2 = (double *)malloc(sizeof(double) * (size_t)H);
    double *y = (double *)malloc(sizeof(double) * (size_t)O), *dy = (double *)malloc(sizeof(double) * (size_t)O);
    double *d2 = (double *)malloc(sizeof(double) * (size_t)H), *d1 = (double *)malloc(sizeof(double) * (size_t)H);
    double loss = 0.0;
    for (int s = 0; s < n; s++) {
        const double *xs = x + (size_t)s * F;
        for (int j = 0; j < H; j++) {
            double a = b1[j];
            for (int i = 0; i < F; i++) a += W1[j * F + i] * xs[i];
            h1[j] = tanh(a);
        }
        for (int j = 0; j < H; j++) {
            double a = b2[j];
            for (int i = 0; i < H; i++) a += W2[j * H + i] * h1[i];
            h2[j] = tanh(a);
        }
        double m = -1e300;
        for (int o = 0; o < O; o++) {
            double a = b3[o];
            for (int i = 0; i < H; i++) a += W3[o * H + i] * h2[i];
            y[o] = a;
            if (a > m) m = a;
        }
        double z = 0.0;
        for (int o = 0; o < O; o++) z += exp(y[o] - m);
        loss += -(y[label[s]] - m - log(z));
        if (!grad) continue;
        for (int o = 0; o < O; o++) dy[o] = (exp(y[o] - m) / z - (o == label[s] ? 1.0 : 0.0)) / n;
        for (int i = 0; i < H; i++) d2[i] = 0.0;
        for (int o = 0; o < O; o++) {
            gb3[o] += dy[o];
            for (int i = 0; i < H; i++) {
                gW3[o * H + i] += dy[o] * h2[i];
                d2[i] += W3[o * H + i] * dy[o];
            }
        }
        for (int i = 0; i < H; i++) d2[i] *= (1.0 - h2[i] * h2[i]);
        for (int i = 0; i < H; i++) d1[i] = 0.0;
        for (int j = 0; j < H; j++) {
            gb2[j] += d2[j];
            for (int i = 0; i < H; i++) {
                gW2[j * H + i] += d2[j] * h1[i];
                d1[i] += W2[j * H + i] * d2[j];
            }
        }
        for (int i = 0; i < H; i++) d1[i] *= (1.0 - h1[i] * h1[i]);
        for (int j = 0; j < H; j++) {
            gb1[j] += d1[j];
            for (int i = 0; i < F; i++) gW1[j * F + i] += d1[j] * xs[i];
        }
    }
    free(h1); free(h2); free(y); free(dy); free(d2); free(d1);
    return loss / n;
}

/* ---------------------------------------------------------------- graph optimisation
 * GraphOptimizationAPI (include/test/optimization/graph_optimization_API.hpp):
 *   reorder_edges_in_adjacency_list_format :14-55  sort edges by (src, dst, weight)
 *   remove_loops_and_multiple_arcs          :60-117 drop loops; drop an edge whose (src, dst) equals the
 *                                                   previous sorted edge's (so the lightest arc is kept)
 *   reorder_edges_for_cache                 :122-166 sort by (src / seg, dst / seg); std::sort leaves the
 *                                                   order inside a segment pair unspecified -- here it is the
 *                                                   (src, dst, weight) order (a stable sort)
 * Weights compare as floats; -0.0 is read as +0.0 first so that equal weights have equal bits. */
typedef struct {
    int32_t s, d;
    float w;
    int64_t pos;
} opt_edge;

static int cmp_sdw(const void *pa, const void *pb)
{
    const opt_edge *a = (const opt_edge *)pa, *b = (const opt_edge *)pb;
    if (a->s != b->s) return a->s < b->s ? -1 : 1;
    if (a->d != b->d) return a->d < b->d ? -1 : 1;
    if (a->w != b->w) return a->w < b->w ? -1 : 1;
    return a->pos < b->pos ? -1 : (a->pos > b->pos);
}

static int32_t g_seg;
static int cmp_segments(const void *pa, const void *pb)
{
    const opt_edge *a = (const opt_edge *)pa, *b = (const opt_edge *)pb;
    const int32_t sa = a->s / g_seg, sb = b->s / g_seg, da = a->d / g_seg, db = b->d / g_seg;
    if (sa != sb) return sa < sb ? -1 : 1;
    if (da != db) return da < db ? -1 : 1;
    return a->pos < b->pos ? -1 : (a->pos > b->pos);
}

int64_t orc_el_optimize(int64_t E, const int32_t *src, const int32_t *dst, const float *w, int32_t segment,
                        int32_t *out_src, int32_t *out_dst, float *out_w)
{
    opt_edge *e = (opt_edge *)malloc(sizeof(opt_edge) * (size_t)(E > 0 ? E : 1));
    for (int64_t i = 0; i < E; i++) {
        e[i].s = src[i];
        e[i].d = dst[i];
        e[i].w = w[i] == 0.0f ? 0.0f : w[i];
        e[i].pos = i;
    }
    qsort(e, (size_t)E, sizeof(opt_edge), cmp_sdw);
    int64_t n = 0;
    for (int64_t i = 0; i < E; i++) {
        if (e[i].s == e[i].d) continue;
        if (i > 0 && e[i].s == e[i - 1].s && e[i].d == e[i - 1].d) continue;
        e[n] = e[i];
        e[n].pos = n;
        n++;
    }
    if (segment > 0) {
        g_seg = segment;
        qsort(e, (size_t)n, sizeof(opt_edge), cmp_segments);
    }
    for (int64_t i = 0; i < n; i++) {
        out_src[i] = e[i].s;
        out_dst[i] = e[i].d;
        out_w[i] = e[i].w;
    }
    free(e);
    return n;
}

/* check_gpu_memory_transactions_count (graph_optimization_API.hpp:229-266): for each warp of 32 consecutive
 * edges, the distinct 128-byte segments of src * elem_size plus those of dst * elem_size.  The reference adds a
 * warp's count when the next warp starts, so the warp holding the last edge is never added; kept. */
int64_t orc_gpu_transactions(int64_t E, const int32_t *src, const int32_t *dst, int32_t elem_size)
{
    const int64_t counted = E > 0 ? (E - 1) / 32 : 0;  /* warps before the one holding the last edge */
    int64_t total = 0;
    for (int64_t k = 0; k < counted; k++) {
        int64_t ss[32], ds[32];
        int ns = 0, nd = 0;
        for (int64_t i = 32 * k; i < 32 * k + 32; i++) {
            const int64_t a = (int64_t)src[i] * elem_size / 128, b = (int64_t)dst[i] * elem_size / 128;
            int j;
            for (j = 0; j < ns && ss[j] != a; j++) {}
            if (j == ns) ss[ns++] = a;
            for (j = 0; j < nd && ds[j] != b; j++) {}
            if (j == nd) ds[nd++] = b;
        }
        total += ns + nd;
    }
    return total;
}
