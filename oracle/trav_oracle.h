/* Test infrastructure, not product code: the CPU oracle for the traversal path.
 *
 * A plain-C restatement of the reference library's single-source traversal
 * algorithms, used only by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline leg, always as the checker.  Each function cites the reference
 * file:line it restates.  It is pinned against the reference itself (the
 * harness in oracle/ref_harness.cpp compiled into oracle/_ref/) and against the
 * golden fixtures in tests/golden/.
 */
#ifndef TRAV_ORACLE_H
#define TRAV_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* glibc rand_r restated (three LCG steps per call, 31 output bits). */
int orc_rand_r(uint32_t *state);
/* Advance the rand_r LCG state by `steps` single LCG steps. */
uint32_t orc_lcg_skip(uint32_t state, uint64_t steps);

/* RMAT edge generator restating GraphGenerationAPI::R_MAT_parallel
 * (include/test/generation/graph_generation_API.hpp:403-484) for a directed
 * graph with V = 2^scale and E = V * avg edges.  Edge e draws scale+2 rand_r
 * values starting at LCG step 3*(scale+2)*e of `seed`, so output does not
 * depend on `threads`; seed 0 equals the reference run with one thread. */
void orc_rmat(int scale, int avg, int a, int b, int c, int d, uint32_t seed, int threads,
              int32_t *src, int32_t *dst, float *w);
/* Stable in-place removal of self-loops; returns the new edge count. */
int64_t orc_drop_self_loops(int64_t E, int32_t *src, int32_t *dst, float *w);

/* cpu_bellman_ford (algorithm/sssp/sssp.hpp:3-71), one thread: in-place sweeps
 * over the edge list in order until a sweep changes nothing. Returns sweeps. */
int orc_bellman_ford(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, const float *w,
                     int32_t source, float *dist);
/* The SCC forward-backward reachability sweep (algorithm/scc/gpu/
 * forward_backward.cu:71-99, 139-170): from pivot, edges whose ends share a
 * tree; visited[v] = 1 / 0.  Returns sweeps. */
int orc_reach_masked(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, int32_t pivot,
                     const int32_t *trees, uint8_t *visited);
/* Same fixpoint by label-setting (binary heap).  Equal bits to the sweep form
 * because fl(x + w) is monotone in x and >= x for w >= 0. */
void orc_dijkstra(int32_t V, const int64_t *offsets, const int32_t *adj, const float *w,
                  int32_t source, float *dist);

/* EL -> CSR in the reference's order (graph.hpp:248-361: each row keeps the
 * edge-list order of its source).  offsets has V+1 entries. */
void orc_build_csr(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, const float *w,
                   int64_t *offsets, int32_t *adj, float *wt);

/* cpu_sequential_bfs (algorithm/bfs/bfs.hpp:3-46) with a level recorded at
 * push time; -1 = unreached.  Returns the number of levels (max level + 1). */
int orc_bfs_levels(int32_t V, const int64_t *offsets, const int32_t *adj, int32_t source, int32_t *levels);

/* Device layout restated for checking the ingest path: vertices relabelled by
 * out-degree descending (ties by id); out rows sorted by (weight, edge order)
 * with -0.0 stored as +0.0; in rows sorted by (neighbour, edge order).
 * new_of_old / old_of_new have V entries; out_off/in_off V+1; out_adj, out_w,
 * in_adj E. */
void orc_device_layout(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, const float *w,
                       int32_t *new_of_old, int32_t *old_of_new,
                       int64_t *out_off, int32_t *out_adj, float *out_w,
                       int64_t *in_off, int32_t *in_adj);

/* Algorithmic bytes of one SSSP query: 4V + 12 V_r + 12 E_r. */
int64_t orc_sssp_bytes(int32_t V, const int64_t *offsets, const float *dist);
/* Algorithmic bytes of one BFS query on the device layout (new ids): 4V plus,
 * per step s with direction dirs[s] (0 top-down, 1 bottom-up):
 *  top-down : 12 B per frontier vertex + 8 B per out-edge + 8 B per new vertex
 *  bottom-up: 12 B per unvisited vertex + 8 B per in-edge examined up to and
 *             including the first parent on the frontier + 4 B per new vertex. */
int64_t orc_bfs_bytes(int32_t V, const int64_t *out_off, const int64_t *in_off, const int32_t *in_adj,
                      const int32_t *levels_new, const uint8_t *dirs, int nsteps);

/* Float64 reference of the schedule MLP (3 layers, tanh hidden units):
 * h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), y = W3 h2 + b3, loss =
 * softmax cross-entropy of y against label, averaged over the batch.
 * Parameters are packed [W1 (H x F), b1 (H), W2 (H x H), b2 (H), W3 (O x H), b3 (O)],
 * row-major.  grad receives d loss / d params (same packing). Returns loss. */
double orc_mlp_loss_grad(int F, int H, int O, const double *params, int n, const double *x,
                         const int32_t *label, double *grad);


/* Graph optimisation pass (GraphOptimizationAPI): sort by (src, dst, w), drop loops and repeated arcs,
 * then (segment > 0) group by (src / segment, dst / segment).  Returns the new edge count. */
int64_t orc_el_optimize(int64_t E, const int32_t *src, const int32_t *dst, const float *w, int32_t segment,
                        int32_t *out_src, int32_t *out_dst, float *out_w);

/* check_gpu_memory_transactions_count: distinct 128-byte segments per warp of 32 edges (last warp excluded). */
int64_t orc_gpu_transactions(int64_t E, const int32_t *src, const int32_t *dst, int32_t elem_size);

#ifdef __cplusplus
}
#endif
#endif
