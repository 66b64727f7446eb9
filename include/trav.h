/* trav.h -- C ABI of the B200 traversal library (libtrav_b200.so).
 *
 * Single-source shortest paths (Bellman-Ford and delta-stepping over the same
 * relaxation) and breadth-first search (top-down / bottom-up) on one NVIDIA
 * B200, behind plain C entry points: pointers, sizes and an int status.
 *
 * Conventions
 *  - Every function returns TRAV_OK (0) or a negative TRAV_ERR_* code; the
 *    message of the last failure on the calling thread is trav_last_error().
 *  - Vertex ids are int32 in [0, V); edge counts are int64 but a graph must
 *    hold fewer than 2^31 edges (the device CSR uses int32 offsets).
 *  - Weights are fp32, finite and >= 0.  Distances are fp32 with FLT_MAX for
 *    unreachable vertices, exactly as the reference library writes them;
 *    every result is bit-identical to the reference's CPU Bellman-Ford.
 *  - BFS levels are int32 hop counts, -1 for unreachable vertices.
 *  - `mem` arguments say where a buffer lives: TRAV_MEM_HOST (pageable or
 *    pinned host memory) or TRAV_MEM_DEVICE (CUDA device memory of the
 *    current device).
 *  - A graph handle is not thread-safe: use one handle per host thread.
 *    Each handle owns a CUDA stream; calls return after their work finishes.
 */
#ifndef TRAV_H
#define TRAV_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TRAV_OK 0
#define TRAV_ERR_BAD_ARG (-1)        /* invalid argument (ids, sizes, weights, options) */
#define TRAV_ERR_OOM (-2)            /* device or host allocation failed */
#define TRAV_ERR_OVERFLOW_INT32 (-3) /* graph has 2^31 or more edges */
#define TRAV_ERR_TIMEOUT (-4)        /* device step budget or bounded wait exhausted */
#define TRAV_ERR_CUDA (-5)           /* CUDA runtime error */
#define TRAV_ERR_NO_DEVICE (-6)      /* no usable CUDA device */
#define TRAV_ERR_IO (-7)             /* file could not be read or written / bad format */

#define TRAV_MEM_HOST 0
#define TRAV_MEM_DEVICE 1

#define TRAV_SCHEDULE_PLAIN 0   /* Beamer alpha/beta switch; fixed delta */
#define TRAV_SCHEDULE_LEARNED 1 /* the schedule MLP decides per step */

typedef struct trav_graph trav_graph;

/* Options of a BFS query.  alpha/beta: Beamer's direction-switch constants
 * (top-down -> bottom-up when frontier out-edges > unvisited out-edges / alpha;
 * back when the frontier shrinks below V / beta).  force_direction: -1 = use
 * the schedule, 0 = top-down only, 1 = bottom-up after the first step. */
typedef struct {
    int32_t schedule;
    float alpha;
    float beta;
    int32_t force_direction;
} trav_bfs_opts;

/* Options of an SSSP query.  delta <= 0 or +inf selects Bellman-Ford (one
 * bucket: every improved vertex is relaxed in the next round); delta > 0
 * selects delta-stepping with buckets [k*delta, (k+1)*delta) processed in
 * order.  The distances are the same bits either way. */
typedef struct {
    int32_t schedule;
    float delta;
} trav_sssp_opts;

/* Per-query record of the most recent query on a handle. */
typedef struct {
    int32_t kind;            /* 0 = BFS, 1 = SSSP */
    int32_t steps;           /* BFS levels expanded / SSSP relaxation rounds */
    int32_t buckets;         /* SSSP buckets opened (0 for BFS) */
    int32_t bottom_up_steps; /* BFS steps run bottom-up */
    int64_t reached;         /* vertices with a finite result */
    int64_t reached_edges;   /* out-edges of reached vertices */
    int64_t algorithmic_bytes; /* schedule-independent byte count of the query */
    float kernel_ms;         /* device time of the query's traversal launch */
    int64_t edges_scanned;   /* out-edges expanded by top-down / relaxation steps (re-expansions included) */
} trav_query_stats;

/* ------------------------------------------------------------------ graphs */

/* Build a device graph from an edge list (src[e] -> dst[e], weight w[e]).
 * w may be NULL (all weights 1.0); weights must be finite and >= 0 (NaN,
 * infinite or negative weights are rejected with TRAV_ERR_BAD_ARG).  The
 * device copy is an int32 CSR with vertices relabelled by out-degree
 * (descending, ties by id), each row sorted by weight (-0.0 read as +0.0,
 * equal weights in edge-list order) so the edges lighter than any delta form
 * a prefix, plus the transposed CSR (rows sorted by source, with each
 * in-edge's weight) for bottom-up BFS and SSSP pull rounds; results are
 * reported in the caller's original ids.  Replaces the per-call edge-list upload of
 * SingleSourceShortestPaths::gpu_bellman_ford (algorithm/sssp/sssp.hpp:219-277)
 * and BFS::gpu_bfs (algorithm/bfs/bfs.hpp:212-254). */
int trav_graph_from_edges(int32_t vertices, int64_t edges, const int32_t *src, const int32_t *dst,
                          const float *w, int32_t mem, trav_graph **out);

/* Generate a seeded RMAT graph directly on the device and build it.  Restates
 * GraphGenerationAPI::R_MAT_parallel (include/test/generation/
 * graph_generation_API.hpp:403-484): V = 2^scale, V*avg edges, integer
 * percent quadrant probabilities a,b,c,d, weights rand_r/RAND_MAX.  Edge e
 * uses the rand_r stream of `seed` from LCG step 3*(scale+2)*e, so seed 0
 * equals the reference run with one thread.  If drop_self_loops, loops are
 * removed (stable).  The edge list is also written to src/dst/w when they
 * are non-NULL device buffers of V*avg entries; *edges_out gets the count. */
int trav_graph_rmat(int32_t scale, int32_t avg, int32_t a, int32_t b, int32_t c, int32_t d, uint32_t seed,
                    int32_t drop_self_loops, int32_t *src, int32_t *dst, float *w, int64_t *edges_out,
                    trav_graph **out);

int trav_graph_free(trav_graph *g);

int trav_graph_info(const trav_graph *g, int32_t *vertices, int64_t *edges, int32_t *max_out_degree);

/* Copy the device layout to host arrays (any may be NULL): new_of_old[V],
 * old_of_new[V], out_off[V+1], out_adj[E], out_w[E], in_off[V+1], in_adj[E]. */
int trav_graph_export(const trav_graph *g, int32_t *new_of_old, int32_t *old_of_new, int32_t *out_off,
                      int32_t *out_adj, float *out_w, int32_t *in_off, int32_t *in_adj);

/* Copy the weight of every in-edge (in_w[E], the order of in_adj) to a host
 * array.  The reference keeps no transposed weights; the SSSP pull rounds
 * read them. */
int trav_graph_export_in_w(const trav_graph *g, float *in_w);

/* ----------------------------------------------------------------- queries */

/* BFS levels from each of n sources: levels[q*V + v].  Replaces
 * BFS::gpu_bfs / bfs_wrapper (algorithm/bfs/bfs.hpp:212-254,
 * algorithm/bfs/gpu/bfs.cu:43-81), which return only reachability. */
int trav_bfs(trav_graph *g, const int32_t *sources, int32_t n, const trav_bfs_opts *opts,
             int32_t *levels, int32_t mem);

/* SSSP distances from each of n sources: dist[q*V + v].  Replaces
 * SingleSourceShortestPaths::gpu_bellman_ford (algorithm/sssp/sssp.hpp:219-277)
 * and bellman_ford_wrapper (algorithm/sssp/gpu/bellman_ford.cu:103-144). */
int trav_sssp(trav_graph *g, const int32_t *sources, int32_t n, const trav_sssp_opts *opts,
              float *dist, int32_t mem);

/* Statistics of the last query (of the last source of a batch). */
int trav_last_stats(trav_graph *g, trav_query_stats *out);

/* Device time (ms, CUDA events on the launching stream) of each traversal
 * launch of the last batch; *n receives the batch size. */
int trav_last_batch_ms(trav_graph *g, float *ms, int32_t cap, int32_t *n);

/* Run this handle's queries on the caller's CUDA stream (a cudaStream_t;
 * NULL restores the handle's own stream).  Calls still return after their
 * work has finished. */
int trav_graph_set_stream(trav_graph *g, void *stream);

/* Per-step trace of the last BFS query: dirs[s] (0 top-down, 1 bottom-up) and
 * frontier[s] (vertices on the frontier of step s), up to cap entries.
 * *nsteps receives the step count. */
int trav_last_bfs_trace(trav_graph *g, uint8_t *dirs, int64_t *frontier, int32_t cap, int32_t *nsteps);

/* Phase log of the last query (the last source of a batch): per grid-wide
 * phase, its kind (0 BFS top-down step, 1 BFS bottom-up step, 2 BFS
 * frontier-bitmap build, 3 SSSP light relaxation round, 4 SSSP bucket
 * opening, 5 SSSP heavy round pushing the heavy list's out-rows, 6 SSSP pull
 * check listing the vertices a heavy edge could still improve, 7 SSSP heavy
 * round pulling over those vertices' in-rows), the frontier size it started
 * from, its end time in microseconds after the query's initialisation
 * and the cumulative out-edges expanded.  Up to cap entries; *n receives the
 * phase count.  New; the reference has no equivalent. */
int trav_last_phase_log(trav_graph *g, uint8_t *kind, int64_t *size, double *end_us, int64_t *edges, int32_t cap,
                        int32_t *n);

/* ------------------------------------- reference-shaped entry points (EL) */

/* init_kernel / init_distances_wrapper<float> (algorithm/sssp/gpu/
 * bellman_ford.cu:10-56): d[i] = FLT_MAX, d[source] = 0 on device memory. */
int trav_init_distances_f32(float *d, int32_t vertices, int32_t source);

/* bellman_ford_wrapper<float> (algorithm/sssp/gpu/bellman_ford.cu:103-144):
 * device edge-list arrays, relaxes the caller's device distance array d to
 * its fixpoint (from whatever d holds, as the reference does). */
int trav_bellman_ford_el_f32(const int32_t *src, const int32_t *dst, const float *w, int32_t vertices,
                             int64_t edges, int32_t source, float *d);

/* bfs_wrapper (algorithm/bfs/gpu/bfs.cu:43-81): device edge-list arrays,
 * writes visited[v] = 1 / 0 (C++ bool layout) to device memory. */
int trav_bfs_el(const int32_t *src, const int32_t *dst, int32_t vertices, int64_t edges, uint8_t *visited,
                int32_t source);

/* The reachability sweep of the reference's SCC forward-backward step
 * (bfs(), algorithm/scc/gpu/forward_backward.cu:139-170, with its kernels
 * init_visited at :71-79 and bfs_kernel at :83-99, called forward and
 * backward at :267-268): from the vertex *pivot, follow the edges
 * src[e] -> dst[e] whose two ends lie in the same tree (trees[src] ==
 * trees[dst]); visited[v] = 1 for every vertex reached, else 0 (C++ bool
 * layout).  All arrays, pivot included, are device memory, as in the
 * reference; the backward sweep passes dst as src.  Runs on this library's
 * BFS kernels (the tree restriction is a vertex mask: only vertices of the
 * pivot's tree are ever reached).  Synchronous. */
int trav_reach_el_masked(const int32_t *src, const int32_t *dst, int32_t vertices, int64_t edges,
                         const int32_t *pivot, const int32_t *trees, uint8_t *visited);

/* ------------------------------------------------- allocation-free BFS */

/* BFS levels (top-down) over a CSR the caller already holds in device
 * memory, without allocating anything.  This entry point has no counterpart
 * in the reference.
 *
 * It is for callers that cannot call cudaMalloc: a process whose device
 * memory is owned by another allocator (for example a framework's caching
 * pool that has reserved the free memory), or a latency-critical service that
 * cannot accept the device-wide synchronisation cudaMalloc / cudaFree imply.
 * Every other entry point here allocates its workspace; this one takes all
 * of its scratch (levels, bitmap, queues, control block) from one static
 * 8 MiB device array that every GPU which loads the library holds until the
 * process exits.  Limits: 1 <= vertices <= 262144, 0 <= edges <= 16777216;
 * larger graphs are rejected with TRAV_ERR_BAD_ARG (use trav_bfs).
 *
 * row_offsets (V+1 int32), adj (E int32, ids in [0, V)) and levels (V int32,
 * written: hop level or -1) are device pointers in the caller's vertex ids;
 * a pointer that is not device (or managed) memory is rejected with
 * TRAV_ERR_BAD_ARG before any launch, and the CSR is checked on the GPU
 * before use.  Runs on `stream` (a cudaStream_t; NULL =
 * the legacy default stream) and returns after the work has finished.
 * The first call on a device looks up the device address of the static array
 * (cudaGetSymbolAddress) once for that device; make that first call before
 * any stream capture begins.  All calls share the one array and leave their
 * contents in it: calls that overlap on the GPU (from two host threads or two
 * streams) race and must be serialised by the caller. */
int trav_bfs_csr_noalloc(const int32_t *row_offsets, const int32_t *adj, int32_t vertices, int64_t edges,
                         int32_t source, int32_t *levels, void *stream);

/* -------------------------------------------------- graph files (host only) */

/* Read an edge-list binary file in the reference format
 * (include/storage/graph_storage_API.hpp:114-160): bool directed, int32 V,
 * int64 E, then E records {int32 src, int32 dst, float w}.  Call with
 * src == NULL to get V, E and directed only.  With unweighted != 0 the records
 * are {int32 src, int32 dst} (generator.cpp:51-72) and w is filled with 1.0. */
int trav_el_file_read(const char *path, int32_t unweighted, int32_t *vertices, int64_t *edges,
                      int32_t *directed, int32_t *src, int32_t *dst, float *w);

/* Write the same format (include/storage/graph_storage_API.hpp:39-65). */
int trav_el_file_write(const char *path, int32_t directed, int32_t vertices, int64_t edges,
                       const int32_t *src, const int32_t *dst, const float *w);

/* Read an adjacency-list binary file in the reference format
 * (GraphStorageAPI::load_from_adjacency_list_bin_file,
 * include/storage/graph_storage_API.hpp:69-111): the same 13-byte header
 * (bool directed, int32 V, int64 E), then per vertex a Vertex<int> record
 * {int32 id, int32 value}, an int32 connection count and that many
 * {int32 dst, float32 w} records.  Call with offsets == NULL to get V, E and
 * directed only; otherwise ids[V], values[V], offsets[V+1] (row v holds
 * edges [offsets[v], offsets[v+1]) in file order, its source is ids[v]),
 * dst[E] and w[E] are filled.  A file whose records do not add up to the
 * header's E, ends inside a record or has bytes after the last one is
 * rejected with TRAV_ERR_IO. */
int trav_adj_file_read(const char *path, int32_t *vertices, int64_t *edges, int32_t *directed, int32_t *ids,
                       int32_t *values, int64_t *offsets, int32_t *dst, float *w);

/* Write the same format (GraphStorageAPI::save_to_adjacency_list_bin_file,
 * include/storage/graph_storage_API.hpp:3-35) from the arrays
 * trav_adj_file_read returns. */
int trav_adj_file_write(const char *path, int32_t directed, int32_t vertices, int64_t edges, const int32_t *ids,
                        const int32_t *values, const int64_t *offsets, const int32_t *dst, const float *w);

/* Read a headerless file of {int32 src, int32 dst} pairs as the BFS sample's
 * read_data_from_file does (sample/bfs.cpp:84-114): V = 2^vertices_pow, and
 * the edge count is file_size / 12 -- the reference sizes it for 12-byte
 * weighted records but reads 8-byte pairs, so it takes the first
 * file_size / 12 pairs of the file, and that count is kept here.  Every
 * weight is 1.0.  Call with src == NULL to get V and E only. */
int trav_pairs_file_read(const char *path, int32_t vertices_pow, int32_t *vertices, int64_t *edges, int32_t *src,
                         int32_t *dst, float *w);

/* ------------------------------------------------------- learned schedule */

/* Install the parameters of a schedule MLP on a handle (copied to the
 * device).  kind 0 = BFS direction (2 outputs: top-down, bottom-up);
 * kind 1 = SSSP bucket width (6 outputs: delta x 1, 4, 16, 64, 256, 1024).  count must be
 * trav_mlp_param_count(kind).  Layout: [W1 (32x10) | b1 (32) | W2 (32x32) |
 * b2 (32) | W3 (Ox32) | b3 (O)], row-major, tanh hidden units.  New; the
 * reference has no learned schedule. */
int trav_mlp_set(trav_graph *g, int32_t kind, const float *params, int32_t count);

/* The learned schedule's choice of delta for this graph: TRAV_SCHEDULE_LEARNED
 * SSSP queries (single and batched) on this handle run with delta x scale as
 * the light/heavy threshold and as the unit of the bucket widths their
 * network picks; plain queries keep the caller's delta.  scale is chosen per
 * graph by the learned split model from the graph's degree and weight
 * statistics (pytrav.learn); default 1.  The distances are the same bits for
 * every delta.  New. */
int trav_set_sssp_split(trav_graph *g, float scale);

/* Mean edge weight of a graph (a schedule feature). */
int trav_graph_mean_weight(const trav_graph *g, float *mean_weight);

/* Abstention margin of the kind's schedule network on this handle: at each
 * decision the network keeps the plain schedule's option (Beamer's direction;
 * delta x 1) unless its best output logit beats that option's logit by at
 * least margin.  0 (the default) takes the plain argmax.  New. */
int trav_mlp_set_margin(trav_graph *g, int32_t kind, float margin);
int32_t trav_mlp_param_count(int32_t kind);

/* Softmax cross-entropy loss of the kind's MLP on n samples (x: n x 10
 * features, labels in [0, outputs)) and its gradient, computed on the GPU by
 * the training kernels (forward + backward, one warp per sample).  Host
 * buffers; grad has trav_mlp_param_count(kind) entries (may be NULL). */
int trav_mlp_loss_grad(int32_t kind, const float *params, const float *x, const int32_t *labels, int32_t n,
                       float *grad, float *loss);

/* Train the kind's MLP in place on the GPU: `epochs` full-batch Adam steps
 * (beta1 0.9, beta2 0.999) with learning rate lr; *final_loss (may be NULL)
 * receives the loss after training. */
int trav_mlp_train(int32_t kind, float *params, const float *x, const int32_t *labels, int32_t n, int32_t epochs,
                   float lr, float *final_loss);

/* CUDA-graph capture (on != 0): a trav_bfs / trav_sssp call with device
 * outputs is recorded into a CUDA graph the first time and replayed, with no
 * per-query launch work on the host, while the call's arguments (sources,
 * output array, options, launch shape, stream) repeat; any change records a
 * new graph.  Off by default.  No counterpart in the reference. */
int trav_graph_set_capture(trav_graph *g, int32_t on);

/* Launch shape of the following queries of one kind on this handle: the
 * persistent kernel runs `ctas` CTAs of 256 threads (1 <= ctas <= the number
 * the device can hold at once, which *max_ctas receives when not NULL);
 * ctas == 0 restores that maximum.  Results do not depend on it; small graphs
 * and long chains of small steps can run faster on fewer CTAs, because every
 * step ends with a grid barrier that all CTAs join.  No counterpart in the
 * reference. */
int trav_set_grid(trav_graph *g, int32_t kind, int32_t ctas, int32_t *max_ctas);

/* Limits of the following trav_bfs / trav_sssp queries on this handle (batch
 * launches keep the defaults).  max_steps caps a query's
 * steps (BFS levels; SSSP relaxation rounds plus bucket openings) below its
 * default budget (BFS V + 1, SSSP 4V + 4096); 0 restores the default.
 * timeout_ns bounds every wait of a grid barrier inside the persistent
 * kernels; 0 restores the default of 10 s.  A query that runs out of either
 * returns TRAV_ERR_TIMEOUT (trav_last_error says which) and leaves the
 * handle usable.  The reference's counterpart is the V-iteration cap of
 * bellman_ford_wrapper (algorithm/sssp/gpu/bellman_ford.cu:126); its BFS
 * loop has none (algorithm/bfs/gpu/bfs.cu:69). */
int trav_set_limits(trav_graph *g, int32_t max_steps, uint64_t timeout_ns);

/* Fault injection for tests of the out-of-memory paths: after `after` more
 * device allocations by this library succeed, the next one fails as
 * cudaMalloc fails when the device is full (TRAV_ERR_OOM), once; -1 disarms.
 * Process-wide.  No counterpart in the reference. */
int trav_inject_alloc_failure(int32_t after);

/* Force the schedule's decisions for the following queries of one kind on
 * this handle (used to time alternatives when building training traces):
 * decision i takes option plan[i] when plan[i] < 255 and follows the schedule
 * otherwise.  BFS decision i is the direction of step i (0 top-down, 1
 * bottom-up); SSSP decision i is the width option of the i-th bucket opening
 * (0..5: delta x 1, 4, 16, 64, 256, 1024).  n == 0 clears the plan. */
int trav_set_plan(trav_graph *g, int32_t kind, const uint8_t *plan, int32_t n);

/* Decisions of the last query (the last source of a batch): per decision the
 * 10 MLP input features (x[i*10 + k]), the option taken, the index of the
 * phase it opened (see trav_last_phase_log) and, for SSSP, the new bucket
 * [lo, hi).  Up to cap entries (any array may be NULL); *n receives the count. */
int trav_last_decisions(trav_graph *g, float *x, uint8_t *choice, int32_t *phase, float *lo, float *hi, int32_t cap,
                        int32_t *n);

/* ------------------------------------------------------------------- misc */

const char *trav_last_error(void);
const char *trav_version(void);

/* ------------------------------------------------------ graph optimisation
 * The optimisation pass of GraphOptimizationAPI on an edge list, in place
 * (replaces remove_loops_and_multiple_arcs and reorder_edges_for_cache,
 * include/test/optimization/graph_optimization_API.hpp:60-166): edges are
 * sorted by (src, dst, weight), self-loops and repeated arcs are dropped (the
 * lightest arc of each (src, dst) pair stays), and when segment > 0 the edges
 * are grouped by (src / segment, dst / segment) -- the reference's segment is
 * its L2 size / elem_size vertices -- keeping the (src, dst, weight) order
 * inside a group.  Weights of -0.0 become +0.0.  *edges_out receives the new
 * count; the arrays keep their capacity.  mem says where the arrays live
 * (TRAV_MEM_HOST arrays are copied to the device and back). */
int trav_el_optimize(int32_t *src, int32_t *dst, float *w, int32_t vertices, int64_t edges, int32_t segment,
                     int32_t mem, int64_t *edges_out);

/* Memory transactions of an edge-per-thread sweep over an edge list
 * (replaces check_gpu_memory_transactions_count,
 * graph_optimization_API.hpp:229-266): for each warp of 32 consecutive edges,
 * the distinct 128-byte segments among src * elem_size plus those among
 * dst * elem_size.  As in the reference, the warp holding the last edge is
 * not counted. */
int trav_el_gpu_transactions(const int32_t *src, const int32_t *dst, int32_t vertices, int64_t edges,
                             int32_t elem_size, int32_t mem, int64_t *count);

/* ----------------------------------------------------------------- batches
 * Many BFS / SSSP queries over several graphs in one persistent launch.  The
 * launch is cut into teams of CTAs; each team runs one query at a time and
 * takes the next one (largest first) when it is done, so graphs of very
 * different sizes share the GPU.  No counterpart in the reference, which runs
 * one query per call. */
typedef struct trav_batch trav_batch;

typedef struct {
    int32_t graph;    /* index into the batch's graph list */
    int32_t kind;     /* 0 = BFS (int32 levels, -1 unreached), 1 = SSSP (float distances, FLT_MAX unreached) */
    int32_t source;   /* vertex id of that graph */
    float delta;      /* SSSP bucket width; <= 0 or +inf = Bellman-Ford.  BFS: ignored */
    int32_t schedule; /* TRAV_SCHEDULE_PLAIN, or TRAV_SCHEDULE_LEARNED with the graph's network */
    void *out;        /* device array of the graph's V results */
} trav_query;

typedef struct {
    int32_t team_ctas; /* CTAs per team (256 threads each) */
    int32_t small_deg; /* rows of at most this many edges expand in warp tiles, 0..1024 */
    int32_t item;      /* longer rows are cut into items of this many edges, 64..8192 */
} trav_batch_shape;

/* A batch over n graph handles of one device (the handles stay the caller's
 * and must outlive the batch).  The shape starts at 16 CTAs per team, 32, 256. */
int trav_batch_create(trav_graph *const *graphs, int32_t n, trav_batch **out);
void trav_batch_free(trav_batch *b);

/* Run n queries in one launch and wait for it; *device_ms (may be NULL)
 * receives the launch's device time.  Every team holds scratch for the
 * batch's largest graph (about 80 bytes per vertex); when the device cannot
 * hold one per team, fewer teams of the same size run. */
int trav_batch_run(trav_batch *b, const trav_query *queries, int32_t n, float *device_ms);

/* The same queries with HOST output arrays (`out` = V results in host
 * memory; pinned memory lets the copies overlap the work).  Each query's
 * results are staged in device memory; the kernel raises a completion flag in
 * mapped host memory once a query's team has written them all, and the
 * calling thread, polling the flags while the launch runs, copies that
 * query's results to the host on a second stream.  So the copies overlap the
 * remaining queries and only the last ones follow the launch.  The queries
 * run as `parts` launches over consecutive slices of the array (slices
 * shrinking in the ratio 2 (parts - p) + 1); parts = 1 is normally fastest.
 * *device_ms (may be NULL) receives the summed device time of the launches.
 * Returns after the last copy has finished.  The reference's counterpart is
 * the per-call upload / kernel / copy-back of gpu_bellman_ford
 * (algorithm/sssp/sssp.hpp:219-277). */
int trav_batch_run_host(trav_batch *b, const trav_query *queries, int32_t n, int32_t parts, float *device_ms);

/* Process-wide table of the launch shapes the autotuner found, keyed by the
 * kind of batch: the device's co-resident CTAs, log2 of the largest queried
 * graph's V and E, log2 of the number of graphs and queries, and the shares
 * of SSSP and learned-schedule queries in eighths.  save writes it as text
 * lines "key team_ctas small_deg item"; load merges a saved table into the
 * current one (*entries, may be NULL, receives its size).  Malformed files
 * are rejected with TRAV_ERR_IO.  New; the reference has no autotuner. */
int trav_tune_table_save(const char *path);
int trav_tune_table_load(const char *path, int32_t *entries);

/* Time candidate shapes on these queries (each run `reps` times, best kept)
 * and keep the fastest for later runs; *best (may be NULL) receives it.  The
 * result is also recorded in the tuning table.  reps == 0 takes the table's
 * shape for this kind of batch without timing anything, and tunes once
 * (reps 1) when the table has none. */
int trav_batch_autotune(trav_batch *b, const trav_query *queries, int32_t n, int32_t reps,
                        trav_batch_shape *best);

int trav_batch_set_shape(trav_batch *b, const trav_batch_shape *shape);
int trav_batch_get_shape(const trav_batch *b, trav_batch_shape *shape);

#ifdef __cplusplus
}
#endif
#endif /* TRAV_H */
