// Internal declarations shared by the traversal library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/trav.h"

namespace trav {

constexpr int kBlock = 256;       // threads per CTA of the persistent kernels
constexpr int kWarps = kBlock / 32;
constexpr int kChunk = 512;       // edges per chunk item (two-phase expansion of the allocation-free BFS)
constexpr int kBigDegree = 512;   // rows longer than this are split into chunks there
constexpr int kSmallDeg = 32;     // one-phase expansion (default): rows up to this length go to the warp-tile queue
constexpr int kItem = 256;        // one-phase expansion (default): edges per chunk item of a longer row
constexpr int kMinItem = 64;      // smallest chunk item a launch may use (sizes the chunk lists)
constexpr int kMaxItem = 8192;
constexpr int kMaxSmallDeg = 1024;
constexpr int kMaxTrace = 4096;   // steps recorded per query
constexpr int kMaxDec = 1024;     // schedule decisions recorded per query
constexpr int kDecFeat = 10;      // features per decision (the schedule MLP's input width)
constexpr int kSlots = 4;         // ring of per-phase counter slots
constexpr unsigned long long kDefaultTimeoutNs = 10ull * 1000000000ull;  // grid-barrier wait limit (10 s)
// Row-class flags in the low bits of an SSSP distance word (dist_bits << 32 |
// round << kClsBits | flags): which parts of the vertex's out-row are non-empty
// and which are longer than the warp-tile threshold.  They depend only on the
// graph and delta, so the 64-bit atomicMin that lowers a distance keeps them.
// A copy in one byte per vertex (written at a query's initialisation) serves
// the pull rounds, which gather no word of the vertex they improve.
constexpr unsigned kClsLight = 1, kClsLightBig = 2, kClsHeavy = 4, kClsHeavyBig = 8;
constexpr unsigned kClsBits = 4, kClsMask = (1u << kClsBits) - 1u;
constexpr int kMaxRounds = (1 << (32 - kClsBits)) - 1;  // round ids of one SSSP launch must fit the stamp

// Device status codes written to Ctl::err.
constexpr int kErrTimeout = 1;    // a bounded grid-barrier wait gave up
constexpr int kErrBudget = 2;     // the step budget of a query ran out

// Counters produced by one phase; read by every CTA after the next barrier.
struct Slot {
    unsigned int q_add;           // entries appended to the next queue
    unsigned int far_add;         // entries appended to the far pile
    unsigned int chunk_add;       // chunk items appended
    int min_far_bits;             // min distance bits pushed to the far pile
    unsigned long long mf;        // out-degree sum of newly reached vertices
    unsigned int big_add;         // vertices pushed as chunk items (rows longer than kSmallDeg)
    unsigned int hq_add;          // SSSP heavy list: short heavy parts appended
    unsigned int hchunk_add;      // SSSP heavy list: chunk items appended
    unsigned int hbig_add;        // SSSP heavy list: vertices pushed as chunk items
    unsigned long long scanned;   // out-edges expanded in the phase
};
static_assert(sizeof(Slot) == 48 && offsetof(Slot, mf) == 16 && offsetof(Slot, scanned) == 40,
              "grid_sync reads Slot as twelve 32-bit words");

// Control block of one persistent launch (zeroed by the host before launch).
struct Ctl {
    unsigned long long bar_count;  // grid-barrier arrivals so far (only grows during a launch)
    int err;
    int err_phase;
    Slot slot[kSlots];
    // written by CTA 0 as the query runs
    int steps;
    int buckets;
    int bottom_up_steps;
    unsigned long long edges_scanned;  // out-edges expanded (push-side work, all steps)
    int nphase;                   // phases logged below
    int ndec;                     // schedule decisions logged below
    int cur_query;                // batch launches: the query the team runs next
    unsigned char dirs[kMaxTrace];       // BFS: direction of step s (0 top-down, 1 bottom-up)
    unsigned int frontier[kMaxTrace];    // BFS: frontier size of step s; SSSP: of expansion s
    // phase log (CTA 0, after each grid barrier): kind (0 top-down, 1 bottom-up,
    // 2 bitmap build, 3 light relaxation round, 4 bucket opening, 5 heavy
    // relaxation round), frontier size,
    // %globaltimer at the phase's end and cumulative edges_scanned
    unsigned char ph_kind[kMaxTrace];
    unsigned int ph_size[kMaxTrace];
    unsigned long long ph_end_ns[kMaxTrace];
    unsigned long long ph_scanned[kMaxTrace];
    unsigned long long t0_ns;     // %globaltimer after initialisation
    // schedule decisions (CTA 0): the MLP features, the choice taken, the
    // phase index the decision opened, and for SSSP the new bucket [lo, hi)
    float dec_x[kMaxDec][kDecFeat];
    unsigned char dec_choice[kMaxDec];
    int dec_phase[kMaxDec];
    float dec_lo[kMaxDec], dec_hi[kMaxDec];
};

// Device graph: int32 CSR over relabelled ids + transposed CSR.
struct DevGraph {
    int32_t V = 0;
    int64_t E = 0;
    int32_t max_out_degree = 0;
    float mean_w = 0.0f;          // mean edge weight (a schedule feature)
    int32_t *out_off = nullptr;   // V+1
    int32_t *out_adj = nullptr;   // E
    float *out_w = nullptr;       // E
    int32_t *in_off = nullptr;    // V+1
    int32_t *in_adj = nullptr;    // E
    float *in_w = nullptr;        // E: weight of each in-edge (the SSSP pull rounds)
    int32_t *new_of_old = nullptr;  // V
    int32_t *old_of_new = nullptr;  // V
};

// Light rows of a graph for one delta: the light-prefix length of every row
// and, when the light rows are packed (TRAV_LIGHT_ROWS), the prefixes
// themselves in a CSR of their own (see TravArgs::loff / ledge).
struct LightRows {
    float delta = -1.0f;          // < 0: not built
    int32_t *nlight = nullptr;    // V
    int32_t *loff = nullptr;      // V + 1; nullptr when the prefixes are not packed
    int2 *ledge = nullptr;        // loff[V] edges {target, weight bits}
    int64_t edges = 0;            // light edges of the graph for delta
};

// Per-handle traversal workspace (scratch memory of the persistent kernels).
struct Workspace {
    int32_t V = 0;
    int64_t chunk_cap = 0;
    // V 64-bit words: BFS levels (int32, the first V words) or SSSP distance
    // words (float bits << 32 | round << kClsBits | row-class flags)
    unsigned int *value = nullptr;
    unsigned char *rcls = nullptr;     // V: SSSP row-class flags (the pull rounds' copy)
    unsigned int *visited = nullptr;   // W words
    unsigned int *front[2] = {nullptr, nullptr};  // W words each
    int32_t *queue[2] = {nullptr, nullptr};       // V each
    int32_t *far[2] = {nullptr, nullptr};         // V each
    int32_t *hq[2] = {nullptr, nullptr};  // SSSP heavy lists (short heavy parts), V each
    int2 *hchunks[2] = {nullptr, nullptr};  // SSSP heavy lists (chunk items), chunk_cap each
    LightRows light;                   // light rows for the last finite delta (rows are sorted by weight)
    int2 *chunks[2] = {nullptr, nullptr};  // chunk_cap items each (current / next frontier)
    Ctl *ctl = nullptr;                // ctl_cap control blocks: one per query of a batch
    int ctl_cap = 0;
    unsigned char *plan[2] = {nullptr, nullptr};  // forced decisions for BFS / SSSP queries (device)
    int plan_len[2] = {0, 0};
    int grid[2] = {0, 0};              // CTAs of the BFS / SSSP launches (0 = as many as fit)
    int small_deg = kSmallDeg;         // expansion thresholds of the launches (see TravArgs)
    int item = kItem;
    int max_steps = 0;                 // step budget of a query; 0 = the default (see launch_bfs / launch_sssp)
    float mlp_margin[2] = {0.0f, 0.0f};  // abstention margins of the BFS / SSSP networks
    float split_scale = 1.0f;          // learned SSSP queries run with delta x split_scale (the learned split)
    unsigned long long timeout_ns = 0;  // bounded wait of a grid barrier; 0 = kDefaultTimeoutNs
};

// Arguments of the persistent kernels (passed by value).
struct TravArgs {
    // graph (read-only for the launch)
    const int32_t *__restrict__ out_off;
    const int32_t *__restrict__ out_adj;
    const float *__restrict__ out_w;
    const int32_t *__restrict__ in_off;
    const int32_t *__restrict__ in_adj;
    const float *__restrict__ in_w;   // in-edge weights; nullptr = no SSSP pull rounds
    const int32_t *__restrict__ new_of_old;
    int32_t V;
    int32_t W;        // bitmap words
    int64_t E;
    // workspace
    unsigned int *value;        // BFS levels
    unsigned long long *dist;   // SSSP distance words (same memory as value)
    unsigned char *rcls;        // SSSP row-class flags of each vertex (pull rounds)
    unsigned int *visited;
    unsigned int *front0, *front1;
    int32_t *q0, *q1;
    int32_t *far0, *far1;
    int32_t *hq0, *hq1;       // SSSP heavy lists
    int2 *hch0, *hch1;
    const int32_t *__restrict__ nlight;  // light-prefix length per vertex; nullptr = every edge is light
    // light rows (nullptr = none): the light prefixes packed by themselves,
    // row v = ledge[loff[v] .. loff[v+1]), each edge {target, weight bits}
    const int32_t *__restrict__ loff;
    const int2 *__restrict__ ledge;
    int2 *chunks;          // chunk items (two-phase expansion)
    int2 *chunks0, *chunks1;  // chunk items of the current / next frontier (one-phase expansion)
    Ctl *ctl;
    // query
    int32_t source;        // new id; -1 = start from the distance bits in init_bits
    const unsigned int *init_bits;  // source -1: V distance bits (new ids), read before the first barrier
    int32_t max_steps;
    // BFS options
    float alpha, beta;
    int32_t force_dir;
    // BFS vertex mask (new ids; nullptr = none): only vertices v with
    // color[v] == color_want are reached (the SCC sweeps' tree restriction)
    const int32_t *color;
    int32_t color_want;
    // SSSP options
    float delta;           // +inf = Bellman-Ford
    float mean_w;          // mean edge weight of the graph
    int32_t max_deg;       // largest out-degree of the graph
    // output (original ids); nullptr = leave results in `value`
    void *out;
    int32_t out_kind;      // 0 = int32 levels, 1 = float distances, 2 = uint8 reached flags
    // learned schedule (nullptr = plain); mlp_margin > 0: the network keeps
    // the plain option unless its best logit beats it by that much
    const float *mlp;
    float mlp_margin;
    // forced decisions: plan[i] (< 255) overrides decision i of the query
    const unsigned char *plan;
    int32_t plan_len;
    unsigned long long timeout_ns;
    // the CTAs that run this query: [cta0, cta0 + ctas) of the launch
    int32_t cta0, ctas;
    // expansion thresholds: rows (or row parts) longer than small_deg are cut
    // into item-edge chunk items, shorter ones go to the warp-tile queue
    int32_t small_deg, item;
};

// One query of a batch launch (device descriptor, built by the host).
struct BatchQuery {
    const int32_t *out_off, *out_adj, *in_off, *in_adj, *new_of_old;
    const float *out_w, *in_w;
    const int32_t *nlight;  // SSSP light-prefix lengths for delta; nullptr = Bellman-Ford
    const int32_t *loff;    // packed light rows (nullptr = none)
    const int2 *ledge;
    const float *mlp;       // schedule network; nullptr = plain schedule
    float mlp_margin;       // logit margin the network needs to leave the plain option
    void *out;              // results in original ids: int32 levels (BFS) or float distances (SSSP)
    int64_t E;
    int32_t V;
    int32_t kind;           // 0 = BFS, 1 = SSSP
    int32_t source;         // new id
    float delta;            // SSSP bucket width (+inf = Bellman-Ford)
    float mean_w;           // mean edge weight
    int32_t max_deg;        // largest out-degree
    int32_t id;             // position in the caller's query array (its completion flag)
};

// Scratch of one team of a batch launch, sized for the batch's largest graph.
struct TeamWs {
    unsigned int *value;  // 2 * Vmax words
    unsigned char *rcls;  // Vmax
    unsigned int *visited, *front0, *front1;
    int32_t *q0, *q1, *far0, *far1, *hq0, *hq1;
    int2 *chunks0, *chunks1, *hch0, *hch1;
    Ctl *ctl;
};

struct BatchArgs {
    const BatchQuery *queries;  // in dispatch order
    int32_t nq;
    unsigned int *next;         // dispatch counter, zero at launch
    const TeamWs *teams;
    int32_t team_ctas;          // CTAs per team; the launch has a whole number of teams
    int32_t full_ctas;          // co-resident CTAs of the device (a single query's grid)
    int32_t small_deg, item;
    unsigned long long timeout_ns;
    // completion flags in mapped host memory, one per query by BatchQuery::id
    // (nullptr = none): set once the query's results are all written
    unsigned *done;
};

__device__ __forceinline__ int team_tid(const TravArgs &a) { return (int)(blockIdx.x - a.cta0) * kBlock + (int)threadIdx.x; }
__device__ __forceinline__ int team_threads(const TravArgs &a) { return a.ctas * kBlock; }

// ---- host-side helpers (capi.cu) ----
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
// True when p is device or managed memory of the current context (a pointer
// the kernels may dereference); false for host memory and unknown pointers.
bool is_device_ptr(const void *p);

// Every device allocation of the library goes through dev_malloc: cudaMalloc,
// unless a test armed trav_inject_alloc_failure, in which case the armed
// allocation fails with cudaErrorMemoryAllocation as cudaMalloc would.
cudaError_t dev_malloc_bytes(void **p, size_t bytes);
template <class T>
inline cudaError_t dev_malloc(T **p, size_t bytes)
{
    return dev_malloc_bytes(reinterpret_cast<void **>(p), bytes);
}

// ingest.cu
int build_graph_device(int32_t V, int64_t E, const int32_t *d_src, const int32_t *d_dst, const float *d_w,
                       cudaStream_t st, DevGraph *out);
void free_graph(DevGraph *g);
int rmat_device(int scale, int avg, int a, int b, int c, int d, uint32_t seed, int drop_loops,
                int32_t *d_src, int32_t *d_dst, float *d_w, int64_t *E_out, cudaStream_t st);
int validate_edges(int32_t V, int64_t E, const int32_t *d_src, const int32_t *d_dst, const float *d_w,
                   cudaStream_t st);

// el_optimize.cu
int el_optimize_device(int32_t *src, int32_t *dst, float *w, int64_t E, int32_t segment, int64_t *E_out,
                       cudaStream_t st);
int el_transactions_device(const int32_t *src, const int32_t *dst, int64_t E, int32_t elem, int64_t *count,
                           cudaStream_t st);

// traverse.cu
int workspace_ensure(Workspace *ws, const DevGraph &g, int nqueries, cudaStream_t st);
void workspace_free(Workspace *ws);
// Enqueue one query on st using control block ws->ctl[q] (no host sync).
// ev0/ev1 (optional) are recorded around the launch.
// color (new ids, may be nullptr): reach only vertices with color[v] == color_want.
int launch_bfs(const DevGraph &g, Workspace *ws, int q, int32_t source_new, const trav_bfs_opts &o,
               const float *mlp, void *out, int out_kind, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
               const int32_t *color = nullptr, int32_t color_want = 0);
int launch_sssp(const DevGraph &g, Workspace *ws, int q, int32_t source_new, float delta, const float *mlp,
                void *out, int out_kind, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1);
// After the stream finished: turn the device status of queries [0, n) into a return code.
int check_queries(Workspace *ws, int n, const char *what);
int check_ctls(const Ctl *ctl, int n, const char *what);  // the same for n device control blocks
// Light-prefix length of every row of g for delta (rows are sorted by weight).
int count_light(const DevGraph &g, float delta, int32_t *nlight, cudaStream_t st);
// Build (or rebuild for a new delta) the light rows of g; no-op when lr already holds delta.
int light_rows_build(const DevGraph &g, float delta, LightRows *lr, cudaStream_t st);
void light_rows_free(LightRows *lr);
int query_bytes(const DevGraph &g, Workspace *ws, int q, int kind, int64_t *bytes, int64_t *reached,
                int64_t *reached_edges, cudaStream_t st);
int persistent_grid_size(int kind);  // kind 2 = the batch kernel
// Enqueue one batch launch of `teams` teams of b.team_ctas CTAs on st.
int launch_batch(BatchArgs b, int teams, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1);

}  // namespace trav
