// Persistent traversal kernels for sm_100a: BFS (top-down / bottom-up) and
// SSSP (Bellman-Ford and delta-stepping over one relaxation).
//
// One cooperative launch runs a whole query: initialisation, every step with
// a device-side decision between steps, and the write-back of results in the
// caller's vertex ids.  Steps are separated by a grid barrier whose wait is
// bounded in time; on timeout the kernel records kErrTimeout and returns.
//
// Reference counterparts (the reference sweeps the whole edge list per round
// with one thread per edge and a host round-trip per round):
//   bellman_ford_kernel / bellman_ford_wrapper  algorithm/sssp/gpu/bellman_ford.cu:62-144
//   init_kernel / init_distances_wrapper        algorithm/sssp/gpu/bellman_ford.cu:10-56
//   level_init_kernel / bfs_kernel / bfs_wrapper algorithm/bfs/gpu/bfs.cu:12-81
//   cpu_bellman_ford relaxation                 algorithm/sssp/sssp.hpp:47-61
//   cpu_parallel_bfs level loop                 algorithm/bfs/bfs.hpp:150-206
#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <climits>
#include <cmath>
#include <algorithm>
#include <cstddef>
#include <mutex>

#include "trav_internal.cuh"
#include "mlp_device.cuh"

namespace trav {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr unsigned kFltMaxBits = 0x7f7fffffu;

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_relaxed_int(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

// L2 eviction priorities.  The adjacency and weight arrays stream through
// once per phase while the distance words (8 B per vertex) are gathered at
// random over and over: streamed lines are marked evict-first and gathered
// ones evict-last, so the stream does not push the distances out of L2.
#ifndef TRAV_L2HINT
#define TRAV_L2HINT 1
#endif
__device__ __forceinline__ unsigned long long l2_policy_evict_first()
{
    unsigned long long pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ unsigned long long l2_policy_evict_last()
{
    unsigned long long pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// read-only stream load (non-coherent path), evict-first in L2
__device__ __forceinline__ int ld_stream(const int *p)
{
#if TRAV_L2HINT
    int v;
    asm("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(l2_policy_evict_first()));
    return v;
#else
    return __ldg(p);
#endif
}

__device__ __forceinline__ float ld_stream(const float *p) { return __int_as_float(ld_stream(reinterpret_cast<const int *>(p))); }

// one light-row edge {target, weight bits}: a single 8-byte load.  The light
// rows are re-read by every light round and by every concurrent query on the
// graph; TRAV_LIGHT_KEEP leaves them at the normal L2 priority instead of
// marking them evict-first like the other edge streams.
#ifndef TRAV_LIGHT_KEEP
#define TRAV_LIGHT_KEEP 0
#endif
__device__ __forceinline__ int2 ld_stream(const int2 *p)
{
#if TRAV_L2HINT && !TRAV_LIGHT_KEEP
    int2 v;
    asm("ld.global.nc.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;"
        : "=r"(v.x), "=r"(v.y)
        : "l"(p), "l"(l2_policy_evict_first()));
    return v;
#else
    return __ldg(p);
#endif
}

// gather of a mutable word at L2 (bypassing L1), evict-last in L2
__device__ __forceinline__ unsigned long long ld_gather(const unsigned long long *p)
{
#if TRAV_L2HINT
    unsigned long long v;
    asm volatile("ld.global.cg.L2::cache_hint.b64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(l2_policy_evict_last()));
    return v;
#else
    return __ldcg(p);
#endif
}

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

struct SlotView {
    unsigned q_add, far_add, chunk_add;
    int min_far_bits;  // kFltMaxBits when nothing was pushed
    unsigned long long mf;
    unsigned big_add;
    unsigned hq_add, hchunk_add, hbig_add;
    unsigned long long scanned;
};

// Grid-wide barrier with a bounded wait.  After the CTA barrier, thread 0 of
// every CTA adds one to a single arrival counter with an acquire-release
// atomic (which orders the CTA's writes of the phase before it).  The counter
// only grows, so barrier k of a launch is passed once it reaches
// k * gridDim.x: there is no reset and no generation word, and the critical
// path is one arrival plus one poll.  (A tree of reset counters puts a chain of
// dependent atomics and fences on that path instead.)  Waiters poll with an
// acquire load and give up after timeout_ns, or when another CTA already
// failed; the barrier then returns false in every thread of the CTA.
//
// With `view`, warp 0 also reads the counter slot of `phase` once for the
// whole CTA (one coalesced load) and leaves it decoded in shared memory: if
// every warp read the slot itself, the thousands of requests to one L2 line
// after each barrier would cost as much as a small phase.
__device__ bool grid_sync(const TravArgs &a, int phase, SlotView *view = nullptr)
{
    Ctl *ctl = a.ctl;
    const unsigned long long timeout_ns = a.timeout_ns;
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) {
            int ok = 1;
            const unsigned long long nb = (unsigned long long)a.ctas;
            unsigned long long old;
            asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], 1;" : "=l"(old) : "l"(&ctl->bar_count) : "memory");
            const unsigned long long target = (old / nb + 1) * nb;
            if (old + 1 != target) {
                const unsigned long long t0 = globaltimer();
                unsigned ns = 32;
                while (true) {
                    unsigned long long c;
                    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(c) : "l"(&ctl->bar_count) : "memory");
                    if (c >= target) break;
                    if (ld_relaxed_int(&ctl->err) != 0) { ok = 0; break; }
                    __nanosleep(ns);
                    if (ns < 128) ns <<= 1;
                    if (globaltimer() - t0 > timeout_ns) {
                        if (atomicCAS(&ctl->err, 0, kErrTimeout) == 0) atomicExch(&ctl->err_phase, phase);
                        ok = 0;
                        break;
                    }
                }
            }
            s_ok = ok;
        }
        __syncwarp();
        if (view) {
            // Slot is 48 bytes: lanes 0-11 load one word each
            const unsigned lane = threadIdx.x;
            const unsigned *w = reinterpret_cast<const unsigned *>(&ctl->slot[phase % kSlots]);
            const unsigned x = lane < sizeof(Slot) / 4 ? ld_relaxed_u32(w + lane) : 0u;
            unsigned f[12];
#pragma unroll
            for (int k = 0; k < 12; k++) f[k] = __shfl_sync(kFull, x, k);
            if (lane == 0) {
                view->q_add = f[0];
                view->far_add = f[1];
                view->chunk_add = f[2];
                const int neg = (int)f[3];  // stored as 0x7fffffff - bits via atomicMax
                view->min_far_bits = neg > 0 ? 0x7fffffff - neg : (int)kFltMaxBits;
                view->mf = (unsigned long long)f[4] | ((unsigned long long)f[5] << 32);
                view->big_add = f[6];
                view->hq_add = f[7];
                view->hchunk_add = f[8];
                view->hbig_add = f[9];
                view->scanned = (unsigned long long)f[10] | ((unsigned long long)f[11] << 32);
            }
        }
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ SlotView read_slot(const Ctl *ctl, int ph)
{
    const volatile Slot *s = &ctl->slot[ph % kSlots];
    SlotView v;
    v.q_add = s->q_add;
    v.far_add = s->far_add;
    v.chunk_add = s->chunk_add;
    int neg = s->min_far_bits;  // stored as 0x7fffffff - bits via atomicMax
    v.min_far_bits = neg > 0 ? 0x7fffffff - neg : (int)kFltMaxBits;
    v.mf = s->mf;
    v.big_add = s->big_add;
    v.hq_add = s->hq_add;
    v.hchunk_add = s->hchunk_add;
    v.hbig_add = s->hbig_add;
    v.scanned = s->scanned;
    return v;
}

// At the start of phase ph, slot ph+2 was last read right after phase ph-1's
// barrier by every CTA, so the first CTA can clear it for reuse in phase ph+2.
__device__ __forceinline__ void clear_ahead(const TravArgs &a, int ph)
{
    Ctl *ctl = a.ctl;
    if ((int)blockIdx.x == a.cta0 && threadIdx.x == 0) {
        Slot *s = &ctl->slot[(ph + 2) % kSlots];
        s->q_add = 0;
        s->far_add = 0;
        s->chunk_add = 0;
        s->min_far_bits = 0;
        s->mf = 0;
        s->big_add = 0;
        s->hq_add = 0;
        s->hchunk_add = 0;
        s->hbig_add = 0;
        s->scanned = 0;
    }
}

// Decision log entry (CTA 0 thread 0).  Returns the plan's override of
// decision `i` or -1.
__device__ __forceinline__ int planned(const TravArgs &a, int i)
{
    return (a.plan && i < a.plan_len && a.plan[i] != 255) ? (int)a.plan[i] : -1;
}

// Log counters.  Every thread that calls the log functions keeps them in
// registers; thread 0 of CTA 0 writes the logs with plain stores, so logging
// adds no load to the step's critical path (every CTA waits for CTA 0 at the
// next barrier).
struct PhaseLog {
    bool leader;                     // thread 0 of the query's first CTA
    int nphase = 0, ndec = 0;
    unsigned long long scanned = 0;  // edges expanded so far (sum of the slots' counts)
};

__device__ __forceinline__ void log_decision(Ctl *ctl, PhaseLog &lg, const Feat &f, int choice, float lo, float hi)
{
    if (lg.leader) {
        const int i = lg.ndec;
        if (i < kMaxDec) {
#pragma unroll
            for (int k = 0; k < kDecFeat; k++) ctl->dec_x[i][k] = f.x[k];
            ctl->dec_choice[i] = (unsigned char)choice;
            ctl->dec_phase[i] = lg.nphase;
            ctl->dec_lo[i] = lo;
            ctl->dec_hi[i] = hi;
        }
        ctl->ndec = i + 1;
    }
    lg.ndec++;
}

// Phase log entry, written by CTA 0 thread 0 right after a grid barrier.
__device__ __forceinline__ void log_phase(Ctl *ctl, PhaseLog &lg, int kind, unsigned size)
{
    if (lg.leader) {
        const int i = lg.nphase;
        if (i < kMaxTrace) {
            ctl->ph_kind[i] = (unsigned char)kind;
            ctl->ph_size[i] = size;
            ctl->ph_end_ns[i] = globaltimer();
            ctl->ph_scanned[i] = lg.scanned;
        }
        ctl->nphase = i + 1;
        ctl->edges_scanned = lg.scanned;
    }
    lg.nphase++;
}

// Warp-aggregated append: lanes with flag set write val to arr[base + k],
// one atomic per warp.  Must be called by all 32 lanes.
__device__ __forceinline__ void warp_append(bool flag, int val, int32_t *arr, unsigned base, unsigned *counter)
{
    unsigned m = __ballot_sync(kFull, flag);
    if (!m) return;
    unsigned leader = __ffs(m) - 1;
    unsigned pos = 0;
    if (lane_id() == leader) pos = atomicAdd(counter, (unsigned)__popc(m));
    pos = __shfl_sync(kFull, pos, leader);
    if (flag) arr[base + pos + __popc(m & lanemask_lt())] = val;
}

__device__ __forceinline__ void warp_add_u64(unsigned x, unsigned long long *counter)
{
    unsigned s = __reduce_add_sync(kFull, x);
    if (s && lane_id() == 0) atomicAdd(counter, (unsigned long long)s);
}

// ------------------------------------------------------------- visitors
// visit() is called by all 32 lanes of a warp together; `valid` marks lanes
// that carry an edge.  begin() returns the per-vertex value used by visit.

struct BfsTopDown {
    const TravArgs *a;
    int level_next;
    int32_t *qn;
    unsigned qbase;
    Slot *slot;

    __device__ __forceinline__ float begin(int) const { return 0.0f; }

    __device__ __forceinline__ void visit(int, float, int e, bool valid) const
    {
        bool fresh = false;
        int v = 0;
        if (valid) {
            v = __ldg(&a->out_adj[e]);
            unsigned bit = 1u << (v & 31);
            unsigned *wp = a->visited + (v >> 5);
            if (!(__ldcg(wp) & bit)) fresh = !(atomicOr(wp, bit) & bit);
        }
        unsigned deg = 0;
        if (fresh) {
            reinterpret_cast<int *>(a->value)[v] = level_next;
            deg = (unsigned)(__ldg(&a->out_off[v + 1]) - __ldg(&a->out_off[v]));
        }
        warp_append(fresh, v, qn, qbase, &slot->q_add);
        warp_add_u64(deg, &slot->mf);
    }
};

// ----------------------------------------------------- frontier expansion
struct TileShared {
    int u[kBlock];
    int rb[kBlock];
    int pre[kBlock];
    float du[kBlock];
    int wsum[kWarps];
    int total;
};

// Block-wide exclusive scan (kBlock threads); total in ts.total.
__device__ __forceinline__ int block_excl_scan(int x, TileShared &ts)
{
    const int lane = lane_id(), wid = threadIdx.x >> 5;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) ts.wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int s = lane < kWarps ? ts.wsum[lane] : 0;
        int si = s;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            int y = __shfl_up_sync(kFull, si, o);
            if (lane >= o) si += y;
        }
        if (lane < kWarps) ts.wsum[lane] = si - s;
        if (lane == kWarps - 1) ts.total = si;
    }
    __syncthreads();
    return incl - x + ts.wsum[wid];
}

// Phase 1 of a frontier expansion: tiles of kBlock frontier vertices per CTA.
// Rows of at most kBigDegree edges are expanded by the whole CTA (edge-
// balanced: a scan of the tile's degrees and a search for each edge's row);
// longer rows are cut into kChunk-edge items for phase 2.
template <class Vis>
__device__ void expand_tiles(const TravArgs &a, const int32_t *q, unsigned qlen, const Vis &vis, TileShared &ts,
                             Slot *slot)
{
    for (unsigned tile = blockIdx.x * kBlock; tile < qlen; tile += gridDim.x * kBlock) {
        unsigned i = tile + threadIdx.x;
        int u = 0, rb = 0, deg = 0;
        if (i < qlen) {
            u = __ldcg(&q[i]);
            rb = __ldg(&a.out_off[u]);
            deg = __ldg(&a.out_off[u + 1]) - rb;
            if (deg > kBigDegree) {
                int nch = (deg + kChunk - 1) / kChunk;
                unsigned base = atomicAdd(&slot->chunk_add, (unsigned)nch);
                for (int c = 0; c < nch; c++) a.chunks[base + c] = make_int2(u, rb + c * kChunk);
                deg = 0;
            }
        }
        int pre = block_excl_scan(deg, ts);
        ts.u[threadIdx.x] = u;
        ts.rb[threadIdx.x] = rb;
        ts.pre[threadIdx.x] = pre;
        ts.du[threadIdx.x] = deg > 0 ? vis.begin(u) : 0.0f;
        __syncthreads();
        const int total = ts.total;
        const int n = (int)min((unsigned)kBlock, qlen - tile);
        for (int base = 0; base < total; base += kBlock) {
            int k = base + threadIdx.x;
            bool valid = k < total;
            int lo = 0;
            if (valid) {
                int hi = n;
                while (hi - lo > 1) {
                    int mid = (lo + hi) >> 1;
                    if (ts.pre[mid] <= k) lo = mid;
                    else hi = mid;
                }
            }
            int e = ts.rb[lo] + (k - ts.pre[lo]);
            if (__any_sync(kFull, valid)) vis.visit(ts.u[lo], ts.du[lo], e, valid);
        }
        __syncthreads();
    }
}

// Phase 2: one warp per chunk item of a long row.
template <class Vis>
__device__ void expand_chunks(const TravArgs &a, unsigned nchunks, const Vis &vis)
{
    const unsigned warp = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const unsigned nwarps = (gridDim.x * kBlock) >> 5;
    for (unsigned c = warp; c < nchunks; c += nwarps) {
        int2 it = __ldcg(&a.chunks[c]);
        int u = it.x;
        int end = min(it.y + kChunk, __ldg(&a.out_off[u + 1]));
        float du = vis.begin(u);
        for (int e = it.y + (int)lane_id(); e - (int)lane_id() < end; e += 32) vis.visit(u, du, e, e < end);
    }
}

// ------------------------------------------------------- result write-back
// kDist: the results are SSSP packed distances (dist), else BFS levels (value).
template <bool kDist = false>
__device__ void write_back(const TravArgs &a)
{
    if (!a.out) return;
    const int gtid = team_tid(a), nth = team_threads(a);
    for (int v = gtid; v < a.V; v += nth) {
        const int r = __ldg(&a.new_of_old[v]);
        const unsigned x = kDist ? (unsigned)(__ldcg(&a.dist[r]) >> 32) : __ldcg(&a.value[r]);
        if (a.out_kind == 0) reinterpret_cast<int32_t *>(a.out)[v] = (int32_t)x;
        else if (a.out_kind == 1) reinterpret_cast<unsigned *>(a.out)[v] = x;
        else if (a.out_kind == 2) reinterpret_cast<unsigned char *>(a.out)[v] = (int32_t)x >= 0 ? 1 : 0;
        else reinterpret_cast<unsigned char *>(a.out)[v] = x != kFltMaxBits ? 1 : 0;
    }
}

// ------------------------------------------------------ one-phase frontier
// The next frontier is written in two parts while it is discovered: vertices
// whose row to expand has at most small_deg edges go to a queue that the next
// step expands in 32-vertex warp tiles; longer rows are cut into item-edge
// items, expanded one warp per item.  Both parts are complete when the step's
// barrier passes, so a step is one phase and one grid barrier, and the work of
// long rows is spread over every warp of the grid.
//
// Expansion is warp-centric: no CTA barrier inside a phase.  Every warp stages
// its pushes in its own shared-memory buffers and writes them out in bulk (one
// global atomic reserves room for up to a few hundred entries); the scalar
// counters are kept per warp and reduced per CTA once at the end of the phase.
//
// A push goes to one of two targets: target 0 is the next frontier (for SSSP
// its rows are the light prefixes, w < delta), target 1 is the SSSP heavy list
// (rows are the heavy suffixes).  Rows are sorted by weight, so both parts are
// contiguous: [off[v], off[v] + nlight[v]) and [off[v] + nlight[v], off[v+1]).
// Launch-shape constants, overridable at build time for tuning sweeps.
#ifndef TRAV_KBATCH_BFS
#define TRAV_KBATCH_BFS 4
#endif
#ifndef TRAV_KBATCH_SSSP
#define TRAV_KBATCH_SSSP 3
#endif
#ifndef TRAV_SSSP_MIN_BLOCKS
#define TRAV_SSSP_MIN_BLOCKS 4
#endif
#ifndef TRAV_BFS_MIN_BLOCKS
#define TRAV_BFS_MIN_BLOCKS 5
#endif
// Flushes run once per 64-128 staged entries.  Out of line they shrink the
// relaxation loop but force the pusher state into local memory, which costs
// more (a 1024x1024 grid SSSP took 90 instead of 52 ms).
// SSSP light rounds read packed light rows (1) or the light prefixes of the
// full rows (0); both give the same results.
#ifndef TRAV_LIGHT_ROWS
#define TRAV_LIGHT_ROWS 1
#endif
// Pull rounds stage one candidate per owner and batch, the min of a warp
// segment (1), or every improving in-edge (0); both give the same results.
#ifndef TRAV_PULL_REDUCE
#define TRAV_PULL_REDUCE 1
#endif
// BFS bottom-up steps count the vertices they find and leave them in the
// frontier bitmap only; a top-down step that follows builds its queue from
// that bitmap in one extra phase (1).  Or every bottom-up step pushes its
// found vertices to the queue as it goes (0).  Both give the same levels.
#ifndef TRAV_BU_LAZY
#define TRAV_BU_LAZY 1
#endif
// SSSP light rounds hold back long light rows more than this many deltas above
// the frontier's lowest distance while short rows remain (negative: never, and
// none of it is compiled in).  Summed over 64-query SSSP batches on four graphs
// (RMAT s23 ef32, s24 ef16, a flatter RMAT 45/25/15/15, uniform 2^23): 850 ms
// never, 822 at 0.5, 821 at 1, 841 at 2 -- the flatter RMAT gains 9% -- but at
// 1 single queries took 12% longer on RMAT s26 ef16 and 5% longer at s22, so it
// is off by default.
#ifndef TRAV_HOLD_SLACK
#define TRAV_HOLD_SLACK -1.0f
#endif
constexpr float kHoldSlack = TRAV_HOLD_SLACK;
// Bitmap words a warp works on at once in a bottom-up step.
#ifndef TRAV_BU_WORDS
#define TRAV_BU_WORDS 3
#endif
constexpr int kBuWords = TRAV_BU_WORDS;
// In-rows longer than this are scanned by the whole warp in a bottom-up step;
// shorter ones by their own lane, four parents per probe.
#ifndef TRAV_BU_COOP
#define TRAV_BU_COOP 512
#endif
constexpr int kBuCoop = TRAV_BU_COOP;
#ifndef TRAV_FLUSH_ATTR
#define TRAV_FLUSH_ATTR __forceinline__
#endif
// Independent edges per lane per round of a relaxation loop.  More edges in
// flight hide more latency but cost registers.  With the atomics deferred
// (SsspPush), SSSP's 64-register budget (4 CTAs per SM) holds 3 without
// spilling; at s23 a batch of 128 queries ran 8% faster with 3 than with 2,
// and 4 gained nothing more.  5 CTAs per SM (48 registers) spill and lose 50%.
constexpr int kBatchBfs = TRAV_KBATCH_BFS, kBatchSssp = TRAV_KBATCH_SSSP;
// Per-warp buffers: a push adds at most 32 entries to a buffer that held
// fewer than its flush mark, so mark + 32 entries always fit.
constexpr int kWQFlush = 128, kWQ = kWQFlush + 32;
constexpr int kWBigFlush = 64, kWBig = kWBigFlush + 32;
constexpr int kWFarFlush = 128, kWFar = kWFarFlush + 32;

constexpr int kPartWhole = 0, kPartLight = 1, kPartHeavy = 2, kPartIn = 3;  // kPartIn: the in-row (CSC)
// An SSSP heavy round considers pulling when its heavy list may hold more than
// 1/kPullCheck of the graph's edges.  The check is a pass over every vertex,
// which a query on a batch team of 1/8 of the grid pays eight times over:
// summed over four graphs (RMAT s23 ef32, s24 ef16, a flatter RMAT, uniform
// 2^23), 64-query SSSP batches took 854 ms at 3, 864 at 4 and 871 at 8, and
// single queries were also fastest at 3.
#ifndef TRAV_PULL_CHECK
#define TRAV_PULL_CHECK 3.0
#endif
constexpr double kPullCheck = TRAV_PULL_CHECK;

struct WarpStage {
    int q[2][kWQ];
    int big[2][kWBig];
    int far[kWFar];
    int tu[32], trb[32], tpre[32];  // the current warp tile
    float tdu[32];
};

// Deferred SSSP relaxations of one warp (see SsspPush): fewer than 32 kept
// between batches, plus up to 32 per edge of a lane's batch.
constexpr int kWDefer = 32 + 32 * kBatchSssp;
// Where a drain takes a candidate's row-class flags from: the gathered
// distance word, staged with the candidate (0), or the byte array, loaded in
// parallel with the atomic (1).  Same results either way.  Measured on the
// bench step (128 queries, RMAT s23): 143.0 ms staged, 148.6 ms from the byte.
#ifndef TRAV_CLS_BYTE
#define TRAV_CLS_BYTE 0
#endif
struct DeferStage {
    int v[kWDefer];
    float d[kWDefer];
#if !TRAV_CLS_BYTE
    unsigned cls[kWDefer];
#endif
};

struct CtaCounters {
    unsigned long long mf, scanned;
    unsigned big_total[2];
    int far_key;
    int light_key;  // SSSP: max of 0x7fffffff - bits(d) over the light frontier pushed (0 = none)
};

// Destination of one phase's pushes.
struct FrontierOut {
    int32_t *q[2];       // short-row queues of the two targets
    int2 *chunks[2];     // chunk items of the two targets
    unsigned qbase[2];   // entries already in each target before this phase
    unsigned cbase[2];
    int part[2];         // which part of a row each target expands
    int32_t *farp;       // far pile (SSSP)
    unsigned fbase;      // far entries already in the pile before this phase
    Slot *slot;
};

// Per-warp push state (counts are warp-uniform registers).
struct Pusher {
    const TravArgs *a;
    const FrontierOut *o;
    WarpStage *s;
    DeferStage *d;                   // the warp's deferred relaxations (SSSP expansions only)
    unsigned nq[2], nbig[2], nfar;
    unsigned ndef;                   // entries staged in d
    unsigned big_total[2];
    unsigned long long mf, scanned;  // lane-partial sums
    int far_key;                     // lane-partial max
    int light_key;                   // lane-partial max (SSSP light frontier; see CtaCounters)
};

// Row part [begin, end) of vertex v.
__device__ __forceinline__ int2 row_part(const TravArgs &a, int v, int part)
{
    if (part == kPartIn) return make_int2(__ldg(&a.in_off[v]), __ldg(&a.in_off[v + 1]));
    // light parts live in the light rows when the query has them (edge indices
    // then count into a.ledge, not into out_adj / out_w)
    if (part == kPartLight && a.loff) return make_int2(__ldg(&a.loff[v]), __ldg(&a.loff[v + 1]));
    int rb = __ldg(&a.out_off[v]), re = __ldg(&a.out_off[v + 1]);
    if (part == kPartLight) re = rb + __ldg(&a.nlight[v]);
    else if (part == kPartHeavy) rb += __ldg(&a.nlight[v]);
    return make_int2(rb, re);
}

__device__ __forceinline__ Pusher make_pusher(const TravArgs &a, const FrontierOut &o, WarpStage *s,
                                              DeferStage *d = nullptr)
{
    Pusher p;
    p.a = &a;
    p.o = &o;
    p.s = s;
    p.d = d;
    p.nq[0] = p.nq[1] = p.nbig[0] = p.nbig[1] = p.nfar = 0;
    p.ndef = 0;
    p.big_total[0] = p.big_total[1] = 0;
    p.mf = p.scanned = 0;
    p.far_key = 0;
    p.light_key = 0;
    return p;
}

__device__ TRAV_FLUSH_ATTR void flush_q(Pusher &p, int t)
{
    __syncwarp();
    unsigned base = 0;
    if (lane_id() == 0) base = p.o->qbase[t] + atomicAdd(t ? &p.o->slot->hq_add : &p.o->slot->q_add, p.nq[t]);
    base = __shfl_sync(kFull, base, 0);
    for (unsigned i = lane_id(); i < p.nq[t]; i += 32) p.o->q[t][base + i] = p.s->q[t][i];
    __syncwarp();
    p.nq[t] = 0;
}

__device__ TRAV_FLUSH_ATTR void flush_big(Pusher &p, int t)
{
    __syncwarp();
    for (unsigned r = 0; r < p.nbig[t]; r += 32) {
        const unsigned i = r + lane_id();
        int v = 0, nch = 0;
        int2 part = make_int2(0, 0);
        if (i < p.nbig[t]) {
            v = p.s->big[t][i];
            part = row_part(*p.a, v, p.o->part[t]);
            nch = (part.y - part.x + p.a->item - 1) / p.a->item;
        }
        int incl = nch;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, d);
            if ((int)lane_id() >= d) incl += y;
        }
        const unsigned total = (unsigned)__shfl_sync(kFull, incl, 31);
        unsigned base = 0;
        if (lane_id() == 0) base = p.o->cbase[t] + atomicAdd(t ? &p.o->slot->hchunk_add : &p.o->slot->chunk_add, total);
        base = __shfl_sync(kFull, base, 0) + (unsigned)(incl - nch);
        for (int c = 0; c < nch; c++) p.o->chunks[t][base + c] = make_int2(v, part.x + c * p.a->item);
    }
    __syncwarp();
    p.nbig[t] = 0;
}

__device__ TRAV_FLUSH_ATTR void flush_far(Pusher &p)
{
    __syncwarp();
    unsigned base = 0;
    if (lane_id() == 0) base = p.o->fbase + atomicAdd(&p.o->slot->far_add, p.nfar);
    base = __shfl_sync(kFull, base, 0);
    for (unsigned i = lane_id(); i < p.nfar; i += 32) p.o->farp[base + i] = p.s->far[i];
    __syncwarp();
    p.nfar = 0;
}

// Warp-collective: lanes with `flag` push vertex v to target t; `len` is the
// length of the row part the target will expand (tile queue or chunk items).
__device__ __forceinline__ void push(Pusher &p, int t, bool flag, int v, unsigned len)
{
    const bool big = flag && len > (unsigned)p.a->small_deg;
    const bool small = flag && !big;
    const unsigned ms = __ballot_sync(kFull, small), mb = __ballot_sync(kFull, big);
    if (ms) {
        if (small) p.s->q[t][p.nq[t] + __popc(ms & lanemask_lt())] = v;
        p.nq[t] += __popc(ms);
        if (p.nq[t] >= (unsigned)kWQFlush) flush_q(p, t);
    }
    if (mb) {
        if (big) p.s->big[t][p.nbig[t] + __popc(mb & lanemask_lt())] = v;
        p.nbig[t] += __popc(mb);
        p.big_total[t] += __popc(mb);
        if (p.nbig[t] >= (unsigned)kWBigFlush) flush_big(p, t);
    }
}

// Warp-collective: lanes with `flag` add v to the far pile; key = 0x7fffffff - distance bits.
__device__ __forceinline__ void push_far(Pusher &p, bool flag, int v, int key)
{
    const unsigned m = __ballot_sync(kFull, flag);
    if (!m) return;
    if (flag) {
        p.s->far[p.nfar + __popc(m & lanemask_lt())] = v;
        p.far_key = max(p.far_key, key);
    }
    p.nfar += __popc(m);
    if (p.nfar >= (unsigned)kWFarFlush) flush_far(p);
}

// End of a phase: every warp writes out what it staged, then the CTA reduces
// the counters and publishes them with one atomic each.  CTA-collective.
__device__ void finish_phase(Pusher &p, CtaCounters &cc)
{
    for (int t = 0; t < 2; t++) {
        if (p.nq[t]) flush_q(p, t);
        if (p.nbig[t]) flush_big(p, t);
    }
    if (p.nfar) flush_far(p);
    const unsigned long long mf = __reduce_add_sync(kFull, (unsigned)p.mf);  // per-lane parts fit 32 bits
    unsigned long long sc = p.scanned;
#pragma unroll
    for (int d = 16; d; d >>= 1) sc += __shfl_xor_sync(kFull, sc, d);
    const int fk = __reduce_max_sync(kFull, p.far_key);
    const int lk = kHoldSlack >= 0.0f ? __reduce_max_sync(kFull, p.light_key) : 0;
    if (lane_id() == 0) {
        if (mf) atomicAdd(&cc.mf, mf);
        if (sc) atomicAdd(&cc.scanned, sc);
        if (p.big_total[0]) atomicAdd(&cc.big_total[0], p.big_total[0]);
        if (p.big_total[1]) atomicAdd(&cc.big_total[1], p.big_total[1]);
        if (fk) atomicMax(&cc.far_key, fk);
        if (lk) atomicMax(&cc.light_key, lk);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Slot *sl = p.o->slot;
        if (cc.mf) atomicAdd(&sl->mf, cc.mf);
        if (cc.scanned) atomicAdd(&sl->scanned, cc.scanned);
        if (cc.big_total[0]) atomicAdd(&sl->big_add, cc.big_total[0]);
        if (cc.big_total[1]) atomicAdd(&sl->hbig_add, cc.big_total[1]);
        if (cc.far_key) atomicMax(&sl->min_far_bits, cc.far_key);
        // SSSP phases that push a light frontier leave mf (a sum only BFS and
        // the pull check use) free: it carries the frontier's lowest distance
        if (cc.light_key) atomicMax(&sl->mf, (unsigned long long)cc.light_key);
        cc.mf = cc.scanned = 0;
        cc.big_total[0] = cc.big_total[1] = 0;
        cc.far_key = 0;
        cc.light_key = 0;
    }
    // the next phase's pushes are staged only after the grid barrier, which
    // begins with __syncthreads, so the reset is seen before any reuse
}

// Expand a frontier (part kPart of each row) in one phase: chunk items one
// warp each, then the short-row queue in 32-vertex warp tiles (edge-balanced
// within the tile).  Every lane carries kBatch independent edges per round so
// their loads and atomics overlap.
template <int kPart, class Vis>
__device__ void expand_frontier(const TravArgs &a, const int32_t *q, unsigned nq, const int2 *chunks, unsigned nch,
                                const Vis &vis, Pusher &p)
{
    constexpr int kBatch = Vis::kBatch;
    const int lane = (int)lane_id();
    const unsigned gwarp = (unsigned)team_tid(a) >> 5, nwarps = (unsigned)team_threads(a) >> 5;
    for (unsigned c = gwarp; c < nch; c += nwarps) {
        const int2 it = chunks[c];
        const int u = it.x, start = it.y;
        const int2 rp = row_part(a, u, kPart);
        const int end = min(start + a.item, rp.y);
        const float du = vis.begin(u);
        if (kHoldSlack >= 0.0f && kPart == kPartLight && nq > 0 && vis.hold(du)) {
            // A long light row (a hub's) whose distance is well above the
            // frontier's lowest would likely be improved again, and rescanned
            // in full each time: while short rows are still being expanded it
            // waits, and the row's first item queues it for the next round.
            const bool carry = start == rp.x && lane == 0 && vis.stamp_carry(u);
            push(p, 0, carry, u, (unsigned)a.small_deg + 1u);
            if (carry) p.light_key = max(p.light_key, 0x7fffffff - __float_as_int(du));
            continue;
        }
        if (lane == 0) p.scanned += (unsigned long long)(end - start);
        for (int e0 = start; e0 < end; e0 += 32 * kBatch) {
            int us[kBatch], e[kBatch];
            float ds[kBatch];
            bool ok[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; j++) {
                e[j] = e0 + lane + 32 * j;
                ok[j] = e[j] < end;
                us[j] = u;
                ds[j] = du;
            }
            vis.template visit_batch<kPart>(us, ds, e, ok, p);
        }
    }
    WarpStage *s = p.s;
    for (unsigned t0 = gwarp * 32; t0 < nq; t0 += nwarps * 32) {
        const unsigned i = t0 + lane;
        int u = 0, rb = 0, deg = 0;
        if (i < nq) {
            u = q[i];
            const int2 pr = row_part(a, u, kPart);
            rb = pr.x;
            deg = pr.y - pr.x;
        }
        int incl = deg;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += y;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        s->tu[lane] = u;
        s->trb[lane] = rb;
        s->tpre[lane] = incl - deg;
        s->tdu[lane] = deg > 0 ? vis.begin(u) : 0.0f;
        __syncwarp();
        if (lane == 0) p.scanned += (unsigned long long)total;
        const int n = (int)min(32u, nq - t0);
        for (int base = 0; base < total; base += 32 * kBatch) {
            int us[kBatch], e[kBatch];
            float ds[kBatch];
            bool ok[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; j++) {
                const int k = base + lane + 32 * j;
                ok[j] = k < total;
                int lo = 0;
                if (ok[j]) {
                    int hi = n;
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (s->tpre[mid] <= k) lo = mid;
                        else hi = mid;
                    }
                }
                e[j] = s->trb[lo] + (k - s->tpre[lo]);
                us[j] = s->tu[lo];
                ds[j] = s->tdu[lo];
            }
            vis.template visit_batch<kPart>(us, ds, e, ok, p);
        }
        __syncwarp();
    }
    vis.finish(p);
}

// One vertex as a frontier of its own (row part [rb, re)): every CTA computes
// the counts; the items are written by the first threads of the grid.
__device__ __forceinline__ void seed_part(const TravArgs &a, int s, int rb, int re, int32_t *q, int2 *chunks,
                                          unsigned &nq, unsigned &nch)
{
    const int gtid = team_tid(a), nth = team_threads(a);
    const int len = re - rb;
    nq = nch = 0;
    if (len <= 0) return;
    if (len > a.small_deg) {
        nch = (unsigned)((len + a.item - 1) / a.item);
        for (int c = gtid; c < (int)nch; c += nth) chunks[c] = make_int2(s, rb + c * a.item);
    } else {
        nq = 1;
        if (gtid == 0) q[0] = s;
    }
}

// visit_batch() is called by all 32 lanes of a warp together; ok[j] marks
// the lanes' edges that exist.  begin() returns the per-vertex value used.
struct BfsPush {
    static constexpr int kBatch = kBatchBfs;
    const TravArgs *a;
    int level_next;

    __device__ __forceinline__ float begin(int) const { return 0.0f; }
    __device__ __forceinline__ bool hold(float) const { return false; }
    __device__ __forceinline__ bool stamp_carry(int) const { return false; }
    __device__ __forceinline__ void finish(Pusher &) const {}

    __device__ __forceinline__ void load_at(const int (&e)[kBatch], const bool (&ok)[kBatch], int (&v)[kBatch],
                                            float (&)[kBatch]) const
    {
#pragma unroll
        for (int j = 0; j < kBatch; j++) v[j] = ok[j] ? ld_stream(&a->out_adj[e[j]]) : 0;
    }

    template <int kPart>
    __device__ __forceinline__ void visit_batch(const int (&)[kBatch], const float (&du)[kBatch],
                                                const int (&e)[kBatch], const bool (&ok)[kBatch], Pusher &p) const
    {
        int v[kBatch];
        float w[kBatch];
        load_at(e, ok, v, w);
        visit_loaded(du, v, w, ok, p);
    }

    __device__ __forceinline__ void visit_loaded(const float (&)[kBatch], const int (&v)[kBatch],
                                                 const float (&)[kBatch], const bool (&ok)[kBatch], Pusher &p) const
    {
        unsigned word[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; j++) word[j] = ok[j] ? __ldcg(&a->visited[v[j] >> 5]) : ~0u;
        bool fresh[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; j++) {
            const unsigned bit = 1u << (v[j] & 31);
            fresh[j] = false;
            if (!(word[j] & bit)) fresh[j] = !(atomicOr(a->visited + (v[j] >> 5), bit) & bit);
        }
        unsigned deg[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; j++) {
            deg[j] = 0;
            if (fresh[j]) {
                reinterpret_cast<int *>(a->value)[v[j]] = level_next;
                deg[j] = (unsigned)(__ldg(&a->out_off[v[j] + 1]) - __ldg(&a->out_off[v[j]]));
            }
            p.mf += deg[j];
        }
#pragma unroll
        for (int j = 0; j < kBatch; j++) push(p, 0, fresh[j], v[j], deg[j]);
    }
};

// SSSP distance word: float bits in the high half, the round stamp in the low
// half.  Distances are >= +0, so the unsigned order of the words is the order
// of the distances (ties broken by the stamp).
__device__ __forceinline__ float dist_of(unsigned long long x) { return __uint_as_float((unsigned)(x >> 32)); }

__device__ __forceinline__ unsigned long long pack_dist(float d, unsigned low)
{
    return (static_cast<unsigned long long>(__float_as_uint(d)) << 32) | low;
}

// SSSP relaxation.  A distance is one 64-bit word: the float bits, then the
// id of the round that last lowered it:
//     dist_bits << 32 | round << 4.
// The atomicMin that lowers a distance writes the current round, and its
// return value tells the thread both whether it improved the vertex and when
// the vertex was last improved -- which, with the vertex's row-class byte, is
// all the push needs to decide, without another atomic, whether the vertex is
// already in the buffer it belongs to:
//   - next frontier (light prefix, this round only): already there when the
//     old word is from this round and below the bound;
//   - heavy list (since h_start): already there when the old word is from a
//     round >= h_start and below the bound;
//   - far pile (since f_start): already there when the old word is from a
//     round >= f_start and at or above the bound.
// Among the threads that lower one vertex in a round, exactly the first one
// sees an old word from an earlier round (distances only fall, so a vertex
// below the bound stays below it).
__device__ __forceinline__ unsigned row_class(const TravArgs &a, int v)
{
    const int deg = __ldg(&a.out_off[v + 1]) - __ldg(&a.out_off[v]);
    const int nl = a.nlight ? __ldg(&a.nlight[v]) : deg, nh = deg - nl;
    return (nl > 0 ? kClsLight : 0u) | (nl > a.small_deg ? kClsLightBig : 0u) | (nh > 0 ? kClsHeavy : 0u) |
           (nh > a.small_deg ? kClsHeavyBig : 0u);
}

// kPull = false relaxes out-rows (push): the row's owner is the source of
// every candidate.  kPull = true scans the in-rows of unsettled vertices
// (pull rounds): the row's owner is the target, and each in-edge u -> owner
// gives the candidate fl(d(u) + w).  Both feed the same deferred atomics and
// push decisions; a pull candidate is just a relaxation of the edge u -> owner.
template <bool kPull>
struct SsspVisit {
    static constexpr int kBatch = kBatchSssp;
    const TravArgs *a;
    float thr;               // bucket upper bound (exclusive)
    unsigned round;          // id of this round (>= 1)
    unsigned h_start;        // round the current heavy list began in
    unsigned f_start;        // round the current far pile began in
    float hold_above = INFINITY;  // light rounds: long rows above this distance wait (see expand_frontier)

    __device__ __forceinline__ float begin(int u) const { return dist_of(__ldcg(&a->dist[u])); }
    __device__ __forceinline__ bool hold(float du) const { return du > hold_above; }

    // Queue a held vertex for the next round without a new distance: stamp its
    // word with this round, keeping the distance and the flags, unless a
    // relaxation of this round already did (and pushed it).  Either way the
    // vertex enters the next frontier once.  A frontier vertex's stamp is from
    // the heavy list's span already, so the heavy-list test reads the same.
    __device__ __forceinline__ bool stamp_carry(int u) const
    {
        unsigned long long w = __ldcg(&a->dist[u]);
        while (((unsigned)w >> kClsBits) < round) {
            const unsigned long long nw =
                (w & ~0xffffffffull) | (unsigned long long)(round << kClsBits | ((unsigned)w & kClsMask));
            const unsigned long long old = atomicCAS(&a->dist[u], w, nw);
            if (old == w) return true;
            w = old;  // lowered (and stamped) meanwhile: look again
        }
        return false;
    }

    template <int kPart>
    __device__ __forceinline__ void load_at(const int (&e)[kBatch], const bool (&ok)[kBatch], int (&v)[kBatch],
                                            float (&w)[kBatch]) const
    {
        if (kPart == kPartLight && a->ledge) {
            // light rows: target and weight of an edge side by side
#pragma unroll
            for (int j = 0; j < kBatch; j++) {
                const int2 x = ok[j] ? ld_stream(&a->ledge[e[j]]) : make_int2(0, 0);
                v[j] = x.x;
                w[j] = __int_as_float(x.y);
            }
            return;
        }
#pragma unroll
        for (int j = 0; j < kBatch; j++) {
            v[j] = ok[j] ? ld_stream(&a->out_adj[e[j]]) : 0;
            w[j] = ok[j] ? ld_stream(&a->out_w[e[j]]) : 0.0f;
        }
    }

    template <int kPart>
    __device__ __forceinline__ void visit_batch(const int (&us)[kBatch], const float (&du)[kBatch],
                                                const int (&e)[kBatch], const bool (&ok)[kBatch], Pusher &p) const
    {
        int v[kBatch];
        float w[kBatch];
        if constexpr (kPull) {
            // in-neighbours and weights; the candidate's target is the row's owner us[j], whose distance is du[j]
#pragma unroll
            for (int j = 0; j < kBatch; j++) {
                v[j] = ok[j] ? ld_stream(&a->in_adj[e[j]]) : 0;
                w[j] = ok[j] ? ld_stream(&a->in_w[e[j]]) : 0.0f;
            }
            float nd[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; j++) nd[j] = ok[j] ? dist_of(ld_gather(&a->dist[v[j]])) : 0.0f;
            DeferStage *d = p.d;
#if TRAV_PULL_REDUCE
            // Lane k of batch j holds edge base + 32 j + k, so for each j the
            // lanes of one owner are contiguous.  A segmented min leaves an
            // owner's best candidate at its first lane, and only that lane
            // stages it: one atomic per owner and batch instead of one per
            // improving in-edge (the owner is unsettled, so most of its
            // in-edges improve on its distance at the round's start).  The
            // candidates are >= +0, so their bits order as unsigned integers.
            const unsigned lane = lane_id();
#pragma unroll
            for (int j = 0; j < kBatch; j++) {
                nd[j] = __fadd_rn(nd[j], w[j]);  // one rounded add, as sssp.hpp:56
                const int o = ok[j] ? us[j] : -1;
                const int prev = __shfl_up_sync(kFull, o, 1);
                const unsigned heads = __ballot_sync(kFull, lane == 0 || prev != o);
                const unsigned later = heads & ~((2u << lane) - 1u);  // heads above this lane (none for lane 31)
                const unsigned end = later ? (unsigned)__ffs(later) - 1u : 32u;  // first lane past this segment
                unsigned key = ok[j] && nd[j] < du[j] ? __float_as_uint(nd[j]) : 0xffffffffu;
#pragma unroll
                for (unsigned s = 1; s < 32; s <<= 1) {
                    const unsigned y = __shfl_down_sync(kFull, key, s);
                    if (lane + s < end) key = min(key, y);
                }
                const bool cand = (heads >> lane & 1u) && key != 0xffffffffu;
                const unsigned m = __ballot_sync(kFull, cand);
                if (cand) {
                    const unsigned i = p.ndef + __popc(m & lanemask_lt());
                    d->v[i] = us[j];
                    d->d[i] = __uint_as_float(key);
                }
                p.ndef += __popc(m);
            }
#else
#pragma unroll
            for (int j = 0; j < kBatch; j++) {
                nd[j] = __fadd_rn(nd[j], w[j]);  // one rounded add, as sssp.hpp:56
                const bool cand = ok[j] && nd[j] < du[j];
                const unsigned m = __ballot_sync(kFull, cand);
                if (cand) {
                    const unsigned i = p.ndef + __popc(m & lanemask_lt());
                    d->v[i] = us[j];
                    d->d[i] = nd[j];
                }
                p.ndef += __popc(m);
            }
#endif
            while (p.ndef >= 32) drain(p, 32);
        } else {
            load_at<kPart>(e, ok, v, w);
            visit_loaded(du, v, w, ok, p);
        }
    }

    // An edge whose candidate beats the gathered distance is not relaxed at
    // once: (v, candidate, row class) goes to the warp's DeferStage, and the
    // atomicMins run 32 at a time (drain).  A batch then waits on its edge
    // loads and its gathers only; the wait for an atomic's return -- which
    // every batch used to pay, since almost every batch of 32 * kBatch edges
    // has an improving lane -- comes once per 32 candidates.  The candidates
    // are relaxed within the same phase, and the push decision reads only the
    // atomic's return value, so the order of the atomics changes nothing.
    __device__ __forceinline__ void visit_loaded(const float (&du)[kBatch], const int (&v)[kBatch],
                                                 const float (&w)[kBatch], const bool (&ok)[kBatch], Pusher &p) const
    {
        float nd[kBatch];
        unsigned long long cur[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; j++) nd[j] = ok[j] ? __fadd_rn(du[j], w[j]) : 0.0f;  // one rounded add, as sssp.hpp:56
#pragma unroll
        for (int j = 0; j < kBatch; j++) cur[j] = ok[j] ? ld_gather(&a->dist[v[j]]) : 0ull;
        DeferStage *d = p.d;
#pragma unroll
        for (int j = 0; j < kBatch; j++) {
            const bool cand = ok[j] && nd[j] < dist_of(cur[j]);
            const unsigned m = __ballot_sync(kFull, cand);
            if (cand) {
                const unsigned i = p.ndef + __popc(m & lanemask_lt());
                d->v[i] = v[j];
                d->d[i] = nd[j];
#if !TRAV_CLS_BYTE
                d->cls[i] = (unsigned)cur[j] & kClsMask;
#endif
            }
            p.ndef += __popc(m);
        }
        while (p.ndef >= 32) drain(p, 32);
    }

    // End of the warp's expansion: relax what is still staged.
    __device__ __forceinline__ void finish(Pusher &p) const
    {
        if (p.ndef) drain(p, p.ndef);
    }

    // Relax the last n (<= 32) staged candidates, one per lane, and push the
    // vertices they improved.  Warp-collective.
    __device__ __forceinline__ void drain(Pusher &p, unsigned n) const
    {
        __syncwarp();
        const DeferStage *d = p.d;
        const unsigned base = p.ndef - n, lane = lane_id();
        const bool ok = lane < n;
        int v = 0;
        float nd = 0.0f;
        unsigned cls = 0;
        if (ok) {
            v = d->v[base + lane];
            nd = d->d[base + lane];
#if !TRAV_CLS_BYTE
            if constexpr (!kPull) cls = d->cls[base + lane];
#endif
        }
        __syncwarp();  // the entries are read before later batches overwrite them
        if (kPull || TRAV_CLS_BYTE) {
            // the flags' byte copy (a pull stages no gathered word of the vertex
            // it improves): written at this query's initialisation, by other
            // CTAs and per query in a team, so read at L2 rather than through
            // the read-only path
            if (ok) cls = __ldcg(&a->rcls[v]);
        }
        p.ndef = base;
        bool light = false, heavy = false, far = false;
        if (ok) {
            const unsigned long long old = atomicMin(&a->dist[v], pack_dist(nd, round << kClsBits | cls));
            const float od = dist_of(old);
            if (nd < od) {
                const unsigned orr = (unsigned)old >> kClsBits;
                if (nd < thr) {
                    const bool seen_below = od < thr;
                    light = (cls & kClsLight) && !(seen_below && orr >= round);
                    heavy = (cls & kClsHeavy) && !(seen_below && orr >= h_start);
                } else {
                    far = !(orr >= f_start);  // od > nd >= thr
                }
            }
        }
        const unsigned big_len = (unsigned)a->small_deg + 1u;  // any length that classifies as a long row
        push(p, 0, light, v, cls & kClsLightBig ? big_len : 1u);
        push(p, 1, heavy, v, cls & kClsHeavyBig ? big_len : 1u);
        push_far(p, far, v, far ? 0x7fffffff - __float_as_int(nd) : 0);
        if (kHoldSlack >= 0.0f && light) p.light_key = max(p.light_key, 0x7fffffff - __float_as_int(nd));
    }
};

using SsspPush = SsspVisit<false>;
using SsspPull = SsspVisit<true>;

__device__ __forceinline__ void init_counters(CtaCounters &cc)
{
    if (threadIdx.x == 0) {
        cc.mf = cc.scanned = 0;
        cc.big_total[0] = cc.big_total[1] = 0;
        cc.far_key = 0;
        cc.light_key = 0;
    }
    __syncthreads();
}

// --------------------------------------------------------------- BFS kernel
// Shared memory of one query's CTA (the bodies below run inside the
// single-query kernels and inside the batch kernel).
struct QueryShared {
    float mlp[kMlpMaxParams];  // the schedule network, copied in when the query has one
    WarpStage wst[kWarps];
    CtaCounters cc;
    SlotView view;
    int dir;
    float bound;
};

// Copy the query's schedule network into shared memory (read there by warp 0
// at every decision); the first grid barrier orders it before any use.
__device__ __forceinline__ void load_mlp(const TravArgs &a, QueryShared &sh, int count)
{
    if (!a.mlp) return;
    for (int i = threadIdx.x; i < count; i += kBlock) sh.mlp[i] = __ldg(&a.mlp[i]);
}

// One query on the CTAs [a.cta0, a.cta0 + a.ctas), starting at phase ph0 of the
// counter-slot ring.  Returns the next phase index, or -1 when the query failed
// (the error is in a.ctl->err).
__device__ __forceinline__ int bfs_query(const TravArgs &a, QueryShared &sh, int ph0)
{
    SlotView &s_view = sh.view;
    PhaseLog lg;
    lg.leader = (int)blockIdx.x == a.cta0 && threadIdx.x == 0;
    WarpStage *wst = sh.wst;
    CtaCounters &cc = sh.cc;
    int &s_dir = sh.dir;
    Ctl *ctl = a.ctl;
    const int gtid = team_tid(a), nth = team_threads(a);
    const unsigned gwarp = gtid >> 5, nwarps = nth >> 5;
    WarpStage *mys = &wst[threadIdx.x >> 5];
    const int s = a.source;
    int ph = ph0;

    load_mlp(a, sh, mlp_param_count(kBfsOut));
    init_counters(cc);
    for (int v = gtid; v < a.V; v += nth) reinterpret_cast<int *>(a.value)[v] = v == s ? 0 : -1;
    if (!a.color) {
        for (int w = gtid; w < a.W; w += nth) a.visited[w] = w == (s >> 5) ? 1u << (s & 31) : 0u;
    } else {
        // vertex mask: vertices of another color start out visited, so no
        // step (top-down or bottom-up) ever reaches them; their levels stay -1
        for (unsigned w = gwarp; w < (unsigned)a.W; w += nwarps) {
            const int v = (int)(w * 32 + lane_id());
            const bool pre = v < a.V && (v == s || __ldg(&a.color[v]) != a.color_want);
            const unsigned m = __ballot_sync(kFull, pre);
            if (lane_id() == 0) a.visited[w] = m;
        }
    }
    unsigned nq, nch;
    seed_part(a, s, __ldg(&a.out_off[s]), __ldg(&a.out_off[s + 1]), a.q0, a.chunks0, nq, nch);
    clear_ahead(a, ph);
    if (!grid_sync(a, ph)) return -1;
    ph++;
    if (gtid == 0) ctl->t0_ns = globaltimer();

    const unsigned long long deg_s = (unsigned long long)(__ldg(&a.out_off[s + 1]) - __ldg(&a.out_off[s]));
    unsigned long long nf = 1, nf_prev = 0, mf = deg_s, mu = (unsigned long long)a.E - deg_s;
    int dir = 0, prev_dir = 0, L = 0, cur = 0, fcur = 0, bu_steps = 0;
    while (nf > 0) {
        if (L >= a.max_steps) {
            if (gtid == 0) atomicCAS(&ctl->err, 0, kErrBudget);
            return -1;
        }
        // direction for this step (same inputs in every CTA -> same answer)
        if (threadIdx.x < 32) {
            int plain = dir;  // Beamer's switch
            if (dir == 0) {
                if ((double)mf > (double)mu / a.alpha) plain = 1;
            } else if (!(nf >= nf_prev || (double)nf > (double)a.V / a.beta)) {
                plain = 0;
            }
            const Feat f = bfs_features(L, nf, mf, mu, nf_prev, a.V, a.E, prev_dir, plain);
            // The network is consulted only near Beamer's switching points
            // (within kBfsGate of either threshold): far from them its answer is
            // Beamer's, and on long chains of tiny steps (a grid has thousands)
            // the inference itself would cost more than any choice can save.
            const bool near = dir == 0 ? (double)mf * a.alpha * kBfsGate > (double)mu
                                       : (double)nf * a.beta < (double)a.V * kBfsGate;
            int d = plain;
            if (a.force_dir >= 0) d = (L == 0) ? 0 : a.force_dir;
            else if (a.mlp && near) d = mlp_argmax_warp<kBfsOut>(sh.mlp, f, plain, a.mlp_margin);
            const int forced = planned(a, L);
            if (forced >= 0) d = forced;
            log_decision(ctl, lg, f, d, 0.0f, 0.0f);
            if (threadIdx.x == 0) s_dir = d;
        }
        __syncthreads();
        dir = s_dir;
        if (gtid == 0 && L < kMaxTrace) {
            ctl->dirs[L] = (unsigned char)dir;
            ctl->frontier[L] = (unsigned)nf;
        }
        if (dir == 1 && prev_dir == 0) {
            // frontier bitmap from the levels: bit v = (level[v] == L)
            clear_ahead(a, ph);
            for (unsigned w = gwarp; w < (unsigned)a.W; w += nwarps) {
                const int v = (int)(w * 32 + lane_id());
                const bool f = v < a.V && (int)a.value[v] == L;
                const unsigned m = __ballot_sync(kFull, f);
                if (lane_id() == 0) (fcur ? a.front1 : a.front0)[w] = m;
            }
            if (!grid_sync(a, ph)) return -1;
            log_phase(ctl, lg, 2, (unsigned)nf);
            ph++;
        }
#if TRAV_BU_LAZY
        if (dir == 0 && prev_dir == 1) {
            // frontier queue from the bitmap of the vertices the last
            // bottom-up step found (bottom-up steps push nothing)
            clear_ahead(a, ph);
            const FrontierOut qo{{(cur ? a.q1 : a.q0), nullptr}, {(cur ? a.chunks1 : a.chunks0), nullptr}, {0u, 0u},
                                 {0u, 0u}, {kPartWhole, kPartWhole}, nullptr, 0u, &ctl->slot[ph % kSlots]};
            Pusher pq = make_pusher(a, qo, mys);
            const unsigned *fc = fcur ? a.front1 : a.front0;
            for (unsigned w = gwarp; w < (unsigned)a.W; w += nwarps) {
                const int v = (int)(w * 32 + lane_id());
                const bool f = v < a.V && ((fc[w] >> lane_id()) & 1u);
                const unsigned deg = f ? (unsigned)(__ldg(&a.out_off[v + 1]) - __ldg(&a.out_off[v])) : 0u;
                push(pq, 0, f, v, deg);
            }
            finish_phase(pq, cc);
            if (!grid_sync(a, ph, &s_view)) return -1;
            log_phase(ctl, lg, 2, (unsigned)nf);
            nq = s_view.q_add;
            nch = s_view.chunk_add;
            ph++;
        }
#endif
        clear_ahead(a, ph);
        const FrontierOut out{{(cur ? a.q0 : a.q1), nullptr}, {(cur ? a.chunks0 : a.chunks1), nullptr}, {0u, 0u},
                              {0u, 0u}, {kPartWhole, kPartWhole}, nullptr, 0u, &ctl->slot[ph % kSlots]};
        Pusher p = make_pusher(a, out, mys);
        if (dir == 0) {
            const BfsPush vis{&a, L + 1};
            expand_frontier<kPartWhole>(a, (cur ? a.q1 : a.q0), nq, (cur ? a.chunks1 : a.chunks0), nch, vis, p);
        } else {
            // bottom-up: each warp owns 32 vertices = one bitmap word, and works
            // on kBuWords words at once (w, w + nwarps, ...) so that the
            // dependent loads of one word (visited -> in_off -> in_adj ->
            // frontier bit) overlap those of the others
            const unsigned *fc = fcur ? a.front1 : a.front0;
            unsigned *fn = fcur ? a.front0 : a.front1;
            constexpr int kW = kBuWords;
            const int lane = (int)lane_id();
            for (unsigned w0 = gwarp; w0 < (unsigned)a.W; w0 += kW * nwarps) {
                // The frontier bitmap and these words of `visited` were written
                // in earlier phases and only this warp writes them now: plain
                // (L1-cacheable) loads are coherent after the grid barrier.
                unsigned wd[kW], vis[kW];
                bool live[kW], cand[kW], found[kW];
                int v[kW], k[kW], kend[kW];
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    wd[i] = w0 + (unsigned)i * nwarps;
                    live[i] = wd[i] < (unsigned)a.W;
                    vis[i] = live[i] ? a.visited[wd[i]] : ~0u;
                    v[i] = (int)(wd[i] * 32 + lane);
                }
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    cand[i] = live[i] && v[i] < a.V && !((vis[i] >> lane) & 1u);
                    found[i] = false;
                    k[i] = kend[i] = 0;
                    if (cand[i]) {
                        k[i] = __ldg(&a.in_off[v[i]]);
                        kend[i] = __ldg(&a.in_off[v[i] + 1]);
                    }
                }
                // long in-rows: the whole warp scans one row 32 entries at a time
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    unsigned coop = __ballot_sync(kFull, cand[i] && kend[i] - k[i] > kBuCoop);
                    while (coop) {
                        const int owner = __ffs(coop) - 1;
                        coop &= coop - 1;
                        const int kb = __shfl_sync(kFull, k[i], owner), ke = __shfl_sync(kFull, kend[i], owner);
                        bool hit = false;
                        for (int kk = kb + lane; kk - lane < ke; kk += 32) {
                            bool h = false;
                            if (kk < ke) {
                                const int u = ld_stream(&a.in_adj[kk]);
                                h = (fc[u >> 5] >> (u & 31)) & 1u;
                            }
                            if (__any_sync(kFull, h)) {
                                hit = true;
                                break;
                            }
                        }
                        if (lane == owner) {
                            found[i] = hit;
                            cand[i] = false;
                        }
                    }
                }
                // short in-rows: one lane each, four parents per row and probe
                // (the probes of the lane's kW rows are independent loads)
                for (;;) {
                    bool act[kW], any = false;
#pragma unroll
                    for (int i = 0; i < kW; i++) {
                        act[i] = cand[i] && !found[i] && k[i] < kend[i];
                        any |= act[i];
                    }
                    if (!any) break;
                    int u[kW][4];
#pragma unroll
                    for (int i = 0; i < kW; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) u[i][j] = act[i] && k[i] + j < kend[i] ? ld_stream(&a.in_adj[k[i] + j]) : -1;
#pragma unroll
                    for (int i = 0; i < kW; i++) {
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            if (u[i][j] >= 0 && ((fc[u[i][j] >> 5] >> (u[i][j] & 31)) & 1u)) found[i] = true;
                        k[i] += 4;
                    }
                }
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    const unsigned m = __ballot_sync(kFull, found[i]);
                    if (lane == 0 && live[i]) {
                        fn[wd[i]] = m;
                        if (m) a.visited[wd[i]] = vis[i] | m;
                    }
                    unsigned deg = 0;
                    if (found[i]) {
                        reinterpret_cast<int *>(a.value)[v[i]] = L + 1;
                        deg = (unsigned)(__ldg(&a.out_off[v[i] + 1]) - __ldg(&a.out_off[v[i]]));
                    }
                    p.mf += deg;
#if TRAV_BU_LAZY
                    // the found vertices are counted (in the slot's hbig_add,
                    // which BFS leaves unused) and queued only if a top-down
                    // step follows
                    p.big_total[1] += __popc(m);
#else
                    push(p, 0, found[i], v[i], deg);
#endif
                }
            }
            fcur ^= 1;
            bu_steps++;
        }
        finish_phase(p, cc);
        if (!grid_sync(a, ph, &s_view)) return -1;
        lg.scanned += s_view.scanned;
        log_phase(ctl, lg, dir, (unsigned)nf);
        const SlotView s0 = s_view;
        ph++;
        nq = s0.q_add;
        nch = s0.chunk_add;
        mu -= s0.mf;
        nf_prev = nf;
        nf = TRAV_BU_LAZY && dir == 1 ? (unsigned long long)s0.hbig_add
                                      : (unsigned long long)s0.q_add + s0.big_add;
        mf = s0.mf;
        prev_dir = dir;
        L++;
        cur ^= 1;
    }
    if (gtid == 0) {
        ctl->steps = L;
        ctl->bottom_up_steps = bu_steps;
        ctl->buckets = 0;
    }
    write_back(a);
    return ph;
}

__global__ void __launch_bounds__(kBlock, TRAV_BFS_MIN_BLOCKS) bfs_persistent(TravArgs a)
{
    __shared__ QueryShared sh;
    bfs_query(a, sh, 0);
}

// -------------------------------------------------------------- SSSP kernel
// Delta-stepping with light and heavy edges over a near/far split.  Inside a
// bucket [lo, thr), relaxation rounds expand only the light prefixes (w <
// delta) of the frontier; improvements below thr feed the next round,
// improvements at or above it go to the far pile.  Every vertex improved below
// thr is also put (once per round of the heavy list) on the heavy list, whose
// heavy suffixes are relaxed once the light rounds drain -- so a vertex whose
// distance is corrected several times inside the bucket re-scans only its light
// edges.  With width = delta a heavy edge always lands at or above thr; with a
// wider bucket (the learned schedule) it may land below, and then its target
// starts new light rounds and joins the next heavy list.  When the frontier
// and the heavy list are empty the bound advances and the far pile is split.
// delta = +inf is Bellman-Ford over active vertices (every edge light).  Any
// order of relaxations reaches the same fixpoint bits: fl(x + w) is monotone
// in x and not below x for w >= 0.
//
// Pushes are deduplicated by the round stamps of the distance words (see
// SsspPush): round ids are phase indices, so the initial words (round 0) are
// older than every buffer.  A bucket opening pushes from the far pile without
// lowering a distance, so it stamps each vertex it pushes with its own round
// (an atomicMax that keeps the distance: nothing lowers distances in that
// phase).
__device__ __forceinline__ int sssp_query(const TravArgs &a, QueryShared &sh, DeferStage *defer, int ph0)
{
    SlotView &s_view = sh.view;
    PhaseLog lg;
    lg.leader = (int)blockIdx.x == a.cta0 && threadIdx.x == 0;
    WarpStage *wst = sh.wst;
    CtaCounters &cc = sh.cc;
    float &s_delta = sh.bound;
    Ctl *ctl = a.ctl;
    const int gtid = team_tid(a), nth = team_threads(a);
    const unsigned gwarp = gtid >> 5, nwarps = nth >> 5;
    WarpStage *mys = &wst[threadIdx.x >> 5];
    DeferStage *myd = &defer[threadIdx.x >> 5];
    const int lpart = a.nlight ? kPartLight : kPartWhole;
    const unsigned big_len = (unsigned)a.small_deg + 1u;  // any length that classifies as a long row
    int ph = ph0;
    load_mlp(a, sh, mlp_param_count(kSsspOut));
    init_counters(cc);
    unsigned nq, nch, nbig;                 // current frontier (light parts)
    unsigned hq = 0, hch = 0, hbig = 0;     // heavy list of the current round
    unsigned long long far_len = 0;
    int min_far = (int)kFltMaxBits;
    float thr = a.delta > 0.0f ? a.delta : INFINITY;
    float lo = 0.0f;                        // lower bound of the current bucket
    int cur = 0, hcur = 0, fcur = 0;

    unsigned h_start = 1, f_start = 1;      // rounds the heavy list / far pile began in
    if (a.source >= 0) {
        const int s = a.source;
        for (int v = gtid; v < a.V; v += nth) {
            const unsigned cls = row_class(a, v);
            a.rcls[v] = (unsigned char)cls;
            a.dist[v] = pack_dist(v == s ? 0.0f : FLT_MAX, cls);
        }
        const int2 lp = row_part(a, s, lpart);
        seed_part(a, s, lp.x, lp.y, a.q0, a.chunks0, nq, nch);
        nbig = nch ? 1u : 0u;
        if (a.nlight) {
            const int2 hp = row_part(a, s, kPartHeavy);
            seed_part(a, s, hp.x, hp.y, a.hq0, a.hch0, hq, hch);
            hbig = hch ? 1u : 0u;
        }
        clear_ahead(a, ph);
        if (!grid_sync(a, ph)) return -1;
        ph++;
        if (gtid == 0) ctl->t0_ns = globaltimer();
    } else {
        // start from the distance bits in init_bits (Bellman-Ford entry point,
        // every edge light): every vertex below FLT_MAX is active.
        thr = INFINITY;
        clear_ahead(a, ph);
        const FrontierOut out{{a.q0, nullptr}, {a.chunks0, nullptr}, {0u, 0u}, {0u, 0u}, {kPartWhole, kPartWhole},
                              nullptr, 0u, &ctl->slot[ph % kSlots]};
        Pusher p = make_pusher(a, out, mys);
        for (unsigned base = gwarp * 32; base < (unsigned)a.V; base += nwarps * 32) {
            const int v = (int)(base + lane_id());
            unsigned bits = kFltMaxBits, cls = 0;
            if (v < a.V) {
                bits = __ldg(&a.init_bits[v]);
                cls = row_class(a, v);
                a.rcls[v] = (unsigned char)cls;
                a.dist[v] = (static_cast<unsigned long long>(bits) << 32) | cls;
            }
            const bool act = bits < kFltMaxBits && (cls & kClsLight);
            push(p, 0, act, v, cls & kClsLightBig ? big_len : 1u);
        }
        finish_phase(p, cc);
        if (!grid_sync(a, ph, &s_view)) return -1;
        lg.scanned += s_view.scanned;
        const SlotView s0 = s_view;
        nq = s0.q_add;
        nch = s0.chunk_add;
        nbig = s0.big_add;
        ph++;
        if (gtid == 0) ctl->t0_ns = globaltimer();
    }

    int steps = 0, buckets = 1;
    // Light rounds hold back long light rows whose distance is more than
    // kHoldSlack x delta above the lowest distance of the round's frontier (a
    // vertex at or below that lowest distance is final: every later candidate
    // comes from a frontier vertex plus a weight >= 0).
    float hold_above = INFINITY;
    auto next_hold = [&](const SlotView &v) {
        return kHoldSlack >= 0.0f && v.mf ? __int_as_float(0x7fffffff - (int)v.mf) + kHoldSlack * a.delta : INFINITY;
    };
    while (true) {
        if (steps + buckets >= a.max_steps) {
            if (gtid == 0) atomicCAS(&ctl->err, 0, kErrBudget);
            return -1;
        }
        if (nq + nch > 0) {
            // light round: frontier (cur) -> next frontier (cur^1) + heavy list (hcur, appended)
            clear_ahead(a, ph);
            const FrontierOut out{{(cur ? a.q0 : a.q1), (hcur ? a.hq1 : a.hq0)},
                                  {(cur ? a.chunks0 : a.chunks1), (hcur ? a.hch1 : a.hch0)},
                                  {0u, hq},
                                  {0u, hch},
                                  {lpart, kPartHeavy},
                                  (fcur ? a.far1 : a.far0),
                                  (unsigned)far_len,
                                  &ctl->slot[ph % kSlots]};
            Pusher p = make_pusher(a, out, mys, myd);
            const SsspPush vis{&a, thr, (unsigned)ph, h_start, f_start, hold_above};
            if (lpart == kPartLight)
                expand_frontier<kPartLight>(a, (cur ? a.q1 : a.q0), nq, (cur ? a.chunks1 : a.chunks0), nch, vis, p);
            else
                expand_frontier<kPartWhole>(a, (cur ? a.q1 : a.q0), nq, (cur ? a.chunks1 : a.chunks0), nch, vis, p);
            finish_phase(p, cc);
            if (!grid_sync(a, ph, &s_view)) return -1;
            lg.scanned += s_view.scanned;
            log_phase(ctl, lg, 3, nq + nbig);
            const SlotView s0 = s_view;
            hold_above = next_hold(s0);
            ph++;
            if (gtid == 0 && steps < kMaxTrace) ctl->frontier[steps] = nq + nbig;
            nq = s0.q_add;
            nch = s0.chunk_add;
            nbig = s0.big_add;
            hq += s0.hq_add;
            hch += s0.hchunk_add;
            hbig += s0.hbig_add;
            far_len += s0.far_add;
            min_far = min(min_far, s0.min_far_bits);
            cur ^= 1;
            steps++;
        } else if (hq + hch > 0) {
            // heavy round: heavy list (hcur) -> frontier (cur, empty) + next heavy list (hcur^1).
            // Direction: when the heavy list's heavy parts may hold more than 1/kPullCheck of the edges, a check
            // phase first lists the vertices that a heavy edge could still improve, in the idle frontier buffer,
            // and counts their in-edges.  If they are fewer than half the heavy edges, the round pulls: it scans
            // those in-rows, and every in-edge u -> v relaxes v from u's distance, instead of pushing the heavy
            // list's out-rows.  The heavy list lies at or above the bucket's lower bound lo and a heavy edge
            // weighs at least delta, so a heavy candidate is at least fl(lo + delta): a vertex at or below that
            // cannot improve, and every other vertex is in the list.
            bool pull = false;
            unsigned pq = 0, pch = 0;
            const double heavy_est = (double)hch * a.item + (double)hq * (0.5 * a.small_deg + 1.0);
            if (a.in_w && heavy_est * kPullCheck > (double)a.E) {
                const float reach = __fadd_rn(lo, a.delta);
                clear_ahead(a, ph);
                const FrontierOut lout{{(cur ? a.q0 : a.q1), nullptr}, {(cur ? a.chunks0 : a.chunks1), nullptr},
                                       {0u, 0u}, {0u, 0u}, {kPartIn, kPartIn}, nullptr, 0u, &ctl->slot[ph % kSlots]};
                Pusher lp = make_pusher(a, lout, mys);
                for (unsigned base = gwarp * 32; base < (unsigned)a.V; base += nwarps * 32) {
                    const int v = (int)(base + lane_id());
                    unsigned len = 0;
                    if (v < a.V && dist_of(__ldcg(&a.dist[v])) > reach)
                        len = (unsigned)(__ldg(&a.in_off[v + 1]) - __ldg(&a.in_off[v]));
                    lp.mf += len;  // a lane's share stays below E < 2^31
                    push(lp, 0, len > 0, v, len);
                }
                finish_phase(lp, cc);
                if (!grid_sync(a, ph, &s_view)) return -1;
                log_phase(ctl, lg, 6, s_view.q_add + s_view.big_add);
                pq = s_view.q_add;
                pch = s_view.chunk_add;
                pull = 2.0 * (double)s_view.mf < heavy_est;
                ph++;
                steps++;
            }
            clear_ahead(a, ph);
            const FrontierOut out{{(cur ? a.q1 : a.q0), (hcur ? a.hq0 : a.hq1)},
                                  {(cur ? a.chunks1 : a.chunks0), (hcur ? a.hch0 : a.hch1)},
                                  {0u, 0u},
                                  {0u, 0u},
                                  {lpart, kPartHeavy},
                                  (fcur ? a.far1 : a.far0),
                                  (unsigned)far_len,
                                  &ctl->slot[ph % kSlots]};
            Pusher p = make_pusher(a, out, mys, myd);
            h_start = (unsigned)ph;  // the next heavy list begins in this round
            if (pull) {
                const SsspPull vis{&a, thr, (unsigned)ph, h_start, f_start};
                expand_frontier<kPartIn>(a, (cur ? a.q0 : a.q1), pq, (cur ? a.chunks0 : a.chunks1), pch, vis, p);
            } else {
                const SsspPush vis{&a, thr, (unsigned)ph, h_start, f_start};
                expand_frontier<kPartHeavy>(a, (hcur ? a.hq1 : a.hq0), hq, (hcur ? a.hch1 : a.hch0), hch, vis, p);
            }
            finish_phase(p, cc);
            if (!grid_sync(a, ph, &s_view)) return -1;
            lg.scanned += s_view.scanned;
            log_phase(ctl, lg, pull ? 7 : 5, hq + hbig);
            const SlotView s0 = s_view;
            hold_above = next_hold(s0);
            ph++;
            nq = s0.q_add;
            nch = s0.chunk_add;
            nbig = s0.big_add;
            hq = s0.hq_add;
            hch = s0.hchunk_add;
            hbig = s0.hbig_add;
            far_len += s0.far_add;
            min_far = min(min_far, s0.min_far_bits);
            hcur ^= 1;
            steps++;
        } else if (far_len > 0) {
            // open the next bucket (skipping empty ones): bound = max(old, min far) + width
            if (threadIdx.x < 32) {
                const Feat f = sssp_features(steps, far_len, __int_as_float(min_far), thr, a.delta, a.V, a.E, buckets, a.mean_w,
                                             a.max_deg);
                int o = 0;
                if (a.mlp) o = mlp_argmax_warp<kSsspOut>(sh.mlp, f, 0, a.mlp_margin);
                const int forced = planned(a, buckets - 1);
                if (forced >= 0) o = forced;
                const float width = a.delta * sssp_width_scale(o);
                float hi = __fadd_rn(fmaxf(thr, __int_as_float(min_far)), width);
                if (!(hi > thr)) hi = nextafterf(thr, INFINITY);
                log_decision(ctl, lg, f, o, thr, hi);
                if (threadIdx.x == 0) s_delta = hi;
            }
            __syncthreads();
            const float told = thr;
            thr = s_delta;  // the new bound, computed once above (same inputs in every CTA)
            lo = fmaxf(told, __int_as_float(min_far));
            const int32_t *fp = fcur ? a.far1 : a.far0;
            clear_ahead(a, ph);
            // the (empty) frontier and heavy list receive the entries of the new bucket
            const FrontierOut out{{(cur ? a.q1 : a.q0), (hcur ? a.hq1 : a.hq0)},
                                  {(cur ? a.chunks1 : a.chunks0), (hcur ? a.hch1 : a.hch0)},
                                  {0u, 0u},
                                  {0u, 0u},
                                  {lpart, kPartHeavy},
                                  (fcur ? a.far0 : a.far1),
                                  0u,
                                  &ctl->slot[ph % kSlots]};
            Pusher p = make_pusher(a, out, mys);
            const unsigned round = (unsigned)ph;
            h_start = f_start = round;  // the heavy list and the far pile begin again here
            for (unsigned long long base = (unsigned long long)gwarp * 32; base < far_len;
                 base += (unsigned long long)nwarps * 32) {
                const unsigned long long i = base + lane_id();
                const bool valid = i < far_len;
                const int v = valid ? fp[i] : 0;
                const unsigned long long dv = valid ? __ldcg(&a.dist[v]) : 0ull;
                const unsigned cls = (unsigned)dv & kClsMask;
                const float d = dist_of(dv);
                const bool in_bucket = valid && d >= told && d < thr;
                // the pile holds each vertex once (see SsspPush), so every entry is pushed on
                const bool light = in_bucket && (cls & kClsLight);
                const bool heavy = in_bucket && (cls & kClsHeavy);
                const bool keep = valid && d >= thr;
                if (in_bucket || keep) atomicMax(&a.dist[v], pack_dist(d, round << kClsBits | cls));
                push(p, 0, light, v, cls & kClsLightBig ? big_len : 1u);
                push(p, 1, heavy, v, cls & kClsHeavyBig ? big_len : 1u);
                push_far(p, keep, v, keep ? 0x7fffffff - __float_as_int(d) : 0);
            }
            finish_phase(p, cc);
            if (!grid_sync(a, ph, &s_view)) return -1;
            lg.scanned += s_view.scanned;
            log_phase(ctl, lg, 4, (unsigned)far_len);
            const SlotView s0 = s_view;
            hold_above = INFINITY;  // a bucket's first round expands everything it opened with
            ph++;
            nq = s0.q_add;
            nch = s0.chunk_add;
            nbig = s0.big_add;
            hq = s0.hq_add;
            hch = s0.hchunk_add;
            hbig = s0.hbig_add;
            far_len = s0.far_add;
            min_far = s0.min_far_bits;
            fcur ^= 1;
            buckets++;
        } else {
            break;
        }
    }
    if (gtid == 0) {
        ctl->steps = steps;
        ctl->buckets = buckets;
        ctl->bottom_up_steps = 0;
    }
    write_back<true>(a);
    return ph;
}

__global__ void __launch_bounds__(kBlock, TRAV_SSSP_MIN_BLOCKS) sssp_persistent(TravArgs a)
{
    __shared__ QueryShared sh;
    __shared__ DeferStage defer[kWarps];
    sssp_query(a, sh, defer, 0);
}

// ------------------------------------------------------------ batch kernel
// Many queries over several graphs in one persistent launch.  The grid is cut
// into teams of b.team_ctas CTAs; a team runs one query at a time with the
// same bodies as the single-query kernels (its grid barrier counts only its
// own CTAs) and then takes the next query from a shared counter, so the
// queries -- issued largest first -- spread over the teams as they free up.
// The team's phase index runs on across its queries, so the counter-slot ring
// stays valid without clearing: every phase clears the slot two ahead.
__global__ void __launch_bounds__(kBlock, TRAV_SSSP_MIN_BLOCKS) batch_persistent(BatchArgs b)
{
    __shared__ QueryShared sh;
    __shared__ DeferStage defer[kWarps];  // used by the SSSP queries
    const int team = (int)blockIdx.x / b.team_ctas;
    const TeamWs w = b.teams[team];
    TravArgs t{};
    t.ctl = w.ctl;
    t.timeout_ns = b.timeout_ns;
    t.cta0 = team * b.team_ctas;
    t.ctas = b.team_ctas;
    const bool leader = (int)blockIdx.x == t.cta0 && threadIdx.x == 0;
    int ph = 0, prev_id = -1;
    while (true) {
        // dispatch phase: the team's first thread takes the next query
        clear_ahead(t, ph);
        if (leader) w.ctl->cur_query = (int)atomicAdd(b.next, 1u);
        if (!grid_sync(t, ph)) return;
        ph++;
        // every CTA of the team has written (and fenced) its part of the
        // previous query's results: raise its completion flag for the host
        if (leader && b.done && prev_id >= 0) {
            __threadfence_system();
            *reinterpret_cast<volatile unsigned *>(&b.done[prev_id]) = 1u;
        }
        const int qi = ld_relaxed_int(&w.ctl->cur_query);
        if (qi >= b.nq) return;
        const BatchQuery &q = b.queries[qi];
        TravArgs a = t;
        a.out_off = q.out_off;
        a.out_adj = q.out_adj;
        a.out_w = q.out_w;
        a.in_off = q.in_off;
        a.in_adj = q.in_adj;
        a.in_w = q.in_w;
        a.new_of_old = q.new_of_old;
        a.V = q.V;
        a.W = (q.V + 31) / 32;
        a.E = q.E;
        a.value = w.value;
        a.dist = reinterpret_cast<unsigned long long *>(w.value);
        a.rcls = w.rcls;
        a.visited = w.visited;
        a.front0 = w.front0;
        a.front1 = w.front1;
        a.q0 = w.q0;
        a.q1 = w.q1;
        a.far0 = w.far0;
        a.far1 = w.far1;
        a.hq0 = w.hq0;
        a.hq1 = w.hq1;
        a.hch0 = w.hch0;
        a.hch1 = w.hch1;
        a.chunks = w.chunks0;
        a.chunks0 = w.chunks0;
        a.chunks1 = w.chunks1;
        a.nlight = q.nlight;
        a.loff = q.loff;
        a.ledge = q.ledge;
        a.source = q.source;
        a.out = q.out;
        a.mlp = q.mlp;
        a.mlp_margin = q.mlp_margin;
        a.plan = nullptr;
        a.plan_len = 0;
        a.small_deg = b.small_deg;
        a.item = b.item;
        if (q.kind == 0) {
            a.max_steps = q.V + 1;
            a.alpha = 15.0f;
            a.beta = 18.0f;
            // The direction network was trained on queries that own the whole
            // grid.  A bottom-up step scans every unvisited vertex, so on a team
            // of a fraction of the grid it costs that much more against a
            // top-down step than the network saw: there a learned query keeps
            // Beamer's switch (on 74-CTA teams at RMAT s23 the network's
            // directions ran 10% slower than Beamer's; on the full grid, even).
            if (2 * b.team_ctas <= b.full_ctas) a.mlp = nullptr;
            a.force_dir = -1;
            a.delta = 0.0f;
            a.out_kind = 0;
            ph = bfs_query(a, sh, ph);
        } else {
            // round stamps are phase indices: the team's whole run must fit them
            a.max_steps = (int32_t)min((long long)4 * q.V + 4096, (long long)(kMaxRounds - 2 - ph));
            a.force_dir = -1;
            a.delta = q.delta;
            a.mean_w = q.mean_w;
            a.max_deg = q.max_deg;
            a.out_kind = 1;
            ph = sssp_query(a, sh, defer, ph);
        }
        if (ph < 0) return;
        if (b.done) __threadfence_system();  // this thread's results, before the next dispatch barrier
        prev_id = q.id;
    }
}

// Light-prefix length of every row for `delta` (rows are sorted by weight):
// the first position whose weight is not below delta.
__global__ void light_count_kernel(const int32_t *__restrict__ out_off, const float *__restrict__ out_w, int32_t V,
                                   float delta, int32_t *__restrict__ nlight)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        int lo = out_off[v], hi = out_off[v + 1];
        const int rb = lo;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (out_w[mid] < delta) lo = mid + 1;
            else hi = mid;
        }
        nlight[v] = lo - rb;
    }
}

// ------------------------------------------------------------- accounting
// Algorithmic bytes of the query just run (see trav_query_stats).
__global__ void sssp_bytes_kernel(const unsigned long long *__restrict__ dist, const int32_t *__restrict__ out_off,
                                  int32_t V, unsigned long long *acc)
{
    unsigned long long r = 0, re = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        if ((unsigned)(dist[v] >> 32) != kFltMaxBits) {
            r++;
            re += (unsigned long long)(out_off[v + 1] - out_off[v]);
        }
    }
    for (int o = 16; o; o >>= 1) {
        r += __shfl_down_sync(kFull, r, o);
        re += __shfl_down_sync(kFull, re, o);
    }
    if (lane_id() == 0) {
        atomicAdd(&acc[0], r);
        atomicAdd(&acc[1], re);
    }
}

__global__ void bfs_bytes_kernel(const int *__restrict__ level, const int32_t *__restrict__ out_off,
                                 const int32_t *__restrict__ in_off, const int32_t *__restrict__ in_adj, int32_t V,
                                 const unsigned char *__restrict__ dirs, int nsteps, unsigned long long *acc)
{
    unsigned long long b = 0, r = 0, re = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const int lv = level[v];
        const int deg = out_off[v + 1] - out_off[v];
        if (lv >= 0) {
            r++;
            re += deg;
            if (lv < nsteps && dirs[lv] == 0) b += 12ull + 8ull * deg;  // expanded top-down at step lv
            if (lv >= 1) b += dirs[lv - 1] == 0 ? 8ull : 4ull;          // discovered at step lv-1
        }
        const int last = lv >= 0 ? min(lv, nsteps) : nsteps;        // BU steps s < lv examine v
        for (int s = 0; s < last; s++) {
            if (dirs[s] == 0) continue;
            b += 12;
            for (int k = in_off[v]; k < in_off[v + 1]; k++) {
                b += 8;
                if (level[in_adj[k]] == s) break;
            }
        }
    }
    for (int o = 16; o; o >>= 1) {
        b += __shfl_down_sync(kFull, b, o);
        r += __shfl_down_sync(kFull, r, o);
        re += __shfl_down_sync(kFull, re, o);
    }
    if (lane_id() == 0) {
        atomicAdd(&acc[0], r);
        atomicAdd(&acc[1], re);
        atomicAdd(&acc[2], b);
    }
}

int g_grid[3] = {0, 0, 0};

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

int device_timeout_err(const Ctl &h, const char *what)
{
    if (h.err == kErrTimeout) {
        set_error(std::string(what) + ": a bounded grid-barrier wait timed out (phase " + std::to_string(h.err_phase) + ")");
        return TRAV_ERR_TIMEOUT;
    }
    if (h.err == kErrBudget) {
        set_error(std::string(what) + ": step budget exhausted");
        return TRAV_ERR_TIMEOUT;
    }
    return TRAV_OK;
}

// Record a timing event; inside a stream capture it becomes an event-record
// node of the graph (an external record), so every replay records it.
int record_event(cudaEvent_t ev, cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    TRY_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs == cudaStreamCaptureStatusActive) TRY_CUDA(cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal));
    else TRY_CUDA(cudaEventRecord(ev, st));
    return TRAV_OK;
}

// A cooperative launch (every CTA co-resident, which the grid barriers need),
// issued through the attribute form so that it can also be captured into a
// CUDA graph.
int launch_cooperative(const void *fn, int grid, void **params, cudaStream_t st)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TRY_CUDA(cudaLaunchKernelExC(&cfg, fn, params));
    return TRAV_OK;
}

// Enqueue one persistent launch: clear its control block, launch
// cooperatively (all CTAs co-resident, which the grid barrier needs).
int enqueue_persistent(int kind, TravArgs &args, int ctas, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1)
{
    int grid = persistent_grid_size(kind);
    if (grid <= 0) return TRAV_ERR_CUDA;
    if (ctas > 0 && ctas < grid) grid = ctas;
    args.cta0 = 0;
    args.ctas = grid;
    TRY_CUDA(cudaMemsetAsync(args.ctl, 0, offsetof(Ctl, dirs), st));
    if (ev0) TRY(record_event(ev0, st));
    void *params[] = {&args};
    TRY(launch_cooperative(kind == 0 ? (const void *)bfs_persistent : (const void *)sssp_persistent, grid, params, st));
    if (ev1) TRY(record_event(ev1, st));
    return TRAV_OK;
}

}  // namespace

int check_queries(Workspace *ws, int n, const char *what) { return check_ctls(ws->ctl, n, what); }

int check_ctls(const Ctl *ctl, int n, const char *what)
{
    for (int q = 0; q < n; q++) {
        Ctl h;
        TRY_CUDA(cudaMemcpy(&h, ctl + q, offsetof(Ctl, slot), cudaMemcpyDeviceToHost));
        int rc = device_timeout_err(h, what);
        if (rc != TRAV_OK) return rc;
    }
    return TRAV_OK;
}

int persistent_grid_size(int kind)
{
    if (g_grid[kind] > 0) return g_grid[kind];
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void *fn = kind == 0 ? (const void *)bfs_persistent
                   : kind == 1 ? (const void *)sssp_persistent : (const void *)batch_persistent;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kBlock, 0);
    if (e != cudaSuccess || per < 1 || sms < 1) {
        cuda_fail(e == cudaSuccess ? cudaErrorInvalidConfiguration : e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        return -1;
    }
    g_grid[kind] = sms * per;
    return g_grid[kind];
}

// Light rows: packed light prefixes {target, weight bits}, one warp per row.
__global__ void light_fill_kernel(const int32_t *__restrict__ out_off, const int32_t *__restrict__ out_adj,
                                  const float *__restrict__ out_w, const int32_t *__restrict__ nlight,
                                  const int32_t *__restrict__ loff, int32_t V, int2 *__restrict__ ledge)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int v = warp; v < V; v += nwarps) {
        const int rb = out_off[v], nl = nlight[v], lb = loff[v];
        for (int k = (int)lane_id(); k < nl; k += 32)
            ledge[lb + k] = make_int2(out_adj[rb + k], __float_as_int(out_w[rb + k]));
    }
}

int count_light(const DevGraph &g, float delta, int32_t *nlight, cudaStream_t st)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (g.V > 0) light_count_kernel<<<sms * 8, 256, 0, st>>>(g.out_off, g.out_w, g.V, delta, nlight);
    TRY_CUDA(cudaGetLastError());
    return TRAV_OK;
}

void light_rows_free(LightRows *lr)
{
    cudaFree(lr->nlight);
    cudaFree(lr->loff);
    cudaFree(lr->ledge);
    *lr = LightRows{};
}

// The light prefix of every row for delta (rows are sorted by weight), and with
// TRAV_LIGHT_ROWS the prefixes packed into rows of their own: the light rounds
// then read 8 contiguous bytes per edge, and a row's bounds from one array,
// instead of two arrays and a prefix length.  Built once per (graph, delta).
int light_rows_build(const DevGraph &g, float delta, LightRows *lr, cudaStream_t st)
{
    if (lr->delta == delta && lr->nlight) return TRAV_OK;
    light_rows_free(lr);
    const int32_t V = g.V > 0 ? g.V : 1;
    TRY_CUDA(dev_malloc(&lr->nlight, sizeof(int32_t) * (size_t)V));
    TRY(count_light(g, delta, lr->nlight, st));
#if TRAV_LIGHT_ROWS
    TRY_CUDA(dev_malloc(&lr->loff, sizeof(int32_t) * ((size_t)V + 1)));
    // loff[0..V) = exclusive scan of nlight; loff[V] = the last offset plus the last length
    size_t tmp_bytes = 0;
    TRY_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, lr->nlight, lr->loff, V, st));
    void *tmp = nullptr;
    TRY_CUDA(dev_malloc(&tmp, tmp_bytes));
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, lr->nlight, lr->loff, g.V, st);
    int32_t last[2] = {0, 0};
    if (e == cudaSuccess && g.V > 0) e = cudaMemcpyAsync(&last[0], lr->loff + g.V - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && g.V > 0) e = cudaMemcpyAsync(&last[1], lr->nlight + g.V - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "light row offsets");
    const int32_t total = last[0] + last[1];
    TRY_CUDA(cudaMemcpyAsync(lr->loff + g.V, &total, sizeof(int32_t), cudaMemcpyHostToDevice, st));
    lr->edges = total;
    TRY_CUDA(dev_malloc(&lr->ledge, sizeof(int2) * (size_t)(total > 0 ? total : 1)));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (g.V > 0)
        light_fill_kernel<<<sms * 8, 256, 0, st>>>(g.out_off, g.out_adj, g.out_w, lr->nlight, lr->loff, g.V,
                                                    lr->ledge);
    TRY_CUDA(cudaGetLastError());
    TRY_CUDA(cudaStreamSynchronize(st));  // the host value `total` is read by the copy above
#endif
    lr->delta = delta;
    return TRAV_OK;
}

int launch_batch(BatchArgs b, int teams, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1)
{
    const int most = persistent_grid_size(2);
    if (most <= 0) return TRAV_ERR_CUDA;
    if (b.team_ctas < 1 || teams < 1 || (int64_t)teams * b.team_ctas > most) {
        set_error("batch launch shape exceeds the co-resident CTAs");
        return TRAV_ERR_BAD_ARG;
    }
    b.full_ctas = most;
    TRY_CUDA(cudaMemsetAsync(b.next, 0, sizeof(unsigned), st));
    if (ev0) TRY_CUDA(cudaEventRecord(ev0, st));
    void *params[] = {&b};
    TRY(launch_cooperative((const void *)batch_persistent, teams * b.team_ctas, params, st));
    if (ev1) TRY_CUDA(cudaEventRecord(ev1, st));
    return TRAV_OK;
}

int workspace_ensure(Workspace *ws, const DevGraph &g, int nqueries, cudaStream_t st)
{
    if (nqueries < 1) nqueries = 1;
    if (ws->ctl && ws->V == g.V) {
        if (nqueries <= ws->ctl_cap) return TRAV_OK;
        TRY_CUDA(cudaStreamSynchronize(st));
        cudaFree(ws->ctl);
        ws->ctl = nullptr;
        ws->ctl_cap = 0;
        TRY_CUDA(dev_malloc(&ws->ctl, sizeof(Ctl) * (size_t)nqueries));
        ws->ctl_cap = nqueries;
        return TRAV_OK;
    }
    workspace_free(ws);
    const int64_t V = g.V > 0 ? g.V : 1;
    const int64_t W = (V + 31) / 32;
    ws->V = g.V;
    ws->chunk_cap = V + g.E / kMinItem + 1;
    TRY_CUDA(dev_malloc(&ws->value, sizeof(unsigned long long) * V));
    TRY_CUDA(dev_malloc(&ws->rcls, sizeof(unsigned char) * V));

    TRY_CUDA(dev_malloc(&ws->visited, sizeof(unsigned) * W));
    TRY_CUDA(dev_malloc(&ws->front[0], sizeof(unsigned) * W));
    TRY_CUDA(dev_malloc(&ws->front[1], sizeof(unsigned) * W));
    for (int i = 0; i < 2; i++) {
        TRY_CUDA(dev_malloc(&ws->queue[i], sizeof(int32_t) * V));
        TRY_CUDA(dev_malloc(&ws->far[i], sizeof(int32_t) * V));
    }
    for (int i = 0; i < 2; i++) {
        TRY_CUDA(dev_malloc(&ws->hq[i], sizeof(int32_t) * V));
        TRY_CUDA(dev_malloc(&ws->hchunks[i], sizeof(int2) * ws->chunk_cap));
    }
    TRY_CUDA(dev_malloc(&ws->chunks[0], sizeof(int2) * ws->chunk_cap));
    TRY_CUDA(dev_malloc(&ws->chunks[1], sizeof(int2) * ws->chunk_cap));
    TRY_CUDA(dev_malloc(&ws->ctl, sizeof(Ctl) * (size_t)nqueries));
    ws->ctl_cap = nqueries;
    return TRAV_OK;
}

void workspace_free(Workspace *ws)
{
    cudaFree(ws->value);
    cudaFree(ws->rcls);
    cudaFree(ws->visited);
    cudaFree(ws->front[0]);
    cudaFree(ws->front[1]);
    for (int i = 0; i < 2; i++) {
        cudaFree(ws->queue[i]);
        cudaFree(ws->far[i]);
    }
    light_rows_free(&ws->light);
    for (int i = 0; i < 2; i++) {
        cudaFree(ws->hq[i]);
        cudaFree(ws->hchunks[i]);
    }
    cudaFree(ws->chunks[0]);
    cudaFree(ws->chunks[1]);
    cudaFree(ws->ctl);
    cudaFree(ws->plan[0]);
    cudaFree(ws->plan[1]);
    *ws = Workspace{};
}

static TravArgs make_args(const DevGraph &g, Workspace *ws)
{
    TravArgs a{};
    a.out_off = g.out_off;
    a.out_adj = g.out_adj;
    a.out_w = g.out_w;
    a.in_off = g.in_off;
    a.in_adj = g.in_adj;
    a.in_w = g.in_w;
    a.new_of_old = g.new_of_old;
    a.V = g.V;
    a.W = (g.V + 31) / 32;
    a.E = g.E;
    a.value = ws->value;
    a.dist = reinterpret_cast<unsigned long long *>(ws->value);
    a.rcls = ws->rcls;
    a.visited = ws->visited;
    a.front0 = ws->front[0];
    a.front1 = ws->front[1];
    a.q0 = ws->queue[0];
    a.q1 = ws->queue[1];
    a.far0 = ws->far[0];
    a.far1 = ws->far[1];
    a.hq0 = ws->hq[0];
    a.hq1 = ws->hq[1];
    a.hch0 = ws->hchunks[0];
    a.hch1 = ws->hchunks[1];
    a.nlight = nullptr;
    a.chunks = ws->chunks[0];
    a.chunks0 = ws->chunks[0];
    a.chunks1 = ws->chunks[1];
    a.timeout_ns = ws->timeout_ns ? ws->timeout_ns : kDefaultTimeoutNs;
    a.mean_w = g.mean_w;
    a.max_deg = g.max_out_degree;
    a.cta0 = 0;
    a.ctas = 0;  // set at launch
    a.small_deg = ws->small_deg;
    a.item = ws->item;
    return a;
}

int launch_bfs(const DevGraph &g, Workspace *ws, int q, int32_t source_new, const trav_bfs_opts &o,
               const float *mlp, void *out, int out_kind, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
               const int32_t *color, int32_t color_want)
{
    TravArgs a = make_args(g, ws);
    a.color = color;
    a.color_want = color_want;
    a.ctl = ws->ctl + q;
    a.source = source_new;
    a.max_steps = g.V + 1;
    if (ws->max_steps > 0 && ws->max_steps < a.max_steps) a.max_steps = ws->max_steps;
    a.alpha = o.alpha;
    a.beta = o.beta;
    a.force_dir = o.force_direction;
    a.delta = 0.0f;
    a.out = out;
    a.out_kind = out_kind;
    a.mlp = mlp;
    a.mlp_margin = ws->mlp_margin[0];
    a.plan = ws->plan[0];
    a.plan_len = ws->plan_len[0];
    return enqueue_persistent(0, a, ws->grid[0], st, ev0, ev1);
}

int launch_sssp(const DevGraph &g, Workspace *ws, int q, int32_t source_new, float delta, const float *mlp,
                void *out, int out_kind, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1)
{
    TravArgs a = make_args(g, ws);
    a.ctl = ws->ctl + q;
    a.source = source_new;
    a.max_steps = (int32_t)std::min<int64_t>(4 * (int64_t)g.V + 4096, kMaxRounds - 2);
    if (ws->max_steps > 0 && ws->max_steps < a.max_steps) a.max_steps = ws->max_steps;
    a.force_dir = -1;
    a.delta = (delta > 0.0f && std::isfinite(delta)) ? delta : INFINITY;
    // the learned schedule also picks the query's delta: its split scales the
    // caller's delta (light/heavy threshold and the unit of the bucket widths)
    if (mlp && std::isfinite(a.delta)) a.delta *= ws->split_scale;
    if (source_new < 0) {
        // start from distance bits gathered into the second queue buffer (read
        // by the initialisation only); every edge is light there
        a.delta = INFINITY;
        a.init_bits = reinterpret_cast<const unsigned *>(ws->queue[1]);
    }
    if (std::isfinite(a.delta)) {
        TRY(light_rows_build(g, a.delta, &ws->light, st));  // once per delta
        a.nlight = ws->light.nlight;
        a.loff = ws->light.loff;
        a.ledge = ws->light.ledge;
    }
    a.out = out;
    a.out_kind = out_kind;
    a.mlp = mlp;
    a.mlp_margin = ws->mlp_margin[1];
    a.plan = ws->plan[1];
    a.plan_len = ws->plan_len[1];
    return enqueue_persistent(1, a, ws->grid[1], st, ev0, ev1);
}

// Byte accounting of query q, which must be the last query run (its results
// are still in the workspace).
int query_bytes(const DevGraph &g, Workspace *ws, int q, int kind, int64_t *bytes, int64_t *reached,
                int64_t *reached_edges, cudaStream_t st)
{
    unsigned long long *acc = nullptr;
    TRY_CUDA(dev_malloc(&acc, sizeof(unsigned long long) * 3));
    TRY_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * 3, st));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = sms * 8;
    if (kind == 1) {
        sssp_bytes_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const unsigned long long *>(ws->value), g.out_off,
                                                g.V, acc);
    } else {
        int nsteps = 0;
        TRY_CUDA(cudaMemcpyAsync(&nsteps, &ws->ctl[q].steps, sizeof(int), cudaMemcpyDeviceToHost, st));
        TRY_CUDA(cudaStreamSynchronize(st));
        bfs_bytes_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const int *>(ws->value), g.out_off, g.in_off, g.in_adj,
                                              g.V, ws->ctl[q].dirs, min(nsteps, kMaxTrace), acc);
    }
    unsigned long long h[3] = {0, 0, 0};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(acc);
    if (e != cudaSuccess) return cuda_fail(e, "query_bytes");
    *reached = (int64_t)h[0];
    *reached_edges = (int64_t)h[1];
    if (kind == 1) *bytes = 4 * (int64_t)g.V + 12 * (int64_t)h[0] + 12 * (int64_t)h[1];
    else *bytes = 4 * (int64_t)g.V + (int64_t)h[2];
    return TRAV_OK;
}

// ------------------------------------------------ allocation-free BFS entry
// For callers that must not allocate device memory: a process whose device
// memory is already owned by another allocator (a framework's caching pool
// that reserved the free memory), or a latency-critical service where the
// device-wide synchronisation of cudaMalloc / cudaFree is not acceptable.
// Those callers hold their graph as a CSR in device memory already; this
// entry point runs the top-down persistent BFS directly on it, taking every
// byte of scratch (levels, visited bitmap, two frontier queues, chunk items,
// the control block) from one statically sized device array of this library.

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;   // 8 MiB on every device that loads the library
constexpr int32_t kNoAllocMaxVertices = 1 << 18;            // 262,144
constexpr int64_t kNoAllocMaxEdges = int64_t(1) << 24;      // 16,777,216
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

void *g_noalloc_base[kNoAllocMaxDevices];  // device address of g_noalloc_scratch, per device
std::mutex g_noalloc_mu;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// The caller's CSR must be well formed before the kernel trusts it.
__global__ void noalloc_validate_csr(const int32_t *__restrict__ off, const int32_t *__restrict__ adj, int32_t V,
                                     int64_t E, int *bad)
{
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
    int flag = 0;
    for (int64_t v = gtid; v <= V; v += nth) {
        int o = off[v];
        if (o < 0 || o > E || (v == 0 && o != 0) || (v == V && o != E) || (v > 0 && off[v - 1] > o)) flag = 1;
    }
    for (int64_t e = gtid; e < E; e += nth) {
        int t = adj[e];
        if (t < 0 || t >= V) flag = 1;
    }
    if (flag) atomicOr(bad, 1);
}

// Top-down-only BFS over the caller's CSR (vertex ids as given, no relabel),
// the same phases as bfs_persistent's top-down step.
__global__ void __launch_bounds__(kBlock) bfs_csr_noalloc_kernel(TravArgs a, int32_t *levels)
{
    __shared__ TileShared ts;
    Ctl *ctl = a.ctl;
    const int gtid = blockIdx.x * kBlock + threadIdx.x, nth = gridDim.x * kBlock;
    const int s = a.source;
    int ph = 0;
    for (int v = gtid; v < a.V; v += nth) reinterpret_cast<int *>(a.value)[v] = v == s ? 0 : -1;
    for (int w = gtid; w < a.W; w += nth) a.visited[w] = w == (s >> 5) ? 1u << (s & 31) : 0u;
    if (gtid == 0) a.q0[0] = s;
    if (!grid_sync(a, ph)) return;
    ph++;
    unsigned long long qlen = 1;
    int L = 0, cur = 0;
    while (qlen > 0) {
        if (L >= a.max_steps) {
            if (gtid == 0) atomicCAS(&ctl->err, 0, kErrBudget);
            return;
        }
        const int32_t *q = cur ? a.q1 : a.q0;
        int32_t *qn = cur ? a.q0 : a.q1;
        clear_ahead(a, ph);
        BfsTopDown vis{&a, L + 1, qn, 0u, &ctl->slot[ph % kSlots]};
        expand_tiles(a, q, (unsigned)qlen, vis, ts, &ctl->slot[ph % kSlots]);
        if (!grid_sync(a, ph)) return;
        SlotView s0 = read_slot(ctl, ph);
        ph++;
        clear_ahead(a, ph);
        vis.qbase = s0.q_add;
        vis.slot = &ctl->slot[ph % kSlots];
        expand_chunks(a, s0.chunk_add, vis);
        if (!grid_sync(a, ph)) return;
        SlotView s1 = read_slot(ctl, ph);
        ph++;
        qlen = (unsigned long long)s0.q_add + s1.q_add;
        L++;
        cur ^= 1;
    }
    if (gtid == 0) ctl->steps = L;
    for (int v = gtid; v < a.V; v += nth) levels[v] = (int32_t)__ldcg(&a.value[v]);
}

}  // namespace

}  // namespace trav

using namespace trav;

// Declared in include/trav.h.  No cudaMalloc, cudaFree or other allocating
// call is made here: scratch comes from g_noalloc_scratch, whose device
// address is looked up once per device (on that device's first call).
extern "C" int trav_bfs_csr_noalloc(const int32_t *row_offsets, const int32_t *adj, int32_t vertices, int64_t edges,
                                    int32_t source, int32_t *levels, void *stream)
{
    if (!row_offsets || !levels || (edges > 0 && !adj)) {
        set_error("trav_bfs_csr_noalloc: row_offsets, adj and levels must be device arrays");
        return TRAV_ERR_BAD_ARG;
    }
    // The CSR check below runs on the GPU, so a host pointer must be caught
    // here, before anything is launched on it.
    if (!is_device_ptr(row_offsets) || !is_device_ptr(levels) || (edges > 0 && !is_device_ptr(adj))) {
        set_error("trav_bfs_csr_noalloc: row_offsets, adj and levels must be device (or managed) memory of the "
                  "current device");
        return TRAV_ERR_BAD_ARG;
    }
    if (vertices < 1 || vertices > kNoAllocMaxVertices || edges < 0 || edges > kNoAllocMaxEdges) {
        set_error("trav_bfs_csr_noalloc: needs 1 <= vertices <= 262144 and 0 <= edges <= 16777216 (its 8 MiB "
                  "static scratch); use trav_bfs for larger graphs");
        return TRAV_ERR_BAD_ARG;
    }
    if (source < 0 || source >= vertices) {
        set_error("trav_bfs_csr_noalloc: source vertex out of range [0, V)");
        return TRAV_ERR_BAD_ARG;
    }
    int dev = 0;
    TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error("trav_bfs_csr_noalloc: device index beyond the supported 64");
        return TRAV_ERR_BAD_ARG;
    }
    unsigned char *base;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_base[dev]) {
            void *p = nullptr;
            TRY_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_noalloc_base[dev] = p;
        }
        base = static_cast<unsigned char *>(g_noalloc_base[dev]);
    }
    const size_t V = (size_t)vertices, W = (V + 31) / 32;
    const size_t chunk_cap = V + (size_t)edges / kChunk + 1;
    size_t at = 0;
    auto carve = [&](size_t bytes) {
        unsigned char *p = base + at;
        at += align256(bytes);
        return p;
    };
    TravArgs a{};
    a.value = reinterpret_cast<unsigned *>(carve(4 * V));
    a.visited = reinterpret_cast<unsigned *>(carve(4 * W));
    a.q0 = reinterpret_cast<int32_t *>(carve(4 * V));
    a.q1 = reinterpret_cast<int32_t *>(carve(4 * V));
    a.chunks = reinterpret_cast<int2 *>(carve(sizeof(int2) * chunk_cap));
    a.ctl = reinterpret_cast<Ctl *>(carve(sizeof(Ctl)));
    int *bad = reinterpret_cast<int *>(carve(sizeof(int)));
    if (at > kNoAllocScratchBytes) {  // cannot happen within the limits above
        set_error("trav_bfs_csr_noalloc: scratch layout exceeds the static array");
        return TRAV_ERR_BAD_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int sms = 0, per = 0;
    TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bfs_csr_noalloc_kernel, kBlock, 0));
    if (per < 1) return cuda_fail(cudaErrorInvalidConfiguration, "bfs_csr_noalloc_kernel occupancy");

    // every call reuses the array: clear the control block and the flag
    TRY_CUDA(cudaMemsetAsync(a.ctl, 0, offsetof(Ctl, dirs), st));
    TRY_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
    noalloc_validate_csr<<<sms * 4, 256, 0, st>>>(row_offsets, adj, vertices, edges, bad);
    TRY_CUDA(cudaGetLastError());
    int hbad = 0;
    TRY_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY_CUDA(cudaStreamSynchronize(st));
    if (hbad) {
        set_error("trav_bfs_csr_noalloc: row_offsets must rise from 0 to edges and adj ids must lie in [0, V)");
        return TRAV_ERR_BAD_ARG;
    }
    a.out_off = row_offsets;
    a.out_adj = adj;
    a.V = vertices;
    a.W = (int32_t)W;
    a.E = edges;
    a.source = source;
    a.max_steps = vertices + 1;
    a.force_dir = 0;
    a.timeout_ns = kDefaultTimeoutNs;
    a.cta0 = 0;
    a.ctas = sms * per;
    a.small_deg = kSmallDeg;
    a.item = kItem;
    void *params[] = {&a, &levels};
    TRY_CUDA(cudaLaunchCooperativeKernel((void *)bfs_csr_noalloc_kernel, dim3(sms * per), dim3(kBlock), params, 0, st));
    // the status is read on the caller's stream, so no other stream is waited for
    Ctl h;
    TRY_CUDA(cudaMemcpyAsync(&h, a.ctl, offsetof(Ctl, slot), cudaMemcpyDeviceToHost, st));
    TRY_CUDA(cudaStreamSynchronize(st));
    return device_timeout_err(h, "trav_bfs_csr_noalloc");
}
