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
#include <cfloat>
#include <climits>
#include <cmath>
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

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_int(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

// Grid-wide barrier with a bounded wait.  Every CTA's thread 0 arrives on a
// counter; the last one resets it and advances the generation.  Waiters give
// up after timeout_ns (or when another CTA already failed) and the barrier
// then returns false in every thread of the CTA.
__device__ bool grid_sync(Ctl *ctl, unsigned long long timeout_ns, int phase)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned gen = ld_acquire(&ctl->bar_gen);
        __threadfence();
        unsigned arrived = atomicAdd(&ctl->bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&ctl->bar_count, 0u);
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            unsigned long long t0 = globaltimer();
            unsigned ns = 32;
            while (ld_acquire(&ctl->bar_gen) == gen) {
                if (ld_relaxed_int(&ctl->err) != 0) { ok = 0; break; }
                __nanosleep(ns);
                if (ns < 256) ns <<= 1;
                if (globaltimer() - t0 > timeout_ns) {
                    if (atomicCAS(&ctl->err, 0, kErrTimeout) == 0) atomicExch(&ctl->err_phase, phase);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (ld_relaxed_int(&ctl->err) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct SlotView {
    unsigned q_add, far_add, chunk_add;
    int min_far_bits;  // kFltMaxBits when nothing was pushed
    unsigned long long mf;
};

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
    return v;
}

// At the start of phase ph, slot ph+2 was last read right after phase ph-1's
// barrier by every CTA, so CTA 0 can clear it for reuse in phase ph+2.
__device__ __forceinline__ void clear_ahead(Ctl *ctl, int ph)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Slot *s = &ctl->slot[(ph + 2) % kSlots];
        s->q_add = 0;
        s->far_add = 0;
        s->chunk_add = 0;
        s->min_far_bits = 0;
        s->mf = 0;
    }
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

struct SsspRelax {
    const TravArgs *a;
    float thr;          // bucket upper bound (exclusive)
    int near_id;        // stamp of the next near queue
    int far_id;         // stamp of the current far epoch
    int32_t *qn;
    unsigned qbase;
    int32_t *farp;
    unsigned fbase;
    Slot *slot;

    __device__ __forceinline__ float begin(int u) const { return __uint_as_float(__ldcg(&a->value[u])); }

    __device__ __forceinline__ void visit(int, float du, int e, bool valid) const
    {
        bool imp = false;
        int v = 0;
        float nd = 0.0f;
        if (valid) {
            v = __ldg(&a->out_adj[e]);
            nd = __fadd_rn(du, __ldg(&a->out_w[e]));  // one rounded add, as sssp.hpp:56
            if (nd < __uint_as_float(__ldcg(&a->value[v]))) {
                int old = atomicMin(reinterpret_cast<int *>(a->value) + v, __float_as_int(nd));
                imp = nd < __int_as_float(old);
            }
        }
        bool near = false, far = false;
        if (imp) {
            if (nd < thr) near = atomicExch(&a->stamp_near[v], near_id) != near_id;
            else far = atomicExch(&a->stamp_far[v], far_id) != far_id;
        }
        warp_append(near, v, qn, qbase, &slot->q_add);
        if (__any_sync(kFull, far)) {
            warp_append(far, v, farp, fbase, &slot->far_add);
            int key = far ? 0x7fffffff - __float_as_int(nd) : 0;
            key = __reduce_max_sync(kFull, key);
            if (lane_id() == 0) atomicMax(&slot->min_far_bits, key);
        }
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
__device__ void write_back(const TravArgs &a)
{
    if (!a.out) return;
    const int gtid = blockIdx.x * kBlock + threadIdx.x, nth = gridDim.x * kBlock;
    for (int v = gtid; v < a.V; v += nth) {
        unsigned x = __ldcg(&a.value[__ldg(&a.new_of_old[v])]);
        if (a.out_kind == 0) reinterpret_cast<int32_t *>(a.out)[v] = (int32_t)x;
        else if (a.out_kind == 1) reinterpret_cast<unsigned *>(a.out)[v] = x;
        else if (a.out_kind == 2) reinterpret_cast<unsigned char *>(a.out)[v] = (int32_t)x >= 0 ? 1 : 0;
        else reinterpret_cast<unsigned char *>(a.out)[v] = x != kFltMaxBits ? 1 : 0;
    }
}

// --------------------------------------------------------------- BFS kernel
__global__ void __launch_bounds__(kBlock) bfs_persistent(TravArgs a)
{
    __shared__ TileShared ts;
    __shared__ int s_dir;
    Ctl *ctl = a.ctl;
    const int gtid = blockIdx.x * kBlock + threadIdx.x, nth = gridDim.x * kBlock;
    const unsigned gwarp = gtid >> 5, nwarps = nth >> 5;
    const int s = a.source;
    int ph = 0;

    for (int v = gtid; v < a.V; v += nth) reinterpret_cast<int *>(a.value)[v] = v == s ? 0 : -1;
    for (int w = gtid; w < a.W; w += nth) a.visited[w] = w == (s >> 5) ? 1u << (s & 31) : 0u;
    if (gtid == 0) a.q0[0] = s;
    if (!grid_sync(ctl, a.timeout_ns, ph)) return;
    ph++;

    const unsigned long long deg_s = (unsigned long long)(__ldg(&a.out_off[s + 1]) - __ldg(&a.out_off[s]));
    unsigned long long qlen = 1, nf_prev = 0, mf = deg_s, mu = (unsigned long long)a.E - deg_s;
    int dir = 0, prev_dir = 0, L = 0, cur = 0, fcur = 0, bu_steps = 0;
    while (qlen > 0) {
        if (L >= a.max_steps) {
            if (gtid == 0) atomicCAS(&ctl->err, 0, kErrBudget);
            return;
        }
        // direction for this step (same inputs in every CTA -> same answer)
        if (threadIdx.x < 32) {
            int d = dir;
            if (a.force_dir >= 0) d = (L == 0) ? 0 : a.force_dir;
            else if (a.mlp) d = mlp_argmax_warp(a.mlp, bfs_features(L, qlen, mf, mu, nf_prev, a.V, a.E, prev_dir), kBfsOut);
            else if (dir == 0) { if ((double)mf > (double)mu / a.alpha) d = 1; }
            else if (!(qlen >= nf_prev || (double)qlen > (double)a.V / a.beta)) d = 0;
            if (threadIdx.x == 0) s_dir = d;
        }
        __syncthreads();
        dir = s_dir;
        if (gtid == 0 && L < kMaxTrace) {
            ctl->dirs[L] = (unsigned char)dir;
            ctl->frontier[L] = (unsigned)qlen;
        }
        const int32_t *q = cur ? a.q1 : a.q0;
        int32_t *qn = cur ? a.q0 : a.q1;
        unsigned long long qnext, mfn;
        if (dir == 0) {
            clear_ahead(ctl, ph);
            BfsTopDown vis{&a, L + 1, qn, 0u, &ctl->slot[ph % kSlots]};
            expand_tiles(a, q, (unsigned)qlen, vis, ts, &ctl->slot[ph % kSlots]);
            if (!grid_sync(ctl, a.timeout_ns, ph)) return;
            SlotView s0 = read_slot(ctl, ph);
            ph++;
            clear_ahead(ctl, ph);
            vis.qbase = s0.q_add;
            vis.slot = &ctl->slot[ph % kSlots];
            expand_chunks(a, s0.chunk_add, vis);
            if (!grid_sync(ctl, a.timeout_ns, ph)) return;
            SlotView s1 = read_slot(ctl, ph);
            ph++;
            qnext = (unsigned long long)s0.q_add + s1.q_add;
            mfn = s0.mf + s1.mf;
        } else {
            unsigned *fc = fcur ? a.front1 : a.front0;
            unsigned *fn = fcur ? a.front0 : a.front1;
            if (prev_dir == 0) {
                // frontier bitmap from the levels: bit v = (level[v] == L)
                clear_ahead(ctl, ph);
                for (unsigned w = gwarp; w < (unsigned)a.W; w += nwarps) {
                    int v = (int)(w * 32 + lane_id());
                    bool f = v < a.V && (int)__ldcg(&a.value[v]) == L;
                    unsigned m = __ballot_sync(kFull, f);
                    if (lane_id() == 0) fc[w] = m;
                }
                if (!grid_sync(ctl, a.timeout_ns, ph)) return;
                ph++;
            }
            clear_ahead(ctl, ph);
            Slot *slot = &ctl->slot[ph % kSlots];
            // bottom-up: each warp owns 32 vertices = one bitmap word
            for (unsigned w = gwarp; w < (unsigned)a.W; w += nwarps) {
                int v = (int)(w * 32 + lane_id());
                unsigned vis = __ldcg(&a.visited[w]);
                bool found = false;
                if (v < a.V && !((vis >> lane_id()) & 1u)) {
                    int k = __ldg(&a.in_off[v]);
                    const int kend = __ldg(&a.in_off[v + 1]);
                    for (; k < kend; k++) {
                        int u = __ldg(&a.in_adj[k]);
                        if ((__ldcg(&fc[u >> 5]) >> (u & 31)) & 1u) { found = true; break; }
                    }
                }
                unsigned m = __ballot_sync(kFull, found);
                if (lane_id() == 0) {
                    fn[w] = m;
                    if (m) a.visited[w] = vis | m;
                }
                unsigned deg = 0;
                if (found) {
                    reinterpret_cast<int *>(a.value)[v] = L + 1;
                    deg = (unsigned)(__ldg(&a.out_off[v + 1]) - __ldg(&a.out_off[v]));
                }
                warp_append(found, v, qn, 0u, &slot->q_add);
                warp_add_u64(deg, &slot->mf);
            }
            if (!grid_sync(ctl, a.timeout_ns, ph)) return;
            SlotView s0 = read_slot(ctl, ph);
            ph++;
            qnext = s0.q_add;
            mfn = s0.mf;
            fcur ^= 1;
            bu_steps++;
        }
        mu -= mfn;
        nf_prev = qlen;
        qlen = qnext;
        mf = mfn;
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
}

// -------------------------------------------------------------- SSSP kernel
// Near/far delta-stepping: the near queue holds vertices whose distance
// improved below the bucket bound `thr`; improvements at or above it go to
// the far pile.  When the near queue drains, the bound advances and the far
// pile is split (entries below the new bound move to the near queue, stale
// ones are dropped).  delta = +inf gives Bellman-Ford over active vertices.
// Any order of relaxations reaches the same fixpoint bits: fl(x + w) is
// monotone in x and not below x for w >= 0.
__global__ void __launch_bounds__(kBlock) sssp_persistent(TravArgs a)
{
    __shared__ TileShared ts;
    __shared__ float s_delta;
    Ctl *ctl = a.ctl;
    const int gtid = blockIdx.x * kBlock + threadIdx.x, nth = gridDim.x * kBlock;
    int ph = 0;
    // Stamp ids continue across queries so the stamp arrays need no clearing;
    // every CTA reads the base before the first barrier, thread 0 of CTA 0
    // advances it after the last one.  Near the int range they are recycled.
    int first_id = *(volatile int *)a.id_base;
    if (first_id > (1 << 30)) {
        for (int v = gtid; v < a.V; v += nth) {
            a.stamp_near[v] = -1;
            a.stamp_far[v] = -1;
        }
        first_id = 0;
    }
    int near_id = first_id, far_id = first_id;
    unsigned long long qlen, far_len = 0;
    int min_far = (int)kFltMaxBits;
    float thr = a.delta > 0.0f ? a.delta : INFINITY;

    if (a.source >= 0) {
        const int s = a.source;
        for (int v = gtid; v < a.V; v += nth) a.value[v] = v == s ? 0u : kFltMaxBits;
        if (gtid == 0) {
            a.q0[0] = s;
            a.stamp_near[s] = near_id;
        }
        if (!grid_sync(ctl, a.timeout_ns, ph)) return;
        ph++;
        qlen = 1;
    } else {
        // start from the distances already in `value` (Bellman-Ford entry
        // point): every vertex below FLT_MAX is active.
        thr = INFINITY;
        clear_ahead(ctl, ph);
        Slot *slot = &ctl->slot[ph % kSlots];
        for (int base = gtid - (int)lane_id(); base < a.V; base += nth) {
            int v = base + (int)lane_id();
            bool act = v < a.V && __ldcg(&a.value[v]) < kFltMaxBits;
            if (act) a.stamp_near[v] = near_id;
            warp_append(act, v, a.q0, 0u, &slot->q_add);
        }
        if (!grid_sync(ctl, a.timeout_ns, ph)) return;
        qlen = read_slot(ctl, ph).q_add;
        ph++;
    }

    int cur = 0, fcur = 0, steps = 0, buckets = 1;
    float dcur = thr;  // width of the current bucket
    while (true) {
        if (qlen > 0) {
            if (steps >= a.max_steps) {
                if (gtid == 0) atomicCAS(&ctl->err, 0, kErrBudget);
                return;
            }
            const int32_t *q = cur ? a.q1 : a.q0;
            int32_t *qn = cur ? a.q0 : a.q1;
            int32_t *fp = fcur ? a.far1 : a.far0;
            clear_ahead(ctl, ph);
            SsspRelax vis{&a, thr, near_id + 1, far_id, qn, 0u, fp, (unsigned)far_len, &ctl->slot[ph % kSlots]};
            expand_tiles(a, q, (unsigned)qlen, vis, ts, &ctl->slot[ph % kSlots]);
            if (!grid_sync(ctl, a.timeout_ns, ph)) return;
            SlotView s0 = read_slot(ctl, ph);
            ph++;
            clear_ahead(ctl, ph);
            vis.qbase = s0.q_add;
            vis.fbase = (unsigned)(far_len + s0.far_add);
            vis.slot = &ctl->slot[ph % kSlots];
            expand_chunks(a, s0.chunk_add, vis);
            if (!grid_sync(ctl, a.timeout_ns, ph)) return;
            SlotView s1 = read_slot(ctl, ph);
            ph++;
            qlen = (unsigned long long)s0.q_add + s1.q_add;
            far_len += (unsigned long long)s0.far_add + s1.far_add;
            min_far = min(min_far, min(s0.min_far_bits, s1.min_far_bits));
            near_id++;
            cur ^= 1;
            steps++;
            if (gtid == 0 && steps - 1 < kMaxTrace) ctl->frontier[steps - 1] = (unsigned)qlen;
        } else if (far_len > 0) {
            if (buckets >= a.max_steps) {
                if (gtid == 0) atomicCAS(&ctl->err, 0, kErrBudget);
                return;
            }
            // open the next bucket (skipping empty ones): bound = max(old, min far) + width
            if (threadIdx.x < 32) {
                float d = a.delta;
                if (a.mlp)
                    d = a.delta * sssp_width_scale(mlp_argmax_warp(
                                      a.mlp, sssp_features(steps, far_len, __int_as_float(min_far), thr, a.delta, a.V, a.E, buckets),
                                      kSsspOut));
                if (threadIdx.x == 0) s_delta = d;
            }
            __syncthreads();
            dcur = s_delta;
            const float told = thr;
            thr = __fadd_rn(fmaxf(told, __int_as_float(min_far)), dcur);
            if (!(thr > told)) thr = nextafterf(told, INFINITY);
            far_id++;
            const int32_t *fp = fcur ? a.far1 : a.far0;
            int32_t *fq = fcur ? a.far0 : a.far1;
            int32_t *q = cur ? a.q1 : a.q0;  // the (empty) current near queue
            clear_ahead(ctl, ph);
            Slot *slot = &ctl->slot[ph % kSlots];
            for (unsigned long long base = gtid - lane_id(); base < far_len; base += nth) {
                unsigned long long i = base + lane_id();
                bool valid = i < far_len;
                int v = valid ? __ldcg(&fp[i]) : 0;
                float d = valid ? __uint_as_float(__ldcg(&a.value[v])) : 0.0f;
                bool to_near = valid && d >= told && d < thr && atomicExch(&a.stamp_near[v], near_id) != near_id;
                bool keep = valid && d >= thr && atomicExch(&a.stamp_far[v], far_id) != far_id;
                warp_append(to_near, v, q, 0u, &slot->q_add);
                warp_append(keep, v, fq, 0u, &slot->far_add);
                int key = keep ? 0x7fffffff - __float_as_int(d) : 0;
                key = __reduce_max_sync(kFull, key);
                if (key && lane_id() == 0) atomicMax(&slot->min_far_bits, key);
            }
            if (!grid_sync(ctl, a.timeout_ns, ph)) return;
            SlotView s0 = read_slot(ctl, ph);
            ph++;
            qlen = s0.q_add;
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
        ctl->next_id = max(near_id, far_id) + 1;
        *a.id_base = ctl->next_id;
    }
    write_back(a);
}

// ------------------------------------------------------------- accounting
// Algorithmic bytes of the query just run (see trav_query_stats).
__global__ void sssp_bytes_kernel(const unsigned *__restrict__ value, const int32_t *__restrict__ out_off, int32_t V,
                                  unsigned long long *acc)
{
    unsigned long long r = 0, re = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        if (value[v] != kFltMaxBits) {
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

int g_grid[2] = {0, 0};

#define TRY_CUDA(expr)                                      \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
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

// Enqueue one persistent launch: clear its control block, launch
// cooperatively (all CTAs co-resident, which the grid barrier needs).
int enqueue_persistent(int kind, TravArgs &args, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1)
{
    int grid = persistent_grid_size(kind);
    if (grid <= 0) return TRAV_ERR_CUDA;
    TRY_CUDA(cudaMemsetAsync(args.ctl, 0, offsetof(Ctl, dirs), st));
    if (ev0) TRY_CUDA(cudaEventRecord(ev0, st));
    void *params[] = {&args};
    TRY_CUDA(cudaLaunchCooperativeKernel(kind == 0 ? (void *)bfs_persistent : (void *)sssp_persistent, dim3(grid),
                                         dim3(kBlock), params, 0, st));
    if (ev1) TRY_CUDA(cudaEventRecord(ev1, st));
    return TRAV_OK;
}

}  // namespace

int check_queries(Workspace *ws, int n, const char *what)
{
    for (int q = 0; q < n; q++) {
        Ctl h;
        TRY_CUDA(cudaMemcpy(&h, ws->ctl + q, offsetof(Ctl, slot), cudaMemcpyDeviceToHost));
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
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per, kind == 0 ? (const void *)bfs_persistent : (const void *)sssp_persistent, kBlock, 0);
    if (e != cudaSuccess || per < 1 || sms < 1) {
        cuda_fail(e == cudaSuccess ? cudaErrorInvalidConfiguration : e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        return -1;
    }
    g_grid[kind] = sms * per;
    return g_grid[kind];
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
        TRY_CUDA(cudaMalloc(&ws->ctl, sizeof(Ctl) * (size_t)nqueries));
        ws->ctl_cap = nqueries;
        return TRAV_OK;
    }
    workspace_free(ws);
    const int64_t V = g.V > 0 ? g.V : 1;
    const int64_t W = (V + 31) / 32;
    ws->V = g.V;
    ws->chunk_cap = V + g.E / kChunk + 1;
    TRY_CUDA(cudaMalloc(&ws->value, sizeof(unsigned) * V));
    TRY_CUDA(cudaMalloc(&ws->visited, sizeof(unsigned) * W));
    TRY_CUDA(cudaMalloc(&ws->front[0], sizeof(unsigned) * W));
    TRY_CUDA(cudaMalloc(&ws->front[1], sizeof(unsigned) * W));
    for (int i = 0; i < 2; i++) {
        TRY_CUDA(cudaMalloc(&ws->queue[i], sizeof(int32_t) * V));
        TRY_CUDA(cudaMalloc(&ws->far[i], sizeof(int32_t) * V));
    }
    TRY_CUDA(cudaMalloc(&ws->stamp_near, sizeof(int32_t) * V));
    TRY_CUDA(cudaMalloc(&ws->stamp_far, sizeof(int32_t) * V));
    TRY_CUDA(cudaMalloc(&ws->chunks, sizeof(int2) * ws->chunk_cap));
    TRY_CUDA(cudaMalloc(&ws->ctl, sizeof(Ctl) * (size_t)nqueries));
    ws->ctl_cap = nqueries;
    TRY_CUDA(cudaMalloc(&ws->id_base, sizeof(int)));
    TRY_CUDA(cudaMemsetAsync(ws->id_base, 0, sizeof(int), st));
    TRY_CUDA(cudaMemsetAsync(ws->stamp_near, 0xff, sizeof(int32_t) * V, st));
    TRY_CUDA(cudaMemsetAsync(ws->stamp_far, 0xff, sizeof(int32_t) * V, st));
    return TRAV_OK;
}

void workspace_free(Workspace *ws)
{
    cudaFree(ws->value);
    cudaFree(ws->visited);
    cudaFree(ws->front[0]);
    cudaFree(ws->front[1]);
    for (int i = 0; i < 2; i++) {
        cudaFree(ws->queue[i]);
        cudaFree(ws->far[i]);
    }
    cudaFree(ws->stamp_near);
    cudaFree(ws->stamp_far);
    cudaFree(ws->chunks);
    cudaFree(ws->ctl);
    cudaFree(ws->id_base);
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
    a.new_of_old = g.new_of_old;
    a.V = g.V;
    a.W = (g.V + 31) / 32;
    a.E = g.E;
    a.value = ws->value;
    a.visited = ws->visited;
    a.front0 = ws->front[0];
    a.front1 = ws->front[1];
    a.q0 = ws->queue[0];
    a.q1 = ws->queue[1];
    a.far0 = ws->far[0];
    a.far1 = ws->far[1];
    a.stamp_near = ws->stamp_near;
    a.stamp_far = ws->stamp_far;
    a.chunks = ws->chunks;
    a.id_base = ws->id_base;
    a.timeout_ns = 10ull * 1000000000ull;
    return a;
}

int launch_bfs(const DevGraph &g, Workspace *ws, int q, int32_t source_new, const trav_bfs_opts &o,
               const float *mlp, void *out, int out_kind, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1)
{
    TravArgs a = make_args(g, ws);
    a.ctl = ws->ctl + q;
    a.source = source_new;
    a.max_steps = g.V + 1;
    a.alpha = o.alpha;
    a.beta = o.beta;
    a.force_dir = o.force_direction;
    a.delta = 0.0f;
    a.out = out;
    a.out_kind = out_kind;
    a.mlp = mlp;
    return enqueue_persistent(0, a, st, ev0, ev1);
}

int launch_sssp(const DevGraph &g, Workspace *ws, int q, int32_t source_new, float delta, const float *mlp,
                void *out, int out_kind, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1)
{
    TravArgs a = make_args(g, ws);
    a.ctl = ws->ctl + q;
    a.source = source_new;
    a.max_steps = 4 * g.V + 4096;
    a.force_dir = -1;
    a.delta = (delta > 0.0f && std::isfinite(delta)) ? delta : INFINITY;
    a.out = out;
    a.out_kind = out_kind;
    a.mlp = mlp;
    return enqueue_persistent(1, a, st, ev0, ev1);
}

// Byte accounting of query q, which must be the last query run (its results
// are still in the workspace).
int query_bytes(const DevGraph &g, Workspace *ws, int q, int kind, int64_t *bytes, int64_t *reached,
                int64_t *reached_edges, cudaStream_t st)
{
    unsigned long long *acc = nullptr;
    TRY_CUDA(cudaMalloc(&acc, sizeof(unsigned long long) * 3));
    TRY_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * 3, st));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = sms * 8;
    if (kind == 1) {
        sssp_bytes_kernel<<<grid, 256, 0, st>>>(ws->value, g.out_off, g.V, acc);
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
    if (!grid_sync(ctl, a.timeout_ns, ph)) return;
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
        clear_ahead(ctl, ph);
        BfsTopDown vis{&a, L + 1, qn, 0u, &ctl->slot[ph % kSlots]};
        expand_tiles(a, q, (unsigned)qlen, vis, ts, &ctl->slot[ph % kSlots]);
        if (!grid_sync(ctl, a.timeout_ns, ph)) return;
        SlotView s0 = read_slot(ctl, ph);
        ph++;
        clear_ahead(ctl, ph);
        vis.qbase = s0.q_add;
        vis.slot = &ctl->slot[ph % kSlots];
        expand_chunks(a, s0.chunk_add, vis);
        if (!grid_sync(ctl, a.timeout_ns, ph)) return;
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
    a.timeout_ns = 10ull * 1000000000ull;
    void *params[] = {&a, &levels};
    TRY_CUDA(cudaLaunchCooperativeKernel((void *)bfs_csr_noalloc_kernel, dim3(sms * per), dim3(kBlock), params, 0, st));
    TRY_CUDA(cudaStreamSynchronize(st));
    Ctl h;
    TRY_CUDA(cudaMemcpy(&h, a.ctl, offsetof(Ctl, slot), cudaMemcpyDeviceToHost));
    return device_timeout_err(h, "trav_bfs_csr_noalloc");
}
