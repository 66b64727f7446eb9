// Graph ingest on the device: seeded RMAT generation, edge validation and the
// edge-list -> CSR build (degree relabel, sorted rows, transposed CSR).
//
// Reference counterparts:
//   GraphGenerationAPI::R_MAT_parallel  include/test/generation/graph_generation_API.hpp:403-484
//   Graph::convert_to_compressed_adjacency_list  include/graph_data_structures/graph.hpp:248-361
//   Graph::transpose                    include/graph_data_structures/graph.hpp:464-497
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <cfloat>
#include <climits>

#include "trav_internal.cuh"

namespace trav {

namespace {

constexpr uint32_t kLcgA = 1103515245u;
constexpr uint32_t kLcgC = 12345u;

struct Affine { uint32_t a, c; };  // x -> a*x + c (mod 2^32)

__host__ __device__ inline Affine affine_pow(uint64_t steps)
{
    Affine acc{1u, 0u}, cur{kLcgA, kLcgC};
    while (steps) {
        if (steps & 1u) acc = Affine{acc.a * cur.a, acc.c * cur.a + cur.c};
        cur = Affine{cur.a * cur.a, cur.c * cur.a + cur.c};
        steps >>= 1;
    }
    return acc;
}

// glibc rand_r: three LCG steps combined into 31 bits.
__device__ __forceinline__ int rand_r_dev(uint32_t &s)
{
    uint32_t n = s;
    int r;
    n = n * kLcgA + kLcgC;
    r = (int)((n >> 16) % 2048u);
    n = n * kLcgA + kLcgC;
    r = (r << 10) ^ (int)((n >> 16) % 1024u);
    n = n * kLcgA + kLcgC;
    r = (r << 10) ^ (int)((n >> 16) % 1024u);
    s = n;
    return r;
}

// One thread per edge stream position: thread t generates edges t, t+T, ...
// Its LCG state starts at step spe*t (spe = steps per edge) and jumps by the
// precomputed map `gap` = spe*(T-1) steps between its edges.
__global__ void rmat_kernel(int scale, int64_t E, int a, int b, int c, int d, uint32_t seed,
                            Affine gap, uint64_t spe, int32_t *__restrict__ src, int32_t *__restrict__ dst,
                            float *__restrict__ w)
{
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= E) return;
    Affine start = affine_pow(spe * (uint64_t)t);
    uint32_t st = start.a * seed + start.c;
    const int V = 1 << scale;
    const int ab = a + b, abc = a + b + c, abcd = a + b + c + d;
    for (int64_t e = t; e < E; e += T) {
        int x = V / 2, y = V / 2;
        for (int i = 1; i < scale; i++) {
            int step = 1 << (scale - (i + 1));
            int p = rand_r_dev(st) % 100;
            if (p < a) { x -= step; y -= step; }
            else if (p < ab) { x -= step; y += step; }
            else if (p < abc) { x += step; y -= step; }
            else if (p < abcd) { x += step; y += step; }
        }
        if (rand_r_dev(st) % 2 == 0) x--;
        if (rand_r_dev(st) % 2 == 0) y--;
        // (float)r / (float)RAND_MAX: (float)2147483647 rounds to 2^31, so the
        // quotient is an exact scaling by 2^-31 of the rounded numerator.
        float wt = __fdiv_rn(__int2float_rn(rand_r_dev(st)), 2147483648.0f);
        src[e] = x;
        dst[e] = y;
        w[e] = wt;
        st = gap.a * st + gap.c;
    }
}

__global__ void loop_flags_kernel(const int32_t *__restrict__ src, const int32_t *__restrict__ dst, int64_t E,
                                  unsigned char *__restrict__ keep)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
        keep[e] = src[e] != dst[e];
}

// bad[0] |= 1 for an id out of range, 2 for a negative weight, 4 for a NaN or
// infinite weight (the fp32 fixpoint is defined for finite weights >= 0).
__global__ void validate_kernel(int32_t V, int64_t E, const int32_t *__restrict__ src,
                                const int32_t *__restrict__ dst, const float *__restrict__ w, int *bad)
{
    int flag = 0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        int s = src[e], t = dst[e];
        if (s < 0 || s >= V || t < 0 || t >= V) flag |= 1;
        if (w) {
            const float x = w[e];
            if (x < 0.0f) flag |= 2;
            if (!isfinite(x)) flag |= 4;
        }
    }
    flag = __reduce_or_sync(0xffffffffu, flag);
    if (flag && (threadIdx.x & 31) == 0) atomicOr(bad, flag);
}

__global__ void degree_kernel(int64_t E, const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                              int32_t *out_deg, int32_t *in_deg)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        atomicAdd(&out_deg[src[e]], 1);
        atomicAdd(&in_deg[dst[e]], 1);
    }
}

__global__ void iota_kernel(int32_t *x, int32_t n)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = i;
}

// new_of_old[old_of_new[r]] = r; degrees in new order (entry V = 0 for the scan).
__global__ void relabel_kernel(int32_t V, const int32_t *__restrict__ old_of_new, const int32_t *__restrict__ out_deg,
                               const int32_t *__restrict__ in_deg, int32_t *__restrict__ new_of_old,
                               int32_t *__restrict__ out_deg_new, int32_t *__restrict__ in_deg_new)
{
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= V; r += gridDim.x * blockDim.x) {
        if (r == V) {
            out_deg_new[V] = 0;
            in_deg_new[V] = 0;
            continue;
        }
        int32_t o = old_of_new[r];
        new_of_old[o] = r;
        out_deg_new[r] = out_deg[o];
        in_deg_new[r] = in_deg[o];
    }
}

// Out-row key (new source, weight bits): rows sorted by weight so the edges
// lighter than any delta form a prefix.  -0.0 is stored as +0.0 (the sum
// d + w is the same for d >= 0) so that zero weights sort first.
__global__ void edge_keys_kernel(int64_t E, int lv, const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                                 const int32_t *__restrict__ new_of_old, const float *__restrict__ w,
                                 unsigned long long *__restrict__ out_keys, unsigned long long *__restrict__ in_keys,
                                 int32_t *__restrict__ out_dst, float *__restrict__ in_wt)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long s = (unsigned)new_of_old[src[e]], t = (unsigned)new_of_old[dst[e]];
        float wt = w ? w[e] : 1.0f;
        if (wt == 0.0f) wt = 0.0f;
        out_keys[e] = (s << 32) | __float_as_uint(wt);
        in_keys[e] = (t << lv) | s;
        out_dst[e] = (int32_t)t;
        in_wt[e] = wt;
    }
}

__global__ void low_word_float_kernel(int64_t E, const unsigned long long *__restrict__ keys, float *__restrict__ out)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = __uint_as_float((unsigned)(keys[e] & 0xffffffffull));
}

__global__ void low_bits_kernel(int64_t E, unsigned long long mask, const unsigned long long *__restrict__ keys,
                                int32_t *__restrict__ out)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = (int32_t)(keys[e] & mask);
}

int grid_for(int64_t n, int block = 256)
{
    int64_t g = (n + block - 1) / block;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t cap = (int64_t)sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// Scoped device allocation.
// Sum of the weights in fixed order: each block adds a grid-stride share in
// double and reduces it in a fixed tree; the host adds the block sums in
// block order.  (The mean weight is a schedule feature, so it must not vary
// from run to run.)
constexpr int kWSumBlocks = 256;

__global__ void weight_sum_kernel(int64_t E, const float *__restrict__ w, double *__restrict__ partial)
{
    __shared__ double sh[256];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x)
        acc += (double)w[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

template <class T>
struct DBuf {
    T *p = nullptr;
    cudaError_t alloc(int64_t n) { return dev_malloc((void **)&p, sizeof(T) * (size_t)(n > 0 ? n : 1)); }
    ~DBuf() { if (p) cudaFree(p); }
    T *release() { T *q = p; p = nullptr; return q; }
};

#define TRY_CUDA(expr)                                   \
    do {                                                 \
        cudaError_t _e = (expr);                         \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

}  // namespace

int rmat_device(int scale, int avg, int a, int b, int c, int d, uint32_t seed, int drop_loops,
                int32_t *d_src, int32_t *d_dst, float *d_w, int64_t *E_out, cudaStream_t st)
{
    if (scale < 1 || scale > 30 || avg < 1 || a < 0 || b < 0 || c < 0 || d < 0) {
        set_error("trav_graph_rmat: scale must be in [1,30], avg >= 1, probabilities >= 0");
        return TRAV_ERR_BAD_ARG;
    }
    int64_t E = ((int64_t)1 << scale) * avg;
    uint64_t spe = 3ull * (uint64_t)(scale + 2);
    int threads = 256;
    int blocks = grid_for(E, threads) * 4;
    int64_t T = (int64_t)blocks * threads;
    if (T > E) { blocks = (int)((E + threads - 1) / threads); T = (int64_t)blocks * threads; }
    Affine gap = affine_pow(spe * (uint64_t)(T - 1));
    rmat_kernel<<<blocks, threads, 0, st>>>(scale, E, a, b, c, d, seed, gap, spe, d_src, d_dst, d_w);
    TRY_CUDA(cudaGetLastError());
    if (drop_loops) {
        DBuf<unsigned char> keep;
        DBuf<int32_t> tmp_i;
        DBuf<float> tmp_f;
        DBuf<int64_t> nsel;
        TRY_CUDA(keep.alloc(E));
        TRY_CUDA(tmp_i.alloc(E));
        TRY_CUDA(tmp_f.alloc(E));
        TRY_CUDA(nsel.alloc(1));
        loop_flags_kernel<<<grid_for(E), 256, 0, st>>>(d_src, d_dst, E, keep.p);
        size_t tb = 0;
        TRY_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, d_src, keep.p, tmp_i.p, nsel.p, E, st));
        DBuf<unsigned char> temp;
        TRY_CUDA(temp.alloc((int64_t)tb));
        int64_t n = 0;
        TRY_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, d_src, keep.p, tmp_i.p, nsel.p, E, st));
        TRY_CUDA(cudaMemcpyAsync(d_src, tmp_i.p, sizeof(int32_t) * E, cudaMemcpyDeviceToDevice, st));
        TRY_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, d_dst, keep.p, tmp_i.p, nsel.p, E, st));
        TRY_CUDA(cudaMemcpyAsync(d_dst, tmp_i.p, sizeof(int32_t) * E, cudaMemcpyDeviceToDevice, st));
        TRY_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, d_w, keep.p, tmp_f.p, nsel.p, E, st));
        TRY_CUDA(cudaMemcpyAsync(d_w, tmp_f.p, sizeof(float) * E, cudaMemcpyDeviceToDevice, st));
        TRY_CUDA(cudaMemcpyAsync(&n, nsel.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        TRY_CUDA(cudaStreamSynchronize(st));
        E = n;
    }
    TRY_CUDA(cudaStreamSynchronize(st));
    *E_out = E;
    return TRAV_OK;
}

int validate_edges(int32_t V, int64_t E, const int32_t *d_src, const int32_t *d_dst, const float *d_w,
                   cudaStream_t st)
{
    if (E == 0) return TRAV_OK;
    DBuf<int> bad;
    TRY_CUDA(bad.alloc(1));
    TRY_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    validate_kernel<<<grid_for(E), 256, 0, st>>>(V, E, d_src, d_dst, d_w, bad.p);
    TRY_CUDA(cudaGetLastError());
    int h = 0;
    TRY_CUDA(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY_CUDA(cudaStreamSynchronize(st));
    if (h & 1) { set_error("edge list holds a vertex id outside [0, V)"); return TRAV_ERR_BAD_ARG; }
    if (h & 2) { set_error("edge list holds a negative weight (only weights >= 0 are supported)"); return TRAV_ERR_BAD_ARG; }
    if (h & 4) { set_error("edge list holds a NaN or infinite weight (weights must be finite)"); return TRAV_ERR_BAD_ARG; }
    return TRAV_OK;
}

void free_graph(DevGraph *g)
{
    cudaFree(g->out_off);
    cudaFree(g->out_adj);
    cudaFree(g->out_w);
    cudaFree(g->in_off);
    cudaFree(g->in_adj);
    cudaFree(g->in_w);
    cudaFree(g->new_of_old);
    cudaFree(g->old_of_new);
    *g = DevGraph{};
}

int build_graph_device(int32_t V, int64_t E, const int32_t *d_src, const int32_t *d_dst, const float *d_w,
                       cudaStream_t st, DevGraph *out)
{
    int rc = validate_edges(V, E, d_src, d_dst, d_w, st);
    if (rc) return rc;
    int lv = 1;
    while (lv < 31 && ((int64_t)1 << lv) < (int64_t)V) lv++;
    const unsigned long long mask = (1ull << lv) - 1ull;

    DBuf<int32_t> out_deg, in_deg, ids, deg_sorted, out_deg_new, in_deg_new;
    DBuf<int32_t> out_off, in_off, new_of_old, old_of_new, out_adj, in_adj;
    DBuf<float> out_w, in_w, iwt;
    DBuf<int32_t> dv;
    DBuf<unsigned long long> okeys, ikeys, skeys;
    TRY_CUDA(out_deg.alloc(V));
    TRY_CUDA(in_deg.alloc(V));
    TRY_CUDA(ids.alloc(V));
    TRY_CUDA(deg_sorted.alloc(V));
    TRY_CUDA(out_deg_new.alloc((int64_t)V + 1));
    TRY_CUDA(in_deg_new.alloc((int64_t)V + 1));
    TRY_CUDA(out_off.alloc((int64_t)V + 1));
    TRY_CUDA(in_off.alloc((int64_t)V + 1));
    TRY_CUDA(new_of_old.alloc(V));
    TRY_CUDA(old_of_new.alloc(V));
    TRY_CUDA(out_adj.alloc(E));
    TRY_CUDA(in_adj.alloc(E));
    TRY_CUDA(out_w.alloc(E));
    TRY_CUDA(in_w.alloc(E));

    TRY_CUDA(cudaMemsetAsync(out_deg.p, 0, sizeof(int32_t) * (size_t)V, st));
    TRY_CUDA(cudaMemsetAsync(in_deg.p, 0, sizeof(int32_t) * (size_t)V, st));
    if (E > 0) degree_kernel<<<grid_for(E), 256, 0, st>>>(E, d_src, d_dst, out_deg.p, in_deg.p);
    iota_kernel<<<grid_for(V), 256, 0, st>>>(ids.p, V);
    TRY_CUDA(cudaGetLastError());

    // Vertex order: out-degree descending, ties by id (the sort is stable).
    size_t tb = 0, tb2 = 0;
    TRY_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, out_deg.p, deg_sorted.p, ids.p, old_of_new.p,
                                                       (int)V, 0, 32, st));
    TRY_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, out_deg_new.p, out_off.p, (int)V + 1, st));
    size_t tb3 = 0, tb4 = 0;
    if (E > 0) {
        TRY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb3, (unsigned long long *)nullptr,
                                                 (unsigned long long *)nullptr, (int32_t *)nullptr, (int32_t *)nullptr,
                                                 (int)E, 0, 32 + lv, st));
        TRY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb4, (unsigned long long *)nullptr,
                                                 (unsigned long long *)nullptr, (float *)nullptr, (float *)nullptr,
                                                 (int)E, 0, 2 * lv, st));
    }
    size_t tmax = tb;
    if (tb2 > tmax) tmax = tb2;
    if (tb3 > tmax) tmax = tb3;
    if (tb4 > tmax) tmax = tb4;
    DBuf<unsigned char> temp;
    TRY_CUDA(temp.alloc((int64_t)tmax));
    TRY_CUDA(cub::DeviceRadixSort::SortPairsDescending(temp.p, tb, out_deg.p, deg_sorted.p, ids.p, old_of_new.p,
                                                       (int)V, 0, 32, st));
    relabel_kernel<<<grid_for((int64_t)V + 1), 256, 0, st>>>(V, old_of_new.p, out_deg.p, in_deg.p, new_of_old.p,
                                                             out_deg_new.p, in_deg_new.p);
    TRY_CUDA(cudaGetLastError());
    TRY_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb2, out_deg_new.p, out_off.p, (int)V + 1, st));
    TRY_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb2, in_deg_new.p, in_off.p, (int)V + 1, st));

    if (E > 0) {
        TRY_CUDA(okeys.alloc(E));
        TRY_CUDA(ikeys.alloc(E));
        TRY_CUDA(skeys.alloc(E));
        TRY_CUDA(dv.alloc(E));
        TRY_CUDA(iwt.alloc(E));
        edge_keys_kernel<<<grid_for(E), 256, 0, st>>>(E, lv, d_src, d_dst, new_of_old.p, d_w, okeys.p, ikeys.p, dv.p,
                                                      iwt.p);
        TRY_CUDA(cudaGetLastError());
        // Out rows by (new source, weight); stable, so equal weights keep
        // their edge-list order.
        TRY_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb3, okeys.p, skeys.p, dv.p, out_adj.p, (int)E, 0, 32 + lv, st));
        low_word_float_kernel<<<grid_for(E), 256, 0, st>>>(E, skeys.p, out_w.p);
        // In rows by (new target, new source), each in-edge with its weight.
        TRY_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb4, ikeys.p, skeys.p, iwt.p, in_w.p, (int)E, 0, 2 * lv, st));
        low_bits_kernel<<<grid_for(E), 256, 0, st>>>(E, mask, skeys.p, in_adj.p);
        TRY_CUDA(cudaGetLastError());
    }
    int32_t maxdeg = 0;
    if (V > 0) TRY_CUDA(cudaMemcpyAsync(&maxdeg, deg_sorted.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    double wsum = 0.0;
    if (E > 0) {
        DBuf<double> part;
        TRY_CUDA(part.alloc(kWSumBlocks));
        weight_sum_kernel<<<kWSumBlocks, 256, 0, st>>>(E, out_w.p, part.p);
        TRY_CUDA(cudaGetLastError());
        double h[kWSumBlocks];
        TRY_CUDA(cudaMemcpyAsync(h, part.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        TRY_CUDA(cudaStreamSynchronize(st));
        for (int b = 0; b < kWSumBlocks; b++) wsum += h[b];
    }
    TRY_CUDA(cudaStreamSynchronize(st));

    out->V = V;
    out->E = E;
    out->max_out_degree = maxdeg;
    out->mean_w = E > 0 ? (float)(wsum / (double)E) : 0.0f;
    out->out_off = out_off.release();
    out->out_adj = out_adj.release();
    out->out_w = out_w.release();
    out->in_off = in_off.release();
    out->in_adj = in_adj.release();
    out->in_w = in_w.release();
    out->new_of_old = new_of_old.release();
    out->old_of_new = old_of_new.release();
    return TRAV_OK;
}

}  // namespace trav
