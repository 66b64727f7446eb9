// Graph optimisation pass on a device edge list, and the memory-transaction
// count of an edge-per-thread sweep: the GPU forms of GraphOptimizationAPI
// (include/test/optimization/graph_optimization_API.hpp).
//
//   reorder_edges_in_adjacency_list_format :14-55   sort by (src, dst, weight)
//   remove_loops_and_multiple_arcs          :60-117  drop loops and repeated arcs (the lightest arc stays)
//   reorder_edges_for_cache                 :122-166 group by (src / segment, dst / segment)
//   check_gpu_memory_transactions_count     :229-266 distinct 128-byte segments per warp of 32 edges
//
// The sorts are stable radix sorts (weight bits, then the 64-bit (src, dst)
// key, then the segment key), so the order inside a segment pair -- which the
// reference's std::sort leaves unspecified -- is the (src, dst, weight) order.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cstdint>

#include "trav_internal.cuh"

namespace trav {
namespace {

#define TRY_CUDA(expr)                                      \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

template <class T>
struct Buf {
    T *p = nullptr;
    cudaError_t alloc(int64_t n) { return dev_malloc((void **)&p, sizeof(T) * (size_t)(n > 0 ? n : 1)); }
    ~Buf() { if (p) cudaFree(p); }
};

int grid_of(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 65535); }

// weight bits with -0.0 read as +0.0 (non-negative floats order like their bits), and the identity permutation
__global__ void weight_keys_kernel(int64_t E, const float *__restrict__ w, unsigned *__restrict__ key,
                                   int32_t *__restrict__ idx)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = w[i];
        key[i] = x == 0.0f ? 0u : __float_as_uint(x);
        idx[i] = (int32_t)i;
    }
}

// (src, dst) of the permuted edges as one 64-bit key
__global__ void pair_keys_kernel(int64_t E, const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                                 const int32_t *__restrict__ idx, unsigned long long *__restrict__ key)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t e = idx[i];
        key[i] = ((unsigned long long)(unsigned)src[e] << 32) | (unsigned)dst[e];
    }
}

// (src / segment, dst / segment) as one 64-bit key, identity permutation
__global__ void segment_keys_kernel(int64_t E, const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                                    int32_t segment, unsigned long long *__restrict__ key, int32_t *__restrict__ idx)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        key[i] = ((unsigned long long)(unsigned)(src[i] / segment) << 32) | (unsigned)(dst[i] / segment);
        idx[i] = (int32_t)i;
    }
}

__global__ void gather_kernel(int64_t E, const int32_t *__restrict__ idx, const int32_t *__restrict__ src,
                              const int32_t *__restrict__ dst, const float *__restrict__ w, int32_t *__restrict__ os,
                              int32_t *__restrict__ od, float *__restrict__ ow)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t e = idx[i];
        os[i] = src[e];
        od[i] = dst[e];
        const float x = w[e];
        ow[i] = x == 0.0f ? 0.0f : x;
    }
}

// keep an edge unless it is a loop or repeats the previous sorted edge's (src, dst)
__global__ void keep_kernel(int64_t E, const int32_t *__restrict__ s, const int32_t *__restrict__ d,
                            unsigned char *__restrict__ keep)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        bool k = s[i] != d[i];
        if (k && i > 0 && s[i] == s[i - 1] && d[i] == d[i - 1]) k = false;
        keep[i] = k ? 1 : 0;
    }
}

// One warp per 32 consecutive edges of the counted warps: the distinct
// 128-byte segments among the warp's src * elem and among its dst * elem.
__global__ void transactions_kernel(int64_t warps, const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                                    int32_t elem, unsigned long long *__restrict__ total)
{
    const unsigned lane = threadIdx.x & 31;
    unsigned long long acc = 0;
    for (int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < warps;
         k += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t i = 32 * k + lane;
        const unsigned long long a = (unsigned long long)((int64_t)src[i] * elem / 128);
        const unsigned long long b = (unsigned long long)((int64_t)dst[i] * elem / 128);
        const unsigned ma = __match_any_sync(0xffffffffu, a), mb = __match_any_sync(0xffffffffu, b);
        // a lane leads its group when no lower lane holds the same segment
        const unsigned lower = (1u << lane) - 1u;
        acc += ((ma & lower) == 0u ? 1u : 0u) + ((mb & lower) == 0u ? 1u : 0u);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0 && acc) atomicAdd(total, acc);
}

}  // namespace

int el_optimize_device(int32_t *src, int32_t *dst, float *w, int64_t E, int32_t segment, int64_t *E_out,
                       cudaStream_t st)
{
    *E_out = 0;
    if (E == 0) return TRAV_OK;
    Buf<unsigned> wkey, wkey2;
    Buf<int32_t> idx, idx2;
    Buf<unsigned long long> key, key2;
    Buf<int32_t> s2, d2;
    Buf<float> w2;
    Buf<unsigned char> keep;
    Buf<int64_t> nsel;
    TRY_CUDA(wkey.alloc(E));
    TRY_CUDA(wkey2.alloc(E));
    TRY_CUDA(idx.alloc(E));
    TRY_CUDA(idx2.alloc(E));
    TRY_CUDA(key.alloc(E));
    TRY_CUDA(key2.alloc(E));
    TRY_CUDA(s2.alloc(E));
    TRY_CUDA(d2.alloc(E));
    TRY_CUDA(w2.alloc(E));
    TRY_CUDA(keep.alloc(E));
    TRY_CUDA(nsel.alloc(1));
    const int n = (int)E;
    size_t tb = 0, t1 = 0;
    TRY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, wkey.p, wkey2.p, idx.p, idx2.p, n, 0, 32, st));
    tb = t1;
    TRY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, key.p, key2.p, idx2.p, idx.p, n, 0, 64, st));
    tb = std::max(tb, t1);
    TRY_CUDA(cub::DeviceSelect::Flagged(nullptr, t1, s2.p, keep.p, src, nsel.p, n, st));
    tb = std::max(tb, t1);
    Buf<unsigned char> temp;
    TRY_CUDA(temp.alloc((int64_t)tb));

    // (src, dst, weight) order: weight first, then a stable sort by (src, dst)
    weight_keys_kernel<<<grid_of(E), 256, 0, st>>>(E, w, wkey.p, idx.p);
    TRY_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb, wkey.p, wkey2.p, idx.p, idx2.p, n, 0, 32, st));
    pair_keys_kernel<<<grid_of(E), 256, 0, st>>>(E, src, dst, idx2.p, key.p);
    TRY_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb, key.p, key2.p, idx2.p, idx.p, n, 0, 64, st));
    gather_kernel<<<grid_of(E), 256, 0, st>>>(E, idx.p, src, dst, w, s2.p, d2.p, w2.p);
    keep_kernel<<<grid_of(E), 256, 0, st>>>(E, s2.p, d2.p, keep.p);
    TRY_CUDA(cudaGetLastError());
    TRY_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, s2.p, keep.p, src, nsel.p, n, st));
    TRY_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, d2.p, keep.p, dst, nsel.p, n, st));
    TRY_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, w2.p, keep.p, w, nsel.p, n, st));
    int64_t kept = 0;
    TRY_CUDA(cudaMemcpyAsync(&kept, nsel.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TRY_CUDA(cudaStreamSynchronize(st));
    if (segment > 0 && kept > 0) {
        segment_keys_kernel<<<grid_of(kept), 256, 0, st>>>(kept, src, dst, segment, key.p, idx.p);
        TRY_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb, key.p, key2.p, idx.p, idx2.p, (int)kept, 0, 64, st));
        gather_kernel<<<grid_of(kept), 256, 0, st>>>(kept, idx2.p, src, dst, w, s2.p, d2.p, w2.p);
        TRY_CUDA(cudaGetLastError());
        TRY_CUDA(cudaMemcpyAsync(src, s2.p, sizeof(int32_t) * (size_t)kept, cudaMemcpyDeviceToDevice, st));
        TRY_CUDA(cudaMemcpyAsync(dst, d2.p, sizeof(int32_t) * (size_t)kept, cudaMemcpyDeviceToDevice, st));
        TRY_CUDA(cudaMemcpyAsync(w, w2.p, sizeof(float) * (size_t)kept, cudaMemcpyDeviceToDevice, st));
        TRY_CUDA(cudaStreamSynchronize(st));
    }
    *E_out = kept;
    return TRAV_OK;
}

int el_transactions_device(const int32_t *src, const int32_t *dst, int64_t E, int32_t elem, int64_t *count,
                           cudaStream_t st)
{
    const int64_t warps = E > 0 ? (E - 1) / 32 : 0;  // the warp holding the last edge is not counted
    Buf<unsigned long long> tot;
    TRY_CUDA(tot.alloc(1));
    TRY_CUDA(cudaMemsetAsync(tot.p, 0, sizeof(unsigned long long), st));
    if (warps > 0) {
        transactions_kernel<<<(int)std::min<int64_t>((warps + 7) / 8, 65535), 256, 0, st>>>(warps, src, dst, elem,
                                                                                             tot.p);
        TRY_CUDA(cudaGetLastError());
    }
    unsigned long long h = 0;
    TRY_CUDA(cudaMemcpyAsync(&h, tot.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    TRY_CUDA(cudaStreamSynchronize(st));
    *count = (int64_t)h;
    return TRAV_OK;
}

}  // namespace trav
