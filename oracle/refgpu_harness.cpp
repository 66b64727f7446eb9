// Test and baseline infrastructure, not product code.
//
// The reference library's own GPU path -- init_distances_wrapper<float> and
// bellman_ford_wrapper<float> (algorithm/sssp/gpu/bellman_ford.cu:38-144) and
// bfs_wrapper (algorithm/bfs/gpu/bfs.cu:43-81) -- compiled unchanged from its
// sources for sm_100a by oracle/build_refgpu.sh and driven here on an edge
// list kept resident in device memory, the way gpu_bellman_ford
// (algorithm/sssp/sssp.hpp:219-277) and gpu_bfs (algorithm/bfs/bfs.hpp:
// 212-254) call them.  Each call is timed as the reference times it: host
// clock (omp_get_wtime) around the wrappers only, uploads excluded
// (sssp.hpp:255-262, bfs.hpp:241-243).  bench.py reports it as the secondary
// GPU baseline; tests/test_gpu_refgpu.py checks its results.
#include <cstdint>
#include <omp.h>
#include <cuda_runtime.h>

template <typename _TEdgeWeight>
void init_distances_wrapper(_TEdgeWeight *_distances, int _vertices_count, int _source_vertex);
template <typename _TEdgeWeight>
void bellman_ford_wrapper(int *_src_ids, int *_dst_ids, _TEdgeWeight *_weights, int _vertices_count,
                          long long _edges_count, int _source_vertex, _TEdgeWeight *_distances);
void bfs_wrapper(int *_src_ids, int *_dst_ids, int _vertices_count, long long _edges_count, bool *_visited,
                 int _source_vertex);

namespace {
int *g_src = nullptr, *g_dst = nullptr;
float *g_w = nullptr, *g_dist = nullptr;
bool *g_vis = nullptr;
int g_V = 0;
long long g_E = 0;
}  // namespace

extern "C" {

void refgpu_free(void)
{
    cudaFree(g_src);
    cudaFree(g_dst);
    cudaFree(g_w);
    cudaFree(g_dist);
    cudaFree(g_vis);
    g_src = g_dst = nullptr;
    g_w = g_dist = nullptr;
    g_vis = nullptr;
    g_V = 0;
    g_E = 0;
}

// Upload an edge list (host arrays) once; 0 on success.
int refgpu_upload(int V, long long E, const int *src, const int *dst, const float *w)
{
    refgpu_free();
    if (cudaMalloc(&g_src, sizeof(int) * E) != cudaSuccess || cudaMalloc(&g_dst, sizeof(int) * E) != cudaSuccess ||
        cudaMalloc(&g_w, sizeof(float) * E) != cudaSuccess || cudaMalloc(&g_dist, sizeof(float) * V) != cudaSuccess ||
        cudaMalloc(&g_vis, sizeof(bool) * V) != cudaSuccess) {
        refgpu_free();
        return -1;
    }
    if (cudaMemcpy(g_src, src, sizeof(int) * E, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g_dst, dst, sizeof(int) * E, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g_w, w, sizeof(float) * E, cudaMemcpyHostToDevice) != cudaSuccess) {
        refgpu_free();
        return -1;
    }
    g_V = V;
    g_E = E;
    return 0;
}

// The reference's SSSP on the resident edge list; distances to dist (host).
// Returns the seconds between the wrappers' start and the device's finish,
// or -1 when a wrapper threw.
double refgpu_sssp(int source, float *dist)
{
    try {
        cudaDeviceSynchronize();
        const double t0 = omp_get_wtime();
        init_distances_wrapper<float>(g_dist, g_V, source);
        bellman_ford_wrapper<float>(g_src, g_dst, g_w, g_V, g_E, source, g_dist);
        cudaDeviceSynchronize();
        const double t1 = omp_get_wtime();
        if (cudaMemcpy(dist, g_dist, sizeof(float) * g_V, cudaMemcpyDeviceToHost) != cudaSuccess) return -1.0;
        return t1 - t0;
    } catch (const char *) {
        return -1.0;
    }
}

// The reference's BFS (reachability) on the resident edge list.
double refgpu_bfs(int source, unsigned char *visited)
{
    try {
        cudaDeviceSynchronize();
        const double t0 = omp_get_wtime();
        bfs_wrapper(g_src, g_dst, g_V, g_E, g_vis, source);
        cudaDeviceSynchronize();
        const double t1 = omp_get_wtime();
        if (cudaMemcpy(visited, g_vis, g_V, cudaMemcpyDeviceToHost) != cudaSuccess) return -1.0;
        return t1 - t0;
    } catch (const char *) {
        return -1.0;
    }
}

}  // extern "C"
