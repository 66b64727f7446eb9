// The reference's C++ CUDA-wrapper entry points (include/trav_reference.h),
// implemented on the C ABI so the reference's own callers link unchanged.
#include <cstdio>

#include "trav.h"
#include "trav_reference.h"

namespace {

[[noreturn]] void fail(const char *what)
{
    printf("CUDA error: %s at call \"%s\"\n", trav_last_error(), what);
    throw "error in CUDA kernel execution, aborting...";
}

[[noreturn]] void no_double(const char *what)
{
    printf("error: %s: double-precision weights are not supported by the B200 traversal library (fp32 only)\n", what);
    throw "error in CUDA kernel execution, aborting...";
}

void init_impl(float *d, int V, int s)
{
    if (trav_init_distances_f32(d, V, s) != TRAV_OK) fail("init_distances_wrapper");
}
void init_impl(double *, int, int) { no_double("init_distances_wrapper<double>"); }

void bf_impl(int *src, int *dst, float *w, int V, long long E, int s, float *d)
{
    if (trav_bellman_ford_el_f32(src, dst, w, V, E, s, d) != TRAV_OK) fail("bellman_ford_wrapper");
}
void bf_impl(int *, int *, double *, int, long long, int, double *) { no_double("bellman_ford_wrapper<double>"); }

}  // namespace

template <typename _TEdgeWeight>
void init_distances_wrapper(_TEdgeWeight *_distances, int _vertices_count, int _source_vertex)
{
    init_impl(_distances, _vertices_count, _source_vertex);
}

template <typename _TEdgeWeight>
void bellman_ford_wrapper(int *_src_ids, int *_dst_ids, _TEdgeWeight *_weights, int _vertices_count,
                          long long _edges_count, int _source_vertex, _TEdgeWeight *_distances)
{
    bf_impl(_src_ids, _dst_ids, _weights, _vertices_count, _edges_count, _source_vertex, _distances);
}

void bfs_wrapper(int *_src_ids, int *_dst_ids, int _vertices_count, long long _edges_count, bool *_visited,
                 int _source_vertex)
{
    static_assert(sizeof(bool) == 1, "bool must be one byte");
    if (trav_bfs_el(_src_ids, _dst_ids, _vertices_count, _edges_count, reinterpret_cast<uint8_t *>(_visited),
                    _source_vertex) != TRAV_OK)
        fail("bfs_wrapper");
}

template void init_distances_wrapper<float>(float *, int, int);
template void init_distances_wrapper<double>(double *, int, int);
template void bellman_ford_wrapper<float>(int *, int *, float *, int, long long, int, float *);
template void bellman_ford_wrapper<double>(int *, int *, double *, int, long long, int, double *);
