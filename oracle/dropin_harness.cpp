// Test infrastructure, not product code.
//
// The reference library's own GPU callers of the traversal path, compiled
// unchanged from its headers where they lie and linked against
// libtrav_b200.so instead of the reference's bellman_ford.cu / bfs.cu.  The
// wrapper declarations they include (algorithm/sssp/gpu/bellman_ford.cuh:13-18,
// algorithm/bfs/gpu/bfs.cuh:10) resolve to the library's definitions of the
// same symbols.  oracle/build_dropin.sh builds it into
// oracle/_ref/libtrav_dropin.so; tests/test_gpu_dropin.py calls it and checks
// its results against the reference's CPU implementations.
//
// Callers driven here (reference file:line):
//   SingleSourceShortestPaths::gpu_bellman_ford  algorithm/sssp/sssp.hpp:219-277
//   BFS::gpu_bfs                                 algorithm/bfs/bfs.hpp:212-254
//   TransitiveClosure::allocate_and_copy_device_arrays / gpu_bfs / free_device_arrays
//                                                algorithm/transitive_closure/transitive_closure.hpp:20-70
// The TransitiveClosure members are private in the reference; the harness
// opens them with a preprocessor switch around the reference's headers, which
// changes no code the callers run.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <queue>
#include <set>
#include <stack>
#include <string>
#include <vector>
#include <omp.h>
#include <cuda_runtime.h>

// Everything include/graph_library.h pulls in, in its order, except the
// transitive closure, whose header is then read with its private members
// opened (its header has no other use of the word); the umbrella header
// itself adds nothing more after that (every header is #pragma once).
#include "include/architectures.h"
#include "include/knl_data.h"
#include "include/graph_data_structures/graph.h"
#include "include/common/file_system.h"
#include "include/visualization/graph_visualization_API.h"
#include "include/test/generation/graph_generation_API.h"
#include "include/test/optimization/graph_optimization_API.h"
#include "include/storage/graph_storage_API.h"
#include "include/node_data/node_data.h"
#include "algorithm/sssp/sssp.h"
#include "algorithm/bfs/bfs.h"
#include "algorithm/scc/scc.h"
#include "algorithm/mst/mst.h"
#define private public
#include "algorithm/transitive_closure/transitive_closure.h"
#undef private
#include "include/graph_library.h"

typedef Graph<int, float> RefGraph;

namespace {

RefGraph *edges_list(int V, long long E, const int *src, const int *dst, const float *w)
{
    RefGraph *g = new RefGraph(V, E, EDGES_LIST, true, false);
    GraphContainerData<int, float> d = g->get_graph_data();
    if (E > 0) {
        memcpy(d.edges_src_ids, src, sizeof(int) * E);
        memcpy(d.edges_dst_ids, dst, sizeof(int) * E);
        memcpy(d.edges_weights, w, sizeof(float) * E);
    }
    return g;
}

}  // namespace

extern "C" {

// SingleSourceShortestPaths<int, float>::gpu_bellman_ford on an edge list;
// returns its MTEPS figure, or -1 when it threw (the message is printed).
double dropin_gpu_bellman_ford(int V, long long E, const int *src, const int *dst, const float *w, int source,
                               float *dist)
{
    RefGraph *g = edges_list(V, E, src, dst, w);
    double mteps = -1.0;
    try {
        SingleSourceShortestPaths<int, float> op(1);
        mteps = op.gpu_bellman_ford(*g, dist, source);
    } catch (const char *e) {
        std::cout << "gpu_bellman_ford threw: " << e << std::endl;
        mteps = -1.0;
    }
    delete g;
    return mteps;
}

// BFS<int, float>::gpu_bfs: reachability into visited[V] (C++ bool bytes).
int dropin_gpu_bfs(int V, long long E, const int *src, const int *dst, int source, unsigned char *visited)
{
    std::vector<float> w((size_t)(E > 0 ? E : 1), 1.0f);
    RefGraph *g = edges_list(V, E, src, dst, w.data());
    int rc = 0;
    try {
        BFS<int, float> op(1);
        op.gpu_bfs(*g, reinterpret_cast<bool *>(visited), source);
    } catch (const char *e) {
        std::cout << "gpu_bfs threw: " << e << std::endl;
        rc = -1;
    }
    delete g;
    return rc;
}

// TransitiveClosure<int, float>'s GPU reachability (the bfs_wrapper caller at
// transitive_closure.hpp:50), with its device-array setup and teardown, for
// each of n sources: visited[q * V + v].
int dropin_tc_gpu_bfs(int V, long long E, const int *src, const int *dst, const int *sources, int n,
                      unsigned char *visited)
{
    std::vector<float> w((size_t)(E > 0 ? E : 1), 1.0f);
    RefGraph *g = edges_list(V, E, src, dst, w.data());
    int rc = 0;
    try {
        TransitiveClosure<int, float> tc(1);
        tc.allocate_and_copy_device_arrays(*g);
        for (int q = 0; q < n; q++) tc.gpu_bfs(*g, reinterpret_cast<bool *>(visited) + (size_t)q * V, sources[q]);
        tc.free_device_arrays();
    } catch (const char *e) {
        std::cout << "TransitiveClosure::gpu_bfs threw: " << e << std::endl;
        rc = -1;
    }
    delete g;
    return rc;
}

}  // extern "C"
