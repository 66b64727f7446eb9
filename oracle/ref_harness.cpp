// Test infrastructure, not product code.
//
// C-linkage harness around the reference library's own CPU implementations of
// the traversal path.  It is compiled by oracle/build_ref.sh directly against
// the reference headers where they lie (nothing from the reference is copied
// into this repository) into oracle/_ref/libtrav_ref.so.  Tests use it to pin
// the C restatement in oracle/trav_oracle.c, the golden-fixture script uses it
// to produce tests/golden/*, and bench.py's reference arm times it.
//
// Functions wrapped (reference file:line):
//   SingleSourceShortestPaths::cpu_bellman_ford   algorithm/sssp/sssp.hpp:3-71
//   BFS::cpu_sequential_bfs                       algorithm/bfs/bfs.hpp:3-46
//   BFS::cpu_parallel_bfs                         algorithm/bfs/bfs.hpp:117-208
//   GraphGenerationAPI::R_MAT_parallel            include/test/generation/graph_generation_API.hpp:403-484
//   GraphStorageAPI::{save,load}_*_bin_file       include/storage/graph_storage_API.hpp:3-160
//   Graph::convert_to_edges_list                  include/graph_data_structures/graph.hpp:366-401
//   Graph::convert_to_compressed_adjacency_list   include/graph_data_structures/graph.hpp:316-361
//   GraphOptimizationAPI::optimize_graph_for_CPU  include/test/optimization/graph_optimization_API.hpp:173-224
//   GraphOptimizationAPI::check_gpu_memory_transactions_count                             :229-266
#include <cstdint>
#include <cstring>
#include <cfloat>
#include <algorithm>
#include <vector>
#include <string>
#include <omp.h>

#include "include/graph_data_structures/graph.h"
#include "include/common/file_system.h"
#include "include/test/generation/graph_generation_API.h"
#include "include/storage/graph_storage_API.h"
#include "algorithm/sssp/sssp.h"
#include "algorithm/bfs/bfs.h"
#include "include/test/optimization/graph_optimization_API.h"

typedef Graph<int, float> RefGraph;

extern "C" {

// Edge-list graph (the container cpu_bellman_ford works on).
void *ref_graph_el(int V, long long E, const int *src, const int *dst, const float *w)
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

// Compressed-adjacency-list graph produced by the reference's own conversion
// (EL -> adjacency list -> CSR).  Slow on large graphs; used for fixtures.
void *ref_graph_csr_via_reference(int V, long long E, const int *src, const int *dst, const float *w)
{
    RefGraph *g = (RefGraph *)ref_graph_el(V, E, src, dst, w);
    g->convert_to_compressed_adjacency_list();
    return g;
}

// Compressed-adjacency-list graph filled through the container's add_vertex
// API from an already-built CSR (row order as given).  Used when the
// reference's own EL->CSR conversion would dominate a timing run.
void *ref_graph_csr(int V, long long E, const long long *offsets, const int *adj, const float *w)
{
    RefGraph *g = new RefGraph(V, E, COMPRESSED_ADJACENCY_LIST, true, true);
    std::vector<int> ids;
    std::vector<float> ws;
    for (int v = 0; v < V; v++) {
        long long b = offsets[v], e = offsets[v + 1];
        ids.assign(adj + b, adj + e);
        ws.assign(w + b, w + e);
        g->add_vertex(v, 0, ids, ws);
    }
    return g;
}

// Export the CSR of a compressed-adjacency-list graph (offsets V+1, adj E, w E).
int ref_graph_export_csr(void *h, long long *offsets, int *adj, float *w)
{
    RefGraph *g = (RefGraph *)h;
    if (g->get_container_type() != COMPRESSED_ADJACENCY_LIST) return -1;
    GraphContainerData<int, float> d = g->get_graph_data();
    int V = g->get_vertices_count();
    long long E = g->get_edges_count();
    memcpy(offsets, d.vertices_to_edges_ptrs, sizeof(long long) * (V + 1));
    if (E > 0) {
        memcpy(adj, d.edges_dst_ids, sizeof(int) * E);
        memcpy(w, d.edges_weights, sizeof(float) * E);
    }
    return 0;
}

int ref_graph_vertices(void *h) { return ((RefGraph *)h)->get_vertices_count(); }
long long ref_graph_edges(void *h) { return ((RefGraph *)h)->get_edges_count(); }
void ref_graph_free(void *h) { delete (RefGraph *)h; }

int ref_cpu_bellman_ford(void *h, int source, float *dist, int threads)
{
    try {
        SingleSourceShortestPaths<int, float> op(threads);
        op.cpu_bellman_ford(*(RefGraph *)h, dist, source);
    } catch (const char *) { return -1; }
    return 0;
}

int ref_cpu_sequential_bfs(void *h, int source, unsigned char *visited)
{
    try {
        BFS<int, float> op(1);
        op.cpu_sequential_bfs(*(RefGraph *)h, (bool *)visited, source);
    } catch (const char *) { return -1; }
    return 0;
}

// cpu_parallel_bfs sizes its team with omp_get_max_threads()
// (algorithm/bfs/bfs.hpp:142), so the thread count is set through the OpenMP ICV.
int ref_cpu_parallel_bfs(void *h, int source, unsigned char *visited, int threads)
{
    try {
        if (threads > 0) omp_set_num_threads(threads);
        BFS<int, float> op(threads > 0 ? threads : 1);
        op.cpu_parallel_bfs(*(RefGraph *)h, (bool *)visited, source);
    } catch (const char *) { return -1; }
    return 0;
}

// R_MAT_parallel writes into a fresh EL graph; copy its arrays out.
// With threads == 1 the reference seeds rand_r with 0 (time * thread 0).
int ref_rmat_parallel(int V, int avg, int a, int b, int c, int d, int threads,
                      int *src, int *dst, float *w)
{
    RefGraph g(0, 0, EDGES_LIST, true);
    GraphGenerationAPI<int, float>::R_MAT_parallel(g, V, avg, a, b, c, d, threads, true);
    GraphContainerData<int, float> gd = g.get_graph_data();
    long long E = g.get_edges_count();
    memcpy(src, gd.edges_src_ids, sizeof(int) * E);
    memcpy(dst, gd.edges_dst_ids, sizeof(int) * E);
    memcpy(w, gd.edges_weights, sizeof(float) * E);
    return 0;
}

int ref_save_edges_list(void *h, const char *path)
{
    return GraphStorageAPI<int, float>::save_to_edges_list_bin_file(*(RefGraph *)h, std::string(path)) ? 0 : -1;
}

int ref_save_adjacency_list(void *h, const char *path)
{
    return GraphStorageAPI<int, float>::save_to_adjacency_list_bin_file(*(RefGraph *)h, std::string(path)) ? 0 : -1;
}

// Load an EL binary through the reference loader into an EL graph handle.
void *ref_load_edges_list(const char *path)
{
    RefGraph *g = new RefGraph(0, 0, EDGES_LIST, true);
    if (!GraphStorageAPI<int, float>::load_from_edges_list_bin_file(*g, std::string(path))) {
        delete g;
        return nullptr;
    }
    return g;
}

// Load an adjacency-list binary through the reference loader
// (load_from_adjacency_list_bin_file, graph_storage_API.hpp:69-111) into an
// adjacency-list graph, then convert it to an edge list the reference's way
// (Graph::convert_to_edges_list, graph.hpp:366-401).
void *ref_load_adjacency_list_as_el(const char *path)
{
    RefGraph *g = new RefGraph(0, 0, ADJACENCY_LIST, true);
    try {
        if (!GraphStorageAPI<int, float>::load_from_adjacency_list_bin_file(*g, std::string(path))) {
            delete g;
            return nullptr;
        }
        g->convert_to_edges_list();
    } catch (const char *) {
        delete g;
        return nullptr;
    }
    return g;
}

int ref_graph_export_el(void *h, int *src, int *dst, float *w)
{
    RefGraph *g = (RefGraph *)h;
    if (g->get_container_type() != EDGES_LIST) return -1;
    GraphContainerData<int, float> d = g->get_graph_data();
    long long E = g->get_edges_count();
    memcpy(src, d.edges_src_ids, sizeof(int) * E);
    memcpy(dst, d.edges_dst_ids, sizeof(int) * E);
    memcpy(w, d.edges_weights, sizeof(float) * E);
    return 0;
}

double ref_wtime(void) { return omp_get_wtime(); }

// The reference's CPU optimisation pass on an edge-list graph, in place
// (loops and repeated arcs removed, edges grouped by CPU_L2_CACHE_SIZE /
// elem_size vertex segments).  Returns the new edge count.
long long ref_optimize_for_cpu(void *h, int elem_size)
{
    RefGraph *g = (RefGraph *)h;
    GraphOptimizationAPI<int, float>::optimize_graph_for_CPU(*g, elem_size);
    return g->get_edges_count();
}

long long ref_gpu_transactions(void *h, int elem_size)
{
    return GraphOptimizationAPI<int, float>::check_gpu_memory_transactions_count(*(RefGraph *)h, elem_size);
}

}  // extern "C"
