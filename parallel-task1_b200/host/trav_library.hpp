// C++ host layer over the C ABI (include/trav.h), shaped like the reference
// library's host API for the traversal path so its sample programs port
// line for line:
//
//   GraphStorageAPI::load_from_edges_list_bin_file / save_to_edges_list_bin_file
//       include/storage/graph_storage_API.hpp:39-65, 114-160
//   GraphStorageAPI::load_from_adjacency_list_bin_file / save_to_adjacency_list_bin_file
//       include/storage/graph_storage_API.hpp:3-35, 69-111
//   read_data_from_file (headerless pairs)        sample/bfs.cpp:84-114
//   GraphGenerationAPI::R_MAT_parallel
//       include/test/generation/graph_generation_API.hpp:403-484
//   SingleSourceShortestPaths::gpu_bellman_ford   algorithm/sssp/sssp.hpp:219-277
//   BFS::gpu_bfs                                  algorithm/bfs/bfs.hpp:212-254
//
// Errors are thrown as `const char *`, as the reference's SAFE_CALL does
// (include/common/cuda_error_hadling.h:4-24), after printing the library's
// message.
#pragma once

#include <climits>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "trav.h"

namespace trav_host {

inline void check(int rc, const char *what)
{
    if (rc != TRAV_OK) {
        printf("trav error %d in %s: %s\n", rc, what, trav_last_error());
        throw "error in B200 traversal library call, aborting...";
    }
}

// Host edge list: the reference's EDGES_LIST container reduced to its arrays.
struct EdgesList {
    int vertices_count = 0;
    bool directed = true;
    std::vector<int32_t> src_ids, dst_ids;
    std::vector<float> weights;
    long long get_edges_count() const { return (long long)src_ids.size(); }
    int get_vertices_count() const { return vertices_count; }
};

struct GraphStorageAPI {
    static bool load_from_edges_list_bin_file(EdgesList &g, const std::string &file_name)
    {
        int32_t V = 0, directed = 1;
        int64_t E = 0;
        if (trav_el_file_read(file_name.c_str(), 0, &V, &E, &directed, nullptr, nullptr, nullptr) != TRAV_OK)
            return false;
        g.vertices_count = V;
        g.directed = directed != 0;
        g.src_ids.resize((size_t)E);
        g.dst_ids.resize((size_t)E);
        g.weights.resize((size_t)E);
        return trav_el_file_read(file_name.c_str(), 0, &V, &E, &directed, g.src_ids.data(), g.dst_ids.data(),
                                 g.weights.data()) == TRAV_OK;
    }

    static bool save_to_edges_list_bin_file(const EdgesList &g, const std::string &file_name)
    {
        return trav_el_file_write(file_name.c_str(), g.directed, g.vertices_count, g.get_edges_count(),
                                  g.src_ids.data(), g.dst_ids.data(), g.weights.data()) == TRAV_OK;
    }

    // Adjacency-list binary: rows in file order become edges grouped by
    // source (the order the reference's conversion to an edge list gives).
    static bool load_from_adjacency_list_bin_file(EdgesList &g, const std::string &file_name)
    {
        int32_t V = 0, directed = 1;
        int64_t E = 0;
        if (trav_adj_file_read(file_name.c_str(), &V, &E, &directed, nullptr, nullptr, nullptr, nullptr, nullptr) !=
            TRAV_OK)
            return false;
        std::vector<int32_t> ids((size_t)V), values((size_t)V), dst((size_t)E);
        std::vector<int64_t> off((size_t)V + 1);
        std::vector<float> w((size_t)E);
        if (trav_adj_file_read(file_name.c_str(), &V, &E, &directed, ids.data(), values.data(), off.data(), dst.data(),
                               w.data()) != TRAV_OK)
            return false;
        g.vertices_count = V;
        g.directed = directed != 0;
        g.src_ids.resize((size_t)E);
        for (int32_t v = 0; v < V; v++)
            for (int64_t e = off[(size_t)v]; e < off[(size_t)v + 1]; e++) g.src_ids[(size_t)e] = ids[(size_t)v];
        g.dst_ids = std::move(dst);
        g.weights = std::move(w);
        return true;
    }

    // Rows of vertices 0..V-1 (vertex values 0), each in edge-list order.
    static bool save_to_adjacency_list_bin_file(const EdgesList &g, const std::string &file_name)
    {
        const int32_t V = g.vertices_count;
        const int64_t E = g.get_edges_count();
        std::vector<int64_t> off((size_t)V + 1, 0);
        for (int64_t e = 0; e < E; e++) {
            const int32_t s = g.src_ids[(size_t)e];
            if (s < 0 || s >= V) return false;
            off[(size_t)s + 1]++;
        }
        for (int32_t v = 0; v < V; v++) off[(size_t)v + 1] += off[(size_t)v];
        std::vector<int64_t> at(off.begin(), off.end() - 1);
        std::vector<int32_t> dst((size_t)E), ids((size_t)V), values((size_t)V, 0);
        std::vector<float> w((size_t)E);
        for (int64_t e = 0; e < E; e++) {
            const int64_t k = at[(size_t)g.src_ids[(size_t)e]]++;
            dst[(size_t)k] = g.dst_ids[(size_t)e];
            w[(size_t)k] = g.weights[(size_t)e];
        }
        for (int32_t v = 0; v < V; v++) ids[(size_t)v] = v;
        return trav_adj_file_write(file_name.c_str(), g.directed, V, E, ids.data(), values.data(), off.data(),
                                   dst.data(), w.data()) == TRAV_OK;
    }

    // The BFS sample's headerless {int32, int32} pairs: V = 2^vertices_pow,
    // the first file_size / 12 pairs, weight 1.0 each.
    static bool read_data_from_file(EdgesList &g, const std::string &file_name, int vertices_pow)
    {
        int32_t V = 0;
        int64_t E = 0;
        if (trav_pairs_file_read(file_name.c_str(), vertices_pow, &V, &E, nullptr, nullptr, nullptr) != TRAV_OK)
            return false;
        g.vertices_count = V;
        g.directed = true;
        g.src_ids.resize((size_t)E);
        g.dst_ids.resize((size_t)E);
        g.weights.resize((size_t)E);
        return trav_pairs_file_read(file_name.c_str(), vertices_pow, &V, &E, g.src_ids.data(), g.dst_ids.data(),
                                    g.weights.data()) == TRAV_OK;
    }
};

// A graph resident on the GPU (int32 CSR + transposed CSR, degree-relabelled).
class DeviceGraph {
    trav_graph *h_ = nullptr;

public:
    explicit DeviceGraph(const EdgesList &g)
    {
        check(trav_graph_from_edges(g.vertices_count, g.get_edges_count(), g.src_ids.data(), g.dst_ids.data(),
                                    g.weights.data(), TRAV_MEM_HOST, &h_),
              "trav_graph_from_edges");
    }
    explicit DeviceGraph(trav_graph *h) : h_(h) {}
    DeviceGraph(const DeviceGraph &) = delete;
    DeviceGraph &operator=(const DeviceGraph &) = delete;
    ~DeviceGraph() { trav_graph_free(h_); }
    trav_graph *handle() const { return h_; }
    int get_vertices_count() const
    {
        int32_t V = 0;
        trav_graph_info(h_, &V, nullptr, nullptr);
        return V;
    }
    long long get_edges_count() const
    {
        int64_t E = 0;
        trav_graph_info(h_, nullptr, &E, nullptr);
        return E;
    }
};

struct GraphGenerationAPI {
    // RMAT as R_MAT_parallel, generated on the device from a seeded rand_r
    // stream (seed 0 reproduces the reference's single-thread output); the
    // edge list is copied into the host container.  `_omp_threads` is kept
    // for signature compatibility: the result does not depend on it.
    static void R_MAT_parallel(EdgesList &g, int vertices_count, int average_connections, int a_prob, int b_prob,
                               int c_prob, int d_prob, int /*omp_threads*/, bool directed, uint32_t seed = 0,
                               bool drop_self_loops = false)
    {
        if (!directed) throw "R_MAT_parallel: only directed graphs are generated";
        int scale = 0;
        while ((1 << scale) < vertices_count) scale++;
        if ((1 << scale) != vertices_count) throw "R_MAT_parallel: vertices_count must be a power of two";
        trav_graph *h = nullptr;
        int64_t E = 0;
        check(trav_graph_rmat(scale, average_connections, a_prob, b_prob, c_prob, d_prob, seed, drop_self_loops,
                              nullptr, nullptr, nullptr, &E, &h),
              "trav_graph_rmat");
        DeviceGraph dg(h);
        // the device keeps only the CSR; rebuild the edge list in CSR order
        int32_t V = vertices_count;
        std::vector<int32_t> n2o((size_t)V), off((size_t)V + 1), adj((size_t)E), o2n((size_t)V);
        std::vector<float> w((size_t)E);
        check(trav_graph_export(h, n2o.data(), o2n.data(), off.data(), adj.data(), w.data(), nullptr, nullptr),
              "trav_graph_export");
        g.vertices_count = V;
        g.directed = true;
        g.src_ids.resize((size_t)E);
        g.dst_ids.resize((size_t)E);
        g.weights = w;
        for (int32_t r = 0; r < V; r++)
            for (int32_t k = off[(size_t)r]; k < off[(size_t)r + 1]; k++) {
                g.src_ids[(size_t)k] = o2n[(size_t)r];
                g.dst_ids[(size_t)k] = o2n[(size_t)adj[(size_t)k]];
            }
    }
};

// GraphOptimizationAPI::optimize_graph_for_GPU and
// check_gpu_memory_transactions_count
// (include/test/optimization/graph_optimization_API.hpp:173-266), run on the
// device: loops and repeated arcs are removed and edges grouped by segments of
// l2_bytes / elem_size vertices (the B200's 126 MB L2 by default, where the
// reference names Kepler's or Pascal's).
struct GraphOptimizationAPI {
    static constexpr long long kB200L2Bytes = 126LL * 1024 * 1024;

    static void optimize_graph_for_GPU(EdgesList &g, int elem_size, long long l2_bytes = kB200L2Bytes)
    {
        int64_t n = 0;
        const long long seg = l2_bytes / (elem_size > 0 ? elem_size : 1);
        check(trav_el_optimize(g.src_ids.data(), g.dst_ids.data(), g.weights.data(), g.vertices_count,
                               g.get_edges_count(), (int32_t)(seg < INT32_MAX ? seg : INT32_MAX), TRAV_MEM_HOST, &n),
              "trav_el_optimize");
        g.src_ids.resize((size_t)n);
        g.dst_ids.resize((size_t)n);
        g.weights.resize((size_t)n);
    }

    static long long check_gpu_memory_transactions_count(const EdgesList &g, int elem_size)
    {
        int64_t n = 0;
        check(trav_el_gpu_transactions(g.src_ids.data(), g.dst_ids.data(), g.vertices_count, g.get_edges_count(),
                                       elem_size, TRAV_MEM_HOST, &n),
              "trav_el_gpu_transactions");
        return (long long)n;
    }
};

template <typename _TVertexValue, typename _TEdgeWeight>
class SingleSourceShortestPaths {
public:
    // Bellman-Ford (delta <= 0) or delta-stepping (delta > 0) from one source;
    // distances in the caller's ids, FLT_MAX unreachable.  Returns MTEPS =
    // E / kernel time, as gpu_bellman_ford does.
    double gpu_bellman_ford(DeviceGraph &g, _TEdgeWeight *distances, int source_vertex, float delta = 0.0f)
    {
        static_assert(sizeof(_TEdgeWeight) == 4, "the B200 library computes in fp32");
        trav_sssp_opts o{TRAV_SCHEDULE_PLAIN, delta};
        int32_t s = source_vertex;
        check(trav_sssp(g.handle(), &s, 1, &o, reinterpret_cast<float *>(distances), TRAV_MEM_HOST), "trav_sssp");
        trav_query_stats st;
        check(trav_last_stats(g.handle(), &st), "trav_last_stats");
        return (double)g.get_edges_count() / ((double)st.kernel_ms * 1e3);
    }
};

template <typename _TVertexValue, typename _TEdgeWeight>
class BFS {
public:
    // Reachability into a bool array (as BFS::gpu_bfs); returns MTEPS.
    double gpu_bfs(DeviceGraph &g, bool *result, int source_vertex)
    {
        std::vector<int32_t> lv((size_t)g.get_vertices_count());
        double mteps = gpu_bfs_levels(g, lv.data(), source_vertex);
        for (size_t i = 0; i < lv.size(); i++) result[i] = lv[i] >= 0;
        return mteps;
    }

    // Hop levels, -1 unreachable (Beamer alpha 15 / beta 18 direction switch).
    double gpu_bfs_levels(DeviceGraph &g, int32_t *levels, int source_vertex, float alpha = 15.0f, float beta = 18.0f)
    {
        trav_bfs_opts o{TRAV_SCHEDULE_PLAIN, alpha, beta, -1};
        int32_t s = source_vertex;
        check(trav_bfs(g.handle(), &s, 1, &o, levels, TRAV_MEM_HOST), "trav_bfs");
        trav_query_stats st;
        check(trav_last_stats(g.handle(), &st), "trav_last_stats");
        return (double)g.get_edges_count() / ((double)st.kernel_ms * 1e3);
    }
};

}  // namespace trav_host
