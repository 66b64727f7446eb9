// SSSP sample on the B200 library: the counterpart of the reference's
// sample/sssp.cpp (argv[1] = edge-list binary file in the reference format).
// Loads the graph, uploads it once, then runs SSSP from pseudo-random sources
// as the reference's loop does (sample/sssp.cpp:117-120), printing the
// GPU-only performance of each run like gpu_bellman_ford (sssp.hpp:274).
//
//   sssp <graph.el> [sources=10] [delta=0 (Bellman-Ford)] [out.bin]
//
// With out.bin, each run appends its int32 source and the V float distances
// (caller ids, FLT_MAX unreachable) to that file.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "host/trav_library.hpp"

using namespace trav_host;

int main(int argc, char *argv[])
{
    try {
        if (argc < 2) {
            printf("usage: %s <graph.el> [sources] [delta]\n", argv[0]);
            return 1;
        }
        std::string file_name = argv[1];
        int runs = argc > 2 ? atoi(argv[2]) : 10;
        float delta = argc > 3 ? (float)atof(argv[3]) : 0.0f;
        FILE *out = nullptr;
        if (argc > 4 && !(out = fopen(argv[4], "wb"))) throw "Error: cannot create the output file";
        EdgesList graph;
        if (!GraphStorageAPI::load_from_edges_list_bin_file(graph, file_name)) throw "Error: no such graph file";
        printf("graph loaded!\n");
        printf("graph size: %f GB\n\n", (double)(graph.get_edges_count() * 12) / (1024.0 * 1024.0 * 1024.0));
        DeviceGraph dg(graph);
        int vertices_count = dg.get_vertices_count();
        SingleSourceShortestPaths<int, float> operation;
        std::vector<float> result((size_t)vertices_count);
        double avg = 0;
        for (int i = 0; i < runs; i++) {
            int source_vertex = rand() % vertices_count;
            double mteps = operation.gpu_bellman_ford(dg, result.data(), source_vertex, delta);
            printf("GPU-only perfomance: %f MTEPS (source %d)\n", mteps, source_vertex);
            avg += mteps;
            if (out && (fwrite(&source_vertex, 4, 1, out) != 1 ||
                        fwrite(result.data(), 4, result.size(), out) != result.size()))
                throw "Error: writing the output file failed";
        }
        if (runs > 0) printf("avg perfomance: %f MTEPS\n", avg / runs);
        if (out) fclose(out);
    } catch (const char *error) {
        printf("%s\n", error);
        return 1;
    }
    return 0;
}
