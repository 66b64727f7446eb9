// BFS sample on the B200 library: the counterpart of the reference's
// sample/bfs.cpp (argv[1] = RMAT scale).  Generates R_MAT_parallel(2^scale,
// 16, 45, 20, 20, 15) as the reference sample does (sample/bfs.cpp:138), then
// runs BFS from vertex 0 and reports reached vertices, levels and MTEPS.
//
//   bfs <scale> [seed=0]
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "host/trav_library.hpp"

using namespace trav_host;

int main(int argc, char **argv)
{
    try {
        if (argc < 2) {
            printf("usage: %s <scale> [seed]\n", argv[0]);
            return 1;
        }
        int scale = atoi(argv[1]);
        uint32_t seed = argc > 2 ? (uint32_t)strtoul(argv[2], nullptr, 10) : 0u;
        printf("Generating graph...\n");
        EdgesList graph;
        GraphGenerationAPI::R_MAT_parallel(graph, 1 << scale, 16, 45, 20, 20, 15, 1, true, seed);
        printf("done!\n\n");
        DeviceGraph dg(graph);
        BFS<int, float> operation;
        std::vector<int32_t> levels((size_t)dg.get_vertices_count());
        double mteps = operation.gpu_bfs_levels(dg, levels.data(), 0);
        long long reached = 0;
        int maxl = 0;
        for (int32_t l : levels)
            if (l >= 0) {
                reached++;
                if (l > maxl) maxl = l;
            }
        printf("reached %lld of %d vertices in %d levels\n", reached, dg.get_vertices_count(), maxl + 1);
        printf("GPU perfomance: %f MTEPS\n", mteps);
    } catch (const char *error) {
        printf("%s\n", error);
        return 1;
    }
    return 0;
}
