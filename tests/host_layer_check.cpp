// Checks of the C++ host layer (parallel-task1_b200/host/trav_library.hpp)
// that run without a GPU: the file APIs shaped like the reference's
// GraphStorageAPI.  tests/test_host_layer.py compiles this file against
// libtrav_b200.so and runs it:
//
//   host_layer_check files <el.bin> <adj.bin> <out_dir>
//
// It loads the reference-written edge-list and adjacency-list fixtures through
// the host layer, saves them again and prints one line per check; the Python
// side compares the bytes and the printed arrays.
#include <cstdio>
#include <cstring>
#include <string>

#include "host/trav_library.hpp"

using namespace trav_host;

static void print_el(const char *tag, const EdgesList &g)
{
    printf("%s V=%d E=%lld directed=%d", tag, g.get_vertices_count(), g.get_edges_count(), g.directed ? 1 : 0);
    for (long long e = 0; e < g.get_edges_count(); e++)
        printf(" %d>%d:%.9g", g.src_ids[(size_t)e], g.dst_ids[(size_t)e], (double)g.weights[(size_t)e]);
    printf("\n");
}

int main(int argc, char **argv)
{
    if (argc != 5 || strcmp(argv[1], "files") != 0) {
        printf("usage: %s files <el.bin> <adj.bin> <out_dir>\n", argv[0]);
        return 2;
    }
    const std::string out = argv[4];
    try {
        EdgesList el, adj;
        if (!GraphStorageAPI::load_from_edges_list_bin_file(el, argv[2])) throw "cannot load the edge list";
        print_el("el", el);
        if (!GraphStorageAPI::save_to_edges_list_bin_file(el, out + "/el_again.bin")) throw "cannot save the edge list";
        if (!GraphStorageAPI::load_from_adjacency_list_bin_file(adj, argv[3])) throw "cannot load the adjacency list";
        print_el("adj", adj);
        if (!GraphStorageAPI::save_to_adjacency_list_bin_file(el, out + "/adj_from_el.bin"))
            throw "cannot save the adjacency list";
        EdgesList pairs;
        if (!GraphStorageAPI::read_data_from_file(pairs, argv[2], 3)) throw "cannot read pairs";
        printf("pairs V=%d E=%lld\n", pairs.get_vertices_count(), pairs.get_edges_count());
        EdgesList missing;
        printf("missing=%d\n", GraphStorageAPI::load_from_edges_list_bin_file(missing, out + "/nope.bin") ? 1 : 0);
    } catch (const char *e) {
        printf("error: %s\n", e);
        return 1;
    }
    return 0;
}
