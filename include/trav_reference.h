/* trav_reference.h -- the reference library's CUDA wrapper declarations,
 * implemented by libtrav_b200.so on the B200 kernels.
 *
 * A reference build that includes this header instead of
 * algorithm/sssp/gpu/bellman_ford.cuh and algorithm/bfs/gpu/bfs.cuh, and
 * links libtrav_b200.so instead of compiling bellman_ford.cu and bfs.cu,
 * runs its unchanged callers (SingleSourceShortestPaths::gpu_bellman_ford,
 * algorithm/sssp/sssp.hpp:257-258; BFS::gpu_bfs, algorithm/bfs/bfs.hpp:242;
 * TransitiveClosure::gpu_bfs, algorithm/transitive_closure/
 * transitive_closure.hpp:50) on this library.
 *
 * Contract kept from the reference: every pointer is a device pointer owned
 * by the caller; calls are synchronous; on failure a message is printed and
 * a `const char *` is thrown, as SAFE_CALL / SAFE_KERNEL_CALL do
 * (include/common/cuda_error_hadling.h:4-24).
 */
#pragma once

#define VISITED true
#define UNVISITED false

/* algorithm/sssp/gpu/bellman_ford.cuh:13-14; instantiated for float and
 * double (bellman_ford.cu:150-151).  The double form is declared for link
 * compatibility and throws: this library computes in fp32. */
template <typename _TEdgeWeight>
void init_distances_wrapper(_TEdgeWeight *_distances, int _vertices_count, int _source_vertex);

/* algorithm/sssp/gpu/bellman_ford.cuh:16-18 (instantiated at
 * bellman_ford.cu:153-156): relaxes _distances to the Bellman-Ford fixpoint of
 * the device edge list, starting from whatever it holds. */
template <typename _TEdgeWeight>
void bellman_ford_wrapper(int *_src_ids, int *_dst_ids, _TEdgeWeight *_weights, int _vertices_count,
                          long long _edges_count, int _source_vertex, _TEdgeWeight *_distances);

/* algorithm/bfs/gpu/bfs.cuh:10: reachability from _source_vertex into the
 * device bool array _visited. */
void bfs_wrapper(int *_src_ids, int *_dst_ids, int _vertices_count, long long _edges_count, bool *_visited,
                 int _source_vertex);
