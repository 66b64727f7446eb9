// Graph handle of the C ABI (shared by the C-ABI translation units).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "trav_internal.cuh"

struct trav_graph {
    trav::DevGraph g;
    trav::Workspace ws;
    cudaStream_t own_st = nullptr;    // the handle's stream
    cudaStream_t st = nullptr;        // stream queries run on (own_st or the caller's)
    cudaStream_t cst = nullptr;       // copy stream for host-bound results
    int device = 0;
    std::vector<int32_t> new_of_old;  // host copy for source mapping
    float *staging[2] = {nullptr, nullptr};  // device buffers for host-bound results (double-buffered)
    cudaEvent_t done[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> ev;      // start/stop event per query of a batch
    std::vector<float> batch_ms;      // device time of each launch of the last batch
    float *mlp[2] = {nullptr, nullptr};  // device MLP parameters: 0 = BFS, 1 = SSSP
    int last_kind = -1;
    int last_n = 0;
    // CUDA-graph capture of multi-source calls with device outputs: the
    // launches of a call are captured once and replayed while the call's
    // arguments repeat (one graph per kind)
    bool capture = false;
    struct Captured {
        cudaGraphExec_t exec = nullptr;
        std::vector<unsigned char> key;
    } cap[2];
};
