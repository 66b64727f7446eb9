// Schedule MLP: features of a traversal step and the fused, warp-cooperative
// forward pass evaluated inside the persistent kernels.
//
// Network: x (kFeat) -> tanh(W1 x + b1) (kHidden) -> tanh(W2 h1 + b2) (kHidden)
//          -> W3 h2 + b3 (O logits); the decision is the argmax.
// Parameters are packed row-major as [W1 | b1 | W2 | b2 | W3 | b3].
// The choice never changes results (BFS levels and SSSP distances are fixed
// points), only which kernel path a step takes.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace trav {

constexpr int kFeat = 10;
constexpr int kHidden = 32;
constexpr int kBfsOut = 2;      // 0 = top-down (push), 1 = bottom-up (pull)
constexpr int kSsspOut = 4;     // bucket width = delta * {1, 4, 16, 64} (merge 1, 4, 16, 64 buckets)

__host__ __device__ constexpr int mlp_param_count(int O)
{
    return kHidden * kFeat + kHidden + kHidden * kHidden + kHidden + O * kHidden + O;
}

struct Feat {
    float x[kFeat];
};

__host__ __device__ inline float flog2p1(double v) { return (float)log2(1.0 + (v > 0 ? v : 0)); }

// BFS step features: frontier size, frontier out-edges, unvisited out-edges,
// previous frontier size, step index, graph size and mean degree, growth,
// edge ratio and the previous step's direction.
__host__ __device__ inline Feat bfs_features(int step, unsigned long long nf, unsigned long long mf,
                                             unsigned long long mu, unsigned long long nf_prev, int V, long long E,
                                             int prev_dir)
{
    Feat f;
    f.x[0] = flog2p1((double)nf) / 32.0f;
    f.x[1] = flog2p1((double)mf) / 32.0f;
    f.x[2] = flog2p1((double)mu) / 32.0f;
    f.x[3] = flog2p1((double)nf_prev) / 32.0f;
    f.x[4] = (float)step / 16.0f;
    f.x[5] = flog2p1((double)V) / 32.0f;
    f.x[6] = flog2p1((double)E / (V > 0 ? V : 1)) / 8.0f;
    f.x[7] = nf >= nf_prev ? 1.0f : 0.0f;
    f.x[8] = (flog2p1((double)mf) - flog2p1((double)mu)) / 8.0f;
    f.x[9] = (float)prev_dir;
    return f;
}

// SSSP bucket features: relaxation rounds so far, far-pile size, distance of
// the nearest far entry relative to the current bound, delta, graph size and
// mean degree.
__host__ __device__ inline Feat sssp_features(int steps, unsigned long long far_len, float min_far, float thr,
                                              float delta, int V, long long E, int buckets)
{
    Feat f;
    f.x[0] = (float)steps / 64.0f;
    f.x[1] = flog2p1((double)far_len) / 32.0f;
    f.x[2] = (min_far - thr) / (delta > 0 ? delta : 1.0f) / 8.0f;
    f.x[3] = thr / (delta > 0 ? delta : 1.0f) / 64.0f;
    f.x[4] = flog2p1((double)V) / 32.0f;
    f.x[5] = flog2p1((double)E / (V > 0 ? V : 1)) / 8.0f;
    f.x[6] = (float)buckets / 64.0f;
    f.x[7] = flog2p1((double)far_len) / (flog2p1((double)V) + 1.0f);
    f.x[8] = delta;
    f.x[9] = 1.0f;
    return f;
}

__host__ __device__ inline float sssp_width_scale(int option) { return (float)(1 << (2 * option)); }

#ifdef __CUDACC__
// Warp-cooperative forward pass: lane j owns hidden unit j.  All 32 lanes
// must call; every lane returns the argmax (lowest index on ties).  The
// summation order is fixed, so every CTA computes the same decision.
__device__ inline int mlp_argmax_warp(const float *__restrict__ p, const Feat &f, int O)
{
    const int j = threadIdx.x & 31;
    const float *W1 = p, *b1 = W1 + kHidden * kFeat, *W2 = b1 + kHidden, *b2 = W2 + kHidden * kHidden;
    const float *W3 = b2 + kHidden, *b3 = W3 + O * kHidden;
    float a = __ldg(&b1[j]);
#pragma unroll
    for (int i = 0; i < kFeat; i++) a = fmaf(__ldg(&W1[j * kFeat + i]), f.x[i], a);
    const float h1 = tanhf(a);
    a = __ldg(&b2[j]);
#pragma unroll 8
    for (int i = 0; i < kHidden; i++) a = fmaf(__ldg(&W2[j * kHidden + i]), __shfl_sync(0xffffffffu, h1, i), a);
    const float h2 = tanhf(a);
    int best = 0;
    float bestv = -INFINITY;
    for (int o = 0; o < O; o++) {
        float t = __ldg(&W3[o * kHidden + j]) * h2;
#pragma unroll
        for (int s = 16; s; s >>= 1) t += __shfl_xor_sync(0xffffffffu, t, s);
        t += __ldg(&b3[o]);
        if (t > bestv) { bestv = t; best = o; }
    }
    // the butterfly sums may round differently per lane: lane 0 decides
    return __shfl_sync(0xffffffffu, best, 0);
}
#endif

}  // namespace trav
