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
constexpr int kSsspOut = 6;     // bucket width = delta * 4^k, k = 0..5 (merge 1 .. 1024 buckets)
constexpr double kBfsGate = 8.0;  // BFS steps within this factor of a Beamer threshold consult the network

__host__ __device__ constexpr int mlp_param_count(int O)
{
    return kHidden * kFeat + kHidden + kHidden * kHidden + kHidden + O * kHidden + O;
}
constexpr int kMlpMaxParams = kHidden * kFeat + kHidden + kHidden * kHidden + kHidden + kSsspOut * kHidden + kSsspOut;

struct Feat {
    float x[kFeat];
};

// Feature arithmetic is single precision (log2f): the features only steer a
// choice, and every CTA evaluates them identically.
__host__ __device__ inline float flog2p1(double v) { return log2f(1.0f + (float)(v > 0 ? v : 0)); }

// sign(v) * log2(1 + |v|): bounded growth for quantities of any scale
__host__ __device__ inline float fslog2p1(double v) { return v < 0 ? -flog2p1(-v) : flog2p1(v); }

// log2(a / b) for counts (a, b >= 1)
__host__ __device__ inline float flog2ratio(double a, double b) { return log2f((float)a) - log2f((float)b); }

// BFS step features, all scale-free so that graphs larger than the training
// graphs stay in range: the two ratios Beamer's switch tests (frontier
// out-edges / unexplored edges, frontier / V), frontier growth, the step
// index, mean degree, the explored and frontier shares of the edges, whether
// the frontier grew, the previous direction and the plain switch's own choice
// (so the network only has to learn where to differ from it).
__host__ __device__ inline Feat bfs_features(int step, unsigned long long nf, unsigned long long mf,
                                             unsigned long long mu, unsigned long long nf_prev, int V, long long E,
                                             int prev_dir, int plain_dir)
{
    Feat f;
    const double v = V > 0 ? (double)V : 1.0, e = E > 0 ? (double)E : 1.0;
    f.x[0] = flog2ratio((double)mf + 1.0, (double)mu + 1.0) / 8.0f;
    f.x[1] = flog2ratio((double)nf + 1.0, v) / 8.0f;
    f.x[2] = flog2ratio((double)nf + 1.0, (double)nf_prev + 1.0) / 8.0f;
    f.x[3] = flog2p1((double)step) / 8.0f;
    f.x[4] = flog2p1(e / v) / 8.0f;
    f.x[5] = flog2ratio((double)mu + 1.0, e) / 8.0f;
    f.x[6] = flog2ratio((double)mf + 1.0, e) / 8.0f;
    f.x[7] = nf >= nf_prev ? 1.0f : 0.0f;
    f.x[8] = (float)prev_dir;
    f.x[9] = (float)plain_dir;
    return f;
}

// SSSP bucket features: relaxation rounds and buckets so far, the far pile's
// share of the vertices, the gap from the current bound to the nearest far
// entry and the bound itself in units of delta and of the mean edge weight,
// mean degree, the mean edge weight in units of delta (how many buckets one
// edge spans), the degree skew (largest out-degree over the mean: wide
// buckets pay on skewed graphs, whose hubs settle early, and cost re-relaxation
// on even ones), and the graph's size: whether wide buckets pay depends on it,
// since they trade fewer rounds (latency) for more re-relaxation (work).
__host__ __device__ inline Feat sssp_features(int steps, unsigned long long far_len, float min_far, float thr,
                                              float delta, int V, long long E, int buckets, float mean_w, int max_deg)
{
    Feat f;
    const double d = delta > 0 ? (double)delta : 1.0;
    const double mw = mean_w > 0 ? (double)mean_w : d;
    const double v = V > 0 ? (double)V : 1.0;
    const double gap = (double)min_far - (double)thr;
    f.x[0] = flog2p1((double)steps) / 16.0f;
    f.x[1] = flog2ratio((double)far_len + 1.0, v) / 8.0f;
    f.x[2] = fslog2p1(gap / d) / 16.0f;
    f.x[3] = flog2p1((double)thr / d) / 16.0f;
    f.x[4] = flog2p1((double)E / v) / 8.0f;
    f.x[5] = flog2p1((double)buckets) / 16.0f;
    f.x[6] = fslog2p1(mw / d) / 8.0f;
    f.x[7] = fslog2p1(gap / mw) / 8.0f;
    f.x[8] = flog2p1((double)max_deg / ((double)E / v + 1.0)) / 16.0f;
    f.x[9] = (flog2p1((double)E) - 16.0f) / 12.0f;  // about 0 at 2^16 edges, 1 at 2^28
    return f;
}

__host__ __device__ inline float sssp_width_scale(int option) { return (float)(1 << (2 * option)); }

#ifdef __CUDACC__
// Warp-cooperative forward pass over parameters held in shared memory: lane j
// owns hidden unit j; the output layer reduces all O logits in one butterfly
// (O independent shuffle chains).  All 32 lanes must call; lane 0's argmax
// (lowest index on ties) is returned in every lane.  The summation order is
// fixed, so every CTA computes the same decision.
//
// Abstention: with margin > 0 the network keeps the plain schedule's option
// `plain` unless its best logit beats plain's by at least margin, so a network
// that is unsure (or wrong by little) does not override its fallback.
template <int O>
__device__ inline int mlp_argmax_warp(const float *p, const Feat &f, int plain = 0, float margin = 0.0f)
{
    const int j = threadIdx.x & 31;
    const float *W1 = p, *b1 = W1 + kHidden * kFeat, *W2 = b1 + kHidden, *b2 = W2 + kHidden * kHidden;
    const float *W3 = b2 + kHidden, *b3 = W3 + O * kHidden;
    float a = b1[j];
#pragma unroll
    for (int i = 0; i < kFeat; i++) a = fmaf(W1[j * kFeat + i], f.x[i], a);
    const float h1 = tanhf(a);
    a = b2[j];
#pragma unroll
    for (int i = 0; i < kHidden; i++) a = fmaf(W2[j * kHidden + i], __shfl_sync(0xffffffffu, h1, i), a);
    const float h2 = tanhf(a);
    float t[O];
#pragma unroll
    for (int o = 0; o < O; o++) t[o] = W3[o * kHidden + j] * h2;
#pragma unroll
    for (int s = 16; s; s >>= 1) {
#pragma unroll
        for (int o = 0; o < O; o++) t[o] += __shfl_xor_sync(0xffffffffu, t[o], s);
    }
    int best = 0;
    float bestv = -INFINITY, plainv = -INFINITY;
#pragma unroll
    for (int o = 0; o < O; o++) {
        const float v = t[o] + b3[o];
        if (o == plain) plainv = v;
        if (v > bestv) {
            bestv = v;
            best = o;
        }
    }
    if (margin > 0.0f && bestv - plainv < margin) best = plain;
    // the butterfly sums may round differently per lane: lane 0 decides
    return __shfl_sync(0xffffffffu, best, 0);
}
#endif

}  // namespace trav
