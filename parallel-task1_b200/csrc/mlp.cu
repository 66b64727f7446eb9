// Training of the schedule MLP on the GPU: forward + backward of the
// softmax cross-entropy loss (one warp per sample, lane j owning hidden unit
// j), a deterministic reduction of the gradients, and Adam.  The network and
// its parameter packing are described in mlp_device.cuh; the float64
// restatement used to check these gradients is orc_mlp_loss_grad.  New: the
// reference has no learned component.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "mlp_device.cuh"
#include "trav_internal.cuh"

namespace trav {

namespace {

constexpr int kMlpBlock = 256;
constexpr int kMlpWarps = kMlpBlock / 32;
constexpr int kMaxParams = kHidden * kFeat + kHidden + kHidden * kHidden + kHidden + kSsspOut * kHidden + kSsspOut;

// Per-CTA partial gradient (fixed summation order: samples by warp, warps in
// order) and partial loss.
template <int O>
__global__ void __launch_bounds__(kMlpBlock) mlp_grad_kernel(const float *__restrict__ params,
                                                             const float *__restrict__ X, const int *__restrict__ y,
                                                             int n, float *__restrict__ partial, float *__restrict__ lpart)
{
    __shared__ float p[kMaxParams];
    __shared__ float acc[kMaxParams];
    __shared__ float wloss[kMlpWarps];
    const int P = mlp_param_count(O);
    for (int i = threadIdx.x; i < P; i += kMlpBlock) p[i] = params[i];
    __syncthreads();
    const float *W1 = p, *b1 = W1 + kHidden * kFeat, *W2 = b1 + kHidden, *b2 = W2 + kHidden * kHidden;
    const float *W3 = b2 + kHidden, *b3 = W3 + O * kHidden;
    const int j = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float gW1[kFeat], gb1 = 0.0f, gW2[kHidden], gb2 = 0.0f, gW3[O], gb3[O];
#pragma unroll
    for (int i = 0; i < kFeat; i++) gW1[i] = 0.0f;
#pragma unroll
    for (int i = 0; i < kHidden; i++) gW2[i] = 0.0f;
#pragma unroll
    for (int o = 0; o < O; o++) gW3[o] = gb3[o] = 0.0f;
    float loss = 0.0f;
    const float inv_n = 1.0f / (float)n;
    for (int s = blockIdx.x * kMlpWarps + wid; s < n; s += gridDim.x * kMlpWarps) {
        float x[kFeat];
#pragma unroll
        for (int i = 0; i < kFeat; i++) x[i] = __ldg(&X[(size_t)s * kFeat + i]);
        float a = b1[j];
#pragma unroll
        for (int i = 0; i < kFeat; i++) a = fmaf(W1[j * kFeat + i], x[i], a);
        const float h1 = tanhf(a);
        a = b2[j];
#pragma unroll 8
        for (int i = 0; i < kHidden; i++) a = fmaf(W2[j * kHidden + i], __shfl_sync(0xffffffffu, h1, i), a);
        const float h2 = tanhf(a);
        float logit[O];
        float m = -INFINITY;
#pragma unroll
        for (int o = 0; o < O; o++) {
            float t = W3[o * kHidden + j] * h2;
#pragma unroll
            for (int k = 16; k; k >>= 1) t += __shfl_xor_sync(0xffffffffu, t, k);
            t = __shfl_sync(0xffffffffu, t, 0) + b3[o];
            logit[o] = t;
            m = fmaxf(m, t);
        }
        float z = 0.0f;
#pragma unroll
        for (int o = 0; o < O; o++) z += expf(logit[o] - m);
        const int label = __ldg(&y[s]);
        float lab_logit = 0.0f;
#pragma unroll
        for (int o = 0; o < O; o++)
            if (o == label) lab_logit = logit[o];
        loss += logf(z) + m - lab_logit;
        float d2 = 0.0f;
#pragma unroll
        for (int o = 0; o < O; o++) {
            const float dy = (expf(logit[o] - m) / z - (o == label ? 1.0f : 0.0f)) * inv_n;
            gW3[o] = fmaf(dy, h2, gW3[o]);
            gb3[o] += dy;
            d2 = fmaf(W3[o * kHidden + j], dy, d2);
        }
        d2 *= 1.0f - h2 * h2;
        gb2 += d2;
#pragma unroll 8
        for (int i = 0; i < kHidden; i++) gW2[i] = fmaf(d2, __shfl_sync(0xffffffffu, h1, i), gW2[i]);
        float d1 = 0.0f;  // lane j: sum over k of W2[k][j] * d2_k
#pragma unroll 8
        for (int k = 0; k < kHidden; k++) d1 = fmaf(W2[k * kHidden + j], __shfl_sync(0xffffffffu, d2, k), d1);
        d1 *= 1.0f - h1 * h1;
        gb1 += d1;
#pragma unroll
        for (int i = 0; i < kFeat; i++) gW1[i] = fmaf(d1, x[i], gW1[i]);
    }
    // per-warp gradients summed into shared memory one warp after the other
    // (a fixed order, so the result does not depend on scheduling)
    const int w3 = kHidden * kFeat + 2 * kHidden + kHidden * kHidden;
    for (int i = threadIdx.x; i < P; i += kMlpBlock) acc[i] = 0.0f;
    if (j == 0) wloss[wid] = loss;
    for (int w = 0; w < kMlpWarps; w++) {
        __syncthreads();
        if (wid == w) {
#pragma unroll
            for (int i = 0; i < kFeat; i++) acc[j * kFeat + i] += gW1[i];
            acc[kHidden * kFeat + j] += gb1;
#pragma unroll
            for (int i = 0; i < kHidden; i++) acc[kHidden * kFeat + kHidden + j * kHidden + i] += gW2[i];
            acc[kHidden * kFeat + kHidden + kHidden * kHidden + j] += gb2;
#pragma unroll
            for (int o = 0; o < O; o++) acc[w3 + o * kHidden + j] += gW3[o];
            if (j == 0)
#pragma unroll
                for (int o = 0; o < O; o++) acc[w3 + O * kHidden + o] += gb3[o];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P; i += kMlpBlock) partial[(size_t)blockIdx.x * P + i] = acc[i];
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < kMlpWarps; w++) t += wloss[w];
        lpart[blockIdx.x] = t;
    }
}

// grad[i] = sum over CTAs of partial[c][i] (in CTA order); loss likewise, / n.
__global__ void mlp_reduce_kernel(const float *__restrict__ partial, const float *__restrict__ lpart, int nblk, int P,
                                  int n, float *__restrict__ grad, float *__restrict__ loss)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) {
        float t = 0.0f;
        for (int c = 0; c < nblk; c++) t += partial[(size_t)c * P + i];
        grad[i] = t;
    }
    if (i == 0) {
        float t = 0.0f;
        for (int c = 0; c < nblk; c++) t += lpart[c];
        *loss = t / (float)n;
    }
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int P, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

#define TRY_CUDA(expr)                                      \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

struct MlpDev {
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr, *x = nullptr, *partial = nullptr, *lpart = nullptr,
          *loss = nullptr;
    int *y = nullptr;
    ~MlpDev()
    {
        cudaFree(p);
        cudaFree(g);
        cudaFree(m);
        cudaFree(v);
        cudaFree(x);
        cudaFree(partial);
        cudaFree(lpart);
        cudaFree(loss);
        cudaFree(y);
    }
};

int outputs_of(int kind) { return kind == 0 ? kBfsOut : kind == 1 ? kSsspOut : -1; }

int mlp_blocks(int n)
{
    int b = (n + kMlpWarps - 1) / kMlpWarps;
    if (b > 296) b = 296;
    return b < 1 ? 1 : b;
}

void launch_grad(int O, int nblk, MlpDev &d, int n)
{
    if (O == kBfsOut) mlp_grad_kernel<kBfsOut><<<nblk, kMlpBlock>>>(d.p, d.x, d.y, n, d.partial, d.lpart);
    else mlp_grad_kernel<kSsspOut><<<nblk, kMlpBlock>>>(d.p, d.x, d.y, n, d.partial, d.lpart);
}

int upload(MlpDev &d, int P, const float *params, const float *x, const int32_t *labels, int n, int nblk)
{
    TRY_CUDA(dev_malloc(&d.p, sizeof(float) * P));
    TRY_CUDA(dev_malloc(&d.g, sizeof(float) * P));
    TRY_CUDA(dev_malloc(&d.x, sizeof(float) * (size_t)n * kFeat));
    TRY_CUDA(dev_malloc(&d.y, sizeof(int) * (size_t)n));
    TRY_CUDA(dev_malloc(&d.partial, sizeof(float) * (size_t)nblk * P));
    TRY_CUDA(dev_malloc(&d.lpart, sizeof(float) * (size_t)nblk));
    TRY_CUDA(dev_malloc(&d.loss, sizeof(float)));
    TRY_CUDA(cudaMemcpy(d.p, params, sizeof(float) * P, cudaMemcpyHostToDevice));
    TRY_CUDA(cudaMemcpy(d.x, x, sizeof(float) * (size_t)n * kFeat, cudaMemcpyHostToDevice));
    TRY_CUDA(cudaMemcpy(d.y, labels, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    return TRAV_OK;
}

int check_args(int kind, const float *params, const float *x, const int32_t *labels, int32_t n)
{
    const int O = outputs_of(kind);
    if (O < 0) {
        set_error("kind must be 0 (BFS) or 1 (SSSP)");
        return TRAV_ERR_BAD_ARG;
    }
    if (!params || !x || !labels || n < 1) {
        set_error("params, x and labels must be host arrays and n >= 1");
        return TRAV_ERR_BAD_ARG;
    }
    for (int32_t i = 0; i < n; i++)
        if (labels[i] < 0 || labels[i] >= O) {
            set_error("labels must lie in [0, outputs)");
            return TRAV_ERR_BAD_ARG;
        }
    return TRAV_OK;
}

}  // namespace

}  // namespace trav

using namespace trav;

extern "C" int trav_mlp_loss_grad(int32_t kind, const float *params, const float *x, const int32_t *labels, int32_t n,
                                  float *grad, float *loss)
{
    int rc = check_args(kind, params, x, labels, n);
    if (rc) return rc;
    const int O = outputs_of(kind), P = mlp_param_count(O), nblk = mlp_blocks(n);
    MlpDev d;
    rc = upload(d, P, params, x, labels, n, nblk);
    if (rc) return rc;
    launch_grad(O, nblk, d, n);
    mlp_reduce_kernel<<<(P + 255) / 256, 256>>>(d.partial, d.lpart, nblk, P, n, d.g, d.loss);
    TRY_CUDA(cudaGetLastError());
    if (grad) TRY_CUDA(cudaMemcpy(grad, d.g, sizeof(float) * P, cudaMemcpyDeviceToHost));
    if (loss) TRY_CUDA(cudaMemcpy(loss, d.loss, sizeof(float), cudaMemcpyDeviceToHost));
    TRY_CUDA(cudaDeviceSynchronize());
    return TRAV_OK;
}

extern "C" int trav_mlp_train(int32_t kind, float *params, const float *x, const int32_t *labels, int32_t n,
                              int32_t epochs, float lr, float *final_loss)
{
    int rc = check_args(kind, params, x, labels, n);
    if (rc) return rc;
    if (epochs < 1 || !(lr > 0.0f)) {
        set_error("epochs must be >= 1 and lr > 0");
        return TRAV_ERR_BAD_ARG;
    }
    const int O = outputs_of(kind), P = mlp_param_count(O), nblk = mlp_blocks(n);
    MlpDev d;
    rc = upload(d, P, params, x, labels, n, nblk);
    if (rc) return rc;
    TRY_CUDA(dev_malloc(&d.m, sizeof(float) * P));
    TRY_CUDA(dev_malloc(&d.v, sizeof(float) * P));
    TRY_CUDA(cudaMemset(d.m, 0, sizeof(float) * P));
    TRY_CUDA(cudaMemset(d.v, 0, sizeof(float) * P));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    double c1 = 1.0, c2 = 1.0;
    for (int t = 1; t <= epochs; t++) {  // full-batch Adam steps
        c1 *= b1;
        c2 *= b2;
        launch_grad(O, nblk, d, n);
        mlp_reduce_kernel<<<(P + 255) / 256, 256>>>(d.partial, d.lpart, nblk, P, n, d.g, d.loss);
        adam_kernel<<<(P + 255) / 256, 256>>>(d.p, d.g, d.m, d.v, P, lr, b1, b2, eps, (float)(1.0 - c1),
                                              (float)(1.0 - c2));
    }
    TRY_CUDA(cudaGetLastError());
    TRY_CUDA(cudaMemcpy(params, d.p, sizeof(float) * P, cudaMemcpyDeviceToHost));
    if (final_loss) {
        launch_grad(O, nblk, d, n);
        mlp_reduce_kernel<<<(P + 255) / 256, 256>>>(d.partial, d.lpart, nblk, P, n, d.g, d.loss);
        TRY_CUDA(cudaMemcpy(final_loss, d.loss, sizeof(float), cudaMemcpyDeviceToHost));
    }
    TRY_CUDA(cudaDeviceSynchronize());
    return TRAV_OK;
}
