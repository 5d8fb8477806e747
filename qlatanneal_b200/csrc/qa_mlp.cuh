// qa_mlp.cuh -- training and inference kernels of the chi_B-curve MLP.
//
// A plain multilayer perceptron: dims d0 -> d1 -> ... -> dL, ReLU between
// layers, linear output.  Weights are held twice: float32 masters (updated by
// Adam) and bfloat16 copies that the forward and backward passes read; all
// products accumulate in float32, in a fixed order (no atomics), so a step is
// reproducible.  The output is 2M wide: M means and M log-variances of a
// Gaussian over the target curve; the loss is the mean negative log-likelihood
//   l = 1/2 (exp(-s) (t - mu)^2 + s),   s clamped to [-12, 12].
// Parameter layout (float32 masters): for each layer l, W_l[d_l][d_l+1]
// row-major, then b_l[d_l+1].
#pragma once
#include <cuda_bf16.h>

#include "qa_device.cuh"

namespace qa {

// Y[b][n] = act(b[n] + sum_k X[b][k] W[k][n])   (thread per output)
__global__ void mlp_fwd_kernel(const float *X, int B, int K, const __nv_bfloat16 *W, const float *bias, float *Y,
                               int N, int relu) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * N) return;
    const int b = idx / N, n = idx - b * N;
    float acc = bias[n];
    const float *x = X + (long long)b * K;
    for (int k = 0; k < K; ++k) acc = __fmaf_rn(x[k], __bfloat162float(W[(long long)k * N + n]), acc);
    Y[idx] = relu ? fmaxf(acc, 0.0f) : acc;
}

// Gaussian NLL over [mu | s] outputs; dY = dl/dY / (B M); per-row loss sums.
__global__ void mlp_loss_kernel(const float *Y, const float *T, int B, int M, float *dY, float *row_loss) {
    const int b = blockIdx.x;
    if (b >= B) return;
    __shared__ float part[256];
    float acc = 0.0f;
    const float inv = 1.0f / (float)(B * M);
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        const float mu = Y[(long long)b * 2 * M + m];
        const float sr = Y[(long long)b * 2 * M + M + m];
        const float s = fminf(fmaxf(sr, -12.0f), 12.0f);
        const float e = expf(-s);
        const float d = T[(long long)b * M + m] - mu;
        acc += 0.5f * (e * d * d + s);
        dY[(long long)b * 2 * M + m] = -e * d * inv;
        dY[(long long)b * 2 * M + M + m] = (sr > -12.0f && sr < 12.0f) ? 0.5f * (1.0f - e * d * d) * inv : 0.0f;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int i = 0; i < (int)blockDim.x; ++i) s += part[i];
        row_loss[b] = s;
    }
}

// dW[k][n] = sum_b X[b][k] dZ[b][n],  db[n] = sum_b dZ[b][n]   (thread per (k, n) / n)
__global__ void mlp_bwd_weight_kernel(const float *X, const float *dZ, int B, int K, int N, float *dW, float *db) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < K * N) {
        const int k = idx / N, n = idx - k * N;
        float acc = 0.0f;
        for (int b = 0; b < B; ++b) acc = __fmaf_rn(X[(long long)b * K + k], dZ[(long long)b * N + n], acc);
        dW[idx] = acc;
    } else if (idx < K * N + N) {
        const int n = idx - K * N;
        float acc = 0.0f;
        for (int b = 0; b < B; ++b) acc += dZ[(long long)b * N + n];
        db[n] = acc;
    }
}

// dX[b][k] = (sum_n dZ[b][n] W[k][n]) * [X[b][k] > 0]   (ReLU of the layer below)
__global__ void mlp_bwd_input_kernel(const float *dZ, const __nv_bfloat16 *W, const float *X, int B, int K, int N,
                                     float *dX) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * K) return;
    const int b = idx / K, k = idx - b * K;
    float acc = 0.0f;
    for (int n = 0; n < N; ++n)
        acc = __fmaf_rn(dZ[(long long)b * N + n], __bfloat162float(W[(long long)k * N + n]), acc);
    dX[idx] = X[idx] > 0.0f ? acc : 0.0f;
}

// Adam on the float32 masters; refreshes the bfloat16 copies of the weights.
__global__ void mlp_adam_kernel(float *W, const float *g, float *m, float *v, long long count, float lr, float b1,
                                float b2, float eps, float c1, float c2, const long long *wmap, __nv_bfloat16 *W16) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float w = W[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    W[i] = w;
    const long long j = wmap[i];
    if (j >= 0) W16[j] = __float2bfloat16_rn(w);
}

__global__ void mlp_to_bf16_kernel(const float *W, long long count, const long long *wmap, __nv_bfloat16 *W16) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long j = wmap[i];
    if (j >= 0) W16[j] = __float2bfloat16_rn(W[i]);
}

}  // namespace qa
