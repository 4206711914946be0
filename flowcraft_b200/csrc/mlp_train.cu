// Training kernels of the learned closure's MLP (5 -> 32 -> 32 -> 1, ReLU,
// linear output): FP32 forward, mean-squared-error loss and gradient, and
// the Adam update. The gradient is deterministic: a fixed grid of blocks
// takes 128-sample tiles in a fixed order, each block keeps its parameter
// partial sums in registers, and one final kernel adds the per-block
// partials in block order.
#include <cuda_runtime.h>

#include <cstdint>

#include "fc_lbm.h"

namespace {

constexpr int kIn = 5, kH = 32;
constexpr int kW1 = 0, kB1 = kW1 + kIn * kH, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH, kB3 = kW3 + kH;
constexpr int kP = kB3 + 1;
static_assert(kP == FC_MLP_PARAMS, "parameter count must match the header");
constexpr int kTile = 128;                         // samples per tile = threads per block
constexpr int kGradBlocks = 148;
constexpr int kPerThread = (kP + kTile - 1) / kTile;  // parameters each thread accumulates
static_assert((size_t)kGradBlocks * kP + 2 * kGradBlocks <= FC_MLP_GRAD_SCRATCH, "scratch size");

__device__ __forceinline__ void forward(const float* __restrict__ w, const float* x, float* z1, float* h1, float* z2,
                                        float* h2, float& out) {
#pragma unroll 4
    for (int j = 0; j < kH; ++j) {
        float s = w[kB1 + j];
        for (int i = 0; i < kIn; ++i) s = fmaf(x[i], w[kW1 + i * kH + j], s);
        z1[j] = s;
        h1[j] = s > 0.0f ? s : 0.0f;
    }
#pragma unroll 4
    for (int k = 0; k < kH; ++k) {
        float s = w[kB2 + k];
        for (int j = 0; j < kH; ++j) s = fmaf(h1[j], w[kW2 + j * kH + k], s);
        z2[k] = s;
        h2[k] = s > 0.0f ? s : 0.0f;
    }
    float o = w[kB3];
    for (int k = 0; k < kH; ++k) o = fmaf(h2[k], w[kW3 + k], o);
    out = o;
}

__global__ void __launch_bounds__(kTile) k_mlp_forward(const float* __restrict__ params, const float* __restrict__ x,
                                                      int64_t n, float* __restrict__ y) {
    __shared__ float w[kP];
    for (int p = threadIdx.x; p < kP; p += blockDim.x) w[p] = params[p];
    __syncthreads();
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        float xi[kIn], z1[kH], h1[kH], z2[kH], h2[kH], o;
        for (int i = 0; i < kIn; ++i) xi[i] = x[s * kIn + i];
        forward(w, xi, z1, h1, z2, h2, o);
        y[s] = o;
    }
}

// One tile per block iteration: every thread runs forward and backward for
// its sample and parks what the parameter gradients need in shared memory;
// then each thread adds the tile's contribution to its own parameters.
__global__ void __launch_bounds__(kTile) k_mlp_grad(const float* __restrict__ params, const float* __restrict__ x,
                                                   const float* __restrict__ y, const int64_t* __restrict__ idx,
                                                   int64_t n, float* __restrict__ partial,
                                                   double* __restrict__ loss_partial) {
    extern __shared__ float sm[];
    float* w = sm;                        // kP
    float* sx = w + kP;                   // [kTile][kIn]
    float* sh1 = sx + kTile * kIn;        // [kTile][kH]
    float* sdh1 = sh1 + kTile * kH;       // dL/dz1
    float* sh2 = sdh1 + kTile * kH;
    float* sdh2 = sh2 + kTile * kH;       // dL/dz2
    float* sd = sdh2 + kTile * kH;        // dL/dout
    for (int p = threadIdx.x; p < kP; p += blockDim.x) w[p] = params[p];
    float acc[kPerThread];
    for (int r = 0; r < kPerThread; ++r) acc[r] = 0.0f;
    double lsum = 0.0;
    const int t = threadIdx.x;
    const int64_t tiles = (n + kTile - 1) / kTile;
    const float inv_n = 1.0f / (float)n;
    __syncthreads();
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t s = tile * kTile + t;
        const bool live = s < n;
        float xi[kIn], z1[kH], h1[kH], z2[kH], h2[kH], o = 0.0f, d = 0.0f;
        if (live) {
            const int64_t row = idx ? idx[s] : s;
            for (int i = 0; i < kIn; ++i) xi[i] = x[row * kIn + i];
            forward(w, xi, z1, h1, z2, h2, o);
            const float e = o - y[row];
            lsum += (double)e * (double)e;
            d = 2.0f * e * inv_n;
        } else {
            for (int i = 0; i < kIn; ++i) xi[i] = 0.0f;
            for (int j = 0; j < kH; ++j) z1[j] = h1[j] = z2[j] = h2[j] = 0.0f;
        }
        float dz2[kH];
        for (int k = 0; k < kH; ++k) dz2[k] = z2[k] > 0.0f ? d * w[kW3 + k] : 0.0f;
        for (int j = 0; j < kH; ++j) {
            float g = 0.0f;
            for (int k = 0; k < kH; ++k) g = fmaf(w[kW2 + j * kH + k], dz2[k], g);
            sdh1[t * kH + j] = z1[j] > 0.0f ? g : 0.0f;
            sh1[t * kH + j] = h1[j];
            sh2[t * kH + j] = h2[j];
            sdh2[t * kH + j] = dz2[j];
        }
        for (int i = 0; i < kIn; ++i) sx[t * kIn + i] = xi[i];
        sd[t] = d;
        __syncthreads();
        for (int r = 0; r < kPerThread; ++r) {
            const int p = t + r * kTile;
            if (p >= kP) break;
            float a = 0.0f;
            if (p < kB1) {
                const int i = (p - kW1) / kH, j = (p - kW1) % kH;
                for (int q = 0; q < kTile; ++q) a = fmaf(sx[q * kIn + i], sdh1[q * kH + j], a);
            } else if (p < kW2) {
                const int j = p - kB1;
                for (int q = 0; q < kTile; ++q) a += sdh1[q * kH + j];
            } else if (p < kB2) {
                const int j = (p - kW2) / kH, k = (p - kW2) % kH;
                for (int q = 0; q < kTile; ++q) a = fmaf(sh1[q * kH + j], sdh2[q * kH + k], a);
            } else if (p < kW3) {
                const int k = p - kB2;
                for (int q = 0; q < kTile; ++q) a += sdh2[q * kH + k];
            } else if (p < kB3) {
                const int k = p - kW3;
                for (int q = 0; q < kTile; ++q) a = fmaf(sh2[q * kH + k], sd[q], a);
            } else {
                for (int q = 0; q < kTile; ++q) a += sd[q];
            }
            acc[r] += a;
        }
        __syncthreads();
    }
    for (int r = 0; r < kPerThread; ++r) {
        const int p = t + r * kTile;
        if (p < kP) partial[(size_t)blockIdx.x * kP + p] = acc[r];
    }
    // block loss sum in thread order
    __shared__ double sl[kTile];
    sl[t] = lsum;
    __syncthreads();
    if (t == 0) {
        double b = 0.0;
        for (int q = 0; q < kTile; ++q) b += sl[q];
        loss_partial[blockIdx.x] = b;
    }
}

__global__ void k_mlp_grad_final(const float* __restrict__ partial, const double* __restrict__ loss_partial,
                                 int blocks, int64_t n, float* __restrict__ grad, double* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kP) {
        float g = 0.0f;
        for (int b = 0; b < blocks; ++b) g += partial[(size_t)b * kP + p];
        grad[p] = g;
    }
    if (p == 0 && loss) {
        double l = 0.0;
        for (int b = 0; b < blocks; ++b) l += loss_partial[b];
        *loss = l / (double)n;
    }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kP) return;
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.0f - b1) * gp;
    const float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    w[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

constexpr size_t kGradSmem = sizeof(float) * (kP + kTile * kIn + 4 * kTile * kH + kTile);

}  // namespace

extern "C" {

FC_LBM_API int fc_lbm_mlp_forward(const float* params, const float* x, int64_t n, float* y, void* stream) {
    if (!params || (n > 0 && (!x || !y)) || n < 0) return FC_LBM_ERR_INVALID_ARG;
    if (n == 0) return FC_LBM_OK;
    const int64_t blocks = (n + kTile - 1) / kTile;
    k_mlp_forward<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), kTile, 0, (cudaStream_t)stream>>>(params, x,
                                                                                                     n, y);
    return cudaGetLastError() == cudaSuccess ? FC_LBM_OK : FC_LBM_ERR_CUDA;
}

FC_LBM_API int fc_lbm_mlp_grad(const float* params, const float* x, const float* y, const int64_t* idx, int64_t n,
                               float* grad, double* loss, float* scratch, void* stream) {
    if (!params || !x || !y || !grad || !scratch || n <= 0) return FC_LBM_ERR_INVALID_ARG;
    // per device and cheap: set on every call
    if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem) != cudaSuccess)
        return FC_LBM_ERR_CUDA;
    float* partial = scratch;
    double* lp = reinterpret_cast<double*>(scratch + (size_t)kGradBlocks * kP + ((size_t)kGradBlocks * kP) % 2);
    cudaStream_t s = (cudaStream_t)stream;
    k_mlp_grad<<<kGradBlocks, kTile, kGradSmem, s>>>(params, x, y, idx, n, partial, lp);
    if (cudaGetLastError() != cudaSuccess) return FC_LBM_ERR_CUDA;
    k_mlp_grad_final<<<(kP + 255) / 256, 256, 0, s>>>(partial, lp, kGradBlocks, n, grad, loss);
    return cudaGetLastError() == cudaSuccess ? FC_LBM_OK : FC_LBM_ERR_CUDA;
}

FC_LBM_API int fc_lbm_mlp_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr,
                               float beta1, float beta2, float eps, void* stream) {
    if (!params || !grad || !m || !v || step < 1) return FC_LBM_ERR_INVALID_ARG;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_adam<<<(kP + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? FC_LBM_OK : FC_LBM_ERR_CUDA;
}

}  // extern "C"
