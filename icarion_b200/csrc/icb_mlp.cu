// icb_mlp.cu — training and evaluation of the learned deflection network
// (2 -> 64 -> 64 -> 1, tanh; parameter layout in icb_mlp.cuh).
//
// Training: Adam on the mean squared error, mini-batches drawn from a
// per-epoch permutation.  One block of 128 threads takes 128 samples of the
// batch: the forward pass keeps h1 and h2 per sample in shared memory, the
// backward pass forms the block's share of every gradient (dW2 as the
// 64 x 64 product D2^T H1 over the block's samples); partial gradients land
// in a [blocks][4417] buffer that one thread per parameter sums in block
// order (deterministic) before its Adam update.  With bf16_forward the
// forward pass rounds weights and the first hidden layer to BF16 exactly as
// the collision path does (quantisation-aware; gradients pass straight
// through the rounding).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/icarion_b200.h"
#include "icb_internal.h"
#include "icb_mlp.cuh"

namespace icb {

namespace {

constexpr int kTB = 128;     // samples per training block
constexpr int kLd = kMlpH + 1;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Forward of one sample in FP32 arithmetic (optionally with BF16-rounded
// weights and first-layer activations); h1, h2 receive the activations.
template <bool BF16>
__device__ float mlp_forward_one(const float* w, float x0, float x1, float* h1, float* h2) {
    for (int c = 0; c < kMlpH; ++c) {
        float w0 = w[kMlpOffW1 + 2 * c], w1 = w[kMlpOffW1 + 2 * c + 1];
        if (BF16) { w0 = bf16r(w0); w1 = bf16r(w1); }
        float a = tanhf(fmaf(w0, x0, fmaf(w1, x1, w[kMlpOffB1 + c])));
        if (BF16) a = bf16r(a);
        h1[c] = a;
    }
    float y = w[kMlpOffB3];
    for (int n = 0; n < kMlpH; ++n) {
        float acc = 0.f;
        const float* row = w + kMlpOffW2 + n * kMlpH;
        for (int k = 0; k < kMlpH; ++k) acc = fmaf(BF16 ? bf16r(row[k]) : row[k], h1[k], acc);
        const float a = tanhf(acc + w[kMlpOffB2 + n]);
        h2[n] = a;
        y = fmaf(BF16 ? bf16r(w[kMlpOffW3 + n]) : w[kMlpOffW3 + n], a, y);
    }
    return y;
}

template <bool BF16>
__global__ void __launch_bounds__(kTB) k_mlp_fwdbwd(const float* __restrict__ params, const float* __restrict__ x,
                                                    const float* __restrict__ y, const uint32_t* __restrict__ perm,
                                                    uint64_t first, uint32_t count, float inv_batch,
                                                    float* __restrict__ partial, double* __restrict__ loss_partial) {
    extern __shared__ float sm[];
    float* w = sm;                               // kMlpParams
    float* H1 = w + kMlpParams + 3;              // [kTB][kLd]
    float* H2 = H1 + kTB * kLd;                  // [kTB][kLd] (holds D2 after the backward step)
    float* dout = H2 + kTB * kLd;                // [kTB]
    float* xs = dout + kTB;                      // [kTB][2]
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) w[k] = params[k];
    __syncthreads();
    const uint32_t local = blockIdx.x * kTB + threadIdx.x;
    const bool valid = local < count;
    float e = 0.f;
    float* h1 = H1 + threadIdx.x * kLd;
    float* h2 = H2 + threadIdx.x * kLd;
    if (valid) {
        const uint32_t sidx = perm ? perm[first + local] : static_cast<uint32_t>(first + local);
        const float x0 = x[2 * static_cast<size_t>(sidx)], x1 = x[2 * static_cast<size_t>(sidx) + 1];
        xs[2 * threadIdx.x] = x0;
        xs[2 * threadIdx.x + 1] = x1;
        const float out = mlp_forward_one<BF16>(w, x0, x1, h1, h2);
        e = out - y[sidx];
        dout[threadIdx.x] = 2.f * e * inv_batch;
    } else {
        xs[2 * threadIdx.x] = 0.f;
        xs[2 * threadIdx.x + 1] = 0.f;
        dout[threadIdx.x] = 0.f;
        for (int c = 0; c < kMlpH; ++c) { h1[c] = 0.f; h2[c] = 0.f; }
    }
    __syncthreads();
    float* g = partial + static_cast<size_t>(blockIdx.x) * kMlpParams;
    // dW3, db2-side: dW3[n] = sum_s dout h2[n]
    if (threadIdx.x < kMlpH) {
        float acc = 0.f;
        for (int s = 0; s < kTB; ++s) acc = fmaf(dout[s], H2[s * kLd + threadIdx.x], acc);
        g[kMlpOffW3 + threadIdx.x] = acc;
    }
    if (threadIdx.x == kMlpH) {
        float acc = 0.f;
        for (int s = 0; s < kTB; ++s) acc += dout[s];
        g[kMlpOffB3] = acc;
    }
    __syncthreads();
    // D2[n] = dout W3[n] (1 - h2^2), in place of h2
    {
        const float d = dout[threadIdx.x];
        for (int n = 0; n < kMlpH; ++n) {
            const float a = h2[n];
            h2[n] = d * w[kMlpOffW3 + n] * (1.f - a * a);
        }
    }
    __syncthreads();
    // dW2[n][k] = sum_s D2[s][n] H1[s][k]; db2[n] = sum_s D2[s][n]
    for (int e2 = threadIdx.x; e2 < kMlpH * kMlpH; e2 += blockDim.x) {
        const int n = e2 / kMlpH, k = e2 % kMlpH;
        float acc = 0.f;
        for (int s = 0; s < kTB; ++s) acc = fmaf(H2[s * kLd + n], H1[s * kLd + k], acc);
        g[kMlpOffW2 + e2] = acc;
    }
    if (threadIdx.x < kMlpH) {
        float acc = 0.f;
        for (int s = 0; s < kTB; ++s) acc += H2[s * kLd + threadIdx.x];
        g[kMlpOffB2 + threadIdx.x] = acc;
    }
    __syncthreads();
    // D1[k] = (1 - h1^2) sum_n D2[n] W2[n][k], in place of h1
    {
        float d1[kMlpH];
        for (int k = 0; k < kMlpH; ++k) d1[k] = 0.f;
        for (int n = 0; n < kMlpH; ++n) {
            const float dn = h2[n];
            const float* row = w + kMlpOffW2 + n * kMlpH;
            for (int k = 0; k < kMlpH; ++k) d1[k] = fmaf(dn, row[k], d1[k]);
        }
        for (int k = 0; k < kMlpH; ++k) {
            const float a = h1[k];
            d1[k] *= (1.f - a * a);
        }
        __syncthreads();
        for (int k = 0; k < kMlpH; ++k) h1[k] = d1[k];
    }
    __syncthreads();
    // dW1[k][j] = sum_s D1[s][k] x_j; db1[k] = sum_s D1[s][k]
    if (threadIdx.x < kMlpH) {
        const int k = threadIdx.x;
        float a0 = 0.f, a1 = 0.f, ab = 0.f;
        for (int s = 0; s < kTB; ++s) {
            const float d = H1[s * kLd + k];
            a0 = fmaf(d, xs[2 * s], a0);
            a1 = fmaf(d, xs[2 * s + 1], a1);
            ab += d;
        }
        g[kMlpOffW1 + 2 * k] = a0;
        g[kMlpOffW1 + 2 * k + 1] = a1;
        g[kMlpOffB1 + k] = ab;
    }
    // block loss: sum of squared errors (thread order)
    __shared__ double red[kTB];
    red[threadIdx.x] = static_cast<double>(e) * e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
        for (int s = 0; s < kTB; ++s) acc += red[s];
        loss_partial[blockIdx.x] = acc;
    }
}

struct AdamState {
    float lr, b1, b2, eps, c1, c2;   // c1 = 1/(1-b1^t), c2 = 1/(1-b2^t)
};

// Sum the blocks' partial gradients in block order, then one Adam step.
__global__ void k_mlp_adam(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ partial, int nblocks, AdamState a,
                           const double* __restrict__ loss_partial, double* __restrict__ loss_acc) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) {
        double l = 0.0;
        for (int b = 0; b < nblocks; ++b) l += loss_partial[b];
        *loss_acc += l;
    }
    if (p >= kMlpParams) return;
    float gsum = 0.f;
    for (int b = 0; b < nblocks; ++b) gsum += partial[static_cast<size_t>(b) * kMlpParams + p];
    const float mm = a.b1 * m[p] + (1.f - a.b1) * gsum;
    const float vv = a.b2 * v[p] + (1.f - a.b2) * gsum * gsum;
    m[p] = mm;
    v[p] = vv;
    params[p] -= a.lr * (mm * a.c1) / (sqrtf(vv * a.c2) + a.eps);
}

__global__ void k_mlp_sum_grad(const float* __restrict__ partial, int nblocks, float* __restrict__ grad,
                               const double* __restrict__ loss_partial, double* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) {
        double l = 0.0;
        for (int b = 0; b < nblocks; ++b) l += loss_partial[b];
        *loss = l;
    }
    if (p >= kMlpParams) return;
    float gsum = 0.f;
    for (int b = 0; b < nblocks; ++b) gsum += partial[static_cast<size_t>(b) * kMlpParams + p];
    grad[p] = gsum;
}

__global__ void k_mlp_forward_fp32(const float* __restrict__ params, uint64_t n, const float* __restrict__ x,
                                   float* __restrict__ y) {
    __shared__ float w[kMlpParams];
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) w[k] = params[k];
    __syncthreads();
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float h1[kMlpH], h2[kMlpH];
    y[i] = mlp_forward_one<false>(w, x[2 * i], x[2 * i + 1], h1, h2);
}

// The collision path's evaluation: each warp takes 32 consecutive samples.
__global__ void k_mlp_forward_mma(const uint32_t* __restrict__ frag, const float* __restrict__ f, uint64_t n,
                                  const float* __restrict__ x, float* __restrict__ y) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool want = i < n;
    const float x0 = want ? x[2 * i] : 0.f, x1 = want ? x[2 * i + 1] : 0.f;
    const float out = mlp_warp_eval(frag, f, x0, x1, want);
    if (want) y[i] = out;
}

float bf16_round_host(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;       // inf / nan unchanged
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;                                    // round to nearest even
    u &= 0xffff0000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

uint32_t bf16_bits_host(float x) {
    const float r = bf16_round_host(x);
    uint32_t u;
    std::memcpy(&u, &r, 4);
    return u >> 16;
}

template <class T>
struct DevVec {
    T* p = nullptr;
    ~DevVec() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)); }
};

}  // namespace

// Collision-path parameter blocks: B fragments of W2 (BF16 pairs) and the
// float block (W1, W3 rounded to BF16; biases FP32).
void mlp_pack(const float* params, std::vector<uint32_t>& frag, std::vector<float>& fblock) {
    frag.assign(kMlpFragWords, 0u);
    // W2 as A fragments of m-tile mt (units 16mt..16mt+15) and k-step ks
    auto pair = [&](int n, int k) {
        const float* row = params + kMlpOffW2 + n * kMlpH;
        return bf16_bits_host(row[k]) | (bf16_bits_host(row[k + 1]) << 16);
    };
    for (int mt = 0; mt < 4; ++mt)
        for (int ks = 0; ks < 4; ++ks)
            for (int lane = 0; lane < 32; ++lane) {
                const int g = lane >> 2, t = lane & 3;
                const int n0 = 16 * mt + g, n1 = n0 + 8;
                const int k0 = 16 * ks + 2 * t, k1 = k0 + 8;
                const size_t base = (static_cast<size_t>(mt * 4 + ks) * 32 + lane) * 4;
                frag[base] = pair(n0, k0);
                frag[base + 1] = pair(n1, k0);
                frag[base + 2] = pair(n0, k1);
                frag[base + 3] = pair(n1, k1);
            }
    // layer 1 as A fragments: rows h of [W1[h][0] twice, W1[h][1] twice,
    // b1[h] hi, b1[h] lo, 0 ...], words for rows 16mt+g and 16mt+g+8
    auto l1 = [&](int h, int t) {
        if (t < 2) {
            const uint32_t b = bf16_bits_host(params[kMlpOffW1 + 2 * h + t]);
            return b | (b << 16);
        }
        if (t == 2) {
            const float b1 = params[kMlpOffB1 + h];
            const float hi = bf16_round_host(b1);
            return bf16_bits_host(hi) | (bf16_bits_host(b1 - hi) << 16);
        }
        return 0u;
    };
    for (int mt = 0; mt < 4; ++mt)
        for (int lane = 0; lane < 32; ++lane) {
            const int g = lane >> 2, t = lane & 3;
            const size_t base = static_cast<size_t>(kMlpFragW1Off) + (static_cast<size_t>(mt) * 32 + lane) * 2;
            frag[base] = l1(16 * mt + g, t);
            frag[base + 1] = l1(16 * mt + g + 8, t);
        }
    fblock.assign(kMlpFSize, 0.f);
    for (int k = 0; k < 128; ++k) fblock[kMlpFW1 + k] = bf16_round_host(params[kMlpOffW1 + k]);
    for (int k = 0; k < kMlpH; ++k) {
        fblock[kMlpFB1 + k] = params[kMlpOffB1 + k];
        fblock[kMlpFB2 + k] = params[kMlpOffB2 + k];
        fblock[kMlpFW3 + k] = bf16_round_host(params[kMlpOffW3 + k]);
    }
    fblock[kMlpFB3] = params[kMlpOffB3];
}

}  // namespace icb

using namespace icb;

#define MLP_CUDA(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            return set_error(e_ == cudaErrorMemoryAllocation ? ICB_ERR_OUT_OF_MEMORY : ICB_ERR_CUDA, \
                             (std::string(#expr) + ": " + cudaGetErrorString(e_)).c_str());        \
        }                                                                                \
    } while (0)

extern "C" {

int icb_mlp_init(uint64_t seed, float* params) {
    if (!params) return set_error(ICB_ERR_INVALID_ARGUMENT, "null params");
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::fill(params, params + kMlpParams, 0.f);
    const double a1 = std::sqrt(6.0 / (2 + kMlpH)), a2 = std::sqrt(6.0 / (kMlpH + kMlpH)), a3 = std::sqrt(6.0 / (kMlpH + 1));
    for (int k = 0; k < 128; ++k) params[kMlpOffW1 + k] = static_cast<float>(a1 * u(rng));
    for (int k = 0; k < kMlpH * kMlpH; ++k) params[kMlpOffW2 + k] = static_cast<float>(a2 * u(rng));
    for (int k = 0; k < kMlpH; ++k) params[kMlpOffW3 + k] = static_cast<float>(a3 * u(rng));
    return ICB_OK;
}

static size_t fwdbwd_smem() {
    return (kMlpParams + 3 + 2 * kTB * kLd + kTB + 2 * kTB) * sizeof(float);
}

static int launch_fwdbwd(bool bf16, const float* params, const float* x, const float* y, const uint32_t* perm,
                         uint64_t first, uint32_t count, float inv_batch, float* partial, double* loss_partial,
                         int nblocks, cudaStream_t s) {
    const size_t smem = fwdbwd_smem();
    if (bf16) {
        MLP_CUDA(cudaFuncSetAttribute(k_mlp_fwdbwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)));
        k_mlp_fwdbwd<true><<<nblocks, kTB, smem, s>>>(params, x, y, perm, first, count, inv_batch, partial,
                                                      loss_partial);
    } else {
        MLP_CUDA(cudaFuncSetAttribute(k_mlp_fwdbwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)));
        k_mlp_fwdbwd<false><<<nblocks, kTB, smem, s>>>(params, x, y, perm, first, count, inv_batch, partial,
                                                       loss_partial);
    }
    MLP_CUDA(cudaGetLastError());
    return ICB_OK;
}

int icb_mlp_train(int device, const icb_mlp_train_config* cfg, uint64_t n, const float* x, const float* y,
                  float* params, double* loss_per_epoch) {
    if (!cfg || !x || !y || !params) return set_error(ICB_ERR_INVALID_ARGUMENT, "null argument");
    if (cfg->epochs < 1 || cfg->batch < 1 || cfg->batch > (1 << 20) || n < static_cast<uint64_t>(cfg->batch) ||
        n >= (1ull << 32))
        return set_error(ICB_ERR_INVALID_ARGUMENT, "need epochs >= 1, 1 <= batch <= min(n, 2^20), n < 2^32");
    if (!(cfg->lr > 0.0) || !(cfg->lr_min >= 0.0)) return set_error(ICB_ERR_INVALID_ARGUMENT, "bad learning rate");
    MLP_CUDA(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    MLP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamDestroy(s); } } guard{s};
    const uint32_t B = static_cast<uint32_t>(cfg->batch);
    const int nblocks = static_cast<int>((B + kTB - 1) / kTB);
    DevVec<float> dx, dy, dp, dm, dv, dpart;
    DevVec<uint32_t> dperm;
    DevVec<double> dlp, dloss;
    MLP_CUDA(dx.alloc(2 * n));
    MLP_CUDA(dy.alloc(n));
    MLP_CUDA(dp.alloc(kMlpParams));
    MLP_CUDA(dm.alloc(kMlpParams));
    MLP_CUDA(dv.alloc(kMlpParams));
    MLP_CUDA(dpart.alloc(static_cast<size_t>(nblocks) * kMlpParams));
    MLP_CUDA(dperm.alloc(n));
    MLP_CUDA(dlp.alloc(nblocks));
    MLP_CUDA(dloss.alloc(1));
    MLP_CUDA(cudaMemcpyAsync(dx.p, x, 2 * n * sizeof(float), cudaMemcpyHostToDevice, s));
    MLP_CUDA(cudaMemcpyAsync(dy.p, y, n * sizeof(float), cudaMemcpyHostToDevice, s));
    MLP_CUDA(cudaMemcpyAsync(dp.p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, s));
    MLP_CUDA(cudaMemsetAsync(dm.p, 0, kMlpParams * sizeof(float), s));
    MLP_CUDA(cudaMemsetAsync(dv.p, 0, kMlpParams * sizeof(float), s));
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::mt19937_64 rng(cfg->seed ^ 0x9e3779b97f4a7c15ull);
    const uint64_t steps_per_epoch = n / B;
    const uint64_t total = steps_per_epoch * static_cast<uint64_t>(cfg->epochs);
    const double b1 = 0.9, b2 = 0.999;
    double b1t = 1.0, b2t = 1.0;
    uint64_t step = 0;
    for (int ep = 0; ep < cfg->epochs; ++ep) {
        // Fisher-Yates with the generator's raw 64-bit output
        for (uint64_t i = n - 1; i > 0; --i) {
            const uint64_t j = rng() % (i + 1);
            std::swap(perm[i], perm[j]);
        }
        MLP_CUDA(cudaMemcpyAsync(dperm.p, perm.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        MLP_CUDA(cudaMemsetAsync(dloss.p, 0, sizeof(double), s));
        for (uint64_t k = 0; k < steps_per_epoch; ++k, ++step) {
            if (int r = launch_fwdbwd(cfg->bf16_forward != 0, dp.p, dx.p, dy.p, dperm.p, k * B, B, 1.f / B, dpart.p,
                                      dlp.p, nblocks, s))
                return r;
            b1t *= b1;
            b2t *= b2;
            const double frac = static_cast<double>(step) / static_cast<double>(total);
            const double lr = cfg->lr_min + 0.5 * (cfg->lr - cfg->lr_min) * (1.0 + std::cos(M_PI * frac));
            AdamState a{static_cast<float>(lr), static_cast<float>(b1), static_cast<float>(b2), 1e-8f,
                        static_cast<float>(1.0 / (1.0 - b1t)), static_cast<float>(1.0 / (1.0 - b2t))};
            k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(dp.p, dm.p, dv.p, dpart.p, nblocks, a, dlp.p,
                                                                dloss.p);
            MLP_CUDA(cudaGetLastError());
        }
        double l = 0.0;
        MLP_CUDA(cudaMemcpyAsync(&l, dloss.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        MLP_CUDA(cudaStreamSynchronize(s));
        if (loss_per_epoch) loss_per_epoch[ep] = l / static_cast<double>(steps_per_epoch * B);
    }
    MLP_CUDA(cudaMemcpyAsync(params, dp.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, s));
    MLP_CUDA(cudaStreamSynchronize(s));
    return ICB_OK;
}

int icb_mlp_forward(int device, const float* params, uint64_t n, const float* x, float* y, int mode) {
    if (!params || (n > 0 && (!x || !y))) return set_error(ICB_ERR_INVALID_ARGUMENT, "null argument");
    if (mode != 0 && mode != 1) return set_error(ICB_ERR_INVALID_ARGUMENT, "mode must be 0 (FP32) or 1 (BF16 MMA)");
    if (n == 0) return ICB_OK;
    MLP_CUDA(cudaSetDevice(device));
    DevVec<float> dx, dy, dp, df;
    DevVec<uint32_t> dfrag;
    MLP_CUDA(dx.alloc(2 * n));
    MLP_CUDA(dy.alloc(n));
    MLP_CUDA(cudaMemcpy(dx.p, x, 2 * n * sizeof(float), cudaMemcpyHostToDevice));
    const unsigned blocks = static_cast<unsigned>((n + 127) / 128);
    if (mode == 0) {
        MLP_CUDA(dp.alloc(kMlpParams));
        MLP_CUDA(cudaMemcpy(dp.p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
        k_mlp_forward_fp32<<<blocks, 128>>>(dp.p, n, dx.p, dy.p);
    } else {
        std::vector<uint32_t> frag;
        std::vector<float> fb;
        mlp_pack(params, frag, fb);
        MLP_CUDA(dfrag.alloc(frag.size()));
        MLP_CUDA(df.alloc(fb.size()));
        MLP_CUDA(cudaMemcpy(dfrag.p, frag.data(), frag.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        MLP_CUDA(cudaMemcpy(df.p, fb.data(), fb.size() * sizeof(float), cudaMemcpyHostToDevice));
        k_mlp_forward_mma<<<blocks, 128>>>(dfrag.p, df.p, n, dx.p, dy.p);
    }
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaMemcpy(y, dy.p, n * sizeof(float), cudaMemcpyDeviceToHost));
    return ICB_OK;
}

int icb_mlp_gradients(int device, const float* params, uint64_t n, const float* x, const float* y, float* grad,
                      double* loss) {
    if (!params || !x || !y || !grad) return set_error(ICB_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0 || n > (1u << 20)) return set_error(ICB_ERR_INVALID_ARGUMENT, "need 1 <= n <= 2^20");
    MLP_CUDA(cudaSetDevice(device));
    const int nblocks = static_cast<int>((n + kTB - 1) / kTB);
    DevVec<float> dx, dy, dp, dpart, dg;
    DevVec<double> dlp, dl;
    MLP_CUDA(dx.alloc(2 * n));
    MLP_CUDA(dy.alloc(n));
    MLP_CUDA(dp.alloc(kMlpParams));
    MLP_CUDA(dpart.alloc(static_cast<size_t>(nblocks) * kMlpParams));
    MLP_CUDA(dg.alloc(kMlpParams));
    MLP_CUDA(dlp.alloc(nblocks));
    MLP_CUDA(dl.alloc(1));
    MLP_CUDA(cudaMemcpy(dx.p, x, 2 * n * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(dy.p, y, n * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(dp.p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
    if (int r = launch_fwdbwd(false, dp.p, dx.p, dy.p, nullptr, 0, static_cast<uint32_t>(n), 1.f / n, dpart.p,
                              dlp.p, nblocks, nullptr))
        return r;
    k_mlp_sum_grad<<<(kMlpParams + 255) / 256, 256>>>(dpart.p, nblocks, dg.p, dlp.p, dl.p);
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaMemcpy(grad, dg.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
    double l = 0.0;
    MLP_CUDA(cudaMemcpy(&l, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
    if (loss) *loss = l / static_cast<double>(n);
    return ICB_OK;
}

}  // extern "C"
