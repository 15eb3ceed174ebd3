// icb_mathcheck.cu — device evaluation of the float clock functions of the
// step kernel (-ln(1 - q) and 1 - e^-x, own series plus hardware log/exp)
// next to CUDA's log1pf / expm1f, compiled with the mixed kernel's flags
// (-use_fast_math), so tests can bound the kernel's forms against CUDA's.
#include <cuda_runtime.h>

#include "../../include/icarion_b200.h"
#include "icb_step_kernel.cuh"

namespace {
__global__ void k_clock_math(uint64_t n, const float* __restrict__ x, int which, float* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = x[i];
    float r;
    switch (which) {
        case ICB_MATH_NEG_LOG1M: r = icb::m_neg_log1m(v); break;
        case ICB_MATH_NEG_LOG1M_CUDA: r = -log1pf(-v); break;
        case ICB_MATH_ONE_MINUS_EXP: r = icb::m_one_minus_exp(v); break;
        default: r = -expm1f(-v); break;
    }
    out[i] = r;
}
}  // namespace

extern "C" int icb_clock_math_eval(int device, uint64_t n, const float* x, int which, float* out) {
    if (!x || !out || n == 0 || which < ICB_MATH_NEG_LOG1M || which > ICB_MATH_ONE_MINUS_EXP_CUDA)
        return ICB_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return ICB_ERR_NO_DEVICE;
    float *dx = nullptr, *dout = nullptr;
    const size_t bytes = n * sizeof(float);
    if (cudaMalloc(&dx, bytes) != cudaSuccess) return ICB_ERR_OUT_OF_MEMORY;
    if (cudaMalloc(&dout, bytes) != cudaSuccess) { cudaFree(dx); return ICB_ERR_OUT_OF_MEMORY; }
    int rc = ICB_OK;
    if (cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice) != cudaSuccess) rc = ICB_ERR_CUDA;
    if (rc == ICB_OK) {
        k_clock_math<<<static_cast<unsigned>((n + 255) / 256), 256>>>(n, dx, which, dout);
        if (cudaGetLastError() != cudaSuccess) rc = ICB_ERR_CUDA;
    }
    if (rc == ICB_OK && cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) rc = ICB_ERR_CUDA;
    cudaFree(dx);
    cudaFree(dout);
    return rc;
}
