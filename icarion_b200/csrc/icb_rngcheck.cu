// icb_rngcheck.cu — device evaluation of the counter-based RNG, used to pin
// the kernel's Philox4x32-10 against the CPU restatement and against
// cuRAND's independent implementation of the same published generator.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include "../../include/icarion_b200.h"
#include "icb_rng.cuh"

namespace {
__global__ void k_philox(uint64_t n, const uint32_t* __restrict__ ctr, uint32_t k0, uint32_t k1, int use_curand,
                         uint32_t* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t* c = ctr + 4 * i;
    uint32_t* o = out + 4 * i;
    if (use_curand) {
        const uint4 r = curand_Philox4x32_10(make_uint4(c[0], c[1], c[2], c[3]), make_uint2(k0, k1));
        o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w;
    } else {
        const icb::U4 r = icb::philox4x32_10(c[0], c[1], c[2], c[3], k0, k1);
        o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w;
    }
}
}  // namespace

extern "C" int icb_philox_eval(int device, uint64_t n, const uint32_t* counters, uint64_t seed, int use_curand,
                               uint32_t* out) {
    if (!counters || !out || n == 0) return ICB_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return ICB_ERR_NO_DEVICE;
    uint32_t *dc = nullptr, *dout = nullptr;
    const size_t bytes = n * 4 * sizeof(uint32_t);
    if (cudaMalloc(&dc, bytes) != cudaSuccess) return ICB_ERR_OUT_OF_MEMORY;
    if (cudaMalloc(&dout, bytes) != cudaSuccess) { cudaFree(dc); return ICB_ERR_OUT_OF_MEMORY; }
    int rc = ICB_OK;
    if (cudaMemcpy(dc, counters, bytes, cudaMemcpyHostToDevice) != cudaSuccess) rc = ICB_ERR_CUDA;
    if (rc == ICB_OK) {
        k_philox<<<static_cast<unsigned>((n + 255) / 256), 256>>>(n, dc, static_cast<uint32_t>(seed),
                                                                  static_cast<uint32_t>(seed >> 32), use_curand, dout);
        if (cudaGetLastError() != cudaSuccess) rc = ICB_ERR_CUDA;
    }
    if (rc == ICB_OK && cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) rc = ICB_ERR_CUDA;
    cudaFree(dc);
    cudaFree(dout);
    return rc;
}
