// icb_mlp.cuh — the learned deflection network (2 -> 64 -> 64 -> 1, tanh)
// evaluated by one warp on the tensor cores: the warp's requesting lanes are
// the rows of m16 tiles, the 64x64 layer is 8 n-tiles x 4 k-steps of
// mma.sync.m16n8k16 (BF16 operands, FP32 accumulation).
//
// Parameter block (FP32): W1[64][2] at 0, b1 at 128, W2[64][64] at 192
// (W2[n][k] feeds h1[k] into h2[n]), b2 at 4288, W3 at 4352, b3 at 4416.
// The collision path reads W2 as pre-packed B fragments:
// frag[((nt * 4 + ks) * 32 + lane) * 2 + {0, 1}] holds the BF16 pairs
// (W2[8nt+g][16ks+2t], W2[8nt+g][16ks+2t+1]) and (.. +8, .. +9),
// g = lane / 4, t = lane % 4 (the PTX m16n8k16 ".col" B layout), and the
// small parameters from a float block: W1 (128), b1 (64), b2 (64), W3 (64),
// b3 (1), all already rounded to BF16 values except the biases.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace icb {

constexpr int kMlpH = 64;
constexpr int kMlpParams = 4417;
constexpr int kMlpOffW1 = 0, kMlpOffB1 = 128, kMlpOffW2 = 192, kMlpOffB2 = 4288, kMlpOffW3 = 4352, kMlpOffB3 = 4416;
// float block of the collision path
constexpr int kMlpFW1 = 0, kMlpFB1 = 128, kMlpFB2 = 192, kMlpFW3 = 256, kMlpFB3 = 320, kMlpFSize = 321;
constexpr int kMlpFragWords = 8 * 4 * 32 * 2;

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Lane index of the (r+1)-th set bit of mask (r < popc(mask)).
__device__ __forceinline__ int nth_set_lane(unsigned mask, int r) {
    for (int i = 0; i < r; ++i) mask &= mask - 1u;
    return __ffs(static_cast<int>(mask)) - 1;
}

// Network output for every lane with want = true (rows in lane order, 16 per
// tile); other lanes get 0.  All 32 lanes must call it together.
__device__ __forceinline__ float mlp_warp_eval(const uint32_t* __restrict__ frag, const float* __restrict__ f,
                                               float x0, float x1, bool want) {
    const unsigned full = 0xffffffffu;
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int g = lane >> 2, t = lane & 3;
    const unsigned mask = __ballot_sync(full, want);
    const int nrows = __popc(mask);
    const int rank = __popc(mask & ((1u << lane) - 1u));
    float mine = 0.f;
    for (int base = 0; base < nrows; base += 16) {
        // rows g and g + 8 of this tile: their inputs from the owning lanes
        const bool v0 = base + g < nrows, v1 = base + g + 8 < nrows;
        const int l0 = v0 ? nth_set_lane(mask, base + g) : lane;
        const int l1 = v1 ? nth_set_lane(mask, base + g + 8) : lane;
        const float xa0 = __shfl_sync(full, x0, l0), xa1 = __shfl_sync(full, x1, l0);
        const float xb0 = __shfl_sync(full, x0, l1), xb1 = __shfl_sync(full, x1, l1);
        // layer 1 straight into the A fragments (4 k-steps of 16 columns)
        uint32_t a[4][4];
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int c = 16 * ks + 2 * t + 8 * half;
                const float w00 = f[kMlpFW1 + 2 * c], w01 = f[kMlpFW1 + 2 * c + 1];
                const float w10 = f[kMlpFW1 + 2 * c + 2], w11 = f[kMlpFW1 + 2 * c + 3];
                const float bb0 = f[kMlpFB1 + c], bb1 = f[kMlpFB1 + c + 1];
                const float h00 = tanh_fast(fmaf(w00, xa0, fmaf(w01, xa1, bb0)));
                const float h01 = tanh_fast(fmaf(w10, xa0, fmaf(w11, xa1, bb1)));
                const float h10 = tanh_fast(fmaf(w00, xb0, fmaf(w01, xb1, bb0)));
                const float h11 = tanh_fast(fmaf(w10, xb0, fmaf(w11, xb1, bb1)));
                a[ks][2 * half + 0] = pack_bf16(h00, h01);   // row g
                a[ks][2 * half + 1] = pack_bf16(h10, h11);   // row g + 8
            }
        }
        // A register order of m16n8k16: {row g, k 0-7}, {row g+8, k 0-7},
        // {row g, k 8-15}, {row g+8, k 8-15}
        float y0 = 0.f, y1 = 0.f;
#pragma unroll 2
        for (int nt = 0; nt < 8; ++nt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const uint2 bw = __ldg(reinterpret_cast<const uint2*>(frag) + (nt * 4 + ks) * 32 + lane);
                const uint32_t af[4] = {a[ks][0], a[ks][1], a[ks][2], a[ks][3]};
                mma_bf16_16816(d, af, bw.x, bw.y);
            }
            const int c = 8 * nt + 2 * t;
            const float b20 = f[kMlpFB2 + c], b21 = f[kMlpFB2 + c + 1];
            const float w30 = f[kMlpFW3 + c], w31 = f[kMlpFW3 + c + 1];
            y0 = fmaf(w30, tanh_fast(d[0] + b20), fmaf(w31, tanh_fast(d[1] + b21), y0));
            y1 = fmaf(w30, tanh_fast(d[2] + b20), fmaf(w31, tanh_fast(d[3] + b21), y1));
        }
        // sum over the four lanes of the group: row g in y0, row g + 8 in y1
        y0 += __shfl_xor_sync(full, y0, 1);
        y0 += __shfl_xor_sync(full, y0, 2);
        y1 += __shfl_xor_sync(full, y1, 1);
        y1 += __shfl_xor_sync(full, y1, 2);
        const float b3 = f[kMlpFB3];
        // row r of the tile lives in group r (y0) or group r - 8 (y1)
        const int r = rank - base;
        const int src = (r >= 0 && r < 16) ? 4 * (r & 7) : 0;
        const float got0 = __shfl_sync(full, y0, src);
        const float got1 = __shfl_sync(full, y1, src);
        if (want && r >= 0 && r < 16) mine = (r < 8 ? got0 : got1) + b3;
    }
    return mine;
}

}  // namespace icb
