// icb_mlp.cuh — the learned deflection network (2 -> 64 -> 64 -> 1, tanh)
// evaluated by one warp on the tensor cores: the warp's requesting lanes are
// the rows of m16 tiles; layer 1 is 8 mma.sync.m16n8k16 (inputs and bias
// as BF16 hi/lo pairs), the 64x64 layer 8 n-tiles x 4 k-steps of them (BF16
// operands, FP32 accumulation).
//
// Parameter block (FP32): W1[64][2] at 0, b1 at 128, W2[64][64] at 192
// (W2[n][k] feeds h1[k] into h2[n]), b2 at 4288, W3 at 4352, b3 at 4416.
// The collision path reads W2 as pre-packed B fragments:
// frag[((nt * 4 + ks) * 32 + lane) * 2 + {0, 1}] holds the BF16 pairs
// (W2[8nt+g][16ks+2t], W2[8nt+g][16ks+2t+1]) and (.. +8, .. +9),
// g = lane / 4, t = lane % 4 (the PTX m16n8k16 ".col" B layout); after them
// frag[kMlpFragW1Off + nt * 32 + lane] holds layer 1's B fragment word of
// hidden unit n = 8nt + g (rows 2t, 2t + 1 of B1): t = 0 (W1[n][0],
// W1[n][0]), t = 1 (W1[n][1], W1[n][1]), t = 2 (b1[n] hi, b1[n] lo), t = 3
// zero (rows 8-15 are zero).  The small parameters come from a float
// block: W1 (128), b1 (64), b2 (64), W3 (64), b3 (1), all already rounded
// to BF16 values except the biases.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace icb {

constexpr int kMlpH = 64;
constexpr int kMlpParams = 4417;
constexpr int kMlpOffW1 = 0, kMlpOffB1 = 128, kMlpOffW2 = 192, kMlpOffB2 = 4288, kMlpOffW3 = 4352, kMlpOffB3 = 4416;
// float block of the collision path
constexpr int kMlpFW1 = 0, kMlpFB1 = 128, kMlpFB2 = 192, kMlpFW3 = 256, kMlpFB3 = 320, kMlpFSize = 321;
// W2 as B fragments (8 n-tiles x 4 k-steps x 32 lanes x 2 words), then the
// layer-1 B fragments (8 n-tiles x 32 lanes x 1 word, see mlp_warp_eval)
constexpr int kMlpFragW2Words = 8 * 4 * 32 * 2;
constexpr int kMlpFragW1Off = kMlpFragW2Words;
constexpr int kMlpFragWords = kMlpFragW2Words + 8 * 32;

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

// x as the pair (hi, lo) of BF16 values with hi + lo = x to ~2^-16
// relative: a product with a BF16 weight summed over both is exact in FP32.
__device__ __forceinline__ uint32_t pack_bf16_hilo(float x) {
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
    return static_cast<uint32_t>(__bfloat16_as_ushort(hi)) | (static_cast<uint32_t>(__bfloat16_as_ushort(lo)) << 16);
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
        // Layer 1 on the tensor cores: one m16n8k16 per 8 hidden units with
        // A1 row = [x0 hi, x0 lo, x1 hi, x1 lo, 1, 1, 0 ...] and B1 column n =
        // [W1[n][0] twice, W1[n][1] twice, b1[n] hi, b1[n] lo, 0 ...] (BF16
        // pairs, FP32 accumulation: W1 x + b1 to ~2^-16).  The C fragments of
        // n-tiles 2 ks and 2 ks + 1 (rows g, g + 8; columns 2t, 2t + 1) are
        // the A fragment of k-step ks of the 64 x 64 layer after tanh.
        uint32_t a1f[4] = {0u, 0u, 0u, 0u};
        if (t == 0) { a1f[0] = pack_bf16_hilo(xa0); a1f[1] = pack_bf16_hilo(xb0); }
        else if (t == 1) { a1f[0] = pack_bf16_hilo(xa1); a1f[1] = pack_bf16_hilo(xb1); }
        else if (t == 2) { a1f[0] = 0x3F803F80u; a1f[1] = 0x3F803F80u; }   // (1, 1)
        uint32_t a[4][4];
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            float d0[4] = {0.f, 0.f, 0.f, 0.f}, d1[4] = {0.f, 0.f, 0.f, 0.f};
            mma_bf16_16816(d0, a1f, __ldg(frag + kMlpFragW1Off + (2 * ks) * 32 + lane), 0u);
            mma_bf16_16816(d1, a1f, __ldg(frag + kMlpFragW1Off + (2 * ks + 1) * 32 + lane), 0u);
            a[ks][0] = pack_bf16(tanh_fast(d0[0]), tanh_fast(d0[1]));   // row g,     k 16ks + 2t, +1
            a[ks][1] = pack_bf16(tanh_fast(d0[2]), tanh_fast(d0[3]));   // row g + 8
            a[ks][2] = pack_bf16(tanh_fast(d1[0]), tanh_fast(d1[1]));   // row g,     k 16ks + 8 + 2t, +1
            a[ks][3] = pack_bf16(tanh_fast(d1[2]), tanh_fast(d1[3]));   // row g + 8
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
