// icb_mlp.cuh — the learned deflection network (2 -> 64 -> 64 -> 1, tanh)
// evaluated by one warp on the tensor cores, with the network's units as
// the MMA rows and up to 8 samples (the warp's requesting lanes) as the
// columns: every layer is D[units x 8] = W[units x k] . H[k x 8] with
// mma.sync.m16n8k16 (BF16 operands, FP32 accumulation).  Layer 1 is 4 MMAs
// (inputs and bias as BF16 hi/lo pairs: W1 x + b1 to ~2^-16), the 64x64
// layer 16; each lane applies tanh to 16 + 16 values per pass of 8 samples,
// so a warp event with few colliding lanes (the common case) does half the
// work of a 16-row tile.  Layer 1's C fragments become layer 2's B
// fragments through movmatrix (an 8x8 transpose in registers).
//
// Parameter block (FP32): W1[64][2] at 0, b1 at 128, W2[64][64] at 192
// (W2[n][k] feeds h1[k] into h2[n]), b2 at 4288, W3 at 4352, b3 at 4416.
// The collision path reads the weights as pre-packed A fragments (g = lane
// / 4, t = lane % 4, the PTX m16n8k16 ".row" A layout):
//   frag[((mt * 4 + ks) * 32 + lane) * 4 + {0, 1, 2, 3}]: the BF16 pairs
//     (W2[16mt+g][16ks+2t], .. +1), (W2[16mt+g+8][16ks+2t], .. +1),
//     (W2[16mt+g][16ks+8+2t], .. +1), (W2[16mt+g+8][16ks+8+2t], .. +1);
//   frag[kMlpFragW1Off + (mt * 32 + lane) * 2 + {0, 1}]: layer 1's rows
//     16mt+g and 16mt+g+8 of [W1[h][0] twice, W1[h][1] twice, b1[h] hi,
//     b1[h] lo, 0 ...]: t = 0 (W1[h][0], W1[h][0]), t = 1 (W1[h][1],
//     W1[h][1]), t = 2 (b1 hi, b1 lo), t = 3 zero (columns 8-15 are zero);
// and the small parameters from a float block: W1 (128), b1 (64), b2 (64),
// W3 (64), b3 (1), all already rounded to BF16 values except the biases.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace icb {

constexpr int kMlpH = 64;
constexpr int kMlpParams = 4417;
constexpr int kMlpOffW1 = 0, kMlpOffB1 = 128, kMlpOffW2 = 192, kMlpOffB2 = 4288, kMlpOffW3 = 4352, kMlpOffB3 = 4416;
// float block of the collision path
constexpr int kMlpFW1 = 0, kMlpFB1 = 128, kMlpFB2 = 192, kMlpFW3 = 256, kMlpFB3 = 320, kMlpFSize = 321;
// W2 as A fragments (4 m-tiles x 4 k-steps x 32 lanes x 4 words), then
// layer 1's A fragments (4 m-tiles x 32 lanes x 2 words)
constexpr int kMlpFragW2Words = 4 * 4 * 32 * 4;
constexpr int kMlpFragW1Off = kMlpFragW2Words;
constexpr int kMlpFragWords = kMlpFragW2Words + 4 * 32 * 2;

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

// 8x8 BF16 transpose across the warp: lane (g, t) holds row g, columns 2t,
// 2t + 1 before and row g of the transpose after (PTX movmatrix).
__device__ __forceinline__ uint32_t movmatrix_trans(uint32_t a) {
    uint32_t d;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;\n" : "=r"(d) : "r"(a));
    return d;
}

// Lane index of the (r+1)-th set bit of mask (r < popc(mask)).
__device__ __forceinline__ int nth_set_lane(unsigned mask, int r) {
    for (int i = 0; i < r; ++i) mask &= mask - 1u;
    return __ffs(static_cast<int>(mask)) - 1;
}

// Network output for every lane with want = true (samples in lane order, 8
// per pass); other lanes get 0.  All 32 lanes must call it together.
__device__ __forceinline__ float mlp_warp_eval(const uint32_t* __restrict__ frag, const float* __restrict__ f,
                                               float x0, float x1, bool want) {
    const unsigned full = 0xffffffffu;
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int g = lane >> 2, t = lane & 3;
    const unsigned mask = __ballot_sync(full, want);
    const int nrows = __popc(mask);
    const int rank = __popc(mask & ((1u << lane) - 1u));
    float mine = 0.f;
    for (int base = 0; base < nrows; base += 8) {
        // sample g of this pass (column g): its inputs from the owning lane
        const bool valid = base + g < nrows;
        const int src = valid ? nth_set_lane(mask, base + g) : lane;
        const float s0 = __shfl_sync(full, x0, src), s1 = __shfl_sync(full, x1, src);
        // layer 1: B1[k][sample g] = [x0 hi, x0 lo, x1 hi, x1 lo, 1, 1, 0 ...]
        uint32_t b1w = 0u;
        if (t == 0) b1w = pack_bf16_hilo(s0);
        else if (t == 1) b1w = pack_bf16_hilo(s1);
        else if (t == 2) b1w = 0x3F803F80u;   // (1, 1)
        // h1 = tanh(W1 x + b1) as layer 2's B fragments: k-step ks takes
        // units 16ks..16ks+15, the transposes of m-tile ks's two halves
        uint32_t hb[4][2];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
            const uint2 aw = __ldg(reinterpret_cast<const uint2*>(frag + kMlpFragW1Off) + mt * 32 + lane);
            const uint32_t a1f[4] = {aw.x, aw.y, 0u, 0u};
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            mma_bf16_16816(d, a1f, b1w, 0u);
            hb[mt][0] = movmatrix_trans(pack_bf16(tanh_fast(d[0]), tanh_fast(d[1])));   // units 16mt + 0..7
            hb[mt][1] = movmatrix_trans(pack_bf16(tanh_fast(d[2]), tanh_fast(d[3])));   // units 16mt + 8..15
        }
        // layer 2 and the W3 dot product: lane (g, t) holds units 16mt + g
        // and 16mt + g + 8 of samples 2t and 2t + 1
        float ye = 0.f, yo = 0.f;
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const uint4 aw = __ldg(reinterpret_cast<const uint4*>(frag) + (mt * 4 + ks) * 32 + lane);
                const uint32_t af[4] = {aw.x, aw.y, aw.z, aw.w};
                mma_bf16_16816(d, af, hb[ks][0], hb[ks][1]);
            }
            const int h0 = 16 * mt + g, h1 = h0 + 8;
            const float b20 = f[kMlpFB2 + h0], b21 = f[kMlpFB2 + h1];
            const float w30 = f[kMlpFW3 + h0], w31 = f[kMlpFW3 + h1];
            ye = fmaf(w30, tanh_fast(d[0] + b20), fmaf(w31, tanh_fast(d[2] + b21), ye));
            yo = fmaf(w30, tanh_fast(d[1] + b20), fmaf(w31, tanh_fast(d[3] + b21), yo));
        }
        // sum over the 8 unit groups g (lanes t, t + 4, ..., t + 28)
        ye += __shfl_xor_sync(full, ye, 4);
        ye += __shfl_xor_sync(full, ye, 8);
        ye += __shfl_xor_sync(full, ye, 16);
        yo += __shfl_xor_sync(full, yo, 4);
        yo += __shfl_xor_sync(full, yo, 8);
        yo += __shfl_xor_sync(full, yo, 16);
        const float b3 = f[kMlpFB3];
        // sample r of the pass is column r: lane r / 2, even or odd
        const int r = rank - base;
        const int from = (r >= 0 && r < 8) ? (r >> 1) : 0;
        const float ge = __shfl_sync(full, ye, from);
        const float go = __shfl_sync(full, yo, from);
        if (want && r >= 0 && r < 8) mine = ((r & 1) ? go : ge) + b3;
    }
    return mine;
}

}  // namespace icb
