// icb_rng.cuh — counter-based Philox4x32-10 and uniform conversions.
//
// Philox4x32-10 restated from Salmon, Moraes, Dror, Shaw, "Parallel Random
// Numbers: As Easy as 1, 2, 3" (SC'11).  Stateless: every draw is a pure
// function of (key, counter), so no RNG state lives in HBM and a resumed or
// re-sharded run reproduces the same numbers.  This replaces the reference's
// per-ion std::mt19937_64 pool (CollisionTypes.h:31-49, RngUtils.cpp:51-118).
//
// Stream layout (shared with the CPU oracle):
//   key     = (lo32(rng_seed), hi32(rng_seed))
//   counter = (ion id, step index, substream, 0)
//   substream 0..2: the draws of a collision candidate at that step,
//   substream 3 at step 0: the initial uniform of the collision clock.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define ICB_HD __host__ __device__ __forceinline__
#else
#define ICB_HD inline
#endif

namespace icb {

struct U4 { uint32_t x, y, z, w; };

ICB_HD U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return U4{c0, c1, c2, c3};
}

// Round keys (k0 + r W0, k1 + r W1), r = 0..9, of a fixed key: computed
// once per launch so the rounds need no key arithmetic.
inline void philox_round_keys(uint64_t seed, uint32_t rk[20]) {
    uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        rk[2 * r] = k0;
        rk[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Philox4x32-10 with precomputed round keys; identical output to
// philox4x32_10(c, k0, k1).
ICB_HD U4 philox4x32_10_rk(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, const uint32_t* rk) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        c0 = hi1 ^ c1 ^ rk[2 * r];
        c1 = lo1;
        c2 = hi0 ^ c3 ^ rk[2 * r + 1];
        c3 = lo0;
    }
    return U4{c0, c1, c2, c3};
}

// 32-bit word -> double in (0, 1]: (w + 1) * 2^-32, exact.
ICB_HD double unit_d(uint32_t w) { return (static_cast<double>(w) + 1.0) * 2.3283064365386963e-10; }
// 32-bit word -> float in (0, 1]: (top 24 bits + 1) * 2^-24, exact.
ICB_HD float unit_f(uint32_t w) { return static_cast<float>((w >> 8) + 1u) * 5.9604644775390625e-08f; }

}  // namespace icb
