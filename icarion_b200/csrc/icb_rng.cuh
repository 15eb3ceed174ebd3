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

// The candidate draws of one ion: counter (id, step, s, 0) for s = 0, 1.
// The first round depends on the step only through c1, and the second
// round's multiply of c2 only on the ion, so both are formed once per ion:
// after round 0 the state is (w_s ^ step, lo(M1 s), hi(M0 id) ^ rk1,
// lo(M0 id)) with w_s = hi(M1 s) ^ rk0; round 1 then needs one multiply.
// philox_ion(pre, step, s) equals philox4x32_10_rk(id, step, s, 0, rk).
struct PhiloxIon {
    uint32_t x1[2];   // round-1 outputs c0 = hi(M1 c2_1) ^ lo(M1 s) ^ rk2, s = 0, 1
    uint32_t y1;      // c1 = lo(M1 c2_1)
    uint32_t z1;      // lo(M0 id) ^ rk3 (folds into c2 of round 1)
};

ICB_HD PhiloxIon philox_ion_setup(uint32_t id, const uint32_t* rk) {
    PhiloxIon q;
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * id;
    const uint32_t c2_1 = static_cast<uint32_t>(p0 >> 32) ^ rk[1];
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2_1;
    for (uint32_t s = 0; s < 2; ++s) {
        const uint32_t lo_s = static_cast<uint32_t>(static_cast<uint64_t>(0xCD9E8D57u) * s);
        q.x1[s] = static_cast<uint32_t>(p1 >> 32) ^ lo_s ^ rk[2];
    }
    q.y1 = static_cast<uint32_t>(p1);
    q.z1 = static_cast<uint32_t>(p0) ^ rk[3];
    return q;
}

ICB_HD U4 philox_ion(const PhiloxIon& q, uint32_t step, uint32_t s, const uint32_t* rk) {
    // round 0: c0 = hi(M1 s) ^ step ^ rk0 (the only step-dependent word)
    const uint32_t hi_s = static_cast<uint32_t>((static_cast<uint64_t>(0xCD9E8D57u) * s) >> 32);
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * (hi_s ^ step ^ rk[0]);
    // round 1
    uint32_t c0 = q.x1[s], c1 = q.y1;
    uint32_t c2 = static_cast<uint32_t>(p0 >> 32) ^ q.z1, c3 = static_cast<uint32_t>(p0);
#pragma unroll
    for (int r = 2; r < 10; ++r) {
        const uint64_t a = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t b = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        c0 = static_cast<uint32_t>(b >> 32) ^ c1 ^ rk[2 * r];
        c1 = static_cast<uint32_t>(b);
        c2 = static_cast<uint32_t>(a >> 32) ^ c3 ^ rk[2 * r + 1];
        c3 = static_cast<uint32_t>(a);
    }
    return U4{c0, c1, c2, c3};
}

// 32-bit word -> double in (0, 1]: (w + 1) * 2^-32, exact.
ICB_HD double unit_d(uint32_t w) { return (static_cast<double>(w) + 1.0) * 2.3283064365386963e-10; }
// 32-bit word -> float in (0, 1]: (top 24 bits + 1) * 2^-24, exact.
ICB_HD float unit_f(uint32_t w) { return static_cast<float>((w >> 8) + 1u) * 5.9604644775390625e-08f; }

}  // namespace icb
