// icb_step1.cuh — the per-step kernel: the engine's step with a stateless
// collision test, for runs that hand the state back every step (the
// engine's per-step loop, icb_config.collision_test = ICB_TEST_PER_STEP).
//
// Every launch advances each ion by n_steps (1 by default) engine steps and
// moves only what a step needs through HBM: positions (3 doubles),
// velocities (3 floats in the float forms) and the flag byte are read and
// written; mass and charge come from the ensemble's species when all its
// ions share them (otherwise from the per-ion arrays); the death and
// arrival times are written only when they happen (an arrival is also
// recorded in the flag byte, so the per-ion arrival time is never read).
// No collision-clock state exists: each step draws Philox(id, step, 0, 0)
// and a candidate occurs with probability Q = A (|v - u| + <|th|>) of the
// current relative speed; the candidate then samples the neutral from the
// size-biased law and accepts with p / (A (|v - u| + |th|)) exactly as the
// per-step clock does (candidate<R, false, COLL>), so the per-step collision
// law is the reference's (HSSCollisionHandler.cpp:331-364) and results do
// not depend on n_steps.
//
// Physics in this kernel: Boris (BorisStrategy.cpp:50-97) in a uniform
// electric field without B, hard-sphere collisions or none, single gas
// with a constant (or axial uniform) flow; the engine's prepare / finalize
// (SimulationEngineLifecycle.cpp:72-195) and the first detector-plane
// crossing.  The host rejects every other configuration for this mode.
#pragma once
#include "icb_step_kernel.cuh"

namespace icb {

constexpr int kStep1Block = 256;
// Resident blocks per SM: 4 (50 % occupancy, <= 64 registers, no spills) in
// the float forms; FP64 needs more registers for the candidate (spills at 64).
template <int PREC>
struct Step1Shape {
    static constexpr int kMinBlocks = PREC == kPrecFP64 ? 2 : 4;
};

template <int PREC, int COLL>
__global__ void __launch_bounds__(kStep1Block, Step1Shape<PREC>::kMinBlocks) k_step1(const __grid_constant__ StepParams p) {
    using R = typename PrecT<PREC>::R;
    using Pos = typename PosOf<PREC>::T;
    constexpr bool kAccumT = PREC == kPrecFP64;   // FP64: the engine clock as the sum t += dt

    const uint64_t i = p.ens_off[0] + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool in_range = i < p.ens_off[p.n_ens];
    uint32_t n_cand = 0, n_coll = 0, n_ovf = 0, n_dead = 0, n_arr = 0;
    const uint8_t flags0 = in_range ? p.flags[i] : static_cast<uint8_t>(0);
    if (flags0 & kFlagActive) {
        int e = 0;
        if (p.n_ens > 1) {
            int lo = 0, hi = static_cast<int>(p.n_ens) - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (p.ens_off[mid] <= i) lo = mid; else hi = mid - 1;
            }
            e = lo;
        }
        const EnsConst& C = p.ens[e];
        Pos x{};
        x.load(p, i);
        R v[3] = {static_cast<const R*>(p.vx)[i], static_cast<const R*>(p.vy)[i], static_cast<const R*>(p.vz)[i]};
        double q, m;
        if (C.sp_m > 0.0) {
            q = C.sp_q;
            m = C.sp_m;
        } else {
            q = p.charge[i];
            m = p.mass[i];
        }
        Consts<R> k;
        load_consts<R, kFieldUniform, false>(k, C, q, m);
        const double dt = C.dt;
        const double t0 = p.t_dev[p.ens_base + static_cast<uint32_t>(e)];
        const uint32_t step0 = static_cast<uint32_t>(*p.step_dev);
        const uint32_t id = static_cast<uint32_t>(p.first_id + i);
        PhiloxIon pq{};
        if constexpr (COLL != kCollNone) pq = philox_ion_setup(id, p.rk);
        uint8_t flags = flags0;
        double tdeath = -1.0, tarr = -1.0;
        double t = t0;
        bool live = true;
        auto kill = [&](double when) {
            flags &= static_cast<uint8_t>(~kFlagActive);
            tdeath = when;
            live = false;
            ++n_dead;
        };
        if (!inside(C, x)) kill(t0);            // prepare_ions_for_integration
        for (uint32_t kk = 0; live && kk < p.n_steps; ++kk) {
            const double ts = kAccumT ? t : fma(static_cast<double>(kk), dt, t0);
            const double zo = x.gz();
            boris<R, kFieldUniform, false>(k, x, v, ts);
            if constexpr (COLL == kCollHSS) {
                const uint32_t gs = step0 + kk;
                const R wx = v[0] - k.ug[0], wy = v[1] - k.ug[1], wz = v[2] - k.ug[2];
                const R b = m_sqrt(wx * wx + wy * wy + wz * wz);
                R Q = k.A * b + k.Amean;
                if (Q > R(1)) { Q = R(1); ++n_ovf; }
                const U4 r0 = philox_ion(pq, gs, 0u, p.rk);
                if (u32(r0.x, R(0)) < Q) {
                    ++n_cand;
                    R clk;
                    const int st = candidate<R, false, kCollHSS>(C, v, clk, R(0), k.Amean, b, m, p.rk, id, gs, p,
                                                                 nullptr, p.ens_base + static_cast<uint32_t>(e), pq);
                    if (st >= 2) ++n_coll;
                }
            }
            x.fold();
            // finalize_ions_after_integration and the detector plane
            const double zn = x.gz();
            if (!(flags & kFlagArrived) && zo < C.zdet && zn >= C.zdet) {
                tarr = ts + dt * ((C.zdet - zo) / (zn - zo));
                flags |= kFlagArrived;
                ++n_arr;
            }
            if (!inside(C, x) || !(x.finite() && isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) kill(ts);
            if (kAccumT) t = t + dt;
        }
        x.store(p, i);
        static_cast<R*>(p.vx)[i] = v[0];
        static_cast<R*>(p.vy)[i] = v[1];
        static_cast<R*>(p.vz)[i] = v[2];
        if (flags != flags0) p.flags[i] = flags;
        if (tdeath >= 0.0) p.t_death[i] = tdeath;
        if (tarr >= 0.0) p.t_arr[i] = tarr;
    }
    const unsigned long long s0 = warp_sum_u32(n_cand), s1 = warp_sum_u32(n_coll), s2 = warp_sum_u32(n_ovf);
    const unsigned long long s3 = warp_sum_u32(n_dead), s4 = warp_sum_u32(n_arr);
    if ((threadIdx.x & 31u) == 0u) {
        if (s0) atomicAdd(&p.counters[kCntCandidates], s0);
        if (s1) atomicAdd(&p.counters[kCntCollisions], s1);
        if (s2) atomicAdd(&p.counters[kCntOverflow], s2);
        if (s3) atomicAdd(&p.counters[kCntDeaths], s3);
        if (s4) atomicAdd(&p.counters[kCntArrivals], s4);
    }
}

template <int PREC>
cudaError_t launch_step1(int coll, const StepParams& p, dim3 grid, cudaStream_t s) {
    const dim3 block(kStep1Block);
    if (coll == kCollNone) k_step1<PREC, kCollNone><<<grid, block, 0, s>>>(p);
    else if (coll == kCollHSS) k_step1<PREC, kCollHSS><<<grid, block, 0, s>>>(p);
    else return cudaErrorNotSupported;
    return cudaGetLastError();
}

}  // namespace icb
