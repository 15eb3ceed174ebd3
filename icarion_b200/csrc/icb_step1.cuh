// icb_step1.cuh — the per-step kernel: the engine's step with a stateless
// collision test, for runs that hand the state back every step (the
// engine's per-step loop, icb_config.collision_test = ICB_TEST_PER_STEP).
//
// Every launch advances each ion by n_steps (1 by default) engine steps and
// moves only what a step needs through HBM: positions (3 doubles, or 6
// floats in the hi/lo form), velocities (3 floats in the float forms) and
// the flag byte are read and written; mass and charge come from the
// ensemble's species when all its ions share them (otherwise from the
// per-ion arrays); the death and arrival times are written only when they
// happen (an arrival is also recorded in the flag byte, so the per-ion
// arrival time is never read).  No collision-clock state exists: each step
// draws one Philox2x32-10 word of (step, id) (step_test_word) and a
// candidate occurs with probability
// Q = A (|v - u| + <|th|>) of the current relative speed; the candidate then
// samples the neutral from the size-biased law and accepts with
// p / (A (|v - u| + |th|)) exactly as the per-step clock does
// (candidate<R, false, COLL>), so the per-step collision law is the
// reference's (HSSCollisionHandler.cpp:331-364) and results do not depend on
// n_steps.
//
// Layout of the work.  The ions are cut into tiles of 256 (absolute index
// k*256 .. k*256+255); each CTA owns one ion per thread of a tile and walks
// the tiles k = first + blockIdx.x + it * gridDim.x of the launch's range,
// with a grid of (resident CTAs per SM) x SMs.  A tile's state arrives in
// shared memory by bulk copies (cp.async.bulk, one per array, completed on
// the stage's mbarrier) issued two tiles ahead, so the loads of
// later tiles are in flight while this one computes and the number of
// bytes in flight does not depend on registers.  Tiles cut by the range's
// ends load with ordinary per-thread loads.  Each step runs in three
// phases: every live ion pushes and draws its test; the candidates are
// queued in shared memory and handled one per thread (a tile has ~9 % of
// candidates, so one warp does the candidate work of eight, instead of
// every warp running it for its one or two lanes); then every ion takes
// back its velocity and finalizes.  Results go straight to global memory
// from registers.
//
// Physics in this kernel: Boris (BorisStrategy.cpp:50-97) in a uniform
// electric field without B, hard-sphere collisions or none, single gas
// with a constant (or axial uniform) flow; the engine's prepare / finalize
// (SimulationEngineLifecycle.cpp:72-195) and the first detector-plane
// crossing.  The host rejects every other configuration for this mode.
#pragma once
#include <atomic>

#include "icb_bulk.cuh"
#include "icb_step_kernel.cuh"

namespace icb {

constexpr int kStep1Block = 256;    // ions per tile = threads per CTA
static_assert(kStep1Block == 256, "tile index arithmetic shifts by 8");
// Tiles loaded ahead per CTA (9.5 KB each in the float forms, 12.5 KB in
// FP64).  Two keep the copies ahead of the push: four measured the same
// (0.348 vs 0.342 ms per 16.8M-ion step), and five CTAs per SM with 40
// registers measured 0.369 ms.
// The per-step collision test's word: Philox2x32-10 (Salmon et al., SC'11;
// multiplier 0xD256D193, key bump 0x9E3779B9) of the counter (step, ion id)
// under the key seed_lo ^ seed_hi (rk[0], rk[1] are the seed's words),
// first output word.  A candidate then draws its Philox4x32-10 blocks
// (id, step, 0 | 1) as the clock form's candidates do.  The first round's
// product depends on the step alone: one value for every ion of a launch.
__device__ __forceinline__ uint32_t step_test_word(uint32_t step, uint32_t id, const uint32_t* rk) {
    uint32_t c0 = step, c1 = id, k = rk[0] ^ rk[1];
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi = __umulhi(0xD256D193u, c0), lo = 0xD256D193u * c0;
        c0 = hi ^ k ^ c1;
        c1 = lo;
        k += 0x9E3779B9u;
    }
    return c0;
}

template <int PREC>
struct Step1Stages {
    static constexpr int kN = 2;
};

// Resident CTAs per SM the register budget is built for.
template <int PREC>
struct Step1Shape {
    static constexpr int kMinBlocks = PREC == kPrecFP64 ? 2 : 4;
};

// Position of the mixed form in the one-step kernel: the double position
// itself.  A step adds (double) fmaf(v, dt, 0) per axis, the value the fused
// kernel's anchor + float offset folds to, without the offset's
// bookkeeping (one step per launch leaves nothing to accumulate).
struct PosS {
    double x, y, z;
    __device__ void load(const StepParams& p, uint64_t i) { x = p.x[i]; y = p.y[i]; z = p.z[i]; }
    __device__ void store(const StepParams& p, uint64_t i) const { p.x[i] = x; p.y[i] = y; p.z[i] = z; }
    __device__ double gx() const { return x; }
    __device__ double gy() const { return y; }
    __device__ double gz() const { return z; }
    __device__ void fold() {}
    __device__ void drift(float vx, float vy, float vz, double, float d) {
        x += static_cast<double>(fmaf(vx, d, 0.0f));
        y += static_cast<double>(fmaf(vy, d, 0.0f));
        z += static_cast<double>(fmaf(vz, d, 0.0f));
    }
    __device__ bool finite() const { return isfinite(x) && isfinite(y) && isfinite(z); }
};
template <int PREC> struct Step1Pos { using T = typename PosOf<PREC>::T; };
template <> struct Step1Pos<kPrecMixed> { using T = PosS; };

// Shared-memory image of one tile: position arrays, velocity arrays, flags.
template <int PREC>
struct Step1Stage {
    using R = typename PrecT<PREC>::R;
    static constexpr int kPosArrays = PREC == kPrecHiLo ? 6 : 3;
    static constexpr int kPosElem = PREC == kPrecHiLo ? 4 : 8;
    static constexpr int kPosBytes = kPosElem * kStep1Block;              // per array
    static constexpr int kVelOff = kPosArrays * kPosBytes;
    static constexpr int kVelBytes = static_cast<int>(sizeof(R)) * kStep1Block;
    static constexpr int kFlagOff = kVelOff + 3 * kVelBytes;
    static constexpr int kBytes = kFlagOff + kStep1Block;
    static_assert(kPosBytes % 16 == 0 && kVelBytes % 16 == 0 && kBytes % 16 == 0, "bulk copy sizes");
};

template <int PREC>
__device__ __forceinline__ void step1_issue(const StepParams& p, uint64_t i0, unsigned char* st, uint64_t* bar) {
    using S = Step1Stage<PREC>;
    using R = typename S::R;
    mbar_arrive_expect_tx(bar, S::kBytes);
    if constexpr (PREC == kPrecHiLo) {
        const float* src[6] = {p.xh, p.xl, p.yh, p.yl, p.zh, p.zl};
#pragma unroll
        for (int a = 0; a < 6; ++a) bulk_g2s(st + a * S::kPosBytes, src[a] + i0, S::kPosBytes, bar);
    } else {
        const double* src[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) bulk_g2s(st + a * S::kPosBytes, src[a] + i0, S::kPosBytes, bar);
    }
    const R* vs[3] = {static_cast<const R*>(p.vx), static_cast<const R*>(p.vy), static_cast<const R*>(p.vz)};
#pragma unroll
    for (int a = 0; a < 3; ++a) bulk_g2s(st + S::kVelOff + a * S::kVelBytes, vs[a] + i0, S::kVelBytes, bar);
    bulk_g2s(st + S::kFlagOff, p.flags + i0, kStep1Block, bar);
}

template <int PREC, class Pos>
__device__ __forceinline__ void step1_pos_from_stage(Pos& x, const unsigned char* st, int j) {
    if constexpr (PREC == kPrecHiLo) {
        const float* f = reinterpret_cast<const float*>(st);
        x.xh = f[j]; x.xl = f[kStep1Block + j];
        x.yh = f[2 * kStep1Block + j]; x.yl = f[3 * kStep1Block + j];
        x.zh = f[4 * kStep1Block + j]; x.zl = f[5 * kStep1Block + j];
    } else {
        const double* d = reinterpret_cast<const double*>(st);
        x.x = d[j]; x.y = d[kStep1Block + j]; x.z = d[2 * kStep1Block + j];
    }
}

// The push and collision-test constants of an ion: from the ensemble's
// species (the host's copy of load_consts' arithmetic) when all its ions
// share mass and charge, else by load_consts from the ion's own.
template <class R>
__device__ __forceinline__ void step1_consts(Consts<R>& k, const EnsConst& C, const StepParams& p, uint64_t i) {
    if (C.sp_m > 0.0) {
        k.dt = C.dt;
        if constexpr (sizeof(R) == 8) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                k.a_uni[a] = C.sp_a64[a];
                k.ug[a] = C.ug[a];
            }
            k.h = C.dt * 0.5;
            k.dt_r = C.dt;
            k.A = C.A;
            k.Amean = C.A * C.mean_th;
        } else {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                k.a_uni[a] = C.sp_fa[a];
                k.ug[a] = C.fug[a];
            }
            k.h = C.sp_fh;
            k.dt_r = C.sp_fdt;
            k.A = C.fA;
            k.Amean = C.sp_fAmean;
        }
    } else {
        load_consts<R, kFieldUniform, false>(k, C, p.charge[i], p.mass[i]);
    }
}

__device__ __forceinline__ int step1_ensemble(const StepParams& p, uint64_t i) {
    int lo = 0, hi = static_cast<int>(p.n_ens) - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.ens_off[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int PREC, int COLL>
__global__ void __launch_bounds__(kStep1Block, Step1Shape<PREC>::kMinBlocks) k_step1(const __grid_constant__ StepParams p) {
    using R = typename PrecT<PREC>::R;
    using Pos = typename Step1Pos<PREC>::T;
    using S = Step1Stage<PREC>;
    constexpr bool kAccumT = PREC == kPrecFP64;   // FP64: the engine clock as the sum t += dt
    constexpr bool kColl = COLL == kCollHSS;
    constexpr int kStep1Stages = Step1Stages<PREC>::kN;

    __shared__ __align__(128) unsigned char stage[kStep1Stages][S::kBytes];
    __shared__ __align__(8) uint64_t bar[kStep1Stages];
    __shared__ R cv[2][3][kStep1Block];          // queued candidates' velocities (two passes)
    __shared__ uint16_t cj[2][kStep1Block];      // ... and their thread in the tile
    __shared__ int n_c[2];

    const int j = static_cast<int>(threadIdx.x);
    const uint64_t b = p.ens_off[0], en = p.ens_off[p.n_ens];
    const uint64_t kb = b / kStep1Block;
    const uint64_t n_tiles = (en + kStep1Block - 1) / kStep1Block - kb;
    const uint64_t n_it = blockIdx.x < n_tiles ? (n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    if (n_it == 0) return;
    auto tile_of = [&](uint64_t it) { return kb + blockIdx.x + it * gridDim.x; };
    // a tile wholly inside the range loads by bulk copies
    auto staged = [&](uint64_t k) { return k * kStep1Block >= b && (k + 1) * kStep1Block <= en; };

    if (j == 0) {
#pragma unroll
        for (int s = 0; s < kStep1Stages; ++s) mbar_init(&bar[s], 1u);
        fence_mbar_init();
        n_c[0] = n_c[1] = 0;
    }
    __syncthreads();
    // per stage: fills issued and fills consumed (every thread keeps the
    // same counts; thread 0 issues)
    uint32_t issued[kStep1Stages], uses[kStep1Stages];
#pragma unroll
    for (int s = 0; s < kStep1Stages; ++s) {
        issued[s] = uses[s] = 0u;
        if (static_cast<uint64_t>(s) < n_it && staged(tile_of(s))) {
            if (j == 0) step1_issue<PREC>(p, tile_of(s) * kStep1Block, stage[s], &bar[s]);
            issued[s] = 1u;
        }
    }
    bool stop = false;

    const uint32_t step0 = static_cast<uint32_t>(*p.step_dev);
    uint32_t n_cand = 0, n_coll = 0, n_ovf = 0, n_dead = 0, n_arr = 0;
    uint32_t pass = 0;                            // candidate passes so far (queue parity)

    for (uint64_t it = 0; it < n_it; ++it) {
        const int s = static_cast<int>(it % kStep1Stages);
        const uint64_t k = tile_of(it);
        const uint64_t i = k * kStep1Block + static_cast<uint64_t>(j);
        const bool bulk = staged(k);
        const bool in_range = i >= b && i < en;
        bool my_stall = false;
        if (bulk) {
#pragma unroll
            for (int q = 0; q < kStep1Stages; ++q)
                if (q == s) {
                    my_stall = !mbar_wait_bounded(&bar[q], uses[q] & 1u);
                    ++uses[q];
                }
        }
        uint8_t flags0 = 0;
        Pos x{};
        R v[3] = {R(0), R(0), R(0)};
        if (bulk) {
            const unsigned char* st = stage[s];
            flags0 = st[S::kFlagOff + j];
            if (flags0 & kFlagActive) {
                step1_pos_from_stage<PREC>(x, st, j);
                const R* vv = reinterpret_cast<const R*>(st + S::kVelOff);
                v[0] = vv[j]; v[1] = vv[kStep1Block + j]; v[2] = vv[2 * kStep1Block + j];
            }
        } else if (in_range) {
            flags0 = p.flags[i];
            if (flags0 & kFlagActive) {
                x.load(p, i);
                v[0] = static_cast<const R*>(p.vx)[i];
                v[1] = static_cast<const R*>(p.vy)[i];
                v[2] = static_cast<const R*>(p.vz)[i];
            }
        }
        // stage s has been read; a wait that gave up anywhere stops the CTA
        if (__syncthreads_or(my_stall ? 1 : 0)) {
            stop = true;
            break;
        }
        if (it + kStep1Stages < n_it && staged(tile_of(it + kStep1Stages))) {
            if (j == 0) {
                fence_proxy_async();
                step1_issue<PREC>(p, tile_of(it + kStep1Stages) * kStep1Block, stage[s], &bar[s]);
            }
#pragma unroll
            for (int q = 0; q < kStep1Stages; ++q)
                if (q == s) ++issued[q];
        }

        bool live = (flags0 & kFlagActive) != 0;
        const int e = (live && p.n_ens > 1) ? step1_ensemble(p, i) : 0;
        const EnsConst& C = p.ens[e];
        Consts<R> kc;
        if (live) step1_consts<R>(kc, C, p, i);
        const double dt = C.dt;
        const double t0 = p.t_dev[p.ens_base + static_cast<uint32_t>(e)];
        const uint32_t id = static_cast<uint32_t>(p.first_id + i);
        uint8_t flags = flags0;
        double t = t0;
        // death and arrival times are stored when they happen
        auto kill = [&](double when) {
            flags &= static_cast<uint8_t>(~kFlagActive);
            p.t_death[i] = when;
            live = false;
            ++n_dead;
        };
        if (live && !p.skip_prepare && !inside(C, x)) kill(t0);   // prepare_ions_for_integration
        for (uint32_t kk = 0; kk < p.n_steps; ++kk) {
            const uint32_t gs = step0 + kk;
            bool out = false;                     // outside the domain or non-finite after the push
            int slot = -1;
            if (live) {
                const double ts = kAccumT ? t : fma(static_cast<double>(kk), dt, t0);
                const double zo = x.gz();
                boris<R, kFieldUniform, false>(kc, x, v, ts);
                // finalize_ions_after_integration's position half (a
                // collision moves no ion, so it goes first): the detector
                // plane and the domain
                x.fold();
                const double zn = x.gz();
                if (!(flags & kFlagArrived) && zo < C.zdet && zn >= C.zdet) {
                    p.t_arr[i] = ts + dt * ((C.zdet - zo) / (zn - zo));
                    flags |= kFlagArrived;
                    ++n_arr;
                }
                // inside() already fails for non-finite x or y and infinite
                // z; of a non-finite position only a NaN z passes it
                out = !inside(C, x) || isnan(x.gz());
            }
            if constexpr (kColl) {
                const int qp = static_cast<int>(pass & 1u);
                bool cand = false;
                if (live) {
                    const R wx = v[0] - kc.ug[0], wy = v[1] - kc.ug[1], wz = v[2] - kc.ug[2];
                    const R bb = m_sqrt(wx * wx + wy * wy + wz * wz);
                    R Q = kc.A * bb + kc.Amean;
                    if (Q > R(1)) { Q = R(1); ++n_ovf; }
                    cand = u32(step_test_word(gs, id, p.rk), R(0)) < Q;
                }
                // queue the candidates (warp-aggregated slots)
                const unsigned ball = __ballot_sync(0xffffffffu, cand);
                int base = 0;
                if ((j & 31) == 0 && ball) base = atomicAdd(&n_c[qp], __popc(ball));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (cand) {
                    ++n_cand;
                    slot = base + __popc(ball & ((1u << (j & 31)) - 1u));
                    cv[qp][0][slot] = v[0]; cv[qp][1][slot] = v[1]; cv[qp][2][slot] = v[2];
                    cj[qp][slot] = static_cast<uint16_t>(j);
                }
                __syncthreads();
                // one queued candidate per thread
                const int nq = n_c[qp];
                if (j < nq) {
                    const int jj = cj[qp][j];
                    const uint64_t ic = k * kStep1Block + static_cast<uint64_t>(jj);
                    const int ec = p.n_ens > 1 ? step1_ensemble(p, ic) : 0;
                    const EnsConst& Cc = p.ens[ec];
                    const double mc = Cc.sp_m > 0.0 ? Cc.sp_m : p.mass[ic];
                    const uint32_t idc = static_cast<uint32_t>(p.first_id + ic);
                    const PhiloxIon pc = philox_ion_setup(idc, p.rk);
                    R vc[3] = {cv[qp][0][j], cv[qp][1][j], cv[qp][2][j]};
                    const R ug0 = static_cast<R>(Cc.ug[0]), ug1 = static_cast<R>(Cc.ug[1]),
                            ug2 = static_cast<R>(Cc.ug[2]);
                    const R wx = vc[0] - ug0, wy = vc[1] - ug1, wz = vc[2] - ug2;
                    const R bb = m_sqrt(wx * wx + wy * wy + wz * wz);
                    R clk;
                    const int st = candidate<R, false, kCollHSS>(Cc, vc, clk, R(0),
                                                                 static_cast<R>(Cc.A * Cc.mean_th), bb, mc, p.rk,
                                                                 idc, gs, p, nullptr,
                                                                 p.ens_base + static_cast<uint32_t>(ec), pc);
                    if (st >= 2) ++n_coll;
                    cv[qp][0][j] = vc[0]; cv[qp][1][j] = vc[1]; cv[qp][2][j] = vc[2];
                }
                if (j == 0) n_c[qp ^ 1] = 0;      // the next pass's queue
                __syncthreads();
                if (slot >= 0) {
                    v[0] = cv[qp][0][slot]; v[1] = cv[qp][1][slot]; v[2] = cv[qp][2][slot];
                }
                ++pass;
            }
            if (live) {
                // the velocity half of finalize, after the collision
                if (out || !(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2])))
                    kill(kAccumT ? t : fma(static_cast<double>(kk), dt, t0));
                if (kAccumT) t = t + dt;
            }
        }
        if (flags0 & kFlagActive) {
            x.store(p, i);
            static_cast<R*>(p.vx)[i] = v[0];
            static_cast<R*>(p.vy)[i] = v[1];
            static_cast<R*>(p.vz)[i] = v[2];
            if (flags != flags0) p.flags[i] = flags;
        }
    }
    if (stop) {
        // a stage never completed: report it, and let the copies still in
        // flight land (bounded) before the CTA's shared memory goes away
        if (j == 0) {
            atomicAdd(&p.counters[kCntStalls], 1ull);
#pragma unroll
            for (int q = 0; q < kStep1Stages; ++q)
                if (issued[q] != uses[q]) (void)mbar_wait_bounded(&bar[q], uses[q] & 1u);
        }
        return;
    }
    const unsigned long long s0 = warp_sum_u32(n_cand), s1 = warp_sum_u32(n_coll), s2 = warp_sum_u32(n_ovf);
    const unsigned long long s3 = warp_sum_u32(n_dead), s4 = warp_sum_u32(n_arr);
    if ((j & 31) == 0) {
        if (s0) atomicAdd(&p.counters[kCntCandidates], s0);
        if (s1) atomicAdd(&p.counters[kCntCollisions], s1);
        if (s2) atomicAdd(&p.counters[kCntOverflow], s2);
        if (s3) atomicAdd(&p.counters[kCntDeaths], s3);
        if (s4) atomicAdd(&p.counters[kCntArrivals], s4);
    }
}

// ---- the one-step form with collision warps --------------------------------
// One engine step per launch (n_steps = 1, the per-step loop) with
// hard-sphere collisions.  Eight push warps hold a tile (one ion per
// thread): they push, take the detector plane and the domain test, draw the
// collision test and queue the candidates in shared memory; two collision
// warps, each owning every other tile with its queue and stage, work through
// the queues meanwhile (the candidate law of the block-synchronous kernel
// above, then the velocity half of finalize and the stores of the candidate
// ions) and refill their stages.  Full and empty queues are mbarriers (eight arrivals
// / one).  A push warp reads its tile's stage before it arrives on the
// tile's full queue, so once a collision warp has that queue the stage is
// free and it issues the stage's next fill: no warp waits for another's
// stage reads or for the candidate chain of its own tile.  Every wait is
// bounded; a wait that gives up sets the CTA's abort flag, which every
// other wait polls, and the CTA reports a stall and returns once its copies
// have landed.
constexpr int kStep1WsPush = 8;
constexpr int kStep1WsColl = 2;          // collision warps: warp w takes the tiles it with it % 2 == w
constexpr int kStep1WsThreads = 32 * (kStep1WsPush + kStep1WsColl);
static_assert(kStep1WsPush * 32 == kStep1Block, "one push thread per ion of a tile");
constexpr uint8_t kQueueOut = 0x80u;    // queue flag bit: the position failed finalize

template <int PREC>
struct Step1WsShape {
    static constexpr int kMinBlocks = PREC == kPrecFP64 ? 2 : 3;
};

template <int PREC, bool ONE>
__global__ void __launch_bounds__(kStep1WsThreads, Step1WsShape<PREC>::kMinBlocks)
    k_step1_ws(const __grid_constant__ StepParams p) {
    using R = typename PrecT<PREC>::R;
    using Pos = typename Step1Pos<PREC>::T;
    using S = Step1Stage<PREC>;
    constexpr int kStep1Stages = Step1Stages<PREC>::kN;

    __shared__ __align__(128) unsigned char stage[kStep1Stages][S::kBytes];
    __shared__ __align__(8) uint64_t bar[kStep1Stages];
    __shared__ __align__(8) uint64_t q_full[2];
    __shared__ __align__(8) uint64_t q_empty[2];
    __shared__ R qv[2][3][kStep1Block];           // candidates' velocities after the push
    __shared__ uint16_t qj[2][kStep1Block];       // ... their ion in the tile
    __shared__ uint8_t qf[2][kStep1Block];        // ... their flags after the push (+ kQueueOut)
    __shared__ int qn[2];
    __shared__ int abort_flag;

    const int tid = static_cast<int>(threadIdx.x);
    const int warp = tid >> 5, lane = tid & 31;
    const unsigned full = 0xffffffffu;
    const uint64_t b = p.ens_off[0], en = p.ens_off[p.n_ens];
    const uint64_t kb = b / kStep1Block;
    const uint64_t n_tiles = (en + kStep1Block - 1) / kStep1Block - kb;
    const uint64_t n_it = blockIdx.x < n_tiles ? (n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    if (n_it == 0) return;
    auto tile_of = [&](uint64_t it) { return kb + blockIdx.x + it * gridDim.x; };
    auto staged = [&](uint64_t k) { return k * kStep1Block >= b && (k + 1) * kStep1Block <= en; };
    volatile int* abortp = &abort_flag;

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < kStep1Stages; ++s) mbar_init(&bar[s], 1u);
        mbar_init(&q_full[0], kStep1WsPush); mbar_init(&q_full[1], kStep1WsPush);
        mbar_init(&q_empty[0], 1u); mbar_init(&q_empty[1], 1u);
        fence_mbar_init();
        qn[0] = qn[1] = 0;
        abort_flag = 0;
    }
    __syncthreads();

    const uint32_t step0 = static_cast<uint32_t>(*p.step_dev);
    uint32_t n_cand = 0, n_coll = 0, n_ovf = 0, n_dead = 0, n_arr = 0;

    if (warp >= kStep1WsPush) {
        // ---- the collision warps: warp w takes the tiles (and their queue
        // q = w and stage s = w) of the iterations it = w, w + 2, ...; its
        // lane 0 also fills that stage ----
        static_assert(kStep1WsColl == 2 && Step1Stages<PREC>::kN == 2, "one queue and one stage per collision warp");
        const int w = warp - kStep1WsPush;
        uint32_t fills[kStep1Stages];
#pragma unroll
        for (int s = 0; s < kStep1Stages; ++s) {
            fills[s] = 0u;
            if (s == w && static_cast<uint64_t>(s) < n_it && staged(tile_of(s))) {
                if (lane == 0) step1_issue<PREC>(p, tile_of(s) * kStep1Block, stage[s], &bar[s]);
                fills[s] = 1u;
            }
        }
        for (uint64_t it = static_cast<uint64_t>(w); it < n_it; it += 2) {
            const int q = static_cast<int>(it & 1u);
            const bool got = mbar_wait_or_abort(&q_full[q], static_cast<uint32_t>(it >> 1) & 1u, abortp);
            if (__any_sync(full, !got)) {
                if (lane == 0) *abortp = 1;
                break;
            }
            // every push warp has read tile it's stage: refill it
            const int s = static_cast<int>(it % kStep1Stages);
            if (it + kStep1Stages < n_it && staged(tile_of(it + kStep1Stages))) {
                if (lane == 0) {
                    fence_proxy_async();
                    step1_issue<PREC>(p, tile_of(it + kStep1Stages) * kStep1Block, stage[s], &bar[s]);
                }
#pragma unroll
                for (int qq = 0; qq < kStep1Stages; ++qq)
                    if (qq == s) ++fills[qq];
            }
            const int n = qn[q];
            const uint64_t k = tile_of(it);
            for (int sl = lane; sl < n; sl += 32) {
                const uint64_t ic = k * kStep1Block + static_cast<uint64_t>(qj[q][sl]);
                const int ec = ONE ? 0 : step1_ensemble(p, ic);
                const EnsConst& Cc = p.ens[ec];
                const double mc = Cc.sp_m > 0.0 ? Cc.sp_m : p.mass[ic];
                const uint32_t idc = static_cast<uint32_t>(p.first_id + ic);
                const PhiloxIon pc = philox_ion_setup(idc, p.rk);
                R vc[3] = {qv[q][0][sl], qv[q][1][sl], qv[q][2][sl]};
                const R wx = vc[0] - static_cast<R>(Cc.ug[0]), wy = vc[1] - static_cast<R>(Cc.ug[1]),
                        wz = vc[2] - static_cast<R>(Cc.ug[2]);
                const R bb = m_sqrt(wx * wx + wy * wy + wz * wz);
                R clk;
                const int st = candidate<R, false, kCollHSS>(Cc, vc, clk, R(0), static_cast<R>(Cc.A * Cc.mean_th), bb,
                                                             mc, p.rk, idc, step0, p, nullptr,
                                                             p.ens_base + static_cast<uint32_t>(ec), pc);
                if (st >= 2) ++n_coll;
                // the velocity half of finalize (the step started at t0)
                uint8_t fl = qf[q][sl];
                const bool out = (fl & kQueueOut) != 0;
                fl = static_cast<uint8_t>(fl & ~kQueueOut);
                if (out || !(isfinite(vc[0]) && isfinite(vc[1]) && isfinite(vc[2]))) {
                    fl = static_cast<uint8_t>(fl & ~kFlagActive);
                    p.t_death[ic] = p.t_dev[p.ens_base + static_cast<uint32_t>(ec)];
                    ++n_dead;
                }
                static_cast<R*>(p.vx)[ic] = vc[0];
                static_cast<R*>(p.vy)[ic] = vc[1];
                static_cast<R*>(p.vz)[ic] = vc[2];
                p.flags[ic] = fl;
            }
            __syncwarp();
            if (lane == 0) {
                qn[q] = 0;
                mbar_arrive(&q_empty[q]);
            }
        }
        // the CTA's shared memory must outlive every fill issued (bounded)
        if (lane == 0) {
#pragma unroll
            for (int s = 0; s < kStep1Stages; ++s)
                if (s == w && fills[s] > 0u) (void)mbar_wait_bounded(&bar[s], (fills[s] - 1u) & 1u);
        }
    } else {
        // ---- the push warps ----
        const int j = tid;
        const double t0_one = ONE ? p.t_dev[p.ens_base] : 0.0;   // the launch's clock (one ensemble)
        uint32_t uses[kStep1Stages];
#pragma unroll
        for (int s = 0; s < kStep1Stages; ++s) uses[s] = 0u;
        // tiles wholly inside the range: [k_lo, k_hi)
        const uint64_t k_lo = (b + kStep1Block - 1) / kStep1Block, k_hi = en / kStep1Block;
        uint64_t k = tile_of(0);
        for (uint64_t it = 0; it < n_it; ++it, k += gridDim.x) {
            const int s = static_cast<int>(it % kStep1Stages);
            const uint64_t i = (k << 8) + static_cast<uint64_t>(j);
            const bool bulk = k >= k_lo && k < k_hi;
            bool give_up = false;
            if (bulk) {
#pragma unroll
                for (int qq = 0; qq < kStep1Stages; ++qq)
                    if (qq == s) {
                        give_up = !mbar_wait_or_abort(&bar[qq], uses[qq] & 1u, abortp);
                        ++uses[qq];
                    }
            }
            if (__any_sync(full, give_up)) {
                if (lane == 0) *abortp = 1;
                break;
            }
            uint8_t flags0 = 0;
            Pos x{};
            R v[3] = {R(0), R(0), R(0)};
            if (bulk) {
                const unsigned char* st = stage[s];
                flags0 = st[S::kFlagOff + j];
                if (flags0 & kFlagActive) {
                    step1_pos_from_stage<PREC>(x, st, j);
                    const R* vv = reinterpret_cast<const R*>(st + S::kVelOff);
                    v[0] = vv[j]; v[1] = vv[kStep1Block + j]; v[2] = vv[2 * kStep1Block + j];
                }
            } else if (i >= b && i < en) {
                flags0 = p.flags[i];
                if (flags0 & kFlagActive) {
                    x.load(p, i);
                    v[0] = static_cast<const R*>(p.vx)[i];
                    v[1] = static_cast<const R*>(p.vy)[i];
                    v[2] = static_cast<const R*>(p.vz)[i];
                }
            }

            bool live = (flags0 & kFlagActive) != 0;
            const int e = (ONE || !live) ? 0 : step1_ensemble(p, i);
            const EnsConst& C = p.ens[e];
            const double t0 = ONE ? t0_one : p.t_dev[p.ens_base + static_cast<uint32_t>(e)];
            uint8_t flags = flags0;
            auto kill = [&]() {
                flags = static_cast<uint8_t>(flags & ~kFlagActive);
                p.t_death[i] = t0;
                live = false;
                ++n_dead;
            };
            if (live && !p.skip_prepare && !inside(C, x)) kill();   // prepare_ions_for_integration
            bool out = false, cand = false;
            if (live) {
                Consts<R> kc;
                step1_consts<R>(kc, C, p, i);
                const double zo = x.gz();
                boris<R, kFieldUniform, false>(kc, x, v, t0);
                x.fold();
                const double zn = x.gz();
                if (!(flags & kFlagArrived) && zo < C.zdet && zn >= C.zdet) {
                    p.t_arr[i] = t0 + C.dt * ((C.zdet - zo) / (zn - zo));
                    flags |= kFlagArrived;
                    ++n_arr;
                }
                // inside() already fails for non-finite x or y and infinite
                // z; of a non-finite position only a NaN z passes it
                out = !inside(C, x) || isnan(x.gz());
                const R wx = v[0] - kc.ug[0], wy = v[1] - kc.ug[1], wz = v[2] - kc.ug[2];
                const R bb = m_sqrt(wx * wx + wy * wy + wz * wz);
                R Q = kc.A * bb + kc.Amean;
                if (Q > R(1)) { Q = R(1); ++n_ovf; }
                cand = u32(step_test_word(step0, static_cast<uint32_t>(p.first_id + i), p.rk), R(0)) < Q;
            }
            // queue the candidates once the collision warp is done with
            // this queue's previous tile
            const int q = static_cast<int>(it & 1u);
            bool ok = true;
            if (it >= 2) ok = mbar_wait_or_abort(&q_empty[q], static_cast<uint32_t>((it >> 1) + 1u) & 1u, abortp);
            if (__any_sync(full, !ok)) {
                if (lane == 0) *abortp = 1;
                break;
            }
            const unsigned ball = __ballot_sync(full, cand);
            int base = 0;
            if (lane == 0 && ball) base = atomicAdd(&qn[q], __popc(ball));
            base = __shfl_sync(full, base, 0);
            if (cand) {
                ++n_cand;
                const int sl = base + __popc(ball & ((1u << lane) - 1u));
                qv[q][0][sl] = v[0]; qv[q][1][sl] = v[1]; qv[q][2][sl] = v[2];
                qj[q][sl] = static_cast<uint16_t>(j);
                qf[q][sl] = static_cast<uint8_t>(flags | (out ? kQueueOut : 0u));
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&q_full[q]);
            if (flags0 & kFlagActive) {
                x.store(p, i);
                if (!cand) {
                    if (live && (out || !(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2])))) kill();
                    static_cast<R*>(p.vx)[i] = v[0];
                    static_cast<R*>(p.vy)[i] = v[1];
                    static_cast<R*>(p.vz)[i] = v[2];
                    if (flags != flags0) p.flags[i] = flags;
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0 && *abortp) atomicAdd(&p.counters[kCntStalls], 1ull);
    const unsigned long long s0 = warp_sum_u32(n_cand), s1 = warp_sum_u32(n_coll), s2 = warp_sum_u32(n_ovf);
    const unsigned long long s3 = warp_sum_u32(n_dead), s4 = warp_sum_u32(n_arr);
    if (lane == 0) {
        if (s0) atomicAdd(&p.counters[kCntCandidates], s0);
        if (s1) atomicAdd(&p.counters[kCntCollisions], s1);
        if (s2) atomicAdd(&p.counters[kCntOverflow], s2);
        if (s3) atomicAdd(&p.counters[kCntDeaths], s3);
        if (s4) atomicAdd(&p.counters[kCntArrivals], s4);
    }
}

// Persistent grid size of a kernel on the current device: resident CTAs
// per SM x SMs, cached per device (a kernel's occupancy does not change).
constexpr int kStep1MaxDevices = 64;
template <class K>
cudaError_t step1_grid_cap(K kernel, int threads, std::atomic<int>* cache, int& cap) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    std::atomic<int>* slot = (dev >= 0 && dev < kStep1MaxDevices) ? &cache[dev] : nullptr;
    cap = slot ? slot->load(std::memory_order_relaxed) : 0;
    if (cap > 0) return cudaSuccess;
    int sms = 0, per_sm = 0;
    err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (err == cudaSuccess) err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    if (err != cudaSuccess) return err;
    cap = (per_sm < 1 ? 1 : per_sm) * (sms < 1 ? 1 : sms);
    if (slot) slot->store(cap, std::memory_order_relaxed);
    return cudaSuccess;
}

// Persistent grid: resident CTAs per SM (as compiled) x SMs, at most one
// CTA per tile of the launch's range.
template <int PREC, int COLL>
cudaError_t launch_step1_coll(const StepParams& p, cudaStream_t s) {
    static std::atomic<int> cached[kStep1MaxDevices];
    int cap_i = 0;
    if (cudaError_t err = step1_grid_cap(k_step1<PREC, COLL>, kStep1Block, cached, cap_i)) return err;
    const uint64_t b = p.ens_off[0], en = p.ens_off[p.n_ens];
    if (en <= b) return cudaSuccess;
    const uint64_t tiles = (en + kStep1Block - 1) / kStep1Block - b / kStep1Block;
    const uint64_t cap = static_cast<uint64_t>(cap_i);
    const dim3 grid(static_cast<unsigned>(tiles < cap ? tiles : cap));
    k_step1<PREC, COLL><<<grid, kStep1Block, 0, s>>>(p);
    return cudaGetLastError();
}

template <int PREC, bool ONE>
cudaError_t launch_step1_ws(const StepParams& p, cudaStream_t s) {
    static std::atomic<int> cached[kStep1MaxDevices];
    int cap_i = 0;
    if (cudaError_t err = step1_grid_cap(k_step1_ws<PREC, ONE>, kStep1WsThreads, cached, cap_i)) return err;
    const uint64_t b = p.ens_off[0], en = p.ens_off[p.n_ens];
    if (en <= b) return cudaSuccess;
    const uint64_t tiles = (en + kStep1Block - 1) / kStep1Block - b / kStep1Block;
    const uint64_t cap = static_cast<uint64_t>(cap_i);
    const dim3 grid(static_cast<unsigned>(tiles < cap ? tiles : cap));
    k_step1_ws<PREC, ONE><<<grid, kStep1WsThreads, 0, s>>>(p);
    return cudaGetLastError();
}

// One step per launch with collisions: the warp-specialized kernel;
// otherwise the block-synchronous one.
template <int PREC>
cudaError_t launch_step1(int coll, const StepParams& p, cudaStream_t s) {
    if (coll == kCollNone) return launch_step1_coll<PREC, kCollNone>(p, s);
    if (coll != kCollHSS) return cudaErrorNotSupported;
    if (p.n_steps == 1) return p.n_ens == 1 ? launch_step1_ws<PREC, true>(p, s) : launch_step1_ws<PREC, false>(p, s);
    return launch_step1_coll<PREC, kCollHSS>(p, s);
}

}  // namespace icb
