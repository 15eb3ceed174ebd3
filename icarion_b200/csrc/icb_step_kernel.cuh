// icb_step_kernel.cuh — the fused, register-resident K-step kernel.
//
// One thread owns one ion for n_steps engine steps.  Each step follows the
// reference engine's order (SimulationEngine::process_timestep,
// SimulationEngine.cpp:374-428):
//   push (BorisStrategy.cpp:18-98 or RK4Strategy.cpp:181-361)
//   -> collision (null-collision form of HSSCollisionHandler.cpp:257-376)
//   -> finalize (SimulationEngineLifecycle.cpp:123-195: domain exit or
//      non-finite state -> inactive with death time = step start time)
//   -> t += dt.
//
// Precision policies:
//   FP64       double everywhere.  Compiled without FMA contraction so that
//              the collision-free push is bit-identical to the reference.
//   MIXED      float velocity, field, collision; double position and time.
//   HILO       float velocity; position as a compensated float hi/lo pair.
//
// Deferred collisions.  A collision candidate fires in ~10% of ion-steps;
// executed in place it would make almost every warp-step run the expensive
// candidate branch with a few lanes active.  Instead a lane whose clock
// fires stops ("pending") while the other lanes keep stepping; once
// `pend_threshold` lanes of the warp are pending (or no lane can step) the
// warp processes all pending collisions together, converged.  Every lane
// still applies its own steps in order, so results do not depend on the
// threshold or the launch shape.
#pragma once
#include <cstdint>
#include <cmath>
#include "icb_params.h"
#include "icb_rng.cuh"

namespace icb {

template <int PREC> struct PrecT;
template <> struct PrecT<kPrecFP64> { using R = double; };
template <> struct PrecT<kPrecMixed> { using R = float; };
template <> struct PrecT<kPrecHiLo> { using R = float; };

// ---- math helpers per precision ------------------------------------------
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_log(float x) { return __logf(x); }
__device__ __forceinline__ double m_expm1(double x) { return expm1(x); }
__device__ __forceinline__ float m_expm1(float x) { return expm1f(x); }
__device__ __forceinline__ double m_cos(double x) { return cos(x); }
__device__ __forceinline__ double m_fmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float m_fmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double unit(uint32_t w, double) { return unit_d(w); }
__device__ __forceinline__ float unit(uint32_t w, float) { return unit_f(w); }

// (cos, sin) of the angle 2*pi*u.  FP64 keeps the oracle's 2*pi*u; the
// float path uses the equally uniform angle 2*pi*(u - 1/2) in (-pi, pi],
// the accurate range of the hardware sin/cos.
__device__ __forceinline__ void angle_cs(double u, double& c, double& s) {
    const double ph = 2.0 * 3.14159265358979323846 * u;
    c = cos(ph);
    s = sin(ph);
}
__device__ __forceinline__ void angle_cs(float u, float& c, float& s) {
    __sincosf(6.28318530717958648f * (u - 0.5f), &s, &c);
}

// ---- positions --------------------------------------------------------------
// Double position (FP64 and MIXED).
struct PosD {
    double x, y, z;
    __device__ void load(const StepParams& p, uint64_t i) { x = p.x[i]; y = p.y[i]; z = p.z[i]; }
    __device__ void store(const StepParams& p, uint64_t i) const { p.x[i] = x; p.y[i] = y; p.z[i] = z; }
    __device__ double gx() const { return x; }
    __device__ double gy() const { return y; }
    __device__ double gz() const { return z; }
    template <class R> __device__ R rel(int a, double c) const {
        const double v = (a == 0) ? x : (a == 1) ? y : z;
        return static_cast<R>(v - c);
    }
    __device__ void drift(double vx, double vy, double vz, double dt) {
        x += vx * dt; y += vy * dt; z += vz * dt;
    }
    __device__ void drift(float vx, float vy, float vz, double dt) {
        x = fma(static_cast<double>(vx), dt, x);
        y = fma(static_cast<double>(vy), dt, y);
        z = fma(static_cast<double>(vz), dt, z);
    }
    __device__ bool finite() const { return isfinite(x) && isfinite(y) && isfinite(z); }
};

// Compensated float pair: value = hi + lo, |lo| <= ulp(hi)/2.
__device__ __forceinline__ void two_sum_acc(float& hi, float& lo, float d) {
    const float s = hi + d;
    const float bp = s - hi;
    const float err = (hi - (s - bp)) + (d - bp);
    const float l = lo + err;
    const float h2 = s + l;
    lo = l - (h2 - s);
    hi = h2;
}

struct PosHL {
    float xh, xl, yh, yl, zh, zl;
    __device__ void load(const StepParams& p, uint64_t i) {
        xh = p.xh[i]; xl = p.xl[i]; yh = p.yh[i]; yl = p.yl[i]; zh = p.zh[i]; zl = p.zl[i];
    }
    __device__ void store(const StepParams& p, uint64_t i) const {
        p.xh[i] = xh; p.xl[i] = xl; p.yh[i] = yh; p.yl[i] = yl; p.zh[i] = zh; p.zl[i] = zl;
    }
    __device__ double gx() const { return static_cast<double>(xh) + static_cast<double>(xl); }
    __device__ double gy() const { return static_cast<double>(yh) + static_cast<double>(yl); }
    __device__ double gz() const { return static_cast<double>(zh) + static_cast<double>(zl); }
    template <class R> __device__ R rel(int a, double c) const {
        const float h = (a == 0) ? xh : (a == 1) ? yh : zh;
        const float l = (a == 0) ? xl : (a == 1) ? yl : zl;
        const float ch = static_cast<float>(c);
        const float cl = static_cast<float>(c - static_cast<double>(ch));
        return static_cast<R>(((h - ch) + l) - cl);
    }
    __device__ void drift(float vx, float vy, float vz, double dt) {
        const float d = static_cast<float>(dt);
        two_sum_acc(xh, xl, vx * d);
        two_sum_acc(yh, yl, vy * d);
        two_sum_acc(zh, zl, vz * d);
    }
    __device__ bool finite() const {
        return isfinite(xh) && isfinite(yh) && isfinite(zh) && isfinite(xl) && isfinite(yl) && isfinite(zl);
    }
};

template <int PREC> struct PosOf { using T = PosD; };
template <> struct PosOf<kPrecHiLo> { using T = PosHL; };

// ---- per-thread copy of the ensemble constants in the working precision --
template <class R>
struct Consts {
    R E0[3], G[3];
    double c[3];
    R rfU0, rfV, r0sq;
    double rfw;
    R tv[3], sv[3];          // Boris rotation vectors for this ion
    R a_uni[3];              // acceleration of a uniform field for this ion
    R q, m, qm, inv_m;
    double dt;
    R h;                     // dt/2 in working precision
    R A, mean_th, ug[3];     // collision clock
};

template <class R, int FIELD, bool MAG>
__device__ void load_consts(Consts<R>& k, const EnsConst& C, double q, double m) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        k.E0[a] = static_cast<R>(C.E0[a]);
        k.G[a] = static_cast<R>(C.G[a]);
        k.c[a] = C.c[a];
        k.ug[a] = static_cast<R>(C.ug[a]);
    }
    k.rfU0 = static_cast<R>(C.rf_U0);
    k.rfV = static_cast<R>(C.rf_V);
    k.r0sq = static_cast<R>(C.r0sq);
    k.rfw = C.rf_omega;
    k.dt = C.dt;
    k.h = static_cast<R>(C.dt * 0.5);
    k.q = static_cast<R>(q);
    k.m = static_cast<R>(m);
    // Reference: qm = charge / mass; t = B * (qm * dt * 0.5); s = 2 t / (1 + t^2);
    // uniform field a = (E * q) / m (ElectricFieldForce.cpp:66-83,
    // BorisStrategy.cpp:50), constant for the whole launch.  FP64 keeps the
    // reference's divisions; the float paths use one reciprocal.
    double qm, inv_m;
    if constexpr (sizeof(R) == 8) {
        qm = q / m;
        inv_m = 1.0 / m;
#pragma unroll
        for (int a = 0; a < 3; ++a) k.a_uni[a] = static_cast<R>((C.E0[a] * q) / m);
    } else {
        inv_m = 1.0 / m;
        qm = q * inv_m;
#pragma unroll
        for (int a = 0; a < 3; ++a) k.a_uni[a] = static_cast<R>((C.E0[a] * q) * inv_m);
    }
    k.qm = static_cast<R>(qm);
    k.inv_m = static_cast<R>(inv_m);
    if (MAG) {
        const double ts = qm * C.dt * 0.5;
        const double tv0 = C.B[0] * ts, tv1 = C.B[1] * ts, tv2 = C.B[2] * ts;
        const double t2 = tv0 * tv0 + tv1 * tv1 + tv2 * tv2;
        const double sf = 2.0 / (1.0 + t2);
        k.tv[0] = static_cast<R>(tv0); k.tv[1] = static_cast<R>(tv1); k.tv[2] = static_cast<R>(tv2);
        k.sv[0] = static_cast<R>(tv0 * sf); k.sv[1] = static_cast<R>(tv1 * sf); k.sv[2] = static_cast<R>(tv2 * sf);
    }
    k.A = static_cast<R>(C.A);
    k.mean_th = static_cast<R>(C.mean_th);
}

// ---- fields -----------------------------------------------------------------
template <class R, int FIELD, class Pos>
__device__ __forceinline__ void efield(const Consts<R>& k, const Pos& x, double t, R E[3]) {
    if constexpr (FIELD == kFieldUniform) {
        E[0] = k.E0[0]; E[1] = k.E0[1]; E[2] = k.E0[2];
        return;
    } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) E[a] = k.E0[a] + k.G[a] * x.template rel<R>(a, k.c[a]);
    }
    if constexpr (FIELD == kFieldLinearRF) {
        // AnalyticalFieldModel.cpp:152-158: U = dc_quad + V cos(w t);
        // E_x = -2 x U / r0^2, E_y = 2 y U / r0^2.
        const R U = k.rfU0 + k.rfV * static_cast<R>(cos(k.rfw * t));
        const R px = x.template rel<R>(0, 0.0), py = x.template rel<R>(1, 0.0);
        E[0] = R(-2.0) * px * U / k.r0sq;
        E[1] = R(2.0) * py * U / k.r0sq;
    }
}

// ---- pushers ------------------------------------------------------------------
// Boris exactly as BorisStrategy.cpp:50-97, including x += v_plus * dt.
// Returns |v_plus|_1, the L1 speed of this step's drift.
template <class R, int FIELD, bool MAG, class Pos>
__device__ __forceinline__ R boris(const Consts<R>& k, Pos& x, R v[3], double t) {
    R a[3];
    if (FIELD == kFieldUniform) {
        a[0] = k.a_uni[0]; a[1] = k.a_uni[1]; a[2] = k.a_uni[2];
    } else {
        R E[3];
        efield<R, FIELD>(k, x, t, E);
        if (sizeof(R) == 8) {
#pragma unroll
            for (int c = 0; c < 3; ++c) a[c] = (E[c] * k.q) / k.m;
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) a[c] = E[c] * k.qm;
        }
    }
    R vm[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) vm[c] = v[c] + a[c] * k.h;
    R vp[3];
    if (MAG) {
        const R c1x = vm[1] * k.tv[2] - vm[2] * k.tv[1];
        const R c1y = vm[2] * k.tv[0] - vm[0] * k.tv[2];
        const R c1z = vm[0] * k.tv[1] - vm[1] * k.tv[0];
        const R ppx = vm[0] + c1x, ppy = vm[1] + c1y, ppz = vm[2] + c1z;
        const R c2x = ppy * k.sv[2] - ppz * k.sv[1];
        const R c2y = ppz * k.sv[0] - ppx * k.sv[2];
        const R c2z = ppx * k.sv[1] - ppy * k.sv[0];
        vp[0] = vm[0] + c2x; vp[1] = vm[1] + c2y; vp[2] = vm[2] + c2z;
    } else {
        vp[0] = vm[0]; vp[1] = vm[1]; vp[2] = vm[2];
    }
    x.drift(vp[0], vp[1], vp[2], k.dt);
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = vp[c] + a[c] * k.h;
    return fabs(vp[0]) + fabs(vp[1]) + fabs(vp[2]);
}

// RK4 acceleration: (E q [+ (v x B) q]) * (1/m)  (RK4Strategy.cpp:236-243,
// MagneticFieldForce.cpp:61-88; magnetic force is registered for non-Boris
// integrators, PhysicsSetup.cpp:206).
template <class R, int FIELD, bool MAG, class Pos>
__device__ __forceinline__ void rk4_acc(const Consts<R>& k, const Pos& x, const R v[3], double t, R acc[3]) {
    R E[3];
    efield<R, FIELD>(k, x, t, E);
    R F[3] = {E[0] * k.q, E[1] * k.q, E[2] * k.q};
    if (MAG) {
        const R B0 = k.tv[0], B1 = k.tv[1], B2 = k.tv[2];  // holds B itself for RK4 (see load)
        const R cx = v[1] * B2 - v[2] * B1;
        const R cy = v[2] * B0 - v[0] * B2;
        const R cz = v[0] * B1 - v[1] * B0;
        F[0] += cx * k.q; F[1] += cy * k.q; F[2] += cz * k.q;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] = F[c] * k.inv_m;
}

// Returns the L1 norm of the step's displacement divided by dt.
template <class R, int FIELD, bool MAG, class Pos>
__device__ __forceinline__ R rk4(const Consts<R>& k, Pos& x, R v[3], double t) {
    const double dt = k.dt;
    const double hd = dt * 0.5;
    const R h = k.h;
    const R dtr = static_cast<R>(dt);
    const Pos x0 = x;
    const R v0[3] = {v[0], v[1], v[2]};
    R k1a[3], k2a[3], k3a[3], k4a[3], v2[3], v3[3], v4[3];
    rk4_acc<R, FIELD, MAG>(k, x0, v0, t, k1a);
    Pos p2 = x0; p2.drift(v0[0], v0[1], v0[2], hd);
#pragma unroll
    for (int c = 0; c < 3; ++c) v2[c] = v0[c] + k1a[c] * h;
    rk4_acc<R, FIELD, MAG>(k, p2, v2, t + hd, k2a);
    Pos p3 = x0; p3.drift(v2[0], v2[1], v2[2], hd);
#pragma unroll
    for (int c = 0; c < 3; ++c) v3[c] = v0[c] + k2a[c] * h;
    rk4_acc<R, FIELD, MAG>(k, p3, v3, t + hd, k3a);
    Pos p4 = x0; p4.drift(v3[0], v3[1], v3[2], dt);
#pragma unroll
    for (int c = 0; c < 3; ++c) v4[c] = v0[c] + k3a[c] * dtr;
    rk4_acc<R, FIELD, MAG>(k, p4, v4, t + dt, k4a);
    R dv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) dv[c] = v0[c] + v2[c] * R(2.0) + v3[c] * R(2.0) + v4[c];
    x = x0;
    x.drift(dv[0], dv[1], dv[2], dt / 6.0);
    const R s = static_cast<R>(dt / 6.0);
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = v0[c] + (k1a[c] + k2a[c] * R(2.0) + k3a[c] * R(2.0) + k4a[c]) * s;
    return (fabs(dv[0]) + fabs(dv[1]) + fabs(dv[2])) * R(1.0 / 6.0);
}

// ---- null-collision HSS -------------------------------------------------------
// Clock update after the push.  Returns true when a candidate fires.
template <class R>
__device__ __forceinline__ bool clock_tick(const Consts<R>& k, const R v[3], R& S, R U, R& gu, uint32_t& ovf) {
    const R wx = v[0] - k.ug[0], wy = v[1] - k.ug[1], wz = v[2] - k.ug[2];
    gu = m_sqrt(wx * wx + wy * wy + wz * wz);
    R Q = k.A * (gu + k.mean_th);
    if (Q > R(1)) { Q = R(1); ++ovf; }
    S = S - S * Q;
    return S < U;
}

// Candidate processing (the same steps as the oracle's hss_nullcoll).
// Returns true when the collision is accepted (v updated).
template <class R>
__device__ __forceinline__ bool candidate(const EnsConst& C, R v[3], R& S, R& U, R gu, double mi_d,
                                          uint64_t seed, uint32_t id, uint32_t step) {
    struct {
        R A, mean_th, sig_n, ug[3], mi, mn, inv_mt, fac;
    } k;
    k.A = static_cast<R>(C.A);
    k.mean_th = static_cast<R>(C.mean_th);
    k.sig_n = static_cast<R>(C.sig_n);
    k.ug[0] = static_cast<R>(C.ug[0]); k.ug[1] = static_cast<R>(C.ug[1]); k.ug[2] = static_cast<R>(C.ug[2]);
    k.mi = static_cast<R>(mi_d);
    k.mn = static_cast<R>(C.m_gas);
    const double inv = 1.0 / (mi_d + C.m_gas);
    k.inv_mt = static_cast<R>(inv);
    k.fac = static_cast<R>(C.m_gas * inv);
    const uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
    const U4 r0 = philox4x32_10(id, step, 0u, 0u, k0, k1);
    const U4 r1 = philox4x32_10(id, step, 1u, 0u, k0, k1);
    U = unit(r0.x, R(0));
    S = R(1);
    R th[3];
    if (unit(r0.y, R(0)) * (gu + k.mean_th) < gu) {
        const R ra = m_sqrt(R(-2.0) * m_log(unit(r1.x, R(0))));
        const R rb = m_sqrt(R(-2.0) * m_log(unit(r1.z, R(0))));
        R ca, sa, cb, sb;
        angle_cs(unit(r1.y, R(0)), ca, sa);
        angle_cs(unit(r1.w, R(0)), cb, sb);
        th[0] = k.sig_n * (ra * ca);
        th[1] = k.sig_n * (ra * sa);
        th[2] = k.sig_n * (rb * cb);
    } else {
        const R rad = k.sig_n * m_sqrt(R(-2.0) * m_log(unit(r1.x, R(0)) * unit(r1.y, R(0))));
        const R ct = R(2.0) * unit(r1.z, R(0)) - R(1.0);
        const R st = m_sqrt(m_fmax(R(0), R(1.0) - ct * ct));
        R cp, sp;
        angle_cs(unit(r1.w, R(0)), cp, sp);
        th[0] = rad * (st * cp);
        th[1] = rad * (st * sp);
        th[2] = rad * ct;
    }
    const R thm = m_sqrt(th[0] * th[0] + th[1] * th[1] + th[2] * th[2]);
    const R vn[3] = {k.ug[0] + th[0], k.ug[1] + th[1], k.ug[2] + th[2]};
    const R gx = v[0] - vn[0], gy = v[1] - vn[1], gz = v[2] - vn[2];
    const R g = m_sqrt(gx * gx + gy * gy + gz * gz);
    const R q = k.A * (gu + thm);
    const R pc = -m_expm1(-k.A * g);
    if (!(unit(r0.z, R(0)) * q < pc)) return false;
    const U4 r2 = philox4x32_10(id, step, 2u, 0u, k0, k1);
    const R ct = R(2.0) * unit(r0.w, R(0)) - R(1.0);
    const R st = m_sqrt(m_fmax(R(0), R(1.0) - ct * ct));
    R cp, sp;
    angle_cs(unit(r2.x, R(0)), cp, sp);
    const R dir[3] = {st * cp, st * sp, ct};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const R vcom = (v[c] * k.mi + vn[c] * k.mn) * k.inv_mt;
        v[c] = vcom + (dir[c] * g) * k.fac;
    }
    return true;
}

// ---- finalize ------------------------------------------------------------------
// CylindricalGeometry::contains (CylindricalGeometry.h:35-40) on the global
// position; returns false for positions outside or non-finite.
template <class Pos>
__device__ __forceinline__ bool inside(const EnsConst& C, const Pos& x) {
    const double lz = x.gz() - C.oz;
    if (lz < -1e-12 || lz >= C.zmax_local) return false;
    const double lx = x.gx() - C.ox, ly = x.gy() - C.oy;
    const double r2 = lx * lx + ly * ly;
    return r2 <= C.rmax2;
}

__device__ __forceinline__ unsigned long long warp_sum_u32(uint32_t v) {
    return static_cast<unsigned long long>(__reduce_add_sync(0xffffffffu, v));
}

// ---- the kernel -----------------------------------------------------------------
// Exact per-step finalize of the reference (domain exit -> death at the step
// start time, non-finite state -> death, first detector-plane crossing) is
// evaluated only when it can change anything: each lane accumulates the L1
// length of its drifts since its last exact check (acc) and re-checks once acc
// may exceed 99% of the distance to the nearest wall, end face or (not yet
// crossed) detector plane (lim).  The L1 length bounds the true path, so no
// exit or crossing is missed; NaN or Inf makes acc non-finite and forces the
// check.  Float accumulation error over <= 16384 steps per launch is < 0.1%.

template <int PREC>
struct KernelShape { static constexpr int kMinBlocks = 6; };
template <>
struct KernelShape<kPrecFP64> { static constexpr int kMinBlocks = 4; };

template <int PREC, int INTEG, int COLL, int FIELD, bool MAG, bool FUSED>
__global__ void __launch_bounds__(128, KernelShape<PREC>::kMinBlocks) k_step(const __grid_constant__ StepParams p) {
    using R = typename PrecT<PREC>::R;
    using Pos = typename PosOf<PREC>::T;
    // FP64 keeps the engine clock as the accumulated sum t += dt (bit-exact
    // death and arrival times); the float paths form t = t0 + k*dt when an
    // event needs it, unless the field itself is time dependent.
    constexpr bool kAccumT = (PREC == kPrecFP64) || (FIELD == kFieldLinearRF);

    const uint64_t i = p.ens_off[0] + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool in_range = i < p.ens_off[p.n_ens];
    int e = 0;
    if (in_range) {
        int lo = 0, hi = static_cast<int>(p.n_ens) - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.ens_off[mid] <= i) lo = mid; else hi = mid - 1;
        }
        e = lo;
    }
    const EnsConst& C = p.ens[e];
    const bool do_push = FUSED || p.do_push;
    const bool do_coll = FUSED || p.do_collide;
    const bool do_fin = FUSED || p.do_finalize;

    uint8_t flags = 0;
    Pos x{};
    R v[3] = {R(0), R(0), R(0)};
    R S = R(1), U = R(0);
    double q = 1.0, m = 1.0, birth = 0.0;
    bool had_arrival = false;
    if (in_range) {
        flags = p.flags[i];
        x.load(p, i);
        v[0] = static_cast<const R*>(p.vx)[i];
        v[1] = static_cast<const R*>(p.vy)[i];
        v[2] = static_cast<const R*>(p.vz)[i];
        if (COLL != kCollNone) {
            S = static_cast<const R*>(p.clkS)[i];
            U = static_cast<const R*>(p.clkU)[i];
        }
        q = p.charge[i];
        m = p.mass[i];
        if (p.birth) birth = p.birth[i];
        had_arrival = p.t_arr[i] >= 0.0;
    }
    Consts<R> k;
    load_consts<R, FIELD, MAG>(k, C, q, m);
    if (INTEG == kRK4 && MAG) {
        // rk4_acc reads B from tv[] (no rotation vectors needed for RK4).
        k.tv[0] = static_cast<R>(C.B[0]); k.tv[1] = static_cast<R>(C.B[1]); k.tv[2] = static_cast<R>(C.B[2]);
    }

    const uint32_t id = static_cast<uint32_t>(p.first_id + i);
    const uint32_t step0 = static_cast<uint32_t>(*p.step_dev);
    const double t0 = p.t_dev[p.ens_base + e];
    const double dt = C.dt;
    const R dt_r = static_cast<R>(dt);
    const double zdet = C.zdet;
    double t = t0;            // accumulated clock (used when kAccumT)
    double tdeath = -1.0, tarr = -1.0;
    bool dead_now = false, arr_now = false;
    uint32_t n_cand = 0, n_coll = 0, n_ovf = 0, n_dead = 0, n_arr = 0;
    const uint32_t K = p.n_steps;
    uint32_t kk = 0;
    bool pending = false;
    R gu = R(0);
    double zold = 0.0;
    R acc = R(0), lim = R(0);

    auto t_step = [&]() -> double { return kAccumT ? t : fma(static_cast<double>(kk), dt, t0); };
    auto kill = [&](double when) {
        flags &= static_cast<uint8_t>(~kFlagActive);
        tdeath = when;
        dead_now = true;
        ++n_dead;
    };
    // Short launches (the per-step form) check exactly every step instead of
    // setting up a displacement budget (lim stays 0).
    const bool budget = FUSED && K >= 8;
    // distance to the nearest wall, end face or pending detector plane
    auto new_limit = [&]() {
        if (!budget) return;
        const double z = x.gz();
        const double lz = z - C.oz;
        double d = fmin(lz + 1e-12, C.zmax_local - lz);
        const double lx = x.gx() - C.ox, ly = x.gy() - C.oy;
        d = fmin(d, C.rmax - sqrt(lx * lx + ly * ly));
        if (!had_arrival) d = fmin(d, fabs(zdet - z));
        lim = static_cast<R>(0.99 * d);
        acc = R(0);
    };

    bool live = in_range && (flags & kFlagActive);
    bool waiting = in_range && !(flags & kFlagBorn);
    if (live && (do_fin || do_push)) {
        if (!inside(C, x)) {       // prepare_ions_for_integration: outside -> inactive
            live = false;
            kill(t0);
        } else {
            new_limit();
        }
    }

    // exact finalize of the current step (SimulationEngineLifecycle.cpp:123-195)
    auto finalize_step = [&]() {
        // the unfused finalize call has no drift history: always exact
        if (do_fin && (!FUSED || !(acc <= lim))) {
            if (!FUSED && !do_push) zold = p.zprev[i];
            const double ts = t_step();
            const double znew = x.gz();
            if (!had_arrival && zold < zdet && znew >= zdet) {
                tarr = ts + dt * ((zdet - zold) / (znew - zold));
                had_arrival = true;
                arr_now = true;
                ++n_arr;
            }
            bool ok = inside(C, x);
            if (ok) ok = x.finite() && isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]);
            if (!ok) {
                live = false;
                kill(ts);
            } else {
                new_limit();
            }
        }
        ++kk;
        if (kAccumT) t = t + dt;
    };

    auto cheap_step = [&]() {
        if (waiting) {
            if (t_step() >= birth) {      // prepare_ions_for_integration birth rule
                waiting = false;
                flags |= static_cast<uint8_t>(kFlagBorn | kFlagActive);
                live = inside(C, x);
                if (!live) kill(t_step());
                else new_limit();
            }
        }
        if (waiting || !live) {
            ++kk;
            if (kAccumT) t = t + dt;
            return;
        }
        zold = x.gz();
        if (!FUSED && do_push) p.zprev[i] = zold;
        if (do_push) {
            R l1;
            if (INTEG == kBoris) l1 = boris<R, FIELD, MAG>(k, x, v, t_step());
            else l1 = rk4<R, FIELD, MAG>(k, x, v, t_step());
            acc += l1 * dt_r;
        }
        if (COLL != kCollNone && do_coll) pending = clock_tick<R>(k, v, S, U, gu, n_ovf);
        if (!pending) finalize_step();
    };

    while (true) {
        // cheap phase: up to steps_per_vote steps for every lane that can
        // step without a collision
#pragma unroll 1
        for (uint32_t j = 0; j < p.steps_per_vote; ++j) {
            if ((live || waiting) && !pending && kk < K) cheap_step();
        }
        const unsigned pend_mask = __ballot_sync(0xffffffffu, pending);
        const unsigned run_mask = __ballot_sync(0xffffffffu, (live || waiting) && !pending && kk < K);
        if (pend_mask != 0u &&
            (run_mask == 0u || static_cast<uint32_t>(__popc(pend_mask)) >= p.pend_threshold)) {
            if (pending) {
                ++n_cand;
                if (candidate<R>(C, v, S, U, gu, m, p.seed, id, step0 + kk)) ++n_coll;
                pending = false;
                finalize_step();
            }
            continue;
        }
        if (run_mask == 0u) break;
    }

    if (in_range) {
        x.store(p, i);
        static_cast<R*>(p.vx)[i] = v[0];
        static_cast<R*>(p.vy)[i] = v[1];
        static_cast<R*>(p.vz)[i] = v[2];
        if (COLL != kCollNone) {
            static_cast<R*>(p.clkS)[i] = S;
            static_cast<R*>(p.clkU)[i] = U;
        }
        p.flags[i] = flags;
        if (dead_now) p.t_death[i] = tdeath;
        if (arr_now) p.t_arr[i] = tarr;
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

}  // namespace icb
