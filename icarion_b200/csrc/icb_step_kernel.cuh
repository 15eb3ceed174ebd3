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
//   MIXED      float velocity, field, collision; position = double anchor +
//              float offset (folded into the anchor at every warp vote).
//   HILO       float velocity; position as a compensated float hi/lo pair.
//
// Two loops run the steps.  The event-to-event form (float precisions, and
// FP64 on request; Boris in a uniform field without B; run_jumps below)
// moves each lane in one closed-form update to its next clock event, exact
// domain check or the launch end, and the warp then handles the events of
// all its lanes together.  The step-by-step loop (FP64 by default, RK4,
// other fields, births, ICB_STEPPING_PER_STEP) defers collisions instead:
// a collision candidate
// fires in ~10% of ion-steps; executed in place it would make almost every
// warp-step run the expensive candidate branch with a few lanes active, so
// a lane whose clock fires stops ("pending") while the other lanes keep
// stepping; once `pend_threshold` lanes of the warp are pending (or no lane
// can step) the warp processes all pending collisions together, converged.
// Every lane still applies its own steps in order, so results do not depend
// on the threshold or the launch shape.
#pragma once
#include <cstdint>
#include <cmath>
#include <type_traits>
#include "icb_params.h"
#include "icb_rng.cuh"
#include "icb_mlp.cuh"
#include "icb_ipm.cuh"

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
__device__ __forceinline__ double m_log1p(double x) { return log1p(x); }
__device__ __forceinline__ float m_log1p(float x) { return log1pf(x); }
__device__ __forceinline__ double m_expm1(double x) { return expm1(x); }
__device__ __forceinline__ float m_expm1(float x) { return expm1f(x); }

// -ln(1 - q), 0 <= q < 1 (a per-step probability -> hazard).  FP64: log1p.
// Float: the Taylor series sum_{k>=1} q^k / k to k = 12 below q = 1/4
// (truncation < q^12 / (13 (1 - q)) < 5e-9 relative), above it -ln(1 - q)
// with the hardware log (1 - q is exact for q >= 1/2; absolute error
// < 4e-7 on a value >= 0.28).
__device__ __forceinline__ double m_neg_log1m(double q) { return -log1p(-q); }
__device__ __forceinline__ float m_neg_log1m(float q) {
    if (q < 0.25f) {
        float s = 1.0f / 12.0f;
        s = fmaf(q, s, 1.0f / 11.0f); s = fmaf(q, s, 1.0f / 10.0f); s = fmaf(q, s, 1.0f / 9.0f);
        s = fmaf(q, s, 1.0f / 8.0f);  s = fmaf(q, s, 1.0f / 7.0f);  s = fmaf(q, s, 1.0f / 6.0f);
        s = fmaf(q, s, 0.2f);         s = fmaf(q, s, 0.25f);        s = fmaf(q, s, 1.0f / 3.0f);
        s = fmaf(q, s, 0.5f);         s = fmaf(q, s, 1.0f);
        return q * s;
    }
    return -__logf(1.0f - q);
}
// 1 - e^-x, x >= 0 (a hazard -> probability).  FP64: -expm1(-x).  Float:
// the series x sum_{k>=0} (-x)^k / (k+1)! to k = 8 below x = 1/4
// (truncation < x^9 / 10! < 1e-11), above it 1 - e^-x with the hardware exp
// (relative error < 2e-6 on a value >= 0.22).
__device__ __forceinline__ double m_one_minus_exp(double x) { return -expm1(-x); }
__device__ __forceinline__ float m_one_minus_exp(float x) {
    if (x < 0.25f) {
        float s = 1.0f / 362880.0f;
        s = fmaf(-x, s, 1.0f / 40320.0f); s = fmaf(-x, s, 1.0f / 5040.0f); s = fmaf(-x, s, 1.0f / 720.0f);
        s = fmaf(-x, s, 1.0f / 120.0f);   s = fmaf(-x, s, 1.0f / 24.0f);   s = fmaf(-x, s, 1.0f / 6.0f);
        s = fmaf(-x, s, 0.5f);            s = fmaf(-x, s, 1.0f);
        return x * s;
    }
    return 1.0f - __expf(-x);
}
__device__ __forceinline__ double m_fmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float m_fmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double m_fmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double m_fabs(double a) { return fabs(a); }
__device__ __forceinline__ float m_fabs(float a) { return fabsf(a); }
__device__ __forceinline__ float m_fmin(float a, float b) { return fminf(a, b); }

// Uniforms from Philox words.  FP64: (w + 1) 2^-32 in (0, 1] and, for a
// 16-bit half k, (k + 1/2) 2^-16 -- the oracle's conversions.  Float: the
// same intervals built from the exponent field (no int->float convert):
// 23-bit words in (0, 1] and the identical (k + 1/2) 2^-16 halves.
__device__ __forceinline__ double u32(uint32_t w, double) { return unit_d(w); }
__device__ __forceinline__ float u32(uint32_t w, float) {
    return 2.0f - __uint_as_float(0x3f800000u | (w >> 9));
}
__device__ __forceinline__ double u16(uint32_t k, double) { return (static_cast<double>(k) + 0.5) * 1.52587890625e-05; }
__device__ __forceinline__ float u16(uint32_t k, float) {
    return __uint_as_float(0x3f800000u | (k << 7)) - 0.99999237060546875f;
}

// (cos, sin) of a uniform angle.  FP64 uses 2*pi*u like the oracle; the
// float path uses the equally uniform 2*pi*(u - 1/2) in (-pi, pi], the
// accurate range of the hardware sin/cos.
__device__ __forceinline__ void angle_cs(double u, double& c, double& s) {
    const double ph = 2.0 * 3.14159265358979323846 * u;
    c = cos(ph);
    s = sin(ph);
}
__device__ __forceinline__ void angle_cs(float u, float& c, float& s) {
    __sincosf(6.28318530717958648f * (u - 0.5f), &s, &c);
}

// ---- positions --------------------------------------------------------------
// Double position (FP64).
struct PosD {
    using Snap = double;
    double x, y, z;
    __device__ void load(const StepParams& p, uint64_t i) { x = p.x[i]; y = p.y[i]; z = p.z[i]; }
    __device__ void store(const StepParams& p, uint64_t i) const { p.x[i] = x; p.y[i] = y; p.z[i] = z; }
    __device__ double gx() const { return x; }
    __device__ double gy() const { return y; }
    __device__ double gz() const { return z; }
    __device__ Snap snap_z() const { return z; }
    __device__ double z_of(Snap s) const { return s; }
    __device__ void fold() {}
    template <class R> __device__ R rel(int a, double c) const {
        const double v = (a == 0) ? x : (a == 1) ? y : z;
        return static_cast<R>(v - c);
    }
    __device__ void drift(double vx, double vy, double vz, double dt, double) {
        x += vx * dt; y += vy * dt; z += vz * dt;
    }
    __device__ void jump(double Dx, double Dy, double Dz) { x += Dx; y += Dy; z += Dz; }
    __device__ bool finite() const { return isfinite(x) && isfinite(y) && isfinite(z); }
};

// Double anchor + float offset (MIXED).  A step adds v*dt to the float
// offset (one FFMA per axis, no conversion); every lane folds the offset
// into the anchor at each warp vote (every steps_per_vote steps), so the
// offset stays below ~1 um and its rounding below ~1e-13 m per step.
struct PosA {
    using Snap = float;
    double ax, ay, az;
    float dx, dy, dz;
    __device__ void load(const StepParams& p, uint64_t i) {
        ax = p.x[i]; ay = p.y[i]; az = p.z[i];
        dx = dy = dz = 0.0f;
    }
    __device__ void store(const StepParams& p, uint64_t i) const { p.x[i] = gx(); p.y[i] = gy(); p.z[i] = gz(); }
    __device__ double gx() const { return ax + static_cast<double>(dx); }
    __device__ double gy() const { return ay + static_cast<double>(dy); }
    __device__ double gz() const { return az + static_cast<double>(dz); }
    __device__ Snap snap_z() const { return dz; }
    __device__ double z_of(Snap s) const { return az + static_cast<double>(s); }
    __device__ void fold() {
        ax += static_cast<double>(dx); ay += static_cast<double>(dy); az += static_cast<double>(dz);
        dx = dy = dz = 0.0f;
    }
    template <class R> __device__ R rel(int a, double c) const {
        const double an = (a == 0) ? ax : (a == 1) ? ay : az;
        const float d = (a == 0) ? dx : (a == 1) ? dy : dz;
        return static_cast<R>(static_cast<float>(an - c) + d);
    }
    __device__ void drift(float vx, float vy, float vz, double, float d) {
        dx = fmaf(vx, d, dx); dy = fmaf(vy, d, dy); dz = fmaf(vz, d, dz);
    }
    // A multi-step displacement goes straight into the anchor (the jump loop
    // never leaves an offset).
    __device__ void jump(float Dx, float Dy, float Dz) {
        ax += static_cast<double>(Dx); ay += static_cast<double>(Dy); az += static_cast<double>(Dz);
    }
    __device__ bool finite() const {
        return isfinite(ax) && isfinite(ay) && isfinite(az) && isfinite(dx) && isfinite(dy) && isfinite(dz);
    }
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

// Compensated float hi/lo position (HILO), TwoSum update (Knuth, TAOCP
// vol. 2, 4.2.2).
struct PosHL {
    struct Snap { float h, l; };
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
    __device__ Snap snap_z() const { return Snap{zh, zl}; }
    __device__ double z_of(Snap s) const { return static_cast<double>(s.h) + static_cast<double>(s.l); }
    __device__ void fold() {}
    template <class R> __device__ R rel(int a, double c) const {
        const float h = (a == 0) ? xh : (a == 1) ? yh : zh;
        const float l = (a == 0) ? xl : (a == 1) ? yl : zl;
        const float ch = static_cast<float>(c);
        const float cl = static_cast<float>(c - static_cast<double>(ch));
        return static_cast<R>(((h - ch) + l) - cl);
    }
    __device__ void drift(float vx, float vy, float vz, double, float d) {
        two_sum_acc(xh, xl, vx * d);
        two_sum_acc(yh, yl, vy * d);
        two_sum_acc(zh, zl, vz * d);
    }
    __device__ void jump(float Dx, float Dy, float Dz) {
        two_sum_acc(xh, xl, Dx);
        two_sum_acc(yh, yl, Dy);
        two_sum_acc(zh, zl, Dz);
    }
    __device__ bool finite() const {
        return isfinite(xh) && isfinite(yh) && isfinite(zh) && isfinite(xl) && isfinite(yl) && isfinite(zl);
    }
};

template <int PREC> struct PosOf;
template <> struct PosOf<kPrecFP64> { using T = PosD; };
template <> struct PosOf<kPrecMixed> { using T = PosA; };
template <> struct PosOf<kPrecHiLo> { using T = PosHL; };

// ---- per-thread constants in the working precision ------------------------
template <class R>
struct Consts {
    R E0[3], G[3];
    double c[3];
    R rfU0, rfV, r0sq;
    double rfw;
    double acA[2], acw[2], acp[2];   // AC drives (time-dependent field only)
    bool ac;
    R tv[3], sv[3];          // Boris rotation vectors (RK4: B itself in tv)
    R a_uni[3];              // acceleration of a uniform field for this ion
    R q, qm, inv_m;
    double m;
    double dt, hd, dt6;      // dt, dt/2, dt/6
    R dt_r, h, dt6_r;        // the same in working precision
    R A, Amean, ug[3];       // collision clock: Q = A |v - u| + A <|th|>
    R escq[3];               // space-charge force E_sc q of this step
    bool sc;                 // space charge on (one step per launch)
    const TimeField* tf;     // time-dependent field (waveforms, TIMS) or null
    const double* tftab;     // its per-step scalars for this launch (k_tf_table)
    const double* tfrow;     // ... of the current step
    uint32_t tfstride;       // doubles per row
    // the time-dependent field's constants read by the float forms each
    // step: instrument, uniform TIMS fields, final-profile flag
    int tfc_inst;
    float tfc_ei, tfc_ef;
    bool tfc_final;
    // the lane's current TIMS profile segment (z in (ts_lo, ts_hi]):
    // mode 0 uniform, 1 constant (outside the nodes), 2 interpolated
    mutable float ts_lo, ts_hi, ts_z0, ts_idz, ts_vi, ts_dvi, ts_vf, ts_dvf;
    mutable int ts_mode;
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
    k.ac = C.ac != 0;
#pragma unroll
    for (int a = 0; a < 2; ++a) { k.acA[a] = C.ac_amp[a]; k.acw[a] = C.ac_omega[a]; k.acp[a] = C.ac_phase[a]; }
    k.dt = C.dt;
    k.hd = C.dt * 0.5;
    k.dt6 = C.dt / 6.0;
    k.dt_r = static_cast<R>(C.dt);
    k.h = static_cast<R>(C.dt * 0.5);
    k.dt6_r = static_cast<R>(C.dt / 6.0);
    k.q = static_cast<R>(q);
    k.m = m;
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
    k.Amean = static_cast<R>(C.A * C.mean_th);
}

// ---- time-dependent fields ------------------------------------------------------
constexpr double kPiD = 3.141592653589793;   // M_PI
constexpr double kMinVoltageD = 1e-12;       // MIN_VOLTAGE_THRESHOLD of the field models

// std::clamp(v, 0, 1) (NaN passes through)
__device__ __forceinline__ double clamp01(double v) { return v < 0.0 ? 0.0 : (1.0 < v ? 1.0 : v); }

// One waveform at time t, each type as WaveformConfig.h:33-188 and
// ArbitraryWaveform::evaluate (WaveformConfig.cpp:10-91) compute it.
static __device__ __noinline__ double wave_eval(const WaveConst& w, double t) {
    const double* p = w.p;
    switch (w.type) {
        case kWaveConstant: return p[0];
        case kWaveLinear: {          // start, end, t_start, t_end
            if (t < p[2]) return p[0];
            if (t >= p[3]) return w.clamp ? p[1] : p[0];
            const double duration = p[3] - p[2];
            const double t_norm = (t - p[2]) / duration;
            return p[0] + (p[1] - p[0]) * t_norm;
        }
        case kWaveQuadratic:         // a, b, c, t_start, t_end
            if (t < p[3] || t > p[4]) return p[0];
            return p[0] + p[1] * t + p[2] * t * t;
        case kWaveExponential: {     // offset, amplitude, rate, t_start, t_end
            double rel = t - p[3];
            if (t < p[3]) rel = 0.0;
            else if (t >= p[4]) rel = w.clamp ? p[4] - p[3] : 0.0;
            return p[0] + p[1] * exp(p[2] * rel);
        }
        case kWaveSinusoidal: {      // offset, amplitude, frequency, phase
            const double omega = 2.0 * kPiD * p[2];
            return p[0] + p[1] * sin(omega * t + p[3]);
        }
        case kWavePWM: {             // low, high, frequency, duty, phase, t_start, t_end
            if (p[2] <= 0.0) return p[0];
            if (t < p[5]) return p[0];
            double t_rel = t - p[5];
            if (t >= p[6]) {
                if (!w.clamp) return p[0];
                t_rel = p[6] - p[5];
            }
            const double period = 1.0 / p[2];
            const double phase_shift = p[4] / (2.0 * kPiD * p[2]);
            double phase = fmod(t_rel + phase_shift, period);
            if (phase < 0.0) phase += period;
            return (phase < p[3] * period) ? p[1] : p[0];
        }
        case kWavePulsed:            // low, high, pulse_start, pulse_width
            return (t >= p[2] && t < p[2] + p[3]) ? p[1] : p[0];
        default: {                   // arbitrary table
            const int n = w.n;
            if (!(t > w.tt[0])) return w.vv[0];          // also a NaN time
            if (t >= w.tt[n - 1]) return w.vv[n - 1];
            int lo = 0, hi = n;      // lower_bound: first tt[i] >= t, 1 <= i <= n - 1 here
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (w.tt[mid] < t) lo = mid + 1; else hi = mid;
            }
            const int i1 = lo, i0 = lo - 1;
            const double t0 = w.tt[i0], t1 = w.tt[i1], v0 = w.vv[i0], v1 = w.vv[i1];
            if (w.interp == 1) return v0;
            const double alpha = (t - t0) / (t1 - t0);
            if (w.interp == 0) return v0 + alpha * (v1 - v0);
            double m0, m1;
            if (i0 == 0) m0 = (v1 - v0) / (t1 - t0);
            else m0 = (v1 - w.vv[i0 - 1]) / (t1 - w.tt[i0 - 1]);
            if (i1 == n - 1) m1 = (v1 - v0) / (t1 - t0);
            else m1 = (w.vv[i1 + 1] - v0) / (w.tt[i1 + 1] - t0);
            const double h00 = 2 * alpha * alpha * alpha - 3 * alpha * alpha + 1;
            const double h10 = alpha * alpha * alpha - 2 * alpha * alpha + alpha;
            const double h01 = -2 * alpha * alpha * alpha + 3 * alpha * alpha;
            const double h11 = alpha * alpha * alpha - alpha * alpha;
            const double dt = t1 - t0;
            return h00 * v0 + h10 * dt * m0 + h01 * v1 + h11 * dt * m1;
        }
    }
}

// TIMS ramp fraction f(t) (TIMSAxialFieldModel.h:66-96).
__device__ __forceinline__ double tims_ramp(const TimeField& F, double t) {
    if (F.ramp_wave) return clamp01(wave_eval(F.ch[kChTimsRamp], t));
    const double t0 = F.tims_t0, t1 = F.tims_t1;
    if (t <= t0) return 0.0;
    if (t >= t1) return 1.0;
    const double duration = t1 - t0;
    if (duration <= 0.0) return 1.0;
    const double rel = t - t0;
    if (F.tims_mode == 1) {
        const double tau = F.tims_tau < 1e-30 ? 1e-30 : F.tims_tau;
        const double denom = 1.0 - exp(-duration / tau);
        if (fabs(denom) < 1e-15) return clamp01(rel / duration);
        return clamp01((1.0 - exp(-rel / tau)) / denom);
    }
    return clamp01(rel / duration);
}

// Piecewise-linear axial profile at local z (TIMSAxialFieldModel.h:98-124);
// n == 0: the uniform value.
__device__ __forceinline__ double tims_sample(const double* zn, const double* val, int n, double z, double uni) {
    if (n == 0) return uni;
    if (!(z > zn[0])) return val[0];                 // also a NaN position
    if (z >= zn[n - 1]) return val[n - 1];
    int lo = 0, hi = n;          // lower_bound, 1 <= result <= n - 1 here
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (zn[mid] < z) lo = mid + 1; else hi = mid;
    }
    const int i1 = lo, i0 = lo - 1;
    const double z0 = zn[i0], z1 = zn[i1];
    const double dz = z1 - z0;
    if (dz <= 0.0) return val[i0];
    const double alpha = (z - z0) / dz;
    return val[i0] + alpha * (val[i1] - val[i0]);
}

// Time-only part of the field of an ensemble with waveforms or the TIMS
// model at time t, in FP64 with the reference's operation order (IMS
// AnalyticalFieldModel.cpp:136-161, QuadrupoleRF :219-248, LQIT :81-134,
// TIMS TIMSAxialFieldModel.h:30-44, 126-148).  Every ion of the ensemble
// shares it at a step, so k_tf_table evaluates it once per step (and RK4
// half step) of a launch:
//   s[0] U = dc_quad + V cos(2 pi f t)      s[1] 1 if the RF term applies
//   s[2] IMS / QuadrupoleRF axial / L, LQIT axial / L^2, TIMS ramp f(t)
//   s[3] 1 if the axial term applies        s[4], s[5] AC drive E_x, E_y
//   s[6], s[7] -2 U / r0^2, 2 U / r0^2 (the float forms' coefficients)
// followed by the float block (8 floats): s[6], s[7], s[2], s[4], s[5] as
// floats, 1.0f / 0.0f for s[1] != 0 and s[3] != 0, and 0.
constexpr int kTfScalars = kTfScalarsFP64;
constexpr int kTfFloats = 8;
static __device__ __noinline__ void tf_scalars(const TimeField& F, double t, double s[kTfScalars]) {
    const double rfv = wave_eval(F.ch[kChRfV], t);
    for (int j = 0; j < kTfScalars; ++j) s[j] = 0.0;
    if (F.inst == 4 || fabs(rfv) > kMinVoltageD) {
        const double rff = wave_eval(F.ch[kChRfF], t);
        const double quad = wave_eval(F.ch[kChQuad], t);
        const double omega = 2.0 * kPiD * rff;
        s[0] = quad + rfv * cos(omega * t);
        s[1] = 1.0;
        s[6] = -2.0 * s[0] / F.r0sq;
        s[7] = 2.0 * s[0] / F.r0sq;
    }
    if (F.inst == 4) {               // TIMS
        s[2] = tims_ramp(F, t);
        s[3] = 1.0;
        return;
    }
    const double axial = wave_eval(F.ch[kChAxial], t);
    if (F.inst == 0 || fabs(axial) > kMinVoltageD) {
        s[2] = F.inst == 3 ? axial / (F.L * F.L) : axial / F.L;
        s[3] = 1.0;
    }
    if (F.inst == 3) {               // LQIT AC drives, AnalyticalFieldModel.cpp:47-61, 104-121
        if (F.ac_dipolar) {
            for (int a = 0; a < 2; ++a) {
                const double amp = wave_eval(F.ch[kChAcA + 3 * a], t);
                if (fabs(amp) <= kMinVoltageD) continue;
                const double f = wave_eval(F.ch[kChAcF + 3 * a], t);
                const double ramp = wave_eval(F.ch[kChAcR + 3 * a], t);
                const double drive = amp * ramp * cos(2.0 * kPiD * f * t + F.ac_phase[a]);
                if (fabs(drive) > kMinVoltageD) s[4 + a] = -drive / F.R;
            }
        } else {
            const double v = wave_eval(F.ch[kChAcA], t);
            if (fabs(v) > kMinVoltageD) {
                const double f = wave_eval(F.ch[kChAcF], t);
                s[4] = -v / F.R * cos(2.0 * kPiD * f * t + F.ac_phase[0]);
            }
        }
    }
}

// Float piecewise-linear profile (the float forms): reciprocal interval
// widths instead of the division.
__device__ __forceinline__ float tims_sample_f(const float* zn, const float* val, const float* idz, int n, float z,
                                               float uni) {
    if (n == 0) return uni;
    if (!(z > zn[0])) return val[0];
    if (z >= zn[n - 1]) return val[n - 1];
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (zn[mid] < z) lo = mid + 1; else hi = mid;
    }
    const int i0 = lo - 1;
    const float alpha = (z - zn[i0]) * idz[i0];
    return fmaf(alpha, val[lo] - val[i0], val[i0]);
}

// The field at one ion from the step's scalars s (tf_scalars): FP64 in the
// reference's operation order; the float forms in float from the row's float
// block, with the field's constants held by the lane (Consts: tfc_*) and the
// TIMS profiles' current segment cached per lane (the same expression as
// tims_sample_f over the cached nodes, so the same values).
template <class R>
__device__ __forceinline__ float tims_segment_sample(const Consts<R>& k, float z) {
    if (!(z > k.ts_lo && z <= k.ts_hi)) {
        const TimeField& F = *k.tf;
        const int n = F.tims_nodes;
        if (n == 0) {
            k.ts_lo = -INFINITY; k.ts_hi = INFINITY; k.ts_mode = 0;
        } else if (!(z > F.tims_zf[0])) {
            k.ts_lo = -INFINITY; k.ts_hi = F.tims_zf[0]; k.ts_mode = 1;
            k.ts_vi = F.tims_pif[0]; k.ts_vf = F.tims_final_profile ? F.tims_pff[0] : static_cast<float>(F.tims_ef);
        } else if (z >= F.tims_zf[n - 1]) {
            // z >= z[n-1] samples the last node; a z just below it lands in
            // the last interval again, so the segment starts at z[n-1] itself
            k.ts_lo = nextafterf(F.tims_zf[n - 1], -INFINITY); k.ts_hi = INFINITY; k.ts_mode = 1;
            k.ts_vi = F.tims_pif[n - 1];
            k.ts_vf = F.tims_final_profile ? F.tims_pff[n - 1] : static_cast<float>(F.tims_ef);
        } else {
            int lo = 0, hi = n;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (F.tims_zf[mid] < z) lo = mid + 1; else hi = mid;
            }
            const int i0 = lo - 1;
            k.ts_lo = F.tims_zf[i0];
            k.ts_hi = lo == n - 1 ? nextafterf(F.tims_zf[lo], -INFINITY) : F.tims_zf[lo];
            k.ts_mode = 2;
            k.ts_z0 = F.tims_zf[i0];
            k.ts_idz = F.tims_idz[i0];
            k.ts_vi = F.tims_pif[i0];
            k.ts_dvi = F.tims_pif[lo] - F.tims_pif[i0];
            if (F.tims_final_profile) {
                k.ts_vf = F.tims_pff[i0];
                k.ts_dvf = F.tims_pff[lo] - F.tims_pff[i0];
            } else {
                k.ts_vf = static_cast<float>(F.tims_ef);
                k.ts_dvf = 0.0f;
            }
        }
    }
    return z;
}

template <class R, class Pos>
__device__ __forceinline__ void tf_apply(const Consts<R>& k, const TimeField& F, const Pos& x, const double* s,
                                         R E[3]) {
    if constexpr (sizeof(R) == 4) {
        const float4 f0 = *reinterpret_cast<const float4*>(s + kTfScalars);
        const float4 f1 = *reinterpret_cast<const float4*>(s + kTfScalars + 2);
        float ex = 0.0f, ey = 0.0f, ez = 0.0f;
        const bool local = k.tfc_inst >= 3;   // LQIT, TIMS: x, y from the cylinder axis
        if (f1.y != 0.0f) {          // RF term
            ex = x.template rel<float>(0, local ? F.ox : 0.0) * f0.x;
            ey = x.template rel<float>(1, local ? F.oy : 0.0) * f0.y;
        }
        if (k.tfc_inst == 4) {
            const float zl = x.template rel<float>(2, F.oz);
            tims_segment_sample<R>(k, zl);
            float ei, ef;
            if (k.ts_mode == 2) {
                const float alpha = (zl - k.ts_z0) * k.ts_idz;
                ei = fmaf(alpha, k.ts_dvi, k.ts_vi);
                ef = k.tfc_final ? fmaf(alpha, k.ts_dvf, k.ts_vf) : k.ts_vf;
            } else if (k.ts_mode == 1) {
                ei = k.ts_vi;
                ef = k.ts_vf;
            } else {
                ei = k.tfc_ei;
                ef = k.tfc_ef;
            }
            ez = fmaf(f0.z, ef - ei, ei);
        } else if (k.tfc_inst == 3) {
            ex += f0.w;
            ey += f1.x;
            if (f1.z != 0.0f) ez = (-2.0f * f0.z) * x.template rel<float>(2, F.oz + 0.5 * F.L);
        } else if (f1.z != 0.0f) {
            ez = f0.z;
        }
        E[0] = ex; E[1] = ey; E[2] = ez;
        return;
    }
    double ex = 0.0, ey = 0.0, ez = 0.0;
    const bool local = F.inst >= 3;  // LQIT, TIMS: x, y from the cylinder axis
    if (s[1] != 0.0) {
        const double u = s[0];
        ex = -2.0 * x.template rel<double>(0, local ? F.ox : 0.0) * u / F.r0sq;
        ey = 2.0 * x.template rel<double>(1, local ? F.oy : 0.0) * u / F.r0sq;
    }
    if (F.inst == 4) {
        const double zl = x.template rel<double>(2, F.oz);
        const double f = s[2];
        const double ei = tims_sample(F.tims_z, F.tims_pi, F.tims_nodes, zl, F.tims_ei);
        const double ef = tims_sample(F.tims_z, F.tims_pf, F.tims_final_profile ? F.tims_nodes : 0, zl, F.tims_ef);
        ez = (1.0 - f) * ei + f * ef;
    } else if (F.inst == 3) {
        ex += s[4];
        ey += s[5];
        if (s[3] != 0.0) ez = -2.0 * s[2] * (x.template rel<double>(2, F.oz) - 0.5 * F.L);
    } else if (s[3] != 0.0) {
        ez = s[2];
    }
    E[0] = static_cast<R>(ex); E[1] = static_cast<R>(ey); E[2] = static_cast<R>(ez);
}

#ifdef ICB_TF_TABLE_UNIT
// Per-step scalars of the launch for the ensembles with a time-dependent
// field (built in the FP64 unit only, without FMA contraction, for every
// precision): block e fills rows k = 0..K of the table of chunk ensemble e
// (global index ens_base + e; stage 0 at t_k, stage 1 at t_k + dt/2 for
// RK4), t_k accumulated as the step kernel does (t_{k+1} = t_k + dt) into
// tseq first, so each lane reads the values it would compute.
__global__ void k_tf_table(const StepParams p, double* tab, double* tseq, uint32_t stride) {
    const uint32_t e = blockIdx.x;
    const EnsConst& C = p.ens[e];
    if (!C.tf) return;
    const uint32_t g = p.ens_base + e;
    const TimeField& F = p.tfield[g];
    const uint32_t rows = p.n_steps + 1u;
    double* T = tab + static_cast<size_t>(g) * rows * stride;
    double* ts = tseq + static_cast<size_t>(g) * rows;
    if (threadIdx.x == 0) {
        double t = p.t_dev[g];
        for (uint32_t k = 0; k < rows; ++k) {
            ts[k] = t;
            t = t + C.dt;
        }
    }
    __syncthreads();
    const double hd = C.dt * 0.5;
    for (uint32_t k = threadIdx.x; k < rows; k += blockDim.x) {
        double* row = T + static_cast<size_t>(k) * stride;
        const double t = ts[k];
        double sc[kTfScalars];
        auto put = [&](double* r) {
            for (int j = 0; j < kTfScalars; ++j) r[j] = sc[j];
            float* f = reinterpret_cast<float*>(r + kTfScalars);
            f[0] = static_cast<float>(sc[6]);
            f[1] = static_cast<float>(sc[7]);
            f[2] = static_cast<float>(sc[2]);
            f[3] = static_cast<float>(sc[4]);
            f[4] = static_cast<float>(sc[5]);
            f[5] = sc[1] != 0.0 ? 1.0f : 0.0f;
            f[6] = sc[3] != 0.0 ? 1.0f : 0.0f;
            f[7] = 0.0f;
        };
        tf_scalars(F, t, sc);
        put(row);
        if (stride > static_cast<uint32_t>(kTfRowScalars)) {
            tf_scalars(F, t + hd, sc);
            put(row + kTfRowScalars);
        }
    }
}
#endif

// ---- fields -----------------------------------------------------------------
template <class R, int FIELD, class Pos>
__device__ __forceinline__ void efield(const Consts<R>& k, const Pos& x, double t, R E[3], int stage = 0) {
    if constexpr (FIELD == kFieldUniform) {
        E[0] = k.E0[0]; E[1] = k.E0[1]; E[2] = k.E0[2];
        return;
    } else if constexpr (FIELD == kFieldLinear) {
#pragma unroll
        for (int a = 0; a < 3; ++a) E[a] = k.E0[a] + k.G[a] * x.template rel<R>(a, k.c[a]);
        return;
    } else {
        if (k.tf != nullptr) {
            // stage 0 at t_k, 1 at t_k + dt/2 (RK4), 2 at t_k + dt = the next row
            const double* row = k.tfrow + (stage == 0 ? 0 : stage == 1 ? kTfRowScalars : static_cast<int>(k.tfstride));
            tf_apply<R>(k, *k.tf, x, row, E);
            return;
        } else {
#pragma unroll
            for (int a = 0; a < 3; ++a) E[a] = k.E0[a] + k.G[a] * x.template rel<R>(a, k.c[a]);
            // AnalyticalFieldModel.cpp:152-158: U = dc_quad + V cos(w t);
            // E_x = -2 x U / r0^2, E_y = 2 y U / r0^2, x and y from the
            // quadrupole axis (c[0], c[1]: 0 for IMS / QuadrupoleRF, the
            // cylinder axis for the LQIT, AnalyticalFieldModel.cpp:90-103).
            // Without an RF voltage the LQIT's x, y come from G = 0.
            if (k.rfV != R(0)) {
                const R U = k.rfU0 + k.rfV * static_cast<R>(cos(k.rfw * t));
                const R px = x.template rel<R>(0, k.c[0]), py = x.template rel<R>(1, k.c[1]);
                E[0] = R(-2.0) * px * U / k.r0sq;
                E[1] = R(2.0) * py * U / k.r0sq;
            }
        }
        // LQIT AC drives (AnalyticalFieldModel.cpp:104-121)
        if (k.ac) {
            E[0] += static_cast<R>(k.acA[0] * cos(k.acw[0] * t + k.acp[0]));
            E[1] += static_cast<R>(k.acA[1] * cos(k.acw[1] * t + k.acp[1]));
        }
    }
}

// ---- pushers ------------------------------------------------------------------
// Boris exactly as BorisStrategy.cpp:50-97, including x += v_plus * dt.
// Returns |v_plus|_1, the L1 speed of this step's drift.
template <class R, int FIELD, bool MAG, class Pos>
__device__ __forceinline__ R boris(const Consts<R>& k, Pos& x, R v[3], double t) {
    R a[3];
    if constexpr (FIELD == kFieldUniform) {
        a[0] = k.a_uni[0]; a[1] = k.a_uni[1]; a[2] = k.a_uni[2];
    } else {
        R E[3];
        efield<R, FIELD>(k, x, t, E);
        // total force q E + q E_sc, then / m (ForceRegistry.cpp:76-87)
        if constexpr (sizeof(R) == 8) {
            if (k.sc) {
#pragma unroll
                for (int c = 0; c < 3; ++c) a[c] = (E[c] * k.q + k.escq[c]) / static_cast<R>(k.m);
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c) a[c] = (E[c] * k.q) / static_cast<R>(k.m);
            }
        } else {
            if (k.sc) {
#pragma unroll
                for (int c = 0; c < 3; ++c) a[c] = (E[c] * k.q + k.escq[c]) * k.inv_m;
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c) a[c] = E[c] * k.qm;
            }
        }
    }
    R vm[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) vm[c] = v[c] + a[c] * k.h;
    R vp[3];
    if constexpr (MAG) {
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
    x.drift(vp[0], vp[1], vp[2], k.dt, k.dt_r);
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = vp[c] + a[c] * k.h;
    return fabs(vp[0]) + fabs(vp[1]) + fabs(vp[2]);
}

// RK4 acceleration: (E q [+ (v x B) q]) * (1/m)  (RK4Strategy.cpp:236-243,
// MagneticFieldForce.cpp:61-88; magnetic force is registered for non-Boris
// integrators, PhysicsSetup.cpp:206).
template <class R, int FIELD, bool MAG, class Pos>
__device__ __forceinline__ void rk4_acc(const Consts<R>& k, const Pos& x, const R v[3], double t, R acc[3],
                                        int stage) {
    R E[3];
    efield<R, FIELD>(k, x, t, E, stage);
    R F[3] = {E[0] * k.q, E[1] * k.q, E[2] * k.q};
    if constexpr (MAG) {
        const R B0 = k.tv[0], B1 = k.tv[1], B2 = k.tv[2];
        const R cx = v[1] * B2 - v[2] * B1;
        const R cy = v[2] * B0 - v[0] * B2;
        const R cz = v[0] * B1 - v[1] * B0;
        F[0] += cx * k.q; F[1] += cy * k.q; F[2] += cz * k.q;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] = F[c] * k.inv_m;
}

// RK4 batch stages (RK4Strategy.cpp:255-358).  Returns the L1 norm of the
// step's displacement divided by dt.
template <class R, int FIELD, bool MAG, class Pos>
__device__ __forceinline__ R rk4(const Consts<R>& k, Pos& x, R v[3], double t) {
    const double dt = k.dt;
    const double hd = k.hd;
    const R h = k.h;
    const R dtr = k.dt_r;
    const Pos x0 = x;
    const R v0[3] = {v[0], v[1], v[2]};
    R k1a[3], k2a[3], k3a[3], k4a[3], v2[3], v3[3], v4[3];
    rk4_acc<R, FIELD, MAG>(k, x0, v0, t, k1a, 0);
    Pos p2 = x0; p2.drift(v0[0], v0[1], v0[2], hd, h);
#pragma unroll
    for (int c = 0; c < 3; ++c) v2[c] = v0[c] + k1a[c] * h;
    rk4_acc<R, FIELD, MAG>(k, p2, v2, t + hd, k2a, 1);
    Pos p3 = x0; p3.drift(v2[0], v2[1], v2[2], hd, h);
#pragma unroll
    for (int c = 0; c < 3; ++c) v3[c] = v0[c] + k2a[c] * h;
    rk4_acc<R, FIELD, MAG>(k, p3, v3, t + hd, k3a, 1);
    Pos p4 = x0; p4.drift(v3[0], v3[1], v3[2], dt, dtr);
#pragma unroll
    for (int c = 0; c < 3; ++c) v4[c] = v0[c] + k3a[c] * dtr;
    rk4_acc<R, FIELD, MAG>(k, p4, v4, t + dt, k4a, 2);
    R dv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) dv[c] = v0[c] + v2[c] * R(2.0) + v3[c] * R(2.0) + v4[c];
    x = x0;
    x.drift(dv[0], dv[1], dv[2], k.dt6, k.dt6_r);
    const R s = k.dt6_r;
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = v0[c] + (k1a[c] + k2a[c] * R(2.0) + k3a[c] * R(2.0) + k4a[c]) * s;
    return (fabs(dv[0]) + fabs(dv[1]) + fabs(dv[2])) * R(1.0 / 6.0);
}

// ---- null-collision HSS -------------------------------------------------------
// The reference draws a Maxwell-Boltzmann neutral every step and collides
// with probability p = 1 - exp(-n sigma |v - v_n| dt).  Here each step has a
// candidate with probability Q = A (b + <|th|>) (A = n sigma dt, b >= |v - u|,
// th = v_n - u the neutral's thermal part); a candidate draws th from
// f(th) (b + |th|) / (b + <|th|>) and is accepted with p / (A (b + |th|)) <= 1,
// so the joint law of (collision, v_n) per step is f(v_n) p, the reference's.
// The mixture is sampled without branches: |th|^2/sigma^2 = -2 ln u1 -
// 2 ln u2 * s with s = cos^2(2 pi u3) (chi^2_3, the thermal part, probability
// b/(b+<|th|>)) or s = 1 (chi^2_4, the |th|-weighted part), and an isotropic
// direction.
//
// FP64 uses b = |v - u| (exact sqrt, as the oracle).  The float path uses
// the sqrt-free bound b = (w^2 + c^2) / (2c) >= |w| (AM-GM), c = |w| at the
// lane's last candidate, which keeps Q within ~0.1% of the tight value.
template <class R>
struct ClockBound {
    R inv2c, halfc;      // b = w2 * inv2c + halfc  (float path)
    __device__ void set(R w2) {
        const R c = m_fmax(m_sqrt(w2), R(1e-3));
        inv2c = R(0.5) / c;
        halfc = R(0.5) * c;
    }
};

template <class R>
__device__ __forceinline__ bool clock_tick(const Consts<R>& k, const R v[3], R& S, R U, R& b,
                                           const ClockBound<R>& cb, uint32_t& ovf) {
    const R wx = v[0] - k.ug[0], wy = v[1] - k.ug[1], wz = v[2] - k.ug[2];
    const R w2 = wx * wx + wy * wy + wz * wz;
    if constexpr (sizeof(R) == 8) b = m_sqrt(w2);
    else b = w2 * cb.inv2c + cb.halfc;
    R Q = k.A * b + k.Amean;
    if (Q > R(1)) { Q = R(1); ++ovf; }
    S = S - S * Q;
    return S < U;
}

// Candidate processing (the steps of the oracle's hss_nullcoll).
// SKIP (skip clock): the event is first thinned with Q(b)/Q*, b = |v - u|
// exact; clk receives the new optical depth.  Otherwise (per-step clock) b
// is the clock's bound and clk receives the new threshold U.
// Returns 0 when the skip-clock event is thinned away, 1 when the candidate
// is rejected, 2 on a collision (v updated).
// cos(chi) from the interaction-potential table: bilinear in (ln E, b),
// E clamped to the table range.
template <class R>
__device__ __forceinline__ R ipm_table_cos(const StepParams& p, R E, R bn) {
    const int nE = p.ipm_nE, nb = p.ipm_nb;
    R t = (m_log(E) - static_cast<R>(p.ipm_lnEmin)) * static_cast<R>(p.ipm_inv_dlnE);
    t = m_fmin(m_fmax(t, R(0)), static_cast<R>(nE - 1));
    const int k = min(static_cast<int>(t), nE - 2);
    const R ft = t - static_cast<R>(k);
    const R u = bn * static_cast<R>(nb - 1);
    const int j = min(static_cast<int>(u), nb - 2);
    const R fu = u - static_cast<R>(j);
    const float* r0 = p.ipm_tab + static_cast<size_t>(k) * nb + j;
    const float* r1 = r0 + nb;
    const R c00 = static_cast<R>(__ldg(r0)), c01 = static_cast<R>(__ldg(r0 + 1));
    const R c10 = static_cast<R>(__ldg(r1)), c11 = static_cast<R>(__ldg(r1 + 1));
    const R lo = c00 + fu * (c01 - c00);
    const R hi = c10 + fu * (c11 - c10);
    return lo + ft * (hi - lo);
}

// Relative velocity g turned by the polar angle chi (cos cx, sin sx) about
// its own direction, azimuth (cp, sp) (Bird 1994, eq. 2.22).
template <class R>
__device__ __forceinline__ void deflect(const R g3[3], R g, R cx, R sx, R cp, R sp, R out[3]) {
    const R gyz = m_sqrt(g3[1] * g3[1] + g3[2] * g3[2]);
    if (gyz > R(1e-6) * g) {
        const R ig = R(1) / gyz;
        out[0] = g3[0] * cx + sx * sp * gyz;
        out[1] = g3[1] * cx + sx * (g * g3[2] * cp - g3[0] * g3[1] * sp) * ig;
        out[2] = g3[2] * cx - sx * (g * g3[1] * cp + g3[0] * g3[2] * sp) * ig;
    } else {
        out[0] = g3[0] * cx;
        out[1] = g * sx * cp;
        out[2] = g * sx * sp;
    }
}

// A collision whose deflection waits for the warp's network evaluation.
template <class R>
struct IpmPend {
    R g3[3], g, vn[3], E, bn, cp, sp;
};

// v after an elastic deflection of the relative velocity by chi.
template <class R>
__device__ __forceinline__ void ipm_apply(const EnsConst& C, R v[3], const IpmPend<R>& ip, R cx, double mi_d) {
    R mi, mn, inv_mt;
    if constexpr (sizeof(R) == 8) {
        mi = mi_d; mn = C.m_gas; inv_mt = 1.0 / (mi_d + C.m_gas);
    } else {
        mi = static_cast<float>(mi_d); mn = C.fm_gas; inv_mt = __frcp_rn(mi + mn);
    }
    const R fac = mn * inv_mt;
    const R sx = m_sqrt(m_fmax(R(0), R(1) - cx * cx));
    R gp[3];
    deflect<R>(ip.g3, ip.g, cx, sx, ip.cp, ip.sp, gp);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const R vcom = (v[c] * mi + ip.vn[c] * mn) * inv_mt;
        v[c] = vcom + gp[c] * fac;
    }
}

// EHSS scattering (CollisionKernels::ehss_collision, CollisionKernels.cpp:
// 13-137, 220-381): a uniformly random orientation of the molecule
// (Shoemake quaternion from three uniforms, CollisionGeometry.cpp:30-59) in
// the frame of the collision axis g/|g|, the maximal impact parameter of the
// rotated atoms plus the gas radius, impact points uniform in that disk
// until the straight trajectory meets an atom (at most 256 draws; the disk
// grows by 1.5 after 64), the earliest contact's normal, specular
// reflection of g and the centre-of-mass transform.  No hit in 256 draws
// leaves v unchanged, as in the reference.  Philox substreams: 2 for the
// orientation, 8 + a/2 for draw a.
template <class R>
__device__ void ehss_scatter(const StepParams& p, uint32_t eg, R v[3], const R vn[3], const R g3[3], R g, R mi,
                             R mn, R inv_mt, R fac, const uint32_t* rk, uint32_t id, uint32_t step) {
    const int a0 = p.ehss_off[eg], a1 = p.ehss_off[eg + 1];
    if (a1 <= a0 || !(g > R(0))) return;
    const R rg = static_cast<R>(p.ehss_rgas[eg]);
    const R ax[3] = {g3[0] / g, g3[1] / g, g3[2] / g};
    // orthonormal basis of the impact plane (CollisionGeometry.cpp:11-28)
    const R ea[3] = {m_fabs(ax[0]) < R(0.9) ? R(1) : R(0), m_fabs(ax[0]) < R(0.9) ? R(0) : R(1), R(0)};
    R t1[3] = {ax[1] * ea[2] - ax[2] * ea[1], ax[2] * ea[0] - ax[0] * ea[2], ax[0] * ea[1] - ax[1] * ea[0]};
    R nt = R(1) / m_sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    t1[0] *= nt; t1[1] *= nt; t1[2] *= nt;
    R t2[3] = {ax[1] * t1[2] - ax[2] * t1[1], ax[2] * t1[0] - ax[0] * t1[2], ax[0] * t1[1] - ax[1] * t1[0]};
    nt = R(1) / m_sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
    t2[0] *= nt; t2[1] *= nt; t2[2] *= nt;
    // random orientation, expressed in the collision-axis frame: Rm = B Q
    const U4 ro = philox4x32_10_rk(id, step, 2u, 0u, rk);
    const R u1 = u32(ro.x, R(0));
    R s2, c2, s3, c3;
    angle_cs(u32(ro.y, R(0)), c2, s2);
    angle_cs(u32(ro.z, R(0)), c3, s3);
    const R qa = m_sqrt(R(1) - u1), qb = m_sqrt(u1);
    const R qx = qa * s2, qy = qa * c2, qz = qb * s3, qw = qb * c3;
    const R Q[3][3] = {{R(1) - R(2) * (qy * qy + qz * qz), R(2) * (qx * qy - qz * qw), R(2) * (qx * qz + qy * qw)},
                       {R(2) * (qx * qy + qz * qw), R(1) - R(2) * (qx * qx + qz * qz), R(2) * (qy * qz - qx * qw)},
                       {R(2) * (qx * qz - qy * qw), R(2) * (qy * qz + qx * qw), R(1) - R(2) * (qx * qx + qy * qy)}};
    const R B[3][3] = {{t1[0], t2[0], ax[0]}, {t1[1], t2[1], ax[1]}, {t1[2], t2[2], ax[2]}};
    R Rm[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Rm[i][j] = B[i][0] * Q[0][j] + B[i][1] * Q[1][j] + B[i][2] * Q[2][j];
    auto rot = [&](const double4& c, R out[3]) {
        const R cx = static_cast<R>(c.x), cy = static_cast<R>(c.y), cz = static_cast<R>(c.z);
#pragma unroll
        for (int i = 0; i < 3; ++i) out[i] = Rm[i][0] * cx + Rm[i][1] * cy + Rm[i][2] * cz;
    };
    R bmax = R(0);
    for (int j = a0; j < a1; ++j) {
        const double4 c = p.ehss_atoms[j];
        R ra[3];
        rot(c, ra);
        const R sra = ax[0] * ra[0] + ax[1] * ra[1] + ax[2] * ra[2];
        const R px = ra[0] - ax[0] * sra, py = ra[1] - ax[1] * sra, pz = ra[2] - ax[2] * sra;
        const R cur = m_sqrt(px * px + py * py + pz * pz) + static_cast<R>(c.w);
        if (cur > bmax) bmax = cur;
    }
    bmax += rg;
    U4 w{};
    for (int at = 0; at < 256; ++at) {
        if ((at & 1) == 0) w = philox4x32_10_rk(id, step, 8u + static_cast<uint32_t>(at >> 1), 0u, rk);
        const uint32_t wa = (at & 1) ? w.z : w.x, wb = (at & 1) ? w.w : w.y;
        const R bb = bmax * m_sqrt(u32(wa, R(0)));
        R cph, sph;
        angle_cs(u32(wb, R(0)), cph, sph);
        const R off[3] = {t1[0] * (bb * cph) + t2[0] * (bb * sph), t1[1] * (bb * cph) + t2[1] * (bb * sph),
                          t1[2] * (bb * cph) + t2[2] * (bb * sph)};
        bool hit = false;
        R best = R(0), nrm[3] = {R(0), R(0), R(0)};
        for (int j = a0; j < a1; ++j) {
            const double4 c = p.ehss_atoms[j];
            R ra[3];
            rot(c, ra);
            const R rs = static_cast<R>(c.w) + rg;
            const R rel[3] = {off[0] - ra[0], off[1] - ra[1], off[2] - ra[2]};
            const R ss = ax[0] * rel[0] + ax[1] * rel[1] + ax[2] * rel[2];
            const R dv[3] = {rel[0] - ax[0] * ss, rel[1] - ax[1] * ss, rel[2] - ax[2] * ss};
            const R d2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
            if (d2 <= rs * rs) {
                const R hgt = m_sqrt(m_fmax(R(0), rs * rs - d2));
                const R sh = ss - hgt;
                if (!hit || sh < best) {
                    const R ph[3] = {rel[0] - ax[0] * sh, rel[1] - ax[1] * sh, rel[2] - ax[2] * sh};
                    const R pr2 = ph[0] * ph[0] + ph[1] * ph[1] + ph[2] * ph[2];
                    if (pr2 <= R(1e-24)) {
                        nrm[0] = -ax[0]; nrm[1] = -ax[1]; nrm[2] = -ax[2];
                    } else {
                        const R ip = R(1) / m_sqrt(pr2);
                        nrm[0] = ph[0] * ip; nrm[1] = ph[1] * ip; nrm[2] = ph[2] * ip;
                        if (ax[0] * nrm[0] + ax[1] * nrm[1] + ax[2] * nrm[2] > R(0)) {
                            nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
                        }
                    }
                    hit = true;
                    best = sh;
                }
            }
        }
        if (hit) {
            const R vd = g3[0] * nrm[0] + g3[1] * nrm[1] + g3[2] * nrm[2];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const R gr = g3[c] - nrm[c] * (R(2) * vd);
                const R vcom = (v[c] * mi + vn[c] * mn) * inv_mt;
                v[c] = vcom + gr * fac;
            }
            return;
        }
        if (at == 64) bmax *= R(1.5);
    }
}

// A parabolic-flow ensemble (C.flow) calls this with v in the local gas
// frame (v_z - u_z at the ion) and C.ug = 0.
template <class R, bool SKIP, int COLL>
__device__ __forceinline__ int candidate(const EnsConst& C, R v[3], R& clk, R qstar, R Amean, R b, double mi_d,
                                         const uint32_t* rk, uint32_t id, uint32_t step, const StepParams& p,
                                         IpmPend<R>* ip, uint32_t eg, const PhiloxIon& pq) {
    constexpr bool LANG = COLL == kCollLangevin;
    R A, mean_th, sig_n, ug[3], mi, mn, inv_mt, fac;
    if constexpr (sizeof(R) == 8) {
        A = C.A; mean_th = C.mean_th; sig_n = C.sig_n;
        ug[0] = C.ug[0]; ug[1] = C.ug[1]; ug[2] = C.ug[2];
        mi = mi_d; mn = C.m_gas;
        inv_mt = 1.0 / (mi_d + C.m_gas);
        fac = mn * inv_mt;
    } else {
        A = C.fA; mean_th = C.fmean_th; sig_n = C.fsig_n;
        ug[0] = C.fug[0]; ug[1] = C.fug[1]; ug[2] = C.fug[2];
        mi = static_cast<float>(mi_d); mn = C.fm_gas;
        inv_mt = __frcp_rn(mi + mn);
        fac = mn * inv_mt;
    }
    // The hard-sphere kinds run without branches: every event lane draws
    // both Philox blocks and forms the scattered velocity, and the outcome
    // (thinned, rejected, collided) selects what is kept.  The values are
    // those of the early-exit form.
    constexpr bool kFlat = COLL == kCollHSS || COLL == kCollLangevin;
    const U4 r0 = philox_ion(pq, step, 0u, rk);   // = philox4x32_10_rk(id, step, 0, 0, rk)
    R uc = u32(r0.y, R(0));
    bool kept = true;                 // not thinned away
    if constexpr (SKIP) {
        clk = -m_log(u32(r0.x, R(0)));
        const R wx = v[0] - ug[0], wy = v[1] - ug[1], wz = v[2] - ug[2];
        b = m_sqrt(wx * wx + wy * wy + wz * wz);
        const R Q = A * b + Amean;
        kept = uc * qstar < Q;
        if constexpr (!kFlat) {
            if (!kept) return 0;
        }
        uc = uc * qstar / Q;          // uniform on (0, 1) given the acceptance
    } else {
        clk = u32(r0.x, R(0));
    }
    const U4 r1 = philox_ion(pq, step, 1u, rk);
    // Langevin capture: Maxwellian neutral (the thermal branch), every event collides
    const bool thermal = LANG || (uc * (b + mean_th) < b);
    R c3, s3;
    angle_cs(u16(r1.y >> 16, R(0)), c3, s3);
    const R sfac = thermal ? c3 * c3 : R(1);
    const R r2 = R(-2.0) * (m_log(u32(r0.w, R(0))) + m_log(u32(r1.x, R(0))) * sfac);
    const R rad = sig_n * m_sqrt(r2);
    const R ct = R(2.0) * u16(r1.y & 0xffffu, R(0)) - R(1.0);
    const R st = m_sqrt(m_fmax(R(0), R(1.0) - ct * ct));
    R cp, sp;
    angle_cs(u16(r1.z >> 16, R(0)), cp, sp);
    const R vn[3] = {ug[0] + rad * (st * cp), ug[1] + rad * (st * sp), ug[2] + rad * ct};
    const R gx = v[0] - vn[0], gy = v[1] - vn[1], gz = v[2] - vn[2];
    const R g = m_sqrt(gx * gx + gy * gy + gz * gz);
    const R q = A * (b + rad);
    const R pc = m_one_minus_exp(A * g);
    const bool hit = kept && (LANG || u32(r0.z, R(0)) * q < pc);
    if constexpr (!kFlat) {
        if (!hit) return 1;
    }
    if constexpr (COLL == kCollEHSS) {
        const R g3[3] = {gx, gy, gz};
        ehss_scatter<R>(p, eg, v, vn, g3, g, mi, mn, inv_mt, fac, rk, id, step);
        return 2;
    }
    if constexpr (COLL == kCollIPMMLP) {
        // deflection after the warp's network evaluation
        const R mu = mi * fac;   // m_i m_n / (m_i + m_n); the product m_i m_n underflows in float
        ip->E = R(0.5) * mu * (g * g);
        ip->bn = m_sqrt(u16(r1.z & 0xffffu, R(0)));
        angle_cs(u16(r1.w >> 16, R(0)), ip->cp, ip->sp);
        ip->g3[0] = gx; ip->g3[1] = gy; ip->g3[2] = gz;
        ip->g = g;
        ip->vn[0] = vn[0]; ip->vn[1] = vn[1]; ip->vn[2] = vn[2];
        return 3;
    }
    if constexpr (COLL == kCollIPMTable || COLL == kCollIPMQuad) {
        // elastic deflection by chi(E, b): b uniform in area below b_max;
        // chi from the table, or (kCollIPMQuad) by the FP64 quadrature of
        // this collision's own (E, b)
        const R mu = mi * fac;   // m_i m_n / (m_i + m_n); the product m_i m_n underflows in float
        const R E = R(0.5) * mu * (g * g);
        const R bn = m_sqrt(u16(r1.z & 0xffffu, R(0)));
        R cx;
        if constexpr (COLL == kCollIPMQuad)
            cx = static_cast<R>(ipm_cos_chi(p.ipm_pot, *static_cast<const GLNodes*>(p.ipm_gl),
                                            static_cast<double>(E), static_cast<double>(bn) * p.ipm_bmax));
        else
            cx = ipm_table_cos<R>(p, E, bn);
        const R sx = m_sqrt(m_fmax(R(0), R(1) - cx * cx));
        R cp2, sp2;
        angle_cs(u16(r1.w >> 16, R(0)), cp2, sp2);
        const R g3[3] = {gx, gy, gz};
        R gp[3];
        deflect<R>(g3, g, cx, sx, cp2, sp2, gp);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const R vcom = (v[c] * mi + vn[c] * mn) * inv_mt;
            v[c] = vcom + gp[c] * fac;
        }
        return 2;
    }
    const R ct2 = R(2.0) * u16(r1.z & 0xffffu, R(0)) - R(1.0);
    const R st2 = m_sqrt(m_fmax(R(0), R(1.0) - ct2 * ct2));
    R cp2, sp2;
    angle_cs(u16(r1.w >> 16, R(0)), cp2, sp2);
    const R dir[3] = {st2 * cp2, st2 * sp2, ct2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const R vcom = (v[c] * mi + vn[c] * mn) * inv_mt;
        const R vs = vcom + (dir[c] * g) * fac;
        v[c] = hit ? vs : v[c];
    }
    return hit ? 2 : (kept ? 1 : 0);
}

// Candidate of an HSS gas mixture (HSSCollisionHandler.cpp:105-249): the
// reference draws a neutral of every component, collides with probability
// 1 - exp(-K), K = sum_j n_j sigma_j |v - v_j| dt, and picks component i
// with probability k_i / K.  Here the candidate (majorant Q = sum_i A_i
// (b + <|th_i|>)) picks component i with probability A_i (b + <|th_i|>) / Q,
// draws its neutral from the size-biased mixture as in the single-gas case,
// draws the other components' neutrals from their Maxwellians (Philox
// substreams 4 + j), and accepts with g_i (1 - exp(-K)) / (K (b + |th_i|)):
// the joint law of (collision, component, v_n) per step is the reference's.
template <class R, bool SKIP>
__device__ __forceinline__ int candidate_mix(const EnsConst& C, const MixConst& M, R v[3], R& clk, R qstar,
                                             R Amean, R b, double mi_d, const uint32_t* rk, uint32_t id,
                                             uint32_t step, const PhiloxIon& pq) {
    constexpr bool D = sizeof(R) == 8;
    R ug[3], mi;
    if constexpr (D) {
        ug[0] = C.ug[0]; ug[1] = C.ug[1]; ug[2] = C.ug[2];
        mi = mi_d;
    } else {
        ug[0] = C.fug[0]; ug[1] = C.fug[1]; ug[2] = C.fug[2];
        mi = static_cast<float>(mi_d);
    }
    const int n = M.n;
    auto Ai = [&](int i) -> R { if constexpr (D) return M.A[i]; else return M.fA[i]; };
    auto Mi = [&](int i) -> R { if constexpr (D) return M.mean_th[i]; else return M.fmean_th[i]; };
    auto Si = [&](int i) -> R { if constexpr (D) return M.sig_n[i]; else return M.fsig_n[i]; };
    auto Gm = [&](int i) -> R { if constexpr (D) return M.m[i]; else return M.fm[i]; };
    const U4 r0 = philox_ion(pq, step, 0u, rk);
    R uc = u32(r0.y, R(0));
    if constexpr (SKIP) {
        clk = -m_log(u32(r0.x, R(0)));
        const R wx = v[0] - ug[0], wy = v[1] - ug[1], wz = v[2] - ug[2];
        b = m_sqrt(wx * wx + wy * wy + wz * wz);
        const R A = D ? static_cast<R>(C.A) : static_cast<R>(C.fA);
        const R Q = A * b + Amean;
        if (!(uc * qstar < Q)) return 0;
        uc = uc * qstar / Q;
    } else {
        clk = u32(r0.x, R(0));
    }
    // component choice
    R qtot = R(0);
    for (int i = 0; i < n; ++i) qtot += Ai(i) * (b + Mi(i));
    const R target = uc * qtot;
    int ci = n - 1;
    R cum = R(0);
    for (int i = 0; i < n - 1; ++i) {
        const R qi = Ai(i) * (b + Mi(i));
        if (target < cum + qi) { ci = i; break; }
        cum += qi;
    }
    const R qsel = Ai(ci) * (b + Mi(ci));
    const R uci = m_fmin((target - cum) / qsel, R(1));
    const U4 r1 = philox_ion(pq, step, 1u, rk);
    const bool thermal = uci * (b + Mi(ci)) < b;
    R c3, s3;
    angle_cs(u16(r1.y >> 16, R(0)), c3, s3);
    const R sfac = thermal ? c3 * c3 : R(1);
    const R r2 = R(-2.0) * (m_log(u32(r0.w, R(0))) + m_log(u32(r1.x, R(0))) * sfac);
    const R rad = Si(ci) * m_sqrt(r2);
    const R ct = R(2.0) * u16(r1.y & 0xffffu, R(0)) - R(1.0);
    const R st = m_sqrt(m_fmax(R(0), R(1.0) - ct * ct));
    R cp, sp;
    angle_cs(u16(r1.z >> 16, R(0)), cp, sp);
    const R vn[3] = {ug[0] + rad * (st * cp), ug[1] + rad * (st * sp), ug[2] + rad * ct};
    const R gx = v[0] - vn[0], gy = v[1] - vn[1], gz = v[2] - vn[2];
    const R g = m_sqrt(gx * gx + gy * gy + gz * gz);
    R K = Ai(ci) * g;
    for (int j = 0; j < n; ++j) {
        if (j == ci) continue;
        const U4 rj = philox4x32_10_rk(id, step, 4u + static_cast<uint32_t>(j), 0u, rk);
        const R ra = m_sqrt(R(-2.0) * m_log(u32(rj.x, R(0))));
        const R rb = m_sqrt(R(-2.0) * m_log(u32(rj.y, R(0))));
        R ca, sa, cb2, sb2;
        angle_cs(u16(rj.z >> 16, R(0)), ca, sa);
        angle_cs(u16(rj.z & 0xffffu, R(0)), cb2, sb2);
        const R s = Si(j);
        const R hx = v[0] - (ug[0] + s * ra * ca);
        const R hy = v[1] - (ug[1] + s * ra * sa);
        const R hz = v[2] - (ug[2] + s * rb * cb2);
        K += Ai(j) * m_sqrt(hx * hx + hy * hy + hz * hz);
    }
    const R pc = m_one_minus_exp(K);
    if (!(u32(r0.z, R(0)) * K * (b + rad) < g * pc)) return 1;
    const R mn = Gm(ci);
    R inv_mt;
    if constexpr (D) inv_mt = R(1) / (mi + mn);
    else inv_mt = __frcp_rn(mi + mn);
    const R fac = mn * inv_mt;
    const R ct2 = R(2.0) * u16(r1.z & 0xffffu, R(0)) - R(1.0);
    const R st2 = m_sqrt(m_fmax(R(0), R(1.0) - ct2 * ct2));
    R cp2, sp2;
    angle_cs(u16(r1.w >> 16, R(0)), cp2, sp2);
    const R dir[3] = {st2 * cp2, st2 * sp2, ct2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const R vcom = (v[c] * mi + vn[c] * mn) * inv_mt;
        v[c] = vcom + (dir[c] * g) * fac;
    }
    return 2;
}

// The reference's per-step HSS form (HSSCollisionHandler.cpp:331-376 with
// VelocitySampling.cpp:9-66 and CollisionKernels.cpp:139-169), with Philox
// in place of the per-ion mt19937_64: every step draws a Maxwell-Boltzmann
// neutral (three Box-Muller cosine normals), collides with probability
// 1 - exp(-n sigma |v - v_n| dt) and scatters isotropically in the centre of
// mass.  This is the plain form the optimised null-collision kernels are
// measured against; returns true on a collision.
template <class R>
__device__ __forceinline__ bool plain_hss(const EnsConst& C, R v[3], double mi_d, const uint32_t* rk, uint32_t id,
                                          uint32_t step, R ugz, R A, uint32_t sub0) {
    const U4 a = philox4x32_10_rk(id, step, sub0 + 0u, 0u, rk);
    const U4 b = philox4x32_10_rk(id, step, sub0 + 1u, 0u, rk);
    const R sn = static_cast<R>(C.sig_n);
    R vn[3];
    const uint32_t w1[3] = {a.x, a.z, b.x}, w2[3] = {a.y, a.w, b.y};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        R cs, ss;
        angle_cs(u32(w2[c], R(0)), cs, ss);
        const R u = (C.flow && c == 2) ? ugz : static_cast<R>(C.ug[c]);
        vn[c] = u + sn * (m_sqrt(R(-2.0) * m_log(u32(w1[c], R(0)))) * cs);
    }
    const R gx = v[0] - vn[0], gy = v[1] - vn[1], gz = v[2] - vn[2];
    const R g = m_sqrt(gx * gx + gy * gy + gz * gz);
    const R P = -m_expm1(-A * g);
    if (!(u32(b.z, R(0)) < P)) return false;
    const U4 c4 = philox4x32_10_rk(id, step, sub0 + 2u, 0u, rk);
    const R mi = static_cast<R>(mi_d), mn = static_cast<R>(C.m_gas);
    const R inv = R(1) / (mi + mn);
    const R fac = mn * inv;
    const R ct = R(2.0) * u32(b.w, R(0)) - R(1.0);
    const R st = m_sqrt(m_fmax(R(0), R(1.0) - ct * ct));
    R cp, sp;
    angle_cs(u32(c4.x, R(0)), cp, sp);
    const R dir[3] = {st * cp, st * sp, ct};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const R vcom = (v[c] * mi + vn[c] * mn) * inv;
        v[c] = vcom + (dir[c] * g) * fac;
    }
    return true;
}

// ---- finalize ------------------------------------------------------------------
// CylindricalGeometry::contains (CylindricalGeometry.h:35-40) on the global
// position; false for positions outside or non-finite.
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
// check.  Float accumulation error over <= kMaxStepsPerLaunch steps is < 0.1%.
// Resident blocks of 128 threads per SM the register budget is set for:
// 6 for the float forms (80 registers), 4 for FP64 (128).  The learned
// deflection measured fastest at 6 too (4 and 5 remove its spills but lose
// more to occupancy).  The float time-dependent instance holds the field's
// constants and its TIMS profile segment per lane: 5 (102 registers).
template <int PREC, int COLL, int FIELD>
struct KernelShape {
    static constexpr int kMinBlocks = PREC == kPrecFP64 ? 4 : (FIELD == kFieldLinearRF ? 5 : 6);
};

template <int PREC, int INTEG, int COLL, int FIELD, bool MAG, bool FUSED>
__global__ void __launch_bounds__(128, KernelShape<PREC, COLL, FIELD>::kMinBlocks) k_step(const __grid_constant__ StepParams p) {
    using R = typename PrecT<PREC>::R;
    using Pos = typename PosOf<PREC>::T;
    using Snap = typename Pos::Snap;
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
        if (COLL != kCollNone && COLL != kCollHSSPlain) {
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
    k.tf = nullptr;
    k.tftab = nullptr;
    k.tfrow = nullptr;
    k.tfstride = p.tf_stride;
    if constexpr (FIELD == kFieldLinearRF) {
        if (C.tf && p.tfield != nullptr && p.tf_tab != nullptr) {
            k.tf = p.tfield + (p.ens_base + static_cast<uint32_t>(e));
            k.tftab = p.tf_tab + static_cast<size_t>(p.ens_base + static_cast<uint32_t>(e)) * (p.n_steps + 1u) *
                                     p.tf_stride;
            k.tfrow = k.tftab;
            if constexpr (sizeof(R) == 4) {
                const TimeField& F = *k.tf;
                k.tfc_inst = F.inst;
                k.tfc_ei = static_cast<float>(F.tims_ei);
                k.tfc_ef = static_cast<float>(F.tims_ef);
                k.tfc_final = F.tims_final_profile != 0;
                k.ts_lo = INFINITY;               // no segment yet
                k.ts_hi = -INFINITY;
                k.ts_mode = 0;
            }
        }
    }
    if constexpr (COLL == kCollLangevin) {
        // speed-independent capture rate nu_i: event probability per step
        // Q = 1 - exp(-nu_i dt) (A = 0)
        const double mu = m * C.m_gas / (m + C.m_gas);
        k.A = R(0);
        k.Amean = static_cast<R>(-expm1(-C.lang_c * fabs(q) / sqrt(mu)));
    }
    k.sc = false;
    if (p.escx != nullptr && in_range) {
        // space charge: this launch advances one step with the field solved
        // for the step's start positions; the uniform-field acceleration
        // becomes (E0 q + E_sc q) / m
        const double es[3] = {p.escx[i], p.escy[i], p.escz[i]};
        k.sc = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            k.escq[a] = static_cast<R>(es[a] * q);
            if constexpr (sizeof(R) == 8) k.a_uni[a] = static_cast<R>((C.E0[a] * q + es[a] * q) / m);
            else k.a_uni[a] = static_cast<R>((C.E0[a] * q + es[a] * q) * (1.0 / m));
        }
    }
    if (INTEG == kRK4 && MAG) {
        k.tv[0] = static_cast<R>(C.B[0]); k.tv[1] = static_cast<R>(C.B[1]); k.tv[2] = static_cast<R>(C.B[2]);
    }
    ClockBound<R> cb;
    if constexpr (sizeof(R) == 4) {
        const R wx = v[0] - k.ug[0], wy = v[1] - k.ug[1], wz = v[2] - k.ug[2];
        cb.set(wx * wx + wy * wy + wz * wz);
    }

    const uint32_t id = static_cast<uint32_t>(p.first_id + i);
    // the ion's share of the candidate draws' first two Philox rounds
    const PhiloxIon pq = philox_ion_setup(id, p.rk);
    const uint32_t step0 = static_cast<uint32_t>(*p.step_dev);
    uint32_t n_cand = 0, n_coll = 0, n_ovf = 0, n_dead = 0, n_arr = 0;

    // Skip clock (Boris): S holds the exponential optical depth tau left at
    // the last restart, U the majorant Q* = A b* + A <|th|> of the current
    // horizon, b* >= |v - u| for every step of the horizon because Boris
    // changes |v| by at most |q/m| Emax dt per step.  A restart computes the
    // step at which tau is used up at rate -ln(1 - Q*) per step (the clock
    // event) or, if that lies beyond the horizon of H steps, a refresh at the
    // horizon's last step; restarts happen at global step indices fixed by
    // the lane's own history, so results do not depend on launch shape.
    constexpr bool kSkip = (INTEG == kBoris) && (COLL != kCollNone) && (COLL != kCollHSSPlain);
    // closed-form event-to-event drift (run_jumps below)
    // (FP64 only when the host asks for it: ICB_STEPPING_EVENTS_ALL)
    constexpr bool kJump = FUSED && (INTEG == kBoris) && (FIELD == kFieldUniform) && !MAG &&
                           (COLL != kCollHSSPlain);
    constexpr uint32_t kRefresh = 0x80000000u, kNeedRestart = 0xFFFFFFFFu;
    uint32_t g_next = kNeedRestart, g_start = 0u, nk = 0xFFFFFFFFu, H = 1u;
    R lam = R(0), dvmax = R(0), absu = R(0);
    if constexpr (kSkip) {
        if (in_range) { g_next = p.clk_next[i]; g_start = p.clk_start[i]; }
        dvmax = static_cast<R>(fabs(k.qm) * static_cast<R>(C.Emax) * static_cast<R>(C.dt));
        absu = m_sqrt(k.ug[0] * k.ug[0] + k.ug[1] * k.ug[1] + k.ug[2] * k.ug[2]);
        if (C.flow) absu = static_cast<R>(C.flow_umax);   // |u(x)| <= u_max
        // Horizon: a longer one thins more events (the majorant's excess
        // A H dv), a shorter one refreshes more often.  With a thinned event
        // costing about four refreshes, H = 1 / (2 sqrt(A dv)) balances them
        // (4 % faster than 1 / sqrt(A dv) at 20 Td, measured).
        R hz = R(0.5) / m_sqrt(k.A * dvmax);
        if (!(hz < R(4096))) hz = R(4096);
        if (hz < R(16)) hz = R(16);
        H = static_cast<uint32_t>(hz);
        if (U > R(0)) lam = m_neg_log1m(U);
        if (g_next != kNeedRestart) nk = (g_next & ~kRefresh) - step0;
    }
    auto clock_restart = [&](uint32_t gs) {
        const R v0 = m_sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const R bstar = (v0 + absu + static_cast<R>(H) * dvmax) * R(1.000001);
        R qs = k.A * bstar + k.Amean;
        if (qs > R(0.99999904632568359375)) { qs = R(0.99999904632568359375); ++n_ovf; }
        U = qs;
        lam = m_neg_log1m(qs);
        const R nf = ceil(S / lam);
        g_start = gs;
        if (nf <= static_cast<R>(H)) g_next = gs + (nf < R(1) ? 1u : static_cast<uint32_t>(nf)) - 1u;
        else g_next = (gs + H - 1u) | kRefresh;
        nk = (g_next & ~kRefresh) - step0;
    };
    const double t0 = p.t_dev[p.ens_base + e];
    const double dt = C.dt;
    const R dt_r = static_cast<R>(dt);
    const double zdet = C.zdet;
    double t = t0;            // accumulated clock (used when kAccumT)
    double tdeath = -1.0, tarr = -1.0;
    bool dead_now = false, arr_now = false;
    const uint32_t K = p.n_steps;
    uint32_t kk = 0;
    bool pending = false;     // lane stopped at this step until the deferred phase
    bool cand = false;        // ... because a collision candidate fired
    R b = R(0);
    Snap zold{};
    R acc = R(0), lim = R(0);

    auto t_step = [&]() -> double { return kAccumT ? t : fma(static_cast<double>(kk), dt, t0); };
    // z component of the parabolic gas flow at the ion
    // (EnvironmentConfig::gas_velocity_at, EnvironmentConfig.h:115-125)
    auto flow_z = [&]() -> R {
        if (!C.flow) return R(0);
        const double lx = x.gx() - C.ox, ly = x.gy() - C.oy;
        const double r2 = lx * lx + ly * ly;
        const double rr = (C.flow_r2 > 0.0) ? r2 / C.flow_r2 : 0.0;
        return static_cast<R>(C.flow_umax * fmax(0.0, 1.0 - rr));
    };
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
    if constexpr (kSkip) {
        // restart from the velocity before this step's push (the unfused
        // push call restarts for the collide call that follows)
        if (live && (do_coll || do_push) && g_next == kNeedRestart) clock_restart(step0);
    }

    // exact finalize of a step that started at time ts with z = zo
    // (SimulationEngineLifecycle.cpp:123-195)
    auto check_exact = [&](double zo, double ts) {
        const double znew = x.gz();
        if (!had_arrival && zo < zdet && znew >= zdet) {
            tarr = ts + dt * ((zdet - zo) / (znew - zo));
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
    };
    auto finalize_step = [&]() {
        // the unfused finalize call has no drift history: always exact
        if (do_fin && (!FUSED || !(acc <= lim))) {
            double zo = x.z_of(zold);
            if (!FUSED && !do_push) zo = p.zprev[i];
            x.fold();
            check_exact(zo, t_step());
        }
        ++kk;
        if (kAccumT) t = t + dt;
    };

    // The clock event of step gs (a lane with has_ev): candidate (or horizon
    // refresh), the warp's shared network evaluation for the learned
    // deflection, and the clock restart from the step after.  Every lane of
    // the warp calls this together.
    auto collide_at = [&](bool has_ev, uint32_t gs) {
        IpmPend<R> ip;
        bool need_net = false;
        // a parabolic flow is handled in the local gas frame: v_z - u_z(x)
        // during the candidate, u_z added back afterwards (x is unchanged)
        bool shifted = false;
        if (has_ev) {
            if constexpr (kSkip) {
                if (g_next & kRefresh) {
                    // horizon end without an event: consume its steps
                    S = S - static_cast<R>(gs + 1u - g_start) * lam;
                } else {
                    if (p.flows && C.flow) { v[2] = v[2] - flow_z(); shifted = true; }
                    int st;
                    if constexpr (COLL == kCollHSSMix)
                        st = candidate_mix<R, true>(C, p.mix[p.ens_base + e], v, S, U, k.Amean, b, m, p.rk, id, gs, pq);
                    else
                        st = candidate<R, true, COLL>(C, v, S, U, k.Amean, b, m, p.rk, id, gs, p, &ip, p.ens_base + e, pq);
                    if (st >= 1) ++n_cand;
                    if (st >= 2) ++n_coll;
                    need_net = st == 3;
                }
            } else {
                if (p.flows && C.flow) { v[2] = v[2] - flow_z(); shifted = true; }
                ++n_cand;
                int st;
                if constexpr (COLL == kCollHSSMix)
                    st = candidate_mix<R, false>(C, p.mix[p.ens_base + e], v, U, R(0), k.Amean, b, m, p.rk, id, gs, pq);
                else
                    st = candidate<R, false, COLL>(C, v, U, R(0), k.Amean, b, m, p.rk, id, gs, p, &ip, p.ens_base + e, pq);
                if (st >= 2) ++n_coll;
                need_net = st == 3;
            }
        }
        if constexpr (COLL == kCollIPMMLP) {
            // the warp's accepted collisions share one tensor-core
            // evaluation of the deflection network; energies outside
            // the trained range use the table
            if (__any_sync(0xffffffffu, need_net)) {
                R xr = R(0);
                bool in_dom = false;
                if (need_net) {
                    xr = (m_log(ip.E) - static_cast<R>(p.ipm_net_lnEmin)) * static_cast<R>(p.ipm_net_scale) - R(1);
                    in_dom = xr >= R(-1) && xr <= R(1);
                }
                const float x0 = static_cast<float>(xr);
                const float x1 = static_cast<float>(R(2) * ip.bn - R(1));
                const float y = mlp_warp_eval(p.mlp_w2, p.mlp_f, x0, x1, need_net && in_dom);
                if (need_net) {
                    R cx = in_dom ? m_fmin(m_fmax(static_cast<R>(y), R(-1)), R(1))
                                  : ipm_table_cos<R>(p, ip.E, ip.bn);
                    ipm_apply<R>(C, v, ip, cx, m);
                }
            }
        }
        if (shifted) v[2] = v[2] + flow_z();
        if (has_ev) {
            if constexpr (kSkip) {
                clock_restart(gs + 1u);
            } else {
                S = R(1);
                if constexpr (sizeof(R) == 4) {
                    const R wx = v[0] - k.ug[0], wy = v[1] - k.ug[1], wz = v[2] - k.ug[2];
                    cb.set(wx * wx + wy * wy + wz * wz);
                }
            }
        }
    };

    // one collision-free step (or a step that leaves the lane pending)
    auto push_and_tick = [&]() {
        zold = x.snap_z();
        if (!FUSED && do_push) p.zprev[i] = x.z_of(zold);
        if (do_push) {
            R l1;
            double tn = 0.0;   // only a time-dependent field reads the clock
            if constexpr (FIELD == kFieldLinearRF) {
                tn = t_step();
                if (k.tf != nullptr) k.tfrow = k.tftab + static_cast<size_t>(kk) * k.tfstride;
            }
            if (INTEG == kBoris) l1 = boris<R, FIELD, MAG>(k, x, v, tn);
            else l1 = rk4<R, FIELD, MAG>(k, x, v, tn);
            acc += l1 * dt_r;
        }
        if constexpr (kSkip) {
            if (do_coll) cand = (kk == nk);
        } else if constexpr (COLL == kCollHSSPlain) {
            if (do_coll) {
                // m collision sub-steps of dt/m at this position; sub-step j
                // draws from Philox substreams 4j, 4j + 1, 4j + 2
                const uint32_t ms = p.subcycles;
                const R A = ms > 1u ? static_cast<R>(C.A / static_cast<double>(ms)) : static_cast<R>(C.A);
                for (uint32_t j = 0; j < ms; ++j) {
                    ++n_cand;
                    if (plain_hss<R>(C, v, m, p.rk, id, step0 + kk, flow_z(), A, 4u * j)) ++n_coll;
                }
            }
        } else if constexpr (COLL != kCollNone) {
            if (do_coll) {
                if (p.flows && C.flow) k.ug[2] = flow_z();
                cand = clock_tick<R>(k, v, S, U, b, cb, n_ovf);
            }
        }
        // A collision candidate or an exhausted displacement budget stops the
        // lane at this step; both are handled in the warp's deferred phase,
        // which keeps the rare exact check out of the per-step path.
        pending = cand || (do_fin && (!FUSED || !(acc <= lim)));
        if (!pending) {
            ++kk;
            if (kAccumT) t = t + dt;
        }
    };

    auto run = [&](auto births) {
        constexpr bool kBirths = decltype(births)::value;
        while (true) {
            // cheap phase: up to steps_per_vote steps for every lane that can
            // step without a collision
#pragma unroll 1
            for (uint32_t j = 0; j < p.steps_per_vote; ++j) {
                if constexpr (kBirths) {
                    if (!((live || waiting) && !pending && kk < K)) continue;
                    if (waiting) {
                        if (t_step() >= birth) {      // prepare_ions_for_integration birth rule
                            waiting = false;
                            flags |= static_cast<uint8_t>(kFlagBorn | kFlagActive);
                            live = inside(C, x);
                            if (!live) {
                                kill(t_step());
                            } else {
                                new_limit();
                                if constexpr (kSkip) {
                                    if ((do_coll || do_push) && g_next == kNeedRestart) clock_restart(step0 + kk);
                                }
                            }
                        }
                    }
                    if (waiting || !live) {
                        ++kk;
                        if (kAccumT) t = t + dt;
                        continue;
                    }
                    push_and_tick();
                } else {
                    if (live && !pending && kk < K) push_and_tick();
                }
            }
            // warp-uniform fold of the float position offsets (anchor mode);
            // pending lanes keep theirs until their step is finalized
            if (!pending) x.fold();
            const bool can_step = (kBirths ? (live || waiting) : live) && !pending && kk < K;
            const unsigned pend_mask = __ballot_sync(0xffffffffu, pending);
            const unsigned run_mask = __ballot_sync(0xffffffffu, can_step);
            if (pend_mask != 0u &&
                (run_mask == 0u || static_cast<uint32_t>(__popc(pend_mask)) >= p.pend_threshold)) {
                collide_at(pending && cand, step0 + kk);
                if (pending) {
                    cand = false;
                    pending = false;
                    finalize_step();
                }
                continue;
            }
            if (run_mask == 0u) break;
        }
    };
    // Event-to-event drift (float forms, Boris in a uniform field without a
    // magnetic field, fused launches).  With a constant acceleration a the
    // Boris steps have a closed form: n steps from velocity v end at
    // v + a n dt after the displacement n dt v + a (n dt)^2 / 2 (the sum of
    // the per-step drifts (v + a dt/2 + (j-1) a dt) dt, j = 1..n).  Each lane
    // moves in one update to the first of: its clock event, the step at
    // which its displacement budget may run out, the end of the launch; the
    // warp then handles the events of all its lanes together, so candidate
    // work runs with most lanes active and no per-step work remains.
    // Events fall on the same steps and draw the same Philox counters as the
    // step-by-step loop; the drift differs from it by float rounding only.
    // Budget: the L1 path of j steps is at most
    //   B(j) = j dt s0 + ca j (j-1) / 2,  s0 = |v + a dt/2|_1,  ca = |a|_1 dt^2,
    // so a jump of n steps with B(n-1) <= lim - acc passes no step at which
    // the exact check could fire; it checks its last step exactly when
    // acc + B(n) exceeds lim.
    auto run_jumps = [&]() {
        const R a0 = k.a_uni[0], a1 = k.a_uni[1], a2 = k.a_uni[2];
        const R ca = (m_fabs(a0) + m_fabs(a1) + m_fabs(a2)) * dt_r * dt_r;
        const R ah0 = a0 * k.h, ah1 = a1 * k.h, ah2 = a2 * k.h;
        while (true) {
            const bool act = live && kk < K;
            if (__ballot_sync(0xffffffffu, act) == 0u) break;
            bool ev = false, exact = false;
            double zo = 0.0;
            if (act) {
                uint32_t n = K - kk;
                uint32_t ne = 0xFFFFFFFFu;
                if constexpr (kSkip) {
                    ne = nk + 1u - kk;    // steps up to and including the clock event
                    if (ne < n) n = ne;
                }
                const R s0 = m_fabs(v[0] + ah0) + m_fabs(v[1] + ah1) + m_fabs(v[2] + ah2);
                const R sd = s0 * dt_r;
                auto bound = [&](uint32_t j) {
                    const R rj = static_cast<R>(j);
                    return rj * (sd + R(0.5) * ca * (rj - R(1)));
                };
                if (budget) {
                    const R rem = lim - acc;
                    // the largest nb with B(nb) <= rem, solved only when the
                    // whole jump does not fit (near a wall or the detector)
                    if (!(bound(n) <= rem)) {
                        uint32_t nb = 0;
                        if (rem >= R(0)) {     // false for a non-finite state
                            const R B = sd - R(0.5) * ca;
                            const R den = B + m_sqrt(m_fmax(B * B + R(2) * ca * rem, R(0)));
                            R nbf = R(0);
                            if (den > R(0)) nbf = (R(2) * rem) / den;
                            else if (den == R(0)) nbf = static_cast<R>(n);
                            nb = nbf >= static_cast<R>(n) ? n : static_cast<uint32_t>(nbf);
                            if (nb > 0u && !(bound(nb) <= rem)) --nb;
                        }
                        if (nb + 1u < n) n = nb + 1u;
                    }
                } else {
                    n = 1u;               // short launches check every step
                }
                ev = n == ne;
                acc += bound(n);
                exact = !budget || !(acc <= lim);
                const R nd = static_cast<R>(n) * dt_r;
                const R hn = R(0.5) * nd;
                x.jump(nd * (v[0] + a0 * hn), nd * (v[1] + a1 * hn), nd * (v[2] + a2 * hn));
                v[0] = v[0] + a0 * nd;
                v[1] = v[1] + a1 * nd;
                v[2] = v[2] + a2 * nd;
                kk += n;
                // z before the last step: minus that step's drift (v - a dt/2) dt
                if (exact) zo = x.gz() - static_cast<double>(dt_r * (v[2] - ah2));
            }
            collide_at(ev, step0 + kk - 1u);
            if (exact) check_exact(zo, fma(static_cast<double>(kk - 1u), dt, t0));
        }
    };
    if (__any_sync(0xffffffffu, waiting)) {
        run(std::true_type{});
    } else {
        if constexpr (kJump) {
            if (p.jumps) run_jumps();
            else run(std::false_type{});
        } else {
            run(std::false_type{});
        }
    }

    if (in_range) {
        x.store(p, i);
        static_cast<R*>(p.vx)[i] = v[0];
        static_cast<R*>(p.vy)[i] = v[1];
        static_cast<R*>(p.vz)[i] = v[2];
        if (COLL != kCollNone && COLL != kCollHSSPlain) {
            static_cast<R*>(p.clkS)[i] = S;
            static_cast<R*>(p.clkU)[i] = U;
        }
        if constexpr (kSkip) {
            p.clk_next[i] = g_next;
            p.clk_start[i] = g_start;
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
