/*
 * ORACLE — test infrastructure only.  Nothing in the icarion_b200 product
 * links, loads or calls this file; only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg use it, as the checker.
 *
 * CPU restatement (plain C, IEEE double, no FP contraction) of ICARION's
 * uniform-dt batch step, written from the reference's behaviour:
 *
 *   - engine order per step: domain check of unborn/outside ions, push,
 *     collision, finalize (domain exit -> inactive + death time, NaN ->
 *     inactive), t += dt          SimulationEngine.cpp:374-428,
 *                                 SimulationEngineLifecycle.cpp:72-195
 *   - Boris push with x += v_plus*dt     BorisStrategy.cpp:18-98
 *   - RK4 batch                          RK4Strategy.cpp:181-361
 *   - analytic E of IMS / FTICR / QuadrupoleRF / LQIT
 *                                        AnalyticalFieldModel.cpp:81-248
 *   - voltages given as waveforms (all eight types), evaluated per field
 *     call                               WaveformConfig.h:33-188,
 *                                        WaveformConfig.cpp:10-91
 *   - the TIMS axial field model         TIMSAxialFieldModel.h:30-148
 *   - magnetic force for RK4             MagneticFieldForce.cpp:61-118
 *   - cylinder containment (eps 1e-12)   CylindricalGeometry.h:35-40
 *   - reference HSS: full Maxwell-Boltzmann neutral every step, P=1-exp,
 *     isotropic COM scatter              HSSCollisionHandler.cpp:257-376,
 *                                        VelocitySampling.cpp:9-66,
 *                                        CollisionKernels.cpp:139-169,383-397
 *   - per-ion std::mt19937_64 seeded rng_seed + ion index, uniform01 via
 *     libstdc++ generate_canonical<double,53>
 *                                        CollisionTypes.h:31-49, RngUtils.cpp:51-53
 *   - the product's null-collision HSS (same per-step collision law in
 *     distribution) with Philox4x32-10 keyed on (seed, ion id, step), FP64,
 *     so GPU FP64 trajectories can be compared ion by ion.
 *
 * Pinned against golden vectors produced by the reference's own code
 * (oracle/ref_harness.cpp compiled from the reference sources), see
 * tests/golden/make_golden.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ORC_N_MOMENTS 20
#define ORC_KB 1.380649e-23          /* utils/constants.h:15 */
#define ORC_EPS0 8.854187817e-12     /* utils/constants.h:19 */
#define ORC_GEOM_EPS 1e-12           /* CylindricalGeometry.h:245 */
#define ORC_MIN_REL_VEL 1e-10        /* HSSCollisionHandler.cpp:20 */
#define ORC_MIN_VEL_MAG 1e-12        /* CollisionKernels.h:172 */
#define ORC_MIN_VOLTAGE 1e-12        /* threshold on |rf voltage| (AnalyticalFieldModel) */

/* Same layout as icb_ensemble_params (include/icarion_b200.h): the oracle
 * defines its own copy so it does not depend on the product headers. */
typedef struct orc_domain {
    int32_t instrument;
    int32_t magnetic_enabled;
    double origin_m[3];
    double length_m;
    double radius_m;
    double axial_V;
    double radial_V;
    double dc_quad_V;
    double rf_voltage_V;
    double rf_frequency_Hz;
    double B_T[3];
    double temperature_K;
    double gas_density_m3;
    double gas_mass_kg;
    double gas_velocity_m_s[3];
    double gas_polarizability_m3;
    double sigma_m2;
    double ipm_bmax_m;
    double dt_s;
    double detector_z_m;
    int32_t n_gas;
    int32_t flow_model;        /* 0 constant, 1 axial uniform, 2 axial parabolic */
    double gas_mix_density_m3[8];
    double gas_mix_mass_kg[8];
    double gas_mix_sigma_m2[8];
    double axial_flow_velocity_m_s;
    double axial_flow_max_velocity_m_s;
    double ac_amplitude_V[2];  /* LQIT AC drives: x (single-axis or dipolar x), y (dipolar y) */
    double ac_frequency_Hz[2];
    double ac_phase_rad[2];
    double ac_ramp[2];
    int32_t ac_dipolar;
    int32_t reserved2_;
} orc_domain;

/* Gas flow velocity at global position p (EnvironmentConfig::gas_velocity_at,
 * EnvironmentConfig.h:96-128, for an unrotated cylinder): the constant
 * vector, (0, 0, u) for the axial uniform profile, and u_z = u_max
 * max(0, 1 - r^2/R^2) for the parabolic one, r measured from the axis. */
static void gas_flow_at(const orc_domain* d, const double p[3], double ug[3]) {
    if (d->flow_model == 1) {
        ug[0] = 0.0; ug[1] = 0.0; ug[2] = d->axial_flow_velocity_m_s;
    } else if (d->flow_model == 2) {
        const double lx = p[0] - d->origin_m[0], ly = p[1] - d->origin_m[1];
        const double r2 = lx * lx + ly * ly;
        const double R2 = d->radius_m * d->radius_m;
        const double rr = (R2 > 0.0) ? r2 / R2 : 0.0;
        ug[0] = 0.0; ug[1] = 0.0; ug[2] = d->axial_flow_max_velocity_m_s * fmax(0.0, 1.0 - rr);
    } else {
        ug[0] = d->gas_velocity_m_s[0]; ug[1] = d->gas_velocity_m_s[1]; ug[2] = d->gas_velocity_m_s[2];
    }
}

/* ======================================================================
 * mt19937_64 (Matsumoto & Nishimura, ACM TOMACS 2000; 64-bit variant of
 * Nishimura 2000), restated from the published algorithm.
 * ==================================================================== */
typedef struct { uint64_t mt[312]; int mti; } orc_mt64;

static void mt64_seed(orc_mt64* s, uint64_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        s->mt[i] = 6364136223846793005ULL * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
    s->mti = 312;
}

static uint64_t mt64_next(orc_mt64* s) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    const uint64_t MATRIX_A = 0xB5026F5AA96619E9ULL;
    if (s->mti >= 312) {
        int i;
        for (i = 0; i < 312 - 156; ++i) {
            uint64_t x = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
            s->mt[i] = s->mt[i + 156] ^ (x >> 1) ^ ((x & 1ULL) ? MATRIX_A : 0ULL);
        }
        for (; i < 311; ++i) {
            uint64_t x = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
            s->mt[i] = s->mt[i + (156 - 312)] ^ (x >> 1) ^ ((x & 1ULL) ? MATRIX_A : 0ULL);
        }
        uint64_t x = (s->mt[311] & UM) | (s->mt[0] & LM);
        s->mt[311] = s->mt[155] ^ (x >> 1) ^ ((x & 1ULL) ? MATRIX_A : 0ULL);
        s->mti = 0;
    }
    uint64_t x = s->mt[s->mti++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}

/* uniform_real_distribution<double>(0,1) over a 64-bit engine: one draw,
 * value / 2^64, clamped below 1 (generate_canonical<double, 53>). */
static double mt64_uniform01(orc_mt64* s) {
    double r = (double)mt64_next(s) / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

void orc_mt64_uniforms(uint64_t seed, int64_t n, double* out) {
    orc_mt64 s;
    mt64_seed(&s, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = mt64_uniform01(&s);
}

/* ======================================================================
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As
 * Easy as 1, 2, 3", SC'11), restated from the paper.
 * ==================================================================== */
static void philox4x32_10(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t out[4]) {
    uint32_t c0 = c_in[0], c1 = c_in[1], c2 = c_in[2], c3 = c_in[3];
    uint32_t k0 = k_in[0], k1 = k_in[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox4x32_10(ctr, key, out);
}

/* Philox2x32-10 (Salmon, Moraes, Dror, Shaw, SC'11; the Random123 round:
 * (hi, lo) = 0xD256D193 * c0, c0' = hi ^ key ^ c1, c1' = lo, then
 * key += 0x9E3779B9) of the counter (c0, c1): both output words. */
void orc_philox2x32_10(uint32_t c0, uint32_t c1, uint32_t key, uint32_t out2[2]) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p = (uint64_t)0xD256D193u * c0;
        const uint32_t hi = (uint32_t)(p >> 32), lo = (uint32_t)p;
        c0 = hi ^ key ^ c1;
        c1 = lo;
        key += 0x9E3779B9u;
    }
    out2[0] = c0;
    out2[1] = c1;
}

/* The per-step kernel's collision test word (icb_step1.cuh,
 * step_test_word): Philox2x32-10 of (step, ion_id) under the key
 * seed_lo ^ seed_hi, first word. */
uint32_t orc_step_test_word(uint64_t seed, uint32_t step, uint32_t ion_id) {
    uint32_t out2[2];
    orc_philox2x32_10(step, ion_id, (uint32_t)seed ^ (uint32_t)(seed >> 32), out2);
    return out2[0];
}

void orc_philox_many(int64_t n, const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    for (int64_t i = 0; i < n; ++i) philox4x32_10(ctr + 4 * i, key, out + 4 * i);
}

/* 32-bit word -> double uniform on (0, 1]: (w + 1) * 2^-32 (exact). */
static double u32_to_unit(uint32_t w) { return ((double)w + 1.0) * 2.3283064365386963e-10; }

/* Philox stream layout of the product (icarion_b200/csrc/icb_rng.cuh):
 * key = (lo32(seed), hi32(seed)), counter = (ion id, step, substream, 0). */
static void draw4(uint64_t seed, uint32_t ion_id, uint32_t step, uint32_t sub, double u[4]) {
    uint32_t c[4] = {ion_id, step, sub, 0u};
    uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    philox4x32_10(c, k, o);
    for (int i = 0; i < 4; ++i) u[i] = u32_to_unit(o[i]);
}

void orc_unit_uniforms(uint64_t seed, uint32_t ion_id, uint32_t step, uint32_t sub, double* out4) {
    draw4(seed, ion_id, step, sub, out4);
}

/* ======================================================================
 * Time-dependent voltages and the TIMS axial field
 * ==================================================================== */
/* Same layouts as icb_waveform / icb_tims_field of the C ABI (own copies). */
#define ORC_MAX_WAVE 64
typedef struct {
    int32_t type, clamp, interp, n_points;
    double p[8];
    double times_s[ORC_MAX_WAVE];
    double values[ORC_MAX_WAVE];
} orc_wave;
typedef struct {
    int32_t ramp_mode, n_nodes, has_final_profile, reserved_;
    double ei, ef, t0, t1, tau;
    double z[ORC_MAX_WAVE], pi[ORC_MAX_WAVE], pf[ORC_MAX_WAVE];
} orc_tims;

/* channels: 0 DC.axial_V, 1 DC.quad_V, 2 RF.voltage_V, 3 RF.frequency_Hz,
 * 4 TIMS.ramp_fraction, 5-7 AC x amplitude / frequency / ramp (the
 * single-axis drive or dipolar_x), 8-10 the same for dipolar_y */
#define ORC_N_CH 11
static orc_wave g_wave[ORC_N_CH];
static int g_wave_set[ORC_N_CH];
static orc_tims g_tims;
static int g_tims_set;

void orc_set_time_field(const orc_tims* tims, const orc_wave* waves, const int32_t* set) {
    g_tims_set = tims != NULL;
    if (tims) g_tims = *tims;
    for (int c = 0; c < ORC_N_CH; ++c) {
        g_wave_set[c] = (waves && set && set[c]) ? 1 : 0;
        if (g_wave_set[c]) g_wave[c] = waves[c];
    }
}

/* Waveform value at t: WaveformConfig.h:33-188 (constant, linear,
 * quadratic, exponential, sinusoidal, PWM, pulsed) and
 * ArbitraryWaveform::evaluate, WaveformConfig.cpp:10-91. */
static double wave_eval(const orc_wave* w, double t) {
    const double* p = w->p;
    switch (w->type) {
    case 0: return p[0];
    case 1:
        if (t < p[2]) return p[0];
        if (t >= p[3]) return w->clamp ? p[1] : p[0];
        return p[0] + (p[1] - p[0]) * ((t - p[2]) / (p[3] - p[2]));
    case 2:
        if (t < p[3] || t > p[4]) return p[0];
        return p[0] + p[1] * t + p[2] * t * t;
    case 3: {
        double rel;
        if (t < p[3]) rel = 0.0;
        else if (t >= p[4]) rel = w->clamp ? (p[4] - p[3]) : 0.0;
        else rel = t - p[3];
        return p[0] + p[1] * exp(p[2] * rel);
    }
    case 4: return p[0] + p[1] * sin(2.0 * M_PI * p[2] * t + p[3]);
    case 5: {
        double tr, period, phase;
        if (p[2] <= 0.0 || t < p[5]) return p[0];
        if (t >= p[6]) {
            if (!w->clamp) return p[0];
            tr = p[6] - p[5];
        } else {
            tr = t - p[5];
        }
        period = 1.0 / p[2];
        phase = fmod(tr + p[4] / (2.0 * M_PI * p[2]), period);
        if (phase < 0.0) phase += period;
        return phase < p[3] * period ? p[1] : p[0];
    }
    case 6: return (t >= p[2] && t < p[2] + p[3]) ? p[1] : p[0];
    default: {
        const int n = w->n_points;
        const double* T = w->times_s;
        const double* V = w->values;
        int i1 = 0;
        if (!(t > T[0])) return V[0];
        if (t >= T[n - 1]) return V[n - 1];
        while (T[i1] < t) ++i1;             /* first T[i] >= t */
        {
            const int i0 = i1 - 1;
            const double t0 = T[i0], t1 = T[i1], v0 = V[i0], v1 = V[i1];
            double a, m0, m1, h00, h10, h01, h11, dt;
            if (w->interp == 1) return v0;
            a = (t - t0) / (t1 - t0);
            if (w->interp == 0) return v0 + a * (v1 - v0);
            m0 = i0 == 0 ? (v1 - v0) / (t1 - t0) : (v1 - V[i0 - 1]) / (t1 - T[i0 - 1]);
            m1 = i1 == n - 1 ? (v1 - v0) / (t1 - t0) : (V[i1 + 1] - v0) / (T[i1 + 1] - t0);
            h00 = 2 * a * a * a - 3 * a * a + 1;
            h10 = a * a * a - 2 * a * a + a;
            h01 = -2 * a * a * a + 3 * a * a;
            h11 = a * a * a - a * a;
            dt = t1 - t0;
            return h00 * v0 + h10 * dt * m0 + h01 * v1 + h11 * dt * m1;
        }
    }
    }
}

double orc_wave_value(const orc_wave* w, double t) { return wave_eval(w, t); }

/* Value of a field channel at t: its waveform, else the constant. */
static double chan(const orc_domain* d, int c, double t) {
    if (g_wave_set[c]) return wave_eval(&g_wave[c], t);
    switch (c) {
    case 0: return d->axial_V;
    case 1: return d->dc_quad_V;
    case 2: return d->rf_voltage_V;
    case 3: return d->rf_frequency_Hz;
    case 5: return d->ac_amplitude_V[0];
    case 6: return d->ac_frequency_Hz[0];
    case 7: return d->ac_ramp[0];
    case 8: return d->ac_amplitude_V[1];
    case 9: return d->ac_frequency_Hz[1];
    case 10: return d->ac_ramp[1];
    default: return 0.0;
    }
}

static double clamp01(double v) { return v < 0.0 ? 0.0 : (1.0 < v ? 1.0 : v); }

/* TIMS ramp fraction (TIMSAxialFieldModel.h:66-96). */
static double tims_ramp(double t) {
    const orc_tims* T = &g_tims;
    double t0, t1, duration, rel;
    if (g_wave_set[4]) return clamp01(wave_eval(&g_wave[4], t));
    t0 = g_tims_set ? T->t0 : 0.0;
    t1 = g_tims_set ? T->t1 : 0.0;
    if (t <= t0) return 0.0;
    if (t >= t1) return 1.0;
    duration = t1 - t0;
    if (duration <= 0.0) return 1.0;
    rel = t - t0;
    if (T->ramp_mode == 1) {
        const double tau = T->tau < 1e-30 ? 1e-30 : T->tau;
        const double denom = 1.0 - exp(-duration / tau);
        if (fabs(denom) < 1e-15) return clamp01(rel / duration);
        return clamp01((1.0 - exp(-rel / tau)) / denom);
    }
    return clamp01(rel / duration);
}

/* Axial profile at local z (TIMSAxialFieldModel.h:98-124). */
static double tims_sample(const double* zn, const double* v, int n, double z, double uni) {
    int i1 = 0;
    if (n == 0) return uni;
    if (!(z > zn[0])) return v[0];
    if (z >= zn[n - 1]) return v[n - 1];
    while (zn[i1] < z) ++i1;
    {
        const int i0 = i1 - 1;
        const double dz = zn[i1] - zn[i0];
        if (dz <= 0.0) return v[i0];
        return v[i0] + ((z - zn[i0]) / dz) * (v[i1] - v[i0]);
    }
}

/* ======================================================================
 * Fields and geometry
 * ==================================================================== */
static void field_E(const orc_domain* d, const double p[3], double t, double E[3]) {
    E[0] = E[1] = E[2] = 0.0;
    if (d->instrument == 0) {               /* IMS: AnalyticalFieldModel.cpp:136-161 */
        const double rfv = chan(d, 2, t);
        E[2] = chan(d, 0, t) / d->length_m;
        if (fabs(rfv) > ORC_MIN_VOLTAGE) {
            double r0_sq = d->radius_m * d->radius_m;
            double omega = 2.0 * M_PI * chan(d, 3, t);
            double U = chan(d, 1, t) + rfv * cos(omega * t);
            E[0] = -2.0 * p[0] * U / r0_sq;
            E[1] = 2.0 * p[1] * U / r0_sq;
        }
    } else if (d->instrument == 1) {        /* FTICR: AnalyticalFieldModel.cpp:174-186 */
        double L = d->length_m, r = d->radius_m;
        double dd = sqrt((L * L / 8.0) + (r * r / 4.0));
        double factor = d->radial_V / (dd * dd);
        double zc = p[2] - 0.5 * L;
        E[0] = factor * p[0];
        E[1] = factor * p[1];
        E[2] = -2.0 * factor * zc;
    } else if (d->instrument == 2) {        /* QuadrupoleRF: AnalyticalFieldModel.cpp:219-248 */
        const double rfv = chan(d, 2, t), axial = chan(d, 0, t);
        if (fabs(rfv) > ORC_MIN_VOLTAGE) {
            double r0_sq = d->radius_m * d->radius_m;
            double omega = 2.0 * M_PI * chan(d, 3, t);
            double U = chan(d, 1, t) + rfv * cos(omega * t);
            E[0] = -2.0 * p[0] * U / r0_sq;
            E[1] = 2.0 * p[1] * U / r0_sq;
        }
        if (fabs(axial) > ORC_MIN_VOLTAGE) E[2] = axial / d->length_m;
    } else if (d->instrument == 4) {        /* TIMS: TIMSAxialFieldModel.h:30-44, 126-148, unrotated */
        const double q[3] = {p[0] - d->origin_m[0], p[1] - d->origin_m[1], p[2] - d->origin_m[2]};
        const orc_tims* T = &g_tims;
        const int n = g_tims_set ? T->n_nodes : 0;
        const double f = tims_ramp(t);
        const double ei = tims_sample(T->z, T->pi, n, q[2], g_tims_set ? T->ei : 0.0);
        const double ef = tims_sample(T->z, T->pf, T->has_final_profile ? n : 0, q[2], g_tims_set ? T->ef : 0.0);
        const double r0_sq = d->radius_m * d->radius_m;
        E[2] = (1.0 - f) * ei + f * ef;
        if (r0_sq > 0.0) {
            const double omega = 2.0 * M_PI * chan(d, 3, t);
            const double u = chan(d, 1, t) + chan(d, 2, t) * cos(omega * t);
            E[0] = -2.0 * q[0] * u / r0_sq;
            E[1] = 2.0 * q[1] * u / r0_sq;
        }
    } else if (d->instrument == 3) {        /* LQIT: AnalyticalFieldModel.cpp:81-134, unrotated */
        const double q[3] = {p[0] - d->origin_m[0], p[1] - d->origin_m[1], p[2] - d->origin_m[2]};
        const double rfv = chan(d, 2, t), axial = chan(d, 0, t);
        if (fabs(rfv) > ORC_MIN_VOLTAGE) {
            double r0_sq = d->radius_m * d->radius_m;
            double omega = 2.0 * M_PI * chan(d, 3, t);
            double U = chan(d, 1, t) + rfv * cos(omega * t);
            E[0] = -2.0 * q[0] * U / r0_sq;
            E[1] = 2.0 * q[1] * U / r0_sq;
        }
        if (d->ac_dipolar) {
            /* two-axis dipolar drive: amplitude * ramp * cos(w t + phase), skipped
             * where |drive| <= threshold (eval_dipolar_axis_voltage) */
            for (int a = 0; a < 2; ++a) {
                const double amp = chan(d, 5 + 3 * a, t);
                if (fabs(amp) <= ORC_MIN_VOLTAGE) continue;
                const double omega = 2.0 * M_PI * chan(d, 6 + 3 * a, t);
                const double drive = amp * chan(d, 7 + 3 * a, t) * cos(omega * t + d->ac_phase_rad[a]);
                if (fabs(drive) > ORC_MIN_VOLTAGE) E[a] += -drive / d->radius_m;
            }
        } else {
            /* single-axis drive on x */
            const double v = chan(d, 5, t);
            if (fabs(v) > ORC_MIN_VOLTAGE) {
                const double omega_ac = 2.0 * M_PI * chan(d, 6, t);
                E[0] += -v / d->radius_m * cos(omega_ac * t + d->ac_phase_rad[0]);
            }
        }
        if (fabs(axial) > ORC_MIN_VOLTAGE) {
            const double L = d->length_m;
            const double alpha = axial / (L * L);
            E[2] = -2.0 * alpha * (q[2] - 0.5 * L);
        }
    }
}

void orc_field(const orc_domain* d, const double p[3], double t, double E[3]) { field_E(d, p, t, E); }

static int contains(const orc_domain* d, const double p[3]) {
    double lx = p[0] - d->origin_m[0], ly = p[1] - d->origin_m[1], lz = p[2] - d->origin_m[2];
    if (lz < -ORC_GEOM_EPS || lz >= d->length_m + ORC_GEOM_EPS) return 0;
    double r2 = lx * lx + ly * ly;
    return r2 <= (d->radius_m + ORC_GEOM_EPS) * (d->radius_m + ORC_GEOM_EPS);
}

/* ======================================================================
 * Pushers
 * ==================================================================== */
static void boris_step(const orc_domain* d, double x[3], double v[3], double m, double q,
                       double t, double dt) {
    double E[3];
    field_E(d, x, t, E);
    double F[3] = {E[0] * q, E[1] * q, E[2] * q};          /* ElectricFieldForce: E * q */
    double a[3] = {F[0] / m, F[1] / m, F[2] / m};          /* F / mass */
    double B[3] = {0.0, 0.0, 0.0};
    if (d->magnetic_enabled) { B[0] = d->B_T[0]; B[1] = d->B_T[1]; B[2] = d->B_T[2]; }
    double qm = q / m;
    double h = dt * 0.5;
    double vm[3] = {v[0] + a[0] * h, v[1] + a[1] * h, v[2] + a[2] * h};
    double ts = qm * dt * 0.5;
    double tv[3] = {B[0] * ts, B[1] * ts, B[2] * ts};
    double t2 = tv[0] * tv[0] + tv[1] * tv[1] + tv[2] * tv[2];
    double sf = 2.0 / (1.0 + t2);
    double sv[3] = {tv[0] * sf, tv[1] * sf, tv[2] * sf};
    double c1[3] = {vm[1] * tv[2] - vm[2] * tv[1], vm[2] * tv[0] - vm[0] * tv[2], vm[0] * tv[1] - vm[1] * tv[0]};
    double vp_[3] = {vm[0] + c1[0], vm[1] + c1[1], vm[2] + c1[2]};
    double c2[3] = {vp_[1] * sv[2] - vp_[2] * sv[1], vp_[2] * sv[0] - vp_[0] * sv[2], vp_[0] * sv[1] - vp_[1] * sv[0]};
    double vplus[3] = {vm[0] + c2[0], vm[1] + c2[1], vm[2] + c2[2]};
    x[0] += vplus[0] * dt; x[1] += vplus[1] * dt; x[2] += vplus[2] * dt;
    v[0] = vplus[0] + a[0] * h; v[1] = vplus[1] + a[1] * h; v[2] = vplus[2] + a[2] * h;
}

/* total force / m for RK4: E force, then magnetic force when enabled
 * (PhysicsSetup.cpp:206 adds MagneticFieldForce for non-Boris integrators),
 * times (1/mass) (RK4Strategy.cpp:242). */
static void rk4_acc(const orc_domain* d, const double x[3], const double v[3], double m, double q,
                    double t, double acc[3]) {
    double E[3];
    field_E(d, x, t, E);
    double F[3] = {E[0] * q, E[1] * q, E[2] * q};
    if (d->magnetic_enabled) {
        const double* B = d->B_T;
        double vxb[3] = {v[1] * B[2] - v[2] * B[1], v[2] * B[0] - v[0] * B[2], v[0] * B[1] - v[1] * B[0]};
        double Fb[3] = {vxb[0] * q, vxb[1] * q, vxb[2] * q};
        F[0] += Fb[0]; F[1] += Fb[1]; F[2] += Fb[2];
    }
    double im = 1.0 / m;
    acc[0] = F[0] * im; acc[1] = F[1] * im; acc[2] = F[2] * im;
}

static void rk4_step(const orc_domain* d, double x[3], double v[3], double m, double q,
                     double t, double dt) {
    double h = dt * 0.5;
    double bx[3] = {x[0], x[1], x[2]}, bv[3] = {v[0], v[1], v[2]};
    double k1v[3] = {bv[0], bv[1], bv[2]}, k1a[3];
    rk4_acc(d, bx, bv, m, q, t, k1a);
    double p2[3], v2[3], k2a[3];
    for (int i = 0; i < 3; ++i) { p2[i] = bx[i] + k1v[i] * h; v2[i] = bv[i] + k1a[i] * h; }
    rk4_acc(d, p2, v2, m, q, t + h, k2a);
    double p3[3], v3[3], k3a[3];
    for (int i = 0; i < 3; ++i) { p3[i] = bx[i] + v2[i] * h; v3[i] = bv[i] + k2a[i] * h; }
    rk4_acc(d, p3, v3, m, q, t + h, k3a);
    double p4[3], v4[3], k4a[3];
    for (int i = 0; i < 3; ++i) { p4[i] = bx[i] + v3[i] * dt; v4[i] = bv[i] + k3a[i] * dt; }
    rk4_acc(d, p4, v4, m, q, t + dt, k4a);
    double s = dt / 6.0;
    for (int i = 0; i < 3; ++i) {
        x[i] = bx[i] + (k1v[i] + v2[i] * 2.0 + v3[i] * 2.0 + v4[i]) * s;
        v[i] = bv[i] + (k1a[i] + k2a[i] * 2.0 + k3a[i] * 2.0 + k4a[i]) * s;
    }
}

/* ======================================================================
 * Collisions
 * ==================================================================== */
/* Reference HSS, single gas (HSSCollisionHandler.cpp:257-376). */
static int hss_reference(const orc_domain* d, const double p[3], double v[3], double mi, orc_mt64* rng) {
    double sig_n = sqrt(ORC_KB * d->temperature_K / d->gas_mass_kg);
    double vn[3];
    for (int c = 0; c < 3; ++c) {
        double u1 = mt64_uniform01(rng), u2 = mt64_uniform01(rng);
        vn[c] = sig_n * sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
    }
    double ug[3];
    gas_flow_at(d, p, ug);
    for (int c = 0; c < 3; ++c) vn[c] = vn[c] + ug[c];
    double vr[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
    double g = sqrt(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
    if (g < ORC_MIN_REL_VEL) return 0;
    double P = 1.0 - exp(-d->gas_density_m3 * d->sigma_m2 * g * d->dt_s);
    if (mt64_uniform01(rng) >= P) return 0;
    /* CollisionKernels::hss_collision */
    double mn = d->gas_mass_kg;
    double vr2[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
    double gm = sqrt(vr2[0] * vr2[0] + vr2[1] * vr2[1] + vr2[2] * vr2[2]);
    if (gm <= ORC_MIN_VEL_MAG) {
        double u1 = mt64_uniform01(rng), u2 = mt64_uniform01(rng);
        (void)u1; (void)u2;
        gm = ORC_MIN_VEL_MAG;
    }
    double u1 = mt64_uniform01(rng), u2 = mt64_uniform01(rng);
    double ct = 2.0 * u1 - 1.0;
    double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    double ph = 2.0 * M_PI * u2;
    double dir[3] = {st * cos(ph), st * sin(ph), ct};
    double mt = mi + mn, inv = 1.0 / mt;
    double fac = mn * inv;
    for (int c = 0; c < 3; ++c) {
        double vcom = (v[c] * mi + vn[c] * mn) * inv;
        v[c] = vcom + (dir[c] * gm) * fac;
    }
    return 1;
}

/* Null-collision HSS with Philox (the product's algorithm, FP64).
 * Each step has a candidate with probability Q = A b + A <|th|> (A = n sigma
 * dt, b = |v-u|).  The neutral's thermal part th is drawn from the mixture
 * f(th)(b + |th|)/(b + <|th|>) -- |th|^2/sigma^2 = -2 ln u1 - 2 ln u2 * s with
 * s = cos^2(2 pi u3) (chi^2_3, probability b/(b+<|th|>)) or s = 1 (chi^2_4),
 * isotropic direction -- and accepted with (1-exp(-n sigma g dt)) /
 * (A (b+|th|)) <= 1; the joint law of (collide, v_n) per step is then
 * f(v_n)(1-exp(-n sigma g dt)), the reference's.
 *
 * Two clocks decide the candidate steps:
 *  - per-step clock (RK4): survival S *= (1-Q), candidate when S < U;
 *  - skip clock (Boris): an exponential optical depth tau is spent at rate
 *    -ln(1-Q*) per step over horizons of H steps, with Q* = A b* + A<|th|>
 *    and b* = (|v| + |u| + H |q/m| Emax dt)(1 + 1e-6) >= |v-u| for every step
 *    of the horizon; at the step where tau runs out the event is thinned with
 *    Q(b)/Q*; at the end of a horizon without event tau is reduced and the
 *    horizon restarted.
 * Words: r0 = (U or tau, choice (thinning), accept, u1), r1 = (u2,
 * u3|cos th, phi th|cos scatter, phi scatter|-), 16-bit halves as
 * (k + 1/2) 2^-16.  Return: 0 thinned away, 1 candidate rejected, 2 collision. */
static double u16_to_unit(uint32_t k) { return ((double)k + 0.5) * 1.52587890625e-05; }

static void philox_words(uint64_t seed, uint32_t ion_id, uint32_t step, uint32_t sub, uint32_t o[4]) {
    uint32_t c[4] = {ion_id, step, sub, 0u};
    uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    philox4x32_10(c, k, o);
}

typedef struct { double A, Amean, mean_th, sig_n, mn, ug[3]; } gas_consts;

static gas_consts gas_of(const orc_domain* d) {
    gas_consts g;
    g.mn = d->gas_mass_kg;
    g.sig_n = sqrt(ORC_KB * d->temperature_K / g.mn);
    g.mean_th = g.sig_n * 1.5957691216057308;   /* E|th| = sigma*2*sqrt(2/pi) */
    g.A = d->gas_density_m3 * d->sigma_m2 * d->dt_s;
    g.Amean = g.A * g.mean_th;
    /* position-independent flows; the parabolic profile is set per collision */
    const double p0[3] = {0.0, 0.0, 0.0};
    gas_flow_at(d, p0, g.ug);
    if (d->flow_model == 2) g.ug[2] = 0.0;
    return g;
}

/* Interaction-potential table (collision 4): cos(chi) [nE][nb] over
 * ln E = lnEmin + k / inv_dlnE, b = b_max j / (nb - 1); bilinear in
 * (ln E, b) with E clamped, as the product samples it. */
static const float* g_ipm_tab = NULL;
static int g_ipm_nE = 0, g_ipm_nb = 0;
static double g_ipm_lnEmin = 0.0, g_ipm_inv_dlnE = 0.0;

void orc_set_ipm_table(const float* tab, int nE, int nb, double lnEmin, double inv_dlnE) {
    g_ipm_tab = tab;
    g_ipm_nE = nE;
    g_ipm_nb = nb;
    g_ipm_lnEmin = lnEmin;
    g_ipm_inv_dlnE = inv_dlnE;
}

static double ipm_table_cos(double E, double bn) {
    double t = (log(E) - g_ipm_lnEmin) * g_ipm_inv_dlnE;
    t = fmin(fmax(t, 0.0), (double)(g_ipm_nE - 1));
    int k = (int)t;
    if (k > g_ipm_nE - 2) k = g_ipm_nE - 2;
    const double ft = t - (double)k;
    const double u = bn * (double)(g_ipm_nb - 1);
    int j = (int)u;
    if (j > g_ipm_nb - 2) j = g_ipm_nb - 2;
    const double fu = u - (double)j;
    const float* r0 = g_ipm_tab + (size_t)k * g_ipm_nb + j;
    const float* r1 = r0 + g_ipm_nb;
    const double c00 = r0[0], c01 = r0[1], c10 = r1[0], c11 = r1[1];
    const double lo = c00 + fu * (c01 - c00);
    const double hi = c10 + fu * (c11 - c10);
    return lo + ft * (hi - lo);
}

/* Relative velocity g turned by chi about its own direction with azimuth
 * (cp, sp): Bird, Molecular Gas Dynamics and the Direct Simulation of Gas
 * Flows (1994), eq. 2.22. */
static void deflect(const double g3[3], double g, double cx, double sx, double cp, double sp, double out[3]) {
    const double gyz = sqrt(g3[1] * g3[1] + g3[2] * g3[2]);
    if (gyz > 1e-6 * g) {
        const double ig = 1.0 / gyz;
        out[0] = g3[0] * cx + sx * sp * gyz;
        out[1] = g3[1] * cx + sx * (g * g3[2] * cp - g3[0] * g3[1] * sp) * ig;
        out[2] = g3[2] * cx - sx * (g * g3[1] * cp + g3[0] * g3[2] * sp) * ig;
    } else {
        out[0] = g3[0] * cx;
        out[1] = g * sx * cp;
        out[2] = g * sx * sp;
    }
}

/* EHSS geometry of the oracle's ensemble (collision 7): atoms x, y, z, r. */
static const double* g_ehss_atoms = NULL;
static int g_ehss_n = 0;
static double g_ehss_rgas = 0.0;

void orc_set_ehss(const double* atoms4, int n, double gas_radius) {
    g_ehss_atoms = atoms4;
    g_ehss_n = n;
    g_ehss_rgas = gas_radius;
}

/* EHSS scattering with Philox words (the product's restatement of
 * CollisionKernels::ehss_collision, CollisionKernels.cpp:13-137, 220-381):
 * orientation quaternion from substream 2 (Shoemake), impact points from
 * substreams 8 + a/2 (words (0,1) for even a, (2,3) for odd a), earliest
 * atom contact, specular reflection, COM transform; v unchanged when 256
 * draws miss. */
static void ehss_scatter_orc(double v[3], const double vn[3], const double g3[3], double g, double mi, double mn,
                             uint64_t seed, uint32_t id, uint32_t step) {
    if (g_ehss_n <= 0 || !(g > 0.0)) return;
    const double ax[3] = {g3[0] / g, g3[1] / g, g3[2] / g};
    const double ea[3] = {fabs(ax[0]) < 0.9 ? 1.0 : 0.0, fabs(ax[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    double t1[3] = {ax[1] * ea[2] - ax[2] * ea[1], ax[2] * ea[0] - ax[0] * ea[2], ax[0] * ea[1] - ax[1] * ea[0]};
    double nt = 1.0 / sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    for (int c = 0; c < 3; ++c) t1[c] *= nt;
    double t2[3] = {ax[1] * t1[2] - ax[2] * t1[1], ax[2] * t1[0] - ax[0] * t1[2], ax[0] * t1[1] - ax[1] * t1[0]};
    nt = 1.0 / sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
    for (int c = 0; c < 3; ++c) t2[c] *= nt;
    uint32_t ro[4];
    philox_words(seed, id, step, 2u, ro);
    const double u1 = u32_to_unit(ro[0]);
    const double p2 = 2.0 * M_PI * u32_to_unit(ro[1]), p3 = 2.0 * M_PI * u32_to_unit(ro[2]);
    const double qa = sqrt(1.0 - u1), qb = sqrt(u1);
    const double qx = qa * sin(p2), qy = qa * cos(p2), qz = qb * sin(p3), qw = qb * cos(p3);
    const double Q[3][3] = {{1.0 - 2.0 * (qy * qy + qz * qz), 2.0 * (qx * qy - qz * qw), 2.0 * (qx * qz + qy * qw)},
                            {2.0 * (qx * qy + qz * qw), 1.0 - 2.0 * (qx * qx + qz * qz), 2.0 * (qy * qz - qx * qw)},
                            {2.0 * (qx * qz - qy * qw), 2.0 * (qy * qz + qx * qw), 1.0 - 2.0 * (qx * qx + qy * qy)}};
    const double B[3][3] = {{t1[0], t2[0], ax[0]}, {t1[1], t2[1], ax[1]}, {t1[2], t2[2], ax[2]}};
    double Rm[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rm[i][j] = B[i][0] * Q[0][j] + B[i][1] * Q[1][j] + B[i][2] * Q[2][j];
    double bmax = 0.0;
    for (int j = 0; j < g_ehss_n; ++j) {
        const double* c = g_ehss_atoms + 4 * j;
        double ra[3];
        for (int i = 0; i < 3; ++i) ra[i] = Rm[i][0] * c[0] + Rm[i][1] * c[1] + Rm[i][2] * c[2];
        const double sra = ax[0] * ra[0] + ax[1] * ra[1] + ax[2] * ra[2];
        const double px = ra[0] - ax[0] * sra, py = ra[1] - ax[1] * sra, pz = ra[2] - ax[2] * sra;
        const double cur = sqrt(px * px + py * py + pz * pz) + c[3];
        if (cur > bmax) bmax = cur;
    }
    bmax += g_ehss_rgas;
    uint32_t w[4] = {0, 0, 0, 0};
    for (int at = 0; at < 256; ++at) {
        if ((at & 1) == 0) philox_words(seed, id, step, 8u + (uint32_t)(at >> 1), w);
        const uint32_t wa = (at & 1) ? w[2] : w[0], wb = (at & 1) ? w[3] : w[1];
        const double bb = bmax * sqrt(u32_to_unit(wa));
        const double ph = 2.0 * M_PI * u32_to_unit(wb);
        const double cph = cos(ph), sph = sin(ph);
        const double off[3] = {t1[0] * (bb * cph) + t2[0] * (bb * sph), t1[1] * (bb * cph) + t2[1] * (bb * sph),
                               t1[2] * (bb * cph) + t2[2] * (bb * sph)};
        int hit = 0;
        double best = 0.0, nrm[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < g_ehss_n; ++j) {
            const double* c = g_ehss_atoms + 4 * j;
            double ra[3];
            for (int i = 0; i < 3; ++i) ra[i] = Rm[i][0] * c[0] + Rm[i][1] * c[1] + Rm[i][2] * c[2];
            const double rs = c[3] + g_ehss_rgas;
            const double rel[3] = {off[0] - ra[0], off[1] - ra[1], off[2] - ra[2]};
            const double ss = ax[0] * rel[0] + ax[1] * rel[1] + ax[2] * rel[2];
            const double dv[3] = {rel[0] - ax[0] * ss, rel[1] - ax[1] * ss, rel[2] - ax[2] * ss};
            const double d2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
            if (d2 <= rs * rs) {
                const double hgt = sqrt(fmax(0.0, rs * rs - d2));
                const double sh = ss - hgt;
                if (!hit || sh < best) {
                    const double phr[3] = {rel[0] - ax[0] * sh, rel[1] - ax[1] * sh, rel[2] - ax[2] * sh};
                    const double pr2 = phr[0] * phr[0] + phr[1] * phr[1] + phr[2] * phr[2];
                    if (pr2 <= 1e-24) {
                        nrm[0] = -ax[0]; nrm[1] = -ax[1]; nrm[2] = -ax[2];
                    } else {
                        const double ip = 1.0 / sqrt(pr2);
                        nrm[0] = phr[0] * ip; nrm[1] = phr[1] * ip; nrm[2] = phr[2] * ip;
                        if (ax[0] * nrm[0] + ax[1] * nrm[1] + ax[2] * nrm[2] > 0.0) {
                            nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
                        }
                    }
                    hit = 1;
                    best = sh;
                }
            }
        }
        if (hit) {
            const double vd = g3[0] * nrm[0] + g3[1] * nrm[1] + g3[2] * nrm[2];
            const double inv = 1.0 / (mi + mn);
            const double fac = mn * inv;
            for (int c = 0; c < 3; ++c) {
                const double gr = g3[c] - nrm[c] * (2.0 * vd);
                const double vcom = (v[c] * mi + vn[c] * mn) * inv;
                v[c] = vcom + gr * fac;
            }
            return;
        }
        if (at == 64) bmax *= 1.5;
    }
}

/* model: 0 hard sphere, 1 Langevin capture, 2 interaction-potential table, 3 EHSS */
static int nullcoll_candidate(const gas_consts* G, double v[3], double mi, uint64_t seed, uint32_t id,
                              uint32_t step, int skip, double* clk, double qstar, double b, int model) {
    const int langevin = model == 1;
    const double* ug = G->ug;
    uint32_t r0[4], r1[4];
    philox_words(seed, id, step, 0u, r0);
    double uc = u32_to_unit(r0[1]);
    if (skip) {
        *clk = -log(u32_to_unit(r0[0]));
        double w[3] = {v[0] - ug[0], v[1] - ug[1], v[2] - ug[2]};
        b = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        const double Q = G->A * b + G->Amean;
        if (!(uc * qstar < Q)) return 0;
        uc = uc * qstar / Q;
    } else {
        *clk = u32_to_unit(r0[0]);
    }
    philox_words(seed, id, step, 1u, r1);
    /* Langevin capture: a Maxwellian neutral (thermal branch), every event collides */
    const int thermal = langevin ? 1 : (uc * (b + G->mean_th) < b);
    const double c3 = cos(2.0 * M_PI * u16_to_unit(r1[1] >> 16));
    const double sfac = thermal ? c3 * c3 : 1.0;
    const double r2 = -2.0 * (log(u32_to_unit(r0[3])) + log(u32_to_unit(r1[0])) * sfac);
    const double rad = G->sig_n * sqrt(r2);
    const double ct = 2.0 * u16_to_unit(r1[1] & 0xffffu) - 1.0;
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    const double ph = 2.0 * M_PI * u16_to_unit(r1[2] >> 16);
    double vn[3] = {ug[0] + rad * (st * cos(ph)), ug[1] + rad * (st * sin(ph)), ug[2] + rad * ct};
    double gv[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
    double g = sqrt(gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2]);
    double q = G->A * (b + rad);
    double p = -expm1(-G->A * g);
    if (!langevin && !(u32_to_unit(r0[2]) * q < p)) return 1;
    if (model == 3) {
        ehss_scatter_orc(v, vn, gv, g, mi, G->mn, seed, id, step);
        return 2;
    }
    if (model == 2) {
        const double mn = G->mn;
        const double inv = 1.0 / (mi + mn);
        const double fac = mn * inv;
        const double mu = mi * fac;
        const double E = 0.5 * mu * (g * g);
        const double bn = sqrt(u16_to_unit(r1[2] & 0xffffu));
        const double cx = ipm_table_cos(E, bn);
        const double sx = sqrt(fmax(0.0, 1.0 - cx * cx));
        const double phi = 2.0 * M_PI * u16_to_unit(r1[3] >> 16);
        double gp[3];
        deflect(gv, g, cx, sx, cos(phi), sin(phi), gp);
        for (int c = 0; c < 3; ++c) {
            double vcom = (v[c] * mi + vn[c] * mn) * inv;
            v[c] = vcom + gp[c] * fac;
        }
        return 2;
    }
    const double ct2 = 2.0 * u16_to_unit(r1[2] & 0xffffu) - 1.0;
    const double st2 = sqrt(fmax(0.0, 1.0 - ct2 * ct2));
    const double ph2 = 2.0 * M_PI * u16_to_unit(r1[3] >> 16);
    double dir[3] = {st2 * cos(ph2), st2 * sin(ph2), ct2};
    const double mn = G->mn;
    double inv = 1.0 / (mi + mn);
    double fac = mn * inv;
    for (int c = 0; c < 3; ++c) {
        double vcom = (v[c] * mi + vn[c] * mn) * inv;
        v[c] = vcom + (dir[c] * g) * fac;
    }
    return 2;
}

/* HSS gas mixture candidate (collision 5), the product's exact restatement
 * of HSSCollisionHandler.cpp:105-249: component i chosen with probability
 * A_i (b + <|th_i|>) / sum, its neutral from the size-biased mixture, the
 * other components' neutrals Maxwellian from Philox substreams 4 + j, accept
 * with g_i (1 - exp(-K)) / (K (b + |th_i|)), K = sum_j A_j |v - v_j|. */
static int mix_candidate(const orc_domain* d, const gas_consts* G, double v[3], double mi, uint64_t seed,
                         uint32_t id, uint32_t step, double* clk, double qstar) {
    const int n = d->n_gas;
    double A[8], mean[8], sig[8];
    for (int i = 0; i < n; ++i) {
        A[i] = d->gas_mix_density_m3[i] * d->gas_mix_sigma_m2[i] * d->dt_s;
        sig[i] = sqrt(ORC_KB * d->temperature_K / d->gas_mix_mass_kg[i]);
        mean[i] = sig[i] * 1.5957691216057308;
    }
    const double* ug = G->ug;
    uint32_t r0[4], r1[4];
    philox_words(seed, id, step, 0u, r0);
    double uc = u32_to_unit(r0[1]);
    *clk = -log(u32_to_unit(r0[0]));
    double w[3] = {v[0] - ug[0], v[1] - ug[1], v[2] - ug[2]};
    const double b = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    const double Q = G->A * b + G->Amean;
    if (!(uc * qstar < Q)) return 0;
    uc = uc * qstar / Q;
    double qtot = 0.0;
    for (int i = 0; i < n; ++i) qtot += A[i] * (b + mean[i]);
    const double target = uc * qtot;
    int ci = n - 1;
    double cum = 0.0;
    for (int i = 0; i < n - 1; ++i) {
        const double qi = A[i] * (b + mean[i]);
        if (target < cum + qi) { ci = i; break; }
        cum += qi;
    }
    const double qsel = A[ci] * (b + mean[ci]);
    const double uci = fmin((target - cum) / qsel, 1.0);
    philox_words(seed, id, step, 1u, r1);
    const int thermal = uci * (b + mean[ci]) < b;
    const double c3 = cos(2.0 * M_PI * u16_to_unit(r1[1] >> 16));
    const double sfac = thermal ? c3 * c3 : 1.0;
    const double r2 = -2.0 * (log(u32_to_unit(r0[3])) + log(u32_to_unit(r1[0])) * sfac);
    const double rad = sig[ci] * sqrt(r2);
    const double ct = 2.0 * u16_to_unit(r1[1] & 0xffffu) - 1.0;
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    const double ph = 2.0 * M_PI * u16_to_unit(r1[2] >> 16);
    double vn[3] = {ug[0] + rad * (st * cos(ph)), ug[1] + rad * (st * sin(ph)), ug[2] + rad * ct};
    double gv[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
    const double g = sqrt(gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2]);
    double K = A[ci] * g;
    for (int j = 0; j < n; ++j) {
        if (j == ci) continue;
        uint32_t rj[4];
        philox_words(seed, id, step, 4u + (uint32_t)j, rj);
        const double ra = sqrt(-2.0 * log(u32_to_unit(rj[0])));
        const double rb = sqrt(-2.0 * log(u32_to_unit(rj[1])));
        const double pa = 2.0 * M_PI * u16_to_unit(rj[2] >> 16);
        const double pb = 2.0 * M_PI * u16_to_unit(rj[2] & 0xffffu);
        const double hx = v[0] - (ug[0] + sig[j] * ra * cos(pa));
        const double hy = v[1] - (ug[1] + sig[j] * ra * sin(pa));
        const double hz = v[2] - (ug[2] + sig[j] * rb * cos(pb));
        K += A[j] * sqrt(hx * hx + hy * hy + hz * hz);
    }
    const double pc = -expm1(-K);
    if (!(u32_to_unit(r0[2]) * K * (b + rad) < g * pc)) return 1;
    const double mn = d->gas_mix_mass_kg[ci];
    const double inv = 1.0 / (mi + mn);
    const double fac = mn * inv;
    const double ct2 = 2.0 * u16_to_unit(r1[2] & 0xffffu) - 1.0;
    const double st2 = sqrt(fmax(0.0, 1.0 - ct2 * ct2));
    const double ph2 = 2.0 * M_PI * u16_to_unit(r1[3] >> 16);
    double dir[3] = {st2 * cos(ph2), st2 * sin(ph2), ct2};
    for (int c = 0; c < 3; ++c) {
        double vcom = (v[c] * mi + vn[c] * mn) * inv;
        v[c] = vcom + (dir[c] * g) * fac;
    }
    return 2;
}

/* The reference's per-step HSS form with Philox words (collision 6): three
 * Box-Muller cosine normals for the neutral (VelocitySampling.cpp:9-66),
 * P = 1 - exp(-n sigma g dt), isotropic COM scatter (CollisionKernels.cpp:
 * 139-169).  Words: a = (u1, u2, u1', u2'), b = (u1'', u2'', accept, cos),
 * c = (phi, -, -, -). */
/* Collision sub-steps per step for the plain form (collision 6): m tests of
 * dt/m at the pushed position (SimulationEngineCollisionRuntime.cpp:79-190),
 * sub-step j from Philox substreams 4j, 4j + 1, 4j + 2. */
static int g_subcycles = 1;
void orc_set_subcycles(int m) { g_subcycles = m > 1 ? m : 1; }

static int plain_hss(const gas_consts* G, double v[3], double mi, uint64_t seed, uint32_t id, uint32_t step,
                     uint32_t sub0) {
    uint32_t a[4], b[4], c[4];
    philox_words(seed, id, step, sub0 + 0u, a);
    philox_words(seed, id, step, sub0 + 1u, b);
    const uint32_t w1[3] = {a[0], a[2], b[0]}, w2[3] = {a[1], a[3], b[1]};
    double vn[3];
    for (int k = 0; k < 3; ++k)
        vn[k] = G->ug[k] + G->sig_n * (sqrt(-2.0 * log(u32_to_unit(w1[k]))) * cos(2.0 * M_PI * u32_to_unit(w2[k])));
    double gv[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
    const double g = sqrt(gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2]);
    const double P = -expm1(-G->A * g);
    if (!(u32_to_unit(b[2]) < P)) return 0;
    philox_words(seed, id, step, sub0 + 2u, c);
    const double mn = G->mn;
    const double inv = 1.0 / (mi + mn);
    const double fac = mn * inv;
    const double ct = 2.0 * u32_to_unit(b[3]) - 1.0;
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    const double ph = 2.0 * M_PI * u32_to_unit(c[0]);
    double dir[3] = {st * cos(ph), st * sin(ph), ct};
    for (int k = 0; k < 3; ++k) {
        double vcom = (v[k] * mi + vn[k] * mn) * inv;
        v[k] = vcom + (dir[k] * g) * fac;
    }
    return 1;
}

/* Per-step clock (RK4). */
static int hss_nullcoll(const orc_domain* d, const double p[3], double v[3], double mi, uint64_t seed, uint32_t id,
                        uint32_t step, double* S, double* U, uint64_t* overflow) {
    const gas_consts G = gas_of(d);
    double ul[3];
    gas_flow_at(d, p, ul);
    double w[3] = {v[0] - ul[0], v[1] - ul[1], v[2] - ul[2]};
    double gu = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    double Q = G.A * gu + G.Amean;
    if (Q > 1.0) { Q = 1.0; ++*overflow; }
    *S = *S - *S * Q;
    if (!(*S < *U)) return -1;
    /* a parabolic flow: the candidate runs in the local gas frame */
    if (d->flow_model == 2) v[2] = v[2] - ul[2];
    const int r = nullcoll_candidate(&G, v, mi, seed, id, step, 0, U, 0.0, gu, 0);
    if (d->flow_model == 2) v[2] = v[2] + ul[2];
    *S = 1.0;
    return r;
}

/* Langevin capture (collision 3): a speed-independent rate per ion,
 * nu = n pi |q| sqrt(alpha' / (4 pi eps0 mu)) — sigma_L(v) v of
 * DampingForce.cpp:170-176 — so the per-step probability is the constant
 * 1 - exp(-nu dt); the skip clock runs with A = 0 and Amean = nu dt, each
 * event draws a Maxwellian neutral and scatters isotropically in the COM
 * frame. */
static double langevin_lambda(const orc_domain* d, double q, double m) {
    const double mu = m * d->gas_mass_kg / (m + d->gas_mass_kg);
    const double c = d->gas_density_m3 * d->dt_s * M_PI * sqrt(d->gas_polarizability_m3 / (4.0 * M_PI * ORC_EPS0));
    return c * fabs(q) / sqrt(mu);
}

/* Largest |value| of a waveform over all t (same expression as the
 * product's bound). */
static double wave_bound(const orc_wave* w) {
    const double* p = w->p;
    switch (w->type) {
    case 0: return fabs(p[0]);
    case 1: return fmax(fabs(p[0]), fabs(p[1]));
    case 2: {
        const double q3 = fabs(p[0] + p[1] * p[3] + p[2] * p[3] * p[3]);
        const double q4 = fabs(p[0] + p[1] * p[4] + p[2] * p[4] * p[4]);
        double b = fmax(fabs(p[0]), fmax(q3, q4));
        if (p[2] != 0.0) {
            const double tv = -p[1] / (2.0 * p[2]);
            if (tv > p[3] && tv < p[4]) b = fmax(b, fabs(p[0] + p[1] * tv + p[2] * tv * tv));
        }
        return b;
    }
    case 3: return fmax(fabs(p[0] + p[1]), fabs(p[0] + p[1] * exp(p[2] * (p[4] - p[3]))));
    case 4: return fabs(p[0]) + fabs(p[1]);
    case 5: case 6: return fmax(fabs(p[0]), fabs(p[1]));
    default: {
        double m = 0.0;
        for (int i = 0; i < w->n_points; ++i) m = fmax(m, fabs(w->values[i]));
        return w->interp == 2 ? 2.0 * m : m;
    }
    }
}

/* Field bound of a domain on the time-dependent path (instrument TIMS or a
 * waveform on any channel; same expression as the product's tf_bound). */
static double tf_field_bound(const orc_domain* d) {
    const double Rp = d->radius_m + ORC_GEOM_EPS;
    const double L = d->length_m;
    double wb[ORC_N_CH], ez, raxis = Rp, e;
    for (int c = 0; c < ORC_N_CH; ++c) wb[c] = g_wave_set[c] ? wave_bound(&g_wave[c]) : fabs(chan(d, c, 0.0));
    if (d->instrument == 4) {
        const orc_tims* T = &g_tims;
        const int n = g_tims_set ? T->n_nodes : 0;
        double m = g_tims_set ? fmax(fabs(T->ei), fabs(T->ef)) : fmax(0.0, 0.0);
        for (int i = 0; i < n; ++i) {
            m = fmax(m, fabs(T->pi[i]));
            if (T->has_final_profile) m = fmax(m, fabs(T->pf[i]));
        }
        ez = m;
    } else if (d->instrument == 3) {
        ez = 2.0 * (wb[0] / (L * L)) * (0.5 * L + ORC_GEOM_EPS);
    } else {
        ez = wb[0] / L;
        raxis = sqrt(d->origin_m[0] * d->origin_m[0] + d->origin_m[1] * d->origin_m[1]) + Rp;
    }
    e = ez + 2.0 * (wb[1] + wb[2]) * raxis / (d->radius_m * d->radius_m);
    if (d->instrument == 3) {
        double ac = 0.0;
        for (int a = 0; a < (d->ac_dipolar ? 2 : 1); ++a) {
            const double A = wb[5 + 3 * a] * (d->ac_dipolar ? wb[7 + 3 * a] : 1.0);
            if (A > ORC_MIN_VOLTAGE) ac += A / d->radius_m;
        }
        if (ac > 0.0) e = e + ac;
    }
    return e;
}

static int time_field_on(const orc_domain* d) {
    int c;
    if (d->instrument == 4) return 1;
    for (c = 0; c < ORC_N_CH; ++c)
        if (g_wave_set[c]) return 1;
    return 0;
}

/* Upper bound of |E| over the cylinder (same expression as the product's
 * field_bound): |E0| + |G .* max|x - c|| + 2 (|U0| + |V|) r_axis / r0^2. */
double orc_field_bound(const orc_domain* d) {
    double E0[3] = {0.0, 0.0, 0.0}, Gv[3] = {0.0, 0.0, 0.0}, c[3] = {0.0, 0.0, 0.0};
    int rf = fabs(d->rf_voltage_V) > ORC_MIN_VOLTAGE;
    if (time_field_on(d)) return tf_field_bound(d);
    if (d->instrument == 0) {
        E0[2] = d->axial_V / d->length_m;
    } else if (d->instrument == 2) {
        if (fabs(d->axial_V) > ORC_MIN_VOLTAGE) E0[2] = d->axial_V / d->length_m;
    } else if (d->instrument == 1) {
        double L = d->length_m, r = d->radius_m;
        double dd = sqrt((L * L / 8.0) + (r * r / 4.0));
        double factor = d->radial_V / (dd * dd);
        Gv[0] = factor; Gv[1] = factor; Gv[2] = -2.0 * factor;
        c[2] = 0.5 * L;
    } else if (d->instrument == 3) {
        c[0] = d->origin_m[0];
        c[1] = d->origin_m[1];
        if (fabs(d->axial_V) > ORC_MIN_VOLTAGE) {
            const double L = d->length_m;
            Gv[2] = -2.0 * (d->axial_V / (L * L));
            c[2] = d->origin_m[2] + 0.5 * L;
        }
    }
    const double Rp = d->radius_m + ORC_GEOM_EPS;
    const double ox = d->origin_m[0], oy = d->origin_m[1], oz = d->origin_m[2];
    const double zmax_local = d->length_m + ORC_GEOM_EPS;
    double e = sqrt(E0[0] * E0[0] + E0[1] * E0[1] + E0[2] * E0[2]);
    const double ex = fabs(ox - c[0]) + Rp;
    const double ey = fabs(oy - c[1]) + Rp;
    const double ez = fmax(fabs(oz - c[2]), fabs(oz + zmax_local - c[2]));
    const double gx = Gv[0] * ex, gy = Gv[1] * ey, gz = Gv[2] * ez;
    e = e + sqrt(gx * gx + gy * gy + gz * gz);
    if (rf) {
        const double dx = ox - c[0], dy = oy - c[1];
        const double raxis = sqrt(dx * dx + dy * dy) + Rp;
        e = e + 2.0 * (fabs(d->dc_quad_V) + fabs(d->rf_voltage_V)) * raxis / (d->radius_m * d->radius_m);
    }
    if (d->instrument == 3) {
        double ac = 0.0;
        for (int a = 0; a < (d->ac_dipolar ? 2 : 1); ++a) {
            const double A = d->ac_amplitude_V[a] * (d->ac_dipolar ? d->ac_ramp[a] : 1.0);
            if (fabs(A) > ORC_MIN_VOLTAGE) ac += fabs(-A / d->radius_m);
        }
        if (ac > 0.0) e = e + ac;
    }
    return e;
}

/* Skip clock of one ion (Boris). */
typedef struct {
    double tau, qstar, lam, dvmax, absu;
    uint32_t next, start, H;
} skip_clock;

#define ORC_REFRESH 0x80000000u
#define ORC_NEED_RESTART 0xFFFFFFFFu
#define ORC_QCAP 0.99999904632568359375

static void skip_setup(skip_clock* k, const orc_domain* d, const gas_consts* G, double q, double m) {
    const double qm = q / m;
    k->dvmax = fabs(qm) * orc_field_bound(d) * d->dt_s;
    k->absu = sqrt(G->ug[0] * G->ug[0] + G->ug[1] * G->ug[1] + G->ug[2] * G->ug[2]);
    if (d->flow_model == 2) k->absu = d->axial_flow_max_velocity_m_s;   /* |u(x)| <= u_max */
    double hz = 0.5 / sqrt(G->A * k->dvmax);   /* the product's horizon */
    if (!(hz < 4096.0)) hz = 4096.0;
    if (hz < 16.0) hz = 16.0;
    k->H = (uint32_t)hz;
    k->lam = (k->qstar > 0.0) ? -log1p(-k->qstar) : 0.0;
}

static void skip_restart(skip_clock* k, const gas_consts* G, const double v[3], uint32_t gs, uint64_t* overflow) {
    const double v0 = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double bstar = (v0 + k->absu + (double)k->H * k->dvmax) * 1.000001;
    double qs = G->A * bstar + G->Amean;
    if (qs > ORC_QCAP) { qs = ORC_QCAP; ++*overflow; }
    k->qstar = qs;
    k->lam = -log1p(-qs);
    const double nf = ceil(k->tau / k->lam);
    k->start = gs;
    if (nf <= (double)k->H) k->next = gs + (nf < 1.0 ? 1u : (uint32_t)nf) - 1u;
    else k->next = (gs + k->H - 1u) | ORC_REFRESH;
}

/* Initial clocks from u = uniform of Philox(id, 0, 3, 0).x: per-step clock
 * S = 1, U = u; skip clock (skip != 0) tau = -ln u, restart pending. */
void orc_clock_init(uint64_t seed, int64_t n, uint64_t first_id, double* S, double* U,
                    uint32_t* next, uint32_t* start, int skip) {
    for (int64_t i = 0; i < n; ++i) {
        double r[4];
        draw4(seed, (uint32_t)(first_id + (uint64_t)i), 0u, 3u, r);
        if (skip) {
            S[i] = -log(r[0]);
            U[i] = 0.0;
            next[i] = ORC_NEED_RESTART;
            start[i] = 0u;
        } else {
            S[i] = 1.0;
            U[i] = r[0];
        }
    }
}

/* ======================================================================
 * Engine loop (one domain)
 * ==================================================================== */
static void add_moments(double* m, const double x[3], const double v[3], const double r[3]) {
    m[0] += 1.0;
    m[1] += x[0]; m[2] += x[1]; m[3] += x[2];
    m[4] += x[0] * x[0]; m[5] += x[1] * x[1]; m[6] += x[2] * x[2];
    m[7] += v[0]; m[8] += v[1]; m[9] += v[2];
    m[10] += v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    m[13] += x[2] * v[2];
    for (int c = 0; c < 3; ++c) {
        double d = x[c] - r[c];
        m[14 + c] += d;
        m[17 + c] += d * d;
    }
}

/*
 * Run n_steps engine steps for n ions of one domain.
 *   integrator: 0 Boris, 1 RK4
 *   collision:  0 none, 1 reference HSS (mt19937_64 seeded seed + id),
 *               2 null-collision HSS (Philox; needs clk_S/clk_U, and for
 *               Boris the skip-clock event arrays clk_next/clk_start)
 *   step0/t0:   engine step index and time at entry
 *   snap_every: moments of the active ions are accumulated after every
 *               snap_every-th step into moments[(k/snap_every) * 14 + ...]
 *               (slot 11 counts arrivals so far, slot 12 deaths so far)
 *               (slots 14..19: displacement moments from the position after
 *               ref_step steps; before that, from the entry position)
 *   counters:   [candidates, collisions, rate_overflows] (nullable)
 * Ions are independent without space charge, so the loop runs ion-major
 * (parallel over ions with OpenMP when n_threads > 1).
 */
int orc_run(const orc_domain* d, int integrator, int collision, uint64_t seed,
            int64_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
            const double* mass, const double* charge, uint8_t* active,
            double* t_death, double* t_arr, double* clk_S, double* clk_U,
            uint32_t* clk_next, uint32_t* clk_start,
            uint64_t first_id, uint64_t step0, double t0, int64_t n_steps,
            int64_t snap_every, int64_t ref_step, double* moments, uint64_t* counters, int n_threads) {
    const int clocked = (collision == 2 || collision == 3 || collision == 4 || collision == 5 || collision == 7);
    if (clocked && (!clk_S || !clk_U)) return 1;
    if (clocked && integrator == 0 && (!clk_next || !clk_start)) return 1;
    if ((collision == 3 || collision == 4 || collision == 5 || collision == 7 || collision == 8) && integrator != 0)
        return 1;
    if (collision == 7 && !g_ehss_atoms) return 1;
    if (collision == 5 && (d->n_gas < 2 || d->n_gas > 8)) return 1;
    if (collision == 4 && !g_ipm_tab) return 1;
    const gas_consts G = gas_of(d);
    const int64_t n_snap = (snap_every > 0) ? n_steps / snap_every : 0;
    if (n_snap > 0 && moments) memset(moments, 0, sizeof(double) * (size_t)(n_snap * ORC_N_MOMENTS));
    uint64_t cand_tot = 0, coll_tot = 0, ovf_tot = 0;
    const double dt = d->dt_s;
    const double zdet = d->detector_z_m;
#ifdef _OPENMP
    if (n_threads < 1) n_threads = 1;
#else
    (void)n_threads;
#endif
#pragma omp parallel num_threads(n_threads) reduction(+ : cand_tot, coll_tot, ovf_tot)
    {
        double* mom = NULL;
        if (n_snap > 0 && moments) mom = (double*)calloc((size_t)(n_snap * ORC_N_MOMENTS), sizeof(double));
        orc_mt64* rng = (collision == 1) ? (orc_mt64*)malloc(sizeof(orc_mt64)) : NULL;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double p[3] = {x[i], y[i], z[i]}, v[3] = {vx[i], vy[i], vz[i]};
            double m = mass[i], q = charge[i];
            uint8_t act = active[i];
            double S = clk_S ? clk_S[i] : 1.0, U = clk_U ? clk_U[i] : 0.0;
            uint32_t id = (uint32_t)(first_id + (uint64_t)i);
            if (collision == 1) mt64_seed(rng, seed + first_id + (uint64_t)i);
            skip_clock sk;
            memset(&sk, 0, sizeof(sk));
            const int skip = (clocked && integrator == 0);
            gas_consts Gi = G;
            if (collision == 3) {
                Gi.A = 0.0;
                Gi.Amean = -expm1(-langevin_lambda(d, q, m));   /* per-step probability */
            } else if (collision == 4) {
                Gi.A = d->gas_density_m3 * (M_PI * d->ipm_bmax_m * d->ipm_bmax_m) * d->dt_s;
                Gi.Amean = Gi.A * Gi.mean_th;
            } else if (collision == 5) {
                double A = 0.0, Am = 0.0;
                for (int g = 0; g < d->n_gas; ++g) {
                    const double Ag = d->gas_mix_density_m3[g] * d->gas_mix_sigma_m2[g] * d->dt_s;
                    A += Ag;
                    Am += Ag * (sqrt(ORC_KB * d->temperature_K / d->gas_mix_mass_kg[g]) * 1.5957691216057308);
                }
                Gi.A = A;
                Gi.mean_th = A > 0.0 ? Am / A : 0.0;
                Gi.Amean = Gi.A * Gi.mean_th;
            }
            if (skip) {
                sk.tau = S;
                sk.qstar = U;
                sk.next = clk_next[i];
                sk.start = clk_start[i];
                skip_setup(&sk, d, &Gi, q, m);
                if (act && contains(d, p) && sk.next == ORC_NEED_RESTART) {
                    uint64_t ov = 0;
                    skip_restart(&sk, &Gi, v, (uint32_t)step0, &ov);
                    ovf_tot += ov;
                }
            }
            double t = t0;
            double ref[3] = {p[0], p[1], p[2]};
            for (int64_t k = 0; k < n_steps; ++k) {
                if (act) {
                    if (!contains(d, p)) {            /* prepare_ions_for_integration */
                        act = 0;
                        t_death[i] = t;
                    }
                }
                if (act) {
                    double zold = p[2];
                    if (integrator == 0) boris_step(d, p, v, m, q, t, dt);
                    else rk4_step(d, p, v, m, q, t, dt);
                    if (collision == 6) {
                        gas_consts Gp = Gi;
                        gas_flow_at(d, p, Gp.ug);            /* flow at the ion after the push */
                        if (g_subcycles > 1) Gp.A = Gi.A / (double)g_subcycles;
                        for (int j = 0; j < g_subcycles; ++j) {
                            ++cand_tot;
                            coll_tot += (uint64_t)plain_hss(&Gp, v, m, seed, id, (uint32_t)(step0 + (uint64_t)k),
                                                            4u * (uint32_t)j);
                        }
                    } else if (collision == 1) {
                        coll_tot += (uint64_t)hss_reference(d, p, v, m, rng);
                    } else if (skip) {
                        const uint32_t gs = (uint32_t)(step0 + (uint64_t)k);
                        if (sk.next != ORC_NEED_RESTART && gs == (sk.next & ~ORC_REFRESH)) {
                            uint64_t ov = 0;
                            if (sk.next & ORC_REFRESH) {
                                sk.tau = sk.tau - (double)(gs + 1u - sk.start) * sk.lam;
                            } else {
                                /* a parabolic flow: the candidate runs in the local gas frame */
                                double ul[3];
                                if (d->flow_model == 2) {
                                    gas_flow_at(d, p, ul);
                                    v[2] = v[2] - ul[2];
                                }
                                int r = (collision == 5)
                                    ? mix_candidate(d, &Gi, v, m, seed, id, gs, &sk.tau, sk.qstar)
                                    : nullcoll_candidate(&Gi, v, m, seed, id, gs, 1, &sk.tau, sk.qstar, 0.0,
                                                         collision == 3 ? 1 : (collision == 4 ? 2 : (collision == 7 ? 3 : 0)));
                                if (d->flow_model == 2) {
                                    gas_flow_at(d, p, ul);
                                    v[2] = v[2] + ul[2];
                                }
                                if (r >= 1) ++cand_tot;
                                if (r == 2) ++coll_tot;
                            }
                            skip_restart(&sk, &Gi, v, gs + 1u, &ov);
                            ovf_tot += ov;
                        }
                    } else if (collision == 8) {
                        /* the per-step kernel's stateless test: a candidate
                         * when the Philox2x32-10 word of (step, id) is below
                         * Q = A |v - u| + A <|th|>, then the per-step clock's
                         * candidate with b exact */
                        const uint32_t gs = (uint32_t)(step0 + (uint64_t)k);
                        const double w[3] = {v[0] - Gi.ug[0], v[1] - Gi.ug[1], v[2] - Gi.ug[2]};
                        const double b = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
                        double Q = Gi.A * b + Gi.Amean;
                        if (Q > 1.0) { Q = 1.0; ++ovf_tot; }
                        if (u32_to_unit(orc_step_test_word(seed, gs, id)) < Q) {
                            double clk = 0.0;
                            ++cand_tot;
                            if (nullcoll_candidate(&Gi, v, m, seed, id, gs, 0, &clk, 0.0, b, 0) == 2) ++coll_tot;
                        }
                    } else if (collision == 2) {
                        uint64_t ov = 0;
                        int r = hss_nullcoll(d, p, v, m, seed, id, (uint32_t)(step0 + (uint64_t)k), &S, &U, &ov);
                        ovf_tot += ov;
                        if (r >= 1) ++cand_tot;
                        if (r == 2) ++coll_tot;
                    }
                    if (t_arr[i] < 0.0 && zold < zdet && p[2] >= zdet)
                        t_arr[i] = t + dt * ((zdet - zold) / (p[2] - zold));
                    if (!contains(d, p)) {
                        act = 0;
                        t_death[i] = t;
                    } else if (!(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]) &&
                                 isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) {
                        act = 0;
                        t_death[i] = t;
                    }
                }
                t = t + dt;
                if (k + 1 == ref_step) { ref[0] = p[0]; ref[1] = p[1]; ref[2] = p[2]; }
                if (mom && ((k + 1) % snap_every) == 0) {
                    double* ms = mom + ((k + 1) / snap_every - 1) * ORC_N_MOMENTS;
                    if (act) add_moments(ms, p, v, ref);
                    if (t_arr[i] >= 0.0) ms[11] += 1.0;
                    if (!act && t_death[i] >= 0.0) ms[12] += 1.0;
                }
            }
            x[i] = p[0]; y[i] = p[1]; z[i] = p[2];
            vx[i] = v[0]; vy[i] = v[1]; vz[i] = v[2];
            active[i] = act;
            if (skip) {
                S = sk.tau;
                U = sk.qstar;
                clk_next[i] = sk.next;
                clk_start[i] = sk.start;
            }
            if (clk_S) clk_S[i] = S;
            if (clk_U) clk_U[i] = U;
        }
        if (mom) {
#pragma omp critical
            for (int64_t j = 0; j < n_snap * ORC_N_MOMENTS; ++j) moments[j] += mom[j];
            free(mom);
        }
        free(rng);
    }
    if (counters) { counters[0] = cand_tot; counters[1] = coll_tot; counters[2] = ovf_tot; }
    return 0;
}

/* Thermal width sqrt(kB T / m) (VelocitySampling.cpp:48-55). */
double orc_thermal_width(double T, double m) { return sqrt(ORC_KB * T / m); }

/* ---- interaction potential: classical deflection by trajectory ---------
 * Restates the reference's offline IPM physics for one isotropic site at
 * the origin: LJ 12-6 V = c12/r^12 - c6/r^6 (compute_vdw_force_and_potential,
 * interaction_potential_precompute.cpp:1386-1420) plus the isotropic
 * induced-dipole term -c4/r^4, c4 = 1/2 alpha' k q^2 (:1457-1508, :905/:929);
 * velocity-Verlet with the adaptive step of integrate_trajectory (:1672-1796:
 * dt <= eta sqrt(m r / |F|), halve when the per-step relative energy drift
 * exceeds tol_high, grow by 1.1 after relax_steps steps under tol_low, stop
 * outbound beyond r_cut once potential and force are negligible); the start
 * point (b, 0, -(b + 50 A)) and the deflection cos(theta) = v0 . v_out / |v0|^2
 * of deflection_weight_for_b (:1798-1835).  max_step_m > 0 is the tool's
 * optional cap |v| dt <= max_step_m (TrajectoryConfig::max_step_m, :504,
 * :1718-1724); without it the first step can jump over the interaction
 * region at high energy.  Returns cos(chi), or NAN when the trajectory did
 * not reach the asymptotic region within max_steps (200000, :503). */
static void ipm_force(double c12, double c6, double c4, const double r[3], double f[3], double* pot) {
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double rn = sqrt(r2);
    const double ir = 1.0 / rn;
    const double ir2 = ir * ir, ir4 = ir2 * ir2, ir6 = ir4 * ir2, ir12 = ir6 * ir6;
    const double ir7 = ir6 * ir, ir13 = ir12 * ir, ir5 = ir4 * ir;
    *pot = c12 * ir12 - c6 * ir6 - c4 * ir4;
    const double dVdr = -12.0 * c12 * ir13 + 6.0 * c6 * ir7 + 4.0 * c4 * ir5;
    const double scale = -dVdr * ir;
    for (int a = 0; a < 3; ++a) f[a] = r[a] * scale;
}

double orc_ipm_cos_chi_trajectory(double c12, double c6, double c4, double m_red, double E, double b,
                                  double max_step_m) {
    const double eta = 0.02, tol_high = 1e-6, tol_low = 1e-8;
    const int relax_steps = 100, max_steps = 200000;
    const double margin = 50e-10;
    const double r_cut = b + margin;
    const double v_rel = sqrt(2.0 * E / m_red);
    double r[3] = {b, 0.0, -(b + margin)}, v[3] = {0.0, 0.0, v_rel};
    double f[3], pot;
    ipm_force(c12, c6, c4, r, f, &pot);
    const double inv_m = 1.0 / m_red;
    double e_prev = 0.5 * m_red * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + pot;
    const double kin0 = 0.5 * m_red * v_rel * v_rel;
    const double e_floor = fmax(1e-30, kin0 * 1e-12);
    double e_scale = fmax(e_floor, fmax(fabs(e_prev), kin0));
    double dt = 0.0;
    int good = 0, approached = 0;
    for (int step = 0; step < max_steps; ++step) {
        const double rn = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        const double fn = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        if (fn > 0.0 && rn > 0.0) {
            const double dtf = eta * sqrt(m_red * rn / fn);
            dt = (dt <= 0.0) ? dtf : fmin(dt, dtf);
        }
        if (max_step_m > 0.0) {
            const double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            if (vn > 1e-12) {
                const double dts = max_step_m / vn;
                dt = (dt <= 0.0) ? dts : fmin(dt, dts);
            }
        }
        if (dt <= 0.0) dt = 1e-15;
        double vh[3], rt[3], fnw[3], pn;
        for (int a = 0; a < 3; ++a) {
            vh[a] = v[a] + f[a] * (0.5 * dt * inv_m);
            rt[a] = r[a] + vh[a] * dt;
        }
        ipm_force(c12, c6, c4, rt, fnw, &pn);
        double vt[3];
        for (int a = 0; a < 3; ++a) vt[a] = vh[a] + fnw[a] * (0.5 * dt * inv_m);
        const double e_new = 0.5 * m_red * (vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]) + pn;
        const double drift = fabs(e_new - e_prev) / e_scale;
        if (drift > tol_high) {
            dt *= 0.5;
            continue;
        }
        for (int a = 0; a < 3; ++a) { r[a] = rt[a]; v[a] = vt[a]; f[a] = fnw[a]; }
        pot = pn;
        e_prev = e_new;
        if (drift < tol_low) {
            if (++good >= relax_steps) { dt *= 1.1; good = 0; }
        } else {
            good = 0;
        }
        const double kin = 0.5 * m_red * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double rn2 = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        const double fn2 = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        const double asym = fmax(e_floor, kin);
        const double radial = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
        if (radial < 0.0) approached = 1;
        if (approached && radial > 0.0 && rn2 > r_cut && fabs(pot) / asym < 1e-6 && (fn2 * rn2) / asym < 1e-6) {
            const double c = (v[2] * v_rel) / fmax(1e-12, v_rel * v_rel);
            return fmax(-1.0, fmin(1.0, c));
        }
    }
    return NAN;
}

/* EHSS scattering alone (for the law check against the reference kernel):
 * ion i collides with its neutral using Philox(seed, id = i, step = 0). */
void orc_ehss_scatter_many(int64_t n, const double* v_ion, const double* v_n, double mi, double mn, uint64_t seed,
                           double* out) {
    for (int64_t i = 0; i < n; ++i) {
        double v[3] = {v_ion[3 * i], v_ion[3 * i + 1], v_ion[3 * i + 2]};
        const double vn[3] = {v_n[3 * i], v_n[3 * i + 1], v_n[3 * i + 2]};
        const double g3[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
        const double g = sqrt(g3[0] * g3[0] + g3[1] * g3[1] + g3[2] * g3[2]);
        ehss_scatter_orc(v, vn, g3, g, mi, mn, seed, (uint32_t)i, 0u);
        out[3 * i] = v[0];
        out[3 * i + 1] = v[1];
        out[3 * i + 2] = v[2];
    }
}

/* ---- interaction potential: classical deflection by quadrature ---------
 * CPU restatement of the library's device quadrature (the same steps):
 *   chi = pi - 2 (b / r0) int_0^1 2 s ds / sqrt(F(r0 / (1 - s^2))),
 *   F(r) = 1 - b^2/r^2 - V(r)/E,  V = c12/r^12 - c6/r^6 - c4/r^4,
 * r0 the outermost zero of F: stepped inwards by 2 % from 4 (b + sigma),
 * then bisected; 64-point Gauss-Legendre on [0, 1].  Used to build cos(chi)
 * tables and the reference-format momentum-transfer sample sets on the CPU.
 * Returns cos(chi); chi itself through chi_out when non-NULL. */
#define ORC_GL 64
static double g_gl_s[ORC_GL], g_gl_w[ORC_GL];
static int g_gl_ready = 0;

static void orc_gl_init(void) {
    if (g_gl_ready) return;
#pragma omp critical(orc_gl)
    {
        if (!g_gl_ready) {
            const int n = ORC_GL;
            for (int i = 0; i < n; ++i) {
                double x = cos(M_PI * (i + 0.75) / (n + 0.5));
                double dp = 0.0;
                for (int it = 0; it < 100; ++it) {
                    double p0 = 1.0, p1 = x;
                    for (int k = 2; k <= n; ++k) {
                        const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                        p0 = p1;
                        p1 = p2;
                    }
                    dp = n * (x * p1 - p0) / (x * x - 1.0);
                    const double dx = p1 / dp;
                    x -= dx;
                    if (fabs(dx) < 1e-16) break;
                }
                g_gl_s[i] = 0.5 * (x + 1.0);
                g_gl_w[i] = 0.5 * (2.0 / ((1.0 - x * x) * dp * dp));
            }
            g_gl_ready = 1;
        }
    }
}

static double ipm_F(double c12, double c6, double c4, double E, double b, double r) {
    const double ir2 = 1.0 / (r * r);
    const double ir4 = ir2 * ir2, ir6 = ir4 * ir2, ir12 = ir6 * ir6;
    const double V = c12 * ir12 - c6 * ir6 - c4 * ir4;
    return 1.0 - b * b * ir2 - V / E;
}

double orc_ipm_chi_quad(double c12, double c6, double c4, double sigma, double E, double b) {
    orc_gl_init();
    if (!(E > 0.0)) return 0.0;
    double r = 4.0 * (b + sigma);
    int it = 0;
    while (ipm_F(c12, c6, c4, E, b, r * 0.98) > 0.0 && it < 4000) {
        r *= 0.98;
        ++it;
    }
    double lo = r * 0.98, hi = r;
    for (int k = 0; k < 200 && hi - lo > 1e-15 * hi; ++k) {
        const double mid = 0.5 * (lo + hi);
        if (ipm_F(c12, c6, c4, E, b, mid) > 0.0) hi = mid; else lo = mid;
    }
    const double r0 = hi;
    double I = 0.0;
    for (int k = 0; k < ORC_GL; ++k) {
        const double s = g_gl_s[k];
        const double u = 1.0 - s * s;
        const double F = fmax(ipm_F(c12, c6, c4, E, b, r0 / u), 1e-300);
        I += g_gl_w[k] * 2.0 * s / sqrt(F);
    }
    return M_PI - 2.0 * (b / r0) * I;
}

/* cos(chi) of n (E, b) pairs (OpenMP over pairs). */
void orc_ipm_cos_chi_many(int64_t n, double c12, double c6, double c4, double sigma, const double* E,
                          const double* b, double* out) {
    orc_gl_init();
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) out[i] = cos(orc_ipm_chi_quad(c12, c6, c4, sigma, E[i], b[i]));
}

/* The reference's per-cell momentum-transfer samples
 * (interaction_potential_precompute.cpp:2692-2880, store_full_cdf) for one
 * isotropic site and a fixed b_max, n_cells relative speeds g[c]: per cell
 * n_trials impact points uniform over the disk of radius b_max (b = b_max
 * sqrt(w), phi = 2 pi u), the deflection chi(E = mu g^2 / 2, b) by the
 * quadrature above, and the centre-of-mass momentum change dp = mu (v_out -
 * v0) in the frame with v0 along +z: v_out = g (sin chi cos phi,
 * sin chi sin phi, cos chi) (chi > 0 deflects away from the scattering
 * centre, i.e. along the impact offset).  The tool draws w and u as
 * independent uniforms (mt19937_64 per cell); stratified = 1 takes w from
 * the t-th of n_trials equal-area annuli instead (w = (t + u') / n_trials),
 * the same uniform-area law without the Monte Carlo noise of the cell's
 * momentum-transfer mean.  dp: 3 n_trials doubles per cell, cells in order
 * (OpenMP over cells). */
void orc_ipm_sample_cells(int64_t n_cells, const double* g, double c12, double c6, double c4, double sigma,
                          double mu, double b_max, int64_t n_trials, uint64_t seed, int stratified, double* dp) {
    orc_gl_init();
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < n_cells; ++c) {
        orc_mt64 rng;
        mt64_seed(&rng, seed * 1000003ull + (uint64_t)c);
        const double E = 0.5 * mu * g[c] * g[c];
        double* out = dp + 3 * n_trials * c;
        for (int64_t t = 0; t < n_trials; ++t) {
            const double u1 = mt64_uniform01(&rng);
            const double u2 = mt64_uniform01(&rng);
            const double w = stratified ? ((double)t + u1) / (double)n_trials : u1;
            const double b = b_max * sqrt(w);
            const double phi = 2.0 * M_PI * u2;
            const double chi = orc_ipm_chi_quad(c12, c6, c4, sigma, E, b);
            const double sn = sin(chi), cs = cos(chi);
            out[3 * t] = mu * (g[c] * sn * cos(phi));
            out[3 * t + 1] = mu * (g[c] * sn * sin(phi));
            out[3 * t + 2] = mu * (g[c] * cs - g[c]);
        }
    }
}
