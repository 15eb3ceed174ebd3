// icb_params.h — plain structs shared by the host library and the kernels.
//
// Per-ensemble constants travel in the kernel's parameter block (a constant
// bank on the device, up to 32 KB), so every launch sees its ensembles'
// field, geometry and gas constants in constant memory without a
// per-handle __constant__ symbol (several handles may coexist in one process).
#pragma once
#include <cstdint>

namespace icb {

constexpr int kMaxLaunchEns = 64;   // ensembles per launch chunk (param space bound)
// Steps per launch are bounded so that the float accumulation of a lane's
// drift length between exact boundary checks stays within 0.1% (the check
// triggers at 99% of the distance to the nearest boundary).
constexpr uint32_t kMaxStepsPerLaunch = 16384;

enum FieldKind : int { kFieldUniform = 0, kFieldLinear = 1, kFieldLinearRF = 2 };
enum CollKind : int { kCollNone = 0, kCollHSS = 1, kCollLangevin = 2, kCollIPMTable = 3, kCollIPMMLP = 4, kCollHSSMix = 5, kCollHSSPlain = 6, kCollEHSS = 7, kCollIPMQuad = 8 };
enum PrecKind : int { kPrecFP64 = 0, kPrecMixed = 1, kPrecHiLo = 2 };
enum IntegKind : int { kBoris = 0, kRK4 = 1 };

// Counter slots (uint64 each) accumulated by the stepping kernels.
enum CounterSlot : int {
    kCntCandidates = 0, kCntCollisions = 1, kCntOverflow = 2, kCntDeaths = 3, kCntArrivals = 4,
    kCntStalls = 5,   // staged copies whose wait ran out (per-step kernel): an error
    kNumCounters = 8
};

// Flags byte per ion.
constexpr uint8_t kFlagActive = 1u;
constexpr uint8_t kFlagBorn = 2u;
constexpr uint8_t kFlagArrived = 4u;   // per-step kernel: arrival time recorded

struct EnsConst {
    // Electric field E = E0 + G .* (x - c); with rf: E_x, E_y from the
    // quadrupole term -2 x U(t)/r0^2, 2 y U(t)/r0^2, U = U0 + V cos(w t).
    double E0[3];
    double G[3];
    double c[3];
    double rf_U0, rf_V, rf_omega, r0sq;
    double B[3];
    // Cylinder (no rotation): local = x - origin; inside iff
    // -eps <= lz < L + eps and lx^2 + ly^2 <= (R + eps)^2.
    double ox, oy, oz, zmax_local, rmax2, rmax;
    double dt;
    // Gas: A = n sigma dt, mean thermal speed <|th|> = sigma_n 2 sqrt(2/pi).
    double A, mean_th, sig_n;
    double ug[3];
    double m_gas;
    double zdet;
    // Upper bound of |E| inside the domain: the skip clock bounds the ion
    // speed change per step by |q/m| Emax dt.
    double Emax;
    // Langevin capture: per-step event probability parameter
    // lambda_i = lang_c |q_i| / sqrt(mu_i)
    double lang_c;
    // parabolic axial gas flow (flow != 0): u_z = flow_umax max(0, 1 - r^2 /
    // flow_r2) at the ion; ug is then zero and refreshed at each collision
    double flow_umax, flow_r2;
    // AC drives (ac != 0): E_a += ac_amp[a] cos(ac_omega[a] t + ac_phase[a]),
    // a = x, y, ac_amp = -amplitude * ramp / r0; the RF quadrupole is
    // centred on (c[0], c[1])
    double ac_amp[2], ac_omega[2], ac_phase[2];
    int32_t magnetic;
    int32_t rf;
    int32_t ac;
    // float copies for the float collision path
    float fA, fmean_th, fsig_n, fm_gas;
    float fug[3];
    int32_t flow;
    int32_t tf;        // time-dependent field of TimeField (waveforms, TIMS)
    // the species of every ion of the ensemble (per-step kernel): mass and
    // charge when all its ions share them, sp_m = 0 otherwise; then also the
    // uniform field's acceleration by the FP64 form's formula (E0 q) / m and
    // by the float forms' (E0 q) (1 / m)
    double sp_m, sp_q;
    double sp_a64[3], sp_a32[3];
    // ... and the float forms' push constants: the acceleration, dt / 2, dt
    // and A <|th|> rounded to float once
    float sp_fa[3], sp_fh, sp_fdt, sp_fAmean;
};

// HSS gas mixture of one ensemble (read by the candidate step only):
// A_i = n_i sigma_i dt, thermal widths and masses per component.  The
// ensemble's EnsConst carries the totals (A = sum A_i, A mean_th =
// sum A_i mean_th_i) for the collision clock.
constexpr int kMaxGas = 8;
struct MixConst {
    int32_t n;
    int32_t pad_;
    double A[kMaxGas], mean_th[kMaxGas], sig_n[kMaxGas], m[kMaxGas];
    float fA[kMaxGas], fmean_th[kMaxGas], fsig_n[kMaxGas], fm[kMaxGas];
};

// Time-dependent field of one ensemble: voltages given as waveforms
// (ValueOrWaveform) and the TIMS axial ramp, evaluated in FP64 at every
// field evaluation.  Lives in device memory, one per ensemble (global index).
constexpr int kMaxWavePoints = 64;
// Per-step field table: per step and stage, kTfScalars doubles (the FP64
// scalars) then kTfFloatDoubles doubles holding 8 floats for the float
// forms (the same values rounded once when the table is built).
constexpr int kTfScalarsFP64 = 8;
constexpr int kTfFloatDoubles = 4;
constexpr int kTfRowScalars = kTfScalarsFP64 + kTfFloatDoubles;   // doubles per step and stage
enum WaveKind : int32_t {
    kWaveConstant = 0, kWaveLinear = 1, kWaveQuadratic = 2, kWaveExponential = 3,
    kWaveSinusoidal = 4, kWavePWM = 5, kWavePulsed = 6, kWaveArbitrary = 7
};
enum WaveChannel : int {
    kChAxial = 0, kChQuad = 1, kChRfV = 2, kChRfF = 3, kChTimsRamp = 4,
    kChAcA = 5, kChAcF = 6, kChAcR = 7,      // AC axis a: kChAc* + 3 a
    kNumChannels = 11
};
struct WaveConst {
    int32_t type, clamp, interp, n;
    double p[8];
    double tt[kMaxWavePoints], vv[kMaxWavePoints];
};
struct TimeField {
    int32_t inst;            // ICB_INSTRUMENT_* (IMS, QuadrupoleRF, LQIT, TIMS)
    int32_t tims_mode;       // 0 linear, 1 exponential ramp
    int32_t tims_nodes;      // 0 = uniform initial / final fields
    int32_t tims_final_profile;
    int32_t ramp_wave;       // ch[kChTimsRamp] replaces the built-in ramp
    int32_t ac_dipolar;      // LQIT AC: two-axis dipolar drive (else x alone, no ramp)
    double L, R, r0sq, ox, oy, oz;
    double ac_phase[2];
    double tims_t0, tims_t1, tims_tau, tims_ei, tims_ef;
    double tims_z[kMaxWavePoints], tims_pi[kMaxWavePoints], tims_pf[kMaxWavePoints];
    // float copies for the float forms: nodes, profiles, 1 / (z[i+1] - z[i])
    float tims_zf[kMaxWavePoints], tims_pif[kMaxWavePoints], tims_pff[kMaxWavePoints], tims_idz[kMaxWavePoints];
    WaveConst ch[kNumChannels];
};

// Ion-neutral interaction potential V = c12/r^12 - c6/r^6 - c4/r^4 (SI).
struct IpmPotential {
    double c12, c6, c4, sigma;
};

struct StepParams {
    // FP64 / mixed positions
    double* x; double* y; double* z;
    // hi/lo positions (mixed hi/lo mode)
    float* xh; float* xl; float* yh; float* yl; float* zh; float* zl;
    // velocities (double in FP64 mode, float otherwise)
    void* vx; void* vy; void* vz;
    // null-collision clock (same type as v): per-step clock (RK4): survival S
    // and threshold U; skip clock (Boris): optical depth tau at the last
    // restart and the majorant Q*.
    void* clkS; void* clkU;
    // skip clock: global step of the next clock event (bit 31 set = horizon
    // refresh, 0xFFFFFFFF = restart needed) and of the last restart
    uint32_t* clk_next;
    uint32_t* clk_start;
    const double* mass;
    const double* charge;
    uint8_t* flags;
    double* t_death;
    double* t_arr;
    const double* birth;               // nullable
    // space-charge field of this step per ion (nullable; launches with
    // space charge advance one step, the field is solved before each)
    const double* escx; const double* escy; const double* escz;
    double* zprev;                     // z before the push, kept between unfused calls
    // interaction-potential collisions: cos(chi) table [nE][nb] over
    // ln E = lnEmin + k / inv_dlnE and b = b_max j / (nb - 1)
    const float* ipm_tab;
    int32_t ipm_nE, ipm_nb;
    double ipm_lnEmin, ipm_inv_dlnE;
    // per-collision quadrature (kCollIPMQuad): the potential, b_max and the
    // Gauss-Legendre nodes (struct GLNodes of icb_ipm.cuh)
    IpmPotential ipm_pot;
    double ipm_bmax;
    const void* ipm_gl;
    // learned deflection input: x0 = (ln E - net_lnEmin) net_scale - 1,
    // inside the trained range when |x0| <= 1
    double ipm_net_lnEmin, ipm_net_scale;
    // learned deflection (MLP 2-64-64-1): packed BF16 weights and FP32
    // biases (nullable unless the MLP model is selected)
    const uint32_t* mlp_w2;            // W2 as mma B fragments
    const float* mlp_f;                // W1 (128), b1 (64), b2 (64), W3 (64), b3 (1)
    const MixConst* mix;               // per ensemble (global index), HSS mixtures
    const TimeField* tfield;           // per ensemble (global index), nullable
    // per-step time-only field scalars of this launch (k_tf_table), rows
    // k = 0..n_steps of tf_stride doubles per chunk ensemble; nullable
    const double* tf_tab;
    uint32_t tf_stride;
    // EHSS molecule geometry: atoms (x, y, z, radius) of ensemble e in
    // [ehss_off[e], ehss_off[e+1]), gas (contact) radius per ensemble
    const double4* ehss_atoms;
    const int32_t* ehss_off;
    const double* ehss_rgas;
    unsigned long long* counters;      // kNumCounters
    const unsigned long long* step_dev;// engine step index at launch start
    const double* t_dev;               // engine time per ensemble at launch start
    uint64_t first_id;
    uint64_t seed;
    uint32_t rk[20];                   // Philox round keys of the seed
    uint32_t n_steps;
    uint32_t pend_threshold;
    uint32_t ens_base;                 // global index of this chunk's ensemble 0
    uint32_t n_ens;
    uint32_t do_push, do_collide, do_finalize, steps_per_vote;
    uint32_t jumps;                    // event-to-event drift where the kernel supports it
    uint32_t subcycles;                // collision sub-steps per step (plain form), >= 1
    uint32_t flows;                    // some ensemble of the launch has a parabolic gas flow
    uint32_t skip_prepare;             // per-step kernel: every live ion was inside after the last step
    uint64_t ens_off[kMaxLaunchEns + 1];  // absolute ion offsets of the chunk's ensembles
    EnsConst ens[kMaxLaunchEns];
};

// The kernel parameter block holds at most 32,764 bytes.
static_assert(sizeof(StepParams) <= 32764, "StepParams exceeds the kernel parameter space");

}  // namespace icb
