/*
 * icarion_b200.h — C ABI of the B200-native ICARION uniform-dt batch step.
 *
 * One handle owns one device-resident ion population (SoA in HBM) and the
 * per-ensemble constants of the physics (domain, fields, gas, time step).
 * Every entry point returns an int status (ICB_OK == 0); nothing throws
 * across the ABI.  On failure icb_last_error() gives a readable message.
 * Handles are not thread-safe: one host thread drives one handle, as one
 * SimulationEngine drives one IIntegrationStrategy / ICollisionHandler.
 *
 * Interfaces replaced (reference paths are relative to the ICARION tree):
 *   IIntegrationStrategy::step_batch
 *       src/core/integrator/strategies/IIntegrationStrategy.h:119-132
 *       -> icb_upload_ions + icb_advance(push only / fused) + icb_download_ions
 *   ICollisionHandler::handle_batch
 *       src/core/physics/collisions/ICollisionHandler.h:121-134
 *       -> icb_collide (unfused) or folded into icb_advance (fused)
 *   SimulationEngine::process_timestep's per-step order
 *       src/core/integrator/SimulationEngine.cpp:374-428
 *       -> icb_advance(n_steps): push -> collide -> finalize -> t += dt, n times
 */
#ifndef ICARION_B200_H
#define ICARION_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ICB_ABI_VERSION 10

/* ---- status codes ------------------------------------------------------ */
enum {
    ICB_OK = 0,
    ICB_ERR_INVALID_ARGUMENT = 1,
    ICB_ERR_CUDA = 2,
    ICB_ERR_OUT_OF_MEMORY = 3,
    ICB_ERR_UNSUPPORTED = 4,
    ICB_ERR_STATE = 5,
    ICB_ERR_NO_DEVICE = 6,
    ICB_ERR_TIMEOUT = 7
};

/* ---- enums ------------------------------------------------------------- */
enum { ICB_PREC_FP64 = 0, ICB_PREC_MIXED = 1, ICB_PREC_MIXED_HILO = 2 };
enum { ICB_INTEGRATOR_BORIS = 0, ICB_INTEGRATOR_RK4 = 1 };
enum {
    ICB_COLLISION_NONE = 0,
    ICB_COLLISION_HSS = 1,
    ICB_COLLISION_IPM_TABLE = 2,
    ICB_COLLISION_IPM_MLP = 3,
    ICB_COLLISION_LANGEVIN = 4,
    /* the reference's per-step HSS form (a Maxwell-Boltzmann neutral and an
     * exp test every step), FP64 + Boris only: the plain baseline the
     * null-collision kernels are measured against */
    ICB_COLLISION_HSS_PLAIN = 5,
    /* exact hard-sphere scattering on a molecule of atoms (EHSS,
     * CollisionKernels.cpp:13-137, 220-381), rate n sigma_m2 |v - v_n|;
     * geometry from icb_ehss_set_geometry */
    ICB_COLLISION_EHSS = 6,
    /* interaction-potential collisions with the deflection computed by the
     * FP64 quadrature at every collision (no table, no network): the plain
     * method the learned deflection is measured against; Boris in a uniform
     * field without B */
    ICB_COLLISION_IPM_QUAD = 7
};
enum {
    ICB_INSTRUMENT_IMS = 0,          /* AnalyticalFieldModel.cpp:136-161 */
    ICB_INSTRUMENT_FTICR = 1,        /* AnalyticalFieldModel.cpp:174-186 */
    ICB_INSTRUMENT_QUADRUPOLE_RF = 2,/* AnalyticalFieldModel.cpp:219-248 */
    /* linear quadrupole ion trap, AnalyticalFieldModel.cpp:81-134: RF
     * quadrupole about the cylinder axis, AC drives (ac_* below) and the
     * axial DC well E_z = -2 axial_V / L^2 (z_local - L/2) */
    ICB_INSTRUMENT_LQIT = 3,
    /* trapped IMS, TIMSAxialFieldModel.h:18-193 (the model of every domain
     * with instrument TIMS or fields.TIMS.enabled, PhysicsSetup.cpp:190-196):
     * E_z(z, t) = (1 - f(t)) E_initial(z) + f(t) E_final(z) in local z from
     * icb_set_tims_field (zero without it), plus the radial quadrupole
     * E_x = -2 x U / r0^2, E_y = 2 y U / r0^2, U = dc_quad + V cos(w t),
     * x, y from the cylinder axis; no dc.axial_V term */
    ICB_INSTRUMENT_TIMS = 4
};

/* Number of doubles per ensemble returned by icb_moments:
 *  0 n_active  1 sum x   2 sum y   3 sum z   4 sum x^2  5 sum y^2  6 sum z^2
 *  7 sum vx    8 sum vy  9 sum vz  10 sum |v|^2  11 n_arrived  12 n_dead
 *  13 sum z*vz
 *  14..16 sum of displacement (x - x_ref) per axis, 17..19 sum of its square,
 *  where x_ref is the position at upload or at the last icb_mark_reference.
 *  Drift and diffusion are fitted from the displacement moments, which do
 *  not carry the initial cloud's spread.                                   */
#define ICB_N_MOMENTS 20

/* One ensemble = one domain + environment + ion species + dt.  The fields
 * follow DomainConfig / EnvironmentConfig of the reference; derived values
 * (gas density, axial_V from E/N) are computed by the caller exactly as the
 * reference loader does (DomainConfigLoader.cpp:410-440,
 * EnvironmentConfig.h:152). */
typedef struct icb_ensemble_params {
    int32_t instrument;        /* ICB_INSTRUMENT_* */
    int32_t magnetic_enabled;  /* fields.magnetic.enabled */
    double origin_m[3];        /* geometry.origin_m (no rotation) */
    double length_m;           /* geometry.length_m */
    double radius_m;           /* geometry.radius_m */
    double axial_V;            /* fields.DC.axial_V */
    double radial_V;           /* fields.DC.radial_V (FTICR trap) */
    double dc_quad_V;          /* fields.DC.quad_V */
    double rf_voltage_V;       /* fields.RF.voltage_V */
    double rf_frequency_Hz;    /* fields.RF.frequency_Hz */
    double B_T[3];             /* fields.magnetic.field_strength_T */
    double temperature_K;      /* env.temperature_K */
    double gas_density_m3;     /* env.particle_density_m_3 = P/(kB T) */
    double gas_mass_kg;        /* env.gas_mass_kg */
    double gas_velocity_m_s[3];/* env.gas_velocity_m_s (constant flow) */
    double gas_polarizability_m3; /* Langevin capture (alpha') */
    double sigma_m2;           /* HSS cross-section of this ensemble's ions */
    double ipm_bmax_m;         /* IPM: event cross-section pi*b_max^2 */
    double dt_s;               /* uniform time step of this ensemble */
    double detector_z_m;       /* arrival plane (first crossing, global z) */
    /* Gas mixture (env.gas_mixture, EnvironmentConfig.h:31-44, 155-205):
     * n_gas = 2..ICB_MAX_GAS components replace gas_density_m3 /
     * gas_mass_kg / sigma_m2 above for HSS collisions
     * (HSSCollisionHandler.cpp:105-249); 0 or 1 = the single gas above. */
    int32_t n_gas;
    int32_t flow_model;        /* ICB_FLOW_* (env.flow_model, EnvironmentConfig.h:81-128) */
    double gas_mix_density_m3[8];
    double gas_mix_mass_kg[8];
    double gas_mix_sigma_m2[8];
    /* Gas flow profile: CONSTANT uses gas_velocity_m_s; AXIAL_UNIFORM
     * (0, 0, axial_flow_velocity_m_s); AXIAL_PARABOLIC u_z =
     * axial_flow_max_velocity_m_s * max(0, 1 - r^2/R^2), r the distance
     * from the cylinder axis, R = radius_m, at the ion's position when it
     * collides (SimulationEngineCollisionRuntime.cpp:124-131). */
    double axial_flow_velocity_m_s;
    double axial_flow_max_velocity_m_s;
    /* AC drives of the LQIT (fields.ac): E_x += -ac_amplitude_V[0] *
     * ac_ramp[0] / radius_m * cos(2 pi ac_frequency_Hz[0] t + ac_phase_rad[0]),
     * E_y the same with [1].  ac_dipolar = 0: the single-axis drive
     * (ac.voltage_V, frequency_Hz, phase_rad) on axis 0 alone, ac_ramp and
     * axis 1 unused; 1: the
     * two-axis dipolar drive (ac.dipolar_x / dipolar_y: amplitude_V, ramp,
     * frequency_Hz, phase_rad; a disabled axis has amplitude 0).  Drives
     * with |amplitude * ramp| <= 1e-12 V are off. */
    double ac_amplitude_V[2];
    double ac_frequency_Hz[2];
    double ac_phase_rad[2];
    double ac_ramp[2];
    int32_t ac_dipolar;
    int32_t reserved2_;
} icb_ensemble_params;
enum { ICB_FLOW_CONSTANT = 0, ICB_FLOW_AXIAL_UNIFORM = 1, ICB_FLOW_AXIAL_PARABOLIC = 2 };
#define ICB_MAX_GAS 8

typedef struct icb_config {
    int32_t precision;         /* ICB_PREC_* */
    int32_t integrator;        /* ICB_INTEGRATOR_* */
    int32_t collision_model;   /* ICB_COLLISION_* */
    int32_t n_ensembles;       /* 1 .. ICB_MAX_ENSEMBLES */
    const icb_ensemble_params* ensembles; /* copied at icb_create */
    uint64_t rng_seed;         /* simulation.rng_seed */
    int32_t device;            /* CUDA device ordinal */
    int32_t block_size;        /* threads per block, 0 = tuned default */
    int32_t steps_per_launch;  /* steps fused per kernel launch, 0 = default */
    int32_t pending_threshold; /* deferred-collision batch size per warp, 0 = default */
    int32_t use_graphs;        /* capture launch sequences in CUDA graphs */
    int32_t steps_per_vote;    /* collision-free steps between warp votes, 0 = default */
    int32_t stepping;          /* ICB_STEPPING_* (0 = event-to-event drift where supported) */
    /* Collision sub-steps per step (physics.collision_subcycles_per_step, or
     * collision_max_events_per_step in multi-event mode;
     * SimulationEngineCollisionRuntime.cpp:79-190): m > 1 repeats the
     * collision test m times per step with dt/m at the pushed position.
     * Needs ICB_COLLISION_HSS_PLAIN; 0 or 1 = one test per step. */
    int32_t collision_subcycles;
    int32_t collision_test;    /* ICB_TEST_* (0 = the collision clock) */
    int32_t reserved[3];
} icb_config;

/* How the null-collision candidates of hard-sphere collisions are found.
 * CLOCK: a collision clock carried per ion between launches (the skip clock
 * for Boris, a survival product for RK4); the fused kernels.  PER_STEP: a
 * stateless test every step (Philox(id, step) against Q = A (|v - u| +
 * <|th|>) of the current velocity), run by the per-step kernel, which moves
 * only positions, velocities and the flag byte through HBM each step:
 * the form for an engine that hands the state back every step.  Same
 * per-step collision law; the two draw different random numbers.  PER_STEP
 * runs Boris in a uniform electric field without B, hard-sphere or no
 * collisions, a single gas with constant or axial-uniform flow, no births,
 * no space charge and no time-dependent field; its steps_per_launch
 * defaults to 1. */
enum { ICB_TEST_CLOCK = 0, ICB_TEST_PER_STEP = 1 };

/* Stepping of the fused float forms (MIXED, MIXED_HILO) with Boris in a
 * uniform field and no magnetic field: EVENTS moves each ion in one
 * closed-form update from one event (collision-clock event, exact domain
 * check, end of launch) to the next; PER_STEP applies the steps one by one.
 * Both draw the same random numbers at the same steps; their drifts differ
 * by float rounding.  FP64 steps one by one under EVENTS (so that its pushes
 * keep the reference's operation order); EVENTS_ALL moves FP64 from event
 * to event too (the same algorithm as the float forms, for measuring what
 * precision alone costs; its drifts differ from the step loop's by double
 * rounding).  RK4, non-uniform fields and the per-step plug points always
 * step one by one. */
enum { ICB_STEPPING_EVENTS = 0, ICB_STEPPING_PER_STEP = 1, ICB_STEPPING_EVENTS_ALL = 2 };

#define ICB_MAX_ENSEMBLES 256

typedef struct icb_run_stats {
    uint64_t steps;            /* time steps advanced by the call */
    uint64_t candidates;       /* null-collision candidates tested */
    uint64_t collisions;       /* accepted collisions */
    uint64_t rate_overflows;   /* steps whose candidate probability was clamped to 1 */
    uint64_t deaths;           /* ions deactivated (domain exit or non-finite state) */
    uint64_t arrivals;         /* first detector-plane crossings */
    double device_ms;          /* device time of the call (CUDA events) */
    double step_kernel_ms;     /* device time inside the fused step kernel launches */
    uint64_t kernel_launches;  /* kernels this call launched */
    double spacecharge_ms;     /* device time of the space-charge solves timed (the first 64 of the call) */
    uint64_t spacecharge_solves_timed;
} icb_run_stats;

/* ---- ion cloud generation (IonLoader semantics) ------------------------ */
enum {
    ICB_POS_POINT = 0, ICB_POS_GAUSSIAN = 1, ICB_POS_UNIFORM_SPHERE = 2,
    ICB_POS_UNIFORM_CYLINDER = 3, ICB_POS_UNIFORM_BOX = 4
};
enum { ICB_VEL_FIXED = 0, ICB_VEL_THERMAL = 1 };

typedef struct icb_species_spec {
    uint64_t count;
    double mass_kg;
    double charge_C;
    int32_t position_type;     /* ICB_POS_* (PositionDistribution) */
    int32_t velocity_type;     /* ICB_VEL_* (VelocityDistribution) */
    double center_m[3];
    double std_m[3];           /* gaussian */
    double radius_m;           /* uniform_sphere / uniform_cylinder */
    double length_m;           /* uniform_cylinder */
    double box_min_m[3];
    double box_max_m[3];
    double velocity_m_s[3];    /* fixed */
    double temperature_K;      /* thermal */
} icb_species_spec;

/* Generate the initial ion cloud of all species in order from one
 * std::mt19937(rng_seed), as IonLoader::generate_species does
 * (IonLoader.cpp:183-238, sample_position/sample_velocity :246-313).
 * Output arrays hold sum(count) entries. */
int icb_generate_ions(uint32_t rng_seed, int32_t n_species, const icb_species_spec* specs,
                      double* x, double* y, double* z, double* vx, double* vy, double* vz,
                      double* mass_kg, double* charge_C);

/* ---- library ----------------------------------------------------------- */
int icb_abi_version(void);
/* Message of the last failing call on this host thread ("" if none). */
const char* icb_last_error(void);
int icb_device_count(int* count);

/* ---- handle lifetime --------------------------------------------------- */
int icb_create(const icb_config* cfg, struct icb_handle** out);
int icb_destroy(struct icb_handle* h);
/* Launch on this stream (a cudaStream_t); NULL = the handle's own stream. */
int icb_set_stream(struct icb_handle* h, void* cuda_stream);
int icb_synchronize(struct icb_handle* h);

/* ---- ion state (IonEnsemble SoA, IonEnsemble.h:267-330) ----------------
 * Ions must be grouped by ensemble: ions [ens_offsets[e], ens_offsets[e+1])
 * belong to ensemble e.  ens_offsets may be NULL when n_ensembles == 1.
 * birth_time_s may be NULL (all born at t = 0).  Ion ids (the Philox key
 * component) are first_ion_id + index. */
int icb_upload_ions(struct icb_handle* h, uint64_t n,
                    const double* x, const double* y, const double* z,
                    const double* vx, const double* vy, const double* vz,
                    const double* mass_kg, const double* charge_C,
                    const uint8_t* active, const double* birth_time_s,
                    const uint64_t* ens_offsets, uint64_t first_ion_id);
/* Copy positions/velocities back; every pointer may be NULL.  death and
 * arrival times are -1 where the event has not happened. */
int icb_download_ions(struct icb_handle* h,
                      double* x, double* y, double* z,
                      double* vx, double* vy, double* vz,
                      uint8_t* active, double* death_time_s,
                      double* arrival_time_s);
/* Overwrite positions/velocities only (engine-side edits between steps);
 * collision clocks, ids and flags stay. */
int icb_update_state(struct icb_handle* h,
                     const double* x, const double* y, const double* z,
                     const double* vx, const double* vy, const double* vz,
                     const uint8_t* active);
uint64_t icb_ion_count(struct icb_handle* h);

/* ---- stepping ---------------------------------------------------------- */
/* Fused uniform-dt batch step, n_steps times: push (Boris/RK4) -> collision
 * -> domain/NaN finalize -> t += dt (SimulationEngine.cpp:374-428). */
int icb_advance(struct icb_handle* h, uint64_t n_steps, icb_run_stats* stats);
/* The engine fast path with host state in one call: icb_update_state (the
 * given positions, velocities and active flags) + icb_advance(n_steps) +
 * icb_download_ions (same arrays), with the ions split into n_chunks whose
 * host<->device copies overlap the steps of the other chunks (copy and
 * copy-back streams, one compute stream per chunk, events, queued chunk by
 * chunk; host arrays should be pinned for the overlap; 24 chunks measured
 * best for 1M ions on a B200).  The overlapped
 * form needs n_steps <= steps_per_launch, no space charge and the
 * double-position forms (on a use_graphs handle its chunks launch directly);
 * otherwise (and for n_chunks = 1) the three calls run in order.  Results
 * equal the three separate calls bit for bit. */
int icb_advance_host(struct icb_handle* h, uint64_t n_steps, int n_chunks,
                     double* x, double* y, double* z, double* vx, double* vy, double* vz,
                     uint8_t* active, icb_run_stats* stats);
/* Unfused parts of one step, for the per-step plug points:
 * icb_push   = IIntegrationStrategy::step_batch (push only, no finalize)
 * icb_collide = ICollisionHandler::handle_batch (collision only)
 * icb_finalize = SimulationEngine::finalize_ions_after_integration + t += dt */
int icb_push(struct icb_handle* h);
int icb_collide(struct icb_handle* h, icb_run_stats* stats);
int icb_finalize(struct icb_handle* h, icb_run_stats* stats);
/* Engine clock: step index and time of ensemble 0 (all ensembles share the
 * step index; time_s[e] = accumulated dt of ensemble e). */
int icb_get_clock(struct icb_handle* h, uint64_t* step, double* time_s);
int icb_set_clock(struct icb_handle* h, uint64_t step, const double* time_s);
/* Per-ensemble moments of the active ions (ICB_N_MOMENTS doubles each). */
int icb_moments(struct icb_handle* h, double* out);
/* Store every ion's current position as its displacement reference. */
int icb_mark_reference(struct icb_handle* h);

/* ---- space charge (ISpaceChargeModel, ISpaceChargeModel.h:22-46) --------
 * Replaces the GPU space-charge model the factory builds when
 * physics.enable_space_charge_gpu is set (SpaceChargeModelFactory.cpp:29-95,
 * GPUSpaceChargeP3M.h:61-92 for the configuration).  Once configured, every
 * step of icb_advance / icb_push first solves the field of the current ion
 * positions (ISpaceChargeModel::update_fields, once per step before the push,
 * SimulationEngineLifecycle.cpp:16-32) and the push adds q E_sc to the force
 * (ForceRegistry.cpp:76-87).  Needs one ensemble and the Boris pusher (the
 * reference's RK4 refreshes space charge per stage).
 *   ICB_SC_P3M_ISOLATED: P3M with free-space boundaries: CIC charges on the
 *     mesh, zero-padded FFT convolution with the long-range part of the
 *     Coulomb field of a Gaussian-screened charge (screening alpha), CIC
 *     interpolation, plus a particle-particle correction to the softened
 *     direct-sum field (SpaceChargeDirectModel.cpp:20-66) within
 *     pp_cutoff_cells mesh cells.  Active ions inside the mesh take part.
 *   ICB_SC_PM_PERIODIC_REF: the reference's GPU particle-mesh solver as it is
 *     (GPUSpaceChargeP3M.cu:36-339): periodic FFT Poisson solve, central
 *     differences, no particle-particle part, all ions deposit.
 * Ions outside the mesh (a grid coordinate outside [0, n-1)) get no field
 * and deposit nothing, as in the reference solver. */
enum { ICB_SC_OFF = 0, ICB_SC_P3M_ISOLATED = 1, ICB_SC_PM_PERIODIC_REF = 2 };
typedef struct icb_spacecharge_config {
    int32_t mode;              /* ICB_SC_* */
    int32_t grid_n[3];         /* mesh nodes per axis (8 .. 512), GPUSpaceChargeP3M::Config::grid_n* */
    double box_min_m[3];       /* domain_min */
    double box_max_m[3];       /* domain_max; node spacing h = (max - min) / n */
    double alpha_h;            /* isolated: screening alpha times max(h); 0 = 1.0 */
    double pp_cutoff_cells;    /* isolated: particle-particle cutoff in units of max(h); 0 = 2 */
    double softening_m;        /* isolated: direct-sum softening; < 0 = 1e-10 (SpaceChargeModelFactory.h:26) */
    double field_bound_V_m;    /* bound on |E_sc| added to the collision majorant's field bound;
                                  0 = 4 x the largest |E_sc| of the configured state */
    int32_t solver_fp32;       /* isolated: 1 = mesh and particle-particle sums in single
                                  precision under an FP64 handle too (the float forms always
                                  use them); E_sc stays FP64 per ion.  0 = the handle's form */
    int32_t reserved[7];
} icb_spacecharge_config;
int icb_spacecharge_configure(struct icb_handle* h, const icb_spacecharge_config* cfg);
/* Space charge across devices (one process per GPU, the ions sharded over
 * the ranks): this handle's solve also deposits, and pairs with, the ions of
 * the other ranks, given as a device array on this handle's device of n
 * (x, y, z, q) double quadruples (16-byte aligned), e.g. an all-gather of
 * every rank's icb_spacecharge_export.  Entries [skip_begin, skip_begin +
 * skip_count) are this handle's own ions in that list and take no part, nor
 * do entries with q = 0.  Every following solve reads the array as it is
 * then (refresh it before each step, after the ranks' previous step); n = 0
 * removes the peers.  The field is computed for this handle's ions only.
 * With an automatic field bound (field_bound_V_m = 0) the first call with
 * peers takes the bound again over the whole state.  Isolated P3M only. */
int icb_spacecharge_set_peers(struct icb_handle* h, uint64_t n, const double* xyzq_device,
                              uint64_t skip_begin, uint64_t skip_count);
/* This handle's ions as (x, y, z, q) quadruples into a device array of
 * n_ions entries on the handle's device (16-byte aligned), on the handle's
 * stream: active, born ions with their charge, the others with q = 0. */
int icb_spacecharge_export(struct icb_handle* h, double* xyzq_device);
/* Solve the field of the current state and copy E_sc (V/m) of every ion to
 * host arrays (any may be NULL): ISpaceChargeModel::sample_electric_field. */
int icb_spacecharge_field(struct icb_handle* h, double* ex, double* ey, double* ez);

/* ---- interaction-potential collisions ----------------------------------
 * Replaces InteractionPotentialCollisionHandler::handle_collision
 * (InteractionPotentialCollisionHandler.cpp:298-552) and its offline table
 * (InteractionPotentialOfflineSampleSet.h:16-98) for an isotropic ion-neutral
 * potential: the reference's LJ1264 form V = c12/r^12 - c6/r^6 - c4/r^4
 * (interaction_potential_precompute.cpp:1386-1508), c12 = 4 eps sigma^12,
 * c6 = 4 eps sigma^6, sigma = r_m 2^(-1/6), c4 = 1/2 alpha' k q^2.
 * A collision event happens at rate n g pi b_max^2 (sigma_event, the
 * ensemble's ipm_bmax_m); the impact parameter is uniform in area below
 * b_max and the relative velocity is deflected elastically by chi(E, b),
 * E = mu g^2 / 2, with a uniform azimuth (the reference applies the
 * equivalent momentum transfer mu (v_out - v0) from its trajectory samples). */
typedef struct icb_ipm_potential {
    double epsilon_J;          /* LJ well depth */
    double r_m_m;              /* LJ minimum position */
    double polarizability_m3;  /* neutral polarizability volume alpha' */
    double charge_C;           /* ion charge in the induced-dipole term */
} icb_ipm_potential;
/* cos(chi) at n (E, b) pairs by the device quadrature (chi = pi - 2 b
 * int dr / (r^2 sqrt(1 - b^2/r^2 - V/E)) from the outermost turning point);
 * host arrays.  Replaces the trajectory integration of
 * interaction_potential_precompute.cpp:1672-1835. */
int icb_ipm_deflection(int device, const icb_ipm_potential* pot, uint64_t n, const double* E_J,
                       const double* b_m, double* cos_chi);
typedef struct icb_ipm_config {
    icb_ipm_potential potential;
    double b_max_m;            /* must equal every ensemble's ipm_bmax_m */
    double E_min_J, E_max_J;   /* table range (log-spaced); energies outside are clamped */
    int32_t n_E, n_b;          /* table size (>= 2 each) */
    /* trained range of the learned deflection (its input normalisation);
     * 0, 0 = the table range */
    double net_E_min_J, net_E_max_J;
    int32_t reserved[2];
} icb_ipm_config;
/* Build the cos(chi) table of the handle on its device (collision models
 * ICB_COLLISION_IPM_TABLE and ICB_COLLISION_IPM_MLP need it; the learned
 * model falls back to it outside [net_E_min, net_E_max]). */
int icb_ipm_configure(struct icb_handle* h, const icb_ipm_config* cfg);
/* Copy the table (n_E * n_b floats, row-major [E][b]) to the host. */
int icb_ipm_table(struct icb_handle* h, float* out);

/* ---- learned deflection (MLP 2 -> 64 -> 64 -> 1, tanh) ------------------
 * No counterpart in the reference: a network trained on the quadrature's
 * cos(chi) replaces the table lookup in the collision path.  Inputs
 * x0 = 2 (ln E - ln net_E_min) / (ln net_E_max - ln net_E_min) - 1,
 * x1 = 2 b / b_max - 1;
 * output cos(chi).  Parameters (ICB_MLP_N_PARAMS floats, in order):
 * W1[64][2], b1[64], W2[64][64], b2[64], W3[64], b3.  In the collision path
 * the weights are BF16 and the 64x64 layer runs on the tensor cores
 * (mma.sync m16n8k16, FP32 accumulation), the warp's colliding ions forming
 * the rows. */
#define ICB_MLP_HIDDEN 64
#define ICB_MLP_N_PARAMS 4417
typedef struct icb_mlp_train_config {
    int32_t epochs;
    int32_t batch;             /* samples per Adam step */
    double lr;                 /* initial learning rate (cosine decay to lr_min) */
    double lr_min;
    uint64_t seed;             /* initialisation and shuffling */
    int32_t bf16_forward;      /* train through the BF16 forward of the collision path */
    int32_t reserved[5];
} icb_mlp_train_config;
/* Xavier-uniform initial parameters from `seed`. */
int icb_mlp_init(uint64_t seed, float* params);
/* Adam on the mean squared error over n samples (x: 2n floats, y: n floats,
 * host); params in/out; loss_per_epoch (epochs doubles) may be NULL. */
int icb_mlp_train(int device, const icb_mlp_train_config* cfg, uint64_t n, const float* x, const float* y,
                  float* params, double* loss_per_epoch);
/* Network output for n inputs: mode 0 = FP32 reference arithmetic, mode 1 =
 * the collision path's BF16 tensor-core evaluation. */
int icb_mlp_forward(int device, const float* params, uint64_t n, const float* x, float* y, int mode);
/* Gradient of the mean squared error (FP32 arithmetic) and the loss. */
int icb_mlp_gradients(int device, const float* params, uint64_t n, const float* x, const float* y,
                      float* grad, double* loss);
/* Load network parameters into the handle (ICB_COLLISION_IPM_MLP). */
int icb_ipm_set_mlp(struct icb_handle* h, const float* params);

/* ---- EHSS molecule geometry ------------------------------------------- */
/* Atoms (centres relative to the ion's centre of mass, n_atoms x 3 doubles,
 * and radii) of the ions of one ensemble, and the gas (contact) radius
 * (EHSSCollisionHandler.cpp:278-297, geometry_map_ of the handler).  Every
 * ensemble needs one before stepping with ICB_COLLISION_EHSS. */
int icb_ehss_set_geometry(struct icb_handle* h, int32_t ensemble, int32_t n_atoms, const double* centers_m,
                          const double* radii_m, double gas_radius_m);

/* ---- time-dependent fields ---------------------------------------------- */
/* A voltage given as a waveform instead of a constant (ValueOrWaveform,
 * WaveformConfig.h:19-276, WaveformConfig.cpp:10-107), evaluated at the
 * field's time at every field evaluation, as the reference does.  p[] holds
 * the type's parameters in this order:
 *   CONSTANT     value
 *   LINEAR       start_value, end_value, start_time_s, end_time_s (clamp)
 *   QUADRATIC    a, b, c, start_time_s, end_time_s
 *   EXPONENTIAL  offset, amplitude, rate_per_s, start_time_s, end_time_s (clamp)
 *   SINUSOIDAL   offset, amplitude, frequency_Hz, phase_rad
 *   PWM          low_value, high_value, frequency_Hz, duty_cycle, phase_rad,
 *                start_time_s, end_time_s (clamp)
 *   PULSED       low_value, high_value, pulse_start_s, pulse_width_s
 *   ARBITRARY    n_points (1..ICB_MAX_WAVE_POINTS) ascending times_s and
 *                values, interp LINEAR / STEP / CUBIC (Catmull-Rom) */
#define ICB_MAX_WAVE_POINTS 64
enum { ICB_WAVE_CONSTANT = 0, ICB_WAVE_LINEAR = 1, ICB_WAVE_QUADRATIC = 2, ICB_WAVE_EXPONENTIAL = 3,
       ICB_WAVE_SINUSOIDAL = 4, ICB_WAVE_PWM = 5, ICB_WAVE_PULSED = 6, ICB_WAVE_ARBITRARY = 7 };
enum { ICB_INTERP_LINEAR = 0, ICB_INTERP_STEP = 1, ICB_INTERP_CUBIC = 2 };
typedef struct icb_waveform {
    int32_t type;              /* ICB_WAVE_* */
    int32_t clamp;             /* LINEAR / EXPONENTIAL / PWM: hold the end value after end_time_s */
    int32_t interp;            /* ARBITRARY: ICB_INTERP_* */
    int32_t n_points;          /* ARBITRARY */
    double p[8];
    double times_s[ICB_MAX_WAVE_POINTS];
    double values[ICB_MAX_WAVE_POINTS];
} icb_waveform;

/* Field channels that may carry a waveform (fields.DC.axial_V, DC.quad_V,
 * RF.voltage_V, RF.frequency_Hz, TIMS.ramp_fraction, and the LQIT AC
 * drives: axis x = AC.voltage_V / frequency_Hz of the single-axis drive or
 * dipolar_x.amplitude_V / frequency_Hz / ramp, axis y = dipolar_y's).  A
 * channel without a waveform uses the constant of icb_ensemble_params (the
 * TIMS ramp its built-in linear / exponential ramp). */
enum { ICB_CHANNEL_DC_AXIAL_V = 0, ICB_CHANNEL_DC_QUAD_V = 1, ICB_CHANNEL_RF_VOLTAGE_V = 2,
       ICB_CHANNEL_RF_FREQUENCY_HZ = 3, ICB_CHANNEL_TIMS_RAMP_FRACTION = 4,
       ICB_CHANNEL_AC_X_AMPLITUDE_V = 5, ICB_CHANNEL_AC_X_FREQUENCY_HZ = 6, ICB_CHANNEL_AC_X_RAMP = 7,
       ICB_CHANNEL_AC_Y_AMPLITUDE_V = 8, ICB_CHANNEL_AC_Y_FREQUENCY_HZ = 9, ICB_CHANNEL_AC_Y_RAMP = 10,
       ICB_N_CHANNELS = 11 };

/* Set (w != NULL) or clear (w == NULL) the waveform of one field channel of
 * one ensemble (IMS, QuadrupoleRF, LQIT or TIMS; the AC channels on an LQIT
 * only, the ramp channels with the two-axis dipolar drive).  An ensemble with a
 * waveform, like every TIMS ensemble, is stepped through the time-dependent
 * field path (one field evaluation per step or RK4 stage). */
int icb_set_waveform(struct icb_handle* h, int32_t ensemble, int32_t channel, const icb_waveform* w);

/* TIMS axial field (fields.TIMS, FieldsConfig.h:244-300): uniform initial /
 * final fields, or profiles over n_nodes local z positions (2..64,
 * ascending; the final profile may be absent, then the final uniform field
 * applies), ramped by f(t) = clamp((t - start) / (end - start)) (linear) or
 * (1 - e^{-(t - start)/tau}) / (1 - e^{-(end - start)/tau}) (exponential),
 * f = 0 before start and 1 after end; a TIMS.ramp_fraction waveform
 * (channel ICB_CHANNEL_TIMS_RAMP_FRACTION, clamped to [0, 1]) replaces the
 * built-in ramp.  Needs instrument ICB_INSTRUMENT_TIMS; f == NULL clears
 * (zero axial field). */
enum { ICB_TIMS_RAMP_LINEAR = 0, ICB_TIMS_RAMP_EXPONENTIAL = 1 };
typedef struct icb_tims_field {
    int32_t ramp_mode;         /* ICB_TIMS_RAMP_* */
    int32_t n_nodes;           /* 0 = uniform fields */
    int32_t has_final_profile; /* final_profile_V_m given */
    int32_t reserved_;
    double initial_uniform_V_m;
    double final_uniform_V_m;
    double ramp_start_s;
    double ramp_end_s;
    double ramp_tau_s;
    double z_positions_m[ICB_MAX_WAVE_POINTS];
    double initial_profile_V_m[ICB_MAX_WAVE_POINTS];
    double final_profile_V_m[ICB_MAX_WAVE_POINTS];
} icb_tims_field;
int icb_set_tims_field(struct icb_handle* h, int32_t ensemble, const icb_tims_field* f);

/* ---- launch-shape tuning ----------------------------------------------- */
typedef struct icb_tuning {
    int32_t block_size;        /* threads per block chosen */
    int32_t steps_per_vote;    /* collision-free steps between warp votes chosen */
    int32_t pending_threshold; /* deferred-collision batch size chosen */
    int32_t steps_per_launch;  /* unchanged by tuning */
    int32_t trials;            /* launch shapes timed */
    int32_t reserved;
    double ion_steps_per_s;    /* trial throughput of the chosen shape */
} icb_tuning;
/* No counterpart in the reference (its batch path has no launch shape).
 * Times trial_steps (0 = 500) fused steps of the uploaded ions under each
 * launch shape (block 64/128 x steps per vote 4/8/16 x pending threshold
 * 6/10/14), each from the same saved copy of the state, keeps the fastest
 * and restores the state and clock: the trajectory continues as if the call
 * had not been made.  In FP64 every shape gives bit-identical results; in
 * the float forms the shape moves where float position offsets are folded
 * into the double anchor, so results change at float rounding level. */
int icb_autotune(struct icb_handle* h, uint64_t trial_steps, icb_tuning* out);

/* ---- moments without device allocation -------------------------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (an engine whose allocator reserves all device memory up front, or a
 * fixed device-memory budget): the ICB_N_MOMENTS moments of one population
 * from caller-owned device arrays (positions, velocities, displacement
 * reference positions, active flags; arrival/death times may be NULL, then
 * slots 11/12 are 0) into `out` (device, ICB_N_MOMENTS doubles), launched on
 * `cuda_stream` (NULL = default stream).  Allocates nothing: partial sums go
 * to a 640 KB file-scope device array, so n <= 33,554,432 ions (larger n is
 * rejected with ICB_ERR_INVALID_ARGUMENT).  The first call on a device (and
 * the first after that device is reset) resolves that array's address and
 * should come before any stream capture.  The caller's current device is
 * unchanged on return.  All calls on a device share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
int icb_moments_noalloc(int device, uint64_t n, const double* x, const double* y, const double* z,
                        const double* vx, const double* vy, const double* vz,
                        const double* x_ref, const double* y_ref, const double* z_ref,
                        const uint8_t* active, const double* arrival_time_s,
                        const double* death_time_s, double* out, void* cuda_stream);

/* ---- counter-based RNG check ------------------------------------------ */
/* Evaluate the device Philox4x32-10 (use_curand = 0) or cuRAND's
 * curand_Philox4x32_10 (use_curand = 1) on n host counters (4 words each)
 * under key (lo32(seed), hi32(seed)) on `device`; results to out (4n).
 * Replaces nothing in the reference: it pins the stateless RNG that stands
 * in for PhysicsRng (CollisionTypes.h:31-49). */
int icb_philox_eval(int device, uint64_t n, const uint32_t* counters, uint64_t seed,
                    int use_curand, uint32_t* out);

/* Evaluate on `device` the float clock functions of the step kernel next to
 * CUDA's: NEG_LOG1M = -ln(1 - q) (series / hardware log), NEG_LOG1M_CUDA =
 * -log1pf(-q), ONE_MINUS_EXP = 1 - e^-x (series / hardware exp),
 * ONE_MINUS_EXP_CUDA = -expm1f(-x); n inputs x, results to out.  Replaces
 * nothing in the reference: it bounds the kernel's float forms. */
enum { ICB_MATH_NEG_LOG1M = 0, ICB_MATH_NEG_LOG1M_CUDA = 1, ICB_MATH_ONE_MINUS_EXP = 2,
       ICB_MATH_ONE_MINUS_EXP_CUDA = 3 };
int icb_clock_math_eval(int device, uint64_t n, const float* x, int which, float* out);

#ifdef __cplusplus
}
#endif

#endif /* ICARION_B200_H */
