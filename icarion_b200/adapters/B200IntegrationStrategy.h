// src/core/integrator/strategies/B200IntegrationStrategy.h
// Reference-side adapter (compiled into the ICARION tree, not into this
// library): IIntegrationStrategy over the icarion_b200 C ABI
// (IIntegrationStrategy.h:44-140).
// Built and exercised against the reference's own headers by oracle/Makefile
// (target _ref/ref_adapters) and tests/test_gpu_adapters.py.
#pragma once
#include "core/integrator/strategies/IIntegrationStrategy.h"
#include "core/config/types/DomainConfig.h"
#include "icarion_b200.h"
#include <stdexcept>
#include <type_traits>
#include <variant>
#include <string>
#include <vector>

namespace ICARION::integrator {

// Device-resident batch step.  One instance owns one icb_handle; the engine
// drives it from one thread.
class B200IntegrationStrategy : public IIntegrationStrategy {
public:
    B200IntegrationStrategy(const config::DomainConfig& d, const std::string& integrator,
                            const std::string& collision_model, uint64_t rng_seed, double dt,
                            double sigma_m2, int precision = ICB_PREC_MIXED) {
        icb_ensemble_params p{};
        // PhysicsSetup.cpp:190-196: TIMS domains and enabled TIMS blocks use
        // TIMSAxialFieldModel
        const bool tims = d.instrument == config::Instrument::TIMS || d.fields.tims.enabled;
        p.instrument = tims ? ICB_INSTRUMENT_TIMS
                     : d.instrument == config::Instrument::FTICR ? ICB_INSTRUMENT_FTICR
                     : d.instrument == config::Instrument::QuadrupoleRF ? ICB_INSTRUMENT_QUADRUPOLE_RF
                     : d.instrument == config::Instrument::LQIT ? ICB_INSTRUMENT_LQIT
                     : ICB_INSTRUMENT_IMS;
        p.magnetic_enabled = d.fields.magnetic.enabled;
        p.origin_m[0] = d.geometry.origin_m.x; p.origin_m[1] = d.geometry.origin_m.y;
        p.origin_m[2] = d.geometry.origin_m.z;
        p.length_m = d.geometry.length_m; p.radius_m = d.geometry.radius_m;
        p.axial_V = d.fields.dc.axial_V.constant_value.value_or(0.0);
        p.radial_V = d.fields.dc.radial_V.constant_value.value_or(0.0);
        p.dc_quad_V = d.fields.dc.quad_V.constant_value.value_or(0.0);
        p.rf_voltage_V = d.fields.rf.voltage_V.constant_value.value_or(0.0);
        p.rf_frequency_Hz = d.fields.rf.frequency_Hz.constant_value.value_or(0.0);
        p.B_T[0] = d.fields.magnetic.field_strength_T.x; p.B_T[1] = d.fields.magnetic.field_strength_T.y;
        p.B_T[2] = d.fields.magnetic.field_strength_T.z;
        // LQIT AC drives (constant values)
        const auto& ac = d.fields.ac;
        p.ac_dipolar = ac.dipolar_excitation_defined;
        if (p.ac_dipolar) {
            const config::ACDipolarAxisConfig* axes[2] = {&ac.dipolar_x, &ac.dipolar_y};
            for (int a = 0; a < 2; ++a) {
                if (!axes[a]->enabled) continue;
                p.ac_amplitude_V[a] = axes[a]->amplitude_V.constant_value.value_or(0.0);
                p.ac_frequency_Hz[a] = axes[a]->frequency_Hz.constant_value.value_or(0.0);
                p.ac_phase_rad[a] = axes[a]->phase_rad;
                p.ac_ramp[a] = axes[a]->ramp.constant_value.value_or(1.0);
            }
        } else {
            p.ac_amplitude_V[0] = ac.voltage_V.constant_value.value_or(0.0);
            p.ac_frequency_Hz[0] = ac.frequency_Hz.constant_value.value_or(0.0);
            p.ac_phase_rad[0] = ac.phase_rad;
        }
        p.temperature_K = d.environment.temperature_K;
        p.gas_density_m3 = d.environment.particle_density_m_3;
        p.gas_mass_kg = d.environment.gas_mass_kg;
        p.gas_velocity_m_s[0] = d.environment.gas_velocity_m_s.x;
        p.gas_velocity_m_s[1] = d.environment.gas_velocity_m_s.y;
        p.gas_velocity_m_s[2] = d.environment.gas_velocity_m_s.z;
        p.flow_model = static_cast<int32_t>(d.environment.flow_model);   // Constant 0, AxialUniform 1, AxialParabolic 2
        p.axial_flow_velocity_m_s = d.environment.axial_flow_velocity_m_s;
        p.axial_flow_max_velocity_m_s = d.environment.axial_flow_max_velocity_m_s;
        p.sigma_m2 = sigma_m2;
        // gas mixture (HSSCollisionHandler.cpp:105-249): the components that
        // take part in collisions, with the loader's derived density and mass
        int ng = 0;
        for (const auto& comp : d.environment.gas_mixture) {
            if (!comp.participates_in_collisions || comp.density_m3 <= 0.0) continue;
            if (ng == ICB_MAX_GAS) throw std::runtime_error("B200: more than ICB_MAX_GAS gas components");
            p.gas_mix_density_m3[ng] = comp.density_m3;
            p.gas_mix_mass_kg[ng] = comp.mass_kg;
            p.gas_mix_sigma_m2[ng] = comp.cross_section_m2 > 0.0 ? comp.cross_section_m2 : sigma_m2;
            ++ng;
        }
        if (ng == 1) {            // one colliding component: the single-gas form
            p.gas_density_m3 = p.gas_mix_density_m3[0];
            p.gas_mass_kg = p.gas_mix_mass_kg[0];
            p.sigma_m2 = p.gas_mix_sigma_m2[0];
        }
        p.n_gas = ng >= 2 ? ng : 0;
        p.dt_s = dt;
        p.detector_z_m = 1e30;
        icb_config c{};
        c.precision = precision;
        c.integrator = integrator == "Boris" ? ICB_INTEGRATOR_BORIS : ICB_INTEGRATOR_RK4;
        c.collision_model = collision_model == "HSS" ? ICB_COLLISION_HSS : ICB_COLLISION_NONE;
        c.n_ensembles = 1;
        c.ensembles = &p;
        c.rng_seed = rng_seed;
        // c.stepping stays ICB_STEPPING_EVENTS (0): the float forms move each
        // ion from event to event in closed form; ICB_STEPPING_PER_STEP keeps
        // the step-by-step loop (same random draws, float rounding differs)
        // Collision sub-steps (PhysicsConfig): m = multi_event_mode
        //   ? max(collision_subcycles_per_step, collision_max_events_per_step)
        //   : collision_subcycles_per_step; m > 1 needs ICB_COLLISION_HSS_PLAIN
        //   (FP64), e.g. c.collision_subcycles = m;
        check(icb_create(&c, &h_));
        set_time_fields(d, tims);
    }
    ~B200IntegrationStrategy() override { icb_destroy(h_); }

    // Waveform voltages and the TIMS axial field (icb_set_waveform,
    // icb_set_tims_field).  IMS / QuadrupoleRF read only constants and
    // waveform_ref values (AnalyticalFieldModel.cpp:140-147, 226-233); the
    // LQIT and TIMS models also read inline waveforms.
    void set_time_fields(const config::DomainConfig& d, bool tims) {
        const auto& lib = d.fields.waveform_library;
        const bool inline_ok = tims || d.instrument == config::Instrument::LQIT;
        auto send = [&](int ch, const config::ValueOrWaveform& v) {
            const config::Waveform* w = nullptr;
            if (v.waveform_ref) w = &lib.at(*v.waveform_ref);
            else if (v.waveform && inline_ok) w = &*v.waveform;
            if (!w) return;
            icb_waveform iw{};
            to_icb(*w, iw);
            check(icb_set_waveform(h_, 0, ch, &iw));
        };
        if (d.instrument != config::Instrument::FTICR) {
            send(ICB_CHANNEL_DC_AXIAL_V, d.fields.dc.axial_V);
            send(ICB_CHANNEL_DC_QUAD_V, d.fields.dc.quad_V);
            send(ICB_CHANNEL_RF_VOLTAGE_V, d.fields.rf.voltage_V);
            send(ICB_CHANNEL_RF_FREQUENCY_HZ, d.fields.rf.frequency_Hz);
        }
        if (!tims) return;
        const auto& t = d.fields.tims;
        icb_tims_field f{};
        f.ramp_mode = t.ramp_mode == "exponential" ? ICB_TIMS_RAMP_EXPONENTIAL : ICB_TIMS_RAMP_LINEAR;
        f.initial_uniform_V_m = t.axial_field_initial_uniform_V_m;
        f.final_uniform_V_m = t.axial_field_final_uniform_V_m;
        f.ramp_start_s = t.ramp_start_s; f.ramp_end_s = t.ramp_end_s; f.ramp_tau_s = t.ramp_tau_s;
        f.n_nodes = static_cast<int32_t>(t.z_positions_m.size());
        f.has_final_profile = !t.axial_field_final_profile_V_m.empty();
        for (int32_t i = 0; i < f.n_nodes; ++i) {
            f.z_positions_m[i] = t.z_positions_m[i];
            f.initial_profile_V_m[i] = t.axial_field_initial_profile_V_m[i];
            if (f.has_final_profile) f.final_profile_V_m[i] = t.axial_field_final_profile_V_m[i];
        }
        check(icb_set_tims_field(h_, 0, &f));
        if (t.ramp_fraction_defined) {
            if (t.ramp_fraction.constant_value) {
                icb_waveform c{};
                c.type = ICB_WAVE_CONSTANT;
                c.p[0] = *t.ramp_fraction.constant_value;
                check(icb_set_waveform(h_, 0, ICB_CHANNEL_TIMS_RAMP_FRACTION, &c));
            } else {
                send(ICB_CHANNEL_TIMS_RAMP_FRACTION, t.ramp_fraction);
            }
        }
    }

    // The Waveform variant -> icb_waveform (parameters in the order the
    // header lists for each type).
    static void to_icb(const config::Waveform& w, icb_waveform& o) {
        std::visit([&](const auto& x) {
            using T = std::decay_t<decltype(x)>;
            if constexpr (std::is_same_v<T, config::ConstantWaveform>) {
                o.type = ICB_WAVE_CONSTANT; o.p[0] = x.value;
            } else if constexpr (std::is_same_v<T, config::LinearWaveform>) {
                o.type = ICB_WAVE_LINEAR; o.clamp = x.clamp;
                o.p[0] = x.start_value; o.p[1] = x.end_value; o.p[2] = x.start_time_s; o.p[3] = x.end_time_s;
            } else if constexpr (std::is_same_v<T, config::QuadraticWaveform>) {
                o.type = ICB_WAVE_QUADRATIC;
                o.p[0] = x.a; o.p[1] = x.b; o.p[2] = x.c; o.p[3] = x.start_time_s; o.p[4] = x.end_time_s;
            } else if constexpr (std::is_same_v<T, config::ExponentialWaveform>) {
                o.type = ICB_WAVE_EXPONENTIAL; o.clamp = x.clamp;
                o.p[0] = x.offset; o.p[1] = x.amplitude; o.p[2] = x.rate_per_s;
                o.p[3] = x.start_time_s; o.p[4] = x.end_time_s;
            } else if constexpr (std::is_same_v<T, config::SinusoidalWaveform>) {
                o.type = ICB_WAVE_SINUSOIDAL;
                o.p[0] = x.offset; o.p[1] = x.amplitude; o.p[2] = x.frequency_Hz; o.p[3] = x.phase_rad;
            } else if constexpr (std::is_same_v<T, config::PWMWaveform>) {
                o.type = ICB_WAVE_PWM; o.clamp = x.clamp;
                o.p[0] = x.low_value; o.p[1] = x.high_value; o.p[2] = x.frequency_Hz; o.p[3] = x.duty_cycle;
                o.p[4] = x.phase_rad; o.p[5] = x.start_time_s; o.p[6] = x.end_time_s;
            } else if constexpr (std::is_same_v<T, config::PulsedWaveform>) {
                o.type = ICB_WAVE_PULSED;
                o.p[0] = x.low_value; o.p[1] = x.high_value; o.p[2] = x.pulse_start_s; o.p[3] = x.pulse_width_s;
            } else {
                o.type = ICB_WAVE_ARBITRARY;
                o.interp = x.interp == config::ArbitraryWaveform::Interpolation::Step ? ICB_INTERP_STEP
                         : x.interp == config::ArbitraryWaveform::Interpolation::Cubic ? ICB_INTERP_CUBIC
                                                                                       : ICB_INTERP_LINEAR;
                if (x.times_s.size() > ICB_MAX_WAVE_POINTS) throw std::runtime_error("B200: waveform table too long");
                o.n_points = static_cast<int32_t>(x.times_s.size());
                for (int32_t i = 0; i < o.n_points; ++i) { o.times_s[i] = x.times_s[i]; o.values[i] = x.values[i]; }
            }
        }, w.data);
    }

    void step(core::IonEnsemble&, size_t, double, double, const physics::ForceRegistry&) override {
        throw std::runtime_error("B200IntegrationStrategy: per-ion step is not offered; use step_batch");
    }
    std::string name() const override { return "B200"; }
    bool is_adaptive() const override { return false; }
    bool supports_batch() const override { return true; }

    bool step_batch(core::IonEnsemble& e, double t, double dt,
                    const std::vector<std::shared_ptr<physics::ForceRegistry>>&,
                    const std::vector<int>& domain_indices) override {
        const uint64_t n = e.size();
        std::vector<uint8_t> act(n);
        for (uint64_t i = 0; i < n; ++i) act[i] = (domain_indices[i] >= 0 && e.is_active(i)) ? 1 : 0;
        if (icb_ion_count(h_) != n) {
            check(icb_upload_ions(h_, n, e.pos_x_data(), e.pos_y_data(), e.pos_z_data(), e.vel_x_data(),
                                  e.vel_y_data(), e.vel_z_data(), e.mass_data(), e.charge_data(), act.data(),
                                  nullptr, nullptr, 0));
        } else {
            check(icb_update_state(h_, e.pos_x_data(), e.pos_y_data(), e.pos_z_data(), e.vel_x_data(),
                                   e.vel_y_data(), e.vel_z_data(), act.data()));
        }
        check(icb_set_clock(h_, step_++, &t));
        (void)dt;   // the handle's ensemble dt is the engine's uniform dt
        check(icb_push(h_));
        check(icb_download_ions(h_, e.pos_x_data(), e.pos_y_data(), e.pos_z_data(), e.vel_x_data(),
                                e.vel_y_data(), e.vel_z_data(), nullptr, nullptr, nullptr));
        return true;
    }

    icb_handle* handle() { return h_; }

private:
    static void check(int rc) {
        if (rc != ICB_OK) throw std::runtime_error(std::string("icarion_b200: ") + icb_last_error());
    }
    icb_handle* h_ = nullptr;
    uint64_t step_ = 0;
};

}  // namespace ICARION::integrator
