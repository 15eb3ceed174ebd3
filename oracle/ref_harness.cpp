// ORACLE — test infrastructure only (never linked into the product).
//
// Drives the reference's own hot-path code, compiled from its sources by
// oracle/Makefile, with the engine's per-step order restated here because
// SimulationEngine itself needs HDF5/jsoncpp which this image lacks:
//
//   per step (SimulationEngine::process_timestep, SimulationEngine.cpp:374-428):
//     prepare:   ion outside the domain -> inactive, death = t
//                (SimulationEngineLifecycle.cpp:72-121)
//     integrate: BorisStrategy::step per ion (SimulationEngineIntegration.cpp:114-146)
//                or RK4Strategy::step_batch (uniform dt, :26-45)
//     collide:   HSSCollisionHandler::handle_collision per ion with
//                PhysicsRng(rng_seed + ion index) (RngUtils.cpp:51-53)
//     finalize:  domain exit -> inactive, death = t; non-finite -> inactive
//                (SimulationEngineLifecycle.cpp:123-195);  t += dt
//   arrival time = first crossing of the detector plane, linearly
//   interpolated within the step (analysis/ims_mobility.py:290-322 convention).
//
// Modes (key=value arguments):
//   uniforms seed= n= out=             PhysicsRng(seed).uniform01() x n
//   init     seed= n= sigma_pos= T= mass= charge= ccs= out=
//            ion cloud as IonLoader::sample_position/sample_velocity
//            (gaussian at the origin, thermal), std::mt19937(seed)
//   derive   <domain keys>             print the loader-derived constants
//   field    <domain keys> in= out=    E of the domain's field model at the
//            (x, y, z, t) rows of in (4 doubles each) into out (3 each)
//
// Time-dependent domain keys: wave_<axial|quad|rfv|rff|ramp|acxA|acxf|acxr|acyA|acyf|acyr>=
// "type|clamp|interp|p0,p1,..|t0,t1,..|v0,v1,.." (type 0..7 in the order of
// WaveformType; acx / acy: AC drive amplitude A, frequency f, ramp r of the
// single-axis drive or dipolar x, and dipolar y), attached inline as the
// loader does, or through the
// waveform library (waveform_ref) with wave_ref=1; TIMS: tims=1 tims_mode=
// tims_ei= tims_ef= tims_t0= tims_t1= tims_tau= tims_z= tims_pi= tims_pf=.
//   run      in= out= <domain keys> integrator= collision= steps= snap=
//            ref_step= threads= seed= schedule=static|faithful mom=
//            moments (20 per snapshot, layout of ICB_N_MOMENTS) of the
//            active ions; slots 14..19 are displacement moments from the
//            positions after ref_step steps.
//            sc=direct softening=: the reference's direct space charge.
//            collision=ipm ipm_samples=<file>: the reference's
//            InteractionPotentialCollisionHandler (random orientation mode)
//            with the offline sample set of <file> for species "ion"
//            (read by oracle/ref_ipm_loader.cpp).
#include "core/integrator/strategies/BorisStrategy.h"
#include "core/integrator/strategies/RK4Strategy.h"
#include "core/physics/collisions/HSSCollisionHandler.h"
#include "core/physics/collisions/InteractionPotentialCollisionHandler.h"
#include "core/config/types/SpeciesConfig.h"
#include "core/physics/forces/ElectricFieldForce.h"
#include "core/physics/forces/MagneticFieldForce.h"
#include "core/config/types/AnalyticalFieldModel.h"
#include "core/config/types/TIMSAxialFieldModel.h"
#include "core/config/types/WaveformConfig.h"
#include "core/config/types/CylindricalGeometry.h"
#include "core/types/IonEnsemble.h"
#include "core/physics/spacecharge/SpaceChargeDirectModel.h"
#include "core/physics/collisions/core/CollisionKernels.h"
#include "core/types/CollisionTypes.h"
#include "utils/constants.h"

#ifdef ICB_WITH_ADAPTERS
// the reference-side adapters of this library (icarion_b200/adapters)
#include "B200IntegrationStrategy.h"
#include "B200CollisionHandler.h"
#endif

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace ICARION;

namespace {

using Args = std::map<std::string, std::string>;

double num(const Args& a, const char* k, double def) {
    auto it = a.find(k);
    return it == a.end() ? def : std::strtod(it->second.c_str(), nullptr);
}
std::string str(const Args& a, const char* k, const char* def) {
    auto it = a.find(k);
    return it == a.end() ? std::string(def) : it->second;
}

// Ion state file: int64 n, then 12 arrays of n doubles:
// x y z vx vy vz mass charge ccs active t_death t_arrival
struct State {
    int64_t n = 0;
    std::vector<double> a[12];
};

State read_state(const std::string& path) {
    State s;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    if (std::fread(&s.n, sizeof(int64_t), 1, f) != 1) throw std::runtime_error("bad state file");
    for (auto& v : s.a) {
        v.resize(static_cast<size_t>(s.n));
        if (std::fread(v.data(), sizeof(double), v.size(), f) != v.size()) throw std::runtime_error("short state file");
    }
    std::fclose(f);
    return s;
}

void write_state(const std::string& path, const State& s) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fwrite(&s.n, sizeof(int64_t), 1, f);
    for (const auto& v : s.a) std::fwrite(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
}

std::vector<double> list(const std::string& v) {
    std::vector<double> out;
    size_t pos = 0;
    while (pos < v.size()) {
        size_t end = v.find(',', pos);
        if (end == std::string::npos) end = v.size();
        if (end > pos) out.push_back(std::strtod(v.substr(pos, end - pos).c_str(), nullptr));
        pos = end + 1;
    }
    return out;
}

// "type|clamp|interp|params|times|values" -> the reference's Waveform variant
config::Waveform parse_wave(const std::string& spec) {
    std::vector<std::string> f;
    size_t pos = 0;
    while (true) {
        size_t end = spec.find('|', pos);
        f.push_back(spec.substr(pos, end == std::string::npos ? std::string::npos : end - pos));
        if (end == std::string::npos) break;
        pos = end + 1;
    }
    while (f.size() < 6) f.push_back("");
    const int type = std::atoi(f[0].c_str());
    const bool clamp = std::atoi(f[1].c_str()) != 0;
    const int interp = std::atoi(f[2].c_str());
    std::vector<double> p = list(f[3]);
    p.resize(8, 0.0);
    config::Waveform w;
    switch (type) {
        case 0: { config::ConstantWaveform c; c.value = p[0]; w.data = c; break; }
        case 1: { config::LinearWaveform c; c.start_value = p[0]; c.end_value = p[1]; c.start_time_s = p[2];
                  c.end_time_s = p[3]; c.clamp = clamp; w.data = c; break; }
        case 2: { config::QuadraticWaveform c; c.a = p[0]; c.b = p[1]; c.c = p[2]; c.start_time_s = p[3];
                  c.end_time_s = p[4]; w.data = c; break; }
        case 3: { config::ExponentialWaveform c; c.offset = p[0]; c.amplitude = p[1]; c.rate_per_s = p[2];
                  c.start_time_s = p[3]; c.end_time_s = p[4]; c.clamp = clamp; w.data = c; break; }
        case 4: { config::SinusoidalWaveform c; c.offset = p[0]; c.amplitude = p[1]; c.frequency_Hz = p[2];
                  c.phase_rad = p[3]; w.data = c; break; }
        case 5: { config::PWMWaveform c; c.low_value = p[0]; c.high_value = p[1]; c.frequency_Hz = p[2];
                  c.duty_cycle = p[3]; c.phase_rad = p[4]; c.start_time_s = p[5]; c.end_time_s = p[6];
                  c.clamp = clamp; w.data = c; break; }
        case 6: { config::PulsedWaveform c; c.low_value = p[0]; c.high_value = p[1]; c.pulse_start_s = p[2];
                  c.pulse_width_s = p[3]; w.data = c; break; }
        default: {
            config::ArbitraryWaveform c;
            c.times_s = list(f[4]);
            c.values = list(f[5]);
            c.interp = interp == 1 ? config::ArbitraryWaveform::Interpolation::Step
                     : interp == 2 ? config::ArbitraryWaveform::Interpolation::Cubic
                                   : config::ArbitraryWaveform::Interpolation::Linear;
            w.data = c;
        }
    }
    return w;
}

// Domain exactly as the loader builds it: E/N -> axial_V via N = P/(kB T)
// (DomainConfigLoader.cpp:417-431), density and gas mass from
// EnvironmentConfig::compute_derived_properties.
config::DomainConfig make_domain(const Args& a) {
    config::DomainConfig d;
    const std::string inst = str(a, "instrument", "IMS");
    if (inst == "IMS") d.instrument = config::Instrument::IMS;
    else if (inst == "FTICR") d.instrument = config::Instrument::FTICR;
    else if (inst == "QuadrupoleRF") d.instrument = config::Instrument::QuadrupoleRF;
    else if (inst == "LQIT") d.instrument = config::Instrument::LQIT;
    else if (inst == "TIMS") d.instrument = config::Instrument::TIMS;
    else throw std::runtime_error("unsupported instrument " + inst);
    d.geometry.origin_m = Vec3{num(a, "origin_x", 0.0), num(a, "origin_y", 0.0), num(a, "origin_z", 0.0)};
    d.geometry.length_m = num(a, "length", 0.1);
    d.geometry.radius_m = num(a, "radius", 0.05);
    d.environment.temperature_K = num(a, "T", 300.0);
    d.environment.pressure_Pa = num(a, "P", 1000.0);
    d.environment.gas_species = str(a, "gas", "N2");
    // gas mixture "species:fraction:sigma_m2,..." (EnvironmentConfig::gas_mixture)
    const std::string mix = str(a, "mix", "");
    size_t pos = 0;
    while (pos < mix.size()) {
        size_t end = mix.find(',', pos);
        if (end == std::string::npos) end = mix.size();
        const std::string item = mix.substr(pos, end - pos);
        const size_t c1 = item.find(':'), c2 = item.find(':', c1 + 1);
        config::GasMixtureComponent comp;
        comp.species = item.substr(0, c1);
        comp.mole_fraction = std::stod(item.substr(c1 + 1, c2 - c1 - 1));
        comp.cross_section_m2 = std::stod(item.substr(c2 + 1));
        d.environment.gas_mixture.push_back(comp);
        pos = end + 1;
    }
    // gas flow profile (EnvironmentConfig::flow_model; DomainConfigLoader.cpp:204-212)
    if (a.count("flow_model")) d.environment.flow_model = config::EnvironmentConfig::parse_flow_model(str(a, "flow_model", ""));
    d.environment.axial_flow_velocity_m_s = num(a, "axial_flow_velocity", 0.0);
    d.environment.axial_flow_max_velocity_m_s = num(a, "axial_flow_max_velocity", 0.0);
    d.environment.compute_derived_properties();
    if (a.count("EN_Td")) {
        const double EN_Td = num(a, "EN_Td", 0.0);
        const double k_B = 1.380649e-23;
        const double N = d.environment.pressure_Pa / (k_B * d.environment.temperature_K);
        const double E_Vm = EN_Td * 1e-21 * N;
        d.fields.dc.axial_V.constant_value = E_Vm * d.geometry.length_m;
    }
    if (a.count("axial_V")) d.fields.dc.axial_V.constant_value = num(a, "axial_V", 0.0);
    d.fields.dc.radial_V.constant_value = num(a, "radial_V", 0.0);
    d.fields.dc.quad_V.constant_value = num(a, "dc_quad_V", 0.0);
    d.fields.rf.voltage_V.constant_value = num(a, "rf_V", 0.0);
    d.fields.rf.frequency_Hz.constant_value = num(a, "rf_f", 0.0);
    d.fields.magnetic.enabled = num(a, "magnetic", 0.0) != 0.0;
    d.fields.magnetic.field_strength_T = Vec3{num(a, "B_x", 0.0), num(a, "B_y", 0.0), num(a, "B_z", 0.0)};
    // LQIT AC excitation (FieldsConfig.h:93-168): single-axis ac_V/ac_f/ac_phase,
    // or the two-axis dipolar drive dip_{x,y}_{A,f,phase,ramp}
    d.fields.ac.voltage_V.constant_value = num(a, "ac_V", 0.0);
    d.fields.ac.frequency_Hz.constant_value = num(a, "ac_f", 0.0);
    d.fields.ac.phase_rad = num(a, "ac_phase", 0.0);
    for (const char* axis : {"x", "y"}) {
        const std::string pre = std::string("dip_") + axis + "_";
        if (!a.count(pre + "A")) continue;
        d.fields.ac.dipolar_excitation_defined = true;
        config::ACDipolarAxisConfig& ax = axis[0] == 'x' ? d.fields.ac.dipolar_x : d.fields.ac.dipolar_y;
        ax.enabled = true;
        ax.amplitude_V.constant_value = num(a, (pre + "A").c_str(), 0.0);
        ax.frequency_Hz.constant_value = num(a, (pre + "f").c_str(), 0.0);
        ax.phase_rad = num(a, (pre + "phase").c_str(), 0.0);
        ax.ramp.constant_value = num(a, (pre + "ramp").c_str(), 1.0);
    }
    d.fields.ac.compute_derived();
    // waveforms: inline (the loader resolves "@id" into an inline copy,
    // WaveformLoader.cpp:290-320) or through the library (wave_ref=1)
    const bool by_ref = num(a, "wave_ref", 0.0) != 0.0;
    const std::pair<const char*, config::ValueOrWaveform*> chans[] = {
        {"wave_axial", &d.fields.dc.axial_V}, {"wave_quad", &d.fields.dc.quad_V},
        {"wave_rfv", &d.fields.rf.voltage_V}, {"wave_rff", &d.fields.rf.frequency_Hz},
        {"wave_ramp", &d.fields.tims.ramp_fraction},
        {"wave_acxA", d.fields.ac.dipolar_excitation_defined ? &d.fields.ac.dipolar_x.amplitude_V : &d.fields.ac.voltage_V},
        {"wave_acxf", d.fields.ac.dipolar_excitation_defined ? &d.fields.ac.dipolar_x.frequency_Hz : &d.fields.ac.frequency_Hz},
        {"wave_acxr", &d.fields.ac.dipolar_x.ramp},
        {"wave_acyA", &d.fields.ac.dipolar_y.amplitude_V}, {"wave_acyf", &d.fields.ac.dipolar_y.frequency_Hz},
        {"wave_acyr", &d.fields.ac.dipolar_y.ramp}};
    for (const auto& [key, slot] : chans) {
        if (!a.count(key)) continue;
        config::Waveform w = parse_wave(str(a, key, ""));
        *slot = config::ValueOrWaveform{};
        if (by_ref) {
            w.id = key;
            d.fields.waveform_library[key] = w;
            slot->waveform_ref = key;
        } else {
            slot->waveform = w;
        }
        if (std::string(key) == "wave_ramp") d.fields.tims.ramp_fraction_defined = true;
    }
    if (num(a, "tims", 0.0) != 0.0) {
        auto& t = d.fields.tims;
        t.enabled = true;
        t.axial_field_initial_uniform_V_m = num(a, "tims_ei", 0.0);
        t.axial_field_final_uniform_V_m = num(a, "tims_ef", 0.0);
        t.ramp_start_s = num(a, "tims_t0", 0.0);
        t.ramp_end_s = num(a, "tims_t1", 0.0);
        t.ramp_mode = num(a, "tims_mode", 0.0) != 0.0 ? "exponential" : "linear";
        t.ramp_tau_s = num(a, "tims_tau", 1e-3);
        t.z_positions_m = list(str(a, "tims_z", ""));
        t.axial_field_initial_profile_V_m = list(str(a, "tims_pi", ""));
        t.axial_field_final_profile_V_m = list(str(a, "tims_pf", ""));
    }
    return d;
}

// The field model PhysicsSetup builds for the domain (PhysicsSetup.cpp:190-196).
std::unique_ptr<config::IFieldModel> make_field_model(const config::DomainConfig& d) {
    if (d.instrument == config::Instrument::TIMS || d.fields.tims.enabled)
        return std::make_unique<config::TIMSAxialFieldModel>(d);
    return std::make_unique<config::AnalyticalFieldModel>(d);
}

int mode_field(const Args& a) {
    config::DomainConfig d = make_domain(a);
    auto model = make_field_model(d);
    FILE* f = std::fopen(str(a, "in", "pts.bin").c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open points");
    std::vector<double> pts;
    double buf[4];
    while (std::fread(buf, sizeof(double), 4, f) == 4) pts.insert(pts.end(), buf, buf + 4);
    std::fclose(f);
    std::vector<double> out;
    for (size_t i = 0; i + 3 < pts.size(); i += 4) {
        const Vec3 E = model->E(Vec3{pts[i], pts[i + 1], pts[i + 2]}, pts[i + 3]);
        out.push_back(E.x); out.push_back(E.y); out.push_back(E.z);
    }
    FILE* g = std::fopen(str(a, "out", "E.bin").c_str(), "wb");
    std::fwrite(out.data(), sizeof(double), out.size(), g);
    std::fclose(g);
    return 0;
}

int mode_uniforms(const Args& a) {
    physics::PhysicsRng rng(static_cast<uint64_t>(std::strtoull(str(a, "seed", "123").c_str(), nullptr, 10)));
    const int64_t n = static_cast<int64_t>(num(a, "n", 64));
    std::vector<double> u(static_cast<size_t>(n));
    for (auto& x : u) x = rng.uniform01();
    FILE* f = std::fopen(str(a, "out", "uniforms.bin").c_str(), "wb");
    std::fwrite(u.data(), sizeof(double), u.size(), f);
    std::fclose(f);
    return 0;
}

int mode_init(const Args& a) {
    std::mt19937 rng(static_cast<uint32_t>(std::strtoul(str(a, "seed", "123").c_str(), nullptr, 10)));
    const int64_t n = static_cast<int64_t>(num(a, "n", 4096));
    const double sp = num(a, "sigma_pos", 5e-4);
    const double T = num(a, "T", 300.0);
    const double m = num(a, "mass", 200.0 * AMU_TO_KG);
    State s;
    s.n = n;
    for (auto& v : s.a) v.assign(static_cast<size_t>(n), 0.0);
    for (int64_t i = 0; i < n; ++i) {
        // IonLoader::sample_position (Gaussian) then sample_velocity (Thermal),
        // each with fresh distribution objects (IonLoader.cpp:246-313).
        std::normal_distribution<double> np(0.0, 1.0);
        const double px = 0.0 + np(rng) * sp;
        const double py = 0.0 + np(rng) * sp;
        const double pz = 0.0 + np(rng) * sp;
        std::normal_distribution<double> nv(0.0, 1.0);
        const double sig = std::sqrt(BOLTZMANN_CONSTANT * T / m);
        const double vx = nv(rng) * sig;
        const double vy = nv(rng) * sig;
        const double vz = nv(rng) * sig;
        const size_t k = static_cast<size_t>(i);
        s.a[0][k] = px; s.a[1][k] = py; s.a[2][k] = pz;
        s.a[3][k] = vx; s.a[4][k] = vy; s.a[5][k] = vz;
        s.a[6][k] = m;
        s.a[7][k] = num(a, "charge", ELEM_CHARGE_C);
        s.a[8][k] = num(a, "ccs", 150e-20);
        s.a[9][k] = 1.0;
        s.a[10][k] = -1.0;
        s.a[11][k] = -1.0;
    }
    write_state(str(a, "out", "state.bin"), s);
    return 0;
}

int mode_derive(const Args& a) {
    auto d = make_domain(a);
    std::printf("{\"gas_density_m3\": %.17g, \"gas_mass_kg\": %.17g, \"axial_V\": %.17g, "
                "\"E_z\": %.17g}\n",
                d.environment.particle_density_m_3, d.environment.gas_mass_kg,
                d.fields.dc.axial_V.constant_value.value_or(0.0),
                d.fields.dc.axial_V.constant_value.value_or(0.0) / d.geometry.length_m);
    return 0;
}

// Space-charge field of every ion from the reference's direct summation
// (SpaceChargeDirectModel::update_fields, SpaceChargeDirectModel.cpp:20-66,
// softening as the factory builds it, SpaceChargeModelFactory.h:26).
// Output file: 3n doubles (Ex[n], Ey[n], Ez[n]).
int mode_direct(const Args& a) {
    State s = read_state(str(a, "in", "state.bin"));
    std::vector<IonState> ions(static_cast<size_t>(s.n));
    for (int64_t i = 0; i < s.n; ++i) {
        auto& ion = ions[static_cast<size_t>(i)];
        const size_t k = static_cast<size_t>(i);
        ion.pos = Vec3{s.a[0][k], s.a[1][k], s.a[2][k]};
        ion.vel = Vec3{s.a[3][k], s.a[4][k], s.a[5][k]};
        ion.mass_kg = s.a[6][k];
        ion.ion_charge_C = s.a[7][k];
        ion.active = s.a[9][k] != 0.0;
        ion.born = true;
        ion.species_id = "ion";
    }
    core::IonEnsemble ens = core::IonEnsemble::from_legacy(ions);
    physics::SpaceChargeDirectModel model(num(a, "softening", 1e-10));
    model.update_fields(ens, 0.0);
    FILE* f = std::fopen(str(a, "out", "field.bin").c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write field file");
    for (int c = 0; c < 3; ++c) {
        for (int64_t i = 0; i < s.n; ++i) {
            const Vec3 e = model.sample_electric_field(static_cast<size_t>(i));
            const double v = c == 0 ? e.x : (c == 1 ? e.y : e.z);
            std::fwrite(&v, sizeof(double), 1, f);
        }
    }
    std::fclose(f);
    return 0;
}

// EHSS scattering law of the reference kernel
// (CollisionKernels::ehss_collision, CollisionKernels.cpp:13-137, 220-381).
// in: int64 n_atoms, then x,y,z,r per atom; int64 n, then v_ion (3n) and
// v_neutral (3n).  out: v_post (3n).  PhysicsRng(seed) drives all draws.
int mode_ehss(const Args& a) {
    FILE* f = std::fopen(str(a, "in", "ehss.bin").c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open ehss input");
    int64_t na = 0, n = 0;
    if (std::fread(&na, sizeof(na), 1, f) != 1) throw std::runtime_error("bad ehss input");
    std::vector<double> atoms(static_cast<size_t>(4 * na));
    if (std::fread(atoms.data(), sizeof(double), atoms.size(), f) != atoms.size()) throw std::runtime_error("short");
    if (std::fread(&n, sizeof(n), 1, f) != 1) throw std::runtime_error("bad ehss input");
    std::vector<double> vi(static_cast<size_t>(3 * n)), vn(static_cast<size_t>(3 * n));
    if (std::fread(vi.data(), sizeof(double), vi.size(), f) != vi.size()) throw std::runtime_error("short");
    if (std::fread(vn.data(), sizeof(double), vn.size(), f) != vn.size()) throw std::runtime_error("short");
    std::fclose(f);
    std::vector<Vec3> centers(static_cast<size_t>(na));
    std::vector<double> radii(static_cast<size_t>(na));
    for (int64_t j = 0; j < na; ++j) {
        centers[static_cast<size_t>(j)] = Vec3{atoms[4 * j], atoms[4 * j + 1], atoms[4 * j + 2]};
        radii[static_cast<size_t>(j)] = atoms[4 * j + 3];
    }
    const double mi = num(a, "mi", 1e-25), mn = num(a, "mn", 4.65e-26), rg = num(a, "rgas", 1.8e-10);
    physics::PhysicsRng rng(static_cast<uint64_t>(std::strtoull(str(a, "seed", "1").c_str(), nullptr, 10)));
    FILE* o = std::fopen(str(a, "out", "ehss_out.bin").c_str(), "wb");
    for (int64_t i = 0; i < n; ++i) {
        const Vec3 v{vi[3 * i], vi[3 * i + 1], vi[3 * i + 2]};
        const Vec3 w{vn[3 * i], vn[3 * i + 1], vn[3 * i + 2]};
        const Vec3 p = physics::collision_core::CollisionKernels::ehss_collision(v, w, mi, mn, rg, centers, radii,
                                                                                   rng);
        const double q[3] = {p.x, p.y, p.z};
        std::fwrite(q, sizeof(double), 3, o);
    }
    std::fclose(o);
    return 0;
}

int mode_run(const Args& a) {
    State s = read_state(str(a, "in", "state.bin"));
    const int64_t n = s.n;
    config::DomainConfig d = make_domain(a);
    const double dt = num(a, "dt", 5e-10);
    const int64_t steps = static_cast<int64_t>(num(a, "steps", 1000));
    const int64_t snap = static_cast<int64_t>(num(a, "snap", 0));
    const int64_t ref_step = static_cast<int64_t>(num(a, "ref_step", 0));
    const double zdet = num(a, "zdet", 1e30);
    const uint64_t seed = std::strtoull(str(a, "seed", "123").c_str(), nullptr, 10);
    const std::string integ = str(a, "integrator", "boris");
    const std::string coll = str(a, "collision", "none");
    const bool faithful = str(a, "schedule", "static") == "faithful";
    const int threads = static_cast<int>(num(a, "threads", 1));
#ifdef _OPENMP
    omp_set_num_threads(threads);
#else
    (void)threads;
#endif

    std::vector<IonState> ions(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        auto& ion = ions[static_cast<size_t>(i)];
        const size_t k = static_cast<size_t>(i);
        ion.pos = Vec3{s.a[0][k], s.a[1][k], s.a[2][k]};
        ion.vel = Vec3{s.a[3][k], s.a[4][k], s.a[5][k]};
        ion.mass_kg = s.a[6][k];
        ion.ion_charge_C = s.a[7][k];
        ion.CCS_m2 = s.a[8][k];
        ion.active = s.a[9][k] != 0.0;
        ion.born = true;
        ion.birth_time_s = 0.0;
        ion.species_id = "ion";
    }
    core::IonEnsemble ens = core::IonEnsemble::from_legacy(ions);

    auto field_model = make_field_model(d);
    auto reg = std::make_shared<physics::ForceRegistry>(d);
    reg->add_force(std::make_unique<physics::ElectricFieldForce>(d));
    if (d.fields.magnetic.enabled && integ != "boris")
        reg->add_force(std::make_unique<physics::MagneticFieldForce>(d.fields.magnetic));
    reg->set_field_model(field_model.get());
    // sc=direct: the reference's O(N^2) space charge (SpaceChargeDirectModel,
    // softening as SpaceChargeModelFactory.h:26), updated once per step
    // before the ions are prepared (SimulationEngineLifecycle.cpp:16-32) and
    // added as q E_sc by the force registry (ForceRegistry.cpp:76-87)
    std::shared_ptr<physics::SpaceChargeDirectModel> sc_model;
    if (str(a, "sc", "none") == "direct") {
        sc_model = std::make_shared<physics::SpaceChargeDirectModel>(num(a, "softening", 1e-10));
        reg->set_space_charge_model(sc_model);
    }
    std::vector<std::shared_ptr<physics::ForceRegistry>> regs{reg};
    config::CylindricalGeometry geom(d);

    integrator::BorisStrategy boris;
    integrator::RK4Strategy rk4;
    rk4.set_parallel_enabled(threads > 1);
    physics::HSSCollisionHandler hss_handler(false, nullptr);
    // interaction-potential collisions: the reference handler reads the
    // sample set named in the species database (the engine's wiring,
    // CollisionHandlerFactory.cpp:94-111, SpeciesConfig.h:39)
    config::SpeciesDatabase species_db;
    std::unique_ptr<physics::InteractionPotentialCollisionHandler> ipm_handler;
    if (coll == "ipm") {
        config::SpeciesProperties sp{};
        sp.id = "ion";
        sp.ipm_samples_file = str(a, "ipm_samples", "ipm_samples.bin");
        species_db.species.emplace("ion", sp);
        ipm_handler = std::make_unique<physics::InteractionPotentialCollisionHandler>(false, &species_db, "random");
    }
    physics::ICollisionHandler& hss = ipm_handler ? static_cast<physics::ICollisionHandler&>(*ipm_handler)
                                                  : static_cast<physics::ICollisionHandler&>(hss_handler);
    const bool colliding = coll == "hss" || coll == "ipm";
    std::vector<physics::PhysicsRng> rng;
    rng.reserve(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) rng.emplace_back(seed + static_cast<uint64_t>(i));

    auto* px = ens.pos_x_data(); auto* py = ens.pos_y_data(); auto* pz = ens.pos_z_data();
    auto* vx = ens.vel_x_data(); auto* vy = ens.vel_y_data(); auto* vz = ens.vel_z_data();
    auto* active = ens.active_data();
    std::vector<double>& t_death = s.a[10];
    std::vector<double>& t_arr = s.a[11];
    std::vector<double> zold(static_cast<size_t>(n));
    std::vector<int> dom(static_cast<size_t>(n), 0);
    const int64_t n_snap = snap > 0 ? steps / snap : 0;
    std::vector<double> mom(static_cast<size_t>(n_snap * 20), 0.0);
    std::vector<double> rx(px, px + n), ry(py, py + n), rz(pz, pz + n);
    uint64_t collisions = 0;
    // the collision environment of ion i: the reference engine evaluates a
    // non-constant gas flow at the ion's position before each collision
    // (SimulationEngineCollisionRuntime.cpp:124-131; unrotated cylinder)
    // collision sub-steps: handle_collision m times with dt / m at the pushed
    // position (SimulationEngineCollisionRuntime.cpp:79-190)
    const int subcycles = std::max(1, static_cast<int>(num(a, "subcycles", 1.0)));
    const bool flow_var = d.environment.flow_model != config::FlowModelKind::Constant;
    auto env_at = [&](int64_t i) -> const config::EnvironmentConfig& {
        if (!flow_var) return d.environment;
        thread_local config::EnvironmentConfig local_env;
        local_env = d.environment;
        local_env.gas_velocity_m_s = d.environment.gas_velocity_at(Vec3{px[i], py[i], pz[i]}, &d.geometry);
        return local_env;
    };

    double t = num(a, "t0", 0.0);
    const auto wall0 = std::chrono::steady_clock::now();
    for (int64_t k = 0; k < steps; ++k) {
        if (sc_model) sc_model->update_fields(ens, t);
        // prepare_ions_for_integration
        for (int64_t i = 0; i < n; ++i) {
            if (!active[i]) { dom[static_cast<size_t>(i)] = -1; continue; }
            if (!geom.contains(Vec3{px[i], py[i], pz[i]})) {
                active[i] = 0;
                t_death[static_cast<size_t>(i)] = t;
                dom[static_cast<size_t>(i)] = -1;
            } else {
                dom[static_cast<size_t>(i)] = 0;
            }
            zold[static_cast<size_t>(i)] = pz[i];
        }
        if (integ == "rk4") {
            rk4.step_batch(ens, t, dt, regs, dom);
            if (colliding) {
#pragma omp parallel for schedule(static) reduction(+ : collisions)
                for (int64_t i = 0; i < n; ++i) {
                    if (!active[i]) continue;
                    auto cv = ens.collision_data(static_cast<size_t>(i));
                    for (int sc = 0; sc < subcycles; ++sc)
                        collisions += hss.handle_collision(cv, dt / subcycles, rng[static_cast<size_t>(i)], env_at(i)) ? 1 : 0;
                }
            }
        } else if (faithful) {
            // Engine order as written: serial Boris loop, OpenMP collision loop.
            for (int64_t i = 0; i < n; ++i)
                if (active[i]) boris.step(ens, static_cast<size_t>(i), t, dt, *reg);
            if (colliding) {
#pragma omp parallel for schedule(guided, 128) reduction(+ : collisions)
                for (int64_t i = 0; i < n; ++i) {
                    if (!active[i]) continue;
                    auto cv = ens.collision_data(static_cast<size_t>(i));
                    for (int sc = 0; sc < subcycles; ++sc)
                        collisions += hss.handle_collision(cv, dt / subcycles, rng[static_cast<size_t>(i)], env_at(i)) ? 1 : 0;
                }
            }
        } else {
            // Best CPU form of the reference code: one OpenMP loop, push then collide.
#pragma omp parallel for schedule(static) reduction(+ : collisions)
            for (int64_t i = 0; i < n; ++i) {
                if (!active[i]) continue;
                boris.step(ens, static_cast<size_t>(i), t, dt, *reg);
                if (colliding) {
                    auto cv = ens.collision_data(static_cast<size_t>(i));
                    for (int sc = 0; sc < subcycles; ++sc)
                        collisions += hss.handle_collision(cv, dt / subcycles, rng[static_cast<size_t>(i)], env_at(i)) ? 1 : 0;
                }
            }
        }
        // finalize_ions_after_integration (+ arrival-plane crossing)
        for (int64_t i = 0; i < n; ++i) {
            const size_t k2 = static_cast<size_t>(i);
            if (dom[k2] < 0) continue;
            const double zo = zold[k2];
            if (t_arr[k2] < 0.0 && zo < zdet && pz[i] >= zdet)
                t_arr[k2] = t + dt * ((zdet - zo) / (pz[i] - zo));
            const Vec3 p{px[i], py[i], pz[i]};
            if (!geom.contains(p)) {
                active[i] = 0;
                t_death[k2] = t;
                continue;
            }
            if (!(std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z) &&
                  std::isfinite(vx[i]) && std::isfinite(vy[i]) && std::isfinite(vz[i]))) {
                active[i] = 0;
                t_death[k2] = t;
            }
        }
        t = t + dt;
        if (k + 1 == ref_step) {
            std::copy(px, px + n, rx.begin());
            std::copy(py, py + n, ry.begin());
            std::copy(pz, pz + n, rz.begin());
        }
        if (snap > 0 && (k + 1) % snap == 0) {
            double* m = &mom[static_cast<size_t>(((k + 1) / snap - 1) * 20)];
            for (int64_t i = 0; i < n; ++i) {
                const size_t k2 = static_cast<size_t>(i);
                if (t_arr[k2] >= 0.0) m[11] += 1.0;
                if (!active[i]) { if (t_death[k2] >= 0.0) m[12] += 1.0; continue; }
                m[0] += 1.0;
                m[1] += px[i]; m[2] += py[i]; m[3] += pz[i];
                m[4] += px[i] * px[i]; m[5] += py[i] * py[i]; m[6] += pz[i] * pz[i];
                m[7] += vx[i]; m[8] += vy[i]; m[9] += vz[i];
                m[10] += vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i];
                m[13] += pz[i] * vz[i];
                const double d[3] = {px[i] - rx[k2], py[i] - ry[k2], pz[i] - rz[k2]};
                for (int c = 0; c < 3; ++c) {
                    m[14 + c] += d[c];
                    m[17 + c] += d[c] * d[c];
                }
            }
        }
    }
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();

    for (int64_t i = 0; i < n; ++i) {
        const size_t k = static_cast<size_t>(i);
        s.a[0][k] = px[i]; s.a[1][k] = py[i]; s.a[2][k] = pz[i];
        s.a[3][k] = vx[i]; s.a[4][k] = vy[i]; s.a[5][k] = vz[i];
        s.a[9][k] = active[i] ? 1.0 : 0.0;
    }
    write_state(str(a, "out", "state_out.bin"), s);
    if (snap > 0) {
        FILE* f = std::fopen(str(a, "mom", "moments.bin").c_str(), "wb");
        std::fwrite(mom.data(), sizeof(double), mom.size(), f);
        std::fclose(f);
    }
    std::printf("{\"ion_steps\": %lld, \"wall_s\": %.6f, \"ion_steps_per_s\": %.6g, \"threads\": %d, "
                "\"collisions\": %llu, \"t_end\": %.17g}\n",
                static_cast<long long>(n * steps), wall, static_cast<double>(n * steps) / wall, threads,
                static_cast<unsigned long long>(collisions), t);
    return 0;
}

#ifdef ICB_WITH_ADAPTERS
// adapters: the reference engine's per-step order (as mode_run) with the
// plug points served by this library's reference-side adapters:
// B200IntegrationStrategy::step_batch (IIntegrationStrategy.h:119-132) and
// B200CollisionHandler::handle_batch (ICollisionHandler.h:121-134) on the
// reference's own IonEnsemble; prepare and finalize stay the engine's.
//   adapters in= out= <domain keys> integrator=boris|rk4 collision=none|hss
//            steps= dt= seed= precision=0|1|2
int mode_adapters(const Args& a) {
    State s = read_state(str(a, "in", "state.bin"));
    const int64_t n = s.n;
    config::DomainConfig d = make_domain(a);
    const double dt = num(a, "dt", 5e-10);
    const int64_t steps = static_cast<int64_t>(num(a, "steps", 100));
    const uint64_t seed = std::strtoull(str(a, "seed", "123").c_str(), nullptr, 10);
    const std::string integ = str(a, "integrator", "boris");
    const std::string coll = str(a, "collision", "hss");
    std::vector<IonState> ions(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        auto& ion = ions[static_cast<size_t>(i)];
        const size_t k = static_cast<size_t>(i);
        ion.pos = Vec3{s.a[0][k], s.a[1][k], s.a[2][k]};
        ion.vel = Vec3{s.a[3][k], s.a[4][k], s.a[5][k]};
        ion.mass_kg = s.a[6][k];
        ion.ion_charge_C = s.a[7][k];
        ion.CCS_m2 = s.a[8][k];
        ion.active = s.a[9][k] != 0.0;
        ion.born = true;
        ion.species_id = "ion";
    }
    core::IonEnsemble ens = core::IonEnsemble::from_legacy(ions);
    integrator::B200IntegrationStrategy strategy(d, integ == "rk4" ? "RK4" : "Boris", coll == "hss" ? "HSS" : "none",
                                                 seed, dt, n > 0 ? s.a[8][0] : 0.0,
                                                 static_cast<int>(num(a, "precision", 0)));
    physics::B200CollisionHandler collisions(strategy);
    auto reg = std::make_shared<physics::ForceRegistry>(d);
    std::vector<std::shared_ptr<physics::ForceRegistry>> regs{reg};
    std::vector<physics::PhysicsRng> rng_pool;     // ignored by the B200 handler (ICollisionHandler.h:118)
    config::CylindricalGeometry geom(d);
    auto* px = ens.pos_x_data(); auto* py = ens.pos_y_data(); auto* pz = ens.pos_z_data();
    auto* vx = ens.vel_x_data(); auto* vy = ens.vel_y_data(); auto* vz = ens.vel_z_data();
    auto* active = ens.active_data();
    std::vector<int> dom(static_cast<size_t>(n), 0);
    std::vector<size_t> idx;
    double t = 0.0;
    for (int64_t k = 0; k < steps; ++k) {
        idx.clear();
        for (int64_t i = 0; i < n; ++i) {           // prepare_ions_for_integration
            const size_t k2 = static_cast<size_t>(i);
            if (!active[i]) { dom[k2] = -1; continue; }
            if (!geom.contains(Vec3{px[i], py[i], pz[i]})) {
                active[i] = 0;
                s.a[10][k2] = t;
                dom[k2] = -1;
                continue;
            }
            dom[k2] = 0;
            idx.push_back(k2);
        }
        if (!strategy.step_batch(ens, t, dt, regs, dom)) throw std::runtime_error("step_batch refused");
        if (coll == "hss" && !collisions.handle_batch(ens, idx, dt, d.environment, rng_pool))
            throw std::runtime_error("handle_batch refused");
        for (int64_t i = 0; i < n; ++i) {           // finalize_ions_after_integration
            const size_t k2 = static_cast<size_t>(i);
            if (dom[k2] < 0) continue;
            const Vec3 p{px[i], py[i], pz[i]};
            if (!geom.contains(p) || !(std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z) &&
                                       std::isfinite(vx[i]) && std::isfinite(vy[i]) && std::isfinite(vz[i]))) {
                active[i] = 0;
                s.a[10][k2] = t;
            }
        }
        t = t + dt;
    }
    for (int64_t i = 0; i < n; ++i) {
        const size_t k = static_cast<size_t>(i);
        s.a[0][k] = px[i]; s.a[1][k] = py[i]; s.a[2][k] = pz[i];
        s.a[3][k] = vx[i]; s.a[4][k] = vy[i]; s.a[5][k] = vz[i];
        s.a[9][k] = active[i] ? 1.0 : 0.0;
    }
    write_state(str(a, "out", "state_out.bin"), s);
    std::printf("{\"ion_steps\": %lld, \"strategy\": \"%s\", \"handler\": \"%s\", \"t_end\": %.17g}\n",
                static_cast<long long>(n * steps), strategy.name().c_str(), collisions.name().c_str(), t);
    return 0;
}
#endif

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_harness uniforms|init|derive|run key=value...\n");
        return 2;
    }
    Args a;
    for (int i = 2; i < argc; ++i) {
        const char* eq = std::strchr(argv[i], '=');
        if (!eq) { std::fprintf(stderr, "bad argument %s\n", argv[i]); return 2; }
        a[std::string(argv[i], static_cast<size_t>(eq - argv[i]))] = std::string(eq + 1);
    }
    try {
        const std::string mode = argv[1];
        if (mode == "uniforms") return mode_uniforms(a);
        if (mode == "init") return mode_init(a);
        if (mode == "derive") return mode_derive(a);
        if (mode == "field") return mode_field(a);
        if (mode == "run") return mode_run(a);
        if (mode == "direct") return mode_direct(a);
        if (mode == "ehss") return mode_ehss(a);
#ifdef ICB_WITH_ADAPTERS
        if (mode == "adapters") return mode_adapters(a);
#endif
        std::fprintf(stderr, "unknown mode %s\n", argv[1]);
        return 2;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_harness: %s\n", e.what());
        return 1;
    }
}
