// icb_ions.cu — host-side ion cloud generation with the reference loader's
// semantics: one std::mt19937(rng_seed) shared by all species in order, and
// per ion sample_position then sample_velocity, each with freshly
// constructed std::normal_distribution / std::uniform_real_distribution
// objects (IonLoader.cpp:183-238, :246-313; FullConfig.cpp:111).  Using the
// same standard library distributions as the reference build gives the
// identical initial state, which both the CPU oracle runs and the device
// runs start from.
#include <cmath>
#include <cstdint>
#include <random>

#include "../../include/icarion_b200.h"

namespace {
constexpr double kBoltzmann = 1.380649e-23;   // utils/constants.h:15
}

extern "C" int icb_generate_ions(uint32_t rng_seed, int32_t n_species, const icb_species_spec* specs,
                                 double* x, double* y, double* z, double* vx, double* vy, double* vz,
                                 double* mass_kg, double* charge_C) {
    if (n_species < 0 || (n_species > 0 && !specs)) return ICB_ERR_INVALID_ARGUMENT;
    if (!x || !y || !z || !vx || !vy || !vz || !mass_kg || !charge_C) return ICB_ERR_INVALID_ARGUMENT;
    std::mt19937 rng(rng_seed);
    uint64_t k = 0;
    for (int s = 0; s < n_species; ++s) {
        const icb_species_spec& sp = specs[s];
        if (!(sp.mass_kg > 0.0)) return ICB_ERR_INVALID_ARGUMENT;
        for (uint64_t i = 0; i < sp.count; ++i, ++k) {
            double px, py, pz;
            {
                std::normal_distribution<double> normal(0.0, 1.0);
                std::uniform_real_distribution<double> uniform(0.0, 1.0);
                switch (sp.position_type) {
                    case ICB_POS_POINT:
                        px = sp.center_m[0]; py = sp.center_m[1]; pz = sp.center_m[2];
                        break;
                    case ICB_POS_GAUSSIAN: {
                        const double ax = sp.center_m[0] + normal(rng) * sp.std_m[0];
                        const double ay = sp.center_m[1] + normal(rng) * sp.std_m[1];
                        const double az = sp.center_m[2] + normal(rng) * sp.std_m[2];
                        px = ax; py = ay; pz = az;
                        break;
                    }
                    case ICB_POS_UNIFORM_SPHERE: {
                        const double r = sp.radius_m * std::cbrt(uniform(rng));
                        const double theta = 2.0 * M_PI * uniform(rng);
                        const double phi = std::acos(2.0 * uniform(rng) - 1.0);
                        px = sp.center_m[0] + r * std::sin(phi) * std::cos(theta);
                        py = sp.center_m[1] + r * std::sin(phi) * std::sin(theta);
                        pz = sp.center_m[2] + r * std::cos(phi);
                        break;
                    }
                    case ICB_POS_UNIFORM_CYLINDER: {
                        const double r = sp.radius_m * std::sqrt(uniform(rng));
                        const double theta = 2.0 * M_PI * uniform(rng);
                        const double zz = sp.length_m * (uniform(rng) - 0.5);
                        px = sp.center_m[0] + r * std::cos(theta);
                        py = sp.center_m[1] + r * std::sin(theta);
                        pz = sp.center_m[2] + zz;
                        break;
                    }
                    case ICB_POS_UNIFORM_BOX: {
                        const double ax = sp.box_min_m[0] + uniform(rng) * (sp.box_max_m[0] - sp.box_min_m[0]);
                        const double ay = sp.box_min_m[1] + uniform(rng) * (sp.box_max_m[1] - sp.box_min_m[1]);
                        const double az = sp.box_min_m[2] + uniform(rng) * (sp.box_max_m[2] - sp.box_min_m[2]);
                        px = ax; py = ay; pz = az;
                        break;
                    }
                    default:
                        return ICB_ERR_INVALID_ARGUMENT;
                }
            }
            double ux, uy, uz;
            {
                std::normal_distribution<double> normal(0.0, 1.0);
                switch (sp.velocity_type) {
                    case ICB_VEL_FIXED:
                        ux = sp.velocity_m_s[0]; uy = sp.velocity_m_s[1]; uz = sp.velocity_m_s[2];
                        break;
                    case ICB_VEL_THERMAL: {
                        const double sigma = std::sqrt(kBoltzmann * sp.temperature_K / sp.mass_kg);
                        const double ax = normal(rng) * sigma;
                        const double ay = normal(rng) * sigma;
                        const double az = normal(rng) * sigma;
                        ux = ax; uy = ay; uz = az;
                        break;
                    }
                    default:
                        return ICB_ERR_INVALID_ARGUMENT;
                }
            }
            x[k] = px; y[k] = py; z[k] = pz;
            vx[k] = ux; vy[k] = uy; vz[k] = uz;
            mass_kg[k] = sp.mass_kg;
            charge_C[k] = sp.charge_C;
        }
    }
    return ICB_OK;
}
