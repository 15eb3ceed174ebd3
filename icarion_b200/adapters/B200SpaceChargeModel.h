// src/core/physics/spacecharge/B200SpaceChargeModel.h
// Reference-side adapter (compiled into the ICARION tree, not into this
// library): ISpaceChargeModel over the icarion_b200 C ABI
// (ISpaceChargeModel.h:22-46).
// Built and exercised against the reference's own headers by oracle/Makefile
// (target _ref/ref_adapters) and tests/test_gpu_adapters.py.
#pragma once
#include "core/physics/spacecharge/ISpaceChargeModel.h"
#include "B200IntegrationStrategy.h"

#include <algorithm>
#include <stdexcept>
#include <vector>

namespace ICARION::physics {

// The field is solved on the device inside icb_push / icb_advance (once per
// step, before the push, as the engine orders it); update_fields only
// refreshes the host copy the reference's per-ion paths sample.
class B200SpaceChargeModel : public ISpaceChargeModel {
public:
    B200SpaceChargeModel(integrator::B200IntegrationStrategy& s, const config::DomainConfig& d, int grid_n) : s_(s) {
        icb_spacecharge_config c{};
        c.mode = ICB_SC_P3M_ISOLATED;            // ICB_SC_PM_PERIODIC_REF = the reference solver as it is
        c.grid_n[0] = c.grid_n[1] = c.grid_n[2] = grid_n;
        const double h = 0.5 * d.geometry.length_m;   // a cube around the cell centre
        for (int a = 0; a < 3; ++a) { c.box_min_m[a] = -h; c.box_max_m[a] = h; }
        c.box_min_m[2] += d.geometry.origin_m.z + h; c.box_max_m[2] += d.geometry.origin_m.z + h;
        c.softening_m = -1.0;                    // 1e-10 m, SpaceChargeModelFactory.h:26
        c.solver_fp32 = 1;                       // single-precision mesh under an FP64 push too
        if (icb_spacecharge_configure(s_.handle(), &c) != ICB_OK)
            throw std::runtime_error(icb_last_error());
    }
    void update_fields(const core::IonEnsemble& e, double) override {
        ex_.resize(e.size()); ey_.resize(e.size()); ez_.resize(e.size());
        if (icb_spacecharge_field(s_.handle(), ex_.data(), ey_.data(), ez_.data()) != ICB_OK)
            std::fill(ex_.begin(), ex_.end(), 0.0);   // as SpaceChargeGPUModel.cpp:25-42 on failure
    }
    core::Vec3 sample_electric_field(size_t i) const override {
        return i < ex_.size() ? core::Vec3{ex_[i], ey_[i], ez_[i]} : core::Vec3{0.0, 0.0, 0.0};
    }
    std::string name() const override { return "P3M (B200)"; }
private:
    integrator::B200IntegrationStrategy& s_;
    std::vector<double> ex_, ey_, ez_;
};

}  // namespace ICARION::physics
