// src/core/physics/collisions/B200CollisionHandler.h
// Reference-side adapter (compiled into the ICARION tree, not into this
// library): ICollisionHandler over the icarion_b200 C ABI
// (ICollisionHandler.h:59-135).
// Built and exercised against the reference's own headers by oracle/Makefile
// (target _ref/ref_adapters) and tests/test_gpu_adapters.py.
#pragma once
#include "core/physics/collisions/ICollisionHandler.h"
#include "B200IntegrationStrategy.h"

namespace ICARION::physics {

// Collisions on the integration strategy's device-resident state.
class B200CollisionHandler : public ICollisionHandler {
public:
    explicit B200CollisionHandler(integrator::B200IntegrationStrategy& s) : s_(s) {}
    bool handle_collision(core::IonCollisionData&, double, PhysicsRng&, const config::EnvironmentConfig&,
                          CollisionEventDiagnostics*) override {
        return false;   // per-ion path: the engine's CPU handler keeps serving it
    }
    std::string name() const override { return "HSS (B200)"; }
    bool supports_batch() const override { return true; }
    bool handle_batch(core::IonEnsemble& e, const std::vector<size_t>&, double, const config::EnvironmentConfig&,
                      std::vector<PhysicsRng>&) override {
        icb_run_stats st{};
        if (icb_collide(s_.handle(), &st) != ICB_OK) return false;   // CPU fallback by the engine
        return icb_download_ions(s_.handle(), nullptr, nullptr, nullptr, e.vel_x_data(), e.vel_y_data(),
                                 e.vel_z_data(), nullptr, nullptr, nullptr) == ICB_OK;
    }
private:
    integrator::B200IntegrationStrategy& s_;
};

}  // namespace ICARION::physics
