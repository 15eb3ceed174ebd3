// ORACLE — test infrastructure only (the checker, never the product).
//
// Runs the reference's own GPU particle-mesh solver
// (GPUSpaceChargeP3M::compute_space_charge_field, GPUSpaceChargeP3M.cpp:20-183
// with the kernels of GPUSpaceChargeP3M.cu:36-339), compiled from the
// reference sources by oracle/Makefile, on ions read from a file:
//
//   ref_p3m in=ions.bin out=field.bin nx= ny= nz= xmin= ymin= zmin= xmax= ymax= zmax=
//
// ions.bin: int64 n, then x[n], y[n], z[n], q[n] (doubles); field.bin: 3n
// doubles (Ex[n], Ey[n], Ez[n]).
#include "core/gpu/core/GPUContext.h"
#include "core/gpu/spacecharge/GPUSpaceChargeP3M.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

using namespace ICARION;

int main(int argc, char** argv) {
    std::map<std::string, std::string> a;
    for (int i = 1; i < argc; ++i) {
        const char* eq = std::strchr(argv[i], '=');
        if (eq) a[std::string(argv[i], static_cast<size_t>(eq - argv[i]))] = eq + 1;
    }
    auto num = [&](const char* k) { return std::stod(a.at(k)); };
    FILE* f = std::fopen(a.at("in").c_str(), "rb");
    if (!f) return 2;
    int64_t n = 0;
    if (std::fread(&n, sizeof(n), 1, f) != 1) return 2;
    std::vector<double> c[4];
    for (auto& v : c) {
        v.resize(static_cast<size_t>(n));
        if (std::fread(v.data(), sizeof(double), v.size(), f) != v.size()) return 2;
    }
    std::fclose(f);
    std::vector<IonState> ions(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        ions[static_cast<size_t>(i)].pos = Vec3{c[0][i], c[1][i], c[2][i]};
        ions[static_cast<size_t>(i)].ion_charge_C = c[3][i];
        ions[static_cast<size_t>(i)].active = true;
    }
    auto ctx = icarion::gpu::GPUContext::create(0);
    if (!ctx) return 3;
    icarion::gpu::GPUSpaceChargeP3M::Config cfg;
    cfg.grid_nx = static_cast<int>(num("nx"));
    cfg.grid_ny = static_cast<int>(num("ny"));
    cfg.grid_nz = static_cast<int>(num("nz"));
    cfg.domain_min = Vec3{num("xmin"), num("ymin"), num("zmin")};
    cfg.domain_max = Vec3{num("xmax"), num("ymax"), num("zmax")};
    auto solver = icarion::gpu::GPUSpaceChargeP3M::create(*ctx, cfg);
    if (!solver) return 4;
    std::vector<Vec3> E;
    if (!solver->compute_space_charge_field(ions, E)) return 5;
    FILE* o = std::fopen(a.at("out").c_str(), "wb");
    if (!o) return 2;
    for (int comp = 0; comp < 3; ++comp)
        for (int64_t i = 0; i < n; ++i) {
            const Vec3& e = E[static_cast<size_t>(i)];
            const double v = comp == 0 ? e.x : (comp == 1 ? e.y : e.z);
            std::fwrite(&v, sizeof(double), 1, o);
        }
    std::fclose(o);
    return 0;
}
