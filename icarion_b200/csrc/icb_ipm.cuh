// icb_ipm.cuh — the classical deflection function of the ion-neutral
// potential by quadrature, shared by the table builder (icb_ipm.cu) and the
// per-collision quadrature collision model of the step kernel.
//
//     chi = pi - 2 (b / r0) \int_0^1 2 s ds / sqrt(F(r0 / (1 - s^2))),
//     F(r) = 1 - b^2/r^2 - V(r)/E,  V = c12/r^12 - c6/r^6 - c4/r^4,
// r0 the outermost zero of F (stepped inwards by 2 % from 4 (b + sigma),
// then bisected), 64-point Gauss-Legendre on [0, 1].  FP64 throughout.
#pragma once
#include <cuda_runtime.h>

#include "icb_params.h"

namespace icb {

constexpr int kGL = 64;

struct GLNodes {
    double s[kGL];   // nodes on [0, 1]
    double w[kGL];   // weights on [0, 1]
};

__device__ __forceinline__ double ipm_F(const IpmPotential& P, double E, double b, double r) {
    const double ir2 = 1.0 / (r * r);
    const double ir4 = ir2 * ir2, ir6 = ir4 * ir2, ir12 = ir6 * ir6;
    const double V = P.c12 * ir12 - P.c6 * ir6 - P.c4 * ir4;
    return 1.0 - b * b * ir2 - V / E;
}

// gl may live in shared or global memory (read through L1).
__device__ __forceinline__ double ipm_cos_chi(const IpmPotential& P, const GLNodes& gl, double E, double b) {
    if (!(E > 0.0)) return 1.0;
    double r = 4.0 * (b + P.sigma);
    int it = 0;
    while (ipm_F(P, E, b, r * 0.98) > 0.0 && it < 4000) {
        r *= 0.98;
        ++it;
    }
    double lo = r * 0.98, hi = r;
    for (int k = 0; k < 200 && hi - lo > 1e-15 * hi; ++k) {
        const double mid = 0.5 * (lo + hi);
        if (ipm_F(P, E, b, mid) > 0.0) hi = mid; else lo = mid;
    }
    const double r0 = hi;
    double I = 0.0;
    for (int k = 0; k < kGL; ++k) {
        const double s = gl.s[k];
        const double u = 1.0 - s * s;
        const double F = fmax(ipm_F(P, E, b, r0 / u), 1e-300);
        I += gl.w[k] * 2.0 * s / sqrt(F);
    }
    const double chi = M_PI - 2.0 * (b / r0) * I;
    return cos(chi);
}

}  // namespace icb
