// icb_step_dispatch.cuh — maps runtime (integrator, collision, field, B)
// choices onto the compiled template instances of k_step.
#pragma once
#include <cuda_runtime.h>
#include "icb_step_kernel.cuh"

namespace icb {

template <int PREC, int INTEG, int COLL, int FIELD, bool MAG>
cudaError_t launch_one(const StepParams& p, dim3 grid, dim3 block, cudaStream_t s) {
    if (p.do_push && p.do_collide && p.do_finalize)
        k_step<PREC, INTEG, COLL, FIELD, MAG, true><<<grid, block, 0, s>>>(p);
    else
        k_step<PREC, INTEG, COLL, FIELD, MAG, false><<<grid, block, 0, s>>>(p);
    return cudaGetLastError();
}

template <int PREC, int INTEG, int COLL>
cudaError_t dispatch_field(int field, bool mag, const StepParams& p, dim3 g, dim3 b, cudaStream_t s) {
    switch (field) {
        case kFieldUniform:
            return mag ? launch_one<PREC, INTEG, COLL, kFieldUniform, true>(p, g, b, s)
                       : launch_one<PREC, INTEG, COLL, kFieldUniform, false>(p, g, b, s);
        case kFieldLinear:
            return mag ? launch_one<PREC, INTEG, COLL, kFieldLinear, true>(p, g, b, s)
                       : launch_one<PREC, INTEG, COLL, kFieldLinear, false>(p, g, b, s);
        case kFieldLinearRF:
            return mag ? launch_one<PREC, INTEG, COLL, kFieldLinearRF, true>(p, g, b, s)
                       : launch_one<PREC, INTEG, COLL, kFieldLinearRF, false>(p, g, b, s);
        default:
            return cudaErrorNotSupported;
    }
}

template <int PREC, bool WITH_RK4>
cudaError_t dispatch_step(int integ, int coll, int field, bool mag, const StepParams& p,
                          dim3 g, dim3 b, cudaStream_t s) {
    if (integ == kBoris) {
        if (coll == kCollNone) return dispatch_field<PREC, kBoris, kCollNone>(field, mag, p, g, b, s);
        if (coll == kCollHSS) return dispatch_field<PREC, kBoris, kCollHSS>(field, mag, p, g, b, s);
        if (coll == kCollLangevin) return dispatch_field<PREC, kBoris, kCollLangevin>(field, mag, p, g, b, s);
        if (coll == kCollIPMTable) return dispatch_field<PREC, kBoris, kCollIPMTable>(field, mag, p, g, b, s);
        if (coll == kCollIPMMLP) return dispatch_field<PREC, kBoris, kCollIPMMLP>(field, mag, p, g, b, s);
        if (coll == kCollIPMQuad) {
            // the per-collision quadrature: built for the uniform drift field
            if (field != kFieldUniform || mag) return cudaErrorNotSupported;
            return launch_one<PREC, kBoris, kCollIPMQuad, kFieldUniform, false>(p, g, b, s);
        }
        if (coll == kCollHSSMix) return dispatch_field<PREC, kBoris, kCollHSSMix>(field, mag, p, g, b, s);
        if (coll == kCollEHSS) return dispatch_field<PREC, kBoris, kCollEHSS>(field, mag, p, g, b, s);
        if constexpr (PREC == kPrecFP64) {
            if (coll == kCollHSSPlain) return dispatch_field<PREC, kBoris, kCollHSSPlain>(field, mag, p, g, b, s);
        }
        return cudaErrorNotSupported;
    }
    if constexpr (WITH_RK4) {
        if (integ == kRK4) {
            if (coll == kCollNone) return dispatch_field<PREC, kRK4, kCollNone>(field, mag, p, g, b, s);
            if (coll == kCollHSS) return dispatch_field<PREC, kRK4, kCollHSS>(field, mag, p, g, b, s);
        }
    }
    return cudaErrorNotSupported;
}

}  // namespace icb
