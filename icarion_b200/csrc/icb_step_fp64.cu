// icb_step_fp64.cu — FP64 instantiations of the fused step kernel.
// Built with --fmad=false: no FMA contraction, so the collision-free push
// performs the reference's IEEE double operations in the reference's order.
#include "icb_internal.h"
#include "icb_step_kernel.cuh"
#include "icb_step_dispatch.cuh"

namespace icb {
cudaError_t launch_step_fp64(int integ, int coll, int field, bool mag, const StepParams& p,
                             dim3 grid, dim3 block, cudaStream_t s) {
    return dispatch_step<kPrecFP64, true>(integ, coll, field, mag, p, grid, block, s);
}
}  // namespace icb
