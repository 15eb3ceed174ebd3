// icb_step_mixed.cu — mixed-precision instantiations of the fused step
// kernel: float velocity, field and collision arithmetic (hardware sqrt,
// log, sin/cos), double position and time.  Built with -use_fast_math.
#include "icb_internal.h"
#include "icb_step_kernel.cuh"
#include "icb_step_dispatch.cuh"

namespace icb {
cudaError_t launch_step_mixed(int integ, int coll, int field, bool mag, const StepParams& p,
                              dim3 grid, dim3 block, cudaStream_t s) {
    return dispatch_step<kPrecMixed, true>(integ, coll, field, mag, p, grid, block, s);
}
}  // namespace icb
