// icb_step_hilo.cu — the compensated float hi/lo position variant (Boris
// only): position = hi + lo with a TwoSum update (Knuth, TAOCP vol. 2,
// 4.2.2), velocity and collisions as in the mixed kernel.
#include "icb_internal.h"
#include "icb_step_kernel.cuh"
#include "icb_step_dispatch.cuh"

namespace icb {
cudaError_t launch_step_hilo(int integ, int coll, int field, bool mag, const StepParams& p,
                             dim3 grid, dim3 block, cudaStream_t s) {
    return dispatch_step<kPrecHiLo, false>(integ, coll, field, mag, p, grid, block, s);
}
}  // namespace icb
