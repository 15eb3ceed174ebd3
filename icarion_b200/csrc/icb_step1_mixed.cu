// icb_step1_mixed.cu — the per-step kernel (icb_step1.cuh) in the
// mixed form.  Built with -use_fast_math like the fused mixed kernel.
#include "icb_internal.h"
#include "icb_step1.cuh"

namespace icb {
cudaError_t launch_step1_mixed(int coll, const StepParams& p, cudaStream_t s) {
    return launch_step1<kPrecMixed>(coll, p, s);
}
}  // namespace icb
