// icb_step1_fp64.cu — the per-step kernel (icb_step1.cuh) in the
// FP64 form.  Built with --fmad=false like the fused FP64 kernel (bit-faithful IEEE double push).
#include "icb_internal.h"
#include "icb_step1.cuh"

namespace icb {
cudaError_t launch_step1_fp64(int coll, const StepParams& p, cudaStream_t s) {
    return launch_step1<kPrecFP64>(coll, p, s);
}
}  // namespace icb
