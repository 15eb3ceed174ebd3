// icb_step1_hilo.cu — the per-step kernel (icb_step1.cuh) in the
// hi/lo form.  Built with -use_fast_math like the fused hi/lo kernel.
#include "icb_internal.h"
#include "icb_step1.cuh"

namespace icb {
cudaError_t launch_step1_hilo(int coll, const StepParams& p, cudaStream_t s) {
    return launch_step1<kPrecHiLo>(coll, p, s);
}
}  // namespace icb
