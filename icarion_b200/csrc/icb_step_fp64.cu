// icb_step_fp64.cu — FP64 instantiations of the fused step kernel.
// Built with --fmad=false: no FMA contraction, so the collision-free push
// performs the reference's IEEE double operations in the reference's order.
#include "icb_internal.h"
#define ICB_TF_TABLE_UNIT
#include "icb_step_kernel.cuh"
#include "icb_step_dispatch.cuh"

namespace icb {
cudaError_t launch_step_fp64(int integ, int coll, int field, bool mag, const StepParams& p,
                             dim3 grid, dim3 block, cudaStream_t s) {
    return dispatch_step<kPrecFP64, true>(integ, coll, field, mag, p, grid, block, s);
}

cudaError_t launch_tf_table(const StepParams& p, double* tab, double* tseq, uint32_t stride, cudaStream_t s) {
    k_tf_table<<<p.n_ens, 128, 0, s>>>(p, tab, tseq, stride);
    return cudaGetLastError();
}
}  // namespace icb
