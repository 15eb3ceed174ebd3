// icb_internal.h — host-side declarations shared by the library's .cu files.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "icb_params.h"

namespace icb {

// Kernel launchers, one per precision translation unit.  Each returns the
// launch's cudaError_t (cudaErrorNotSupported for an absent combination).
cudaError_t launch_step_fp64(int integ, int coll, int field, bool mag, const StepParams& p,
                             dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_step_mixed(int integ, int coll, int field, bool mag, const StepParams& p,
                              dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_step_hilo(int integ, int coll, int field, bool mag, const StepParams& p,
                             dim3 grid, dim3 block, cudaStream_t s);

// Records the message icb_last_error() returns on this host thread and
// passes `code` through.
int set_error(int code, const char* msg);

}  // namespace icb
