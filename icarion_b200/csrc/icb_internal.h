// icb_internal.h — host-side declarations shared by the library's .cu files.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/icarion_b200.h"
#include "icb_params.h"

namespace icb {

// Kernel launchers, one per precision translation unit.  Each returns the
// launch's cudaError_t (cudaErrorNotSupported for an absent combination).
// Per-step time-only field scalars of one launch (tf_tab of StepParams).
cudaError_t launch_tf_table(const StepParams& p, double* tab, double* tseq, uint32_t stride, cudaStream_t s);
cudaError_t launch_step_fp64(int integ, int coll, int field, bool mag, const StepParams& p,
                             dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_step_mixed(int integ, int coll, int field, bool mag, const StepParams& p,
                              dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_step_hilo(int integ, int coll, int field, bool mag, const StepParams& p,
                             dim3 grid, dim3 block, cudaStream_t s);
// The per-step kernel (icb_step1.cuh) of each precision: coll kCollNone or
// kCollHSS; a persistent grid over the launch's tiles of its own shape.
cudaError_t launch_step1_fp64(int coll, const StepParams& p, cudaStream_t s);
cudaError_t launch_step1_mixed(int coll, const StepParams& p, cudaStream_t s);
cudaError_t launch_step1_hilo(int coll, const StepParams& p, cudaStream_t s);

// Space-charge solver (icb_p3m.cu).  Functions return ICB_* status codes
// and put a message into `err` on failure.
struct SpaceChargeSolver;
int sc_create(const icb_spacecharge_config& cfg, uint64_t n_ions, bool pp_float, cudaStream_t s,
              SpaceChargeSolver** out, std::string& err);
void sc_destroy(SpaceChargeSolver* sc);
int sc_solve(SpaceChargeSolver* sc, const double* x, const double* y, const double* z, const double* q,
             const uint8_t* flags, uint64_t n, cudaStream_t s, std::string& err);
const double* sc_field(const SpaceChargeSolver* sc, int axis);
int sc_set_peers(SpaceChargeSolver* sc, const double* xyzq, uint64_t n, uint64_t skip_b, uint64_t skip_n,
                 cudaStream_t s, std::string& err);
int sc_export(const double* x, const double* y, const double* z, const double* q, const uint8_t* flags, uint64_t n,
              double* out, cudaStream_t s, std::string& err);
int sc_kernel_count(const SpaceChargeSolver* sc);

// Interaction-potential physics (icb_ipm.cu).
int ipm_potential_from(const icb_ipm_potential& p, IpmPotential& P, std::string& err);
// Device Gauss-Legendre nodes of the deflection quadrature (one copy per
// device, made on first use).
struct GLNodes;
int ipm_gl_nodes(int device, const GLNodes** out, std::string& err);
int ipm_build_table(int device, const IpmPotential& P, int nE, int nb, double Emin, double Emax, double bmax,
                    float* dev_table, cudaStream_t s, std::string& err);

// Learned deflection (icb_mlp.cu): the collision path's parameter blocks.
void mlp_pack(const float* params, std::vector<uint32_t>& frag, std::vector<float>& fblock);

// Records the message icb_last_error() returns on this host thread and
// passes `code` through.
int set_error(int code, const char* msg);

}  // namespace icb
