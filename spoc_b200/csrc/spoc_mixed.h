// Mixed-precision form of the RK4 DG right-hand side (spoc_mixed.cu).
//
// The contractions run in FP32 in an orthonormal modal basis psi = U^-T phi
// (U the upper Cholesky factor of the mass matrix, amm = U^T U): there the
// mass matrix is the identity, so every mass solve of the reference becomes
// the identity and every wall solve (reduc_gn, amml solve, reduc_inv_gn)
// becomes an orthogonal projector.  The RK4 state and its accumulation stay in
// FP64 (psi coefficients); the conversions phi <-> psi (c = U a, a = U^-1 c)
// are FP64.  In the reference basis FP32 contractions are not usable: the
// mass solves amplify their rounding by up to cond(amm) (2e8 at degree 6).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/spoc_gpu.h"
#include "spoc_kernels.h"

namespace spoc {

struct MixedCtx;

bool mixed_available(int nc, int ng, int ngf);

// Builds the psi-basis operators from the COMMON-block tables and allocates
// the device buffers for ne elements.
int mixed_create(MixedCtx **out, const spoc_tables *t, int variant, int ne, int sms,
                 std::string *err);
void mixed_destroy(MixedCtx *c);

// Time-constant fields (device, packed (ne, nm), reference basis): hb, fc, w0,
// z0 are evaluated at the quadrature points once.
cudaError_t mixed_set_params(MixedCtx *c, const DevOps &op, const double *hb, const double *fc,
                             const double *w0, const double *z0, bool w0z0_zero, double mu0,
                             double mb0, double g0, double hh0, cudaStream_t st);

// State in the reference basis (device, packed) -> psi state, and back.
cudaError_t mixed_set_state(MixedCtx *c, const DevMesh &m, const double *const phi[3],
                            cudaStream_t st, long long *launches);
cudaError_t mixed_get_state(MixedCtx *c, double *const phi[3], cudaStream_t st,
                            long long *launches);

// nsteps RK4 steps of the resident psi state.  ev (optional, 4 events) marks
// the kernel boundaries of the first stage of the last step.
cudaError_t mixed_steps(MixedCtx *c, const DevMesh &m, double dt, int nsteps, int *flag,
                        cudaStream_t st, long long *launches, cudaEvent_t *ev = nullptr);

// One right-hand side: phi-basis input -> phi-basis tendency (device, packed).
// Leaves the resident state untouched.
cudaError_t mixed_rhs(MixedCtx *c, const DevMesh &m, const double *const in[3],
                      double *const out[3], int *flag, cudaStream_t st, long long *launches);

// Kernels per right-hand side (1 linear, 2 nonlinear).
int mixed_kernels_per_rhs(const MixedCtx *c);

// Nonlinear volume kernel on the tensor cores (tcgen05) or on the FP32 pipes;
// false if the tensor-core kernel is not available.
bool mixed_set_tensor(MixedCtx *c, bool on);
// back to the default family (FP32 pipes)
void mixed_default_path(MixedCtx *c);
bool mixed_uses_tensor(const MixedCtx *c);

// Ensemble of members (mixed precision, free-slip, degree 3-6) stepped
// together: one cooperative launch per RK4 stage for all members, optionally
// replayed from a CUDA graph.  Blocks are dealt to members in proportion to
// their work, modelled as ne nm^p with p = 2, 1, 0.5, 0 for weight 0..3, or
// measured (weight 4, mixed_ens_balance);
// bps resident blocks per SM.
struct MixedEns;
int mixed_ens_create(MixedEns **out, MixedCtx *const *ctx, const DevMesh *meshes,
                     int *const *flags, int n, int sms, std::string *err);
void mixed_ens_destroy(MixedEns *e);
int mixed_ens_configure(MixedEns *e, int bps, int weight);
void mixed_ens_info(const MixedEns *e, int *bps, int *max_bps, int *weight, int *blocks,
                    int *graph);
int mixed_ens_member_blocks(const MixedEns *e, int i);
cudaError_t mixed_ens_steps(MixedEns *e, const double *dt, int nsteps, bool use_graph);
// Measured work model: `rounds` steps (they advance the members), each with
// per-block cycle counters; after each, blocks are dealt again in proportion
// to every member's total block cycles (weight 4).
cudaError_t mixed_ens_balance(MixedEns *e, const double *dt, int rounds);

}  // namespace spoc
