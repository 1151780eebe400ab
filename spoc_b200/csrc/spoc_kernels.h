// Launch interface between the C ABI (spoc_api.cu) and the kernels.
#pragma once
#include <cuda_runtime.h>

#include "spoc_device.cuh"

namespace spoc {

enum { kLIN = 0, kFS = 1, kNS = 2, kINV = 3 };

// RK4 stage bookkeeping (src/shwwnl.f:242-284).  stage < 0: write the
// tendency to `tend` (a plain cal_var call).  Fields are u, v, h.
struct StageArgs {
  int stage;
  double dt, dt6;
  double *base[3];  // u0, v0, h0 (updated in place at stage 3)
  double *out[3];   // next stage input
  double *acc[3];   // du1 + 2 du2 + 2 du3
  double *tend[3];  // tendency output when stage < 0
  int *flag;        // set non-zero on a non-finite tendency
};

struct NlArgs {
  const double *su, *sv, *sh, *hb, *w0, *z0, *fc, *q;
  double *gx0, *gy0, *uh, *vh, *f;
  double mu0, mb0, g0;
};

struct TendArgs {
  const double *gx0, *gy0, *uh, *vh, *f;
};

struct LinArgs {
  const double *su, *sv, *sh;
  double g0, hh0;
};

struct RhsBuffers {
  const double *su, *sv, *sh;          // stage input
  const double *hb, *w0, *z0, *fc;     // time-constant fields
  double *q, *f, *gx0, *gy0, *uh, *vh; // nonlinear intermediates
  double mu0, mb0, g0, hh0;
};

cudaError_t launch_rhs(int variant, const DevOps &op, const DevMesh &m, const RhsBuffers &b,
                       const StageArgs &sa, cudaStream_t st, int sms, long long *launches,
                       cudaEvent_t *ev = nullptr);
cudaError_t launch_energy(const DevOps &op, const DevMesh &m, const double *su, const double *sv,
                          const double *sh, const double *hb, double g0, double *terms,
                          double *out, cudaStream_t st, int sms, long long *launches);
cudaError_t launch_cfl(int ne, int nc, const int *in, const double *xg, const double *yg,
                       const double *hb, int nm, double g0, unsigned long long *out,
                       cudaStream_t st, int sms, long long *launches);

// Compile-time-sized kernels (spoc_fast.cu) for the tabulated degree /
// quadrature combinations; identical results to launch_rhs.
bool fast_available(int nc, int ng, int ngf);
cudaError_t launch_rhs_fast(int variant, const DevOps &op, const DevMesh &m, const RhsBuffers &b,
                            const StageArgs &sa, cudaStream_t st, int sms, long long *launches,
                            cudaEvent_t *ev = nullptr);

// The same kernels with fused multiply-adds (spoc_fast.cu built with SPOC_FMA=1).
bool fast_available_fma(int nc, int ng, int ngf);
cudaError_t launch_rhs_fast_fma(int variant, const DevOps &op, const DevMesh &m,
                                const RhsBuffers &b, const StageArgs &sa, cudaStream_t st, int sms,
                                long long *launches, cudaEvent_t *ev = nullptr);

// 8 independent chains of `iters` FP64 operations per thread, sms*8 blocks of 256
cudaError_t launch_fp64_peak(int mode, int sms, int iters, double *out, cudaStream_t st);

}  // namespace spoc
