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
  // stage 3 only, optional: the new state is also stored to these
  // (ld-strided) arrays, mapped pinned host memory of the caller
  double *host[3];
  int host_ld;
};

struct NlArgs {
  const double *su, *sv, *sh, *hb, *w0, *z0, *fc, *q;
  double *gx0, *gy0, *uh, *vh, *f;
  double mu0, mb0, g0;
};

struct TendArgs {
  const double *gx0, *gy0, *uh, *vh, *f;
  const double *fv = nullptr;  // [nf][6][ngf] face values of f, uh, vh, or null
};

struct LinArgs {
  const double *su, *sv, *sh;
  double g0, hh0;
};

// Several RK4 steps of the linear variant in one launch: sa carries dt, dt6,
// base (u0, updated in place), acc, flag and host_ld; bufa / bufb are the
// two stage buffers; host (optional) receives the final state; count is a
// device word for the grid barrier (zeroed by the launcher).
struct LinSteps {
  StageArgs sa;
  double *bufa[3];
  double *bufb[3];
  double *host[3];
  double g0, hh0;
  int nsteps;
  unsigned *count;
  // optional element order of the 16-lane tiles (order[t] = element of tile t,
  // -1 for none; norder entries): pairs the two elements of a warp by their
  // wall flag, so that a warp's halves take the same wall or interior branch
  const int *order = nullptr;
  int norder = 0;
};

// Tangent-linear quadrature-point stage: base state (su.., q) and perturbation
// (du, dv, dh, dq) in; perturbations of gx0, gy0, uh, vh, F out.
struct TlmArgs {
  const double *su, *sv, *sh, *hb, *w0, *z0, *fc, *q;
  const double *du, *dv, *dh, *dq;
  double *gx0, *gy0, *uh, *vh, *f;
  double mu0, mb0, g0;
};

// Adjoint of the tendency stage: adjoints (bu, bv, bh) of the tendencies in;
// adjoints of gx0, gy0, F (4 fields), uh, vh out; side-lift scratch lx, ly, lh
// (ne*3*ngf each).
struct AdjTendArgs {
  const double *bu, *bv, *bh;
  double *gx0b, *gy0b, *fb, *uhb, *vhb;
  double *lx, *ly, *lh;
};

// Adjoint of the quadrature-point stage: base state and the adjoints from the
// tendency stage in; adjoints of u, v, h (written) and q (4 fields) out.
struct AdjNlArgs {
  const double *su, *sv, *sh, *hb, *w0, *z0, *fc, *q;
  const double *fb, *gx0b, *gy0b, *uhb, *vhb;
  double *ub, *vb, *hbo, *qb;
  double mu0, mb0, g0;
};

// Adjoint of the q-phase: adjoint of q in; adjoints of u, v accumulated;
// side-lift scratch lq (4 * ne*3*ngf).
struct AdjQArgs {
  const double *qb;
  double *ub, *vb;
  double *lq;
};

// Adjoint of the linear variant.
struct AdjLinArgs {
  const double *bu, *bv, *bh;
  double *ub, *vb, *hbo;
  double *lx, *ly, *lh;
  double g0, hh0;
};

struct RhsBuffers {
  const double *su, *sv, *sh;          // stage input
  const double *hb, *w0, *z0, *fc;     // time-constant fields
  double *q, *f, *gx0, *gy0, *uh, *vh; // nonlinear intermediates
  // optional: [nf][6][ngf] face values of the tendency kernel's six fields
  // (computed once per face instead of once per side)
  double *fv = nullptr;
  double mu0, mb0, g0, hh0;
  // optional: recorded when sh is in place (the kernels that read sh wait
  // for it; the q-phase, which reads only su and sv, does not)
  cudaEvent_t sh_ready = nullptr;
};

cudaError_t launch_rhs(int variant, const DevOps &op, const DevMesh &m, const RhsBuffers &b,
                       const StageArgs &sa, cudaStream_t st, int sms, long long *launches,
                       cudaEvent_t *ev = nullptr);
// Single generic kernels (the tangent-linear model reuses them: the q-phase,
// the tendency kernel and the linear kernel are linear in their inputs).
cudaError_t launch_qphase(int variant, const DevOps &op, const DevMesh &m, const double *su,
                          const double *sv, double *q, cudaStream_t st, int sms);
cudaError_t launch_tend(int variant, const DevOps &op, const DevMesh &m, const TendArgs &ta,
                        const StageArgs &sa, cudaStream_t st, int sms);
cudaError_t launch_lin(const DevOps &op, const DevMesh &m, const LinArgs &la, const StageArgs &sa,
                       cudaStream_t st, int sms);


cudaError_t launch_energy(const DevOps &op, const DevMesh &m, const double *su, const double *sv,
                          const double *sh, const double *hb, double g0, double *terms,
                          double *out, cudaStream_t st, int sms, long long *launches);
cudaError_t launch_cfl(int ne, int nc, const int *in, const double *xg, const double *yg,
                       const double *hb, int nm, double g0, unsigned long long *out,
                       cudaStream_t st, int sms, long long *launches);

// Tangent-linear and adjoint kernels (spoc_adjoint.cu).
cudaError_t launch_nlvol_tlm(int variant, const DevOps &op, const DevMesh &m, const TlmArgs &a,
                             cudaStream_t st, int sms);
cudaError_t launch_adj_nl(int variant, const DevOps &op, const DevMesh &m, const AdjTendArgs &ta,
                          const AdjNlArgs &na, const AdjQArgs &qa, cudaStream_t st, int sms);
cudaError_t launch_adj_lin(const DevOps &op, const DevMesh &m, const AdjLinArgs &a,
                           cudaStream_t st, int sms);
cudaError_t launch_axpy(size_t n, const double *x, double c, const double *y, double *out,
                        cudaStream_t st, int sms);
cudaError_t launch_axpby(size_t n, double a, const double *x, double b, const double *y,
                         double *out, cudaStream_t st, int sms);
// Regridding (spoc_regrid.cu).  Scratch of the error indicator: amax_bits
// (3 ne), small_bits (4: mode-0 maxima of u, v, h, then the largest
// normalised jump), amax (3 ne, normalised), fconv / fderaff (ne, or null),
// deraff (1).
struct RegridScratch {
  unsigned long long *amax_bits, *small_bits;
  double *amax;
  int *fconv, *fderaff, *deraff;
};
cudaError_t launch_checkconv(const DevOps &op, const DevMesh &m, const double *su,
                             const double *sv, const double *sh, double fac1, double fac2,
                             RegridScratch s, cudaStream_t st, int sms, long long *launches);
cudaError_t launch_interpol(const DevOps &op, int ne_new, int src_ne, const int *tinter,
                            const int *pel, const double *px, const double *py,
                            const double *const src[3], double *const dst[3], int *flag,
                            cudaStream_t st, int sms, long long *launches);
cudaError_t launch_verif_rot(const DevOps &op, const DevMesh &m, double *u, double *v,
                             cudaStream_t st, int sms, long long *launches);
cudaError_t launch_cfl2(int ne, int nc, int nm, int n, double *pg, const int *in,
                        const double *xg, const double *yg, const double *hb, const double *u,
                        const double *v, double g0, unsigned long long *out, cudaStream_t st,
                        int sms, long long *launches);

cudaError_t launch_eval_points(int nc, int nm, int ne, int npts, const int *elem,
                               const double *px, const double *py, const double *const f[3],
                               double *out, int *flag, cudaStream_t st, int sms,
                               long long *launches);
cudaError_t launch_lattice(int ne, int nc, int nm, int n, double *pg, const int *in,
                           const double *xg, const double *yg, const double *const f[3],
                           double *out, cudaStream_t st, int sms, long long *launches);

// Adjoint RK4 bookkeeping over the three fields in one launch.  kInit:
// kb = a lam + b lam.  kFirst: acc = sb, kb = a sb + b lam.  kMid: acc += sb,
// kb = a sb + b lam.  kLast: lam += acc + sb.
struct AdjCombine {
  enum Mode { kInit = 0, kFirst = 1, kMid = 2, kLast = 3 };
  const double *sb[3];
  double *acc[3], *lam[3], *kb[3];
  double a, b;
  int mode;
};
cudaError_t launch_adj_combine(size_t n, const AdjCombine &c, cudaStream_t st, int sms);
cudaError_t launch_obs_eval(int nobs, int nm, const int *elem, const double *basis,
                            const double *h, double *val, cudaStream_t st);
cudaError_t launch_obs_adj(int nel, int nm, const int *el_list, const int *el_start,
                           const int *obs_of, const double *basis, const double *resid, double *hb,
                           cudaStream_t st);

// Compile-time-sized kernels (spoc_fast.cu) for the tabulated degree /
// quadrature combinations; identical results to launch_rhs.
bool fast_available(int nc, int ng, int ngf);
// Bytes of the operator images of the compile-time-sized kernels (which 0:
// q-phase / tendency / linear kernels, 1: quadrature-point kernel; 0 when the
// degree is not tabulated), and the kernel that writes them from op's tables.
size_t fast_image_bytes(int nc, int ng, int ngf, int which);
cudaError_t fast_build_images(const DevOps &op, void *img, void *imgq, cudaStream_t st);
cudaError_t launch_rhs_fast(int variant, const DevOps &op, const DevMesh &m, const RhsBuffers &b,
                            const StageArgs &sa, cudaStream_t st, int sms, long long *launches,
                            cudaEvent_t *ev = nullptr);

// The compile-time-sized q-phase alone (nonlinear variants, tabulated sizes;
// cudaErrorNotSupported otherwise); bit-identical to launch_qphase.
cudaError_t launch_qphase_fast(int variant, const DevOps &op, const DevMesh &m, const double *su,
                               const double *sv, double *q, cudaStream_t st, int sms);

// Several RK4 steps of the linear variant in one cooperative launch of the
// compile-time-sized kernel, bit-identical to one launch per stage; returns
// cudaErrorNotSupported (nothing launched) when the degree is not tabulated
// or the mesh needs more than one pass of the resident warps.
cudaError_t lin_steps_fast(const DevOps &op, const DevMesh &m, const LinSteps &ls, cudaStream_t st,
                           int sms, long long *launches);

// The same kernels with fused multiply-adds (spoc_fast.cu built with SPOC_FMA=1).
bool fast_available_fma(int nc, int ng, int ngf);
cudaError_t launch_rhs_fast_fma(int variant, const DevOps &op, const DevMesh &m,
                                const RhsBuffers &b, const StageArgs &sa, cudaStream_t st, int sms,
                                long long *launches, cudaEvent_t *ev = nullptr);
cudaError_t lin_steps_fast_fma(const DevOps &op, const DevMesh &m, const LinSteps &ls,
                               cudaStream_t st, int sms, long long *launches);

// 8 independent chains of `iters` multiply-adds per thread, sms*8 blocks of 256;
// mode 0 FP64 fused, 1 FP64 separately rounded, 2 FP32 fused
cudaError_t launch_fp64_peak(int mode, int sms, int iters, double *out, cudaStream_t st);

}  // namespace spoc
