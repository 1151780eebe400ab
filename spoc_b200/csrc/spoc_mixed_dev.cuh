// Device definitions shared by the mixed-precision kernels (spoc_mixed.cu,
// spoc_mixed_tc.cu): compile-time dimensions, kernel arguments, face
// references and the mean-free trace records.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/spoc_gpu.h"
#include "spoc_kernels.h"

namespace spoc {
namespace mx {

constexpr int kMxWarps = 8;  // warps (elements in flight) per block

template <int NC_, int Q_, int G_>
struct MDims {
  static constexpr int N = (NC_ + 1) * (NC_ + 2) / 2;
  static constexpr int Q = Q_;
  static constexpr int G = G_;
  static constexpr int TG = 3 * G_;
  static constexpr int TS = TG + 1;  // trace record: TG mean-free traces + the mean
  // lanes per element: 16 when the modes, the trace record and two passes
  // over the quadrature points fit (degrees 3 and 4: two elements per warp)
  static constexpr int LW = (N <= 16 && TS <= 16 && Q <= 32) ? 16 : 32;
  static constexpr int SLOTS = kMxWarps * 32 / LW;  // elements in flight per block
  static constexpr int R = (N + LW - 1) / LW;
  // resident blocks per SM the register budget is sized for (shared memory
  // allows about 4 blocks of 8 warps at degree <= 6 and 3 at degree 7; the
  // one-kernel linear variant keeps 2 at degree 7, where 3 would spill)
  static constexpr int MINB = R == 1 ? 4 : 3;
  static constexpr int MINB_LIN = R == 1 ? 4 : 2;
  // operator image in shared memory (floats)
  static constexpr int PPT = 0;               // [n*Q + q]  = Pp(q, n)
  static constexpr int PW = PPT + N * Q;      // [q*N + i]  = Pp(q, i) wi(q)
  static constexpr int GX = PW + Q * N;       // [k*N + i]  = GX(i, k)
  static constexpr int GY = GX + N * N;       // [k*N + i]  = GY(i, k)
  static constexpr int TRT = GY + N * N;      // [n*TG + l] = TR(l, n), l = s*G + j
  static constexpr int LIFT = TRT + N * TG;   // [l*N + i]  = TR(l, i)
  static constexpr int PWALL = LIFT + TG * N; // [k*N + i]  = Pwall(i, k)
  static constexpr int WIF = PWALL + N * N;   // [j] = wif(j)
  static constexpr int NOPS = (WIF + G + 3) / 4 * 4;
  // per-warp scratch (floats)
  static constexpr int S_U = 0, S_V = N, S_H = 2 * N;
  static constexpr int S_Q = 3 * N;           // qxx, qxy, qyx, qyy
  static constexpr int S_VEC = 7 * N;         // six combined vectors
  static constexpr int S_UH = 13 * N, S_VH = 14 * N, S_TMP = 15 * N;
  static constexpr int S_GL = 16 * N;         // 4 face vectors of TG
  static constexpr int S_QP = S_GL + 4 * TG;  // 7 quadrature vectors of Q
  static constexpr int WS = (S_QP + 7 * Q + 3) / 4 * 4;
  static_assert(TS <= LW, "face points of one element must fit its lanes");
  static_assert(Q <= 2 * LW, "two passes over the quadrature points at most");
  static_assert(N <= 64 && Q <= 64, "two rows per lane at most");
};

struct MxArgs {
  int ne;
  const float *ops;
  DevMesh m;
  const float *tr_in;  // [3][ne][TS] trace records of the stage input (u, v, h)
  float *tr_out;       // [3][ne][TS] trace records of the next stage input
  float *y;            // [3][ne][N] stage input (FP32); replaced by the next one
  float *part;         // [3][ne][N] partial load vectors (u, v, h)
  float *trq;          // [6][ne][TS] trace records of qxx, qxy, qyx, qyy, uh, vh
  const float *hbq, *fcq, *w0q, *z0q;  // [ne][Q]; w0q / z0q null when zero
  float mu0, mb0, g0, hh0;
  int stage;           // 0..3 RK4 stage; -1: write the tendency to k64
  double dt, dt6;
  double *c64, *acc, *k64;  // [3][ne][N] psi coefficients, FP64
  int *flag;                // bit 0: non-finite tendency; bit 1: tensor-core wait limit
  float psi0;               // value of the constant psi mode
  float wif[10];            // edge quadrature weights
};

__device__ __forceinline__ float fma32(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <class Dm>
__device__ void stage_mx_ops(float *s, const float *g) {
  const float4 *src = reinterpret_cast<const float4 *>(g);
  float4 *dst = reinterpret_cast<float4 *>(s);
  for (int i = threadIdx.x; i < Dm::NOPS / 4; i += blockDim.x) dst[i] = src[i];
}

// The face of side k of element e as element e sees it.
struct FaceRef {
  int f, nb, s2;
  float sig, nx, ny;  // sig = its * 0.5 (the tri_f factor); nx, ny = norm(., f)
  bool wall;
};

__device__ __forceinline__ FaceRef face_ref(const DevMesh &m, int e, int k) {
  FaceRef r;
  r.f = m.itm[3 * e + k];
  const int isg = m.its[3 * e + k];
  const int t1 = m.tseg[2 * r.f], t2 = m.tseg[2 * r.f + 1];
  r.nb = isg > 0 ? t2 : t1;
  r.s2 = isg > 0 ? m.ssit[2 * r.f + 1] : m.ssit[2 * r.f];
  r.wall = t2 < 0;
  r.sig = isg > 0 ? 0.5f : -0.5f;
  r.nx = (float)m.norm[2 * r.f];
  r.ny = (float)m.norm[2 * r.f + 1];
  return r;
}

// Trace records.  The weak derivative of a field F on an element,
// -int F dpsi/dx + sum_faces int psi F* n_x, is a small difference of two large
// terms when F has a large element mean m (Gauss's theorem makes the mean's two
// contributions cancel exactly).  In FP32 that cancellation loses up to three
// digits, so the mean is taken out of both terms: the volume contractions skip
// the constant mode (psi_0 = const) and the face terms use F* - m.  A trace
// record of an element holds, for each of its 3 x ngf face points, the trace
// of F - m, followed by m itself.
//
// cal_flu central value minus the own mean, on the face seen from side k,
// point j of element e: own trace and the neighbour's trace at the mirrored
// point (src/calflu.f:45-62); a wall face keeps the own trace
// (src/calflu.f:35-39).
template <int G>
__device__ __forceinline__ float face_value(const float *tr, const FaceRef &r, int e, int l, int j) {
  constexpr int TG = 3 * G, TS = TG + 1;
  const float own = tr[(size_t)e * TS + l];
  if (r.wall) return own;
  const float *nb = tr + (size_t)r.nb * TS;
  return 0.5f * (own + nb[r.s2 * G + (G - 1 - j)] + (nb[TG] - tr[(size_t)e * TS + TG]));
}

// RK4 bookkeeping of src/shwwnl.f:242-284 on one psi coefficient, FP64;
// returns the next stage input.
__device__ __forceinline__ double rk4_update(const MxArgs &a, size_t i, double d) {
  double *c = a.c64 + i, *acc = a.acc + i;
  const double u0 = *c;
  switch (a.stage) {
    case 0: *acc = d; return u0 + a.dt * d * 0.5;
    case 1: *acc = *acc + 2.0 * d; return u0 + a.dt * d * 0.5;
    case 2: *acc = *acc + 2.0 * d; return u0 + a.dt * d;
    default: {
      const double u1 = u0 + a.dt6 * (*acc + d);
      *c = u1;
      return u1;
    }
  }
}

}  // namespace mx

// psi-basis operators built on the host in FP64 (spoc_mixed.cu).
struct PsiOps {
  int N, Q, G;
  std::vector<double> U, Ui, Pp, GX, GY, TR, PWALL;
};

// Tensor-core volume kernel (spoc_mixed_tc.cu): operator image and launch.
bool mixed_tc_available(int nc, int ng, int ngf);
std::vector<float> mixed_tc_image(int nc, int ng, int ngf, const PsiOps &p, const double *wi);
cudaError_t mixed_tc_vol(int variant, int nc, int ng, int ngf, const mx::MxArgs &a, const float *img,
                         int sms, cudaStream_t st);
// The tendency kernel on the tensor cores (face lifts, wall projection, traces).
cudaError_t mixed_tc_tend(int variant, int nc, int ng, int ngf, const mx::MxArgs &a, const float *img,
                         int sms, cudaStream_t st);

}  // namespace spoc
