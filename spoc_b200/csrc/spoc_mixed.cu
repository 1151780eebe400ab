// Mixed-precision form of the RK4 DG shallow-water right-hand side.
//
// Basis.  The reference expands each field in phi = P_k1(x) P_k2(y) (mode
// order of src/mat1.f) and solves with the Cholesky factor U of the mass
// matrix amm = U^T U (src/shwwnl.f:153-156, DTRSM4 src/dtrsm1.f:47-82).  Here
// the contractions use psi = U^-T phi, which is orthonormal on the reference
// triangle.  With c = U a the psi coefficients of a field and b_psi = U^-T b
// the psi load vector of a load vector b:
//   * a mass solve a = amm^-1 b becomes c = b_psi (no work);
//   * cal_b (b += coeff agx^T a, src/calb2.f:3-24) becomes b_psi += coeff GX c
//     with GX = U^-T agx^T U^-1 (likewise GY);
//   * spectoxy / xytospec (src/nonlin.f:35-107) become Pp = pi2 U^-1 and
//     Pp^T diag(wi);
//   * the face trace of cal_flu (src/calflu.f:6-71) and the lift of tri_f
//     (src/mat1.f:172-209) become TR_s = pico(.,.,s) U^-1 and TR_s^T;
//   * the wall solve reduc_gn -> amml solve -> reduc_inv_gn
//     (src/mat1.f:418-473, amml = R^T amm R with R the map of reduc_inv_gn)
//     becomes the orthogonal projector onto span(U R).
// All of these are well conditioned, so FP32 contractions keep FP32 accuracy;
// in the reference basis the mass solves amplify contraction rounding by up to
// cond(amm) (2.1e8 at degree 6).  The RK4 state (psi coefficients) and its
// accumulation stay FP64 (src/shwwnl.f:242-284); the conversions between the
// bases are FP64.
//
// Kernels (one warp per element, lanes over modes, quadrature points or the
// 3*ngf face points; operators staged in shared memory per persistent block):
//   kx_vol<VAR>  nonlinear variants, phases A, B and the volume parts of C, D
//                of calvarnl_*.f (q, quadrature products, F and h volume
//                terms), writing partial load vectors and the face traces of
//                q, uh, vh;
//   kx_tend<VAR> face lifts of phases C, D, wall projections, RK4 update in
//                FP64, and the face traces of the next stage input;
//   kx_lin       calvar_lin.f in one kernel.
// Face values are the central averages of cal_flu, formed from traces that
// each element writes for its own three sides (no face arrays).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "spoc_launch.h"
#include "spoc_mixed.h"
#include "spoc_mixed_dev.cuh"

namespace spoc {
using namespace mx;

namespace {

// The lanes of this thread's element (all 32, or its half of the warp).
template <class Dm>
__device__ __forceinline__ unsigned lane_mask() {
  return Dm::LW == 32 ? 0xffffffffu : (0xffffu << (threadIdx.x & 16));
}

// f(k, v) for k = k0..L-1 in order, v[c] = x[c][k] for NX shared vectors of
// length L.  The entries are read W = 4 or 2 at a time (16- or 8-byte
// broadcast loads) when W divides L; every x[c] must then be W-aligned.  The
// arithmetic f does, and its order, do not depend on W.
template <int L, int NX, class F>
__device__ __forceinline__ void sweep(int k0, const float *const (&x)[NX], F &&f) {
  constexpr int W = L % 4 == 0 ? 4 : (L % 2 == 0 ? 2 : 1);
  const int kp = (k0 + W - 1) / W * W;
  for (int k = k0; k < kp && k < L; ++k) {
    float v[NX];
#pragma unroll
    for (int c = 0; c < NX; ++c) v[c] = x[c][k];
    f(k, v);
  }
#pragma unroll 1
  for (int k = kp; k < L; k += W) {
    float v[W][NX];
#pragma unroll
    for (int c = 0; c < NX; ++c) {
      if constexpr (W == 4) {
        const float4 t = *reinterpret_cast<const float4 *>(x[c] + k);
        v[0][c] = t.x;
        v[1][c] = t.y;
        v[2][c] = t.z;
        v[3][c] = t.w;
      } else if constexpr (W == 2) {
        const float2 t = *reinterpret_cast<const float2 *>(x[c] + k);
        v[0][c] = t.x;
        v[1][c] = t.y;
      } else {
        v[0][c] = x[c][k];
      }
    }
#pragma unroll
    for (int j = 0; j < W; ++j) f(k + j, v[j]);
  }
}

// Trace record (mean-free traces, then the mean) of up to six fields held in
// the warp's shared vectors x[f] (psi coefficients); written by lanes 0..TG.
template <class Dm, int NF>
__device__ __forceinline__ void write_traces(const float *o, const float *const (&x)[NF], float *out,
                                             size_t stride, int e) {
  constexpr int N = Dm::N, TG = Dm::TG, TS = Dm::TS;
  const int lane = threadIdx.x & (Dm::LW - 1);
  if (lane > TG) return;
  float t[NF];
  if (lane < TG) {
#pragma unroll
    for (int f = 0; f < NF; ++f) t[f] = 0.f;
#pragma unroll 4
    for (int n = 1; n < N; ++n) {
      const float p = o[Dm::TRT + n * TG + lane];
#pragma unroll
      for (int f = 0; f < NF; ++f) t[f] = fma32(p, x[f][n], t[f]);
    }
  } else {
    const float p0 = o[Dm::TRT];  // psi_0, the constant mode's value
#pragma unroll
    for (int f = 0; f < NF; ++f) t[f] = p0 * x[f][0];
  }
  const size_t off = (size_t)e * TS + lane;
#pragma unroll
  for (int f = 0; f < NF; ++f) out[f * stride + off] = t[f];
}

// Orthogonal projection of the warp's vector x (shared, length N) onto the
// wall-compatible subspace; lanes receive rows i = lane + LW r (LW = lanes per element).
template <class Dm>
__device__ __forceinline__ void project_rows(const float *o, const float *x, float (&out)[Dm::R]) {
  constexpr int N = Dm::N;
  const int lane = threadIdx.x & (Dm::LW - 1);
#pragma unroll
  for (int r = 0; r < Dm::R; ++r) {
    const int i = lane + Dm::LW * r;
    float a = 0.f;
    if (i < N) {
#pragma unroll 4
      for (int k = 0; k < N; ++k) a = fma32(o[Dm::PWALL + k * N + i], x[k], a);
    }
    out[r] = a;
  }
}

// Wall solves of a vector tendency (gx, gy) in the psi basis.
//  no-slip (calvarnl_ns.f:404-421): both components projected;
//  free-slip / inviscid / linear (wall_solve_rot): normal component
//  gn = nx gx + ny gy projected, tangential one untouched.
template <class Dm, bool NOSLIP>
__device__ void wall_vec(const float *o, float *tmp, float (&gx)[Dm::R], float (&gy)[Dm::R],
                         float nx, float ny) {
  constexpr int N = Dm::N;
  const int lane = threadIdx.x & (Dm::LW - 1);
  if (NOSLIP) {
    float px[Dm::R], py[Dm::R];
#pragma unroll
    for (int r = 0; r < Dm::R; ++r)
      if (lane + Dm::LW * r < N) tmp[lane + Dm::LW * r] = gx[r];
    __syncwarp(lane_mask<Dm>());
    project_rows<Dm>(o, tmp, px);
    __syncwarp(lane_mask<Dm>());
#pragma unroll
    for (int r = 0; r < Dm::R; ++r)
      if (lane + Dm::LW * r < N) tmp[lane + Dm::LW * r] = gy[r];
    __syncwarp(lane_mask<Dm>());
    project_rows<Dm>(o, tmp, py);
    __syncwarp(lane_mask<Dm>());
#pragma unroll
    for (int r = 0; r < Dm::R; ++r) {
      gx[r] = px[r];
      gy[r] = py[r];
    }
  } else {
    float gn[Dm::R], pg[Dm::R];
#pragma unroll
    for (int r = 0; r < Dm::R; ++r) {
      gn[r] = nx * gx[r] + ny * gy[r];
      if (lane + Dm::LW * r < N) tmp[lane + Dm::LW * r] = gn[r];
    }
    __syncwarp(lane_mask<Dm>());
    project_rows<Dm>(o, tmp, pg);
    __syncwarp(lane_mask<Dm>());
#pragma unroll
    for (int r = 0; r < Dm::R; ++r) {
      const float d = pg[r] - gn[r];
      gx[r] += nx * d;
      gy[r] += ny * d;
    }
  }
}

// Finishes an element: non-finite check, RK4 update (or tendency output),
// next stage input and its traces.  t[3][R] holds the psi tendencies.
template <class Dm>
__device__ void finish_element(const MxArgs &a, const float *o, float *w, int e,
                               float (&t)[3][Dm::R]) {
  constexpr int N = Dm::N;
  const int lane = threadIdx.x & (Dm::LW - 1);
  const size_t fn = (size_t)a.ne * N;
  bool bad = false;
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int r = 0; r < Dm::R; ++r) {
      const int i = lane + Dm::LW * r;
      if (i >= N) continue;
      const float d = t[f][r];
      bad |= !isfinite(d);
      const size_t gi = f * fn + (size_t)e * N + i;
      if (a.stage < 0) {
        a.k64[gi] = (double)d;
      } else {
        const double yn = rk4_update(a, gi, (double)d);
        const float y32 = (float)yn;
        a.y[gi] = y32;
        w[f * N + i] = y32;
      }
    }
  if (__any_sync(lane_mask<Dm>(), bad) && lane == 0) atomicOr(a.flag, 1);
  if (a.stage < 0) return;
  __syncwarp(lane_mask<Dm>());
  const float *const x[3] = {w, w + N, w + 2 * N};
  write_traces<Dm, 3>(o, x, a.tr_out, (size_t)a.ne * Dm::TS, e);
  __syncwarp(lane_mask<Dm>());
}

// ---------------------------------------------------------------------------
// Nonlinear variants: volume kernel (calvarnl_fs.f:88-332 and the volume terms
// of :341-544).
// Body shared by kx_vol and the ensemble kernel: block blk of nblk working
// on the elements of one member; the operators are already in sm.
template <class Dm, int VAR>
__device__ __forceinline__ void vol_body(const MxArgs &a, float *sm, int blk, int nblk) {
  constexpr int N = Dm::N, Q = Dm::Q, G = Dm::G, TG = Dm::TG, R = Dm::R;
  float *o = sm;
  const int lane = threadIdx.x & (Dm::LW - 1), wib = threadIdx.x / Dm::LW;
  float *w = sm + Dm::NOPS + wib * Dm::WS;
  float *su = w + Dm::S_U, *sv = w + Dm::S_V, *sh = w + Dm::S_H, *sq = w + Dm::S_Q;
  float *vec = w + Dm::S_VEC, *suh = w + Dm::S_UH, *svh = w + Dm::S_VH, *tmp = w + Dm::S_TMP;
  float *gl = w + Dm::S_GL, *qp = w + Dm::S_QP;
  const size_t fn = (size_t)a.ne * N, tn = (size_t)a.ne * Dm::TS;
  const int stride = nblk * Dm::SLOTS;
  for (int e = blk * Dm::SLOTS + wib; e < a.ne; e += stride) {
    const double *vp = a.m.vect + 5 * (size_t)e;
    const float ax = (float)vp[0], bx = (float)vp[1], ay = (float)vp[2], by = (float)vp[3],
                di = (float)vp[4];
    for (int i = lane; i < N; i += Dm::LW) {
      const size_t gi = (size_t)e * N + i;
      su[i] = a.y[gi];
      sv[i] = a.y[fn + gi];
      sh[i] = a.y[2 * fn + gi];
    }
    // face values of u and v, as lift inputs of the four q components
    if (lane < TG) {
      const int k = lane / G, j = lane - k * G;
      const FaceRef r = face_ref(a.m, e, k);
      const float fu = face_value<G>(a.tr_in, r, e, lane, j);
      const float fv = face_value<G>(a.tr_in + tn, r, e, lane, j);
      const float s = r.sig * di * o[Dm::WIF + (r.sig > 0.f ? j : G - 1 - j)];
      gl[lane] = s * r.nx * fu;
      gl[TG + lane] = s * r.ny * fu;
      gl[2 * TG + lane] = s * r.nx * fv;
      gl[3 * TG + lane] = s * r.ny * fv;
    }
    __syncwarp(lane_mask<Dm>());
    // u, v, h + hb at the quadrature points (spectoxy); points past the
    // element's last lane run as (field, point) chains spread over the lanes
    if (lane < Q) {
      const int q = lane;
      float U = 0.f, V = 0.f, H = 0.f;
      const float *const x3[3] = {su, sv, sh};
      sweep<N, 3>(0, x3, [&](int n, const float (&v)[3]) {
        const float p = o[Dm::PPT + n * Q + q];
        U = fma32(p, v[0], U);
        V = fma32(p, v[1], V);
        H = fma32(p, v[2], H);
      });
      qp[q] = U;
      qp[Q + q] = V;
      qp[2 * Q + q] = H + a.hbq[(size_t)e * Q + q];
    }
    if (Q > Dm::LW) {
      constexpr int T = Q > Dm::LW ? Q - Dm::LW : 1;
      for (int c = lane; c < 3 * T; c += Dm::LW) {
        const int f = c / T, q = Dm::LW + c - f * T;
        const float *const x1[1] = {f == 0 ? su : (f == 1 ? sv : sh)};
        float acc = 0.f;
        sweep<N, 1>(0, x1, [&](int n, const float (&v)[1]) {
          acc = fma32(o[Dm::PPT + n * Q + q], v[0], acc);
        });
        qp[f * Q + q] = f == 2 ? acc + a.hbq[(size_t)e * Q + q] : acc;
      }
    }
    // q = weak gradients of u, v (calvarnl_fs.f:115-164): cal_b with coeff -1,
    // geometry, then tri_f of the traces; the mass solve is the identity
    // Rows past the last lane (degree 7: 4 of 36) would cost every row loop a
    // second pass with a few lanes busy: their (output, row) chains are spread
    // over the lanes instead, each summed in the same order.
    constexpr int RL = R == 2 ? 1 : R;  // rows computed lane by lane
    constexpr int T2 = R == 2 ? N - Dm::LW : 1;
    static_assert(R == 1 || (8 * T2 <= 4 * Q && 4 * T2 <= N && 3 * T2 <= Dm::LW), "row tail");
    float qv[4][R];
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int i = lane + Dm::LW * r;
      float gxu = 0.f, gyu = 0.f, gxv = 0.f, gyv = 0.f;
      float l0 = 0.f, l1 = 0.f, l2 = 0.f, l3 = 0.f;
      if (i < N) {
        const float *const x2[2] = {su, sv};
        sweep<N, 2>(1, x2, [&](int k, const float (&v)[2]) {  // constant mode: see the trace records
          const float cx = o[Dm::GX + k * N + i], cy = o[Dm::GY + k * N + i];
          gxu = fma32(cx, v[0], gxu);
          gyu = fma32(cy, v[0], gyu);
          gxv = fma32(cx, v[1], gxv);
          gyv = fma32(cy, v[1], gyv);
        });
#pragma unroll
        for (int l = 0; l < TG; ++l) {
          const float L = o[Dm::LIFT + l * N + i];
          l0 = fma32(L, gl[l], l0);
          l1 = fma32(L, gl[TG + l], l1);
          l2 = fma32(L, gl[2 * TG + l], l2);
          l3 = fma32(L, gl[3 * TG + l], l3);
        }
      }
      qv[0][r] = (ay * gyu - by * gxu) * di + l0;
      qv[1][r] = (bx * gxu - ax * gyu) * di + l1;
      qv[2][r] = (ay * gyv - by * gxv) * di + l2;
      qv[3][r] = (bx * gxv - ax * gyv) * di + l3;
    }
    if constexpr (R == 2) {
      // chains c = out * T2 + t: out 0-3 the cal_b sums, 4-7 the lift sums of
      // row LW + t, parked in the free qp slots of the products
      float *cs = qp + 3 * Q;
      for (int c = lane; c < 8 * T2; c += Dm::LW) {
        const int out = c / T2, i = Dm::LW + c - out * T2;
        float acc = 0.f;
        if (out < 4) {
          const int op = (out & 1) ? Dm::GY : Dm::GX;
          const float *const x1[1] = {out < 2 ? su : sv};
          sweep<N, 1>(1, x1, [&](int k, const float (&v)[1]) { acc = fma32(o[op + k * N + i], v[0], acc); });
        } else {
          const float *g = gl + (out - 4) * TG;
#pragma unroll 9
          for (int l = 0; l < TG; ++l) acc = fma32(o[Dm::LIFT + l * N + i], g[l], acc);
        }
        cs[c] = acc;
      }
      __syncwarp(lane_mask<Dm>());
      const bool own = lane < T2;
      const float gxu = own ? cs[lane] : 0.f, gyu = own ? cs[T2 + lane] : 0.f;
      const float gxv = own ? cs[2 * T2 + lane] : 0.f, gyv = own ? cs[3 * T2 + lane] : 0.f;
      const float l0 = own ? cs[4 * T2 + lane] : 0.f, l1 = own ? cs[5 * T2 + lane] : 0.f;
      const float l2 = own ? cs[6 * T2 + lane] : 0.f, l3 = own ? cs[7 * T2 + lane] : 0.f;
      qv[0][R - 1] = (ay * gyu - by * gxu) * di + l0;
      qv[1][R - 1] = (bx * gxu - ax * gyu) * di + l1;
      qv[2][R - 1] = (ay * gyv - by * gxv) * di + l2;
      qv[3][R - 1] = (bx * gxv - ax * gyv) * di + l3;
      __syncwarp(lane_mask<Dm>());
    }
    if (VAR == SPOC_FS && a.m.bdl[e]) {
      // calvarnl_fs.f:165-205: of the rotated tensor only the tangential-normal
      // component gtn is solved in the wall sub-basis
      const float nx = (float)a.m.normt[2 * (size_t)e], ny = (float)a.m.normt[2 * (size_t)e + 1];
      float gtn[R], pg[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        gtn[r] = nx * ny * qv[0][r] - nx * nx * qv[2][r] + ny * ny * qv[1][r] - nx * ny * qv[3][r];
        if (lane + Dm::LW * r < N) tmp[lane + Dm::LW * r] = gtn[r];
      }
      __syncwarp(lane_mask<Dm>());
      project_rows<Dm>(o, tmp, pg);
      __syncwarp(lane_mask<Dm>());
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float d = pg[r] - gtn[r];
        qv[0][r] += d * nx * ny;
        qv[2][r] -= d * nx * nx;
        qv[1][r] += d * ny * ny;
        qv[3][r] -= d * nx * ny;
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + Dm::LW * r;
      if (i < N)
#pragma unroll
        for (int c = 0; c < 4; ++c) sq[c * N + i] = qv[c][r];
    }
    __syncwarp(lane_mask<Dm>());
    // quadrature-point products (calvarnl_fs.f:243-332); xytospec is linear,
    // so the four projections of -adu + w1, -adv + z1, uh, vh take combined
    // integrands
    auto qproducts = [&](int q, float gxx, float gxy, float gyx, float gyy) {
      const float fc = a.fcq[(size_t)e * Q + q];
      gxy -= fc;
      gyx += fc;
      const float U = qp[q], V = qp[Q + q], H = qp[2 * Q + q];
      float wk = -a.mb0 * U, zk = -a.mb0 * V;
      if (a.w0q) {
        wk += a.w0q[(size_t)e * Q + q];
        zk += a.z0q[(size_t)e * Q + q];
      }
      qp[3 * Q + q] = wk / H - (U * gxx + V * gxy);
      qp[4 * Q + q] = zk / H - (U * gyx + V * gyy);
      qp[5 * Q + q] = U * H;
      qp[6 * Q + q] = V * H;
    };
    if (lane < Q) {
      const int q = lane;
      float gxx = 0.f, gxy = 0.f, gyx = 0.f, gyy = 0.f;
      const float *const x4[4] = {sq, sq + N, sq + 2 * N, sq + 3 * N};
      sweep<N, 4>(0, x4, [&](int n, const float (&v)[4]) {
        const float p = o[Dm::PPT + n * Q + q];
        gxx = fma32(p, v[0], gxx);
        gxy = fma32(p, v[1], gxy);
        gyx = fma32(p, v[2], gyx);
        gyy = fma32(p, v[3], gyy);
      });
      qproducts(q, gxx, gxy, gyx, gyy);
    }
    if (Q > Dm::LW) {
      // the four gradient values at points past the last lane as spread
      // chains, parked in the qp slots their products overwrite
      constexpr int T = Q > Dm::LW ? Q - Dm::LW : 1;
      __syncwarp(lane_mask<Dm>());
      for (int c = lane; c < 4 * T; c += Dm::LW) {
        const int f = c / T, q = Dm::LW + c - f * T;
        float acc = 0.f;
        const float *const x1[1] = {sq + f * N};
        sweep<N, 1>(0, x1, [&](int n, const float (&v)[1]) {
          acc = fma32(o[Dm::PPT + n * Q + q], v[0], acc);
        });
        qp[(3 + f) * Q + q] = acc;
      }
      __syncwarp(lane_mask<Dm>());
      if (lane < T) {
        const int q = Dm::LW + lane;
        qproducts(q, qp[3 * Q + q], qp[4 * Q + q], qp[5 * Q + q], qp[6 * Q + q]);
      }
    }
    __syncwarp(lane_mask<Dm>());
    float bxr[R], byr[R], uh[R], vh[R];
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int i = lane + Dm::LW * r;
      float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
      if (i < N) {
        const float *const x4[4] = {qp + 3 * Q, qp + 4 * Q, qp + 5 * Q, qp + 6 * Q};
        sweep<Q, 4>(0, x4, [&](int q, const float (&v)[4]) {
          const float p = o[Dm::PW + q * N + i];
          s0 = fma32(p, v[0], s0);
          s1 = fma32(p, v[1], s1);
          s2 = fma32(p, v[2], s2);
          s3 = fma32(p, v[3], s3);
        });
      }
      bxr[r] = s0;
      byr[r] = s1;
      uh[r] = s2;
      vh[r] = s3;
    }
    if constexpr (R == 2) {
      // the 4 T2 projections of the rows past the last lane as spread chains
      for (int c = lane; c < 4 * T2; c += Dm::LW) {
        const int out = c / T2, i = Dm::LW + c - out * T2;
        float acc = 0.f;
        const float *const x1[1] = {qp + (3 + out) * Q};
        sweep<Q, 1>(0, x1, [&](int q, const float (&v)[1]) { acc = fma32(o[Dm::PW + q * N + i], v[0], acc); });
        tmp[c] = acc;
      }
      __syncwarp(lane_mask<Dm>());
      const bool own = lane < T2;
      bxr[R - 1] = own ? tmp[lane] : 0.f;
      byr[R - 1] = own ? tmp[T2 + lane] : 0.f;
      uh[R - 1] = own ? tmp[2 * T2 + lane] : 0.f;
      vh[R - 1] = own ? tmp[3 * T2 + lane] : 0.f;
      __syncwarp(lane_mask<Dm>());
    }
    if (a.m.bdl[e]) {
      // uh, vh wall solves (calvarnl_fs.f:333-340, calvarnl_ns.f:249-265)
      const float nx = (float)a.m.normt[2 * (size_t)e], ny = (float)a.m.normt[2 * (size_t)e + 1];
      wall_vec<Dm, VAR == SPOC_NS>(o, tmp, uh, vh, nx, ny);
    }
    // combined vectors of the cal_b chains: F = mu0 q - g0 h (phase C) and
    // uh, vh (phase D)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + Dm::LW * r;
      if (i >= N) continue;
      const float hh = sh[i];
      const float fxx = a.mu0 * sq[i] - a.g0 * hh, fxy = a.mu0 * sq[N + i];
      const float fyx = a.mu0 * sq[2 * N + i], fyy = a.mu0 * sq[3 * N + i] - a.g0 * hh;
      vec[i] = di * (bx * fxy - by * fxx);
      vec[N + i] = di * (ay * fxx - ax * fxy);
      vec[2 * N + i] = di * (bx * fyy - by * fyx);
      vec[3 * N + i] = di * (ay * fyx - ax * fyy);
      vec[4 * N + i] = di * (by * uh[r] - bx * vh[r]);
      vec[5 * N + i] = di * (ax * vh[r] - ay * uh[r]);
      suh[i] = uh[r];
      svh[i] = vh[r];
    }
    __syncwarp(lane_mask<Dm>());
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int i = lane + Dm::LW * r;
      if (i >= N) continue;
      float gx = bxr[r], gy = byr[r], hp = 0.f;
      const float *const x6[6] = {vec, vec + N, vec + 2 * N, vec + 3 * N, vec + 4 * N, vec + 5 * N};
      sweep<N, 6>(1, x6, [&](int k, const float (&v)[6]) {  // constant mode: see the trace records
        const float cx = o[Dm::GX + k * N + i], cy = o[Dm::GY + k * N + i];
        gx = fma32(cx, v[0], gx);
        gx = fma32(cy, v[1], gx);
        gy = fma32(cx, v[2], gy);
        gy = fma32(cy, v[3], gy);
        hp = fma32(cx, v[4], hp);
        hp = fma32(cy, v[5], hp);
      });
      const size_t gi = (size_t)e * N + i;
      a.part[gi] = gx;
      a.part[fn + gi] = gy;
      a.part[2 * fn + gi] = hp;
    }
    if constexpr (R == 2) {
      // gx, gy, hp of the rows past the last lane: chains c = out * T2 + t,
      // started from row LW + t's bxr / byr (held by lane t)
      const int out = lane / T2, t = lane - out * T2;
      const float b0 = __shfl_sync(lane_mask<Dm>(), bxr[R - 1], t);
      const float b1 = __shfl_sync(lane_mask<Dm>(), byr[R - 1], t);
      if (lane < 3 * T2) {
        const int i = Dm::LW + t;
        float acc = out == 0 ? b0 : (out == 1 ? b1 : 0.f);
        const float *const x2[2] = {vec + 2 * out * N, vec + (2 * out + 1) * N};
        sweep<N, 2>(1, x2, [&](int k, const float (&v)[2]) {
          acc = fma32(o[Dm::GX + k * N + i], v[0], acc);
          acc = fma32(o[Dm::GY + k * N + i], v[1], acc);
        });
        a.part[out * fn + (size_t)e * N + i] = acc;
      }
    }
    // trace records of q and uh, vh for the face terms of phases C and D
    {
      const float *const x[6] = {sq, sq + N, sq + 2 * N, sq + 3 * N, suh, svh};
      write_traces<Dm, 6>(o, x, a.trq, tn, e);
    }
    __syncwarp(lane_mask<Dm>());
  }
}

template <class Dm, int VAR>
__global__ void __launch_bounds__(32 * kMxWarps, Dm::MINB) kx_vol(const MxArgs a) {
  extern __shared__ __align__(16) float sm[];
  stage_mx_ops<Dm>(sm, a.ops);
  __syncthreads();
  vol_body<Dm, VAR>(a, sm, blockIdx.x, gridDim.x);
}

// Nonlinear variants: face lifts of phases C and D (calvarnl_fs.f:350-544),
// wall solves, RK4 update.
template <class Dm, int VAR>
__device__ __forceinline__ void tend_body(const MxArgs &a, float *sm, int blk, int nblk) {
  constexpr int N = Dm::N, G = Dm::G, TG = Dm::TG, R = Dm::R;
  float *o = sm;
  const int lane = threadIdx.x & (Dm::LW - 1), wib = threadIdx.x / Dm::LW;
  float *w = sm + Dm::NOPS + wib * Dm::WS;
  float *gl = w + Dm::S_GL, *tmp = w + Dm::S_TMP;
  const size_t fn = (size_t)a.ne * N, tn = (size_t)a.ne * Dm::TS;
  const int stride = nblk * Dm::SLOTS;
  for (int e = blk * Dm::SLOTS + wib; e < a.ne; e += stride) {
    const float di = (float)a.m.vect[5 * (size_t)e + 4];
    if (lane < TG) {
      const int k = lane / G, j = lane - k * G;
      const FaceRef r = face_ref(a.m, e, k);
      const float fqxx = face_value<G>(a.trq, r, e, lane, j);
      const float fqxy = face_value<G>(a.trq + tn, r, e, lane, j);
      const float fqyx = face_value<G>(a.trq + 2 * tn, r, e, lane, j);
      const float fqyy = face_value<G>(a.trq + 3 * tn, r, e, lane, j);
      const float fuh = face_value<G>(a.trq + 4 * tn, r, e, lane, j);
      const float fvh = face_value<G>(a.trq + 5 * tn, r, e, lane, j);
      const float fh = face_value<G>(a.tr_in + 2 * tn, r, e, lane, j);
      const float Fxx = a.mu0 * fqxx - a.g0 * fh, Fxy = a.mu0 * fqxy;
      const float Fyx = a.mu0 * fqyx, Fyy = a.mu0 * fqyy - a.g0 * fh;
      const float s = r.sig * di * o[Dm::WIF + (r.sig > 0.f ? j : G - 1 - j)];
      gl[lane] = s * (r.nx * Fxx + r.ny * Fxy);
      gl[TG + lane] = s * (r.nx * Fyx + r.ny * Fyy);
      gl[2 * TG + lane] = -s * (r.nx * fuh + r.ny * fvh);
    }
    __syncwarp(lane_mask<Dm>());
    float t[3][R];
    constexpr int RL = R == 2 ? 1 : R;  // rows computed lane by lane
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int i = lane + Dm::LW * r;
      float gx = 0.f, gy = 0.f, hh = 0.f;
      if (i < N) {
        const size_t gi = (size_t)e * N + i;
        gx = a.part[gi];
        gy = a.part[fn + gi];
        hh = a.part[2 * fn + gi];
#pragma unroll
        for (int l = 0; l < TG; ++l) {
          const float L = o[Dm::LIFT + l * N + i];
          gx = fma32(L, gl[l], gx);
          gy = fma32(L, gl[TG + l], gy);
          hh = fma32(L, gl[2 * TG + l], hh);
        }
      }
      t[0][r] = gx;
      t[1][r] = gy;
      t[2][r] = hh;
    }
    if constexpr (R == 2) {
      // rows past the last lane (degree 7: 4 of 36): the lift sums of row
      // LW + t as chains on lanes out * T2 + t, in the same order, then
      // gathered to lane t
      constexpr int T2 = N - Dm::LW;
      static_assert(3 * T2 <= Dm::LW, "row tail");
      const int out = lane / T2, tt = lane - out * T2;
      float acc = 0.f;
      if (lane < 3 * T2) {
        const int i = Dm::LW + tt;
        acc = a.part[out * fn + (size_t)e * N + i];
        const float *g = gl + out * TG;
#pragma unroll 9
        for (int l = 0; l < TG; ++l) acc = fma32(o[Dm::LIFT + l * N + i], g[l], acc);
      }
      const bool own = lane < T2;
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        const float v = __shfl_sync(lane_mask<Dm>(), acc, f * T2 + tt);
        t[f][R - 1] = own ? v : 0.f;
      }
    }
    if (a.m.bdl[e]) {
      const float nx = (float)a.m.normt[2 * (size_t)e], ny = (float)a.m.normt[2 * (size_t)e + 1];
      wall_vec<Dm, VAR == SPOC_NS>(o, tmp, t[0], t[1], nx, ny);
    }
    finish_element<Dm>(a, o, w, e, t);
  }
}

template <class Dm, int VAR>
__global__ void __launch_bounds__(32 * kMxWarps, Dm::MINB) kx_tend(const MxArgs a) {
  extern __shared__ __align__(16) float sm[];
  stage_mx_ops<Dm>(sm, a.ops);
  __syncthreads();
  tend_body<Dm, VAR>(a, sm, blockIdx.x, gridDim.x);
}

// Linear variant (calvar_lin.f:7-287) in one kernel.
template <class Dm>
__global__ void __launch_bounds__(32 * kMxWarps, Dm::MINB_LIN) kx_lin(const MxArgs a) {
  constexpr int N = Dm::N, G = Dm::G, TG = Dm::TG, R = Dm::R;
  extern __shared__ __align__(16) float sm[];
  float *o = sm;
  stage_mx_ops<Dm>(o, a.ops);
  __syncthreads();
  const int lane = threadIdx.x & (Dm::LW - 1), wib = threadIdx.x / Dm::LW;
  float *w = sm + Dm::NOPS + wib * Dm::WS;
  float *su = w + Dm::S_U, *sv = w + Dm::S_V, *sh = w + Dm::S_H;
  float *gl = w + Dm::S_GL, *tmp = w + Dm::S_TMP;
  const size_t fn = (size_t)a.ne * N, tn = (size_t)a.ne * Dm::TS;
  const int stride = gridDim.x * Dm::SLOTS;
  for (int e = blockIdx.x * Dm::SLOTS + wib; e < a.ne; e += stride) {
    const double *vp = a.m.vect + 5 * (size_t)e;
    const float ax = (float)vp[0], bx = (float)vp[1], ay = (float)vp[2], by = (float)vp[3],
                di = (float)vp[4];
    for (int i = lane; i < N; i += Dm::LW) {
      const size_t gi = (size_t)e * N + i;
      su[i] = a.y[gi];
      sv[i] = a.y[fn + gi];
      sh[i] = a.y[2 * fn + gi];
    }
    if (lane < TG) {
      const int k = lane / G, j = lane - k * G;
      const FaceRef r = face_ref(a.m, e, k);
      const float fu = face_value<G>(a.tr_in, r, e, lane, j);
      const float fv = face_value<G>(a.tr_in + tn, r, e, lane, j);
      const float fh = face_value<G>(a.tr_in + 2 * tn, r, e, lane, j);
      const float s = r.sig * di * o[Dm::WIF + (r.sig > 0.f ? j : G - 1 - j)];
      const float fxx = -a.g0 * fh;
      gl[lane] = s * r.nx * fxx;
      gl[TG + lane] = s * r.ny * fxx;
      gl[2 * TG + lane] = -s * a.hh0 * (r.nx * fu + r.ny * fv);
    }
    __syncwarp(lane_mask<Dm>());
    float t[3][R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + Dm::LW * r;
      float gxh = 0.f, gyh = 0.f, gxu = 0.f, gyu = 0.f, gxv = 0.f, gyv = 0.f;
      float l0 = 0.f, l1 = 0.f, l2 = 0.f;
      if (i < N) {
#pragma unroll 4
        for (int k = 1; k < N; ++k) {  // constant mode: see the trace records
          const float cx = o[Dm::GX + k * N + i], cy = o[Dm::GY + k * N + i];
          gxh = fma32(cx, sh[k], gxh);
          gyh = fma32(cy, sh[k], gyh);
          gxu = fma32(cx, su[k], gxu);
          gyu = fma32(cy, su[k], gyu);
          gxv = fma32(cx, sv[k], gxv);
          gyv = fma32(cy, sv[k], gyv);
        }
#pragma unroll
        for (int l = 0; l < TG; ++l) {
          const float L = o[Dm::LIFT + l * N + i];
          l0 = fma32(L, gl[l], l0);
          l1 = fma32(L, gl[TG + l], l1);
          l2 = fma32(L, gl[2 * TG + l], l2);
        }
      }
      // fxx = fyy = -g0 h: gx = cal_b(agx, fxx, -by di) + cal_b(agy, fxx, ay di) + lift
      t[0][r] = -a.g0 * di * (ay * gyh - by * gxh) + l0;
      t[1][r] = -a.g0 * di * (bx * gxh - ax * gyh) + l1;
      t[2][r] = a.hh0 * di * (by * gxu - ay * gyu - bx * gxv + ax * gyv) + l2;
    }
    if (a.m.bdl[e]) {
      const float nx = (float)a.m.normt[2 * (size_t)e], ny = (float)a.m.normt[2 * (size_t)e + 1];
      wall_vec<Dm, false>(o, tmp, t[0], t[1], nx, ny);
    }
    __syncwarp(lane_mask<Dm>());
    finish_element<Dm>(a, o, w, e, t);
  }
}

// Stage input and its traces from the FP64 psi state.
template <class Dm>
__global__ void __launch_bounds__(32 * kMxWarps, Dm::MINB) kx_prep(const MxArgs a) {
  constexpr int N = Dm::N;
  extern __shared__ __align__(16) float sm[];
  float *o = sm;
  stage_mx_ops<Dm>(o, a.ops);
  __syncthreads();
  const int lane = threadIdx.x & (Dm::LW - 1), wib = threadIdx.x / Dm::LW;
  float *w = sm + Dm::NOPS + wib * Dm::WS;
  const size_t fn = (size_t)a.ne * N, tn = (size_t)a.ne * Dm::TS;
  const int stride = gridDim.x * Dm::SLOTS;
  for (int e = blockIdx.x * Dm::SLOTS + wib; e < a.ne; e += stride) {
    for (int f = 0; f < 3; ++f)
      for (int i = lane; i < N; i += Dm::LW) {
        const size_t gi = f * fn + (size_t)e * N + i;
        const float v = (float)a.c64[gi];
        a.y[gi] = v;
        w[f * N + i] = v;
      }
    __syncwarp(lane_mask<Dm>());
    const float *const x[3] = {w, w + N, w + 2 * N};
    write_traces<Dm, 3>(o, x, a.tr_out, tn, e);
    __syncwarp(lane_mask<Dm>());
  }
}

// FP64 basis changes: out = T x per element with T upper triangular (row-major).
__global__ void kx_upper(int ne, int n, const double *T, const double *x, double *out) {
  const size_t total = (size_t)ne * n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t e = t / n;
    const int i = (int)(t - e * n);
    const double *xe = x + e * n;
    double s = 0.0;
    for (int k = i; k < n; ++k) s += T[i * n + k] * xe[k];
    out[t] = s;
  }
}

// Values of a reference-basis field at the quadrature points (spectoxy), FP64
// sum, stored as FP32: out[e*ng + q] = sum_n pi2(q, n) x[e*nm + n].
__global__ void kx_quad(int ne, int nm, int ng, const double *p2, const double *x, float *out) {
  const size_t total = (size_t)ne * ng;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t e = t / ng;
    const int q = (int)(t - e * ng);
    double s = 0.0;
    for (int n = 0; n < nm; ++n) s += p2[(size_t)n * ng + q] * x[e * nm + n];
    out[t] = (float)s;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
struct MixedCtx {
  int variant = 0, nc = 0, N = 0, Q = 0, G = 0, ne = 0, sms = 148;
  int cur = 0;  // which trace buffer holds the traces of the current stage input
  bool w0z0 = false;
  float mu0 = 0, mb0 = 0, g0 = 0, hh0 = 0;
  std::vector<void *> allocs;
  float *ops = nullptr;
  double *U = nullptr, *Ui = nullptr;
  double *c64 = nullptr, *acc = nullptr, *k64 = nullptr, *cin = nullptr;
  float *y = nullptr, *tr[2]{}, *part = nullptr, *trq = nullptr;
  float *hbq = nullptr, *fcq = nullptr, *w0q = nullptr, *z0q = nullptr;
  float *tcimg = nullptr;  // operator image of the tensor-core volume kernel
  bool tc = false;         // nonlinear volume work on the tensor cores
  float psi0 = 0.f, wif[10]{};
  template <class T>
  cudaError_t alloc(T **p, size_t n) {
    cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (n ? n : 1));
    if (e == cudaSuccess) allocs.push_back((void *)*p);
    return e;
  }
  ~MixedCtx() {
    for (void *p : allocs) cudaFree(p);
  }
};

namespace {

// Host construction of the psi-basis operators, FP64 (PsiOps: spoc_mixed_dev.cuh).

bool build_psi(const spoc_tables *t, PsiOps &p, std::string *err) {
  const int nc = t->nc, N = t->nm, Q = t->ng, G = t->ngf, NR = N - nc - 1;
  const int lm = t->ld_mat, lq = t->ld_pi2, lp1 = t->ld_pico1, lp2 = t->ld_pico2;
  auto MAT = [&](const double *a, int i, int j) { return a[(size_t)j * lm + i]; };  // a(i,j)
  p.N = N;
  p.Q = Q;
  p.G = G;
  p.U.assign(N * N, 0.0);
  p.Ui.assign(N * N, 0.0);
  for (int i = 0; i < N; ++i)
    for (int k = i; k < N; ++k) p.U[i * N + k] = MAT(t->amm, i, k);
  // U^-1 by back substitution, column by column
  for (int c = 0; c < N; ++c)
    for (int i = N - 1; i >= 0; --i) {
      double s = i == c ? 1.0 : 0.0;
      for (int k = i + 1; k < N; ++k) s -= p.U[i * N + k] * p.Ui[k * N + c];
      p.Ui[i * N + c] = s / p.U[i * N + i];
    }
  p.Pp.assign(Q * N, 0.0);
  for (int q = 0; q < Q; ++q)
    for (int n = 0; n < N; ++n) {
      double s = 0.0;
      for (int m = 0; m <= n; ++m) s += t->pi2[(size_t)m * lq + q] * p.Ui[m * N + n];
      p.Pp[q * N + n] = s;
    }
  // GX = U^-T A U^-1 with A(i, j) = agx(j, i): cal_b adds coeff * sum_j agx(j,i) a_j
  auto conj = [&](const double *ag, std::vector<double> &out) {
    std::vector<double> tmp(N * N, 0.0);
    for (int i = 0; i < N; ++i)
      for (int n = 0; n < N; ++n) {
        double s = 0.0;
        for (int j = 0; j <= n; ++j) s += MAT(ag, j, i) * p.Ui[j * N + n];
        tmp[i * N + n] = s;
      }
    out.assign(N * N, 0.0);
    for (int m = 0; m < N; ++m)
      for (int n = 0; n < N; ++n) {
        double s = 0.0;
        for (int i = 0; i <= m; ++i) s += p.Ui[i * N + m] * tmp[i * N + n];
        out[m * N + n] = s;
      }
  };
  conj(t->agx, p.GX);
  conj(t->agy, p.GY);
  p.TR.assign(3 * G * N, 0.0);
  for (int s = 0; s < 3; ++s)
    for (int j = 0; j < G; ++j)
      for (int n = 0; n < N; ++n) {
        double acc = 0.0;
        for (int m = 0; m <= n; ++m)
          acc += t->pico[((size_t)s * lp2 + m) * lp1 + j] * p.Ui[m * N + n];
        p.TR[(s * G + j) * N + n] = acc;
      }
  // wall sub-basis: R = matrix of reduc_inv_gn (src/mat1.f:445-473), columns
  // mapped to psi and orthonormalised (modified Gram-Schmidt, two passes)
  std::vector<double> R(N * NR, 0.0);
  for (int j = 0; j <= nc - 1; ++j) {
    const int c1 = t->cip[2 * j], c2 = t->cip[2 * j + 1];
    for (int l = 0; l <= nc - j - 1; ++l) {
      const int r = c2 + l;
      if (r < 0 || r >= NR || c1 < 0 || c1 + l + 1 >= N) {
        if (err) *err = "cip table inconsistent with nc";
        return false;
      }
      R[c1 * NR + r] = (l % 2 == 0) ? 1.0 : -1.0;
      R[(c1 + l + 1) * NR + r] = 1.0;
    }
  }
  std::vector<double> B(N * NR, 0.0);  // U R
  for (int i = 0; i < N; ++i)
    for (int r = 0; r < NR; ++r) {
      double s = 0.0;
      for (int k = i; k < N; ++k) s += p.U[i * N + k] * R[k * NR + r];
      B[i * NR + r] = s;
    }
  for (int r = 0; r < NR; ++r) {
    for (int pass = 0; pass < 2; ++pass)
      for (int r2 = 0; r2 < r; ++r2) {
        double d = 0.0;
        for (int i = 0; i < N; ++i) d += B[i * NR + r] * B[i * NR + r2];
        for (int i = 0; i < N; ++i) B[i * NR + r] -= d * B[i * NR + r2];
      }
    double nrm = 0.0;
    for (int i = 0; i < N; ++i) nrm += B[i * NR + r] * B[i * NR + r];
    nrm = std::sqrt(nrm);
    if (!(nrm > 0.0)) {
      if (err) *err = "wall sub-basis is rank deficient";
      return false;
    }
    for (int i = 0; i < N; ++i) B[i * NR + r] /= nrm;
  }
  p.PWALL.assign(N * N, 0.0);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int r = 0; r < NR; ++r) s += B[i * NR + r] * B[k * NR + r];
      p.PWALL[i * N + k] = s;
    }
  return true;
}

template <class Dm>
std::vector<float> ops_image(const PsiOps &p, const spoc_tables *t) {
  constexpr int N = Dm::N, Q = Dm::Q, G = Dm::G, TG = Dm::TG;
  std::vector<float> o(Dm::NOPS, 0.f);
  for (int n = 0; n < N; ++n)
    for (int q = 0; q < Q; ++q) o[Dm::PPT + n * Q + q] = (float)p.Pp[q * N + n];
  for (int q = 0; q < Q; ++q)
    for (int i = 0; i < N; ++i) o[Dm::PW + q * N + i] = (float)(p.Pp[q * N + i] * t->wi[q]);
  for (int k = 0; k < N; ++k)
    for (int i = 0; i < N; ++i) {
      o[Dm::GX + k * N + i] = (float)p.GX[i * N + k];
      o[Dm::GY + k * N + i] = (float)p.GY[i * N + k];
      o[Dm::PWALL + k * N + i] = (float)p.PWALL[i * N + k];
    }
  for (int n = 0; n < N; ++n)
    for (int l = 0; l < TG; ++l) {
      o[Dm::TRT + n * TG + l] = (float)p.TR[l * N + n];
      o[Dm::LIFT + l * N + n] = (float)p.TR[l * N + n];
    }
  for (int j = 0; j < G; ++j) o[Dm::WIF + j] = (float)t->wif[j];
  return o;
}

// Persistent grid: as many blocks as stay resident (occupancy x SMs on the
// current device), or fewer when the elements run out.
using MxKernel = void (*)(MxArgs);
cudaError_t grid_for(MxKernel kernel, size_t smem, int sms, int ne, int slots, int *grid) {
  return resident_grid(kernel, 32 * kMxWarps, smem, sms, ne, slots, grid);
}

template <class Dm>
constexpr size_t mx_smem() {
  return sizeof(float) * (Dm::NOPS + (size_t)Dm::SLOTS * Dm::WS);
}

// Launches of one right-hand side (stage >= 0: with the RK4 update).
template <class Dm>
cudaError_t run_stage(MixedCtx *c, const MxArgs &a, cudaStream_t st, long long *launches,
                      cudaEvent_t *ev) {
  constexpr size_t smem = mx_smem<Dm>();
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], st);
  };
  if (c->variant == SPOC_LIN) {
    int g = 0;
    const cudaError_t ge = grid_for(kx_lin<Dm>, smem, c->sms, c->ne, Dm::SLOTS, &g);
    if (ge != cudaSuccess) return ge;
    mark(0);
    kx_lin<Dm><<<g, 32 * kMxWarps, smem, st>>>(a);
    mark(1);
    if (launches) *launches += 1;
    return cudaGetLastError();
  }
  cudaError_t tce = cudaSuccess;
  auto go = [&](MxKernel kv, MxKernel kt) {
    int gv = 0, gt = 0;
    tce = grid_for(kv, smem, c->sms, c->ne, Dm::SLOTS, &gv);
    if (tce == cudaSuccess) tce = grid_for(kt, smem, c->sms, c->ne, Dm::SLOTS, &gt);
    if (tce != cudaSuccess) return;
    mark(0);
    if (c->tc) {
      tce = mixed_tc_vol(c->variant, c->nc, c->Q, c->G, a, c->tcimg, c->sms, st);
      if (tce != cudaSuccess) return;
    } else {
      kv<<<gv, 32 * kMxWarps, smem, st>>>(a);
    }
    mark(1);
    if (c->tc) {
      tce = mixed_tc_tend(c->variant, c->nc, c->Q, c->G, a, c->tcimg, c->sms, st);
      if (tce != cudaSuccess) return;
    } else {
      kt<<<gt, 32 * kMxWarps, smem, st>>>(a);
    }
    mark(2);
    if (launches) *launches += 2;
  };
  if (c->variant == SPOC_FS) go(kx_vol<Dm, SPOC_FS>, kx_tend<Dm, SPOC_FS>);
  else if (c->variant == SPOC_NS) go(kx_vol<Dm, SPOC_NS>, kx_tend<Dm, SPOC_NS>);
  else go(kx_vol<Dm, SPOC_INV>, kx_tend<Dm, SPOC_INV>);
  if (tce != cudaSuccess) return tce;
  return cudaGetLastError();
}

template <class Dm>
cudaError_t run_prep(MixedCtx *c, const MxArgs &a, cudaStream_t st, long long *launches) {
  constexpr size_t smem = mx_smem<Dm>();
  int g = 0;
  const cudaError_t ge = grid_for(kx_prep<Dm>, smem, c->sms, c->ne, Dm::SLOTS, &g);
  if (ge != cudaSuccess) return ge;
  kx_prep<Dm><<<g, 32 * kMxWarps, smem, st>>>(a);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

// Dispatch over the tabulated (nc, ng, ngf) combinations.
template <class F>
bool with_dims(int nc, int ng, int ngf, F &&f) {
  if (nc == 3 && ng == 12 && ngf == 4) return f(MDims<3, 12, 4>{}), true;
  if (nc == 4 && ng == 25 && ngf == 5) return f(MDims<4, 25, 5>{}), true;
  if (nc == 5 && ng == 27 && ngf == 6) return f(MDims<5, 27, 6>{}), true;
  if (nc == 6 && ng == 33 && ngf == 7) return f(MDims<6, 33, 7>{}), true;
  if (nc == 7 && ng == 42 && ngf == 9) return f(MDims<7, 42, 9>{}), true;
  return false;
}

MxArgs base_args(MixedCtx *c, const DevMesh &m) {
  MxArgs a{};
  a.ne = c->ne;
  a.ops = c->ops;
  a.m = m;
  a.y = c->y;
  a.part = c->part;
  a.trq = c->trq;
  a.hbq = c->hbq;
  a.fcq = c->fcq;
  a.w0q = c->w0z0 ? nullptr : c->w0q;
  a.z0q = c->w0z0 ? nullptr : c->z0q;
  a.mu0 = c->mu0;
  a.mb0 = c->mb0;
  a.g0 = c->g0;
  a.hh0 = c->hh0;
  a.c64 = c->c64;
  a.acc = c->acc;
  a.k64 = c->k64;
  a.psi0 = c->psi0;
  for (int j = 0; j < 10; ++j) a.wif[j] = c->wif[j];
  return a;
}

int blocks_for(size_t n) {
  const size_t b = (n + 255) / 256;
  return (int)(b < 4096 ? (b ? b : 1) : 4096);
}

}  // namespace

bool mixed_available(int nc, int ng, int ngf) {
  return with_dims(nc, ng, ngf, [](auto) {});
}

int mixed_kernels_per_rhs(const MixedCtx *c) { return c->variant == SPOC_LIN ? 1 : 2; }

bool mixed_set_tensor(MixedCtx *c, bool on) {
  if (on && !c->tcimg) return false;
  c->tc = on;
  return true;
}

void mixed_default_path(MixedCtx *c) { c->tc = false; }

bool mixed_uses_tensor(const MixedCtx *c) { return c->tc; }

int mixed_create(MixedCtx **out, const spoc_tables *t, int variant, int ne, int sms,
                 std::string *err) {
  *out = nullptr;
  if (!mixed_available(t->nc, t->ng, t->ngf)) {
    if (err) *err = "mixed precision is built for (nc, ng, ngf) = (3,12,4), (4,25,5), (5,27,6), (6,33,7), (7,42,9)";
    return SPOC_E_UNSUPPORTED;
  }
  PsiOps p;
  if (!build_psi(t, p, err)) return SPOC_E_MATRIX;
  MixedCtx *c = new (std::nothrow) MixedCtx();
  if (!c) return SPOC_E_NOMEM;
  c->variant = variant;
  c->nc = t->nc;
  c->N = p.N;
  c->Q = p.Q;
  c->G = p.G;
  c->ne = ne;
  c->sms = sms;
  std::vector<float> img;
  with_dims(t->nc, t->ng, t->ngf, [&](auto d) {
    using Dm = decltype(d);
    img = ops_image<Dm>(p, t);
  });
  c->psi0 = (float)p.TR[0];  // trace of the constant mode: its value
  for (int j = 0; j < t->ngf && j < 10; ++j) c->wif[j] = (float)t->wif[j];
  std::vector<float> tcimg;
  if (variant != SPOC_LIN && mixed_tc_available(t->nc, t->ng, t->ngf))
    tcimg = mixed_tc_image(t->nc, t->ng, t->ngf, p, t->wi);
  const size_t fn = (size_t)ne * p.N, tn = (size_t)ne * (3 * p.G + 1), qn = (size_t)ne * p.Q;
  cudaError_t ce = c->alloc(&c->ops, img.size());
  if (ce == cudaSuccess) ce = cudaMemcpy(c->ops, img.data(), sizeof(float) * img.size(), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess && !tcimg.empty()) ce = c->alloc(&c->tcimg, tcimg.size());
  if (ce == cudaSuccess && !tcimg.empty())
    ce = cudaMemcpy(c->tcimg, tcimg.data(), sizeof(float) * tcimg.size(), cudaMemcpyHostToDevice);
  // default kernel family: the FP32 pipes.  The tensor-core kernel is faster
  // at degree 7 but its three-term TF32 products are less accurate than FP32
  // multiply-adds (C3, 1000 steps: 1.0e-5 against 2.0e-6 relative eta
  // error), so it is chosen explicitly with SPOC_PATH_TENSOR.
  c->tc = false;
  if (ce == cudaSuccess) ce = c->alloc(&c->U, p.U.size());
  if (ce == cudaSuccess) ce = cudaMemcpy(c->U, p.U.data(), sizeof(double) * p.U.size(), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = c->alloc(&c->Ui, p.Ui.size());
  if (ce == cudaSuccess) ce = cudaMemcpy(c->Ui, p.Ui.data(), sizeof(double) * p.Ui.size(), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = c->alloc(&c->c64, 3 * fn);
  if (ce == cudaSuccess) ce = c->alloc(&c->acc, 3 * fn);
  if (ce == cudaSuccess) ce = c->alloc(&c->k64, 3 * fn);
  if (ce == cudaSuccess) ce = c->alloc(&c->cin, 3 * fn);
  if (ce == cudaSuccess) ce = c->alloc(&c->y, 3 * fn);
  if (ce == cudaSuccess) ce = c->alloc(&c->tr[0], 3 * tn);
  if (ce == cudaSuccess) ce = c->alloc(&c->tr[1], 3 * tn);
  if (ce == cudaSuccess && variant != SPOC_LIN) ce = c->alloc(&c->part, 3 * fn);
  if (ce == cudaSuccess && variant != SPOC_LIN) ce = c->alloc(&c->trq, 6 * tn);
  if (ce == cudaSuccess) ce = c->alloc(&c->hbq, qn);
  if (ce == cudaSuccess) ce = c->alloc(&c->fcq, qn);
  if (ce == cudaSuccess) ce = c->alloc(&c->w0q, qn);
  if (ce == cudaSuccess) ce = c->alloc(&c->z0q, qn);
  if (ce == cudaSuccess) ce = cudaMemset(c->c64, 0, sizeof(double) * 3 * fn);
  if (ce != cudaSuccess) {
    if (err) *err = std::string("mixed-precision device set-up: ") + cudaGetErrorString(ce);
    delete c;
    return ce == cudaErrorMemoryAllocation ? SPOC_E_NOMEM : SPOC_E_CUDA;
  }
  *out = c;
  return SPOC_OK;
}

void mixed_destroy(MixedCtx *c) { delete c; }

cudaError_t mixed_set_params(MixedCtx *c, const DevOps &op, const double *hb, const double *fc,
                             const double *w0, const double *z0, bool w0z0_zero, double mu0,
                             double mb0, double g0, double hh0, cudaStream_t st) {
  c->mu0 = (float)mu0;
  c->mb0 = (float)mb0;
  c->g0 = (float)g0;
  c->hh0 = (float)hh0;
  c->w0z0 = w0z0_zero;
  const int b = blocks_for((size_t)c->ne * c->Q);
  kx_quad<<<b, 256, 0, st>>>(c->ne, c->N, c->Q, op.p2, hb, c->hbq);
  kx_quad<<<b, 256, 0, st>>>(c->ne, c->N, c->Q, op.p2, fc, c->fcq);
  kx_quad<<<b, 256, 0, st>>>(c->ne, c->N, c->Q, op.p2, w0, c->w0q);
  kx_quad<<<b, 256, 0, st>>>(c->ne, c->N, c->Q, op.p2, z0, c->z0q);
  return cudaGetLastError();
}

cudaError_t mixed_set_state(MixedCtx *c, const DevMesh &m, const double *const phi[3],
                            cudaStream_t st, long long *launches) {
  const size_t fn = (size_t)c->ne * c->N;
  const int b = blocks_for(fn);
  for (int f = 0; f < 3; ++f) kx_upper<<<b, 256, 0, st>>>(c->ne, c->N, c->U, phi[f], c->c64 + f * fn);
  if (launches) *launches += 3;
  MxArgs a = base_args(c, m);
  c->cur = 0;
  a.tr_out = c->tr[0];
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return ce;
  with_dims(c->nc, c->Q, c->G, [&](auto d) { ce = run_prep<decltype(d)>(c, a, st, launches); });
  return ce;
}

cudaError_t mixed_get_state(MixedCtx *c, double *const phi[3], cudaStream_t st, long long *launches) {
  const size_t fn = (size_t)c->ne * c->N;
  const int b = blocks_for(fn);
  for (int f = 0; f < 3; ++f) kx_upper<<<b, 256, 0, st>>>(c->ne, c->N, c->Ui, c->c64 + f * fn, phi[f]);
  if (launches) *launches += 3;
  return cudaGetLastError();
}

cudaError_t mixed_steps(MixedCtx *c, const DevMesh &m, double dt, int nsteps, int *flag,
                        cudaStream_t st, long long *launches, cudaEvent_t *ev) {
  MxArgs a = base_args(c, m);
  a.dt = dt;
  a.dt6 = dt / 6.0;
  a.flag = flag;
  cudaError_t ce = cudaSuccess;
  for (int it = 0; it < nsteps && ce == cudaSuccess; ++it)
    for (int s = 0; s < 4 && ce == cudaSuccess; ++s) {
      a.stage = s;
      a.tr_in = c->tr[c->cur];
      a.tr_out = c->tr[c->cur ^ 1];
      cudaEvent_t *e = (ev && it == nsteps - 1 && s == 0) ? ev : nullptr;
      with_dims(c->nc, c->Q, c->G, [&](auto d) { ce = run_stage<decltype(d)>(c, a, st, launches, e); });
      c->cur ^= 1;
    }
  return ce;
}

cudaError_t mixed_rhs(MixedCtx *c, const DevMesh &m, const double *const in[3],
                      double *const out[3], int *flag, cudaStream_t st, long long *launches) {
  // the resident state is kept: the input goes through cin and the stage
  // buffers, which the next mixed_steps call rebuilds from c64
  const size_t fn = (size_t)c->ne * c->N;
  const int b = blocks_for(fn);
  for (int f = 0; f < 3; ++f) kx_upper<<<b, 256, 0, st>>>(c->ne, c->N, c->U, in[f], c->cin + f * fn);
  if (launches) *launches += 3;
  MxArgs a = base_args(c, m);
  a.c64 = c->cin;
  a.flag = flag;
  a.tr_out = c->tr[c->cur ^ 1];
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess)
    with_dims(c->nc, c->Q, c->G, [&](auto d) { ce = run_prep<decltype(d)>(c, a, st, launches); });
  a.stage = -1;
  a.tr_in = c->tr[c->cur ^ 1];
  a.tr_out = nullptr;
  if (ce == cudaSuccess)
    with_dims(c->nc, c->Q, c->G, [&](auto d) { ce = run_stage<decltype(d)>(c, a, st, launches, nullptr); });
  for (int f = 0; f < 3 && ce == cudaSuccess; ++f) {
    kx_upper<<<b, 256, 0, st>>>(c->ne, c->N, c->Ui, c->k64 + f * fn, out[f]);
    ce = cudaGetLastError();
  }
  if (launches) *launches += 3;
  // restore the stage input of the resident state
  a = base_args(c, m);
  a.tr_out = c->tr[c->cur];
  if (ce == cudaSuccess)
    with_dims(c->nc, c->Q, c->G, [&](auto d) { ce = run_prep<decltype(d)>(c, a, st, launches); });
  return ce;
}


// ---------------------------------------------------------------------------
// Ensemble: members with their own meshes, degrees 3-6 and time steps advance
// together, one cooperative launch per RK4 stage for all of them.  Blocks are
// dealt to members in proportion to their work; a block stages its member's
// operators once, runs the volume phase on the member's elements, waits for
// the whole grid (the face terms of the tendency phase read neighbour trace
// records), then runs the tendency phase.  All members are free-slip
// (calvarnl_fs.f) and use the FP32-pipe kernels.

struct EnsMember {
  MxArgs a;        // stage, tr_in and tr_out are set per launch
  float *tr[2];
  int nc, first_block, nblocks;
};

namespace {

template <class F>
__device__ __forceinline__ void ens_dims(int nc, F &&f) {
  switch (nc) {
    case 3: f(MDims<3, 12, 4>{}); break;
    case 4: f(MDims<4, 25, 5>{}); break;
    case 5: f(MDims<5, 27, 6>{}); break;
    default: f(MDims<6, 33, 7>{}); break;
  }
}

constexpr int kEnsMinBlocks = 4;  // degrees 3-6: one row per lane, 64 registers

// bt (null except when balancing): each block adds the SM cycles of its
// volume phase (operator staging included) and of its tendency phase to
// bt[2 b] and bt[2 b + 1].
__global__ void __launch_bounds__(32 * kMxWarps, kEnsMinBlocks)
    kx_ens_stage(const EnsMember *__restrict__ mem, const int *__restrict__ blk_member, int stage,
                 int cur, unsigned long long *bt) {
  extern __shared__ __align__(16) float sm[];
  const EnsMember &em = mem[blk_member[blockIdx.x]];
  MxArgs a = em.a;
  a.stage = stage;
  a.tr_in = em.tr[cur];
  a.tr_out = em.tr[cur ^ 1];
  const int lb = blockIdx.x - em.first_block, nb = em.nblocks;
  const long long c0 = bt ? clock64() : 0;
  ens_dims(em.nc, [&](auto d) { stage_mx_ops<decltype(d)>(sm, a.ops); });
  __syncthreads();
  ens_dims(em.nc, [&](auto d) { vol_body<decltype(d), SPOC_FS>(a, sm, lb, nb); });
  if (bt) {
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(bt + 2 * blockIdx.x, (unsigned long long)(clock64() - c0));
  }
  cooperative_groups::this_grid().sync();
  const long long c1 = bt ? clock64() : 0;
  ens_dims(em.nc, [&](auto d) { tend_body<decltype(d), SPOC_FS>(a, sm, lb, nb); });
  if (bt) {
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(bt + 2 * blockIdx.x + 1, (unsigned long long)(clock64() - c1));
  }
}

size_t ens_smem() {
  const size_t s[4] = {mx_smem<MDims<3, 12, 4>>(), mx_smem<MDims<4, 25, 5>>(),
                       mx_smem<MDims<5, 27, 6>>(), mx_smem<MDims<6, 33, 7>>()};
  size_t m = 0;
  for (size_t v : s) m = v > m ? v : m;
  return m;
}

}  // namespace

struct MixedEns {
  std::vector<MixedCtx *> mem;
  std::vector<DevMesh> mesh;
  std::vector<int *> flag;
  std::vector<double> dt;
  std::vector<int> nb;  // blocks of each member under the current layout
  std::vector<double> mw;  // measured work per member (weight 4)
  int sms = 148, bps = 0, weight = 0, nblk = 0, max_bps = 1;
  EnsMember *d_mem = nullptr;
  int *d_blk = nullptr;
  unsigned long long *d_bt = nullptr;  // block cycles while balancing
  cudaStream_t st = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool graph_ok = true;
  ~MixedEns() {
    if (exec) cudaGraphExecDestroy(exec);
    cudaFree(d_mem);
    cudaFree(d_blk);
    cudaFree(d_bt);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

// Blocks per member in proportion to its work, modelled as ne nm^p with
// p = 2, 1, 0.5, 0 for weight 0..3, or measured (weight 4: the member's
// block cycles of a balancing step); at least one block each.
int ens_layout(MixedEns *e) {
  const int n = (int)e->mem.size();
  const int total = e->bps * e->sms;
  if (total < n) return SPOC_E_UNSUPPORTED;
  std::vector<double> w(n);
  double sw = 0.0;
  for (int i = 0; i < n; ++i) {
    const double N = e->mem[i]->N;
    static const double expo[4] = {2.0, 1.0, 0.5, 0.0};
    w[i] = e->weight == 4 ? e->mw[i] : (double)e->mem[i]->ne * std::pow(N, expo[e->weight]);
    sw += w[i];
  }
  std::vector<int> nb(n, 1);
  int left = total - n;
  for (int i = 0; i < n; ++i) {
    const int extra = (int)std::floor(left * w[i] / sw);
    nb[i] += extra;
  }
  int used = 0;
  for (int v : nb) used += v;
  for (int i = 0; used < total; i = (i + 1) % n, ++used) ++nb[i];  // remainder
  e->nb = nb;
  std::vector<EnsMember> hm(n);
  std::vector<int> blk;
  for (int i = 0; i < n; ++i) {
    MixedCtx *c = e->mem[i];
    EnsMember &m = hm[i];
    m.a = base_args(c, e->mesh[i]);
    m.a.dt = e->dt[i];
    m.a.dt6 = e->dt[i] / 6.0;
    m.a.flag = e->flag[i];
    m.tr[0] = c->tr[0];
    m.tr[1] = c->tr[1];
    m.nc = c->nc;
    m.first_block = (int)blk.size();
    m.nblocks = nb[i];
    for (int b = 0; b < nb[i]; ++b) blk.push_back(i);
  }
  e->nblk = (int)blk.size();
  cudaFree(e->d_mem);
  cudaFree(e->d_blk);
  e->d_mem = nullptr;
  e->d_blk = nullptr;
  cudaError_t ce = cudaMalloc(&e->d_mem, sizeof(EnsMember) * n);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_blk, sizeof(int) * blk.size());
  if (ce == cudaSuccess)
    ce = cudaMemcpy(e->d_mem, hm.data(), sizeof(EnsMember) * n, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess)
    ce = cudaMemcpy(e->d_blk, blk.data(), sizeof(int) * blk.size(), cudaMemcpyHostToDevice);
  if (e->exec) {
    cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
  }
  return ce == cudaSuccess ? SPOC_OK : SPOC_E_CUDA;
}

cudaError_t ens_launch_step(MixedEns *e, int cur0, unsigned long long *bt = nullptr) {
  const size_t smem = ens_smem();
  for (int s = 0; s < 4; ++s) {
    int stage = s, cur = (cur0 + s) & 1;
    void *args[] = {(void *)&e->d_mem, (void *)&e->d_blk, (void *)&stage, (void *)&cur,
                    (void *)&bt};
    cudaError_t ce = cudaLaunchCooperativeKernel((const void *)kx_ens_stage, dim3(e->nblk),
                                                 dim3(32 * kMxWarps), args, smem, e->st);
    if (ce != cudaSuccess) return ce;
  }
  return cudaSuccess;
}

}  // namespace

int mixed_ens_create(MixedEns **out, MixedCtx *const *ctx, const DevMesh *meshes,
                     int *const *flags, int n, int sms, std::string *err) {
  *out = nullptr;
  for (int i = 0; i < n; ++i)
    if (ctx[i]->variant != SPOC_FS || ctx[i]->nc < 3 || ctx[i]->nc > 6) {
      if (err) *err = "ensemble members: free-slip variant, degree 3-6, mixed precision";
      return SPOC_E_UNSUPPORTED;
    }
  int coop = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop) {
    if (err) *err = "device has no cooperative launch";
    return SPOC_E_UNSUPPORTED;
  }
  MixedEns *e = new (std::nothrow) MixedEns();
  if (!e) return SPOC_E_NOMEM;
  e->mem.assign(ctx, ctx + n);
  e->mesh.assign(meshes, meshes + n);
  e->flag.assign(flags, flags + n);
  e->dt.assign(n, 0.0);
  e->sms = sms;
  const size_t smem = ens_smem();
  cudaError_t ce = cudaFuncSetAttribute(kx_ens_stage, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem);
  int occ = 0;
  if (ce == cudaSuccess)
    ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kx_ens_stage, 32 * kMxWarps, smem);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
  if (ce != cudaSuccess || occ < 1) {
    if (err) *err = std::string("ensemble set-up: ") + cudaGetErrorString(ce);
    delete e;
    return SPOC_E_CUDA;
  }
  e->max_bps = occ;
  e->bps = occ;
  const int rc = ens_layout(e);
  if (rc) {
    if (err) *err = "ensemble: more members than resident blocks";
    delete e;
    return rc;
  }
  *out = e;
  return SPOC_OK;
}

void mixed_ens_destroy(MixedEns *e) { delete e; }

int mixed_ens_configure(MixedEns *e, int bps, int weight) {
  if (bps < 1 || bps > e->max_bps || weight < 0 || weight > 4) return SPOC_E_ARG;
  if (weight == 4 && e->mw.size() != e->mem.size()) return SPOC_E_ARG;
  e->bps = bps;
  e->weight = weight;
  return ens_layout(e);
}

void mixed_ens_info(const MixedEns *e, int *bps, int *max_bps, int *weight, int *blocks,
                    int *graph) {
  *bps = e->bps;
  *max_bps = e->max_bps;
  *weight = e->weight;
  *blocks = e->nblk;
  *graph = e->exec != nullptr;
}

int mixed_ens_member_blocks(const MixedEns *e, int i) {
  return (i >= 0 && i < (int)e->nb.size()) ? e->nb[i] : -1;
}

cudaError_t mixed_ens_balance(MixedEns *e, const double *dt, int rounds) {
  const int n = (int)e->mem.size();
  for (int i = 0; i < n; ++i) e->dt[i] = dt[i];
  const int cur0 = e->mem[0]->cur;
  for (MixedCtx *c : e->mem)
    if (c->cur != cur0) return cudaErrorInvalidValue;
  const size_t cap = 2 * (size_t)e->max_bps * e->sms;
  cudaError_t ce = cudaSuccess;
  if (!e->d_bt) ce = cudaMalloc(&e->d_bt, sizeof(unsigned long long) * cap);
  std::vector<unsigned long long> bt(cap);
  for (int r = 0; r < rounds && ce == cudaSuccess; ++r) {
    if (ens_layout(e)) return cudaErrorMemoryAllocation;
    ce = cudaMemsetAsync(e->d_bt, 0, sizeof(unsigned long long) * 2 * e->nblk, e->st);
    if (ce == cudaSuccess) ce = ens_launch_step(e, cur0, e->d_bt);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(bt.data(), e->d_bt, sizeof(unsigned long long) * 2 * e->nblk,
                           cudaMemcpyDeviceToHost, e->st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
    if (ce != cudaSuccess) break;
    // a member's work: the cycles of all its blocks in both phases
    std::vector<double> w(n, 0.0);
    for (int i = 0, b = 0; i < n; ++i)
      for (int k = 0; k < e->nb[i]; ++k, ++b) w[i] += (double)bt[2 * b] + (double)bt[2 * b + 1];
    e->mw = w;
    e->weight = 4;
  }
  if (ce == cudaSuccess && ens_layout(e)) return cudaErrorMemoryAllocation;
  return ce;
}

cudaError_t mixed_ens_steps(MixedEns *e, const double *dt, int nsteps, bool use_graph) {
  bool changed = false;
  for (size_t i = 0; i < e->mem.size(); ++i)
    if (e->dt[i] != dt[i]) {
      e->dt[i] = dt[i];
      changed = true;
    }
  if (changed && ens_layout(e)) return cudaErrorMemoryAllocation;
  // members step in lockstep from the trace buffer their state set-up filled
  const int cur0 = e->mem[0]->cur;
  for (MixedCtx *c : e->mem)
    if (c->cur != cur0) return cudaErrorInvalidValue;
  cudaError_t ce = cudaSuccess;
  if (use_graph && e->graph_ok && !e->exec) {
    cudaGraph_t g = nullptr;
    ce = cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      const cudaError_t le = ens_launch_step(e, cur0);
      ce = cudaStreamEndCapture(e->st, &g);
      if (le != cudaSuccess) ce = le;
    }
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      e->graph_ok = false;  // fall back to direct launches
      e->exec = nullptr;
      cudaGetLastError();
      ce = cudaSuccess;
    }
  }
  for (int it = 0; it < nsteps && ce == cudaSuccess; ++it)
    ce = (use_graph && e->exec) ? cudaGraphLaunch(e->exec, e->st) : ens_launch_step(e, cur0);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
  return ce;
}

}  // namespace spoc
