// Tangent-linear and adjoint kernels of the SPOC right-hand side (FP64).
//
// The right-hand side (calvarnl_*.f, calvar_lin.f) is linear in the state
// except for the pointwise products and divisions at quadrature points
// (calvarnl_fs.f:263-296).  Hence
//   * tangent-linear model: the forward q-phase, tendency and linear kernels
//     applied to the perturbation (they are linear in their inputs) plus one
//     linearised quadrature-point kernel (k_nlvol_tlm);
//   * adjoint: the transpose of every stage, in reverse order.  The mass
//     solves and every wall projection are self-adjoint (the rotations are
//     symmetric reflections and reduc_inv_gn is the transpose of reduc_gn), so
//     the adjoint reuses the forward solve code.  Face-flux transposes are
//     done in two kernels without atomics: each element writes the adjoint of
//     its three side lifts (in face-point order), then each element gathers
//     both sides of its faces and applies the transposed trace.
// One warp per element, lanes over modes / points, as the generic forward
// kernels.  Fused multiply-adds are used freely: these kernels are checked
// by dot-product and finite-difference tests, not bit for bit.
#include <cuda_runtime.h>

#include <algorithm>

#include "spoc_device.cuh"
#include "spoc_kernels.h"

namespace spoc {
namespace {

constexpr int kT = 256;
constexpr int kWB = kT / kWarp;

// Sizes known at compile time for the tabulated (nc, ng, ngf): the kernels
// read their sizes from op, so fixing them here lets every loop be unrolled
// and every index be folded; RtDims keeps the runtime sizes.
struct RtDims {
  static constexpr int NC = 0, NG = 0, NGF = 0;
};
template <int NC_, int NG_, int NGF_>
struct FixDims {
  static constexpr int NC = NC_, NG = NG_, NGF = NGF_;
};
template <class D>
__device__ __forceinline__ DevOps fixed_dims(const DevOps &in) {
  DevOps o = in;
  if (D::NC > 0) {
    o.nc = D::NC;
    o.nm = (D::NC + 1) * (D::NC + 2) / 2;
    o.nmr = D::NC * (D::NC + 1) / 2;
    o.ng = D::NG;
    o.ngf = D::NGF;
  }
  return o;
}

// Resident blocks per SM asked of the compiler for the heavier adjoint
// kernels: with compile-time sizes up to degree 6 a cap of 80 registers
// costs a few spilled words and raises the resident warps from 16 to 24
// (these kernels are latency-bound).
template <class D>
constexpr int adj_min_blocks() {
  return D::NC >= 1 && D::NC <= 6 ? 3 : 1;
}

__device__ __forceinline__ int wg() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int wc() { return (gridDim.x * blockDim.x) >> 5; }
__device__ __forceinline__ double fmac(double acc, double a, double b) { return __fma_rn(a, b, acc); }

__device__ __forceinline__ V2 vadd(V2 a, V2 b) { return V2{a.a + b.a, a.b + b.b}; }
__device__ __forceinline__ V2 vscale(V2 a, double c) { return V2{a.a * c, a.b * c}; }
// c1*a + c2*b
__device__ __forceinline__ V2 vlin(double c1, V2 a, double c2, V2 b) {
  return V2{fmac(c1 * a.a, c2, b.a), fmac(c1 * a.b, c2, b.b)};
}

struct Geo {
  double ax, bx, ay, by, detai;
};
__device__ __forceinline__ Geo geo(const DevMesh &m, int e) {
  const double *v = m.vect + 5 * (size_t)e;
  return Geo{__ldg(v), __ldg(v + 1), __ldg(v + 2), __ldg(v + 3), __ldg(v + 4)};
}

// Adjoint of the three side lifts of tri_f (src/mat1.f:189-206) for one
// load vector g (smem, nm): L[(e*3+k)*G + j] = sig_k * wif(j) * sum_n
// pico(j1(j), n, k) g(n), j in face-point order, sig_k = its_k * coeff / 2.
__device__ __forceinline__ void side_lift_adj(const DevOps &op, const DevMesh &m, int e,
                                              const double *g, double coeff, double *L) {
  const int l = lane_id(), G = op.ngf, nm = op.nm;
  if (l < 3 * G) {
    const int k = l / G, j = l - k * G;  // j 0-based face point
    const int isg = __ldg(m.its + 3 * e + k);
    const int j1 = isg > 0 ? j : G - 1 - j;  // element-local point
    const double sig = isg * coeff * 0.5;
    const double *p = op.picoF + (size_t)k * nm * G + j1;
    double s = 0.0;
    for (int n = 0; n < nm; ++n) s = fmac(s, __ldg(p + n * G), g[n]);
    L[(3 * (size_t)e + k) * G + j] = sig * __ldg(op.wif + j) * s;
  }
}

// Sum over the (one or two) elements of each face of element e of their side
// lift adjoints, in face-point order: S[k*G + j].  Also returns the trace
// weight (0.5 interior, 1 wall) per side through wt[k].
__device__ __forceinline__ void face_sums(const DevOps &op, const DevMesh &m, int e,
                                          const double *L, double *S) {
  const int l = lane_id(), G = op.ngf;
  if (l < 3 * G) {
    const int k = l / G, j = l - k * G;
    const int f = __ldg(m.itm + 3 * e + k);
    const int t1 = __ldg(m.tseg + 2 * f), t2 = __ldg(m.tseg + 2 * f + 1);
    double s = L[(3 * (size_t)e + k) * G + j];
    if (t2 >= 0) {
      const int nb = (t1 == e) ? t2 : t1;
      const int kn = (t1 == e) ? __ldg(m.ssit + 2 * f + 1) : __ldg(m.ssit + 2 * f);
      s += L[(3 * (size_t)nb + kn) * G + j];
    }
    S[l] = s;
  }
}

// Transposed cal_flu (src/calflu.f:31-62) for element e: a(n) = sum_k w_k
// sum_j pico(j_e(j), n, k) * c_k(j) * S[k*G + j], with c_k(j) = norm(comp,
// face_k) * scale and w_k = 0.5 (interior) or 1 (wall, traced on side 1).
__device__ __forceinline__ V2 trace_adj(const DevOps &op, const DevMesh &m, int e, const double *S,
                                        int comp, double scale) {
  const int l = lane_id(), G = op.ngf, nm = op.nm;
  V2 a = vzero();
  for (int k = 0; k < 3; ++k) {
    const int f = __ldg(m.itm + 3 * e + k);
    const int t1 = __ldg(m.tseg + 2 * f), t2 = __ldg(m.tseg + 2 * f + 1);
    const double w = (t2 < 0 ? 1.0 : 0.5) * __ldg(m.norm + 2 * f + comp) * scale;
    const bool first = (t1 == e);
    const double *pk = op.picoT + (size_t)k * G * nm;
    for (int j = 0; j < G; ++j) {
      const int je = first ? j : G - 1 - j;
      const double c = w * S[k * G + j];
      const double *pr = pk + (size_t)je * nm;
      if (l < nm) a.a = fmac(a.a, __ldg(pr + l), c);
      if (l + kWarp < nm) a.b = fmac(a.b, __ldg(pr + l + kWarp), c);
    }
  }
  return a;
}

// ans_i = sum_j A(i,j) x_j through the non-transposed copy (AN[j*nm + i] = A(i,j))
__device__ __forceinline__ V2 matvecN(const double *AN, const double *x, int nm) {
  const int l = lane_id();
  double s0 = 0.0, s1 = 0.0;
  for (int j = 0; j < nm; ++j) {
    const double xj = x[j];
    if (l < nm) s0 = fmac(s0, __ldg(AN + j * nm + l), xj);
    if (l + kWarp < nm) s1 = fmac(s1, __ldg(AN + j * nm + l + kWarp), xj);
  }
  return V2{s0, s1};
}

// FS q-phase wall transform (calvarnl_fs.f:171-204): symmetric, used both ways.
__device__ __forceinline__ void qwall_fs(const DevOps &op, V2 &gxx, V2 &gxy, V2 &gyx, V2 &gyy,
                                         double dnx, double dny, double *sm) {
  V2 gnx, gtx, gny, gty, gnn, gnt, gtn, gtt;
  rot_vec(gnx, gtx, gxx, gyx, dnx, dny);
  rot_vec(gny, gty, gxy, gyy, dnx, dny);
  rot_vec(gnn, gnt, gnx, gny, dnx, dny);
  rot_vec(gtn, gtt, gtx, gty, dnx, dny);
  V2 bu = reduc_gn(op, gtn, sm);
  gnn = solve_full(op, gnn);
  gnt = solve_full(op, gnt);
  bu = solve_red(op, bu);
  gtt = solve_full(op, gtt);
  gtn = reduc_inv_gn(op, bu, sm);
  rot_vec(gnx, gny, gnn, gnt, dnx, dny);
  rot_vec(gtx, gty, gtn, gtt, dnx, dny);
  rot_vec(gxx, gyx, gnx, gtx, dnx, dny);
  rot_vec(gxy, gyy, gny, gty, dnx, dny);
}

// Mass solve of a vector pair with the variant's wall projection (symmetric).
template <int VAR>
__device__ __forceinline__ void pair_solve(const DevOps &op, const DevMesh &m, int e, V2 &gx,
                                           V2 &gy, double *sm) {
  if (__ldg(m.bdl + e)) {
    if (VAR == kNS)
      wall_solve_zero(op, gx, gy, sm);
    else
      wall_solve_rot(op, gx, gy, __ldg(m.normt + 2 * e), __ldg(m.normt + 2 * e + 1), sm);
  } else {
    gx = solve_full(op, gx);
    gy = solve_full(op, gy);
  }
}

// ---------------------------------------------------------------------------
// tangent-linear quadrature-point kernel (linearisation of k_nlvol)
// ---------------------------------------------------------------------------
struct TlmSmem {
  double vin[18][kMaxModes];  // 9 base + 9 perturbation modal inputs
  double wp[8][kMaxQuad];
  double sm[kMaxModes];
};

template <int VAR>
__global__ void __launch_bounds__(64) k_nlvol_tlm(DevOps op, DevMesh m, TlmArgs a) {
  __shared__ TlmSmem sall[2];
  TlmSmem &S = sall[threadIdx.x >> 5];
  const int nm = op.nm, ng = op.ng, ne = m.ne, l = lane_id();
  const size_t fs = (size_t)ne * nm;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    const V2 uk = vload(a.su + o, nm), vk = vload(a.sv + o, nm), hh = vload(a.sh + o, nm);
    const V2 hb = vload(a.hb + o, nm), w0 = vload(a.w0 + o, nm), z0 = vload(a.z0 + o, nm);
    const V2 fc = vload(a.fc + o, nm);
    const V2 q0 = vload(a.q + o, nm), q1 = vload(a.q + fs + o, nm);
    const V2 q2 = vload(a.q + 2 * fs + o, nm), q3 = vload(a.q + 3 * fs + o, nm);
    const V2 du = vload(a.du + o, nm), dv = vload(a.dv + o, nm), dh = vload(a.dh + o, nm);
    const V2 d0 = vload(a.dq + o, nm), d1 = vload(a.dq + fs + o, nm);
    const V2 d2 = vload(a.dq + 2 * fs + o, nm), d3 = vload(a.dq + 3 * fs + o, nm);
    vstore(S.vin[0], uk, nm);
    vstore(S.vin[1], vk, nm);
    vstore(S.vin[2], q0, nm);
    vstore(S.vin[3], V2{q1.a - fc.a, q1.b - fc.b}, nm);
    vstore(S.vin[4], V2{q2.a + fc.a, q2.b + fc.b}, nm);
    vstore(S.vin[5], q3, nm);
    vstore(S.vin[6], vadd(hh, hb), nm);
    vstore(S.vin[7], V2{w0.a - a.mb0 * uk.a, w0.b - a.mb0 * uk.b}, nm);
    vstore(S.vin[8], V2{z0.a - a.mb0 * vk.a, z0.b - a.mb0 * vk.b}, nm);
    vstore(S.vin[9], du, nm);
    vstore(S.vin[10], dv, nm);
    vstore(S.vin[11], d0, nm);
    vstore(S.vin[12], d1, nm);
    vstore(S.vin[13], d2, nm);
    vstore(S.vin[14], d3, nm);
    vstore(S.vin[15], dh, nm);
    vstore(S.vin[16], vscale(du, -a.mb0), nm);
    vstore(S.vin[17], vscale(dv, -a.mb0), nm);
    __syncwarp();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int qp = l + h * kWarp;
      if (qp < ng) {
        double b[9], d[9];
#pragma unroll
        for (int f = 0; f < 9; ++f) b[f] = d[f] = 0.0;
        for (int n = 0; n < nm; ++n) {
          const double p = __ldg(op.p2 + (size_t)n * ng + qp);
#pragma unroll
          for (int f = 0; f < 9; ++f) {
            b[f] = fmac(b[f], S.vin[f][n], p);
            d[f] = fmac(d[f], S.vin[9 + f][n], p);
          }
        }
        const double w = __ldg(op.wi + qp), ih = 1.0 / b[6];
        // d(products) of calvarnl_fs.f:263-296
        S.wp[0][qp] = w * (d[0] * b[2] + b[0] * d[2]);
        S.wp[1][qp] = w * (d[1] * b[3] + b[1] * d[3]);
        S.wp[2][qp] = w * (d[0] * b[4] + b[0] * d[4]);
        S.wp[3][qp] = w * (d[1] * b[5] + b[1] * d[5]);
        S.wp[4][qp] = w * (d[0] * b[6] + b[0] * d[6]);
        S.wp[5][qp] = w * (d[1] * b[6] + b[1] * d[6]);
        S.wp[6][qp] = w * (d[7] - b[7] * ih * d[6]) * ih;
        S.wp[7][qp] = w * (d[8] - b[8] * ih * d[6]) * ih;
      }
    }
    __syncwarp();
    double X[8][2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = l + h * kWarp;
#pragma unroll
      for (int f = 0; f < 8; ++f) X[f][h] = 0.0;
      if (n < nm)
        for (int qp = 0; qp < ng; ++qp) {
          const double p = __ldg(op.p2t + (size_t)qp * nm + n);
#pragma unroll
          for (int f = 0; f < 8; ++f) X[f][h] = fmac(X[f][h], S.wp[f][qp], p);
        }
    }
    V2 uhk{X[4][0], X[4][1]}, vhk{X[5][0], X[5][1]};
    pair_solve<VAR>(op, m, e, uhk, vhk, S.sm);
    V2 gx0{-(X[0][0] + X[1][0]) + X[6][0], -(X[0][1] + X[1][1]) + X[6][1]};
    V2 gy0{-(X[2][0] + X[3][0]) + X[7][0], -(X[2][1] + X[3][1]) + X[7][1]};
    vstore(a.gx0 + o, gx0, nm);
    vstore(a.gy0 + o, gy0, nm);
    vstore(a.uh + o, uhk, nm);
    vstore(a.vh + o, vhk, nm);
    const double mu0 = a.mu0, g0 = a.g0;
    vstore(a.f + o, vlin(mu0, d0, -g0, dh), nm);
    vstore(a.f + fs + o, vscale(d1, mu0), nm);
    vstore(a.f + 2 * fs + o, vscale(d2, mu0), nm);
    vstore(a.f + 3 * fs + o, vlin(mu0, d3, -g0, dh), nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// adjoint of the tendency stage (calvarnl_fs.f:382-544)
// ---------------------------------------------------------------------------
struct TaSmem {
  double g[3][kMaxModes];
};

template <int VAR, class D = RtDims>
__global__ void __launch_bounds__(kT, adj_min_blocks<D>()) k_adj_tend_a(DevOps op_in, DevMesh m, AdjTendArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ TaSmem sall[kWB];
  __shared__ double smw[kWB][kMaxModes];
  TaSmem &S = sall[threadIdx.x >> 5];
  double *sm = smw[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  const size_t fs = (size_t)ne * nm;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
    V2 gx = vload(a.bu + o, nm), gy = vload(a.bv + o, nm), b = vload(a.bh + o, nm);
    pair_solve<VAR>(op, m, e, gx, gy, sm);
    b = solve_full(op, b);
    vstore(a.gx0b + o, gx, nm);
    vstore(a.gy0b + o, gy, nm);
    vstore(S.g[0], gx, nm);
    vstore(S.g[1], gy, nm);
    vstore(S.g[2], b, nm);
    __syncwarp();
    const V2 axg = matvecN(op.agxN, S.g[0], nm), ayg = matvecN(op.agyN, S.g[0], nm);
    const V2 bxg = matvecN(op.agxN, S.g[1], nm), byg = matvecN(op.agyN, S.g[1], nm);
    const V2 ah = matvecN(op.agxN, S.g[2], nm), bh = matvecN(op.agyN, S.g[2], nm);
    const double cby = g.by * g.detai, cay = g.ay * g.detai, cbx = g.bx * g.detai, cax = g.ax * g.detai;
    vstore(a.fb + o, vlin(-cby, axg, cay, ayg), nm);
    vstore(a.fb + fs + o, vlin(cbx, axg, -cax, ayg), nm);
    vstore(a.fb + 2 * fs + o, vlin(-cby, bxg, cay, byg), nm);
    vstore(a.fb + 3 * fs + o, vlin(cbx, bxg, -cax, byg), nm);
    vstore(a.uhb + o, vlin(cby, ah, -cay, bh), nm);
    vstore(a.vhb + o, vlin(-cbx, ah, cax, bh), nm);
    side_lift_adj(op, m, e, S.g[0], g.detai, a.lx);
    side_lift_adj(op, m, e, S.g[1], g.detai, a.ly);
    side_lift_adj(op, m, e, S.g[2], -g.detai, a.lh);
    __syncwarp();
  }
}

template <class D = RtDims>
__global__ void __launch_bounds__(kT) k_adj_tend_b(DevOps op_in, DevMesh m, AdjTendArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kWB][3][32];
  double(*S)[32] = sall[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  const size_t fs = (size_t)ne * nm;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    face_sums(op, m, e, a.lx, S[0]);
    face_sums(op, m, e, a.ly, S[1]);
    face_sums(op, m, e, a.lh, S[2]);
    __syncwarp();
    // fbdxx = fbd(fxx)*n1, fbdxy = fbd(fxy)*n2 lifted into gx; likewise gy, h
    vstore(a.fb + o, vadd(vload(a.fb + o, nm), trace_adj(op, m, e, S[0], 0, 1.0)), nm);
    vstore(a.fb + fs + o, vadd(vload(a.fb + fs + o, nm), trace_adj(op, m, e, S[0], 1, 1.0)), nm);
    vstore(a.fb + 2 * fs + o, vadd(vload(a.fb + 2 * fs + o, nm), trace_adj(op, m, e, S[1], 0, 1.0)), nm);
    vstore(a.fb + 3 * fs + o, vadd(vload(a.fb + 3 * fs + o, nm), trace_adj(op, m, e, S[1], 1, 1.0)), nm);
    vstore(a.uhb + o, vadd(vload(a.uhb + o, nm), trace_adj(op, m, e, S[2], 0, 1.0)), nm);
    vstore(a.vhb + o, vadd(vload(a.vhb + o, nm), trace_adj(op, m, e, S[2], 1, 1.0)), nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// adjoint of the quadrature-point stage (calvarnl_fs.f:243-348)
// ---------------------------------------------------------------------------
// Per-warp scratch, sized by the compile-time dimensions when there are
// some (the maximum sizes would limit the kernel to 16 resident warps per SM).
template <class D>
struct NaSmem {
  static constexpr int M = D::NC > 0 ? (D::NC + 1) * (D::NC + 2) / 2 : kMaxModes;
  static constexpr int Q = D::NC > 0 ? D::NG : kMaxQuad;
  double vin[9][M];
  double xb[8][M];
  double qb[9][Q];  // quadrature-point adjoints: U V Gxx Gxy Gyx Gyy H Wk Zk
  double sm[M];
};

template <int VAR, class D = RtDims>
__global__ void __launch_bounds__(64, 4 * adj_min_blocks<D>()) k_nlvol_adj(DevOps op_in, DevMesh m, AdjNlArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ NaSmem<D> sall[2];
  NaSmem<D> &S = sall[threadIdx.x >> 5];
  const int nm = op.nm, ng = op.ng, ne = m.ne, l = lane_id();
  const size_t fs = (size_t)ne * nm;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    const V2 uk = vload(a.su + o, nm), vk = vload(a.sv + o, nm), hh = vload(a.sh + o, nm);
    const V2 hb = vload(a.hb + o, nm), w0 = vload(a.w0 + o, nm), z0 = vload(a.z0 + o, nm);
    const V2 fc = vload(a.fc + o, nm);
    const V2 q0 = vload(a.q + o, nm), q1 = vload(a.q + fs + o, nm);
    const V2 q2 = vload(a.q + 2 * fs + o, nm), q3 = vload(a.q + 3 * fs + o, nm);
    const V2 f0 = vload(a.fb + o, nm), f1 = vload(a.fb + fs + o, nm);
    const V2 f2 = vload(a.fb + 2 * fs + o, nm), f3 = vload(a.fb + 3 * fs + o, nm);
    const V2 gx0 = vload(a.gx0b + o, nm), gy0 = vload(a.gy0b + o, nm);
    V2 uhb = vload(a.uhb + o, nm), vhb = vload(a.vhb + o, nm);
    vstore(S.vin[0], uk, nm);
    vstore(S.vin[1], vk, nm);
    vstore(S.vin[2], q0, nm);
    vstore(S.vin[3], V2{q1.a - fc.a, q1.b - fc.b}, nm);
    vstore(S.vin[4], V2{q2.a + fc.a, q2.b + fc.b}, nm);
    vstore(S.vin[5], q3, nm);
    vstore(S.vin[6], vadd(hh, hb), nm);
    vstore(S.vin[7], V2{w0.a - a.mb0 * uk.a, w0.b - a.mb0 * uk.b}, nm);
    vstore(S.vin[8], V2{z0.a - a.mb0 * vk.a, z0.b - a.mb0 * vk.b}, nm);
    // uh = W(uhk) (self-adjoint)
    pair_solve<VAR>(op, m, e, uhb, vhb, S.sm);
    const V2 ngx = vscale(gx0, -1.0), ngy = vscale(gy0, -1.0);
    vstore(S.xb[0], ngx, nm);
    vstore(S.xb[1], ngx, nm);
    vstore(S.xb[2], ngy, nm);
    vstore(S.xb[3], ngy, nm);
    vstore(S.xb[4], uhb, nm);
    vstore(S.xb[5], vhb, nm);
    vstore(S.xb[6], gx0, nm);
    vstore(S.xb[7], gy0, nm);
    __syncwarp();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int qp = l + h * kWarp;
      if (qp < ng) {
        double b[9], pb[8];
#pragma unroll
        for (int f = 0; f < 9; ++f) b[f] = 0.0;
#pragma unroll
        for (int f = 0; f < 8; ++f) pb[f] = 0.0;
        for (int n = 0; n < nm; ++n) {
          const double p = __ldg(op.p2 + (size_t)n * ng + qp);
#pragma unroll
          for (int f = 0; f < 9; ++f) b[f] = fmac(b[f], S.vin[f][n], p);
#pragma unroll
          for (int f = 0; f < 8; ++f) pb[f] = fmac(pb[f], S.xb[f][n], p);
        }
        const double w = __ldg(op.wi + qp), ih = 1.0 / b[6];
#pragma unroll
        for (int f = 0; f < 8; ++f) pb[f] *= w;  // xytospec^T
        S.qb[0][qp] = pb[0] * b[2] + pb[2] * b[4] + pb[4] * b[6];  // U
        S.qb[1][qp] = pb[1] * b[3] + pb[3] * b[5] + pb[5] * b[6];  // V
        S.qb[2][qp] = pb[0] * b[0];                                // Gxx
        S.qb[3][qp] = pb[1] * b[1];                                // Gxy
        S.qb[4][qp] = pb[2] * b[0];                                // Gyx
        S.qb[5][qp] = pb[3] * b[1];                                // Gyy
        S.qb[6][qp] = pb[4] * b[0] + pb[5] * b[1] - (pb[6] * b[7] + pb[7] * b[8]) * ih * ih;  // H
        S.qb[7][qp] = pb[6] * ih;                                  // Wk
        S.qb[8][qp] = pb[7] * ih;                                  // Zk
      }
    }
    __syncwarp();
    // spectoxy^T: modal adjoint a(n) = sum_q pi2(q,n) qb(q)
    double M[9][2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = l + h * kWarp;
#pragma unroll
      for (int f = 0; f < 9; ++f) M[f][h] = 0.0;
      if (n < nm)
        for (int qp = 0; qp < ng; ++qp) {
          const double p = __ldg(op.p2t + (size_t)qp * nm + n);
#pragma unroll
          for (int f = 0; f < 9; ++f) M[f][h] = fmac(M[f][h], S.qb[f][qp], p);
        }
    }
    const double mu0 = a.mu0, g0 = a.g0, mb0 = a.mb0;
    V2 ub{M[0][0] - mb0 * M[7][0], M[0][1] - mb0 * M[7][1]};
    V2 vb{M[1][0] - mb0 * M[8][0], M[1][1] - mb0 * M[8][1]};
    V2 hbar{M[6][0] - g0 * (f0.a + f3.a), M[6][1] - g0 * (f0.b + f3.b)};
    vstore(a.ub + o, ub, nm);
    vstore(a.vb + o, vb, nm);
    vstore(a.hbo + o, hbar, nm);
    vstore(a.qb + o, V2{M[2][0] + mu0 * f0.a, M[2][1] + mu0 * f0.b}, nm);
    vstore(a.qb + fs + o, V2{M[3][0] + mu0 * f1.a, M[3][1] + mu0 * f1.b}, nm);
    vstore(a.qb + 2 * fs + o, V2{M[4][0] + mu0 * f2.a, M[4][1] + mu0 * f2.b}, nm);
    vstore(a.qb + 3 * fs + o, V2{M[5][0] + mu0 * f3.a, M[5][1] + mu0 * f3.b}, nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// adjoint of the q-phase (calvarnl_fs.f:88-226)
// ---------------------------------------------------------------------------
template <int VAR, class D = RtDims>
__global__ void __launch_bounds__(kT, adj_min_blocks<D>()) k_adj_qphase_a(DevOps op_in, DevMesh m, AdjQArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kWB][5][kMaxModes];
  double(*S)[kMaxModes] = sall[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  const size_t fs = (size_t)ne * nm;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
    V2 gxx = vload(a.qb + o, nm), gxy = vload(a.qb + fs + o, nm);
    V2 gyx = vload(a.qb + 2 * fs + o, nm), gyy = vload(a.qb + 3 * fs + o, nm);
    if (VAR == kFS && __ldg(m.bdl + e)) {
      qwall_fs(op, gxx, gxy, gyx, gyy, __ldg(m.normt + 2 * e), __ldg(m.normt + 2 * e + 1), S[4]);
    } else {
      gxx = solve_full(op, gxx);
      gxy = solve_full(op, gxy);
      gyx = solve_full(op, gyx);
      gyy = solve_full(op, gyy);
    }
    // gxx = (by gx1 - ay gy1) detai, gxy = (-bx gx1 + ax gy1) detai, gx1 = -agx^T u ...
    const double d = g.detai;
    const V2 gx1u = vlin(d * g.by, gxx, -d * g.bx, gxy), gy1u = vlin(-d * g.ay, gxx, d * g.ax, gxy);
    const V2 gx1v = vlin(d * g.by, gyx, -d * g.bx, gyy), gy1v = vlin(-d * g.ay, gyx, d * g.ax, gyy);
    vstore(S[0], gx1u, nm);
    vstore(S[1], gy1u, nm);
    vstore(S[2], gx1v, nm);
    vstore(S[3], gy1v, nm);
    __syncwarp();
    const V2 uvol = vscale(vadd(matvecN(op.agxN, S[0], nm), matvecN(op.agyN, S[1], nm)), -1.0);
    const V2 vvol = vscale(vadd(matvecN(op.agxN, S[2], nm), matvecN(op.agyN, S[3], nm)), -1.0);
    vstore(a.ub + o, vadd(vload(a.ub + o, nm), uvol), nm);
    vstore(a.vb + o, vadd(vload(a.vb + o, nm), vvol), nm);
    __syncwarp();
    vstore(S[0], gxx, nm);
    vstore(S[1], gxy, nm);
    vstore(S[2], gyx, nm);
    vstore(S[3], gyy, nm);
    __syncwarp();
    for (int c = 0; c < 4; ++c) side_lift_adj(op, m, e, S[c], d, a.lq + (size_t)c * ne * 3 * op.ngf);
    __syncwarp();
  }
}

template <class D = RtDims>
__global__ void __launch_bounds__(kT) k_adj_qphase_b(DevOps op_in, DevMesh m, AdjQArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kWB][4][32];
  double(*S)[32] = sall[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  const size_t ls = (size_t)ne * 3 * op.ngf;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    for (int c = 0; c < 4; ++c) face_sums(op, m, e, a.lq + c * ls, S[c]);
    __syncwarp();
    // u is traced into fbdxx (n1, lifted into gxx) and fbdxy (n2, into gxy)
    V2 ut = vadd(trace_adj(op, m, e, S[0], 0, 1.0), trace_adj(op, m, e, S[1], 1, 1.0));
    V2 vt = vadd(trace_adj(op, m, e, S[2], 0, 1.0), trace_adj(op, m, e, S[3], 1, 1.0));
    vstore(a.ub + o, vadd(vload(a.ub + o, nm), ut), nm);
    vstore(a.vb + o, vadd(vload(a.vb + o, nm), vt), nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Two elements per warp for the tabulated degrees with nm <= 16 (degrees 3
// and 4): a 16-lane tile owns an element, one mode (or point) per lane, so
// the mode loops keep 15 of 16 lanes busy instead of 15 of 32.  Same
// arithmetic as the kernels above; shuffles and barriers are per tile.
// ---------------------------------------------------------------------------
namespace t16 {

constexpr int W = 16;
__device__ __forceinline__ int lane() { return threadIdx.x & (W - 1); }
__device__ __forceinline__ unsigned mask() { return 0xffffu << (threadIdx.x & 16); }
__device__ __forceinline__ void sync() { __syncwarp(mask()); }
__device__ __forceinline__ double shfl(double x, int k) { return __shfl_sync(mask(), x, k, W); }
// tile slot of this thread: in the block, in the grid, and the grid's count
__device__ __forceinline__ int bslot() { return threadIdx.x >> 4; }
__device__ __forceinline__ int gslot() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 4; }
__device__ __forceinline__ int nslot() { return (gridDim.x * blockDim.x) >> 4; }

__device__ __forceinline__ double load(const double *__restrict__ g, int n) {
  const int l = lane();
  return l < n ? g[l] : 0.0;
}
__device__ __forceinline__ void store(double *g, double v, int n) {
  if (lane() < n) g[lane()] = v;
}

// DTRSM4 (src/dtrsm1.f:47-82) on the tile, as dtrsm4 in spoc_device.cuh
__device__ __forceinline__ double dtrsm(double t, int m, const double *__restrict__ uT,
                                        const double *__restrict__ uC,
                                        const double *__restrict__ dia, int ld) {
  const int l = lane();
  for (int k = 0; k < m; ++k) {
    if (l == k) t = mul(t, __ldg(dia + k));
    const double xk = shfl(t, k);
    if (l > k && l < m) t = sub(t, mul(__ldg(uT + k * ld + l), xk));
  }
  for (int k = m - 1; k >= 0; --k) {
    if (l == k) t = mul(t, __ldg(dia + k));
    const double bk = shfl(t, k);
    if (l < k) t = sub(t, mul(bk, __ldg(uC + k * ld + l)));
  }
  return t;
}
__device__ __forceinline__ double solve_full(const DevOps &op, double b) {
  return dtrsm(b, op.nm, op.uT, op.uC, op.dia1, op.nm);
}
__device__ __forceinline__ double solve_red(const DevOps &op, double b) {
  return dtrsm(b, op.nmr, op.ulT, op.ulC, op.dia2, op.nm);
}

// reduc_gn / reduc_inv_gn (src/mat1.f:418-473) through the tile's scratch
__device__ __forceinline__ double reduc_gn(const DevOps &op, double gn, double *sm) {
  const int l = lane();
  store(sm, gn, op.nm);
  sync();
  double v = 0.0;
  if (l < op.nmr) {
    const double a = sm[__ldg(op.red_k + l)], c = sm[__ldg(op.red_i0 + l)];
    v = __ldg(op.red_sg + l) > 0 ? add(a, c) : sub(a, c);
  }
  sync();
  return v;
}
__device__ __forceinline__ double reduc_inv_gn(const DevOps &op, double gnr, double *sm) {
  const int l = lane();
  store(sm, gnr, op.nmr);
  sync();
  double v = 0.0;
  if (l < op.nm) {
    const int kind = __ldg(op.inv_kind + l);
    if (kind == 1) {
      const int a = __ldg(op.inv_a + l), cnt = __ldg(op.inv_cnt + l);
      for (int ll = 0; ll < cnt; ll += 2) v = add(v, sm[a + ll]);
      for (int ll = 1; ll < cnt; ll += 2) v = sub(v, sm[a + ll]);
    } else if (kind == 2) {
      v = sm[__ldg(op.inv_a + l)];
    }
  }
  sync();
  return v;
}
__device__ __forceinline__ void rot(double &gn, double &gt, double gx, double gy, double dnx,
                                    double dny) {
  gn = add(mul(gx, dnx), mul(gy, dny));
  gt = sub(mul(gx, dny), mul(gy, dnx));
}

template <int VAR>
__device__ __forceinline__ void pair_solve(const DevOps &op, const DevMesh &m, int e, double &gx,
                                           double &gy, double *sm) {
  if (__ldg(m.bdl + e)) {
    if (VAR == kNS) {
      double bu = reduc_gn(op, gx, sm), bv = reduc_gn(op, gy, sm);
      bu = solve_red(op, bu);
      bv = solve_red(op, bv);
      gx = reduc_inv_gn(op, bu, sm);
      gy = reduc_inv_gn(op, bv, sm);
    } else {
      const double dnx = __ldg(m.normt + 2 * e), dny = __ldg(m.normt + 2 * e + 1);
      double gn, gt;
      rot(gn, gt, gx, gy, dnx, dny);
      double bu = reduc_gn(op, gn, sm);
      bu = solve_red(op, bu);
      gt = solve_full(op, gt);
      gn = reduc_inv_gn(op, bu, sm);
      rot(gx, gy, gn, gt, dnx, dny);
    }
  } else {
    gx = solve_full(op, gx);
    gy = solve_full(op, gy);
  }
}

// ans_i = sum_j A(i,j) x_j through AN[j*nm + i] = A(i,j); x in shared memory
__device__ __forceinline__ double matvecN(const double *AN, const double *x, int nm) {
  const int l = lane();
  double s = 0.0;
  if (l < nm)
    for (int j = 0; j < nm; ++j) s = fmac(s, __ldg(AN + j * nm + l), x[j]);
  return s;
}

// the three side lifts' adjoints (as side_lift_adj)
__device__ __forceinline__ void side_lift_adj(const DevOps &op, const DevMesh &m, int e,
                                              const double *g, double coeff, double *L) {
  const int l = lane(), G = op.ngf, nm = op.nm;
  if (l < 3 * G) {
    const int k = l / G, j = l - k * G;
    const int isg = __ldg(m.its + 3 * e + k);
    const int j1 = isg > 0 ? j : G - 1 - j;
    const double sig = isg * coeff * 0.5;
    const double *p = op.picoF + (size_t)k * nm * G + j1;
    double s = 0.0;
    for (int n = 0; n < nm; ++n) s = fmac(s, __ldg(p + n * G), g[n]);
    L[(3 * (size_t)e + k) * G + j] = sig * __ldg(op.wif + j) * s;
  }
}

// face sums of the side-lift adjoints (as face_sums)
__device__ __forceinline__ void face_sums(const DevOps &op, const DevMesh &m, int e,
                                          const double *L, double *S) {
  const int l = lane(), G = op.ngf;
  if (l < 3 * G) {
    const int k = l / G, j = l - k * G;
    const int f = __ldg(m.itm + 3 * e + k);
    const int t1 = __ldg(m.tseg + 2 * f), t2 = __ldg(m.tseg + 2 * f + 1);
    double s = L[(3 * (size_t)e + k) * G + j];
    if (t2 >= 0) {
      const int nb = (t1 == e) ? t2 : t1;
      const int kn = (t1 == e) ? __ldg(m.ssit + 2 * f + 1) : __ldg(m.ssit + 2 * f);
      s += L[(3 * (size_t)nb + kn) * G + j];
    }
    S[l] = s;
  }
}

// transposed cal_flu (as trace_adj)
__device__ __forceinline__ double trace_adj(const DevOps &op, const DevMesh &m, int e,
                                            const double *S, int comp, double scale) {
  const int l = lane(), G = op.ngf, nm = op.nm;
  double a = 0.0;
  for (int k = 0; k < 3; ++k) {
    const int f = __ldg(m.itm + 3 * e + k);
    const int t1 = __ldg(m.tseg + 2 * f), t2 = __ldg(m.tseg + 2 * f + 1);
    const double w = (t2 < 0 ? 1.0 : 0.5) * __ldg(m.norm + 2 * f + comp) * scale;
    const bool first = (t1 == e);
    const double *pk = op.picoT + (size_t)k * G * nm;
    for (int j = 0; j < G; ++j) {
      const int je = first ? j : G - 1 - j;
      const double c = w * S[k * G + j];
      if (l < nm) a = fmac(a, __ldg(pk + (size_t)je * nm + l), c);
    }
  }
  return a;
}

__device__ __forceinline__ double lin(double c1, double a, double c2, double b) {
  return fmac(c1 * a, c2, b);
}

}  // namespace t16

constexpr int kT16 = 256;              // threads per block of the 16-lane-tile kernels
constexpr int kS16 = kT16 / t16::W;    // element slots per block
constexpr int kT16N = 128;             // the quadrature-point kernel (static scratch <= 48 KB)
constexpr int kS16N = kT16N / t16::W;

template <int VAR, class D>
__global__ void __launch_bounds__(kT16, 3) k16_adj_tend_a(DevOps op_in, DevMesh m, AdjTendArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sg[kS16][3][t16::W];
  __shared__ double smw[kS16][t16::W];
  double(*S)[t16::W] = sg[t16::bslot()];
  double *sm = smw[t16::bslot()];
  const int nm = op.nm, ne = m.ne;
  const size_t fs = (size_t)ne * nm;
  for (int e = t16::gslot(); e < ne; e += t16::nslot()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
    double gx = t16::load(a.bu + o, nm), gy = t16::load(a.bv + o, nm), b = t16::load(a.bh + o, nm);
    t16::pair_solve<VAR>(op, m, e, gx, gy, sm);
    b = t16::solve_full(op, b);
    t16::store(a.gx0b + o, gx, nm);
    t16::store(a.gy0b + o, gy, nm);
    t16::store(S[0], gx, nm);
    t16::store(S[1], gy, nm);
    t16::store(S[2], b, nm);
    t16::sync();
    const double axg = t16::matvecN(op.agxN, S[0], nm), ayg = t16::matvecN(op.agyN, S[0], nm);
    const double bxg = t16::matvecN(op.agxN, S[1], nm), byg = t16::matvecN(op.agyN, S[1], nm);
    const double ah = t16::matvecN(op.agxN, S[2], nm), bh = t16::matvecN(op.agyN, S[2], nm);
    const double cby = g.by * g.detai, cay = g.ay * g.detai, cbx = g.bx * g.detai, cax = g.ax * g.detai;
    t16::store(a.fb + o, t16::lin(-cby, axg, cay, ayg), nm);
    t16::store(a.fb + fs + o, t16::lin(cbx, axg, -cax, ayg), nm);
    t16::store(a.fb + 2 * fs + o, t16::lin(-cby, bxg, cay, byg), nm);
    t16::store(a.fb + 3 * fs + o, t16::lin(cbx, bxg, -cax, byg), nm);
    t16::store(a.uhb + o, t16::lin(cby, ah, -cay, bh), nm);
    t16::store(a.vhb + o, t16::lin(-cbx, ah, cax, bh), nm);
    t16::side_lift_adj(op, m, e, S[0], g.detai, a.lx);
    t16::side_lift_adj(op, m, e, S[1], g.detai, a.ly);
    t16::side_lift_adj(op, m, e, S[2], -g.detai, a.lh);
    t16::sync();
  }
}

template <class D>
__global__ void __launch_bounds__(kT16) k16_adj_tend_b(DevOps op_in, DevMesh m, AdjTendArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kS16][3][t16::W];
  double(*S)[t16::W] = sall[t16::bslot()];
  const int nm = op.nm, ne = m.ne;
  const size_t fs = (size_t)ne * nm;
  for (int e = t16::gslot(); e < ne; e += t16::nslot()) {
    const size_t o = (size_t)e * nm;
    t16::face_sums(op, m, e, a.lx, S[0]);
    t16::face_sums(op, m, e, a.ly, S[1]);
    t16::face_sums(op, m, e, a.lh, S[2]);
    t16::sync();
    t16::store(a.fb + o, t16::load(a.fb + o, nm) + t16::trace_adj(op, m, e, S[0], 0, 1.0), nm);
    t16::store(a.fb + fs + o, t16::load(a.fb + fs + o, nm) + t16::trace_adj(op, m, e, S[0], 1, 1.0), nm);
    t16::store(a.fb + 2 * fs + o, t16::load(a.fb + 2 * fs + o, nm) + t16::trace_adj(op, m, e, S[1], 0, 1.0), nm);
    t16::store(a.fb + 3 * fs + o, t16::load(a.fb + 3 * fs + o, nm) + t16::trace_adj(op, m, e, S[1], 1, 1.0), nm);
    t16::store(a.uhb + o, t16::load(a.uhb + o, nm) + t16::trace_adj(op, m, e, S[2], 0, 1.0), nm);
    t16::store(a.vhb + o, t16::load(a.vhb + o, nm) + t16::trace_adj(op, m, e, S[2], 1, 1.0), nm);
    t16::sync();
  }
}

template <class D>
struct Na16 {
  static constexpr int M = (D::NC + 1) * (D::NC + 2) / 2, Q = D::NG;
  double vin[9][M];
  double xb[8][M];
  double qb[9][Q];
  double sm[t16::W];
};

template <int VAR, class D>
__global__ void __launch_bounds__(kT16N, 4) k16_nlvol_adj(DevOps op_in, DevMesh m, AdjNlArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ Na16<D> sall[kS16N];
  Na16<D> &S = sall[t16::bslot()];
  const int nm = op.nm, ng = op.ng, ne = m.ne, l = t16::lane();
  const size_t fs = (size_t)ne * nm;
  for (int e = t16::gslot(); e < ne; e += t16::nslot()) {
    const size_t o = (size_t)e * nm;
    const double uk = t16::load(a.su + o, nm), vk = t16::load(a.sv + o, nm), hh = t16::load(a.sh + o, nm);
    const double hb = t16::load(a.hb + o, nm), w0 = t16::load(a.w0 + o, nm), z0 = t16::load(a.z0 + o, nm);
    const double fc = t16::load(a.fc + o, nm);
    const double q0 = t16::load(a.q + o, nm), q1 = t16::load(a.q + fs + o, nm);
    const double q2 = t16::load(a.q + 2 * fs + o, nm), q3 = t16::load(a.q + 3 * fs + o, nm);
    const double f0 = t16::load(a.fb + o, nm), f1 = t16::load(a.fb + fs + o, nm);
    const double f2 = t16::load(a.fb + 2 * fs + o, nm), f3 = t16::load(a.fb + 3 * fs + o, nm);
    const double gx0 = t16::load(a.gx0b + o, nm), gy0 = t16::load(a.gy0b + o, nm);
    double uhb = t16::load(a.uhb + o, nm), vhb = t16::load(a.vhb + o, nm);
    t16::store(S.vin[0], uk, nm);
    t16::store(S.vin[1], vk, nm);
    t16::store(S.vin[2], q0, nm);
    t16::store(S.vin[3], q1 - fc, nm);
    t16::store(S.vin[4], q2 + fc, nm);
    t16::store(S.vin[5], q3, nm);
    t16::store(S.vin[6], hh + hb, nm);
    t16::store(S.vin[7], w0 - a.mb0 * uk, nm);
    t16::store(S.vin[8], z0 - a.mb0 * vk, nm);
    t16::pair_solve<VAR>(op, m, e, uhb, vhb, S.sm);
    t16::store(S.xb[0], -gx0, nm);
    t16::store(S.xb[1], -gx0, nm);
    t16::store(S.xb[2], -gy0, nm);
    t16::store(S.xb[3], -gy0, nm);
    t16::store(S.xb[4], uhb, nm);
    t16::store(S.xb[5], vhb, nm);
    t16::store(S.xb[6], gx0, nm);
    t16::store(S.xb[7], gy0, nm);
    t16::sync();
    for (int qp = l; qp < ng; qp += t16::W) {
      double b[9], pb[8];
#pragma unroll
      for (int f = 0; f < 9; ++f) b[f] = 0.0;
#pragma unroll
      for (int f = 0; f < 8; ++f) pb[f] = 0.0;
      for (int n = 0; n < nm; ++n) {
        const double p = __ldg(op.p2 + (size_t)n * ng + qp);
#pragma unroll
        for (int f = 0; f < 9; ++f) b[f] = fmac(b[f], S.vin[f][n], p);
#pragma unroll
        for (int f = 0; f < 8; ++f) pb[f] = fmac(pb[f], S.xb[f][n], p);
      }
      const double w = __ldg(op.wi + qp), ih = 1.0 / b[6];
#pragma unroll
      for (int f = 0; f < 8; ++f) pb[f] *= w;
      S.qb[0][qp] = pb[0] * b[2] + pb[2] * b[4] + pb[4] * b[6];
      S.qb[1][qp] = pb[1] * b[3] + pb[3] * b[5] + pb[5] * b[6];
      S.qb[2][qp] = pb[0] * b[0];
      S.qb[3][qp] = pb[1] * b[1];
      S.qb[4][qp] = pb[2] * b[0];
      S.qb[5][qp] = pb[3] * b[1];
      S.qb[6][qp] = pb[4] * b[0] + pb[5] * b[1] - (pb[6] * b[7] + pb[7] * b[8]) * ih * ih;
      S.qb[7][qp] = pb[6] * ih;
      S.qb[8][qp] = pb[7] * ih;
    }
    t16::sync();
    double M[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) M[f] = 0.0;
    if (l < nm)
      for (int qp = 0; qp < ng; ++qp) {
        const double p = __ldg(op.p2t + (size_t)qp * nm + l);
#pragma unroll
        for (int f = 0; f < 9; ++f) M[f] = fmac(M[f], S.qb[f][qp], p);
      }
    const double mu0 = a.mu0, g0 = a.g0, mb0 = a.mb0;
    t16::store(a.ub + o, M[0] - mb0 * M[7], nm);
    t16::store(a.vb + o, M[1] - mb0 * M[8], nm);
    t16::store(a.hbo + o, M[6] - g0 * (f0 + f3), nm);
    t16::store(a.qb + o, M[2] + mu0 * f0, nm);
    t16::store(a.qb + fs + o, M[3] + mu0 * f1, nm);
    t16::store(a.qb + 2 * fs + o, M[4] + mu0 * f2, nm);
    t16::store(a.qb + 3 * fs + o, M[5] + mu0 * f3, nm);
    t16::sync();
  }
}

template <int VAR, class D>
__global__ void __launch_bounds__(kT16, 3) k16_adj_qphase_a(DevOps op_in, DevMesh m, AdjQArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kS16][5][t16::W];
  double(*S)[t16::W] = sall[t16::bslot()];
  const int nm = op.nm, ne = m.ne;
  const size_t fs = (size_t)ne * nm;
  for (int e = t16::gslot(); e < ne; e += t16::nslot()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
    double gxx = t16::load(a.qb + o, nm), gxy = t16::load(a.qb + fs + o, nm);
    double gyx = t16::load(a.qb + 2 * fs + o, nm), gyy = t16::load(a.qb + 3 * fs + o, nm);
    if (VAR == kFS && __ldg(m.bdl + e)) {
      // calvarnl_fs.f:171-204, symmetric
      const double dnx = __ldg(m.normt + 2 * e), dny = __ldg(m.normt + 2 * e + 1);
      double gnx, gtx, gny, gty, gnn, gnt, gtn, gtt;
      t16::rot(gnx, gtx, gxx, gyx, dnx, dny);
      t16::rot(gny, gty, gxy, gyy, dnx, dny);
      t16::rot(gnn, gnt, gnx, gny, dnx, dny);
      t16::rot(gtn, gtt, gtx, gty, dnx, dny);
      double bu = t16::reduc_gn(op, gtn, S[4]);
      gnn = t16::solve_full(op, gnn);
      gnt = t16::solve_full(op, gnt);
      bu = t16::solve_red(op, bu);
      gtt = t16::solve_full(op, gtt);
      gtn = t16::reduc_inv_gn(op, bu, S[4]);
      t16::rot(gnx, gny, gnn, gnt, dnx, dny);
      t16::rot(gtx, gty, gtn, gtt, dnx, dny);
      t16::rot(gxx, gyx, gnx, gtx, dnx, dny);
      t16::rot(gxy, gyy, gny, gty, dnx, dny);
    } else {
      gxx = t16::solve_full(op, gxx);
      gxy = t16::solve_full(op, gxy);
      gyx = t16::solve_full(op, gyx);
      gyy = t16::solve_full(op, gyy);
    }
    const double d = g.detai;
    t16::store(S[0], t16::lin(d * g.by, gxx, -d * g.bx, gxy), nm);
    t16::store(S[1], t16::lin(-d * g.ay, gxx, d * g.ax, gxy), nm);
    t16::store(S[2], t16::lin(d * g.by, gyx, -d * g.bx, gyy), nm);
    t16::store(S[3], t16::lin(-d * g.ay, gyx, d * g.ax, gyy), nm);
    t16::sync();
    const double uvol = -(t16::matvecN(op.agxN, S[0], nm) + t16::matvecN(op.agyN, S[1], nm));
    const double vvol = -(t16::matvecN(op.agxN, S[2], nm) + t16::matvecN(op.agyN, S[3], nm));
    t16::store(a.ub + o, t16::load(a.ub + o, nm) + uvol, nm);
    t16::store(a.vb + o, t16::load(a.vb + o, nm) + vvol, nm);
    t16::sync();
    t16::store(S[0], gxx, nm);
    t16::store(S[1], gxy, nm);
    t16::store(S[2], gyx, nm);
    t16::store(S[3], gyy, nm);
    t16::sync();
    for (int c = 0; c < 4; ++c)
      t16::side_lift_adj(op, m, e, S[c], d, a.lq + (size_t)c * ne * 3 * op.ngf);
    t16::sync();
  }
}

template <class D>
__global__ void __launch_bounds__(kT16) k16_adj_qphase_b(DevOps op_in, DevMesh m, AdjQArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kS16][4][t16::W];
  double(*S)[t16::W] = sall[t16::bslot()];
  const int nm = op.nm, ne = m.ne;
  const size_t ls = (size_t)ne * 3 * op.ngf;
  for (int e = t16::gslot(); e < ne; e += t16::nslot()) {
    const size_t o = (size_t)e * nm;
    for (int c = 0; c < 4; ++c) t16::face_sums(op, m, e, a.lq + c * ls, S[c]);
    t16::sync();
    const double ut = t16::trace_adj(op, m, e, S[0], 0, 1.0) + t16::trace_adj(op, m, e, S[1], 1, 1.0);
    const double vt = t16::trace_adj(op, m, e, S[2], 0, 1.0) + t16::trace_adj(op, m, e, S[3], 1, 1.0);
    t16::store(a.ub + o, t16::load(a.ub + o, nm) + ut, nm);
    t16::store(a.vb + o, t16::load(a.vb + o, nm) + vt, nm);
    t16::sync();
  }
}

// ---------------------------------------------------------------------------
// adjoint of the linear variant (calvar_lin.f:7-287)
// ---------------------------------------------------------------------------
template <class D = RtDims>
__global__ void __launch_bounds__(kT) k_adj_lin_a(DevOps op_in, DevMesh m, AdjLinArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kWB][3][kMaxModes];
  __shared__ double smw[kWB][kMaxModes];
  double(*S)[kMaxModes] = sall[threadIdx.x >> 5];
  double *sm = smw[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
    V2 gx = vload(a.bu + o, nm), gy = vload(a.bv + o, nm), b = vload(a.bh + o, nm);
    if (__ldg(m.bdl + e)) {
      wall_solve_rot(op, gx, gy, __ldg(m.normt + 2 * e), __ldg(m.normt + 2 * e + 1), sm);
    } else {
      gx = solve_full(op, gx);
      gy = solve_full(op, gy);
    }
    b = solve_full(op, b);
    vstore(S[0], gx, nm);
    vstore(S[1], gy, nm);
    vstore(S[2], b, nm);
    __syncwarp();
    const double cby = g.by * g.detai, cay = g.ay * g.detai, cbx = g.bx * g.detai, cax = g.ax * g.detai;
    const V2 axg = matvecN(op.agxN, S[0], nm), ayg = matvecN(op.agyN, S[0], nm);
    const V2 bxg = matvecN(op.agxN, S[1], nm), byg = matvecN(op.agyN, S[1], nm);
    const V2 ah = matvecN(op.agxN, S[2], nm), bh = matvecN(op.agyN, S[2], nm);
    // fxx = fyy = -g0 h: gx uses (agx,-by d), (agy, ay d); gy uses (agx, bx d), (agy, -ax d)
    const V2 fb = vadd(vlin(-cby, axg, cay, ayg), vlin(cbx, bxg, -cax, byg));
    vstore(a.hbo + o, vscale(fb, -a.g0), nm);
    vstore(a.ub + o, vscale(vlin(cby, ah, -cay, bh), a.hh0), nm);
    vstore(a.vb + o, vscale(vlin(-cbx, ah, cax, bh), a.hh0), nm);
    side_lift_adj(op, m, e, S[0], g.detai, a.lx);
    side_lift_adj(op, m, e, S[1], g.detai, a.ly);
    side_lift_adj(op, m, e, S[2], -g.detai, a.lh);
    __syncwarp();
  }
}

template <class D = RtDims>
__global__ void __launch_bounds__(kT) k_adj_lin_b(DevOps op_in, DevMesh m, AdjLinArgs a) {
  const DevOps op = fixed_dims<D>(op_in);
  __shared__ double sall[kWB][3][32];
  double(*S)[32] = sall[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  for (int e = wg(); e < ne; e += wc()) {
    const size_t o = (size_t)e * nm;
    face_sums(op, m, e, a.lx, S[0]);
    face_sums(op, m, e, a.ly, S[1]);
    face_sums(op, m, e, a.lh, S[2]);
    __syncwarp();
    const V2 ht = vadd(trace_adj(op, m, e, S[0], 0, 1.0), trace_adj(op, m, e, S[1], 1, 1.0));
    vstore(a.hbo + o, vadd(vload(a.hbo + o, nm), vscale(ht, -a.g0)), nm);
    vstore(a.ub + o, vadd(vload(a.ub + o, nm), trace_adj(op, m, e, S[2], 0, a.hh0)), nm);
    vstore(a.vb + o, vadd(vload(a.vb + o, nm), trace_adj(op, m, e, S[2], 1, a.hh0)), nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// element-wise helpers of the RK4 tangent-linear / adjoint steps
// ---------------------------------------------------------------------------
// out = x + c * y (n doubles)
__global__ void k_axpy(size_t n, const double *x, double c, const double *y, double *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = fma(c, y[i], x[i]);
}

// out = a*x + b*y
__global__ void k_axpby(size_t n, double a, const double *x, double b, const double *y,
                        double *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = fma(a, x[i], b * y[i]);
}

// Bookkeeping of the adjoint RK4 step after one stage adjoint sbar (3 fields,
// n values each, one launch): see AdjCombine in spoc_kernels.h.
__global__ void k_adj_combine(size_t n, AdjCombine c) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < 3 * n;
       j += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(j / n);
    const size_t i = j - (size_t)f * n;
    const double L = c.lam[f][i];
    if (c.mode == AdjCombine::kInit) {
      c.kb[f][i] = fma(c.a, L, c.b * L);
      continue;
    }
    const double sb = c.sb[f][i];
    const double acc = c.mode == AdjCombine::kFirst ? sb : fma(1.0, sb, c.acc[f][i]);
    if (c.mode == AdjCombine::kLast) {
      c.lam[f][i] = fma(1.0, acc, L);
      continue;
    }
    c.acc[f][i] = acc;
    c.kb[f][i] = fma(c.a, sb, c.b * L);
  }
}

// Observation values: obs o lies in element elem[o] with basis values
// basis[o*nm + n]; val[o] = sum_n h(elem, n) basis(n).
__global__ void k_obs_eval(int nobs, int nm, const int *elem, const double *basis, const double *h,
                           double *val) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < nobs) {
    const double *hv = h + (size_t)elem[o] * nm;
    double s = 0.0;
    for (int n = 0; n < nm; ++n) s = fma(hv[n], basis[(size_t)o * nm + n], s);
    val[o] = s;
  }
}

// Adjoint forcing of 0.5 sum_o (val_o - y_o)^2: hb(elem, n) += sum over the
// observations of that element (CSR, fixed order) of r_o basis(o, n).
__global__ void k_obs_adj(int nel, int nm, const int *el_list, const int *el_start,
                          const int *obs_of, const double *basis, const double *resid, double *hb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nel * nm) {
    const int k = i / nm, n = i - k * nm;
    double s = 0.0;
    for (int p = el_start[k]; p < el_start[k + 1]; ++p) {
      const int o = obs_of[p];
      s = fma(resid[o], basis[(size_t)o * nm + n], s);
    }
    hb[(size_t)el_list[k] * nm + n] += s;
  }
}

inline int grid_for(int ne, int sms, int wpb) {
  const int need = (ne + wpb - 1) / wpb;
  return need < sms * 8 ? need : sms * 8;
}

}  // namespace

cudaError_t launch_nlvol_tlm(int variant, const DevOps &op, const DevMesh &m, const TlmArgs &a,
                             cudaStream_t st, int sms) {
  const int grid = grid_for(m.ne, sms, 2);
  switch (variant) {
    case kFS: k_nlvol_tlm<kFS><<<grid, 64, 0, st>>>(op, m, a); break;
    case kNS: k_nlvol_tlm<kNS><<<grid, 64, 0, st>>>(op, m, a); break;
    default: k_nlvol_tlm<kINV><<<grid, 64, 0, st>>>(op, m, a); break;
  }
  return cudaGetLastError();
}

namespace {
template <class D>
constexpr bool tile16() {
  return D::NC > 0 && (D::NC + 1) * (D::NC + 2) / 2 <= t16::W && 3 * D::NGF <= t16::W;
}

template <class D, int VAR>
void adj_nl16(const DevOps &op, const DevMesh &m, const AdjTendArgs &ta, const AdjNlArgs &na,
              const AdjQArgs &qa, cudaStream_t st, int sms) {
  int g = (m.ne + kS16 - 1) / kS16;
  if (g > sms * 8) g = sms * 8;
  int gn = (m.ne + kS16N - 1) / kS16N;
  if (gn > sms * 16) gn = sms * 16;
  k16_adj_tend_a<VAR, D><<<g, kT16, 0, st>>>(op, m, ta);
  k16_adj_tend_b<D><<<g, kT16, 0, st>>>(op, m, ta);
  k16_nlvol_adj<VAR, D><<<gn, kT16N, 0, st>>>(op, m, na);
  k16_adj_qphase_a<VAR, D><<<g, kT16, 0, st>>>(op, m, qa);
  k16_adj_qphase_b<D><<<g, kT16, 0, st>>>(op, m, qa);
}

template <class D>
void adj_nl_kernels(int variant, const DevOps &op, const DevMesh &m, const AdjTendArgs &ta,
                    const AdjNlArgs &na, const AdjQArgs &qa, cudaStream_t st, int g8, int g2,
                    int sms) {
  if constexpr (tile16<D>()) {
    switch (variant) {
      case kFS: adj_nl16<D, kFS>(op, m, ta, na, qa, st, sms); return;
      case kNS: adj_nl16<D, kNS>(op, m, ta, na, qa, st, sms); return;
      default: adj_nl16<D, kINV>(op, m, ta, na, qa, st, sms); return;
    }
  }
  switch (variant) {
    case kFS:
      k_adj_tend_a<kFS, D><<<g8, kT, 0, st>>>(op, m, ta);
      k_adj_tend_b<D><<<g8, kT, 0, st>>>(op, m, ta);
      k_nlvol_adj<kFS, D><<<g2, 64, 0, st>>>(op, m, na);
      k_adj_qphase_a<kFS, D><<<g8, kT, 0, st>>>(op, m, qa);
      break;
    case kNS:
      k_adj_tend_a<kNS, D><<<g8, kT, 0, st>>>(op, m, ta);
      k_adj_tend_b<D><<<g8, kT, 0, st>>>(op, m, ta);
      k_nlvol_adj<kNS, D><<<g2, 64, 0, st>>>(op, m, na);
      k_adj_qphase_a<kNS, D><<<g8, kT, 0, st>>>(op, m, qa);
      break;
    default:
      k_adj_tend_a<kINV, D><<<g8, kT, 0, st>>>(op, m, ta);
      k_adj_tend_b<D><<<g8, kT, 0, st>>>(op, m, ta);
      k_nlvol_adj<kINV, D><<<g2, 64, 0, st>>>(op, m, na);
      k_adj_qphase_a<kINV, D><<<g8, kT, 0, st>>>(op, m, qa);
      break;
  }
  k_adj_qphase_b<D><<<g8, kT, 0, st>>>(op, m, qa);
}

template <class D>
void adj_lin_kernels(const DevOps &op, const DevMesh &m, const AdjLinArgs &a, cudaStream_t st, int g) {
  k_adj_lin_a<D><<<g, kT, 0, st>>>(op, m, a);
  k_adj_lin_b<D><<<g, kT, 0, st>>>(op, m, a);
}

template <class F>
bool with_fixed(const DevOps &op, F &&f) {
  if (op.nc == 3 && op.ng == 12 && op.ngf == 4) return f(FixDims<3, 12, 4>{}), true;
  if (op.nc == 4 && op.ng == 25 && op.ngf == 5) return f(FixDims<4, 25, 5>{}), true;
  if (op.nc == 5 && op.ng == 27 && op.ngf == 6) return f(FixDims<5, 27, 6>{}), true;
  if (op.nc == 6 && op.ng == 33 && op.ngf == 7) return f(FixDims<6, 33, 7>{}), true;
  if (op.nc == 7 && op.ng == 42 && op.ngf == 9) return f(FixDims<7, 42, 9>{}), true;
  return false;
}
}  // namespace

cudaError_t launch_adj_nl(int variant, const DevOps &op, const DevMesh &m, const AdjTendArgs &ta,
                          const AdjNlArgs &na, const AdjQArgs &qa, cudaStream_t st, int sms) {
  // k_nlvol_adj: 2-warp blocks, up to 12 resident per SM
  const int g8 = grid_for(m.ne, sms, kWB), g2 = std::min((m.ne + 1) / 2, sms * 24);
  if (!with_fixed(op, [&](auto d) { adj_nl_kernels<decltype(d)>(variant, op, m, ta, na, qa, st, g8, g2, sms); }))
    adj_nl_kernels<RtDims>(variant, op, m, ta, na, qa, st, g8, g2, sms);
  return cudaGetLastError();
}

cudaError_t launch_adj_lin(const DevOps &op, const DevMesh &m, const AdjLinArgs &a,
                           cudaStream_t st, int sms) {
  const int g = grid_for(m.ne, sms, kWB);
  if (!with_fixed(op, [&](auto d) { adj_lin_kernels<decltype(d)>(op, m, a, st, g); }))
    adj_lin_kernels<RtDims>(op, m, a, st, g);
  return cudaGetLastError();
}

cudaError_t launch_axpy(size_t n, const double *x, double c, const double *y, double *out,
                        cudaStream_t st, int sms) {
  size_t blocks = (n + 255) / 256;
  if (blocks > (size_t)sms * 16) blocks = (size_t)sms * 16;
  if (blocks < 1) blocks = 1;
  k_axpy<<<(unsigned)blocks, 256, 0, st>>>(n, x, c, y, out);
  return cudaGetLastError();
}

cudaError_t launch_axpby(size_t n, double a, const double *x, double b, const double *y,
                         double *out, cudaStream_t st, int sms) {
  size_t blocks = (n + 255) / 256;
  if (blocks > (size_t)sms * 16) blocks = (size_t)sms * 16;
  if (blocks < 1) blocks = 1;
  k_axpby<<<(unsigned)blocks, 256, 0, st>>>(n, a, x, b, y, out);
  return cudaGetLastError();
}

cudaError_t launch_adj_combine(size_t n, const AdjCombine &c, cudaStream_t st, int sms) {
  size_t blocks = (3 * n + 255) / 256;
  if (blocks > (size_t)sms * 16) blocks = (size_t)sms * 16;
  if (blocks < 1) blocks = 1;
  k_adj_combine<<<(unsigned)blocks, 256, 0, st>>>(n, c);
  return cudaGetLastError();
}

cudaError_t launch_obs_eval(int nobs, int nm, const int *elem, const double *basis,
                            const double *h, double *val, cudaStream_t st) {
  k_obs_eval<<<(nobs + 127) / 128, 128, 0, st>>>(nobs, nm, elem, basis, h, val);
  return cudaGetLastError();
}

cudaError_t launch_obs_adj(int nel, int nm, const int *el_list, const int *el_start,
                           const int *obs_of, const double *basis, const double *resid, double *hb,
                           cudaStream_t st) {
  const int n = nel * nm;
  k_obs_adj<<<(n + 127) / 128, 128, 0, st>>>(nel, nm, el_list, el_start, obs_of, basis, resid, hb);
  return cudaGetLastError();
}

}  // namespace spoc
