// FP64 kernels of the SPOC RK4 DG shallow-water right-hand side (sm_100a).
//
// One warp per element; operators are read through the read-only L1 path.
// Per right-hand side the nonlinear variants run three element kernels,
// separated by the three global dependencies of the reference
// (calvarnl_fs.f:88-101, :341-373, :487-498):
//   k_qphase  -> q = grad(u), grad(v)                  (calvarnl_fs.f:115-226)
//   k_nlvol   -> uh, vh, -adu+w1, -adv+z1, F = mu0 q - g h (:243-348)
//   k_tend    -> lifts, wall projection, mass solves, RK4 stage update (:382-544)
// The linear variant (calvar_lin.f) is a single kernel k_lin.  Face values
// are recomputed by both elements of a face with the cal_flu chain
// (src/calflu.f:22-66), so no face arrays are stored.
#include <cuda_runtime.h>

#include "spoc_device.cuh"
#include "spoc_kernels.h"

namespace spoc {

namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerBlock = kThreads / kWarp;
// k_nlvol keeps 9.2 KB of per-warp staging; 4 warps fit the static limit
constexpr int kThreadsNl = 128;
constexpr int kWarpsPerBlockNl = kThreadsNl / kWarp;

__device__ __forceinline__ int warp_global() {
  return (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}
__device__ __forceinline__ int warp_count() { return (gridDim.x * blockDim.x) >> 5; }

// Face value of a modal field at face point j of the face of side k of
// element e, by the cal_flu chain (src/calflu.f:31-62).  `coef(t, n)` returns
// coefficient n of element t.  Lanes k*ngf + j, k < 3, compute; the result is
// written to fb[k*ngf + j] (face-ordered).
template <class Coef>
__device__ __forceinline__ void face_values(const DevOps &op, const DevMesh &m, int e, Coef coef,
                                            double *fb) {
  const int l = lane_id(), G = op.ngf, nm = op.nm;
  if (l < 3 * G) {
    const int k = l / G, j = l - k * G;
    const int f = __ldg(m.itm + 3 * e + k);
    const int t1 = __ldg(m.tseg + 2 * f), t2 = __ldg(m.tseg + 2 * f + 1);
    double s = 0.0;
    if (t2 < 0) {
      const double *p = op.picoF + j;  // side 1 of the wall element
      for (int n = 0; n < nm; ++n) s = add(s, mul(coef(t1, n), __ldg(p + n * G)));
    } else {
      const int s1 = __ldg(m.ssit + 2 * f), s2 = __ldg(m.ssit + 2 * f + 1);
      const double *p1 = op.picoF + (size_t)s1 * nm * G + j;
      const double *p2 = op.picoF + (size_t)s2 * nm * G + (G - 1 - j);
      for (int n = 0; n < nm; ++n) s = add(s, mul(coef(t1, n), __ldg(p1 + n * G)));
      for (int n = 0; n < nm; ++n) s = add(s, mul(coef(t2, n), __ldg(p2 + n * G)));
      s = mul(0.5, s);
    }
    fb[l] = s;
  }
}

// fbs[l] = fb[l] * norm(c, face(l)) [* scale]
__device__ __forceinline__ void scale_face(const DevOps &op, const DevMesh &m, int e,
                                           const double *fb, double *out, int c) {
  const int l = lane_id(), G = op.ngf;
  if (l < 3 * G) {
    const int k = l / G;
    const int f = __ldg(m.itm + 3 * e + k);
    out[l] = mul(fb[l], __ldg(m.norm + 2 * f + c));
  }
}
__device__ __forceinline__ void scale_face2(const DevOps &op, const DevMesh &m, int e,
                                            const double *fb, double *out, int c, double scale) {
  const int l = lane_id(), G = op.ngf;
  if (l < 3 * G) {
    const int k = l / G;
    const int f = __ldg(m.itm + 3 * e + k);
    out[l] = mul(mul(fb[l], __ldg(m.norm + 2 * f + c)), scale);
  }
}

// tri_f (src/mat1.f:172-209): b(n) += sig_k * sum_j wif(j) * (pico(j1,n,k) * fbs(j))
__device__ __forceinline__ V2 tri_f(const DevOps &op, const DevMesh &m, int e, const double *fbs,
                                    V2 b, double coeff) {
  const int l = lane_id(), G = op.ngf, nm = op.nm;
  for (int k = 0; k < 3; ++k) {
    const int isg = __ldg(m.its + 3 * e + k);
    const int isg2 = (G + 1) * (1 - isg) / 2;
    const double sig = mul(mul((double)isg, coeff), 0.5);
    const double *pk = op.picoT + (size_t)k * G * nm;
    double a0 = 0.0, a1 = 0.0;
    for (int jj = 1; jj <= G; ++jj) {
      const int j1 = isg2 + isg * jj;  // 1-based point of this element's side
      const double fv = fbs[k * G + jj - 1], w = __ldg(op.wif + jj - 1);
      const double *pr = pk + (size_t)(j1 - 1) * nm;
      if (l < nm) a0 = add(a0, mul(w, mul(__ldg(pr + l), fv)));
      if (l + kWarp < nm) a1 = add(a1, mul(w, mul(__ldg(pr + l + kWarp), fv)));
    }
    b.a = add(b.a, mul(a0, sig));
    b.b = add(b.b, mul(a1, sig));
  }
  return b;
}

struct Geo {
  double ax, bx, ay, by, detai;
};
__device__ __forceinline__ Geo geo(const DevMesh &m, int e) {
  const double *v = m.vect + 5 * (size_t)e;
  return Geo{__ldg(v), __ldg(v + 1), __ldg(v + 2), __ldg(v + 3), __ldg(v + 4)};
}

// RK4 stage bookkeeping of src/shwwnl.f:242-284 for one field of element e.
__device__ __forceinline__ void stage_update(const StageArgs &sa, int fld, int e, int nm, V2 d) {
  const int l = lane_id();
  const size_t off = (size_t)e * nm;
  double dv[2] = {d.a, d.b};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int n = l + h * kWarp;
    if (n >= nm) continue;
    const size_t i = off + n;
    const double dd = dv[h];
    if (!isfinite(dd)) atomicOr(sa.flag, 1);
    if (sa.stage < 0) {
      sa.tend[fld][i] = dd;
      continue;
    }
    const double u0 = sa.base[fld][i];
    if (sa.stage == 0) {
      sa.acc[fld][i] = dd;
      sa.out[fld][i] = add(u0, mul(mul(sa.dt, dd), 0.5));
    } else if (sa.stage == 1) {
      sa.acc[fld][i] = add(sa.acc[fld][i], mul(2.0, dd));
      sa.out[fld][i] = add(u0, mul(mul(sa.dt, dd), 0.5));
    } else if (sa.stage == 2) {
      sa.acc[fld][i] = add(sa.acc[fld][i], mul(2.0, dd));
      sa.out[fld][i] = add(u0, mul(sa.dt, dd));
    } else {
      const double nv = add(u0, mul(sa.dt6, add(sa.acc[fld][i], dd)));
      sa.base[fld][i] = nv;
      if (sa.host[fld]) sa.host[fld][(size_t)e * sa.host_ld + n] = nv;
    }
  }
}

// ---------------------------------------------------------------------------
// q-phase: weak gradients of u and v (calvarnl_fs.f:88-226)
// ---------------------------------------------------------------------------
struct QSmem {
  double x[kMaxModes];
  double sm[kMaxModes];
  double fu[32], fv[32];
  double fxx[32], fxy[32], fyx[32], fyy[32];
};

template <int VAR>
__global__ void __launch_bounds__(kThreads) k_qphase(DevOps op, DevMesh m, const double *su,
                                                      const double *sv, double *q) {
  __shared__ QSmem smem_all[kWarpsPerBlock];
  QSmem &S = smem_all[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  const size_t fstride = (size_t)ne * nm;
  for (int e = warp_global(); e < ne; e += warp_count()) {
    const Geo g = geo(m, e);
    face_values(op, m, e, [&](int t, int n) { return __ldg(su + (size_t)t * nm + n); }, S.fu);
    face_values(op, m, e, [&](int t, int n) { return __ldg(sv + (size_t)t * nm + n); }, S.fv);
    __syncwarp();
    scale_face(op, m, e, S.fu, S.fxx, 0);
    scale_face(op, m, e, S.fu, S.fxy, 1);
    scale_face(op, m, e, S.fv, S.fyx, 0);
    scale_face(op, m, e, S.fv, S.fyy, 1);
    // u
    V2 uk = vload(su + (size_t)e * nm, nm);
    vstore(S.x, uk, nm);
    __syncwarp();
    V2 gx1 = axpy_ans(vzero(), matvecT(op.agx, S.x, nm), -1.0);
    V2 gy1 = axpy_ans(vzero(), matvecT(op.agy, S.x, nm), -1.0);
    __syncwarp();
    V2 gxx, gxy, gyx, gyy;
    gxx.a = mul(sub(mul(g.by, gx1.a), mul(g.ay, gy1.a)), g.detai);
    gxx.b = mul(sub(mul(g.by, gx1.b), mul(g.ay, gy1.b)), g.detai);
    gxy.a = mul(add(-mul(g.bx, gx1.a), mul(g.ax, gy1.a)), g.detai);
    gxy.b = mul(add(-mul(g.bx, gx1.b), mul(g.ax, gy1.b)), g.detai);
    gxx = tri_f(op, m, e, S.fxx, gxx, g.detai);
    gxy = tri_f(op, m, e, S.fxy, gxy, g.detai);
    // v
    V2 vk = vload(sv + (size_t)e * nm, nm);
    vstore(S.x, vk, nm);
    __syncwarp();
    gx1 = axpy_ans(vzero(), matvecT(op.agx, S.x, nm), -1.0);
    gy1 = axpy_ans(vzero(), matvecT(op.agy, S.x, nm), -1.0);
    __syncwarp();
    gyx.a = mul(sub(mul(g.by, gx1.a), mul(g.ay, gy1.a)), g.detai);
    gyx.b = mul(sub(mul(g.by, gx1.b), mul(g.ay, gy1.b)), g.detai);
    gyy.a = mul(add(-mul(g.bx, gx1.a), mul(g.ax, gy1.a)), g.detai);
    gyy.b = mul(add(-mul(g.bx, gx1.b), mul(g.ax, gy1.b)), g.detai);
    gyx = tri_f(op, m, e, S.fyx, gyx, g.detai);
    gyy = tri_f(op, m, e, S.fyy, gyy, g.detai);
    if (VAR == kFS && __ldg(m.bdl + e)) {
      // calvarnl_fs.f:171-204
      const double dnx = __ldg(m.normt + 2 * e), dny = __ldg(m.normt + 2 * e + 1);
      V2 gnx, gtx, gny, gty, gnn, gnt, gtn, gtt;
      rot_vec(gnx, gtx, gxx, gyx, dnx, dny);
      rot_vec(gny, gty, gxy, gyy, dnx, dny);
      rot_vec(gnn, gnt, gnx, gny, dnx, dny);
      rot_vec(gtn, gtt, gtx, gty, dnx, dny);
      V2 bu = reduc_gn(op, gtn, S.sm);
      gnn = solve_full(op, gnn);
      gnt = solve_full(op, gnt);
      bu = solve_red(op, bu);
      gtt = solve_full(op, gtt);
      gtn = reduc_inv_gn(op, bu, S.sm);
      rot_vec(gnx, gny, gnn, gnt, dnx, dny);
      rot_vec(gtx, gty, gtn, gtt, dnx, dny);
      rot_vec(gxx, gyx, gnx, gtx, dnx, dny);
      rot_vec(gxy, gyy, gny, gty, dnx, dny);
    } else {
      gxx = solve_full(op, gxx);
      gxy = solve_full(op, gxy);
      gyx = solve_full(op, gyx);
      gyy = solve_full(op, gyy);
    }
    vstore(q + 0 * fstride + (size_t)e * nm, gxx, nm);
    vstore(q + 1 * fstride + (size_t)e * nm, gxy, nm);
    vstore(q + 2 * fstride + (size_t)e * nm, gyx, nm);
    vstore(q + 3 * fstride + (size_t)e * nm, gyy, nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// nonlinear volume terms at quadrature points (calvarnl_fs.f:243-348)
// ---------------------------------------------------------------------------
struct BSmem {
  double vin[9][kMaxModes];  // modal inputs of the nine spectoxy calls
  double wp[8][kMaxQuad];    // wi * (pointwise products)
  double sm[kMaxModes];
};

template <int VAR>
__global__ void __launch_bounds__(kThreadsNl) k_nlvol(DevOps op, DevMesh m, NlArgs a) {
  __shared__ BSmem smem_all[kWarpsPerBlockNl];
  BSmem &S = smem_all[threadIdx.x >> 5];
  const int nm = op.nm, ng = op.ng, ne = m.ne, l = lane_id();
  const size_t fs = (size_t)ne * nm;
  for (int e = warp_global(); e < ne; e += warp_count()) {
    const size_t o = (size_t)e * nm;
    const V2 uk = vload(a.su + o, nm), vk = vload(a.sv + o, nm), hh = vload(a.sh + o, nm);
    const V2 hbk = vload(a.hb + o, nm), w0 = vload(a.w0 + o, nm), z0 = vload(a.z0 + o, nm);
    const V2 fc = vload(a.fc + o, nm);
    const V2 qxx = vload(a.q + 0 * fs + o, nm), qxy = vload(a.q + 1 * fs + o, nm);
    const V2 qyx = vload(a.q + 2 * fs + o, nm), qyy = vload(a.q + 3 * fs + o, nm);
    // uk,vk,hk=h+hb,wk=w-mb0 u,zk=z-mb0 v,gxx=qxx,gxy=qxy-fc,gyx=qyx+fc,gyy=qyy (:245-255)
    vstore(S.vin[0], uk, nm);
    vstore(S.vin[1], vk, nm);
    vstore(S.vin[2], qxx, nm);
    vstore(S.vin[3], V2{sub(qxy.a, fc.a), sub(qxy.b, fc.b)}, nm);
    vstore(S.vin[4], V2{add(qyx.a, fc.a), add(qyx.b, fc.b)}, nm);
    vstore(S.vin[5], qyy, nm);
    vstore(S.vin[6], V2{add(hh.a, hbk.a), add(hh.b, hbk.b)}, nm);
    vstore(S.vin[7], V2{sub(w0.a, mul(a.mb0, uk.a)), sub(w0.b, mul(a.mb0, uk.b))}, nm);
    vstore(S.vin[8], V2{sub(z0.a, mul(a.mb0, vk.a)), sub(z0.b, mul(a.mb0, vk.b))}, nm);
    __syncwarp();
    // spectoxy (src/nonlin.f:62-86) of the nine fields, lanes over points
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int qp = l + h * kWarp;
      if (qp < ng) {
        double mv[9];
#pragma unroll
        for (int f = 0; f < 9; ++f) mv[f] = 0.0;
        for (int n = 0; n < nm; ++n) {
          const double p = __ldg(op.p2 + (size_t)n * ng + qp);
#pragma unroll
          for (int f = 0; f < 9; ++f) mv[f] = add(mv[f], mul(S.vin[f][n], p));
        }
        const double w = __ldg(op.wi + qp);
        // multiply / divide (src/nonlin.f:111-133), then wi * mff of inttri2
        S.wp[0][qp] = mul(w, mul(mv[0], mv[2]));  // u * gxx   -> uux
        S.wp[1][qp] = mul(w, mul(mv[1], mv[3]));  // v * gxy   -> vuy
        S.wp[2][qp] = mul(w, mul(mv[0], mv[4]));  // u * gyx   -> uvx
        S.wp[3][qp] = mul(w, mul(mv[1], mv[5]));  // v * gyy   -> vvy
        S.wp[4][qp] = mul(w, mul(mv[0], mv[6]));  // u * H     -> uhk
        S.wp[5][qp] = mul(w, mul(mv[1], mv[6]));  // v * H     -> vhk
        S.wp[6][qp] = mul(w, __ddiv_rn(mv[7], mv[6]));  // wk / H -> w1
        S.wp[7][qp] = mul(w, __ddiv_rn(mv[8], mv[6]));  // zk / H -> z1
      }
    }
    __syncwarp();
    // xytospec (src/nonlin.f:35-57, inttri2 :91-107), lanes over modes
    double X[8][2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = l + h * kWarp;
#pragma unroll
      for (int f = 0; f < 8; ++f) X[f][h] = 0.0;
      if (n < nm) {
        for (int qp = 0; qp < ng; ++qp) {
          const double p = __ldg(op.p2t + (size_t)qp * nm + n);
#pragma unroll
          for (int f = 0; f < 8; ++f) X[f][h] = add(X[f][h], mul(S.wp[f][qp], p));
        }
      }
    }
    V2 uhk{X[4][0], X[4][1]}, vhk{X[5][0], X[5][1]};
    if (__ldg(m.bdl + e)) {
      if (VAR == kNS) {
        wall_solve_zero(op, uhk, vhk, S.sm);  // calvarnl_ns.f:249-265
      } else {
        wall_solve_rot(op, uhk, vhk, __ldg(m.normt + 2 * e), __ldg(m.normt + 2 * e + 1), S.sm);
      }
    } else {
      uhk = solve_full(op, uhk);
      vhk = solve_full(op, vhk);
    }
    // adu = uux + vuy ; adv = uvx + vvy ; gx = -adu + w1 ; gy = -adv + z1 (:324-326, :393-396)
    V2 gx0, gy0;
    gx0.a = add(-add(X[0][0], X[1][0]), X[6][0]);
    gx0.b = add(-add(X[0][1], X[1][1]), X[6][1]);
    gy0.a = add(-add(X[2][0], X[3][0]), X[7][0]);
    gy0.b = add(-add(X[2][1], X[3][1]), X[7][1]);
    vstore(a.gx0 + o, gx0, nm);
    vstore(a.gy0 + o, gy0, nm);
    vstore(a.uh + o, uhk, nm);
    vstore(a.vh + o, vhk, nm);
    // F = mu0 q - g0 h I  (:341-348)
    const double mu0 = a.mu0, g0 = a.g0;
    vstore(a.f + 0 * fs + o, V2{sub(mul(mu0, qxx.a), mul(g0, hh.a)), sub(mul(mu0, qxx.b), mul(g0, hh.b))}, nm);
    vstore(a.f + 1 * fs + o, V2{mul(mu0, qxy.a), mul(mu0, qxy.b)}, nm);
    vstore(a.f + 2 * fs + o, V2{mul(mu0, qyx.a), mul(mu0, qyx.b)}, nm);
    vstore(a.f + 3 * fs + o, V2{sub(mul(mu0, qyy.a), mul(g0, hh.a)), sub(mul(mu0, qyy.b), mul(g0, hh.b))}, nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// u, v, h tendencies and the RK4 stage update (calvarnl_fs.f:350-544)
// ---------------------------------------------------------------------------
struct CSmem {
  double fld[6][kMaxModes];  // own fxx, fxy, fyx, fyy, uh, vh
  double fb[32];
  double fs[6][32];          // fbdxx, fbdxy, fbdyx, fbdyy, fbdx, fbdy
  double sm[kMaxModes];
};

template <int VAR>
__global__ void __launch_bounds__(kThreads) k_tend(DevOps op, DevMesh m, TendArgs a, StageArgs sa) {
  __shared__ CSmem smem_all[kWarpsPerBlock];
  CSmem &S = smem_all[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  const size_t fsz = (size_t)ne * nm;
  const double *src[6] = {a.f, a.f + fsz, a.f + 2 * fsz, a.f + 3 * fsz, a.uh, a.vh};
  const int comp[6] = {0, 1, 0, 1, 0, 1};
  for (int e = warp_global(); e < ne; e += warp_count()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
#pragma unroll 1
    for (int f = 0; f < 6; ++f) {
      const double *p = src[f];
      vstore(S.fld[f], vload(p + o, nm), nm);
      face_values(op, m, e, [&](int t, int n) { return __ldg(p + (size_t)t * nm + n); }, S.fb);
      __syncwarp();
      scale_face(op, m, e, S.fb, S.fs[f], comp[f]);
      __syncwarp();
    }
    // u
    V2 gx = vload(a.gx0 + o, nm);
    gx = axpy_ans(gx, matvecT(op.agx, S.fld[0], nm), -mul(g.by, g.detai));
    gx = axpy_ans(gx, matvecT(op.agy, S.fld[0], nm), mul(g.ay, g.detai));
    gx = axpy_ans(gx, matvecT(op.agx, S.fld[1], nm), mul(g.bx, g.detai));
    gx = axpy_ans(gx, matvecT(op.agy, S.fld[1], nm), -mul(g.ax, g.detai));
    gx = tri_f(op, m, e, S.fs[0], gx, g.detai);
    gx = tri_f(op, m, e, S.fs[1], gx, g.detai);
    // v
    V2 gy = vload(a.gy0 + o, nm);
    gy = axpy_ans(gy, matvecT(op.agx, S.fld[2], nm), -mul(g.by, g.detai));
    gy = axpy_ans(gy, matvecT(op.agy, S.fld[2], nm), mul(g.ay, g.detai));
    gy = axpy_ans(gy, matvecT(op.agx, S.fld[3], nm), mul(g.bx, g.detai));
    gy = axpy_ans(gy, matvecT(op.agy, S.fld[3], nm), -mul(g.ax, g.detai));
    gy = tri_f(op, m, e, S.fs[2], gy, g.detai);
    gy = tri_f(op, m, e, S.fs[3], gy, g.detai);
    if (__ldg(m.bdl + e)) {
      if (VAR == kNS)
        wall_solve_zero(op, gx, gy, S.sm);
      else
        wall_solve_rot(op, gx, gy, __ldg(m.normt + 2 * e), __ldg(m.normt + 2 * e + 1), S.sm);
    } else {
      gx = solve_full(op, gx);
      gy = solve_full(op, gy);
    }
    // h
    V2 b = vzero();
    b = axpy_ans(b, matvecT(op.agx, S.fld[4], nm), mul(g.by, g.detai));
    b = axpy_ans(b, matvecT(op.agy, S.fld[4], nm), -mul(g.ay, g.detai));
    b = axpy_ans(b, matvecT(op.agx, S.fld[5], nm), -mul(g.bx, g.detai));
    b = axpy_ans(b, matvecT(op.agy, S.fld[5], nm), mul(g.ax, g.detai));
    b = tri_f(op, m, e, S.fs[4], b, -g.detai);
    b = tri_f(op, m, e, S.fs[5], b, -g.detai);
    b = solve_full(op, b);
    stage_update(sa, 0, e, nm, gx);
    stage_update(sa, 1, e, nm, gy);
    stage_update(sa, 2, e, nm, b);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// linear variant (calvar_lin.f:7-287), one kernel per right-hand side
// ---------------------------------------------------------------------------
struct LSmem {
  double x[kMaxModes];
  double sm[kMaxModes];
  double fb[32];
  double fxx[32], fyy[32], fx[32], fy[32];
};

__global__ void __launch_bounds__(kThreads) k_lin(DevOps op, DevMesh m, LinArgs a, StageArgs sa) {
  __shared__ LSmem smem_all[kWarpsPerBlock];
  LSmem &S = smem_all[threadIdx.x >> 5];
  const int nm = op.nm, ne = m.ne;
  const double g0 = a.g0, hh0 = a.hh0, mg0 = -g0;
  for (int e = warp_global(); e < ne; e += warp_count()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
    // fxx = fyy = -g0 h (calvar_lin.f:74-81) traced on each face (:83-106)
    face_values(op, m, e, [&](int t, int n) { return mul(mg0, __ldg(a.sh + (size_t)t * nm + n)); }, S.fb);
    __syncwarp();
    scale_face(op, m, e, S.fb, S.fxx, 0);
    scale_face(op, m, e, S.fb, S.fyy, 1);
    __syncwarp();
    face_values(op, m, e, [&](int t, int n) { return __ldg(a.su + (size_t)t * nm + n); }, S.fb);
    __syncwarp();
    scale_face2(op, m, e, S.fb, S.fx, 0, hh0);
    __syncwarp();
    face_values(op, m, e, [&](int t, int n) { return __ldg(a.sv + (size_t)t * nm + n); }, S.fb);
    __syncwarp();
    scale_face2(op, m, e, S.fb, S.fy, 1, hh0);
    const V2 hk = vload(a.sh + o, nm);
    vstore(S.x, V2{mul(mg0, hk.a), mul(mg0, hk.b)}, nm);
    __syncwarp();
    // u, v (calvar_lin.f:143-166; the terms of the zero fields fxy, fyx are
    // exact zeros and are not formed)
    const V2 ax_f = matvecT(op.agx, S.x, nm), ay_f = matvecT(op.agy, S.x, nm);
    V2 gx = axpy_ans(vzero(), ax_f, -mul(g.by, g.detai));
    gx = axpy_ans(gx, ay_f, mul(g.ay, g.detai));
    gx = tri_f(op, m, e, S.fxx, gx, g.detai);
    V2 gy = axpy_ans(vzero(), ax_f, mul(g.bx, g.detai));
    gy = axpy_ans(gy, ay_f, -mul(g.ax, g.detai));
    gy = tri_f(op, m, e, S.fyy, gy, g.detai);
    __syncwarp();
    if (__ldg(m.bdl + e)) {
      wall_solve_rot(op, gx, gy, __ldg(m.normt + 2 * e), __ldg(m.normt + 2 * e + 1), S.sm);
    } else {
      gx = solve_full(op, gx);
      gy = solve_full(op, gy);
    }
    // h (calvar_lin.f:244-280)
    const V2 uk = vload(a.su + o, nm), vk = vload(a.sv + o, nm);
    vstore(S.x, V2{mul(uk.a, hh0), mul(uk.b, hh0)}, nm);
    __syncwarp();
    V2 b = axpy_ans(vzero(), matvecT(op.agx, S.x, nm), mul(g.by, g.detai));
    b = axpy_ans(b, matvecT(op.agy, S.x, nm), -mul(g.ay, g.detai));
    __syncwarp();
    vstore(S.x, V2{mul(vk.a, hh0), mul(vk.b, hh0)}, nm);
    __syncwarp();
    b = axpy_ans(b, matvecT(op.agx, S.x, nm), -mul(g.bx, g.detai));
    b = axpy_ans(b, matvecT(op.agy, S.x, nm), mul(g.ax, g.detai));
    b = tri_f(op, m, e, S.fx, b, -g.detai);
    b = tri_f(op, m, e, S.fy, b, -g.detai);
    b = solve_full(op, b);
    stage_update(sa, 0, e, nm, gx);
    stage_update(sa, 1, e, nm, gy);
    stage_update(sa, 2, e, nm, b);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// diagnostics
// ---------------------------------------------------------------------------
// Per-element energy terms of src/energy.f:307-370: ke_e, pe_e, mass_e.
__global__ void __launch_bounds__(kThreads) k_energy_terms(DevOps op, DevMesh m, const double *su,
                                                            const double *sv, const double *sh,
                                                            const double *hb, double g0,
                                                            double *terms) {
  __shared__ double smq[kWarpsPerBlock][2][kMaxQuad];
  const int w = threadIdx.x >> 5, l = lane_id(), nm = op.nm, ng = op.ng, ne = m.ne;
  for (int e = warp_global(); e < ne; e += warp_count()) {
    const size_t o = (size_t)e * nm;
    const Geo g = geo(m, e);
    const double deta = sub(mul(g.ax, g.by), mul(g.ay, g.bx));
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int qp = l + h * kWarp;
      if (qp < ng) {
        double mu = 0.0, mv = 0.0, mh = 0.0, mhb = 0.0;
        for (int n = 0; n < nm; ++n) {
          const double p = __ldg(op.p2 + (size_t)n * ng + qp);
          const double hv = __ldg(sh + o + n);
          mu = add(mu, mul(__ldg(su + o + n), p));
          mv = add(mv, mul(__ldg(sv + o + n), p));
          mh = add(mh, mul(hv, p));
          mhb = add(mhb, mul(add(hv, __ldg(hb + o + n)), p));
        }
        const double wq = __ldg(op.wi + qp), p1 = __ldg(op.p2 + qp);
        smq[w][0][qp] = mul(mul(wq, mul(mhb, add(mul(mu, mu), mul(mv, mv)))), p1);
        smq[w][1][qp] = mul(mul(wq, mul(mh, mh)), p1);
      }
    }
    __syncwarp();
    if (l == 0) {
      double k = 0.0, p = 0.0, ms = 0.0;
      for (int qp = 0; qp < ng; ++qp) k = add(k, smq[w][0][qp]);
      for (int qp = 0; qp < ng; ++qp) p = add(p, smq[w][1][qp]);
      for (int n = 0; n < nm; ++n) ms = add(ms, mul(mul(__ldg(op.ammo1 + n), deta), __ldg(sh + o + n)));
      terms[3 * (size_t)e + 0] = mul(mul(k, deta), 0.5);
      terms[3 * (size_t)e + 1] = mul(mul(mul(p, deta), 0.5), g0);
      terms[3 * (size_t)e + 2] = ms;
    }
    __syncwarp();
  }
}

// Fixed-order (deterministic) sum of the per-element terms: one block.
__global__ void __launch_bounds__(1024) k_energy_sum(const double *terms, int ne, double *out) {
  __shared__ double part[3][1024];
  const int t = threadIdx.x;
  double s[3] = {0.0, 0.0, 0.0};
  for (int e = t; e < ne; e += blockDim.x)
    for (int c = 0; c < 3; ++c) s[c] = add(s[c], terms[3 * (size_t)e + c]);
  for (int c = 0; c < 3; ++c) part[c][t] = s[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w)
      for (int c = 0; c < 3; ++c) part[c][t] = add(part[c][t], part[c][t + w]);
    __syncthreads();
  }
  if (t == 0)
    for (int c = 0; c < 3; ++c) out[c] = part[c][0];
}

// CFL bound of src/cfl.f:15-32: min over elements and edges of
// (|edge| / nc * ra) / sqrt(g0 * hb(1,e)).  Exact (min is order-free).
__global__ void __launch_bounds__(256) k_cfl(int ne, int nc, const int *in, const double *xg,
                                             const double *yg, const double *hb, int nm, double g0,
                                             unsigned long long *out) {
  const double ra = 0.30;
  double best = 6000.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const int i1 = in[3 * e] - 1, i2 = in[3 * e + 1] - 1, i3 = in[3 * e + 2] - 1;
    double ax = sub(xg[i2], xg[i1]), ay = sub(yg[i2], yg[i1]);
    const double dd1 = mul(__ddiv_rn(__dsqrt_rn(add(mul(ax, ax), mul(ay, ay))), (double)nc), ra);
    ax = sub(xg[i3], xg[i1]);
    ay = sub(yg[i3], yg[i1]);
    const double dd2 = mul(__ddiv_rn(__dsqrt_rn(add(mul(ax, ax), mul(ay, ay))), (double)nc), ra);
    ax = sub(xg[i3], xg[i2]);
    ay = sub(yg[i3], yg[i2]);
    const double dd3 = mul(__ddiv_rn(__dsqrt_rn(add(mul(ax, ax), mul(ay, ay))), (double)nc), ra);
    const double cc0 = __dsqrt_rn(mul(g0, hb[(size_t)e * nm]));
    best = fmin(best, __ddiv_rn(dd1, cc0));
    best = fmin(best, __ddiv_rn(dd2, cc0));
    best = fmin(best, __ddiv_rn(dd3, cc0));
  }
  // positive doubles order like their bit patterns
  atomicMin(out, (unsigned long long)__double_as_longlong(best));
}

inline int grid_for(int ne, int sms, int warps_per_block = kWarpsPerBlock) {
  const int need = (ne + warps_per_block - 1) / warps_per_block;
  const int cap = sms * 8 * (kWarpsPerBlock / warps_per_block);
  return need < cap ? need : cap;
}

}  // namespace

cudaError_t launch_rhs(int variant, const DevOps &op, const DevMesh &m, const RhsBuffers &b,
                       const StageArgs &sa, cudaStream_t st, int sms, long long *launches,
                       cudaEvent_t *ev) {
  const int grid = grid_for(m.ne, sms);
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], st);
  };
  if (variant == kLIN) {
    LinArgs la{b.su, b.sv, b.sh, b.g0, b.hh0};
    if (b.sh_ready) cudaStreamWaitEvent(st, b.sh_ready, 0);
    mark(0);
    k_lin<<<grid, kThreads, 0, st>>>(op, m, la, sa);
    mark(1);
    *launches += 1;
    return cudaGetLastError();
  }
  const int gridnl = grid_for(m.ne, sms, kWarpsPerBlockNl);
  NlArgs na{b.su, b.sv, b.sh, b.hb, b.w0, b.z0, b.fc, b.q, b.gx0, b.gy0, b.uh, b.vh, b.f,
            b.mu0, b.mb0, b.g0};
  TendArgs ta{b.gx0, b.gy0, b.uh, b.vh, b.f};
  switch (variant) {
    case kFS:
      mark(0);
      k_qphase<kFS><<<grid, kThreads, 0, st>>>(op, m, b.su, b.sv, b.q);
      if (b.sh_ready) cudaStreamWaitEvent(st, b.sh_ready, 0);
      mark(1);
      k_nlvol<kFS><<<gridnl, kThreadsNl, 0, st>>>(op, m, na);
      mark(2);
      k_tend<kFS><<<grid, kThreads, 0, st>>>(op, m, ta, sa);
      mark(3);
      break;
    case kNS:
      mark(0);
      k_qphase<kNS><<<grid, kThreads, 0, st>>>(op, m, b.su, b.sv, b.q);
      if (b.sh_ready) cudaStreamWaitEvent(st, b.sh_ready, 0);
      mark(1);
      k_nlvol<kNS><<<gridnl, kThreadsNl, 0, st>>>(op, m, na);
      mark(2);
      k_tend<kNS><<<grid, kThreads, 0, st>>>(op, m, ta, sa);
      mark(3);
      break;
    default:
      mark(0);
      k_qphase<kINV><<<grid, kThreads, 0, st>>>(op, m, b.su, b.sv, b.q);
      if (b.sh_ready) cudaStreamWaitEvent(st, b.sh_ready, 0);
      mark(1);
      k_nlvol<kINV><<<gridnl, kThreadsNl, 0, st>>>(op, m, na);
      mark(2);
      k_tend<kINV><<<grid, kThreads, 0, st>>>(op, m, ta, sa);
      mark(3);
      break;
  }
  *launches += 3;
  return cudaGetLastError();
}

cudaError_t launch_qphase(int variant, const DevOps &op, const DevMesh &m, const double *su,
                          const double *sv, double *q, cudaStream_t st, int sms) {
  const int grid = grid_for(m.ne, sms);
  switch (variant) {
    case kFS: k_qphase<kFS><<<grid, kThreads, 0, st>>>(op, m, su, sv, q); break;
    case kNS: k_qphase<kNS><<<grid, kThreads, 0, st>>>(op, m, su, sv, q); break;
    default: k_qphase<kINV><<<grid, kThreads, 0, st>>>(op, m, su, sv, q); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_tend(int variant, const DevOps &op, const DevMesh &m, const TendArgs &ta,
                        const StageArgs &sa, cudaStream_t st, int sms) {
  const int grid = grid_for(m.ne, sms);
  switch (variant) {
    case kFS: k_tend<kFS><<<grid, kThreads, 0, st>>>(op, m, ta, sa); break;
    case kNS: k_tend<kNS><<<grid, kThreads, 0, st>>>(op, m, ta, sa); break;
    default: k_tend<kINV><<<grid, kThreads, 0, st>>>(op, m, ta, sa); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_lin(const DevOps &op, const DevMesh &m, const LinArgs &la, const StageArgs &sa,
                       cudaStream_t st, int sms) {
  k_lin<<<grid_for(m.ne, sms), kThreads, 0, st>>>(op, m, la, sa);
  return cudaGetLastError();
}

cudaError_t launch_energy(const DevOps &op, const DevMesh &m, const double *su, const double *sv,
                          const double *sh, const double *hb, double g0, double *terms,
                          double *out, cudaStream_t st, int sms, long long *launches) {
  k_energy_terms<<<grid_for(m.ne, sms), kThreads, 0, st>>>(op, m, su, sv, sh, hb, g0, terms);
  k_energy_sum<<<1, 1024, 0, st>>>(terms, m.ne, out);
  *launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_cfl(int ne, int nc, const int *in, const double *xg, const double *yg,
                       const double *hb, int nm, double g0, unsigned long long *out,
                       cudaStream_t st, int sms, long long *launches) {
  int grid = (ne + 255) / 256;
  if (grid > sms * 4) grid = sms * 4;
  if (grid < 1) grid = 1;
  k_cfl<<<grid, 256, 0, st>>>(ne, nc, in, xg, yg, hb, nm, g0, out);
  *launches += 1;
  return cudaGetLastError();
}

}  // namespace spoc

// ---------------------------------------------------------------------------
// FP64 pipe microbenchmark: the roofline denominator for the FP64 kernels.
// mode 0: independent DFMA chains; mode 1: separately rounded DMUL + DADD.
// ---------------------------------------------------------------------------
namespace spoc {
namespace {
template <int MODE>
__global__ void __launch_bounds__(256) k_fp64_peak(double *out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = threadIdx.x * 1e-3 + i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (MODE == 0)
        x[i] = __fma_rn(x[i], a, b);
      else
        x[i] = __dadd_rn(__dmul_rn(x[i], a), b);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += x[i];
  if (s == 12345.678) out[0] = s;  // keeps the loop live
}
// FP32 fused multiply-add chains (the arithmetic of the mixed-precision kernels).
__global__ void __launch_bounds__(256) k_fp32_peak(double *out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = threadIdx.x * 1e-3f + i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = __fmaf_rn(x[i], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += x[i];
  if (s == 12345.678f) out[0] = s;  // keeps the loop live
}
}  // namespace

cudaError_t launch_fp64_peak(int mode, int sms, int iters, double *out, cudaStream_t st) {
  const int grid = sms * 8;
  if (mode == 0)
    k_fp64_peak<0><<<grid, 256, 0, st>>>(out, iters, 0.999999, 1e-9);
  else if (mode == 1)
    k_fp64_peak<1><<<grid, 256, 0, st>>>(out, iters, 0.999999, 1e-9);
  else
    k_fp32_peak<<<grid, 256, 0, st>>>(out, iters, 0.999999f, 1e-9f);
  return cudaGetLastError();
}
}  // namespace spoc
