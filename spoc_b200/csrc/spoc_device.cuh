// Device-side data layout and warp helpers of the SPOC RK4 DG right-hand side.
//
// Execution model: one warp per element.  A modal vector of nm <= 64
// coefficients lives in two registers per lane (row = lane and lane + 32);
// quadrature vectors (ng <= 64) likewise; the 3*ngf <= 32 face points of an
// element map to lanes k*ngf + j.  Every dot product is accumulated in the
// reference's loop order with separately rounded products (__dmul_rn /
// __dadd_rn), so results are bit-identical to a sequential IEEE double
// evaluation of the Fortran.
#pragma once
#include <cstdint>

namespace spoc {

constexpr int kWarp = 32;
constexpr int kMaxModes = 64;   // nm
constexpr int kMaxQuad = 64;    // ng
constexpr int kMaxEdge = 10;    // ngf (3*ngf <= 32 lanes)

// Reference-element operators in the layouts the warp helpers read
// (row index fastest so lanes read consecutive addresses).
struct DevOps {
  int nc, nm, nmr, ng, ngf;
  const double *agx;    // [j*nm + i] = agx(j,i)
  const double *agy;    // [j*nm + i] = agy(j,i)
  const double *agxN;   // [i*nm + j] = agx(j,i)  (non-transposed products, adjoint)
  const double *agyN;   // [i*nm + j] = agy(j,i)
  const double *p2;     // [n*ng + q] = pi2(q,n)       (spectoxy)
  const double *p2t;    // [q*nm + n] = pi2(q,n)       (xytospec)
  const double *wi;     // [ng]
  const double *wif;    // [ngf]
  const double *picoF;  // [(s*nm + n)*ngf + j] = pico(j,n,s)  (cal_flu)
  const double *picoT;  // [(s*ngf + j)*nm + n] = pico(j,n,s)  (tri_f)
  const double *uT;     // [k*nm + i] = U(k,i)   amm factor, forward sweep
  const double *uC;     // [k*nm + i] = U(i,k)   backward sweep
  const double *dia1;   // 1/U(i,i)
  const double *ulT;    // [k*nm + i] = Ul(k,i)  amml factor (nmr x nmr, ld nm)
  const double *ulC;    // [k*nm + i] = Ul(i,k)
  const double *dia2;   // 1/Ul(i,i)
  const int *red_k;     // reduc_gn: reduced r <- gn[red_k[r]] +/- gn[red_i0[r]]
  const int *red_i0;
  const int *red_sg;    // +1 / -1
  const int *inv_kind;  // reduc_inv_gn per full mode n: 0 zero, 1 head chain, 2 copy
  const int *inv_a;     // kind 1: first reduced index; kind 2: reduced source
  const int *inv_cnt;   // kind 1: chain length
  const double *ammo1;  // ammo(j,1), for the mass diagnostic
  const double *ammoT;  // [j*nm + i] = ammo(j,i)   (cal_b with ammo, verif_rot)
  // images of the operators in the shared-memory layouts of the
  // compile-time-sized kernels (copied into shared memory whole by the bulk
  // copy engine); null where the degree has no such kernels
  const void *img_ops;  // q-phase, tendency and linear kernels
  const void *img_q;    // quadrature-point kernel
  int *flag;            // the handle's error flags (bit 2: a wait limit ran out)
};

// Mesh pointers with 0-based ids; -1 marks a wall in tseg.
struct DevMesh {
  int ne, nf;
  const int *itm;       // [e*3 + k]
  const int *its;       // [e*3 + k]
  const int *tseg;      // [f*2 + s]
  const int *ssit;      // [f*2 + s] (0-based side)
  const double *norm;   // [f*2 + c]
  const double *vect;   // [e*5 + c]
  const double *normt;  // [e*2 + c]
  const int *bdl;       // [e]
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// A modal (or quadrature) vector distributed over the warp.
struct V2 {
  double a, b;  // rows lane, lane + 32
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & (kWarp - 1); }

__device__ __forceinline__ V2 vzero() { return V2{0.0, 0.0}; }

__device__ __forceinline__ V2 vload(const double *__restrict__ g, int n) {
  const int l = lane_id();
  V2 v;
  v.a = l < n ? g[l] : 0.0;
  v.b = l + kWarp < n ? g[l + kWarp] : 0.0;
  return v;
}

__device__ __forceinline__ void vstore(double *g, V2 v, int n) {
  const int l = lane_id();
  if (l < n) g[l] = v.a;
  if (l + kWarp < n) g[l + kWarp] = v.b;
}

// Broadcast row k of a distributed vector to all lanes.
__device__ __forceinline__ double vget(V2 v, int k) {
  const double x = k < kWarp ? v.a : v.b;
  return __shfl_sync(0xffffffffu, x, k & (kWarp - 1));
}

// ans_i = sum_j op[j*nm + i] * x[j]  (cal_b inner product, src/calb2.f:86-91)
__device__ __forceinline__ V2 matvecT(const double *__restrict__ op, const double *x, int nm) {
  const int l = lane_id();
  double s0 = 0.0, s1 = 0.0;
  const bool r0 = l < nm, r1 = l + kWarp < nm;
  for (int j = 0; j < nm; ++j) {
    const double xj = x[j];
    if (r0) s0 = add(s0, mul(__ldg(op + j * nm + l), xj));
    if (r1) s1 = add(s1, mul(__ldg(op + j * nm + l + kWarp), xj));
  }
  return V2{s0, s1};
}

// b := b + ans * coeff
__device__ __forceinline__ V2 axpy_ans(V2 b, V2 ans, double coeff) {
  return V2{add(b.a, mul(ans.a, coeff)), add(b.b, mul(ans.b, coeff))};
}

// (U^T U) x = b by DTRSM4 (src/dtrsm1.f:47-82): the forward sweep is run
// column-wise (row i subtracts k = 1..i-1 in order, as the row-wise loop does),
// the backward sweep is column-wise as written.
__device__ __forceinline__ V2 dtrsm4(V2 b, int m, const double *__restrict__ uT,
                                     const double *__restrict__ uC,
                                     const double *__restrict__ dia, int ld) {
  const int l = lane_id();
  const int i0 = l, i1 = l + kWarp;
  double t0 = b.a, t1 = b.b;
  for (int k = 0; k < m; ++k) {
    // row k is complete: x_k = temp_k * diag(k)
    double xk;
    if (k < kWarp) {
      if (l == k) t0 = mul(t0, __ldg(dia + k));
      xk = __shfl_sync(0xffffffffu, t0, k);
    } else {
      if (l == k - kWarp) t1 = mul(t1, __ldg(dia + k));
      xk = __shfl_sync(0xffffffffu, t1, k - kWarp);
    }
    if (i0 > k && i0 < m) t0 = sub(t0, mul(__ldg(uT + k * ld + i0), xk));
    if (i1 > k && i1 < m) t1 = sub(t1, mul(__ldg(uT + k * ld + i1), xk));
  }
  for (int k = m - 1; k >= 0; --k) {
    double bk;
    if (k < kWarp) {
      if (l == k) t0 = mul(t0, __ldg(dia + k));
      bk = __shfl_sync(0xffffffffu, t0, k);
    } else {
      if (l == k - kWarp) t1 = mul(t1, __ldg(dia + k));
      bk = __shfl_sync(0xffffffffu, t1, k - kWarp);
    }
    if (i0 < k) t0 = sub(t0, mul(bk, __ldg(uC + k * ld + i0)));
    if (i1 < k) t1 = sub(t1, mul(bk, __ldg(uC + k * ld + i1)));
  }
  return V2{t0, t1};
}

__device__ __forceinline__ V2 solve_full(const DevOps &op, V2 b) {
  return dtrsm4(b, op.nm, op.uT, op.uC, op.dia1, op.nm);
}
__device__ __forceinline__ V2 solve_red(const DevOps &op, V2 b) {
  return dtrsm4(b, op.nmr, op.ulT, op.ulC, op.dia2, op.nm);
}

// reduc_gn (src/mat1.f:418-439): full-basis load -> wall-vanishing sub-basis
// load, gnr(r) = gn(k) +/- gn(ind0).  `sm` is a 64-double warp scratch.
__device__ __forceinline__ V2 reduc_gn(const DevOps &op, V2 gn, double *sm) {
  const int l = lane_id();
  vstore(sm, gn, op.nm);
  __syncwarp();
  V2 r = vzero();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int rr = l + h * kWarp;
    double v = 0.0;
    if (rr < op.nmr) {
      const double a = sm[__ldg(op.red_k + rr)], c = sm[__ldg(op.red_i0 + rr)];
      v = __ldg(op.red_sg + rr) > 0 ? add(a, c) : sub(a, c);
    }
    if (h == 0) r.a = v; else r.b = v;
  }
  __syncwarp();
  return r;
}

// reduc_inv_gn (src/mat1.f:445-473): sub-basis coefficients -> full basis
__device__ __forceinline__ V2 reduc_inv_gn(const DevOps &op, V2 gnr, double *sm) {
  const int l = lane_id();
  vstore(sm, gnr, op.nmr);
  __syncwarp();
  V2 out = vzero();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int n = l + h * kWarp;
    double v = 0.0;
    if (n < op.nm) {
      const int kind = __ldg(op.inv_kind + n);
      if (kind == 1) {
        const int a = __ldg(op.inv_a + n), cnt = __ldg(op.inv_cnt + n);
        v = 0.0;
        for (int ll = 0; ll < cnt; ll += 2) v = add(v, sm[a + ll]);
        for (int ll = 1; ll < cnt; ll += 2) v = sub(v, sm[a + ll]);
      } else if (kind == 2) {
        v = sm[__ldg(op.inv_a + n)];
      }
    }
    if (h == 0) out.a = v; else out.b = v;
  }
  __syncwarp();
  return out;
}

// rot_vec (src/mat1.f:478-488): gn = gx*dnx + gy*dny ; gt = gx*dny - gy*dnx
__device__ __forceinline__ void rot_vec(V2 &gn, V2 &gt, V2 gx, V2 gy, double dnx, double dny) {
  gn.a = add(mul(gx.a, dnx), mul(gy.a, dny));
  gn.b = add(mul(gx.b, dnx), mul(gy.b, dny));
  gt.a = sub(mul(gx.a, dny), mul(gy.a, dnx));
  gt.b = sub(mul(gx.b, dny), mul(gy.b, dnx));
}

// Free-slip / inviscid wall solve of a vector (gx, gy) (calvarnl_fs.f:436-459)
__device__ __forceinline__ void wall_solve_rot(const DevOps &op, V2 &gx, V2 &gy, double dnx,
                                               double dny, double *sm) {
  V2 gn, gt;
  rot_vec(gn, gt, gx, gy, dnx, dny);
  V2 bu = reduc_gn(op, gn, sm);
  bu = solve_red(op, bu);
  gt = solve_full(op, gt);
  gn = reduc_inv_gn(op, bu, sm);
  rot_vec(gx, gy, gn, gt, dnx, dny);
}

// No-slip wall solve: both components in the sub-basis (calvarnl_ns.f:404-421)
__device__ __forceinline__ void wall_solve_zero(const DevOps &op, V2 &gx, V2 &gy, double *sm) {
  V2 bu = reduc_gn(op, gx, sm), bv = reduc_gn(op, gy, sm);
  bu = solve_red(op, bu);
  bv = solve_red(op, bv);
  gx = reduc_inv_gn(op, bu, sm);
  gy = reduc_inv_gn(op, bv, sm);
}

}  // namespace spoc
