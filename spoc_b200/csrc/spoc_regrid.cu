// Solution-driven regridding on the device (FP64, bit-identical to the
// reference arithmetic): the trace-jump error indicator of checkconv /
// cal_conv (src/adapt.f:1122-1334), the re-projection of interpol
// (src/adapt.f:1662-1745) onto a new mesh, the wall re-projection verif_rot
// (src/shwwnl_adap.f:481-596) and the velocity-aware time step checkcfl2
// (src/cfl.f:57-140).
//
// Every sum runs in the reference order with separately rounded products
// (mul/add), and every max / min is taken with atomics on the bit patterns of
// non-negative doubles, which order like the values: the results do not
// depend on the launch shape.  The point location of interpol (interlin's
// walk from the previous point's element) is sequential and stays on the
// host; the kernel receives each quadrature point's element and reference
// coordinates.
#include <cuda_runtime.h>

#include "spoc_device.cuh"
#include "spoc_kernels.h"

namespace spoc {
namespace {

constexpr int kRT = 256;
constexpr int kRW = kRT / kWarp;

__device__ __forceinline__ int gwarp() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int nwarps() { return (gridDim.x * blockDim.x) >> 5; }

__device__ __forceinline__ void max_bits(unsigned long long *p, double v) {
  atomicMax(p, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ double bits_value(unsigned long long b) {
  return __longlong_as_double((long long)b);
}

// Legendre P_0..: one step of the recurrence of src/legendre2.f:5-30,
// P_i = ((2i-1) x P_{i-1} - (i-1) P_{i-2}) / i, as po evaluates it.
__device__ __forceinline__ double po_step(int i, double x, double p1, double p0) {
  const double a0 = (double)i, a2 = (double)(2 * i - 1), a3 = (double)(i - 1);
  return __ddiv_rn(sub(mul(mul(a2, x), p1), mul(a3, p0)), a0);
}

// ---------------------------------------------------------------------------
// checkconv (src/adapt.f:1260-1334): one warp per face, lanes over
// (field, edge point); the jump |fbdy2 - fbdy1| raises both elements' maxima.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRT) k_checkconv(DevOps op, DevMesh m, const double *su,
                                                   const double *sv, const double *sh,
                                                   unsigned long long *amax) {
  const int l = lane_id(), G = op.ngf, nm = op.nm, ne = m.ne;
  const int fld = l / G, j = l - fld * G;
  const double *a0 = fld == 0 ? su : (fld == 1 ? sv : sh);
  for (int f = gwarp(); f < m.nf; f += nwarps()) {
    const int k1 = m.tseg[2 * f], k2 = m.tseg[2 * f + 1];
    if (k2 < 0) continue;  // warp-uniform
    double dif = 0.0;
    if (fld < 3) {
      const int c1 = m.ssit[2 * f], c2 = m.ssit[2 * f + 1];
      const double *p1 = op.picoF + (size_t)c1 * nm * G + j;
      const double *p2 = op.picoF + (size_t)c2 * nm * G + (G - 1 - j);
      const double *x1 = a0 + (size_t)k1 * nm, *x2 = a0 + (size_t)k2 * nm;
      double f1 = 0.0, f2 = 0.0;
#pragma unroll 8
      for (int n = 0; n < nm; ++n) {
        f1 = add(f1, mul(__ldg(x1 + n), __ldg(p1 + (size_t)n * G)));
        f2 = add(f2, mul(__ldg(x2 + n), __ldg(p2 + (size_t)n * G)));
      }
      dif = fabs(sub(f2, f1));
    }
    // largest jump of each field over the face's points (max is exact in any
    // order), then one update per field and element
    double mx = dif;
    for (int t = 1; t < G; ++t) {
      const double v = __shfl_sync(0xffffffffu, dif, l + t < kWarp ? l + t : l);
      if (j + t < G) mx = fmax(mx, v);
    }
    if (fld < 3 && j == 0 && mx > 0.0) {  // amax(k) < dif: zero and NaN jumps leave it
      max_bits(amax + (size_t)fld * ne + k1, mx);
      max_bits(amax + (size_t)fld * ne + k2, mx);
    }
  }
}

// vmax = max_i |a0(1,i)| per field
__global__ void __launch_bounds__(kRT) k_mode0_max(int ne, int nm, const double *su,
                                                   const double *sv, const double *sh,
                                                   unsigned long long *vmax) {
  double b[3] = {0.0, 0.0, 0.0};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    b[0] = fmax(b[0], fabs(su[(size_t)e * nm]));
    b[1] = fmax(b[1], fabs(sv[(size_t)e * nm]));
    b[2] = fmax(b[2], fabs(sh[(size_t)e * nm]));
  }
  for (int f = 0; f < 3; ++f) {
    double v = b[f];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane_id() == 0) max_bits(vmax + f, v);
  }
}

// amax / vmax (0 when vmax <= 1e-6), then the cal_conv flags
// (src/adapt.f:1155-1180): fconv = some field > fac1, fderaff = all < fac2;
// sup = the largest normalised jump, deraff = some fderaff.
__global__ void __launch_bounds__(kRT) k_conv_flags(int ne, const unsigned long long *amax_bits,
                                                    const unsigned long long *vmax_bits,
                                                    double fac1, double fac2, double *amax,
                                                    int *fconv, int *fderaff,
                                                    unsigned long long *sup, int *deraff) {
  double vm[3];
  for (int f = 0; f < 3; ++f) vm[f] = bits_value(vmax_bits[f]);
  double best = 0.0;
  int any = 0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    double a[3];
    for (int f = 0; f < 3; ++f) {
      const double v = bits_value(amax_bits[(size_t)f * ne + e]);
      a[f] = vm[f] > 1.0e-6 ? __ddiv_rn(v, vm[f]) : 0.0;
      amax[(size_t)f * ne + e] = a[f];
      best = fmax(best, a[f]);
    }
    if (fconv) fconv[e] = (a[0] > fac1) || (a[1] > fac1) || (a[2] > fac1);
    const int d = (a[0] < fac2) && (a[1] < fac2) && (a[2] < fac2);
    if (fderaff) fderaff[e] = d;
    any |= d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    any |= __shfl_xor_sync(0xffffffffu, any, o);
  }
  if (lane_id() == 0) {
    max_bits(sup, best);
    if (any) atomicOr(deraff, 1);
  }
}

// ---------------------------------------------------------------------------
// interpol (src/adapt.f:1662-1745): one warp per new element.  Inherited
// elements copy their old element; the others evaluate the old expansion at
// each quadrature point (fsol, src/compare.f:203-219: sum_j b_j P_kc1(x)
// P_kc2(y), modes kc1 outer), project (xytospec + inttri2,
// src/nonlin.f:35-57, :91-107) and solve with the mass matrix (DTRSM3,
// src/dtrsm1.f:1-46, the same sweeps as DTRSM4).
// ---------------------------------------------------------------------------
struct InterpSmem {
  double mff[3][kMaxQuad];
};

// Element ids outside 1..src_ne raise bit 4 of *flag and are not read.
__global__ void __launch_bounds__(kRT) k_interpol(DevOps op, int ne_new, int src_ne,
                                                  const int *tinter, const int *pel,
                                                  const double *px, const double *py,
                                                  const double *su, const double *sv,
                                                  const double *sh, double *du, double *dv,
                                                  double *dh, int *flag) {
  __shared__ InterpSmem sall[kRW];
  InterpSmem &S = sall[threadIdx.x >> 5];
  const int l = lane_id(), nm = op.nm, ng = op.ng, nc = op.nc;
  for (int e = gwarp(); e < ne_new; e += nwarps()) {
    const size_t o = (size_t)e * nm;
    const int t = tinter[e];
    if (t < 0 || t > src_ne) {
      if (l == 0) atomicOr(flag, 4);
      continue;
    }
    if (t > 0) {
      const size_t so = (size_t)(t - 1) * nm;
      for (int n = l; n < nm; n += kWarp) {
        du[o + n] = su[so + n];
        dv[o + n] = sv[so + n];
        dh[o + n] = sh[so + n];
      }
      continue;
    }
    for (int q = l; q < ng; q += kWarp) {
      const size_t pi = (size_t)e * ng + q;
      const int k = pel[pi];
      const bool ok = k >= 1 && k <= src_ne;
      if (!ok) atomicOr(flag, 4);
      const size_t so = ok ? (size_t)(k - 1) * nm : 0;
      const double x = px[pi], y = py[pi];
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      double xa = 1.0, xb = 0.0;  // P_kc1(x), P_kc1-1(x)
      int j = 0;
      for (int kc1 = 0; kc1 <= nc; ++kc1) {
        if (kc1 == 1) {
          xb = xa;
          xa = x;
        } else if (kc1 >= 2) {
          const double pn = po_step(kc1, x, xa, xb);
          xb = xa;
          xa = pn;
        }
        double ya = 1.0, yb = 0.0;  // P_kc2(y), P_kc2-1(y)
        for (int kc2 = 0; kc2 <= nc - kc1; ++kc2, ++j) {
          if (kc2 == 1) {
            yb = ya;
            ya = y;
          } else if (kc2 >= 2) {
            const double pn = po_step(kc2, y, ya, yb);
            yb = ya;
            ya = pn;
          }
          s0 = add(s0, mul(mul(su[so + j], xa), ya));
          s1 = add(s1, mul(mul(sv[so + j], xa), ya));
          s2 = add(s2, mul(mul(sh[so + j], xa), ya));
        }
      }
      S.mff[0][q] = s0;
      S.mff[1][q] = s1;
      S.mff[2][q] = s2;
    }
    __syncwarp();
    V2 b[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      double r[2] = {0.0, 0.0};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = l + h * kWarp;
        if (n < nm) {
          double ans = 0.0;
          for (int q = 0; q < ng; ++q)
            ans = add(ans, mul(mul(__ldg(op.wi + q), S.mff[f][q]), __ldg(op.p2t + (size_t)q * nm + n)));
          r[h] = ans;
        }
      }
      b[f] = solve_full(op, V2{r[0], r[1]});
    }
    vstore(du + o, b[0], nm);
    vstore(dv + o, b[1], nm);
    vstore(dh + o, b[2], nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// verif_rot (src/shwwnl_adap.f:481-596): mass-matrix load cal_b(ammo) of u and
// v, then the interior solve, or on wall elements the rotated solve with the
// wall-vanishing sub-basis for the normal component.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRT) k_verif_rot(DevOps op, DevMesh m, double *u, double *v) {
  __shared__ double sx[kRW][2][kMaxModes];
  __shared__ double smw[kRW][kMaxModes];
  double(*X)[kMaxModes] = sx[threadIdx.x >> 5];
  double *sm = smw[threadIdx.x >> 5];
  const int nm = op.nm;
  for (int e = gwarp(); e < m.ne; e += nwarps()) {
    const size_t o = (size_t)e * nm;
    vstore(X[0], vload(u + o, nm), nm);
    vstore(X[1], vload(v + o, nm), nm);
    __syncwarp();
    V2 gx = axpy_ans(vzero(), matvecT(op.ammoT, X[0], nm), 1.0);
    V2 gy = axpy_ans(vzero(), matvecT(op.ammoT, X[1], nm), 1.0);
    if (m.bdl[e]) {
      wall_solve_rot(op, gx, gy, m.normt[2 * e], m.normt[2 * e + 1], sm);
    } else {
      gx = solve_full(op, gx);
      gy = solve_full(op, gy);
    }
    vstore(u + o, gx, nm);
    vstore(v + o, gy, nm);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// checkcfl2 (src/cfl.f:57-140) with the lattice basis of cal_pgraph
// (src/visu2.f:4-25)
// ---------------------------------------------------------------------------
// pg[p * nm + i1] = P_kc1(x_l) P_kc2(y_k), lattice point p = (k, l) in the
// order k = 1..n, l = 1..n-k+1
__global__ void k_pgraph(int nc, int n, double *pg) {
  const int nm = (nc + 1) * (nc + 2) / 2;
  const int np = n * (n + 1) / 2;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    int k = 1, r = p;
    while (r >= n - k + 1) {
      r -= n - k + 1;
      ++k;
    }
    const int ll = r + 1;
    const double y = __ddiv_rn((double)(2 * k - n - 1), (double)(n - 1));
    const double x = __ddiv_rn((double)(2 * ll - n - 1), (double)(n - 1));
    int i1 = 0;
    double xa = 1.0, xb = 0.0;
    for (int kc1 = 0; kc1 <= nc; ++kc1) {
      if (kc1 == 1) {
        xb = xa;
        xa = x;
      } else if (kc1 >= 2) {
        const double pn = po_step(kc1, x, xa, xb);
        xb = xa;
        xa = pn;
      }
      double ya = 1.0, yb = 0.0;
      for (int kc2 = 0; kc2 <= nc - kc1; ++kc2, ++i1) {
        if (kc2 == 1) {
          yb = ya;
          ya = y;
        } else if (kc2 >= 2) {
          const double pn = po_step(kc2, y, ya, yb);
          yb = ya;
          ya = pn;
        }
        pg[(size_t)p * nm + i1] = mul(xa, ya);
      }
    }
  }
}

// One warp per element, lanes over lattice points.
__global__ void __launch_bounds__(kRT) k_cfl2(int ne, int nc, int nm, int np, const double *pg,
                                              const int *in, const double *xg, const double *yg,
                                              const double *hb, const double *u, const double *v,
                                              double g0, unsigned long long *out) {
  const int l = lane_id();
  const double ra = 0.35;
  for (int e = gwarp(); e < ne; e += nwarps()) {
    const size_t o = (size_t)e * nm;
    double maxdepth = 0.0, maxvel = 0.0;
    for (int p = l; p < np; p += kWarp) {
      const double *pp = pg + (size_t)p * nm;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      for (int i1 = 0; i1 < nm; ++i1) {
        const double w = __ldg(pp + i1);
        s0 = add(s0, mul(hb[o + i1], w));
        s1 = add(s1, mul(u[o + i1], w));
        s2 = add(s2, mul(v[o + i1], w));
      }
      maxdepth = fmax(maxdepth, s0);
      maxvel = fmax(maxvel, __dsqrt_rn(add(mul(s1, s1), mul(s2, s2))));
    }
    for (int k = 16; k > 0; k >>= 1) {
      maxdepth = fmax(maxdepth, __shfl_xor_sync(0xffffffffu, maxdepth, k));
      maxvel = fmax(maxvel, __shfl_xor_sync(0xffffffffu, maxvel, k));
    }
    if (l == 0) {
      const int i1 = in[3 * e] - 1, i2 = in[3 * e + 1] - 1, i3 = in[3 * e + 2] - 1;
      double ax = sub(xg[i2], xg[i1]), ay = sub(yg[i2], yg[i1]);
      const double dd1 = mul(__ddiv_rn(__dsqrt_rn(add(mul(ax, ax), mul(ay, ay))), (double)nc), ra);
      ax = sub(xg[i3], xg[i1]);
      ay = sub(yg[i3], yg[i1]);
      const double dd2 = mul(__ddiv_rn(__dsqrt_rn(add(mul(ax, ax), mul(ay, ay))), (double)nc), ra);
      ax = sub(xg[i3], xg[i2]);
      ay = sub(yg[i3], yg[i2]);
      const double dd3 = mul(__ddiv_rn(__dsqrt_rn(add(mul(ax, ax), mul(ay, ay))), (double)nc), ra);
      const double cc0 = add(__dsqrt_rn(mul(g0, maxdepth)), maxvel);
      double best = __ddiv_rn(dd1, cc0);
      best = fmin(best, __ddiv_rn(dd2, cc0));
      best = fmin(best, __ddiv_rn(dd3, cc0));
      atomicMin(out, (unsigned long long)__double_as_longlong(best));
    }
  }
}

// ---------------------------------------------------------------------------
// Point evaluation of the modal fields (fsol, src/compare.f:203-219): one
// thread per point, the three fields at once; out[f * npts + i].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRT) k_eval_points(int nc, int nm, int ne, int npts,
                                                     const int *elem, const double *px,
                                                     const double *py, const double *su,
                                                     const double *sv, const double *sh,
                                                     double *out, int *flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x) {
    const int k = elem[i];
    if (k < 1 || k > ne) {
      atomicOr(flag, 4);
      continue;
    }
    const size_t so = (size_t)(k - 1) * nm;
    const double x = px[i], y = py[i];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, xa = 1.0, xb = 0.0;
    int j = 0;
    for (int kc1 = 0; kc1 <= nc; ++kc1) {
      if (kc1 == 1) {
        xb = xa;
        xa = x;
      } else if (kc1 >= 2) {
        const double pn = po_step(kc1, x, xa, xb);
        xb = xa;
        xa = pn;
      }
      double ya = 1.0, yb = 0.0;
      for (int kc2 = 0; kc2 <= nc - kc1; ++kc2, ++j) {
        if (kc2 == 1) {
          yb = ya;
          ya = y;
        } else if (kc2 >= 2) {
          const double pn = po_step(kc2, y, ya, yb);
          yb = ya;
          ya = pn;
        }
        s0 = add(s0, mul(mul(su[so + j], xa), ya));
        s1 = add(s1, mul(mul(sv[so + j], xa), ya));
        s2 = add(s2, mul(mul(sh[so + j], xa), ya));
      }
    }
    out[i] = s0;
    out[(size_t)npts + i] = s1;
    out[2 * (size_t)npts + i] = s2;
  }
}

// ---------------------------------------------------------------------------
// write_gra's values (src/visu2.f:86-149): for element e and lattice point p
// (k outer, l inner), the physical point and the three fields:
// out[((e * np + p) * 5 + c)], c = x, y, u, v, h.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRT) k_lattice(int ne, int nm, int n, const double *pg,
                                                 const int *in, const double *xg,
                                                 const double *yg, const double *su,
                                                 const double *sv, const double *sh,
                                                 double *out) {
  const int np = n * (n + 1) / 2;
  const size_t total = (size_t)ne * np;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(t / np), p = (int)(t - (size_t)e * np);
    int k = 1, r = p;
    while (r >= n - k + 1) {
      r -= n - k + 1;
      ++k;
    }
    const int ll = r + 1;
    const int i1 = in[3 * e] - 1, i2 = in[3 * e + 1] - 1, i3 = in[3 * e + 2] - 1;
    const double ax = mul(sub(xg[i2], xg[i1]), 0.5), bx = mul(sub(xg[i3], xg[i1]), 0.5);
    const double ay = mul(sub(yg[i2], yg[i1]), 0.5), by = mul(sub(yg[i3], yg[i1]), 0.5);
    const double xof = xg[i1], yof = yg[i1];
    const double y1 = __ddiv_rn((double)(2 * k - n - 1), (double)(n - 1));
    const double x1 = __ddiv_rn((double)(2 * ll - n - 1), (double)(n - 1));
    const double x = add(add(xof, mul(ax, add(x1, 1.0))), mul(bx, add(y1, 1.0)));
    const double y = add(add(yof, mul(ay, add(x1, 1.0))), mul(by, add(y1, 1.0)));
    const double *pp = pg + (size_t)p * nm;
    const size_t o = (size_t)e * nm;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < nm; ++j) {
      const double w = __ldg(pp + j);
      s0 = add(s0, mul(su[o + j], w));
      s1 = add(s1, mul(sv[o + j], w));
      s2 = add(s2, mul(sh[o + j], w));
    }
    double *q = out + t * 5;
    q[0] = x;
    q[1] = y;
    q[2] = s0;
    q[3] = s1;
    q[4] = s2;
  }
}

int grid_warps(int items, int sms) {
  const int need = (items + kRW - 1) / kRW;
  const int cap = sms * 8;
  return need < 1 ? 1 : (need < cap ? need : cap);
}

}  // namespace

cudaError_t launch_checkconv(const DevOps &op, const DevMesh &m, const double *su,
                             const double *sv, const double *sh, double fac1, double fac2,
                             RegridScratch s, cudaStream_t st, int sms, long long *launches) {
  cudaError_t e = cudaMemsetAsync(s.amax_bits, 0, sizeof(unsigned long long) * 3 * m.ne, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.small_bits, 0, sizeof(unsigned long long) * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.deraff, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  k_checkconv<<<grid_warps(m.nf, sms), kRT, 0, st>>>(op, m, su, sv, sh, s.amax_bits);
  int g = (m.ne + kRT - 1) / kRT;
  if (g > sms * 4) g = sms * 4;
  k_mode0_max<<<g, kRT, 0, st>>>(m.ne, op.nm, su, sv, sh, s.small_bits);
  k_conv_flags<<<g, kRT, 0, st>>>(m.ne, s.amax_bits, s.small_bits, fac1, fac2, s.amax, s.fconv,
                                  s.fderaff, s.small_bits + 3, s.deraff);
  *launches += 3;
  return cudaGetLastError();
}

cudaError_t launch_interpol(const DevOps &op, int ne_new, int src_ne, const int *tinter,
                            const int *pel, const double *px, const double *py,
                            const double *const src[3], double *const dst[3], int *flag,
                            cudaStream_t st, int sms, long long *launches) {
  k_interpol<<<grid_warps(ne_new, sms), kRT, 0, st>>>(op, ne_new, src_ne, tinter, pel, px, py,
                                                      src[0], src[1], src[2], dst[0], dst[1],
                                                      dst[2], flag);
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_verif_rot(const DevOps &op, const DevMesh &m, double *u, double *v,
                             cudaStream_t st, int sms, long long *launches) {
  k_verif_rot<<<grid_warps(m.ne, sms), kRT, 0, st>>>(op, m, u, v);
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_cfl2(int ne, int nc, int nm, int n, double *pg, const int *in,
                        const double *xg, const double *yg, const double *hb, const double *u,
                        const double *v, double g0, unsigned long long *out, cudaStream_t st,
                        int sms, long long *launches) {
  const int np = n * (n + 1) / 2;
  k_pgraph<<<(np + 127) / 128, 128, 0, st>>>(nc, n, pg);
  k_cfl2<<<grid_warps(ne, sms), kRT, 0, st>>>(ne, nc, nm, np, pg, in, xg, yg, hb, u, v, g0, out);
  *launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_eval_points(int nc, int nm, int ne, int npts, const int *elem,
                               const double *px, const double *py, const double *const f[3],
                               double *out, int *flag, cudaStream_t st, int sms,
                               long long *launches) {
  int g = (npts + kRT - 1) / kRT;
  if (g > sms * 8) g = sms * 8;
  if (g < 1) g = 1;
  k_eval_points<<<g, kRT, 0, st>>>(nc, nm, ne, npts, elem, px, py, f[0], f[1], f[2], out, flag);
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_lattice(int ne, int nc, int nm, int n, double *pg, const int *in,
                           const double *xg, const double *yg, const double *const f[3],
                           double *out, cudaStream_t st, int sms, long long *launches) {
  const int np = n * (n + 1) / 2;
  k_pgraph<<<(np + 127) / 128, 128, 0, st>>>(nc, n, pg);
  const size_t total = (size_t)ne * np;
  size_t g = (total + kRT - 1) / kRT;
  if (g > (size_t)sms * 16) g = (size_t)sms * 16;
  if (g < 1) g = 1;
  k_lattice<<<(unsigned)g, kRT, 0, st>>>(ne, nm, n, pg, in, xg, yg, f[0], f[1], f[2], out);
  *launches += 2;
  return cudaGetLastError();
}

}  // namespace spoc
