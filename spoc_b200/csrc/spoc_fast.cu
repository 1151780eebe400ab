// Compile-time-sized FP64 kernels of the SPOC RK4 DG right-hand side.
//
// Same arithmetic as spoc_kernels.cu (every sum in the reference order, every
// product separately rounded, bit-identical results), organised for
// throughput:
//   * dimensions (nm, ng, ngf) are template parameters, so every loop is
//     unrolled and every shared-memory offset is an immediate;
//   * the reference-element operators are staged once per block in shared
//     memory (persistent blocks loop over elements);
//   * the modal coefficients of the element and of its three neighbours are
//     staged with coalesced loads before the face-value chains;
//   * independent chains are batched so each lane carries several at once:
//     the mat-vecs of one kernel share their operator loads, the face values
//     of all traced fields run together, the lifts of all fields and sides
//     run together, and the mass solves of one element run together.
// One warp still handles one element; lanes map to modes, quadrature points
// or face points.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "spoc_bulk.cuh"
#include "spoc_device.cuh"
#include "spoc_kernels.h"
#include "spoc_launch.h"

// SPOC_FMA selects the arithmetic of the multiply-add chains: 0 (default)
// rounds every product separately, as the reference; 1 fuses each
// multiply-add (one rounding), which halves the FP64 instructions of the
// contractions and solves but no longer reproduces the reference bit for bit.
// This file is compiled once per setting.
#ifndef SPOC_FMA
#define SPOC_FMA 0
#endif

namespace spoc {
namespace {

#if SPOC_FMA
__device__ __forceinline__ double macc(double acc, double a, double b) { return __fma_rn(a, b, acc); }
__device__ __forceinline__ double msub(double acc, double a, double b) { return __fma_rn(-a, b, acc); }
#else
__device__ __forceinline__ double macc(double acc, double a, double b) { return add(acc, mul(a, b)); }
__device__ __forceinline__ double msub(double acc, double a, double b) { return sub(acc, mul(a, b)); }
#endif

template <int NC_, int Q_, int G_>
struct Dims {
  static constexpr int N = (NC_ + 1) * (NC_ + 2) / 2;
  static constexpr int NMR = NC_ * (NC_ + 1) / 2;
  static constexpr int Q = Q_;
  static constexpr int G = G_;
  static constexpr int R = (N + 31) / 32;    // modal rows per lane
  static constexpr int RQ = (Q + 31) / 32;   // quadrature rows per lane
  // threads per block of the tendency kernel: its per-warp scratch leaves
  // room for 6 warps at two rows per lane (two blocks per SM)
  static constexpr int TEND_THREADS = R == 1 ? 256 : 192;
  static constexpr int TRI = N * (N + 1) / 2;
  static constexpr int TRIR = NMR * (NMR + 1) / 2;
  static constexpr int LW = 32;              // lanes per element
  static_assert(3 * G <= 32, "face points must fit one warp");
  static_assert(N <= 64 && Q <= 64, "two rows per lane at most");
};

// The same sizes with two elements per warp, one per 16-lane half (degrees
// whose modes and 3 * ngf face points fit 16 lanes).  The operator layouts
// (SOps) are those of D.
template <class D>
struct Half : D {
  static constexpr int LW = 16;
  static_assert(D::N <= 16 && 3 * D::G <= 16 && D::R == 1, "one element per 16 lanes");
};
template <class D>
constexpr bool fits_half() {
  return D::N <= 16 && 3 * D::G <= 16;
}

// Packed upper-triangular factor U (row k of U is U(k, k..m-1); column k is
// U(0..k, k)).  Row k starts at k*m - k*(k-1)/2; column k at k*(k+1)/2.
__host__ __device__ constexpr int row_off(int k, int m) { return k * m - k * (k - 1) / 2; }
__host__ __device__ constexpr int col_off(int k) { return k * (k + 1) / 2; }

// Operators of the q-phase, tendency and linear kernels.
template <class Dm>
struct __align__(16) SOps {
  double agx[Dm::N * Dm::N];      // [j*N + i] = agx(j,i)
  double agy[Dm::N * Dm::N];
  double pf[3 * Dm::N * Dm::G];   // [(s*N + n)*G + j] = pico(j,n,s)
  double pt[3 * Dm::G * Dm::N];   // [(s*G + j)*N + n] = pico(j,n,s)
  double urow[Dm::TRI];           // U(k,i), i >= k, row-packed
  double ucol[Dm::TRI];           // U(i,k), i <= k, column-packed
  double lrow[Dm::TRIR];          // Ul(k,i)
  double lcol[Dm::TRIR];          // Ul(i,k)
  double dia1[Dm::N];
  double dia2[Dm::NMR > 0 ? Dm::NMR : 1];
  double wif[Dm::G];
  int red_k[Dm::NMR > 0 ? Dm::NMR : 1], red_i0[Dm::NMR > 0 ? Dm::NMR : 1],
      red_sg[Dm::NMR > 0 ? Dm::NMR : 1];
  int inv_kind[Dm::N], inv_a[Dm::N], inv_cnt[Dm::N];
};

// Operators of the quadrature-point kernel.
template <class Dm>
struct __align__(16) SOpsQ {
  double p2[Dm::N * Dm::Q];       // [n*Q + q] = pi2(q,n)
  double p2t[Dm::Q * Dm::N];      // [q*N + n] = pi2(q,n)
  double wi[Dm::Q];
  double urow[Dm::TRI];
  double ucol[Dm::TRI];
  double lrow[Dm::TRIR];
  double lcol[Dm::TRIR];
  double dia1[Dm::N];
  double dia2[Dm::NMR > 0 ? Dm::NMR : 1];
  int red_k[Dm::NMR > 0 ? Dm::NMR : 1], red_i0[Dm::NMR > 0 ? Dm::NMR : 1],
      red_sg[Dm::NMR > 0 ? Dm::NMR : 1];
  int inv_kind[Dm::N], inv_a[Dm::N], inv_cnt[Dm::N];
};

template <class Dm, class S>
__device__ void stage_solve_ops(S &s, const DevOps &op) {
  constexpr int N = Dm::N, NMR = Dm::NMR;
  const int t = threadIdx.x, nt = blockDim.x;
  for (int k = 0; k < N; ++k)
    for (int i = k + t; i < N; i += nt) s.urow[row_off(k, N) + i - k] = op.uT[k * N + i];
  for (int k = 0; k < N; ++k)
    for (int i = t; i <= k; i += nt) s.ucol[col_off(k) + i] = op.uC[k * N + i];
  for (int k = 0; k < NMR; ++k)
    for (int i = k + t; i < NMR; i += nt) s.lrow[row_off(k, NMR) + i - k] = op.ulT[k * N + i];
  for (int k = 0; k < NMR; ++k)
    for (int i = t; i <= k; i += nt) s.lcol[col_off(k) + i] = op.ulC[k * N + i];
  for (int i = t; i < N; i += nt) {
    s.dia1[i] = op.dia1[i];
    s.inv_kind[i] = op.inv_kind[i];
    s.inv_a[i] = op.inv_a[i];
    s.inv_cnt[i] = op.inv_cnt[i];
  }
  for (int i = t; i < NMR; i += nt) {
    s.dia2[i] = op.dia2[i];
    s.red_k[i] = op.red_k[i];
    s.red_i0[i] = op.red_i0[i];
    s.red_sg[i] = op.red_sg[i];
  }
}

template <class Dm>
__device__ void stage_ops(SOps<Dm> &s, const DevOps &op) {
  constexpr int N = Dm::N, G = Dm::G;
  const int t = threadIdx.x, nt = blockDim.x;
  for (int i = t; i < N * N; i += nt) {
    s.agx[i] = op.agx[i];
    s.agy[i] = op.agy[i];
  }
  for (int i = t; i < 3 * N * G; i += nt) {
    s.pf[i] = op.picoF[i];
    s.pt[i] = op.picoT[i];
  }
  for (int i = t; i < G; i += nt) s.wif[i] = op.wif[i];
  stage_solve_ops<Dm>(s, op);
}

template <class Dm>
__device__ void stage_ops_q(SOpsQ<Dm> &s, const DevOps &op) {
  constexpr int N = Dm::N, Q = Dm::Q;
  const int t = threadIdx.x, nt = blockDim.x;
  for (int i = t; i < N * Q; i += nt) {
    s.p2[i] = op.p2[i];
    s.p2t[i] = op.p2t[i];
  }
  for (int i = t; i < Q; i += nt) s.wi[i] = op.wi[i];
  stage_solve_ops<Dm>(s, op);
}

__device__ __forceinline__ int warp_in_block() { return threadIdx.x >> 5; }
__device__ __forceinline__ int warp_global() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int warp_count() { return (gridDim.x * blockDim.x) >> 5; }

// Lanes of one element: the whole warp (LW = 32), or a 16-lane half of it for
// degrees whose modes and face points fit 16 lanes (two elements per warp).
template <int LW>
__device__ __forceinline__ int tile_lane() {
  if constexpr (LW == 32) return lane_id(); else return lane_id() & (LW - 1);
}
template <int LW>
__device__ __forceinline__ unsigned tile_mask() {
  if constexpr (LW == 32) return 0xffffffffu;
  else return ((1u << LW) - 1) << (lane_id() & ~(LW - 1));
}

// ---------------------------------------------------------------------------
// warp building blocks (lanes over modes unless stated otherwise)
// ---------------------------------------------------------------------------

// own field: lanes load v[e*N + i] into sm[i]
template <class Dm>
__device__ __forceinline__ void load_vec(double *sm, const double *__restrict__ g, int e) {
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int r = 0; r < Dm::R; ++r) {
    const int i = l + Dm::LW * r;
    if (i < Dm::N) sm[i] = g[(size_t)e * Dm::N + i];
  }
}

template <class Dm>
__device__ __forceinline__ void load_reg(double (&x)[Dm::R], const double *__restrict__ g, int e) {
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int r = 0; r < Dm::R; ++r) {
    const int i = l + Dm::LW * r;
    x[r] = i < Dm::N ? g[(size_t)e * Dm::N + i] : 0.0;
  }
}

template <class Dm>
__device__ __forceinline__ void store_reg(double *g, const double (&x)[Dm::R], int e) {
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int r = 0; r < Dm::R; ++r) {
    const int i = l + Dm::LW * r;
    if (i < Dm::N) g[(size_t)e * Dm::N + i] = x[r];
  }
}

template <class Dm>
__device__ __forceinline__ void reg_to_sm(double *sm, const double (&x)[Dm::R]) {
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int r = 0; r < Dm::R; ++r) {
    const int i = l + Dm::LW * r;
    if (i < Dm::N) sm[i] = x[r];
  }
}

// Neighbour across each side k of element e (-1 for a wall) and whether e is
// tseg(1) of that face.
struct Sides {
  int face[3], nb[3];
  bool first[3];
};
__device__ __forceinline__ Sides sides_of(const DevMesh &m, int e) {
  Sides s;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int f = __ldg(m.itm + 3 * e + k);
    const int t1 = __ldg(m.tseg + 2 * f), t2 = __ldg(m.tseg + 2 * f + 1);
    s.face[k] = f;
    s.first[k] = (t1 == e);
    s.nb[k] = s.first[k] ? t2 : t1;
  }
  return s;
}

// Neighbour buffers hold side k's NF fields at nb + k * nb_stride: NF*N
// doubles and the least padding (an even number of doubles, keeping 16-byte
// pairs aligned) that puts the three sides' entries a face loop reads at once
// in different shared-memory bank groups (unpadded, NF*N = 168 doubles is a
// multiple of 128 bytes: a 3-way conflict on every neighbour load).
__host__ __device__ constexpr bool nb_banks_apart(int s) {
  // 16-byte groups (8 per 128 bytes) of offsets 0, s, 2s doubles
  return (s % 2) ? (s % 16 != 0 && (2 * s) % 16 != 0)
                 : ((s / 2) % 8 != 0 && s % 8 != 0 && (s / 2) % 8 != s % 8);
}
template <class Dm, int NF>
__host__ __device__ constexpr int nb_stride() {
  const int base = NF * Dm::N;
  for (int pad = 0; pad < 16; pad += 2)
    if (nb_banks_apart(base + pad)) return base + pad;
  return base;
}

// Stage NF fields of the three neighbours: nb[k*nb_stride + f*N + i].
template <class Dm, int NF, class Fetch>
__device__ __forceinline__ void stage_neighbours(const Sides &sd, double *nb, Fetch fetch) {
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int t = sd.nb[k];
    if (t < 0) continue;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int r = 0; r < Dm::R; ++r) {
        const int i = l + Dm::LW * r;
        if (i < Dm::N) nb[k * nb_stride<Dm, NF>() + f * Dm::N + i] = fetch(f, t, i);
      }
  }
}

// Asynchronous copy of one double from global to shared memory (LDGSTS: no
// register round trip, the warp keeps computing while the copy is in flight).
__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
// Waits for every copy this thread has issued.
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Start the copies of NF fields of element e and of its three neighbours into
// own[f*N + i] and nb[k*nb_stride + f*N + i] (the layouts of load_vec and
// stage_neighbours); field f is read from fields[f].  The buffers must not be
// read until cp_async_wait_all() and a __syncwarp().
template <class Dm, int NF>
__device__ __forceinline__ void prefetch_element(const double *const (&fields)[NF], int e,
                                                 const Sides &sd, double *own, double *nb) {
  const int l = lane_id();
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int r = 0; r < Dm::R; ++r) {
      const int i = l + 32 * r;
      if (i < Dm::N) cp_async8(own + f * Dm::N + i, fields[f] + (size_t)e * Dm::N + i);
    }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int t = sd.nb[k];
    if (t < 0) continue;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int r = 0; r < Dm::R; ++r) {
        const int i = l + 32 * r;
        if (i < Dm::N)
          cp_async8(nb + k * nb_stride<Dm, NF>() + f * Dm::N + i, fields[f] + (size_t)t * Dm::N + i);
      }
  }
}

// The copies of prefetch_element, made by the bulk-copy (TMA) engine where
// a coefficient row is a whole number of 16-byte units (even N): lane r
// issues row r (the element's NF rows, then NF rows per existing neighbour),
// all completing on the warp's mbarrier; at odd N the per-value cp.async
// copies of prefetch_element.  Rows land in the same layout either way.
template <class Dm, int NF>
struct RowCopy {
  static constexpr bool kBulk = Dm::N % 2 == 0;
  uint64_t *bar;
  uint32_t phase;
  __device__ __forceinline__ void init(uint64_t *b) {
    bar = b;
    phase = 0;
    if (kBulk && lane_id() == 0) {
      tc::mbar_init(bar, 1);
      tc::fence_mbar_init();
    }
    __syncwarp();
  }
  __device__ __forceinline__ void issue(const double *const (&fields)[NF], int e, const Sides &sd,
                                        double *own, double *nb) {
    if constexpr (kBulk) {
      constexpr uint32_t RB = Dm::N * sizeof(double);
      const int have[3] = {sd.nb[0] >= 0, sd.nb[1] >= 0, sd.nb[2] >= 0};
      const int rows = NF * (1 + have[0] + have[1] + have[2]);
      const int l = lane_id();
      if (l == 0) bulk::arrive_expect_tx(bar, (uint32_t)rows * RB);
      __syncwarp();
      if (l < rows) {
        const int slot = l / NF;  // 0: the element, then the existing neighbours in side order
        const int f = l - slot * NF;
        const double *src = fields[f] + (size_t)e * Dm::N;
        double *dst = own + f * Dm::N;
        if (slot > 0) {
          // side of the slot-th existing neighbour
          const int k = (slot == 1) ? (have[0] ? 0 : have[1] ? 1 : 2)
                      : (slot == 2) ? ((have[0] && have[1]) ? 1 : 2)
                                    : 2;
          src = fields[f] + (size_t)sd.nb[k] * Dm::N;
          dst = nb + k * nb_stride<Dm, NF>() + f * Dm::N;
        }
        bulk::copy_g2s(dst, src, RB, bar);
      }
    } else {
      prefetch_element<Dm, NF>(fields, e, sd, own, nb);
    }
  }
  // The element's NF rows and the records of its three faces (rec doubles
  // each, from frec + face * rec into fdst + k * rec): bulk copies at even N
  // (lanes 0..NF-1 the rows, NF..NF+2 the records; rec * 8 a multiple of
  // 16), else 8-byte cp.async copies spread over the lanes.
  __device__ __forceinline__ void issue_own_faces(const double *const (&fields)[NF], int e,
                                                  const Sides &sd, double *own,
                                                  const double *frec, double *fdst, int rec) {
    if constexpr (!kBulk) {
      const int l = lane_id();
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int r = 0; r < Dm::R; ++r) {
          const int i = l + 32 * r;
          if (i < Dm::N) cp_async8(own + f * Dm::N + i, fields[f] + (size_t)e * Dm::N + i);
        }
      for (int i = l; i < 3 * rec; i += 32) {
        const int k = i / rec, j = i - k * rec;
        const int face = k == 0 ? sd.face[0] : (k == 1 ? sd.face[1] : sd.face[2]);
        cp_async8(fdst + i, frec + (size_t)face * rec + j);
      }
      return;
    }
    constexpr uint32_t RB = Dm::N * sizeof(double);
    const int l = lane_id();
    if (l == 0) bulk::arrive_expect_tx(bar, NF * RB + 3u * (uint32_t)rec * sizeof(double));
    __syncwarp();
    if (l < NF) {
      bulk::copy_g2s(own + l * Dm::N, fields[l] + (size_t)e * Dm::N, RB, bar);
    } else if (l < NF + 3) {
      const int k = l - NF;
      bulk::copy_g2s(fdst + k * rec, frec + (size_t)sd.face[k] * rec, (uint32_t)rec * sizeof(double),
                     bar);
    }
  }
  // Waits for the rows of the last issue(); false when the wait limit ran
  // out (bit 2 of *flag set, after one more bounded wait for the copies).
  __device__ __forceinline__ bool wait(int *flag) {
    if constexpr (kBulk) {
      const bool ok = tc::mbar_wait(bar, phase, bulk::kWaitLimit);
      if (!ok) {
        if (lane_id() == 0 && flag) atomicOr(flag, 2);
        tc::mbar_wait(bar, phase, bulk::kWaitLimit);
      }
      phase ^= 1;
      return __all_sync(0xffffffffu, ok);
    } else {
      cp_async_wait_all();
      return true;
    }
  }
};

// Face values of NF fields by the cal_flu chain (src/calflu.f:31-62): lane
// k*G + j computes point j of the face of side k; fb[f*32 + k*G + j].
template <class Dm, int NF>
__device__ __forceinline__ void face_values(const double *pf, const DevMesh &m, const Sides &sd,
                                            const double *own, const double *nb, double *fb) {
  constexpr int N = Dm::N, G = Dm::G;
  const int l = tile_lane<Dm::LW>();
  if (l < 3 * G) {
    const int k = l / G, j = l - k * G;
    const int f = sd.face[k];
    double acc[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q) acc[q] = 0.0;
    if (sd.nb[k] < 0) {
      const double *p = pf + j;  // wall faces are traced on side 1 of their element
#pragma unroll
      for (int n = 0; n < N; ++n) {
        const double pv = p[n * G];
#pragma unroll
        for (int q = 0; q < NF; ++q) acc[q] = macc(acc[q], own[q * N + n], pv);
      }
    } else {
      const double *nbk = nb + k * nb_stride<Dm, NF>();
      const double *a1 = sd.first[k] ? own : nbk;
      const double *a2 = sd.first[k] ? nbk : own;
      const int s1 = __ldg(m.ssit + 2 * f), s2 = __ldg(m.ssit + 2 * f + 1);
      const double *p1 = pf + s1 * N * G + j;
      const double *p2 = pf + s2 * N * G + (G - 1 - j);
      // the chain over side 1's modes, then side 2's; with an even mode count
      // the coefficients come in 16-byte pairs (same operations, same order)
      auto chain = [&](const double *a, const double *p) {
        if constexpr (N % 2 == 0) {
#pragma unroll
          for (int n = 0; n < N; n += 2) {
            const double pv0 = p[n * G], pv1 = p[(n + 1) * G];
#pragma unroll
            for (int q = 0; q < NF; ++q) {
              const double2 c = *reinterpret_cast<const double2 *>(a + q * N + n);
              acc[q] = macc(acc[q], c.x, pv0);
              acc[q] = macc(acc[q], c.y, pv1);
            }
          }
        } else {
#pragma unroll
          for (int n = 0; n < N; ++n) {
            const double pv = p[n * G];
#pragma unroll
            for (int q = 0; q < NF; ++q) acc[q] = macc(acc[q], a[q * N + n], pv);
          }
        }
      };
      chain(a1, p1);
      chain(a2, p2);
#pragma unroll
      for (int q = 0; q < NF; ++q) acc[q] = mul(0.5, acc[q]);
    }
#pragma unroll
    for (int q = 0; q < NF; ++q) fb[q * 32 + l] = acc[q];
  }
}

// ax[f] = agx^T x_f, bx[f] = agy^T x_f for NF smem vectors x_f = X + f*XS
template <class Dm, int NF>
__device__ __forceinline__ void matvec2(const double *A, const double *B, const double *X, int XS,
                                        double (&ax)[NF][Dm::R], double (&bx)[NF][Dm::R]) {
  constexpr int N = Dm::N, R = Dm::R;
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int r = 0; r < R; ++r) ax[f][r] = bx[f][r] = 0.0;
  auto step = [&](int j, const double (&xv)[NF]) {
    double a[R], b[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = l + Dm::LW * r;
      a[r] = (i < N) ? A[j * N + i] : 0.0;
      b[r] = (i < N) ? B[j * N + i] : 0.0;
    }
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        ax[f][r] = macc(ax[f][r], a[r], xv[f]);
        bx[f][r] = macc(bx[f][r], b[r], xv[f]);
      }
  };
  // with an even mode count (XS == N, 16-byte aligned vectors) the inputs
  // come in 16-byte pairs; the operations and their order are unchanged
  if constexpr (N % 2 == 0) {
#pragma unroll
    for (int j = 0; j < N; j += 2) {
      double x0[NF], x1[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double2 c = *reinterpret_cast<const double2 *>(X + f * XS + j);
        x0[f] = c.x;
        x1[f] = c.y;
      }
      step(j, x0);
      step(j + 1, x1);
    }
  } else {
#pragma unroll
    for (int j = 0; j < N; ++j) {
      double x0[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) x0[f] = X[f * XS + j];
      step(j, x0);
    }
  }
}

// b := b + ans * c (cal_b epilogue, src/calb2.f:91)
template <int R>
__device__ __forceinline__ void axpy(double (&b)[R], const double (&ans)[R], double c) {
#pragma unroll
  for (int r = 0; r < R; ++r) b[r] = macc(b[r], ans[r], c);
}

// Lift sums of tri_f (src/mat1.f:189-206) for NF face-value sets:
// t[f][k][r] = sum_j wif(j) * (pico(j1,n,k) * fb[f*32 + k*G + j]).
template <class Dm, int NF>
__device__ __forceinline__ void lift_sums(const SOps<Dm> &s, const int (&isg)[3], const double *fb,
                                          double (&t)[NF][3][Dm::R]) {
  constexpr int N = Dm::N, G = Dm::G, R = Dm::R;
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int isg2 = (G + 1) * (1 - isg[k]) / 2;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int r = 0; r < R; ++r) t[f][k][r] = 0.0;
#pragma unroll
    for (int jj = 1; jj <= G; ++jj) {
      const int j1 = isg2 + isg[k] * jj;
      const double w = s.wif[jj - 1];
      const double *pr = s.pt + (k * G + j1 - 1) * N;
      double p[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = l + Dm::LW * r;
        p[r] = i < N ? pr[i] : 0.0;
      }
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double fv = fb[f * 32 + k * G + jj - 1];
#pragma unroll
        for (int r = 0; r < R; ++r) t[f][k][r] = macc(t[f][k][r], w, mul(p[r], fv));
      }
    }
  }
}

// b := b + t_k * sig_k, k = 1..3, sig_k = (isg_k * coeff) * 0.5
template <int R>
__device__ __forceinline__ void apply_lift(double (&b)[R], const double (&t)[3][R],
                                           const int (&isg)[3], double coeff) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double sig = mul(mul((double)isg[k], coeff), 0.5);
#pragma unroll
    for (int r = 0; r < R; ++r) b[r] = macc(b[r], t[k][r], sig);
  }
}

// S simultaneous DTRSM4 solves (src/dtrsm1.f:47-82) of size M with a packed
// factor; rows i = lane + 32 r.
template <int M, int R, int S, int LW = 32>
__device__ __forceinline__ void solve_batch(double (&t)[S][R], const double *row, const double *col,
                                            const double *dia) {
  const int l = tile_lane<LW>();
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const int kl = k % LW, kr = k / LW;
    const double d = dia[k];
    double xk[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      if (l == kl) t[s][kr] = mul(t[s][kr], d);
      xk[s] = __shfl_sync(tile_mask<LW>(), t[s][kr], kl, LW);
    }
    const double *u = row + row_off(k, M) - k;  // u[i] = U(k,i)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = l + LW * r;
      if (i > k && i < M) {
        const double uk = u[i];
#pragma unroll
        for (int s = 0; s < S; ++s) t[s][r] = msub(t[s][r], uk, xk[s]);
      }
    }
  }
#pragma unroll
  for (int k = M - 1; k >= 0; --k) {
    const int kl = k % LW, kr = k / LW;
    const double d = dia[k];
    double bk[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      if (l == kl) t[s][kr] = mul(t[s][kr], d);
      bk[s] = __shfl_sync(tile_mask<LW>(), t[s][kr], kl, LW);
    }
    const double *u = col + col_off(k);  // u[i] = U(i,k)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = l + LW * r;
      if (i < k) {
        const double uk = u[i];
#pragma unroll
        for (int s = 0; s < S; ++s) t[s][r] = msub(t[s][r], bk[s], uk);
      }
    }
  }
}

template <class Dm, class Ops, int S>
__device__ __forceinline__ void solve_full_b(const Ops &s, double (&t)[S][Dm::R]) {
  solve_batch<Dm::N, Dm::R, S, Dm::LW>(t, s.urow, s.ucol, s.dia1);
}
template <class Dm, class Ops, int S>
__device__ __forceinline__ void solve_red_b(const Ops &s, double (&t)[S][Dm::R]) {
  solve_batch<Dm::NMR, Dm::R, S, Dm::LW>(t, s.lrow, s.lcol, s.dia2);
}

// reduc_gn (src/mat1.f:418-439) through a warp scratch vector
template <class Dm, class Ops>
__device__ __forceinline__ void reduc(const Ops &s, const double (&gn)[Dm::R], double (&r)[Dm::R],
                                      double *sm) {
  const int l = tile_lane<Dm::LW>();
  reg_to_sm<Dm>(sm, gn);
  __syncwarp(tile_mask<Dm::LW>());
#pragma unroll
  for (int h = 0; h < Dm::R; ++h) {
    const int rr = l + Dm::LW * h;
    double v = 0.0;
    if (rr < Dm::NMR) {
      const double a = sm[s.red_k[rr]], c = sm[s.red_i0[rr]];
      v = s.red_sg[rr] > 0 ? add(a, c) : sub(a, c);
    }
    r[h] = v;
  }
  __syncwarp(tile_mask<Dm::LW>());
}

// reduc_inv_gn (src/mat1.f:445-473)
template <class Dm, class Ops>
__device__ __forceinline__ void reduc_inv(const Ops &s, const double (&gr)[Dm::R],
                                          double (&gn)[Dm::R], double *sm) {
  const int l = tile_lane<Dm::LW>();
#pragma unroll
  for (int h = 0; h < Dm::R; ++h) {
    const int i = l + Dm::LW * h;
    if (i < Dm::NMR) sm[i] = gr[h];
  }
  __syncwarp(tile_mask<Dm::LW>());
#pragma unroll
  for (int h = 0; h < Dm::R; ++h) {
    const int n = l + Dm::LW * h;
    double v = 0.0;
    if (n < Dm::N) {
      const int kind = s.inv_kind[n];
      if (kind == 1) {
        const int a = s.inv_a[n], cnt = s.inv_cnt[n];
        for (int ll = 0; ll < cnt; ll += 2) v = add(v, sm[a + ll]);
        for (int ll = 1; ll < cnt; ll += 2) v = sub(v, sm[a + ll]);
      } else if (kind == 2) {
        v = sm[s.inv_a[n]];
      }
    }
    gn[h] = v;
  }
  __syncwarp(tile_mask<Dm::LW>());
}

template <int R>
__device__ __forceinline__ void rot(double (&gn)[R], double (&gt)[R], const double (&gx)[R],
                                    const double (&gy)[R], double dnx, double dny) {
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const double a = gx[r], b = gy[r];
    gn[r] = add(mul(a, dnx), mul(b, dny));
    gt[r] = sub(mul(a, dny), mul(b, dnx));
  }
}

template <int R>
__device__ __forceinline__ void copy(double (&d)[R], const double (&s)[R]) {
#pragma unroll
  for (int r = 0; r < R; ++r) d[r] = s[r];
}

struct Geo {
  double ax, bx, ay, by, detai;
};
__device__ __forceinline__ Geo geo(const DevMesh &m, int e) {
  const double *v = m.vect + 5 * (size_t)e;
  return Geo{__ldg(v), __ldg(v + 1), __ldg(v + 2), __ldg(v + 3), __ldg(v + 4)};
}

// scaled face values: out[l] = fb[l] * norm(c, face of side l/G) [* scale]
template <class Dm>
__device__ __forceinline__ void scale_face(const DevMesh &m, const Sides &sd, const double *fb,
                                           double *out, int c) {
  const int l = tile_lane<Dm::LW>();
  if (l < 3 * Dm::G) out[l] = mul(fb[l], __ldg(m.norm + 2 * sd.face[l / Dm::G] + c));
}
template <class Dm>
__device__ __forceinline__ void scale_face_h(const DevMesh &m, const Sides &sd, const double *fb,
                                             double *out, int c, double scale) {
  const int l = tile_lane<Dm::LW>();
  if (l < 3 * Dm::G) out[l] = mul(mul(fb[l], __ldg(m.norm + 2 * sd.face[l / Dm::G] + c)), scale);
}

// RK4 stage bookkeeping (src/shwwnl.f:242-284)
template <class Dm>
__device__ __forceinline__ void stage_update(const StageArgs &sa, int fld, int e,
                                             const double (&d)[Dm::R]) {
  const int l = lane_id();
#pragma unroll
  for (int r = 0; r < Dm::R; ++r) {
    const int n = l + 32 * r;
    if (n >= Dm::N) continue;
    const size_t i = (size_t)e * Dm::N + n;
    const double dd = d[r];
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
// q-phase (calvarnl_fs.f:88-226)
// ---------------------------------------------------------------------------
template <class Dm, bool FACES = false>
struct __align__(16) QWarp {
  double own[2 * Dm::N];
  double nb[FACES ? 2 : 3 * nb_stride<Dm, 2>()];
  double fvs[FACES ? 3 * 2 * Dm::G : 2];  // face records of u, v (FACES)
  double fr[2 * 32];
  double fb[4 * 32];
  double sm[64];
  uint64_t bar;  // completion of the bulk row copies
};

// One element of the q-phase from the face-value chains on: own / nb hold the
// element's and its neighbours' u, v (FACES: nb holds the face records of
// kf_faces, [side][field][point]); prefetch() is called once they are free
// (after the mat-vecs); gq receives gxx, gxy, gyx, gyy.
template <class Dm, int VAR, bool FACES = false, class Prefetch>
__device__ __forceinline__ void qphase_elem(const SOps<Dm> &S, const DevMesh &m, int e,
                                            const Sides &sd, const double *own, const double *nb,
                                            double *fr, double *fb, double *sm, Prefetch prefetch,
                                            double (&gq)[4][Dm::R]) {
  constexpr int N = Dm::N, R = Dm::R, G = Dm::G;
  const Geo g = geo(m, e);
  int isg[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) isg[k] = __ldg(m.its + 3 * e + k);
  if constexpr (FACES) {
    const int l = lane_id();
    if (l < 3 * G) {
      const int k = l / G, j = l - k * G;
      fr[l] = nb[(k * 2) * G + j];
      fr[32 + l] = nb[(k * 2 + 1) * G + j];
    }
  } else {
    face_values<Dm, 2>(S.pf, m, sd, own, nb, fr);
  }
  __syncwarp();
  scale_face<Dm>(m, sd, fr, fb + 0, 0);
  scale_face<Dm>(m, sd, fr, fb + 32, 1);
  scale_face<Dm>(m, sd, fr + 32, fb + 64, 0);
  scale_face<Dm>(m, sd, fr + 32, fb + 96, 1);
  double ax[2][R], bx[2][R];
  matvec2<Dm, 2>(S.agx, S.agy, own, N, ax, bx);
  __syncwarp();  // own / nb are free from here on
  prefetch();
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double gx1 = add(0.0, mul(ax[c][r], -1.0)), gy1 = add(0.0, mul(bx[c][r], -1.0));
      gq[2 * c][r] = mul(sub(mul(g.by, gx1), mul(g.ay, gy1)), g.detai);
      gq[2 * c + 1][r] = mul(add(-mul(g.bx, gx1), mul(g.ax, gy1)), g.detai);
    }
  double t[4][3][R];
  lift_sums<Dm, 4>(S, isg, fb, t);
#pragma unroll
  for (int c = 0; c < 4; ++c) apply_lift<R>(gq[c], t[c], isg, g.detai);
  if (VAR == kFS && __ldg(m.bdl + e)) {
    // calvarnl_fs.f:171-204
    const double dnx = __ldg(m.normt + 2 * e), dny = __ldg(m.normt + 2 * e + 1);
    double gnx[R], gtx[R], gny[R], gty[R], gtn[R], bu[1][R];
    double fs3[3][R];  // gnn, gnt, gtt
    rot<R>(gnx, gtx, gq[0], gq[2], dnx, dny);
    rot<R>(gny, gty, gq[1], gq[3], dnx, dny);
    rot<R>(fs3[0], fs3[1], gnx, gny, dnx, dny);
    rot<R>(gtn, fs3[2], gtx, gty, dnx, dny);
    reduc<Dm>(S, gtn, bu[0], sm);
    solve_full_b<Dm, SOps<Dm>, 3>(S, fs3);
    solve_red_b<Dm, SOps<Dm>, 1>(S, bu);
    reduc_inv<Dm>(S, bu[0], gtn, sm);
    rot<R>(gnx, gny, fs3[0], fs3[1], dnx, dny);
    rot<R>(gtx, gty, gtn, fs3[2], dnx, dny);
    rot<R>(gq[0], gq[2], gnx, gtx, dnx, dny);
    rot<R>(gq[1], gq[3], gny, gty, dnx, dny);
  } else {
    solve_full_b<Dm, SOps<Dm>, 4>(S, gq);
  }
}

template <class Dm, int VAR, bool FACES = false>
__device__ __forceinline__ void qphase_body(DevOps op, DevMesh m, const double *__restrict__ su,
                                            const double *__restrict__ sv, double *q,
                                            const double *fv = nullptr) {
  extern __shared__ __align__(16) unsigned char smem[];
  SOps<Dm> &S = *reinterpret_cast<SOps<Dm> *>(smem);
  QWarp<Dm, FACES> &W =
      reinterpret_cast<QWarp<Dm, FACES> *>(smem + sizeof(SOps<Dm>))[warp_in_block()];
  constexpr int N = Dm::N, R = Dm::R, G = Dm::G;
  static_assert(!FACES || Dm::R == 1, "face records with one row per lane");
  const double *const fields[2] = {su, sv};
  // the copies of element e: its rows and its neighbours' rows, or its rows
  // and its three face records (FACES: W.fvs stands in for W.nb)
  double *const nbs = FACES ? W.fvs : W.nb;
  auto issue = [&](RowCopy<Dm, 2> &rc, int e, const Sides &sd) {
    if constexpr (FACES)
      rc.issue_own_faces(fields, e, sd, W.own, fv, W.fvs, 2 * G);
    else
      rc.issue(fields, e, sd, W.own, W.nb);
  };
  // the coefficients of the warp's next element are copied into W.own / W.nb
  // while it works on the current one (the first copy overlaps the staging
  // of the operators)
  // (one row per lane only: at two rows the registers are not there)
  constexpr bool PF = Dm::R == 1;
  Sides sd_next{};
  RowCopy<Dm, 2> rows;
  if (PF) rows.init(&W.bar);
  if (PF && warp_global() < m.ne) {
    sd_next = sides_of(m, warp_global());
    issue(rows, warp_global(), sd_next);
  }
  // the operator image arrives whole through one bulk copy (TMA engine)
  __shared__ __align__(8) uint64_t ops_bar;
  if (!bulk::stage_block(&S, op.img_ops, sizeof(SOps<Dm>), &ops_bar, op.flag)) {
    if (PF && warp_global() < m.ne) rows.wait(op.flag);
    return;
  }
  const size_t fs = (size_t)m.ne * N;
  for (int e = warp_global(); e < m.ne; e += warp_count()) {
    const Sides sd = PF ? sd_next : sides_of(m, e);
    const int en = e + warp_count();
    if (PF && en < m.ne) sd_next = sides_of(m, en);
    if constexpr (PF) {
      if (!rows.wait(op.flag)) return;
    } else {
      load_vec<Dm>(W.own, su, e);
      load_vec<Dm>(W.own + N, sv, e);
      stage_neighbours<Dm, 2>(sd, W.nb, [&](int f, int t, int i) { return fields[f][(size_t)t * N + i]; });
    }
    __syncwarp();
    double gq[4][R];  // gxx, gxy, gyx, gyy
    qphase_elem<Dm, VAR, FACES>(S, m, e, sd, W.own, nbs, W.fr, W.fb, W.sm, [&] {
      if (PF && en < m.ne) issue(rows, en, sd_next);
    }, gq);
#pragma unroll
    for (int c = 0; c < 4; ++c) store_reg<Dm>(q + c * fs, gq[c], e);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// nonlinear terms at quadrature points (calvarnl_fs.f:243-348)
// ---------------------------------------------------------------------------
template <class Dm>
struct __align__(16) BWarp {
  static constexpr int T = Dm::Q > 32 ? Dm::Q - 32 : 1;  // quadrature points past lane 31
  double vin[9 * Dm::N];
  double wp[8 * Dm::Q];
  double tail[9 * T];  // values of the nine fields at those points
  double sm[64];
  // one row per lane: the element's su, sv, sh, hb, w0, z0, fc and q (4
  // fields), copied ahead while the previous element is computed
  double rows[Dm::R == 1 ? 11 * Dm::N : 2];
};

// cp.async copies of element e's eleven input rows of the quadrature-point
// phase into rows[f*N + lane]
template <class Dm>
__device__ __forceinline__ void prefetch_nl_rows(const NlArgs &a, int e, size_t fs, double *rows) {
  const int l = lane_id();
  if (l >= Dm::N) return;
  const size_t o = (size_t)e * Dm::N + l;
  const double *const src[11] = {a.su, a.sv, a.sh, a.hb, a.w0, a.z0, a.fc,
                                 a.q, a.q + fs, a.q + 2 * fs, a.q + 3 * fs};
#pragma unroll
  for (int f = 0; f < 11; ++f) cp_async8(rows + f * Dm::N + l, src[f] + o);
}

// One element of the quadrature-point phase, given its q (qq): spectoxy of
// the nine fields, the products, xytospec, the uh / vh solves (wall
// projections included) and the stores of gx0, gy0, uh, vh, F.  so holds the
// solve operators and index maps (SOps or SOpsQ), p2 / p2t / wi the
// quadrature tables; vin, wp, tail, sm are the warp's scratch.
// rows: the element's input rows already in shared memory (one row per
// lane), or null to load them from global memory; after_load() runs once
// they are in registers.
template <class Dm, int VAR, class Ops, class AfterLoad>
__device__ __forceinline__ void nlvol_elem(const Ops &S, const double *p2, const double *p2t,
                                           const double *wi, double *vin, double *wp, double *tail,
                                           double *sm, const DevMesh &m, const NlArgs &a, int e,
                                           const double (&qq)[4][Dm::R], const double *rows,
                                           AfterLoad after_load) {
  constexpr int N = Dm::N, Q = Dm::Q, R = Dm::R, RQ = Dm::RQ;
  constexpr int T = Dm::Q > 32 ? Dm::Q - 32 : 1;  // quadrature points past lane 31
  const int l = lane_id();
  const size_t fs = (size_t)m.ne * N;
  double uk[R], vk[R], hh[R], fc[R], hb[R], w0[R], z0[R];
  if (rows) {
    const bool in = l < N;
    uk[0] = in ? rows[0 * N + l] : 0.0;
    vk[0] = in ? rows[1 * N + l] : 0.0;
    hh[0] = in ? rows[2 * N + l] : 0.0;
    hb[0] = in ? rows[3 * N + l] : 0.0;
    w0[0] = in ? rows[4 * N + l] : 0.0;
    z0[0] = in ? rows[5 * N + l] : 0.0;
    fc[0] = in ? rows[6 * N + l] : 0.0;
  } else {
    load_reg<Dm>(uk, a.su, e);
    load_reg<Dm>(vk, a.sv, e);
    load_reg<Dm>(hh, a.sh, e);
    load_reg<Dm>(hb, a.hb, e);
    load_reg<Dm>(w0, a.w0, e);
    load_reg<Dm>(z0, a.z0, e);
    load_reg<Dm>(fc, a.fc, e);
  }
  after_load();
  // uk,vk,hk=h+hb,wk=w-mb0 u,zk=z-mb0 v,gxx=qxx,gxy=qxy-fc,gyx=qyx+fc,gyy=qyy (:245-255)
  {
    double v9[9][R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      v9[0][r] = uk[r];
      v9[1][r] = vk[r];
      v9[2][r] = qq[0][r];
      v9[3][r] = sub(qq[1][r], fc[r]);
      v9[4][r] = add(qq[2][r], fc[r]);
      v9[5][r] = qq[3][r];
      v9[6][r] = add(hh[r], hb[r]);
      v9[7][r] = sub(w0[r], mul(a.mb0, uk[r]));
      v9[8][r] = sub(z0[r], mul(a.mb0, vk[r]));
    }
#pragma unroll
    for (int f = 0; f < 9; ++f) reg_to_sm<Dm>(vin + f * N, v9[f]);
  }
  __syncwarp();
  // spectoxy (src/nonlin.f:62-86) for the nine fields; lanes over points.
  // Points past lane 31 (degree 6: one, degree 7: ten) would cost a second
  // pass of nine full chains on a few lanes: their (field, point) chains are
  // spread over the lanes instead, each still summed over n in order.
  auto products = [&](int qp, const double (&mv)[9]) {
    const double w = wi[qp];
    wp[0 * Q + qp] = mul(w, mul(mv[0], mv[2]));
    wp[1 * Q + qp] = mul(w, mul(mv[1], mv[3]));
    wp[2 * Q + qp] = mul(w, mul(mv[0], mv[4]));
    wp[3 * Q + qp] = mul(w, mul(mv[1], mv[5]));
    wp[4 * Q + qp] = mul(w, mul(mv[0], mv[6]));
    wp[5 * Q + qp] = mul(w, mul(mv[1], mv[6]));
    wp[6 * Q + qp] = mul(w, __ddiv_rn(mv[7], mv[6]));
    wp[7 * Q + qp] = mul(w, __ddiv_rn(mv[8], mv[6]));
  };
  if (l < Q) {
    double mv[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) mv[f] = 0.0;
#pragma unroll 4
    for (int n = 0; n < N; ++n) {
      const double p = p2[n * Q + l];
#pragma unroll
      for (int f = 0; f < 9; ++f) mv[f] = macc(mv[f], vin[f * N + n], p);
    }
    products(l, mv);
  }
  if (RQ > 1) {
#pragma unroll
    for (int c0 = 0; c0 < 9 * T; c0 += 32) {
      const int c = c0 + l;
      if (c < 9 * T) {
        const int f = c / T, t = c - f * T;
        double v = 0.0;
#pragma unroll 4
        for (int n = 0; n < N; ++n) v = macc(v, vin[f * N + n], p2[n * Q + 32 + t]);
        tail[c] = v;
      }
    }
    __syncwarp();
    if (l < T) {
      double mv[9];
#pragma unroll
      for (int f = 0; f < 9; ++f) mv[f] = tail[f * T + l];
      products(32 + l, mv);
    }
  }
  __syncwarp();
  // xytospec (src/nonlin.f:35-57, :91-107); lanes over modes
  double X[8][R];
#pragma unroll
  for (int f = 0; f < 8; ++f)
#pragma unroll
    for (int r = 0; r < R; ++r) X[f][r] = 0.0;
#pragma unroll 4
  for (int qp = 0; qp < Q; ++qp) {
    double p[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = l + 32 * r;
      p[r] = n < N ? p2t[qp * N + n] : 0.0;
    }
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      const double wv = wp[f * Q + qp];
#pragma unroll
      for (int r = 0; r < R; ++r) X[f][r] = macc(X[f][r], wv, p[r]);
    }
  }
  double uv[2][R];
  copy<R>(uv[0], X[4]);
  copy<R>(uv[1], X[5]);
  if (__ldg(m.bdl + e)) {
    if (VAR == kNS) {
      double bu[2][R];  // calvarnl_ns.f:249-265
      reduc<Dm>(S, uv[0], bu[0], sm);
      reduc<Dm>(S, uv[1], bu[1], sm);
      solve_red_b<Dm, Ops, 2>(S, bu);
      reduc_inv<Dm>(S, bu[0], uv[0], sm);
      reduc_inv<Dm>(S, bu[1], uv[1], sm);
    } else {
      const double dnx = __ldg(m.normt + 2 * e), dny = __ldg(m.normt + 2 * e + 1);
      double gn[R], gt[1][R], bu[1][R];
      rot<R>(gn, gt[0], uv[0], uv[1], dnx, dny);
      reduc<Dm>(S, gn, bu[0], sm);
      solve_red_b<Dm, Ops, 1>(S, bu);
      solve_full_b<Dm, Ops, 1>(S, gt);
      reduc_inv<Dm>(S, bu[0], gn, sm);
      rot<R>(uv[0], uv[1], gn, gt[0], dnx, dny);
    }
  } else {
    solve_full_b<Dm, Ops, 2>(S, uv);
  }
  double gx0[R], gy0[R], f4[4][R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    gx0[r] = add(-add(X[0][r], X[1][r]), X[6][r]);
    gy0[r] = add(-add(X[2][r], X[3][r]), X[7][r]);
    f4[0][r] = sub(mul(a.mu0, qq[0][r]), mul(a.g0, hh[r]));
    f4[1][r] = mul(a.mu0, qq[1][r]);
    f4[2][r] = mul(a.mu0, qq[2][r]);
    f4[3][r] = sub(mul(a.mu0, qq[3][r]), mul(a.g0, hh[r]));
  }
  store_reg<Dm>(a.gx0, gx0, e);
  store_reg<Dm>(a.gy0, gy0, e);
  store_reg<Dm>(a.uh, uv[0], e);
  store_reg<Dm>(a.vh, uv[1], e);
#pragma unroll
  for (int c = 0; c < 4; ++c) store_reg<Dm>(a.f + c * fs, f4[c], e);
}

template <class Dm, int VAR>
__device__ __forceinline__ void nlvol_body(DevOps op, DevMesh m, NlArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  SOpsQ<Dm> &S = *reinterpret_cast<SOpsQ<Dm> *>(smem);
  BWarp<Dm> &W = reinterpret_cast<BWarp<Dm> *>(smem + sizeof(SOpsQ<Dm>))[warp_in_block()];
  constexpr int N = Dm::N, R = Dm::R;
  __shared__ __align__(8) uint64_t ops_bar;
  if (!bulk::stage_block(&S, op.img_q, sizeof(SOpsQ<Dm>), &ops_bar, op.flag)) return;
  const size_t fs = (size_t)m.ne * N;
  // one row per lane: the next element's input rows are copied into W.rows
  // while the current one is computed
  constexpr bool PF = Dm::R == 1;
  if (PF && warp_global() < m.ne) prefetch_nl_rows<Dm>(a, warp_global(), fs, W.rows);
  for (int e = warp_global(); e < m.ne; e += warp_count()) {
    const int en = e + warp_count();
    double qq[4][R];
    if constexpr (PF) {
      cp_async_wait_all();
      __syncwarp();
      const int l = lane_id();
#pragma unroll
      for (int c = 0; c < 4; ++c) qq[c][0] = l < N ? W.rows[(7 + c) * N + l] : 0.0;
      nlvol_elem<Dm, VAR>(S, S.p2, S.p2t, S.wi, W.vin, W.wp, W.tail, W.sm, m, a, e, qq, W.rows, [&] {
        __syncwarp();  // every lane has its rows in registers
        if (en < m.ne) prefetch_nl_rows<Dm>(a, en, fs, W.rows);
      });
    } else {
#pragma unroll
      for (int c = 0; c < 4; ++c) load_reg<Dm>(qq[c], a.q + c * fs, e);
      nlvol_elem<Dm, VAR>(S, S.p2, S.p2t, S.wi, W.vin, W.wp, W.tail, W.sm, m, a, e, qq,
                          static_cast<const double *>(nullptr), [] {});
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// face values once per face (src/calflu.f:22-66): the cal_flu chain of NF
// fields at every point of every face, in the order of the first element of
// the face (the values face_values computes on either side, bit for bit)
// ---------------------------------------------------------------------------
struct FaceArgs {
  const double *f[6];  // the fields, [ne][N] each
  double *out;         // [nf][NF][G]
};

template <class Dm, int NF>
__global__ void __launch_bounds__(256) kf_faces(DevOps op, DevMesh m, FaceArgs fa) {
  constexpr int N = Dm::N, G = Dm::G;
  __shared__ double spf[3 * N * G];  // [(s*N + n)*G + j] = pico(j,n,s)
  for (int i = threadIdx.x; i < 3 * N * G; i += blockDim.x) spf[i] = op.picoF[i];
  __syncthreads();
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= m.nf * G) return;
  const int f = item / G, j = item - f * G;
  const int t1 = __ldg(m.tseg + 2 * f), t2 = __ldg(m.tseg + 2 * f + 1);
  double acc[NF];
#pragma unroll
  for (int q = 0; q < NF; ++q) acc[q] = 0.0;
  // the chain over one element's modes (16-byte pairs at even N: the same
  // operations in the same order)
  auto chain = [&](int t, const double *p) {
    if constexpr (N % 2 == 0) {
#pragma unroll 2
      for (int n = 0; n < N; n += 2) {
        const double pv0 = p[n * G], pv1 = p[(n + 1) * G];
#pragma unroll
        for (int q = 0; q < NF; ++q) {
          const double2 c = __ldg(reinterpret_cast<const double2 *>(fa.f[q] + (size_t)t * N + n));
          acc[q] = macc(acc[q], c.x, pv0);
          acc[q] = macc(acc[q], c.y, pv1);
        }
      }
    } else {
#pragma unroll 2
      for (int n = 0; n < N; ++n) {
        const double pv = p[n * G];
#pragma unroll
        for (int q = 0; q < NF; ++q) acc[q] = macc(acc[q], __ldg(fa.f[q] + (size_t)t * N + n), pv);
      }
    }
  };
  if (t2 < 0) {
    chain(t1, spf + j);  // wall faces are traced on side 1 of their element
  } else {
    const int s1 = __ldg(m.ssit + 2 * f), s2 = __ldg(m.ssit + 2 * f + 1);
    chain(t1, spf + s1 * N * G + j);
    chain(t2, spf + s2 * N * G + (G - 1 - j));
#pragma unroll
    for (int q = 0; q < NF; ++q) acc[q] = mul(0.5, acc[q]);
  }
#pragma unroll
  for (int q = 0; q < NF; ++q) fa.out[((size_t)f * NF + q) * G + j] = acc[q];
}

// ---------------------------------------------------------------------------
// tendencies and the RK4 stage update (calvarnl_fs.f:350-544)
// ---------------------------------------------------------------------------
// FACES: the face values come from kf_faces (the records of the element's
// three faces are copied instead of its neighbours' coefficients).
template <class Dm, bool FACES = false>
struct __align__(16) TWarp {
  double own[6 * Dm::N];       // fxx, fxy, fyx, fyy, uh, vh
  double nb[FACES ? 2 : 3 * nb_stride<Dm, 6>()];
  double fvs[FACES ? 3 * 6 * Dm::G : 2];  // side k: [k][field][point]
  double fb[6 * 32];           // face values, then fbdxx, fbdxy, fbdyx, fbdyy, fbdx, fbdy
  double sm[64];
  // one row per lane: the element's gx0, gy0 and the RK4 base and
  // accumulator rows of u, v, h, copied ahead like the coefficients
  double aux[Dm::R == 1 ? 8 * Dm::N : 2];
  uint64_t bar;  // completion of the bulk row copies
};

// cp.async copies of element e's gx0, gy0 rows into aux[0..2N)
template <class Dm>
__device__ __forceinline__ void prefetch_gxy(const TendArgs &a, int e, double *aux) {
  const int l = lane_id();
  if (l < Dm::N) {
    cp_async8(aux + l, a.gx0 + (size_t)e * Dm::N + l);
    cp_async8(aux + Dm::N + l, a.gy0 + (size_t)e * Dm::N + l);
  }
}
// cp.async copies of element e's RK4 base rows (aux[2N..5N)) and, from the
// second stage on, accumulator rows (aux[5N..8N))
template <class Dm>
__device__ __forceinline__ void prefetch_stage(const StageArgs &sa, int e, double *aux) {
  const int l = lane_id();
  if (sa.stage < 0 || l >= Dm::N) return;
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    cp_async8(aux + (2 + f) * Dm::N + l, sa.base[f] + (size_t)e * Dm::N + l);
    if (sa.stage > 0) cp_async8(aux + (5 + f) * Dm::N + l, sa.acc[f] + (size_t)e * Dm::N + l);
  }
}

// stage_update with the element's base and accumulator rows already in
// shared memory (one row per lane); same operations
template <class Dm>
__device__ __forceinline__ void stage_update_sm(const StageArgs &sa, int fld, int e, double d,
                                                const double *aux) {
  const int n = lane_id();
  if (n >= Dm::N) return;
  const size_t i = (size_t)e * Dm::N + n;
  if (!isfinite(d)) atomicOr(sa.flag, 1);
  if (sa.stage < 0) {
    sa.tend[fld][i] = d;
    return;
  }
  const double u0 = aux[(2 + fld) * Dm::N + n];
  if (sa.stage == 0) {
    sa.acc[fld][i] = d;
    sa.out[fld][i] = add(u0, mul(mul(sa.dt, d), 0.5));
  } else if (sa.stage == 1) {
    sa.acc[fld][i] = add(aux[(5 + fld) * Dm::N + n], mul(2.0, d));
    sa.out[fld][i] = add(u0, mul(mul(sa.dt, d), 0.5));
  } else if (sa.stage == 2) {
    sa.acc[fld][i] = add(aux[(5 + fld) * Dm::N + n], mul(2.0, d));
    sa.out[fld][i] = add(u0, mul(sa.dt, d));
  } else {
    const double nv = add(u0, mul(sa.dt6, add(aux[(5 + fld) * Dm::N + n], d)));
    sa.base[fld][i] = nv;
    if (sa.host[fld]) sa.host[fld][(size_t)e * sa.host_ld + n] = nv;
  }
}

template <class Dm, int VAR, bool FACES = false>
__device__ __forceinline__ void tend_body(DevOps op, DevMesh m, TendArgs a, StageArgs sa) {
  extern __shared__ __align__(16) unsigned char smem[];
  SOps<Dm> &S = *reinterpret_cast<SOps<Dm> *>(smem);
  TWarp<Dm, FACES> &W =
      reinterpret_cast<TWarp<Dm, FACES> *>(smem + sizeof(SOps<Dm>))[warp_in_block()];
  constexpr int N = Dm::N, R = Dm::R, G = Dm::G;
  static_assert(!FACES || Dm::R == 1, "face records with one row per lane");
  // issue the copies of element e: its rows and its neighbours' rows, or its
  // rows and its three face records
  auto issue = [&](RowCopy<Dm, 6> &rc, const double *const (&fields)[6], int e, const Sides &sd) {
    if constexpr (FACES)
      rc.issue_own_faces(fields, e, sd, W.own, a.fv, W.fvs, 6 * G);
    else
      rc.issue(fields, e, sd, W.own, W.nb);
  };
  const size_t fs = (size_t)m.ne * N;
  const double *const src[6] = {a.f, a.f + fs, a.f + 2 * fs, a.f + 3 * fs, a.uh, a.vh};
  // the coefficients of the warp's next element are copied into W.own / W.nb
  // while it works on the current one (the first copy overlaps the staging
  // of the operators)
  // (one row per lane only: at two rows the registers are not there)
  constexpr bool PF = Dm::R == 1;
  Sides sd_next{};
  RowCopy<Dm, 6> rows;
  if (PF) rows.init(&W.bar);
  if (PF && warp_global() < m.ne) {
    sd_next = sides_of(m, warp_global());
    issue(rows, src, warp_global(), sd_next);
    prefetch_gxy<Dm>(a, warp_global(), W.aux);
    prefetch_stage<Dm>(sa, warp_global(), W.aux);
  }
  __shared__ __align__(8) uint64_t ops_bar;
  if (!bulk::stage_block(&S, op.img_ops, sizeof(SOps<Dm>), &ops_bar, op.flag)) {
    if (PF && warp_global() < m.ne) rows.wait(op.flag);
    cp_async_wait_all();
    return;
  }
  for (int e = warp_global(); e < m.ne; e += warp_count()) {
    const Sides sd = PF ? sd_next : sides_of(m, e);
    const int en = e + warp_count();
    if (PF && en < m.ne) sd_next = sides_of(m, en);
    const Geo g = geo(m, e);
    int isg[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) isg[k] = __ldg(m.its + 3 * e + k);
    if constexpr (PF) {
      const bool ok = rows.wait(op.flag);
      cp_async_wait_all();
      if (!ok) return;
    } else {
#pragma unroll
      for (int f = 0; f < 6; ++f) load_vec<Dm>(W.own + f * N, src[f], e);
      stage_neighbours<Dm, 6>(sd, W.nb, [&](int f, int t, int i) { return src[f][(size_t)t * N + i]; });
    }
    __syncwarp();
    if constexpr (FACES) {
      const int l = lane_id();
      if (l < 3 * G) {
        const int k = l / G, j = l - k * G;
#pragma unroll
        for (int f = 0; f < 6; ++f) W.fb[f * 32 + l] = W.fvs[(k * 6 + f) * G + j];
      }
    } else {
      face_values<Dm, 6>(S.pf, m, sd, W.own, W.nb, W.fb);
    }
    __syncwarp();
    // each lane scales the values it computed (fbd * norm(1|2, face))
#pragma unroll
    for (int f = 0; f < 6; ++f) scale_face<Dm>(m, sd, W.fb + 32 * f, W.fb + 32 * f, f & 1);
    double ax[6][R], bx[6][R];
    matvec2<Dm, 6>(S.agx, S.agy, W.own, N, ax, bx);
    double gx[R], gy[R], hb[R];
    if constexpr (PF) {
      gx[0] = lane_id() < N ? W.aux[lane_id()] : 0.0;
      gy[0] = lane_id() < N ? W.aux[N + lane_id()] : 0.0;
    } else {
      load_reg<Dm>(gx, a.gx0, e);
      load_reg<Dm>(gy, a.gy0, e);
    }
    const double cby = mul(g.by, g.detai), cay = mul(g.ay, g.detai);
    const double cbx = mul(g.bx, g.detai), cax = mul(g.ax, g.detai);
    axpy<R>(gx, ax[0], -cby);
    axpy<R>(gx, bx[0], cay);
    axpy<R>(gx, ax[1], cbx);
    axpy<R>(gx, bx[1], -cax);
    axpy<R>(gy, ax[2], -cby);
    axpy<R>(gy, bx[2], cay);
    axpy<R>(gy, ax[3], cbx);
    axpy<R>(gy, bx[3], -cax);
#pragma unroll
    for (int r = 0; r < R; ++r) hb[r] = 0.0;
    axpy<R>(hb, ax[4], cby);
    axpy<R>(hb, bx[4], -cay);
    axpy<R>(hb, ax[5], -cbx);
    axpy<R>(hb, bx[5], cax);
    __syncwarp();  // W.own / W.nb and the gx0, gy0 rows are free from here on
    if (PF && en < m.ne) {
      issue(rows, src, en, sd_next);
      prefetch_gxy<Dm>(a, en, W.aux);
    }
    double t[6][3][R];
    lift_sums<Dm, 6>(S, isg, W.fb, t);
    apply_lift<R>(gx, t[0], isg, g.detai);
    apply_lift<R>(gx, t[1], isg, g.detai);
    apply_lift<R>(gy, t[2], isg, g.detai);
    apply_lift<R>(gy, t[3], isg, g.detai);
    apply_lift<R>(hb, t[4], isg, -g.detai);
    apply_lift<R>(hb, t[5], isg, -g.detai);
    if (__ldg(m.bdl + e)) {
      if (VAR == kNS) {
        double bu[2][R], hs[1][R];
        reduc<Dm>(S, gx, bu[0], W.sm);
        reduc<Dm>(S, gy, bu[1], W.sm);
        solve_red_b<Dm, SOps<Dm>, 2>(S, bu);
        copy<R>(hs[0], hb);
        solve_full_b<Dm, SOps<Dm>, 1>(S, hs);
        copy<R>(hb, hs[0]);
        reduc_inv<Dm>(S, bu[0], gx, W.sm);
        reduc_inv<Dm>(S, bu[1], gy, W.sm);
      } else {
        const double dnx = __ldg(m.normt + 2 * e), dny = __ldg(m.normt + 2 * e + 1);
        double gn[R], full2[2][R], bu[1][R];
        rot<R>(gn, full2[0], gx, gy, dnx, dny);
        copy<R>(full2[1], hb);
        reduc<Dm>(S, gn, bu[0], W.sm);
        solve_red_b<Dm, SOps<Dm>, 1>(S, bu);
        solve_full_b<Dm, SOps<Dm>, 2>(S, full2);
        reduc_inv<Dm>(S, bu[0], gn, W.sm);
        rot<R>(gx, gy, gn, full2[0], dnx, dny);
        copy<R>(hb, full2[1]);
      }
    } else {
      double s3[3][R];
      copy<R>(s3[0], gx);
      copy<R>(s3[1], gy);
      copy<R>(s3[2], hb);
      solve_full_b<Dm, SOps<Dm>, 3>(S, s3);
      copy<R>(gx, s3[0]);
      copy<R>(gy, s3[1]);
      copy<R>(hb, s3[2]);
    }
    if constexpr (PF) {
      stage_update_sm<Dm>(sa, 0, e, gx[0], W.aux);
      stage_update_sm<Dm>(sa, 1, e, gy[0], W.aux);
      stage_update_sm<Dm>(sa, 2, e, hb[0], W.aux);
      __syncwarp();  // the base and accumulator rows are free
      if (en < m.ne) prefetch_stage<Dm>(sa, en, W.aux);
    } else {
      stage_update<Dm>(sa, 0, e, gx);
      stage_update<Dm>(sa, 1, e, gy);
      stage_update<Dm>(sa, 2, e, hb);
    }
    __syncwarp();
  }
}

// The nonlinear kernels.  At one row per lane the registers are left to the
// compiler (about 120); at two rows per lane (degree 7) they are held to two
// resident blocks per SM (kf_tend: 6 warps per block, which its per-warp
// scratch allows), trading a few spilled words for twice the resident warps.
template <class Dm, int VAR>
__global__ void __launch_bounds__(256) kf_qphase(DevOps op, DevMesh m, const double *__restrict__ su,
                                                 const double *__restrict__ sv, double *q) {
  qphase_body<Dm, VAR>(op, m, su, sv, q);
}
// the q-phase on the face values of kf_faces (one row per lane)
template <class Dm, int VAR>
__global__ void __launch_bounds__(256) kf_qphasef(DevOps op, DevMesh m,
                                                  const double *__restrict__ su,
                                                  const double *__restrict__ sv, double *q,
                                                  const double *__restrict__ fv) {
  if constexpr (Dm::R == 1) qphase_body<Dm, VAR, true>(op, m, su, sv, q, fv);
}
template <class Dm, int VAR>
__global__ void __launch_bounds__(256, 2) kf_qphase_r2(DevOps op, DevMesh m,
                                                       const double *__restrict__ su,
                                                       const double *__restrict__ sv, double *q) {
  qphase_body<Dm, VAR>(op, m, su, sv, q);
}
template <class Dm, int VAR>
__global__ void __launch_bounds__(256, 2) kf_nlvol(DevOps op, DevMesh m, NlArgs a) {
  nlvol_body<Dm, VAR>(op, m, a);
}
template <class Dm, int VAR>
__global__ void __launch_bounds__(256, 2) kf_nlvol_r2(DevOps op, DevMesh m, NlArgs a) {
  nlvol_body<Dm, VAR>(op, m, a);
}
template <class Dm, int VAR>
__global__ void __launch_bounds__(256) kf_tend(DevOps op, DevMesh m, TendArgs a, StageArgs sa) {
  tend_body<Dm, VAR>(op, m, a, sa);
}
// the tendency kernel on the face values of kf_faces (one row per lane)
template <class Dm, int VAR>
__global__ void __launch_bounds__(256) kf_tendf(DevOps op, DevMesh m, TendArgs a, StageArgs sa) {
  if constexpr (Dm::R == 1) tend_body<Dm, VAR, true>(op, m, a, sa);
}
template <class Dm, int VAR>
__global__ void __launch_bounds__(Dm::TEND_THREADS, 2) kf_tend_r2(DevOps op, DevMesh m, TendArgs a,
                                                                  StageArgs sa) {
  tend_body<Dm, VAR>(op, m, a, sa);
}
template <class Dm, int VAR>
constexpr auto qphase_kernel() {
  if constexpr (Dm::R == 1) return kf_qphase<Dm, VAR>; else return kf_qphase_r2<Dm, VAR>;
}
template <class Dm, int VAR>
constexpr auto nlvol_kernel() {
  if constexpr (Dm::R == 1) return kf_nlvol<Dm, VAR>; else return kf_nlvol_r2<Dm, VAR>;
}
template <class Dm, int VAR>
constexpr auto tend_kernel() {
  if constexpr (Dm::R == 1) return kf_tend<Dm, VAR>; else return kf_tend_r2<Dm, VAR>;
}

// ---------------------------------------------------------------------------
// linear variant (calvar_lin.f:7-287)
// ---------------------------------------------------------------------------
template <class Dm>
struct __align__(16) LWarp {
  double own[3 * Dm::N];  // fxx = -g0 h, u, v
  double nb[3 * nb_stride<Dm, 3>()];
  double xs[2 * Dm::N];   // u*hh0, v*hh0
  double fr[3 * 32];
  double fb[4 * 32];      // fbdxx, fbdyy, fbdx, fbdy
  double sm[64];
};

// A load of the stage state: plain, or through L2 only (ld.global.cg) in the
// multi-step kernel, whose blocks read rows that other blocks wrote earlier
// in the same launch (behind a grid barrier).
template <bool CG>
__device__ __forceinline__ double ld_state(const double *p) {
  if constexpr (CG) return __ldcg(p); else return *p;
}

// The mesh record of one element of the linear kernels (read once per
// element; the multi-step kernel keeps it for the whole launch).
struct LinElem {
  Sides sd;
  Geo g;
  int isg[3];
  bool wall;
  double dnx, dny;
};
__device__ __forceinline__ LinElem lin_elem_mesh(const DevMesh &m, int e) {
  LinElem r;
  r.sd = sides_of(m, e);
  r.g = geo(m, e);
#pragma unroll
  for (int k = 0; k < 3; ++k) r.isg[k] = __ldg(m.its + 3 * e + k);
  r.wall = __ldg(m.bdl + e) != 0;
  r.dnx = r.wall ? __ldg(m.normt + 2 * e) : 0.0;
  r.dny = r.wall ? __ldg(m.normt + 2 * e + 1) : 0.0;
  return r;
}

// The linear right-hand side of one element (calvar_lin.f:7-287) from its
// own u, v, h (registers) and its neighbours' rows of a.su, a.sv, a.sh:
// gx, gy, hb receive the tendencies of u, v, h after the mass solves.
template <class Dm, bool CG>
__device__ __forceinline__ void lin_rhs(const SOps<Dm> &S, LWarp<Dm> &W, const DevMesh &m,
                                        const LinElem &lm, const LinArgs &a,
                                        const double (&uk)[Dm::R], const double (&vk)[Dm::R],
                                        const double (&hk)[Dm::R], double (&gx)[Dm::R],
                                        double (&gy)[Dm::R], double (&hb)[Dm::R]) {
  constexpr int N = Dm::N, R = Dm::R;
  const int l = tile_lane<Dm::LW>();
  const double mg0 = -a.g0, hh0 = a.hh0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = l + Dm::LW * r;
    if (i < N) {
      W.own[i] = mul(mg0, hk[r]);  // fxx = fyy = -g0 h (calvar_lin.f:76-79)
      W.own[N + i] = uk[r];
      W.own[2 * N + i] = vk[r];
      W.xs[i] = mul(uk[r], hh0);
      W.xs[N + i] = mul(vk[r], hh0);
    }
  }
  stage_neighbours<Dm, 3>(lm.sd, W.nb, [&](int f, int t, int i) {
    const size_t o = (size_t)t * N + i;
    return f == 0 ? mul(mg0, ld_state<CG>(a.sh + o))
                  : (f == 1 ? ld_state<CG>(a.su + o) : ld_state<CG>(a.sv + o));
  });
  __syncwarp(tile_mask<Dm::LW>());
  face_values<Dm, 3>(S.pf, m, lm.sd, W.own, W.nb, W.fr);
  __syncwarp(tile_mask<Dm::LW>());
  scale_face<Dm>(m, lm.sd, W.fr, W.fb, 0);        // fbdxx
  scale_face<Dm>(m, lm.sd, W.fr, W.fb + 32, 1);   // fbdyy
  scale_face_h<Dm>(m, lm.sd, W.fr + 32, W.fb + 64, 0, hh0);  // fbdx
  scale_face_h<Dm>(m, lm.sd, W.fr + 64, W.fb + 96, 1, hh0);  // fbdy
  double af[1][R], bf[1][R], ah[2][R], bh[2][R];
  matvec2<Dm, 1>(S.agx, S.agy, W.own, N, af, bf);
  matvec2<Dm, 2>(S.agx, S.agy, W.xs, N, ah, bh);
  __syncwarp(tile_mask<Dm::LW>());
  const double cby = mul(lm.g.by, lm.g.detai), cay = mul(lm.g.ay, lm.g.detai);
  const double cbx = mul(lm.g.bx, lm.g.detai), cax = mul(lm.g.ax, lm.g.detai);
#pragma unroll
  for (int r = 0; r < R; ++r) gx[r] = gy[r] = hb[r] = 0.0;
  // u, v (calvar_lin.f:143-166); the zero fields fxy, fyx contribute exact zeros
  axpy<R>(gx, af[0], -cby);
  axpy<R>(gx, bf[0], cay);
  axpy<R>(gy, af[0], cbx);
  axpy<R>(gy, bf[0], -cax);
  // h (calvar_lin.f:256-270)
  axpy<R>(hb, ah[0], cby);
  axpy<R>(hb, bh[0], -cay);
  axpy<R>(hb, ah[1], -cbx);
  axpy<R>(hb, bh[1], cax);
  double t[4][3][R];
  lift_sums<Dm, 4>(S, lm.isg, W.fb, t);
  apply_lift<R>(gx, t[0], lm.isg, lm.g.detai);
  apply_lift<R>(gy, t[1], lm.isg, lm.g.detai);
  apply_lift<R>(hb, t[2], lm.isg, -lm.g.detai);
  apply_lift<R>(hb, t[3], lm.isg, -lm.g.detai);
  if (lm.wall) {
    const double dnx = lm.dnx, dny = lm.dny;
    double gn[R], full2[2][R], bu[1][R];
    rot<R>(gn, full2[0], gx, gy, dnx, dny);
    copy<R>(full2[1], hb);
    reduc<Dm>(S, gn, bu[0], W.sm);
    solve_red_b<Dm, SOps<Dm>, 1>(S, bu);
    solve_full_b<Dm, SOps<Dm>, 2>(S, full2);
    reduc_inv<Dm>(S, bu[0], gn, W.sm);
    rot<R>(gx, gy, gn, full2[0], dnx, dny);
    copy<R>(hb, full2[1]);
  } else {
    double s3[3][R];
    copy<R>(s3[0], gx);
    copy<R>(s3[1], gy);
    copy<R>(s3[2], hb);
    solve_full_b<Dm, SOps<Dm>, 3>(S, s3);
    copy<R>(gx, s3[0]);
    copy<R>(gy, s3[1]);
    copy<R>(hb, s3[2]);
  }
}

// One element of the linear right-hand side and its RK4 stage update.
template <class Dm>
__device__ __forceinline__ void lin_elem(const SOps<Dm> &S, LWarp<Dm> &W, const DevMesh &m,
                                         const LinArgs &a, const StageArgs &sa, int e) {
  constexpr int R = Dm::R;
  const LinElem lm = lin_elem_mesh(m, e);
  double uk[R], vk[R], hk[R];
  load_reg<Dm>(uk, a.su, e);
  load_reg<Dm>(vk, a.sv, e);
  load_reg<Dm>(hk, a.sh, e);
  double gx[R], gy[R], hb[R];
  lin_rhs<Dm, false>(S, W, m, lm, a, uk, vk, hk, gx, gy, hb);
  stage_update<Dm>(sa, 0, e, gx);
  stage_update<Dm>(sa, 1, e, gy);
  stage_update<Dm>(sa, 2, e, hb);
  __syncwarp();
}

template <class Dm>
__global__ void __launch_bounds__(256) kf_lin(DevOps op, DevMesh m, LinArgs a, StageArgs sa) {
  extern __shared__ __align__(16) unsigned char smem[];
  SOps<Dm> &S = *reinterpret_cast<SOps<Dm> *>(smem);
  LWarp<Dm> &W = reinterpret_cast<LWarp<Dm> *>(smem + sizeof(SOps<Dm>))[warp_in_block()];
  __shared__ __align__(8) uint64_t ops_bar;
  if (!bulk::stage_block(&S, op.img_ops, sizeof(SOps<Dm>), &ops_bar, op.flag)) return;
  for (int e = warp_global(); e < m.ne; e += warp_count()) lin_elem<Dm>(S, W, m, a, sa, e);
}

// Grid-wide barrier of a cooperative launch: every block adds one to *count
// and waits until it reaches `target` (a multiple of the grid size).  The
// wait is bounded: past kGridWaitLimit polls bit 2 of *flag is set and false
// returned (the caller leaves the kernel).
constexpr long long kGridWaitLimit = 1ll << 24;
__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned target, int *flag) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    // release: the block's stores (ordered before this thread by the block
    // barrier) are visible to whoever acquires the count after this add
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(count) : "memory");
    bool done = false;
    for (long long it = 0; it < kGridWaitLimit; ++it) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
      if (v >= target) {
        done = true;
        break;
      }
      __nanosleep(32);
    }
    if (!done) atomicOr(flag, 2);
    ok = done;
  }
  __syncthreads();
  return ok;
}

// Several RK4 steps of the linear variant in one cooperative launch (every
// block resident), one element per warp or half-warp for the whole launch:
// the operator image is staged once, the element's mesh record, its u0 and
// RK4 accumulator rows and its stage values stay in registers, and only the
// neighbours' stage rows are read (through L2 only: other blocks wrote them
// earlier in the launch, behind a grid barrier).  The stage buffers rotate as
// in one launch per stage (input u0, A, B, A; output A, B, A, u0 in place);
// the arithmetic and its order are those of kf_lin and stage_update.  (Per-
// element stage counters polled by the neighbours instead of the barrier
// measured three times slower.)
// MAXW: the most warps per block the instance is built for (8: the
// registers are left to the compiler; 20: held to 96)
constexpr int kLinStepsMaxWarps = 20;
template <class Dm, int MAXW>
__global__ void __launch_bounds__(32 * MAXW) kf_lin_steps(DevOps op, DevMesh m, LinSteps ls) {
  extern __shared__ __align__(16) unsigned char smem[];
  SOps<Dm> &S = *reinterpret_cast<SOps<Dm> *>(smem);
  constexpr int N = Dm::N, R = Dm::R, TPW = 32 / Dm::LW;  // elements per warp
  LWarp<Dm> &W = reinterpret_cast<LWarp<Dm> *>(
      smem + sizeof(SOps<Dm>))[warp_in_block() * TPW + lane_id() / Dm::LW];
  __shared__ __align__(8) uint64_t ops_bar;
  const bool staged = bulk::stage_block(&S, op.img_ops, sizeof(SOps<Dm>), &ops_bar, op.flag);
  const int l = tile_lane<Dm::LW>();
  const int tile = warp_global() * TPW + lane_id() / Dm::LW;
  const int e = ls.order ? (tile < ls.norder ? __ldg(ls.order + tile) : -1) : tile;
  const bool active = staged && e >= 0 && e < m.ne;
  LinElem lm{};
  double u0[3][R], acc[3][R], x[3][R];  // u0, du1 + 2 du2 + 2 du3, stage input
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < R; ++r) u0[c][r] = acc[c][r] = x[c][r] = 0.0;
  if (active) {
    lm = lin_elem_mesh(m, e);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = l + Dm::LW * r;
        u0[c][r] = x[c][r] = i < N ? __ldcg(ls.sa.base[c] + (size_t)e * N + i) : 0.0;
      }
  }
  const double dt = ls.sa.dt, dt6 = ls.sa.dt6;
  unsigned target = 0;
  for (int it = 0; it < ls.nsteps; ++it) {
    for (int st = 0; st < 4; ++st) {
      const bool last = it == ls.nsteps - 1 && st == 3;
      if (active) {
        const LinArgs a{st == 0 ? ls.sa.base[0] : (st == 2 ? ls.bufb[0] : ls.bufa[0]),
                        st == 0 ? ls.sa.base[1] : (st == 2 ? ls.bufb[1] : ls.bufa[1]),
                        st == 0 ? ls.sa.base[2] : (st == 2 ? ls.bufb[2] : ls.bufa[2]), ls.g0,
                        ls.hh0};
        double d[3][R];
        lin_rhs<Dm, true>(S, W, m, lm, a, x[0], x[1], x[2], d[0], d[1], d[2]);
        // stage_update with u0 and the accumulator in registers
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double *const out = st == 1 ? ls.bufb[c] : ls.bufa[c];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = l + Dm::LW * r;
            if (i >= N) continue;
            const size_t o = (size_t)e * N + i;
            const double dd = d[c][r];
            if (!isfinite(dd)) atomicOr(ls.sa.flag, 1);
            if (st == 0) {
              acc[c][r] = dd;
              x[c][r] = add(u0[c][r], mul(mul(dt, dd), 0.5));
              out[o] = x[c][r];
            } else if (st == 1) {
              acc[c][r] = add(acc[c][r], mul(2.0, dd));
              x[c][r] = add(u0[c][r], mul(mul(dt, dd), 0.5));
              out[o] = x[c][r];
            } else if (st == 2) {
              acc[c][r] = add(acc[c][r], mul(2.0, dd));
              x[c][r] = add(u0[c][r], mul(dt, dd));
              out[o] = x[c][r];
            } else {
              const double nv = add(u0[c][r], mul(dt6, add(acc[c][r], dd)));
              u0[c][r] = x[c][r] = nv;
              ls.sa.base[c][o] = nv;
              if (last && ls.host[c]) ls.host[c][(size_t)e * ls.sa.host_ld + i] = nv;
            }
          }
        }
        __syncwarp(tile_mask<Dm::LW>());
      }
      if (last) return;
      target += gridDim.x;
      if (!grid_barrier(ls.count, target, op.flag)) return;
    }
  }
}

// ---------------------------------------------------------------------------
// operator images: the shared-memory layouts of SOps / SOpsQ, written once per
// handle into global memory so that each block stages them with bulk copies
// ---------------------------------------------------------------------------
template <class Dm>
__global__ void __launch_bounds__(256) k_fast_images(DevOps op, SOps<Dm> *img, SOpsQ<Dm> *imgq) {
  stage_ops(*img, op);
  stage_ops_q(*imgq, op);
}

// ---------------------------------------------------------------------------
// launch plumbing
// ---------------------------------------------------------------------------
// warps per block so that the per-block shared memory stays under ~113 KB
// (two blocks per SM) when possible, else one block up to 8 warps.
constexpr int pick_warps(size_t ops, size_t per_warp) {
  for (int w = 8; w >= 2; --w)
    if (ops + w * per_warp <= 113 * 1024) return w;
  for (int w = 8; w >= 1; --w)
    if (ops + w * per_warp <= 220 * 1024) return w;
  return 1;
}

template <class Dm, int VAR>
cudaError_t run_nl(const DevOps &op, const DevMesh &m, const RhsBuffers &b, const StageArgs &sa,
                   cudaStream_t st, int sms, cudaEvent_t *ev, long long *launches) {
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], st);
  };
  NlArgs na{b.su, b.sv, b.sh, b.hb, b.w0, b.z0, b.fc, b.q, b.gx0, b.gy0, b.uh, b.vh, b.f,
            b.mu0, b.mb0, b.g0};
  TendArgs ta{b.gx0, b.gy0, b.uh, b.vh, b.f, b.fv};
  constexpr int wq = pick_warps(sizeof(SOps<Dm>), sizeof(QWarp<Dm>));
  constexpr int wb = pick_warps(sizeof(SOpsQ<Dm>), sizeof(BWarp<Dm>));
  constexpr int wt = std::min(pick_warps(sizeof(SOps<Dm>), sizeof(TWarp<Dm>)), Dm::TEND_THREADS / 32);
  constexpr size_t sq = sizeof(SOps<Dm>) + wq * sizeof(QWarp<Dm>);
  constexpr size_t sb = sizeof(SOpsQ<Dm>) + wb * sizeof(BWarp<Dm>);
  constexpr size_t stt = sizeof(SOps<Dm>) + wt * sizeof(TWarp<Dm>);
  int gq = 0, gb = 0, gt = 0;
  cudaError_t e = resident_grid(tend_kernel<Dm, VAR>(), 32 * wt, stt, sms, m.ne, wt, &gt);
  if (e != cudaSuccess) return e;
  e = resident_grid(qphase_kernel<Dm, VAR>(), 32 * wq, sq, sms, m.ne, wq, &gq);
  if (e == cudaSuccess) e = resident_grid(nlvol_kernel<Dm, VAR>(), 32 * wb, sb, sms, m.ne, wb, &gb);
  if (e != cudaSuccess) return e;
  mark(0);
  const auto kq = qphase_kernel<Dm, VAR>();
  const auto kb = nlvol_kernel<Dm, VAR>();
  const auto kt = tend_kernel<Dm, VAR>();
  // face values of u, v once per face (counted with the q-phase)
  bool qfaces = false;
  if constexpr (Dm::R == 1) {
    if (b.fv) {
      constexpr int wf = pick_warps(sizeof(SOps<Dm>), sizeof(QWarp<Dm, true>));
      constexpr size_t sf = sizeof(SOps<Dm>) + wf * sizeof(QWarp<Dm, true>);
      int gf = 0;
      e = resident_grid(kf_qphasef<Dm, VAR>, 32 * wf, sf, sms, m.ne, wf, &gf);
      if (e != cudaSuccess) return e;
      FaceArgs fa{{b.su, b.sv}, b.fv};
      const int items = m.nf * Dm::G;
      kf_faces<Dm, 2><<<(items + 255) / 256, 256, 0, st>>>(op, m, fa);
      kf_qphasef<Dm, VAR><<<gf, 32 * wf, sf, st>>>(op, m, b.su, b.sv, b.q, b.fv);
      *launches += 1;
      qfaces = true;
    }
  }
  if (!qfaces) kq<<<gq, 32 * wq, sq, st>>>(op, m, b.su, b.sv, b.q);
  if (b.sh_ready) cudaStreamWaitEvent(st, b.sh_ready, 0);
  mark(1);
  kb<<<gb, 32 * wb, sb, st>>>(op, m, na);
  mark(2);
  if constexpr (Dm::R == 1) {
    if (b.fv) {
      // face values once per face, then the tendency kernel on them (the
      // face kernel's time is counted with the tendency kernel's)
      constexpr int wf = std::min(pick_warps(sizeof(SOps<Dm>), sizeof(TWarp<Dm, true>)),
                                  Dm::TEND_THREADS / 32);
      constexpr size_t sf = sizeof(SOps<Dm>) + wf * sizeof(TWarp<Dm, true>);
      int gf = 0;
      e = resident_grid(kf_tendf<Dm, VAR>, 32 * wf, sf, sms, m.ne, wf, &gf);
      if (e != cudaSuccess) return e;
      const size_t fs = (size_t)m.ne * Dm::N;
      FaceArgs fa{{b.f, b.f + fs, b.f + 2 * fs, b.f + 3 * fs, b.uh, b.vh}, b.fv};
      const int items = m.nf * Dm::G;
      kf_faces<Dm, 6><<<(items + 255) / 256, 256, 0, st>>>(op, m, fa);
      kf_tendf<Dm, VAR><<<gf, 32 * wf, sf, st>>>(op, m, ta, sa);
      mark(3);
      e = cudaGetLastError();
      if (e == cudaSuccess) *launches += 4;
      return e;
    }
  }
  kt<<<gt, 32 * wt, stt, st>>>(op, m, ta, sa);
  mark(3);
  e = cudaGetLastError();
  if (e == cudaSuccess) *launches += 3;
  return e;
}

// The q-phase alone (the base state's q of the tangent-linear and adjoint
// right-hand sides).
template <class Dm, int VAR>
cudaError_t run_q(const DevOps &op, const DevMesh &m, const double *su, const double *sv, double *q,
                  cudaStream_t st, int sms) {
  constexpr int wq = pick_warps(sizeof(SOps<Dm>), sizeof(QWarp<Dm>));
  constexpr size_t sq = sizeof(SOps<Dm>) + wq * sizeof(QWarp<Dm>);
  int gq = 0;
  const cudaError_t e = resident_grid(qphase_kernel<Dm, VAR>(), 32 * wq, sq, sms, m.ne, wq, &gq);
  if (e != cudaSuccess) return e;
  const auto kq = qphase_kernel<Dm, VAR>();
  kq<<<gq, 32 * wq, sq, st>>>(op, m, su, sv, q);
  return cudaGetLastError();
}

// The multi-step linear kernel when the mesh fits one block per SM with one
// element per warp (small meshes, where the per-stage launches and
// the operator staging dominate): the elements are spread evenly, ceil(ne /
// sms) warps per block, so no SM carries twice the work of another between
// two barriers.  Else cudaErrorNotSupported.
template <class D>
cudaError_t run_lin_steps(const DevOps &op, const DevMesh &m, const LinSteps &ls, cudaStream_t st,
                          int sms, long long *launches) {
  // two elements per warp where an element fits 16 lanes
  using Dm = std::conditional_t<fits_half<D>(), Half<D>, D>;
  static_assert(sizeof(SOps<Dm>) == sizeof(SOps<D>), "one operator image for both layouts");
  constexpr int TPW = 32 / Dm::LW;
  if (m.ne < 1 || sms < 1) return cudaErrorNotSupported;
  // the element order pairs the halves of a warp; one element per warp has
  // no halves to pair
  LinSteps l = ls;
  if (TPW == 1 || l.norder < m.ne) {
    l.order = nullptr;
    l.norder = 0;
  }
  const int tiles = l.order ? l.norder : m.ne;
  const int w = (tiles + TPW * sms - 1) / (TPW * sms);
  if (w > kLinStepsMaxWarps) return cudaErrorNotSupported;
  const size_t sm = sizeof(SOps<Dm>) + TPW * w * sizeof(LWarp<Dm>);
  const auto kern = w <= 8 ? kf_lin_steps<Dm, 8> : kf_lin_steps<Dm, kLinStepsMaxWarps>;
  int per_sm = 0;
  cudaError_t e = device_blocks_per_sm(kern, 32 * w, sm, &per_sm);
  if (e == cudaErrorInvalidConfiguration) return cudaErrorNotSupported;  // no room on an SM
  if (e != cudaSuccess) return e;
  const int grid = (tiles + TPW * w - 1) / (TPW * w);  // <= sms blocks, one per SM
  if (ls.nsteps <= 0) return cudaSuccess;
  e = cudaMemsetAsync(ls.count, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  DevOps o = op;
  DevMesh mm = m;
  void *args[] = {&o, &mm, &l};
  e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kern), dim3(grid),
                                  dim3(32 * w), args, sm, st);
  if (e == cudaSuccess) *launches += 1;
  return e;
}

template <class Dm>
cudaError_t run_lin(const DevOps &op, const DevMesh &m, const RhsBuffers &b, const StageArgs &sa,
                    cudaStream_t st, int sms, cudaEvent_t *ev) {
  constexpr int w = pick_warps(sizeof(SOps<Dm>), sizeof(LWarp<Dm>));
  constexpr size_t sm = sizeof(SOps<Dm>) + w * sizeof(LWarp<Dm>);
  int grid = 0;
  const cudaError_t e = resident_grid(kf_lin<Dm>, 32 * w, sm, sms, m.ne, w, &grid);
  if (e != cudaSuccess) return e;
  LinArgs la{b.su, b.sv, b.sh, b.g0, b.hh0};
  if (b.sh_ready) cudaStreamWaitEvent(st, b.sh_ready, 0);
  if (ev) cudaEventRecord(ev[0], st);
  kf_lin<Dm><<<grid, 32 * w, sm, st>>>(op, m, la, sa);
  if (ev) cudaEventRecord(ev[1], st);
  return cudaGetLastError();
}

template <class Dm>
cudaError_t run_any(int variant, const DevOps &op, const DevMesh &m, const RhsBuffers &b,
                    const StageArgs &sa, cudaStream_t st, int sms, cudaEvent_t *ev,
                    long long *launches) {
  switch (variant) {
    case kLIN: return run_lin<Dm>(op, m, b, sa, st, sms, ev);
    case kFS: return run_nl<Dm, kFS>(op, m, b, sa, st, sms, ev, launches);
    case kNS: return run_nl<Dm, kNS>(op, m, b, sa, st, sms, ev, launches);
    default: return run_nl<Dm, kINV>(op, m, b, sa, st, sms, ev, launches);
  }
}

}  // namespace

#if SPOC_FMA
#define FAST_AVAILABLE fast_available_fma
#define LAUNCH_FAST launch_rhs_fast_fma
#define LIN_STEPS_FAST lin_steps_fast_fma
#else
#define FAST_AVAILABLE fast_available
#define LAUNCH_FAST launch_rhs_fast
#define LIN_STEPS_FAST lin_steps_fast
#endif

bool FAST_AVAILABLE(int nc, int ng, int ngf) {
  return (nc == 3 && ng == 12 && ngf == 4) || (nc == 4 && ng == 25 && ngf == 5) ||
         (nc == 5 && ng == 27 && ngf == 6) || (nc == 6 && ng == 33 && ngf == 7) ||
         (nc == 7 && ng == 42 && ngf == 9);
}

#if !SPOC_FMA
template <class F>
bool with_fast_dims(int nc, int ng, int ngf, F &&f) {
  if (nc == 3 && ng == 12 && ngf == 4) return f(Dims<3, 12, 4>{}), true;
  if (nc == 4 && ng == 25 && ngf == 5) return f(Dims<4, 25, 5>{}), true;
  if (nc == 5 && ng == 27 && ngf == 6) return f(Dims<5, 27, 6>{}), true;
  if (nc == 6 && ng == 33 && ngf == 7) return f(Dims<6, 33, 7>{}), true;
  if (nc == 7 && ng == 42 && ngf == 9) return f(Dims<7, 42, 9>{}), true;
  return false;
}

size_t fast_image_bytes(int nc, int ng, int ngf, int which) {
  size_t n = 0;
  with_fast_dims(nc, ng, ngf, [&](auto d) {
    using Dm = decltype(d);
    n = which == 0 ? sizeof(SOps<Dm>) : sizeof(SOpsQ<Dm>);
  });
  return n;
}

cudaError_t fast_build_images(const DevOps &op, void *img, void *imgq, cudaStream_t st) {
  cudaError_t e = cudaErrorNotSupported;
  with_fast_dims(op.nc, op.ng, op.ngf, [&](auto d) {
    using Dm = decltype(d);
    e = cudaMemsetAsync(img, 0, sizeof(SOps<Dm>), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(imgq, 0, sizeof(SOpsQ<Dm>), st);
    if (e != cudaSuccess) return;
    k_fast_images<Dm><<<1, 256, 0, st>>>(op, static_cast<SOps<Dm> *>(img),
                                          static_cast<SOpsQ<Dm> *>(imgq));
    e = cudaGetLastError();
  });
  return e;
}

cudaError_t launch_qphase_fast(int variant, const DevOps &op, const DevMesh &m, const double *su,
                               const double *sv, double *q, cudaStream_t st, int sms) {
  const int nc = op.nc, ng = op.ng, ngf = op.ngf;
  auto go = [&](auto d) -> cudaError_t {
    using Dm = decltype(d);
    switch (variant) {
      case kFS: return run_q<Dm, kFS>(op, m, su, sv, q, st, sms);
      case kNS: return run_q<Dm, kNS>(op, m, su, sv, q, st, sms);
      case kINV: return run_q<Dm, kINV>(op, m, su, sv, q, st, sms);
      default: return cudaErrorNotSupported;
    }
  };
  if (nc == 3 && ng == 12 && ngf == 4) return go(Dims<3, 12, 4>{});
  if (nc == 4 && ng == 25 && ngf == 5) return go(Dims<4, 25, 5>{});
  if (nc == 5 && ng == 27 && ngf == 6) return go(Dims<5, 27, 6>{});
  if (nc == 6 && ng == 33 && ngf == 7) return go(Dims<6, 33, 7>{});
  if (nc == 7 && ng == 42 && ngf == 9) return go(Dims<7, 42, 9>{});
  return cudaErrorNotSupported;
}
#endif

cudaError_t LAUNCH_FAST(int variant, const DevOps &op, const DevMesh &m, const RhsBuffers &b,
                        const StageArgs &sa, cudaStream_t st, int sms, long long *launches,
                        cudaEvent_t *ev) {
  cudaError_t e = cudaErrorNotSupported;
  const int nc = op.nc, ng = op.ng, ngf = op.ngf;
  if (nc == 3 && ng == 12 && ngf == 4) e = run_any<Dims<3, 12, 4>>(variant, op, m, b, sa, st, sms, ev, launches);
  else if (nc == 4 && ng == 25 && ngf == 5) e = run_any<Dims<4, 25, 5>>(variant, op, m, b, sa, st, sms, ev, launches);
  else if (nc == 5 && ng == 27 && ngf == 6) e = run_any<Dims<5, 27, 6>>(variant, op, m, b, sa, st, sms, ev, launches);
  else if (nc == 6 && ng == 33 && ngf == 7) e = run_any<Dims<6, 33, 7>>(variant, op, m, b, sa, st, sms, ev, launches);
  else if (nc == 7 && ng == 42 && ngf == 9) e = run_any<Dims<7, 42, 9>>(variant, op, m, b, sa, st, sms, ev, launches);
  if (e == cudaSuccess && variant == kLIN) *launches += 1;
  return e;
}

cudaError_t LIN_STEPS_FAST(const DevOps &op, const DevMesh &m, const LinSteps &ls, cudaStream_t st,
                           int sms, long long *launches) {
  const int nc = op.nc, ng = op.ng, ngf = op.ngf;
  if (nc == 3 && ng == 12 && ngf == 4) return run_lin_steps<Dims<3, 12, 4>>(op, m, ls, st, sms, launches);
  if (nc == 4 && ng == 25 && ngf == 5) return run_lin_steps<Dims<4, 25, 5>>(op, m, ls, st, sms, launches);
  if (nc == 5 && ng == 27 && ngf == 6) return run_lin_steps<Dims<5, 27, 6>>(op, m, ls, st, sms, launches);
  if (nc == 6 && ng == 33 && ngf == 7) return run_lin_steps<Dims<6, 33, 7>>(op, m, ls, st, sms, launches);
  if (nc == 7 && ng == 42 && ngf == 9) return run_lin_steps<Dims<7, 42, 9>>(op, m, ls, st, sms, launches);
  return cudaErrorNotSupported;
}

}  // namespace spoc
