// Tensor-core (tcgen05) volume kernel of the mixed-precision right-hand side.
//
// Same mathematics as kx_vol (spoc_mixed.cu: orthonormal basis, mean-free
// face terms), organised for the 5th-generation tensor cores: a CTA owns a
// tile of 128 elements, element t of the tile is row t of every MMA and lane t
// of TMEM, and every contraction with a reference-element operator is one
// M = 128 TF32 MMA group D (128 x n) = A (128 x K) B^T with the operator as B.
// Each operand is split into a TF32 head and an FP32 tail and the group runs
// the three products hi*hi + lo*hi + hi*lo (FP32-level accuracy).  Thread t
// does the pointwise work of its element between the groups, reading its
// accumulators with tcgen05.ld and writing its A rows to shared memory.
//
// Per tile (W = 16-padded nm, WQ = 16-padded ng, WT = 16-padded 3 ngf):
//   1. u, v -> [GXm; GYm; Pp]; h -> Pp   (weak-gradient volume parts, u v h
//      at the quadrature points)
//   2. q = volume part (geometry applied in place in TMEM) + lift of the u, v
//      face values (MMA accumulating onto it); free-slip wall: the
//      tangential-normal component projected (calvarnl_fs.f:165-205)
//   3. F = mu0 q - g0 h -> [GXm; GYm]    (phase C volume terms)
//   4. q -> mean-free traces              (trace records for kx_tend)
//   5. q -> Pp, products at the quadrature points, Pp^T diag(w) -> load
//      vectors of -adu + w1, -adv + z1, uh, vh (phase B)
//   6. uh, vh wall projection; h volume terms -> [GXm, GYm]; uh, vh traces
// GXm / GYm / TRm skip the constant mode (its volume and face contributions
// cancel exactly; the face terms use the mean-free trace records).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "spoc_mixed.h"
#include "spoc_mixed_dev.cuh"
#include "spoc_tc.cuh"

namespace spoc {
using namespace mx;
namespace {

__host__ __device__ constexpr int rnd(int x, int m) { return (x + m - 1) / m * m; }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int pow2_cols(int c) {
  return c <= 32 ? 32 : (c <= 64 ? 64 : (c <= 128 ? 128 : (c <= 256 ? 256 : 512)));
}

template <class Dm>
struct TcDims {
  static constexpr int N = Dm::N, Q = Dm::Q, TG = Dm::TG;
  static constexpr int KN = rnd(N, 8), KQ = rnd(Q, 8), KT = rnd(TG, 8);
  static constexpr int KA = imax(KN, imax(KQ, KT));
  static constexpr int W = rnd(N, 16), WQ = rnd(Q, 16), WT = rnd(TG, 16);
  // operator rows (K = KN): GXm | GYm | Pp | TRm | Pwall
  static constexpr int R_GX = 0, R_GY = W, R_PP = 2 * W, R_TR = 2 * W + WQ;
  static constexpr int R_PW = 2 * W + WQ + WT, RB = 3 * W + WQ + WT;
  // image (floats): each operator head then tail; lift (K = KT), projection (K = KQ)
  static constexpr int O_BK = 0, L_BK = RB * KN;
  static constexpr int O_BL = 2 * L_BK, L_BL = W * KT;
  static constexpr int O_BP = O_BL + 2 * L_BL, L_BP = W * KQ;
  static constexpr int IMG = O_BP + 2 * L_BP;
  static constexpr int O_A = IMG, ABUF = 2 * 128 * KA;  // one A buffer: head, tail
  static constexpr size_t SMEM_NEED = sizeof(float) * (IMG + 2 * ABUF) + 64;
  // one CTA per SM: TMEM is allocated whole
  static constexpr size_t SMEM = SMEM_NEED > 118 * 1024 ? SMEM_NEED : 118 * 1024;
  // TMEM columns
  static constexpr int C_U = 0, C_V = 2 * W + WQ, C_H = 2 * (2 * W + WQ), S = C_H + WQ;
  static constexpr int C_END = S + imax(imax(2 * WQ + W, 4 * WT), 2 * W + 2 * WT);
  static constexpr int TCOLS = pow2_cols(C_END);
  static_assert(C_END <= 512, "tensor memory plan exceeds 512 columns");
  static_assert(W <= WQ && KN <= W, "layout assumes nm <= ng");
  static_assert(2 * W + WQ <= 256, "MMA N <= 256");
  static_assert(SMEM_NEED <= 227 * 1024, "shared memory plan exceeds 227 KB");
  static_assert(IMG % 4 == 0 && ABUF % 4 == 0, "16-byte staging");
};

constexpr uint32_t kWaitLimit = 1u << 26;

// Two A buffers, one mbarrier each, one commit per group; a buffer is
// rewritten, or the accumulators of its group read, only after waiting for
// its last commit.  All threads keep the same counts.
struct Pipe {
  uint64_t *mbar;
  uint32_t issued[2], waited[2];
  int *flag;
  __device__ __forceinline__ void wait(int b) {
    if (issued[b] > waited[b]) {
      if (!tc::mbar_wait(&mbar[b], (issued[b] - 1) & 1u, kWaitLimit) && threadIdx.x == 0)
        atomicOr(flag, 2);
      waited[b] = issued[b];
      tc::fence_after();
    }
  }
  __device__ __forceinline__ void commit(int b) {
    if (threadIdx.x == 0) tc::commit(&mbar[b]);
    ++issued[b];
  }
};

// A rows, TMEM stores and generic shared writes made visible to the MMA issue
__device__ __forceinline__ void sync_for_mma() {
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
}

// this thread's row of A buffer b (kpad columns): four values at column k
template <class T>
__device__ __forceinline__ void put4(float *sm, int b, int kpad, int k, float x0, float x1,
                                     float x2, float x3) {
  float4 h, l;
  tc::split_tf32(x0, h.x, l.x);
  tc::split_tf32(x1, h.y, l.y);
  tc::split_tf32(x2, h.z, l.z);
  tc::split_tf32(x3, h.w, l.w);
  float *hi = sm + T::O_A + b * T::ABUF;
  const uint32_t o = tc::kmaj_off(threadIdx.x, k, kpad) / 4;
  *reinterpret_cast<float4 *>(hi + o) = h;
  *reinterpret_cast<float4 *>(hi + 128 * T::KA + o) = l;
}
template <class T>
__device__ __forceinline__ void put8(float *sm, int b, int kpad, int k, const float (&x)[8]) {
  put4<T>(sm, b, kpad, k, x[0], x[1], x[2], x[3]);
  put4<T>(sm, b, kpad, k + 4, x[4], x[5], x[6], x[7]);
}

// MMA group (issued by thread 0): D[dcol .. dcol+n) (+)= A(b) B^T with B the
// rows r0 .. r0+n of the operator whose head starts at image offset bo and
// whose tail follows `tail` floats later; three-term TF32 split.
template <class T>
__device__ __forceinline__ void issue(float *sm, uint32_t tm, int b, int kpad, int bo, int tail,
                                      int r0, int n, int dcol, bool acc0) {
  if (threadIdx.x != 0) return;
  const uint32_t ah = tc::smem_u32(sm + T::O_A + b * T::ABUF);
  const uint32_t al = ah + 128u * T::KA * 4u;
  const uint32_t roff = (uint32_t)(r0 / 8) * (uint32_t)(kpad * 32);
  const uint32_t bh = tc::smem_u32(sm + bo) + roff, bl = tc::smem_u32(sm + bo + tail) + roff;
  const uint32_t id = tc::idesc_tf32(128, n);
  for (int s = 0; s < kpad / 8; ++s) {
    const uint32_t o = (uint32_t)s * 256u;
    tc::mma_tf32(tm + dcol, tc::sdesc(ah + o, kpad), tc::sdesc(bh + o, kpad), id,
                 (s > 0 || acc0) ? 1u : 0u);
    tc::mma_tf32(tm + dcol, tc::sdesc(al + o, kpad), tc::sdesc(bh + o, kpad), id, 1u);
    tc::mma_tf32(tm + dcol, tc::sdesc(ah + o, kpad), tc::sdesc(bl + o, kpad), id, 1u);
  }
}

template <class Dm, int VAR>
__global__ void __launch_bounds__(128, 1) kt_vol(const MxArgs a, const float *__restrict__ img) {
  using T = TcDims<Dm>;
  constexpr int N = Dm::N, Q = Dm::Q, G = Dm::G, TG = Dm::TG, TS = Dm::TS;
  constexpr int W = T::W, WQ = T::WQ, WT = T::WT, KN = T::KN, KQ = T::KQ, KT = T::KT;
  constexpr int BK = T::O_BK, BKT = T::L_BK;
  extern __shared__ __align__(1024) float sm[];
  const int t = threadIdx.x, warp = t >> 5;
  {
    const float4 *src = reinterpret_cast<const float4 *>(img);
    float4 *dst = reinterpret_cast<float4 *>(sm);
    for (int i = t; i < T::IMG / 4; i += 128) dst[i] = src[i];
  }
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + T::O_A + 2 * T::ABUF);
  uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 2);
  if (warp == 0) tc::tmem_alloc(slot, T::TCOLS);
  if (t == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    tc::fence_mbar_init();
  }
  sync_for_mma();
  const uint32_t tm = *slot;
  const uint32_t lrow = (uint32_t)(warp * 32) << 16;
  Pipe p{mbar, {0u, 0u}, {0u, 0u}, a.flag};
  const size_t fn = (size_t)a.ne * N, tn = (size_t)a.ne * TS;
  auto ld8 = [&](int col, float (&v)[8]) {
    tc::tmem_ld8(tm + lrow + (uint32_t)col, v);
    tc::tmem_wait_ld();
  };
  auto st8 = [&](int col, const float (&v)[8]) { tc::tmem_st8(tm + lrow + (uint32_t)col, v); };

  for (int tile = blockIdx.x; tile * 128 < a.ne; tile += gridDim.x) {
    const int e = tile * 128 + t;
    const bool valid = e < a.ne;
    float ax = 0.f, bx = 0.f, ay = 0.f, by = 0.f, di = 0.f, wnx = 0.f, wny = 0.f;
    bool wall = false;
    FaceRef fr[3];
    if (valid) {
      const double *vp = a.m.vect + 5 * (size_t)e;
      ax = (float)vp[0];
      bx = (float)vp[1];
      ay = (float)vp[2];
      by = (float)vp[3];
      di = (float)vp[4];
      wall = a.m.bdl[e] != 0;
      wnx = (float)a.m.normt[2 * (size_t)e];
      wny = (float)a.m.normt[2 * (size_t)e + 1];
#pragma unroll
      for (int k = 0; k < 3; ++k) fr[k] = face_ref(a.m, e, k);
    }
    auto Y = [&](int f, int k) -> float {
      return (valid && k < N) ? a.y[f * fn + (size_t)e * N + k] : 0.f;
    };

    // ---- 1. u, v -> [GXm; GYm; Pp], h -> Pp
    p.wait(0);
    for (int k = 0; k < KN; k += 4) put4<T>(sm, 0, KN, k, Y(0, k), Y(0, k + 1), Y(0, k + 2), Y(0, k + 3));
    sync_for_mma();
    issue<T>(sm, tm, 0, KN, BK, BKT, T::R_GX, 2 * W + WQ, T::C_U, false);
    p.commit(0);
    p.wait(1);
    for (int k = 0; k < KN; k += 4) put4<T>(sm, 1, KN, k, Y(1, k), Y(1, k + 1), Y(1, k + 2), Y(1, k + 3));
    sync_for_mma();
    issue<T>(sm, tm, 1, KN, BK, BKT, T::R_GX, 2 * W + WQ, T::C_V, false);
    p.commit(1);
    p.wait(0);
    for (int k = 0; k < KN; k += 4) put4<T>(sm, 0, KN, k, Y(2, k), Y(2, k + 1), Y(2, k + 2), Y(2, k + 3));
    sync_for_mma();
    issue<T>(sm, tm, 0, KN, BK, BKT, T::R_PP, WQ, T::C_H, false);
    p.commit(0);
    p.wait(1);
    p.wait(0);

    // ---- 2. q: geometry on the volume parts (calvarnl_fs.f:115-164), in place
    for (int c = 0; c < W; c += 8) {
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const int base = f == 0 ? T::C_U : T::C_V;
        float gx[8], gy[8], q0[8], q1[8];
        ld8(base + c, gx);
        ld8(base + W + c, gy);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          q0[j] = (ay * gy[j] - by * gx[j]) * di;
          q1[j] = (bx * gx[j] - ax * gy[j]) * di;
        }
        st8(base + c, q0);
        st8(base + W + c, q1);
      }
    }
    tc::tmem_wait_st();
    // lifts of the u (then v) face values, accumulated onto the volume parts
#pragma unroll 1
    for (int f = 0; f < 2; ++f) {
      p.wait(0);
      p.wait(1);
      const float *tr = a.tr_in + f * tn;
      for (int k4 = 0; k4 < KT; k4 += 4) {
        float x[4], z[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int l = k4 + jj;
          x[jj] = 0.f;
          z[jj] = 0.f;
          if (valid && l < TG) {
            const int side = l / G, j = l - side * G;
            const FaceRef &r = fr[side];
            const float fv = face_value<G>(tr, r, e, l, j);
            const float s = r.sig * di * a.wif[r.sig > 0.f ? j : G - 1 - j];
            x[jj] = s * r.nx * fv;
            z[jj] = s * r.ny * fv;
          }
        }
        put4<T>(sm, 0, KT, k4, x[0], x[1], x[2], x[3]);
        put4<T>(sm, 1, KT, k4, z[0], z[1], z[2], z[3]);
      }
      sync_for_mma();
      const int base = f == 0 ? T::C_U : T::C_V;
      issue<T>(sm, tm, 0, KT, T::O_BL, T::L_BL, 0, W, base, true);
      p.commit(0);
      issue<T>(sm, tm, 1, KT, T::O_BL, T::L_BL, 0, W, base + W, true);
      p.commit(1);
    }
    p.wait(0);
    p.wait(1);
    if (VAR == SPOC_FS && __syncthreads_or(wall)) {
      // calvarnl_fs.f:165-205: gtn = n.(grad u) t projected onto the wall sub-basis
      for (int c = 0; c < KN; c += 8) {
        float qa[8], qb[8], qc[8], qd[8], g[8];
        ld8(T::C_U + c, qa);
        ld8(T::C_U + W + c, qb);
        ld8(T::C_V + c, qc);
        ld8(T::C_V + W + c, qd);
#pragma unroll
        for (int j = 0; j < 8; ++j)
          g[j] = wall ? wnx * wny * qa[j] - wnx * wnx * qc[j] + wny * wny * qb[j] - wnx * wny * qd[j]
                      : 0.f;
        put8<T>(sm, 0, KN, c, g);
      }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_PW, W, T::S, false);
      p.commit(0);
      p.wait(0);
      for (int c = 0; c < W; c += 8) {
        float qa[8], qb[8], qc[8], qd[8], pg[8];
        ld8(T::C_U + c, qa);
        ld8(T::C_U + W + c, qb);
        ld8(T::C_V + c, qc);
        ld8(T::C_V + W + c, qd);
        ld8(T::S + c, pg);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float g = wnx * wny * qa[j] - wnx * wnx * qc[j] + wny * wny * qb[j] - wnx * wny * qd[j];
          const float d = wall ? pg[j] - g : 0.f;
          qa[j] += d * wnx * wny;
          qc[j] -= d * wnx * wnx;
          qb[j] += d * wny * wny;
          qd[j] -= d * wnx * wny;
        }
        st8(T::C_U + c, qa);
        st8(T::C_U + W + c, qb);
        st8(T::C_V + c, qc);
        st8(T::C_V + W + c, qd);
      }
      tc::tmem_wait_st();
    }

    // ---- 3. phase C volume terms: F = mu0 q - g0 h through [GXm; GYm]
#pragma unroll 1
    for (int pr = 0; pr < 2; ++pr) {
      // pr 0: (Fxx, Fxy) -> gx;  pr 1: (Fyx, Fyy) -> gy
      const int qa = pr == 0 ? T::C_U : T::C_V;
      p.wait(0);
      for (int c = 0; c < KN; c += 8) {
        float q[8], f[8];
        ld8(qa + c, q);
#pragma unroll
        for (int j = 0; j < 8; ++j) f[j] = a.mu0 * q[j] - (pr == 0 ? a.g0 * Y(2, c + j) : 0.f);
        put8<T>(sm, 0, KN, c, f);
      }
      p.wait(1);
      for (int c = 0; c < KN; c += 8) {
        float q[8], f[8];
        ld8(qa + W + c, q);
#pragma unroll
        for (int j = 0; j < 8; ++j) f[j] = a.mu0 * q[j] - (pr == 1 ? a.g0 * Y(2, c + j) : 0.f);
        put8<T>(sm, 1, KN, c, f);
      }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_GX, 2 * W, T::S, false);
      p.commit(0);
      p.wait(0);
      float acc[W];
#pragma unroll
      for (int c = 0; c < W; c += 8) {
        float gx[8], gy[8];
        ld8(T::S + c, gx);
        ld8(T::S + W + c, gy);
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[c + j] = di * (ay * gy[j] - by * gx[j]);
      }
      sync_for_mma();
      issue<T>(sm, tm, 1, KN, BK, BKT, T::R_GX, 2 * W, T::S, false);
      p.commit(1);
      p.wait(1);
#pragma unroll
      for (int c = 0; c < W; c += 8) {
        float gx[8], gy[8];
        ld8(T::S + c, gx);
        ld8(T::S + W + c, gy);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float v = acc[c + j] + di * (bx * gx[j] - ax * gy[j]);
          if (valid && c + j < N) a.part[pr * fn + (size_t)e * N + c + j] = v;
        }
      }
    }

    // ---- 4. trace records of q (mean-free traces, then the mean)
#pragma unroll 1
    for (int pr = 0; pr < 2; ++pr) {
      const int qa = pr == 0 ? T::C_U : T::C_V;
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        p.wait(b);
        for (int c = 0; c < KN; c += 8) {
          float q[8];
          ld8(qa + b * W + c, q);
          put8<T>(sm, b, KN, c, q);
        }
      }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_TR, WT, T::S + (2 * pr) * WT, false);
      p.commit(0);
      issue<T>(sm, tm, 1, KN, BK, BKT, T::R_TR, WT, T::S + (2 * pr + 1) * WT, false);
      p.commit(1);
    }
    p.wait(0);
    p.wait(1);
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
      const int qcol = (f < 2 ? T::C_U : T::C_V) + (f & 1) * W;
      float q0[8];
      ld8(qcol, q0);
      float *rec = a.trq + f * tn + (size_t)(valid ? e : 0) * TS;
      for (int c = 0; c < WT; c += 8) {
        float v[8];
        ld8(T::S + f * WT + c, v);
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (valid && c + j < TG) rec[c + j] = v[j];
      }
      if (valid) rec[TG] = a.psi0 * q0[0];
    }

    // ---- 5. phase B: q at the quadrature points, products, projections
#pragma unroll 1
    for (int pr = 0; pr < 2; ++pr) {
      const int qa = pr == 0 ? T::C_U : T::C_V;
      p.wait(0);
      for (int c = 0; c < KN; c += 8) {
        float q[8];
        ld8(qa + c, q);
        put8<T>(sm, 0, KN, c, q);
      }
      p.wait(1);
      for (int c = 0; c < KN; c += 8) {
        float q[8];
        ld8(qa + W + c, q);
        put8<T>(sm, 1, KN, c, q);
      }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_PP, WQ, T::S, false);
      p.commit(0);
      issue<T>(sm, tm, 1, KN, BK, BKT, T::R_PP, WQ, T::S + WQ, false);
      p.commit(1);
      p.wait(0);
      p.wait(1);
      // integrand: pr 0: wk/H - (U Gxx + V (Gxy - fc)); pr 1: zk/H - (U (Gyx + fc) + V Gyy)
      const int b = pr;  // buffer for the integrand
      for (int c = 0; c < KQ; c += 8) {
        float U[8], V[8], H[8], G1[8], G2[8], r[8];
        ld8(T::C_U + 2 * W + c, U);
        ld8(T::C_V + 2 * W + c, V);
        ld8(T::C_H + c, H);
        ld8(T::S + c, G1);
        ld8(T::S + WQ + c, G2);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int q = c + j;
          r[j] = 0.f;
          if (valid && q < Q) {
            const size_t qi = (size_t)e * Q + q;
            const float hq = H[j] + a.hbq[qi], fc = a.fcq[qi];
            if (pr == 0) {
              float wk = -a.mb0 * U[j];
              if (a.w0q) wk += a.w0q[qi];
              r[j] = wk / hq - (U[j] * G1[j] + V[j] * (G2[j] - fc));
            } else {
              float zk = -a.mb0 * V[j];
              if (a.z0q) zk += a.z0q[qi];
              r[j] = zk / hq - (U[j] * (G1[j] + fc) + V[j] * G2[j]);
            }
          }
        }
        put8<T>(sm, b, KQ, c, r);
      }
      sync_for_mma();
      // load vector of -adu + w1 -> S + 2 WQ; of -adv + z1 -> C_U (q_xx consumed)
      issue<T>(sm, tm, b, KQ, T::O_BP, T::L_BP, 0, W, pr == 0 ? T::S + 2 * WQ : T::C_U, false);
      p.commit(b);
    }
    // uh, vh integrands (U H, V H)
    p.wait(0);
    p.wait(1);
    for (int c = 0; c < KQ; c += 8) {
      float U[8], V[8], H[8], ru[8], rv[8];
      ld8(T::C_U + 2 * W + c, U);
      ld8(T::C_V + 2 * W + c, V);
      ld8(T::C_H + c, H);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int q = c + j;
        const float hq = (valid && q < Q) ? H[j] + a.hbq[(size_t)e * Q + q] : 0.f;
        ru[j] = (valid && q < Q) ? U[j] * hq : 0.f;
        rv[j] = (valid && q < Q) ? V[j] * hq : 0.f;
      }
      put8<T>(sm, 0, KQ, c, ru);
      put8<T>(sm, 1, KQ, c, rv);
    }
    sync_for_mma();
    issue<T>(sm, tm, 0, KQ, T::O_BP, T::L_BP, 0, W, T::C_U + W, false);  // uh
    p.commit(0);
    issue<T>(sm, tm, 1, KQ, T::O_BP, T::L_BP, 0, W, T::C_V, false);      // vh
    p.commit(1);
    p.wait(0);
    p.wait(1);
    // partial load vectors of u, v: projection + phase C volume terms
    for (int c = 0; c < W; c += 8) {
      float gx[8], gy[8];
      ld8(T::S + 2 * WQ + c, gx);
      ld8(T::C_U + c, gy);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (valid && c + j < N) {
          const size_t gi = (size_t)e * N + c + j;
          a.part[gi] += gx[j];
          a.part[fn + gi] += gy[j];
        }
    }

    // ---- 6. uh, vh: wall solves (calvarnl_fs.f:333-340, calvarnl_ns.f:249-265)
    if (__syncthreads_or(wall)) {
      for (int c = 0; c < KN; c += 8) {
        float uh[8], vh[8], g0v[8], g1v[8];
        ld8(T::C_U + W + c, uh);
        ld8(T::C_V + c, vh);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (VAR == SPOC_NS) {
            g0v[j] = wall ? uh[j] : 0.f;
            g1v[j] = wall ? vh[j] : 0.f;
          } else {
            g0v[j] = wall ? wnx * uh[j] + wny * vh[j] : 0.f;
            g1v[j] = 0.f;
          }
        }
        put8<T>(sm, 0, KN, c, g0v);
        if (VAR == SPOC_NS) put8<T>(sm, 1, KN, c, g1v);
      }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_PW, W, T::S, false);
      p.commit(0);
      if (VAR == SPOC_NS) {
        issue<T>(sm, tm, 1, KN, BK, BKT, T::R_PW, W, T::S + W, false);
        p.commit(1);
      }
      p.wait(0);
      p.wait(1);
      for (int c = 0; c < W; c += 8) {
        float uh[8], vh[8], p0[8], p1[8];
        ld8(T::C_U + W + c, uh);
        ld8(T::C_V + c, vh);
        ld8(T::S + c, p0);
        if (VAR == SPOC_NS) ld8(T::S + W + c, p1);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (VAR == SPOC_NS) {
            if (wall) {
              uh[j] = p0[j];
              vh[j] = p1[j];
            }
          } else {
            const float d = wall ? p0[j] - (wnx * uh[j] + wny * vh[j]) : 0.f;
            uh[j] += wnx * d;
            vh[j] += wny * d;
          }
        }
        st8(T::C_U + W + c, uh);
        st8(T::C_V + c, vh);
      }
      tc::tmem_wait_st();
    }
    // h volume terms (phase D): GXm (di (by uh - bx vh)) + GYm (di (ax vh - ay uh))
    p.wait(0);
    p.wait(1);
    for (int c = 0; c < KN; c += 8) {
      float uh[8], vh[8], hx[8], hy[8];
      ld8(T::C_U + W + c, uh);
      ld8(T::C_V + c, vh);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        hx[j] = di * (by * uh[j] - bx * vh[j]);
        hy[j] = di * (ax * vh[j] - ay * uh[j]);
      }
      put8<T>(sm, 0, KN, c, hx);
      put8<T>(sm, 1, KN, c, hy);
    }
    sync_for_mma();
    issue<T>(sm, tm, 0, KN, BK, BKT, T::R_GX, W, T::S + W, false);
    issue<T>(sm, tm, 1, KN, BK, BKT, T::R_GY, W, T::S + W, true);
    p.commit(0);
    p.commit(1);
    p.wait(0);
    p.wait(1);
    for (int c = 0; c < W; c += 8) {
      float hp[8];
      ld8(T::S + W + c, hp);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (valid && c + j < N) a.part[2 * fn + (size_t)e * N + c + j] = hp[j];
    }
    // trace records of uh, vh
    for (int c = 0; c < KN; c += 8) {
      float uh[8], vh[8];
      ld8(T::C_U + W + c, uh);
      ld8(T::C_V + c, vh);
      put8<T>(sm, 0, KN, c, uh);
      put8<T>(sm, 1, KN, c, vh);
    }
    sync_for_mma();
    issue<T>(sm, tm, 0, KN, BK, BKT, T::R_TR, WT, T::S + 2 * W, false);
    p.commit(0);
    issue<T>(sm, tm, 1, KN, BK, BKT, T::R_TR, WT, T::S + 2 * W + WT, false);
    p.commit(1);
    p.wait(0);
    p.wait(1);
#pragma unroll 1
    for (int f = 0; f < 2; ++f) {
      float m0[8];
      ld8(f == 0 ? T::C_U + W : T::C_V, m0);
      float *rec = a.trq + (4 + f) * tn + (size_t)(valid ? e : 0) * TS;
      for (int c = 0; c < WT; c += 8) {
        float v[8];
        ld8(T::S + 2 * W + f * WT + c, v);
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (valid && c + j < TG) rec[c + j] = v[j];
      }
      if (valid) rec[TG] = a.psi0 * m0[0];
    }
    // the next tile's first A writes wait on the buffers; TMEM reads above
    // completed (tcgen05.wait::ld) before any later MMA is issued
  }
  p.wait(0);
  p.wait(1);
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tm, T::TCOLS);
}

// tf32 head of x: round to nearest on the 13 dropped mantissa bits, ties away
float tf32_head(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// operator block (rows x kpad, K-major core-matrix layout): head at o, tail
// at o + rows * kpad
void put_block(std::vector<float> &img, int o, int rows, int kpad, int r, int k, double v) {
  const float x = (float)v, h = tf32_head(x);
  const uint32_t off = tc::kmaj_off(r, k, kpad) / 4;
  img[o + off] = h;
  img[o + rows * kpad + off] = x - h;
}

template <class Dm>
std::vector<float> image(const PsiOps &p, const double *wi) {
  using T = TcDims<Dm>;
  constexpr int N = Dm::N, Q = Dm::Q, TG = Dm::TG;
  std::vector<float> img(T::IMG, 0.f);
  for (int i = 0; i < N; ++i)
    for (int k = 1; k < N; ++k) {  // constant mode skipped (mean-free volume terms)
      put_block(img, T::O_BK, T::RB, T::KN, T::R_GX + i, k, p.GX[i * N + k]);
      put_block(img, T::O_BK, T::RB, T::KN, T::R_GY + i, k, p.GY[i * N + k]);
    }
  for (int q = 0; q < Q; ++q)
    for (int k = 0; k < N; ++k) put_block(img, T::O_BK, T::RB, T::KN, T::R_PP + q, k, p.Pp[q * N + k]);
  for (int l = 0; l < TG; ++l)
    for (int k = 1; k < N; ++k) put_block(img, T::O_BK, T::RB, T::KN, T::R_TR + l, k, p.TR[l * N + k]);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < N; ++k) put_block(img, T::O_BK, T::RB, T::KN, T::R_PW + i, k, p.PWALL[i * N + k]);
  for (int i = 0; i < N; ++i)
    for (int l = 0; l < TG; ++l) put_block(img, T::O_BL, T::W, T::KT, i, l, p.TR[l * N + i]);
  for (int i = 0; i < N; ++i)
    for (int q = 0; q < Q; ++q) put_block(img, T::O_BP, T::W, T::KQ, i, q, p.Pp[q * N + i] * wi[q]);
  return img;
}

template <class F>
bool tc_dims(int nc, int ng, int ngf, F &&f) {
  if (nc == 3 && ng == 12 && ngf == 4) return f(MDims<3, 12, 4>{}), true;
  if (nc == 4 && ng == 25 && ngf == 5) return f(MDims<4, 25, 5>{}), true;
  if (nc == 5 && ng == 27 && ngf == 6) return f(MDims<5, 27, 6>{}), true;
  if (nc == 6 && ng == 33 && ngf == 7) return f(MDims<6, 33, 7>{}), true;
  if (nc == 7 && ng == 42 && ngf == 9) return f(MDims<7, 42, 9>{}), true;
  return false;
}

}  // namespace

bool mixed_tc_available(int nc, int ng, int ngf) {
  return tc_dims(nc, ng, ngf, [](auto) {});
}

std::vector<float> mixed_tc_image(int nc, int ng, int ngf, const PsiOps &p, const double *wi) {
  std::vector<float> img;
  tc_dims(nc, ng, ngf, [&](auto d) { img = image<decltype(d)>(p, wi); });
  return img;
}

cudaError_t mixed_tc_vol(int variant, int nc, int ng, int ngf, const MxArgs &a, const float *img,
                         int sms, cudaStream_t st) {
  cudaError_t ce = cudaErrorInvalidValue;
  tc_dims(nc, ng, ngf, [&](auto d) {
    using Dm = decltype(d);
    using T = TcDims<Dm>;
    auto go = [&](auto kern) {
      ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
      if (ce != cudaSuccess) return;
      const int tiles = (a.ne + 127) / 128;
      const int grid = tiles < sms ? tiles : sms;
      kern<<<grid, 128, T::SMEM, st>>>(a, img);
      ce = cudaGetLastError();
    };
    if (variant == SPOC_FS) go(kt_vol<Dm, SPOC_FS>);
    else if (variant == SPOC_NS) go(kt_vol<Dm, SPOC_NS>);
    else go(kt_vol<Dm, SPOC_INV>);
  });
  return ce;
}

}  // namespace spoc
