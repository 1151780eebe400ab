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
constexpr int kTcThreads = 256;  // two threads per element of the 128-element tile

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
__device__ __forceinline__ void put4(float *sm, int b, int kpad, int row, int k, float x0, float x1,
                                     float x2, float x3) {
  float4 h, l;
  tc::split_tf32(x0, h.x, l.x);
  tc::split_tf32(x1, h.y, l.y);
  tc::split_tf32(x2, h.z, l.z);
  tc::split_tf32(x3, h.w, l.w);
  float *hi = sm + T::O_A + b * T::ABUF;
  const uint32_t o = tc::kmaj_off(row, k, kpad) / 4;
  *reinterpret_cast<float4 *>(hi + o) = h;
  *reinterpret_cast<float4 *>(hi + 128 * T::KA + o) = l;
}
template <class T>
__device__ __forceinline__ void put8(float *sm, int b, int kpad, int row, int k, const float (&x)[8]) {
  put4<T>(sm, b, kpad, row, k, x[0], x[1], x[2], x[3]);
  put4<T>(sm, b, kpad, row, k + 4, x[4], x[5], x[6], x[7]);
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
__global__ void __launch_bounds__(kTcThreads, 1) kt_vol(const MxArgs a, const float *__restrict__ img) {
  using T = TcDims<Dm>;
  constexpr int N = Dm::N, Q = Dm::Q, G = Dm::G, TG = Dm::TG, TS = Dm::TS;
  constexpr int W = T::W, WQ = T::WQ, WT = T::WT, KN = T::KN, KQ = T::KQ, KT = T::KT;
  constexpr int BK = T::O_BK, BKT = T::L_BK;
  extern __shared__ __align__(1024) float sm[];
  // two threads per element: thread t owns row t % 128 (its TMEM lane) and
  // the 8-column chunks of parity t / 128
  const int t = threadIdx.x, warp = t >> 5, row = t & 127, half = t >> 7;
  auto own = [&](int c) { return ((c >> 3) & 1) == half; };
  {
    const float4 *src = reinterpret_cast<const float4 *>(img);
    float4 *dst = reinterpret_cast<float4 *>(sm);
    for (int i = t; i < T::IMG / 4; i += kTcThreads) dst[i] = src[i];
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
  const uint32_t lrow = (uint32_t)((warp & 3) * 32) << 16;
  Pipe p{mbar, {0u, 0u}, {0u, 0u}, a.flag};
  const size_t fn = (size_t)a.ne * N, tn = (size_t)a.ne * TS;
  // TMEM loads are issued in batches and completed with one wait
  auto ld = [&](int col, float (&v)[8]) { tc::tmem_ld8(tm + lrow + (uint32_t)col, v); };
  auto ldw = [&]() { tc::tmem_wait_ld(); };
  auto st8 = [&](int col, const float (&v)[8]) { tc::tmem_st8(tm + lrow + (uint32_t)col, v); };

  for (int tile = blockIdx.x; tile * 128 < a.ne; tile += gridDim.x) {
    const int e = tile * 128 + row;
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
    const float *yrow = a.y + (size_t)(valid ? e : 0) * N;
    auto Y8 = [&](int f, int c, float (&v)[8]) {
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = (valid && c + j < N) ? __ldg(yrow + f * fn + c + j) : 0.f;
    };

    // ---- 1. u, v -> [GXm; GYm; Pp], h -> Pp
#pragma unroll 1
    for (int f = 0; f < 3; ++f) {
      const int b = f == 1 ? 1 : 0;
      p.wait(b);
      for (int c = 0; c < KN; c += 8)
        if (own(c)) {
          float v[8];
          Y8(f, c, v);
          put8<T>(sm, b, KN, row, c, v);
        }
      sync_for_mma();
      if (f < 2)
        issue<T>(sm, tm, b, KN, BK, BKT, T::R_GX, 2 * W + WQ, f == 0 ? T::C_U : T::C_V, false);
      else
        issue<T>(sm, tm, b, KN, BK, BKT, T::R_PP, WQ, T::C_H, false);
      p.commit(b);
    }
    p.wait(0);
    p.wait(1);

    // ---- 2. q: geometry on the volume parts (calvarnl_fs.f:115-164), in place
    for (int c = 0; c < W; c += 8)
      if (own(c)) {
        float gxu[8], gyu[8], gxv[8], gyv[8], r[8];
        ld(T::C_U + c, gxu);
        ld(T::C_U + W + c, gyu);
        ld(T::C_V + c, gxv);
        ld(T::C_V + W + c, gyv);
        ldw();
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = (ay * gyu[j] - by * gxu[j]) * di;
        st8(T::C_U + c, r);
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = (bx * gxu[j] - ax * gyu[j]) * di;
        st8(T::C_U + W + c, r);
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = (ay * gyv[j] - by * gxv[j]) * di;
        st8(T::C_V + c, r);
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = (bx * gxv[j] - ax * gyv[j]) * di;
        st8(T::C_V + W + c, r);
      }
    tc::tmem_wait_st();
    // lifts of the u (then v) face values, accumulated onto the volume parts
#pragma unroll 1
    for (int f = 0; f < 2; ++f) {
      p.wait(0);
      p.wait(1);
      const float *tr = a.tr_in + f * tn;
      // unrolled: the face of each point is known at compile time, so the
      // face references stay in registers
#pragma unroll
      for (int c = 0; c < KT; c += 8)
        if (own(c)) {
          float x[8], z[8];
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int l = c + jj;
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
          put8<T>(sm, 0, KT, row, c, x);
          put8<T>(sm, 1, KT, row, c, z);
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
      for (int c = 0; c < KN; c += 8)
        if (own(c)) {
          float qa[8], qb[8], qc[8], qd[8], g[8];
          ld(T::C_U + c, qa);
          ld(T::C_U + W + c, qb);
          ld(T::C_V + c, qc);
          ld(T::C_V + W + c, qd);
          ldw();
#pragma unroll
          for (int j = 0; j < 8; ++j)
            g[j] = wall ? wnx * wny * qa[j] - wnx * wnx * qc[j] + wny * wny * qb[j] - wnx * wny * qd[j]
                        : 0.f;
          put8<T>(sm, 0, KN, row, c, g);
        }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_PW, W, T::S, false);
      p.commit(0);
      p.wait(0);
      for (int c = 0; c < W; c += 8)
        if (own(c)) {
          float qa[8], qb[8], qc[8], qd[8], pg[8];
          ld(T::C_U + c, qa);
          ld(T::C_U + W + c, qb);
          ld(T::C_V + c, qc);
          ld(T::C_V + W + c, qd);
          ld(T::S + c, pg);
          ldw();
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
      p.wait(1);
      for (int c = 0; c < KN; c += 8)
        if (own(c)) {
          float q0[8], q1[8], h[8], f0[8], f1[8];
          ld(qa + c, q0);
          ld(qa + W + c, q1);
          Y8(2, c, h);
          ldw();
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            f0[j] = a.mu0 * q0[j] - (pr == 0 ? a.g0 * h[j] : 0.f);
            f1[j] = a.mu0 * q1[j] - (pr == 1 ? a.g0 * h[j] : 0.f);
          }
          put8<T>(sm, 0, KN, row, c, f0);
          put8<T>(sm, 1, KN, row, c, f1);
        }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_GX, 2 * W, T::S, false);
      p.commit(0);
      p.wait(0);
      float acc[W];
#pragma unroll
      for (int c = 0; c < W; c += 8)
        if (own(c)) {
          float gx[8], gy[8];
          ld(T::S + c, gx);
          ld(T::S + W + c, gy);
          ldw();
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[c + j] = di * (ay * gy[j] - by * gx[j]);
        }
      sync_for_mma();
      issue<T>(sm, tm, 1, KN, BK, BKT, T::R_GX, 2 * W, T::S, false);
      p.commit(1);
      p.wait(1);
#pragma unroll
      for (int c = 0; c < W; c += 8)
        if (own(c)) {
          float gx[8], gy[8];
          ld(T::S + c, gx);
          ld(T::S + W + c, gy);
          ldw();
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
      p.wait(0);
      p.wait(1);
      for (int c = 0; c < KN; c += 8)
        if (own(c)) {
          float q0[8], q1[8];
          ld(qa + c, q0);
          ld(qa + W + c, q1);
          ldw();
          put8<T>(sm, 0, KN, row, c, q0);
          put8<T>(sm, 1, KN, row, c, q1);
        }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_TR, WT, T::S + (2 * pr) * WT, false);
      p.commit(0);
      issue<T>(sm, tm, 1, KN, BK, BKT, T::R_TR, WT, T::S + (2 * pr + 1) * WT, false);
      p.commit(1);
    }
    p.wait(0);
    p.wait(1);
    {
      float m[4][8];
      ld(T::C_U, m[0]);
      ld(T::C_U + W, m[1]);
      ld(T::C_V, m[2]);
      ld(T::C_V + W, m[3]);
      ldw();
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        float *rec = a.trq + f * tn + (size_t)(valid ? e : 0) * TS;
        for (int c = 0; c < WT; c += 8)
          if (own(c)) {
            float v[8];
            ld(T::S + f * WT + c, v);
            ldw();
#pragma unroll
            for (int j = 0; j < 8; ++j)
              if (valid && c + j < TG) rec[c + j] = v[j];
          }
        if (valid && half == 0) rec[TG] = a.psi0 * m[f][0];
      }
    }

    // ---- 5. phase B: q at the quadrature points, products, projections
#pragma unroll 1
    for (int pr = 0; pr < 2; ++pr) {
      const int qa = pr == 0 ? T::C_U : T::C_V;
      p.wait(0);
      p.wait(1);
      for (int c = 0; c < KN; c += 8)
        if (own(c)) {
          float q0[8], q1[8];
          ld(qa + c, q0);
          ld(qa + W + c, q1);
          ldw();
          put8<T>(sm, 0, KN, row, c, q0);
          put8<T>(sm, 1, KN, row, c, q1);
        }
      sync_for_mma();
      issue<T>(sm, tm, 0, KN, BK, BKT, T::R_PP, WQ, T::S, false);
      p.commit(0);
      issue<T>(sm, tm, 1, KN, BK, BKT, T::R_PP, WQ, T::S + WQ, false);
      p.commit(1);
      p.wait(0);
      p.wait(1);
      // integrand: pr 0: wk/H - (U Gxx + V (Gxy - fc)); pr 1: zk/H - (U (Gyx + fc) + V Gyy)
      const int b = pr;
      for (int c = 0; c < KQ; c += 8)
        if (own(c)) {
          float U[8], V[8], H[8], G1[8], G2[8], r[8];
          ld(T::C_U + 2 * W + c, U);
          ld(T::C_V + 2 * W + c, V);
          ld(T::C_H + c, H);
          ld(T::S + c, G1);
          ld(T::S + WQ + c, G2);
          float hb[8], fc[8], w[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int q = c + j;
            const bool in = valid && q < Q;
            const size_t qi = (size_t)(valid ? e : 0) * Q + (q < Q ? q : 0);
            hb[j] = in ? __ldg(a.hbq + qi) : 1.f;
            fc[j] = in ? __ldg(a.fcq + qi) : 0.f;
            const float *wz = pr == 0 ? a.w0q : a.z0q;
            w[j] = (in && wz) ? __ldg(wz + qi) : 0.f;
          }
          ldw();
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float hq = H[j] + hb[j];
            if (pr == 0)
              r[j] = (w[j] - a.mb0 * U[j]) / hq - (U[j] * G1[j] + V[j] * (G2[j] - fc[j]));
            else
              r[j] = (w[j] - a.mb0 * V[j]) / hq - (U[j] * (G1[j] + fc[j]) + V[j] * G2[j]);
            if (!(valid && c + j < Q)) r[j] = 0.f;
          }
          put8<T>(sm, b, KQ, row, c, r);
        }
      sync_for_mma();
      // load vector of -adu + w1 -> S + 2 WQ; of -adv + z1 -> C_U (q_xx consumed)
      issue<T>(sm, tm, b, KQ, T::O_BP, T::L_BP, 0, W, pr == 0 ? T::S + 2 * WQ : T::C_U, false);
      p.commit(b);
    }
    // uh, vh integrands (U H, V H)
    p.wait(0);
    p.wait(1);
    for (int c = 0; c < KQ; c += 8)
      if (own(c)) {
        float U[8], V[8], H[8], ru[8], rv[8], hb[8];
        ld(T::C_U + 2 * W + c, U);
        ld(T::C_V + 2 * W + c, V);
        ld(T::C_H + c, H);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int q = c + j;
          hb[j] = (valid && q < Q) ? __ldg(a.hbq + (size_t)e * Q + q) : 0.f;
        }
        ldw();
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const bool in = valid && c + j < Q;
          const float hq = H[j] + hb[j];
          ru[j] = in ? U[j] * hq : 0.f;
          rv[j] = in ? V[j] * hq : 0.f;
        }
        put8<T>(sm, 0, KQ, row, c, ru);
        put8<T>(sm, 1, KQ, row, c, rv);
      }
    sync_for_mma();
    issue<T>(sm, tm, 0, KQ, T::O_BP, T::L_BP, 0, W, T::C_U + W, false);  // uh
    p.commit(0);
    issue<T>(sm, tm, 1, KQ, T::O_BP, T::L_BP, 0, W, T::C_V, false);      // vh
    p.commit(1);
    p.wait(0);
    p.wait(1);
    // partial load vectors of u, v: projection + phase C volume terms
    for (int c = 0; c < W; c += 8)
      if (own(c)) {
        float gx[8], gy[8];
        ld(T::S + 2 * WQ + c, gx);
        ld(T::C_U + c, gy);
        ldw();
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
      for (int c = 0; c < KN; c += 8)
        if (own(c)) {
          float uh[8], vh[8], g0v[8], g1v[8];
          ld(T::C_U + W + c, uh);
          ld(T::C_V + c, vh);
          ldw();
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
          put8<T>(sm, 0, KN, row, c, g0v);
          if (VAR == SPOC_NS) put8<T>(sm, 1, KN, row, c, g1v);
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
      for (int c = 0; c < W; c += 8)
        if (own(c)) {
          float uh[8], vh[8], p0[8], p1[8];
          ld(T::C_U + W + c, uh);
          ld(T::C_V + c, vh);
          ld(T::S + c, p0);
          if (VAR == SPOC_NS) ld(T::S + W + c, p1);
          ldw();
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
    // h volume terms (phase D)
    p.wait(0);
    p.wait(1);
    for (int c = 0; c < KN; c += 8)
      if (own(c)) {
        float uh[8], vh[8], hx[8], hy[8];
        ld(T::C_U + W + c, uh);
        ld(T::C_V + c, vh);
        ldw();
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          hx[j] = di * (by * uh[j] - bx * vh[j]);
          hy[j] = di * (ax * vh[j] - ay * uh[j]);
        }
        put8<T>(sm, 0, KN, row, c, hx);
        put8<T>(sm, 1, KN, row, c, hy);
      }
    sync_for_mma();
    issue<T>(sm, tm, 0, KN, BK, BKT, T::R_GX, W, T::S + W, false);
    issue<T>(sm, tm, 1, KN, BK, BKT, T::R_GY, W, T::S + W, true);
    p.commit(0);
    p.commit(1);
    p.wait(0);
    p.wait(1);
    // h partial load vector, and the A rows of uh, vh for their traces
    for (int c = 0; c < KN; c += 8)
      if (own(c)) {
        float hp[8], uh[8], vh[8];
        ld(T::S + W + c, hp);
        ld(T::C_U + W + c, uh);
        ld(T::C_V + c, vh);
        ldw();
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (valid && c + j < N) a.part[2 * fn + (size_t)e * N + c + j] = hp[j];
        put8<T>(sm, 0, KN, row, c, uh);
        put8<T>(sm, 1, KN, row, c, vh);
      }
    sync_for_mma();
    issue<T>(sm, tm, 0, KN, BK, BKT, T::R_TR, WT, T::S + 2 * W, false);
    p.commit(0);
    issue<T>(sm, tm, 1, KN, BK, BKT, T::R_TR, WT, T::S + 2 * W + WT, false);
    p.commit(1);
    p.wait(0);
    p.wait(1);
    {
      float m0[8], m1[8];
      ld(T::C_U + W, m0);
      ld(T::C_V, m1);
      ldw();
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        float *rec = a.trq + (4 + f) * tn + (size_t)(valid ? e : 0) * TS;
        for (int c = 0; c < WT; c += 8)
          if (own(c)) {
            float v[8];
            ld(T::S + 2 * W + f * WT + c, v);
            ldw();
#pragma unroll
            for (int j = 0; j < 8; ++j)
              if (valid && c + j < TG) rec[c + j] = v[j];
          }
        if (valid && half == 0) rec[TG] = a.psi0 * (f == 0 ? m0[0] : m1[0]);
      }
    }
    // the next tile waits on the A buffers before rewriting them; every TMEM
    // read above completed (tcgen05.wait::ld) before the next MMA issue
  }
  p.wait(0);
  p.wait(1);
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tm, T::TCOLS);
}

// ---------------------------------------------------------------------------
// Tensor-core tendency kernel (kt_tend): the face lifts of phases C, D, the
// wall projections and the traces of the next stage input as tcgen05 MMA
// groups, the RK4 update in FP64 between them; the same mathematics as
// kx_tend (spoc_mixed.cu).  Per 128-element tile:
//   1. face fluxes of the three tendencies at the 3 ngf face points (from the
//      trace records of q, uh, vh and of the stage input's h) -> three A
//      tiles; D_f (128 x W) = A_f TR  (the lift TR_s^T, all modes);
//   2. t_f = D_f + the partial load vectors of the volume kernel; wall
//      elements: projection onto the wall subspace by an MMA with Pwall;
//   3. RK4 update (FP64 psi state and accumulator) -> next stage input y;
//   4. D_f (128 x WT) = y_f TRm^T -> mean-free trace records, then the mean.
// Shared memory: the TRm, Pwall and lift blocks of the tensor-core image
// (head and TF32 tail of each) and three A tiles (head and tail).
template <class Dm>
struct TcTend {
  using T = TcDims<Dm>;
  static constexpr int W = T::W, WT = T::WT, KN = T::KN, KT = T::KT;
  static constexpr int KA = KN > KT ? KN : KT;
  static constexpr int O_TR = 0, L_TR = WT * KN;        // trace rows (K = KN)
  static constexpr int O_PW = O_TR + 2 * L_TR, L_PW = W * KN;
  static constexpr int O_L = O_PW + 2 * L_PW, L_L = W * KT;
  static constexpr int IMG = O_L + 2 * L_L;
  static constexpr int O_A = IMG, ABUF = 2 * 128 * KA;  // one A tile: head, tail
  static constexpr size_t SMEM = sizeof(float) * (IMG + 3 * ABUF) + 64;
  // TMEM: the three lifted tendencies, then two projection outputs; the
  // trace outputs reuse columns 0 .. 3 WT once the lifts are read
  static constexpr int C_S = 3 * W, C_END = 5 * W;
  static constexpr int TCOLS = pow2_cols(C_END);
  static_assert(C_END <= 512 && 3 * WT <= 3 * W, "tensor memory plan");
  static_assert(SMEM <= 227 * 1024, "shared memory plan exceeds 227 KB");
  static_assert(IMG % 4 == 0 && ABUF % 4 == 0 && T::R_TR % 8 == 0 && T::R_PW % 8 == 0,
                "16-byte staging of whole row groups");
};

// MMA group on explicit operand addresses (thread 0): D[dcol .. dcol+n) (+)=
// A B^T, A and B K-major with kpad columns, heads at ah / bh, tails at al / bl.
__device__ __forceinline__ void issue_ab(uint32_t tm, uint32_t ah, uint32_t al, uint32_t bh,
                                         uint32_t bl, int kpad, int n, int dcol, bool acc0) {
  if (threadIdx.x != 0) return;
  const uint32_t id = tc::idesc_tf32(128, n);
  for (int s = 0; s < kpad / 8; ++s) {
    const uint32_t o = (uint32_t)s * 256u;
    tc::mma_tf32(tm + dcol, tc::sdesc(ah + o, kpad), tc::sdesc(bh + o, kpad), id,
                 (s > 0 || acc0) ? 1u : 0u);
    tc::mma_tf32(tm + dcol, tc::sdesc(al + o, kpad), tc::sdesc(bh + o, kpad), id, 1u);
    tc::mma_tf32(tm + dcol, tc::sdesc(ah + o, kpad), tc::sdesc(bl + o, kpad), id, 1u);
  }
}

// Three A tiles, one mbarrier each (the two-buffer Pipe of kt_vol, widened).
struct Pipe3 {
  uint64_t *mbar;
  uint32_t issued[3], waited[3];
  int *flag;
  __device__ __forceinline__ void wait(int b) {
    if (issued[b] > waited[b]) {
      if (!tc::mbar_wait(&mbar[b], (issued[b] - 1) & 1u, kWaitLimit) && threadIdx.x == 0)
        atomicOr(flag, 2);
      waited[b] = issued[b];
      tc::fence_after();
    }
  }
  __device__ __forceinline__ void wait_all() {
    wait(0);
    wait(1);
    wait(2);
  }
  __device__ __forceinline__ void commit(int b) {
    if (threadIdx.x == 0) tc::commit(&mbar[b]);
    ++issued[b];
  }
};

template <class Dm, int VAR>
__global__ void __launch_bounds__(kTcThreads, 1) kt_tend(const MxArgs a, const float *__restrict__ img) {
  using T = TcDims<Dm>;
  using U = TcTend<Dm>;
  constexpr int N = Dm::N, G = Dm::G, TG = Dm::TG, TS = Dm::TS;
  constexpr int W = U::W, WT = U::WT, KN = U::KN, KT = U::KT, KA = U::KA;
  extern __shared__ __align__(1024) float sm[];
  const int t = threadIdx.x, warp = t >> 5, row = t & 127, half = t >> 7;
  auto own = [&](int c) { return ((c >> 3) & 1) == half; };
  // the TRm and Pwall row groups of the operator block and the lift block
  {
    const float4 *g = reinterpret_cast<const float4 *>(img);
    float4 *d = reinterpret_cast<float4 *>(sm);
    auto copy = [&](int dst, int src, int n) {
      for (int i = t; i < n / 4; i += kTcThreads) d[dst / 4 + i] = g[src / 4 + i];
    };
    const int tr = T::O_BK + (T::R_TR / 8) * (KN * 8), pw = T::O_BK + (T::R_PW / 8) * (KN * 8);
    const int tail = T::RB * KN;
    copy(U::O_TR, tr, U::L_TR);
    copy(U::O_TR + U::L_TR, tr + tail, U::L_TR);
    copy(U::O_PW, pw, U::L_PW);
    copy(U::O_PW + U::L_PW, pw + tail, U::L_PW);
    copy(U::O_L, T::O_BL, U::L_L);
    copy(U::O_L + U::L_L, T::O_BL + T::L_BL, U::L_L);
  }
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + U::O_A + 3 * U::ABUF);
  uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 3);
  if (warp == 0) tc::tmem_alloc(slot, U::TCOLS);
  if (t == 0) {
    for (int b = 0; b < 3; ++b) tc::mbar_init(&mbar[b], 1);
    tc::fence_mbar_init();
  }
  sync_for_mma();
  const uint32_t tm = *slot;
  const uint32_t lrow = (uint32_t)((warp & 3) * 32) << 16;
  Pipe3 p{mbar, {0u, 0u, 0u}, {0u, 0u, 0u}, a.flag};
  const size_t fn = (size_t)a.ne * N, tn = (size_t)a.ne * TS;
  auto ld = [&](int col, float (&v)[8]) { tc::tmem_ld8(tm + lrow + (uint32_t)col, v); };
  auto ldw = [&]() { tc::tmem_wait_ld(); };
  auto abuf = [&](int b) { return sm + U::O_A + b * U::ABUF; };
  // this thread's row of A tile b (kpad columns): eight values at column k
  auto put8a = [&](int b, int kpad, int k, const float (&x)[8]) {
    float *hi = abuf(b);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      float4 h, l;
      tc::split_tf32(x[4 * q + 0], h.x, l.x);
      tc::split_tf32(x[4 * q + 1], h.y, l.y);
      tc::split_tf32(x[4 * q + 2], h.z, l.z);
      tc::split_tf32(x[4 * q + 3], h.w, l.w);
      const uint32_t o = tc::kmaj_off(row, k + 4 * q, kpad) / 4;
      *reinterpret_cast<float4 *>(hi + o) = h;
      *reinterpret_cast<float4 *>(hi + 128 * KA + o) = l;
    }
  };
  auto group = [&](int b, int kpad, int bo, int lb, int n, int dcol) {
    const uint32_t ah = tc::smem_u32(abuf(b)), al = ah + 128u * KA * 4u;
    issue_ab(tm, ah, al, tc::smem_u32(sm + bo), tc::smem_u32(sm + bo + lb), kpad, n, dcol, false);
  };

  for (int tile = blockIdx.x; tile * 128 < a.ne; tile += gridDim.x) {
    const int e = tile * 128 + row;
    const bool valid = e < a.ne;
    float di = 0.f, wnx = 0.f, wny = 0.f;
    bool wall = false;
    FaceRef fr[3];
    if (valid) {
      di = (float)a.m.vect[5 * (size_t)e + 4];
      wall = a.m.bdl[e] != 0;
      wnx = (float)a.m.normt[2 * (size_t)e];
      wny = (float)a.m.normt[2 * (size_t)e + 1];
#pragma unroll
      for (int k = 0; k < 3; ++k) fr[k] = face_ref(a.m, e, k);
    }

    // ---- 1. face fluxes of the three tendencies, lifted by the MMA
    p.wait_all();
#pragma unroll
    for (int c = 0; c < KT; c += 8)
      if (own(c)) {
        float x[3][8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int l = c + jj;
          x[0][jj] = x[1][jj] = x[2][jj] = 0.f;
          if (valid && l < TG) {
            const int side = l / G, j = l - side * G;
            const FaceRef &r = fr[side];
            const float fqxx = face_value<G>(a.trq, r, e, l, j);
            const float fqxy = face_value<G>(a.trq + tn, r, e, l, j);
            const float fqyx = face_value<G>(a.trq + 2 * tn, r, e, l, j);
            const float fqyy = face_value<G>(a.trq + 3 * tn, r, e, l, j);
            const float fuh = face_value<G>(a.trq + 4 * tn, r, e, l, j);
            const float fvh = face_value<G>(a.trq + 5 * tn, r, e, l, j);
            const float fh = face_value<G>(a.tr_in + 2 * tn, r, e, l, j);
            const float Fxx = a.mu0 * fqxx - a.g0 * fh, Fxy = a.mu0 * fqxy;
            const float Fyx = a.mu0 * fqyx, Fyy = a.mu0 * fqyy - a.g0 * fh;
            const float s = r.sig * di * a.wif[r.sig > 0.f ? j : G - 1 - j];
            x[0][jj] = s * (r.nx * Fxx + r.ny * Fxy);
            x[1][jj] = s * (r.nx * Fyx + r.ny * Fyy);
            x[2][jj] = -s * (r.nx * fuh + r.ny * fvh);
          }
        }
#pragma unroll
        for (int f = 0; f < 3; ++f) put8a(f, KT, c, x[f]);
      }
    sync_for_mma();
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      group(f, KT, U::O_L, U::L_L, W, f * W);
      p.commit(f);
    }
    p.wait_all();

    // ---- 2. tendencies: lifts + partial load vectors; wall projection
    const bool any_wall = __syncthreads_or(wall);
    if (any_wall) {
      // FS / INV: the normal component gn = n.(gx, gy) is projected; NS:
      // both components
      for (int c = 0; c < KN; c += 8)
        if (own(c)) {
          float dx[8], dy[8], g0v[8], g1v[8];
          ld(0 * W + c, dx);
          ld(1 * W + c, dy);
          ldw();
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int i = c + jj;
            const bool in = valid && i < N;
            const float tx = in ? dx[jj] + a.part[(size_t)e * N + i] : 0.f;
            const float ty = in ? dy[jj] + a.part[fn + (size_t)e * N + i] : 0.f;
            if (VAR == SPOC_NS) {
              g0v[jj] = wall ? tx : 0.f;
              g1v[jj] = wall ? ty : 0.f;
            } else {
              g0v[jj] = wall ? wnx * tx + wny * ty : 0.f;
              g1v[jj] = 0.f;
            }
          }
          put8a(0, KN, c, g0v);
          if (VAR == SPOC_NS) put8a(1, KN, c, g1v);
        }
      sync_for_mma();
      group(0, KN, U::O_PW, U::L_PW, W, U::C_S);
      p.commit(0);
      if (VAR == SPOC_NS) {
        group(1, KN, U::O_PW, U::L_PW, W, U::C_S + W);
        p.commit(1);
      }
      p.wait_all();
    }

    // ---- 3. RK4 update (FP64 psi state); the next stage input as A tiles
    bool bad = false;
    for (int c = 0; c < KN; c += 8)
      if (own(c)) {
        float d[3][8], pg0[8], pg1[8];
        ld(0 * W + c, d[0]);
        ld(1 * W + c, d[1]);
        ld(2 * W + c, d[2]);
        if (any_wall) {
          ld(U::C_S + c, pg0);
          if (VAR == SPOC_NS) ld(U::C_S + W + c, pg1);
        }
        ldw();
        float y[3][8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int i = c + jj;
          const bool in = valid && i < N;
          float tf[3];
#pragma unroll
          for (int f = 0; f < 3; ++f)
            tf[f] = in ? d[f][jj] + a.part[f * fn + (size_t)e * N + i] : 0.f;
          if (in && wall) {
            if (VAR == SPOC_NS) {
              tf[0] = pg0[jj];
              tf[1] = pg1[jj];
            } else {
              const float gn = wnx * tf[0] + wny * tf[1];
              const float dd = pg0[jj] - gn;
              tf[0] += wnx * dd;
              tf[1] += wny * dd;
            }
          }
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            y[f][jj] = 0.f;
            if (!in) continue;
            bad |= !isfinite(tf[f]);
            const size_t gi = f * fn + (size_t)e * N + i;
            if (a.stage < 0) {
              a.k64[gi] = (double)tf[f];
            } else {
              const float y32 = (float)rk4_update(a, gi, (double)tf[f]);
              a.y[gi] = y32;
              y[f][jj] = y32;
            }
          }
        }
        if (a.stage >= 0) {
#pragma unroll
          for (int f = 0; f < 3; ++f) put8a(f, KN, c, y[f]);
        }
        if (a.stage >= 0 && c == 0 && valid) {
          // the mean of each field: the constant mode's coefficient
#pragma unroll
          for (int f = 0; f < 3; ++f) a.tr_out[f * tn + (size_t)e * TS + TG] = a.psi0 * y[f][0];
        }
      }
    if (bad) atomicOr(a.flag, 1);
    if (a.stage < 0) continue;

    // ---- 4. mean-free traces of the next stage input
    tc::tmem_wait_ld();  // the lifted columns are read: the traces reuse them
    sync_for_mma();
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      group(f, KN, U::O_TR, U::L_TR, WT, f * WT);
      p.commit(f);
    }
    p.wait_all();
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      float *rec = a.tr_out + f * tn + (size_t)(valid ? e : 0) * TS;
      for (int c = 0; c < WT; c += 8)
        if (own(c)) {
          float v[8];
          ld(f * WT + c, v);
          ldw();
#pragma unroll
          for (int jj = 0; jj < 8; ++jj)
            if (valid && c + jj < TG) rec[c + jj] = v[jj];
        }
    }
    // the trace columns are read before the next tile's lifts overwrite them
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
  }
  p.wait_all();
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tm, U::TCOLS);
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
  // head and tail both rounded to TF32 (the tensor core truncates the bits
  // below), the tail taken from the FP64 value
  const float h = tf32_head((float)v), l = tf32_head((float)(v - (double)h));
  const uint32_t off = tc::kmaj_off(r, k, kpad) / 4;
  img[o + off] = h;
  img[o + rows * kpad + off] = l;
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
      kern<<<grid, kTcThreads, T::SMEM, st>>>(a, img);
      ce = cudaGetLastError();
    };
    if (variant == SPOC_FS) go(kt_vol<Dm, SPOC_FS>);
    else if (variant == SPOC_NS) go(kt_vol<Dm, SPOC_NS>);
    else go(kt_vol<Dm, SPOC_INV>);
  });
  return ce;
}

cudaError_t mixed_tc_tend(int variant, int nc, int ng, int ngf, const MxArgs &a, const float *img,
                          int sms, cudaStream_t st) {
  cudaError_t ce = cudaErrorInvalidValue;
  tc_dims(nc, ng, ngf, [&](auto d) {
    using Dm = decltype(d);
    using U = TcTend<Dm>;
    auto go = [&](auto kern) {
      ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)U::SMEM);
      if (ce != cudaSuccess) return;
      const int tiles = (a.ne + 127) / 128;
      const int grid = tiles < sms ? tiles : sms;
      kern<<<grid, kTcThreads, U::SMEM, st>>>(a, img);
      ce = cudaGetLastError();
    };
    if (variant == SPOC_FS) go(kt_tend<Dm, SPOC_FS>);
    else if (variant == SPOC_NS) go(kt_tend<Dm, SPOC_NS>);
    else go(kt_tend<Dm, SPOC_INV>);
  });
  return ce;
}

}  // namespace spoc
