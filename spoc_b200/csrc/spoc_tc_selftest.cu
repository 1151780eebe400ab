// Self-test of the tcgen05 building blocks (spoc_tc.cuh): one CTA computes
// D (128 x N) = A (128 x K) B^T (B: N x K) with TF32 MMAs into TMEM, either as
// one TF32 product or as the three-term split hi*hi + lo*hi + hi*lo, optionally
// accumulating onto a D first stored into TMEM by the threads.  The mixed
// kernels rely on exactly these layouts, descriptors and TMEM access shapes.
#include <cuda_runtime.h>

#include "../../include/spoc_gpu.h"
#include "spoc_tc.cuh"

namespace spoc {
namespace {

template <int KPAD, int N>
__global__ void __launch_bounds__(128) k_tc_selftest(const float *A, const float *B, float *D,
                                                     const float *Dinit, int K, int split,
                                                     int *err) {
  constexpr int NCOLS = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  extern __shared__ __align__(128) float sm[];
  float *ahi = sm, *alo = ahi + 128 * KPAD, *bhi = alo + 128 * KPAD, *blo = bhi + N * KPAD;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(blo + N * KPAD);
  uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int t = threadIdx.x, warp = t >> 5;
  for (int idx = t; idx < 128 * KPAD; idx += 128) {
    const int r = idx / KPAD, k = idx - r * KPAD;
    float h, l;
    tc::split_tf32(k < K ? A[r * K + k] : 0.f, h, l);
    ahi[tc::kmaj_off(r, k, KPAD) / 4] = h;
    alo[tc::kmaj_off(r, k, KPAD) / 4] = l;
  }
  for (int idx = t; idx < N * KPAD; idx += 128) {
    const int r = idx / KPAD, k = idx - r * KPAD;
    float h, l;
    tc::split_tf32(k < K ? B[r * K + k] : 0.f, h, l);
    bhi[tc::kmaj_off(r, k, KPAD) / 4] = h;
    blo[tc::kmaj_off(r, k, KPAD) / 4] = l;
  }
  tc::fence_async_smem();
  if (warp == 0) tc::tmem_alloc(slot, NCOLS);
  if (t == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = *slot;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  if (Dinit) {
#pragma unroll 1
    for (int c = 0; c < N; c += 8) {
      float v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = Dinit[t * N + c + j];
      tc::tmem_st8(tbase + lane_base + c, v);
    }
    tc::tmem_wait_st();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (t == 0) {
    constexpr uint32_t idesc = tc::idesc_tf32(128, N);
    const uint32_t a0 = tc::smem_u32(ahi), a1 = tc::smem_u32(alo);
    const uint32_t b0 = tc::smem_u32(bhi), b1 = tc::smem_u32(blo);
    uint32_t acc = Dinit ? 1u : 0u;
    for (int s = 0; s < KPAD / 8; ++s) {
      const uint32_t o = (uint32_t)s * 256u;
      tc::mma_tf32(tbase, tc::sdesc(a0 + o, KPAD), tc::sdesc(b0 + o, KPAD), idesc, acc);
      acc = 1u;
      if (split) {
        tc::mma_tf32(tbase, tc::sdesc(a1 + o, KPAD), tc::sdesc(b0 + o, KPAD), idesc, 1u);
        tc::mma_tf32(tbase, tc::sdesc(a0 + o, KPAD), tc::sdesc(b1 + o, KPAD), idesc, 1u);
      }
    }
    tc::commit(mbar);
  }
  const bool ok = tc::mbar_wait(mbar, 0, 1u << 24);
  if (!ok) atomicOr(err, 1);
  tc::fence_after();
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < N; c += 8) {
      float v[8];
      tc::tmem_ld8(tbase + lane_base + c, v);
      tc::tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 8; ++j) D[t * N + c + j] = v[j];
    }
  } else {
    tc::mbar_wait(mbar, 0, 1u << 24);  // give an in-flight MMA a last bounded chance
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, NCOLS);
}

template <int KPAD, int N>
cudaError_t run(const float *A, const float *B, float *D, const float *Dinit, int K, int split,
                int *err) {
  const size_t smem = sizeof(float) * (2 * 128 * KPAD + 2 * N * KPAD) + 16;
  cudaError_t e = cudaFuncSetAttribute(k_tc_selftest<KPAD, N>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_tc_selftest<KPAD, N><<<1, 128, smem>>>(A, B, D, Dinit, K, split, err);
  return cudaGetLastError();
}

}  // namespace
}  // namespace spoc

// Host pointers: A (128 x K), B (n x K) row-major, D (128 x n) out, dinit
// (128 x n) or null.  Supported (kpad, n): (8, 16), (40, 48), (48, 144),
// (32, 32), with K <= kpad.  split: 0 one TF32 product, 1 three-term split.
extern "C" int spoc_tc_selftest(int K, int kpad, int n, int split, const float *A, const float *B,
                                const float *dinit, float *D) {
  using namespace spoc;
  if (!A || !B || !D || K < 1 || K > kpad) return SPOC_E_ARG;
  float *dA = nullptr, *dB = nullptr, *dD = nullptr, *dI = nullptr;
  int *derr = nullptr;
  cudaError_t e = cudaMalloc(&dA, sizeof(float) * 128 * K);
  if (e == cudaSuccess) e = cudaMalloc(&dB, sizeof(float) * n * K);
  if (e == cudaSuccess) e = cudaMalloc(&dD, sizeof(float) * 128 * n);
  if (e == cudaSuccess && dinit) e = cudaMalloc(&dI, sizeof(float) * 128 * n);
  if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(dA, A, sizeof(float) * 128 * K, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dB, B, sizeof(float) * n * K, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && dinit) e = cudaMemcpy(dI, dinit, sizeof(float) * 128 * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
  int rc = SPOC_OK;
  if (e == cudaSuccess) {
    if (kpad == 8 && n == 16) e = run<8, 16>(dA, dB, dD, dI, K, split, derr);
    else if (kpad == 40 && n == 48) e = run<40, 48>(dA, dB, dD, dI, K, split, derr);
    else if (kpad == 48 && n == 144) e = run<48, 144>(dA, dB, dD, dI, K, split, derr);
    else if (kpad == 32 && n == 32) e = run<32, 32>(dA, dB, dD, dI, K, split, derr);
    else rc = SPOC_E_UNSUPPORTED;
  }
  int herr = 0;
  if (e == cudaSuccess && !rc) e = cudaMemcpy(D, dD, sizeof(float) * 128 * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && !rc) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(dI);
  cudaFree(derr);
  if (e != cudaSuccess) return SPOC_E_CUDA;
  if (herr) return SPOC_E_CUDA;
  return rc;
}
