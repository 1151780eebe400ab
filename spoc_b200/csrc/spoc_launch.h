// Launch configuration shared by the persistent-grid kernels.
//
// The dynamic shared-memory limit of a kernel (cudaFuncSetAttribute) and its
// resident blocks per SM are properties of the kernel on one device: they are
// cached per (device, kernel, block size, shared memory), under a mutex, so
// handles on different GPUs and handles used from several host threads each
// see their own device's figures.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

namespace spoc {

// Resident blocks per SM of `kernel` at `threads` threads and `smem` bytes of
// dynamic shared memory on the current device; raises the kernel's dynamic
// shared-memory limit there on first use (cudaErrorInvalidConfiguration: the
// block does not fit an SM).
template <class K>
cudaError_t device_blocks_per_sm(K kernel, int threads, size_t smem, int *per_sm) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void *, int, size_t>, int> cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const auto key = std::make_tuple(dev, reinterpret_cast<const void *>(kernel), threads, smem);
  std::lock_guard<std::mutex> lk(mu);
  const auto it = cache.find(key);
  if (it != cache.end()) {
    *per_sm = it->second;
    return cudaSuccess;
  }
  // the limit is raised to the most the device allows beside the kernel's
  // static shared memory, not to `smem`: a kernel launched with several
  // shared-memory sizes keeps them all valid
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa{};
  e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  const int dyn_max = optin - (int)fa.sharedSizeBytes;
  if (dyn_max < 0 || smem > (size_t)dyn_max) return cudaErrorInvalidConfiguration;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max);
  if (e != cudaSuccess) return e;
  int n = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem);
  if (e != cudaSuccess) return e;
  if (n < 1) return cudaErrorInvalidConfiguration;  // the block does not fit an SM
  cache.emplace(key, n);
  *per_sm = n;
  return cudaSuccess;
}

// Persistent grid: as many blocks as stay resident on `sms` SMs, or fewer when
// the `ne` elements (`per_block` per block and pass) run out.
template <class K>
cudaError_t resident_grid(K kernel, int threads, size_t smem, int sms, int ne, int per_block,
                          int *grid) {
  int per_sm = 0;
  const cudaError_t e = device_blocks_per_sm(kernel, threads, smem, &per_sm);
  if (e != cudaSuccess) return e;
  const int need = (ne + per_block - 1) / per_block;
  const int cap = sms * per_sm;
  *grid = need < cap ? need : cap;
  return cudaSuccess;
}

}  // namespace spoc
