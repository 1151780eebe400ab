// Energy diagnostic that allocates nothing: spoc_energy_noalloc.
//
// Why it exists: some callers cannot call cudaMalloc.  cudaMalloc and
// cudaFree are prohibited while a stream is captured into a CUDA graph in the
// default capture mode and cudaFree synchronises the device, so a caller in
// the middle of a capture, or one that must not stall other streams, cannot
// use them; and some host programs own all device memory themselves (a
// Fortran driver with OpenACC or CUDA Fortran device arrays, a framework
// with its own pool).  Such callers cannot use spoc_create, which allocates.
// This entry point takes every input and the output as device pointers the
// caller already owns, and keeps its only scratch -- the per-element
// (ke, pe, mass) terms summed afterwards -- in a file-scope static device
// array of fixed size.
//
// Limits and sharing: at most SPOC_NOALLOC_MAX_NE elements (the array holds
// 3 doubles per element, 3 MiB, resident on every GPU that loads the library
// until the process exits); larger meshes get SPOC_E_UNSUPPORTED.  In host
// code the array's name is not a device address: the first call on a device
// looks up the address (cudaGetSymbolAddress, with that device current) and
// caches it for that device's context; the lookup is made again after the
// context is re-created (cudaDeviceReset), so the first call on a device, and
// the first after a reset, should come before any stream capture.  All calls
// on a device share the array and it keeps the previous call's contents;
// every call overwrites the ne*3 terms it reads, so nothing needs clearing,
// but two calls that overlap on the GPU (different streams, no ordering
// between them) race on it.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "../../include/spoc_gpu.h"
#include "spoc_device.cuh"

namespace {

using namespace spoc;

static __device__ __align__(256) double g_energy_scratch[3 * SPOC_NOALLOC_MAX_NE];

constexpr int kMaxDevices = 64;
struct ScratchAddr {
  double *ptr = nullptr;
  unsigned long long ctx_id = 0;  // context the address belongs to
};
ScratchAddr g_scratch[kMaxDevices];
std::mutex g_scratch_mu;

// Per-element terms of src/energy.f:307-370, as k_energy_terms computes them,
// for fields with leading dimension ld.
__global__ void __launch_bounds__(256) k_energy_terms_ld(int nm, int ng, int ne, int ld,
                                                         const double *__restrict__ su,
                                                         const double *__restrict__ sv,
                                                         const double *__restrict__ sh,
                                                         const double *__restrict__ hb,
                                                         const double *__restrict__ vect,
                                                         const double *__restrict__ pi2,
                                                         const double *__restrict__ wi,
                                                         const double *__restrict__ ammo1,
                                                         double g0, double *terms) {
  __shared__ double smq[8][2][kMaxQuad];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < ne; e += nw) {
    const size_t o = (size_t)e * ld;
    const double *v = vect + 5 * (size_t)e;
    const double deta = sub(mul(v[0], v[3]), mul(v[2], v[1]));
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int qp = l + h * 32;
      if (qp < ng) {
        double mu = 0.0, mv = 0.0, mh = 0.0, mhb = 0.0;
        for (int n = 0; n < nm; ++n) {
          const double p = pi2[(size_t)n * ng + qp];
          const double hv = sh[o + n];
          mu = add(mu, mul(su[o + n], p));
          mv = add(mv, mul(sv[o + n], p));
          mh = add(mh, mul(hv, p));
          mhb = add(mhb, mul(add(hv, hb[o + n]), p));
        }
        const double wq = wi[qp], p1 = pi2[qp];
        smq[w][0][qp] = mul(mul(wq, mul(mhb, add(mul(mu, mu), mul(mv, mv)))), p1);
        smq[w][1][qp] = mul(mul(wq, mul(mh, mh)), p1);
      }
    }
    __syncwarp();
    if (l == 0) {
      double k = 0.0, p = 0.0, ms = 0.0;
      for (int qp = 0; qp < ng; ++qp) k = add(k, smq[w][0][qp]);
      for (int qp = 0; qp < ng; ++qp) p = add(p, smq[w][1][qp]);
      for (int n = 0; n < nm; ++n) ms = add(ms, mul(mul(ammo1[n], deta), sh[o + n]));
      terms[3 * (size_t)e + 0] = mul(mul(k, deta), 0.5);
      terms[3 * (size_t)e + 1] = mul(mul(mul(p, deta), 0.5), g0);
      terms[3 * (size_t)e + 2] = ms;
    }
    __syncwarp();
  }
}

// Same fixed-order tree sum as k_energy_sum.
__global__ void __launch_bounds__(1024) k_energy_sum_to(const double *terms, int ne, double *out) {
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

// Unique id of the current context (cuCtxGetId through the runtime's driver
// entry points, so the library needs no link against the driver library);
// it changes when cudaDeviceReset re-creates the device's context.  With no
// context current on this thread, cudaSetDevice makes the device's primary
// context current (it allocates nothing).
cudaError_t current_context_id(int dev, unsigned long long *id) {
  static PFN_cuCtxGetCurrent get_current = nullptr;
  static PFN_cuCtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<PFN_cuCtxGetCurrent>(f);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PFN_cuCtxGetId>(f);
  });
  if (!get_current || !get_id) return cudaErrorNotSupported;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  if (!ctx) {
    const cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return e;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorDeviceUninitialized;
  }
  return get_id(ctx, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorDeviceUninitialized;
}

// Device address of the static scratch on the current device: looked up with
// that device current, once per device context.
cudaError_t scratch_for_current_device(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  unsigned long long id = 0;
  e = current_context_id(dev, &id);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  ScratchAddr &a = g_scratch[dev];
  if (!a.ptr || a.ctx_id != id) {
    double *p = nullptr;
    e = cudaGetSymbolAddress((void **)&p, g_energy_scratch);
    if (e != cudaSuccess) return e;
    a.ptr = p;
    a.ctx_id = id;
  }
  *out = a.ptr;
  return cudaSuccess;
}

}  // namespace

extern "C" int spoc_energy_noalloc(int nc, int ng, int ne, int ld, double g0, const double *u,
                                   const double *v, const double *h, const double *hb,
                                   const double *vect, const double *pi2, const double *wi,
                                   const double *ammo1, double *out, void *stream) {
  const int nm = (nc + 1) * (nc + 2) / 2;
  if (nc < 1 || nm > kMaxModes || ng < 1 || ng > kMaxQuad || ne < 1 || ld < nm)
    return SPOC_E_ARG;
  if (ne > SPOC_NOALLOC_MAX_NE) return SPOC_E_UNSUPPORTED;  // beyond the static scratch
  if (!u || !v || !h || !hb || !vect || !pi2 || !wi || !ammo1 || !out) return SPOC_E_ARG;
  double *scratch = nullptr;
  if (scratch_for_current_device(&scratch) != cudaSuccess) return SPOC_E_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return SPOC_E_CUDA;
  int grid = (ne + 7) / 8;
  if (grid > sms * 8) grid = sms * 8;
  // cudaLaunchKernel returns the status of this launch itself, not an error
  // left over from earlier work of the caller
  void *ta[] = {(void *)&nm, (void *)&ng, (void *)&ne, (void *)&ld, (void *)&u, (void *)&v,
                (void *)&h, (void *)&hb, (void *)&vect, (void *)&pi2, (void *)&wi,
                (void *)&ammo1, (void *)&g0, (void *)&scratch};
  if (cudaLaunchKernel((const void *)k_energy_terms_ld, dim3(grid), dim3(256), ta, 0, st) !=
      cudaSuccess)
    return SPOC_E_CUDA;
  const double *terms = scratch;
  void *sa[] = {(void *)&terms, (void *)&ne, (void *)&out};
  if (cudaLaunchKernel((const void *)k_energy_sum_to, dim3(1), dim3(1024), sa, 0, st) !=
      cudaSuccess)
    return SPOC_E_CUDA;
  return SPOC_OK;
}
