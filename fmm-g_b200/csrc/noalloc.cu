// noalloc.cu -- a dense direct sum that allocates no memory.
//
// fmmg_check() and the evaluator allocate their device buffers (cudaMalloc)
// at setup.  Some callers cannot allocate at the point where they need a
// result: code running while a stream is being captured into a CUDA graph,
// code inside a framework that owns all device memory through its own pool
// and forbids driver allocations, or code on a latency path that must not
// pay for (or synchronise on) an allocation.  fmmg_dense_noalloc() serves
// them: the caller passes device inputs and outputs, and the only scratch the
// kernel needs -- the accumulation buffer that the dense-sum kernel adds its
// per-chunk partial sums into -- is a file-scope __device__ array of fixed
// size that every GPU loading this library holds until the process exits.
//
// In host code the array's name is only a host-side stand-in for the device
// symbol, so its device address is taken once per device with
// cudaGetSymbolAddress (with that device current) and cached; the first call
// on a device does that set-up and should therefore come before any stream
// capture.  Every call on a device shares the one array: calls that overlap on
// the GPU (different streams, no ordering between them) race and give wrong
// results.  The array keeps the last call's contents; each call clears the
// part it accumulates into before use.  The cached address belongs to the
// device's current context: after cudaDeviceReset() (or any destruction of
// the primary context) the module is loaded again and the array may move, so
// this entry point must not be used across such a reset in one process.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/fmmg.h"
#include "dense_kernel.cuh"
#include "kernels.hpp"

namespace fmmg {

// 2^20 doubles (8 MiB): the largest n_trg * trgDOF one call may produce
static constexpr int64_t kNoallocMaxValues = (int64_t)1 << 20;
static __device__ __align__(256) double g_noalloc_scratch[kNoallocMaxValues];

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[256] = {};

// Device address of g_noalloc_scratch on the current device (set-up once per device).
static cudaError_t noalloc_scratch(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = (double*)p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace fmmg

using namespace fmmg;

extern "C" {

fmmg_status fmmg_dense_noalloc(int kernel_type, const double* coefs, int64_t n_src, const double* d_src,
                               const double* d_nrm, const double* d_den, int64_t n_trg, const double* d_trg,
                               double* d_val, void* stream) {
  const int td = kernel_trg_dof(kernel_type);
  if (kernel_mm(kernel_type) < 0 || td == 0) {
    return FMMG_NOT_SUPPORTED;
  }
  if (n_src < 1 || n_trg < 0 || !d_src || !d_den || (n_trg > 0 && (!d_trg || !d_val)) ||
      (kernel_has_normal(kernel_type) && !d_nrm)) {
    return FMMG_INVALID_ARG;
  }
  if (n_trg * td > kNoallocMaxValues) {
    return FMMG_INVALID_ARG;
  }
  const double mu = coefs ? coefs[0] : 1.0, ve = coefs ? coefs[1] : 0.25;
  if (!std::isfinite(mu) || !std::isfinite(ve) || mu == 0.0) {
    return FMMG_INVALID_ARG;
  }
  // the Navier kernels divide by 1 - nu (kernels.hpp), as fmmg_create refuses
  if (kernel_mm(kernel_type) == NAV_S_U && ve == 1.0) {
    return FMMG_INVALID_ARG;
  }
  if (n_trg == 0) {  // no targets: nothing to sum (fmmg_setup accepts zero targets too)
    return FMMG_OK;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  double* scratch = nullptr;
  if (e == cudaSuccess) e = noalloc_scratch(dev, &scratch);
  if (e != cudaSuccess) {
    return FMMG_CUDA_ERROR;
  }
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemsetAsync(scratch, 0, sizeof(double) * n_trg * td, st);
  if (e != cudaSuccess) {
    return FMMG_CUDA_ERROR;
  }
  const int64_t chunk = 8192;
  dim3 grid((unsigned)((n_trg + 127) / 128), (unsigned)((n_src + chunk - 1) / chunk));
  FMMG_DISPATCH_KT(kernel_type, KT,
                   k_dense<KT><<<grid, 128, 0, st>>>(n_trg, d_trg, n_src, chunk, d_src, d_nrm, d_den, scratch, mu,
                                                     ve));
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_val, scratch, sizeof(double) * n_trg * td, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) {
    return FMMG_CUDA_ERROR;
  }
  return FMMG_OK;
}

}  // extern "C"
