// dense_kernel.cuh -- the FP64 dense direct sum of the reference check()
// (fmm3d_mpi/fmm3d_check_mpi.cpp:122-131, dense3d_mpi.cpp:75-141): every
// point of pos against every source.  Sources are split in chunks over
// grid.y; each CTA adds its partial sums into out with atomics, so out must
// start at zero.
#pragma once

#include <cuda_runtime.h>

#include "kernels.hpp"

namespace fmmg {

template <int KT>
__global__ void __launch_bounds__(128)
    k_dense(int64_t nchk, const double* __restrict__ pos, int64_t ns, int64_t chunk, const double* __restrict__ src,
            const double* __restrict__ nrm, const double* __restrict__ den, double* __restrict__ out, double mu,
            double ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  __shared__ double sPos[128 * 3];
  __shared__ double sNrm[NRM ? 128 * 3 : 1];
  __shared__ double sDen[128 * SD];
  const int64_t i = blockIdx.x * 128 + threadIdx.x;
  const bool act = i < nchk;
  double px = act ? pos[3 * i] : 0, py = act ? pos[3 * i + 1] : 0, pz = act ? pos[3 * i + 2] : 0;
  double acc[TD];
#pragma unroll
  for (int c = 0; c < TD; c++) acc[c] = 0;
  const int64_t s0 = blockIdx.y * chunk, s1 = min(ns, s0 + chunk);
  for (int64_t b = s0; b < s1; b += 128) {
    int cnt = (int)min((int64_t)128, s1 - b);
    __syncthreads();
    if (threadIdx.x < cnt) {
      int64_t s = b + threadIdx.x;
      for (int d = 0; d < 3; d++) sPos[3 * threadIdx.x + d] = src[3 * s + d];
      if (NRM)
        for (int d = 0; d < 3; d++) sNrm[3 * threadIdx.x + d] = nrm[3 * s + d];
      for (int c = 0; c < SD; c++) sDen[SD * threadIdx.x + c] = den[s * SD + c];
    }
    __syncthreads();
    if (act)
      for (int j = 0; j < cnt; j++)
        kaccum<KT, double, double>(px - sPos[3 * j], py - sPos[3 * j + 1], pz - sPos[3 * j + 2],
                                   NRM ? &sNrm[3 * j] : nullptr, &sDen[SD * j], acc, mu, ve);
  }
  if (act)
    for (int c = 0; c < TD; c++) atomicAdd(&out[i * TD + c], acc[c]);
}

}  // namespace fmmg
