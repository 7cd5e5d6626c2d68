// had_smem.cuh -- the M2L Hadamard step for scalar equivalent kernels
// (SDM = TDM = 1), shared by the FP64 and FP32 forms.
//
//   effVal(c)[f] = (1/(2np)^3) sum_{v in V(c)} T_{v-c}[f] effDen(v)[f]
//   (cptwvv, fmm3d_mpi/matmgnt3d_mpi.cpp:414-429)
//
// One CTA owns a 32-frequency slice (lane = frequency) and stages that slice
// of all 316 translation spectra in shared memory once.  Each warp then takes
// one output box at a time and walks its expanded interaction list of
// (input spectrum slot, translation id) pairs -- a warp-uniform load, one
// shared-memory load and KB spectrum loads per pair.  Sibling output boxes are
// adjacent in the slot order, so concurrent warps share most input spectra in
// L1.  With CONJ the conjugated spectra are used: run on the lists inverted per
// source box, that is the transposed operator (circular correlation).
#pragma once

#include <cuda_runtime.h>

namespace fmmg {

constexpr int HS_THREADS = 1024;
constexpr int HS_BOXES = 128;  // output boxes per CTA

template <typename C>
struct CplxOps;
template <>
struct CplxOps<double2> {
  typedef double R;
  static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
};
template <>
struct CplxOps<float2> {
  typedef float R;
  static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
};

template <typename C, int KB, bool CONJ>
__global__ void __launch_bounds__(HS_THREADS)
    k_m2l_had_list(int nOut, const int64_t* __restrict__ lptr, const int2* __restrict__ lent,
                   const C* __restrict__ effIn, int64_t inRhs, const C* __restrict__ T, C* __restrict__ effOut,
                   int64_t outRhs, int nEff, int nrhs, typename CplxOps<C>::R nrmfc) {
  typedef typename CplxOps<C>::R R;
  extern __shared__ unsigned char hs_smem[];
  C* Ts = reinterpret_cast<C*>(hs_smem);  // [316][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int f0 = blockIdx.y * 32;
  const int f = f0 + lane;
  const int rhs0 = blockIdx.z * KB;
  for (int i = threadIdx.x; i < 316 * 32; i += blockDim.x) {
    const int id = i >> 5, ff = f0 + (i & 31);
    Ts[i] = ff < nEff ? T[(int64_t)id * nEff + ff] : CplxOps<C>::zero();
  }
  __syncthreads();
  if (f >= nEff) return;
  const int tEnd = min(nOut, (int)(blockIdx.x + 1) * HS_BOXES);
  for (int t = blockIdx.x * HS_BOXES + warp; t < tEnd; t += HS_THREADS / 32) {
    C acc[KB];
#pragma unroll
    for (int q = 0; q < KB; q++) acc[q] = CplxOps<C>::zero();
    const int64_t e1 = lptr[t + 1];
#pragma unroll 4
    for (int64_t e = lptr[t]; e < e1; e++) {
      const int2 en = lent[e];
      C w = Ts[en.y * 32 + lane];
      if (CONJ) w.y = -w.y;
      const C* dp = effIn + (int64_t)en.x * nEff + f;
#pragma unroll
      for (int q = 0; q < KB; q++) {
        if (rhs0 + q < nrhs) {
          const C d = dp[(rhs0 + q) * inRhs];
          acc[q].x += w.x * d.x - w.y * d.y;
          acc[q].y += w.x * d.y + w.y * d.x;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < KB; q++)
      if (rhs0 + q < nrhs) {
        C o;
        o.x = acc[q].x * (R)nrmfc;
        o.y = acc[q].y * (R)nrmfc;
        effOut[(rhs0 + q) * outRhs + (int64_t)t * nEff + f] = o;
      }
  }
}

template <typename C>
inline size_t had_smem_bytes() {
  return 316 * 32 * sizeof(C);
}

}  // namespace fmmg
