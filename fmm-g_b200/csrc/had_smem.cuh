// had_smem.cuh -- the M2L Hadamard step for scalar equivalent kernels
// (SDM = TDM = 1), shared by the FP64 and FP32 forms.
//
//   effVal(c)[f] = (1/(2np)^3) sum_{v in V(c)} T_{v-c}[f] effDen(v)[f]
//   (cptwvv, fmm3d_mpi/matmgnt3d_mpi.cpp:414-429)
//
// One CTA owns a 32-frequency slice (lane = frequency) and stages the slice
// of all 316 translation spectra in shared memory once; it then walks a block
// of HS_PPB target parents, HS_SLOTS of them at a time: warp w handles child
// w % 8 of parent slot w / 8.  The loop over the 8 children of a neighbour
// parent is unrolled so their slot, spectrum and translation loads issue
// together.  With ADJ the same kernel applies the transposed operator on the
// inverted lists: the translation index is reflected and the spectrum
// conjugated (circular correlation instead of convolution).
#pragma once

#include <cuda_runtime.h>

namespace fmmg {

constexpr int HS_SLOTS = 4;   // parents in flight per CTA
constexpr int HS_PPB = 32;    // parents per CTA
constexpr int HS_THREADS = HS_SLOTS * 256;

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

template <typename C, int KB, bool ADJ>
__global__ void __launch_bounds__(HS_THREADS)
    k_m2l_had_smem(int nP, const int32_t* __restrict__ parents, const int64_t* __restrict__ vPtr,
                   const int32_t* __restrict__ vIdx, const int8_t* __restrict__ vOff, const int32_t* __restrict__ chd,
                   const int32_t* __restrict__ srcSlot, const int32_t* __restrict__ trgSlot,
                   const int16_t* __restrict__ transId, const C* __restrict__ effDen, int64_t denRhs,
                   const C* __restrict__ T, C* __restrict__ effVal, int64_t valRhs, int nEff, int nrhs,
                   typename CplxOps<C>::R nrmfc) {
  typedef typename CplxOps<C>::R R;
  extern __shared__ unsigned char hs_smem[];
  C* Ts = reinterpret_cast<C*>(hs_smem);                            // [316][32]
  int16_t* ids = reinterpret_cast<int16_t*>(Ts + 316 * 32);          // [343]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slotP = warp >> 3, c = warp & 7;
  const int f0 = blockIdx.y * 32;
  const int f = f0 + lane;
  const int rhs0 = blockIdx.z * KB;
  for (int i = threadIdx.x; i < 316 * 32; i += blockDim.x) {
    const int id = i >> 5, ff = f0 + (i & 31);
    Ts[i] = ff < nEff ? T[(int64_t)id * nEff + ff] : CplxOps<C>::zero();
  }
  for (int i = threadIdx.x; i < 343; i += blockDim.x) ids[i] = transId[i];
  __syncthreads();
  const bool fin = f < nEff;
  const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
  const int pEnd = min(nP, (int)(blockIdx.x + 1) * HS_PPB);
  for (int b = blockIdx.x * HS_PPB + slotP; b < pEnd; b += HS_SLOTS) {
    const int P = parents[b];
    const int ts = trgSlot[chd[P] + c];
    if (ts < 0) continue;
    C acc[KB];
#pragma unroll
    for (int q = 0; q < KB; q++) acc[q] = CplxOps<C>::zero();
    const int64_t e1 = vPtr[b + 1];
    for (int64_t e = vPtr[b]; e < e1; e++) {
      const int Q = vIdx[e];
      const int off = vOff[e];
      const int dx = off / 9 - 1, dy = (off / 3) % 3 - 1, dz = off % 3 - 1;
      const int q0 = chd[Q];
      int sl[8];
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++) sl[c2] = srcSlot[q0 + c2];
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++) {
        int rx = 2 * dx + (c2 >> 2) - cx, ry = 2 * dy + ((c2 >> 1) & 1) - cy, rz = 2 * dz + (c2 & 1) - cz;
        const bool use = sl[c2] >= 0 && max(abs(rx), max(abs(ry), abs(rz))) > 1 && fin;
        if (!use) continue;
        if (ADJ) { rx = -rx; ry = -ry; rz = -rz; }
        C w = Ts[ids[(rx + 3) * 49 + (ry + 3) * 7 + (rz + 3)] * 32 + lane];
        if (ADJ) w.y = -w.y;
        const C* dp = effDen + (int64_t)sl[c2] * nEff + f;
#pragma unroll
        for (int q = 0; q < KB; q++) {
          if (rhs0 + q < nrhs) {
            const C d = dp[(rhs0 + q) * denRhs];
            acc[q].x += w.x * d.x - w.y * d.y;
            acc[q].y += w.x * d.y + w.y * d.x;
          }
        }
      }
    }
    if (fin) {
#pragma unroll
      for (int q = 0; q < KB; q++)
        if (rhs0 + q < nrhs) {
          C o;
          o.x = acc[q].x * (R)nrmfc;
          o.y = acc[q].y * (R)nrmfc;
          effVal[(rhs0 + q) * valRhs + (int64_t)ts * nEff + f] = o;
        }
    }
  }
}

template <typename C>
inline size_t had_smem_bytes() {
  return 316 * 32 * sizeof(C) + 343 * sizeof(int16_t);
}

}  // namespace fmmg
