// had_pq.cuh -- the M2L Hadamard step for scalar equivalent kernels, grouped
// by parent pairs and register-blocked over the 8 x 8 child pairs.
//
//   effVal(c)[f] = (1/(2np)^3) sum_{v in V(c)} T_{v-c}[f] effDen(v)[f]
//   (cptwvv, fmm3d_mpi/matmgnt3d_mpi.cpp:414-429)
//
// V(c) for a child c of a parent P is the set of children c2 of P's
// same-depth non-leaf neighbours Q that do not touch c (let3d_mpi.cpp:
// 1687-1698).  For a fixed neighbour offset o = Q - P the relative position of
// the pair is r = 2o + (c2 - c), so the 64 pairs use at most 27 distinct
// translations, and whether a pair interacts depends on (o, c2 - c) only.
// One warp owns one output parent and 32 frequencies (lane = frequency): per
// neighbour it loads the 8 child spectra of Q once into registers and applies
// each distinct translation to every pair that uses it.  The 64 pairs are
// unrolled by child offset e = c2 - c (27 groups); a [26 x 27] table in shared
// memory gives the translation of (neighbour offset, e), or -1 for touching
// pairs, so one code path serves every neighbour offset.  The 316 translation
// spectra of the CTA's 32 frequencies sit in shared memory.
//
// ADJ selects the transposed operator: rows are the source parents Q with
// their target parents P at offset o' = P - Q, outputs the source children,
// and each pair uses conj(T) of the forward relative position -(2o' + c - c2).
#pragma once

#include <cuda_runtime.h>

#include "had_smem.cuh"

namespace fmmg {

constexpr int PQ_THREADS = 512;
constexpr int PQ_PARENTS = 128;  // output parents per CTA

template <typename C>
__device__ __forceinline__ void pq_cfma(C& acc, const C t, const C d) {
  acc.x = fma(t.x, d.x, acc.x);
  acc.x = fma(-t.y, d.y, acc.x);
  acc.y = fma(t.x, d.y, acc.y);
  acc.y = fma(t.y, d.x, acc.y);
}

// child offset e = E (0..26): every pair (c out, c2 = c + e in), when the
// pair's relative position is far (sId >= 0 for this neighbour offset); then E + 1.
// One code path serves all 26 neighbour offsets (the skip is warp-uniform).
template <typename C, int KB, bool ADJ, int E>
__device__ __forceinline__ void pq_delta(C (&acc)[8][KB], const C (&in)[8][KB], const C* __restrict__ Ts,
                                         const int16_t* __restrict__ sIdRow, int lane) {
  if constexpr (E < 27) {
    constexpr int ex = E / 9 - 1, ey = (E / 3) % 3 - 1, ez = E % 3 - 1;
    const int id = sIdRow[E];
    if (id >= 0) {
      C t = Ts[id * 32 + lane];
      if (ADJ) t.y = -t.y;
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int x2 = (c >> 2) + ex, y2 = ((c >> 1) & 1) + ey, z2 = (c & 1) + ez;
        if (x2 < 0 || x2 > 1 || y2 < 0 || y2 > 1 || z2 < 0 || z2 > 1) continue;
        const int c2 = x2 * 4 + y2 * 2 + z2;
#pragma unroll
        for (int q = 0; q < KB; q++) pq_cfma(acc[c][q], t, in[c2][q]);
      }
    }
    pq_delta<C, KB, ADJ, E + 1>(acc, in, Ts, sIdRow, lane);
  }
}

// rows: output parents; per row the neighbour parents (idx) and their offset
// codes (off, (dx+1)*9+(dy+1)*3+(dz+1) of neighbour - row); inSlot/outSlot map
// a child node to its spectrum row (or -1).  effIn/effOut hold nrhs
// right-hand sides at strides inRhs/outRhs; transId maps (rx+3)*49+(ry+3)*7+
// (rz+3) to a translation id or -1; grid (rows/PQ_PARENTS, nEff/32,
// ceil(nrhs/KB)); dynamic shared memory had_smem_bytes<C>().
template <typename C, int KB, bool ADJ>
__global__ void __launch_bounds__(PQ_THREADS)
    k_m2l_had_pq(int nRows, const int32_t* __restrict__ rows, const int64_t* __restrict__ nPtr,
                 const int32_t* __restrict__ nIdx, const int8_t* __restrict__ nOff, const int32_t* __restrict__ chd,
                 const int32_t* __restrict__ inSlot, const int32_t* __restrict__ outSlot, const C* __restrict__ effIn,
                 int64_t inRhs, const C* __restrict__ T, C* __restrict__ effOut, int64_t outRhs, int nEff, int nrhs,
                 typename CplxOps<C>::R nrmfc, const int16_t* __restrict__ transId) {
  typedef typename CplxOps<C>::R R;
  extern __shared__ unsigned char pq_smem[];
  C* Ts = reinterpret_cast<C*>(pq_smem);  // [316][32]
  __shared__ int16_t sId[27 * 27];        // [neighbour offset][child offset] -> translation id or -1
  for (int i = threadIdx.x; i < 27 * 27; i += blockDim.x) {
    const int o = i / 27, e = i % 27;
    int rx = 2 * (o / 9 - 1) + (e / 9 - 1), ry = 2 * ((o / 3) % 3 - 1) + ((e / 3) % 3 - 1),
        rz = 2 * (o % 3 - 1) + (e % 3 - 1);
    if (ADJ) {
      rx = -rx;
      ry = -ry;
      rz = -rz;
    }
    sId[i] = o == 13 ? (int16_t)-1 : transId[(rx + 3) * 49 + (ry + 3) * 7 + (rz + 3)];
  }
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
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * PQ_PARENTS);
  for (int b = blockIdx.x * PQ_PARENTS + warp; b < bEnd; b += PQ_THREADS / 32) {
    C acc[8][KB];
#pragma unroll
    for (int c = 0; c < 8; c++)
#pragma unroll
      for (int q = 0; q < KB; q++) acc[c][q] = CplxOps<C>::zero();
    const int64_t e1 = nPtr[b + 1];
    for (int64_t e = nPtr[b]; e < e1; e++) {
      const int q0 = chd[nIdx[e]];
      const int off = nOff[e];
      C in[8][KB];
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++) {
        const int s = inSlot[q0 + c2];
#pragma unroll
        for (int q = 0; q < KB; q++)
          in[c2][q] = (s >= 0 && rhs0 + q < nrhs) ? effIn[(int64_t)(rhs0 + q) * inRhs + (int64_t)s * nEff + f]
                                                  : CplxOps<C>::zero();
      }
      pq_delta<C, KB, ADJ, 0>(acc, in, Ts, &sId[off * 27], lane);
    }
    const int p0 = chd[rows[b]];
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int t = outSlot[p0 + c];
      if (t < 0) continue;
#pragma unroll
      for (int q = 0; q < KB; q++)
        if (rhs0 + q < nrhs) {
          C o;
          o.x = acc[c][q].x * (R)nrmfc;
          o.y = acc[c][q].y * (R)nrmfc;
          effOut[(int64_t)(rhs0 + q) * outRhs + (int64_t)t * nEff + f] = o;
        }
    }
  }
}

}  // namespace fmmg
