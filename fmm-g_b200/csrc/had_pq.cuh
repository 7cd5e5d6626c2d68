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
// memory gives the translation of (neighbour offset, e), or a zero row for
// touching pairs, so one branch-free code path serves every neighbour offset.
// The 316 translation spectra of the CTA's frequencies (plus the zero row) sit
// in shared memory.
//
// ADJ selects the transposed operator: rows are the source parents Q with
// their target parents P at offset o' = P - Q, outputs the source children,
// and each pair uses conj(T) of the forward relative position -(2o' + c - c2).
#pragma once

#include <cuda_runtime.h>

#include "had_smem.cuh"

namespace fmmg {

constexpr int PQ_THREADS = 512;
// dynamic shared memory of the kernels below: 316 translations + the zero row, fw frequencies
template <typename C>
inline size_t pq_smem_bytes(int fw) {
  return (size_t)317 * fw * sizeof(C);
}
constexpr int PQ_PARENTS = 128;  // output parents per CTA

template <typename C>
__device__ __forceinline__ void pq_cfma(C& acc, const C t, const C d) {
  acc.x = fma(t.x, d.x, acc.x);
  acc.x = fma(-t.y, d.y, acc.x);
  acc.y = fma(t.x, d.y, acc.y);
  acc.y = fma(t.y, d.x, acc.y);
}

// child offset e = E (0..26): every pair (c out, c2 = c + e in) with the
// translation of this (neighbour offset, e) -- zero for touching pairs; then E + 1.
// One branch-free code path serves all 26 neighbour offsets.
template <typename C, int KB, bool ADJ, int E, int FW = 32>
__device__ __forceinline__ void pq_delta(C (&acc)[8][KB], const C (&in)[8][KB], const C* __restrict__ Ts,
                                         const int16_t* __restrict__ sIdRow, int lane) {
  if constexpr (E < 27) {
    constexpr int ex = E / 9 - 1, ey = (E / 3) % 3 - 1, ez = E % 3 - 1;
    C t = Ts[sIdRow[E] * FW + lane];
    if (ADJ) t.y = -t.y;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int x2 = (c >> 2) + ex, y2 = ((c >> 1) & 1) + ey, z2 = (c & 1) + ez;
      if (x2 < 0 || x2 > 1 || y2 < 0 || y2 > 1 || z2 < 0 || z2 > 1) continue;
      const int c2 = x2 * 4 + y2 * 2 + z2;
#pragma unroll
      for (int q = 0; q < KB; q++) pq_cfma(acc[c][q], t, in[c2][q]);
    }
    pq_delta<C, KB, ADJ, E + 1, FW>(acc, in, Ts, sIdRow, lane);
  }
}

template <bool ADJ>
__device__ __forceinline__ void pq_id_table(int16_t* sId, const int16_t* __restrict__ transId) {
  for (int i = threadIdx.x; i < 27 * 27; i += blockDim.x) {
    const int o = i / 27, e = i % 27;
    int rx = 2 * (o / 9 - 1) + (e / 9 - 1), ry = 2 * ((o / 3) % 3 - 1) + ((e / 3) % 3 - 1),
        rz = 2 * (o % 3 - 1) + (e % 3 - 1);
    if (ADJ) {
      rx = -rx;
      ry = -ry;
      rz = -rz;
    }
    const int id = o == 13 ? -1 : transId[(rx + 3) * 49 + (ry + 3) * 7 + (rz + 3)];
    sId[i] = (int16_t)(id < 0 ? 316 : id);  // row 316 of the staged slice is zero
  }
}

// Rows are output parents.  rowOut[8*b + c] is the spectrum row of child c of
// row b (or -1); per row the neighbour entries nPtr[b]..nPtr[b+1] carry the
// offset code nOff (dx+1)*9+(dy+1)*3+(dz+1) of neighbour - row and the input
// spectrum rows of the neighbour's 8 children nIn[8*e + c2] (or -1).  effIn /
// effOut hold nrhs right-hand sides at strides inRhs / outRhs; transId maps
// (rx+3)*49+(ry+3)*7+(rz+3) to a translation id or -1.  Grid (rows /
// PQ_PARENTS, nEff / 32, ceil(nrhs / KB)); dynamic shared memory
// pq_smem_bytes<C>(32).  The child slots of the next entry are fetched while
// the current one is applied, so each neighbour costs one dependent load.
template <typename C, int KB, bool ADJ>
__global__ void __launch_bounds__(PQ_THREADS)
    k_m2l_had_pq(int nRows, const int32_t* __restrict__ rowOut, const int64_t* __restrict__ nPtr,
                 const int8_t* __restrict__ nOff, const int32_t* __restrict__ nIn, const C* __restrict__ effIn,
                 int64_t inRhs, const C* __restrict__ T, C* __restrict__ effOut, int64_t outRhs, int nEff, int nrhs,
                 typename CplxOps<C>::R nrmfc, const int16_t* __restrict__ transId) {
  typedef typename CplxOps<C>::R R;
  extern __shared__ unsigned char pq_smem[];
  C* Ts = reinterpret_cast<C*>(pq_smem);  // [316][32]
  __shared__ int16_t sId[27 * 27];        // [neighbour offset][child offset] -> translation id or -1
  pq_id_table<ADJ>(sId, transId);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int f0 = blockIdx.y * 32;
  const int f = f0 + lane;
  const int rhs0 = blockIdx.z * KB;
  for (int i = threadIdx.x; i < 317 * 32; i += blockDim.x) {
    const int id = i >> 5, ff = f0 + (i & 31);
    Ts[i] = (ff < nEff && id < 316) ? T[(int64_t)id * nEff + ff] : CplxOps<C>::zero();
  }
  __syncthreads();
  if (f >= nEff) return;
  const C* inF = effIn + (int64_t)rhs0 * inRhs + f;
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * PQ_PARENTS);
  for (int b = blockIdx.x * PQ_PARENTS + warp; b < bEnd; b += PQ_THREADS / 32) {
    C acc[8][KB];
#pragma unroll
    for (int c = 0; c < 8; c++)
#pragma unroll
      for (int q = 0; q < KB; q++) acc[c][q] = CplxOps<C>::zero();
    int64_t e = nPtr[b];
    const int64_t e1 = nPtr[b + 1];
    int4 sa = make_int4(-1, -1, -1, -1), sb = sa;
    int off = 13;
    if (e < e1) {
      sa = reinterpret_cast<const int4*>(nIn)[2 * e];
      sb = reinterpret_cast<const int4*>(nIn)[2 * e + 1];
      off = nOff[e];
    }
    for (; e < e1; e++) {
      const int sl[8] = {sa.x, sa.y, sa.z, sa.w, sb.x, sb.y, sb.z, sb.w};
      C in[8][KB];
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++)
#pragma unroll
        for (int q = 0; q < KB; q++)
          in[c2][q] = (sl[c2] >= 0 && rhs0 + q < nrhs) ? inF[(int64_t)q * inRhs + (int64_t)sl[c2] * nEff]
                                                       : CplxOps<C>::zero();
      const int offCur = off;
      if (e + 1 < e1) {
        sa = reinterpret_cast<const int4*>(nIn)[2 * (e + 1)];
        sb = reinterpret_cast<const int4*>(nIn)[2 * (e + 1) + 1];
        off = nOff[e + 1];
      }
      pq_delta<C, KB, ADJ, 0>(acc, in, Ts, &sId[offCur * 27], lane);
    }
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int t = rowOut[8 * b + c];
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

// ---------------------------------------------------------------- FP32 form
// Complex FP32 products on the packed FP32x2 FMA of sm_100: with t the
// translation and d the input spectrum, acc += t * d is
//   acc = fma2((t.x, t.x), (d.x, d.y), acc);  acc = fma2((t.y, t.y), (-d.y, d.x), acc)
// -- the same per-component FMAs as the scalar form, in half the instructions.
__device__ __forceinline__ unsigned long long pq_pk(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 pq_unpk(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ void pq_fma2(unsigned long long& acc, unsigned long long a, unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}

template <bool ADJ, int E, int FW>
__device__ __forceinline__ void pq_delta_x2(unsigned long long (&acc)[8], const unsigned long long (&inD)[8],
                                            const unsigned long long (&inR)[8], const float2* __restrict__ Ts,
                                            const int16_t* __restrict__ sIdRow, int fl) {
  if constexpr (E < 27) {
    constexpr int ex = E / 9 - 1, ey = (E / 3) % 3 - 1, ez = E % 3 - 1;
    const float2 t = Ts[sIdRow[E] * FW + fl];
    const unsigned long long tx = pq_pk(t.x, t.x), ty = ADJ ? pq_pk(-t.y, -t.y) : pq_pk(t.y, t.y);
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int x2 = (c >> 2) + ex, y2 = ((c >> 1) & 1) + ey, z2 = (c & 1) + ez;
      if (x2 < 0 || x2 > 1 || y2 < 0 || y2 > 1 || z2 < 0 || z2 > 1) continue;
      const int c2 = x2 * 4 + y2 * 2 + z2;
      pq_fma2(acc[c], tx, inD[c2]);
      pq_fma2(acc[c], ty, inR[c2]);
    }
    pq_delta_x2<ADJ, E + 1, FW>(acc, inD, inR, Ts, sIdRow, fl);
  }
}

// FW frequencies x (32 / FW) right-hand sides per warp (lane = rhs * FW +
// frequency), one right-hand side per thread: FW = 32 for a single
// right-hand side, FW = 4 for blocks of 8, where every translation value read
// from shared memory serves 8 lanes and the CTA stages only 4 frequencies of
// the 316 translations (10 KB), so residency is set by registers.  Grid (rows
// / PQX_ROWS, nEff / FW, ceil(nrhs / (32 / FW))); blockIdx.z selects the
// right-hand-side block of the layout below; dynamic shared memory
// 317 * FW * sizeof(float2) (row 316 is the zero row of touching pairs).
constexpr int PQX_THREADS = 256;
constexpr int PQX_ROWS = 64;

// Spectrum layout: value (right-hand side r, slot s, frequency f) of effIn
// sits at (r / RW) * in.blk + s * in.slot + f * fStride + (r % RW) * rStride
// (effOut likewise): planes of one right-hand side (RW = 1, fStride = 1), or
// blocks of 8 interleaved right-hand sides (RW = 8, fStride = 8, rStride = 1).
struct PqLayout {
  int64_t blk, slot;
};

template <int FW, bool ADJ>
__global__ void __launch_bounds__(PQX_THREADS, 3)
    k_m2l_had_pqx2(int nRows, const int32_t* __restrict__ rowOut, const int64_t* __restrict__ nPtr,
                   const int8_t* __restrict__ nOff, const int32_t* __restrict__ nIn, const float2* __restrict__ effIn,
                   PqLayout inL, const float2* __restrict__ T, float2* __restrict__ effOut, PqLayout outL,
                   int fStride, int rStride, int nEff, int nrhs, float nrmfc, const int16_t* __restrict__ transId) {
  constexpr int RW = 32 / FW;
  extern __shared__ unsigned char pqx_smem[];
  float2* Ts = reinterpret_cast<float2*>(pqx_smem);  // [316][FW]
  __shared__ int16_t sId[27 * 27];
  pq_id_table<ADJ>(sId, transId);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fl = lane % FW, rl = lane / FW;
  const int f0 = blockIdx.y * FW;
  const int f = f0 + fl;
  const int rhs = blockIdx.z * RW + rl;
  for (int i = threadIdx.x; i < 317 * FW; i += blockDim.x) {
    const int id = i / FW, ff = f0 + i % FW;
    Ts[i] = (ff < nEff && id < 316) ? T[(int64_t)id * nEff + ff] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const bool act = f < nEff && rhs < nrhs;
  const int64_t lanePos = act ? (int64_t)f * fStride + (int64_t)rl * rStride : 0;
  const float2* inF = effIn + (act ? blockIdx.z * inL.blk : 0) + lanePos;
  float2* outF = effOut + blockIdx.z * outL.blk + lanePos;
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * PQX_ROWS);
  for (int b = blockIdx.x * PQX_ROWS + warp; b < bEnd; b += PQX_THREADS / 32) {
    unsigned long long acc[8];
#pragma unroll
    for (int c = 0; c < 8; c++) acc[c] = 0ull;
    int64_t e = nPtr[b];
    const int64_t e1 = nPtr[b + 1];
    int4 sa = make_int4(-1, -1, -1, -1), sb = sa;
    int off = 13;
    if (e < e1) {
      sa = reinterpret_cast<const int4*>(nIn)[2 * e];
      sb = reinterpret_cast<const int4*>(nIn)[2 * e + 1];
      off = nOff[e];
    }
    for (; e < e1; e++) {
      const int sl[8] = {sa.x, sa.y, sa.z, sa.w, sb.x, sb.y, sb.z, sb.w};
      unsigned long long inD[8], inR[8];
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++) {
        const float2 d = (act && sl[c2] >= 0) ? inF[(int64_t)sl[c2] * inL.slot] : make_float2(0.f, 0.f);
        inD[c2] = pq_pk(d.x, d.y);
        inR[c2] = pq_pk(-d.y, d.x);
      }
      const int offCur = off;
      if (e + 1 < e1) {
        sa = reinterpret_cast<const int4*>(nIn)[2 * (e + 1)];
        sb = reinterpret_cast<const int4*>(nIn)[2 * (e + 1) + 1];
        off = nOff[e + 1];
      }
      pq_delta_x2<ADJ, 0, FW>(acc, inD, inR, Ts, &sId[offCur * 27], fl);
    }
    if (!act) continue;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int t = rowOut[8 * b + c];
      if (t < 0) continue;
      const float2 a = pq_unpk(acc[c]);
      outF[(int64_t)t * outL.slot] = make_float2(a.x * nrmfc, a.y * nrmfc);
    }
  }
}

}  // namespace fmmg
