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
// rows per CTA, nEff / 32, ceil(nrhs / KB)) (PQ_PARENTS rows per CTA by default); dynamic shared memory
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
  const int per = (nRows + gridDim.x - 1) / gridDim.x;  // rows per CTA: the grid sets it (tunable)
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * per);
  for (int b = blockIdx.x * per + warp; b < bEnd; b += PQ_THREADS / 32) {
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

// The translation of this group as the two packed operands (t.x, t.x) and
// (t.y, t.y): for FW = 4 the CTA stages each translation pre-duplicated as
// {t.x, t.x, t.y, t.y} (conjugated for ADJ), so one 16-byte shared load gives
// both; for FW = 32 it stages plain complex values and packs in registers.
template <bool ADJ, int FW>
__device__ __forceinline__ void pq_tpair(const void* __restrict__ Ts, int row, int fl, unsigned long long& tx,
                                         unsigned long long& ty) {
  if constexpr (FW == 4) {
    const ulonglong2 t = reinterpret_cast<const ulonglong2*>(Ts)[row * FW + fl];
    tx = t.x;
    ty = t.y;
  } else {
    const float2 t = reinterpret_cast<const float2*>(Ts)[row * FW + fl];
    tx = pq_pk(t.x, t.x);
    ty = ADJ ? pq_pk(-t.y, -t.y) : pq_pk(t.y, t.y);
  }
}

template <bool ADJ, int E, int FW>
__device__ __forceinline__ void pq_delta_x2(unsigned long long (&acc)[8], const unsigned long long (&inD)[8],
                                            const unsigned long long (&inR)[8], const void* __restrict__ Ts,
                                            const int16_t* __restrict__ sIdRow, int fl) {
  if constexpr (E < 27) {
    constexpr int ex = E / 9 - 1, ey = (E / 3) % 3 - 1, ez = E % 3 - 1;
    unsigned long long tx, ty;
    pq_tpair<ADJ, FW>(Ts, sIdRow[E], fl, tx, ty);
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
// per CTA, nEff / FW, ceil(nrhs / (32 / FW))) (PQX_ROWS rows per CTA by default); blockIdx.z selects the
// right-hand-side block of the layout below; dynamic shared memory
// pqx_smem_bytes<FW>() (row 316 is the zero row of touching pairs).
constexpr int PQX_THREADS = 256;
constexpr int PQX_ROWS = 64;
template <int FW>
inline size_t pqx_smem_bytes() {
  return (size_t)317 * FW * (FW == 4 ? 16 : 8);
}

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
  extern __shared__ __align__(16) unsigned char pqx_smem[];
  __shared__ int16_t sId[27 * 27];
  pq_id_table<ADJ>(sId, transId);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fl = lane % FW, rl = lane / FW;
  const int f0 = blockIdx.y * FW;
  const int f = f0 + fl;
  const int rhs = blockIdx.z * RW + rl;
  for (int i = threadIdx.x; i < 317 * FW; i += blockDim.x) {
    const int id = i / FW, ff = f0 + i % FW;
    const float2 t = (ff < nEff && id < 316) ? T[(int64_t)id * nEff + ff] : make_float2(0.f, 0.f);
    if constexpr (FW == 4) {
      const float ty = ADJ ? -t.y : t.y;
      reinterpret_cast<float4*>(pqx_smem)[i] = make_float4(t.x, t.x, ty, ty);
    } else {
      reinterpret_cast<float2*>(pqx_smem)[i] = t;
    }
  }
  __syncthreads();
  const void* Ts = pqx_smem;
  const bool act = f < nEff && rhs < nrhs;
  const int64_t lanePos = act ? (int64_t)f * fStride + (int64_t)rl * rStride : 0;
  const float2* inF = effIn + (act ? blockIdx.z * inL.blk : 0) + lanePos;
  float2* outF = effOut + blockIdx.z * outL.blk + lanePos;
  const int per = (nRows + gridDim.x - 1) / gridDim.x;  // rows per CTA: the grid sets it (tunable)
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * per);
  for (int b = blockIdx.x * per + warp; b < bEnd; b += PQX_THREADS / 32) {
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

namespace fmmg {

// ---------------------------------------------------------------- 27-product form
// For a neighbour offset o the 8 x 8 child-pair matrix is block-Toeplitz over
// the 2 x 2 x 2 child grid (entry (c, c2) depends on c2 - c only; touching
// pairs are zero for the whole (o, c2 - c) class), so per axis
//   [y0; y1] = [[t0, t1], [t_-1, t0]] [x0; x1]
// needs the three products m1 = t0 (x0 + x1), m2 = (t1 - t0) x1,
// m3 = (t_-1 - t0) x0, with y0 = m1 + m2 and y1 = m1 + m3.  Taken over the
// three axes this is 27 complex products per parent pair instead of 64:
// combined translations T'[o][j] (j = (jx, jy, jz), each m1/m2/m3) come from
// the host, the input combinations are sums of child spectra, and the output
// combination runs once per parent after all neighbours (it is linear).
//
// k_m2l_had_w8: FP32, blocks of 8 right-hand sides in the interleaved layout,
// a warp owns one parent, 4 frequencies and 8 right-hand sides.  The CTA
// stages T'[27][27][4 frequencies]; with u an input combination and
// s(u) = (u.y, u.x) a complex MAC is
//   acc = fma2((t.x, t.x), u, acc);  acc = fma2((-t.y, t.y), s(u), acc).
// The translations are read as 8-byte values (the kernel is bound by shared-
// memory wavefronts: 16-byte reads cost 4 per warp, 8-byte ones 2).
// Grid (rows / rows per CTA, nEff / 4, ceil(nrhs / 8)); dynamic shared memory
// 27 * 27 * 4 * 8 bytes.
constexpr int W8_OFFS = 27;  // offset codes 0..26 (13 unused)

__device__ __forceinline__ unsigned long long w8_add(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// Sum over the children (bx, by, bz) selected by the y and z combination
// codes jy, jz (0: both, 1: b = 1, 2: b = 0) for a fixed bx.
template <int JY, int JZ>
__device__ __forceinline__ unsigned long long w8_yz(const unsigned long long (&x)[8], int bx) {
  unsigned long long s = 0ull;
  bool first = true;
#pragma unroll
  for (int by = 0; by < 2; by++)
#pragma unroll
    for (int bz = 0; bz < 2; bz++) {
      if ((JY == 1 && by == 0) || (JY == 2 && by == 1) || (JZ == 1 && bz == 0) || (JZ == 2 && bz == 1)) continue;
      const unsigned long long v = x[bx * 4 + by * 2 + bz];
      s = first ? v : w8_add(s, v);
      first = false;
    }
  return s;
}

// acc += t * u for the combined translation t = Tw[i] (8-byte shared load,
// served per half-warp: 2 wavefronts) and u packed (re, im): the t.x terms as
// one packed FMA on (t.x, t.x), the t.y terms (re -= t.y im, im += t.y re) as
// two scalar FMAs, which take the negation and the crossed halves as operand
// forms instead of a swapped copy of u and a (-t.y, t.y) pair.  Per component
// the same two roundings as two packed FMAs.
__device__ __forceinline__ void w8_cmac(unsigned long long& acc, const float2* __restrict__ Tw, int i,
                                        unsigned long long u) {
  const float2 t = Tw[i];
  pq_fma2(acc, pq_pk(t.x, t.x), u);
  float2 a = pq_unpk(acc);
  const float2 v = pq_unpk(u);
  a.x = fmaf(-t.y, v.y, a.x);
  a.y = fmaf(t.y, v.x, a.y);
  acc = pq_pk(a.x, a.y);
}

template <int J>
__device__ __forceinline__ void w8_group(unsigned long long (&acc)[27], const unsigned long long (&x)[8],
                                         const float2* __restrict__ Tw, int fl) {
  if constexpr (J < 9) {
    constexpr int JY = J / 3, JZ = J % 3;
    const unsigned long long p0 = w8_yz<JY, JZ>(x, 0), p1 = w8_yz<JY, JZ>(x, 1);
    // jx = m1 (x0 + x1), m2 (x1), m3 (x0); j = jx * 9 + jy * 3 + jz
    w8_cmac(acc[0 * 9 + J], Tw, (0 * 9 + J) * 4 + fl, w8_add(p0, p1));
    w8_cmac(acc[1 * 9 + J], Tw, (1 * 9 + J) * 4 + fl, p1);
    w8_cmac(acc[2 * 9 + J], Tw, (2 * 9 + J) * 4 + fl, p0);
    w8_group<J + 1>(acc, x, Tw, fl);
  }
}

static __global__ void __launch_bounds__(PQX_THREADS, 2)
    k_m2l_had_w8(int nRows, const int32_t* __restrict__ rowOut, const int64_t* __restrict__ nPtr,
                 const int8_t* __restrict__ nOff, const int32_t* __restrict__ nIn, const float2* __restrict__ effIn,
                 PqLayout inL, const float2* __restrict__ Tw, float2* __restrict__ effOut, PqLayout outL, int nEff,
                 int nrhs, float nrmfc) {
  extern __shared__ __align__(16) unsigned char w8_smem[];
  float2* Ts = reinterpret_cast<float2*>(w8_smem);  // [27 offsets][27 combinations][4 frequencies]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fl = lane & 3, rl = lane >> 2;
  const int f0 = blockIdx.y * 4;
  const int f = f0 + fl;
  const int rhs = blockIdx.z * 8 + rl;
  for (int i = threadIdx.x; i < W8_OFFS * 27 * 4; i += blockDim.x) {
    const int oj = i >> 2, ff = f0 + (i & 3);
    Ts[i] = ff < nEff ? Tw[(int64_t)oj * nEff + ff] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const bool act = f < nEff && rhs < nrhs;
  const int64_t lanePos = act ? (int64_t)f * 8 + rl : 0;
  const float2* inF = effIn + (act ? blockIdx.z * inL.blk : 0) + lanePos;
  float2* outF = effOut + blockIdx.z * outL.blk + lanePos;
  const int per = (nRows + gridDim.x - 1) / gridDim.x;  // rows per CTA: the grid sets it (tunable)
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * per);
  for (int b = blockIdx.x * per + warp; b < bEnd; b += PQX_THREADS / 32) {
    unsigned long long acc[27];
#pragma unroll
    for (int j = 0; j < 27; j++) acc[j] = 0ull;
    // software pipeline: the spectra of neighbour e + 1 load while neighbour e
    // multiplies; the child slots run one neighbour further ahead
    int64_t e = nPtr[b];
    const int64_t e1 = nPtr[b + 1];
    float2 raw[8];
    int offNext = 13;
    int4 sa = make_int4(-1, -1, -1, -1), sb = sa;
    if (e < e1) {
      const int4 a0 = reinterpret_cast<const int4*>(nIn)[2 * e];
      const int4 b0 = reinterpret_cast<const int4*>(nIn)[2 * e + 1];
      const int sl[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++)
        raw[c2] = (act && sl[c2] >= 0) ? inF[(int64_t)sl[c2] * inL.slot] : make_float2(0.f, 0.f);
      offNext = nOff[e];
      if (e + 1 < e1) {
        sa = reinterpret_cast<const int4*>(nIn)[2 * (e + 1)];
        sb = reinterpret_cast<const int4*>(nIn)[2 * (e + 1) + 1];
      }
    }
    for (; e < e1; e++) {
      unsigned long long x[8];
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++) x[c2] = pq_pk(raw[c2].x, raw[c2].y);
      const int offCur = offNext;
      if (e + 1 < e1) {
        const int sl[8] = {sa.x, sa.y, sa.z, sa.w, sb.x, sb.y, sb.z, sb.w};
#pragma unroll
        for (int c2 = 0; c2 < 8; c2++)
          raw[c2] = (act && sl[c2] >= 0) ? inF[(int64_t)sl[c2] * inL.slot] : make_float2(0.f, 0.f);
        offNext = nOff[e + 1];
        if (e + 2 < e1) {
          sa = reinterpret_cast<const int4*>(nIn)[2 * (e + 2)];
          sb = reinterpret_cast<const int4*>(nIn)[2 * (e + 2) + 1];
        }
      }
      w8_group<0>(acc, x, Ts + offCur * 27 * 4, fl);
    }
    if (!act) continue;
    // output combination: child (cx, cy, cz) sums the products whose codes are
    // m1 or (m2 for c = 0, m3 for c = 1) on every axis
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int t = rowOut[8 * b + c];
      if (t < 0) continue;
      const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
      unsigned long long s = 0ull;
#pragma unroll
      for (int j = 0; j < 27; j++) {
        const int jx = j / 9, jy = (j / 3) % 3, jz = j % 3;
        const bool use = (jx == 0 || jx == 1 + cx) && (jy == 0 || jy == 1 + cy) && (jz == 0 || jz == 1 + cz);
        if (use) s = w8_add(s, acc[j]);
      }
      const float2 a = pq_unpk(s);
      outF[(int64_t)t * outL.slot] = make_float2(a.x * nrmfc, a.y * nrmfc);
    }
  }
}


// k_m2l_had_w8x2: the 27-product form with two right-hand sides per thread.
// Lanes = 8 frequencies x 4 pairs of right-hand sides (one block of 8), a
// warp per target parent as in k_m2l_had_w8.  Each combined translation read
// from shared memory feeds both right-hand sides, which halves the table
// traffic per FMA (the L1 data path bounds the one-per-thread form); the two
// right-hand sides of a lane are adjacent in the interleaved layout, so every
// child spectrum is one 16-byte load.  Per right-hand side the arithmetic is
// the same operations in the same order as k_m2l_had_w8, so the results are
// identical.
constexpr int W8X2_F = 8;  // frequencies per CTA

template <int J>
__device__ __forceinline__ void w8x2_group(unsigned long long (&acc)[2][27], const unsigned long long (&x)[2][8],
                                           const float2* __restrict__ Tw, int fl) {
  if constexpr (J < 9) {
    constexpr int JY = J / 3, JZ = J % 3;
#pragma unroll
    for (int jx = 0; jx < 3; jx++) {
      const float2 t = Tw[(jx * 9 + J) * W8X2_F + fl];
      const unsigned long long tx = pq_pk(t.x, t.x);
#pragma unroll
      for (int r = 0; r < 2; r++) {
        const unsigned long long p0 = w8_yz<JY, JZ>(x[r], 0), p1 = w8_yz<JY, JZ>(x[r], 1);
        const unsigned long long u = jx == 0 ? w8_add(p0, p1) : (jx == 1 ? p1 : p0);
        unsigned long long& a = acc[r][jx * 9 + J];
        pq_fma2(a, tx, u);
        float2 av = pq_unpk(a);
        const float2 v = pq_unpk(u);
        av.x = fmaf(-t.y, v.y, av.x);
        av.y = fmaf(t.y, v.x, av.y);
        a = pq_pk(av.x, av.y);
      }
    }
    w8x2_group<J + 1>(acc, x, Tw, fl);
  }
}

static __global__ void __launch_bounds__(PQX_THREADS, 1)
    k_m2l_had_w8x2(int nRows, const int32_t* __restrict__ rowOut, const int64_t* __restrict__ nPtr,
                   const int8_t* __restrict__ nOff, const int32_t* __restrict__ nIn, const float2* __restrict__ effIn,
                   PqLayout inL, const float2* __restrict__ Tw, float2* __restrict__ effOut, PqLayout outL, int nEff,
                   int nrhs, float nrmfc) {
  extern __shared__ __align__(16) unsigned char w8x2_smem[];
  float2* Ts = reinterpret_cast<float2*>(w8x2_smem);  // [27 offsets][27 combinations][8 frequencies]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fl = lane & 7, rp = lane >> 3;
  const int f0 = blockIdx.y * W8X2_F;
  const int f = f0 + fl;
  const int rhs = blockIdx.z * 8 + 2 * rp;  // this lane's two right-hand sides: rhs, rhs + 1
  for (int i = threadIdx.x; i < W8_OFFS * 27 * W8X2_F; i += blockDim.x) {
    const int oj = i / W8X2_F, ff = f0 + (i % W8X2_F);
    Ts[i] = ff < nEff ? Tw[(int64_t)oj * nEff + ff] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const bool act = f < nEff && rhs < nrhs;
  const bool two = rhs + 1 < nrhs;
  // the block holds 8 right-hand-side slots, so rhs + 1 is in the buffer
  const int64_t lanePos = act ? (int64_t)f * 8 + 2 * rp : 0;
  const float4* inF = reinterpret_cast<const float4*>(effIn + (act ? blockIdx.z * inL.blk : 0) + lanePos);
  float2* outF = effOut + blockIdx.z * outL.blk + lanePos;
  const int64_t inSlot4 = inL.slot / 2;  // float4 units (slot strides are multiples of 8 float2)
  const int per = (nRows + gridDim.x - 1) / gridDim.x;
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * per);
  for (int b = blockIdx.x * per + warp; b < bEnd; b += PQX_THREADS / 32) {
    unsigned long long acc[2][27];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
      for (int j = 0; j < 27; j++) acc[r][j] = 0ull;
    int64_t e = nPtr[b];
    const int64_t e1 = nPtr[b + 1];
    float4 raw[8];
    int offNext = 13;
    int4 sa = make_int4(-1, -1, -1, -1), sb = sa;
    if (e < e1) {
      const int4 a0 = reinterpret_cast<const int4*>(nIn)[2 * e];
      const int4 b0 = reinterpret_cast<const int4*>(nIn)[2 * e + 1];
      const int sl[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++)
        raw[c2] = (act && sl[c2] >= 0) ? inF[(int64_t)sl[c2] * inSlot4] : make_float4(0.f, 0.f, 0.f, 0.f);
      offNext = nOff[e];
      if (e + 1 < e1) {
        sa = reinterpret_cast<const int4*>(nIn)[2 * (e + 1)];
        sb = reinterpret_cast<const int4*>(nIn)[2 * (e + 1) + 1];
      }
    }
    for (; e < e1; e++) {
      unsigned long long x[2][8];
#pragma unroll
      for (int c2 = 0; c2 < 8; c2++) {
        x[0][c2] = pq_pk(raw[c2].x, raw[c2].y);
        x[1][c2] = pq_pk(raw[c2].z, raw[c2].w);
      }
      const int offCur = offNext;
      if (e + 1 < e1) {
        const int sl[8] = {sa.x, sa.y, sa.z, sa.w, sb.x, sb.y, sb.z, sb.w};
#pragma unroll
        for (int c2 = 0; c2 < 8; c2++)
          raw[c2] = (act && sl[c2] >= 0) ? inF[(int64_t)sl[c2] * inSlot4] : make_float4(0.f, 0.f, 0.f, 0.f);
        offNext = nOff[e + 1];
        if (e + 2 < e1) {
          sa = reinterpret_cast<const int4*>(nIn)[2 * (e + 2)];
          sb = reinterpret_cast<const int4*>(nIn)[2 * (e + 2) + 1];
        }
      }
      w8x2_group<0>(acc, x, Ts + offCur * 27 * W8X2_F, fl);
    }
    if (!act) continue;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int t = rowOut[8 * b + c];
      if (t < 0) continue;
      const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
      unsigned long long s0 = 0ull, s1 = 0ull;
#pragma unroll
      for (int j = 0; j < 27; j++) {
        const int jx = j / 9, jy = (j / 3) % 3, jz = j % 3;
        const bool use = (jx == 0 || jx == 1 + cx) && (jy == 0 || jy == 1 + cy) && (jz == 0 || jz == 1 + cz);
        if (use) {
          s0 = w8_add(s0, acc[0][j]);
          s1 = w8_add(s1, acc[1][j]);
        }
      }
      const float2 a0 = pq_unpk(s0), a1 = pq_unpk(s1);
      float2* o = outF + (int64_t)t * outL.slot;
      if (two)
        *reinterpret_cast<float4*>(o) = make_float4(a0.x * nrmfc, a0.y * nrmfc, a1.x * nrmfc, a1.y * nrmfc);
      else
        o[0] = make_float2(a0.x * nrmfc, a0.y * nrmfc);
    }
  }
}


// k_m2l_had_o<R>: the 27-product Hadamard accumulated in the space of the 8
// output children, R = 2 or 4 right-hand sides a lane.  The 27-product form
// above keeps 27 accumulators per right-hand side, so a lane holds one
// right-hand side and every combined translation read from shared memory
// feeds one complex multiply-add: the kernel is bound by the L1 data path
// (27 translation and 8 spectrum reads per neighbour).  Here each neighbour's
// 27 products are folded into the 8 children at once, along one axis at a
// time (m0 + m1 | m0 + m2 per axis, 28 adds for the three axes), so the state
// per right-hand side is 8 accumulators and a lane can hold R of them: the 27
// translations of a neighbour are read once into registers and used for all R
// right-hand sides.  The input combinations go the same way (19 adds), the
// products are 9 complex multiplies and 18 complex multiply-adds.  Per right-
// hand side that is a few more FP32 operations than the 27-product kernel but
// R times fewer translation reads.
// Lanes: FB = 4 R frequencies x (8 / R) groups of R right-hand sides of a
// block of 8; a warp owns one target parent; the CTA stages T'[27][27][FB].
// Grid (rows / rows per CTA, nEff / FB, ceil(nrhs / 8)); dynamic shared
// memory 27 * 27 * FB * 8 bytes.
__device__ __forceinline__ unsigned long long ho_cmul(float2 t, unsigned long long u) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pq_pk(t.x, t.x)), "l"(u));
  float2 a = pq_unpk(r);
  const float2 v = pq_unpk(u);
  a.x = fmaf(-t.y, v.y, a.x);
  a.y = fmaf(t.y, v.x, a.y);
  return pq_pk(a.x, a.y);
}
__device__ __forceinline__ unsigned long long ho_cmac(unsigned long long acc, float2 t, unsigned long long u) {
  pq_fma2(acc, pq_pk(t.x, t.x), u);
  float2 a = pq_unpk(acc);
  const float2 v = pq_unpk(u);
  a.x = fmaf(-t.y, v.y, a.x);
  a.y = fmaf(t.y, v.x, a.y);
  return pq_pk(a.x, a.y);
}

// One neighbour's contribution for one right-hand side: children x[8]
// (index 4 bx + 2 by + bz), translations t[27] (index 9 jx + 3 jy + jz),
// added into acc[8] (index 4 cx + 2 cy + cz).  Codes per axis: inputs
// 0: x0 + x1, 1: x1, 2: x0; outputs c = 0 take codes 0 and 1, c = 1 codes 0 and 2.
__device__ __forceinline__ void ho_apply(unsigned long long (&acc)[8], const unsigned long long (&x)[8],
                                         const float2 (&t)[27]) {
#pragma unroll
  for (int jz = 0; jz < 3; jz++) {
    unsigned long long uz[4];  // [bx][by], z combined by code jz
#pragma unroll
    for (int q = 0; q < 4; q++) uz[q] = jz == 0 ? w8_add(x[2 * q], x[2 * q + 1]) : (jz == 1 ? x[2 * q + 1] : x[2 * q]);
    unsigned long long uy[2][3];  // [bx][jy]
#pragma unroll
    for (int bx = 0; bx < 2; bx++) {
      uy[bx][0] = w8_add(uz[2 * bx], uz[2 * bx + 1]);
      uy[bx][1] = uz[2 * bx + 1];
      uy[bx][2] = uz[2 * bx];
    }
    unsigned long long vx[2][3];  // [cx][jy]: the products folded along x
#pragma unroll
    for (int jy = 0; jy < 3; jy++) {
      const int jyz = 3 * jy + jz;
      const unsigned long long m0 = ho_cmul(t[jyz], w8_add(uy[0][jy], uy[1][jy]));
      vx[0][jy] = ho_cmac(m0, t[9 + jyz], uy[1][jy]);
      vx[1][jy] = ho_cmac(m0, t[18 + jyz], uy[0][jy]);
    }
#pragma unroll
    for (int cx = 0; cx < 2; cx++) {
      const unsigned long long w0 = w8_add(vx[cx][0], vx[cx][1]), w1 = w8_add(vx[cx][0], vx[cx][2]);  // cy = 0, 1
      // fold along z into the children: cz = 0 takes jz 0, 1; cz = 1 takes jz 0, 2
#pragma unroll
      for (int cy = 0; cy < 2; cy++) {
        const unsigned long long w = cy ? w1 : w0;
        const int c = 4 * cx + 2 * cy;
        if (jz == 0) {
          acc[c] = w8_add(acc[c], w);
          acc[c + 1] = w8_add(acc[c + 1], w);
        } else if (jz == 1) {
          acc[c] = w8_add(acc[c], w);
        } else {
          acc[c + 1] = w8_add(acc[c + 1], w);
        }
      }
    }
  }
}

// 32 bytes from global memory in one 256-bit load (sm_100); p is 32-byte aligned
__device__ __forceinline__ void ho_ld256(const float* p, float4& a, float4& b) {
  asm("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

template <int R>
static __global__ void __launch_bounds__(PQX_THREADS, 1)
    k_m2l_had_o(int nRows, const int32_t* __restrict__ rowOut, const int64_t* __restrict__ nPtr,
                const int8_t* __restrict__ nOff, const int32_t* __restrict__ nIn, const float2* __restrict__ effIn,
                PqLayout inL, const float2* __restrict__ Tw, float2* __restrict__ effOut, PqLayout outL, int nEff,
                int nrhs, float nrmfc) {
  static_assert(R == 2 || R == 4, "two or four right-hand sides a lane");
  constexpr int G = 8 / R, FB = 32 / G;
  extern __shared__ __align__(16) unsigned char ho_smem[];
  float2* Ts = reinterpret_cast<float2*>(ho_smem);  // [27 offsets][27 combinations][FB frequencies]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fl = lane % FB, rg = lane / FB;
  const int f0 = blockIdx.y * FB;
  const int f = f0 + fl;
  const int rhs0 = blockIdx.z * 8 + rg * R;  // this lane's right-hand sides rhs0 .. rhs0 + R - 1
  for (int i = threadIdx.x; i < W8_OFFS * 27 * FB; i += blockDim.x) {
    const int oj = i / FB, ff = f0 + (i % FB);
    Ts[i] = ff < nEff ? Tw[(int64_t)oj * nEff + ff] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const bool act = f < nEff && rhs0 < nrhs;
  // the block holds 8 right-hand-side slots, so rhs0 + R - 1 is in the buffer
  const int64_t lanePos = act ? (int64_t)f * 8 + rg * R : 0;
  const float4* inF = reinterpret_cast<const float4*>(effIn + (act ? blockIdx.z * inL.blk : 0) + lanePos);
  float2* outF = effOut + blockIdx.z * outL.blk + lanePos;
  const int64_t inSlot4 = inL.slot / 2;  // float4 units (slot strides are multiples of 8 float2)
  // the warp's parent's neighbour entries (input child slots, offset code),
  // up to 32 at a time, so each neighbour starts on shared-memory reads
  __shared__ int4 sIn[PQX_THREADS / 32][32][2];
  __shared__ int sOff[PQX_THREADS / 32][32];
  const int per = (nRows + gridDim.x - 1) / gridDim.x;
  const int bEnd = min(nRows, (int)(blockIdx.x + 1) * per);
  for (int b = blockIdx.x * per + warp; b < bEnd; b += PQX_THREADS / 32) {
    unsigned long long acc[R][8];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int c = 0; c < 8; c++) acc[r][c] = 0ull;
    const int64_t e1 = nPtr[b + 1];
    for (int64_t c0 = nPtr[b]; c0 < e1; c0 += 32) {  // one pass: a parent has at most 26 neighbours
    const int ne = (int)min((int64_t)32, e1 - c0);
    __syncwarp();
    if (lane < ne) {
      sIn[warp][lane][0] = reinterpret_cast<const int4*>(nIn)[2 * (c0 + lane)];
      sIn[warp][lane][1] = reinterpret_cast<const int4*>(nIn)[2 * (c0 + lane) + 1];
      sOff[warp][lane] = nOff[c0 + lane];
    }
    __syncwarp();
    for (int j = 0; j < ne; j++) {
      const int4 a0 = sIn[warp][j][0];
      const int4 b0 = sIn[warp][j][1];
      const int sl[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
      const float2* Tn = Ts + sOff[warp][j] * 27 * FB + fl;
      float2 t[27];
#pragma unroll
      for (int jj = 0; jj < 27; jj++) t[jj] = Tn[jj * FB];
      if constexpr (R == 4) {
        // the lane's 4 right-hand sides of a child are 32 contiguous bytes:
        // one 256-bit load each, so a warp's load of a child covers whole
        // 128-byte lines (two 16-byte loads each read half of 8 lines)
        float4 lo[8], hi[8];
#pragma unroll
        for (int c2 = 0; c2 < 8; c2++) {
          if (act && sl[c2] >= 0) {
            ho_ld256(reinterpret_cast<const float*>(inF + (int64_t)sl[c2] * inSlot4), lo[c2], hi[c2]);
          } else {
            lo[c2] = hi[c2] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
#pragma unroll
        for (int p = 0; p < 2; p++) {
          unsigned long long x[8];
#pragma unroll
          for (int c2 = 0; c2 < 8; c2++) x[c2] = p ? pq_pk(hi[c2].x, hi[c2].y) : pq_pk(lo[c2].x, lo[c2].y);
          ho_apply(acc[2 * p], x, t);
#pragma unroll
          for (int c2 = 0; c2 < 8; c2++) x[c2] = p ? pq_pk(hi[c2].z, hi[c2].w) : pq_pk(lo[c2].z, lo[c2].w);
          ho_apply(acc[2 * p + 1], x, t);
        }
      } else {
#pragma unroll
        for (int p = 0; p < R / 2; p++) {  // right-hand sides 2p, 2p + 1 of this lane
          float4 raw[8];
#pragma unroll
          for (int c2 = 0; c2 < 8; c2++)
            raw[c2] = (act && sl[c2] >= 0) ? inF[(int64_t)sl[c2] * inSlot4 + p] : make_float4(0.f, 0.f, 0.f, 0.f);
          unsigned long long x[8];
#pragma unroll
          for (int c2 = 0; c2 < 8; c2++) x[c2] = pq_pk(raw[c2].x, raw[c2].y);
          ho_apply(acc[2 * p], x, t);
#pragma unroll
          for (int c2 = 0; c2 < 8; c2++) x[c2] = pq_pk(raw[c2].z, raw[c2].w);
          ho_apply(acc[2 * p + 1], x, t);
        }
      }
    }
    }
    if (!act) continue;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int tt = rowOut[8 * b + c];
      if (tt < 0) continue;
      float4* o = reinterpret_cast<float4*>(outF + (int64_t)tt * outL.slot);
#pragma unroll
      for (int p = 0; p < R / 2; p++) {
        const float2 a0 = pq_unpk(acc[2 * p][c]), a1 = pq_unpk(acc[2 * p + 1][c]);
        o[p] = make_float4(a0.x * nrmfc, a0.y * nrmfc, a1.x * nrmfc, a1.y * nrmfc);
      }
    }
  }
}

}  // namespace fmmg
