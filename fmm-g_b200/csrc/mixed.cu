// mixed.cu -- the mixed-precision, multi-right-hand-side evaluate
// (FMMG_PREC_MIXED).
//
// Same stage sequence and work lists as the FP64 form (stages.cu); the bulk
// arithmetic is FP32 and every kernel handles a block of KB right-hand sides
// per launch (grid.y or the row index runs over the blocks), so geometry,
// kernel evaluations, operator tiles and M2L translation spectra are loaded
// once per block instead of once per density:
//  * direct sums (near-field P2P, S2M, S2L, M2T, L2T) evaluate the kernel in
//    FP32 on coordinates taken relative to the centre of the target box (the
//    subtraction happens in FP64 before rounding), add each shared-memory tile
//    of at most 128 sources in FP32 and carry the tile sums in FP64; target
//    values are accumulated in FP64;
//  * the equivalent-density GEMMs and the spectral M2L (FFTs and Hadamard
//    products) run in FP32 with FP32 operator tables.
#include <stdexcept>
#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <cmath>
#include <string>
#include <vector>

#include "cuda_common.cuh"
#include "engine.hpp"
#include "gemm_rows.cuh"
#include "gemm_tc.cuh"
#include "had_pq.cuh"
#include "had_smem.cuh"
#include "kernels.hpp"

namespace fmmg {

__constant__ int16_t c_transId32[343];

constexpr int MX_THREADS = 128;
constexpr int MX_THREADS_FAR = 192;  // M2T: 2^6 x 3 also allows target groups of 24, 48, 96
constexpr int MX_TILE = 128;
// staged sources (or surface points) per round: 256 when a source carries at
// most 8 density values and no normal (the static shared memory stays under
// 48 KB), else 128
template <int DEN, bool NRM>
constexpr int mx_tile() {
  return (DEN <= 8 && !NRM) ? 256 : 128;
}
constexpr int MX_MAXE = 256;

// fill eBeg/ePre for entries [ec, ec+ne) and return the total source count
__device__ __forceinline__ int load_entries(const int32_t* __restrict__ idx, int64_t ec, int ne, int self,
                                            const int64_t* __restrict__ srcBeg, const int64_t* __restrict__ srcCnt,
                                            int64_t* eBeg, int32_t* ePre) {
  __syncthreads();
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    int s = idx ? idx[ec + e] : self;
    eBeg[e] = srcBeg[s];
    ePre[e + 1] = (int32_t)srcCnt[s];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ePre[0] = 0;
    for (int e = 0; e < ne; e++) ePre[e + 1] += ePre[e];
  }
  __syncthreads();
  return ePre[ne];
}

__device__ __forceinline__ int64_t entry_source(int j, int ne, const int64_t* eBeg, const int32_t* ePre) {
  int lo = 0, hi = ne;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (ePre[mid] <= j) lo = mid; else hi = mid;
  }
  return eBeg[lo] + (j - ePre[lo]);
}

// Shared epilogue of the target-side kernels: reduce the S source splits of
// each target and add the KB x TD values into val (FP64).
template <int TD, int KB>
__device__ __forceinline__ void reduce_store(double* sRed, const double* acc, int tid, int tl, int sp, int TG, int S,
                                             bool act, double* __restrict__ val, int64_t trgIdx, int rhs0, int nrhs,
                                             int64_t valStride, bool assign = false) {
  __syncthreads();
#pragma unroll
  for (int c = 0; c < TD * KB; c++) sRed[tid * TD * KB + c] = acc[c];
  __syncthreads();
  if (sp == 0 && act) {
#pragma unroll
    for (int r = 0; r < KB; r++) {
      if (rhs0 + r >= nrhs) break;
#pragma unroll
      for (int c = 0; c < TD; c++) {
        double s = 0;
        for (int k = 0; k < S; k++) s += sRed[(tl + k * TG) * TD * KB + r * TD + c];
        double& v = val[(int64_t)(rhs0 + r) * valStride + trgIdx * TD + c];
        v = assign ? s : v + s;
      }
    }
  }
}

// Lanes per target group of a leaf with tn targets: the smallest of 8, 16,
// 24, 32, 48, 64, 96, 128 that divides the CTA size, is at least gmin and
// holds them, else the whole CTA (a leaf holds ~ptsMax/4..ptsMax points); the
// rest of the CTA splits the sources.
template <int THREADS>
__device__ __forceinline__ int mx_group(int64_t tn, int gmin = 8) {
  if constexpr ((THREADS & (THREADS - 1)) == 0) {  // power of two: 8, 16, 32, ...
    int g = gmin;
    while (g < THREADS && g < tn) g *= 2;
    return g;
  } else {
    constexpr int G[7] = {8, 16, 24, 32, 48, 64, 96};
#pragma unroll
    for (int i = 0; i < 7; i++)
      if (THREADS % G[i] == 0 && G[i] >= gmin && G[i] >= tn) return G[i];
    return THREADS;
  }
}

// The N staged densities of one source from shared memory into registers,
// as 16-byte vectors when N is a multiple of 4 (the row is 16-byte aligned).
template <int N>
__device__ __forceinline__ void mx_den(const float* __restrict__ s, float (&d)[N]) {
  if constexpr (N % 4 == 0) {
#pragma unroll
    for (int c = 0; c < N; c += 4) {
      const float4 v = *reinterpret_cast<const float4*>(s + c);
      d[c] = v.x;
      d[c + 1] = v.y;
      d[c + 2] = v.z;
      d[c + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int c = 0; c < N; c++) d[c] = s[c];
  }
}

// near field: U-list, direct W and X entries; grid (evaluator leaves, RHS blocks).
// The offsets are formed from hi/lo FP32 pairs of the box-centred
// coordinates, (x_hi - y_hi) + (x_lo - y_lo): the hi difference of close
// points is exact, so near-coincident pairs keep their separation.  For the
// double-layer kernels (source normal, NRM) n.(x - y) is formed in FP64 from
// those pairs and the normal's hi/lo pair: on densely sampled surfaces
// near-coincident pairs dominate the sum and n.(x - y) cancels to curvature
// size, O(r^2), while any FP32 rounding of the offset or the normal leaves an
// O(eps r) error in it (relative error eps / (kappa r), 1e-3 at r = 1e-6).
template <int KT, int KB>
__global__ void __launch_bounds__(MX_THREADS)
    k_p2p_near32(const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                 const int64_t* __restrict__ srcBeg, const int64_t* __restrict__ srcCnt,
                 const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt,
                 const double* __restrict__ src, const double* __restrict__ nrm, const float* __restrict__ den32,
                 int64_t den32Blk, const double* __restrict__ trg, const double* __restrict__ ctr,
                 double* __restrict__ val, int64_t valStride, int nrhs, float mu, float ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  constexpr int MX_TILE = mx_tile<SD * KB, NRM != 0>();
  __shared__ float4 sPos[MX_TILE];
  __shared__ float4 sPosLo[MX_TILE];
  __shared__ float4 sNrm[NRM ? MX_TILE : 1];
  __shared__ double sPosD[NRM ? 3 * MX_TILE : 1];  // FP64 box-centred source positions and normals (NRM)
  __shared__ double sNrmD[NRM ? 3 * MX_TILE : 1];
  __shared__ __align__(16) float sDen[MX_TILE * SD * KB];
  __shared__ int64_t eBeg[MX_MAXE];
  __shared__ int32_t ePre[MX_MAXE + 1];
  __shared__ double sRed[MX_THREADS * TD * KB];
  const int row = blockIdx.x;
  const int rhs0 = blockIdx.y * KB;
  const int g = rows[row];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const int64_t e0 = ptr[row], e1 = ptr[row + 1];
  const double cx = ctr[3 * g], cy = ctr[3 * g + 1], cz = ctr[3 * g + 2];
  const int tid = threadIdx.x;
  const int TG = mx_group<MX_THREADS>(tn);
  const int S = MX_THREADS / TG;
  const int tl = tid % TG, sp = tid / TG;
  for (int64_t t0 = 0; t0 < tn; t0 += TG) {
    const int64_t t = t0 + tl;
    const bool act = t < tn;
    float tx = 0, ty = 0, tz = 0, txl = 0, tyl = 0, tzl = 0;
    double tdx = 0, tdy = 0, tdz = 0;  // FP64 box-centred target (NRM)
    if (act) {
      const double dx = trg[3 * (tb + t)] - cx, dy = trg[3 * (tb + t) + 1] - cy, dz = trg[3 * (tb + t) + 2] - cz;
      tdx = dx;
      tdy = dy;
      tdz = dz;
      tx = (float)dx;
      ty = (float)dy;
      tz = (float)dz;
      txl = (float)(dx - tx);
      tyl = (float)(dy - ty);
      tzl = (float)(dz - tz);
    }
    double acc[TD * KB];
#pragma unroll
    for (int c = 0; c < TD * KB; c++) acc[c] = 0.0;
    for (int64_t ec = e0; ec < e1; ec += MX_MAXE) {
      const int ne = (int)min((int64_t)MX_MAXE, e1 - ec);
      const int total = load_entries(idx, ec, ne, 0, srcBeg, srcCnt, eBeg, ePre);
      for (int base = 0; base < total; base += MX_TILE) {
        const int cnt = min(MX_TILE, total - base);
        __syncthreads();
        for (int i = tid; i < cnt; i += MX_THREADS) {
          const int64_t s = entry_source(base + i, ne, eBeg, ePre);
          const double dx = src[3 * s] - cx, dy = src[3 * s + 1] - cy, dz = src[3 * s + 2] - cz;
          sPos[i] = make_float4((float)dx, (float)dy, (float)dz, 0.f);
          sPosLo[i] = make_float4((float)(dx - (float)dx), (float)(dy - (float)dy), (float)(dz - (float)dz), 0.f);
          if (NRM) {
            const double nx = nrm[3 * s], ny = nrm[3 * s + 1], nz = nrm[3 * s + 2];
            sNrm[i] = make_float4((float)nx, (float)ny, (float)nz, 0.f);
            sPosD[3 * i] = dx;
            sPosD[3 * i + 1] = dy;
            sPosD[3 * i + 2] = dz;
            sNrmD[3 * i] = nx;
            sNrmD[3 * i + 1] = ny;
            sNrmD[3 * i + 2] = nz;
          }
          // the block's KB x SD densities: contiguous in the FP32 copy (rows of
          // 8 right-hand sides per source, zeros past the last one)
          const float* ds = den32 + (rhs0 >> 3) * den32Blk + s * 8 * SD + (rhs0 & 7) * SD;
#pragma unroll
          for (int r = 0; r < KB * SD; r++) sDen[i * KB * SD + r] = ds[r];
        }
        __syncthreads();
        if (act) {
          float part[TD * KB];
#pragma unroll
          for (int c = 0; c < TD * KB; c++) part[c] = 0.f;
          for (int i = sp; i < cnt; i += S) {
            // offsets from hi/lo FP32 pairs of the box-centred coordinates:
            // the hi difference of close points is exact, so a near-coincident
            // pair keeps its separation to FP32 precision of the separation
            const float4 q = sPos[i], ql = sPosLo[i];
            const float ox = (tx - q.x) + (txl - ql.x), oy = (ty - q.y) + (tyl - ql.y), oz = (tz - q.z) + (tzl - ql.z);
            float nv[3] = {0.f, 0.f, 0.f};
            float rn = 0.f;
            if (NRM) {
              const float4 qn = sNrm[i];
              nv[0] = qn.x;
              nv[1] = qn.y;
              nv[2] = qn.z;
              rn = (float)((tdx - sPosD[3 * i]) * sNrmD[3 * i] + (tdy - sPosD[3 * i + 1]) * sNrmD[3 * i + 1] +
                           (tdz - sPosD[3 * i + 2]) * sNrmD[3 * i + 2]);
            }
            float d[KB * SD];
            mx_den<KB * SD>(&sDen[i * KB * SD], d);
            kaccum_multi<KT, KB, float, float>(ox, oy, oz, NRM ? nv : nullptr, d, part, mu, ve, NRM ? &rn : nullptr);
          }
#pragma unroll
          for (int c = 0; c < TD * KB; c++) acc[c] += (double)part[c];
        }
      }
    }
    reduce_store<TD, KB>(sRed, acc, tid, tl, sp, TG, S, act, val, tb + t, rhs0, nrhs, valStride);
  }
}

// Packed FP32x2 helpers of the Laplace near field below.
__device__ __forceinline__ unsigned long long nl_pk(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 nl_unpk(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ unsigned long long nl_add(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long nl_sub(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long nl_mul(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long nl_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// The Laplace single layer near field (the headline kernel): one warp per
// evaluator leaf (four leaves a CTA) and no CTA-wide barrier.  Each warp
// builds its own entry table (source leaves of the near list, prefix sums by
// warp shuffles) and stages its sources in chunks of NW_CH into its slice of
// shared memory; its lanes take two targets each and split each chunk's
// sources in 32 / TG strides.  The offsets, r^2 and 1/(4 pi r) of a source
// against both targets and the KB multiply-adds of its densities run as
// packed FP32x2 operations (half the instructions of a one-target loop), with
// the offsets from hi/lo pairs and the coincidence rule (r^2 < 1e-16 adds
// nothing) of k_p2p_near32; per-chunk FP32 partial sums go into FP64
// accumulators, which meet through warp shuffles at the end.  The leaves come
// in order[] (rows by decreasing targets x near sources), so the four warps of
// a CTA carry similar work and the longest leaves start first.  Six CTAs an SM
// (80 registers) measured faster than four without spills (1.73 vs 2.00 ms).
constexpr int NW_WARPS = 4, NW_CH = 64, NW_MAXE = 128;
template <int KB>
__global__ void __launch_bounds__(32 * NW_WARPS, 6)
    k_p2p_near32_lap2w(int nLeaves, const int32_t* __restrict__ order, const int32_t* __restrict__ rows,
                       const int64_t* __restrict__ ptr,
                       const int32_t* __restrict__ idx, const int64_t* __restrict__ srcBeg,
                       const int64_t* __restrict__ srcCnt, const int64_t* __restrict__ trgBeg,
                       const int64_t* __restrict__ trgCnt, const double* __restrict__ src,
                       const float* __restrict__ den32, int64_t den32Blk, const double* __restrict__ trg,
                       const double* __restrict__ ctr, double* __restrict__ val, int64_t valStride, int nrhs) {
  __shared__ float4 sPos[NW_WARPS][NW_CH];
  __shared__ float4 sPosLo[NW_WARPS][NW_CH];
  __shared__ __align__(16) float sDen[NW_WARPS][NW_CH * KB];
  __shared__ int64_t eBeg[NW_WARPS][NW_MAXE];
  __shared__ int32_t ePre[NW_WARPS][NW_MAXE + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (blockIdx.x * NW_WARPS + warp >= nLeaves) return;
  const int row = order[blockIdx.x * NW_WARPS + warp];
  const int rhs0 = blockIdx.y * KB;
  const int g = rows[row];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const int64_t e0 = ptr[row], e1 = ptr[row + 1];
  const double cx = ctr[3 * g], cy = ctr[3 * g + 1], cz = ctr[3 * g + 2];
  const int64_t pairs = (tn + 1) / 2;
  const int TG = pairs > 16 ? 32 : (pairs > 8 ? 16 : 8), S = 32 / TG;
  const int tl = lane % TG, sp = lane / TG;
  const float c4pi = (float)(1.0 / (4.0 * 3.14159265358979323846));
  for (int64_t t0 = 0; t0 < tn; t0 += 2 * TG) {
    const int64_t ta = t0 + tl, tbb = t0 + tl + TG;
    const bool actA = ta < tn, actB = tbb < tn;
    unsigned long long txh = 0, tyh = 0, tzh = 0, txl = 0, tyl = 0, tzl = 0;
    {
      float h[2][3] = {{0, 0, 0}, {0, 0, 0}}, l[2][3] = {{0, 0, 0}, {0, 0, 0}};
      for (int q = 0; q < 2; q++) {
        const int64_t t = q ? tbb : ta;
        if (!(q ? actB : actA)) continue;
        const double d[3] = {trg[3 * (tb + t)] - cx, trg[3 * (tb + t) + 1] - cy, trg[3 * (tb + t) + 2] - cz};
        for (int c = 0; c < 3; c++) {
          h[q][c] = (float)d[c];
          l[q][c] = (float)(d[c] - h[q][c]);
        }
      }
      txh = nl_pk(h[0][0], h[1][0]);
      tyh = nl_pk(h[0][1], h[1][1]);
      tzh = nl_pk(h[0][2], h[1][2]);
      txl = nl_pk(l[0][0], l[1][0]);
      tyl = nl_pk(l[0][1], l[1][1]);
      tzl = nl_pk(l[0][2], l[1][2]);
    }
    double acc[2][KB];
#pragma unroll
    for (int r = 0; r < KB; r++) acc[0][r] = acc[1][r] = 0.0;
    for (int64_t ec = e0; ec < e1; ec += NW_MAXE) {
      const int ne = (int)min((int64_t)NW_MAXE, e1 - ec);
      __syncwarp();
      int running = 0;  // the warp's entry table: starts and prefix counts
      for (int eb = 0; eb < ne; eb += 32) {
        const int e = eb + lane;
        int c = 0;
        if (e < ne) {
          const int s2 = idx[ec + e];
          eBeg[warp][e] = srcBeg[s2];
          c = (int)srcCnt[s2];
        }
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        if (e < ne) ePre[warp][e + 1] = running + incl;
        running += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) ePre[warp][0] = 0;
      __syncwarp();
      const int total = running;
      for (int base = 0; base < total; base += NW_CH) {
        const int cnt = min(NW_CH, total - base);
        __syncwarp();
        for (int i = lane; i < cnt; i += 32) {
          const int64_t s2 = entry_source(base + i, ne, eBeg[warp], ePre[warp]);
          const double dx = src[3 * s2] - cx, dy = src[3 * s2 + 1] - cy, dz = src[3 * s2 + 2] - cz;
          sPos[warp][i] = make_float4((float)dx, (float)dy, (float)dz, 0.f);
          sPosLo[warp][i] = make_float4((float)(dx - (float)dx), (float)(dy - (float)dy), (float)(dz - (float)dz), 0.f);
          const float* ds = den32 + (rhs0 >> 3) * den32Blk + s2 * 8 + (rhs0 & 7);
          if constexpr (KB % 4 == 0) {
#pragma unroll
            for (int r = 0; r < KB; r += 4)
              *reinterpret_cast<float4*>(&sDen[warp][i * KB + r]) = *reinterpret_cast<const float4*>(ds + r);
          } else {
#pragma unroll
            for (int r = 0; r < KB; r++) sDen[warp][i * KB + r] = ds[r];
          }
        }
        __syncwarp();
        if (actA) {
          unsigned long long part[KB];  // (target A, target B) for each right-hand side
#pragma unroll
          for (int r = 0; r < KB; r++) part[r] = 0ull;
          for (int i = sp; i < cnt; i += S) {
            const float4 q = sPos[warp][i], ql = sPosLo[warp][i];
            const unsigned long long ox = nl_add(nl_sub(txh, nl_pk(q.x, q.x)), nl_sub(txl, nl_pk(ql.x, ql.x)));
            const unsigned long long oy = nl_add(nl_sub(tyh, nl_pk(q.y, q.y)), nl_sub(tyl, nl_pk(ql.y, ql.y)));
            const unsigned long long oz = nl_add(nl_sub(tzh, nl_pk(q.z, q.z)), nl_sub(tzl, nl_pk(ql.z, ql.z)));
            const float2 r2 = nl_unpk(nl_fma(oz, oz, nl_fma(oy, oy, nl_mul(ox, ox))));
            const float ka = r2.x < 1e-16f ? 0.f : c4pi * rsqrtf(r2.x);
            const float kb = r2.y < 1e-16f ? 0.f : c4pi * rsqrtf(r2.y);
            const unsigned long long k2 = nl_pk(ka, kb);
            float d[KB];
            mx_den<KB>(&sDen[warp][i * KB], d);
#pragma unroll
            for (int r = 0; r < KB; r++) part[r] = nl_fma(k2, nl_pk(d[r], d[r]), part[r]);
          }
#pragma unroll
          for (int r = 0; r < KB; r++) {
            const float2 v = nl_unpk(part[r]);
            acc[0][r] += (double)v.x;
            acc[1][r] += (double)v.y;
          }
        }
      }
    }
    if (S > 1) {
#pragma unroll
      for (int r = 0; r < KB; r++)
        for (int o = TG; o < 32; o <<= 1) {
          acc[0][r] += __shfl_xor_sync(0xffffffffu, acc[0][r], o);
          acc[1][r] += __shfl_xor_sync(0xffffffffu, acc[1][r], o);
        }
    }
    if (sp == 0) {
#pragma unroll
      for (int r = 0; r < KB; r++) {
        if (rhs0 + r >= nrhs) break;
        if (actA) val[(int64_t)(rhs0 + r) * valStride + tb + ta] += acc[0][r];
        if (actB) val[(int64_t)(rhs0 + r) * valStride + tb + tbb] += acc[1][r];
      }
    }
  }
}

// equivalent surfaces -> targets: L2T (own DE surface, downward density) and
// M2T (UE surfaces of the W nodes, upward densities), equivalent kernel
template <int KM, int KB, int THREADS>
__global__ void __launch_bounds__(THREADS)
    k_e2t32(const int32_t* __restrict__ rows, const int64_t* __restrict__ farPtr, const int32_t* __restrict__ farIdx,
            int useOwn, int useFar, const int32_t* __restrict__ depth, const double* __restrict__ ctr,
            const double* __restrict__ rad, const double* __restrict__ samUE, int nUE,
            const double* __restrict__ samDE, int nDE, const float* __restrict__ uden,
            const float* __restrict__ dden, int64_t rhsStrideU, int64_t rhsStrideD,
            const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt, const double* __restrict__ trg,
            double* __restrict__ val, int64_t valStride, int nrhs, float mu, float ve, int gmin,
            const int4* __restrict__ items, double* __restrict__ partial, int64_t partStride) {
  constexpr int SD = KTraits<KM>::SD, TD = KTraits<KM>::TD;
  // scalar kernels: a whole equivalent surface (up to 256 points: np <= 7)
  // a tile, so each node takes one staging round and two barriers
  constexpr int TILE = SD * KB <= 8 ? 256 : MX_TILE;
  __shared__ float4 sPos[TILE];
  __shared__ __align__(16) float sDen[TILE * SD * KB];
  __shared__ double sRed[THREADS * TD * KB];
  // with work items (M2T): item = (row, first far entry, end far entry,
  // partial-sum base); base >= 0 stores the sums in partial[rhs][base + t]
  // (a row split in several items, combined by k_e2t_combine), else they
  // are added to the targets' values
  const int4 it = items ? items[blockIdx.x] : make_int4(blockIdx.x, 0, 0, -1);
  const int row = it.x;
  const int rhs0 = blockIdx.y * KB;
  const int g = rows[row];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const double gx = ctr[3 * g], gy = ctr[3 * g + 1], gz = ctr[3 * g + 2];
  const int tid = threadIdx.x;
  const int TG = mx_group<THREADS>(tn, gmin);
  const int S = THREADS / TG;
  const int tl = tid % TG, sp = tid / TG;
  const int own = (useOwn && depth[g] >= 2) ? 1 : 0;
  const int64_t f0 = !useFar ? 0 : items ? it.y : farPtr[row];
  const int64_t nf = !useFar ? 0 : items ? it.z - it.y : farPtr[row + 1] - f0;
  const bool toPart = it.w >= 0;
  for (int64_t t0 = 0; t0 < tn; t0 += TG) {
    const int64_t t = t0 + tl;
    const bool act = t < tn;
    float tx = 0, ty = 0, tz = 0;
    if (act) {
      tx = (float)(trg[3 * (tb + t)] - gx);
      ty = (float)(trg[3 * (tb + t) + 1] - gy);
      tz = (float)(trg[3 * (tb + t) + 2] - gz);
    }
    double acc[TD * KB];
#pragma unroll
    for (int c = 0; c < TD * KB; c++) acc[c] = 0.0;
    for (int64_t e = 0; e < own + nf; e++) {
      const bool isOwn = e < own;
      const int node = isOwn ? g : farIdx[f0 + e - own];
      const double* sam = isOwn ? samDE : samUE;
      const int ns = isOwn ? nDE : nUE;
      const float* dsrc = isOwn ? dden + (int64_t)node * ns * SD : uden + (int64_t)node * ns * SD;
      const int64_t rstr = isOwn ? rhsStrideD : rhsStrideU;
      const double ox = ctr[3 * node] - gx, oy = ctr[3 * node + 1] - gy, oz = ctr[3 * node + 2] - gz;
      const double r = rad[node];
      for (int base = 0; base < ns; base += TILE) {
        const int cnt = min(TILE, ns - base);
        __syncthreads();
        for (int i = tid; i < cnt; i += THREADS) {
          const int j = base + i;
          sPos[i] = make_float4((float)(ox + r * sam[3 * j]), (float)(oy + r * sam[3 * j + 1]),
                                (float)(oz + r * sam[3 * j + 2]), 0.f);
#pragma unroll
          for (int q = 0; q < KB; q++)
#pragma unroll
            for (int c = 0; c < SD; c++)
              sDen[(i * KB + q) * SD + c] = rhs0 + q < nrhs ? dsrc[(rhs0 + q) * rstr + (int64_t)j * SD + c] : 0.f;
        }
        __syncthreads();
        if (act) {
          float part[TD * KB];
#pragma unroll
          for (int c = 0; c < TD * KB; c++) part[c] = 0.f;
          for (int i = sp; i < cnt; i += S) {
            const float4 q = sPos[i];
            float d[KB * SD];
            mx_den<KB * SD>(&sDen[i * KB * SD], d);
            kaccum_multi<KM, KB, float, float>(tx - q.x, ty - q.y, tz - q.z, nullptr, d, part, mu, ve);
          }
#pragma unroll
          for (int c = 0; c < TD * KB; c++) acc[c] += (double)part[c];
        }
      }
    }
    if (toPart)
      reduce_store<TD, KB>(sRed, acc, tid, tl, sp, TG, S, act, partial, it.w + t, rhs0, nrhs, partStride, true);
    else
      reduce_store<TD, KB>(sRed, acc, tid, tl, sp, TG, S, act, val, tb + t, rhs0, nrhs, valStride);
  }
}

// L2T, one warp per leaf (four leaves a CTA): the leaf's downward
// equivalent densities (KB right-hand sides) are staged in the warp's slice of
// shared memory, the DE surface (scaled per leaf) is shared by the CTA, and
// the lanes split as TG targets x (32 / TG) source strides whose partial sums
// meet through warp shuffles -- no CTA-wide barriers after the staging of the
// surface, so the four leaves run independently.  The leaves come from the
// list of leaves at depth >= 2.  Dynamic shared memory
// nDE * 16 + 4 * nDE * KB * SD * 4 bytes.
constexpr int L2T_WARPS = 4;
template <int KM, int KB>
__global__ void __launch_bounds__(32 * L2T_WARPS)
    k_l2t32w(int nLeaves, const int32_t* __restrict__ leaves, const double* __restrict__ ctr,
             const double* __restrict__ rad, const double* __restrict__ samDE, int nDE, const float* __restrict__ dden,
             int64_t rhsStride, const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt,
             const double* __restrict__ trg, double* __restrict__ val, int64_t valStride, int nrhs, float mu,
             float ve) {
  constexpr int SD = KTraits<KM>::SD, TD = KTraits<KM>::TD;
  extern __shared__ __align__(16) unsigned char l2t_smem[];
  float4* sSam = reinterpret_cast<float4*>(l2t_smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* sDen = reinterpret_cast<float*>(sSam + nDE) + (size_t)warp * nDE * KB * SD;
  for (int j = threadIdx.x; j < nDE; j += blockDim.x)
    sSam[j] = make_float4((float)samDE[3 * j], (float)samDE[3 * j + 1], (float)samDE[3 * j + 2], 0.f);
  __syncthreads();
  const int li = blockIdx.x * L2T_WARPS + warp;
  if (li >= nLeaves) return;
  const int g = leaves[li];
  const int rhs0 = blockIdx.y * KB;
  const float* dsrc = dden + (int64_t)g * nDE * SD;
  if (SD == 1 && KB == 8 && nDE % 4 == 0 && rhsStride % 4 == 0 && (reinterpret_cast<uintptr_t>(dsrc) & 15) == 0) {
    // lane = (right-hand side q, run of 4 points v): a warp load reads 64
    // contiguous bytes of each of the 8 right-hand sides (whole sectors),
    // and the stores of one point meet 4-way at most in a bank
    const int q = lane & 7;
    for (int v = lane >> 3; v < nDE / 4; v += 4) {
      const float4 x = rhs0 + q < nrhs
                           ? *reinterpret_cast<const float4*>(dsrc + (int64_t)(rhs0 + q) * rhsStride + 4 * v)
                           : make_float4(0.f, 0.f, 0.f, 0.f);
      sDen[(4 * v) * KB + q] = x.x;
      sDen[(4 * v + 1) * KB + q] = x.y;
      sDen[(4 * v + 2) * KB + q] = x.z;
      sDen[(4 * v + 3) * KB + q] = x.w;
    }
  } else {
    for (int i = lane; i < nDE * KB; i += 32) {
      const int j = i % nDE, q = i / nDE;
#pragma unroll
      for (int c = 0; c < SD; c++)
        sDen[(j * KB + q) * SD + c] =
            rhs0 + q < nrhs ? dsrc[(int64_t)(rhs0 + q) * rhsStride + (int64_t)j * SD + c] : 0.f;
    }
  }
  __syncwarp();
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const double gx = ctr[3 * g], gy = ctr[3 * g + 1], gz = ctr[3 * g + 2];
  const float r = (float)rad[g];
  const int TG = tn > 16 ? 32 : (tn > 8 ? 16 : 8), S = 32 / TG;
  const int tl = lane % TG, sp = lane / TG;
  for (int64_t t0 = 0; t0 < tn; t0 += TG) {
    const int64_t t = t0 + tl;
    const bool act = t < tn;
    float tx = 0, ty = 0, tz = 0;
    if (act) {
      tx = (float)(trg[3 * (tb + t)] - gx);
      ty = (float)(trg[3 * (tb + t) + 1] - gy);
      tz = (float)(trg[3 * (tb + t) + 2] - gz);
    }
    float part[TD * KB];
#pragma unroll
    for (int c = 0; c < TD * KB; c++) part[c] = 0.f;
    if (act) {
      for (int j = sp; j < nDE; j += S) {
        const float4 q = sSam[j];
        float d[KB * SD];
        mx_den<KB * SD>(&sDen[j * KB * SD], d);
        kaccum_multi<KM, KB, float, float>(tx - r * q.x, ty - r * q.y, tz - r * q.z, nullptr, d, part, mu, ve);
      }
    }
#pragma unroll
    for (int c = 0; c < TD * KB; c++)
      for (int o = TG; o < 32; o <<= 1) part[c] += __shfl_xor_sync(0xffffffffu, part[c], o);
    if (act && sp == 0) {
#pragma unroll
      for (int q = 0; q < KB; q++) {
        if (rhs0 + q >= nrhs) break;
#pragma unroll
        for (int c = 0; c < TD; c++) val[(int64_t)(rhs0 + q) * valStride + (tb + t) * TD + c] += (double)part[q * TD + c];
      }
    }
  }
}

// The rows split into several M2T items: per split row (a run of items with
// consecutive partial bases, the first base in splitBase[i], splitCnt[i]
// items of tn targets each) the partial sums are added in item order, then
// to the targets' values -- the same order on every run.  One thread per
// (target component, right-hand side).
__global__ void k_e2t_combine(int nSplit, const int32_t* __restrict__ splitLeaf,
                              const int32_t* __restrict__ splitBase, const int32_t* __restrict__ splitCnt,
                              const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt, int td,
                              const double* __restrict__ partial, int64_t partStride, double* __restrict__ val,
                              int64_t valStride, int nrhs) {
  const int i = blockIdx.x;
  if (i >= nSplit) return;
  const int g = splitLeaf[i];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const int base = splitBase[i], cnt = splitCnt[i];
  for (int64_t q = threadIdx.x; q < tn * td * nrhs; q += blockDim.x) {
    const int r = (int)(q / (tn * td));
    const int64_t tc = q % (tn * td);
    double s = 0.0;
    for (int c = 0; c < cnt; c++) s += partial[(int64_t)r * partStride + (base + c * tn) * td + tc];
    val[(int64_t)r * valStride + tb * td + tc] += s;
  }
}

// point sources -> check surface of a box (S2M onto UC, S2L onto DC), FP32
// out.  One thread per surface point: a CTA of mx_surf_threads(nSurf) (the
// surface rounded up to whole warps, at most 512 points: np <= 8).  With no
// entry list (ptr == nullptr) the sources are the box's own, one contiguous
// run, and need no prefix table.  assign: store the sums (S2M, the only
// writer of a leaf's check surface) instead of adding them (S2L).
constexpr int MX_SURF = 512;
static inline int mx_surf_threads(int nSurf) { return std::min(MX_SURF, (nSurf + 31) / 32 * 32); }
template <int KT, int KB>
__global__ void __launch_bounds__(MX_SURF)
    k_src2surf32(const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                 const int64_t* __restrict__ srcBeg, const int64_t* __restrict__ srcCnt,
                 const double* __restrict__ src, const double* __restrict__ nrm, const float* __restrict__ den32,
                 int64_t den32Blk, const double* __restrict__ ctr, const double* __restrict__ rad,
                 const double* __restrict__ sam, int nSurf, float* __restrict__ out, int64_t ldo,
                 int64_t outRhsStride, int nrhs, float mu, float ve, int assign) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  __shared__ float4 sPos[MX_TILE];
  __shared__ float4 sNrm[NRM ? MX_TILE : 1];
  __shared__ __align__(16) float sDen[MX_TILE * SD * KB];
  __shared__ int64_t eBeg[MX_MAXE];
  __shared__ int32_t ePre[MX_MAXE + 1];
  const int row = blockIdx.x;
  const int rhs0 = blockIdx.y * KB;
  const int g = rows[row];
  const int tid = threadIdx.x;
  const double cx = ctr[3 * g], cy = ctr[3 * g + 1], cz = ctr[3 * g + 2], r = rad[g];
  const bool act = tid < nSurf;
  const float px = act ? (float)(r * sam[3 * tid]) : 0.f;
  const float py = act ? (float)(r * sam[3 * tid + 1]) : 0.f;
  const float pz = act ? (float)(r * sam[3 * tid + 2]) : 0.f;
  float acc[TD * KB];  // the check surface is FP32: one FP32 sum over all tiles
#pragma unroll
  for (int c = 0; c < TD * KB; c++) acc[c] = 0.f;
  const int64_t e0 = ptr ? ptr[row] : 0, e1 = ptr ? ptr[row + 1] : 1;
  for (int64_t ec = e0; ec < e1; ec += MX_MAXE) {
    const int ne = (int)min((int64_t)MX_MAXE, e1 - ec);
    int total;
    if (ptr) {
      total = load_entries(idx, ec, ne, g, srcBeg, srcCnt, eBeg, ePre);
    } else {
      __syncthreads();
      if (tid == 0) {
        eBeg[0] = srcBeg[g];
        ePre[0] = 0;
        ePre[1] = (int32_t)srcCnt[g];
      }
      __syncthreads();
      total = ePre[1];
    }
    for (int base = 0; base < total; base += MX_TILE) {
      const int cnt = min(MX_TILE, total - base);
      __syncthreads();
      for (int i = tid; i < cnt; i += blockDim.x) {
        const int64_t s = entry_source(base + i, ne, eBeg, ePre);
        sPos[i] = make_float4((float)(src[3 * s] - cx), (float)(src[3 * s + 1] - cy), (float)(src[3 * s + 2] - cz),
                              0.f);
        if (NRM) sNrm[i] = make_float4((float)nrm[3 * s], (float)nrm[3 * s + 1], (float)nrm[3 * s + 2], 0.f);
        const float* ds = den32 + (rhs0 >> 3) * den32Blk + s * 8 * SD + (rhs0 & 7) * SD;
#pragma unroll
        for (int q = 0; q < KB * SD; q++) sDen[i * KB * SD + q] = ds[q];
      }
      __syncthreads();
      if (act) {
        for (int i = 0; i < cnt; i++) {
          const float4 q = sPos[i];
          float nv[3] = {0.f, 0.f, 0.f};
          if (NRM) {
            const float4 qn = sNrm[i];
            nv[0] = qn.x;
            nv[1] = qn.y;
            nv[2] = qn.z;
          }
          float d[KB * SD];
          mx_den<KB * SD>(&sDen[i * KB * SD], d);
          kaccum_multi<KT, KB, float, float>(px - q.x, py - q.y, pz - q.z, NRM ? nv : nullptr, d, acc, mu, ve);
        }
      }
    }
  }
  if (act)
#pragma unroll
    for (int q = 0; q < KB; q++) {
      if (rhs0 + q >= nrhs) break;
#pragma unroll
      for (int c = 0; c < TD; c++) {
        float* o = &out[(rhs0 + q) * outRhsStride + (int64_t)g * ldo + (int64_t)tid * TD + c];
        *o = assign ? acc[q * TD + c] : *o + acc[q * TD + c];
      }
    }
}

// S2M (a leaf's own sources onto its UC check surface), one warp per leaf
// and S2M_WARPS leaves a CTA: the warp stages up to S2M_CH of the leaf's
// sources (positions, normals, the KB x SD FP32 densities) in its slice of
// shared memory, its lanes own the surface points j = lane + 32 m and sum the
// staged sources in order into FP32 -- for leaves of up to S2M_CH sources the
// same sums as k_src2surf32, without CTA-wide barriers.  Later chunks of a
// larger leaf add to the stored sums.
constexpr int S2M_WARPS = 4, S2M_CH = 64;
template <int KT, int KB>
__global__ void __launch_bounds__(32 * S2M_WARPS)
    k_s2m32w(int nLeaves, const int32_t* __restrict__ leaves, const int64_t* __restrict__ srcBeg,
             const int64_t* __restrict__ srcCnt, const double* __restrict__ src, const double* __restrict__ nrm,
             const float* __restrict__ den32, int64_t den32Blk, const double* __restrict__ ctr,
             const double* __restrict__ rad, const double* __restrict__ sam, int nSurf, float* __restrict__ out,
             int64_t ldo, int64_t outRhsStride, int nrhs, float mu, float ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  __shared__ float4 sPos[S2M_WARPS][S2M_CH];
  __shared__ float4 sNrm[S2M_WARPS][NRM ? S2M_CH : 1];
  __shared__ __align__(16) float sDen[S2M_WARPS][S2M_CH * KB * SD];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li = blockIdx.x * S2M_WARPS + warp;
  if (li >= nLeaves) return;
  const int g = leaves[li];
  const int rhs0 = blockIdx.y * KB;
  const int64_t sb = srcBeg[g], sn = srcCnt[g];
  const double cx = ctr[3 * g], cy = ctr[3 * g + 1], cz = ctr[3 * g + 2], r = rad[g];
  for (int64_t c0 = 0; c0 < sn; c0 += S2M_CH) {
    const int cnt = (int)min((int64_t)S2M_CH, sn - c0);
    __syncwarp();
    for (int i = lane; i < cnt; i += 32) {
      const int64_t s = sb + c0 + i;
      sPos[warp][i] = make_float4((float)(src[3 * s] - cx), (float)(src[3 * s + 1] - cy),
                                  (float)(src[3 * s + 2] - cz), 0.f);
      if (NRM) sNrm[warp][i] = make_float4((float)nrm[3 * s], (float)nrm[3 * s + 1], (float)nrm[3 * s + 2], 0.f);
      const float* ds = den32 + (rhs0 >> 3) * den32Blk + s * 8 * SD + (rhs0 & 7) * SD;
#pragma unroll
      for (int q = 0; q < KB * SD; q++) sDen[warp][i * KB * SD + q] = ds[q];
    }
    __syncwarp();
    for (int j = lane; j < nSurf; j += 32) {
      const float px = (float)(r * sam[3 * j]), py = (float)(r * sam[3 * j + 1]), pz = (float)(r * sam[3 * j + 2]);
      float acc[TD * KB];
#pragma unroll
      for (int c = 0; c < TD * KB; c++) acc[c] = 0.f;
      for (int i = 0; i < cnt; i++) {
        const float4 q = sPos[warp][i];
        float nv[3] = {0.f, 0.f, 0.f};
        if (NRM) {
          const float4 qn = sNrm[warp][i];
          nv[0] = qn.x;
          nv[1] = qn.y;
          nv[2] = qn.z;
        }
        float d[KB * SD];
        mx_den<KB * SD>(&sDen[warp][i * KB * SD], d);
        kaccum_multi<KT, KB, float, float>(px - q.x, py - q.y, pz - q.z, NRM ? nv : nullptr, d, acc, mu, ve);
      }
#pragma unroll
      for (int q = 0; q < KB; q++) {
        if (rhs0 + q >= nrhs) break;
#pragma unroll
        for (int c = 0; c < TD; c++) {
          float* o = &out[(rhs0 + q) * outRhsStride + (int64_t)g * ldo + (int64_t)j * TD + c];
          *o = c0 == 0 ? acc[q * TD + c] : *o + acc[q * TD + c];
        }
      }
    }
  }
}

// s += a b and s += a conj(b) as four FMAs into the accumulator (a product
// formed first and then added costs a multiply and an add more: IEEE rules
// keep the compiler from reassociating it)
__device__ __forceinline__ void r8_cmac(float2& s, float2 a, float2 b) {
  s.x = fmaf(a.x, b.x, s.x);
  s.x = fmaf(-a.y, b.y, s.x);
  s.y = fmaf(a.x, b.y, s.y);
  s.y = fmaf(a.y, b.x, s.y);
}
__device__ __forceinline__ void r8_cmacc(float2& s, float2 a, float2 b) {
  s.x = fmaf(a.x, b.x, s.x);
  s.x = fmaf(a.y, b.y, s.x);
  s.y = fmaf(a.y, b.x, s.y);
  s.y = fmaf(-a.x, b.y, s.y);
}

// ------------------------------------------------------------------ FP32 M2L
// grid (source slots, right-hand sides)
template <int NP>
__global__ void __launch_bounds__(128)
    k_m2l_fwd32(const int32_t* __restrict__ nodes, const int32_t* __restrict__ depth, int rootLevel, Scale4 deg,
                int sdm, const float* __restrict__ uden, int64_t udenRhs, const int32_t* __restrict__ ijk, int nUE,
                float2* __restrict__ effDen, int64_t effRhs, int nEff) {
  using F = FftDims32<NP>;
  constexpr int N = F::N, NH = F::NH, H = F::H;
  __shared__ float cube[NP * NP * NP];
  __shared__ float2 X1[NP * NP * NH];
  __shared__ float2 X2[NP * N * NH];
  __shared__ float2 tw[N];
  const int slot = blockIdx.x;
  const int v = nodes[slot];
  const int tid = threadIdx.x;
  if (tid < N) {
    double s, c;
    sincospi(2.0 * tid / N, &s, &c);
    tw[tid] = make_float2((float)c, (float)-s);
  }
  const int l = depth[v] + rootLevel;
  const float* ud = uden + blockIdx.y * udenRhs + (int64_t)v * nUE * sdm;
  float2* out = effDen + blockIdx.y * effRhs + (int64_t)slot * nEff * sdm;
  for (int m = 0; m < sdm; m++) {
    const float scl = (float)exp2(l * deg.v[m]);
    for (int i = tid; i < NP * NP * NP; i += blockDim.x) cube[i] = 0.f;
    __syncthreads();
    for (int i = tid; i < nUE; i += blockDim.x) {
      int p = ijk[i];
      cube[((p >> 16) * NP + ((p >> 8) & 255)) * NP + (p & 255)] = ud[(int64_t)i * sdm + m] * scl;
    }
    __syncthreads();
    for (int e = tid; e < NP * NP * NH; e += blockDim.x) {
      int kx = e % NH, yb = (e / NH) % NP, zb = e / (NH * NP);
      float2 s = make_float2(0.f, 0.f);
      const float* row = &cube[(zb * NP + yb) * NP];
#pragma unroll
      for (int xb = 0; xb < NP; xb++) {
        float2 w = tw[(kx * (xb + H)) % N];
        s.x += row[xb] * w.x;
        s.y += row[xb] * w.y;
      }
      X1[e] = s;
    }
    __syncthreads();
    for (int e = tid; e < NP * N * NH; e += blockDim.x) {
      int kx = e % NH, ky = (e / NH) % N, zb = e / (NH * N);
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int yb = 0; yb < NP; yb++) {
        r8_cmac(s, X1[(zb * NP + yb) * NH + kx], tw[(ky * (yb + H)) % N]);
      }
      X2[e] = s;
    }
    __syncthreads();
    for (int e = tid; e < N * N * NH; e += blockDim.x) {
      int kx = e % NH, ky = (e / NH) % N, kz = e / (NH * N);
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int zb = 0; zb < NP; zb++) {
        r8_cmac(s, X2[(zb * N + ky) * NH + kx], tw[(kz * (zb + H)) % N]);
      }
      out[(int64_t)e * sdm + m] = s;
    }
    __syncthreads();
  }
}

// grid (target parents, 32-frequency chunks, RHS blocks); warp c owns child c;
// each translation spectrum value is loaded once and applied to KB densities.
// The parent's neighbour entries (the 8 input child slots resolved at setup,
// the offset code) are staged in shared memory once for the CTA, 32 at a
// time, so each (neighbour, child) pair starts on shared-memory reads instead
// of a chain of dependent global loads (neighbour -> its children -> slot).
template <int SDM, int TDM, int KB>
__global__ void __launch_bounds__(256)
    k_m2l_had32(const int32_t* __restrict__ rowOut, const int64_t* __restrict__ vPtr,
                const int8_t* __restrict__ vOff, const int32_t* __restrict__ nIn,
                const float2* __restrict__ effDen, int64_t denRhs, const float2* __restrict__ T,
                float2* __restrict__ effVal, int64_t valRhs, int nEff, int nrhs, float nrmfc) {
  __shared__ int sSl[32 * 8];
  __shared__ int sOf[32];
  const int b = blockIdx.x;
  const int c = threadIdx.x >> 5;
  const int f = blockIdx.y * 32 + (threadIdx.x & 31);
  const int rhs0 = blockIdx.z * KB;
  const int ts = rowOut[8 * b + c];
  const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
  float2 acc[KB][TDM];
#pragma unroll
  for (int q = 0; q < KB; q++)
#pragma unroll
    for (int i = 0; i < TDM; i++) acc[q][i] = make_float2(0.f, 0.f);
  const bool live = ts >= 0 && f < nEff;  // every thread stays for the CTA's barriers
  const int64_t e1 = vPtr[b + 1];
  for (int64_t e0 = vPtr[b]; e0 < e1; e0 += 32) {
    const int ne = (int)min((int64_t)32, e1 - e0);
    __syncthreads();
    for (int i = threadIdx.x; i < ne * 8; i += blockDim.x) sSl[i] = nIn[8 * e0 + i];
    if (threadIdx.x < ne) sOf[threadIdx.x] = vOff[e0 + threadIdx.x];
    __syncthreads();
    if (!live) continue;
    for (int j = 0; j < ne; j++) {
      const int off = sOf[j];
      const int dx = off / 9 - 1, dy = (off / 3) % 3 - 1, dz = off % 3 - 1;
#pragma unroll 1
      for (int c2 = 0; c2 < 8; c2++) {
        const int s = sSl[j * 8 + c2];
        if (s < 0) continue;
        const int rx = 2 * dx + (c2 >> 2) - cx, ry = 2 * dy + ((c2 >> 1) & 1) - cy, rz = 2 * dz + (c2 & 1) - cz;
        if (max(abs(rx), max(abs(ry), abs(rz))) <= 1) continue;
        const int id = c_transId32[(rx + 3) * 49 + (ry + 3) * 7 + (rz + 3)];
        const float2* Tf = T + ((int64_t)id * nEff + f) * (SDM * TDM);
        float2 tv[SDM * TDM];
#pragma unroll
        for (int jj = 0; jj < SDM * TDM; jj++) tv[jj] = Tf[jj];
#pragma unroll
        for (int q = 0; q < KB; q++) {
          if (rhs0 + q >= nrhs) break;
          const float2* dp = effDen + (rhs0 + q) * denRhs + ((int64_t)s * nEff + f) * SDM;
#pragma unroll
          for (int jj = 0; jj < SDM; jj++) {
            const float2 d = dp[jj];
#pragma unroll
            for (int i = 0; i < TDM; i++) {
              const float2 w = tv[jj * TDM + i];
              acc[q][i].x += w.x * d.x - w.y * d.y;
              acc[q][i].y += w.x * d.y + w.y * d.x;
            }
          }
        }
      }
    }
  }
  if (live) {
#pragma unroll
    for (int q = 0; q < KB; q++) {
      if (rhs0 + q >= nrhs) break;
#pragma unroll
      for (int i = 0; i < TDM; i++)
        effVal[(rhs0 + q) * valRhs + ((int64_t)ts * nEff + f) * TDM + i] =
            make_float2(acc[q][i].x * nrmfc, acc[q][i].y * nrmfc);
    }
  }
}

// grid (target slots, right-hand sides)
template <int NP>
__global__ void __launch_bounds__(128)
    k_m2l_inv32(const int32_t* __restrict__ nodes, const float2* __restrict__ effVal, int64_t valRhs, int nEff,
                int tdm, const int32_t* __restrict__ ijk, int nDC, float* __restrict__ dchk, int64_t dchkRhs) {
  using F = FftDims32<NP>;
  constexpr int N = F::N, NH = F::NH, H = F::H;
  __shared__ float2 Y2[NP * N * NH];
  __shared__ float2 Y1[NP * NP * NH];
  __shared__ float2 tw[N];
  const int slot = blockIdx.x;
  const int node = nodes[slot];
  const int tid = threadIdx.x;
  if (tid < N) {
    double s, c;
    sincospi(2.0 * tid / N, &s, &c);
    tw[tid] = make_float2((float)c, (float)-s);
  }
  __syncthreads();
  const float2* in = effVal + blockIdx.y * valRhs + (int64_t)slot * nEff * tdm;
  float* dc = dchk + blockIdx.y * dchkRhs + (int64_t)node * nDC * tdm;
  for (int m = 0; m < tdm; m++) {
    for (int e = tid; e < NP * N * NH; e += blockDim.x) {
      int kx = e % NH, ky = (e / NH) % N, zb = e / (NH * N);
      float2 s = make_float2(0.f, 0.f);
#pragma unroll 4
      for (int kz = 0; kz < N; kz++) {
        r8_cmacc(s, in[((int64_t)(kz * N + ky) * NH + kx) * tdm + m], tw[(kz * (zb + H)) % N]);
      }
      Y2[e] = s;
    }
    __syncthreads();
    for (int e = tid; e < NP * NP * NH; e += blockDim.x) {
      int kx = e % NH, yb = (e / NH) % NP, zb = e / (NH * NP);
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int ky = 0; ky < N; ky++) {
        r8_cmacc(s, Y2[(zb * N + ky) * NH + kx], tw[(ky * (yb + H)) % N]);
      }
      Y1[e] = s;
    }
    __syncthreads();
    for (int i = tid; i < nDC; i += blockDim.x) {
      int p = ijk[i];
      int a = p & 255, b = (p >> 8) & 255, cc = p >> 16;
      const float2* y1 = &Y1[(cc * NP + b) * NH];
      const int x = a + H;
      float s = 0.f;
#pragma unroll
      for (int kx = 0; kx < NH; kx++) {
        float2 t = cmulc(y1[kx], tw[(kx * x) % N]);
        s += (kx == 0 || 2 * kx == N) ? t.x : 2.f * t.x;  // the Nyquist term only for even N
      }
      dc[(int64_t)i * tdm + m] += s;
    }
    __syncthreads();
  }
}

// Scalar equivalent kernels, blocks of 8 right-hand sides: one CTA per
// (slot, block) transforms the 8 densities together.  Each pass is a set of
// 1-D DFTs along one axis: a thread owns one line of one right-hand side,
// reads its np (or N) inputs from shared memory once and produces all the
// line's outputs, so shared-memory traffic is one read per input (the kernels
// are bound by it otherwise).  Shared staging arrays are planes [8][...]
// padded against bank conflicts; in global memory the spectra are written
// (and read back by k_m2l_inv32r8) as [block][slot][frequency][8], the
// forward's last pass ordered right-hand side fastest for contiguous writes.
// The grid is FftDims32 (N = 2np - 1 points per axis); the twiddles of every
// pass come from one table twb[k][b] = exp(-2 pi i k (b + np/2) / N).  Dynamic
// shared memory r8_fwd_smem<NP>() / r8_inv_smem<NP>().
// plane length rounded so that consecutive planes start 8 words apart modulo
// the 32 shared-memory banks (2-way conflicts at most across right-hand sides)
constexpr int r8_pad(int s) { return s + ((4 - s % 16) + 16) % 16; }
template <int NP>
constexpr size_t r8_fwd_smem() {  // cube + X1 + X2 (padded planes) + twiddles + roots
  using F = FftDims32<NP>;
  return sizeof(float) * NP * NP * NP * 8 +
         sizeof(float2) * (8 * r8_pad(NP * NP * F::NH) + 8 * r8_pad(NP * F::N * F::NH) + F::N * NP + F::N);
}
template <int NP>
constexpr size_t r8_inv_smem() {  // Y1 + Y2 (padded planes) + twiddles + roots
  using F = FftDims32<NP>;
  return sizeof(float2) * (8 * r8_pad(NP * NP * F::NH) + 8 * r8_pad(NP * F::N * F::NH) + F::N * NP + F::N);
}

__device__ __forceinline__ void r8_load(const float2* p, float2 (&v)[8]) {
  const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const float4 t = q[i];
    v[2 * i] = make_float2(t.x, t.y);
    v[2 * i + 1] = make_float2(t.z, t.w);
  }
}
__device__ __forceinline__ void r8_store(float2* p, const float2 (&v)[8]) {
  float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
  for (int i = 0; i < 4; i++) q[i] = make_float4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y);
}
template <int NP>
__device__ __forceinline__ void r8_twiddles(float2* twb, float2* roots) {
  using F = FftDims32<NP>;
  for (int i = threadIdx.x; i < F::N * NP + F::N; i += blockDim.x) {
    const int m = i < F::N * NP ? ((i / NP) * (i % NP + F::H)) % F::N : i - F::N * NP;
    double sn, cs;
    sincospi(2.0 * m / F::N, &sn, &cs);
    (i < F::N * NP ? twb[i] : roots[m]) = make_float2((float)cs, (float)-sn);
  }
}
// The line transforms with the twiddles in registers: twb[k][b] is the root
// w^m, m = k (b + H) mod N, so with both loops unrolled each product names
// its root at compile time and the N roots are held per thread as packed
// pairs.  Forward products s += a w (r8_cmac) take (w.x, w.y) and (w.y, w.x);
// inverse products s += a conj(w) (r8_cmacc) take (w.x, w.x) and (w.y, w.y).
// Each is two packed FP32x2 FMAs with the same per-component order as the
// scalar helpers, so the results are the same.
template <int N, int H>
struct R8Idx {
  static constexpr int at(int k, int b) { return (k * (b + H)) % N; }
};
__device__ __forceinline__ void r8_cmac2(unsigned long long& s, unsigned long long axx, unsigned long long nayy,
                                         unsigned long long wp, unsigned long long ws) {
  pq_fma2(s, axx, wp);   // (s.x + a.x w.x, s.y + a.x w.y)
  pq_fma2(s, nayy, ws);  // (s.x - a.y w.y, s.y + a.y w.x)
}
__device__ __forceinline__ void r8_cmacc2(unsigned long long& s, unsigned long long a, unsigned long long aswp,
                                          unsigned long long wxx, unsigned long long wyy) {
  pq_fma2(s, a, wxx);     // (s.x + a.x w.x, s.y + a.y w.x)
  pq_fma2(s, aswp, wyy);  // (s.x + a.y w.y, s.y - a.x w.y)
}

template <int NP>
__global__ void __launch_bounds__(256)
    k_m2l_fwd32r8(const int32_t* __restrict__ nodes, const int32_t* __restrict__ depth, int rootLevel, float deg,
                  const float* __restrict__ uden, int64_t udenRhs, const int32_t* __restrict__ ijk, int nUE,
                  float2* __restrict__ effDen, int64_t blkStride, int nEff, int kc) {
  using F = FftDims32<NP>;
  constexpr int N = F::N, NH = F::NH;
  constexpr int S1 = r8_pad(NP * NP * NH), S2 = r8_pad(NP * N * NH), S3 = NP * NP * NP;
  extern __shared__ __align__(16) unsigned char r8_smem[];
  float2* X1 = reinterpret_cast<float2*>(r8_smem);      // [8][NP][NP][NH]
  float2* X2 = X1 + S1 * 8;                              // [8][NP][N][NH]
  float2* twb = X2 + S2 * 8;                             // [N][NP]
  float2* roots = twb + N * NP;                          // [N]
  float* cube = reinterpret_cast<float*>(roots + N);     // [8][NP][NP][NP]
  const int slot = blockIdx.x;
  const int v = nodes[slot];
  const int r0 = blockIdx.y * 8;
  const int tid = threadIdx.x;
  using IX = R8Idx<N, F::H>;
  r8_twiddles<NP>(twb, roots);
  const float scl = (float)exp2((double)(depth[v] + rootLevel) * deg);
  for (int i = tid; i < S3 * 8; i += blockDim.x) cube[i] = 0.f;
  __syncthreads();
  for (int i = tid; i < nUE * 8; i += blockDim.x) {  // surface point fastest: coalesced reads of each plane
    const int j = i % nUE, r = i / nUE;
    if (r0 + r >= kc) continue;
    const int p = ijk[j];
    cube[r * S3 + ((p >> 16) * NP + ((p >> 8) & 255)) * NP + (p & 255)] =
        uden[(int64_t)(r0 + r) * udenRhs + (int64_t)v * nUE + j] * scl;
  }
  __syncthreads();
  unsigned long long wp[N], ws[N];  // the roots as (w.x, w.y) and (w.y, w.x)
#pragma unroll
  for (int m = 0; m < N; m++) {
    const float2 w = roots[m];
    wp[m] = pq_pk(w.x, w.y);
    ws[m] = pq_pk(w.y, w.x);
  }
  // x pass (real -> half spectrum): a thread owns one x line of one right-hand side
  for (int i = tid; i < NP * NP * 8; i += blockDim.x) {
    const int row = i % (NP * NP), r = i / (NP * NP);  // row = zb * NP + yb
    unsigned long long cc[NP];
#pragma unroll
    for (int xb = 0; xb < NP; xb++) {
      const float c = cube[r * S3 + row * NP + xb];
      cc[xb] = pq_pk(c, c);
    }
#pragma unroll
    for (int kx = 0; kx < NH; kx++) {
      unsigned long long s = 0ull;
#pragma unroll
      for (int xb = 0; xb < NP; xb++) pq_fma2(s, cc[xb], wp[IX::at(kx, xb)]);
      X1[r * S1 + row * NH + kx] = pq_unpk(s);
    }
  }
  __syncthreads();
  // y pass: a thread owns one y line (kx, zb) of one right-hand side and all N
  // ky outputs
  for (int i = tid; i < NH * NP * 8; i += blockDim.x) {
    const int kx = i % NH, zb = (i / NH) % NP, r = i / (NH * NP);
    unsigned long long axx[NP], nayy[NP];
#pragma unroll
    for (int yb = 0; yb < NP; yb++) {
      const float2 c = X1[r * S1 + (zb * NP + yb) * NH + kx];
      axx[yb] = pq_pk(c.x, c.x);
      nayy[yb] = pq_pk(-c.y, c.y);
    }
#pragma unroll
    for (int ky = 0; ky < N; ky++) {
      unsigned long long s = 0ull;
#pragma unroll
      for (int yb = 0; yb < NP; yb++) r8_cmac2(s, axx[yb], nayy[yb], wp[IX::at(ky, yb)], ws[IX::at(ky, yb)]);
      X2[r * S2 + (zb * N + ky) * NH + kx] = pq_unpk(s);
    }
  }
  __syncthreads();
  // z pass: a thread owns one z line (kx, ky) of one right-hand side and all N kz
  // outputs; right-hand side fastest so the global writes are contiguous
  float2* out = effDen + blockIdx.y * blkStride + (int64_t)slot * nEff * 8;
  for (int i = tid; i < NH * N * 8; i += blockDim.x) {
    const int r = i & 7, kx = (i >> 3) % NH, ky = (i >> 3) / NH;
    unsigned long long axx[NP], nayy[NP];
#pragma unroll
    for (int zb = 0; zb < NP; zb++) {
      const float2 c = X2[r * S2 + (zb * N + ky) * NH + kx];
      axx[zb] = pq_pk(c.x, c.x);
      nayy[zb] = pq_pk(-c.y, c.y);
    }
#pragma unroll
    for (int kz = 0; kz < N; kz++) {
      unsigned long long s = 0ull;
#pragma unroll
      for (int zb = 0; zb < NP; zb++) r8_cmac2(s, axx[zb], nayy[zb], wp[IX::at(kz, zb)], ws[IX::at(kz, zb)]);
      out[((int64_t)(kz * N + ky) * NH + kx) * 8 + r] = pq_unpk(s);
    }
  }
}

// The z pass reads the node's spectra from global memory directly: a warp's
// 32 lanes read 256 contiguous bytes and every element is read once, so the
// CTA needs no staging space (4 CTAs per SM at np = 6; staging the 64.5 KB
// block in shared memory first allowed 2 and measured 1.3x slower).
template <int NP>
__global__ void __launch_bounds__(256)
    k_m2l_inv32r8(const int32_t* __restrict__ nodes, const float2* __restrict__ effVal, int64_t blkStride, int nEff,
                  const int32_t* __restrict__ ijk, int nDC, float* __restrict__ dchk, int64_t dchkRhs, int kc) {
  using F = FftDims32<NP>;
  constexpr int N = F::N, NH = F::NH;
  constexpr int S1 = r8_pad(NP * NP * NH), S2 = r8_pad(NP * N * NH);
  extern __shared__ __align__(16) unsigned char r8_smem[];
  float2* Y1 = reinterpret_cast<float2*>(r8_smem);  // [8][NP][NP][NH]
  float2* Y2 = Y1 + S1 * 8;                          // [8][NP][N][NH]
  float2* twb = Y2 + S2 * 8;                         // [N][NP]
  float2* roots = twb + N * NP;                      // [N]
  const int slot = blockIdx.x;
  const int node = nodes[slot];
  const int r0 = blockIdx.y * 8;
  const int tid = threadIdx.x;
  using IX = R8Idx<N, F::H>;
  const float2* Xg = effVal + blockIdx.y * blkStride + (int64_t)slot * nEff * 8;
  r8_twiddles<NP>(twb, roots);
  __syncthreads();
  unsigned long long wxx[N], wyy[N];  // the roots as (w.x, w.x) and (w.y, w.y)
#pragma unroll
  for (int m = 0; m < N; m++) {
    const float2 w = roots[m];
    wxx[m] = pq_pk(w.x, w.x);
    wyy[m] = pq_pk(w.y, w.y);
  }
  // z pass, band outputs only: a thread owns one z line (kx, ky) of one
  // right-hand side, right-hand side fastest as in HBM
  for (int i = tid; i < NH * N * 8; i += blockDim.x) {
    const int r = i & 7, kx = (i >> 3) % NH, ky = (i >> 3) / NH;
    float2 c[N];
#pragma unroll
    for (int kz = 0; kz < N; kz++) c[kz] = Xg[((kz * N + ky) * NH + kx) * 8 + r];  // all loads of the line first
    unsigned long long s[NP];
#pragma unroll
    for (int zb = 0; zb < NP; zb++) s[zb] = 0ull;
#pragma unroll
    for (int kz = 0; kz < N; kz++) {
      const unsigned long long a = pq_pk(c[kz].x, c[kz].y), asw = pq_pk(c[kz].y, -c[kz].x);
#pragma unroll
      for (int zb = 0; zb < NP; zb++) r8_cmacc2(s[zb], a, asw, wxx[IX::at(kz, zb)], wyy[IX::at(kz, zb)]);
    }
#pragma unroll
    for (int zb = 0; zb < NP; zb++) Y2[r * S2 + (zb * N + ky) * NH + kx] = pq_unpk(s[zb]);
  }
  __syncthreads();
  // y pass: a thread owns one y line (kx, zb) of one right-hand side
  for (int i = tid; i < NH * NP * 8; i += blockDim.x) {
    const int kx = i % NH, zb = (i / NH) % NP, r = i / (NH * NP);
    unsigned long long s[NP];
#pragma unroll
    for (int yb = 0; yb < NP; yb++) s[yb] = 0ull;
#pragma unroll
    for (int ky = 0; ky < N; ky++) {
      const float2 c = Y2[r * S2 + (zb * N + ky) * NH + kx];
      const unsigned long long a = pq_pk(c.x, c.y), asw = pq_pk(c.y, -c.x);
#pragma unroll
      for (int yb = 0; yb < NP; yb++) r8_cmacc2(s[yb], a, asw, wxx[IX::at(ky, yb)], wyy[IX::at(ky, yb)]);
    }
#pragma unroll
    for (int yb = 0; yb < NP; yb++) Y1[r * S1 + (zb * NP + yb) * NH + kx] = pq_unpk(s[yb]);
  }
  __syncthreads();
  for (int i = tid; i < nDC * 8; i += blockDim.x) {  // x pass (c2r) at the surface points
    const int j = i % nDC, r = i / nDC;
    if (r0 + r >= kc) continue;
    const int p = ijk[j];
    const int a = p & 255, b = (p >> 8) & 255, cc = p >> 16;
    const float2* y1 = &Y1[r * S1 + (cc * NP + b) * NH];
    float s = 0.f;
#pragma unroll
    for (int kx = 0; kx < NH; kx++) {
      const float2 w = twb[kx * NP + a];
      s += ((kx == 0 || 2 * kx == N) ? 1.f : 2.f) * cmulc(y1[kx], w).x;
    }
    dchk[(int64_t)(r0 + r) * dchkRhs + (int64_t)node * nDC + j] += s;
  }
}

// ------------------------------------------------------------------ launcher
template <typename T>
static std::string dalloc(DevState& D, T*& p, size_t n) {
  void* q = nullptr;
  cudaError_t e = dev_alloc(D, &q, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return std::string("cudaMalloc: ") + cudaGetErrorString(e);
  p = (T*)q;
  return std::string();
}

static int pad4(int k) { return (k + 3) & ~3; }
// F1 is k x n row-major: append zero rows up to pad4(k)
static std::vector<double> pad_rows(const std::vector<double>& F, int k, int n) {
  std::vector<double> r((size_t)pad4(k) * n, 0.0);
  std::copy(F.begin(), F.begin() + (size_t)k * n, r.begin());
  return r;
}
// F2 is m x k row-major: widen each row to pad4(k) with zeros
static std::vector<double> pad_cols(const std::vector<double>& F, int m, int k) {
  const int kp = pad4(k);
  std::vector<double> r((size_t)m * kp, 0.0);
  for (int i = 0; i < m; i++) std::copy(F.begin() + (size_t)i * k, F.begin() + (size_t)(i + 1) * k, r.begin() + (size_t)i * kp);
  return r;
}

// W row-major n x k -> Wt[k][n] in FP32, K padded to a multiple of GW_BK and N
// to a multiple of GW_BN (ld) with zeros: the wide-tile GEMM reads whole tiles
static std::vector<float> transpose_pad(const std::vector<double>& W, int n, int k, int& ld) {
  const int kp = (k + GW_BK - 1) / GW_BK * GW_BK;
  ld = (n + GW_BN - 1) / GW_BN * GW_BN;
  std::vector<float> t((size_t)kp * ld, 0.f);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < k; j++) t[(size_t)j * ld + i] = (float)W[(size_t)i * k + j];
  return t;
}

// Work arrays for a chunk of kc right-hand sides, and the FP32 operator copies.
// M2T work items.  A far row's cost is its targets x W entries x UE points;
// rows above a cap (the total over 6 items per SM, at least 8,192 pairs) are
// split into near-equal runs of entries, each item writing its own partial
// sums; items run longest first.
static void m2t_items(const Plan& P, int numSMs, std::vector<int4>& items, std::vector<int32_t>& splitLeaf,
                      std::vector<int32_t>& splitBase, std::vector<int32_t>& splitCnt, int64_t& partTargets) {
  items.clear();
  splitLeaf.clear();
  splitBase.clear();
  splitCnt.clear();
  partTargets = 0;
  const int nr = (int)P.farLeaves.size();
  std::vector<double> cost;
  double total = 0;
  for (int r = 0; r < nr; r++)
    total += (double)P.trgCnt[P.farLeaves[r]] * P.nUE * (P.farUE.ptr[r + 1] - P.farUE.ptr[r]);
  const double cap = std::max(8192.0, total / (6.0 * numSMs));
  for (int r = 0; r < nr; r++) {
    const int64_t e0 = P.farUE.ptr[r], ne = P.farUE.ptr[r + 1] - e0;
    const int64_t tn = P.trgCnt[P.farLeaves[r]];
    const double per = (double)std::max<int64_t>(tn, 1) * P.nUE;
    const int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(ne, (int64_t)std::ceil(per * ne / cap)));
    if (chunks == 1) {
      items.push_back(make_int4(r, (int)e0, (int)(e0 + ne), -1));
      cost.push_back(per * ne);
      continue;
    }
    splitLeaf.push_back(P.farLeaves[r]);
    splitBase.push_back((int32_t)partTargets);
    splitCnt.push_back((int32_t)chunks);
    for (int64_t c = 0; c < chunks; c++) {
      const int64_t a = e0 + ne * c / chunks, b = e0 + ne * (c + 1) / chunks;
      items.push_back(make_int4(r, (int)a, (int)b, (int)(partTargets + c * tn)));
      cost.push_back(per * (b - a));
    }
    partTargets += chunks * tn;
  }
  std::vector<int> order(items.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<int4> sorted(items.size());
  for (size_t i = 0; i < order.size(); i++) sorted[i] = items[order[i]];
  items.swap(sorted);
}

static std::string dev_prepare_mixed(const Plan& P, DevState& D, int kc) {
  const size_t ue = (size_t)P.nUE * P.sdm, uc = (size_t)P.nUC * P.tdm;
  const size_t de = (size_t)P.nDE * P.sdm, dc = (size_t)P.nDC * P.tdm;
  if (!D.nearOrder && !P.evtrLeaves.empty()) {  // near-field rows by decreasing pair count
    const size_t nl = P.evtrLeaves.size();
    std::vector<int64_t> cost(nl);
    for (size_t r = 0; r < nl; r++) {
      int64_t sc = 0;
      for (int64_t e = P.nearSrc.ptr[r]; e < P.nearSrc.ptr[r + 1]; e++) sc += P.srcCnt[P.nearSrc.idx[e]];
      cost[r] = sc * P.trgCnt[P.evtrLeaves[r]];
    }
    std::vector<int32_t> order(nl);
    for (size_t r = 0; r < nl; r++) order[r] = (int32_t)r;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
    FMMG_TRY(dalloc(D, D.nearOrder, nl));
    FMMG_CK(cudaMemcpy(D.nearOrder, order.data(), nl * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (!D.m2tItems && !P.farLeaves.empty()) {
    std::vector<int4> items;
    std::vector<int32_t> sl, sb, sc;
    m2t_items(P, D.numSMs, items, sl, sb, sc, D.m2tPartTargets);
    FMMG_TRY(dalloc(D, D.m2tItems, items.size()));
    FMMG_CK(cudaMemcpy(D.m2tItems, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
    D.nM2tItems = (int)items.size();
    D.nM2tSplit = (int)sl.size();
    auto put = [&](int32_t*& dst, const std::vector<int32_t>& v) -> std::string {
      FMMG_TRY(dalloc(D, dst, v.size()));
      FMMG_CK(cudaMemcpy(dst, v.data(), v.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
      return std::string();
    };
    if (!sl.empty()) {
      FMMG_TRY(put(D.m2tSplitLeaf, sl));
      FMMG_TRY(put(D.m2tSplitBase, sb));
      FMMG_TRY(put(D.m2tSplitCnt, sc));
    }
  }
  // rank-sized buffers take the largest rank a pinv can have, so factors
  // recomputed for a replaced table (Plan::refactor_c2e) always fit
  const int kUpMax = pad4((int)std::min(ue, uc)), kDnMax = pad4((int)std::min(de, dc));
  if (!D.mixedReady || kc > D.mixedK) {
    // grow: the old buffers stay in D.allocs until the handle is freed
    FMMG_TRY(dalloc(D, D.uchk32, (size_t)kc * P.nn * uc));
    FMMG_TRY(dalloc(D, D.uden32, (size_t)kc * P.nn * ue));
    // rows of nodes without sources are read (M2M children, V and W sources)
    // but never written: zero once here
    FMMG_CK(cudaMemsetAsync(D.uden32, 0, sizeof(float) * kc * P.nn * ue, D.stream));
    FMMG_TRY(dalloc(D, D.dchk32, (size_t)kc * P.nn * dc));
    FMMG_TRY(dalloc(D, D.dden32, (size_t)kc * P.nn * de));
    const size_t kc8 = (size_t)(kc + 7) / 8 * 8;  // the scalar k >= 2 layout stores blocks of 8
    FMMG_TRY(dalloc(D, D.effDen32, kc8 * P.vSrcNodes.size() * P.nEff32 * P.sdm));
    FMMG_TRY(dalloc(D, D.effVal32, kc8 * P.vTrgNodes.size() * P.nEff32 * P.tdm));
    FMMG_TRY(dalloc(D, D.upT32, (size_t)kc * P.nn * kUpMax));
    FMMG_TRY(dalloc(D, D.dnT32, (size_t)kc * P.nn * kDnMax));
    FMMG_TRY(dalloc(D, D.denK, (size_t)kc * P.ns * P.sd));
    FMMG_TRY(dalloc(D, D.den32, kc8 * P.ns * P.sd));
    FMMG_TRY(dalloc(D, D.valK, (size_t)kc * std::max<int64_t>(P.nt, 1) * P.td));
    FMMG_TRY(dalloc(D, D.m2tPart, (size_t)kc * std::max<int64_t>(D.m2tPartTargets, 1) * P.tdm));
    if (!D.l2l32) {
      FMMG_TRY(dalloc(D, D.l2l32, P.l2l.size()));
      FMMG_TRY(dalloc(D, D.m2lT32, P.m2lT32.size()));
      if (P.sdm == 1 && P.tdm == 1) FMMG_TRY(dalloc(D, D.m2lTw32, (size_t)27 * 27 * P.nEff32));
      FMMG_TRY(dalloc(D, D.upF1, (size_t)kUpMax * uc));
      FMMG_TRY(dalloc(D, D.upF2, ue * kUpMax));
      FMMG_TRY(dalloc(D, D.dnF1, (size_t)kDnMax * dc));
      FMMG_TRY(dalloc(D, D.dnF2, de * kDnMax));
      FMMG_TRY(dalloc(D, D.m2mUp32, ue * 8 * ue));
    }
    D.mixedReady = true;
    D.mixedK = kc;
  }
  if (D.mixedOpsStale) {
    auto put = [&](float* dst, const std::vector<double>& v) -> std::string {
      std::vector<float> f(v.begin(), v.end());
      FMMG_CK(cudaMemcpy(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
      return std::string();
    };
    FMMG_TRY(put(D.l2l32, P.l2l));
    // the factors padded to a rank that is a multiple of 4 (zero rows of F1,
    // zero columns of F2), so the intermediate rows allow 16-byte tile fetches
    FMMG_TRY(put(D.upF1, pad_rows(P.uc2ueF1, P.kUp, (int)uc)));
    FMMG_TRY(put(D.upF2, pad_cols(P.uc2ueF2, (int)ue, P.kUp)));
    FMMG_TRY(put(D.dnF1, pad_rows(P.dc2deF1, P.kDn, (int)dc)));
    FMMG_TRY(put(D.dnF2, pad_cols(P.dc2deF2, (int)de, P.kDn)));
    // the same operators transposed and padded for the wide-tile GEMM
    auto putT = [&](DevState::OpT& op, const std::vector<double>& W, int n, int k) -> std::string {
      int ld = 0;
      const std::vector<float> t = transpose_pad(W, n, k, ld);
      if (!op.p || t.size() > op.cap) {
        FMMG_TRY(dalloc(D, op.p, t.size()));
        op.cap = t.size();
      }
      op.ld = ld;
      FMMG_CK(cudaMemcpy(op.p, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
      return std::string();
    };
    const int kUp4 = pad4(P.kUp), kDn4 = pad4(P.kDn);
    FMMG_TRY(putT(D.tL2L, P.l2l, (int)(8 * dc), (int)de));
    FMMG_TRY(putT(D.tUpF1, pad_rows(P.uc2ueF1, P.kUp, (int)uc), kUp4, (int)uc));
    FMMG_TRY(putT(D.tUpF2, pad_cols(P.uc2ueF2, (int)ue, P.kUp), (int)ue, kUp4));
    FMMG_TRY(putT(D.tDnF1, pad_rows(P.dc2deF1, P.kDn, (int)dc), kDn4, (int)dc));
    FMMG_TRY(putT(D.tDnF2, pad_cols(P.dc2deF2, (int)de, P.kDn), (int)de, kDn4));
    // a parent's upward density straight from its children's: C2E up x M2M
    const std::vector<double>& fold = [&]() -> const std::vector<double>& {
      LinalgDeviceScope scope(D.device);  // formed on this GPU on first use (the host's sums, bit for bit)
      return P.folded_upward();
    }();
    FMMG_TRY(put(D.m2mUp32, fold));
    FMMG_TRY(putT(D.tM2MUp, fold, (int)ue, (int)(8 * ue)));
    // the same six operators split into TF32 hi / lo parts for the tensor cores
    auto tcAlloc = [&](float*& p, size_t n) { return dalloc(D, p, n); };
    FMMG_TRY(tc_prepare_operator(D.cL2L, P.l2l, (int)(8 * dc), (int)de, tcAlloc));
    FMMG_TRY(tc_prepare_operator(D.cUpF1, pad_rows(P.uc2ueF1, P.kUp, (int)uc), kUp4, (int)uc, tcAlloc));
    FMMG_TRY(tc_prepare_operator(D.cUpF2, pad_cols(P.uc2ueF2, (int)ue, P.kUp), (int)ue, kUp4, tcAlloc));
    FMMG_TRY(tc_prepare_operator(D.cDnF1, pad_rows(P.dc2deF1, P.kDn, (int)dc), kDn4, (int)dc, tcAlloc));
    FMMG_TRY(tc_prepare_operator(D.cDnF2, pad_cols(P.dc2deF2, (int)de, P.kDn), (int)de, kDn4, tcAlloc));
    FMMG_TRY(tc_prepare_operator(D.cM2MUp, fold, (int)ue, (int)(8 * ue), tcAlloc));
    std::vector<float2> t(P.m2lT32.size());
    for (size_t i = 0; i < t.size(); i++) t[i] = make_float2((float)P.m2lT32[i].real(), (float)P.m2lT32[i].imag());
    FMMG_CK(cudaMemcpy(D.m2lT32, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice));
    if (D.m2lTw32) {  // combined translations of the 27-product Hadamard (had_pq.cuh), FP64 sums
      auto w = [](int code, int d) -> double {
        if (code == 0) return d == 0 ? 1.0 : 0.0;
        if (code == 1) return d == 1 ? 1.0 : (d == 0 ? -1.0 : 0.0);
        return d == -1 ? 1.0 : (d == 0 ? -1.0 : 0.0);
      };
      const int ne = P.nEff32;
      std::vector<float2> tw((size_t)27 * 27 * ne, make_float2(0.f, 0.f));
      std::vector<std::complex<double>> acc(ne);
      for (int o = 0; o < 27; o++) {
        if (o == 13) continue;
        const int ox = o / 9 - 1, oy = (o / 3) % 3 - 1, oz = o % 3 - 1;
        for (int j = 0; j < 27; j++) {
          const int jx = j / 9, jy = (j / 3) % 3, jz = j % 3;
          std::fill(acc.begin(), acc.end(), std::complex<double>(0.0, 0.0));
          for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++)
              for (int dz = -1; dz <= 1; dz++) {
                const double wt = w(jx, dx) * w(jy, dy) * w(jz, dz);
                if (wt == 0.0) continue;
                const int id = P.transId[2 * ox + dx + 3][2 * oy + dy + 3][2 * oz + dz + 3];
                if (id < 0) continue;  // touching pair
                const std::complex<double>* Tt = &P.m2lT32[(size_t)id * ne];
                for (int f = 0; f < ne; f++) acc[f] += wt * Tt[f];
              }
          float2* dst = &tw[((size_t)o * 27 + j) * ne];
          for (int f = 0; f < ne; f++) dst[f] = make_float2((float)acc[f].real(), (float)acc[f].imag());
        }
      }
      FMMG_CK(cudaMemcpy(D.m2lTw32, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
    }
    int16_t tid[343];
    for (int i = 0; i < 343; i++) tid[i] = (int16_t)P.transId[i / 49][(i / 7) % 7][i % 7];
    FMMG_CK(cudaMemcpyToSymbol(c_transId32, tid, sizeof(tid)));
    D.mixedOpsStale = false;
  }
  return std::string();
}

// one pass over a chunk of kc right-hand sides, KB of them per launch block
// overlap: run the near field and the W list on D.side (an untimed pass; a
// timed one keeps every stage on the main stream so the events bracket it)
template <int KT, int KB>
static void run_mixed_blocks(const Plan& P, DevState& D, int kc, int mask, bool overlap, LaunchStats* ls) {
  cudaStream_t st = D.stream;
  const int64_t ue = (int64_t)P.nUE * P.sdm, uc = (int64_t)P.nUC * P.tdm;
  const int64_t de = (int64_t)P.nDE * P.sdm, dc = (int64_t)P.nDC * P.tdm;
  const int64_t nn = P.nn;
  const int kUp4 = pad4(P.kUp), kDn4 = pad4(P.kDn);
  const int rl = P.o.rootLevel;
  const float mu = (float)P.o.coefs[0], ve = (float)P.o.coefs[1];
  const int nl = (int)P.evtrLeaves.size();
  const int kb = (kc + KB - 1) / KB;
  const int64_t valStride = std::max<int64_t>(P.nt, 1) * P.td;
  const int64_t den32Blk = P.ns * 8 * P.sd;  // floats per block of 8 right-hand sides in D.den32
  // tc: the operator split for the tensor cores (3xTF32), used when that
  // path is on and the class is in the tuning mask (the wide CUDA-core tiles
  // otherwise)
  auto useTc = [&](const TcOp& tc) {
    const int cls = &tc == &D.cUpF1 ? 0 : &tc == &D.cUpF2 ? 1 : &tc == &D.cM2MUp ? 2 : &tc == &D.cL2L ? 3
                    : &tc == &D.cDnF1 ? 4 : 5;
    return D.gemmPath == 1 && ((D.tune.tcMask >> cls) & 1);
  };
  auto gemm = [&](int nrows, const int32_t* rows, int xChild, int yChild, const float* X, int64_t ldx, int64_t xR,
                  const float* W, const DevState::OpT& wt, float* Y, int64_t ldy, int64_t yR, int K, int N, Scale4 xs,
                  Scale4 ys, float beta, const TcOp& tc) {
    if (nrows <= 0) return;
    GrScale<float> gx, gy;
    gx.mod = xs.mod;
    gy.mod = ys.mod;
    for (int k = 0; k < 4; k++) {
      gx.v[k] = (float)xs.v[k];
      gy.v[k] = (float)ys.v[k];
    }
    ls->launches += launch_gemm_rows_f32(st, D.numSMs * D.tune.gemmSplitMul, reinterpret_cast<float*>(D.gemmScratch),
                                         D.gemmScratchBytes / sizeof(float), useTc(tc) ? &tc : nullptr,
                                         D.tune.tcProducts, D.devErr, nrows,
                                         kc, rows, D.chd, xChild, yChild, X, ldx, xR, W,
                                         D.gemmPath == 2 ? nullptr : wt.p, wt.ld, Y, ldy, yR, K, N, gx, gy, beta);
  };
  const bool ovl = overlap && D.side;
  if (ovl) {  // fork: the densities are gathered and the target values cleared
    cudaEventRecord(D.evFork, st);
    cudaStreamWaitEvent(D.side, D.evFork, 0);
  }
  if ((mask & 1) && !P.s2mLeaves.empty()) {
    const int nlv = (int)P.s2mLeaves.size();
    k_s2m32w<KT, KB><<<dim3((nlv + S2M_WARPS - 1) / S2M_WARPS, kb), 32 * S2M_WARPS, 0, st>>>(
        nlv, D.s2mLeaves, D.srcBeg, D.srcCnt, D.src, D.nrm, D.den32, den32Blk, D.ctr, D.rad, D.sam[1], P.nUC,
        D.uchk32, uc, nn * uc, kc, mu, ve);
    ls->launches++;
  }
  cudaEventRecord(D.ev[EV_S2M], st);
  if (mask & 1) {
    for (int d = P.maxDepth; d >= 1; d--) {
      // leaves with sources: C2E as F2 (F1 uchk), so the large-norm pinv
      // never multiplies in FP32
      int64_t a = D.offUpLeaf[d], b = D.offUpLeaf[d + 1];
      gemm((int)(b - a), D.levelRows + a, 0, 0, D.uchk32, uc, nn * uc, D.upF1, D.tUpF1, D.upT32, kUp4, nn * kUp4, uc,
           kUp4, unit_scale(), unit_scale(), 0.f, D.cUpF1);
      gemm((int)(b - a), D.levelRows + a, 0, 0, D.upT32, kUp4, nn * kUp4, D.upF2, D.tUpF2, D.uden32, ue, nn * ue, kUp4,
           ue, unit_scale(), level_scale(P, d + rl, -1.0), 0.f, D.cUpF2);
      // parents: C2E up x M2M folded on the host in FP64 (its norm is O(1)
      // where the pinv's is ~1e6), one product from the children's upward
      // densities (depth d + 1, done in the previous iteration) with no check
      // surface in between
      a = D.offUpM2M[d];
      b = D.offUpM2M[d + 1];
      gemm((int)(b - a), D.levelRows + a, 1, 0, D.uden32, ue, nn * ue, D.m2mUp32, D.tM2MUp, D.uden32, ue, nn * ue,
           8 * ue, ue, level_scale(P, d + 1 + rl, +1.0), level_scale(P, d + rl, -1.0), 0.f, D.cM2MUp);
    }
  }
  cudaEventRecord(D.ev[EV_UP_GEMM], st);
  auto near = [&](const int64_t* ptr, const int32_t* idx, cudaStream_t sn) {
    if (nl == 0) return;
    if constexpr (KT == LAP_S_U)  // two targets a thread, packed FP32x2, a warp per leaf
      k_p2p_near32_lap2w<KB><<<dim3((nl + NW_WARPS - 1) / NW_WARPS, kb), 32 * NW_WARPS, 0, sn>>>(
          nl, D.nearOrder, D.evtrLeaves, ptr, idx, D.srcBeg, D.srcCnt, D.trgBeg, D.trgCnt, D.src, D.den32, den32Blk,
          D.trg, D.ctr, D.valK, valStride, kc);
    else
      k_p2p_near32<KT, KB><<<dim3(nl, kb), MX_THREADS, 0, sn>>>(D.evtrLeaves, ptr, idx, D.srcBeg, D.srcCnt, D.trgBeg,
                                                               D.trgCnt, D.src, D.nrm, D.den32, den32Blk, D.trg, D.ctr,
                                                               D.valK, valStride, kc, mu, ve);
    ls->launches++;
  };
  auto nearAll = [&](cudaStream_t sn) {
    if ((mask & 2) && (mask & 8) && (mask & 16)) {
      near(D.nearPtr, D.nearIdx, sn);
    } else {
      if (mask & 2) near(D.nearUPtr, D.nearUIdx, sn);
      if (mask & 8) near(D.nearWPtr, D.nearWIdx, sn);
      if (mask & 16) near(D.nearXPtr, D.nearXIdx, sn);
    }
  };
  if (ovl) {  // the up pass is done: the W list (own upward densities) joins the near field
    nearAll(D.side);
    cudaEventRecord(D.evUp, st);
    cudaStreamWaitEvent(D.side, D.evUp, 0);
  } else {
    nearAll(st);
  }
  cudaEventRecord(D.ev[EV_NEAR], st);
  const int nsrc = (int)P.vSrcNodes.size(), ntrg = (int)P.vTrgNodes.size(), npar = (int)P.vParents.size();
  const int64_t effDR = (int64_t)nsrc * P.nEff32 * P.sdm, effVR = (int64_t)ntrg * P.nEff32 * P.tdm;
  const bool r8 = P.sdm == 1 && P.tdm == 1 && kc >= 2 && D.hadPQ;  // blocks of 8 interleaved right-hand sides
  const int nblk = (kc + 7) / 8;
  const int64_t blkDen = (int64_t)nsrc * P.nEff32 * 8, blkVal = (int64_t)ntrg * P.nEff32 * 8;
  if ((mask & 4) && nsrc > 0 && r8) {
#define FMMG_FWD32R8(NP_)                                                                                      \
  do {                                                                                                         \
    constexpr size_t sm = r8_fwd_smem<NP_>();                                                                  \
    cudaFuncSetAttribute(k_m2l_fwd32r8<NP_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);            \
    k_m2l_fwd32r8<NP_><<<dim3(nsrc, nblk), 256, sm, st>>>(D.vSrcNodes, D.depth, rl, (float)P.deg[0], D.uden32, \
                                                          nn * ue, D.surfIJK, P.nUE, D.effDen32, blkDen,       \
                                                          P.nEff32, kc);                                         \
  } while (0)
    switch (P.o.np) {
      case 3: FMMG_FWD32R8(3); break;
      case 4: FMMG_FWD32R8(4); break;
      case 5: FMMG_FWD32R8(5); break;
      case 6: FMMG_FWD32R8(6); break;
      case 7: FMMG_FWD32R8(7); break;
      case 8: FMMG_FWD32R8(8); break;
    }
#undef FMMG_FWD32R8
    ls->launches++;
  } else if ((mask & 4) && nsrc > 0) {
    Scale4 deg;
    deg.mod = P.sdm;
    for (int k = 0; k < 4; k++) deg.v[k] = P.deg[k];
#define FMMG_FWD32(NP_)                                                                                         \
  k_m2l_fwd32<NP_><<<dim3(nsrc, kc), 128, 0, st>>>(D.vSrcNodes, D.depth, rl, deg, P.sdm, D.uden32, nn * ue,    \
                                                    D.surfIJK, P.nUE, D.effDen32, effDR, P.nEff32)
    switch (P.o.np) {
      case 3: FMMG_FWD32(3); break;
      case 4: FMMG_FWD32(4); break;
      case 5: FMMG_FWD32(5); break;
      case 6: FMMG_FWD32(6); break;
      case 7: FMMG_FWD32(7); break;
      case 8: FMMG_FWD32(8); break;
    }
#undef FMMG_FWD32
    ls->launches++;
  }
  cudaEventRecord(D.ev[EV_M2L_FWD], st);
  if ((mask & 4) && npar > 0 && ntrg > 0) {
    dim3 grid(npar, (P.nEff32 + 31) / 32, kb);
    const float nrmfc = 1.0f / float(P.nReg32);
    // vector kernels: 8 right-hand sides a thread when there are more than 4
    // (each translation value loaded serves twice the multiply-adds; the pair
    // kernels keep their 4)
#define FMMG_HAD32(SD_, TD_)                                                                                   \
  do {                                                                                                         \
    if (kc > 4)                                                                                                \
      k_m2l_had32<SD_, TD_, 8><<<dim3(npar, (P.nEff32 + 31) / 32, (kc + 7) / 8), 256, 0, st>>>(                \
          D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen32, effDR, D.m2lT32, D.effVal32, effVR, P.nEff32, kc,   \
          nrmfc);                                                                                              \
    else                                                                                                       \
      k_m2l_had32<SD_, TD_, KB><<<grid, 256, 0, st>>>(D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen32, effDR, \
                                                       D.m2lT32, D.effVal32, effVR, P.nEff32, kc, nrmfc);      \
  } while (0)
    if (P.sdm == 1 && P.tdm == 1 && D.hadPQ) {
      if (!r8) {  // planes of one right-hand side
        const size_t smem = pqx_smem_bytes<32>();
        cudaFuncSetAttribute(k_m2l_had_pqx2<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dim3 g1((npar + D.tune.hadRows - 1) / D.tune.hadRows, (P.nEff32 + 31) / 32, kc);
        k_m2l_had_pqx2<32, false><<<g1, PQX_THREADS, smem, st>>>(
            npar, D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen32, PqLayout{effDR, P.nEff32}, D.m2lT32, D.effVal32,
            PqLayout{effVR, P.nEff32}, 1, 0, P.nEff32, kc, nrmfc, D.transIdDev);
      } else if (D.hadW && D.m2lTw32 && D.tune.hadRhsPerThread >= 3) {  // output-child accumulators
#define FMMG_HADO(R_)                                                                                         \
  do {                                                                                                        \
    constexpr int FB = 4 * (R_);                                                                              \
    const size_t smem = (size_t)W8_OFFS * 27 * FB * sizeof(float2);                                           \
    cudaFuncSetAttribute(k_m2l_had_o<R_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);            \
    dim3 go((npar + D.tune.hadRows - 1) / D.tune.hadRows, (P.nEff32 + FB - 1) / FB, nblk);                    \
    k_m2l_had_o<R_><<<go, PQX_THREADS, smem, st>>>(npar, D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen32,     \
                                                   PqLayout{blkDen, (int64_t)P.nEff32 * 8}, D.m2lTw32,        \
                                                   D.effVal32, PqLayout{blkVal, (int64_t)P.nEff32 * 8},       \
                                                   P.nEff32, kc, nrmfc);                                      \
  } while (0)
        if (D.tune.hadRhsPerThread == 4) FMMG_HADO(4);
        else FMMG_HADO(2);
#undef FMMG_HADO
      } else if (D.hadW && D.m2lTw32 && D.tune.hadRhsPerThread == 2) {  // 27-product form, 2 RHS a thread
        const size_t smem = (size_t)W8_OFFS * 27 * W8X2_F * sizeof(float2);
        cudaFuncSetAttribute(k_m2l_had_w8x2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dim3 g8((npar + D.tune.hadRows - 1) / D.tune.hadRows, (P.nEff32 + W8X2_F - 1) / W8X2_F, nblk);
        k_m2l_had_w8x2<<<g8, PQX_THREADS, smem, st>>>(npar, D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen32,
                                                       PqLayout{blkDen, (int64_t)P.nEff32 * 8}, D.m2lTw32, D.effVal32,
                                                       PqLayout{blkVal, (int64_t)P.nEff32 * 8}, P.nEff32, kc, nrmfc);
      } else if (D.hadW && D.m2lTw32) {  // 27-product form
        const size_t smem = (size_t)W8_OFFS * 27 * 4 * sizeof(float2);
        cudaFuncSetAttribute(k_m2l_had_w8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dim3 g8((npar + D.tune.hadRows - 1) / D.tune.hadRows, (P.nEff32 + 3) / 4, nblk);
        k_m2l_had_w8<<<g8, PQX_THREADS, smem, st>>>(npar, D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen32,
                                                     PqLayout{blkDen, (int64_t)P.nEff32 * 8}, D.m2lTw32, D.effVal32,
                                                     PqLayout{blkVal, (int64_t)P.nEff32 * 8}, P.nEff32, kc, nrmfc);
      } else {
        const size_t smem = pqx_smem_bytes<4>();
        dim3 g8((npar + D.tune.hadRows - 1) / D.tune.hadRows, (P.nEff32 + 3) / 4, nblk);
        k_m2l_had_pqx2<4, false><<<g8, PQX_THREADS, smem, st>>>(
            npar, D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen32, PqLayout{blkDen, (int64_t)P.nEff32 * 8}, D.m2lT32,
            D.effVal32, PqLayout{blkVal, (int64_t)P.nEff32 * 8}, 8, 1, P.nEff32, kc, nrmfc, D.transIdDev);
      }
    } else if (P.sdm == 1 && P.tdm == 1) {
      if (!D.vListsReady) throw std::logic_error("the expanded V lists are not on the device (dev_upload_vlists)");
      const size_t smem = had_smem_bytes<float2>();
      cudaFuncSetAttribute(k_m2l_had_list<float2, KB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      dim3 g2((ntrg + HS_BOXES - 1) / HS_BOXES, (P.nEff32 + 31) / 32, kb);
      k_m2l_had_list<float2, KB, false><<<g2, HS_THREADS, smem, st>>>(
          ntrg, D.vTrgPtr, (const int2*)D.vTrgEnt, D.effDen32, effDR, D.m2lT32, D.effVal32, effVR, P.nEff32, kc,
          nrmfc);
    } else if (P.sdm == 4 && P.tdm == 3) FMMG_HAD32(4, 3);
    else FMMG_HAD32(3, 3);
#undef FMMG_HAD32
    ls->launches++;
  }
  cudaEventRecord(D.ev[EV_M2L_HAD], st);
  if ((mask & 4) && npar > 0 && ntrg > 0 && r8) {
#define FMMG_INV32R8(NP_)                                                                                      \
  do {                                                                                                         \
    constexpr size_t sm = r8_inv_smem<NP_>();                                                                  \
    cudaFuncSetAttribute(k_m2l_inv32r8<NP_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);            \
    k_m2l_inv32r8<NP_><<<dim3(ntrg, nblk), 256, sm, st>>>(D.vTrgNodes, D.effVal32, blkVal, P.nEff32, D.surfIJK,  \
                                                          P.nDC, D.dchk32, nn * dc, kc);                       \
  } while (0)
    switch (P.o.np) {
      case 3: FMMG_INV32R8(3); break;
      case 4: FMMG_INV32R8(4); break;
      case 5: FMMG_INV32R8(5); break;
      case 6: FMMG_INV32R8(6); break;
      case 7: FMMG_INV32R8(7); break;
      case 8: FMMG_INV32R8(8); break;
    }
#undef FMMG_INV32R8
    ls->launches++;
  } else if ((mask & 4) && npar > 0 && ntrg > 0) {
#define FMMG_INV32(NP_)                                                                                   \
  k_m2l_inv32<NP_><<<dim3(ntrg, kc), 128, 0, st>>>(D.vTrgNodes, D.effVal32, effVR, P.nEff32, P.tdm, D.surfIJK, \
                                                    P.nDC, D.dchk32, nn * dc)
    switch (P.o.np) {
      case 3: FMMG_INV32(3); break;
      case 4: FMMG_INV32(4); break;
      case 5: FMMG_INV32(5); break;
      case 6: FMMG_INV32(6); break;
      case 7: FMMG_INV32(7); break;
      case 8: FMMG_INV32(8); break;
    }
#undef FMMG_INV32
    ls->launches++;
  }
  cudaEventRecord(D.ev[EV_M2L_INV], st);
  // L2T (one surface per leaf): 128-thread CTAs, target groups from 8 lanes;
  // M2T (many small W-list surfaces per leaf): 192-thread CTAs, groups from
  // 32 lanes -- the choices that measured fastest on B200
  auto e2t = [&](int own, int far, cudaStream_t se) {
    const int nr = far ? (int)P.farLeaves.size() : (int)P.l2tLeaves.size();
    const int32_t* rows = far ? D.farLeaves : D.l2tLeaves;
    if (nr == 0) return;
    constexpr int KM = kernel_mm(KT) < 0 ? KT : kernel_mm(KT);  // the equivalent kernel of KT (301 is its own)
    const int64_t partStride = std::max<int64_t>(D.m2tPartTargets, 1) * P.tdm;
    if (far) {
      k_e2t32<KM, KB, MX_THREADS_FAR><<<dim3(D.nM2tItems, kb), MX_THREADS_FAR, 0, se>>>(
          rows, D.farPtr, D.farIdx, own, far, D.depth, D.ctr, D.rad, D.sam[0], P.nUE, D.sam[2], P.nDE, D.uden32,
          D.dden32, nn * ue, nn * de, D.trgBeg, D.trgCnt, D.trg, D.valK, valStride, kc, mu, ve, 32, D.m2tItems,
          D.m2tPart, partStride);
      ls->launches++;
      if (D.nM2tSplit > 0) {
        k_e2t_combine<<<D.nM2tSplit, 256, 0, se>>>(D.nM2tSplit, D.m2tSplitLeaf, D.m2tSplitBase, D.m2tSplitCnt,
                                                    D.trgBeg, D.trgCnt, P.tdm, D.m2tPart, partStride, D.valK,
                                                    valStride, kc);
        ls->launches++;
      }
    } else {
      const size_t smem = (size_t)P.nDE * sizeof(float4) + (size_t)L2T_WARPS * P.nDE * KB * P.sdm * sizeof(float);
      cudaFuncSetAttribute(k_l2t32w<KM, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_l2t32w<KM, KB><<<dim3((nr + L2T_WARPS - 1) / L2T_WARPS, kb), 32 * L2T_WARPS, smem, se>>>(
          nr, rows, D.ctr, D.rad, D.sam[2], P.nDE, D.dden32, nn * de, D.trgBeg, D.trgCnt, D.trg, D.valK, valStride,
          kc, mu, ve);
      ls->launches++;
    }
  };
  if (mask & 8) e2t(0, 1, ovl ? D.side : st);
  if (ovl) cudaEventRecord(D.evSide, D.side);
  cudaEventRecord(D.ev[EV_M2T], st);
  if ((mask & 16) && !P.s2lNodes.empty()) {
    k_src2surf32<KT, KB><<<dim3((unsigned)P.s2lNodes.size(), kb), mx_surf_threads(P.nDC), 0, st>>>(
        D.s2lNodes, D.s2lPtr, D.s2lIdx, D.srcBeg, D.srcCnt, D.src, D.nrm, D.den32, den32Blk, D.ctr, D.rad, D.sam[3],
        P.nDC, D.dchk32, dc, nn * dc, kc, mu, ve, 0);
    ls->launches++;
  }
  cudaEventRecord(D.ev[EV_S2L], st);
  if (mask & 32) {
    for (int d = 2; d <= P.maxDepth; d++) {
      if (d >= 3) {
        int64_t a = D.offDnL2L[d - 1], b = D.offDnL2L[d];
        gemm((int)(b - a), D.levelRows + a, 0, 1, D.dden32, de, nn * de, D.l2l32, D.tL2L, D.dchk32, dc, nn * dc, de, 8 * dc,
             level_scale(P, d - 1 + rl, +1.0), unit_scale(), 1.f, D.cL2L);
      }
      int64_t a = D.offDnC2E[d], b = D.offDnC2E[d + 1];
      gemm((int)(b - a), D.levelRows + a, 0, 0, D.dchk32, dc, nn * dc, D.dnF1, D.tDnF1, D.dnT32, kDn4, nn * kDn4, dc,
           kDn4, unit_scale(), unit_scale(), 0.f, D.cDnF1);
      gemm((int)(b - a), D.levelRows + a, 0, 0, D.dnT32, kDn4, nn * kDn4, D.dnF2, D.tDnF2, D.dden32, de, nn * de, kDn4,
           de, unit_scale(), level_scale(P, d + rl, -1.0), 0.f, D.cDnF2);
    }
  }
  cudaEventRecord(D.ev[EV_DN_GEMM], st);
  if (ovl) cudaStreamWaitEvent(st, D.evSide, 0);  // join: the target values are complete but for L2T
  if (mask & 32) e2t(1, 0, st);
  cudaEventRecord(D.ev[EV_L2T], st);
}

// blocks of KB right-hand sides; vector targets take at most 4 a block (pick_kb
// never asks for more), so those instantiations are never built
template <int KT, int KB>
static void run_mixed(const Plan& P, DevState& D, int kc, int mask, bool overlap, LaunchStats* ls) {
  if constexpr (KTraits<KT>::TD != 1 && KB > 4)
    run_mixed_blocks<KT, 4>(P, D, kc, mask, overlap, ls);
  else
    run_mixed_blocks<KT, KB>(P, D, kc, mask, overlap, ls);
}

// the densities of a pass in source (leaf) order: FP64 [rhs][n][sd] in out, and
// the FP32 copy the pair kernels stage, den32[rhs / 8][n][8][sd], each source's
// block of 8 right-hand sides contiguous (zeros past the last right-hand side)
__global__ void k_gather_den_k(int64_t n, int sd, int kc, int64_t stride, const int64_t* __restrict__ perm,
                               const double* __restrict__ in, double* __restrict__ out, float* __restrict__ den32) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = perm[i];
  const int kc8 = (kc + 7) & ~7;
  for (int q = 0; q < kc8; q++)
    for (int c = 0; c < sd; c++) {
      const double v = q < kc ? in[q * stride + s * sd + c] : 0.0;
      if (q < kc) out[q * stride + i * sd + c] = v;
      den32[((int64_t)(q >> 3) * n + i) * 8 * sd + (q & 7) * sd + c] = (float)v;
    }
}
__global__ void k_scatter_val_k(int64_t n, int td, int kc, int64_t stride, const int64_t* __restrict__ perm,
                                const double* __restrict__ in, double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t t = perm[i];
  for (int q = 0; q < kc; q++)
    for (int c = 0; c < td; c++) out[q * stride + t * td + c] = in[q * stride + i * td + c];
}

// right-hand sides per launch block: up to 8 for scalar targets, 4 otherwise
static int pick_kb(int kc, int td) {
  int cap = td == 1 ? 8 : 4;
  int kb = 1;
  while (kb * 2 <= std::min(kc, cap)) kb *= 2;
  return kb;
}

std::string dev_wait_selftest(int device, int arrive, long long limitNs, int* flag) {
  *flag = 0;
  FMMG_CK(cudaSetDevice(device));
  int* d = nullptr;
  FMMG_CK(cudaMalloc(&d, sizeof(int)));
  cudaError_t e = cudaMemset(d, 0, sizeof(int));
  if (e == cudaSuccess) {
    k_wait_selftest<<<1, TC_THREADS>>>(arrive, limitNs, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(flag, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return std::string("wait self-test: ") + cudaGetErrorString(e);
  return std::string();
}

std::string dev_evaluate_mixed(const Plan& P, DevState& D, const double* dDen, double* dVal, int k, int mask,
                               bool timed, LaunchStats* lsIn) {
  LaunchStats local;
  LaunchStats* ls = lsIn ? lsIn : &local;
  FMMG_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  const int64_t ns = P.ns, nt = P.nt;
  const int64_t ue = (int64_t)P.nUE * P.sdm, uc = (int64_t)P.nUC * P.tdm;
  const int64_t de = (int64_t)P.nDE * P.sdm, dc = (int64_t)P.nDC * P.tdm;
  // right-hand sides per pass, bounded by a device-memory budget for the
  // per-density work arrays (node rows and M2L spectra)
  const double perRhs = 4.0 * P.nn * (ue + uc + de + dc + pad4(P.kUp) + pad4(P.kDn)) +
                        8.0 * P.nEff32 * (P.vSrcNodes.size() * P.sdm + P.vTrgNodes.size() * P.tdm) +
                        8.0 * (ns * P.sd + nt * P.td);
  // the budget: at most mixedBudgetBytes and 70% of the free device memory;
  // arrays already held for mixedK right-hand sides are reused as they are.
  // The pass size of a k is fixed by its first call (a graph capture of a
  // later call queries nothing).
  int kc = 0;
  if (D.mixedReady && k <= D.mixedK) {
    kc = k;
  } else if (D.mixedReady && k == D.mixedPassFor) {
    kc = D.mixedPassK;
  } else {
    size_t freeB = 0, totalB = 0;
    FMMG_CK(cudaMemGetInfo(&freeB, &totalB));
    for (const DevState::Block& b : D.spare) freeB += b.bytes;  // the previous setup's blocks are this handle's
    const double budget = std::min(D.mixedBudgetBytes, 0.7 * (double)freeB);
    int kmax = std::max(D.mixedReady ? D.mixedK : 0, (int)std::floor(budget / std::max(perRhs, 1.0)));
    kmax = std::max(1, std::min(kmax, 32));
    // several passes: a whole number of launch blocks (8 right-hand sides for
    // scalar targets, 4 otherwise) per pass, so no block runs part-empty
    const int blk = P.td == 1 ? 8 : 4;
    if (k > kmax && kmax > blk) kmax -= kmax % blk;
    kc = std::min(k, kmax);
    D.mixedPassFor = k;
    D.mixedPassK = kc;
  }
  FMMG_TRY(dev_prepare_mixed(P, D, kc));
  const int64_t denStride = ns * P.sd, valStride = std::max<int64_t>(nt, 1) * P.td;
  int passes = 0;
  for (int r0 = 0; r0 < k; r0 += kc, passes++) {
    const int kk = std::min(kc, k - r0);
    cudaEventRecord(D.ev[EV_BEGIN], st);
    k_gather_den_k<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(ns, P.sd, kk, denStride, D.srcPerm,
                                                                  dDen + r0 * denStride, D.denK, D.den32);
    ls->launches++;
    // Cleared per pass: the accumulated target values and downward check
    // potentials.  The upward C2E reads only the check rows of leaves with
    // sources, which S2M assigns; the upward densities of the nodes with
    // sources are assigned (leaf C2E, the folded product for parents) and the
    // others stay zero from allocation; every downward density that L2L or
    // L2T reads is assigned by C2E at its level before.  With the upward stage
    // masked off the densities are cleared so the V and W stages see zeros.
    FMMG_CK(cudaMemsetAsync(D.valK, 0, sizeof(double) * kk * valStride, st));
    FMMG_CK(cudaMemsetAsync(D.dchk32, 0, sizeof(float) * kk * P.nn * dc, st));
    if (!(mask & 1)) FMMG_CK(cudaMemsetAsync(D.uden32, 0, sizeof(float) * kk * P.nn * ue, st));
    cudaEventRecord(D.ev[EV_PREP], st);
    const int KBv = pick_kb(kk, P.td);
#define FMMG_RUN_KB(KBC) FMMG_DISPATCH_KT(P.o.kt, KT, run_mixed<KT, KBC>(P, D, kk, mask, !timed, ls))
    if (KBv == 8) { FMMG_RUN_KB(8); }
    else if (KBv == 4) { FMMG_RUN_KB(4); }
    else if (KBv == 2) { FMMG_RUN_KB(2); }
    else { FMMG_RUN_KB(1); }
#undef FMMG_RUN_KB
    if (nt > 0) {
      k_scatter_val_k<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nt, P.td, kk, valStride, D.trgPerm, D.valK,
                                                                     dVal + r0 * valStride);
      ls->launches++;
    }
    cudaEventRecord(D.ev[EV_END], st);
  }
  D.lastLaunches = ls->launches;
  FMMG_CK(cudaGetLastError());
  if (timed) {
    FMMG_CK(cudaEventSynchronize(D.ev[EV_END]));
    for (int q = 0; q < EV_COUNT - 1; q++) cudaEventElapsedTime(&D.kernMs[q], D.ev[q], D.ev[q + 1]);
    const float* m = D.kernMs;
    D.stageMs[0] = m[EV_S2M - 1] + m[EV_UP_GEMM - 1];
    D.stageMs[1] = m[EV_NEAR - 1];
    D.stageMs[2] = m[EV_M2L_FWD - 1] + m[EV_M2L_HAD - 1] + m[EV_M2L_INV - 1];
    D.stageMs[3] = m[EV_M2T - 1];
    D.stageMs[4] = m[EV_S2L - 1];
    D.stageMs[5] = m[EV_DN_GEMM - 1] + m[EV_L2T - 1];
    cudaEventElapsedTime(&D.stageMs[6], D.ev[EV_BEGIN], D.ev[EV_END]);
  }
  (void)passes;
  return std::string();
}

}  // namespace fmmg
