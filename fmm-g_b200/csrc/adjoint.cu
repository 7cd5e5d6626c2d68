// adjoint.cu -- the transposed FMM and target-position gradients (FP64).
//
// For the linear map phi = A sigma computed by evaluate() (fmm3d_eval_mpi.cpp
// :396-1515) this file computes g = A^T w exactly, stage by stage in reverse
// order, each stage replaced by its transpose:
//   L2T^T (targets -> DE surface), downward C2E^T and L2L^T per level
//   (transposed operator tables), S2L^T (DC surface -> sources), M2T^T
//   (targets -> UE surface of W nodes), M2L^T (the same spectral step with
//   conjugated translation spectra on the inverted V-lists), near-field
//   P2P^T (targets -> sources), upward C2E^T and M2M^T per level, S2M^T
//   (UC surface -> sources).
// The direct sums use the transposed kernel block K(x_t - y_s; n_s)^T, so the
// source normal stays attached to the output point.  The target-position
// gradient of <w, A sigma> (sources fixed) is the kernel gradient applied in
// the near-field, L2T and M2T sums of a forward evaluate.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cuda_common.cuh"
#include "engine.hpp"
#include "kernels.hpp"

namespace fmmg {

constexpr int AJ_THREADS = 128;
constexpr int AJ_TILE = 128;
constexpr int AJ_MAXE = 256;

__device__ __forceinline__ int aj_load_entries(const int32_t* __restrict__ idx, int64_t ec, int ne, int self,
                                               const int64_t* __restrict__ beg, const int64_t* __restrict__ cnt,
                                               int64_t* eBeg, int32_t* ePre) {
  __syncthreads();
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    int s = idx ? idx[ec + e] : self;
    eBeg[e] = beg[s];
    ePre[e + 1] = (int32_t)cnt[s];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ePre[0] = 0;
    for (int e = 0; e < ne; e++) ePre[e + 1] += ePre[e];
  }
  __syncthreads();
  return ePre[ne];
}

__device__ __forceinline__ int64_t aj_entry(int j, int ne, const int64_t* eBeg, const int32_t* ePre) {
  int lo = 0, hi = ne;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (ePre[mid] <= j) lo = mid; else hi = mid;
  }
  return eBeg[lo] + (j - ePre[lo]);
}

// acc[c] += sum_t K[t][c] w[t]  (transposed block; n is the output point's normal)
template <int KT>
__device__ __forceinline__ void kaccum_t(double x, double y, double z, const double* n, const double* w,
                                         double* acc, double mu, double ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  double K[SD * TD];
  if (!kblock<KT, double>(x, y, z, n, K, mu, ve)) return;
#pragma unroll
  for (int c = 0; c < SD; c++) {
    double s = 0;
#pragma unroll
    for (int t = 0; t < TD; t++) s += K[t * SD + c] * w[t];
    acc[c] += s;
  }
}

// Points -> points, transposed (near-field P2P^T): for one source leaf (row),
// g[s] += sum over the targets of the leaves listing it of K(x_t - y_s; n_s)^T w_t.
template <int KT>
__global__ void __launch_bounds__(AJ_THREADS)
    k_pp_t(const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
           const int64_t* __restrict__ srcBeg, const int64_t* __restrict__ srcCnt,
           const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt, const double* __restrict__ src,
           const double* __restrict__ nrm, const double* __restrict__ trg, const double* __restrict__ w,
           double* __restrict__ g, double mu, double ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  __shared__ double sPos[AJ_TILE * 3];
  __shared__ double sW[AJ_TILE * TD];
  __shared__ int64_t eBeg[AJ_MAXE];
  __shared__ int32_t ePre[AJ_MAXE + 1];
  __shared__ double sRed[AJ_THREADS * SD];
  const int row = blockIdx.x;
  const int a = rows[row];
  const int64_t ob = srcBeg[a], on = srcCnt[a];
  const int64_t e0 = ptr[row], e1 = ptr[row + 1];
  const int tid = threadIdx.x;
  const int TG = on <= 32 ? 32 : (on <= 64 ? 64 : 128);
  const int S = AJ_THREADS / TG;
  const int tl = tid % TG, sp = tid / TG;
  for (int64_t o0 = 0; o0 < on; o0 += TG) {
    const int64_t o = o0 + tl;
    const bool act = o < on;
    double px = 0, py = 0, pz = 0, n3[3] = {0, 0, 0};
    if (act) {
      px = src[3 * (ob + o)];
      py = src[3 * (ob + o) + 1];
      pz = src[3 * (ob + o) + 2];
      if (NRM)
        for (int d = 0; d < 3; d++) n3[d] = nrm[3 * (ob + o) + d];
    }
    double acc[SD];
#pragma unroll
    for (int c = 0; c < SD; c++) acc[c] = 0.0;
    for (int64_t ec = e0; ec < e1; ec += AJ_MAXE) {
      const int ne = (int)min((int64_t)AJ_MAXE, e1 - ec);
      const int total = aj_load_entries(idx, ec, ne, 0, trgBeg, trgCnt, eBeg, ePre);
      for (int base = 0; base < total; base += AJ_TILE) {
        const int cnt = min(AJ_TILE, total - base);
        __syncthreads();
        for (int i = tid; i < cnt; i += AJ_THREADS) {
          const int64_t t = aj_entry(base + i, ne, eBeg, ePre);
          sPos[3 * i] = trg[3 * t];
          sPos[3 * i + 1] = trg[3 * t + 1];
          sPos[3 * i + 2] = trg[3 * t + 2];
#pragma unroll
          for (int c = 0; c < TD; c++) sW[TD * i + c] = w[t * TD + c];
        }
        __syncthreads();
        if (act)
          for (int i = sp; i < cnt; i += S)
            kaccum_t<KT>(sPos[3 * i] - px, sPos[3 * i + 1] - py, sPos[3 * i + 2] - pz, n3, &sW[TD * i], acc, mu, ve);
      }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < SD; c++) sRed[tid * SD + c] = acc[c];
    __syncthreads();
    if (sp == 0 && act)
#pragma unroll
      for (int c = 0; c < SD; c++) {
        double s = 0;
        for (int k = 0; k < S; k++) s += sRed[(tl + k * TG) * SD + c];
        g[(ob + o) * SD + c] += s;
      }
  }
}

// Points -> equivalent surface of a node, transposed equivalent kernel
// (L2T^T onto the own DE surface with ptr == nullptr, M2T^T onto the UE surface
// of a W node from the targets of the leaves listing it).
constexpr int AJ_PPT = 4;
template <int KM>
__global__ void __launch_bounds__(AJ_THREADS)
    k_pts2surf_t(const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                 const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt,
                 const double* __restrict__ trg, const double* __restrict__ w, const double* __restrict__ ctr,
                 const double* __restrict__ rad, const double* __restrict__ sam, int nSurf, double* __restrict__ out,
                 int64_t ldo, double mu, double ve) {
  constexpr int SD = KTraits<KM>::SD, TD = KTraits<KM>::TD;
  __shared__ double sPos[AJ_TILE * 3];
  __shared__ double sW[AJ_TILE * TD];
  __shared__ int64_t eBeg[AJ_MAXE];
  __shared__ int32_t ePre[AJ_MAXE + 1];
  const int row = blockIdx.x;
  const int g = rows[row];
  const int tid = threadIdx.x;
  const double cx = ctr[3 * g], cy = ctr[3 * g + 1], cz = ctr[3 * g + 2], r = rad[g];
  double px[AJ_PPT], py[AJ_PPT], pz[AJ_PPT], acc[AJ_PPT][SD];
#pragma unroll
  for (int k = 0; k < AJ_PPT; k++) {
    int i = tid + k * AJ_THREADS;
    px[k] = py[k] = pz[k] = 0;
    if (i < nSurf) {
      px[k] = cx + r * sam[3 * i];
      py[k] = cy + r * sam[3 * i + 1];
      pz[k] = cz + r * sam[3 * i + 2];
    }
#pragma unroll
    for (int c = 0; c < SD; c++) acc[k][c] = 0.0;
  }
  const int64_t e0 = ptr ? ptr[row] : 0, e1 = ptr ? ptr[row + 1] : 1;
  for (int64_t ec = e0; ec < e1; ec += AJ_MAXE) {
    const int ne = (int)min((int64_t)AJ_MAXE, e1 - ec);
    const int total = aj_load_entries(ptr ? idx : nullptr, ec, ne, g, trgBeg, trgCnt, eBeg, ePre);
    for (int base = 0; base < total; base += AJ_TILE) {
      const int cnt = min(AJ_TILE, total - base);
      __syncthreads();
      for (int i = tid; i < cnt; i += AJ_THREADS) {
        const int64_t t = aj_entry(base + i, ne, eBeg, ePre);
        sPos[3 * i] = trg[3 * t];
        sPos[3 * i + 1] = trg[3 * t + 1];
        sPos[3 * i + 2] = trg[3 * t + 2];
#pragma unroll
        for (int c = 0; c < TD; c++) sW[TD * i + c] = w[t * TD + c];
      }
      __syncthreads();
      for (int i = 0; i < cnt; i++)
#pragma unroll
        for (int k = 0; k < AJ_PPT; k++)
          if (tid + k * AJ_THREADS < nSurf)
            kaccum_t<KM>(sPos[3 * i] - px[k], sPos[3 * i + 1] - py[k], sPos[3 * i + 2] - pz[k], nullptr,
                         &sW[TD * i], acc[k], mu, ve);
    }
  }
#pragma unroll
  for (int k = 0; k < AJ_PPT; k++) {
    int i = tid + k * AJ_THREADS;
    if (i < nSurf)
#pragma unroll
      for (int c = 0; c < SD; c++) out[(int64_t)g * ldo + (int64_t)i * SD + c] += acc[k][c];
  }
}

// Check surface -> points, transposed true kernel: S2L^T (DC surfaces of the
// nodes listing the row leaf) and S2M^T (own UC surface, ptr == nullptr).
template <int KT>
__global__ void __launch_bounds__(AJ_THREADS)
    k_surf2pts_t(const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                 const int64_t* __restrict__ srcBeg, const int64_t* __restrict__ srcCnt,
                 const double* __restrict__ src, const double* __restrict__ nrm, const double* __restrict__ ctr,
                 const double* __restrict__ rad, const double* __restrict__ sam, int nSurf,
                 const double* __restrict__ gchk, int64_t ldc, double* __restrict__ g, double mu, double ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  __shared__ double sPos[AJ_TILE * 3];
  __shared__ double sW[AJ_TILE * TD];
  __shared__ double sRed[AJ_THREADS * SD];
  const int row = blockIdx.x;
  const int a = rows[row];
  const int64_t ob = srcBeg[a], on = srcCnt[a];
  const int tid = threadIdx.x;
  const int TG = on <= 32 ? 32 : (on <= 64 ? 64 : 128);
  const int S = AJ_THREADS / TG;
  const int tl = tid % TG, sp = tid / TG;
  const int64_t e0 = ptr ? ptr[row] : 0, ne = ptr ? ptr[row + 1] - e0 : 1;
  for (int64_t o0 = 0; o0 < on; o0 += TG) {
    const int64_t o = o0 + tl;
    const bool act = o < on;
    double px = 0, py = 0, pz = 0, n3[3] = {0, 0, 0};
    if (act) {
      px = src[3 * (ob + o)];
      py = src[3 * (ob + o) + 1];
      pz = src[3 * (ob + o) + 2];
      if (NRM)
        for (int d = 0; d < 3; d++) n3[d] = nrm[3 * (ob + o) + d];
    }
    double acc[SD];
#pragma unroll
    for (int c = 0; c < SD; c++) acc[c] = 0.0;
    for (int64_t e = 0; e < ne; e++) {
      const int node = ptr ? idx[e0 + e] : a;
      const double cx = ctr[3 * node], cy = ctr[3 * node + 1], cz = ctr[3 * node + 2], r = rad[node];
      const double* gc = gchk + (int64_t)node * ldc;
      for (int base = 0; base < nSurf; base += AJ_TILE) {
        const int cnt = min(AJ_TILE, nSurf - base);
        __syncthreads();
        for (int i = tid; i < cnt; i += AJ_THREADS) {
          const int j = base + i;
          sPos[3 * i] = cx + r * sam[3 * j];
          sPos[3 * i + 1] = cy + r * sam[3 * j + 1];
          sPos[3 * i + 2] = cz + r * sam[3 * j + 2];
#pragma unroll
          for (int c = 0; c < TD; c++) sW[TD * i + c] = gc[(int64_t)j * TD + c];
        }
        __syncthreads();
        if (act)
          for (int i = sp; i < cnt; i += S)
            kaccum_t<KT>(sPos[3 * i] - px, sPos[3 * i + 1] - py, sPos[3 * i + 2] - pz, n3, &sW[TD * i], acc, mu, ve);
      }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < SD; c++) sRed[tid * SD + c] = acc[c];
    __syncthreads();
    if (sp == 0 && act)
#pragma unroll
      for (int c = 0; c < SD; c++) {
        double s = 0;
        for (int k = 0; k < S; k++) s += sRed[(tl + k * TG) * SD + c];
        g[(ob + o) * SD + c] += s;
      }
  }
}

// Multi-DOF transposed Hadamard step on the V-lists inverted per source slot:
// out[s][f][j] = nrmfc * sum_{(t, id)} sum_i conj(T[id][f][j*TDM + i]) in[t][f][i].
// A warp owns one source slot and 32 frequencies (lane = frequency).
template <int SDM, int TDM>
__global__ void __launch_bounds__(256)
    k_m2l_had_t(int nOut, const int64_t* __restrict__ lptr, const int2* __restrict__ lent,
                const double2* __restrict__ in, const double2* __restrict__ T, double2* __restrict__ out, int nEff,
                double nrmfc) {
  const int s = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int f = blockIdx.y * 32 + (threadIdx.x & 31);
  if (s >= nOut || f >= nEff) return;
  double2 acc[SDM];
#pragma unroll
  for (int j = 0; j < SDM; j++) acc[j] = make_double2(0, 0);
  for (int64_t e = lptr[s]; e < lptr[s + 1]; e++) {
    const int2 en = lent[e];
    double2 d[TDM];
#pragma unroll
    for (int i = 0; i < TDM; i++) d[i] = in[((int64_t)en.x * nEff + f) * TDM + i];
    const double2* Tf = T + ((int64_t)en.y * nEff + f) * (SDM * TDM);
#pragma unroll
    for (int j = 0; j < SDM; j++)
#pragma unroll
      for (int i = 0; i < TDM; i++) {
        const double2 tv = Tf[j * TDM + i];  // conj(tv) * d[i]
        acc[j].x += tv.x * d[i].x + tv.y * d[i].y;
        acc[j].y += tv.x * d[i].y - tv.y * d[i].x;
      }
  }
#pragma unroll
  for (int j = 0; j < SDM; j++)
    out[((int64_t)s * nEff + f) * SDM + j] = make_double2(acc[j].x * nrmfc, acc[j].y * nrmfc);
}

// Gradient of a scalar kernel with respect to the target position:
// G[d] = dK/dx_d at the offset (x, y, z) = target - source.
template <int KT>
__device__ __forceinline__ bool kgrad(double x, double y, double z, const double* n, double* G) {
  const double r2 = x * x + y * y + z * z;
  if (r2 < 1e-16) return false;
  const double ir = rsqrt(r2);
  const double ir3 = ir * ir * ir;
  constexpr double C = 1.0 / (4.0 * 3.14159265358979323846);
  if constexpr (KT == LAP_S_U) {  // K = C / r
    G[0] = -C * ir3 * x;
    G[1] = -C * ir3 * y;
    G[2] = -C * ir3 * z;
  } else {  // LAP_D_U: K = -C (d.n) / r^3
    const double rn = x * n[0] + y * n[1] + z * n[2];
    const double ir5 = ir3 * ir * ir;
    G[0] = -C * (n[0] * ir3 - 3.0 * rn * ir5 * x);
    G[1] = -C * (n[1] * ir3 - 3.0 * rn * ir5 * y);
    G[2] = -C * (n[2] * ir3 - 3.0 * rn * ir5 * z);
  }
  return true;
}

// Near-field part of the target gradient: for one evaluator leaf,
// grad[t] += w[t] * sum_s grad_x K(x_t - y_s; n_s) den[s] over its near list.
template <int KT>
__global__ void __launch_bounds__(AJ_THREADS)
    k_grad_near(const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                const int64_t* __restrict__ srcBeg, const int64_t* __restrict__ srcCnt,
                const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt,
                const double* __restrict__ src, const double* __restrict__ nrm, const double* __restrict__ den,
                const double* __restrict__ trg, const double* __restrict__ w, double* __restrict__ grad) {
  constexpr int NRM = KTraits<KT>::NRM;
  __shared__ double sPos[AJ_TILE * 3];
  __shared__ double sNrm[NRM ? AJ_TILE * 3 : 1];
  __shared__ double sDen[AJ_TILE];
  __shared__ int64_t eBeg[AJ_MAXE];
  __shared__ int32_t ePre[AJ_MAXE + 1];
  __shared__ double sRed[AJ_THREADS * 3];
  const int row = blockIdx.x;
  const int g = rows[row];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const int64_t e0 = ptr[row], e1 = ptr[row + 1];
  const int tid = threadIdx.x;
  const int TG = tn <= 32 ? 32 : (tn <= 64 ? 64 : 128);
  const int S = AJ_THREADS / TG;
  const int tl = tid % TG, sp = tid / TG;
  for (int64_t t0 = 0; t0 < tn; t0 += TG) {
    const int64_t t = t0 + tl;
    const bool act = t < tn;
    double tx = 0, ty = 0, tz = 0;
    if (act) {
      tx = trg[3 * (tb + t)];
      ty = trg[3 * (tb + t) + 1];
      tz = trg[3 * (tb + t) + 2];
    }
    double acc[3] = {0, 0, 0};
    for (int64_t ec = e0; ec < e1; ec += AJ_MAXE) {
      const int ne = (int)min((int64_t)AJ_MAXE, e1 - ec);
      const int total = aj_load_entries(idx, ec, ne, 0, srcBeg, srcCnt, eBeg, ePre);
      for (int base = 0; base < total; base += AJ_TILE) {
        const int cnt = min(AJ_TILE, total - base);
        __syncthreads();
        for (int i = tid; i < cnt; i += AJ_THREADS) {
          const int64_t s = aj_entry(base + i, ne, eBeg, ePre);
          sPos[3 * i] = src[3 * s];
          sPos[3 * i + 1] = src[3 * s + 1];
          sPos[3 * i + 2] = src[3 * s + 2];
          if (NRM) {
            sNrm[3 * i] = nrm[3 * s];
            sNrm[3 * i + 1] = nrm[3 * s + 1];
            sNrm[3 * i + 2] = nrm[3 * s + 2];
          }
          sDen[i] = den[s];
        }
        __syncthreads();
        if (act)
          for (int i = sp; i < cnt; i += S) {
            double G[3];
            if (kgrad<KT>(tx - sPos[3 * i], ty - sPos[3 * i + 1], tz - sPos[3 * i + 2], NRM ? &sNrm[3 * i] : nullptr,
                          G)) {
              acc[0] += G[0] * sDen[i];
              acc[1] += G[1] * sDen[i];
              acc[2] += G[2] * sDen[i];
            }
          }
      }
    }
    __syncthreads();
    for (int d = 0; d < 3; d++) sRed[tid * 3 + d] = acc[d];
    __syncthreads();
    if (sp == 0 && act) {
      const double wt = w[tb + t];
      for (int d = 0; d < 3; d++) {
        double s = 0;
        for (int k = 0; k < S; k++) s += sRed[(tl + k * TG) * 3 + d];
        grad[(tb + t) * 3 + d] += wt * s;
      }
    }
  }
}

// Far-field part of the target gradient through the equivalent densities
// (Laplace single-layer equivalent kernel): the leaf's own DE surface (L2T)
// and the UE surfaces of its W nodes (M2T).
__global__ void __launch_bounds__(AJ_THREADS)
    k_grad_e2t(const int32_t* __restrict__ rows, const int64_t* __restrict__ farPtr,
               const int32_t* __restrict__ farIdx, int useOwn, int useFar, const int32_t* __restrict__ depth,
               const double* __restrict__ ctr, const double* __restrict__ rad, const double* __restrict__ samUE,
               int nUE, const double* __restrict__ samDE, int nDE, const double* __restrict__ uden,
               const double* __restrict__ dden, const int64_t* __restrict__ trgBeg,
               const int64_t* __restrict__ trgCnt, const double* __restrict__ trg, const double* __restrict__ w,
               double* __restrict__ grad) {
  __shared__ double sPos[AJ_TILE * 3];
  __shared__ double sDen[AJ_TILE];
  __shared__ double sRed[AJ_THREADS * 3];
  const int row = blockIdx.x;
  const int g = rows[row];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const int tid = threadIdx.x;
  const int TG = tn <= 32 ? 32 : (tn <= 64 ? 64 : 128);
  const int S = AJ_THREADS / TG;
  const int tl = tid % TG, sp = tid / TG;
  const int own = (useOwn && depth[g] >= 2) ? 1 : 0;
  const int64_t f0 = useFar ? farPtr[row] : 0, nf = useFar ? farPtr[row + 1] - f0 : 0;
  for (int64_t t0 = 0; t0 < tn; t0 += TG) {
    const int64_t t = t0 + tl;
    const bool act = t < tn;
    double tx = 0, ty = 0, tz = 0;
    if (act) {
      tx = trg[3 * (tb + t)];
      ty = trg[3 * (tb + t) + 1];
      tz = trg[3 * (tb + t) + 2];
    }
    double acc[3] = {0, 0, 0};
    for (int64_t e = 0; e < own + nf; e++) {
      const bool isOwn = e < own;
      const int node = isOwn ? g : farIdx[f0 + e - own];
      const double* sam = isOwn ? samDE : samUE;
      const int ns = isOwn ? nDE : nUE;
      const double* dsrc = isOwn ? dden + (int64_t)node * ns : uden + (int64_t)node * ns;
      const double cx = ctr[3 * node], cy = ctr[3 * node + 1], cz = ctr[3 * node + 2], r = rad[node];
      for (int base = 0; base < ns; base += AJ_TILE) {
        const int cnt = min(AJ_TILE, ns - base);
        __syncthreads();
        for (int i = tid; i < cnt; i += AJ_THREADS) {
          const int j = base + i;
          sPos[3 * i] = cx + r * sam[3 * j];
          sPos[3 * i + 1] = cy + r * sam[3 * j + 1];
          sPos[3 * i + 2] = cz + r * sam[3 * j + 2];
          sDen[i] = dsrc[j];
        }
        __syncthreads();
        if (act)
          for (int i = sp; i < cnt; i += S) {
            double G[3];
            if (kgrad<LAP_S_U>(tx - sPos[3 * i], ty - sPos[3 * i + 1], tz - sPos[3 * i + 2], nullptr, G)) {
              acc[0] += G[0] * sDen[i];
              acc[1] += G[1] * sDen[i];
              acc[2] += G[2] * sDen[i];
            }
          }
      }
    }
    __syncthreads();
    for (int d = 0; d < 3; d++) sRed[tid * 3 + d] = acc[d];
    __syncthreads();
    if (sp == 0 && act) {
      const double wt = w[tb + t];
      for (int d = 0; d < 3; d++) {
        double s = 0;
        for (int k = 0; k < S; k++) s += sRed[(tl + k * TG) * 3 + d];
        grad[(tb + t) * 3 + d] += wt * s;
      }
    }
  }
}

// ------------------------------------------------------------------ host side
template <typename T>
static std::string aj_put(DevState& D, T*& dst, const T* src, size_t n) {
  if (n == 0) {
    dst = nullptr;
    return std::string();
  }
  if (!dst) {
    void* p = nullptr;
    cudaError_t e = dev_alloc(D, &p, n * sizeof(T));
    if (e != cudaSuccess) return std::string("cudaMalloc: ") + cudaGetErrorString(e);
    dst = (T*)p;
  }
  if (src) FMMG_CK(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return std::string();
}

// W is N x K row-major; returns W^T (K x N row-major)
static std::vector<double> transposed(const std::vector<double>& W, int N, int K) {
  std::vector<double> T((size_t)N * K);
  for (int n = 0; n < N; n++)
    for (int k = 0; k < K; k++) T[(size_t)k * N + n] = W[(size_t)n * K + k];
  return T;
}

static std::string adj_prepare(const Plan& P, DevState& D) {
  P.build_adjoint_lists();
  if (!(P.sdm == 1 && P.tdm == 1 && D.hadPQ)) FMMG_TRY(dev_upload_vlists(P, D));  // the list-form M2L^T
  if (!D.adjListsReady) {
    FMMG_TRY(aj_put(D, D.adjNearRows, P.adjNearRows.data(), P.adjNearRows.size()));
    FMMG_TRY(aj_put(D, D.adjNearPtr, P.adjNear.ptr.data(), P.adjNear.ptr.size()));
    FMMG_TRY(aj_put(D, D.adjNearIdx, P.adjNear.idx.data(), P.adjNear.idx.size()));
    FMMG_TRY(aj_put(D, D.adjFarRows, P.adjFarRows.data(), P.adjFarRows.size()));
    FMMG_TRY(aj_put(D, D.adjFarPtr, P.adjFar.ptr.data(), P.adjFar.ptr.size()));
    FMMG_TRY(aj_put(D, D.adjFarIdx, P.adjFar.idx.data(), P.adjFar.idx.size()));
    FMMG_TRY(aj_put(D, D.adjS2lRows, P.adjS2lRows.data(), P.adjS2lRows.size()));
    FMMG_TRY(aj_put(D, D.adjS2lPtr, P.adjS2l.ptr.data(), P.adjS2l.ptr.size()));
    FMMG_TRY(aj_put(D, D.adjS2lIdx, P.adjS2l.idx.data(), P.adjS2l.idx.size()));
    FMMG_TRY(aj_put<double>(D, D.gradT, nullptr, 3 * (size_t)std::max<int64_t>(P.nt, 1)));
    FMMG_TRY(aj_put(D, D.vParentsT, P.vParentsT.data(), P.vParentsT.size()));
    FMMG_TRY(aj_put(D, D.vNbrTPtr, P.vNbrT.ptr.data(), P.vNbrT.ptr.size()));
    FMMG_TRY(aj_put(D, D.vNbrTIdx, P.vNbrT.idx.data(), P.vNbrT.idx.size()));
    FMMG_TRY(aj_put(D, D.vNbrOffT, P.vNbrOffT.data(), P.vNbrOffT.size()));
    FMMG_TRY(aj_put(D, D.vRowOutT, P.vRowOutT.data(), P.vRowOutT.size()));
    FMMG_TRY(aj_put(D, D.vNbrInT, P.vNbrInT.data(), P.vNbrInT.size()));
    D.adjListsReady = true;
  }
  if (D.adjOpsStale) {
    const int ue = P.nUE * P.sdm, uc = P.nUC * P.tdm, de = P.nDE * P.sdm, dc = P.nDC * P.tdm;
    std::vector<double> t;
    t = transposed(P.uc2ue, ue, uc);
    FMMG_TRY(aj_put(D, D.uc2ueT, t.data(), t.size()));
    t = transposed(P.m2m, uc, 8 * ue);
    FMMG_TRY(aj_put(D, D.m2mT, t.data(), t.size()));
    t = transposed(P.dc2de, de, dc);
    FMMG_TRY(aj_put(D, D.dc2deT, t.data(), t.size()));
    t = transposed(P.l2l, 8 * dc, de);
    FMMG_TRY(aj_put(D, D.l2lT, t.data(), t.size()));
    D.adjOpsStale = false;
  }
  return std::string();
}

static Scale4 deg_scale(const Plan& P) {  // 2^(l * deg) per equivalent-density component
  Scale4 s;
  s.mod = P.sdm;
  for (int k = 0; k < 4; k++) s.v[k] = k < P.sdm ? P.deg[k] : 0.0;
  return s;
}

// g += A^T w: the forward stages of run_stages in reverse order, each transposed.
// Work arrays: D.val holds w (permuted), D.den accumulates g (permuted), and
// D.uchk / D.uden / D.dchk / D.dden hold the adjoint surface quantities.
template <int KT>
static void run_adjoint(const Plan& P, DevState& D, int& launches) {
  constexpr int KM = KTraits<KT>::MM;
  cudaStream_t st = D.stream;
  const int ue = P.nUE * P.sdm, uc = P.nUC * P.tdm, de = P.nDE * P.sdm, dc = P.nDC * P.tdm;
  const int rl = P.o.rootLevel;
  const double mu = P.o.coefs[0], ve = P.o.coefs[1];
  const double* w = D.val;
  double* g = D.den;
  auto rows_at = [&](const std::vector<int64_t>& off, int d, const int32_t*& rows) {
    rows = D.levelRows + off[d];
    return (int)(off[d + 1] - off[d]);
  };
  // L2T^T: targets -> DE surface of each evaluator leaf at depth >= 2
  if (!P.l2tLeaves.empty()) {
    k_pts2surf_t<KM><<<(unsigned)P.l2tLeaves.size(), AJ_THREADS, 0, st>>>(
        D.l2tLeaves, nullptr, nullptr, D.trgBeg, D.trgCnt, D.trg, w, D.ctr, D.rad, D.sam[2], P.nDE, D.dden, de, mu,
        ve);
    launches++;
  }
  // downward, transposed: C2E^T then L2L^T per level, deepest first
  for (int d = P.maxDepth; d >= 2; d--) {
    const int32_t* rows;
    int n = rows_at(D.offDnC2E, d, rows);
    if (n > 0) {
      gemm_rows(D, n, rows, D.chd, 0, 0, D.dden, de, D.dc2deT, D.dchk, dc, de, dc, level_scale(P, d + rl, -1.0),
                unit_scale(), 0.0, nullptr);
      launches++;
    }
    if (d >= 3) {
      n = rows_at(D.offDnL2L, d - 1, rows);
      if (n > 0) {
        gemm_rows(D, n, rows, D.chd, 1, 0, D.dchk, dc, D.l2lT, D.dden, de, 8 * dc, de, unit_scale(),
                  level_scale(P, d - 1 + rl, +1.0), 1.0, nullptr);
        launches++;
      }
    }
  }
  // S2L^T: DC surfaces -> sources of the X-list leaves
  if (!P.adjS2lRows.empty()) {
    k_surf2pts_t<KT><<<(unsigned)P.adjS2lRows.size(), AJ_THREADS, 0, st>>>(
        D.adjS2lRows, D.adjS2lPtr, D.adjS2lIdx, D.srcBeg, D.srcCnt, D.src, D.nrm, D.ctr, D.rad, D.sam[3], P.nDC,
        D.dchk, dc, g, mu, ve);
    launches++;
  }
  // M2T^T: targets -> UE surfaces of the W nodes evaluated through them
  if (!P.adjFarRows.empty()) {
    k_pts2surf_t<KM><<<(unsigned)P.adjFarRows.size(), AJ_THREADS, 0, st>>>(
        D.adjFarRows, D.adjFarPtr, D.adjFarIdx, D.trgBeg, D.trgCnt, D.trg, w, D.ctr, D.rad, D.sam[0], P.nUE,
        D.uden, ue, mu, ve);
    launches++;
  }
  // M2L^T: r2c of the DC adjoints, conjugated translations on the V-lists
  // inverted per source box, c2r onto the UE surface times 2^(l * deg)
  const int nsrc = (int)P.vSrcNodes.size(), ntrg = (int)P.vTrgNodes.size();
  if (nsrc > 0 && ntrg > 0) {
    Scale4 none;
    none.mod = 1;
    none.v[0] = none.v[1] = none.v[2] = none.v[3] = 0.0;
    spectral_fwd(P, D, ntrg, D.vTrgNodes, none, P.tdm, D.dchk, D.effVal);
    if (P.sdm == 1 && P.tdm == 1 && D.hadPQ) {
      hadamard_pq64_adj(P, D, D.effVal, D.effDen);
    } else if (P.sdm == 1 && P.tdm == 1) {
      hadamard_list64(P, D, nsrc, D.vSrcPtr, D.vSrcEnt, D.effVal, D.effDen, true);
    } else {
      dim3 grid((nsrc + 7) / 8, (P.nEff + 31) / 32);
      const double nrmfc = 1.0 / double(P.nReg);
      if (P.sdm == 4 && P.tdm == 3)
        k_m2l_had_t<4, 3><<<grid, 256, 0, st>>>(nsrc, D.vSrcPtr, (const int2*)D.vSrcEnt, D.effVal, D.m2lT, D.effDen,
                                               P.nEff, nrmfc);
      else
        k_m2l_had_t<3, 3><<<grid, 256, 0, st>>>(nsrc, D.vSrcPtr, (const int2*)D.vSrcEnt, D.effVal, D.m2lT, D.effDen,
                                               P.nEff, nrmfc);
    }
    spectral_inv(P, D, nsrc, D.vSrcNodes, P.sdm, D.effDen, D.uden, deg_scale(P));
    launches += 3;
  }
  // near field, transposed: targets -> sources of the U, direct W and direct X leaves
  if (!P.adjNearRows.empty()) {
    k_pp_t<KT><<<(unsigned)P.adjNearRows.size(), AJ_THREADS, 0, st>>>(D.adjNearRows, D.adjNearPtr, D.adjNearIdx,
                                                                      D.srcBeg, D.srcCnt, D.trgBeg, D.trgCnt, D.src,
                                                                      D.nrm, D.trg, w, g, mu, ve);
    launches++;
  }
  // upward, transposed: C2E^T then M2M^T per level, root side first
  for (int d = 1; d <= P.maxDepth; d++) {
    const int32_t* rows;
    int n = rows_at(D.offUpC2E, d, rows);
    if (n > 0) {
      gemm_rows(D, n, rows, D.chd, 0, 0, D.uden, ue, D.uc2ueT, D.uchk, uc, ue, uc, level_scale(P, d + rl, -1.0),
                unit_scale(), 0.0, nullptr);
      launches++;
    }
    n = rows_at(D.offUpM2M, d, rows);
    if (n > 0) {
      gemm_rows(D, n, rows, D.chd, 0, 1, D.uchk, uc, D.m2mT, D.uden, ue, uc, 8 * ue, unit_scale(),
                level_scale(P, d + 1 + rl, +1.0), 1.0, nullptr);
      launches++;
    }
  }
  // S2M^T: UC surfaces -> the leaf's own sources
  if (!P.s2mLeaves.empty()) {
    k_surf2pts_t<KT><<<(unsigned)P.s2mLeaves.size(), AJ_THREADS, 0, st>>>(
        D.s2mLeaves, nullptr, nullptr, D.srcBeg, D.srcCnt, D.src, D.nrm, D.ctr, D.rad, D.sam[1], P.nUC, D.uchk, uc,
        g, mu, ve);
    launches++;
  }
}

template <int KT>
static void run_target_grad(const Plan& P, DevState& D, int& launches) {
  cudaStream_t st = D.stream;
  if (!P.evtrLeaves.empty()) {
    k_grad_near<KT><<<(unsigned)P.evtrLeaves.size(), AJ_THREADS, 0, st>>>(
        D.evtrLeaves, D.nearPtr, D.nearIdx, D.srcBeg, D.srcCnt, D.trgBeg, D.trgCnt, D.src, D.nrm, D.den, D.trg,
        D.val, D.gradT);
    launches++;
  }
  if (!P.l2tLeaves.empty()) {
    k_grad_e2t<<<(unsigned)P.l2tLeaves.size(), AJ_THREADS, 0, st>>>(
        D.l2tLeaves, D.farPtr, D.farIdx, 1, 0, D.depth, D.ctr, D.rad, D.sam[0], P.nUE, D.sam[2], P.nDE, D.uden,
        D.dden, D.trgBeg, D.trgCnt, D.trg, D.val, D.gradT);
    launches++;
  }
  if (!P.farLeaves.empty()) {
    k_grad_e2t<<<(unsigned)P.farLeaves.size(), AJ_THREADS, 0, st>>>(
        D.farLeaves, D.farPtr, D.farIdx, 0, 1, D.depth, D.ctr, D.rad, D.sam[0], P.nUE, D.sam[2], P.nDE, D.uden,
        D.dden, D.trgBeg, D.trgCnt, D.trg, D.val, D.gradT);
    launches++;
  }
}

std::string dev_adjoint(const Plan& P, DevState& D, const double* dDen, const double* dW, double* dG,
                        double* dGradT, bool timed) {
  FMMG_CK(cudaSetDevice(D.device));
  if (P.mm != LAP_S_U && P.mm != STK_F_U && P.mm != NAV_S_U) return "adjoint: unsupported kernel";
  if (dGradT && P.o.kt != LAP_S_U && P.o.kt != LAP_D_U)
    return "target-position gradient is implemented for the Laplace kernels 111 and 121";
  if (dGradT && !dDen) return "target-position gradient needs the source density";
  FMMG_TRY(adj_prepare(P, D));
  cudaStream_t st = D.stream;
  const int ue = P.nUE * P.sdm, uc = P.nUC * P.tdm, de = P.nDE * P.sdm, dc = P.nDC * P.tdm;
  int launches = 0;
  if (timed) cudaEventRecord(D.ev[EV_BEGIN], st);
  if (dGradT) {
    FMMG_TRY(dev_far_field(P, D, dDen));
    gather_rows(st, P.nt, P.td, D.trgPerm, dW, D.val);
    FMMG_CK(cudaMemsetAsync(D.gradT, 0, sizeof(double) * 3 * (size_t)std::max<int64_t>(P.nt, 1), st));
    if (P.o.kt == LAP_S_U) run_target_grad<LAP_S_U>(P, D, launches);
    else run_target_grad<LAP_D_U>(P, D, launches);
    scatter_rows(st, P.nt, 3, D.trgPerm, D.gradT, dGradT);
  }
  if (dG) {
    gather_rows(st, P.nt, P.td, D.trgPerm, dW, D.val);
    FMMG_CK(cudaMemsetAsync(D.den, 0, sizeof(double) * (size_t)std::max<int64_t>(P.ns, 1) * P.sd, st));
    FMMG_CK(cudaMemsetAsync(D.uchk, 0, sizeof(double) * (size_t)P.nn * uc, st));
    FMMG_CK(cudaMemsetAsync(D.uden, 0, sizeof(double) * (size_t)P.nn * ue, st));
    FMMG_CK(cudaMemsetAsync(D.dchk, 0, sizeof(double) * (size_t)P.nn * dc, st));
    FMMG_CK(cudaMemsetAsync(D.dden, 0, sizeof(double) * (size_t)P.nn * de, st));
    FMMG_DISPATCH_KT(P.o.kt, KT, run_adjoint<KT>(P, D, launches));
    scatter_rows(st, P.ns, P.sd, D.srcPerm, D.den, dG);
  }
  FMMG_CK(cudaGetLastError());
  D.lastLaunches = launches;
  if (timed) {
    cudaEventRecord(D.ev[EV_END], st);
    FMMG_CK(cudaEventSynchronize(D.ev[EV_END]));
    cudaEventElapsedTime(&D.adjMs, D.ev[EV_BEGIN], D.ev[EV_END]);
  }
  return std::string();
}

}  // namespace fmmg
