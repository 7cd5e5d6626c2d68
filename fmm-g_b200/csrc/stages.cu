// stages.cu -- sm_100a kernels for every stage of evaluate() and the launcher.
//
// Stage map (reference fmm3d_mpi/fmm3d_eval_mpi.cpp):
//   upward  :557-595  S2M (k_src2surf on each leaf's UC surface), then per level
//                     M2M + C2E as batched row GEMMs (k_gemm_rows)
//   U-list  :773-785  k_p2p_near_w (true kernel, sources of adjacent leaves)
//   V-list  :1015-1051 k_m2l_fwd (r2c of each upward density on the (2np)^3
//                     grid), k_m2l_had (per-frequency products grouped by
//                     parent pairs), k_m2l_inv (c2r + gather onto DC)
//   W-list  :1139-1175 S2T entries folded into k_p2p_near_w, M2T in k_e2t
//   X-list  :1241-1257 S2T entries folded into k_p2p_near_w, S2L in k_src2surf
//   downward:1368-1438 per level L2L + C2E row GEMMs, L2T in k_e2t
// Every output row (a leaf's targets, a box's check surface, a node's
// spectrum) is owned by exactly one CTA, so no atomics are needed and the
// stages are plain stream-ordered launches.
#include <stdexcept>
#include <cuda_runtime.h>

#include <chrono>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>

#include "cuda_common.cuh"
#include "engine.hpp"
#include "plan_pool.cuh"
#include "dense_kernel.cuh"
#include "gemm_rows.cuh"
#include "had_pq.cuh"
#include "had_smem.cuh"
#include "kernels.hpp"

namespace fmmg {


__constant__ int16_t c_transId[343];  // (rx+3)*49+(ry+3)*7+(rz+3) -> 0..315 or -1

// ------------------------------------------------------------------ helpers
__global__ void k_gather_den(int64_t n, int sd, const int64_t* __restrict__ perm, const double* __restrict__ in,
                             double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = perm[i];
  for (int c = 0; c < sd; c++) out[i * sd + c] = in[s * sd + c];
}

__global__ void k_scatter_val(int64_t n, int td, const int64_t* __restrict__ perm, const double* __restrict__ in,
                              double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t t = perm[i];
  for (int c = 0; c < td; c++) out[t * td + c] = in[i * td + c];
}

// ------------------------------------------------------------------ near field
// The CTA-per-box FP64 kernels below (k_e2t, k_src2surf) stage their sources
// in tiles of P2P_TILE in shared memory; when a box has few targets the CTA
// splits the tile between thread groups and reduces the partial sums at the
// end.  The near field itself, for one evaluator leaf val[targets] +=
// K(trg, src) den(src) over the source leaves of its near list (U-list,
// direct W and X entries), is k_p2p_near_w: one warp per leaf.
constexpr int P2P_THREADS = 128;
constexpr int P2P_TILE = 128;
constexpr int P2P_MAXE = 256;


// k_p2p_near_w: the same sums, one warp per evaluator leaf (P2PW_WARPS
// leaves a CTA) and no CTA-wide barrier: the warp builds its entry table
// (source ranges and their prefix counts, a shuffle scan per 32 entries),
// stages P2PW_CH sources at a time in its own slice of shared memory, and
// splits them over S = 32 / TG lane groups of TG = 8, 16 or 32 targets; the
// groups' FP64 partial sums meet through warp shuffles.  A leaf with few
// targets no longer leaves most of a CTA idle behind block barriers.
constexpr int P2PW_WARPS = 4, P2PW_CH = 64, P2PW_MAXE = 128;
template <int KT>
__global__ void __launch_bounds__(32 * P2PW_WARPS)
    k_p2p_near_w(int nLeaves, const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr,
                 const int32_t* __restrict__ idx, const int64_t* __restrict__ srcBeg,
                 const int64_t* __restrict__ srcCnt, const int64_t* __restrict__ trgBeg,
                 const int64_t* __restrict__ trgCnt, const double* __restrict__ src, const double* __restrict__ nrm,
                 const double* __restrict__ den, const double* __restrict__ trg, double* __restrict__ val, double mu,
                 double ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  __shared__ double sPos[P2PW_WARPS][P2PW_CH * 3];
  __shared__ double sNrm[P2PW_WARPS][NRM ? P2PW_CH * 3 : 1];
  __shared__ double sDen[P2PW_WARPS][P2PW_CH * SD];
  __shared__ int64_t eBeg[P2PW_WARPS][P2PW_MAXE];
  __shared__ int32_t ePre[P2PW_WARPS][P2PW_MAXE + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * P2PW_WARPS + warp;
  if (row >= nLeaves) return;  // no CTA-wide barrier below
  const int g = rows[row];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const int64_t e0 = ptr[row], e1 = ptr[row + 1];
  const int TG = tn > 16 ? 32 : (tn > 8 ? 16 : 8), S = 32 / TG;
  const int tl = lane % TG, sp = lane / TG;
  for (int64_t t0 = 0; t0 < tn; t0 += TG) {
    const int64_t t = t0 + tl;
    const bool act = t < tn;
    double tx = 0, ty = 0, tz = 0;
    if (act) {
      tx = trg[3 * (tb + t)];
      ty = trg[3 * (tb + t) + 1];
      tz = trg[3 * (tb + t) + 2];
    }
    double acc[TD];
#pragma unroll
    for (int c = 0; c < TD; c++) acc[c] = 0.0;
    for (int64_t ec = e0; ec < e1; ec += P2PW_MAXE) {
      const int ne = (int)min((int64_t)P2PW_MAXE, e1 - ec);
      __syncwarp();
      int running = 0;
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
      for (int base = 0; base < total; base += P2PW_CH) {
        const int cnt = min(P2PW_CH, total - base);
        __syncwarp();
        for (int i = lane; i < cnt; i += 32) {
          const int j = base + i;
          int lo = 0, hi = ne;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (ePre[warp][mid] <= j) lo = mid; else hi = mid;
          }
          const int64_t s2 = eBeg[warp][lo] + (j - ePre[warp][lo]);
          sPos[warp][3 * i] = src[3 * s2];
          sPos[warp][3 * i + 1] = src[3 * s2 + 1];
          sPos[warp][3 * i + 2] = src[3 * s2 + 2];
          if (NRM) {
            sNrm[warp][3 * i] = nrm[3 * s2];
            sNrm[warp][3 * i + 1] = nrm[3 * s2 + 1];
            sNrm[warp][3 * i + 2] = nrm[3 * s2 + 2];
          }
#pragma unroll
          for (int c = 0; c < SD; c++) sDen[warp][SD * i + c] = den[s2 * SD + c];
        }
        __syncwarp();
        if (act) {
          for (int i = sp; i < cnt; i += S)
            kaccum<KT, double, double>(tx - sPos[warp][3 * i], ty - sPos[warp][3 * i + 1], tz - sPos[warp][3 * i + 2],
                                       NRM ? &sNrm[warp][3 * i] : nullptr, &sDen[warp][SD * i], acc, mu, ve);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < TD; c++)
      for (int o = TG; o < 32; o <<= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if (act && sp == 0) {
#pragma unroll
      for (int c = 0; c < TD; c++) val[(tb + t) * TD + c] += acc[c];
    }
  }
}

// k_e2t: target values from equivalent surfaces with the equivalent kernel:
// the leaf's own DE surface with its downward density (L2T,
// fmm3d_mpi.cpp:159-202) and the UE surfaces of its W nodes with their
// upward densities (M2T, fmm3d_mpi.cpp:208-249).
template <int KM>
__global__ void __launch_bounds__(P2P_THREADS)
    k_e2t(const int32_t* __restrict__ rows, const int64_t* __restrict__ farPtr, const int32_t* __restrict__ farIdx,
          int useOwn, int useFar, const int32_t* __restrict__ depth, const double* __restrict__ ctr,
          const double* __restrict__ rad, const double* __restrict__ samUE, int nUE,
          const double* __restrict__ samDE, int nDE, const double* __restrict__ uden,
          const double* __restrict__ dden, const int64_t* __restrict__ trgBeg, const int64_t* __restrict__ trgCnt,
          const double* __restrict__ trg, double* __restrict__ val, double mu, double ve) {
  constexpr int SD = KTraits<KM>::SD, TD = KTraits<KM>::TD;
  __shared__ double sPos[P2P_TILE * 3];
  __shared__ double sDen[P2P_TILE * SD];
  __shared__ double sRed[P2P_THREADS * TD];
  const int row = blockIdx.x;
  const int g = rows[row];
  const int64_t tb = trgBeg[g], tn = trgCnt[g];
  const int tid = threadIdx.x;
  const int TG = tn <= 32 ? 32 : (tn <= 64 ? 64 : 128);
  const int S = P2P_THREADS / TG;
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
    double acc[TD];
#pragma unroll
    for (int c = 0; c < TD; c++) acc[c] = 0.0;
    for (int64_t e = 0; e < own + nf; e++) {
      const bool isOwn = e < own;
      const int node = isOwn ? g : farIdx[f0 + e - own];
      const double* sam = isOwn ? samDE : samUE;
      const int ns = isOwn ? nDE : nUE;
      const double* dsrc = isOwn ? dden + (int64_t)node * ns * SD : uden + (int64_t)node * ns * SD;
      const double cx = ctr[3 * node], cy = ctr[3 * node + 1], cz = ctr[3 * node + 2], r = rad[node];
      for (int base = 0; base < ns; base += P2P_TILE) {
        const int cnt = min(P2P_TILE, ns - base);
        __syncthreads();
        for (int i = tid; i < cnt; i += P2P_THREADS) {
          const int j = base + i;
          sPos[3 * i] = cx + r * sam[3 * j];
          sPos[3 * i + 1] = cy + r * sam[3 * j + 1];
          sPos[3 * i + 2] = cz + r * sam[3 * j + 2];
#pragma unroll
          for (int c = 0; c < SD; c++) sDen[SD * i + c] = dsrc[(int64_t)j * SD + c];
        }
        __syncthreads();
        if (act)
          for (int i = sp; i < cnt; i += S)
            kaccum<KM, double, double>(tx - sPos[3 * i], ty - sPos[3 * i + 1], tz - sPos[3 * i + 2], nullptr,
                                       &sDen[SD * i], acc, mu, ve);
      }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < TD; c++) sRed[tid * TD + c] = acc[c];
    __syncthreads();
    if (sp == 0 && act) {
#pragma unroll
      for (int c = 0; c < TD; c++) {
        double s = 0;
        for (int k = 0; k < S; k++) s += sRed[(tl + k * TG) * TD + c];
        val[(tb + t) * TD + c] += s;
      }
    }
  }
}

// k_src2surf: check values on a box surface from point sources with the
// true kernel.  S2M (fmm3d_mpi.cpp:124-137): each leaf's own sources onto its
// UC surface (ptr == nullptr).  S2L (fmm3d_mpi.cpp:142-154): the X-list
// leaves' sources onto the DC surface.
constexpr int SURF_THREADS = 128;
constexpr int SURF_PPT = 4;  // surface points per thread: up to 512 points

template <int KT>
__global__ void __launch_bounds__(SURF_THREADS)
    k_src2surf(const int32_t* __restrict__ rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
               const int64_t* __restrict__ srcBeg, const int64_t* __restrict__ srcCnt,
               const double* __restrict__ src, const double* __restrict__ nrm, const double* __restrict__ den,
               const double* __restrict__ ctr, const double* __restrict__ rad, const double* __restrict__ sam,
               int nSurf, double* __restrict__ out, int64_t ldo, double mu, double ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD, NRM = KTraits<KT>::NRM;
  __shared__ double sPos[P2P_TILE * 3];
  __shared__ double sNrm[NRM ? P2P_TILE * 3 : 1];
  __shared__ double sDen[P2P_TILE * SD];
  __shared__ int64_t eBeg[P2P_MAXE];
  __shared__ int32_t ePre[P2P_MAXE + 1];
  const int row = blockIdx.x;
  const int g = rows[row];
  const int tid = threadIdx.x;
  const double cx = ctr[3 * g], cy = ctr[3 * g + 1], cz = ctr[3 * g + 2], r = rad[g];
  double px[SURF_PPT], py[SURF_PPT], pz[SURF_PPT];
  double acc[SURF_PPT][TD];
#pragma unroll
  for (int k = 0; k < SURF_PPT; k++) {
    int i = tid + k * SURF_THREADS;
    px[k] = py[k] = pz[k] = 0;
    if (i < nSurf) {
      px[k] = cx + r * sam[3 * i];
      py[k] = cy + r * sam[3 * i + 1];
      pz[k] = cz + r * sam[3 * i + 2];
    }
#pragma unroll
    for (int c = 0; c < TD; c++) acc[k][c] = 0.0;
  }
  const int64_t e0 = ptr ? ptr[row] : 0, e1 = ptr ? ptr[row + 1] : 1;
  for (int64_t ec = e0; ec < e1; ec += P2P_MAXE) {
    const int ne = (int)min((int64_t)P2P_MAXE, e1 - ec);
    __syncthreads();
    for (int e = tid; e < ne; e += SURF_THREADS) {
      int s = ptr ? idx[ec + e] : g;
      eBeg[e] = srcBeg[s];
      ePre[e + 1] = (int32_t)srcCnt[s];
    }
    __syncthreads();
    if (tid == 0) {
      ePre[0] = 0;
      for (int e = 0; e < ne; e++) ePre[e + 1] += ePre[e];
    }
    __syncthreads();
    const int total = ePre[ne];
    for (int base = 0; base < total; base += P2P_TILE) {
      const int cnt = min(P2P_TILE, total - base);
      __syncthreads();
      for (int i = tid; i < cnt; i += SURF_THREADS) {
        const int j = base + i;
        int lo = 0, hi = ne;
        while (hi - lo > 1) {
          int mid = (lo + hi) >> 1;
          if (ePre[mid] <= j) lo = mid; else hi = mid;
        }
        const int64_t s = eBeg[lo] + (j - ePre[lo]);
        sPos[3 * i] = src[3 * s];
        sPos[3 * i + 1] = src[3 * s + 1];
        sPos[3 * i + 2] = src[3 * s + 2];
        if (NRM) {
          sNrm[3 * i] = nrm[3 * s];
          sNrm[3 * i + 1] = nrm[3 * s + 1];
          sNrm[3 * i + 2] = nrm[3 * s + 2];
        }
#pragma unroll
        for (int c = 0; c < SD; c++) sDen[SD * i + c] = den[s * SD + c];
      }
      __syncthreads();
      for (int i = 0; i < cnt; i++) {
#pragma unroll
        for (int k = 0; k < SURF_PPT; k++)
          if (tid + k * SURF_THREADS < nSurf)
            kaccum<KT, double, double>(px[k] - sPos[3 * i], py[k] - sPos[3 * i + 1], pz[k] - sPos[3 * i + 2],
                                       NRM ? &sNrm[3 * i] : nullptr, &sDen[SD * i], acc[k], mu, ve);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < SURF_PPT; k++) {
    int i = tid + k * SURF_THREADS;
    if (i < nSurf)
#pragma unroll
      for (int c = 0; c < TD; c++) out[(int64_t)g * ldo + (int64_t)i * TD + c] += acc[k][c];
  }
}

// ------------------------------------------------------------------ M2L
// Spectral M2L of fmm3d_mpi/matmgnt3d_mpi.cpp:276-431.  The upward density
// of a box (on the surface of an np^3 lattice) is embedded at offset np/2 in
// the (2np)^3 grid, x index fastest; the r2c/c2r transforms follow FFTW's
// rank-3 layout with the x axis halved.  Because only the np^3 band of each
// axis is non-zero on input (and needed on output), the three 1-D passes are
// evaluated as small dense DFTs restricted to that band.


template <int NP>
__global__ void __launch_bounds__(128)
    k_m2l_fwd(const int32_t* __restrict__ nodes, const int32_t* __restrict__ depth, int rootLevel, Scale4 deg,
              int sdm, const double* __restrict__ uden, const int32_t* __restrict__ ijk, int nUE,
              double2* __restrict__ effDen, int nEff) {
  using F = FftDims<NP>;
  constexpr int N = F::N, NH = F::NH, H = F::H;
  __shared__ double cube[NP * NP * NP];
  __shared__ double2 X1[NP * NP * NH];
  __shared__ double2 X2[NP * N * NH];
  __shared__ double2 tw[N];
  const int slot = blockIdx.x;
  const int v = nodes[slot];
  const int tid = threadIdx.x;
  if (tid < N) {
    double s, c;
    sincospi(2.0 * tid / N, &s, &c);
    tw[tid] = make_double2(c, -s);
  }
  const int l = depth[v] + rootLevel;
  const double* ud = uden + (int64_t)v * nUE * sdm;
  for (int m = 0; m < sdm; m++) {
    const double scl = exp2(l * deg.v[m]);
    for (int i = tid; i < NP * NP * NP; i += blockDim.x) cube[i] = 0.0;
    __syncthreads();
    for (int i = tid; i < nUE; i += blockDim.x) {
      int p = ijk[i];
      int a = p & 255, b = (p >> 8) & 255, c = p >> 16;
      cube[(c * NP + b) * NP + a] = ud[(int64_t)i * sdm + m] * scl;
    }
    __syncthreads();
    for (int e = tid; e < NP * NP * NH; e += blockDim.x) {  // x pass (real -> half spectrum)
      int kx = e % NH, yb = (e / NH) % NP, zb = e / (NH * NP);
      double2 s = make_double2(0, 0);
      const double* row = &cube[(zb * NP + yb) * NP];
#pragma unroll
      for (int xb = 0; xb < NP; xb++) {
        double2 w = tw[(kx * (xb + H)) % N];
        s.x += row[xb] * w.x;
        s.y += row[xb] * w.y;
      }
      X1[e] = s;
    }
    __syncthreads();
    for (int e = tid; e < NP * N * NH; e += blockDim.x) {  // y pass
      int kx = e % NH, ky = (e / NH) % N, zb = e / (NH * N);
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int yb = 0; yb < NP; yb++) {
        double2 t = cmul(X1[(zb * NP + yb) * NH + kx], tw[(ky * (yb + H)) % N]);
        s.x += t.x;
        s.y += t.y;
      }
      X2[e] = s;
    }
    __syncthreads();
    double2* out = effDen + (int64_t)slot * nEff * sdm;
    for (int e = tid; e < N * N * NH; e += blockDim.x) {  // z pass
      int kx = e % NH, ky = (e / NH) % N, kz = e / (NH * N);
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int zb = 0; zb < NP; zb++) {
        double2 t = cmul(X2[(zb * N + ky) * NH + kx], tw[(kz * (zb + H)) % N]);
        s.x += t.x;
        s.y += t.y;
      }
      out[(int64_t)e * sdm + m] = s;
    }
    __syncthreads();
  }
}

// k_m2l_had: effVal(c) = (1/(2np)^3) sum_{v in V(c)} T_{idx(c,v)} .* effDen(v)
// (cptwvv, matmgnt3d_mpi.cpp:414-429).  One CTA per (target parent P,
// 32-frequency chunk); warp w owns child c = w of P.  The V-list of c is the
// set of children v of P's same-depth non-leaf neighbours Q that do not touch
// c; idx = v - c in child widths.
template <int SDM, int TDM>
__global__ void __launch_bounds__(256)
    k_m2l_had(const int32_t* __restrict__ rowOut, const int64_t* __restrict__ vPtr, const int8_t* __restrict__ vOff,
              const int32_t* __restrict__ nIn, const double2* __restrict__ effDen, const double2* __restrict__ T,
              double2* __restrict__ effVal, int nEff, double nrmfc) {
  // the parent's neighbour entries (input child slots resolved at setup,
  // offset code), 32 at a time in shared memory for the CTA
  __shared__ int sSl[32 * 8];
  __shared__ int sOf[32];
  const int b = blockIdx.x;
  const int c = threadIdx.x >> 5;
  const int f = blockIdx.y * 32 + (threadIdx.x & 31);
  const int ts = rowOut[8 * b + c];
  const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
  double2 acc[TDM];
#pragma unroll
  for (int i = 0; i < TDM; i++) acc[i] = make_double2(0, 0);
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
        const int id = c_transId[(rx + 3) * 49 + (ry + 3) * 7 + (rz + 3)];
        double2 d[SDM];
#pragma unroll
        for (int jj = 0; jj < SDM; jj++) d[jj] = effDen[((int64_t)s * nEff + f) * SDM + jj];
        const double2* Tf = T + ((int64_t)id * nEff + f) * (SDM * TDM);
#pragma unroll
        for (int jj = 0; jj < SDM; jj++)
#pragma unroll
          for (int i = 0; i < TDM; i++) {
            double2 tv = Tf[jj * TDM + i];
            acc[i].x += tv.x * d[jj].x - tv.y * d[jj].y;
            acc[i].y += tv.x * d[jj].y + tv.y * d[jj].x;
          }
      }
    }
  }
  if (live) {
#pragma unroll
    for (int i = 0; i < TDM; i++)
      effVal[((int64_t)ts * nEff + f) * TDM + i] = make_double2(acc[i].x * nrmfc, acc[i].y * nrmfc);
  }
}

// k_m2l_inv: c2r of a target box's accumulated spectrum and gather onto its
// DC surface, added to the downward check values (effVal2PlnVal,
// matmgnt3d_mpi.cpp:333-371).  The x pass is FFTW's halved c2r: the kx = 0 and
// kx = N/2 terms enter once and by their real part, the others twice.
template <int NP>
__global__ void __launch_bounds__(128)
    k_m2l_inv(const int32_t* __restrict__ nodes, const double2* __restrict__ effVal, int nEff, int tdm,
              const int32_t* __restrict__ ijk, int nDC, double* __restrict__ dchk, const int32_t* __restrict__ depth,
              int rootLevel, Scale4 outScale) {
  using F = FftDims<NP>;
  constexpr int N = F::N, NH = F::NH, H = F::H;
  __shared__ double2 Y2[NP * N * NH];
  __shared__ double2 Y1[NP * NP * NH];
  __shared__ double2 tw[N];
  const int slot = blockIdx.x;
  const int node = nodes[slot];
  const int tid = threadIdx.x;
  if (tid < N) {
    double s, c;
    sincospi(2.0 * tid / N, &s, &c);
    tw[tid] = make_double2(c, -s);
  }
  __syncthreads();
  const double2* in = effVal + (int64_t)slot * nEff * tdm;
  for (int m = 0; m < tdm; m++) {
    for (int e = tid; e < NP * N * NH; e += blockDim.x) {  // z pass, band outputs only
      int kx = e % NH, ky = (e / NH) % N, zb = e / (NH * N);
      double2 s = make_double2(0, 0);
#pragma unroll 4
      for (int kz = 0; kz < N; kz++) {
        double2 t = cmulc(in[((int64_t)(kz * N + ky) * NH + kx) * tdm + m], tw[(kz * (zb + H)) % N]);
        s.x += t.x;
        s.y += t.y;
      }
      Y2[e] = s;
    }
    __syncthreads();
    for (int e = tid; e < NP * NP * NH; e += blockDim.x) {  // y pass
      int kx = e % NH, yb = (e / NH) % NP, zb = e / (NH * NP);
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int ky = 0; ky < N; ky++) {
        double2 t = cmulc(Y2[(zb * N + ky) * NH + kx], tw[(ky * (yb + H)) % N]);
        s.x += t.x;
        s.y += t.y;
      }
      Y1[e] = s;
    }
    __syncthreads();
    for (int i = tid; i < nDC; i += blockDim.x) {  // x pass (c2r) at the surface points
      int p = ijk[i];
      int a = p & 255, b = (p >> 8) & 255, c = p >> 16;
      const double2* y1 = &Y1[(c * NP + b) * NH];
      const int x = a + H;
      double s = 0;
#pragma unroll
      for (int kx = 0; kx < NH; kx++) {
        double2 t = cmulc(y1[kx], tw[(kx * x) % N]);
        s += (kx == 0 || kx == N / 2) ? t.x : 2.0 * t.x;
      }
      dchk[(int64_t)node * nDC * tdm + (int64_t)i * tdm + m] +=
          outScale.mod ? s * exp2((depth[node] + rootLevel) * outScale.v[m]) : s;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ upload
template <typename T>
static std::string dput(DevState& D, T*& dst, const T* src, size_t n) {
  dst = nullptr;
  if (n == 0) return std::string();
  void* p = nullptr;
  cudaError_t e = dev_alloc(D, &p, n * sizeof(T));
  if (e != cudaSuccess) return std::string("cudaMalloc: ") + cudaGetErrorString(e);
  dst = (T*)p;
  if (src) {
    e = cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return std::string("cudaMemcpy: ") + cudaGetErrorString(e);
  }
  return std::string();
}
template <typename T>
static std::string dput(DevState& D, T*& dst, const std::vector<T>& v) {
  return dput(D, dst, v.data(), v.size());
}


cudaError_t dev_alloc(DevState& D, void** p, size_t bytes) {
  bytes = std::max<size_t>(bytes, 1);
  int best = -1;
  for (int i = 0; i < (int)D.spare.size(); i++) {
    const size_t b = D.spare[i].bytes;
    if (b >= bytes && b <= bytes + bytes / 2 && (best < 0 || b < D.spare[best].bytes)) best = i;
  }
  void* q = nullptr;
  if (best >= 0) {
    q = D.spare[best].p;
    bytes = D.spare[best].bytes;
    D.spare[best] = D.spare.back();
    D.spare.pop_back();
  } else {
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e == cudaErrorMemoryAllocation && !D.spare.empty()) {  // the kept blocks give way
      cudaGetLastError();
      dev_trim(D);
      e = cudaMalloc(&q, bytes);
    }
    if (e != cudaSuccess) {
      *p = nullptr;
      return e;
    }
  }
  D.allocs.push_back(q);
  D.allocBytes.push_back(bytes);
  *p = q;
  return cudaSuccess;
}

void dev_trim(DevState& D) {
  for (const DevState::Block& b : D.spare) cudaFree(b.p);
  D.spare.clear();
}

static void dev_clear(DevState& D);

void dev_release_for_reuse(DevState& D) {
  // the blocks may still be read by queued work of the handle
  if (D.stream) cudaStreamSynchronize(D.stream);
  if (D.side) cudaStreamSynchronize(D.side);
  for (size_t i = 0; i < D.allocs.size(); i++) D.spare.push_back(DevState::Block{D.allocs[i], D.allocBytes[i]});
  D.allocs.clear();
  D.allocBytes.clear();
  dev_clear(D);
}

void dev_free(DevState& D) {
  for (void* p : D.allocs) cudaFree(p);
  D.allocs.clear();
  D.allocBytes.clear();
  dev_trim(D);
  dev_clear(D);
}

// every pointer and flag of D back to "nothing uploaded" (the memory itself
// is freed or kept by the callers)
static void dev_clear(DevState& D) {
  if (D.evReady) {
    for (auto& e : D.ev) cudaEventDestroy(e);
    for (cudaEvent_t e : {D.evFork, D.evUp, D.evSide}) cudaEventDestroy(e);
    if (D.side) cudaStreamDestroy(D.side);
    D.side = nullptr;
    D.evFork = D.evUp = D.evSide = nullptr;
  }
  D.evReady = false;
  D.uc2ue = D.m2m = D.dc2de = D.l2l = nullptr;
  D.m2lT = nullptr;
  D.chkPos = D.chkOut = nullptr;
  D.chkCap = 0;
  D.uchk32 = D.uden32 = D.dchk32 = D.dden32 = nullptr;
  D.effDen32 = D.effVal32 = nullptr;
  D.l2l32 = nullptr;
  D.upF1 = D.upF2 = D.dnF1 = D.dnF2 = D.upT32 = D.dnT32 = nullptr;
  D.m2mUp32 = nullptr;
  for (DevState::OpT* op : {&D.tL2L, &D.tUpF1, &D.tUpF2, &D.tDnF1, &D.tDnF2, &D.tM2MUp}) *op = DevState::OpT();
  for (TcOp* op : {&D.cL2L, &D.cUpF1, &D.cUpF2, &D.cDnF1, &D.cDnF2, &D.cM2MUp}) *op = TcOp();  // memory freed above
  D.transIdDev = nullptr;
  D.m2lT32 = nullptr;
  D.m2lTw32 = nullptr;
  D.denK = D.valK = nullptr;
  D.den32 = nullptr;
  D.adjNearRows = D.adjNearIdx = D.adjFarRows = D.adjFarIdx = D.adjS2lRows = D.adjS2lIdx = nullptr;
  D.adjNearPtr = D.adjFarPtr = D.adjS2lPtr = nullptr;
  D.vParentsT = D.vNbrTIdx = nullptr;
  D.vRowOut = D.vNbrIn = D.vRowOutT = D.vNbrInT = nullptr;
  D.gemmScratch = nullptr;
  D.gemmScratchBytes = 0;
  D.devErr = nullptr;
  D.vNbrTPtr = nullptr;
  D.vNbrOffT = nullptr;
  D.uc2ueT = D.m2mT = D.dc2deT = D.l2lT = D.gradT = nullptr;
  D.adjListsReady = false;
  D.vListsReady = false;
  D.vTrgPtr = D.vSrcPtr = nullptr;
  D.vTrgEnt = D.vSrcEnt = nullptr;
  D.adjOpsStale = true;
  D.mixedReady = false;
  D.mixedOpsStale = true;
  D.mixedK = 0;
  D.mixedPassFor = D.mixedPassK = 0;
  D.m2tItems = nullptr;
  D.nearOrder = nullptr;
  D.nM2tItems = D.nM2tSplit = 0;
  D.m2tSplitLeaf = D.m2tSplitBase = D.m2tSplitCnt = nullptr;
  D.m2tPartTargets = 0;
  D.m2tPart = nullptr;
}

std::string dev_upload_operators(const Plan& P, DevState& D) {
  FMMG_CK(cudaSetDevice(D.device));
  auto put = [&](double*& dst, const std::vector<double>& v) -> std::string {
    if (!dst) return dput(D, dst, v);
    FMMG_CK(cudaMemcpy(dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    return std::string();
  };
  FMMG_TRY(put(D.uc2ue, P.uc2ue));
  FMMG_TRY(put(D.m2m, P.m2m));
  FMMG_TRY(put(D.dc2de, P.dc2de));
  FMMG_TRY(put(D.l2l, P.l2l));
  if (!D.m2lT) {
    FMMG_TRY(dput(D, D.m2lT, (const double2*)P.m2lT.data(), P.m2lT.size()));
  } else {
    FMMG_CK(cudaMemcpy(D.m2lT, P.m2lT.data(), P.m2lT.size() * sizeof(double2), cudaMemcpyHostToDevice));
  }
  int16_t tid[343];
  for (int i = 0; i < 343; i++) tid[i] = (int16_t)P.transId[i / 49][(i / 7) % 7][i % 7];
  FMMG_CK(cudaMemcpyToSymbol(c_transId, tid, sizeof(tid)));
  if (!D.transIdDev) FMMG_TRY(dput(D, D.transIdDev, tid, 343));
  D.mixedOpsStale = true;
  D.adjOpsStale = true;
  return std::string();
}

std::string dev_upload_vlists(const Plan& P, DevState& D) {
  if (D.vListsReady) return std::string();
  FMMG_CK(cudaSetDevice(D.device));
  P.expand_v_lists();
  FMMG_TRY(dput(D, D.vTrgPtr, P.vTrgPtr));
  FMMG_TRY(dput(D, D.vTrgEnt, P.vTrgEnt));
  FMMG_TRY(dput(D, D.vSrcPtr, P.vSrcPtr));
  FMMG_TRY(dput(D, D.vSrcEnt, P.vSrcEnt));
  D.vListsReady = true;
  return std::string();
}

static void csr_rows(const CSR& L, const std::vector<int32_t>& rows, std::vector<int64_t>& ptr,
                     std::vector<int32_t>& idx, const std::function<bool(int, int)>& keep) {
  ptr.assign(1, 0);
  idx.clear();
  for (int g : rows) {
    for (int64_t e = L.ptr[g]; e < L.ptr[g + 1]; e++)
      if (keep(g, L.idx[e])) idx.push_back(L.idx[e]);
    ptr.push_back((int64_t)idx.size());
  }
}

// out[i] = in[perm[i]] for xyz triples
__global__ void k_gather3(int64_t n, const int64_t* __restrict__ perm, const double* __restrict__ in,
                          double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = perm[i];
  out[3 * i] = in[3 * s];
  out[3 * i + 1] = in[3 * s + 1];
  out[3 * i + 2] = in[3 * s + 2];
}

std::string dev_upload(const Plan& P, DevState& D, const double* src, const double* nrm, const double* trg) {
  using Clock = std::chrono::steady_clock;
  auto t0 = Clock::now();
  auto lap = [&](int i) {
    const auto t1 = Clock::now();
    D.uploadMs[i] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    t0 = t1;
  };
  FMMG_CK(cudaSetDevice(D.device));
  const int64_t ns = P.ns, nt = P.nt;
  // targets that are the sources share their partition: a device copy
  const bool trgIsSrc = trg == src && nt == ns && P.trgPerm == P.srcPerm;
  FMMG_TRY(dput(D, D.srcPerm, P.srcPerm));
  if (trgIsSrc) {
    FMMG_TRY(dput<int64_t>(D, D.trgPerm, nullptr, (size_t)nt));
    if (nt > 0) FMMG_CK(cudaMemcpy(D.trgPerm, D.srcPerm, sizeof(int64_t) * nt, cudaMemcpyDeviceToDevice));
  } else {
    FMMG_TRY(dput(D, D.trgPerm, P.trgPerm));
  }
  {  // permuted geometry: the caller's arrays go up as they are and are
     // gathered into tree order on the device, through a staging block of
     // the plan builder's pool (the tree build's own copy of the sources
     // left one of this size there)
    double* raw = nullptr;
    PlanBufs stage;
    stage.device = D.device;
    FMMG_CK(stage.get(raw, 3 * (size_t)std::max<int64_t>(std::max(ns, nt), 1)));
    auto gather = [&](const double* host, int64_t n, const int64_t* dPerm, double*& dst) -> std::string {
      FMMG_TRY(dput<double>(D, dst, nullptr, 3 * (size_t)n));
      if (n == 0) return std::string();
      FMMG_CK(cudaMemcpy(raw, host, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
      k_gather3<<<(unsigned)((n + 255) / 256), 256>>>(n, dPerm, raw, dst);
      FMMG_CK(cudaGetLastError());
      return std::string();
    };
    FMMG_TRY(gather(src, ns, D.srcPerm, D.src));
    if (P.nrm) FMMG_TRY(gather(nrm, ns, D.srcPerm, D.nrm));
    if (trgIsSrc) {
      FMMG_TRY(dput<double>(D, D.trg, nullptr, 3 * (size_t)nt));
      if (nt > 0) FMMG_CK(cudaMemcpy(D.trg, D.src, sizeof(double) * 3 * nt, cudaMemcpyDeviceToDevice));
    } else {
      FMMG_TRY(gather(trg, nt, D.trgPerm, D.trg));
    }
    FMMG_CK(cudaDeviceSynchronize());
  }
  FMMG_TRY(dput(D, D.ctr, P.center));
  FMMG_TRY(dput(D, D.rad, P.radius));
  FMMG_TRY(dput(D, D.srcBeg, P.srcBeg));
  FMMG_TRY(dput(D, D.srcCnt, P.srcCnt));
  FMMG_TRY(dput(D, D.trgBeg, P.trgBeg));
  FMMG_TRY(dput(D, D.trgCnt, P.trgCnt));
  FMMG_TRY(dput(D, D.chd, P.chd));
  FMMG_TRY(dput(D, D.depth, P.depth));
  for (int k = 0; k < 4; k++) FMMG_TRY(dput(D, D.sam[k], P.sam[k]));
  {
    std::vector<int32_t> ijk;
    const int np = P.o.np;
    for (int i = 0; i < np; i++)
      for (int j = 0; j < np; j++)
        for (int k = 0; k < np; k++)
          if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1)
            ijk.push_back(i | (j << 8) | (k << 16));
    FMMG_TRY(dput(D, D.surfIJK, ijk));
  }
  lap(0);
  // work lists
  FMMG_TRY(dput(D, D.evtrLeaves, P.evtrLeaves));
  FMMG_TRY(dput(D, D.nearPtr, P.nearSrc.ptr));
  FMMG_TRY(dput(D, D.nearIdx, P.nearSrc.idx));
  {
    const int64_t ueSize = (int64_t)P.nUE * P.sdm, dcSize = (int64_t)P.nDC * P.tdm;
    std::vector<int64_t> ptr;
    std::vector<int32_t> idx;
    csr_rows(P.U, P.evtrLeaves, ptr, idx, [](int, int) { return true; });
    FMMG_TRY(dput(D, D.nearUPtr, ptr));
    FMMG_TRY(dput(D, D.nearUIdx, idx));
    csr_rows(P.W, P.evtrLeaves, ptr, idx,
             [&](int, int w) { return (P.flags[w] & NF_LSRC) && P.srcCnt[w] * P.sd < ueSize; });
    FMMG_TRY(dput(D, D.nearWPtr, ptr));
    FMMG_TRY(dput(D, D.nearWIdx, idx));
    csr_rows(P.X, P.evtrLeaves, ptr, idx, [&](int g, int) { return P.trgCnt[g] * P.td < dcSize; });
    FMMG_TRY(dput(D, D.nearXPtr, ptr));
    FMMG_TRY(dput(D, D.nearXIdx, idx));
  }
  FMMG_TRY(dput(D, D.farLeaves, P.farLeaves));
  FMMG_TRY(dput(D, D.l2tLeaves, P.l2tLeaves));
  FMMG_TRY(dput(D, D.farPtr, P.farUE.ptr));
  FMMG_TRY(dput(D, D.farIdx, P.farUE.idx));
  FMMG_TRY(dput(D, D.s2lNodes, P.s2lNodes));
  FMMG_TRY(dput(D, D.s2lPtr, P.s2lSrc.ptr));
  FMMG_TRY(dput(D, D.s2lIdx, P.s2lSrc.idx));
  FMMG_TRY(dput(D, D.s2mLeaves, P.s2mLeaves));
  {
    std::vector<int32_t> rows;
    auto cat = [&](const std::vector<std::vector<int32_t>>& L, std::vector<int64_t>& off) {
      off.assign(L.size() + 1, 0);
      for (size_t d = 0; d < L.size(); d++) {
        off[d] = (int64_t)rows.size();
        rows.insert(rows.end(), L[d].begin(), L[d].end());
      }
      off[L.size()] = (int64_t)rows.size();
    };
    cat(P.upC2E, D.offUpC2E);
    cat(P.upM2M, D.offUpM2M);
    cat(P.dnL2L, D.offDnL2L);
    cat(P.dnC2E, D.offDnC2E);
    cat(P.upLeaf, D.offUpLeaf);
    FMMG_TRY(dput(D, D.levelRows, rows));
  }
  FMMG_TRY(dput(D, D.vParents, P.vParents));
  FMMG_TRY(dput(D, D.vPtr, P.vNbr.ptr));
  FMMG_TRY(dput(D, D.vIdx, P.vNbr.idx));
  FMMG_TRY(dput(D, D.vOff, P.vNbrOff));
  FMMG_TRY(dput(D, D.vSrcSlot, P.vSrcSlot));
  FMMG_TRY(dput(D, D.vTrgSlot, P.vTrgSlot));
  FMMG_TRY(dput(D, D.vSrcNodes, P.vSrcNodes));
  FMMG_TRY(dput(D, D.vTrgNodes, P.vTrgNodes));
  FMMG_TRY(dput(D, D.vRowOut, P.vRowOut));
  FMMG_TRY(dput(D, D.vNbrIn, P.vNbrIn));
  lap(1);
  FMMG_TRY(dev_upload_operators(P, D));
  lap(2);
  // work arrays
  const int64_t ue = (int64_t)P.nUE * P.sdm, uc = (int64_t)P.nUC * P.tdm;
  const int64_t de = (int64_t)P.nDE * P.sdm, dc = (int64_t)P.nDC * P.tdm;
  FMMG_TRY(dput<double>(D, D.den, nullptr, (size_t)ns * P.sd));
  FMMG_TRY(dput<double>(D, D.val, nullptr, (size_t)std::max<int64_t>(nt, 1) * P.td));
  FMMG_TRY(dput<double>(D, D.uchk, nullptr, (size_t)P.nn * uc));
  FMMG_TRY(dput<double>(D, D.uden, nullptr, (size_t)P.nn * ue));
  FMMG_TRY(dput<double>(D, D.dchk, nullptr, (size_t)P.nn * dc));
  FMMG_TRY(dput<double>(D, D.dden, nullptr, (size_t)P.nn * de));
  FMMG_TRY(dput<double2>(D, D.effDen, nullptr, P.vSrcNodes.size() * (size_t)P.nEff * P.sdm));
  FMMG_TRY(dput<double2>(D, D.effVal, nullptr, P.vTrgNodes.size() * (size_t)P.nEff * P.tdm));
  D.gemmScratchBytes = (size_t)64 << 20;  // split-K partial tiles of the FP32 row GEMMs
  FMMG_TRY(dput<double>(D, D.gemmScratch, nullptr, D.gemmScratchBytes / sizeof(double)));
  FMMG_CK(cudaDeviceGetAttribute(&D.numSMs, cudaDevAttrMultiProcessorCount, D.device));
  FMMG_TRY(dput<int>(D, D.devErr, nullptr, 1));
  FMMG_CK(cudaMemset(D.devErr, 0, sizeof(int)));
  {
    const char* hk = std::getenv("FMMG_HADAMARD");
    D.hadPQ = !(hk && std::strcmp(hk, "list") == 0);
  }
  if (!D.evReady) {
    for (auto& e : D.ev) FMMG_CK(cudaEventCreate(&e));
    {
      int least = 0, greatest = 0;
      FMMG_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      FMMG_CK(cudaStreamCreateWithPriority(&D.side, cudaStreamNonBlocking, least));
    }
    for (cudaEvent_t* e : {&D.evFork, &D.evUp, &D.evSide}) FMMG_CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    D.evReady = true;
  }
  lap(3);
  return std::string();
}

// ------------------------------------------------------------------ launcher
void gemm_rows(DevState& D, int nrows, const int32_t* rows, const int32_t* chd, int xChild, int yChild,
               const double* X, int64_t ldx, const double* W, double* Y, int64_t ldy, int K, int N, Scale4 xs,
               Scale4 ys, double beta, LaunchStats* ls) {
  if (nrows <= 0) return;
  GrScale<double> gx, gy;
  gx.mod = xs.mod;
  gy.mod = ys.mod;
  for (int k = 0; k < 4; k++) {
    gx.v[k] = xs.v[k];
    gy.v[k] = ys.v[k];
  }
  // FP64 keeps each output's K sum in sequential order (no split-K scratch):
  // the 1e-10 parity with the oracle's sequential sums depends on it at np = 7
  const int n = launch_gemm_rows<double, 8>(D.stream, D.numSMs, nullptr, 0, nrows, 1, rows, chd, xChild, yChild, X,
                                            ldx, 0, W, Y, ldy, 0, K, N, gx, gy, beta);
  if (ls) ls->launches += n;
}

template <int KT>
static void launch_near(const Plan& P, DevState& D, const int64_t* ptr, const int32_t* idx, LaunchStats* ls,
                        cudaStream_t sn) {
  int n = (int)P.evtrLeaves.size();
  if (n == 0) return;
  k_p2p_near_w<KT><<<(n + P2PW_WARPS - 1) / P2PW_WARPS, 32 * P2PW_WARPS, 0, sn>>>(
      n, D.evtrLeaves, ptr, idx, D.srcBeg, D.srcCnt, D.trgBeg, D.trgCnt, D.src, D.nrm, D.den, D.trg, D.val,
      P.o.coefs[0], P.o.coefs[1]);
  if (ls) ls->launches++;
}

template <int KT>
static void launch_s2surf(const Plan& P, DevState& D, int nrows, const int32_t* rows, const int64_t* ptr,
                          const int32_t* idx, const double* sam, int nSurf, double* out, int64_t ldo,
                          LaunchStats* ls) {
  if (nrows <= 0) return;
  k_src2surf<KT><<<nrows, SURF_THREADS, 0, D.stream>>>(rows, ptr, idx, D.srcBeg, D.srcCnt, D.src, D.nrm, D.den,
                                                       D.ctr, D.rad, sam, nSurf, out, ldo, P.o.coefs[0],
                                                       P.o.coefs[1]);
  if (ls) ls->launches++;
}

static void launch_e2t(const Plan& P, DevState& D, int useOwn, int useFar, LaunchStats* ls, cudaStream_t se) {
  // L2T runs over the leaves at depth >= 2, M2T over the leaves with W nodes
  const int n = useFar ? (int)P.farLeaves.size() : (int)P.l2tLeaves.size();
  const int32_t* rows = useFar ? D.farLeaves : D.l2tLeaves;
  if (n == 0) return;
  switch (P.mm) {
#define FMMG_E2T(KM)                                                                                          \
  case KM:                                                                                                    \
    k_e2t<KM><<<n, P2P_THREADS, 0, se>>>(rows, D.farPtr, D.farIdx, useOwn, useFar, D.depth, D.ctr, D.rad,       \
                                               D.sam[0], P.nUE, D.sam[2], P.nDE, D.uden, D.dden, D.trgBeg,     \
                                               D.trgCnt, D.trg, D.val, P.o.coefs[0], P.o.coefs[1]);            \
    break;
    FMMG_E2T(LAP_S_U)
    FMMG_E2T(STK_F_U)
    FMMG_E2T(NAV_S_U)
#undef FMMG_E2T
  }
  if (ls) ls->launches++;
}

template <int NP>
static void launch_m2l_np(const Plan& P, DevState& D, LaunchStats* ls) {
  const int nsrc = (int)P.vSrcNodes.size(), ntrg = (int)P.vTrgNodes.size(), npar = (int)P.vParents.size();
  if (nsrc > 0) {
    Scale4 deg;
    deg.mod = P.sdm;
    for (int k = 0; k < 4; k++) deg.v[k] = P.deg[k];
    k_m2l_fwd<NP><<<nsrc, 128, 0, D.stream>>>(D.vSrcNodes, D.depth, P.o.rootLevel, deg, P.sdm, D.uden, D.surfIJK,
                                              P.nUE, D.effDen, P.nEff);
    if (ls) ls->launches++;
  }
  cudaEventRecord(D.ev[EV_M2L_FWD], D.stream);
  if (npar > 0 && ntrg > 0) {
    dim3 grid(npar, (P.nEff + 31) / 32);
    const double nrmfc = 1.0 / double(P.nReg);
    if (P.sdm == 1 && P.tdm == 1 && D.hadPQ) {
      const size_t smem = pq_smem_bytes<double2>(32);
      cudaFuncSetAttribute(k_m2l_had_pq<double2, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      dim3 g2((npar + D.tune.pqParents - 1) / D.tune.pqParents, (P.nEff + 31) / 32, 1);
      k_m2l_had_pq<double2, 1, false><<<g2, PQ_THREADS, smem, D.stream>>>(
          npar, D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen, 0, D.m2lT, D.effVal, 0, P.nEff, 1, nrmfc,
          D.transIdDev);
    } else if (P.sdm == 1 && P.tdm == 1) {
      if (!D.vListsReady) throw std::logic_error("the expanded V lists are not on the device (dev_upload_vlists)");
      const size_t smem = had_smem_bytes<double2>();
      cudaFuncSetAttribute(k_m2l_had_list<double2, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      dim3 g2((ntrg + HS_BOXES - 1) / HS_BOXES, (P.nEff + 31) / 32, 1);
      k_m2l_had_list<double2, 1, false><<<g2, HS_THREADS, smem, D.stream>>>(
          ntrg, D.vTrgPtr, (const int2*)D.vTrgEnt, D.effDen, 0, D.m2lT, D.effVal, 0, P.nEff, 1, nrmfc);
    }
    else if (P.sdm == 4 && P.tdm == 3)
      k_m2l_had<4, 3><<<grid, 256, 0, D.stream>>>(D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen, D.m2lT, D.effVal,
                                                  P.nEff, nrmfc);
    else
      k_m2l_had<3, 3><<<grid, 256, 0, D.stream>>>(D.vRowOut, D.vPtr, D.vOff, D.vNbrIn, D.effDen, D.m2lT, D.effVal,
                                                  P.nEff, nrmfc);
    cudaEventRecord(D.ev[EV_M2L_HAD], D.stream);
    Scale4 none;
    none.mod = 0;
    k_m2l_inv<NP><<<ntrg, 128, 0, D.stream>>>(D.vTrgNodes, D.effVal, P.nEff, P.tdm, D.surfIJK, P.nDC, D.dchk,
                                              D.depth, P.o.rootLevel, none);
    if (ls) ls->launches += 2;
  } else {
    cudaEventRecord(D.ev[EV_M2L_HAD], D.stream);
  }
}

// FP64 spectral transforms on arbitrary node lists (used by the adjoint):
// r2c of 2^(l*deg) .* x[node] on the np-surface, and c2r + gather added into
// y[node] (times 2^(l*outDeg) when outDeg.mod != 0).
template <int NP>
static void fwd_np(const Plan& P, DevState& D, int n, const int32_t* nodes, Scale4 deg, int dof, const double* x,
                   double2* spec) {
  k_m2l_fwd<NP><<<n, 128, 0, D.stream>>>(nodes, D.depth, P.o.rootLevel, deg, dof, x, D.surfIJK, P.nUE, spec, P.nEff);
}
template <int NP>
static void inv_np(const Plan& P, DevState& D, int n, const int32_t* nodes, int dof, const double2* spec, double* y,
                   Scale4 outDeg) {
  k_m2l_inv<NP><<<n, 128, 0, D.stream>>>(nodes, spec, P.nEff, dof, D.surfIJK, P.nDC, y, D.depth, P.o.rootLevel,
                                         outDeg);
}
void spectral_fwd(const Plan& P, DevState& D, int n, const int32_t* nodes, Scale4 deg, int dof, const double* x,
                  double2* spec) {
  if (n <= 0) return;
  switch (P.o.np) {
    case 3: fwd_np<3>(P, D, n, nodes, deg, dof, x, spec); break;
    case 4: fwd_np<4>(P, D, n, nodes, deg, dof, x, spec); break;
    case 5: fwd_np<5>(P, D, n, nodes, deg, dof, x, spec); break;
    case 6: fwd_np<6>(P, D, n, nodes, deg, dof, x, spec); break;
    case 7: fwd_np<7>(P, D, n, nodes, deg, dof, x, spec); break;
    case 8: fwd_np<8>(P, D, n, nodes, deg, dof, x, spec); break;
  }
}
void spectral_inv(const Plan& P, DevState& D, int n, const int32_t* nodes, int dof, const double2* spec, double* y,
                  Scale4 outDeg) {
  if (n <= 0) return;
  switch (P.o.np) {
    case 3: inv_np<3>(P, D, n, nodes, dof, spec, y, outDeg); break;
    case 4: inv_np<4>(P, D, n, nodes, dof, spec, y, outDeg); break;
    case 5: inv_np<5>(P, D, n, nodes, dof, spec, y, outDeg); break;
    case 6: inv_np<6>(P, D, n, nodes, dof, spec, y, outDeg); break;
    case 7: inv_np<7>(P, D, n, nodes, dof, spec, y, outDeg); break;
    case 8: inv_np<8>(P, D, n, nodes, dof, spec, y, outDeg); break;
  }
}
// the scalar Hadamard step on expanded lists; conj selects the transposed operator
void hadamard_pq64_adj(const Plan& P, DevState& D, const double2* in, double2* out) {
  const int nrow = (int)P.vParentsT.size();
  if (nrow <= 0) return;
  const size_t smem = pq_smem_bytes<double2>(32);
  cudaFuncSetAttribute(k_m2l_had_pq<double2, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g2((nrow + D.tune.pqParents - 1) / D.tune.pqParents, (P.nEff + 31) / 32, 1);
  k_m2l_had_pq<double2, 1, true><<<g2, PQ_THREADS, smem, D.stream>>>(
      nrow, D.vRowOutT, D.vNbrTPtr, D.vNbrOffT, D.vNbrInT, in, 0, D.m2lT, out, 0, P.nEff, 1, 1.0 / double(P.nReg),
      D.transIdDev);
}
void hadamard_list64(const Plan& P, DevState& D, int nOut, const int64_t* ptr, const int32_t* ent, const double2* in,
                     double2* out, bool conj) {
  if (nOut <= 0) return;
  const size_t smem = had_smem_bytes<double2>();
  dim3 g2((nOut + HS_BOXES - 1) / HS_BOXES, (P.nEff + 31) / 32, 1);
  const double nrmfc = 1.0 / double(P.nReg);
  if (conj) {
    cudaFuncSetAttribute(k_m2l_had_list<double2, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_m2l_had_list<double2, 1, true><<<g2, HS_THREADS, smem, D.stream>>>(nOut, ptr, (const int2*)ent, in, 0, D.m2lT,
                                                                         out, 0, P.nEff, 1, nrmfc);
  } else {
    cudaFuncSetAttribute(k_m2l_had_list<double2, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_m2l_had_list<double2, 1, false><<<g2, HS_THREADS, smem, D.stream>>>(nOut, ptr, (const int2*)ent, in, 0,
                                                                          D.m2lT, out, 0, P.nEff, 1, nrmfc);
  }
}

static void launch_m2l(const Plan& P, DevState& D, LaunchStats* ls) {
  switch (P.o.np) {
    case 3: launch_m2l_np<3>(P, D, ls); break;
    case 4: launch_m2l_np<4>(P, D, ls); break;
    case 5: launch_m2l_np<5>(P, D, ls); break;
    case 6: launch_m2l_np<6>(P, D, ls); break;
    case 7: launch_m2l_np<7>(P, D, ls); break;
    case 8: launch_m2l_np<8>(P, D, ls); break;
  }
}

template <int KT>
// overlap: the near field and the W list run on D.side (an untimed pass; a
// timed one keeps every stage on the main stream so the events bracket it);
// the target values still receive near field, M2T and L2T in that order
static void run_stages(const Plan& P, DevState& D, int mask, LaunchStats* ls, bool overlap) {
  cudaStream_t st = D.stream;
  const int ue = P.nUE * P.sdm, uc = P.nUC * P.tdm, de = P.nDE * P.sdm, dc = P.nDC * P.tdm;
  const int rl = P.o.rootLevel;
  const bool trgOut = !(mask & STAGE_NO_TARGETS);
  const bool ovl = overlap && trgOut && D.side;
  if (ovl) {  // fork: the densities are gathered and the target values cleared
    cudaEventRecord(D.evFork, st);
    cudaStreamWaitEvent(D.side, D.evFork, 0);
  }
  cudaStream_t sn = ovl ? D.side : st;
  if (mask & 1)  // upward: S2M
    launch_s2surf<KT>(P, D, (int)P.s2mLeaves.size(), D.s2mLeaves, nullptr, nullptr, D.sam[1], P.nUC, D.uchk, uc, ls);
  cudaEventRecord(D.ev[EV_S2M], st);
  if (mask & 1) {  // upward: M2M + C2E per level
    for (int d = P.maxDepth; d >= 1; d--) {
      int64_t a = D.offUpM2M[d], b = D.offUpM2M[d + 1];
      gemm_rows(D, (int)(b - a), D.levelRows + a, D.chd, 1, 0, D.uden, ue, D.m2m, D.uchk, uc, 8 * ue, uc,
                level_scale(P, d + 1 + rl, +1.0), unit_scale(), 0.0, ls);
      a = D.offUpC2E[d]; b = D.offUpC2E[d + 1];
      gemm_rows(D, (int)(b - a), D.levelRows + a, D.chd, 0, 0, D.uchk, uc, D.uc2ue, D.uden, ue, uc, ue, unit_scale(),
                level_scale(P, d + rl, -1.0), 0.0, ls);
    }
  }
  cudaEventRecord(D.ev[EV_UP_GEMM], st);
  if (!trgOut) {
  } else if ((mask & 2) && (mask & 8) && (mask & 16)) {
    launch_near<KT>(P, D, D.nearPtr, D.nearIdx, ls, sn);
  } else {
    if (mask & 2) launch_near<KT>(P, D, D.nearUPtr, D.nearUIdx, ls, sn);
    if (mask & 8) launch_near<KT>(P, D, D.nearWPtr, D.nearWIdx, ls, sn);
    if (mask & 16) launch_near<KT>(P, D, D.nearXPtr, D.nearXIdx, ls, sn);
  }
  if (ovl) {  // the up pass is done: the W list (upward densities) follows the near field
    cudaEventRecord(D.evUp, st);
    cudaStreamWaitEvent(D.side, D.evUp, 0);
  }
  cudaEventRecord(D.ev[EV_NEAR], st);
  if (mask & 4) {
    launch_m2l(P, D, ls);
  } else {
    cudaEventRecord(D.ev[EV_M2L_FWD], st);
    cudaEventRecord(D.ev[EV_M2L_HAD], st);
  }
  cudaEventRecord(D.ev[EV_M2L_INV], st);
  if ((mask & 8) && trgOut) launch_e2t(P, D, 0, 1, ls, sn);
  if (ovl) cudaEventRecord(D.evSide, D.side);
  cudaEventRecord(D.ev[EV_M2T], st);
  if (mask & 16)
    launch_s2surf<KT>(P, D, (int)P.s2lNodes.size(), D.s2lNodes, D.s2lPtr, D.s2lIdx, D.sam[3], P.nDC, D.dchk, dc, ls);
  cudaEventRecord(D.ev[EV_S2L], st);
  if (mask & 32) {  // downward: L2L + C2E per level
    for (int d = 2; d <= P.maxDepth; d++) {
      if (d >= 3) {
        int64_t a = D.offDnL2L[d - 1], b = D.offDnL2L[d];
        gemm_rows(D, (int)(b - a), D.levelRows + a, D.chd, 0, 1, D.dden, de, D.l2l, D.dchk, dc, de, 8 * dc,
                  level_scale(P, d - 1 + rl, +1.0), unit_scale(), 1.0, ls);
      }
      int64_t a = D.offDnC2E[d], b = D.offDnC2E[d + 1];
      gemm_rows(D, (int)(b - a), D.levelRows + a, D.chd, 0, 0, D.dchk, dc, D.dc2de, D.dden, de, dc, de,
                unit_scale(), level_scale(P, d + rl, -1.0), 0.0, ls);
    }
  }
  cudaEventRecord(D.ev[EV_DN_GEMM], st);
  if (ovl) cudaStreamWaitEvent(st, D.evSide, 0);  // join before the last writer of the target values
  if ((mask & 32) && trgOut) launch_e2t(P, D, 1, 0, ls, st);  // L2T
  cudaEventRecord(D.ev[EV_L2T], st);
}

std::string dev_evaluate(const Plan& P, DevState& D, const double* dDen, double* dVal, int precision, int mask,
                         bool timed, LaunchStats* lsIn) {
  if (precision == 1) return dev_evaluate_mixed(P, D, dDen, dVal, 1, mask, timed, lsIn);
  LaunchStats local;
  LaunchStats* ls = lsIn ? lsIn : &local;
  FMMG_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  const int64_t ns = P.ns, nt = P.nt;
  const int ue = P.nUE * P.sdm, uc = P.nUC * P.tdm, de = P.nDE * P.sdm, dc = P.nDC * P.tdm;
  cudaEventRecord(D.ev[EV_BEGIN], st);
  k_gather_den<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(ns, P.sd, D.srcPerm, dDen, D.den);
  if (ls) ls->launches++;
  FMMG_CK(cudaMemsetAsync(D.val, 0, sizeof(double) * std::max<int64_t>(nt, 1) * P.td, st));
  FMMG_CK(cudaMemsetAsync(D.uchk, 0, sizeof(double) * (size_t)P.nn * uc, st));
  FMMG_CK(cudaMemsetAsync(D.uden, 0, sizeof(double) * (size_t)P.nn * ue, st));
  FMMG_CK(cudaMemsetAsync(D.dchk, 0, sizeof(double) * (size_t)P.nn * dc, st));
  FMMG_CK(cudaMemsetAsync(D.dden, 0, sizeof(double) * (size_t)P.nn * de, st));
  cudaEventRecord(D.ev[EV_PREP], st);
  FMMG_DISPATCH_KT(P.o.kt, KT, run_stages<KT>(P, D, mask, ls, !timed));
  if (nt > 0) {
    k_scatter_val<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nt, P.td, D.trgPerm, D.val, dVal);
    if (ls) ls->launches++;
  }
  cudaEventRecord(D.ev[EV_END], st);
  D.lastLaunches = ls->launches;
  FMMG_CK(cudaGetLastError());
  if (timed) {
    FMMG_CK(cudaEventSynchronize(D.ev[EV_END]));
    for (int k = 0; k < EV_COUNT - 1; k++) cudaEventElapsedTime(&D.kernMs[k], D.ev[k], D.ev[k + 1]);
    const float* m = D.kernMs;
    // stage view: upward, U, V, W, X, downward, total
    D.stageMs[0] = m[EV_S2M - 1] + m[EV_UP_GEMM - 1];
    D.stageMs[1] = m[EV_NEAR - 1];
    D.stageMs[2] = m[EV_M2L_FWD - 1] + m[EV_M2L_HAD - 1] + m[EV_M2L_INV - 1];
    D.stageMs[3] = m[EV_M2T - 1];
    D.stageMs[4] = m[EV_S2L - 1];
    D.stageMs[5] = m[EV_DN_GEMM - 1] + m[EV_L2T - 1];
    cudaEventElapsedTime(&D.stageMs[6], D.ev[EV_BEGIN], D.ev[EV_END]);
  }
  return std::string();
}

void gather_rows(cudaStream_t st, int64_t n, int dof, const int64_t* perm, const double* in, double* out) {
  if (n > 0) k_gather_den<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, dof, perm, in, out);
}
void scatter_rows(cudaStream_t st, int64_t n, int dof, const int64_t* perm, const double* in, double* out) {
  if (n > 0) k_scatter_val<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, dof, perm, in, out);
}

std::string dev_take_error(DevState& D, int* flag) {
  *flag = 0;
  if (!D.devErr) return std::string();
  FMMG_CK(cudaSetDevice(D.device));
  FMMG_CK(cudaStreamSynchronize(D.stream));
  FMMG_CK(cudaMemcpy(flag, D.devErr, sizeof(int), cudaMemcpyDeviceToHost));
  FMMG_CK(cudaMemset(D.devErr, 0, sizeof(int)));
  return std::string();
}

std::string dev_far_field(const Plan& P, DevState& D, const double* dDen) {
  cudaStream_t st = D.stream;
  const int ue = P.nUE * P.sdm, uc = P.nUC * P.tdm, de = P.nDE * P.sdm, dc = P.nDC * P.tdm;
  gather_rows(st, P.ns, P.sd, D.srcPerm, dDen, D.den);
  FMMG_CK(cudaMemsetAsync(D.uchk, 0, sizeof(double) * (size_t)P.nn * uc, st));
  FMMG_CK(cudaMemsetAsync(D.uden, 0, sizeof(double) * (size_t)P.nn * ue, st));
  FMMG_CK(cudaMemsetAsync(D.dchk, 0, sizeof(double) * (size_t)P.nn * dc, st));
  FMMG_CK(cudaMemsetAsync(D.dden, 0, sizeof(double) * (size_t)P.nn * de, st));
  FMMG_DISPATCH_KT(P.o.kt, KT, run_stages<KT>(P, D, 63 | STAGE_NO_TARGETS, nullptr, false));
  FMMG_CK(cudaGetLastError());
  return std::string();
}

std::string dev_dense(const Plan& P, DevState& D, const double* dDen, int64_t nchk, const double* hPos,
                      double* hOut) {
  FMMG_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  if ((size_t)nchk > D.chkCap) {
    size_t cap = (size_t)std::max<int64_t>(nchk, 1024);
    FMMG_TRY(dput<double>(D, D.chkPos, nullptr, 3 * cap));
    FMMG_TRY(dput<double>(D, D.chkOut, nullptr, 3 * cap));
    D.chkCap = cap;
  }
  k_gather_den<<<(unsigned)((P.ns + 255) / 256), 256, 0, st>>>(P.ns, P.sd, D.srcPerm, dDen, D.den);
  FMMG_CK(cudaMemcpyAsync(D.chkPos, hPos, sizeof(double) * 3 * nchk, cudaMemcpyHostToDevice, st));
  FMMG_CK(cudaMemsetAsync(D.chkOut, 0, sizeof(double) * P.td * nchk, st));
  const int64_t chunk = 8192;
  dim3 grid((unsigned)((nchk + 127) / 128), (unsigned)((P.ns + chunk - 1) / chunk));
  FMMG_DISPATCH_KT(P.o.kt, KT,
                   k_dense<KT><<<grid, 128, 0, st>>>(nchk, D.chkPos, P.ns, chunk, D.src, D.nrm, D.den, D.chkOut,
                                                     P.o.coefs[0], P.o.coefs[1]));
  FMMG_CK(cudaMemcpyAsync(hOut, D.chkOut, sizeof(double) * P.td * nchk, cudaMemcpyDeviceToHost, st));
  FMMG_CK(cudaStreamSynchronize(st));
  FMMG_CK(cudaGetLastError());
  return std::string();
}


}  // namespace fmmg
