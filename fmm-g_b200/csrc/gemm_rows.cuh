// gemm_rows.cuh -- batched row GEMM of the translation stages, FP64 and FP32.
//
// For every listed node (and every right-hand side),
//   Y[row] = beta * Y[row] + ys .* (W (xs .* X[row])),
// W N x K row-major.  The X (Y) row of a node starts at its own id or at its
// first child's id, so the 8 children of a parent form one contiguous row of
// length 8 * ld.  Serves C2E (pinv GEMV, matmgnt3d_mpi.cpp:107-149, :196-229),
// M2M (:151-193) and L2L (:231-274) over all nodes of a level at once, and
// their transposes in the adjoint.
//
// Tiling: 128 (rows x right-hand sides) x 64 (outputs) per CTA, K in steps of
// BK (16 for FP32, 8 for FP64: four 16-byte vectors per tile row), 256
// threads each owning an 8 x 4 register tile.  The next K step is
// fetched into registers while the current one is multiplied from shared
// memory (two buffers, one barrier per step).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace fmmg {

constexpr int GR_BM = 128, GR_BN = 64, GR_BK = 16, GR_THREADS = 256;

template <typename T>
struct GrScale {
  T v[4];
  int mod;
};

// v[i % mod] without dynamic indexing of the by-value parameter (which
// would place it in local memory)
template <typename T>
__device__ __forceinline__ T gr_sel(const GrScale<T>& s, int i) {
  const int m = s.mod == 1 ? 0 : i % s.mod;
  return m == 0 ? s.v[0] : (m == 1 ? s.v[1] : (m == 2 ? s.v[2] : s.v[3]));
}

template <typename T>
struct GrVec;
template <>
struct GrVec<float> {
  typedef float4 V;
};
template <>
struct GrVec<double> {
  typedef double2 V;
};

// VEC: X rows and W rows are 16-byte aligned with K a multiple of the vector
// width, so the tiles are fetched as 16-byte vectors along K (4 vectors per
// row of a K step, consecutive threads on consecutive vectors); otherwise
// element by element.  Shared tiles are padded against bank conflicts.
template <typename T, int BK, bool VEC>
__global__ void __launch_bounds__(GR_THREADS, 2)
    k_gemm_rows_t(int nrows, int nrhs, const int32_t* __restrict__ rows, const int32_t* __restrict__ chd, int xChild,
                  int yChild, const T* __restrict__ X, int64_t ldx, int64_t xRhs, const T* __restrict__ W,
                  T* __restrict__ Y, int64_t ldy, int64_t yRhs, int K, int N, GrScale<T> xs, GrScale<T> ys, T beta,
                  int kChunk, T* __restrict__ part) {
  typedef typename GrVec<T>::V V;
  constexpr int VW = sizeof(V) / sizeof(T);  // 4 floats or 2 doubles
  static_assert(BK / VW == 4, "four vectors per tile row");
  constexpr int PA = GR_BM + VW, PB = GR_BN + VW;  // padded tile rows
  __shared__ __align__(16) T As[2][BK][PA];
  __shared__ __align__(16) T Bs[2][BK][PB];
  __shared__ const T* xrow[GR_BM];
  __shared__ T* yrow[GR_BM];
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * GR_BM, n0 = blockIdx.y * GR_BN;
  if (tid < GR_BM) {
    const int r = r0 + tid;
    if (r < nrows * nrhs) {
      const int q = r / nrows;
      const int node = rows[r - q * nrows];
      xrow[tid] = X + q * xRhs + (int64_t)(xChild ? chd[node] : node) * ldx;
      yrow[tid] = Y + q * yRhs + (int64_t)(yChild ? chd[node] : node) * ldy;
    } else {
      xrow[tid] = nullptr;
      yrow[tid] = nullptr;
    }
  }
  __syncthreads();
  // K range of this split (blockIdx.z); the whole of K without splitting
  const int kBeg = blockIdx.z * kChunk, kEnd = min(K, kBeg + kChunk);
  // fetch mapping: A vectors (row tid/4 and 64 + tid/4, K quad tid%4), B vector (output tid/4, K quad tid%4)
  const int fr = tid >> 2, fq = (tid & 3) * VW;
  const T* xa0 = xrow[fr];
  const T* xa1 = xrow[fr + 64];
  const bool bIn = n0 + fr < N;
  const T* wr = W + (int64_t)(bIn ? n0 + fr : 0) * K;
  T fa0[VW], fa1[VW], fb[VW];
  auto fetch = [&](int k0) {
    const int k = k0 + fq;
    if (VEC) {
      const bool kin = k < kEnd;  // VW | K and VW | kChunk: the whole vector is in range
      V a0 = {}, a1 = {}, bv = {};
      if (xa0 && kin) a0 = *reinterpret_cast<const V*>(xa0 + k);
      if (xa1 && kin) a1 = *reinterpret_cast<const V*>(xa1 + k);
      if (bIn && kin) bv = *reinterpret_cast<const V*>(wr + k);
      const T* pa0 = reinterpret_cast<const T*>(&a0);
      const T* pa1 = reinterpret_cast<const T*>(&a1);
      const T* pb = reinterpret_cast<const T*>(&bv);
#pragma unroll
      for (int j = 0; j < VW; j++) {
        const T sc = gr_sel(xs, k + j);
        fa0[j] = pa0[j] * sc;
        fa1[j] = pa1[j] * sc;
        fb[j] = pb[j];
      }
    } else {
#pragma unroll
      for (int j = 0; j < VW; j++) {
        const bool kin = k + j < kEnd;
        const T sc = gr_sel(xs, k + j);
        fa0[j] = (xa0 && kin) ? xa0[k + j] * sc : T(0);
        fa1[j] = (xa1 && kin) ? xa1[k + j] * sc : T(0);
        fb[j] = (bIn && kin) ? wr[k + j] : T(0);
      }
    }
  };
  auto stash = [&](int b) {
#pragma unroll
    for (int j = 0; j < VW; j++) {
      As[b][fq + j][fr] = fa0[j];
      As[b][fq + j][fr + 64] = fa1[j];
      Bs[b][fq + j][fr] = fb[j];
    }
  };
  const int tm = tid >> 4, tn = tid & 15;  // rows tm*8 .. +7, outputs tn*4 .. +3
  T acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = T(0);
  fetch(kBeg);
  stash(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = kBeg; k0 < kEnd; k0 += BK) {
    const bool more = k0 + BK < kEnd;
    if (more) fetch(k0 + BK);
#pragma unroll
    for (int k = 0; k < BK; k++) {
      T a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; i += VW) {
        const V v = *reinterpret_cast<const V*>(&As[buf][k][tm * 8 + i]);
        const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int j = 0; j < VW; j++) a[i + j] = pv[j];
      }
#pragma unroll
      for (int j0 = 0; j0 < 4; j0 += VW) {
        const V v = *reinterpret_cast<const V*>(&Bs[buf][k][tn * 4 + j0]);
        const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int j = 0; j < VW; j++) b[j0 + j] = pv[j];
      }
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (more) {
      stash(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
  if (part) {  // split K: raw partial tile, reduced by k_gemm_reduce_t
    const int64_t M = (int64_t)nrows * nrhs;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = r0 + tm * 8 + i;
      if (r >= M) continue;
      T* pr = part + ((int64_t)blockIdx.z * M + r) * N;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int n = n0 + tn * 4 + j;
        if (n < N) pr[n] = acc[i][j];
      }
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    T* yr = yrow[tm * 8 + i];
    if (!yr) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = n0 + tn * 4 + j;
      if (n < N) {
        const T v = acc[i][j] * gr_sel(ys, n);
        yr[n] = beta == T(0) ? v : beta * yr[n] + v;
      }
    }
  }
}

// Y[row] = beta * Y[row] + ys .* sum over splits of part[split][row]
template <typename T>
__global__ void __launch_bounds__(256)
    k_gemm_reduce_t(int nrows, int nrhs, const int32_t* __restrict__ rows, const int32_t* __restrict__ chd,
                    int yChild, T* __restrict__ Y, int64_t ldy, int64_t yRhs, int N, int splits,
                    const T* __restrict__ part, GrScale<T> ys, T beta) {
  const int64_t M = (int64_t)nrows * nrhs;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  const int64_t r = i / N;
  const int n = (int)(i - r * N);
  T s = T(0);
  for (int z = 0; z < splits; z++) s += part[((int64_t)z * M + r) * N + n];
  const int q = (int)(r / nrows);
  const int node = rows[r - (int64_t)q * nrows];
  T* yr = Y + q * yRhs + (int64_t)(yChild ? chd[node] : node) * ldy;
  const T v = s * gr_sel(ys, n);
  yr[n] = beta == T(0) ? v : beta * yr[n] + v;
}

// ------------------------------------------------------------------ FP32 wide tile
// The FP32 row GEMM with a 128 x 160 CTA tile: one column tile covers the
// 152-wide surfaces (the 296-wide check surface and the 1216-wide L2L output
// take 2 and 8), where 64-wide tiles left a fifth of the FMAs on padding.
// Each of the 256 threads owns 8 rows x 10 outputs: columns 4t..4t+3,
// 64+4t..+3 and 128+2t, +1 (t = thread % 16), so its shared reads are two
// 16-byte and one 8-byte vector per k.  The operator arrives transposed and
// zero padded, Wt[k][n] (K to a multiple of 16, N to a multiple of 160), and
// streams into shared memory with cp.async (no registers); the X rows are
// gathered through registers and stored transposed.  A uniform X scale
// (one value, xs.mod == 1) is applied to the accumulators at the end instead
// of to every fetched value.
constexpr int GW_BM = 128, GW_BN = 160, GW_BK = 16, GW_THREADS = 256;
constexpr int GW_PA = GW_BM + 4, GW_PB = GW_BN + 4;

__device__ __forceinline__ void gw_cp16(void* dst, const void* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ int gw_col(int tn, int j) {
  return j < 4 ? tn * 4 + j : (j < 8 ? 64 + tn * 4 + (j - 4) : 128 + tn * 2 + (j - 8));
}

static __global__ void __launch_bounds__(GW_THREADS, 2)
    k_gemm_rows_w(int nrows, int nrhs, const int32_t* __restrict__ rows, const int32_t* __restrict__ chd, int xChild,
                  int yChild, const float* __restrict__ X, int64_t ldx, int64_t xRhs, const float* __restrict__ Wt,
                  int ldw, float* __restrict__ Y, int64_t ldy, int64_t yRhs, int K, int N, GrScale<float> xs,
                  GrScale<float> ys, float beta, int kChunk, float* __restrict__ part, int yVec) {
  __shared__ __align__(16) float As[2][GW_BK][GW_PA];
  __shared__ __align__(16) float Bs[2][GW_BK][GW_PB];
  __shared__ const float* xrow[GW_BM];
  __shared__ float* yrow[GW_BM];
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * GW_BM, n0 = blockIdx.y * GW_BN;
  if (tid < GW_BM) {
    const int r = r0 + tid;
    if (r < nrows * nrhs) {
      const int q = r / nrows;
      const int node = rows[r - q * nrows];
      xrow[tid] = X + q * xRhs + (int64_t)(xChild ? chd[node] : node) * ldx;
      yrow[tid] = Y + q * yRhs + (int64_t)(yChild ? chd[node] : node) * ldy;
    } else {
      xrow[tid] = nullptr;
      yrow[tid] = nullptr;
    }
  }
  __syncthreads();
  const int kBeg = blockIdx.z * kChunk, kEnd = min(K, kBeg + kChunk);
  const bool xsUni = xs.mod == 1;
  // X fetch: rows fr and 64 + fr, K quad fq (16-byte vectors)
  const int fr = tid >> 2, fq = (tid & 3) * 4;
  const float* xa0 = xrow[fr];
  const float* xa1 = xrow[fr + 64];
  float4 ra0, ra1;
  auto fetchA = [&](int k0) {
    const int k = k0 + fq;
    const bool kin = k < kEnd;  // 4 | K and 16 | kChunk: the whole vector is in range
    ra0 = (xa0 && kin) ? *reinterpret_cast<const float4*>(xa0 + k) : make_float4(0.f, 0.f, 0.f, 0.f);
    ra1 = (xa1 && kin) ? *reinterpret_cast<const float4*>(xa1 + k) : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  auto stashA = [&](int b, int k0) {
    float a0[4] = {ra0.x, ra0.y, ra0.z, ra0.w}, a1[4] = {ra1.x, ra1.y, ra1.z, ra1.w};
    if (!xsUni) {
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const float sc = gr_sel(xs, k0 + fq + j);
        a0[j] *= sc;
        a1[j] *= sc;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      As[b][fq + j][fr] = a0[j];
      As[b][fq + j][fr + 64] = a1[j];
    }
  };
  // operator tile: BK rows of Wt, 160 columns, 640 16-byte pieces
  auto loadB = [&](int b, int k0) {
    for (int i = tid; i < GW_BK * GW_BN / 4; i += GW_THREADS) {
      const int kk = i / (GW_BN / 4), c = (i - kk * (GW_BN / 4)) * 4;
      gw_cp16(&Bs[b][kk][c], Wt + (int64_t)(k0 + kk) * ldw + n0 + c);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  const int tm = tid >> 4, tn = tid & 15;
  float acc[8][10];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 10; j++) acc[i][j] = 0.f;
  fetchA(kBeg);
  loadB(0, kBeg);
  stashA(0, kBeg);
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  int buf = 0;
  for (int k0 = kBeg; k0 < kEnd; k0 += GW_BK) {
    const bool more = k0 + GW_BK < kEnd;
    if (more) {
      fetchA(k0 + GW_BK);
      loadB(buf ^ 1, k0 + GW_BK);
    }
#pragma unroll
    for (int k = 0; k < GW_BK; k++) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][k][tm * 8]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][k][tm * 8 + 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][k][tn * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][k][64 + tn * 4]);
      const float2 b2 = *reinterpret_cast<const float2*>(&Bs[buf][k][128 + tn * 2]);
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float b[10] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w, b2.x, b2.y};
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 10; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (more) {
      stashA(buf ^ 1, k0 + GW_BK);
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      __syncthreads();
      buf ^= 1;
    }
  }
  const float xsc = xsUni ? xs.v[0] : 1.f;
  if (part) {  // split K: raw partial tile, reduced by k_gemm_reduce_t
    const int64_t M = (int64_t)nrows * nrhs;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = r0 + tm * 8 + i;
      if (r >= M) continue;
      float* pr = part + ((int64_t)blockIdx.z * M + r) * N;
#pragma unroll
      for (int j = 0; j < 10; j++) {
        const int n = n0 + gw_col(tn, j);
        if (n < N) pr[n] = acc[i][j] * xsc;
      }
    }
    return;
  }
  float ysc[10];
#pragma unroll
  for (int j = 0; j < 10; j++) ysc[j] = gr_sel(ys, n0 + gw_col(tn, j)) * xsc;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    float* yr = yrow[tm * 8 + i];
    if (!yr) continue;
#pragma unroll
    for (int g = 0; g < 2; g++) {  // the two 4-column groups
      const int n = n0 + g * 64 + tn * 4;
      float v[4];
#pragma unroll
      for (int j = 0; j < 4; j++) v[j] = acc[i][g * 4 + j] * ysc[g * 4 + j];
      if (yVec && n + 3 < N) {
        float4* dst = reinterpret_cast<float4*>(yr + n);
        if (beta != 0.f) {
          const float4 o = *dst;
          v[0] += beta * o.x;
          v[1] += beta * o.y;
          v[2] += beta * o.z;
          v[3] += beta * o.w;
        }
        *dst = make_float4(v[0], v[1], v[2], v[3]);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (n + j < N) yr[n + j] = beta == 0.f ? v[j] : beta * yr[n + j] + v[j];
      }
    }
#pragma unroll
    for (int j = 8; j < 10; j++) {
      const int n = n0 + gw_col(tn, j);
      if (n < N) {
        const float v = acc[i][j] * ysc[j];
        yr[n] = beta == 0.f ? v : beta * yr[n] + v;
      }
    }
  }
}

// Launches the wide-tile FP32 GEMM (Wt transposed and padded as above, ldw
// its row length); split K as in launch_gemm_rows.  Returns the launches.
inline int launch_gemm_rows_w(cudaStream_t st, int splitCtas, float* scratch, size_t scratchElems, int nrows, int nrhs,
                              const int32_t* rows, const int32_t* chd, int xChild, int yChild, const float* X,
                              int64_t ldx, int64_t xRhs, const float* Wt, int ldw, float* Y, int64_t ldy,
                              int64_t yRhs, int K, int N, GrScale<float> xs, GrScale<float> ys, float beta) {
  if (nrows <= 0 || nrhs <= 0) return 0;
  const int64_t M = (int64_t)nrows * nrhs;
  const int tiles = (int)((M + GW_BM - 1) / GW_BM) * ((N + GW_BN - 1) / GW_BN);
  int splits = 1;
  if (scratch && tiles < splitCtas && K >= 8 * GW_BK) {
    splits = std::min(8, (splitCtas + tiles - 1) / tiles);
    splits = std::min(splits, K / (4 * GW_BK));
    while (splits > 1 && (size_t)splits * M * N > scratchElems) splits--;
  }
  const int kChunk = splits > 1 ? ((K + splits - 1) / splits + GW_BK - 1) / GW_BK * GW_BK : K;
  if (splits > 1) splits = (K + kChunk - 1) / kChunk;
  const int yVec = ((uintptr_t)Y % 16 == 0) && ldy % 4 == 0 && yRhs % 4 == 0;
  dim3 grid((unsigned)((M + GW_BM - 1) / GW_BM), (N + GW_BN - 1) / GW_BN, splits);
  float* pt = splits > 1 ? scratch : nullptr;
  k_gemm_rows_w<<<grid, GW_THREADS, 0, st>>>(nrows, nrhs, rows, chd, xChild, yChild, X, ldx, xRhs, Wt, ldw, Y, ldy,
                                             yRhs, K, N, xs, ys, beta, kChunk, pt, yVec);
  if (splits == 1) return 1;
  const int64_t tot = M * N;
  k_gemm_reduce_t<float><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(nrows, nrhs, rows, chd, yChild, Y, ldy, yRhs,
                                                                         N, splits, scratch, ys, beta);
  return 2;
}

// Launches the row GEMM; when the output tiles alone would leave the GPU
// underfilled (fewer than splitCtas CTAs: 2 per SM by default, set by the
// autotuner, 0 never splits) and K is long, K is split into up to 8 chunks whose partial tiles go to `scratch` (scratchElems values) and are
// summed in a fixed order by k_gemm_reduce_t, so results stay deterministic.
// Returns the number of kernels launched.
template <typename T, int BK>
inline int launch_gemm_rows(cudaStream_t st, int splitCtas, T* scratch, size_t scratchElems, int nrows, int nrhs,
                            const int32_t* rows, const int32_t* chd, int xChild, int yChild, const T* X, int64_t ldx,
                            int64_t xRhs, const T* W, T* Y, int64_t ldy, int64_t yRhs, int K, int N, GrScale<T> xs,
                            GrScale<T> ys, T beta) {
  if (nrows <= 0 || nrhs <= 0) return 0;
  const int64_t M = (int64_t)nrows * nrhs;
  const int tiles = (int)((M + GR_BM - 1) / GR_BM) * ((N + GR_BN - 1) / GR_BN);
  int splits = 1;
  if (scratch && tiles < splitCtas && K >= 8 * BK) {
    splits = std::min(8, (splitCtas + tiles - 1) / tiles);
    splits = std::min(splits, K / (4 * BK));
    while (splits > 1 && (size_t)splits * M * N > scratchElems) splits--;
  }
  const int kChunk = splits > 1 ? ((K + splits - 1) / splits + BK - 1) / BK * BK : K;
  if (splits > 1) splits = (K + kChunk - 1) / kChunk;
  constexpr int VW = 16 / sizeof(T);
  const bool vec = ((uintptr_t)X % 16 == 0) && ((uintptr_t)W % 16 == 0) && ldx % VW == 0 && xRhs % VW == 0 &&
                   K % VW == 0;
  dim3 grid((unsigned)((M + GR_BM - 1) / GR_BM), (N + GR_BN - 1) / GR_BN, splits);
  T* pt = splits > 1 ? scratch : nullptr;
  if (vec)
    k_gemm_rows_t<T, BK, true><<<grid, GR_THREADS, 0, st>>>(nrows, nrhs, rows, chd, xChild, yChild, X, ldx, xRhs, W,
                                                             Y, ldy, yRhs, K, N, xs, ys, beta, kChunk, pt);
  else
    k_gemm_rows_t<T, BK, false><<<grid, GR_THREADS, 0, st>>>(nrows, nrhs, rows, chd, xChild, yChild, X, ldx, xRhs, W,
                                                              Y, ldy, yRhs, K, N, xs, ys, beta, kChunk, pt);
  if (splits == 1) return 1;
  const int64_t tot = M * N;
  k_gemm_reduce_t<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(nrows, nrhs, rows, chd, yChild, Y, ldy, yRhs, N,
                                                                     splits, scratch, ys, beta);
  return 2;
}

}  // namespace fmmg
