// gemm_tc.cuh -- the FP32 row GEMMs of the translation stages (C2E factors,
// folded C2E x M2M, L2L) on the 5th-generation tensor cores (tcgen05,
// kind::tf32) as 3xTF32 split products.
//
// Same contract as k_gemm_rows_t (gemm_rows.cuh):
//   Y[row] = beta * Y[row] + ys .* (W (xs .* X[row]))  for every listed node
// and right-hand side, W N x K, or raw partial tiles for split K.
//
// Precision.  Every operand value v is carried as two TF32 numbers, hi =
// rna_tf32(v) and lo = rna_tf32(v - hi), both rounded to nearest, so the
// tensor core (which reads only the TF32 bits) sees them exactly and v is
// represented to 2^-22 relative.  The constant operator W is split once on
// the host from its FP64 value; the runtime rows X are split in registers as
// they are staged.  Each 32-wide K block's hi*hi + hi*lo + lo*hi is
// accumulated by the tensor core in a fresh TMEM accumulator (12 MMA steps),
// and the block sums are added in FP32, rounded to nearest, on the CUDA
// cores: accumulating the whole K inside TMEM loses accuracy with K (on the
// 1M-point workload it moved the evaluate from 1.7e-6 to 1.5e-5 against the
// dense sum, per block it stays at 2.6e-6).
//
// Warp roles (416 threads): warps 0-3 stage the gathered X rows (128 rows x
// 32 K values per block as 16-byte loads, two blocks in flight, split and
// stored K-major with the 128-byte swizzle); warps 4-11 drain each block's
// accumulator into FP32 register sums (warp w reads TMEM lanes 32 (w % 4) ..,
// half the columns each) and run the epilogue; lane 0 of warp 12 loads the
// pre-split operator tiles (BN rows x 32 K, hi and lo) by TMA
// (cp.async.bulk.tensor, this GPU's own memory, no multicast) and issues per
// K block 4 K steps x 3 products of tcgen05.mma M = 128, N = BN, K = 8 into
// one of three TMEM accumulators, so the tensor core runs up to two blocks
// ahead of the drain.  Issuing a block's MMAs occupies the lane for about the
// tensor core's time on it, so that lane does nothing else.  Three smem
// stages.
//
// Every mbarrier wait is bounded (TC_WAIT_NS): a wait that runs out sets the
// CTA's abort flag and the kernel's error flag, nobody writes a stage the
// tensor core may still read, the MMA lane stops issuing, the epilogue is
// skipped, and the TMEM is freed only after a last bounded wait for the
// issued MMAs.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "gemm_rows.cuh"
#include "tc_op.hpp"

namespace fmmg {

constexpr int TC_THREADS = 128;                 // the wait self-test's CTA
constexpr uint32_t TC_TMEM_COLS = 64;           // the wait self-test's TMEM
constexpr long long TC_WAIT_NS = 1000000000ll;  // a bounded mbarrier wait gives up after 1 s

constexpr int T3_BM = 128, T3_BK = 32, T3_STAGES = 3, T3_AWARPS = 4, T3_DWARPS = 8;
constexpr int T3_DWARP0 = T3_AWARPS, T3_MWARP = T3_AWARPS + T3_DWARPS, T3_THREADS = 32 * (T3_MWARP + 1);
constexpr int T3_NACC = 3;  // block accumulators in TMEM: the tensor core runs up to two blocks ahead of the drain
constexpr int T3_A_BYTES = T3_BM * T3_BK * 4;  // 16 KB per A part (hi or lo)

template <int BN>
struct T3Cfg {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "tcgen05 M=128 needs N % 16 == 0, 16..256");
  static constexpr int B_BYTES = BN * T3_BK * 4;                          // one B part
  static constexpr int STAGE_BYTES = 2 * T3_A_BYTES + 2 * B_BYTES;        // A hi, A lo, B hi, B lo
  static constexpr size_t SMEM = (size_t)T3_STAGES * STAGE_BYTES + 1024;  // + 1024-byte alignment slack
  static constexpr uint32_t TMEM_COLS = 512;  // T3_NACC block accumulators of BN columns each
  // kind::tf32, FP32 accumulator, A and B K-major, N = BN, M = 128
  static constexpr uint32_t IDESC =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(T3_BM >> 4) << 24);
};

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major operand tile with the 128-byte swizzle: 8-row groups 1024 B apart
// (SBO), descriptor version 1, layout type 2; start address advanced by 32 B
// per K step of 8 TF32 values.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ uint64_t tc_clock_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase of the mbarrier at `bar` with the given parity to
// complete; gives up (returns false) once limitNs nanoseconds have passed.
// The global timer is read only between rounds of 256 polls: a wait that
// completes soon never reads it (the read is slow next to a poll).
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, long long limitNs = TC_WAIT_NS) {
  uint64_t t0 = 0;
  for (int round = 0;; round++) {
    for (int i = 0; i < 256; i++) {
      uint32_t done;
      asm volatile(
          "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
          "selp.b32 %0, 1, 0, P1;\n\t}"
          : "=r"(done)
          : "r"(bar), "r"(parity)
          : "memory");
      if (done) return true;
    }
    const uint64_t t = tc_clock_ns();
    if (round == 0) t0 = t;
    else if ((long long)(t - t0) >= limitNs) return false;
  }
}

__device__ __forceinline__ void tc_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}

// round to nearest TF32, ties away from zero (the rounding of
// cvt.rna.tf32.f32), with two integer operations on the magnitude bits
__device__ __forceinline__ float tc_rna(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
}

// v = hi + lo with both parts TF32 numbers rounded to nearest
__device__ __forceinline__ void tc_split(float x, float& hi, float& lo) {
  hi = tc_rna(x);
  lo = tc_rna(x - hi);
}

// float4 chunk c (elements 4c..4c+3) of tile row r, 128-byte swizzle
__device__ __forceinline__ uint32_t tc_swz(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

template <int BN>
__global__ void __launch_bounds__(T3_THREADS, 1)
    k_gemm_tc3(const __grid_constant__ CUtensorMap tmW, int nPad, int nrows, int nrhs, const int32_t* __restrict__ rows,
               const int32_t* __restrict__ chd, int xChild, int yChild, const float* __restrict__ X, int64_t ldx,
               int64_t xRhs, float* __restrict__ Y, int64_t ldy, int64_t yRhs, int K, int N, GrScale<float> xs,
               GrScale<float> ys, float beta, int kChunk, float* __restrict__ part, int nProd,
               int* __restrict__ errFlag) {
  using C = T3Cfg<BN>;
  static_assert(T3_NACC * BN <= 512 && BN % 32 == 0, "the block accumulators fit 512 TMEM columns");
  static_assert(T3_DWARPS == 8, "two drain warps per TMEM lane group, half the columns each");
  extern __shared__ unsigned char t3_smem_raw[];
  __shared__ const float* xrow[T3_BM];
  __shared__ float* yrow[T3_BM];
  __shared__ __align__(8) uint64_t fullA[T3_STAGES], fullB[T3_STAGES], empty[T3_STAGES], accFull[T3_NACC],
      accEmpty[T3_NACC];
  __shared__ uint32_t tmemSlot;
  __shared__ int abortFlag, lastCommit;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rawAddr = tc_smem_u32(t3_smem_raw);
  const uint32_t base = (rawAddr + 1023u) & ~1023u;  // 1024-byte aligned stages (the swizzle atom)
  unsigned char* baseP = t3_smem_raw + (base - rawAddr);
  const int r0 = blockIdx.x * T3_BM, n0 = blockIdx.y * BN;
  const int64_t M = (int64_t)nrows * nrhs;
  if (tid < T3_BM) {
    const int64_t r = r0 + tid;
    if (r < M) {
      const int q = (int)(r / nrows);
      const int node = rows[r - (int64_t)q * nrows];
      xrow[tid] = X + q * xRhs + (int64_t)(xChild ? chd[node] : node) * ldx;
      yrow[tid] = Y + q * yRhs + (int64_t)(yChild ? chd[node] : node) * ldy;
    } else {
      xrow[tid] = nullptr;
      yrow[tid] = nullptr;
    }
  }
  if (tid == 0) {
    abortFlag = 0;
    lastCommit = -1;
    for (int s = 0; s < T3_STAGES; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&fullA[s])), "r"(T3_AWARPS * 32));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&fullB[s])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&empty[s])), "r"(1));
    }
    for (int b = 0; b < T3_NACC; b++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&accFull[b])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&accEmpty[b])), "r"(T3_DWARPS * 32));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&tmemSlot)),
                 "r"(C::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (warp == T3_MWARP && lane == 0)
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmW)) : "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmemSlot;
  const int kBeg = blockIdx.z * kChunk, kEnd = min(K, kBeg + kChunk);
  const int nKB = (kEnd - kBeg + T3_BK - 1) / T3_BK;
  float R[BN / 2];  // drain warps: FP32 sums of half the row's columns

  if (warp == T3_MWARP) {
    // ------------------------------------------------- TMA + MMA (one lane)
    const bool mma = lane == 0;
    const uint64_t tmAddr = reinterpret_cast<uint64_t>(&tmW);
    auto loadB = [&](int kb) {  // operator block kb into stage kb % S (hi rows n0.., lo rows nPad + n0..)
      const int s = kb % T3_STAGES;
      const uint32_t bar = tc_smem_u32(&fullB[s]);
      const uint32_t dst = base + s * C::STAGE_BYTES + 2 * T3_A_BYTES;
      const int kx = kBeg + kb * T3_BK;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(2 * C::B_BYTES)
                   : "memory");
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
          "[%4];" ::"r"(dst),
          "l"(tmAddr), "r"(kx), "r"(n0), "r"(bar)
          : "memory");
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
          "[%4];" ::"r"(dst + C::B_BYTES),
          "l"(tmAddr), "r"(kx), "r"(nPad + n0), "r"(bar)
          : "memory");
    };
    // block kb's MMAs into accumulator kb % T3_NACC; false once the CTA aborts
    auto issue = [&](int kb) -> bool {
      const int s = kb % T3_STAGES, b = kb % T3_NACC;
      const uint32_t ph = (uint32_t)((kb / T3_STAGES) & 1);
      if (!tc_wait(tc_smem_u32(&fullA[s]), ph) || !tc_wait(tc_smem_u32(&fullB[s]), ph) ||
          (kb >= T3_NACC && !tc_wait(tc_smem_u32(&accEmpty[b]), (uint32_t)(((kb - T3_NACC) / T3_NACC) & 1))) ||
          *(volatile int*)&abortFlag) {
        atomicExch(&abortFlag, 1);
        return false;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sA = base + s * C::STAGE_BYTES, sAl = sA + T3_A_BYTES;
      const uint32_t sB = sA + 2 * T3_A_BYTES, sBl = sB + C::B_BYTES;
      const uint32_t acc = tmem + (uint32_t)(b * BN);
#pragma unroll
      for (int ks = 0; ks < T3_BK / 8; ks++) {
        const uint64_t aH = tc_desc(sA + ks * 32), aL = tc_desc(sAl + ks * 32);
        const uint64_t bH = tc_desc(sB + ks * 32), bL = tc_desc(sBl + ks * 32);
        const uint64_t ad[4] = {aH, aH, aL, aL}, bd[4] = {bH, bL, bH, bL};
#pragma unroll
        for (int t = 0; t < 4; t++) {
          if (t == 3 && nProd < 4) break;
          const uint32_t accum = (ks > 0 || t > 0) ? 1u : 0u;  // a fresh accumulator per K block
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(acc),
              "l"(ad[t]), "l"(bd[t]), "r"(C::IDESC), "r"(accum));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc_smem_u32(&empty[s]))
                   : "memory");
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc_smem_u32(&accFull[b]))
                   : "memory");
      lastCommit = kb;
      // refill the stage the previous block used once its MMAs are done
      if (kb >= 1 && kb - 1 + T3_STAGES < nKB) {
        const int sp = (kb - 1) % T3_STAGES;
        if (!tc_wait(tc_smem_u32(&empty[sp]), (uint32_t)(((kb - 1) / T3_STAGES) & 1))) {
          atomicExch(&abortFlag, 1);
          return false;
        }
        loadB(kb - 1 + T3_STAGES);
      }
      return true;
    };
    if (mma) {
      for (int kb = 0; kb < nKB && kb < T3_STAGES; kb++) loadB(kb);
      for (int kb = 0; kb < nKB; kb++)
        if (!issue(kb)) break;
    }
  } else if (warp >= T3_DWARP0) {
    // ------------------------------------------------------------- drain
    // block kb's accumulator columns [half * BN/2, +BN/2) into R; false once the CTA aborts
    const int half = (warp - T3_DWARP0) / 4;
    const uint32_t lanes = (uint32_t)((warp % 4) * 32) << 16;
    auto ld16 = [&](uint32_t addr, uint32_t(&v)[16]) {
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(addr));
    };
    auto drain = [&](int kb) -> bool {
      const int b = kb % T3_NACC;
      if (!tc_wait(tc_smem_u32(&accFull[b]), (uint32_t)((kb / T3_NACC) & 1))) atomicExch(&abortFlag, 1);
      if (__any_sync(0xffffffffu, *(volatile int*)&abortFlag != 0)) return false;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int cb = 0; cb < BN / 32; cb++) {
        uint32_t v[16];
        ld16(tmem + lanes + (uint32_t)(b * BN + half * (BN / 2) + cb * 16), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; j++) R[cb * 16 + j] += __uint_as_float(v[j]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      tc_arrive(tc_smem_u32(&accEmpty[b]));
      return true;
    };
#pragma unroll
    for (int j = 0; j < BN / 2; j++) R[j] = 0.f;
    for (int kb = 0; kb < nKB; kb++)
      if (!drain(kb)) break;
  } else {
    // ---------------------------------------------------------- X rows (A)
    const bool xsUni = xs.mod == 1;
    const float xs0 = xs.v[0];
    float4 ra[2][8];  // two K blocks in flight
    auto fetch = [&](float4(&dst)[8], int kb) {
      const int k0 = kBeg + kb * T3_BK;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int idx = tid + i * T3_AWARPS * 32, r = idx >> 3, c = idx & 7;
        const int k = k0 + 4 * c;
        const float* xr = xrow[r];
        dst[i] = (xr && k < kEnd) ? __ldcs(reinterpret_cast<const float4*>(xr + k)) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    };
    // stores block kb (in src) into its stage; false once the CTA aborts
    auto stage = [&](const float4(&src)[8], int kb) -> bool {
      const int s = kb % T3_STAGES;
      if (kb >= T3_STAGES && !tc_wait(tc_smem_u32(&empty[s]), (uint32_t)(((kb - T3_STAGES) / T3_STAGES) & 1)))
        atomicExch(&abortFlag, 1);
      if (*(volatile int*)&abortFlag) return false;  // the tensor core may still read this stage: nobody writes it
      unsigned char* pA = baseP + s * C::STAGE_BYTES;
      const int k0 = kBeg + kb * T3_BK;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int idx = tid + i * T3_AWARPS * 32, r = idx >> 3, c = idx & 7;
        float v[4] = {src[i].x, src[i].y, src[i].z, src[i].w};
        if (!xsUni || xs0 != 1.f) {
#pragma unroll
          for (int j = 0; j < 4; j++) v[j] *= xsUni ? xs0 : gr_sel(xs, k0 + 4 * c + j);
        }
        float4 h, l;
        tc_split(v[0], h.x, l.x);
        tc_split(v[1], h.y, l.y);
        tc_split(v[2], h.z, l.z);
        tc_split(v[3], h.w, l.w);
        *reinterpret_cast<float4*>(pA + tc_swz(r, c)) = h;
        *reinterpret_cast<float4*>(pA + T3_A_BYTES + tc_swz(r, c)) = l;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic stores -> tensor-core reads
      tc_arrive(tc_smem_u32(&fullA[s]));
      return true;
    };
    if (nKB > 0) fetch(ra[0], 0);
    if (nKB > 1) fetch(ra[1], 1);
    for (int kb = 0; kb < nKB; kb += 2) {
      if (!stage(ra[0], kb)) break;
      if (kb + 2 < nKB) fetch(ra[0], kb + 2);
      if (kb + 1 >= nKB) break;
      if (!stage(ra[1], kb + 1)) break;
      if (kb + 3 < nKB) fetch(ra[1], kb + 3);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const bool ok = abortFlag == 0 && nKB > 0;
  if (abortFlag && tid == 0) atomicExch(errFlag, 1);
  if (abortFlag && warp == T3_MWARP && lane == 0 && lastCommit >= 0) {
    // an aborted CTA may have MMAs in flight: one last bounded wait on the
    // most recent commit (it covers every earlier MMA) before the TMEM is freed
    const int lc = lastCommit;
    tc_wait(tc_smem_u32(&empty[lc % T3_STAGES]), (uint32_t)((lc / T3_STAGES) & 1));
  }
  if (ok && warp >= T3_DWARP0 && warp < T3_MWARP) {
    // epilogue: the drain warps hold the rows' sums (row m = 32 (w % 4) + lane,
    // columns half * BN/2 ..)
    const int m = (warp % 4) * 32 + lane;
    const int half = (warp - T3_DWARP0) / 4;
    float* yr = yrow[m];
    const bool vecY = ((uintptr_t)yr % 16 == 0);
#pragma unroll
    for (int cb = 0; cb < BN / 32; cb++) {
      const int nb = n0 + half * (BN / 2) + cb * 16;
      if (part) {
        if (r0 + m < M) {
          float* pr = part + ((int64_t)blockIdx.z * M + r0 + m) * N;
#pragma unroll
          for (int j = 0; j < 16; j++)
            if (nb + j < N) pr[nb + j] = R[cb * 16 + j];
        }
      } else if (yr) {
        float a[16];
#pragma unroll
        for (int j = 0; j < 16; j++) a[j] = R[cb * 16 + j] * gr_sel(ys, nb + j);
        if (vecY && nb + 16 <= N) {
#pragma unroll
          for (int j = 0; j < 16; j += 4) {
            float4* p = reinterpret_cast<float4*>(yr + nb + j);
            float4 o = make_float4(a[j], a[j + 1], a[j + 2], a[j + 3]);
            if (beta != 0.f) {
              const float4 y = *p;
              o = make_float4(beta * y.x + o.x, beta * y.y + o.y, beta * y.z + o.z, beta * y.w + o.w);
            }
            *p = o;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; j++)
            if (nb + j < N) yr[nb + j] = beta == 0.f ? a[j] : beta * yr[nb + j] + a[j];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::TMEM_COLS));
}

// The error path of the bounded waits, on its own: one CTA allocates TMEM
// like the GEMM, inits an mbarrier and waits for its first phase with a wait
// limit of limitNs.  With arrive != 0 thread 0 arrives first and the wait
// completes; otherwise nothing arrives (no MMA is ever issued), the wait runs
// out, the kernel sets *errFlag, frees its TMEM and returns.
__global__ void __launch_bounds__(TC_THREADS) k_wait_selftest(int arrive, long long limitNs, int* errFlag) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmemSlot;
  __shared__ int abortFlag;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    abortFlag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&tmemSlot)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (arrive && tid == 0) tc_arrive(tc_smem_u32(&bar));
  if (!tc_wait(tc_smem_u32(&bar), 0u, limitNs)) atomicExch(&abortFlag, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (abortFlag && tid == 0) atomicExch(errFlag, 1);
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmemSlot), "r"(TC_TMEM_COLS));
}

// ------------------------------------------------------------------ host side

constexpr int T3_BN = 160;  // covers the 152-wide surfaces of np = 6 in one tile

// round to nearest TF32 (ties away from zero), as cvt.rna.tf32.f32
inline float host_rna_tf32(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// The hi / lo parts of W (from FP64) in the padded stacked layout.
inline std::vector<float> tc_split_operator(const std::vector<double>& W, int n, int k, int nPad, int kPad) {
  std::vector<float> t((size_t)2 * nPad * kPad, 0.f);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < k; j++) {
      const double w = W[(size_t)i * k + j];
      const float hi = host_rna_tf32((float)w);
      const float lo = host_rna_tf32((float)(w - (double)hi));
      t[(size_t)i * kPad + j] = hi;
      t[(size_t)(nPad + i) * kPad + j] = lo;
    }
  return t;
}

// The TMA tensor map of a TcOp: box 32 K values x T3_BN rows, 128-byte swizzle.
inline std::string tc_encode_map(TcOp& op) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return "cuTensorMapEncodeTiled not available";
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)op.kPad, (cuuint64_t)(2 * op.nPad)};
  const cuuint64_t strides[1] = {(cuuint64_t)op.kPad * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)T3_BK, (cuuint32_t)T3_BN};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(&op.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, op.p, dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
  return std::string();
}

// Uploads W (n x k, FP64 row-major) as a TcOp; `alloc(float*&, size_t)`
// returns device memory that lives as long as the handle.
template <typename Alloc>
inline std::string tc_prepare_operator(TcOp& op, const std::vector<double>& W, int n, int k, Alloc alloc) {
  op.ready = false;
  op.n = n;
  op.k = k;
  op.nPad = (n + T3_BN - 1) / T3_BN * T3_BN;
  op.kPad = (k + T3_BK - 1) / T3_BK * T3_BK;
  const std::vector<float> t = tc_split_operator(W, n, k, op.nPad, op.kPad);
  if (!op.p || t.size() > op.cap) {
    std::string e = alloc(op.p, t.size());
    if (!e.empty()) return e;
    op.cap = t.size();
  }
  cudaError_t ce = cudaMemcpy(op.p, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) return std::string("operator upload: ") + cudaGetErrorString(ce);
  std::string e = tc_encode_map(op);
  op.ready = e.empty();
  return e;
}

// Whether the tensor-core GEMM takes these operands: X rows 16-byte aligned
// with K a multiple of 4 (the rows are staged as float4), and the operator
// prepared for the same N and K.
inline bool tc_usable(const TcOp* op, const float* X, int64_t ldx, int64_t xRhs, int K, int N) {
  return op && op->ready && op->n == N && op->k == K && ((uintptr_t)X % 16 == 0) && ldx % 4 == 0 &&
         xRhs % 4 == 0 && K % 4 == 0;
}

// Launches k_gemm_tc3; splits K into chunks (partial tiles reduced in a
// fixed order by k_gemm_reduce_t) when the tiles alone would leave fewer
// than splitCtas CTAs.  Returns the number of kernels launched.
inline int launch_gemm_tc3(cudaStream_t st, int splitCtas, float* scratch, size_t scratchElems, const TcOp& op,
                           int nProd, int* errFlag, int nrows, int nrhs, const int32_t* rows, const int32_t* chd,
                           int xChild, int yChild, const float* X, int64_t ldx, int64_t xRhs, float* Y, int64_t ldy,
                           int64_t yRhs, int K, int N, GrScale<float> xs, GrScale<float> ys, float beta) {
  if (nrows <= 0 || nrhs <= 0) return 0;
  const int64_t M = (int64_t)nrows * nrhs;
  const int tiles = (int)((M + T3_BM - 1) / T3_BM) * ((N + T3_BN - 1) / T3_BN);
  int splits = 1;
  if (scratch && tiles < splitCtas && K >= 8 * T3_BK) {
    splits = std::min(8, (splitCtas + tiles - 1) / tiles);
    splits = std::min(splits, K / (4 * T3_BK));
    while (splits > 1 && (size_t)splits * M * N > scratchElems) splits--;
  }
  const int kChunk = splits > 1 ? ((K + splits - 1) / splits + T3_BK - 1) / T3_BK * T3_BK : K;
  if (splits > 1) splits = (K + kChunk - 1) / kChunk;
  static bool attrSet = false;  // per process; the attribute is per function, not per device context
  if (!attrSet) {
    cudaFuncSetAttribute(k_gemm_tc3<T3_BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T3Cfg<T3_BN>::SMEM);
    attrSet = true;
  }
  dim3 grid((unsigned)((M + T3_BM - 1) / T3_BM), (N + T3_BN - 1) / T3_BN, splits);
  float* pt = splits > 1 ? scratch : nullptr;
  k_gemm_tc3<T3_BN><<<grid, T3_THREADS, T3Cfg<T3_BN>::SMEM, st>>>(op.map, op.nPad, nrows, nrhs, rows, chd, xChild,
                                                                   yChild, X, ldx, xRhs, Y, ldy, yRhs, K, N, xs, ys,
                                                                   beta, kChunk, pt, nProd, errFlag);
  if (splits == 1) return 1;
  const int64_t tot = M * N;
  k_gemm_reduce_t<float><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(nrows, nrhs, rows, chd, yChild, Y, ldy, yRhs,
                                                                         N, splits, scratch, ys, beta);
  return 2;
}

// FP32 row GEMM launcher: the tensor-core kernel when `tc` names a prepared
// operator and the X rows allow it; else the wide-tile CUDA-core kernel when
// the transposed operator Wt (ldw per row) is given and the X rows allow
// 16-byte fetches; else the 128 x 64 CUDA-core kernel.
inline int launch_gemm_rows_f32(cudaStream_t st, int splitCtas, float* scratch, size_t scratchElems, const TcOp* tc,
                                int nProd, int* errFlag, int nrows, int nrhs, const int32_t* rows, const int32_t* chd,
                                int xChild, int yChild, const float* X, int64_t ldx, int64_t xRhs, const float* W,
                                const float* Wt, int ldw, float* Y, int64_t ldy, int64_t yRhs, int K, int N,
                                GrScale<float> xs, GrScale<float> ys, float beta) {
  if (nrows <= 0 || nrhs <= 0) return 0;
  if (errFlag && tc_usable(tc, X, ldx, xRhs, K, N))
    return launch_gemm_tc3(st, splitCtas, scratch, scratchElems, *tc, nProd, errFlag, nrows, nrhs, rows, chd, xChild,
                           yChild, X, ldx, xRhs, Y, ldy, yRhs, K, N, xs, ys, beta);
  const bool xvec = ((uintptr_t)X % 16 == 0) && ldx % 4 == 0 && xRhs % 4 == 0 && K % 4 == 0;
  if (Wt && xvec && ((uintptr_t)Wt % 16 == 0) && ldw % GW_BN == 0)
    return launch_gemm_rows_w(st, splitCtas, scratch, scratchElems, nrows, nrhs, rows, chd, xChild, yChild, X, ldx,
                              xRhs, Wt, ldw, Y, ldy, yRhs, K, N, xs, ys, beta);
  return launch_gemm_rows<float, 16>(st, splitCtas, scratch, scratchElems, nrows, nrhs, rows, chd, xChild, yChild, X,
                                     ldx, xRhs, W, Y, ldy, yRhs, K, N, xs, ys, beta);
}

}  // namespace fmmg
