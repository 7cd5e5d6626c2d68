// gemm_tc.cuh -- the FP32 row GEMM of the translation stages on the 5th-
// generation tensor cores (tcgen05, kind::tf32) as 3xTF32 split products.
//
// Same contract as k_gemm_rows_t (gemm_rows.cuh):
//   Y[row] = beta * Y[row] + ys .* (W (xs .* X[row]))  for every listed node
// and right-hand side, W N x K row-major, or raw partial tiles for split K.
// Each operand value x is split into hi = tf32(x) (round to nearest) and
// lo = x - hi; the tensor core accumulates hi*hi + hi*lo + lo*hi in FP32 in
// tensor memory, which restores FP32-level accuracy from TF32 products.
//
// CTA = 128 threads, tile 128 rows x 64 outputs, K in blocks of 32 (one
// 128-byte row of FP32 per operand row).  Per K block all threads fetch X and
// W rows as 16-byte vectors (rows gathered by node; the next block's loads
// are issued while the current block multiplies), split them and store
// A_hi, A_lo (128 x 32) and B_hi, B_lo (64 x 32) K-major in shared memory with
// the 128-byte swizzle; one elected thread issues 12 tcgen05.mma (4 K steps x
// 3 products, M = 128, N = 64, K = 8) into a 128 x 64 FP32 accumulator in
// TMEM and commits them to the stage's mbarrier.  Two stages: block b + 1 is
// fetched while block b multiplies.  The epilogue reads TMEM with
// tcgen05.ld (warp w owns lanes 32w..32w+31, i.e. tile rows) and applies the
// scale and beta.  Every mbarrier wait is bounded: on timeout the kernel
// records an error flag, stops issuing work, waits (bounded) for what it
// issued, frees its TMEM and returns.
//
// Requires the VEC layout of k_gemm_rows_t (16-byte aligned rows, K % 4 == 0).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "gemm_rows.cuh"

namespace fmmg {

constexpr int TC_BM = 128, TC_BN = 64, TC_BK = 32, TC_THREADS = 128, TC_STAGES = 2;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 4;                    // 16 KB per A part
constexpr int TC_B_BYTES = TC_BN * TC_BK * 4;                    // 8 KB per B part
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_B_BYTES;  // hi + lo of both
constexpr size_t TC_SMEM_BYTES = (size_t)TC_STAGES * TC_STAGE_BYTES + 1024;  // + alignment slack
constexpr uint32_t TC_TMEM_COLS = 64;
constexpr long long TC_WAIT_NS = 1000000000ll;  // a bounded mbarrier wait gives up after 1 s

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major operand tile with the 128-byte swizzle: 8-row groups 1024 B apart
// (SBO), version 1, layout type 2; start address advanced by 32 B per K step.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::tf32, FP32 accumulator, both operands K-major, M = 128, N = 64
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                              ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ uint64_t tc_clock_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase of the mbarrier at `bar` with the given parity to
// complete; gives up (returns false) once limitNs nanoseconds have passed.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, long long limitNs = TC_WAIT_NS) {
  const uint64_t t0 = tc_clock_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((long long)(tc_clock_ns() - t0) >= limitNs) return false;
  }
}

__device__ __forceinline__ void tc_split(float x, float& hi, float& lo) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  hi = __uint_as_float(h);
  lo = x - hi;
}

// float4 chunk c (elements 4c..4c+3) of tile row r, 128-byte swizzle
__device__ __forceinline__ uint32_t tc_swz(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

__global__ void __launch_bounds__(TC_THREADS)
    k_gemm_rows_tc(int nrows, int nrhs, const int32_t* __restrict__ rows, const int32_t* __restrict__ chd, int xChild,
                   int yChild, const float* __restrict__ X, int64_t ldx, int64_t xRhs, const float* __restrict__ W,
                   float* __restrict__ Y, int64_t ldy, int64_t yRhs, int K, int N, GrScale<float> xs,
                   GrScale<float> ys, float beta, int kChunk, float* __restrict__ part, int* __restrict__ errFlag) {
  extern __shared__ unsigned char tc_smem_raw[];
  __shared__ const float* xrow[TC_BM];
  __shared__ float* yrow[TC_BM];
  __shared__ __align__(8) uint64_t mbar[TC_STAGES];
  __shared__ uint32_t tmemSlot;
  __shared__ int abortFlag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // 1024-byte aligned operand stages inside the dynamic shared memory
  const uint32_t rawAddr = tc_smem_u32(tc_smem_raw);
  const uint32_t base = (rawAddr + 1023u) & ~1023u;
  unsigned char* baseP = tc_smem_raw + (base - rawAddr);
  const int r0 = blockIdx.x * TC_BM, n0 = blockIdx.y * TC_BN;
  {
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
  if (tid == 0) {
    abortFlag = 0;
    for (int s = 0; s < TC_STAGES; s++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&mbar[s])), "r"(1));
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
  const uint32_t tmem = tmemSlot;

  const int kBeg = blockIdx.z * kChunk, kEnd = min(K, kBeg + kChunk);
  const int nKB = (kEnd - kBeg + TC_BK - 1) / TC_BK;
  bool ok;
  int issued = -1;  // last K block whose MMAs were issued (the same on every thread)
  // the next K block's raw operands travel in registers while the current block multiplies
  float4 ra[8], rb[4];
  auto fetch = [&](int kb) {
    const int k0 = kBeg + kb * TC_BK;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int idx = tid + i * TC_THREADS, r = idx >> 3, c = idx & 7;
      const int k = k0 + 4 * c;
      const float* xr = xrow[r];
      ra[i] = (xr && k < kEnd) ? *reinterpret_cast<const float4*>(xr + k) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int idx = tid + i * TC_THREADS, r = idx >> 3, c = idx & 7;
      const int k = k0 + 4 * c, n = n0 + r;
      rb[i] = (n < N && k < kEnd) ? *reinterpret_cast<const float4*>(W + (int64_t)n * K + k)
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  if (nKB > 0) fetch(0);
  for (int kb = 0; kb < nKB; kb++) {
    const int s = kb & 1;
    const uint32_t sA = base + s * TC_STAGE_BYTES;  // A_hi, A_lo, B_hi, B_lo
    const uint32_t sAl = sA + TC_A_BYTES, sB = sA + 2 * TC_A_BYTES, sBl = sB + TC_B_BYTES;
    unsigned char* pA = baseP + s * TC_STAGE_BYTES;
    if (kb >= TC_STAGES) {  // the MMAs of block kb - 2 read this stage
      if (!tc_wait(tc_smem_u32(&mbar[s]), (uint32_t)(((kb - TC_STAGES) / TC_STAGES) & 1))) atomicExch(&abortFlag, 1);
      __syncthreads();  // every thread's wait has ended: abortFlag is final for this block
      if (abortFlag) break;  // the tensor core may still read this stage: nobody writes it
    }
    const int k0 = kBeg + kb * TC_BK;
#pragma unroll
    for (int i = 0; i < 8; i++) {  // A: 128 rows x 8 float4 chunks (8 threads per row)
      const int idx = tid + i * TC_THREADS, r = idx >> 3, c = idx & 7;
      const int k = k0 + 4 * c;
      float4 h, l;
      tc_split(ra[i].x * gr_sel(xs, k), h.x, l.x);
      tc_split(ra[i].y * gr_sel(xs, k + 1), h.y, l.y);
      tc_split(ra[i].z * gr_sel(xs, k + 2), h.z, l.z);
      tc_split(ra[i].w * gr_sel(xs, k + 3), h.w, l.w);
      *reinterpret_cast<float4*>(pA + tc_swz(r, c)) = h;
      *reinterpret_cast<float4*>(pA + TC_A_BYTES + tc_swz(r, c)) = l;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {  // B: 64 output rows x 8 chunks
      const int idx = tid + i * TC_THREADS, r = idx >> 3, c = idx & 7;
      float4 h, l;
      tc_split(rb[i].x, h.x, l.x);
      tc_split(rb[i].y, h.y, l.y);
      tc_split(rb[i].z, h.z, l.z);
      tc_split(rb[i].w, h.w, l.w);
      *reinterpret_cast<float4*>(pA + 2 * TC_A_BYTES + tc_swz(r, c)) = h;
      *reinterpret_cast<float4*>(pA + 2 * TC_A_BYTES + TC_B_BYTES + tc_swz(r, c)) = l;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic stores -> tensor-core reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    issued = kb;
    if (tid == 0) {
#pragma unroll
      for (int ks = 0; ks < TC_BK / 8; ks++) {
        const uint64_t aH = tc_desc(sA + ks * 32), aL = tc_desc(sAl + ks * 32);
        const uint64_t bH = tc_desc(sB + ks * 32), bL = tc_desc(sBl + ks * 32);
        const uint64_t ad[3] = {aH, aH, aL}, bd[3] = {bH, bL, bH};
#pragma unroll
        for (int t = 0; t < 3; t++) {
          const uint32_t accum = (kb > 0 || ks > 0 || t > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
              "l"(ad[t]), "l"(bd[t]), "r"(TC_IDESC), "r"(accum));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc_smem_u32(&mbar[s]))
                   : "memory");
    }
    if (kb + 1 < nKB) fetch(kb + 1);
  }
  // wait for the last issued block (its commit covers every earlier MMA); if
  // that wait runs out, wait once more (bounded) so that the MMAs are done
  // before the accumulator's TMEM is freed, and skip the epilogue
  if (issued >= 0) {
    const uint32_t lb = tc_smem_u32(&mbar[issued & 1]), lp = (uint32_t)((issued / TC_STAGES) & 1);
    if (!tc_wait(lb, lp)) {
      atomicExch(&abortFlag, 1);
      tc_wait(lb, lp);
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  ok = abortFlag == 0;
  if (!ok && tid == 0) atomicExch(errFlag, 1);
  // epilogue: warp w reads TMEM lanes 32w..32w+31 (tile rows), 64 columns in 4 loads of 16
  const int m = warp * 32 + lane;
  float* yr = yrow[m];
  const int64_t M = (int64_t)nrows * nrhs;
  // every thread reads the same abortFlag after the barrier: the warps skip
  // the (warp-collective) TMEM loads together
#pragma unroll
  for (int cb = 0; cb < TC_BN / 16; cb++) {
    if (!ok || issued < 0) break;
    uint32_t v[16];
    const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (part) {
      if (r0 + m < M) {
        float* pr = part + ((int64_t)blockIdx.z * M + r0 + m) * N;
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int n = n0 + cb * 16 + j;
          if (n < N) pr[n] = __uint_as_float(v[j]);
        }
      }
    } else if (yr) {
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int n = n0 + cb * 16 + j;
        if (n < N) {
          const float a = __uint_as_float(v[j]) * gr_sel(ys, n);
          yr[n] = beta == 0.f ? a : beta * yr[n] + a;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
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
  if (arrive && tid == 0) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(tc_smem_u32(&bar))
                 : "memory");
  }
  if (!tc_wait(tc_smem_u32(&bar), 0u, limitNs)) atomicExch(&abortFlag, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (abortFlag && tid == 0) atomicExch(errFlag, 1);
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmemSlot), "r"(TC_TMEM_COLS));
}

// FP32 row GEMM launcher: the tensor-core kernel when useTC and the operands
// have the 16-byte row layout; else the wide-tile CUDA-core kernel when the
// transposed operator Wt (ldw per row) is given and the X rows allow 16-byte
// fetches; else the 128 x 64 CUDA-core kernel.  Split K as in
// launch_gemm_rows (chunks a multiple of 32 on the tensor-core path).
inline int launch_gemm_rows_f32(cudaStream_t st, int splitCtas, float* scratch, size_t scratchElems, bool useTC,
                                int* errFlag, int nrows, int nrhs, const int32_t* rows, const int32_t* chd,
                                int xChild, int yChild, const float* X, int64_t ldx, int64_t xRhs, const float* W,
                                const float* Wt, int ldw, float* Y, int64_t ldy, int64_t yRhs, int K, int N,
                                GrScale<float> xs, GrScale<float> ys, float beta) {
  if (nrows <= 0 || nrhs <= 0) return 0;
  const bool xvec = ((uintptr_t)X % 16 == 0) && ldx % 4 == 0 && xRhs % 4 == 0 && K % 4 == 0;
  const bool vec = xvec && ((uintptr_t)W % 16 == 0);
  if ((!useTC || !vec || !errFlag) && Wt && xvec && ((uintptr_t)Wt % 16 == 0) && ldw % GW_BN == 0)
    return launch_gemm_rows_w(st, splitCtas, scratch, scratchElems, nrows, nrhs, rows, chd, xChild, yChild, X, ldx,
                              xRhs, Wt, ldw, Y, ldy, yRhs, K, N, xs, ys, beta);
  if (!useTC || !vec || !errFlag)
    return launch_gemm_rows<float, 16>(st, splitCtas, scratch, scratchElems, nrows, nrhs, rows, chd, xChild, yChild, X,
                                       ldx, xRhs, W, Y, ldy, yRhs, K, N, xs, ys, beta);
  const int64_t M = (int64_t)nrows * nrhs;
  const int tiles = (int)((M + TC_BM - 1) / TC_BM) * ((N + TC_BN - 1) / TC_BN);
  int splits = 1;
  if (scratch && tiles < splitCtas && K >= 4 * TC_BK) {
    splits = std::min(8, (splitCtas + tiles - 1) / tiles);
    splits = std::min(splits, K / (2 * TC_BK));
    while (splits > 1 && (size_t)splits * M * N > scratchElems) splits--;
  }
  const int kChunk = splits > 1 ? ((K + splits - 1) / splits + TC_BK - 1) / TC_BK * TC_BK : K;
  if (splits > 1) splits = (K + kChunk - 1) / kChunk;
  static bool attrSet = false;  // per process; the attribute is per function, not per device context
  if (!attrSet) {
    cudaFuncSetAttribute(k_gemm_rows_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_BYTES);
    attrSet = true;
  }
  dim3 grid((unsigned)((M + TC_BM - 1) / TC_BM), (N + TC_BN - 1) / TC_BN, splits);
  float* pt = splits > 1 ? scratch : nullptr;
  k_gemm_rows_tc<<<grid, TC_THREADS, TC_SMEM_BYTES, st>>>(nrows, nrhs, rows, chd, xChild, yChild, X, ldx, xRhs, W, Y,
                                                          ldy, yRhs, K, N, xs, ys, beta, kChunk, pt, errFlag);
  if (splits == 1) return 1;
  const int64_t tot = M * N;
  k_gemm_reduce_t<float><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(nrows, nrhs, rows, chd, yChild, Y, ldy, yRhs,
                                                                         N, splits, scratch, ys, beta);
  return 2;
}

}  // namespace fmmg
