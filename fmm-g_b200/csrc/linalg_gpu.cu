// linalg_gpu.cu -- the operator builder's dense FP64 linear algebra on the GPU
// (setup only): the one-sided Jacobi SVD behind the truncated pseudo-inverses
// (common/vecmatop.cpp:129-164, common/svdrep.cpp:38-80) and the C2E x M2M
// fold.  Both reproduce linalg.cpp's host arithmetic operation for operation
// -- every sum in the host's order, products and sums rounded separately (no
// FMA contraction, as the host build), the same tournament pairing and the
// same rotation formulas -- so the tables are bit-identical to the host's
// whichever side builds them.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "plan.hpp"

namespace fmmg {

#define LG_CK(x)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return std::string("linalg device: ") + cudaGetErrorString(e_); \
  } while (0)

// sqrt(1 + z^2) as the host computes it (jacobi_hyp1 in linalg.cpp)
__device__ __forceinline__ double lg_hyp1(double z) {
  const double az = fabs(z);
  return az > 1e100 ? az : __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(z, z)));
}

// One tournament round: warp w takes pair w (columns p < q of Z, ld apart,
// first m rows the working matrix, then the n rows of V).  Lane l sums the
// rows i = l (mod 32) in increasing i and a butterfly over offsets 16 .. 1
// combines the 32 partial sums (the host's jacobi_dots32 order; every lane
// ends with the same value); when the pair is not yet orthogonal all lanes
// apply the rotation to both full columns.
__global__ void __launch_bounds__(256) k_jacobi_round(double* __restrict__ Z, long long ld, int m, int n,
                                                      const int2* __restrict__ pairs, int npair,
                                                      int* __restrict__ rotated) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= npair) return;
  const int2 pq = pairs[w];
  if (pq.y >= n) return;
  double* zp = Z + (long long)pq.x * ld;
  double* zq = Z + (long long)pq.y * ld;
  double a = 0.0, b = 0.0, g = 0.0;
  for (int i = lane; i < m; i += 32) {
    const double x = zp[i], y = zq[i];
    a = __dadd_rn(a, __dmul_rn(x, x));
    b = __dadd_rn(b, __dmul_rn(y, y));
    g = __dadd_rn(g, __dmul_rn(x, y));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    a = __dadd_rn(a, __shfl_xor_sync(0xffffffffu, a, off));
    b = __dadd_rn(b, __shfl_xor_sync(0xffffffffu, b, off));
    g = __dadd_rn(g, __shfl_xor_sync(0xffffffffu, g, off));
  }
  if (a == 0.0 || b == 0.0 || fabs(g) <= __dmul_rn(1e-15, __dsqrt_rn(__dmul_rn(a, b)))) return;
  const double zeta = __ddiv_rn(__dsub_rn(b, a), __dmul_rn(2.0, g));
  const double t = __ddiv_rn(copysign(1.0, zeta), __dadd_rn(fabs(zeta), lg_hyp1(zeta)));
  const double c = __ddiv_rn(1.0, lg_hyp1(t));
  const double s = __dmul_rn(c, t);
  if (lane == 0) atomicAdd(rotated, 1);
  for (long long i = lane; i < ld; i += 32) {
    const double x = zp[i], y = zq[i];
    zp[i] = __dsub_rn(__dmul_rn(c, x), __dmul_rn(s, y));
    zq[i] = __dadd_rn(__dmul_rn(s, x), __dmul_rn(c, y));
  }
}

// Z (ld x n column-major, ld = m + n) in place, the host's sweep loop: at most
// 80 sweeps of nn - 1 tournament rounds, stopping after a sweep that rotated
// no pair.  Returns an empty string on success.
std::string svd_onesided_device(int device, int m, int n, std::vector<double>& Z) {
  const long long ld = (long long)m + n;
  const int nn = n + (n & 1), npair = nn / 2;
  // the host's pairing, round by round
  std::vector<int> top(npair), bot(npair);
  for (int i = 0; i < npair; i++) {
    top[i] = 2 * i;
    bot[i] = 2 * i + 1;
  }
  std::vector<int2> sched((size_t)(nn - 1) * npair);
  for (int round = 0; round < nn - 1; round++) {
    for (int k = 0; k < npair; k++)
      sched[(size_t)round * npair + k] = make_int2(std::min(top[k], bot[k]), std::max(top[k], bot[k]));
    if (npair > 1) {
      int tlast = top[npair - 1], b0 = bot[0];
      for (int i = npair - 1; i > 1; i--) top[i] = top[i - 1];
      top[1] = b0;
      for (int i = 0; i < npair - 1; i++) bot[i] = bot[i + 1];
      bot[npair - 1] = tlast;
    }
  }
  LG_CK(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  LG_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  double* dZ = nullptr;
  int2* dP = nullptr;
  int* dRot = nullptr;
  std::string err;
  auto run = [&]() -> std::string {
    LG_CK(cudaMalloc(&dZ, sizeof(double) * Z.size()));
    LG_CK(cudaMalloc(&dP, sizeof(int2) * sched.size()));
    LG_CK(cudaMalloc(&dRot, sizeof(int)));
    LG_CK(cudaMemcpyAsync(dZ, Z.data(), sizeof(double) * Z.size(), cudaMemcpyHostToDevice, st));
    LG_CK(cudaMemcpyAsync(dP, sched.data(), sizeof(int2) * sched.size(), cudaMemcpyHostToDevice, st));
    const int threads = 256, blocks = (npair * 32 + threads - 1) / threads;
    for (int sweep = 0; sweep < 80; sweep++) {
      LG_CK(cudaMemsetAsync(dRot, 0, sizeof(int), st));
      for (int round = 0; round < nn - 1; round++)
        k_jacobi_round<<<blocks, threads, 0, st>>>(dZ, ld, m, n, dP + (size_t)round * npair, npair, dRot);
      LG_CK(cudaGetLastError());
      int rot = 0;
      LG_CK(cudaMemcpyAsync(&rot, dRot, sizeof(int), cudaMemcpyDeviceToHost, st));
      LG_CK(cudaStreamSynchronize(st));
      if (!rot) break;
    }
    LG_CK(cudaMemcpyAsync(Z.data(), dZ, sizeof(double) * Z.size(), cudaMemcpyDeviceToHost, st));
    LG_CK(cudaStreamSynchronize(st));
    return std::string();
  };
  err = run();
  cudaFree(dZ);
  cudaFree(dP);
  cudaFree(dRot);
  cudaStreamDestroy(st);
  return err;
}

// C += A B for row-major A (rows x inner), B (inner x w), C (rows x w): one
// thread per element of C, its inner terms added in order (the host's
// blocked loop keeps that order per element).
__global__ void __launch_bounds__(256) k_gemm_rows_seq(int rows, int inner, int w, const double* __restrict__ A,
                                                       const double* __restrict__ B, double* __restrict__ C) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (j >= w || r >= rows) return;
  const double* a = A + (size_t)r * inner;
  double acc = C[(size_t)r * w + j];
  for (int c = 0; c < inner; c++) acc = __dadd_rn(acc, __dmul_rn(a[c], B[(size_t)c * w + j]));
  C[(size_t)r * w + j] = acc;
}

std::string gemm_rows_device(int device, int rows, int inner, int w, const double* A, const double* B, double* C) {
  LG_CK(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  LG_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  double *dA = nullptr, *dB = nullptr, *dC = nullptr;
  auto run = [&]() -> std::string {
    LG_CK(cudaMalloc(&dA, sizeof(double) * (size_t)rows * inner));
    LG_CK(cudaMalloc(&dB, sizeof(double) * (size_t)inner * w));
    LG_CK(cudaMalloc(&dC, sizeof(double) * (size_t)rows * w));
    LG_CK(cudaMemcpyAsync(dA, A, sizeof(double) * (size_t)rows * inner, cudaMemcpyHostToDevice, st));
    LG_CK(cudaMemcpyAsync(dB, B, sizeof(double) * (size_t)inner * w, cudaMemcpyHostToDevice, st));
    LG_CK(cudaMemcpyAsync(dC, C, sizeof(double) * (size_t)rows * w, cudaMemcpyHostToDevice, st));
    k_gemm_rows_seq<<<dim3((w + 255) / 256, rows), 256, 0, st>>>(rows, inner, w, dA, dB, dC);
    LG_CK(cudaGetLastError());
    LG_CK(cudaMemcpyAsync(C, dC, sizeof(double) * (size_t)rows * w, cudaMemcpyDeviceToHost, st));
    LG_CK(cudaStreamSynchronize(st));
    return std::string();
  };
  std::string err = run();
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dC);
  cudaStreamDestroy(st);
  return err;
}

}  // namespace fmmg
