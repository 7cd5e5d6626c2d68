// cuda_common.cuh -- helpers shared by the FP64 (stages.cu) and mixed-precision
// (mixed.cu) stage kernels.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "plan.hpp"

namespace fmmg {

#define FMMG_CK(x)                                                                  \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess) return std::string(#x) + ": " + cudaGetErrorString(e_); \
  } while (0)

#define FMMG_TRY(x)             \
  do {                          \
    std::string e_ = (x);       \
    if (!e_.empty()) return e_; \
  } while (0)

// per-component scale of a row (the homogeneous level factors 2^(+-l*deg))
struct Scale4 {
  double v[4];
  int mod;
};

inline Scale4 level_scale(const Plan& P, int level, double sign) {
  Scale4 s;
  s.mod = P.sdm;
  for (int k = 0; k < 4; k++) s.v[k] = k < P.sdm ? std::exp2(sign * level * P.deg[k]) : 1.0;
  return s;
}
inline Scale4 unit_scale() {
  Scale4 s;
  s.mod = 1;
  s.v[0] = s.v[1] = s.v[2] = s.v[3] = 1.0;
  return s;
}

// (2np)^3 grid of the spectral M2L: N points per axis, NH kept x frequencies,
// the np^3 lattice sits at offset H = np/2 (matmgnt3d_mpi.cpp:321)
template <int NP>
struct FftDims {
  static constexpr int N = 2 * NP, NH = NP + 1, H = NP / 2;
};
// The FP32 pass's grid: 2np - 1 points per axis, the smallest on which the
// band-to-band convolution of M2L does not wrap (offsets -(np-1)..np-1);
// odd, so the r2c half spectrum has no Nyquist term.
template <int NP>
struct FftDims32 {
  static constexpr int N = 2 * NP - 1, NH = NP, H = NP / 2;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

}  // namespace fmmg
