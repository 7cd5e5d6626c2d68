// tc_op.hpp -- an FP32 row-GEMM operator prepared for the tensor-core kernel
// k_gemm_tc3 (gemm_tc.cuh).  Host-side data only, so both the CUDA sources
// and the host C++ (the DevState that owns it) can hold one.
#pragma once

#include <cuda.h>

#include <cstddef>

namespace fmmg {

// W (N x K) as hi and lo TF32 parts, N padded to a multiple of the kernel's
// N tile and K to a multiple of 32 with zeros, stacked [2 * nPad][kPad] FP32
// (hi rows first) in device memory at p, and the TMA tensor map over it.
struct TcOp {
  float* p = nullptr;
  size_t cap = 0;  // allocated floats
  int n = 0, k = 0, nPad = 0, kPad = 0;
  CUtensorMap map;  // 64-byte aligned by its declaration
  bool ready = false;
};

}  // namespace fmmg
