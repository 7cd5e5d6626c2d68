// plan_pool.cuh -- device work buffers of the GPU plan build (tree_gpu.cu,
// lists_gpu.cu) and of the coordinate staging of the upload.  Released blocks stay with the process, per device, for the
// next build (a setup per time step for moving points), so repeated setups
// allocate nothing; the best-fitting free block is taken.  The blocks are
// freed at process exit.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

namespace fmmg {

struct PlanBlock {
  int device;
  size_t bytes;
  void* p;
};

inline std::mutex& plan_pool_mutex() {
  static std::mutex m;
  return m;
}
inline std::vector<PlanBlock>& plan_pool_free() {
  static std::vector<PlanBlock> v;
  return v;
}

// The buffers one build holds; they go back to the pool when it ends (the
// caller drains its stream first).
struct PlanBufs {
  int device = 0;
  std::vector<PlanBlock> held;
  template <typename T>
  cudaError_t get(T*& p, size_t n) {
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    {
      std::lock_guard<std::mutex> g(plan_pool_mutex());
      std::vector<PlanBlock>& fr = plan_pool_free();
      int best = -1;
      for (int i = 0; i < (int)fr.size(); i++)
        if (fr[i].device == device && fr[i].bytes >= bytes && (best < 0 || fr[i].bytes < fr[best].bytes)) best = i;
      if (best >= 0) {
        held.push_back(fr[best]);
        fr.erase(fr.begin() + best);
        p = (T*)held.back().p;
        return cudaSuccess;
      }
    }
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e == cudaSuccess) held.push_back(PlanBlock{device, bytes, q});
    p = (T*)q;
    return e;
  }
  ~PlanBufs() {
    std::lock_guard<std::mutex> g(plan_pool_mutex());
    for (const PlanBlock& b : held) plan_pool_free().push_back(b);
  }
};

}  // namespace fmmg
