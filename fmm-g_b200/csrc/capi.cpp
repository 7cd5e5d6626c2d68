// capi.cpp -- the C ABI of include/fmmg.h over the host plan and the device
// engine.  Every entry point validates its arguments, catches host
// exceptions and reports CUDA failures as status codes.
#include <chrono>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/fmmg.h"
#include "engine.hpp"
#include "kernels.hpp"
#include "plan.hpp"

struct fmmg_handle {
  fmmg::Options opt;
  int device = 0;
  bool hostOnly = false;
  bool setupDone = false;
  bool opsDirty = false;
  bool tablesReplaced = false;  // fmmg_operator replaced a table since the last setup
  bool timing = false;
  int64_t launches = 0;
  int hostPrecision = FMMG_PREC_FP64;
  fmmg::Plan plan;
  fmmg::DevState dev;
  double* dDenIO = nullptr;
  double* dValIO = nullptr;
  double* dDenK = nullptr;  // k-RHS host-call staging
  double* dValK = nullptr;
  int ioK = 0;
  double *dAdjW = nullptr, *dAdjG = nullptr, *dAdjGrad = nullptr, *dAdjDen = nullptr;  // host-call adjoint staging
  int adjK = 0;
  // CUDA-graph replay of fmmg_evaluate_device (one cached (k, precision, buffers) key)
  bool graphOn = false;
  struct GraphKey {
    int k = -1, precision = -1;
    const void* den = nullptr;
    void* val = nullptr;
    bool operator==(const GraphKey& o) const { return k == o.k && precision == o.precision && den == o.den && val == o.val; }
  } graphKey, warmKey;
  cudaGraphExec_t graphExec = nullptr;
  int64_t graphLaunches = 0;
  std::string graphNote;
  std::vector<double> trgHost;  // caller-order targets for check(), read back on its first call
  double setupMs[3] = {0, 0, 0};  // last setup: input checks, plan build, device upload (ms)
  bool treeOnDevice = true;       // device handles build the tree and bin the targets on the GPU
  int callsSinceSetup = 0;        // device calls since the last setup (ready())
  std::string err;
};

static thread_local std::string g_create_err;

static void drop_graph(fmmg_handle* h) {
  if (h->graphExec) cudaGraphExecDestroy(h->graphExec);
  h->graphExec = nullptr;
  h->graphKey = fmmg_handle::GraphKey();
  h->warmKey = fmmg_handle::GraphKey();
}

static fmmg_status fail(fmmg_handle* h, fmmg_status s, const std::string& msg) {
  if (h) h->err = msg;
  else g_create_err = msg;
  return s;
}

// After a synchronised call: FMMG_TIMEOUT if a kernel of the handle gave up a
// bounded device wait (its results are then invalid), else FMMG_OK.
static fmmg_status take_timeout(fmmg_handle* h) {
  int flag = 0;
  std::string e = fmmg::dev_take_error(h->dev, &flag);
  if (!e.empty()) return fail(h, FMMG_CUDA_ERROR, e);
  if (flag) return fail(h, FMMG_TIMEOUT, "a bounded device wait ran out; the results of this call are invalid");
  return FMMG_OK;
}

#define FMMG_GUARD(h)                                                    \
  catch (const std::bad_alloc&) { return fail(h, FMMG_OOM, "host allocation failed"); } \
  catch (const std::exception& ex) { return fail(h, FMMG_INVALID_ARG, ex.what()); }

extern "C" {

fmmg_status fmmg_default_options(fmmg_options* opt) {
  if (!opt) return FMMG_INVALID_ARG;
  std::memset(opt, 0, sizeof(*opt));
  opt->kernel_type = FMMG_KNL_LAP_S_U;
  opt->coefs[0] = 1.0;
  opt->coefs[1] = 0.25;
  opt->np = 6;
  opt->pts_max = 150;
  opt->max_level = 30;
  opt->ctr[0] = opt->ctr[1] = opt->ctr[2] = 0.5;
  opt->root_level = 1;
  opt->device = 0;
  opt->stream = nullptr;
  return FMMG_OK;
}

fmmg_status fmmg_create(const fmmg_options* o, fmmg_handle** out) {
  if (!out) return fail(nullptr, FMMG_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!o) return fail(nullptr, FMMG_INVALID_ARG, "options is NULL");
  if (fmmg::kernel_mm(o->kernel_type) < 0)
    return fail(nullptr, FMMG_NOT_SUPPORTED, "kernel type not supported by setup() (fmm3d_setup_mpi.cpp:113-126)");
  if (o->np < 3 || o->np > 8) return fail(nullptr, FMMG_NOT_SUPPORTED, "np must be in [3, 8]");
  if (o->pts_max < 1) return fail(nullptr, FMMG_INVALID_ARG, "pts_max must be >= 1");
  if (o->max_level < 1 || o->max_level > 30) return fail(nullptr, FMMG_INVALID_ARG, "max_level must be in [1, 30]");
  if (o->root_level < 0 || o->root_level > 30) return fail(nullptr, FMMG_INVALID_ARG, "root_level must be in [0, 30]");
  for (int d = 0; d < 3; d++)
    if (!std::isfinite(o->ctr[d])) return fail(nullptr, FMMG_INVALID_ARG, "ctr is not finite");
  if (!std::isfinite(o->coefs[0]) || !std::isfinite(o->coefs[1]) || o->coefs[0] == 0.0)
    return fail(nullptr, FMMG_INVALID_ARG, "coefs must be finite with mu != 0");
  if ((o->kernel_type == FMMG_KNL_NAV_S_U || o->kernel_type == FMMG_KNL_NAV_D_U) && o->coefs[1] == 1.0)
    return fail(nullptr, FMMG_INVALID_ARG, "Navier kernels need nu != 1");
  fmmg_handle* h = nullptr;
  try {
    h = new fmmg_handle();
    h->opt.kt = o->kernel_type;
    h->opt.coefs[0] = o->coefs[0];
    h->opt.coefs[1] = o->coefs[1];
    h->opt.np = o->np;
    h->opt.ptsMax = o->pts_max;
    h->opt.maxLevel = o->max_level;
    for (int d = 0; d < 3; d++) h->opt.ctr[d] = o->ctr[d];
    h->opt.rootLevel = o->root_level;
    h->device = o->device;
    h->hostOnly = o->device < 0;
    h->plan.o = h->opt;
    if (!h->hostOnly) {
      int ndev = 0;
      cudaError_t ce = cudaGetDeviceCount(&ndev);
      if (ce != cudaSuccess || o->device >= ndev) {
        std::string m = std::string("no such CUDA device: ") + (ce != cudaSuccess ? cudaGetErrorString(ce) : "index");
        delete h;
        return fail(nullptr, FMMG_CUDA_ERROR, m);
      }
    }
    {
      // a device handle builds the operator tables' SVDs on its GPU (the same
      // tables as the host build)
      fmmg::LinalgDeviceScope scope(h->hostOnly ? -1 : o->device);
      std::string e = h->plan.build_operators();
      if (!e.empty()) {
        delete h;
        return fail(nullptr, FMMG_NOT_SUPPORTED, e);
      }
    }
    if (!h->hostOnly) {
      cudaError_t ce = cudaSuccess;
      h->dev.device = o->device;
      ce = cudaSetDevice(o->device);
      if (ce == cudaSuccess) {
        if (o->stream) {
          h->dev.stream = (cudaStream_t)o->stream;
        } else {
          // the highest priority: the side stream of the mixed pass (lowest)
          // then fills the gaps of the main stream's kernels
          int least = 0, greatest = 0;
          cudaDeviceGetStreamPriorityRange(&least, &greatest);
          ce = cudaStreamCreateWithPriority(&h->dev.stream, cudaStreamNonBlocking, greatest);
          h->dev.ownStream = true;
        }
      }
      if (ce != cudaSuccess) {
        std::string m = cudaGetErrorString(ce);
        delete h;
        return fail(nullptr, FMMG_CUDA_ERROR, m);
      }
    }
  } catch (const std::bad_alloc&) {
    delete h;
    return fail(nullptr, FMMG_OOM, "host allocation failed");
  }
  *out = h;
  return FMMG_OK;
}

fmmg_status fmmg_setup(fmmg_handle* h, int64_t ns, const double* src, const double* nrm, int64_t nt,
                       const double* trg) {
  if (!h) return fail(nullptr, FMMG_INVALID_ARG, "handle is NULL");
  if (ns < 1 || !src) return fail(h, FMMG_INVALID_ARG, "need n_src >= 1 and src_xyz");
  if (nt < 0 || (nt > 0 && !trg)) return fail(h, FMMG_INVALID_ARG, "need n_trg >= 0 and trg_xyz");
  if (ns > (int64_t)1 << 31 || nt > (int64_t)1 << 31) return fail(h, FMMG_INVALID_ARG, "too many points");
  using Clock = std::chrono::steady_clock;
  auto t0 = Clock::now();
  auto lap = [&](int i) {
    const auto t1 = Clock::now();
    h->setupMs[i] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    t0 = t1;
  };
  if (fmmg::kernel_has_normal(h->opt.kt) && !nrm)
    return fail(h, FMMG_INVALID_ARG, "double-layer kernel needs src_nrm");
  const double R = std::pow(2.0, -h->opt.rootLevel);
  // branch-free over blocks of points so the compiler vectorises the scan: a
  // NaN fails both comparisons and an infinity the range, so one test per
  // coordinate covers "finite and inside the root box"
  const double lo[3] = {h->opt.ctr[0] - R, h->opt.ctr[1] - R, h->opt.ctr[2] - R};
  const double hi[3] = {h->opt.ctr[0] + R, h->opt.ctr[1] + R, h->opt.ctr[2] + R};
  auto inside = [&](const double* p, int64_t n) {
    constexpr int64_t B = 4096;
    for (int64_t i0 = 0; i0 < n; i0 += B) {
      const int64_t i1 = std::min(n, i0 + B);
      int bad = 0;
      for (int64_t i = i0; i < i1; i++)
        for (int d = 0; d < 3; d++) {
          const double v = p[3 * i + d];
          bad |= !(v >= lo[d] && v <= hi[d]);
        }
      if (bad) return false;
    }
    return true;
  };
  auto finite = [](const double* p, int64_t n) {
    int bad = 0;
    for (int64_t i = 0; i < n; i++) bad |= !(std::fabs(p[i]) <= DBL_MAX);
    return !bad;
  };
  if (!inside(src, ns)) return fail(h, FMMG_INVALID_ARG, "a source lies outside the root box or is not finite");
  if (nt > 0 && trg != src && !inside(trg, nt))
    return fail(h, FMMG_INVALID_ARG, "a target lies outside the root box or is not finite");
  if (nrm && !finite(nrm, 3 * ns)) return fail(h, FMMG_INVALID_ARG, "a normal is not finite");
  try {
    if (h->setupDone) {
      drop_graph(h);
      // the blocks of this setup serve the next one (dev_alloc), and what is
      // left over is freed at its end
      fmmg::dev_release_for_reuse(h->dev);
      h->dDenIO = h->dValIO = nullptr;
      h->dDenK = h->dValK = nullptr;
      h->dAdjW = h->dAdjG = h->dAdjGrad = h->dAdjDen = nullptr;
      h->adjK = 0;
      h->ioK = 0;
      fmmg::Plan fresh;
      fresh.o = h->opt;
      if (h->tablesReplaced) {  // back to the built tables
        fmmg::LinalgDeviceScope scope(h->hostOnly ? -1 : h->device);
        std::string e = fresh.build_operators();
        if (!e.empty()) return fail(h, FMMG_NOT_SUPPORTED, e);
      } else {
        fresh.take_operators(std::move(h->plan));  // the handle's own, never replaced
      }
      h->plan = std::move(fresh);
      h->tablesReplaced = false;
      h->setupDone = false;
    }
    lap(0);
    std::string e = h->plan.build(h->opt, ns, src, nrm, nt, nt > 0 ? trg : src,
                                  !h->hostOnly && h->treeOnDevice ? h->device : -1);
    if (!e.empty()) return fail(h, FMMG_INVALID_ARG, e);
    lap(1);
    h->trgHost.clear();  // check() reads the targets back from the device when it needs them
    if (!h->hostOnly) {
      e = fmmg::dev_upload(h->plan, h->dev, src, nrm, nt > 0 ? trg : src);
      if (!e.empty()) {
        fmmg::dev_free(h->dev);
        return fail(h, e.find("cudaMalloc") != std::string::npos ? FMMG_OOM : FMMG_CUDA_ERROR, e);
      }
      void* p = nullptr;
      if (fmmg::dev_alloc(h->dev, &p, sizeof(double) * (size_t)ns * h->plan.sd) != cudaSuccess)
        return fail(h, FMMG_OOM, "cudaMalloc density buffer");
      h->dDenIO = (double*)p;
      if (fmmg::dev_alloc(h->dev, &p, sizeof(double) * (size_t)std::max<int64_t>(nt, 1) * h->plan.td) != cudaSuccess)
        return fail(h, FMMG_OOM, "cudaMalloc value buffer");
      h->dValIO = (double*)p;
      // the previous setup's blocks that nothing reused wait for the first
      // call's lazily allocated work arrays (the mixed pass, the adjoint) and
      // are freed at the start of the second (ready())
      h->callsSinceSetup = 0;
    }
    lap(2);
    h->opsDirty = false;
    h->setupDone = true;
  }
  FMMG_GUARD(h)
  return FMMG_OK;
}

fmmg_status fmmg_set_tree_device(fmmg_handle* h, int on) {
  if (!h) return fail(nullptr, FMMG_INVALID_ARG, "handle is NULL");
  if (h->hostOnly && on) return fail(h, FMMG_STATE, "host-only handle");
  h->treeOnDevice = on != 0;
  return FMMG_OK;
}

fmmg_status fmmg_setup_times(const fmmg_handle* h, double* ms, int n) {
  if (!h || !ms || n < 9) return FMMG_INVALID_ARG;
  if (!h->setupDone) return FMMG_STATE;
  ms[0] = h->setupMs[0];
  for (int i = 0; i < 6; i++) ms[1 + i] = h->plan.buildMs[i];
  ms[7] = h->setupMs[2];
  ms[8] = h->setupMs[0] + h->setupMs[1] + h->setupMs[2];
  for (int i = 0; i < 4 && 9 + i < n; i++) ms[9 + i] = h->plan.opsMs[i];
  for (int i = 0; i < 4 && 13 + i < n; i++) ms[13 + i] = h->dev.uploadMs[i];
  return FMMG_OK;
}

static fmmg_status ready(fmmg_handle* h) {
  if (!h) return fail(nullptr, FMMG_INVALID_ARG, "handle is NULL");
  if (!h->setupDone) return fail(h, FMMG_STATE, "evaluate before setup");
  if (h->hostOnly) return fail(h, FMMG_STATE, "handle was created host-only (device < 0)");
  if (++h->callsSinceSetup == 2) fmmg::dev_trim(h->dev);
  if (h->opsDirty) {
    std::string e = fmmg::dev_upload_operators(h->plan, h->dev);
    if (!e.empty()) return fail(h, FMMG_CUDA_ERROR, e);
    h->opsDirty = false;
  }
  if (!h->dev.hadPQ) {  // FMMG_HADAMARD=list: the expanded-list M2L reads them
    std::string e = fmmg::dev_upload_vlists(h->plan, h->dev);
    if (!e.empty()) return fail(h, e.find("cudaMalloc") != std::string::npos ? FMMG_OOM : FMMG_CUDA_ERROR, e);
  }
  return FMMG_OK;
}

fmmg_status fmmg_evaluate_stages(fmmg_handle* h, const double* dDen, double* dVal, int precision, int mask) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (!dDen || (!dVal && h->plan.nt > 0)) return fail(h, FMMG_INVALID_ARG, "NULL density or value pointer");
  if (precision != FMMG_PREC_FP64 && precision != FMMG_PREC_MIXED)
    return fail(h, FMMG_INVALID_ARG, "unknown precision");
  try {
    std::string e = fmmg::dev_evaluate(h->plan, h->dev, dDen, dVal, precision, mask & 63, h->timing, nullptr);
    if (!e.empty()) return fail(h, FMMG_CUDA_ERROR, e);
    h->launches = h->dev.lastLaunches;
  }
  FMMG_GUARD(h)
  return FMMG_OK;
}

static fmmg_status evaluate_eager(fmmg_handle* h, int k, const double* dDen, double* dVal, int precision, bool timed) {
  fmmg_status s = FMMG_OK;
  (void)s;
  if (k < 1) return fail(h, FMMG_INVALID_ARG, "k must be >= 1");
  if (!dDen || (!dVal && h->plan.nt > 0)) return fail(h, FMMG_INVALID_ARG, "NULL density or value pointer");
  if (precision != FMMG_PREC_FP64 && precision != FMMG_PREC_MIXED)
    return fail(h, FMMG_INVALID_ARG, "unknown precision");
  try {
    const int64_t sdn = h->plan.ns * h->plan.sd, tdn = h->plan.nt * h->plan.td;
    h->launches = 0;
    if (precision == FMMG_PREC_MIXED) {
      std::string e = fmmg::dev_evaluate_mixed(h->plan, h->dev, dDen, dVal, k, 63, timed, nullptr);
      if (!e.empty()) return fail(h, e.find("cudaMalloc") != std::string::npos ? FMMG_OOM : FMMG_CUDA_ERROR, e);
      h->launches = h->dev.lastLaunches;
      return FMMG_OK;
    }
    for (int r = 0; r < k; r++) {
      std::string e = fmmg::dev_evaluate(h->plan, h->dev, dDen + r * sdn, dVal + r * tdn, precision, 63,
                                         timed, nullptr);
      if (!e.empty()) return fail(h, FMMG_CUDA_ERROR, e);
      h->launches += h->dev.lastLaunches;
    }
  }
  FMMG_GUARD(h)
  return FMMG_OK;
}

fmmg_status fmmg_evaluate_device(fmmg_handle* h, int k, const double* dDen, double* dVal, int precision) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (k < 1) return fail(h, FMMG_INVALID_ARG, "k must be >= 1");
  if (!dDen || (!dVal && h->plan.nt > 0)) return fail(h, FMMG_INVALID_ARG, "NULL density or value pointer");
  if (precision != FMMG_PREC_FP64 && precision != FMMG_PREC_MIXED)
    return fail(h, FMMG_INVALID_ARG, "unknown precision");
  if (!h->graphOn || !h->dev.stream) return evaluate_eager(h, k, dDen, dVal, precision, h->timing);
  fmmg_handle::GraphKey key;
  key.k = k;
  key.precision = precision;
  key.den = dDen;
  key.val = dVal;
  cudaStream_t st = h->dev.stream;
  if (h->graphExec && h->graphKey == key) {  // replay
    cudaError_t ce = cudaGraphLaunch(h->graphExec, st);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    h->launches = h->graphLaunches;
    return FMMG_OK;
  }
  if (!(h->warmKey == key)) {  // first call with these buffers: eager (allocates what it needs)
    s = evaluate_eager(h, k, dDen, dVal, precision, false);
    if (s == FMMG_OK) h->warmKey = key;
    return s;
  }
  // second call: capture the whole evaluate into a graph, then launch it
  if (h->graphExec) cudaGraphExecDestroy(h->graphExec);
  h->graphExec = nullptr;
  cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (ce != cudaSuccess) {
    h->graphNote = std::string("capture not started: ") + cudaGetErrorString(ce);
    return evaluate_eager(h, k, dDen, dVal, precision, false);
  }
  s = evaluate_eager(h, k, dDen, dVal, precision, false);
  cudaGraph_t g = nullptr;
  cudaError_t ce2 = cudaStreamEndCapture(st, &g);
  if (s != FMMG_OK || ce2 != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    h->graphNote = std::string("capture failed: ") + (ce2 != cudaSuccess ? cudaGetErrorString(ce2) : h->err);
    h->graphOn = false;  // stay eager from now on
    return evaluate_eager(h, k, dDen, dVal, precision, false);
  }
  // keep the captured streams' priorities (the side stream yields to the main one)
  ce = cudaGraphInstantiateWithFlags(&h->graphExec, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    h->graphExec = nullptr;
    h->graphNote = std::string("instantiate failed: ") + cudaGetErrorString(ce);
    h->graphOn = false;
    return evaluate_eager(h, k, dDen, dVal, precision, false);
  }
  h->graphKey = key;
  h->graphLaunches = h->launches;
  ce = cudaGraphLaunch(h->graphExec, st);
  if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
  return FMMG_OK;
}

fmmg_status fmmg_set_graph(fmmg_handle* h, int on) {
  if (!h) return fail(nullptr, FMMG_INVALID_ARG, "handle is NULL");
  if (h->hostOnly) return fail(h, FMMG_STATE, "host-only handle");
  drop_graph(h);
  h->graphOn = on != 0;
  h->graphNote.clear();
  return FMMG_OK;
}

fmmg_status fmmg_set_gemm_path(fmmg_handle* h, int path) {
  if (!h) return fail(nullptr, FMMG_INVALID_ARG, "handle is NULL");
  if (path < 0 || path > 2) return fail(h, FMMG_INVALID_ARG, "gemm path must be 0, 1 or 2");
  h->dev.gemmPath = path;
  drop_graph(h);
  return FMMG_OK;
}

fmmg_status fmmg_selftest_wait(int device, int arrive, int64_t limit_ns) {
  if (device < 0 || limit_ns < 0 || limit_ns > 2000000000ll) return FMMG_INVALID_ARG;
  int flag = 0;
  std::string e = fmmg::dev_wait_selftest(device, arrive, (long long)limit_ns, &flag);
  if (!e.empty()) return fail(nullptr, FMMG_CUDA_ERROR, e);
  return flag ? FMMG_TIMEOUT : FMMG_OK;
}

fmmg_status fmmg_device_error(fmmg_handle* h, int* flag) {
  if (!h || !flag) return fail(h, FMMG_INVALID_ARG, "NULL argument");
  *flag = 0;
  if (h->hostOnly || !h->setupDone) return FMMG_OK;
  std::string e = fmmg::dev_take_error(h->dev, flag);
  if (!e.empty()) return fail(h, FMMG_CUDA_ERROR, e);
  return FMMG_OK;
}

// Autotuner: times real evaluates of (k, precision) on the caller's buffers
// with CUDA events for each candidate launch shape and keeps the fastest.
// Coordinate search: Hadamard rows per CTA first, then the split-K threshold
// of the FP32 GEMMs (mixed form) -- 8 candidates, reps evaluates each.
fmmg_status fmmg_autotune(fmmg_handle* h, int k, int precision, const double* dDen, double* dVal, int reps,
                          double* bestMs) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (k < 1 || reps < 1 || !dDen || (!dVal && h->plan.nt > 0)) return fail(h, FMMG_INVALID_ARG, "bad autotune arguments");
  if (precision != FMMG_PREC_FP64 && precision != FMMG_PREC_MIXED) return fail(h, FMMG_INVALID_ARG, "precision");
  try {
    cudaStream_t st = h->dev.stream;
    const bool wasGraph = h->graphOn;
    h->graphOn = false;
    drop_graph(h);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timeIt = [&](float& ms) -> fmmg_status {
      fmmg_status r = evaluate_eager(h, k, dDen, dVal, precision, false);  // warm (allocations, caches)
      if (r != FMMG_OK) return r;
      cudaEventRecord(e0, st);
      for (int i = 0; i < reps; i++) {
        r = evaluate_eager(h, k, dDen, dVal, precision, false);
        if (r != FMMG_OK) return r;
      }
      cudaEventRecord(e1, st);
      cudaError_t ce = cudaEventSynchronize(e1);
      if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= reps;
      return FMMG_OK;
    };
    fmmg::DevState::Tune& T = h->dev.tune;
    float best = 1e30f, ms = 0.f;
    const bool mixed = precision == FMMG_PREC_MIXED;
    int* rowsKnob = mixed ? &T.hadRows : &T.pqParents;
    if (mixed && k >= 2) {  // the Hadamard's form: 27-product accumulators (1, 2) or output-child ones (3, 4)
      int bestForm = T.hadRhsPerThread;
      for (int c : {4, 3, 2, 1}) {
        T.hadRhsPerThread = c;
        if ((s = timeIt(ms)) != FMMG_OK) break;
        if (ms < best) {
          best = ms;
          bestForm = c;
        }
      }
      T.hadRhsPerThread = bestForm;
      best = 1e30f;
    }
    const int rowsCand[4] = {32, 64, 128, 256};
    int bestRows = *rowsKnob;
    for (int c : rowsCand) {
      if (s != FMMG_OK) break;
      *rowsKnob = c;
      if ((s = timeIt(ms)) != FMMG_OK) break;
      if (ms < best) {
        best = ms;
        bestRows = c;
      }
    }
    *rowsKnob = bestRows;
    if (s == FMMG_OK && mixed) {
      const int splitCand[4] = {0, 1, 2, 4};
      int bestSplit = T.gemmSplitMul;
      best = 1e30f;
      for (int c : splitCand) {
        T.gemmSplitMul = c;
        if ((s = timeIt(ms)) != FMMG_OK) break;
        if (ms < best) {
          best = ms;
          bestSplit = c;
        }
      }
      T.gemmSplitMul = bestSplit;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->graphOn = wasGraph;
    if (s != FMMG_OK) return s;
    if (bestMs) *bestMs = best;
  }
  FMMG_GUARD(h)
  return FMMG_OK;
}

fmmg_status fmmg_tuning(fmmg_handle* h, int* vals, int n, int set) {
  if (!h || !vals || n < 3) return fail(h, FMMG_INVALID_ARG, "need 3 values");
  fmmg::DevState::Tune& T = h->dev.tune;
  if (set) {
    if (vals[0] < 1 || vals[1] < 1 || vals[2] < 0 || (n >= 4 && (vals[3] < 1 || vals[3] > 4)) ||
        (n >= 5 && (vals[4] < 0 || vals[4] > 63)) || (n >= 6 && vals[5] != 3 && vals[5] != 4))
      return fail(h, FMMG_INVALID_ARG, "tuning values");
    T.hadRows = vals[0];
    T.pqParents = vals[1];
    T.gemmSplitMul = vals[2];
    if (n >= 4) T.hadRhsPerThread = vals[3];
    if (n >= 5) T.tcMask = vals[4];
    if (n >= 6) T.tcProducts = vals[5];
    drop_graph(h);
  } else {
    vals[0] = T.hadRows;
    vals[1] = T.pqParents;
    vals[2] = T.gemmSplitMul;
    if (n >= 4) vals[3] = T.hadRhsPerThread;
    if (n >= 5) vals[4] = T.tcMask;
    if (n >= 6) vals[5] = T.tcProducts;
  }
  return FMMG_OK;
}

fmmg_status fmmg_graph_state(const fmmg_handle* h, int* active, const char** note) {
  if (!h) return FMMG_INVALID_ARG;
  if (active) *active = h->graphExec ? 1 : 0;
  if (note) *note = h->graphNote.c_str();
  return FMMG_OK;
}

fmmg_status fmmg_adjoint_device(fmmg_handle* h, int k, const double* dDen, const double* dW, double* dG,
                                double* dGradT) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (k < 1) return fail(h, FMMG_INVALID_ARG, "k must be >= 1");
  if ((!dW && h->plan.nt > 0) || (dGradT && !dDen)) return fail(h, FMMG_INVALID_ARG, "NULL weight or density pointer");
  if (dGradT && h->opt.kt != 111 && h->opt.kt != 121)
    return fail(h, FMMG_NOT_SUPPORTED, "target-position gradient: Laplace kernels 111 and 121 only");
  try {
    const int64_t sdn = h->plan.ns * h->plan.sd, tdn = h->plan.nt * h->plan.td, gtn = 3 * h->plan.nt;
    h->launches = 0;
    for (int r = 0; r < k; r++) {
      std::string e = fmmg::dev_adjoint(h->plan, h->dev, dDen ? dDen + r * sdn : nullptr, dW ? dW + r * tdn : nullptr,
                                        dG ? dG + r * sdn : nullptr, dGradT ? dGradT + r * gtn : nullptr, h->timing);
      if (!e.empty()) return fail(h, e.find("cudaMalloc") != std::string::npos ? FMMG_OOM : FMMG_CUDA_ERROR, e);
      h->launches += h->dev.lastLaunches;
    }
  }
  FMMG_GUARD(h)
  return FMMG_OK;
}

fmmg_status fmmg_adjoint_host(fmmg_handle* h, int k, const double* den, const double* w, double* g, double* gradT) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (k < 1) return fail(h, FMMG_INVALID_ARG, "k must be >= 1");
  if ((!w && h->plan.nt > 0) || (gradT && !den)) return fail(h, FMMG_INVALID_ARG, "NULL weight or density pointer");
  try {
    const size_t bs = sizeof(double) * (size_t)h->plan.ns * h->plan.sd;
    const size_t bt = sizeof(double) * (size_t)h->plan.nt * h->plan.td;
    const size_t bg = sizeof(double) * 3 * (size_t)h->plan.nt;
    if (k > h->adjK) {
      auto get = [&](double*& p, size_t n) {
        void* q = nullptr;
        if (fmmg::dev_alloc(h->dev, &q, std::max<size_t>(n, 8)) != cudaSuccess) return false;
        p = (double*)q;
        return true;
      };
      if (!get(h->dAdjW, bt * k) || !get(h->dAdjG, bs * k) || !get(h->dAdjGrad, bg * k) || !get(h->dAdjDen, bs * k))
        return fail(h, FMMG_OOM, "cudaMalloc adjoint buffers");
      h->adjK = k;
    }
    cudaStream_t st = h->dev.stream;
    cudaError_t ce = cudaSuccess;
    if (bt) ce = cudaMemcpyAsync(h->dAdjW, w, bt * k, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && gradT) ce = cudaMemcpyAsync(h->dAdjDen, den, bs * k, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    s = fmmg_adjoint_device(h, k, gradT ? h->dAdjDen : nullptr, h->dAdjW, g ? h->dAdjG : nullptr,
                            gradT ? h->dAdjGrad : nullptr);
    if (s != FMMG_OK) return s;
    if (g) ce = cudaMemcpyAsync(g, h->dAdjG, bs * k, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess && gradT && bg) ce = cudaMemcpyAsync(gradT, h->dAdjGrad, bg * k, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    return take_timeout(h);
  }
  FMMG_GUARD(h)
}

fmmg_status fmmg_synchronize(fmmg_handle* h) {
  if (!h) return fail(nullptr, FMMG_INVALID_ARG, "handle is NULL");
  if (h->hostOnly || !h->dev.stream) return FMMG_OK;
  cudaError_t ce = cudaStreamSynchronize(h->dev.stream);
  if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
  return FMMG_OK;
}

fmmg_status fmmg_evaluate(fmmg_handle* h, const double* den, double* val) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (!den || (!val && h->plan.nt > 0)) return fail(h, FMMG_INVALID_ARG, "NULL density or value pointer");
  try {
    cudaStream_t st = h->dev.stream;
    const size_t bi = sizeof(double) * (size_t)h->plan.ns * h->plan.sd;
    const size_t bo = sizeof(double) * (size_t)h->plan.nt * h->plan.td;
    cudaError_t ce = cudaMemcpyAsync(h->dDenIO, den, bi, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    std::string e = fmmg::dev_evaluate(h->plan, h->dev, h->dDenIO, h->dValIO, h->hostPrecision, 63, true, nullptr);
    if (!e.empty()) return fail(h, FMMG_CUDA_ERROR, e);
    h->launches = h->dev.lastLaunches;
    if (bo) {
      ce = cudaMemcpyAsync(val, h->dValIO, bo, cudaMemcpyDeviceToHost, st);
      if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    }
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    return take_timeout(h);
  }
  FMMG_GUARD(h)
}

fmmg_status fmmg_evaluate_host(fmmg_handle* h, int k, const double* den, double* val, int precision) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (k < 1 || !den || (!val && h->plan.nt > 0)) return fail(h, FMMG_INVALID_ARG, "bad k or NULL pointer");
  try {
    const size_t bi = sizeof(double) * (size_t)h->plan.ns * h->plan.sd;
    const size_t bo = sizeof(double) * (size_t)h->plan.nt * h->plan.td;
    if (k > h->ioK) {
      void* p = nullptr;
      if (fmmg::dev_alloc(h->dev, &p, bi * k) != cudaSuccess) return fail(h, FMMG_OOM, "cudaMalloc density buffers");
      h->dDenK = (double*)p;
      if (fmmg::dev_alloc(h->dev, &p, std::max<size_t>(bo, 8) * k) != cudaSuccess)
        return fail(h, FMMG_OOM, "cudaMalloc values");
      h->dValK = (double*)p;
      h->ioK = k;
    }
    cudaStream_t st = h->dev.stream;
    cudaError_t ce = cudaMemcpyAsync(h->dDenK, den, bi * k, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    s = fmmg_evaluate_device(h, k, h->dDenK, h->dValK, precision);
    if (s != FMMG_OK) return s;
    if (bo) {
      ce = cudaMemcpyAsync(val, h->dValK, bo * k, cudaMemcpyDeviceToHost, st);
      if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    }
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    return take_timeout(h);
  }
  FMMG_GUARD(h)
}

fmmg_status fmmg_check(fmmg_handle* h, const double* den, const double* val, int64_t nchk, const int64_t* idx,
                       double* rel, double* maxabs, double* denseOut) {
  fmmg_status s = ready(h);
  if (s != FMMG_OK) return s;
  if (!den || !val || !idx || nchk < 1) return fail(h, FMMG_INVALID_ARG, "bad check arguments");
  try {
    const int td = h->plan.td;
    const int64_t nt = h->plan.nt;
    if ((int64_t)h->trgHost.size() != 3 * nt) {  // the caller-order targets, once per setup
      std::vector<double> tree(3 * (size_t)nt);
      cudaError_t ce = cudaMemcpy(tree.data(), h->dev.trg, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost);
      if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
      h->trgHost.resize(3 * (size_t)nt);
      const std::vector<int64_t>& perm = h->plan.trgPerm;
      for (int64_t q = 0; q < nt; q++)
        for (int d = 0; d < 3; d++) h->trgHost[3 * perm[q] + d] = tree[3 * q + d];
    }
    std::vector<double> pos(3 * (size_t)nchk), dense((size_t)nchk * td);
    for (int64_t i = 0; i < nchk; i++) {
      if (idx[i] < 0 || idx[i] >= h->plan.nt) return fail(h, FMMG_INVALID_ARG, "check index out of range");
      for (int d = 0; d < 3; d++) pos[3 * i + d] = h->trgHost[3 * idx[i] + d];
    }
    cudaError_t ce = cudaMemcpyAsync(h->dDenIO, den, sizeof(double) * h->plan.ns * h->plan.sd,
                                     cudaMemcpyHostToDevice, h->dev.stream);
    if (ce != cudaSuccess) return fail(h, FMMG_CUDA_ERROR, cudaGetErrorString(ce));
    std::string e = fmmg::dev_dense(h->plan, h->dev, h->dDenIO, nchk, pos.data(), dense.data());
    if (!e.empty()) return fail(h, FMMG_CUDA_ERROR, e);
    double en = 0, dn = 0, mx = 0;
    for (int64_t i = 0; i < nchk; i++)
      for (int c = 0; c < td; c++) {
        double a = val[idx[i] * td + c], b = dense[i * td + c];
        en += (a - b) * (a - b);
        dn += b * b;
        mx = std::max(mx, std::fabs(a - b));
      }
    if (rel) *rel = dn > 0 ? std::sqrt(en / dn) : std::sqrt(en);
    if (maxabs) *maxabs = mx;
    if (denseOut) std::copy(dense.begin(), dense.end(), denseOut);
  }
  FMMG_GUARD(h)
  return FMMG_OK;
}

fmmg_status fmmg_info(const fmmg_handle* h, int* sd, int* td, int64_t* nn, int64_t* nl, int* md) {
  if (!h) return FMMG_INVALID_ARG;
  if (sd) *sd = fmmg::kernel_src_dof(h->opt.kt);
  if (td) *td = fmmg::kernel_trg_dof(h->opt.kt);
  if (nn) *nn = h->setupDone ? h->plan.nn : 0;
  if (nl) {
    int64_t c = 0;
    if (h->setupDone)
      for (int n = 0; n < h->plan.nn; n++) c += h->plan.chd[n] < 0;
    *nl = c;
  }
  if (md) *md = h->setupDone ? h->plan.maxDepth : 0;
  return FMMG_OK;
}

fmmg_status fmmg_stage_times(const fmmg_handle* h, double* ms, int n) {
  if (!h || !ms || n < 7) return FMMG_INVALID_ARG;
  for (int i = 0; i < 7; i++) ms[i] = h->dev.stageMs[i];
  return FMMG_OK;
}

fmmg_status fmmg_kernel_times(const fmmg_handle* h, double* ms, int n) {
  if (!h || !ms || n < fmmg::EV_COUNT - 1) return FMMG_INVALID_ARG;
  for (int i = 0; i < fmmg::EV_COUNT - 1; i++) ms[i] = h->dev.kernMs[i];
  return FMMG_OK;
}

fmmg_status fmmg_plan_stats(const fmmg_handle* h, int64_t* st, int n) {
  if (!h || !st || n < 16) return FMMG_INVALID_ARG;
  if (!h->setupDone) return FMMG_STATE;
  const fmmg::Plan& P = h->plan;
  const int64_t ue = (int64_t)P.nUE * P.sdm, uc = (int64_t)P.nUC * P.tdm;
  const int64_t de = (int64_t)P.nDE * P.sdm, dc = (int64_t)P.nDC * P.tdm;
  int64_t nearPairs = 0, s2mPairs = 0, s2lPairs = 0, m2tPairs = 0, l2tPairs = 0, upFlops = 0, dnFlops = 0;
  for (size_t r = 0; r < P.evtrLeaves.size(); r++) {
    int g = P.evtrLeaves[r];
    int64_t s = 0;
    for (int64_t e = P.nearSrc.ptr[r]; e < P.nearSrc.ptr[r + 1]; e++) s += P.srcCnt[P.nearSrc.idx[e]];
    nearPairs += P.trgCnt[g] * s;
    if (P.depth[g] >= 2) l2tPairs += P.trgCnt[g] * P.nDE;
  }
  for (size_t r = 0; r < P.farLeaves.size(); r++)
    m2tPairs += P.trgCnt[P.farLeaves[r]] * (P.farUE.ptr[r + 1] - P.farUE.ptr[r]) * P.nUE;
  for (int g : P.s2mLeaves) s2mPairs += P.srcCnt[g] * P.nUC;
  for (size_t r = 0; r < P.s2lNodes.size(); r++)
    for (int64_t e = P.s2lSrc.ptr[r]; e < P.s2lSrc.ptr[r + 1]; e++) s2lPairs += P.srcCnt[P.s2lSrc.idx[e]] * P.nDC;
  for (int d = 0; d <= P.maxDepth; d++) {
    upFlops += (int64_t)P.upM2M[d].size() * 2 * uc * 8 * ue + (int64_t)P.upC2E[d].size() * 2 * ue * uc;
    if (d >= 3) dnFlops += (int64_t)P.dnL2L[d - 1].size() * 2 * 8 * dc * de;
    dnFlops += (int64_t)P.dnC2E[d].size() * 2 * de * dc;
  }
  // the FP32 pass: parents take the folded C2E x M2M product, leaves and the
  // downward pass the factored pseudo-inverses (ranks padded to 4)
  const int64_t kUp4 = (P.kUp + 3) & ~3, kDn4 = (P.kDn + 3) & ~3;
  int64_t upFlops32 = 0, dnFlops32 = 0;
  for (int d = 0; d <= P.maxDepth; d++) {
    upFlops32 += (int64_t)P.upM2M[d].size() * 2 * ue * 8 * ue + (int64_t)P.upLeaf[d].size() * 2 * kUp4 * (uc + ue);
    if (d >= 3) dnFlops32 += (int64_t)P.dnL2L[d - 1].size() * 2 * 8 * dc * de;
    dnFlops32 += (int64_t)P.dnC2E[d].size() * 2 * kDn4 * (dc + de);
  }
  int64_t v[19] = {nearPairs, s2mPairs, s2lPairs, m2tPairs, l2tPairs,
                   (int64_t)P.vSrcNodes.size(), (int64_t)P.vTrgNodes.size(), (int64_t)P.vParents.size(),
                   (int64_t)P.vNbr.idx.size(), (int64_t)P.V.idx.size(), upFlops, dnFlops,
                   (int64_t)P.nEff, (int64_t)P.sdm, (int64_t)P.tdm, (int64_t)P.nn,
                   (int64_t)P.nEff32, upFlops32, dnFlops32};
  std::copy(v, v + std::min(n, 19), st);
  return FMMG_OK;
}

fmmg_status fmmg_launch_count(const fmmg_handle* h, int64_t* n) {
  if (!h || !n) return FMMG_INVALID_ARG;
  *n = h->launches;
  return FMMG_OK;
}

fmmg_status fmmg_set_precision(fmmg_handle* h, int precision) {
  if (!h) return fail(nullptr, FMMG_INVALID_ARG, "handle is NULL");
  if (precision != FMMG_PREC_FP64 && precision != FMMG_PREC_MIXED) return fail(h, FMMG_INVALID_ARG, "precision");
  h->hostPrecision = precision;
  return FMMG_OK;
}

fmmg_status fmmg_set_timing(fmmg_handle* h, int on) {
  if (!h) return FMMG_INVALID_ARG;
  h->timing = on != 0;
  return FMMG_OK;
}

fmmg_status fmmg_tree(const fmmg_handle* h, int32_t* rec, int64_t* ps, int64_t* pt) {
  if (!h) return FMMG_INVALID_ARG;
  if (!h->setupDone) return FMMG_STATE;
  const fmmg::Plan& P = h->plan;
  if (rec)
    for (int n = 0; n < P.nn; n++) {
      int32_t* r = rec + 9 * (size_t)n;
      r[0] = P.depth[n];
      r[1] = P.path[3 * (size_t)n];
      r[2] = P.path[3 * (size_t)n + 1];
      r[3] = P.path[3 * (size_t)n + 2];
      r[4] = P.par[n];
      r[5] = P.chd[n];
      uint8_t f = P.flags[n];
      r[6] = ((f & fmmg::NF_CBTR) ? 1 : 0) | ((f & fmmg::NF_USER) ? 2 : 0) | ((f & fmmg::NF_EVTR) ? 4 : 0) |
             ((f & fmmg::NF_SRCE) ? 24 : 0);
      r[7] = (int32_t)P.srcCnt[n];
      r[8] = (int32_t)P.trgCnt[n];
    }
  if (ps) std::copy(P.srcPerm.begin(), P.srcPerm.end(), ps);
  if (pt) std::copy(P.trgPerm.begin(), P.trgPerm.end(), pt);
  return FMMG_OK;
}

fmmg_status fmmg_lists(const fmmg_handle* h, int which, int64_t* ptr, int32_t* idx, int64_t* total) {
  if (!h || which < 0 || which > 3) return FMMG_INVALID_ARG;
  if (!h->setupDone) return FMMG_STATE;
  const fmmg::CSR& L = which == 0 ? h->plan.U : which == 1 ? h->plan.V : which == 2 ? h->plan.W : h->plan.X;
  if (ptr) std::copy(L.ptr.begin(), L.ptr.end(), ptr);
  if (idx) std::copy(L.idx.begin(), L.idx.end(), idx);
  if (total) *total = (int64_t)L.idx.size();
  return FMMG_OK;
}

fmmg_status fmmg_worklist(const fmmg_handle* h, int which, int32_t* rows, int64_t* ptr, int32_t* idx,
                          int64_t* n_rows, int64_t* total) {
  if (!h || which < 0 || which > 7) return FMMG_INVALID_ARG;
  if (!h->setupDone) return FMMG_STATE;
  const fmmg::Plan& P = h->plan;
  if (which >= 6) {  // expanded V lists: (slot, translation id) pairs per slot
    P.expand_v_lists();
    const std::vector<int32_t>& R = which == 6 ? P.vTrgNodes : P.vSrcNodes;
    const std::vector<int64_t>& Lp = which == 6 ? P.vTrgPtr : P.vSrcPtr;
    const std::vector<int32_t>& Le = which == 6 ? P.vTrgEnt : P.vSrcEnt;
    if (rows) std::copy(R.begin(), R.end(), rows);
    if (n_rows) *n_rows = (int64_t)R.size();
    if (ptr) std::copy(Lp.begin(), Lp.end(), ptr);
    if (idx) std::copy(Le.begin(), Le.end(), idx);
    if (total) *total = (int64_t)Le.size();
    return FMMG_OK;
  }
  static const fmmg::CSR none;
  const std::vector<int32_t>* R = nullptr;
  const fmmg::CSR* L = &none;
  switch (which) {
    case 0: R = &P.evtrLeaves; L = &P.nearSrc; break;
    case 1: R = &P.farLeaves; L = &P.farUE; break;
    case 2: R = &P.s2lNodes; L = &P.s2lSrc; break;
    case 3: R = &P.vParents; L = &P.vNbr; break;
    case 4: R = &P.s2mLeaves; break;
    default: R = &P.l2tLeaves; break;
  }
  if (rows) std::copy(R->begin(), R->end(), rows);
  if (n_rows) *n_rows = (int64_t)R->size();
  const bool csr = which <= 3;
  if (ptr && csr) std::copy(L->ptr.begin(), L->ptr.end(), ptr);
  if (idx && csr) std::copy(L->idx.begin(), L->idx.end(), idx);
  if (total) *total = csr ? (int64_t)L->idx.size() : 0;
  return FMMG_OK;
}

fmmg_status fmmg_operator(fmmg_handle* h, int which, int idx, double* get, const double* set, int64_t* count) {
  if (!h) return FMMG_INVALID_ARG;
  if (set) drop_graph(h);  // a captured graph holds the FP32 operator copies of the old tables
  fmmg::Plan& P = h->plan;
  const int64_t ue = (int64_t)P.nUE * P.sdm, uc = (int64_t)P.nUC * P.tdm;
  const int64_t de = (int64_t)P.nDE * P.sdm, dc = (int64_t)P.nDC * P.tdm;
  int64_t n = 0;
  switch (which) {
    case 0:  // reference (ue x uc) column-major
      n = ue * uc;
      for (int64_t i = 0; i < ue; i++)
        for (int64_t j = 0; j < uc; j++) {
          if (get) get[j * ue + i] = P.uc2ue[i * uc + j];
          if (set) P.uc2ue[i * uc + j] = set[j * ue + i];
        }
      break;
    case 1:  // octant idx: (uc x ue)
      if (idx < 0 || idx > 7) return fail(h, FMMG_INVALID_ARG, "octant index");
      n = uc * ue;
      for (int64_t r = 0; r < uc; r++)
        for (int64_t c = 0; c < ue; c++) {
          if (get) get[c * uc + r] = P.m2m[r * 8 * ue + idx * ue + c];
          if (set) P.m2m[r * 8 * ue + idx * ue + c] = set[c * uc + r];
        }
      break;
    case 2:
      n = de * dc;
      for (int64_t i = 0; i < de; i++)
        for (int64_t j = 0; j < dc; j++) {
          if (get) get[j * de + i] = P.dc2de[i * dc + j];
          if (set) P.dc2de[i * dc + j] = set[j * de + i];
        }
      break;
    case 3:
      if (idx < 0 || idx > 7) return fail(h, FMMG_INVALID_ARG, "octant index");
      n = dc * de;
      for (int64_t r = 0; r < dc; r++)
        for (int64_t c = 0; c < de; c++) {
          if (get) get[c * dc + r] = P.l2l[((int64_t)idx * dc + r) * de + c];
          if (set) P.l2l[((int64_t)idx * dc + r) * de + c] = set[c * dc + r];
        }
      break;
    case 4: {
      if (idx < 0 || idx > 315) return fail(h, FMMG_INVALID_ARG, "translation index");
      const int64_t m = (int64_t)P.nEff * P.sdm * P.tdm;
      n = 2 * m;
      double* base = (double*)(P.m2lT.data() + (size_t)idx * m);
      if (get) std::memcpy(get, base, sizeof(double) * n);
      if (set) std::memcpy(base, set, sizeof(double) * n);
    } break;
    case 5: {  // the mixed form's translation spectra on the (2np-1)^3 grid, read only
      if (idx < 0 || idx > 315) return fail(h, FMMG_INVALID_ARG, "translation index");
      if (set) return fail(h, FMMG_INVALID_ARG, "operator 5 is read only (set operator 4)");
      const int64_t m = (int64_t)P.nEff32 * P.sdm * P.tdm;
      n = 2 * m;
      if (get) std::memcpy(get, (const double*)(P.m2lT32.data() + (size_t)idx * m), sizeof(double) * n);
    } break;
    case 6: {  // the mixed form's folded C2E up x M2M, (ue x 8 ue) column-major, read only
      if (set) return fail(h, FMMG_INVALID_ARG, "operator 6 is read only (set operators 0 and 1)");
      n = ue * 8 * ue;
      if (get) {
        try {
          const std::vector<double>& f = P.folded_upward();  // row-major [ue][8 ue]
          for (int64_t i = 0; i < ue; i++)
            for (int64_t j = 0; j < 8 * ue; j++) get[j * ue + i] = f[i * 8 * ue + j];
        }
        FMMG_GUARD(h)
      }
    } break;
    default:
      return fail(h, FMMG_INVALID_ARG, "operator id");
  }
  if (count) *count = n;
  if (set) {
    h->opsDirty = true;
    h->tablesReplaced = true;
    if (which == 0 || which == 1) P.drop_folded_upward();
    try {
      if (which == 0 || which == 2) P.refactor_c2e(which);  // the FP32 pass applies the pinv factored
      if (which == 4) P.m2l_spectrum32(idx);                 // and transforms on the (2np-1)^3 grid
    }
    FMMG_GUARD(h)
  }
  return FMMG_OK;
}

const char* fmmg_last_error(const fmmg_handle* h) {
  return h ? h->err.c_str() : g_create_err.c_str();
}

fmmg_status fmmg_destroy(fmmg_handle* h) {
  if (!h) return FMMG_OK;
  if (!h->hostOnly) {
    cudaSetDevice(h->dev.device);
    if (h->dev.stream) cudaStreamSynchronize(h->dev.stream);
    drop_graph(h);
    fmmg::dev_free(h->dev);
    if (h->dev.ownStream && h->dev.stream) cudaStreamDestroy(h->dev.stream);
  }
  delete h;
  return FMMG_OK;
}

}  // extern "C"
