// engine.hpp -- device-resident state of one evaluator handle and the stage
// launcher.  All kernels live in stages.cu; the C ABI is capi.cpp.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "plan.hpp"
#include "tc_op.hpp"

namespace fmmg {

// timing marks recorded on the handle's stream around each kernel class;
// interval k runs from mark k to mark k+1
enum {
  EV_BEGIN = 0, EV_PREP, EV_S2M, EV_UP_GEMM, EV_NEAR, EV_M2L_FWD, EV_M2L_HAD, EV_M2L_INV, EV_M2T, EV_S2L,
  EV_DN_GEMM, EV_L2T, EV_END, EV_COUNT
};

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
};

struct DevState {
  int device = 0;
  cudaStream_t stream = nullptr;
  // second stream of an untimed pass: the near field and the W list run on it
  // beside the upward pass and the V list (they only add into the target
  // values); evFork/evUp/evSide order it against the main stream
  cudaStream_t side = nullptr;
  cudaEvent_t evFork = nullptr, evUp = nullptr, evSide = nullptr;
  bool ownStream = false;
  // geometry (permuted order)
  double *src = nullptr, *nrm = nullptr, *trg = nullptr;
  int64_t *srcPerm = nullptr, *trgPerm = nullptr;
  double *ctr = nullptr, *rad = nullptr;
  int64_t *srcBeg = nullptr, *srcCnt = nullptr, *trgBeg = nullptr, *trgCnt = nullptr;
  int32_t *chd = nullptr, *depth = nullptr;
  double* sam[4] = {nullptr, nullptr, nullptr, nullptr};
  int32_t* surfIJK = nullptr;  // np-surface point -> packed (i, j, k)
  // work lists
  int32_t *evtrLeaves = nullptr;
  int64_t *nearPtr = nullptr; int32_t *nearIdx = nullptr;     // merged near list
  int64_t *nearUPtr = nullptr; int32_t *nearUIdx = nullptr;   // stage-split forms
  int64_t *nearWPtr = nullptr; int32_t *nearWIdx = nullptr;
  int64_t *nearXPtr = nullptr; int32_t *nearXIdx = nullptr;
  int32_t *farLeaves = nullptr; int64_t *farPtr = nullptr; int32_t *farIdx = nullptr;
  // FP32 M2T work items (rows with long W lists split in chunks of far
  // entries), the split rows, and their partial sums
  int4* m2tItems = nullptr; int nM2tItems = 0;
  int32_t* nearOrder = nullptr;  // FP32 near-field rows by decreasing pair count
  int32_t *m2tSplitLeaf = nullptr, *m2tSplitBase = nullptr, *m2tSplitCnt = nullptr; int nM2tSplit = 0;
  int64_t m2tPartTargets = 0;  // partial-sum rows per right-hand side
  double* m2tPart = nullptr;
  int32_t *l2tLeaves = nullptr;
  int32_t *s2lNodes = nullptr; int64_t *s2lPtr = nullptr; int32_t *s2lIdx = nullptr;
  int32_t *s2mLeaves = nullptr;
  int32_t *levelRows = nullptr;  // concatenated per-level row lists
  std::vector<int64_t> offUpC2E, offUpM2M, offDnL2L, offDnC2E, offUpLeaf;  // host offsets into levelRows, size maxDepth+2
  int32_t *vParents = nullptr; int64_t *vPtr = nullptr; int32_t *vIdx = nullptr; int8_t *vOff = nullptr;
  int32_t *vSrcSlot = nullptr, *vTrgSlot = nullptr, *vSrcNodes = nullptr, *vTrgNodes = nullptr;
  int64_t *vTrgPtr = nullptr, *vSrcPtr = nullptr;   // expanded V-lists per target / source slot
  int32_t *vTrgEnt = nullptr, *vSrcEnt = nullptr;   // (slot, translation id) pairs
  // operators
  double *uc2ue = nullptr, *m2m = nullptr, *dc2de = nullptr, *l2l = nullptr;
  double2* m2lT = nullptr;
  int16_t* transIdDev = nullptr;  // (rx+3)*49+(ry+3)*7+(rz+3) -> translation 0..315 or -1
  // per-evaluate work arrays
  double *den = nullptr, *val = nullptr, *uchk = nullptr, *uden = nullptr, *dchk = nullptr, *dden = nullptr;
  double2 *effDen = nullptr, *effVal = nullptr;
  // mixed-precision work arrays and FP32 operator copies (allocated on first use)
  float *uchk32 = nullptr, *uden32 = nullptr, *dchk32 = nullptr, *dden32 = nullptr;
  float2 *effDen32 = nullptr, *effVal32 = nullptr;
  float* l2l32 = nullptr;
  float *upF1 = nullptr, *upF2 = nullptr, *dnF1 = nullptr, *dnF2 = nullptr;  // factored pinvs
  float *upT32 = nullptr, *dnT32 = nullptr;  // [k][nn][kUp|kDn] intermediate of the factored C2E
  float2* m2lT32 = nullptr;
  float2* m2lTw32 = nullptr;  // combined translations of the 27-product Hadamard [27][27][nEff] (scalar kernels)
  bool hadW = true;           // FP32 k >= 2 Hadamard in the 27-product form
  double *denK = nullptr, *valK = nullptr;  // permuted densities / values of a RHS chunk
  float* den32 = nullptr;  // the chunk's densities in FP32, [rhs / 8][n][8][sd] (what the pair kernels stage)
  bool mixedReady = false, mixedOpsStale = true;
  int mixedK = 0;                           // right-hand sides the mixed arrays hold
  int mixedPassFor = 0, mixedPassK = 0;     // the last k that needed several passes, and its pass size
  double mixedBudgetBytes = 120e9;          // device bytes for per-density work arrays (at most)
  // transposed FMM: inverted work lists, transposed operator tables, target-gradient buffer
  int32_t *adjNearRows = nullptr, *adjNearIdx = nullptr; int64_t *adjNearPtr = nullptr;
  int32_t *adjFarRows = nullptr, *adjFarIdx = nullptr; int64_t *adjFarPtr = nullptr;
  int32_t *adjS2lRows = nullptr, *adjS2lIdx = nullptr; int64_t *adjS2lPtr = nullptr;
  double *uc2ueT = nullptr, *m2mT = nullptr, *dc2deT = nullptr, *l2lT = nullptr;
  double* gradT = nullptr;  // [nt][3] permuted order
  int32_t *vParentsT = nullptr, *vNbrTIdx = nullptr; int64_t *vNbrTPtr = nullptr; int8_t *vNbrOffT = nullptr;
  int32_t *vRowOut = nullptr, *vNbrIn = nullptr, *vRowOutT = nullptr, *vNbrInT = nullptr;  // [rows|entries][8]
  bool adjListsReady = false, adjOpsStale = true;
  bool vListsReady = false;  // the expanded V lists (vTrgPtr .. vSrcEnt) are on the device
  bool hadPQ = true;
  // split-K partial tiles of the FP32 row GEMMs, and the SM count
  double* gemmScratch = nullptr;
  size_t gemmScratchBytes = 0;
  int numSMs = 148;
  // launch shapes chosen by fmmg_autotune (defaults otherwise): rows per CTA of
  // the FP32 and FP64 Hadamard kernels, and split-K when a GEMM's tiles fill
  // fewer than gemmSplitMul CTAs per SM (0: never split)
  // fmmg_autotune (defaults otherwise), and the form of the FP32 Hadamard
  // (1, 2: 27-product accumulators, 1 or 2 right-hand sides a thread; 3, 4:
  // output-child accumulators, 2 or 4 right-hand sides a thread)
  // tcMask: which FP32 GEMM classes the tensor-core path takes (bit 0 leaf
  // C2E F1, 1 leaf C2E F2, 2 folded C2E x M2M, 3 L2L, 4 downward C2E F1,
  // 5 downward C2E F2); tcProducts: 3 (hi*hi + hi*lo + lo*hi) or 4 (+ lo*lo)
  struct Tune {
    int hadRows = 128, pqParents = 128, gemmSplitMul = 2, hadRhsPerThread = 4, tcMask = 63, tcProducts = 3;
  } tune;
  // FP32 row GEMMs: 1 on the tensor cores (3xTF32, default), 0 the wide-tile
  // CUDA-core kernel, 2 the 128 x 64 CUDA-core kernel
  int gemmPath = 1;
  // the same operators split and laid out for the tensor-core kernel
  TcOp cL2L, cUpF1, cUpF2, cDnF1, cDnF2, cM2MUp;
  // FP32 operators transposed and zero padded for the wide-tile GEMM,
  // Wt[k][n]: K to a multiple of 16, N to a multiple of 160 (ld)
  struct OpT {
    float* p = nullptr;
    int ld = 0;
    size_t cap = 0;  // allocated floats
  };
  OpT tL2L, tUpF1, tUpF2, tDnF1, tDnF2, tM2MUp;
  // C2E up x M2M folded (Plan fold_c2e_m2m), FP32 [ue][8 ue]: the FP32 pass
  // takes a parent's upward density from its children's in one product
  float* m2mUp32 = nullptr;
  int* devErr = nullptr;  // set by kernels whose bounded waits gave up
  float adjMs = 0.f;
  // dense check scratch
  double *chkPos = nullptr, *chkOut = nullptr;
  size_t chkCap = 0;
  // timing
  cudaEvent_t ev[EV_COUNT] = {};
  bool evReady = false;
  float stageMs[7] = {0, 0, 0, 0, 0, 0, 0};
  float kernMs[EV_COUNT - 1] = {};
  // wall time of the last dev_upload, ms: geometry and tree arrays, work
  // lists, operator tables, work arrays and the rest
  double uploadMs[4] = {0, 0, 0, 0};
  int lastLaunches = 0;  // kernels launched by the last single-RHS evaluate  // interval k = ev[k] .. ev[k+1]
  // every device block of the handle (sizes in allocBytes); after a re-setup
  // the previous setup's blocks wait in spare for dev_alloc to reuse them
  std::vector<void*> allocs;
  std::vector<size_t> allocBytes;
  struct Block {
    void* p;
    size_t bytes;
  };
  std::vector<Block> spare;
};

// counts of the last stage launch list (for reporting)
struct LaunchStats {
  int launches = 0;
};

std::string dev_upload(const Plan& P, DevState& D, const double* src, const double* nrm, const double* trg);
std::string dev_upload_operators(const Plan& P, DevState& D);
// the expanded V lists on the device (formed on the host first if need be);
// a no-op once done.  Call before any capture of a path that reads them
std::string dev_upload_vlists(const Plan& P, DevState& D);
// a device block owned by D: a spare block of the previous setup when one
// fits (bytes .. 1.5 bytes), else cudaMalloc
cudaError_t dev_alloc(DevState& D, void** p, size_t bytes);
void dev_free(DevState& D);
// re-setup: after the handle's streams drain, every block moves to D.spare
// for the next setup's dev_alloc calls and the pointers are cleared as by
// dev_free; dev_trim then frees the blocks nothing reused
void dev_release_for_reuse(DevState& D);
void dev_trim(DevState& D);
// run one right-hand side; den/val are device arrays in caller order
std::string dev_evaluate(const Plan& P, DevState& D, const double* dDenCaller, double* dValCaller,
                         int precision, int stageMask, bool timed, LaunchStats* st);
// k right-hand sides in caller order ([k][n*DOF]); with timed, the kernel
// times are those of the last chunk of right-hand sides
std::string dev_evaluate_mixed(const Plan& P, DevState& D, const double* dDenCaller, double* dValCaller, int k,
                               int stageMask, bool timed, LaunchStats* st);
// FP64 building blocks shared with the adjoint (stages.cu)
struct Scale4;
void gemm_rows(DevState& D, int nrows, const int32_t* rows, const int32_t* chd, int xChild, int yChild,
               const double* X, int64_t ldx, const double* W, double* Y, int64_t ldy, int K, int N, Scale4 xs,
               Scale4 ys, double beta, LaunchStats* ls);
void spectral_fwd(const Plan& P, DevState& D, int n, const int32_t* nodes, Scale4 deg, int dof, const double* x,
                  double2* spec);
void spectral_inv(const Plan& P, DevState& D, int n, const int32_t* nodes, int dof, const double2* spec, double* y,
                  Scale4 outDeg);
// transposed scalar Hadamard on the parent pairs inverted per source parent
void hadamard_pq64_adj(const Plan& P, DevState& D, const double2* in, double2* out);
void hadamard_list64(const Plan& P, DevState& D, int nOut, const int64_t* ptr, const int32_t* ent, const double2* in,
                     double2* out, bool conj);
// internal stage bit: run upward, V, X (S2L) and downward stages only, leaving
// the target values untouched (the far field the target gradient needs)
constexpr int STAGE_NO_TARGETS = 256;
// permutation helpers: out[i] = in[perm[i]] (gather), out[perm[i]] = in[i] (scatter)
void gather_rows(cudaStream_t st, int64_t n, int dof, const int64_t* perm, const double* in, double* out);
void scatter_rows(cudaStream_t st, int64_t n, int dof, const int64_t* perm, const double* in, double* out);
// forward stages into the handle's work arrays for density dDen (caller order)
std::string dev_far_field(const Plan& P, DevState& D, const double* dDen);
// reads and clears the device error flag (synchronises the handle's stream)
std::string dev_take_error(DevState& D, int* flag);
// Runs the bounded-wait error path on `device` (k_wait_selftest); *flag = 1
// when the wait ran out.
std::string dev_wait_selftest(int device, int arrive, long long limitNs, int* flag);
// transposed FMM: g = A^T w for one right-hand side (caller order), and with
// gradT != nullptr the target-position gradient of <w, A sigma> ([nt][3])
std::string dev_adjoint(const Plan& P, DevState& D, const double* dDen, const double* dW, double* dG,
                        double* dGradT, bool timed);
// dense FP64 sums at device positions (caller-order source arrays are the
// permuted copies held on the device plus the permuted density)
std::string dev_dense(const Plan& P, DevState& D, const double* dDenCaller, int64_t nchk,
                      const double* hPos, double* hOut);

}  // namespace fmmg
