// plan.hpp -- host-side setup of the evaluator: the adaptive octree, the
// U/V/W/X interaction lists, their flattened GPU work lists, and the
// operator tables.  This is the setup() half of the reference FMM3d_MPI
// (fmm3d_mpi/fmm3d_setup_mpi.cpp, fmm3d_mpi/let3d_mpi.cpp,
// fmm3d_mpi/matmgnt3d_mpi.cpp) re-laid-out for the GPU:
//  * nodes are numbered level by level (depth-major) and the 8 children of a
//    node are consecutive, so per-node arrays of one level are contiguous and
//    "all children of P" is a single row range;
//  * sources and targets are permuted so that every leaf (and every subtree)
//    owns a contiguous range, in Morton order of the leaves;
//  * each interaction list becomes a CSR array of node ids.
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <vector>

namespace fmmg {

struct Options {
  int kt = 111;
  double coefs[2] = {1.0, 0.25};
  int np = 6;
  int ptsMax = 150;
  int maxLevel = 30;
  double ctr[3] = {0.5, 0.5, 0.5};
  int rootLevel = 1;
};

// node flag bits (fmm3d_mpi/let3d_mpi.hpp:28-39 meanings at one rank)
enum : uint8_t {
  NF_CBTR = 1,   // has sources, not the root: carries an upward density
  NF_USER = 2,   // appears in some list
  NF_EVTR = 4,   // has targets: carries downward data / target values
  NF_SRCE = 16,  // non-root and (non-leaf or has sources)
  NF_LEAF = 32,
  NF_LSRC = 64,  // leaf with sources (glbSrcExaNum > 0 in the reference)
};

struct CSR {
  std::vector<int64_t> ptr;  // size rows + 1
  std::vector<int32_t> idx;
  void clear() { ptr.assign(1, 0); idx.clear(); }
};

struct Plan {
  Options o;
  int sd = 0, td = 0, mm = 0, sdm = 0, tdm = 0;
  double deg[4] = {0, 0, 0, 0};
  bool nrm = false;
  // surfaces and grid (matmgnt3d_mpi.cpp:451-499)
  int nUE = 0, nUC = 0, nDE = 0, nDC = 0, nReg = 0, nEff = 0;
  // the FP32 pass transforms on the (2np-1)^3 grid, the smallest on which the
  // band-to-band M2L convolution does not wrap (offsets -(np-1)..np-1)
  int nReg32 = 0, nEff32 = 0;
  std::vector<double> sam[4];  // UE, UC, DE, DC templates at unit radius scale, [n][3]

  // wall time of the phases of the last build(), ms: sources into the tree,
  // targets binned, node flags and centres, U/V/W/X lists, work lists, and a
  // last phase that is now empty (the adjoint's lists are formed on first use)
  double buildMs[6] = {0, 0, 0, 0, 0, 0};
  // wall time of the operator set's build, ms (0 when it came from the
  // process cache): C2E up pseudo-inverse, C2E down, M2M / L2L tables, M2L
  // translation spectra
  double opsMs[4] = {0, 0, 0, 0};

  // ---- tree
  int64_t ns = 0, nt = 0;
  int nn = 0, maxDepth = 0;
  std::vector<int> levelBeg;  // nodes of depth d: [levelBeg[d], levelBeg[d+1])
  std::vector<int32_t> depth, par, chd;
  std::vector<int32_t> path;  // [nn][3]
  std::vector<uint8_t> flags;
  std::vector<int64_t> srcBeg, srcCnt, trgBeg, trgCnt;  // subtree ranges in permuted order
  std::vector<double> center;                           // [nn][3]
  std::vector<double> radius;                           // [nn]
  std::vector<int64_t> srcPerm, trgPerm;                // permuted position -> caller index

  // ---- lists in the reference form (sorted node ids)
  CSR U, V, W, X;

  // ---- GPU work lists
  std::vector<int32_t> evtrLeaves;  // EVTR leaves (rows of near/far-to-target work)
  CSR nearSrc;                      // per EVTR leaf: source leaves for true-kernel direct sums
  std::vector<int32_t> farLeaves;   // EVTR leaves with W nodes evaluated from their UE surface (M2T)
  CSR farUE;                        // per farLeaves row: those W nodes
  std::vector<int32_t> l2tLeaves;   // EVTR leaves at depth >= 2 (L2T)
  std::vector<int32_t> s2lNodes;    // EVTR nodes with X entries evaluated on the DC surface
  CSR s2lSrc;                       // per s2lNodes row: source leaves
  std::vector<int32_t> s2mLeaves;   // leaves with sources (S2M)
  // per level d: CBTR nodes (upward C2E), CBTR non-leaf parents at d (M2M
  // into them), EVTR non-leaves at d (L2L from them), EVTR nodes at d (C2E down)
  std::vector<std::vector<int32_t>> upC2E, upM2M, dnL2L, dnC2E;
  // the leaves with sources per depth: the upward C2E rows of the FP32 pass,
  // where a parent's upward density comes from the folded C2E x M2M product
  std::vector<std::vector<int32_t>> upLeaf;
  // M2L grouped by parent pairs: for each target parent P (non-leaf, depth >=1,
  // with an EVTR child) the same-depth non-leaf neighbours Q and offset code
  std::vector<int32_t> vParents;  // rows
  CSR vNbr;                       // idx = Q node id
  std::vector<int8_t> vNbrOff;    // parallel to vNbr.idx: (dx+1)*9+(dy+1)*3+(dz+1)
  std::vector<int32_t> vSrcSlot;  // per node: row in the source-spectrum array or -1
  std::vector<int32_t> vSrcNodes; // slot -> node
  std::vector<int32_t> vTrgSlot;  // per node: row in the target-spectrum array or -1
  std::vector<int32_t> vTrgNodes; // slot -> node
  // the same V-lists expanded per target slot: (source slot, translation id),
  // and inverted per source slot for the transposed operator.  Only the
  // expanded-list Hadamards read them (the vector kernels' transposed M2L and
  // the list form chosen by FMMG_HADAMARD=list), so they are formed on first
  // use by expand_v_lists(), not by build()
  mutable std::vector<int64_t> vTrgPtr;   // [nTrgSlots + 1]
  mutable std::vector<int32_t> vTrgEnt;   // pairs (source slot, translation id)
  mutable std::vector<int64_t> vSrcPtr;   // [nSrcSlots + 1]
  mutable std::vector<int32_t> vSrcEnt;   // pairs (target slot, translation id)
  void expand_v_lists() const;            // idempotent until the next build()

  // the parent-pair lists with child slots resolved: per row its 8 output
  // child slots, per neighbour entry its 8 input child slots (-1: no spectrum)
  std::vector<int32_t> vRowOut, vNbrIn;     // forward: target slots of P, source slots of Q

  // ---- adjoint (transposed FMM) work lists: every forward list inverted.
  // Formed on the first adjoint call by build_adjoint_lists(), not by build()
  mutable std::vector<int32_t> adjNearRows;  // source leaves in some near list
  mutable CSR adjNear;                       // per row: the evaluator leaves that list it
  mutable std::vector<int32_t> adjFarRows;   // nodes used through their UE surface (M2T)
  mutable CSR adjFar;                        // per row: the evaluator leaves that list it
  mutable std::vector<int32_t> adjS2lRows;   // source leaves used by S2L
  mutable CSR adjS2l;                        // per row: the nodes whose DC surface they feed
  mutable std::vector<int32_t> vParentsT;    // source parents Q of the grouped M2L
  mutable CSR vNbrT;                         // per row: target parents P
  mutable std::vector<int8_t> vNbrOffT;      // offset code of P - Q
  mutable std::vector<int32_t> vRowOutT, vNbrInT;  // transposed: source slots of Q, target slots of P
  void build_adjoint_lists() const;                // idempotent until the next build()

  // ---- operators (homogeneous equivalent kernels: unit-radius tables)
  // row-major for the GPU GEMMs:
  std::vector<double> uc2ue;     // [nUE*sdm][nUC*tdm]       C2E up (pinv)
  std::vector<double> m2m;       // [nUC*tdm][8*nUE*sdm]     8 octant UE->UC matrices side by side
  std::vector<double> dc2de;     // [nDE*sdm][nDC*tdm]       C2E down (pinv)
  std::vector<double> l2l;       // [8*nDC*tdm][nDE*sdm]     8 octant DE->DC matrices stacked
  std::vector<std::complex<double>> m2lT;  // [316][nEff][sdm*tdm] (FFTW r2c layout)
  std::vector<std::complex<double>> m2lT32;  // [316][nEff32][sdm*tdm]: the same translations, (2np-1)^3 grid
  // the two pseudo-inverses in factored form for the FP32 path:
  // C2E = F2 (F1 x), F1 = diag(1/s) U^T [k][check], F2 = V [equiv][k]
  int kUp = 0, kDn = 0;
  std::vector<double> uc2ueF1, uc2ueF2, dc2deF1, dc2deF2;
  int transId[7][7][7];
  // fold_c2e_m2m of these tables, formed on first use (the FP32 pass and
  // fmmg_operator 6); cleared when the caller replaces C2E up or M2M
  const std::vector<double>& folded_upward() const;
  void drop_folded_upward() { upFold.clear(); }

  // treeDevice >= 0: the tree, the target binning and the U/V/W/X lists on
  // that GPU (tree_gpu.cu, lists_gpu.cu; the same result as the host's)
  std::string build(const Options& opt, int64_t ns, const double* src, const double* nrm, int64_t nt,
                    const double* trg, int treeDevice = -1);
  // the operator tables of (kt, coefs, np), copied from the process's most
  // recent sets when they hold it
  std::string build_operators();
  // the operator tables of s (built by build_operators), moved into this plan
  void take_operators(Plan&& s);
  // refactor the pinv the caller replaced (0: C2E up, 2: C2E down) from its
  // explicit table, so the FP32 pass applies the same operator
  void refactor_c2e(int which);
  // m2lT32[id] from m2lT[id] (after the caller replaced it): inverse r2c to
  // the kernel samples, keep the offsets -(np-1)..np-1, r2c on the odd grid
  void m2l_spectrum32(int id);
  int child(int n, int o) const { return chd[n] + o; }
  bool leaf(int n) const { return chd[n] < 0; }

 private:
  mutable std::vector<double> upFold;  // [nUE*sdm][8*nUE*sdm], empty until formed
  mutable bool vExpanded = false, adjBuilt = false;  // the lazily formed lists are current
  std::string build_operators_uncached();
  template <class S> void assign_operators(S&& s);  // copies or moves, as S is
  void build_tree(const double* src);
  void bin_targets(const double* trg);
  void build_lists();
  void build_worklists();
  int find_node(int wntDepth, const int* p) const;
  bool adjacent(int a, int b) const;
  void node_center(int depth, const int* path, double* c) const;
};

// linear algebra used by the operator builder (linalg.cpp); with a device
// set (>= 0) on the calling thread the SVDs and the fold run there
// (linalg_gpu.cu), with bit-identical results
void set_linalg_device(int device);
// Plan::build_tree + bin_targets on a GPU (tree_gpu.cu); trgIsSrc: the
// targets are the sources
std::string tree_build_device(int device, Plan& P, const double* src, const double* trg, bool trgIsSrc);
// Plan::build_lists on a GPU (lists_gpu.cu): the same U/V/W/X lists
std::string lists_build_device(int device, Plan& P);
struct LinalgDeviceScope {
  explicit LinalgDeviceScope(int device) { set_linalg_device(device); }
  ~LinalgDeviceScope() { set_linalg_device(-1); }
};
// the truncated pseudo-inverse of A (m x n column-major) from one SVD, both as
// the explicit table R (n x m column-major; skipped when R is NULL) and in
// factored form R = F2 F1, F1 = diag(1/s) U^T (k x m, row-major), F2 = V
// (n x k, row-major); returns k, the singular values kept (s >= eps s_max)
int pinv_truncated(int m, int n, const double* A_colmajor, double eps, double* R_colmajor,
                   std::vector<double>& F1, std::vector<double>& F2);
void rfft3_host(int n, int howmany, const double* in, std::complex<double>* out);
int svd_factors(int m, int n, const double* B_rowmajor, double relCut, std::vector<double>& F1,
                std::vector<double>& F2);
// [nUE*sdm][8*nUE*sdm] row-major: C2E up times the 8 side-by-side M2M
// matrices, F2 (F1 M2M) in FP64 -- a parent's upward equivalent density from
// its children's in one product (the FP32 pass)
std::vector<double> fold_c2e_m2m(const Plan& P);

}  // namespace fmmg
