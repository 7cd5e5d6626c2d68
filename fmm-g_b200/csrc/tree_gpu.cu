// tree_gpu.cu -- the adaptive octree and the target binning on the GPU
// (stands in for DENDRO points2Octree + CreateAncestors and the binning of
// fmm3d_mpi/let3d_mpi.cpp:268-288, 611-726, 1230-1285, 1470-1538).
//
// The same tree, permutations and ranges as Plan::build_tree / bin_targets,
// bit for bit: level by level, a node splits while it holds more than ptsMax
// sources and is above maxLevel (the root always), making 8 children numbered
// after the level in parent order; its points go to the octant of the box
// centre (the host's centre expression, rounded the same way) by a stable
// partition of its range.  The stable partition is a rank: a point's new
// position is its child's start plus the number of points of the same octant
// before it in the parent's range, from a device-wide scan of 8 octant
// counters over the positions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "plan.hpp"
#include "plan_pool.cuh"

namespace fmmg {

#define TG_CK(x)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) return std::string("tree device: ") + cudaGetErrorString(e_); \
  } while (0)
#define FMMG_STRTRY(x)               \
  do {                               \
    std::string e_ = (x);            \
    if (!e_.empty()) return e_;      \
  } while (0)

constexpr int TG_THREADS = 256, TG_PER = 16, TG_CHUNK = TG_THREADS * TG_PER;
constexpr uint8_t TG_IDLE = 255;  // a position whose node does not split at this level

struct TgGeom {
  double R2;       // 2 R, R = 2^-rootLevel
  double ll[3];    // ctr - R
};

// Plan::node_center: ll + (2R) (p + 1/2) / 2^d, each operation rounded once
__device__ __forceinline__ double tg_coord(const TgGeom& g, int k, int p, int d) {
  return __dadd_rn(g.ll[k], __ddiv_rn(__dmul_rn(g.R2, __dadd_rn((double)p, 0.5)), (double)(1 << d)));
}

// split flags of the level's nodes [lvS, lvS + nl): sources (mode 0) split
// when the root or above ptsMax and maxLevel; targets (mode 1) follow the
// tree's children
__global__ void k_tg_flags(int lvS, int nl, int d, const int64_t* __restrict__ cnt, const int32_t* __restrict__ chd,
                           int ptsMax, int maxLevel, int mode, int32_t* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nl) return;
  const int n = lvS + i;
  flag[i] = mode == 0 ? ((n == 0) || (cnt[n] > ptsMax && d < maxLevel)) : (chd[n] >= 0);
}

// exclusive scan of nl flags in one CTA (levels hold at most a few million
// nodes); total -> *tot
__global__ void k_tg_scan_flags(int nl, const int32_t* __restrict__ flag, int32_t* __restrict__ off,
                                int32_t* __restrict__ tot) {
  __shared__ int32_t part[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const int per = (nl + T - 1) / T, a = min(nl, t * per), b = min(nl, a + per);
  int s = 0;
  for (int i = a; i < b; i++) s += flag[i];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int i = 0; i < T; i++) {
      const int v = part[i];
      part[i] = run;
      run += v;
    }
    *tot = run;
  }
  __syncthreads();
  int run = part[t];
  for (int i = a; i < b; i++) {
    off[i] = run;
    run += flag[i];
  }
}

// the children of the level's split nodes (sources): ids first = lvE + 8 off
__global__ void k_tg_children(int lvS, int nl, int lvE, int d, const int32_t* __restrict__ flag,
                              const int32_t* __restrict__ off, int32_t* __restrict__ depth, int32_t* __restrict__ par,
                              int32_t* __restrict__ chd, int32_t* __restrict__ path, int64_t* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nl || !flag[i]) return;
  const int n = lvS + i, f = lvE + 8 * off[i];
  chd[n] = f;
  for (int k = 0; k < 8; k++) {
    const int c = f + k;
    depth[c] = d + 1;
    par[c] = n;
    chd[c] = -1;
    path[3 * c + 0] = 2 * path[3 * n + 0] + (k >> 2);
    path[3 * c + 1] = 2 * path[3 * n + 1] + ((k >> 1) & 1);
    path[3 * c + 2] = 2 * path[3 * n + 2] + (k & 1);
    cnt[c] = 0;
  }
}

// octant code of every position whose node splits at this level, and the
// children's counts
__global__ void k_tg_codes(int64_t np, int lvS, int lvE, int d, TgGeom g, const double* __restrict__ pts,
                           const int64_t* __restrict__ perm, const int32_t* __restrict__ posNode,
                           const int32_t* __restrict__ chd, const int32_t* __restrict__ path,
                           uint8_t* __restrict__ code, unsigned long long* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int n = posNode[i];
  if (n < lvS || n >= lvE || chd[n] < 0) {
    code[i] = TG_IDLE;
    return;
  }
  const double* p = pts + 3 * perm[i];
  const int k = (p[0] >= tg_coord(g, 0, path[3 * n], d)) * 4 + (p[1] >= tg_coord(g, 1, path[3 * n + 1], d)) * 2 +
                (p[2] >= tg_coord(g, 2, path[3 * n + 2], d));
  code[i] = (uint8_t)k;
  atomicAdd(&cnt[chd[n] + k], 1ull);
}

// children's ranges: beg[child k] = beg[n] + counts of children 0..k-1
__global__ void k_tg_ranges(int lvS, int nl, const int32_t* __restrict__ chd, int64_t* __restrict__ beg,
                            const int64_t* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nl) return;
  const int n = lvS + i;
  if (chd[n] < 0) return;
  int64_t off = beg[n];
  for (int k = 0; k < 8; k++) {
    beg[chd[n] + k] = off;
    off += cnt[chd[n] + k];
  }
}

// 8 octant counters over each chunk of TG_CHUNK positions
__global__ void __launch_bounds__(TG_THREADS) k_tg_chunk_totals(int64_t np, const uint8_t* __restrict__ code,
                                                                 int32_t* __restrict__ tot) {
  __shared__ int32_t s[8];
  if (threadIdx.x < 8) s[threadIdx.x] = 0;
  __syncthreads();
  int c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int64_t a = (int64_t)blockIdx.x * TG_CHUNK + (int64_t)threadIdx.x * TG_PER;
  for (int j = 0; j < TG_PER; j++) {
    const int64_t i = a + j;
    if (i < np && code[i] != TG_IDLE) c[code[i]]++;
  }
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int v = c[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s[k], v);
  }
  __syncthreads();
  if (threadIdx.x < 8) tot[(int64_t)blockIdx.x * 8 + threadIdx.x] = s[threadIdx.x];
}

// exclusive scan of the chunk totals, one thread per octant
__global__ void k_tg_scan_totals(int64_t nchunks, int32_t* __restrict__ tot) {
  const int k = threadIdx.x;
  if (k >= 8) return;
  int32_t run = 0;
  for (int64_t b = 0; b < nchunks; b++) {
    const int32_t v = tot[b * 8 + k];
    tot[b * 8 + k] = run;
    run += v;
  }
}

// per position: the count of earlier positions with its octant (own), and at
// a splitting node's first position all 8 counters (base, per level node)
__global__ void __launch_bounds__(TG_THREADS) k_tg_prefix(int64_t np, int lvS, const uint8_t* __restrict__ code,
                                                          const int32_t* __restrict__ tot,
                                                          const int32_t* __restrict__ posNode,
                                                          const int64_t* __restrict__ beg, int32_t* __restrict__ own,
                                                          int32_t* __restrict__ base) {
  __shared__ int32_t sc[8][TG_THREADS];
  int c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int64_t a = (int64_t)blockIdx.x * TG_CHUNK + (int64_t)threadIdx.x * TG_PER;
  for (int j = 0; j < TG_PER; j++) {
    const int64_t i = a + j;
    if (i < np && code[i] != TG_IDLE) c[code[i]]++;
  }
#pragma unroll
  for (int k = 0; k < 8; k++) sc[k][threadIdx.x] = c[k];
  __syncthreads();
  if (threadIdx.x < 8) {  // exclusive scan of each octant's thread counts
    const int k = threadIdx.x;
    int32_t run = tot[(int64_t)blockIdx.x * 8 + k];
    for (int t = 0; t < TG_THREADS; t++) {
      const int32_t v = sc[k][t];
      sc[k][t] = run;
      run += v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; k++) c[k] = sc[k][threadIdx.x];
  for (int j = 0; j < TG_PER; j++) {
    const int64_t i = a + j;
    if (i >= np || code[i] == TG_IDLE) continue;
    const int n = posNode[i];
    if (beg[n] == i) {
#pragma unroll
      for (int k = 0; k < 8; k++) base[(int64_t)(n - lvS) * 8 + k] = c[k];
    }
    const int k = code[i];
    own[i] = c[k];
    c[k]++;
  }
}

// the stable partition: a splitting node's point moves to its child's start
// plus its rank among the node's points of that octant
__global__ void k_tg_scatter(int64_t np, int lvS, const uint8_t* __restrict__ code,
                             const int32_t* __restrict__ posNode, const int32_t* __restrict__ chd,
                             const int64_t* __restrict__ beg, const int32_t* __restrict__ own,
                             const int32_t* __restrict__ base, const int64_t* __restrict__ perm,
                             int64_t* __restrict__ perm2, int32_t* __restrict__ posNode2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int n = posNode[i];
  if (code[i] == TG_IDLE) {
    perm2[i] = perm[i];
    posNode2[i] = n;
    return;
  }
  const int k = code[i], c = chd[n] + k;
  const int64_t to = beg[c] + (own[i] - base[(int64_t)(n - lvS) * 8 + k]);
  perm2[to] = perm[i];
  posNode2[to] = c;
}

__global__ void k_tg_iota(int64_t n, int64_t* __restrict__ perm, int32_t* __restrict__ posNode) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  perm[i] = i;
  posNode[i] = 0;
}


// One level's stable partition of the positions whose node in [lvS, lvE) has
// children: octant codes and the children's counts, the children's ranges,
// the ranks, the scatter.  perm / posNode are swapped with their spares.
struct TgLevelBufs {
  int64_t *perm, *perm2;
  int32_t *posNode, *posNode2, *own, *base, *tot;
  uint8_t* code;
};
static void tg_level(cudaStream_t st, TgLevelBufs& L, int64_t np, int lvS, int lvE, int d, const TgGeom& g,
                     const double* dPts, const int32_t* chd, const int32_t* path, int64_t* beg, int64_t* cnt) {
  const int nl = lvE - lvS;
  const unsigned gl = (unsigned)((nl + 255) / 256);
  if (np > 0)
    k_tg_codes<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(np, lvS, lvE, d, g, dPts, L.perm, L.posNode, chd, path,
                                                             L.code, reinterpret_cast<unsigned long long*>(cnt));
  k_tg_ranges<<<gl, 256, 0, st>>>(lvS, nl, chd, beg, cnt);
  if (np == 0) return;
  const int64_t nchunks = (np + TG_CHUNK - 1) / TG_CHUNK;
  k_tg_chunk_totals<<<(unsigned)nchunks, TG_THREADS, 0, st>>>(np, L.code, L.tot);
  k_tg_scan_totals<<<1, 32, 0, st>>>(nchunks, L.tot);
  k_tg_prefix<<<(unsigned)nchunks, TG_THREADS, 0, st>>>(np, lvS, L.code, L.tot, L.posNode, beg, L.own, L.base);
  k_tg_scatter<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(np, lvS, L.code, L.posNode, chd, beg, L.own, L.base,
                                                             L.perm, L.perm2, L.posNode2);
  std::swap(L.perm, L.perm2);
  std::swap(L.posNode, L.posNode2);
}

static std::string tg_level_bufs(PlanBufs& B, int64_t np, int maxLevelNodes, TgLevelBufs& L) {
  const int64_t nchunks = (np + TG_CHUNK - 1) / TG_CHUNK;
  TG_CK(B.get(L.perm, np));
  TG_CK(B.get(L.perm2, np));
  TG_CK(B.get(L.posNode, np));
  TG_CK(B.get(L.posNode2, np));
  TG_CK(B.get(L.own, np));
  TG_CK(B.get(L.code, np));
  TG_CK(B.get(L.tot, std::max<int64_t>(nchunks, 1) * 8));
  TG_CK(B.get(L.base, (size_t)std::max(maxLevelNodes, 1) * 8));
  return std::string();
}

// Plan::build_tree and Plan::bin_targets on the device (trgIsSrc: the targets
// are the sources, whose partition they repeat exactly, so it is copied).
std::string tree_build_device(int device, Plan& P, const double* src, const double* trg, bool trgIsSrc) {
  const Options& o = P.o;
  const int64_t ns = P.ns, nt = P.nt;
  TG_CK(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  TG_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  PlanBufs B;  // released after the stream has drained (sg is destroyed first)
  B.device = device;
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } sg{st};
  TgGeom g;
  const double R = std::pow(2.0, -o.rootLevel);
  g.R2 = 2 * R;
  for (int k = 0; k < 3; k++) g.ll[k] = o.ctr[k] - R;
  double* dSrc = nullptr;
  TG_CK(B.get(dSrc, 3 * (size_t)ns));
  TG_CK(cudaMemcpyAsync(dSrc, src, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, st));
  // ---- sources: the tree grows level by level
  int cap = 1024, nn = 1;
  int32_t *depth = nullptr, *par = nullptr, *chd = nullptr, *path = nullptr, *flag = nullptr, *off = nullptr,
          *tot1 = nullptr;
  int64_t *beg = nullptr, *cnt = nullptr;
  TG_CK(B.get(depth, cap));
  TG_CK(B.get(par, cap));
  TG_CK(B.get(chd, cap));
  TG_CK(B.get(path, 3 * (size_t)cap));
  TG_CK(B.get(beg, cap));
  TG_CK(B.get(cnt, cap));
  TG_CK(B.get(tot1, 1));
  {
    const int32_t r4[4] = {0, -1, -1, 0};  // depth, parent, first child, path x (y, z follow)
    const int32_t p3[3] = {0, 0, 0};
    const int64_t b0 = 0, c0 = ns;
    TG_CK(cudaMemcpyAsync(depth, &r4[0], sizeof(int32_t), cudaMemcpyHostToDevice, st));
    TG_CK(cudaMemcpyAsync(par, &r4[1], sizeof(int32_t), cudaMemcpyHostToDevice, st));
    TG_CK(cudaMemcpyAsync(chd, &r4[2], sizeof(int32_t), cudaMemcpyHostToDevice, st));
    TG_CK(cudaMemcpyAsync(path, p3, sizeof(p3), cudaMemcpyHostToDevice, st));
    TG_CK(cudaMemcpyAsync(beg, &b0, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    TG_CK(cudaMemcpyAsync(cnt, &c0, sizeof(int64_t), cudaMemcpyHostToDevice, st));
  }
  // the widest level holds at most 8 children per split node, and a split
  // node holds more than ptsMax points (the root: any)
  const int maxLevelNodes = (int)std::min<int64_t>(8 * (ns / (o.ptsMax + 1) + 1), (int64_t)1 << 30);
  TgLevelBufs L;
  FMMG_STRTRY(tg_level_bufs(B, ns, maxLevelNodes, L));
  TG_CK(B.get(flag, maxLevelNodes));
  TG_CK(B.get(off, maxLevelNodes));
  if (ns > 0) k_tg_iota<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(ns, L.perm, L.posNode);
  std::vector<int> levelBeg(1, 0);
  int lvS = 0, lvE = 1, d = 0;
  while (lvS < lvE) {
    const int nl = lvE - lvS;
    const unsigned gl = (unsigned)((nl + 255) / 256);
    k_tg_flags<<<gl, 256, 0, st>>>(lvS, nl, d, cnt, chd, o.ptsMax, o.maxLevel, 0, flag);
    k_tg_scan_flags<<<1, 1024, 0, st>>>(nl, flag, off, tot1);
    int splits = 0;
    TG_CK(cudaMemcpyAsync(&splits, tot1, sizeof(int), cudaMemcpyDeviceToHost, st));
    TG_CK(cudaStreamSynchronize(st));
    const int total = lvE + 8 * splits;
    if (total > cap) {  // grow the node arrays
      const int ncap = std::max(total, 2 * cap);
      int32_t *dp = nullptr, *pp = nullptr, *cp = nullptr, *ph = nullptr;
      int64_t *bg = nullptr, *ct = nullptr;
      TG_CK(B.get(dp, ncap));
      TG_CK(B.get(pp, ncap));
      TG_CK(B.get(cp, ncap));
      TG_CK(B.get(ph, 3 * (size_t)ncap));
      TG_CK(B.get(bg, ncap));
      TG_CK(B.get(ct, ncap));
      TG_CK(cudaMemcpyAsync(dp, depth, sizeof(int32_t) * nn, cudaMemcpyDeviceToDevice, st));
      TG_CK(cudaMemcpyAsync(pp, par, sizeof(int32_t) * nn, cudaMemcpyDeviceToDevice, st));
      TG_CK(cudaMemcpyAsync(cp, chd, sizeof(int32_t) * nn, cudaMemcpyDeviceToDevice, st));
      TG_CK(cudaMemcpyAsync(ph, path, sizeof(int32_t) * 3 * nn, cudaMemcpyDeviceToDevice, st));
      TG_CK(cudaMemcpyAsync(bg, beg, sizeof(int64_t) * nn, cudaMemcpyDeviceToDevice, st));
      TG_CK(cudaMemcpyAsync(ct, cnt, sizeof(int64_t) * nn, cudaMemcpyDeviceToDevice, st));
      depth = dp; par = pp; chd = cp; path = ph; beg = bg; cnt = ct;
      cap = ncap;
    }
    if (splits > 0) {
      k_tg_children<<<gl, 256, 0, st>>>(lvS, nl, lvE, d, flag, off, depth, par, chd, path, cnt);
      tg_level(st, L, ns, lvS, lvE, d, g, dSrc, chd, path, beg, cnt);
    }
    TG_CK(cudaGetLastError());
    nn = total;
    levelBeg.push_back(lvE);
    lvS = lvE;
    lvE = total;
    d++;
  }
  P.nn = nn;
  P.depth.resize(nn);
  P.par.resize(nn);
  P.chd.resize(nn);
  P.path.resize(3 * (size_t)nn);
  P.srcBeg.resize(nn);
  P.srcCnt.resize(nn);
  P.srcPerm.resize(ns);
  TG_CK(cudaMemcpyAsync(P.depth.data(), depth, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaMemcpyAsync(P.par.data(), par, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaMemcpyAsync(P.chd.data(), chd, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaMemcpyAsync(P.path.data(), path, sizeof(int32_t) * 3 * nn, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaMemcpyAsync(P.srcBeg.data(), beg, sizeof(int64_t) * nn, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaMemcpyAsync(P.srcCnt.data(), cnt, sizeof(int64_t) * nn, cudaMemcpyDeviceToHost, st));
  if (ns > 0) TG_CK(cudaMemcpyAsync(P.srcPerm.data(), L.perm, sizeof(int64_t) * ns, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaStreamSynchronize(st));
  P.maxDepth = 0;
  for (int n = 0; n < nn; n++) P.maxDepth = std::max(P.maxDepth, P.depth[n]);
  levelBeg.resize(P.maxDepth + 2);
  levelBeg[P.maxDepth + 1] = nn;
  P.levelBeg = levelBeg;
  // ---- targets through the tree
  if (trgIsSrc) {
    P.trgBeg = P.srcBeg;
    P.trgCnt = P.srcCnt;
    P.trgPerm = P.srcPerm;
    return std::string();
  }
  double* dTrg = nullptr;
  int64_t *tbeg = nullptr, *tcnt = nullptr;
  TG_CK(B.get(dTrg, 3 * (size_t)nt));
  TG_CK(B.get(tbeg, nn));
  TG_CK(B.get(tcnt, nn));
  TG_CK(cudaMemsetAsync(tbeg, 0, sizeof(int64_t) * nn, st));
  TG_CK(cudaMemsetAsync(tcnt, 0, sizeof(int64_t) * nn, st));
  TG_CK(cudaMemcpyAsync(tcnt, &nt, sizeof(int64_t), cudaMemcpyHostToDevice, st));
  if (nt > 0) TG_CK(cudaMemcpyAsync(dTrg, trg, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, st));
  TgLevelBufs T;
  int widest = 1;
  for (int dd = 0; dd <= P.maxDepth; dd++) widest = std::max(widest, P.levelBeg[dd + 1] - P.levelBeg[dd]);
  FMMG_STRTRY(tg_level_bufs(B, nt, widest, T));
  if (nt > 0) k_tg_iota<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nt, T.perm, T.posNode);
  for (int dd = 0; dd <= P.maxDepth; dd++) tg_level(st, T, nt, P.levelBeg[dd], P.levelBeg[dd + 1], dd, g, dTrg, chd, path, tbeg, tcnt);
  TG_CK(cudaGetLastError());
  P.trgBeg.resize(nn);
  P.trgCnt.resize(nn);
  P.trgPerm.resize(nt);
  TG_CK(cudaMemcpyAsync(P.trgBeg.data(), tbeg, sizeof(int64_t) * nn, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaMemcpyAsync(P.trgCnt.data(), tcnt, sizeof(int64_t) * nn, cudaMemcpyDeviceToHost, st));
  if (nt > 0) TG_CK(cudaMemcpyAsync(P.trgPerm.data(), T.perm, sizeof(int64_t) * nt, cudaMemcpyDeviceToHost, st));
  TG_CK(cudaStreamSynchronize(st));
  return std::string();
}

}  // namespace fmmg
