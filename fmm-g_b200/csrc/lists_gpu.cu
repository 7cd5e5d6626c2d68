// lists_gpu.cu -- the U/V/W/X interaction lists on the GPU (the rules of
// fmm3d_mpi/let3d_mpi.cpp:1637-1768, as Plan::build_lists restates them).
//
// One thread per node.  For an evaluator node g it resolves the parent's 27
// neighbour boxes one level up (find_node), walks the 216 candidate positions
// of its own level, steps one level down where the parent-level box has
// children, and classifies each candidate with `adjacent` -- coarser and
// touching: U (leaves only); coarser and apart: X; same level and apart: V;
// same level and touching a leaf: descend, apart boxes to W and touching
// leaves to U.  A leaf adds itself to U.  A count pass sizes each node's raw
// candidates, a fill pass writes them, each node's runs are sorted, made
// unique and filtered by the source flags the list needs (U, X: leaves with
// sources; V, W: non-root nodes with sources below), and a compaction gives
// the CSR arrays -- the host build's lists, entry for entry.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "plan.hpp"
#include "plan_pool.cuh"

namespace fmmg {

#define LS_CK(x)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) return std::string("lists device: ") + cudaGetErrorString(e_); \
  } while (0)

struct LsTree {
  const int32_t *depth, *chd, *par, *path;
  const uint8_t* flags;
};

__device__ __forceinline__ int ls_find(const LsTree& T, int want, int p0, int p1, int p2) {
  int cur = 0;
  while (T.depth[cur] < want && T.chd[cur] >= 0) {
    const int t = 1 << (want - T.depth[cur] - 1);
    const int c0 = p0 / t, c1 = p1 / t, c2 = p2 / t;
    p0 -= c0 * t;
    p1 -= c1 * t;
    p2 -= c2 * t;
    cur = T.chd[cur] + c0 * 4 + c1 * 2 + c2;
  }
  return cur;
}

// Plan::adjacent: the boxes touch (face, edge or corner)
__device__ __forceinline__ bool ls_adjacent(const LsTree& T, int a, int b) {
  const int md = max(T.depth[a], T.depth[b]);
  const int ra = 1 << (md - T.depth[a]), rb = 1 << (md - T.depth[b]);
  const int rs = ra + rb;
  int linf = 0;
  bool le = true;
  for (int k = 0; k < 3; k++) {
    const int dif = abs((2 * T.path[3 * a + k] + 1) * ra - (2 * T.path[3 * b + k] + 1) * rb);
    le = le && dif <= rs;
    linf = max(linf, dif);
  }
  return le && linf == rs;
}

constexpr int LS_STACK = 256;  // the W descent's depth-first stack (7 per level at most, plus one)

// Raw candidates of node g: counts (out == nullptr) or the entries (written
// at out[l] + running count), in the host's visiting order.
__device__ void ls_candidates(const LsTree& T, int g, int* cnt, int32_t* const* out) {
  const bool term = T.chd[g] < 0;
  int c[4] = {0, 0, 0, 0};
  auto put = [&](int l, int v) {
    if (out) out[l][c[l]] = v;
    c[l]++;
  };
  if (g != 0) {
    const int P = T.par[g], dg = T.depth[g];
    const int lim = 1 << dg, plim = lim >> 1;
    const int pp0 = T.path[3 * P], pp1 = T.path[3 * P + 1], pp2 = T.path[3 * P + 2];
    const int pg0 = T.path[3 * g], pg1 = T.path[3 * g + 1], pg2 = T.path[3 * g + 2];
    int nb[27];
    for (int a = 0; a < 27; a++) {
      const int q0 = pp0 + a / 9 - 1, q1 = pp1 + (a / 3) % 3 - 1, q2 = pp2 + a % 3 - 1;
      nb[a] = (q0 < 0 || q1 < 0 || q2 < 0 || q0 >= plim || q1 >= plim || q2 >= plim) ? -1
                                                                                      : ls_find(T, dg - 1, q0, q1, q2);
    }
    int stack[LS_STACK];
    for (int i = -2; i < 4; i++)
      for (int j = -2; j < 4; j++)
        for (int k = -2; k < 4; k++) {
          const int t0 = 2 * pp0 + i, t1 = 2 * pp1 + j, t2 = 2 * pp2 + k;
          if (t0 < 0 || t1 < 0 || t2 < 0 || t0 >= lim || t1 >= lim || t2 >= lim) continue;
          if (t0 == pg0 && t1 == pg1 && t2 == pg2) continue;
          const int a = ((i + 2) / 2) * 9 + ((j + 2) / 2) * 3 + (k + 2) / 2;
          int res = nb[a];
          if (T.depth[res] == dg - 1 && T.chd[res] >= 0) res = T.chd[res] + (t0 & 1) * 4 + (t1 & 1) * 2 + (t2 & 1);
          const bool adj = ls_adjacent(T, res, g);
          if (T.depth[res] < dg) {
            if (adj) {
              if (term) put(0, res);
            } else {
              put(3, res);
            }
          } else if (!adj) {
            put(1, res);
          } else if (term) {
            int sp = 0;
            stack[sp++] = res;
            while (sp > 0) {
              const int f = stack[--sp];
              if (!ls_adjacent(T, f, g)) {
                put(2, f);
              } else if (T.chd[f] < 0) {
                put(0, f);
              } else {
                for (int cc = 0; cc < 8 && sp < LS_STACK; cc++) stack[sp++] = T.chd[f] + cc;
              }
            }
          }
        }
  }
  if (term) put(0, g);
  for (int l = 0; l < 4; l++) cnt[l] = c[l];
}

__global__ void k_ls_count(int nn, LsTree T, int64_t* __restrict__ raw) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nn) return;
  int c[4] = {0, 0, 0, 0};
  if (T.flags[g] & NF_EVTR) ls_candidates(T, g, c, nullptr);
  for (int l = 0; l < 4; l++) raw[(int64_t)l * (nn + 1) + g] = c[l];
}

// in-place insertion sort, unique and flag filter of each node's raw run;
// the kept count goes to keep[l][g]
__global__ void k_ls_fill(int nn, LsTree T, const int64_t* __restrict__ rawOff, int32_t* __restrict__ rawIdx,
                          int64_t* __restrict__ keep) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nn) return;
  int c[4] = {0, 0, 0, 0};
  int32_t* out[4];
  for (int l = 0; l < 4; l++) out[l] = rawIdx + rawOff[(int64_t)l * (nn + 1) + g];
  if (T.flags[g] & NF_EVTR) ls_candidates(T, g, c, out);
  const uint8_t need[4] = {NF_LSRC, NF_SRCE, NF_SRCE, NF_LSRC};
  for (int l = 0; l < 4; l++) {
    int32_t* a = out[l];
    const int n = c[l];
    for (int x = 1; x < n; x++) {
      const int32_t v = a[x];
      int y = x - 1;
      while (y >= 0 && a[y] > v) {
        a[y + 1] = a[y];
        y--;
      }
      a[y + 1] = v;
    }
    int m = 0;
    for (int x = 0; x < n; x++) {
      if (x > 0 && a[x] == a[x - 1]) continue;
      if (!(T.flags[a[x]] & need[l])) continue;
      a[m++] = a[x];
    }
    keep[(int64_t)l * (nn + 1) + g] = m;
  }
}

// exclusive scan of 4 x (nn + 1) counts in place, one CTA per list
__global__ void k_ls_scan(int nn, int64_t* __restrict__ v) {
  __shared__ int64_t part[1024];
  int64_t* a = v + (int64_t)blockIdx.x * (nn + 1);
  const int t = threadIdx.x, T = blockDim.x, n = nn + 1;
  const int per = (n + T - 1) / T, lo = min(n, t * per), hi = min(n, lo + per);
  int64_t s = 0;
  for (int i = lo; i < hi; i++) s += a[i];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    int64_t run = 0;
    for (int i = 0; i < T; i++) {
      const int64_t x = part[i];
      part[i] = run;
      run += x;
    }
  }
  __syncthreads();
  int64_t run = part[t];
  for (int i = lo; i < hi; i++) {
    const int64_t x = a[i];
    a[i] = run;
    run += x;
  }
}

// each node's kept entries to their CSR place (both offset tables hold the
// global positions, the four lists one after another)
__global__ void k_ls_compact(int nn, const int64_t* __restrict__ rawOff, const int32_t* __restrict__ rawIdx,
                             const int64_t* __restrict__ keepOff, int32_t* __restrict__ idx) {
  const int g = blockIdx.x, l = blockIdx.y;
  if (g >= nn) return;
  const int64_t s = rawOff[(int64_t)l * (nn + 1) + g];
  const int64_t d = keepOff[(int64_t)l * (nn + 1) + g], e = keepOff[(int64_t)l * (nn + 1) + g + 1];
  for (int64_t x = threadIdx.x; x < e - d; x += blockDim.x) idx[d + x] = rawIdx[s + x];
}

// NF_USER: every node that some list names (one byte per node; several
// threads may store the same 1)
__global__ void k_ls_user(int64_t n, const int32_t* __restrict__ idx, uint8_t* __restrict__ user) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    user[idx[i]] = 1;
}

// Plan::build_lists on a GPU: P's tree and flags in, P.U/V/W/X out.
std::string lists_build_device(int device, Plan& P) {
  const int nn = P.nn;
  LS_CK(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  LS_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  PlanBufs B;
  B.device = device;
  auto get = [&](auto*& p, size_t n) -> cudaError_t { return B.get(p, n); };
  auto run = [&]() -> std::string {
    int32_t *depth, *chd, *par, *path, *rawIdx;
    uint8_t* flags;
    int64_t *raw, *keep;
    LS_CK(get(depth, nn));
    LS_CK(get(chd, nn));
    LS_CK(get(par, nn));
    LS_CK(get(path, 3 * (size_t)nn));
    LS_CK(get(flags, nn));
    LS_CK(get(raw, 4 * ((size_t)nn + 1)));
    LS_CK(get(keep, 4 * ((size_t)nn + 1)));
    LS_CK(cudaMemcpyAsync(depth, P.depth.data(), sizeof(int32_t) * nn, cudaMemcpyHostToDevice, st));
    LS_CK(cudaMemcpyAsync(chd, P.chd.data(), sizeof(int32_t) * nn, cudaMemcpyHostToDevice, st));
    LS_CK(cudaMemcpyAsync(par, P.par.data(), sizeof(int32_t) * nn, cudaMemcpyHostToDevice, st));
    LS_CK(cudaMemcpyAsync(path, P.path.data(), sizeof(int32_t) * 3 * nn, cudaMemcpyHostToDevice, st));
    LS_CK(cudaMemcpyAsync(flags, P.flags.data(), nn, cudaMemcpyHostToDevice, st));
    LS_CK(cudaMemsetAsync(raw, 0, sizeof(int64_t) * 4 * ((size_t)nn + 1), st));
    LS_CK(cudaMemsetAsync(keep, 0, sizeof(int64_t) * 4 * ((size_t)nn + 1), st));
    const LsTree T{depth, chd, par, path, flags};
    const unsigned gb = (unsigned)((nn + 127) / 128);
    k_ls_count<<<gb, 128, 0, st>>>(nn, T, raw);
    k_ls_scan<<<4, 1024, 0, st>>>(nn, raw);
    int64_t rawTot[4];
    for (int l = 0; l < 4; l++)
      LS_CK(cudaMemcpyAsync(&rawTot[l], raw + (int64_t)l * (nn + 1) + nn, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    LS_CK(cudaStreamSynchronize(st));
    // one raw array for the four lists: list l's runs start at its offsets
    // plus the totals of the lists before it
    std::vector<int64_t> base(5, 0);
    for (int l = 0; l < 4; l++) base[l + 1] = base[l] + rawTot[l];
    LS_CK(get(rawIdx, (size_t)base[4]));
    std::vector<int64_t> rawOffH(4 * ((size_t)nn + 1));
    LS_CK(cudaMemcpyAsync(rawOffH.data(), raw, sizeof(int64_t) * rawOffH.size(), cudaMemcpyDeviceToHost, st));
    LS_CK(cudaStreamSynchronize(st));
    for (int l = 0; l < 4; l++)
      for (int g = 0; g <= nn; g++) rawOffH[(size_t)l * (nn + 1) + g] += base[l];
    LS_CK(cudaMemcpyAsync(raw, rawOffH.data(), sizeof(int64_t) * rawOffH.size(), cudaMemcpyHostToDevice, st));
    k_ls_fill<<<gb, 128, 0, st>>>(nn, T, raw, rawIdx, keep);
    k_ls_scan<<<4, 1024, 0, st>>>(nn, keep);
    std::vector<int64_t> keepOff(4 * ((size_t)nn + 1));
    LS_CK(cudaMemcpyAsync(keepOff.data(), keep, sizeof(int64_t) * keepOff.size(), cudaMemcpyDeviceToHost, st));
    LS_CK(cudaStreamSynchronize(st));
    std::vector<int64_t> kbase(5, 0);
    for (int l = 0; l < 4; l++) kbase[l + 1] = kbase[l] + keepOff[(size_t)l * (nn + 1) + nn];
    for (int l = 0; l < 4; l++)
      for (int g = 0; g <= nn; g++) keepOff[(size_t)l * (nn + 1) + g] += kbase[l];
    int32_t* idx = nullptr;
    LS_CK(get(idx, (size_t)kbase[4]));
    LS_CK(cudaMemcpyAsync(keep, keepOff.data(), sizeof(int64_t) * keepOff.size(), cudaMemcpyHostToDevice, st));
    k_ls_compact<<<dim3(nn, 4), 32, 0, st>>>(nn, raw, rawIdx, keep, idx);
    LS_CK(cudaGetLastError());
    uint8_t* user = nullptr;
    LS_CK(get(user, nn));
    LS_CK(cudaMemsetAsync(user, 0, nn, st));
    if (kbase[4] > 0) k_ls_user<<<1184, 256, 0, st>>>(kbase[4], idx, user);
    LS_CK(cudaGetLastError());
    // each list straight into its host CSR, while the host fills the offsets
    CSR* outs[4] = {&P.U, &P.V, &P.W, &P.X};
    for (int l = 0; l < 4; l++) {
      CSR& o = *outs[l];
      o.idx.resize((size_t)(kbase[l + 1] - kbase[l]));
      if (!o.idx.empty())
        LS_CK(cudaMemcpyAsync(o.idx.data(), idx + kbase[l], sizeof(int32_t) * o.idx.size(), cudaMemcpyDeviceToHost,
                              st));
    }
    std::vector<uint8_t> userH((size_t)nn);
    LS_CK(cudaMemcpyAsync(userH.data(), user, nn, cudaMemcpyDeviceToHost, st));
    for (int l = 0; l < 4; l++) {
      CSR& o = *outs[l];
      o.ptr.resize((size_t)nn + 1);
      for (int g = 0; g <= nn; g++) o.ptr[g] = keepOff[(size_t)l * (nn + 1) + g] - kbase[l];
    }
    LS_CK(cudaStreamSynchronize(st));
    for (int g = 0; g < nn; g++)
      if (userH[g]) P.flags[g] |= NF_USER;
    return std::string();
  };
  std::string err = run();
  cudaStreamSynchronize(st);  // the buffers go back to the pool after this
  cudaStreamDestroy(st);
  return err;
}

}  // namespace fmmg
