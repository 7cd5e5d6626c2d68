// plan.cpp -- host setup: octree, lists, GPU work lists, operator tables.
#include "plan.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <numeric>
#include <omp.h>
#include <utility>

#include "kernels.hpp"

namespace fmmg {

// ------------------------------------------------------------------ geometry
// Centre of a box: fmm3d_mpi/let3d_mpi.cpp:1808-1818.  The expression order
// is kept so that the point binning (p >= centre) is reproducible bit for bit.
void Plan::node_center(int d, const int* p, double* c) const {
  double R = std::pow(2.0, -o.rootLevel);
  double ll[3] = {o.ctr[0] - R, o.ctr[1] - R, o.ctr[2] - R};
  int tmp = 1 << d;
  for (int k = 0; k < 3; k++) c[k] = ll[k] + (2 * R) * (p[k] + 0.5) / double(tmp);
}

// Stable partition of perm[b, e) into the 8 octants about centre c (code
// (p >= c) per axis, x most significant); cnt receives the octant sizes.
// With `chunked` (called outside a parallel region, for big ranges) the range
// is cut into one chunk per thread: each chunk counts its codes, then places
// its points after the earlier chunks' points of the same octant, which gives
// the order of the sequential pass.
static void octant_partition(const double* pts, int64_t* perm, int64_t* tmp, int64_t b, int64_t e,
                             const double* c, int64_t cnt[8], bool chunked) {
  auto code_of = [&](int64_t i) {
    const double* p = pts + 3 * perm[i];
    return (p[0] >= c[0]) * 4 + (p[1] >= c[1]) * 2 + (p[2] >= c[2]);
  };
  if (!chunked) {
    for (int k = 0; k < 8; k++) cnt[k] = 0;
    for (int64_t i = b; i < e; i++) cnt[code_of(i)]++;
    int64_t off[8];
    off[0] = b;
    for (int k = 1; k < 8; k++) off[k] = off[k - 1] + cnt[k - 1];
    for (int64_t i = b; i < e; i++) tmp[off[code_of(i)]++] = perm[i];
    std::memcpy(&perm[b], &tmp[b], sizeof(int64_t) * (e - b));
    return;
  }
  const int T = std::max(1, omp_get_max_threads());
  const int64_t chunk = (e - b + T - 1) / T;
  std::vector<int64_t> pos((size_t)T * 8, 0);
  std::vector<uint8_t> code(e - b);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < T; t++)
    for (int64_t i = b + t * chunk; i < std::min(e, b + (t + 1) * chunk); i++) {
      const int k = code_of(i);
      code[i - b] = (uint8_t)k;
      pos[(size_t)t * 8 + k]++;
    }
  int64_t at = b;
  for (int k = 0; k < 8; k++) {
    cnt[k] = 0;
    for (int t = 0; t < T; t++) {
      const int64_t n = pos[(size_t)t * 8 + k];
      pos[(size_t)t * 8 + k] = at;
      at += n;
      cnt[k] += n;
    }
  }
#pragma omp parallel for schedule(static)
  for (int t = 0; t < T; t++)
    for (int64_t i = b + t * chunk; i < std::min(e, b + (t + 1) * chunk); i++)
      tmp[pos[(size_t)t * 8 + code[i - b]]++] = perm[i];
#pragma omp parallel for schedule(static)
  for (int64_t i = b; i < e; i++) perm[i] = tmp[i];
}

// Ranges at least this long are partitioned by all threads at once (the top
// levels hold few nodes with many points each).
constexpr int64_t kChunkedPartition = 1 << 16;

// Adaptive octree (stands in for DENDRO points2Octree + CreateAncestors,
// fmm3d_mpi/let3d_mpi.cpp:268-288, 611-726): an octant is split while it
// holds more than ptsMax sources and is above maxLevel, the root is always
// split, a split makes all 8 children.  Sources are binned by p >= centre per
// axis (let3d_mpi.cpp:1255-1267) with a stable partition, which leaves every
// subtree's sources contiguous in Morton order.
void Plan::build_tree(const double* src) {
  depth.assign(1, 0); par.assign(1, -1); chd.assign(1, -1);
  path.assign(3, 0);
  srcBeg.assign(1, 0); srcCnt.assign(1, ns);
  srcPerm.resize(ns);
  std::iota(srcPerm.begin(), srcPerm.end(), (int64_t)0);
  std::vector<int64_t> tmp(ns);
  levelBeg.assign(1, 0);
  int lvS = 0, lvE = 1, d = 0;
  while (lvS < lvE) {
    // child ids in parent order
    std::vector<int> first(lvE - lvS, -1);
    int next = lvE;
    for (int n = lvS; n < lvE; n++) {
      bool split = (n == 0) || (srcCnt[n] > o.ptsMax && d < o.maxLevel);
      if (split) { first[n - lvS] = next; next += 8; }
    }
    int total = next;
    depth.resize(total); par.resize(total); chd.resize(total); path.resize(3 * (size_t)total);
    srcBeg.resize(total); srcCnt.resize(total);
    auto split_node = [&](int n, bool chunked) {
      const int f = first[n - lvS];
      chd[n] = f;
      double c[3];
      node_center(d, &path[3 * (size_t)n], c);
      const int64_t b = srcBeg[n], e = b + srcCnt[n];
      int64_t cnt[8];
      octant_partition(src, srcPerm.data(), tmp.data(), b, e, c, cnt, chunked);
      int64_t off = b;
      for (int k = 0; k < 8; k++) {
        int ch = f + k;
        depth[ch] = d + 1; par[ch] = n; chd[ch] = -1;
        path[3 * (size_t)ch + 0] = 2 * path[3 * (size_t)n + 0] + (k >> 2);
        path[3 * (size_t)ch + 1] = 2 * path[3 * (size_t)n + 1] + ((k >> 1) & 1);
        path[3 * (size_t)ch + 2] = 2 * path[3 * (size_t)n + 2] + (k & 1);
        srcBeg[ch] = off; srcCnt[ch] = cnt[k];
        off += cnt[k];
      }
    };
    for (int n = lvS; n < lvE; n++)
      if (first[n - lvS] >= 0 && srcCnt[n] >= kChunkedPartition) split_node(n, true);
#pragma omp parallel for schedule(dynamic, 8)
    for (int n = lvS; n < lvE; n++)
      if (first[n - lvS] >= 0 && srcCnt[n] < kChunkedPartition) split_node(n, false);
    levelBeg.push_back(lvE);
    lvS = lvE; lvE = total; d++;
  }
  nn = (int)depth.size();
  maxDepth = 0;
  for (int n = 0; n < nn; n++) maxDepth = std::max(maxDepth, depth[n]);
  levelBeg.resize(maxDepth + 2);
  levelBeg[maxDepth + 1] = nn;
}

// Targets binned into the source tree (fmm3d_mpi/let3d_mpi.cpp:1470-1538).
void Plan::bin_targets(const double* trg) {
  trgBeg.assign(nn, 0); trgCnt.assign(nn, 0);
  trgPerm.resize(nt);
  std::iota(trgPerm.begin(), trgPerm.end(), (int64_t)0);
  std::vector<int64_t> tmp(nt);
  trgCnt[0] = nt;
  for (int d = 0; d <= maxDepth; d++) {
    auto bin_node = [&](int n, bool chunked) {
      double c[3];
      node_center(d, &path[3 * (size_t)n], c);
      const int64_t b = trgBeg[n], e = b + trgCnt[n];
      int64_t cnt[8];
      octant_partition(trg, trgPerm.data(), tmp.data(), b, e, c, cnt, chunked);
      int64_t off = b;
      for (int k = 0; k < 8; k++) {
        trgBeg[chd[n] + k] = off;
        trgCnt[chd[n] + k] = cnt[k];
        off += cnt[k];
      }
    };
    for (int n = levelBeg[d]; n < levelBeg[d + 1]; n++)
      if (chd[n] >= 0 && trgCnt[n] >= kChunkedPartition) bin_node(n, true);
#pragma omp parallel for schedule(dynamic, 8)
    for (int n = levelBeg[d]; n < levelBeg[d + 1]; n++)
      if (chd[n] >= 0 && trgCnt[n] < kChunkedPartition) bin_node(n, false);
  }
}

// fmm3d_mpi/let3d_mpi.cpp:1833-1853
int Plan::find_node(int wntDepth, const int* wp) const {
  int cur = 0;
  int p[3] = {wp[0], wp[1], wp[2]};
  while (depth[cur] < wntDepth && chd[cur] >= 0) {
    int t = 1 << (wntDepth - depth[cur] - 1);
    int c0 = p[0] / t, c1 = p[1] / t, c2 = p[2] / t;
    p[0] -= c0 * t; p[1] -= c1 * t; p[2] -= c2 * t;
    cur = chd[cur] + c0 * 4 + c1 * 2 + c2;
  }
  return cur;
}

// fmm3d_mpi/let3d_mpi.cpp:1856-1876: boxes touch (face, edge or corner)
bool Plan::adjacent(int a, int b) const {
  int md = std::max(depth[a], depth[b]);
  int ra = 1 << (md - depth[a]), rb = 1 << (md - depth[b]);
  int rs = ra + rb, linf = 0;
  bool le = true;
  for (int k = 0; k < 3; k++) {
    int dif = std::abs((2 * path[3 * (size_t)a + k] + 1) * ra - (2 * path[3 * (size_t)b + k] + 1) * rb);
    le = le && dif <= rs;
    linf = std::max(linf, dif);
  }
  return le && linf == rs;
}

// U/V/W/X lists of every evaluator node (fmm3d_mpi/let3d_mpi.cpp:1637-1768):
// the candidates are the children of the parent's neighbours at the node's
// depth, resolved to the deepest existing box; lists hold sorted unique ids.
// A candidate's box is found from the parent's 27 neighbour boxes (its parent
// position is one of them), one level down when that box has children; nodes
// go in chunks whose lists are appended to per-chunk arrays in node order.
void Plan::build_lists() {
  constexpr int CH = 128;
  const int nch = (nn + CH - 1) / CH;
  std::vector<std::vector<int32_t>> part[4];
  for (auto& pv : part) pv.assign(nch, {});
  std::vector<int64_t> cnt[4];
  for (auto& c : cnt) c.assign(nn, 0);
#pragma omp parallel
  {
    std::vector<int32_t> L[4], rest;  // U, V, W, X of one node; W descent work
#pragma omp for schedule(dynamic, 1)
    for (int ch = 0; ch < nch; ch++)
      for (int g = ch * CH; g < std::min(nn, (ch + 1) * CH); g++) {
        if (!(flags[g] & NF_EVTR)) continue;
        for (auto& l : L) l.clear();
        std::vector<int32_t>&Us = L[0], &Vs = L[1], &Ws = L[2], &Xs = L[3];
        const bool term = leaf(g);
        if (g != 0) {
          const int P = par[g], dg = depth[g];
          const int lim = 1 << dg, plim = lim >> 1;
          const int* pp = &path[3 * (size_t)P];
          const int* pg = &path[3 * (size_t)g];
          int nb[27];  // the box holding each neighbour position of P at depth dg - 1
          for (int a = 0; a < 27; a++) {
            const int q[3] = {pp[0] + a / 9 - 1, pp[1] + (a / 3) % 3 - 1, pp[2] + a % 3 - 1};
            nb[a] = (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= plim || q[1] >= plim || q[2] >= plim)
                        ? -1 : find_node(dg - 1, q);
          }
          for (int i = -2; i < 4; i++)
            for (int j = -2; j < 4; j++)
              for (int k = -2; k < 4; k++) {
                int tp[3] = {2 * pp[0] + i, 2 * pp[1] + j, 2 * pp[2] + k};
                if (tp[0] < 0 || tp[1] < 0 || tp[2] < 0 || tp[0] >= lim || tp[1] >= lim || tp[2] >= lim) continue;
                if (tp[0] == pg[0] && tp[1] == pg[1] && tp[2] == pg[2]) continue;
                // i, j, k in [-2, 4): the parent-level offset floor(i / 2) is -1, 0 or 1,
                // and an in-range position has an in-range parent position
                const int a = ((i + 2) / 2) * 9 + ((j + 2) / 2) * 3 + (k + 2) / 2;
                int res = nb[a];
                if (depth[res] == dg - 1 && !leaf(res)) res = chd[res] + (tp[0] & 1) * 4 + (tp[1] & 1) * 2 + (tp[2] & 1);
                bool adj = adjacent(res, g);
                if (depth[res] < dg) {
                  if (adj) { if (term) Us.push_back(res); }
                  else Xs.push_back(res);
                } else if (!adj) {
                  Vs.push_back(res);
                } else if (term) {
                  rest.assign(1, res);
                  while (!rest.empty()) {
                    int f = rest.back();
                    rest.pop_back();
                    if (!adjacent(f, g)) Ws.push_back(f);
                    else if (leaf(f)) Us.push_back(f);
                    else for (int c = 0; c < 8; c++) rest.push_back(chd[f] + c);
                  }
                }
              }
        }
        if (term) Us.push_back(g);
        const uint8_t need[4] = {NF_LSRC, NF_SRCE, NF_SRCE, NF_LSRC};
        for (int l = 0; l < 4; l++) {
          std::sort(L[l].begin(), L[l].end());
          L[l].erase(std::unique(L[l].begin(), L[l].end()), L[l].end());
          L[l].erase(std::remove_if(L[l].begin(), L[l].end(), [&](int32_t s) { return !(flags[s] & need[l]); }),
                     L[l].end());
          part[l][ch].insert(part[l][ch].end(), L[l].begin(), L[l].end());
          cnt[l][g] = (int64_t)L[l].size();
        }
      }
  }
  CSR* out[4] = {&U, &V, &W, &X};
  for (int l = 0; l < 4; l++) {
    CSR& o = *out[l];
    o.ptr.assign(nn + 1, 0);
    for (int n = 0; n < nn; n++) o.ptr[n + 1] = o.ptr[n] + cnt[l][n];
    o.idx.resize(o.ptr[nn]);
#pragma omp parallel for schedule(static)
    for (int ch = 0; ch < nch; ch++)
      std::copy(part[l][ch].begin(), part[l][ch].end(), o.idx.begin() + o.ptr[ch * CH]);
    for (int32_t s : o.idx) flags[s] |= NF_USER;
  }
}

// Flattened work for the GPU stages, following the per-node decisions of
// fmm3d_mpi/fmm3d_eval_mpi.cpp: W sources with fewer than |UE|*srcDOF values
// and X sources of a leaf with fewer than |DC|*trgDOF values are summed
// directly (S2T, :1146 and :1249); the others go through the UE surface (M2T)
// or the DC surface (S2L).
void Plan::build_worklists() {
  const int64_t ueSize = (int64_t)nUE * sdm, dcSize = (int64_t)nDC * tdm;
  evtrLeaves.clear(); nearSrc.clear(); farUE.clear(); farLeaves.clear(); l2tLeaves.clear();
  s2lNodes.clear(); s2lSrc.clear(); s2mLeaves.clear();
  // A W node is summed directly (near list) when it is a source leaf with
  // fewer source values than its UE surface, else through that surface (far
  // list); a leaf's X list is summed directly when the leaf has fewer target
  // values than its DC surface, else onto the DC surface (S2L).  Per node the
  // entry counts are found in parallel, the row lists and offsets follow in
  // node order, and the entries are written in parallel at those offsets, in
  // the order U, direct W, direct X (near) and W order (far).
  auto wDirect = [&](int w) { return (flags[w] & NF_LSRC) && srcCnt[w] * sd < ueSize; };
  auto xDirect = [&](int g) { return leaf(g) && trgCnt[g] * td < dcSize; };
  std::vector<int32_t> cNear(nn, 0), cFar(nn, 0);
#pragma omp parallel for schedule(static, 1024)
  for (int g = 0; g < nn; g++) {
    if (!(flags[g] & NF_EVTR) || !leaf(g)) continue;
    int nd = 0;
    for (int64_t e = W.ptr[g]; e < W.ptr[g + 1]; e++) nd += wDirect(W.idx[e]) ? 1 : 0;
    cNear[g] = (int32_t)(U.ptr[g + 1] - U.ptr[g]) + nd + (xDirect(g) ? (int32_t)(X.ptr[g + 1] - X.ptr[g]) : 0);
    cFar[g] = (int32_t)(W.ptr[g + 1] - W.ptr[g]) - nd;
  }
  std::vector<int64_t> oNear(nn, -1), oFar(nn, -1), oS2l(nn, -1);
  for (int g = 0; g < nn; g++) {
    if ((flags[g] & NF_LSRC)) s2mLeaves.push_back(g);
    if (!(flags[g] & NF_EVTR)) continue;
    if (leaf(g)) {
      evtrLeaves.push_back(g);
      if (depth[g] >= 2) l2tLeaves.push_back(g);
      oNear[g] = nearSrc.ptr.back();
      nearSrc.ptr.push_back(oNear[g] + cNear[g]);
      if (cFar[g] > 0) {
        farLeaves.push_back(g);
        oFar[g] = farUE.ptr.back();
        farUE.ptr.push_back(oFar[g] + cFar[g]);
      }
    }
    if (!xDirect(g) && X.ptr[g + 1] > X.ptr[g]) {
      s2lNodes.push_back(g);
      oS2l[g] = s2lSrc.ptr.back();
      s2lSrc.ptr.push_back(oS2l[g] + (X.ptr[g + 1] - X.ptr[g]));
    }
  }
  nearSrc.idx.resize((size_t)nearSrc.ptr.back());
  farUE.idx.resize((size_t)farUE.ptr.back());
  s2lSrc.idx.resize((size_t)s2lSrc.ptr.back());
#pragma omp parallel for schedule(static, 1024)
  for (int g = 0; g < nn; g++) {
    if (oNear[g] >= 0) {
      int64_t o = oNear[g], of = oFar[g];
      for (int64_t e = U.ptr[g]; e < U.ptr[g + 1]; e++) nearSrc.idx[o++] = U.idx[e];
      for (int64_t e = W.ptr[g]; e < W.ptr[g + 1]; e++) {
        const int w = W.idx[e];
        if (wDirect(w)) nearSrc.idx[o++] = w;
        else farUE.idx[of++] = w;
      }
      if (xDirect(g))
        for (int64_t e = X.ptr[g]; e < X.ptr[g + 1]; e++) nearSrc.idx[o++] = X.idx[e];
    }
    if (oS2l[g] >= 0) {
      int64_t o = oS2l[g];
      for (int64_t e = X.ptr[g]; e < X.ptr[g + 1]; e++) s2lSrc.idx[o++] = X.idx[e];
    }
  }
  // level lists for the batched equivalent-density GEMMs
  upC2E.assign(maxDepth + 1, {}); upM2M.assign(maxDepth + 1, {}); upLeaf.assign(maxDepth + 1, {});
  dnL2L.assign(maxDepth + 1, {}); dnC2E.assign(maxDepth + 1, {});
  for (int g = 0; g < nn; g++) {
    int d = depth[g];
    if (flags[g] & NF_CBTR) {
      upC2E[d].push_back(g);
      if (!leaf(g)) upM2M[d].push_back(g);
      else upLeaf[d].push_back(g);
    }
    if ((flags[g] & NF_EVTR) && d >= 2) {
      dnC2E[d].push_back(g);
      if (!leaf(g)) dnL2L[d].push_back(g);
    }
  }
  // M2L by parent pairs: V(c) for a child c of P is the set of children of
  // P's same-depth non-leaf neighbours Q that do not touch c
  // (let3d_mpi.cpp:1687-1698); grouping by (P, Q) lets the 8 x 8 child pairs
  // share one pass over Q's spectra.
  vParents.clear(); vNbr.clear(); vNbrOff.clear();
  vSrcSlot.assign(nn, -1); vTrgSlot.assign(nn, -1);
  vSrcNodes.clear(); vTrgNodes.clear();
  // Per level: the 26 same-depth non-leaf neighbours of every non-leaf node
  // (in parallel; the relation is symmetric), the rows (non-leaf parents with
  // an evaluator child and a neighbour) numbered in node order with their
  // target slots, the entries written in parallel, and the source slots in
  // first-seen order: a source parent Q is first seen in the earliest row
  // that lists it -- its earliest row neighbour P, at P's offset code for Q --
  // and its children with sources take the next slots there, child by child.
  std::vector<int32_t> nbrQ, rowOf, keyQ;
  std::vector<int64_t> base;
  for (int d = 1; d < maxDepth; d++) {
    const int l0 = levelBeg[d], l1 = levelBeg[d + 1], nL = l1 - l0;
    nbrQ.assign(27 * (size_t)nL, -1);
#pragma omp parallel for schedule(dynamic, 256)
    for (int P = l0; P < l1; P++) {
      if (leaf(P)) continue;
      const int* pp = &path[3 * (size_t)P];
      const int lim = 1 << d;
      for (int j = 0; j < 27; j++) {  // offset code (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)
        const int dx = j / 9 - 1, dy = (j / 3) % 3 - 1, dz = j % 3 - 1;
        if (!dx && !dy && !dz) continue;
        int q[3] = {pp[0] + dx, pp[1] + dy, pp[2] + dz};
        if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= lim || q[1] >= lim || q[2] >= lim) continue;
        const int Q = find_node(d, q);
        if (depth[Q] == d && !leaf(Q)) nbrQ[27 * (size_t)(P - l0) + j] = Q;
      }
    }
    // rows in node order
    rowOf.assign(nL, -1);
    base.assign(nL, 0);
    const size_t row0 = vParents.size();
    for (int P = l0; P < l1; P++) {
      if (leaf(P)) continue;
      bool anyE = false;
      for (int c = 0; c < 8; c++) anyE = anyE || (flags[chd[P] + c] & NF_EVTR);
      if (!anyE) continue;
      int n = 0;
      for (int j = 0; j < 27; j++) n += nbrQ[27 * (size_t)(P - l0) + j] >= 0 ? 1 : 0;
      if (n == 0) continue;
      rowOf[P - l0] = (int32_t)(vParents.size() - row0);
      base[P - l0] = (int64_t)vNbr.idx.size();
      vParents.push_back(P);
      vNbr.idx.resize(vNbr.idx.size() + n);
      vNbr.ptr.push_back((int64_t)vNbr.idx.size());
      for (int c = 0; c < 8; c++) {
        const int t = chd[P] + c;
        if ((flags[t] & NF_EVTR) && vTrgSlot[t] < 0) {
          vTrgSlot[t] = (int32_t)vTrgNodes.size();
          vTrgNodes.push_back(t);
        }
      }
    }
    const int nRows = (int)(vParents.size() - row0);
    vNbrOff.resize(vNbr.idx.size());
    keyQ.assign(27 * (size_t)nRows, -1);
#pragma omp parallel for schedule(dynamic, 256)
    for (int X = l0; X < l1; X++) {
      const int32_t* nb = &nbrQ[27 * (size_t)(X - l0)];
      if (rowOf[X - l0] >= 0) {  // X as a row: its entries
        int64_t o = base[X - l0];
        for (int j = 0; j < 27; j++)
          if (nb[j] >= 0) {
            vNbr.idx[o] = nb[j];
            vNbrOff[o++] = (int8_t)j;
          }
      }
      // X as a source parent: its earliest row neighbour P, which lists X at
      // the opposite offset
      int best = -1;
      for (int j = 0; j < 27; j++) {
        const int P = nb[j];
        if (P < 0 || rowOf[P - l0] < 0) continue;
        const int k = rowOf[P - l0] * 27 + (26 - j);
        if (best < 0 || k < best) best = k;
      }
      if (best >= 0) keyQ[best] = X;
    }
    for (size_t k = 0; k < keyQ.size(); k++) {
      const int Q = keyQ[k];
      if (Q < 0) continue;
      for (int c = 0; c < 8; c++) {
        const int v = chd[Q] + c;
        if ((flags[v] & NF_CBTR) && vSrcSlot[v] < 0) {
          vSrcSlot[v] = (int32_t)vSrcNodes.size();
          vSrcNodes.push_back(v);
        }
      }
    }
  }
  auto slots8 = [&](const std::vector<int32_t>& nodes, const std::vector<int32_t>& slot, std::vector<int32_t>& out) {
    out.resize(8 * nodes.size());
#pragma omp parallel for schedule(static, 4096)
    for (size_t i = 0; i < nodes.size(); i++)
      for (int c = 0; c < 8; c++) out[8 * i + c] = slot[chd[nodes[i]] + c];
  };
  slots8(vParents, vTrgSlot, vRowOut);
  slots8(vNbr.idx, vSrcSlot, vNbrIn);
}

// Expanded per-target lists: v = child c2 of Q, c = child of P, idx = v - c.
// A target slot is one child c of one row P, so the slots are counted, then
// filled, row by row in parallel; each keeps its entries neighbour by
// neighbour, child by child.
void Plan::expand_v_lists() const {
  if (vExpanded) return;
  const size_t nTrgSlots = vTrgNodes.size(), nSrcSlots = vSrcNodes.size();
  auto expand = [&](size_t r, int c, auto&& emit) {
    for (int64_t e = vNbr.ptr[r]; e < vNbr.ptr[r + 1]; e++) {
      const int Q = vNbr.idx[e], off = vNbrOff[e];
      const int dx = off / 9 - 1, dy = (off / 3) % 3 - 1, dz = off % 3 - 1;
      for (int c2 = 0; c2 < 8; c2++) {
        const int s = vSrcSlot[chd[Q] + c2];
        if (s < 0) continue;
        const int rx = 2 * dx + (c2 >> 2) - (c >> 2), ry = 2 * dy + ((c2 >> 1) & 1) - ((c >> 1) & 1),
                  rz = 2 * dz + (c2 & 1) - (c & 1);
        if (std::max(std::abs(rx), std::max(std::abs(ry), std::abs(rz))) <= 1) continue;
        emit(s, transId[rx + 3][ry + 3][rz + 3]);
      }
    }
  };
  vTrgPtr.assign(nTrgSlots + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t r = 0; r < vParents.size(); r++)
    for (int c = 0; c < 8; c++) {
      const int ts = vTrgSlot[chd[vParents[r]] + c];
      if (ts < 0) continue;
      int64_t n = 0;
      expand(r, c, [&](int, int) { n++; });
      vTrgPtr[ts + 1] = n;
    }
  for (size_t t = 0; t < nTrgSlots; t++) vTrgPtr[t + 1] += vTrgPtr[t];
  vTrgEnt.resize(2 * (size_t)vTrgPtr[nTrgSlots]);
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t r = 0; r < vParents.size(); r++)
    for (int c = 0; c < 8; c++) {
      const int ts = vTrgSlot[chd[vParents[r]] + c];
      if (ts < 0) continue;
      int64_t o = vTrgPtr[ts];
      expand(r, c, [&](int s, int id) {
        vTrgEnt[2 * o] = s;
        vTrgEnt[2 * o + 1] = id;
        o++;
      });
    }
  // inverted per source slot, in the order of the target-slot lists: a stable
  // counting sort over chunks of target slots, each chunk placing its entries
  // after the earlier chunks' entries of the same source slot
  const int64_t nEnt = vTrgPtr[nTrgSlots];
  const int T = std::max(1, omp_get_max_threads());
  const size_t tchunk = (nTrgSlots + T - 1) / T;
  std::vector<int64_t> pos((size_t)T * nSrcSlots, 0);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < T; t++) {
    int64_t* pc = &pos[(size_t)t * nSrcSlots];
    for (size_t ts = t * tchunk; ts < std::min(nTrgSlots, (t + 1) * tchunk); ts++)
      for (int64_t i = vTrgPtr[ts]; i < vTrgPtr[ts + 1]; i++) pc[vTrgEnt[2 * i]]++;
  }
  vSrcPtr.assign(nSrcSlots + 1, 0);
  int64_t at = 0;
  for (size_t sl = 0; sl < nSrcSlots; sl++) {
    vSrcPtr[sl] = at;
    for (int t = 0; t < T; t++) {
      const int64_t n = pos[(size_t)t * nSrcSlots + sl];
      pos[(size_t)t * nSrcSlots + sl] = at;
      at += n;
    }
  }
  vSrcPtr[nSrcSlots] = at;
  vSrcEnt.resize(2 * (size_t)nEnt);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < T; t++) {
    int64_t* pc = &pos[(size_t)t * nSrcSlots];
    for (size_t ts = t * tchunk; ts < std::min(nTrgSlots, (t + 1) * tchunk); ts++)
      for (int64_t i = vTrgPtr[ts]; i < vTrgPtr[ts + 1]; i++) {
        const int64_t o = pc[vTrgEnt[2 * i]]++;
        vSrcEnt[2 * o] = (int32_t)ts;
        vSrcEnt[2 * o + 1] = vTrgEnt[2 * i + 1];
      }
  }
  vExpanded = true;
}

// Inverse of a CSR (rows -> column ids): for every id that occurs, the rows
// (given by their own node ids) that list it, in increasing row order.
static void invert_csr(const std::vector<int32_t>& rows, const CSR& L, int nn, std::vector<int32_t>& outRows,
                       CSR& out) {
  std::vector<int64_t> cnt(nn + 1, 0);
  for (int32_t v : L.idx) cnt[v + 1]++;
  for (int i = 0; i < nn; i++) cnt[i + 1] += cnt[i];
  std::vector<int32_t> tmp(L.idx.size());
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (size_t r = 0; r < rows.size(); r++)
    for (int64_t e = L.ptr[r]; e < L.ptr[r + 1]; e++) tmp[fill[L.idx[e]]++] = rows[r];
  outRows.clear();
  out.clear();
  for (int v = 0; v < nn; v++) {
    if (cnt[v + 1] == cnt[v]) continue;
    outRows.push_back(v);
    out.idx.insert(out.idx.end(), tmp.begin() + cnt[v], tmp.begin() + cnt[v + 1]);
    out.ptr.push_back((int64_t)out.idx.size());
  }
}

// The transposed FMM runs every forward stage backwards: its direct sums go
// from the forward targets to the forward sources, so each forward work list
// is needed grouped by its other end.
void Plan::build_adjoint_lists() const {
  if (adjBuilt) return;
  invert_csr(evtrLeaves, nearSrc, nn, adjNearRows, adjNear);
  invert_csr(farLeaves, farUE, nn, adjFarRows, adjFar);
  invert_csr(s2lNodes, s2lSrc, nn, adjS2lRows, adjS2l);
  // grouped M2L: (P, Q, d) -> (Q, P, -d)
  std::vector<std::vector<std::pair<int32_t, int8_t>>> byQ(nn);
  for (size_t r = 0; r < vParents.size(); r++)
    for (int64_t e = vNbr.ptr[r]; e < vNbr.ptr[r + 1]; e++) {
      int off = vNbrOff[e];
      int dx = off / 9 - 1, dy = (off / 3) % 3 - 1, dz = off % 3 - 1;
      byQ[vNbr.idx[e]].push_back({vParents[r], (int8_t)((-dx + 1) * 9 + (-dy + 1) * 3 + (-dz + 1))});
    }
  vParentsT.clear();
  vNbrT.clear();
  vNbrOffT.clear();
  for (int q = 0; q < nn; q++) {
    if (byQ[q].empty()) continue;
    vParentsT.push_back(q);
    for (auto& pr : byQ[q]) {
      vNbrT.idx.push_back(pr.first);
      vNbrOffT.push_back(pr.second);
    }
    vNbrT.ptr.push_back((int64_t)vNbrT.idx.size());
  }
  auto slots8 = [&](const std::vector<int32_t>& nodes, const std::vector<int32_t>& slot, std::vector<int32_t>& out) {
    out.resize(8 * nodes.size());
    for (size_t i = 0; i < nodes.size(); i++)
      for (int c = 0; c < 8; c++) out[8 * i + c] = slot[chd[nodes[i]] + c];
  };
  slots8(vParentsT, vSrcSlot, vRowOutT);
  slots8(vNbrT.idx, vTrgSlot, vNbrInT);
  adjBuilt = true;
}

std::string Plan::build(const Options& opt, int64_t ns_, const double* src, const double* nrmIn, int64_t nt_,
                        const double* trg, int treeDevice) {
  o = opt;
  ns = ns_; nt = nt_;
  using Clock = std::chrono::steady_clock;
  auto t0 = Clock::now();
  auto lap = [&](int i) {
    const auto t1 = Clock::now();
    buildMs[i] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    t0 = t1;
  };
  // targets that are the sources repeat the sources' partition exactly
  const bool trgIsSrc = trg == src && nt == ns;
  if (treeDevice >= 0) {
    std::string e = tree_build_device(treeDevice, *this, src, trg, trgIsSrc);
    if (!e.empty()) return e;
    lap(0);
  } else {
    build_tree(src);
    lap(0);
    if (trgIsSrc) {
      trgBeg = srcBeg;
      trgCnt = srcCnt;
      trgPerm = srcPerm;
    } else {
      bin_targets(trg);
    }
  }
  lap(1);
  flags.assign(nn, 0);
  center.resize(3 * (size_t)nn);
  radius.resize(nn);
  const double R0 = std::pow(2.0, -o.rootLevel);
#pragma omp parallel for schedule(static, 2048)
  for (int n = 0; n < nn; n++) {
    uint8_t f = 0;
    bool lf = chd[n] < 0;
    if (lf) f |= NF_LEAF;
    if (n != 0 && srcCnt[n] > 0) f |= NF_CBTR;
    if (n != 0 && (!lf || srcCnt[n] > 0)) f |= NF_SRCE;
    if (lf && srcCnt[n] > 0) f |= NF_LSRC;
    if (trgCnt[n] > 0) f |= NF_EVTR;
    flags[n] = f;
    node_center(depth[n], &path[3 * (size_t)n], &center[3 * (size_t)n]);
    radius[n] = R0 / double(1 << depth[n]);  // let3d_mpi.cpp:1824-1827
  }
  lap(2);
  if (treeDevice >= 0) {
    std::string e = lists_build_device(treeDevice, *this);
    if (!e.empty()) return e;
  } else {
    build_lists();
  }
  lap(3);
  build_worklists();
  lap(4);
  // the expanded V lists and the adjoint's lists wait for their first use
  vExpanded = adjBuilt = false;
  vTrgPtr.clear(); vTrgEnt.clear(); vSrcPtr.clear(); vSrcEnt.clear();
  lap(5);
  (void)nrmIn;
  return std::string();
}

// ------------------------------------------------------------------ operators
static void sam_pos(int np, double R, std::vector<double>& pos) {  // matmgnt3d_mpi.cpp:451-475
  pos.clear();
  double step = 2.0 / (np - 1);
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++)
      for (int k = 0; k < np; k++)
        if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
          pos.push_back(R * (-1.0 + i * step));
          pos.push_back(R * (-1.0 + j * step));
          pos.push_back(R * (-1.0 + k * step));
        }
}

// column-major kernel matrix (nt*TD) x (ns*SD) of the equivalent kernel
template <int KT>
static void mm_matrix(const double* coefs, int ns, const double* sp, int nt, const double* tp,
                      std::vector<double>& out) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  const int64_t m = (int64_t)nt * TD;
  out.assign((size_t)m * ns * SD, 0.0);
  double K[16];
  for (int j = 0; j < ns; j++)
    for (int i = 0; i < nt; i++) {
      double x = tp[3 * i] - sp[3 * j], y = tp[3 * i + 1] - sp[3 * j + 1], z = tp[3 * i + 2] - sp[3 * j + 2];
      if (!kblock<KT, double>(x, y, z, sp + 3 * j, K, coefs[0], coefs[1])) continue;
      for (int t = 0; t < TD; t++)
        for (int s = 0; s < SD; s++) out[(size_t)(j * SD + s) * m + i * TD + t] = K[t * SD + s];
    }
}

static void mm_matrix_rt(int kt, const double* coefs, int ns, const double* sp, int nt, const double* tp,
                         std::vector<double>& out) {
  switch (kt) {
    case LAP_S_U: mm_matrix<LAP_S_U>(coefs, ns, sp, nt, tp, out); break;
    case STK_F_U: mm_matrix<STK_F_U>(coefs, ns, sp, nt, tp, out); break;
    case NAV_S_U: mm_matrix<NAV_S_U>(coefs, ns, sp, nt, tp, out); break;
  }
}

// The operator tables depend on the kernel, its two coefficients and np only.
// The process keeps the most recent sets, so that new handles and repeated
// setups of one handle (points that move between evaluations) copy them
// instead of rebuilding them, as the reference shares one operator manager per
// kernel and order among its FMM objects (fmm3d_mpi/matmgnt3d_mpi.cpp:526-543).
namespace {
struct OpKey {
  int kt, np;
  double c0, c1;
  bool operator==(const OpKey& b) const { return kt == b.kt && np == b.np && c0 == b.c0 && c1 == b.c1; }
};
constexpr size_t kOperatorSetsKept = 4;
std::mutex gOpMu;
std::list<std::pair<OpKey, std::shared_ptr<const Plan>>> gOps;  // most recent first
}  // namespace

std::string Plan::build_operators() {
  const OpKey key{o.kt, o.np, o.coefs[0], o.coefs[1]};
  std::shared_ptr<const Plan> set;
  {
    std::lock_guard<std::mutex> g(gOpMu);
    for (auto it = gOps.begin(); it != gOps.end(); ++it)
      if (it->first == key) {
        set = it->second;
        gOps.splice(gOps.begin(), gOps, it);
        break;
      }
  }
  if (!set) {
    auto fresh = std::make_shared<Plan>();
    fresh->o = o;
    std::string e = fresh->build_operators_uncached();
    if (!e.empty()) return e;
    std::lock_guard<std::mutex> g(gOpMu);
    gOps.emplace_front(key, fresh);
    if (gOps.size() > kOperatorSetsKept) gOps.pop_back();
    set = fresh;
  }
  assign_operators(*set);
  return std::string();
}

// Every member build_operators sets: copied from a const set, moved from an
// rvalue one.
template <class S> void Plan::assign_operators(S&& s) {
  sd = s.sd; td = s.td; mm = s.mm; sdm = s.sdm; tdm = s.tdm;
  std::memcpy(deg, s.deg, sizeof(deg));
  nrm = s.nrm;
  nUE = s.nUE; nUC = s.nUC; nDE = s.nDE; nDC = s.nDC; nReg = s.nReg; nEff = s.nEff;
  nReg32 = s.nReg32; nEff32 = s.nEff32;
  for (int i = 0; i < 4; i++) sam[i] = std::forward<S>(s).sam[i];
  uc2ue = std::forward<S>(s).uc2ue; m2m = std::forward<S>(s).m2m;
  dc2de = std::forward<S>(s).dc2de; l2l = std::forward<S>(s).l2l;
  m2lT = std::forward<S>(s).m2lT; m2lT32 = std::forward<S>(s).m2lT32;
  kUp = s.kUp; kDn = s.kDn;
  uc2ueF1 = std::forward<S>(s).uc2ueF1; uc2ueF2 = std::forward<S>(s).uc2ueF2;
  dc2deF1 = std::forward<S>(s).dc2deF1; dc2deF2 = std::forward<S>(s).dc2deF2;
  std::memcpy(transId, s.transId, sizeof(transId));
  upFold = std::forward<S>(s).upFold;
  std::memcpy(opsMs, s.opsMs, sizeof(opsMs));
}

const std::vector<double>& Plan::folded_upward() const {
  if (upFold.empty()) upFold = fold_c2e_m2m(*this);
  return upFold;
}

void Plan::take_operators(Plan&& s) { assign_operators(std::move(s)); }

// The operator set of MatMgnt3d_MPI (fmm3d_mpi/matmgnt3d_mpi.cpp:52-71,
// 107-274, 373-411) for a homogeneous equivalent kernel: unit-radius tables,
// level scaling 2^(+-l*deg) applied by the GPU stages.
std::string Plan::build_operators_uncached() {
  sd = kernel_src_dof(o.kt);
  td = kernel_trg_dof(o.kt);
  mm = kernel_mm(o.kt);
  if (mm < 0 || sd == 0) return "unsupported kernel type";
  sdm = kernel_src_dof(mm);
  tdm = kernel_trg_dof(mm);
  nrm = kernel_has_normal(o.kt);
  kernel_hom_deg(mm, deg);
  const int np = o.np;
  sam_pos(np, 1.0, sam[0]);
  sam_pos(np + 2, 3.0, sam[1]);
  sam_pos(np, 3.0, sam[2]);
  sam_pos(np, 1.0, sam[3]);
  nUE = (int)sam[0].size() / 3; nUC = (int)sam[1].size() / 3;
  nDE = (int)sam[2].size() / 3; nDC = (int)sam[3].size() / 3;
  const int n = 2 * np;
  nReg = n * n * n;
  nEff = n * n * (n / 2 + 1);
  {
    const int n32 = 2 * np - 1;
    nReg32 = n32 * n32 * n32;
    nEff32 = n32 * n32 * (n32 / 2 + 1);
  }
  const double eps = std::pow(0.1, np + 1);  // matmgnt3d_mpi.cpp:37-40
  const int ue = nUE * sdm, uc = nUC * tdm, de = nDE * sdm, dc = nDC * tdm;
  using Clock = std::chrono::steady_clock;
  auto t0 = Clock::now();
  auto lap = [&](int i) {
    const auto t1 = Clock::now();
    opsMs[i] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    t0 = t1;
  };
  std::vector<double> A, Rm;
  // C2E up: pinv of the UE -> UC matrix
  mm_matrix_rt(mm, o.coefs, nUE, sam[0].data(), nUC, sam[1].data(), A);
  Rm.assign((size_t)ue * uc, 0.0);
  kUp = pinv_truncated(uc, ue, A.data(), eps, Rm.data(), uc2ueF1, uc2ueF2);
  uc2ue.resize((size_t)ue * uc);
  for (int r = 0; r < ue; r++)
    for (int c = 0; c < uc; c++) uc2ue[(size_t)r * uc + c] = Rm[(size_t)c * ue + r];
  lap(0);
  // C2E down
  mm_matrix_rt(mm, o.coefs, nDE, sam[2].data(), nDC, sam[3].data(), A);
  Rm.assign((size_t)de * dc, 0.0);
  kDn = pinv_truncated(dc, de, A.data(), eps, Rm.data(), dc2deF1, dc2deF2);
  dc2de.resize((size_t)de * dc);
  for (int r = 0; r < de; r++)
    for (int c = 0; c < dc; c++) dc2de[(size_t)r * dc + c] = Rm[(size_t)c * de + r];
  lap(1);
  // (refactor_c2e recovers these factors from the explicit tables)
  // M2M / L2L octant matrices
  m2m.assign((size_t)uc * 8 * ue, 0.0);
  l2l.assign((size_t)8 * dc * de, 0.0);
  for (int oc = 0; oc < 8; oc++) {
    int id[3] = {oc >> 2, (oc >> 1) & 1, oc & 1};
    std::vector<double> chk(3 * (size_t)nUC), den(3 * (size_t)nUE);
    for (int j = 0; j < nUC; j++)
      for (int k = 0; k < 3; k++) chk[3 * j + k] = 2.0 * sam[1][3 * j + k];
    for (int j = 0; j < nUE; j++)
      for (int k = 0; k < 3; k++) den[3 * j + k] = sam[0][3 * j + k] + (2 * id[k] - 1) * 1.0;
    mm_matrix_rt(mm, o.coefs, nUE, den.data(), nUC, chk.data(), A);  // uc x ue, col-major
    for (int r = 0; r < uc; r++)
      for (int c = 0; c < ue; c++) m2m[(size_t)r * 8 * ue + oc * ue + c] = A[(size_t)c * uc + r];
    std::vector<double> chk2(3 * (size_t)nDC), den2(sam[2]);
    for (int j = 0; j < nDC; j++)
      for (int k = 0; k < 3; k++) chk2[3 * j + k] = 0.5 * sam[3][3 * j + k] + (double(id[k]) - 0.5) * 1.0;
    mm_matrix_rt(mm, o.coefs, nDE, den2.data(), nDC, chk2.data(), A);  // dc x de
    for (int r = 0; r < dc; r++)
      for (int c = 0; c < de; c++) l2l[((size_t)oc * dc + r) * de + c] = A[(size_t)c * dc + r];
  }
  lap(2);
  // M2L translation spectra: the kernel from a point at 2*idx sampled on the
  // (2np)^3 regular grid, r2c transformed (matmgnt3d_mpi.cpp:385-411)
  int cnt = 0;
  for (int i1 = -3; i1 <= 3; i1++)
    for (int i2 = -3; i2 <= 3; i2++)
      for (int i3 = -3; i3 <= 3; i3++)
        transId[i1 + 3][i2 + 3][i3 + 3] =
            (std::abs(i1) > 1 || std::abs(i2) > 1 || std::abs(i3) > 1) ? cnt++ : -1;
  // the translations sampled on the n^3 regular grid (offsets
  // (i < np ? i : i - n) steps per axis), r2c transformed
  const int mdof = sdm * tdm;
  auto spectra = [&](int n_, int nEff_, std::vector<std::complex<double>>& out) {
    const int nReg_ = n_ * n_ * n_;
    std::vector<double> reg(3 * (size_t)nReg_);
    double step = 2.0 / (np - 1);
    size_t c = 0;
    for (int k = 0; k < n_; k++)
      for (int j = 0; j < n_; j++)
        for (int i = 0; i < n_; i++, c++) {
          reg[3 * c + 0] = (i < np ? i : i - n_) * step;
          reg[3 * c + 1] = (j < np ? j : j - n_) * step;
          reg[3 * c + 2] = (k < np ? k : k - n_) * step;
        }
    out.assign((size_t)316 * nEff_ * mdof, std::complex<double>(0, 0));
#pragma omp parallel for schedule(dynamic, 2)
    for (int t = 0; t < 343; t++) {
      int i1 = t / 49 - 3, i2 = (t / 7) % 7 - 3, i3 = t % 7 - 3;
      int id = transId[i1 + 3][i2 + 3][i3 + 3];
      if (id < 0) continue;
      double sp[3] = {i1 * 2.0, i2 * 2.0, i3 * 2.0};
      std::vector<double> tt;
      mm_matrix_rt(mm, o.coefs, 1, sp, nReg_, reg.data(), tt);  // (nReg*tdm) x sdm
      std::vector<double> grid((size_t)nReg_ * mdof);
      for (int k = 0; k < nReg_; k++)
        for (int i = 0; i < tdm; i++)
          for (int j = 0; j < sdm; j++)
            grid[(size_t)k * mdof + j * tdm + i] = tt[(size_t)j * nReg_ * tdm + i + (size_t)k * tdm];
      rfft3_host(n_, mdof, grid.data(), &out[(size_t)id * nEff_ * mdof]);
    }
  };
  spectra(n, nEff, m2lT);
  spectra(2 * np - 1, nEff32, m2lT32);
  lap(3);
  return std::string();
}

void Plan::refactor_c2e(int which) {
  // the kept singular values of a truncated pinv span at most 1/eps; the
  // dropped ones are rounding noise
  const double cut = 1e-13;
  if (which == 0)
    kUp = svd_factors(nUE * sdm, nUC * tdm, uc2ue.data(), cut, uc2ueF1, uc2ueF2);
  else if (which == 2)
    kDn = svd_factors(nDE * sdm, nDC * tdm, dc2de.data(), cut, dc2deF1, dc2deF2);
}

void Plan::m2l_spectrum32(int id) {
  typedef std::complex<double> C;
  const int n = 2 * o.np, m = 2 * o.np - 1, nh = n / 2 + 1, mdof = sdm * tdm;
  const C* X = &m2lT[(size_t)id * nEff * mdof];
  std::vector<C> w(n);
  for (int j = 0; j < n; j++) w[j] = C(std::cos(2.0 * M_PI * j / n), std::sin(2.0 * M_PI * j / n));
  // z and y complex inverse transforms: B[z][y][kx][h]
  std::vector<C> A((size_t)n * n * nh * mdof), B((size_t)n * n * nh * mdof);
  for (int z = 0; z < n; z++)
    for (int ky = 0; ky < n; ky++)
      for (int kx = 0; kx < nh; kx++)
        for (int h = 0; h < mdof; h++) {
          C s(0, 0);
          for (int kz = 0; kz < n; kz++) s += X[(((size_t)kz * n + ky) * nh + kx) * mdof + h] * w[(kz * z) % n];
          A[(((size_t)z * n + ky) * nh + kx) * mdof + h] = s;
        }
  for (int z = 0; z < n; z++)
    for (int y = 0; y < n; y++)
      for (int kx = 0; kx < nh; kx++)
        for (int h = 0; h < mdof; h++) {
          C s(0, 0);
          for (int ky = 0; ky < n; ky++) s += A[(((size_t)z * n + ky) * nh + kx) * mdof + h] * w[(ky * y) % n];
          B[(((size_t)z * n + y) * nh + kx) * mdof + h] = s;
        }
  // x c2r at the offsets the odd grid keeps, written into the m^3 grid
  std::vector<double> grid((size_t)m * m * m * mdof);
  auto src = [&](int i) { return i < o.np ? i : i - m + n; };  // odd-grid index -> even-grid index
  const double scale = 1.0 / ((double)n * n * n);
  for (int z = 0; z < m; z++)
    for (int y = 0; y < m; y++)
      for (int x = 0; x < m; x++)
        for (int h = 0; h < mdof; h++) {
          const int zz = src(z), yy = src(y), xx = src(x);
          double s = 0;
          for (int kx = 0; kx < nh; kx++) {
            const C v = B[(((size_t)zz * n + yy) * nh + kx) * mdof + h] * w[(kx * xx) % n];
            s += (kx == 0 || kx == n / 2 ? 1.0 : 2.0) * v.real();
          }
          grid[(((size_t)z * m + y) * m + x) * mdof + h] = s * scale;
        }
  rfft3_host(m, mdof, grid.data(), &m2lT32[(size_t)id * nEff32 * mdof]);
}

}  // namespace fmmg
