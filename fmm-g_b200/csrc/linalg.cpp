// linalg.cpp -- dense linear algebra for the operator builder (setup only).
//
// pinv_truncated: the truncated pseudo-inverse of common/vecmatop.cpp:129-164
// (common/svdrep.cpp:38-80 keeps the singular values >= eps * s_max), computed
// from a one-sided Jacobi SVD, which is accurate in the small singular values
// that the truncation tests (LAPACK dgesvd, which the reference calls, is not
// installed here).  rfft3_host: the r2c transform with FFTW's rank-3
// layout used for the M2L translation tables (fmm3d_mpi/matmgnt3d_mpi.cpp:408).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "plan.hpp"

namespace fmmg {

// The device that builds the operator tables on this thread (-1: the host).
// linalg_gpu.cu repeats the host arithmetic exactly, so the tables do not
// depend on the choice.
static thread_local int tl_linalgDevice = -1;
void set_linalg_device(int device) { tl_linalgDevice = device; }
std::string svd_onesided_device(int device, int m, int n, std::vector<double>& Z);
std::string gemm_rows_device(int device, int rows, int inner, int w, const double* A, const double* B, double* C);

// sqrt(1 + z^2), the Jacobi rotation's hypot(1, z): 1 + z^2 rounds to z^2
// long before z^2 overflows, where the root is |z|
static inline double jacobi_hyp1(double z) {
  const double az = std::fabs(z);
  return az > 1e100 ? az : std::sqrt(1.0 + z * z);
}

// The three dot products of a column pair in the order the GPU forms them:
// 32 partial sums over the rows i = l (mod 32), each in increasing i, then
// combined pairwise as a butterfly over offsets 16, 8, 4, 2, 1 (every lane of
// a warp ends with the same value; IEEE addition is commutative).
static void jacobi_dots32(const double* p, const double* q, int m, double& a, double& b, double& g) {
  double pa[32], pb[32], pg[32];
  for (int l = 0; l < 32; l++) pa[l] = pb[l] = pg[l] = 0.0;
  for (int i = 0; i < m; i++) {
    const int l = i & 31;
    pa[l] += p[i] * p[i];
    pb[l] += q[i] * q[i];
    pg[l] += p[i] * q[i];
  }
  for (int off = 16; off > 0; off >>= 1) {
    double ta[32], tb[32], tg[32];
    for (int l = 0; l < 32; l++) {
      ta[l] = pa[l] + pa[l ^ off];
      tb[l] = pb[l] + pb[l ^ off];
      tg[l] = pg[l] + pg[l ^ off];
    }
    for (int l = 0; l < 32; l++) {
      pa[l] = ta[l];
      pb[l] = tb[l];
      pg[l] = tg[l];
    }
  }
  a = pa[0];
  b = pb[0];
  g = pg[0];
}

// A is m x n column-major with m >= n after an optional transpose.  Columns
// are orthogonalised pairwise in tournament order (n/2 disjoint pairs per
// round, so rounds parallelise and the result is thread-count independent).
// Each column of V is kept right below its column of W, so one pass applies a
// rotation to both.
static void svd_onesided(int m, int n, std::vector<double>& W /* m x n, becomes U*S */,
                         std::vector<double>& V /* n x n */) {
  const size_t ld = (size_t)m + n;
  std::vector<double> Z(ld * n, 0.0);  // column j: W_j (m) then V_j (n), V = I
  for (int j = 0; j < n; j++) {
    std::copy(W.begin() + (size_t)j * m, W.begin() + (size_t)(j + 1) * m, Z.begin() + j * ld);
    Z[j * ld + m + j] = 1.0;
  }
  bool onDevice = false;
  if (tl_linalgDevice >= 0 && n >= 64) {  // on a copy: a failed device run leaves Z for the host loop
    std::vector<double> Zd(Z);
    onDevice = svd_onesided_device(tl_linalgDevice, m, n, Zd).empty();
    if (onDevice) Z.swap(Zd);
  }
  const int nn = n + (n & 1);
  std::vector<int> top(nn / 2), bot(nn / 2);
  for (int i = 0; i < nn / 2; i++) { top[i] = 2 * i; bot[i] = 2 * i + 1; }
  for (int sweep = 0; sweep < (onDevice ? 0 : 80); sweep++) {
    int rotated = 0;
    for (int round = 0; round < nn - 1; round++) {
      // two pairs per iteration: their dot products share one loop (six
      // independent sums hide the add latency; each pair sums in its own order)
      const int npair = nn / 2;
#pragma omp parallel for schedule(static) reduction(+ : rotated)
      for (int k2 = 0; k2 < (npair + 1) / 2; k2++) {
        double* zp[2] = {nullptr, nullptr};
        double* zq[2] = {nullptr, nullptr};
        for (int h = 0; h < 2; h++) {
          const int k = 2 * k2 + h;
          if (k >= npair) break;
          int p = std::min(top[k], bot[k]), q = std::max(top[k], bot[k]);
          if (q >= n) continue;
          zp[h] = &Z[p * ld];
          zq[h] = &Z[q * ld];
        }
        double a[2] = {0, 0}, b[2] = {0, 0}, g[2] = {0, 0};
        for (int h = 0; h < 2; h++)
          if (zp[h]) jacobi_dots32(zp[h], zq[h], m, a[h], b[h], g[h]);
        for (int h = 0; h < 2; h++) {
          if (!zp[h]) continue;
          if (a[h] == 0.0 || b[h] == 0.0) continue;
          if (std::fabs(g[h]) <= 1e-15 * std::sqrt(a[h] * b[h])) continue;
          rotated++;
          double zeta = (b[h] - a[h]) / (2.0 * g[h]);
          double t = std::copysign(1.0, zeta) / (std::fabs(zeta) + jacobi_hyp1(zeta));
          double c = 1.0 / jacobi_hyp1(t), s = c * t;
          double *zph = zp[h], *zqh = zq[h];
#pragma omp simd
          for (size_t i = 0; i < ld; i++) {  // element-wise: the same arithmetic vectorised
            double x = zph[i], y = zqh[i];
            zph[i] = c * x - s * y;
            zqh[i] = s * x + c * y;
          }
        }
      }
      // tournament rotation (player 0 stays)
      if (nn / 2 > 1) {
        int tlast = top[nn / 2 - 1], b0 = bot[0];
        for (int i = nn / 2 - 1; i > 1; i--) top[i] = top[i - 1];
        top[1] = b0;
        for (int i = 0; i < nn / 2 - 1; i++) bot[i] = bot[i + 1];
        bot[nn / 2 - 1] = tlast;
      }
    }
    if (!rotated) break;
  }
  V.resize((size_t)n * n);
  for (int j = 0; j < n; j++) {
    std::copy(Z.begin() + j * ld, Z.begin() + j * ld + m, W.begin() + (size_t)j * m);
    std::copy(Z.begin() + j * ld + m, Z.begin() + (j + 1) * ld, V.begin() + (size_t)j * n);
  }
}

// One SVD gives both forms: the explicit table R (n x m column-major, skipped
// when R is NULL) and the factors F1 = diag(1/s_k) U_k^T (k x m, row-major)
// and F2 = V_k (n x k, row-major).  Applying F1 then F2 keeps the rounding
// error of each factor relative to the size of its own result, which a single
// product with the large-norm explicit pinv does not (used by the FP32 path).
int pinv_truncated(int m, int n, const double* A, double eps, double* R, std::vector<double>& F1,
                   std::vector<double>& F2) {
  bool tr = m < n;
  int M = tr ? n : m, N = tr ? m : n;
  std::vector<double> W((size_t)M * N), V;
  if (!tr) std::memcpy(W.data(), A, sizeof(double) * M * N);
  else
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) W[(size_t)i * n + j] = A[(size_t)j * m + i];
  svd_onesided(M, N, W, V);
  std::vector<double> S(N);
  for (int j = 0; j < N; j++) {
    double s = 0;
    for (int i = 0; i < M; i++) s += W[(size_t)j * M + i] * W[(size_t)j * M + i];
    S[j] = std::sqrt(s);
  }
  double smax = *std::max_element(S.begin(), S.end());
  double cutoff = eps * smax;
  bool rDone = false;
  if (R && tl_linalgDevice >= 0) {
    // the same sums on the device: R(i, j) = sum over kept c, in order, of
    // a_c(i) * (b_c(j) / s_c^2), one rounding per product and per sum
    std::vector<int> cs;
    for (int c = 0; c < N; c++)
      if (S[c] >= cutoff && S[c] != 0.0) cs.push_back(c);
    const int K = (int)cs.size();
    std::vector<double> Ad((size_t)n * K), Bd((size_t)K * m), Cd((size_t)n * m, 0.0);
    for (int r = 0; r < K; r++) {
      const int c = cs[r];
      const double inv2 = 1.0 / (S[c] * S[c]);
      const double* w = &W[(size_t)c * M];
      const double* v = &V[(size_t)c * N];
      const double* a = tr ? w : v;  // length n
      const double* b = tr ? v : w;  // length m
      for (int i = 0; i < n; i++) Ad[(size_t)i * K + r] = a[i];
      for (int j = 0; j < m; j++) Bd[(size_t)r * m + j] = b[j] * inv2;
    }
    if (gemm_rows_device(tl_linalgDevice, n, K, m, Ad.data(), Bd.data(), Cd.data()).empty()) {
      for (int j = 0; j < m; j++)
        for (int i = 0; i < n; i++) R[(size_t)j * n + i] = Cd[(size_t)i * m + j];
      rDone = true;
    }
  }
  if (R && !rDone) {
    std::fill(R, R + (size_t)n * m, 0.0);
    // For A = W V^T with W = U S: pinv(A) = V S^-2 W^T restricted to kept columns.
    for (int c = 0; c < N; c++) {
      if (!(S[c] >= cutoff) || S[c] == 0.0) continue;
      double inv2 = 1.0 / (S[c] * S[c]);
      const double* w = &W[(size_t)c * M];
      const double* v = &V[(size_t)c * N];
      if (!tr) {  // R(i, j) += v_i w_j / s^2, R is n x m
        for (int j = 0; j < m; j++) {
          double f = w[j] * inv2;
          double* r = R + (size_t)j * n;
          for (int i = 0; i < n; i++) r[i] += v[i] * f;
        }
      } else {  // A^T = W V^T  ->  pinv(A) = W S^-2 V^T : R(i, j) += w_i v_j / s^2
        for (int j = 0; j < m; j++) {
          double f = v[j] * inv2;
          double* r = R + (size_t)j * n;
          for (int i = 0; i < n; i++) r[i] += w[i] * f;
        }
      }
    }
  }
  std::vector<int> keep;
  for (int c = 0; c < N; c++)
    if (S[c] >= cutoff && S[c] > 0.0) keep.push_back(c);
  const int k = (int)keep.size();
  F1.assign((size_t)k * m, 0.0);
  F2.assign((size_t)n * k, 0.0);
  for (int r = 0; r < k; r++) {
    const int c = keep[r];
    const double s = S[c];
    const double* w = &W[(size_t)c * M];  // U_c * s_c (length M)
    const double* v = &V[(size_t)c * N];  // V_c (length N)
    if (!tr) {  // A = U S V^T: F1 row = U_c^T / s = w^T / s^2, F2 column = v
      for (int j = 0; j < m; j++) F1[(size_t)r * m + j] = w[j] / (s * s);
      for (int i = 0; i < n; i++) F2[(size_t)i * k + r] = v[i];
    } else {  // A^T = W V^T: A = V S U'^T with U' = W / s: F1 row = v^T / s, F2 column = w / s
      for (int j = 0; j < m; j++) F1[(size_t)r * m + j] = v[j] / s;
      for (int i = 0; i < n; i++) F2[(size_t)i * k + r] = w[i] / s;
    }
  }
  return k;
}

// B (m x n, row-major) as F2 (m x k, row-major) times F1 (k x n, row-major):
// F2 holds the left singular vectors and F1 = diag(s) times the right ones,
// singular values below relCut * s_max dropped.  Applied to an explicit
// truncated pseudo-inverse this recovers the factors of pinv_truncated (the
// singular vectors are shared and s = 1/s_A), for tables the caller replaces.
int svd_factors(int m, int n, const double* B, double relCut, std::vector<double>& F1, std::vector<double>& F2) {
  const bool tr = m < n;  // factor B^T (n x m) so the one-sided SVD sees M >= N
  const int M = tr ? n : m, N = tr ? m : n;
  std::vector<double> W((size_t)M * N), V;
  if (tr) std::memcpy(W.data(), B, sizeof(double) * M * N);  // row-major B = column-major B^T
  else
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) W[(size_t)j * m + i] = B[(size_t)i * n + j];
  svd_onesided(M, N, W, V);
  std::vector<double> S(N);
  for (int c = 0; c < N; c++) {
    double s = 0;
    for (int i = 0; i < M; i++) s += W[(size_t)c * M + i] * W[(size_t)c * M + i];
    S[c] = std::sqrt(s);
  }
  const double smax = N ? *std::max_element(S.begin(), S.end()) : 0.0;
  std::vector<int> keep;
  for (int c = 0; c < N; c++)
    if (S[c] > relCut * smax && S[c] > 0.0) keep.push_back(c);
  const int k = (int)keep.size();
  F1.assign((size_t)k * n, 0.0);
  F2.assign((size_t)m * k, 0.0);
  for (int r = 0; r < k; r++) {
    const int c = keep[r];
    const double s = S[c];
    const double* w = &W[(size_t)c * M];  // U_c * s_c (length M)
    const double* v = &V[(size_t)c * N];  // V_c (length N)
    if (tr) {  // B^T = U S V^T: B = V S U^T, F2 column = V_c, F1 row = s U_c^T = w^T
      for (int i = 0; i < m; i++) F2[(size_t)i * k + r] = v[i];
      for (int j = 0; j < n; j++) F1[(size_t)r * n + j] = w[j];
    } else {  // B = U S V^T: F2 column = U_c = w / s, F1 row = s V_c^T
      for (int i = 0; i < m; i++) F2[(size_t)i * k + r] = w[i] / s;
      for (int j = 0; j < n; j++) F1[(size_t)r * n + j] = s * v[j];
    }
  }
  return k;
}

// C2E up x M2M through the factored pinv, in FP64: F2 (F1 M2M)
// C = A B for row-major A (rows x inner), B (inner x w), C (rows x w), in
// blocks of 32 rows by 256 columns so that each row of B serves a block of C
// rows from cache; every element still sums its inner terms in order.
static void gemm_rows_blocked(int rows, int inner, int w, const double* A, const double* B, double* C) {
  constexpr int RB = 32, JT = 256;
  const int nrb = (rows + RB - 1) / RB, njt = (w + JT - 1) / JT;
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int rb = 0; rb < nrb; rb++)
    for (int jt = 0; jt < njt; jt++) {
      const int r0 = rb * RB, r1 = std::min(rows, r0 + RB), j0 = jt * JT, j1 = std::min(w, j0 + JT);
      for (int c = 0; c < inner; c++) {
        const double* __restrict brow = &B[(size_t)c * w];
        int r = r0;
        for (; r + 4 <= r1; r += 4) {  // four rows of C per pass over the row of B
          const double f0 = A[(size_t)r * inner + c], f1 = A[(size_t)(r + 1) * inner + c];
          const double f2 = A[(size_t)(r + 2) * inner + c], f3 = A[(size_t)(r + 3) * inner + c];
          double* __restrict c0 = &C[(size_t)r * w];
          double* __restrict c1 = c0 + w;
          double* __restrict c2 = c1 + w;
          double* __restrict c3 = c2 + w;
#pragma omp simd
          for (int j = j0; j < j1; j++) {
            const double b = brow[j];
            c0[j] += f0 * b;
            c1[j] += f1 * b;
            c2[j] += f2 * b;
            c3[j] += f3 * b;
          }
        }
        for (; r < r1; r++) {
          const double f = A[(size_t)r * inner + c];
          double* __restrict crow = &C[(size_t)r * w];
#pragma omp simd
          for (int j = j0; j < j1; j++) crow[j] += f * brow[j];
        }
      }
    }
}

std::vector<double> fold_c2e_m2m(const Plan& P) {
  const int ue = P.nUE * P.sdm, uc = P.nUC * P.tdm, k = P.kUp, w = 8 * ue;
  std::vector<double> T((size_t)k * w, 0.0), R((size_t)ue * w, 0.0);
  if (tl_linalgDevice >= 0 &&
      gemm_rows_device(tl_linalgDevice, k, uc, w, P.uc2ueF1.data(), P.m2m.data(), T.data()).empty() &&
      gemm_rows_device(tl_linalgDevice, ue, k, w, P.uc2ueF2.data(), T.data(), R.data()).empty())
    return R;
  std::fill(T.begin(), T.end(), 0.0);
  std::fill(R.begin(), R.end(), 0.0);
  gemm_rows_blocked(k, uc, w, P.uc2ueF1.data(), P.m2m.data(), T.data());
  gemm_rows_blocked(ue, k, w, P.uc2ueF2.data(), T.data(), R.data());
  return R;
}

// out[kz][ky][kx][h], kx in [0, n/2]; in[z][y][x][h] (x fastest), e^{-2 pi i}
void rfft3_host(int n, int howmany, const double* in, std::complex<double>* out) {
  typedef std::complex<double> C;
  const int nh = n / 2 + 1;
  std::vector<C> w(n);
  for (int j = 0; j < n; j++) w[j] = C(std::cos(2.0 * M_PI * j / n), -std::sin(2.0 * M_PI * j / n));
  std::vector<C> a((size_t)n * n * nh), b((size_t)n * n * nh);
  for (int h = 0; h < howmany; h++) {
    for (int z = 0; z < n; z++)
      for (int y = 0; y < n; y++)
        for (int kx = 0; kx < nh; kx++) {
          C s = 0;
          for (int x = 0; x < n; x++) s += in[(((size_t)z * n + y) * n + x) * howmany + h] * w[(kx * x) % n];
          a[((size_t)z * n + y) * nh + kx] = s;
        }
    for (int z = 0; z < n; z++)
      for (int ky = 0; ky < n; ky++)
        for (int kx = 0; kx < nh; kx++) {
          C s = 0;
          for (int y = 0; y < n; y++) s += a[((size_t)z * n + y) * nh + kx] * w[(ky * y) % n];
          b[((size_t)z * n + ky) * nh + kx] = s;
        }
    for (int kz = 0; kz < n; kz++)
      for (int ky = 0; ky < n; ky++)
        for (int kx = 0; kx < nh; kx++) {
          C s = 0;
          for (int z = 0; z < n; z++) s += b[((size_t)z * n + ky) * nh + kx] * w[(kz * z) % n];
          out[(((size_t)kz * n + ky) * nh + kx) * howmany + h] = s;
        }
  }
}

}  // namespace fmmg
