// linalg.cpp -- dense linear algebra for the operator builder (setup only).
//
// pinv_truncated: the truncated pseudo-inverse of common/vecmatop.cpp:129-164
// (common/svdrep.cpp:38-80 keeps the singular values >= eps * s_max), computed
// from a Jacobi SVD preconditioned by a pivoted QR, which is accurate in the
// small singular values that the truncation tests (LAPACK dgesvd, which the
// reference calls, is not installed here).  rfft3_host: the r2c transform with FFTW's rank-3
// layout used for the M2L translation tables (fmm3d_mpi/matmgnt3d_mpi.cpp:408).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "plan.hpp"

namespace fmmg {

// A is m x n column-major with m >= n after an optional transpose.  Columns
// are orthogonalised pairwise in tournament order (n/2 disjoint pairs per
// round, so rounds parallelise and the result is thread-count independent).
static void svd_onesided(int m, int n, std::vector<double>& W /* m x n, becomes U*S */,
                         std::vector<double>& V /* n x n */) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  const int nn = n + (n & 1);
  std::vector<int> top(nn / 2), bot(nn / 2);
  for (int i = 0; i < nn / 2; i++) { top[i] = 2 * i; bot[i] = 2 * i + 1; }
  std::vector<double> norms(n);
  for (int sweep = 0; sweep < 80; sweep++) {
    int rotated = 0;
    for (int j = 0; j < n; j++) {
      double s = 0;
      const double* w = &W[(size_t)j * m];
      for (int i = 0; i < m; i++) s += w[i] * w[i];
      norms[j] = s;
    }
    for (int round = 0; round < nn - 1; round++) {
#pragma omp parallel for schedule(static) reduction(+ : rotated)
      for (int k = 0; k < nn / 2; k++) {
        int p = std::min(top[k], bot[k]), q = std::max(top[k], bot[k]);
        if (q >= n) continue;
        double* wp = &W[(size_t)p * m];
        double* wq = &W[(size_t)q * m];
        double a = 0, b = 0, g = 0;
#pragma omp simd reduction(+ : a, b, g)
        for (int i = 0; i < m; i++) {
          a += wp[i] * wp[i];
          b += wq[i] * wq[i];
          g += wp[i] * wq[i];
        }
        if (a == 0.0 || b == 0.0) continue;
        if (std::fabs(g) <= 1e-15 * std::sqrt(a * b)) continue;
        rotated++;
        double zeta = (b - a) / (2.0 * g);
        double t = std::copysign(1.0, zeta) / (std::fabs(zeta) + std::hypot(1.0, zeta));
        double c = 1.0 / std::hypot(1.0, t), s = c * t;
#pragma omp simd
        for (int i = 0; i < m; i++) {
          double x = wp[i], y = wq[i];
          wp[i] = c * x - s * y;
          wq[i] = s * x + c * y;
        }
        double* vp = &V[(size_t)p * n];
        double* vq = &V[(size_t)q * n];
#pragma omp simd
        for (int i = 0; i < n; i++) {
          double x = vp[i], y = vq[i];
          vp[i] = c * x - s * y;
          vq[i] = s * x + c * y;
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
}

// Householder QR with column pivoting of A (M x N column-major, M >= N):
// A P = Q R.  On return W holds R on and above the diagonal and the reflector
// tails below it (H_k = I - tau_k v v^T, v = [1, W[k+1.., k]]), and column j of
// A P is column perm[j] of A.  The pivot is the trailing column of largest
// remaining norm, recomputed exactly at every step.
static void qr_pivoted(int M, int N, std::vector<double>& W, std::vector<double>& tau, std::vector<int>& perm) {
  tau.assign(N, 0.0);
  perm.resize(N);
  for (int j = 0; j < N; j++) perm[j] = j;
  std::vector<double> nrm(N);
  for (int k = 0; k < N; k++) {
#pragma omp parallel for schedule(static)
    for (int j = k; j < N; j++) {
      const double* w = &W[(size_t)j * M];
      double s = 0;
      for (int i = k; i < M; i++) s += w[i] * w[i];
      nrm[j] = s;
    }
    int p = k;
    for (int j = k + 1; j < N; j++)
      if (nrm[j] > nrm[p]) p = j;
    if (p != k) {
      std::swap_ranges(W.begin() + (size_t)k * M, W.begin() + (size_t)(k + 1) * M, W.begin() + (size_t)p * M);
      std::swap(perm[k], perm[p]);
    }
    double* v = &W[(size_t)k * M];
    double xn = 0;
    for (int i = k + 1; i < M; i++) xn += v[i] * v[i];
    if (xn == 0.0) continue;  // nothing below the diagonal: H_k = I
    const double alpha = v[k];
    const double beta = -std::copysign(std::sqrt(alpha * alpha + xn), alpha);
    const double t = (beta - alpha) / beta, sc = 1.0 / (alpha - beta);
    tau[k] = t;
    for (int i = k + 1; i < M; i++) v[i] *= sc;
    v[k] = beta;
#pragma omp parallel for schedule(static)
    for (int j = k + 1; j < N; j++) {
      double* w = &W[(size_t)j * M];
      double d = w[k];
      for (int i = k + 1; i < M; i++) d += v[i] * w[i];
      d *= t;
      w[k] -= d;
      for (int i = k + 1; i < M; i++) w[i] -= d * v[i];
    }
  }
}

// Thin SVD A = U diag(S) V^T of A (M x N column-major, M >= N); U is M x N
// and V N x N, column-major, with unit columns where S > 0.  Pivoted QR first,
// then one-sided Jacobi on X = R^T, which the pivoting leaves close to
// column-orthogonal so that few sweeps remain (Z. Drmac and K. Veselic, "New
// fast and accurate Jacobi SVD algorithm", SIAM J. Matrix Anal. Appl. 29,
// 2008): with X = Ux S Vx^T, R = Vx S Ux^T and A = (Q Vx) S (P Ux)^T.
static void svd_thin(int M, int N, const double* A, std::vector<double>& U, std::vector<double>& S,
                     std::vector<double>& V) {
  std::vector<double> W(A, A + (size_t)M * N), tau, Vx;
  std::vector<int> perm;
  qr_pivoted(M, N, W, tau, perm);
  std::vector<double> X((size_t)N * N, 0.0);
  for (int j = 0; j < N; j++)  // column j of X = row j of R
    for (int i = j; i < N; i++) X[(size_t)j * N + i] = W[(size_t)i * M + j];
  svd_onesided(N, N, X, Vx);  // X becomes Ux S
  S.assign(N, 0.0);
  V.assign((size_t)N * N, 0.0);
  for (int c = 0; c < N; c++) {
    double s = 0;
    const double* x = &X[(size_t)c * N];
    for (int i = 0; i < N; i++) s += x[i] * x[i];
    S[c] = std::sqrt(s);
    if (S[c] > 0.0)
      for (int j = 0; j < N; j++) V[(size_t)c * N + perm[j]] = x[j] / S[c];
  }
  U.assign((size_t)M * N, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
  for (int c = 0; c < N; c++) {  // U_c = Q (Vx_c, 0) = H_0 H_1 .. H_{N-1} (Vx_c, 0)
    double* y = &U[(size_t)c * M];
    for (int i = 0; i < N; i++) y[i] = Vx[(size_t)c * N + i];
    for (int k = N - 1; k >= 0; k--) {
      if (tau[k] == 0.0) continue;
      const double* v = &W[(size_t)k * M];
      double d = y[k];
      for (int i = k + 1; i < M; i++) d += v[i] * y[i];
      d *= tau[k];
      y[k] -= d;
      for (int i = k + 1; i < M; i++) y[i] -= d * v[i];
    }
  }
}

// The singular triplets of A (m x n column-major) as left/right vector arrays
// of lengths m and n: the SVD is taken of A or, when m < n, of A^T.
struct Svd {
  std::vector<double> U, S, V;
  const double* left = nullptr;   // column c: the left singular vector c (length m)
  const double* right = nullptr;  // column c: the right singular vector c (length n)
  int lstride = 0, rstride = 0, N = 0;
  Svd(int m, int n, const double* A_colmajor) {
    const bool tr = m < n;
    const int M = tr ? n : m;
    N = tr ? m : n;
    std::vector<double> B((size_t)M * N);
    if (!tr) std::memcpy(B.data(), A_colmajor, sizeof(double) * M * N);
    else
      for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) B[(size_t)i * n + j] = A_colmajor[(size_t)j * m + i];
    svd_thin(M, N, B.data(), U, S, V);
    left = tr ? V.data() : U.data();
    right = tr ? U.data() : V.data();
    lstride = tr ? N : M;
    rstride = tr ? M : N;
  }
  std::vector<int> keep(double relCut, bool inclusive) const {
    const double smax = N ? *std::max_element(S.begin(), S.end()) : 0.0;
    std::vector<int> k;
    for (int c = 0; c < N; c++)
      if ((inclusive ? S[c] >= relCut * smax : S[c] > relCut * smax) && S[c] > 0.0) k.push_back(c);
    return k;
  }
};

int pinv_truncated(int m, int n, const double* A, double eps, double* R, std::vector<double>& F1,
                   std::vector<double>& F2) {
  const Svd d(m, n, A);
  const std::vector<int> keep = d.keep(eps, true);  // svdrep.cpp:38-80: s >= eps * s_max
  const int k = (int)keep.size();
  F1.assign((size_t)k * m, 0.0);
  F2.assign((size_t)n * k, 0.0);
  for (int r = 0; r < k; r++) {
    const int c = keep[r];
    const double s = d.S[c];
    const double* u = d.left + (size_t)c * d.lstride;
    const double* v = d.right + (size_t)c * d.rstride;
    for (int j = 0; j < m; j++) F1[(size_t)r * m + j] = u[j] / s;
    for (int i = 0; i < n; i++) F2[(size_t)i * k + r] = v[i];
  }
  if (R) {  // R = F2 F1, n x m column-major
    std::vector<double> F1t((size_t)m * k);
    for (int r = 0; r < k; r++)
      for (int j = 0; j < m; j++) F1t[(size_t)j * k + r] = F1[(size_t)r * m + j];
#pragma omp parallel for schedule(static)
    for (int j = 0; j < m; j++)
      for (int i = 0; i < n; i++) {
        double s = 0;
        const double* a = &F2[(size_t)i * k];
        const double* b = &F1t[(size_t)j * k];
        for (int r = 0; r < k; r++) s += a[r] * b[r];
        R[(size_t)j * n + i] = s;
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
  std::vector<double> Bc((size_t)m * n);
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) Bc[(size_t)j * m + i] = B[(size_t)i * n + j];
  const Svd d(m, n, Bc.data());
  const std::vector<int> keep = d.keep(relCut, false);
  const int k = (int)keep.size();
  F1.assign((size_t)k * n, 0.0);
  F2.assign((size_t)m * k, 0.0);
  for (int r = 0; r < k; r++) {
    const int c = keep[r];
    const double* u = d.left + (size_t)c * d.lstride;
    const double* v = d.right + (size_t)c * d.rstride;
    for (int i = 0; i < m; i++) F2[(size_t)i * k + r] = u[i];
    for (int j = 0; j < n; j++) F1[(size_t)r * n + j] = d.S[c] * v[j];
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
