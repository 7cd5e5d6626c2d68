// ref_shims.cpp -- the third-party arithmetic the reference's kernel and
// operator sources call, so that those sources build here without BLAS,
// LAPACK or FFTW (test infrastructure: linked only into oracle/_ref).
//
//  * BLAS dgemv / dgemm / daxpy / dger / dscal: the published netlib
//    reference algorithms (column-major, the column loop outermost for
//    dgemv 'N' and dgemm 'N','N'), as the reference links them through
//    common/blas.h.
//  * LAPACK dgesvd, dgetrf, dgetri: forwarded to the LAPACK routines the
//    caller registers at load time (oracle/ref_code.py hands over scipy's LAPACK); a call
//    before registration reports INFO = -1000.
//  * FFTW 3 fftw_plan_many_dft_r2c / _c2r / fftw_execute /
//    fftw_destroy_plan: FFTW's documented semantics, restated as separable
//    DFTs (row-major dimensions, the last one halved to n/2+1 for r2c,
//    howmany interleaved transforms addressed by stride and distance, forward
//    sign -1, both directions unnormalised).
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "fftw3.h"

typedef std::complex<double> cplx;

extern "C" {

// ------------------------------------------------------------------ BLAS
static bool is_n(const char* t) { return *t == 'N' || *t == 'n'; }

void dscal_(int* N, double* ALPHA, double* X, int* INCX) {
  for (int i = 0; i < *N; i++) X[(long)i * *INCX] *= *ALPHA;
}

void daxpy_(int* N, double* ALPHA, double* X, int* INCX, double* Y, int* INCY) {
  if (*N <= 0 || *ALPHA == 0.0) return;
  for (int i = 0; i < *N; i++) Y[(long)i * *INCY] += *ALPHA * X[(long)i * *INCX];
}

void dger_(int* M, int* N, double* ALPHA, double* X, int* INCX, double* Y, int* INCY, double* A, int* LDA) {
  for (int j = 0; j < *N; j++) {
    const double yj = Y[(long)j * *INCY];
    if (yj == 0.0) continue;
    const double t = *ALPHA * yj;
    for (int i = 0; i < *M; i++) A[i + (long)j * *LDA] += X[(long)i * *INCX] * t;
  }
}

void dgemv_(char* TRANS, int* M, int* N, double* ALPHA, double* A, int* LDA, double* X, int* INCX, double* BETA,
            double* Y, int* INCY) {
  const int m = *M, n = *N;
  if (m == 0 || n == 0) return;
  const bool nt = is_n(TRANS);
  const int leny = nt ? m : n, lenx = nt ? n : m;
  if (*BETA != 1.0)
    for (int i = 0; i < leny; i++) Y[(long)i * *INCY] = *BETA == 0.0 ? 0.0 : *BETA * Y[(long)i * *INCY];
  if (*ALPHA == 0.0) return;
  if (nt) {  // y := alpha A x + y, one column at a time
    for (int j = 0; j < lenx; j++) {
      const double t = *ALPHA * X[(long)j * *INCX];
      for (int i = 0; i < m; i++) Y[(long)i * *INCY] += t * A[i + (long)j * *LDA];
    }
  } else {  // y := alpha A' x + y, one dot product per column
    for (int j = 0; j < n; j++) {
      double t = 0.0;
      for (int i = 0; i < m; i++) t += A[i + (long)j * *LDA] * X[(long)i * *INCX];
      Y[(long)j * *INCY] += *ALPHA * t;
    }
  }
}

void dgemm_(char* TRANSA, char* TRANSB, int* M, int* N, int* K, double* ALPHA, double* A, int* LDA, double* B, int* LDB,
            double* BETA, double* C, int* LDC) {
  const int m = *M, n = *N, k = *K;
  const bool na = is_n(TRANSA), nb = is_n(TRANSB);
  auto a = [&](int i, int l) { return na ? A[i + (long)l * *LDA] : A[l + (long)i * *LDA]; };
  auto b = [&](int l, int j) { return nb ? B[l + (long)j * *LDB] : B[j + (long)l * *LDB]; };
  for (int j = 0; j < n; j++) {
    double* c = C + (long)j * *LDC;
    if (*BETA == 0.0) {
      for (int i = 0; i < m; i++) c[i] = 0.0;
    } else if (*BETA != 1.0) {
      for (int i = 0; i < m; i++) c[i] *= *BETA;
    }
    if (*ALPHA == 0.0) continue;
    if (na) {  // C(:,j) += (alpha B(l,j)) A(:,l), l in order
      for (int l = 0; l < k; l++) {
        const double t = *ALPHA * b(l, j);
        for (int i = 0; i < m; i++) c[i] += t * a(i, l);
      }
    } else {  // C(i,j) += alpha (A(:,i) . B(:,j))
      for (int i = 0; i < m; i++) {
        double t = 0.0;
        for (int l = 0; l < k; l++) t += a(i, l) * b(l, j);
        c[i] += *ALPHA * t;
      }
    }
  }
}

// ---------------------------------------------------------------- LAPACK
typedef void (*dgesvd_fn)(char*, char*, int*, int*, double*, int*, double*, double*, int*, double*, int*, double*,
                          int*, int*);
typedef void (*dgetrf_fn)(int*, int*, double*, int*, int*, int*);
typedef void (*dgetri_fn)(int*, double*, int*, int*, double*, int*, int*);
static dgesvd_fn g_dgesvd = nullptr;
static dgetrf_fn g_dgetrf = nullptr;
static dgetri_fn g_dgetri = nullptr;

// name: "dgesvd", "dgetrf" or "dgetri"; returns 0, or -1 for another name
int fmmg_ref_register_lapack(const char* name, void* fn) {
  if (!std::strcmp(name, "dgesvd")) g_dgesvd = (dgesvd_fn)fn;
  else if (!std::strcmp(name, "dgetrf")) g_dgetrf = (dgetrf_fn)fn;
  else if (!std::strcmp(name, "dgetri")) g_dgetri = (dgetri_fn)fn;
  else return -1;
  return 0;
}

void dgetrf_(int* M, int* N, double* A, int* LDA, int* IPIV, int* INFO) {
  if (!g_dgetrf) {
    *INFO = -1000;
    return;
  }
  g_dgetrf(M, N, A, LDA, IPIV, INFO);
}

void dgetri_(int* N, double* A, int* LDA, int* IPIV, double* WORK, int* LWORK, int* INFO) {
  if (!g_dgetri) {
    *INFO = -1000;
    return;
  }
  g_dgetri(N, A, LDA, IPIV, WORK, LWORK, INFO);
}

void dgesvd_(char* JOBU, char* JOBVT, int* M, int* N, double* A, int* LDA, double* S, double* U, int* LDU, double* VT,
             int* LDVT, double* WORK, int* LWORK, int* INFO) {
  if (!g_dgesvd) {
    *INFO = -1000;
    return;
  }
  g_dgesvd(JOBU, JOBVT, M, N, A, LDA, S, U, LDU, VT, LDVT, WORK, LWORK, INFO);
}

}  // extern "C"

// ------------------------------------------------------------------ FFTW
struct fmmg_ref_fftw_plan_s {
  bool r2c;
  std::vector<int> n;
  int howmany, istride, idist, ostride, odist;
  double* rin;
  fftw_complex* cin;
  double* rout;
  fftw_complex* cout;
};

// exp(sign 2 pi i m / n) for m = 0..n-1
static std::vector<cplx> twiddles(int n, int sign) {
  std::vector<cplx> w(n);
  for (int m = 0; m < n; m++) {
    const double a = 2.0 * M_PI * (double)m / (double)n;
    w[m] = cplx(std::cos(a), sign * std::sin(a));
  }
  return w;
}

// In-place complex DFT along dimension d of a row-major array with dims
// `dims` (direct sums, twiddle index (j k) mod n).
static void dft_axis(std::vector<cplx>& a, const std::vector<int>& dims, int d, int sign) {
  const int n = dims[d];
  long inner = 1, outer = 1;
  for (size_t e = d + 1; e < dims.size(); e++) inner *= dims[e];
  for (int e = 0; e < d; e++) outer *= dims[e];
  const std::vector<cplx> w = twiddles(n, sign);
  std::vector<cplx> line(n), res(n);
  for (long o = 0; o < outer; o++)
    for (long i = 0; i < inner; i++) {
      const long base = o * n * inner + i;
      for (int j = 0; j < n; j++) line[j] = a[base + (long)j * inner];
      for (int k = 0; k < n; k++) {
        cplx s(0.0, 0.0);
        for (int j = 0; j < n; j++) s += line[j] * w[((long)j * k) % n];
        res[k] = s;
      }
      for (int k = 0; k < n; k++) a[base + (long)k * inner] = res[k];
    }
}

extern "C" {

fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int*, int istride, int idist,
                                 fftw_complex* out, const int*, int ostride, int odist, unsigned) {
  fftw_plan p = new fmmg_ref_fftw_plan_s();
  p->r2c = true;
  p->n.assign(n, n + rank);
  p->howmany = howmany;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->rin = in;
  p->cout = out;
  return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int*, int istride,
                                 int idist, double* out, const int*, int ostride, int odist, unsigned) {
  fftw_plan p = new fmmg_ref_fftw_plan_s();
  p->r2c = false;
  p->n.assign(n, n + rank);
  p->howmany = howmany;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->cin = in;
  p->rout = out;
  return p;
}

void fftw_execute(const fftw_plan p) {
  const int r = (int)p->n.size();
  const int nl = p->n[r - 1], nh = nl / 2 + 1;
  std::vector<int> half(p->n);
  half[r - 1] = nh;
  long rows = 1;
  for (int d = 0; d < r - 1; d++) rows *= p->n[d];
  const long nreal = rows * nl, ncplx = rows * nh;
  for (int h = 0; h < p->howmany; h++) {
    if (p->r2c) {
      std::vector<cplx> a(nreal);
      for (long i = 0; i < nreal; i++) a[i] = cplx(p->rin[i * p->istride + (long)h * p->idist], 0.0);
      for (int d = r - 1; d >= 0; d--) dft_axis(a, p->n, d, -1);
      for (long row = 0; row < rows; row++)
        for (int k = 0; k < nh; k++) {
          const cplx v = a[row * nl + k];
          double* o = p->cout[(row * nh + k) * p->ostride + (long)h * p->odist];
          o[0] = v.real();
          o[1] = v.imag();
        }
    } else {
      std::vector<cplx> a(ncplx);
      for (long i = 0; i < ncplx; i++) {
        const double* v = p->cin[i * p->istride + (long)h * p->idist];
        a[i] = cplx(v[0], v[1]);
      }
      for (int d = r - 2; d >= 0; d--) dft_axis(a, half, d, +1);
      // the halved last axis: x_j = sum over the Hermitian extension; only
      // the real parts of the k = 0 and (even n) k = n/2 terms enter
      const std::vector<cplx> w = twiddles(nl, +1);
      for (long row = 0; row < rows; row++)
        for (int j = 0; j < nl; j++) {
          double s = a[row * nh].real();
          for (int k = 1; k < nh; k++) {
            const cplx t = a[row * nh + k] * w[((long)j * k) % nl];
            s += (2 * k == nl) ? t.real() : 2.0 * t.real();
          }
          p->rout[(row * nl + j) * p->ostride + (long)h * p->odist] = s;
        }
    }
  }
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
