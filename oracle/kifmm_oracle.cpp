// kifmm_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A CPU, FP64 restatement of the single-rank evaluate() path of the reference
// kernel-independent FMM (aashays/fmm-g, class FMM3d_MPI).  It exists only to
// check the GPU library: tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load it; the library never links or calls it.
//
// Parity status: UNPINNED against the reference itself.  The reference ships no
// tests, golden vectors or fixtures, and it cannot be compiled here (it needs
// PETSc 2.3.3, DENDRO 1.0, FFTW3, Fortran BLAS/LAPACK and MPI, none of which is
// installed).  The pieces that stand in for third-party code are pinned
// against independent implementations in tests/: the FFTW r2c/c2r layout
// against numpy.fft, the truncated-SVD pseudo-inverse against numpy.linalg.svd,
// and the whole evaluate against an FP64 dense direct sum (the reference's own
// check() protocol, fmm3d_mpi/fmm3d_check_mpi.cpp:122-165).
//
// Reference files restated (paths relative to the reference root):
//   fmm3d_mpi/kernel3d_mpi.cpp:35-466      kernels, DOFs, homogeneity
//   fmm3d_mpi/fmm3d_setup_mpi.cpp:113-126  user kernel -> equivalent kernel
//   fmm3d_mpi/matmgnt3d_mpi.cpp:37-512     surfaces, operators, FFT M2L
//   common/vecmatop.cpp:102-164, common/svdrep.cpp:38-80   dgemv, pinv
//   fmm3d_mpi/let3d_mpi.cpp:611-726, 1209-1876             tree, binning, lists
//   fmm3d_mpi/fmm3d_mpi.cpp:81-249          direct-evaluation helpers
//   fmm3d_mpi/fmm3d_eval_mpi.cpp:396-1515   evaluate() stage order (CPU paths)
//   fmm3d_mpi/fmm3d_check_mpi.cpp:34-172    dense check
//
// Third-party arithmetic restated from its published definition:
//   FFTW 3.x fftw_plan_many_dft_r2c / _c2r (rank 3, n = 2np per axis, row-major
//   with the x index fastest, the x axis halved, howmany = DOF interleaved with
//   stride DOF and distance 1, unnormalised, forward sign -1) -- restated as a
//   mixed-radix (2, 3) Cooley-Tukey transform.
//   LAPACK dgesvd (JOBU=JOBVT='S') -- restated as a one-sided (Hestenes) Jacobi
//   SVD; only the truncated pseudo-inverse built from it is used.
//   DENDRO ot::points2Octree -- restated as "split an octant while it holds more
//   than ptsMax sources and is above maxLevel; every split makes 8 children; the
//   root is always split" (let3d_mpi.cpp:268-288).  DENDRO's exact leaf set is
//   not reproduced; both this oracle and the GPU library use this rule.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <queue>
#include <set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

typedef std::complex<double> cplx;

// ---------------------------------------------------------------- kernels
// kernel3d_mpi.hpp:37-78
enum {
  LAP_S_U = 111, LAP_D_U = 121, STK_F_U = 301, STK_S_U = 311, STK_S_P = 312,
  STK_D_U = 321, STK_D_P = 322, NAV_S_U = 511, NAV_D_U = 521
};

static const double MINDIF = 1e-8;  // kernel3d_mpi.cpp:35

// kernel3d_mpi.cpp:40-69
static int src_dof(int t) {
  switch (t) {
    case LAP_S_U: case LAP_D_U: return 1;
    case STK_F_U: return 4;
    case STK_S_U: case STK_S_P: case STK_D_U: case STK_D_P: return 3;
    case NAV_S_U: case NAV_D_U: return 3;
  }
  return 0;
}
// kernel3d_mpi.cpp:74-103
static int trg_dof(int t) {
  switch (t) {
    case LAP_S_U: case LAP_D_U: return 1;
    case STK_F_U: case STK_S_U: case STK_D_U: return 3;
    case STK_S_P: case STK_D_P: return 1;
    case NAV_S_U: case NAV_D_U: return 3;
  }
  return 0;
}
// kernel3d_mpi.cpp:122-131 (only the three equivalent kernels are homogeneous)
static bool hom_deg(int t, std::vector<double>& deg) {
  switch (t) {
    case LAP_S_U: deg.assign(1, 1.0); return true;
    case STK_F_U: deg = {1, 1, 1, 2}; return true;
    case NAV_S_U: deg.assign(3, 1.0); return true;
  }
  return false;
}
// fmm3d_setup_mpi.cpp:113-126
static int knl_mm_type(int t) {
  switch (t) {
    case LAP_S_U: case LAP_D_U: return LAP_S_U;
    case STK_S_U: case STK_D_U: return STK_F_U;
    case STK_S_P: case STK_D_P: return LAP_S_U;
    case NAV_S_U: case NAV_D_U: return NAV_S_U;
  }
  return -1;
}

// One (target, source) block of buildKnlIntCtx, kernel3d_mpi.cpp:142-466.
// K is row-major [trgDOF][srcDOF]; returns false (block = 0) when r < 1e-8.
static bool kernel_block(int type, const double* coefs, double x, double y, double z,
                         const double* nrm, double* K) {
  const int sd = src_dof(type), td = trg_dof(type);
  double r2 = x * x + y * y + z * z;
  double r = std::sqrt(r2);
  if (r < MINDIF) {
    for (int i = 0; i < sd * td; i++) K[i] = 0.0;
    return false;
  }
  switch (type) {
    case LAP_S_U: {  // :152-167
      double OOFP = 1.0 / (4.0 * M_PI);
      K[0] = OOFP / r;
    } break;
    case LAP_D_U: {  // :169-185
      double OOFP = 1.0 / (4.0 * M_PI);
      double rn = x * nrm[0] + y * nrm[1] + z * nrm[2];
      double r3 = r2 * r;
      K[0] = -OOFP / r3 * rn;
    } break;
    case STK_F_U: {  // :194-219
      double mu = coefs[0];
      double OOFP = 1.0 / (4.0 * M_PI), OOEP = 1.0 / (8.0 * M_PI), oomu = 1.0 / mu;
      double r3 = r2 * r;
      double G = oomu * OOEP / r, H = oomu * OOEP / r3, A = OOFP / r3;
      K[0] = G + H * x * x; K[1] = H * x * y;     K[2] = H * x * z;      K[3] = A * x;
      K[4] = H * y * x;     K[5] = G + H * y * y; K[6] = H * y * z;      K[7] = A * y;
      K[8] = H * z * x;     K[9] = H * z * y;     K[10] = G + H * z * z; K[11] = A * z;
    } break;
    case STK_S_U: {  // :221-242
      double mu = coefs[0];
      double OOEP = 1.0 / (8.0 * M_PI), oomu = 1.0 / mu;
      double r3 = r2 * r;
      double G = OOEP / r, H = OOEP / r3;
      K[0] = oomu * (G + H * x * x); K[1] = oomu * (H * x * y); K[2] = oomu * (H * x * z);
      K[3] = oomu * (H * y * x); K[4] = oomu * (G + H * y * y); K[5] = oomu * (H * y * z);
      K[6] = oomu * (H * z * x); K[7] = oomu * (H * z * y); K[8] = oomu * (G + H * z * z);
    } break;
    case STK_S_P: {  // :244-260
      double OOFP = 1.0 / (4.0 * M_PI);
      double r3 = r2 * r;
      K[0] = OOFP * x / r3; K[1] = OOFP * y / r3; K[2] = OOFP * z / r3;
    } break;
    case STK_D_U: {  // :262-283
      double SOEP = 6.0 / (8.0 * M_PI);
      double rn = x * nrm[0] + y * nrm[1] + z * nrm[2];
      double r5 = r2 * r2 * r;
      double C = -SOEP / r5;
      K[0] = C * rn * x * x; K[1] = C * rn * x * y; K[2] = C * rn * x * z;
      K[3] = C * rn * y * x; K[4] = C * rn * y * y; K[5] = C * rn * y * z;
      K[6] = C * rn * z * x; K[7] = C * rn * z * y; K[8] = C * rn * z * z;
    } break;
    case STK_D_P: {  // :285-308
      double mu = coefs[0];
      double OOTP = 1.0 / (2.0 * M_PI);
      double coef = mu * OOTP;
      double nx = nrm[0], ny = nrm[1], nz = nrm[2];
      double rn = x * nx + y * ny + z * nz;
      double r3 = r2 * r, r5 = r3 * r2;
      K[0] = coef * (nx / r3 - 3 * rn * x / r5);
      K[1] = coef * (ny / r3 - 3 * rn * y / r5);
      K[2] = coef * (nz / r3 - 3 * rn * z / r5);
    } break;
    case NAV_S_U: {  // :362-385
      double mu = coefs[0], ve = coefs[1];
      double sc1 = (3.0 - 4.0 * ve) / (16.0 * M_PI * (1.0 - ve));
      double sc2 = 1.0 / (16.0 * M_PI * (1.0 - ve));
      double oomu = 1.0 / mu;
      double r3 = r2 * r;
      double G = sc1 / r, H = sc2 / r3;
      K[0] = oomu * (G + H * x * x); K[1] = oomu * (H * x * y); K[2] = oomu * (H * x * z);
      K[3] = oomu * (H * y * x); K[4] = oomu * (G + H * y * y); K[5] = oomu * (H * y * z);
      K[6] = oomu * (H * z * x); K[7] = oomu * (H * z * y); K[8] = oomu * (G + H * z * z);
    } break;
    case NAV_D_U: {  // :387-419
      double ve = coefs[1];
      double dc1 = -(1 - 2.0 * ve) / (8.0 * M_PI * (1.0 - ve));
      double dc2 = (1 - 2.0 * ve) / (8.0 * M_PI * (1.0 - ve));
      double dc3 = -3.0 / (8.0 * M_PI * (1.0 - ve));
      double nx = nrm[0], ny = nrm[1], nz = nrm[2];
      double rn = x * nx + y * ny + z * nz;
      double r3 = r2 * r, r5 = r3 * r2;
      double A = dc1 / r3, B = dc2 / r3, C = dc3 / r5;
      double rx = x, ry = y, rz = z;
      K[0] = A * (rn + nx * rx) + B * (rx * nx) + C * rn * rx * rx;
      K[1] = A * (nx * ry) + B * (rx * ny) + C * rn * rx * ry;
      K[2] = A * (nx * rz) + B * (rx * nz) + C * rn * rx * rz;
      K[3] = A * (ny * rx) + B * (ry * nx) + C * rn * ry * rx;
      K[4] = A * (rn + ny * ry) + B * (ry * ny) + C * rn * ry * ry;
      K[5] = A * (ny * rz) + B * (ry * nz) + C * rn * ry * rz;
      K[6] = A * (nz * rx) + B * (rz * nx) + C * rn * rz * rx;
      K[7] = A * (nz * ry) + B * (rz * ny) + C * rn * rz * ry;
      K[8] = A * (rn + nz * rz) + B * (rz * nz) + C * rn * rz * rz;
    } break;
  }
  return true;
}

// Dense kernel matrix, column-major (nt*td) x (ns*sd), as buildKnlIntCtx.
static void kernel_matrix(int type, const double* coefs, int ns, const double* src,
                          const double* nrm, int nt, const double* trg, double* out) {
  const int sd = src_dof(type), td = trg_dof(type);
  const long m = (long)nt * td;
  double K[16];
  for (int j = 0; j < ns; j++)
    for (int i = 0; i < nt; i++) {
      kernel_block(type, coefs, trg[3 * i] - src[3 * j], trg[3 * i + 1] - src[3 * j + 1],
                   trg[3 * i + 2] - src[3 * j + 2], nrm + 3 * j, K);
      for (int t = 0; t < td; t++)
        for (int s = 0; s < sd; s++) out[(long)(j * sd + s) * m + i * td + t] = K[t * sd + s];
    }
}

// y += K(trg, src) * den, accumulated in BLAS dgemv('N') order: for every target
// component the columns (source j, component s) are added in increasing order
// (common/vecmatop.cpp:110-118, fmm3d_mpi.cpp:81-154).
static void direct_accum(int type, const double* coefs, int ns, const double* src,
                         const double* nrm, const double* den, int nt, const double* trg,
                         double* val) {
  const int sd = src_dof(type), td = trg_dof(type);
  double K[16];
  for (int i = 0; i < nt; i++) {
    double acc[3];
    for (int t = 0; t < td; t++) acc[t] = val[i * td + t];
    for (int j = 0; j < ns; j++) {
      kernel_block(type, coefs, trg[3 * i] - src[3 * j], trg[3 * i + 1] - src[3 * j + 1],
                   trg[3 * i + 2] - src[3 * j + 2], nrm + 3 * j, K);
      for (int s = 0; s < sd; s++) {
        double x = den[j * sd + s];
        for (int t = 0; t < td; t++) acc[t] += K[t * sd + s] * x;
      }
    }
    for (int t = 0; t < td; t++) val[i * td + t] = acc[t];
  }
}

// ---------------------------------------------------------------- surfaces
// matmgnt3d_mpi.cpp:451-475; pos is 3 x n, point-major (x,y,z per point)
static void sam_pos(int np, double R, std::vector<double>& pos) {
  int n = np * np * np - (np - 2) * (np - 2) * (np - 2);
  pos.assign(3 * n, 0.0);
  double step = 2.0 / (np - 1), init = -1.0;
  int cnt = 0;
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++)
      for (int k = 0; k < np; k++)
        if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
          pos[3 * cnt + 0] = R * (init + i * step);
          pos[3 * cnt + 1] = R * (init + j * step);
          pos[3 * cnt + 2] = R * (init + k * step);
          cnt++;
        }
}
// matmgnt3d_mpi.cpp:478-499
static void reg_pos(int np, double R, std::vector<double>& pos) {
  int n = 8 * np * np * np;
  pos.assign(3 * n, 0.0);
  double step = 2.0 / (np - 1);
  int cnt = 0;
  for (int k = 0; k < 2 * np; k++)
    for (int j = 0; j < 2 * np; j++)
      for (int i = 0; i < 2 * np; i++) {
        int gi = (i < np) ? i : i - 2 * np;
        int gj = (j < np) ? j : j - 2 * np;
        int gk = (k < np) ? k : k - 2 * np;
        pos[3 * cnt + 0] = R * gi * step;
        pos[3 * cnt + 1] = R * gj * step;
        pos[3 * cnt + 2] = R * gk * step;
        cnt++;
      }
}

// ---------------------------------------------------------------- FFT
// Mixed-radix decimation-in-time DFT of length n (n = 2^a 3^b, or any n with a
// direct-DFT fallback for other prime factors); sign -1 forward, +1 backward.
static void dft1(int n, const cplx* in, int is, cplx* out, int sign) {
  if (n == 1) { out[0] = in[0]; return; }
  int p = 2;
  while (n % p) p++;
  int m = n / p;
  if (m == 1) {  // direct DFT of prime length
    for (int k = 0; k < n; k++) {
      cplx s = 0;
      for (int j = 0; j < n; j++) {
        double a = sign * 2.0 * M_PI * (double)((long)j * k % n) / n;
        s += in[(long)j * is] * cplx(std::cos(a), std::sin(a));
      }
      out[k] = s;
    }
    return;
  }
  std::vector<cplx> Y((size_t)n);
  for (int q = 0; q < p; q++) dft1(m, in + (long)q * is, is * p, Y.data() + q * m, sign);
  for (int s = 0; s < p; s++)
    for (int k = 0; k < m; k++) {
      int kk = k + m * s;
      cplx acc = 0;
      for (int q = 0; q < p; q++) {
        double a = sign * 2.0 * M_PI * (double)((long)q * kk % n) / n;
        acc += Y[q * m + k] * cplx(std::cos(a), std::sin(a));
      }
      out[kk] = acc;
    }
}

// Full complex 3-D DFT in place on a row-major [n][n][n] array (x fastest).
static void dft3(int n, std::vector<cplx>& a, int sign) {
  std::vector<cplx> line(n), res(n);
  for (int axis = 0; axis < 3; axis++) {
    long st = axis == 0 ? 1 : (axis == 1 ? n : (long)n * n);
    for (int u = 0; u < n; u++)
      for (int v = 0; v < n; v++) {
        long base;
        if (axis == 0) base = ((long)u * n + v) * n;
        else if (axis == 1) base = (long)u * n * n + v;
        else base = (long)u * n + v;
        for (int w = 0; w < n; w++) line[w] = a[base + w * st];
        dft1(n, line.data(), 1, res.data(), sign);
        for (int w = 0; w < n; w++) a[base + w * st] = res[w];
      }
  }
}

// fftw_plan_many_dft_r2c(3, {n,n,n}, howmany, in, NULL, howmany, 1, out, NULL,
// howmany, 1): in is real [n^3][howmany], out complex [n][n][n/2+1][howmany].
static void rfft3(int n, int howmany, const double* in, cplx* out) {
  const long n3 = (long)n * n * n;
  const int nh = n / 2 + 1;
  std::vector<cplx> a(n3);
  for (int h = 0; h < howmany; h++) {
    for (long i = 0; i < n3; i++) a[i] = cplx(in[i * howmany + h], 0.0);
    dft3(n, a, -1);
    for (int kz = 0; kz < n; kz++)
      for (int ky = 0; ky < n; ky++)
        for (int kx = 0; kx < nh; kx++)
          out[(((long)kz * n + ky) * nh + kx) * howmany + h] = a[((long)kz * n + ky) * n + kx];
  }
}

// fftw_plan_many_dft_c2r with the same layout: the missing half of the x axis
// is the Hermitian mirror; the transform is unnormalised.  For the kx = 0 and
// kx = n/2 planes only the real part enters (as in FFTW's halved 1-D c2r).
static void irfft3(int n, int howmany, const cplx* in, double* out) {
  const long n3 = (long)n * n * n;
  const int nh = n / 2 + 1;
  std::vector<cplx> a(n3);
  for (int h = 0; h < howmany; h++) {
    for (int kz = 0; kz < n; kz++)
      for (int ky = 0; ky < n; ky++)
        for (int kx = 0; kx < n; kx++) {
          cplx v;
          if (kx < nh) v = in[(((long)kz * n + ky) * nh + kx) * howmany + h];
          else {
            int mz = (n - kz) % n, my = (n - ky) % n, mx = n - kx;
            v = std::conj(in[(((long)mz * n + my) * nh + mx) * howmany + h]);
          }
          a[((long)kz * n + ky) * n + kx] = v;
        }
    dft3(n, a, +1);
    for (long i = 0; i < n3; i++) out[i * howmany + h] = a[i].real();
  }
}

// ---------------------------------------------------------------- pinv
// One-sided Jacobi SVD of a column-major m x n matrix A (m >= n): returns
// U (m x n), S (n, descending), V (n x n).  Column pairs are rotated in a
// fixed round-robin order, so the result does not depend on the thread count.
static void jacobi_svd(int m, int n, const double* A, std::vector<double>& U,
                       std::vector<double>& S, std::vector<double>& V) {
  U.assign(A, A + (long)m * n);
  V.assign((long)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(long)i * n + i] = 1.0;
  int nn = n + (n & 1);
  std::vector<int> ring(nn);
  for (int i = 0; i < nn; i++) ring[i] = i;
  const double tol = 1e-15;
  for (int sweep = 0; sweep < 60; sweep++) {
    double offmax = 0.0;
    for (int round = 0; round < nn - 1; round++) {
      double rmax = 0.0;
#pragma omp parallel for schedule(static) reduction(max : rmax)
      for (int k = 0; k < nn / 2; k++) {
        int p = ring[k], q = ring[nn - 1 - k];
        if (p >= n || q >= n) continue;
        if (p > q) std::swap(p, q);
        double* up = &U[(long)p * m];
        double* uq = &U[(long)q * m];
        double alpha = 0, beta = 0, gamma = 0;
        for (int i = 0; i < m; i++) {
          alpha += up[i] * up[i];
          beta += uq[i] * uq[i];
          gamma += up[i] * uq[i];
        }
        if (alpha == 0.0 || beta == 0.0) continue;
        double off = std::fabs(gamma) / std::sqrt(alpha * beta);
        rmax = std::max(rmax, off);
        if (off <= tol) continue;
        double zeta = (beta - alpha) / (2.0 * gamma);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (int i = 0; i < m; i++) {
          double a = up[i], b = uq[i];
          up[i] = c * a - s * b;
          uq[i] = s * a + c * b;
        }
        double* vp = &V[(long)p * n];
        double* vq = &V[(long)q * n];
        for (int i = 0; i < n; i++) {
          double a = vp[i], b = vq[i];
          vp[i] = c * a - s * b;
          vq[i] = s * a + c * b;
        }
      }
      offmax = std::max(offmax, rmax);
      // rotate the ring, keeping ring[0] fixed
      int last = ring[nn - 1];
      for (int i = nn - 1; i > 1; i--) ring[i] = ring[i - 1];
      ring[1] = last;
    }
    if (offmax <= tol) break;
  }
  S.assign(n, 0.0);
  for (int j = 0; j < n; j++) {
    double s = 0;
    for (int i = 0; i < m; i++) s += U[(long)j * m + i] * U[(long)j * m + i];
    S[j] = std::sqrt(s);
    if (S[j] > 0)
      for (int i = 0; i < m; i++) U[(long)j * m + i] /= S[j];
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; i++) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return S[a] > S[b]; });
  std::vector<double> U2((long)m * n), V2((long)n * n), S2(n);
  for (int j = 0; j < n; j++) {
    S2[j] = S[ord[j]];
    std::memcpy(&U2[(long)j * m], &U[(long)ord[j] * m], sizeof(double) * m);
    std::memcpy(&V2[(long)j * n], &V[(long)ord[j] * n], sizeof(double) * n);
  }
  U.swap(U2); V.swap(V2); S.swap(S2);
}

// common/vecmatop.cpp:129-164 with common/svdrep.cpp:38-80: keep the singular
// values >= eps * s_max, R = V_k diag(1/s_k) U_k^T.  A is m x n column-major;
// R is n x m column-major.
static void pinv(int m, int n, const double* A, double eps, double* R) {
  std::vector<double> U, S, V;
  bool tr = m < n;
  if (!tr) {
    jacobi_svd(m, n, A, U, S, V);
  } else {  // A^T = V S U^T
    std::vector<double> At((long)m * n);
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) At[(long)i * n + j] = A[(long)j * m + i];
    jacobi_svd(n, m, At.data(), V, S, U);
  }
  int k = (int)S.size();
  int rows_u = m, rows_v = n;
  double cutoff = eps * S[0];
  int cnt = 0;
  while (cnt < k && std::fabs(S[cnt]) >= cutoff) cnt++;
  for (long i = 0; i < (long)n * m; i++) R[i] = 0.0;
  // R(i,j) = sum_c V(i,c) / S(c) * U(j,c)
  for (int c = 0; c < cnt; c++) {
    double inv = 1.0 / S[c];
    const double* vc = &V[(long)c * rows_v];
    const double* uc = &U[(long)c * rows_u];
    for (int j = 0; j < m; j++) {
      double f = uc[j] * inv;
      double* rc = &R[(long)j * n];
      for (int i = 0; i < n; i++) rc[i] += vc[i] * f;
    }
  }
}

// ---------------------------------------------------------------- tree
struct Node {
  int par, chd, depth;
  int path[3];
  int tag;           // LET_* bits as in let3d_mpi.hpp:28-39
  long glbSrcExaNum;  // > 0 only for leaves with sources (let3d_mpi.cpp:1357-1384)
  int srcBeg, srcNum;  // contiguous range in the leaf-ordered source arrays
  int trgBeg, trgNum;
  int srcCount, trgCount;  // points in the subtree
  std::vector<int> U, V, W, X;
};
enum { CBTR = 1, USER = 2, EVTR = 4, OWNR = 8, SRCE = 16 };

struct Oracle {
  // options
  int ktype, mmtype, np, ptsMax, maxLevel, rootLevel, nthreads;
  double coefs[2];
  double ctr[3];
  // dims
  int sd, td, sdm, tdm;  // user kernel and equivalent kernel DOFs
  std::vector<double> deg;
  // geometry
  long ns = 0, nt = 0;
  std::vector<double> srcPos, srcNor, trgPos;  // leaf-ordered copies
  std::vector<long> srcPerm, trgPerm;           // leaf-order -> input index
  std::vector<Node> nodes;
  // operators (column-major, as NumMat)
  std::vector<double> samPos[4], regPosv;
  int nUE, nUC, nDE, nDC, nReg, nEff;  // points / complex per component
  std::vector<double> uc2ue, dc2de;    // pinv matrices
  std::vector<double> ue2uc[8], de2dc[8];
  std::vector<cplx> ue2dc[316];  // [nEff][sdm*tdm] each
  int trans_id[7][7][7];

  double root_radius() const { return std::pow(2.0, -rootLevel); }
  double radius(int n) const { return root_radius() / double(1 << nodes[n].depth); }
  void center(int n, double* res) const {  // let3d_mpi.cpp:1808-1818
    double R = root_radius();
    double ll[3] = {ctr[0] - R, ctr[1] - R, ctr[2] - R};
    int tmp = 1 << nodes[n].depth;
    for (int d = 0; d < 3; d++) res[d] = ll[d] + (2 * R) * (nodes[n].path[d] + 0.5) / double(tmp);
  }
  bool terminal(int n) const { return nodes[n].chd == -1; }
  int child(int n, int a, int b, int c) const { return nodes[n].chd + (a * 4 + b * 2 + c); }

  // let3d_mpi.cpp:1833-1853
  int findGlbNode(int wntDepth, const int* wntPath) const {
    int cur = 0;
    int tmp[3] = {wntPath[0], wntPath[1], wntPath[2]};
    while (nodes[cur].depth < wntDepth && !terminal(cur)) {
      int dif = wntDepth - nodes[cur].depth;
      int t = 1 << (dif - 1);
      int ch[3] = {tmp[0] / t, tmp[1] / t, tmp[2] / t};
      for (int d = 0; d < 3; d++) tmp[d] -= ch[d] * t;
      cur = child(cur, ch[0], ch[1], ch[2]);
    }
    return cur;
  }
  // let3d_mpi.cpp:1856-1876
  bool adjacent(int me, int you) const {
    int md = std::max(nodes[me].depth, nodes[you].depth);
    int meRad = 1 << (md - nodes[me].depth), youRad = 1 << (md - nodes[you].depth);
    int radius = meRad + youRad;
    int linf = 0;
    bool le = true;
    for (int d = 0; d < 3; d++) {
      int mc = (2 * nodes[me].path[d] + 1) * meRad;
      int yc = (2 * nodes[you].path[d] + 1) * youRad;
      int dif = std::abs(mc - yc);
      le = le && (dif <= radius);
      linf = std::max(linf, dif);
    }
    return le && linf == radius;
  }

  // Split rule standing in for DENDRO points2Octree + CreateAncestors
  // (let3d_mpi.cpp:268-288, 611-726): pre-order, children appended when a
  // split node is first visited, child index a*4+b*2+c.
  void build_tree(std::vector<std::vector<long>>& srcIdx) {
    nodes.clear();
    Node root{};
    root.par = -1; root.chd = -1; root.depth = 0; root.path[0] = root.path[1] = root.path[2] = 0;
    nodes.push_back(root);
    srcIdx.assign(1, std::vector<long>());
    srcIdx[0].resize(ns);
    for (long i = 0; i < ns; i++) srcIdx[0][i] = i;
    visit(0, srcIdx);
  }
  void visit(int n, std::vector<std::vector<long>>& srcIdx) {
    bool split = (n == 0) || ((long)srcIdx[n].size() > ptsMax && nodes[n].depth < maxLevel);
    if (!split) return;
    int first = (int)nodes.size();
    nodes[n].chd = first;
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++)
        for (int c = 0; c < 2; c++) {
          Node ch{};
          ch.par = n; ch.chd = -1; ch.depth = nodes[n].depth + 1;
          ch.path[0] = 2 * nodes[n].path[0] + a;
          ch.path[1] = 2 * nodes[n].path[1] + b;
          ch.path[2] = 2 * nodes[n].path[2] + c;
          nodes.push_back(ch);
          srcIdx.push_back(std::vector<long>());
        }
    // srcData binning, let3d_mpi.cpp:1255-1267 (index order preserved)
    double cc[3];
    center(n, cc);
    for (long k : srcIdx[n]) {
      const double* p = &srcIn[3 * k];
      int a = p[0] >= cc[0], b = p[1] >= cc[1], c = p[2] >= cc[2];
      srcIdx[first + a * 4 + b * 2 + c].push_back(k);
    }
    std::vector<long>().swap(srcIdx[n]);  // let3d_mpi.cpp:1267
    for (int c = 0; c < 8; c++) visit(first + c, srcIdx);
  }

  const double* srcIn = nullptr;  // caller arrays during setup
  const double* nrmIn = nullptr;
  const double* trgIn = nullptr;

  // let3d_mpi.cpp:1637-1768
  void calGlbNodeLists(int g) {
    std::set<int> Us, Vs, Ws, Xs;
    if (nodes[g].par != -1) {
      int par = nodes[g].par;
      int maxIdx = 1 << nodes[g].depth;
      for (int i = -2; i < 4; i++)
        for (int j = -2; j < 4; j++)
          for (int k = -2; k < 4; k++) {
            int tp[3] = {2 * nodes[par].path[0] + i, 2 * nodes[par].path[1] + j,
                         2 * nodes[par].path[2] + k};
            bool ok = true;
            for (int d = 0; d < 3; d++) ok = ok && tp[d] >= 0 && tp[d] < maxIdx;
            bool same = tp[0] == nodes[g].path[0] && tp[1] == nodes[g].path[1] &&
                        tp[2] == nodes[g].path[2];
            if (!ok || same) continue;
            int res = findGlbNode(nodes[g].depth, tp);
            bool adj = adjacent(res, g);
            if (nodes[res].depth < nodes[g].depth) {
              if (adj) {
                if (terminal(g)) Us.insert(res);
              } else {
                Xs.insert(res);
              }
            }
            if (nodes[res].depth == nodes[g].depth) {
              if (!adj) {
                Vs.insert(res);
              } else if (terminal(g)) {
                std::queue<int> rest;
                rest.push(res);
                while (!rest.empty()) {
                  int f = rest.front();
                  rest.pop();
                  if (!adjacent(f, g)) {
                    Ws.insert(f);
                  } else if (terminal(f)) {
                    Us.insert(f);
                  } else {
                    for (int a = 0; a < 2; a++)
                      for (int b = 0; b < 2; b++)
                        for (int c = 0; c < 2; c++) rest.push(child(f, a, b, c));
                  }
                }
              }
            }
          }
    }
    if (terminal(g)) Us.insert(g);
    Node& nd = nodes[g];
    for (int s : Us) if (nodes[s].glbSrcExaNum > 0) nd.U.push_back(s);
    for (int s : Vs) if (nodes[s].tag & SRCE) nd.V.push_back(s);
    for (int s : Ws) if (nodes[s].tag & SRCE) nd.W.push_back(s);
    for (int s : Xs) if (nodes[s].glbSrcExaNum > 0) nd.X.push_back(s);
  }

  void setup(long ns_, const double* src, const double* nrm, long nt_, const double* trg) {
    ns = ns_; nt = nt_;
    srcIn = src; nrmIn = nrm; trgIn = trg;
    std::vector<std::vector<long>> srcIdx;
    build_tree(srcIdx);
    const int nn = (int)nodes.size();
    // tags and leaf source ranges (let3d_mpi.cpp:1301-1326, 1357-1384, 1436-1462)
    srcPos.clear(); srcNor.clear(); srcPerm.clear();
    for (int i = 0; i < nn; i++) {
      Node& nd = nodes[i];
      nd.tag = 0;
      nd.glbSrcExaNum = -1;
      nd.srcBeg = 0; nd.srcNum = 0;
    }
    // subtree source counts
    for (int i = nn - 1; i >= 0; i--) {
      if (terminal(i)) nodes[i].srcCount = (int)srcIdx[i].size();
      else {
        int s = 0;
        for (int c = 0; c < 8; c++) s += nodes[nodes[i].chd + c].srcCount;
        nodes[i].srcCount = s;
      }
    }
    for (int i = 1; i < nn; i++) {
      Node& nd = nodes[i];
      if (!terminal(i) || nd.srcCount > 0) nd.tag |= OWNR | SRCE;
      if (nd.srcCount > 0) nd.tag |= CBTR;
      if (terminal(i) && nd.srcCount > 0) {
        nd.glbSrcExaNum = nd.srcCount;
        nd.srcBeg = (int)srcPerm.size();
        nd.srcNum = nd.srcCount;
        for (long k : srcIdx[i]) {
          srcPerm.push_back(k);
          for (int d = 0; d < 3; d++) {
            srcPos.push_back(src[3 * k + d]);
            srcNor.push_back(nrm ? nrm[3 * k + d] : 0.0);
          }
        }
      }
    }
    // trgData binning, let3d_mpi.cpp:1470-1560
    std::vector<std::vector<long>> trgIdx(nn);
    trgIdx[0].resize(nt);
    for (long i = 0; i < nt; i++) trgIdx[0][i] = i;
    for (int i = 0; i < nn; i++) {
      nodes[i].trgCount = (int)trgIdx[i].size();
      if (!terminal(i)) {
        double cc[3];
        center(i, cc);
        for (long k : trgIdx[i]) {
          const double* p = &trg[3 * k];
          int a = p[0] >= cc[0], b = p[1] >= cc[1], c = p[2] >= cc[2];
          trgIdx[child(i, a, b, c)].push_back(k);
        }
        std::vector<long>().swap(trgIdx[i]);
      }
    }
    trgPos.clear(); trgPerm.clear();
    for (int i = 0; i < nn; i++) {
      Node& nd = nodes[i];
      nd.trgBeg = 0; nd.trgNum = 0;
      if (nd.trgCount > 0) {
        nd.tag |= EVTR;
        if (terminal(i)) {
          nd.trgBeg = (int)trgPerm.size();
          nd.trgNum = nd.trgCount;
          for (long k : trgIdx[i]) {
            trgPerm.push_back(k);
            for (int d = 0; d < 3; d++) trgPos.push_back(trg[3 * k + d]);
          }
        }
      }
    }
    for (int i = 0; i < nn; i++) {
      nodes[i].U.clear(); nodes[i].V.clear(); nodes[i].W.clear(); nodes[i].X.clear();
    }
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
    for (int i = 0; i < nn; i++)
      if (nodes[i].tag & EVTR) calGlbNodeLists(i);
    srcIn = nrmIn = trgIn = nullptr;
  }

  // ---------------------------------------------------------- operators
  // matmgnt3d_mpi.cpp:52-71, 107-274, 373-411 (homogeneous kernels: one set
  // of unit-radius operators, level scaling by 2^(l*deg) applied at use).
  void build_operators() {
    sam_pos(np, 1.0, samPos[0]);      // UE
    sam_pos(np + 2, 3.0, samPos[1]);  // UC
    sam_pos(np, 3.0, samPos[2]);      // DE
    sam_pos(np, 1.0, samPos[3]);      // DC
    reg_pos(np, 1.0, regPosv);
    nUE = (int)samPos[0].size() / 3; nUC = (int)samPos[1].size() / 3;
    nDE = (int)samPos[2].size() / 3; nDC = (int)samPos[3].size() / 3;
    nReg = (int)regPosv.size() / 3;
    int n = 2 * np;
    nEff = n * n * (n / 2 + 1);
    double eps = std::pow(0.1, np + 1);  // matmgnt3d_mpi.cpp:37-40
    {  // UpwChk2UpwEqu, :112-127
      std::vector<double> ud2c((long)nUC * tdm * nUE * sdm);
      kernel_matrix(mmtype, coefs, nUE, samPos[0].data(), samPos[0].data(), nUC, samPos[1].data(),
                    ud2c.data());
      uc2ue.assign((long)nUE * sdm * nUC * tdm, 0.0);
      pinv(nUC * tdm, nUE * sdm, ud2c.data(), eps, uc2ue.data());
    }
    {  // DwnChk2DwnEqu, :201-210
      std::vector<double> dd2c((long)nDC * tdm * nDE * sdm);
      kernel_matrix(mmtype, coefs, nDE, samPos[2].data(), samPos[2].data(), nDC, samPos[3].data(),
                    dd2c.data());
      dc2de.assign((long)nDE * sdm * nDC * tdm, 0.0);
      pinv(nDC * tdm, nDE * sdm, dd2c.data(), eps, dc2de.data());
    }
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++)
        for (int c = 0; c < 2; c++) {
          int o = a * 4 + b * 2 + c;
          int idx[3] = {a, b, c};
          {  // UpwEqu2UpwChk, :158-174
            std::vector<double> chk(3 * nUC), den(3 * nUE);
            for (int j = 0; j < nUC; j++)
              for (int d = 0; d < 3; d++) chk[3 * j + d] = 2.0 * samPos[1][3 * j + d];
            for (int j = 0; j < nUE; j++)
              for (int d = 0; d < 3; d++) den[3 * j + d] = samPos[0][3 * j + d] + (2 * idx[d] - 1) * 1.0;
            ue2uc[o].assign((long)nUC * tdm * nUE * sdm, 0.0);
            kernel_matrix(mmtype, coefs, nUE, den.data(), den.data(), nUC, chk.data(), ue2uc[o].data());
          }
          {  // DwnEqu2DwnChk, :239-255
            std::vector<double> chk(3 * nDC), den(3 * nDE);
            for (int j = 0; j < nDE; j++)
              for (int d = 0; d < 3; d++) den[3 * j + d] = samPos[2][3 * j + d];
            for (int j = 0; j < nDC; j++)
              for (int d = 0; d < 3; d++)
                chk[3 * j + d] = 0.5 * samPos[3][3 * j + d] + (double(idx[d]) - 0.5) * 1.0;
            de2dc[o].assign((long)nDC * tdm * nDE * sdm, 0.0);
            kernel_matrix(mmtype, coefs, nDE, den.data(), den.data(), nDC, chk.data(), de2dc[o].data());
          }
        }
    // UpwEqu2DwnChk translation spectra, :385-411; enumerated like
    // fmm3d_eval_mpi.cpp:841-849
    int cnt = 0;
    for (int i1 = -3; i1 <= 3; i1++)
      for (int i2 = -3; i2 <= 3; i2++)
        for (int i3 = -3; i3 <= 3; i3++) {
          if (std::abs(i1) > 1 || std::abs(i2) > 1 || std::abs(i3) > 1) trans_id[i1 + 3][i2 + 3][i3 + 3] = cnt++;
          else trans_id[i1 + 3][i2 + 3][i3 + 3] = -1;
        }
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int t = 0; t < 343; t++) {
      int i1 = t / 49 - 3, i2 = (t / 7) % 7 - 3, i3 = t % 7 - 3;
      int id = trans_id[i1 + 3][i2 + 3][i3 + 3];
      if (id < 0) continue;
      double denPos[3] = {i1 * 2.0, i2 * 2.0, i3 * 2.0};
      int m = sdm * tdm;
      // tt is (nReg*tdm) x sdm column-major; tmp(i, j + k*sdm) = tt(i + k*tdm, j)
      std::vector<double> tt((long)nReg * tdm * sdm), tmp((long)m * nReg);
      kernel_matrix(mmtype, coefs, 1, denPos, denPos, nReg, regPosv.data(), tt.data());
      for (int k = 0; k < nReg; k++)
        for (int i = 0; i < tdm; i++)
          for (int j = 0; j < sdm; j++)
            tmp[(long)(j + k * sdm) * tdm + i] = tt[(long)j * nReg * tdm + i + k * tdm];
      ue2dc[id].assign((long)nEff * m, cplx(0, 0));
      rfft3(2 * np, m, tmp.data(), ue2dc[id].data());
    }
  }

  // ---------------------------------------------------------- evaluate helpers
  void loc_pos(int tp, int node, std::vector<double>& pos) const {  // matmgnt3d_mpi.cpp:434-448
    double c[3];
    center(node, c);
    double r = radius(node);
    const std::vector<double>& bas = samPos[tp];
    pos.resize(bas.size());
    for (size_t j = 0; j < bas.size() / 3; j++)
      for (int d = 0; d < 3; d++) pos[3 * j + d] = c[d] + r * bas[3 * j + d];
  }
  // gemvOrder: bit b set sums the columns of operator class b in reverse
  // (b = 0 upward C2E, 1 M2M, 2 downward C2E, 3 L2L); clear bits keep the
  // reference BLAS column order (j = 0 .. n-1).  Reversed is an equally valid
  // summation order, used by the tests to measure how far two FP64
  // evaluations of the same operators that only sum in another order drift
  // apart (the pseudo-inverses amplify rounding).
  int gemvOrder = 0;
  void dgemv_acc(long m, long n, const double* A, const double* x, double* y, int cls) const {
    const bool rev = (gemvOrder >> cls) & 1;
    for (long jj = 0; jj < n; jj++) {
      const long j = rev ? n - 1 - jj : jj;
      double t = x[j];
      const double* a = A + j * m;
      for (long i = 0; i < m; i++) y[i] += t * a[i];
    }
  }
  // matmgnt3d_mpi.cpp:107-149
  void upwChk2UpwEqu(int l, const double* chk, double* den) const {
    long m = (long)nUE * sdm, n = (long)nUC * tdm;
    std::vector<double> tmp(m, 0.0);
    dgemv_acc(m, n, uc2ue.data(), chk, tmp.data(), 0);
    for (int i = 0; i < nUE; i++)
      for (int s = 0; s < sdm; s++) den[i * sdm + s] += tmp[i * sdm + s] * std::pow(2.0, -l * deg[s]);
  }
  // :151-193
  void upwEqu2UpwChk(int l, int o, const double* den, double* chk) const {
    long m = (long)nUC * tdm, n = (long)nUE * sdm;
    std::vector<double> tmp(n);
    for (int i = 0; i < nUE; i++)
      for (int s = 0; s < sdm; s++) tmp[i * sdm + s] = den[i * sdm + s] * std::pow(2.0, l * deg[s]);
    dgemv_acc(m, n, ue2uc[o].data(), tmp.data(), chk, 1);
  }
  // :196-229
  void dwnChk2DwnEqu(int l, const double* chk, double* den) const {
    long m = (long)nDE * sdm, n = (long)nDC * tdm;
    std::vector<double> tmp(m, 0.0);
    dgemv_acc(m, n, dc2de.data(), chk, tmp.data(), 2);
    for (int i = 0; i < nDE; i++)
      for (int s = 0; s < sdm; s++) den[i * sdm + s] += tmp[i * sdm + s] * std::pow(2.0, -l * deg[s]);
  }
  // :231-274
  void dwnEqu2DwnChk(int l, int o, const double* den, double* chk) const {
    long m = (long)nDC * tdm, n = (long)nDE * sdm;
    std::vector<double> tmp(n);
    for (int i = 0; i < nDE; i++)
      for (int s = 0; s < sdm; s++) tmp[i * sdm + s] = den[i * sdm + s] * std::pow(2.0, l * deg[s]);
    dgemv_acc(m, n, de2dc[o].data(), tmp.data(), chk, 3);
  }
  // :276-331
  void plnDen2EffDen(int l, const double* plnDen, cplx* effDen) const {
    int n = 2 * np;
    std::vector<double> regDen((long)nReg * sdm, 0.0);
    int cnt = 0;
    for (int i = 0; i < np; i++)
      for (int j = 0; j < np; j++)
        for (int k = 0; k < np; k++)
          if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
            int rgoff = (k + np / 2) * n * n + (j + np / 2) * n + (i + np / 2);
            for (int f = 0; f < sdm; f++)
              regDen[(long)sdm * rgoff + f] += plnDen[sdm * cnt + f] * std::pow(2.0, l * deg[f]);
            cnt++;
          }
    rfft3(n, sdm, regDen.data(), effDen);
  }
  // :333-371
  void effVal2PlnVal(const cplx* effVal, double* plnVal) const {
    int n = 2 * np;
    std::vector<double> regVal((long)nReg * tdm);
    irfft3(n, tdm, effVal, regVal.data());
    int cnt = 0;
    for (int i = 0; i < np; i++)
      for (int j = 0; j < np; j++)
        for (int k = 0; k < np; k++)
          if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
            int rgoff = (k + np / 2) * n * n + (j + np / 2) * n + (i + np / 2);
            for (int f = 0; f < tdm; f++) plnVal[tdm * cnt + f] += regVal[(long)tdm * rgoff + f];
            cnt++;
          }
  }
  // :373-431 with cptwvv :502-512
  void upwEqu2DwnChk(const int* idx, const cplx* effDen, cplx* effVal) const {
    const cplx* mat = ue2dc[trans_id[idx[0] + 3][idx[1] + 3][idx[2] + 3]].data();
    double nrmfc = 1.0 / double(nReg);
    int matstp = sdm * tdm;
    for (int i = 0; i < tdm; i++)
      for (int j = 0; j < sdm; j++) {
        const cplx* x = mat + j * tdm + i;
        const cplx* y = effDen + j;
        cplx* z = effVal + i;
        for (int f = 0; f < nEff; f++) {
          double re = z->real() + nrmfc * (x->real() * y->real() - x->imag() * y->imag());
          double im = z->imag() + nrmfc * (x->real() * y->imag() + x->imag() * y->real());
          *z = cplx(re, im);
          x += matstp; y += sdm; z += tdm;
        }
      }
  }

  // ---------------------------------------------------------- evaluate
  // fmm3d_eval_mpi.cpp:396-1515 (CPU paths; MPI scatters are identities at 1
  // rank).  stage bits: 1 upward, 2 U, 4 V, 8 W, 16 X, 32 downward.
  void evaluate(const double* denIn, double* valOut, int stages) {
    const int nn = (int)nodes.size();
    const long ue = (long)nUE * sdm, uc = (long)nUC * tdm, de = (long)nDE * sdm, dc = (long)nDC * tdm;
    std::vector<double> den((long)ns * sd), val((long)nt * td, 0.0);
    for (long i = 0; i < ns; i++)
      for (int d = 0; d < sd; d++) den[i * sd + d] = denIn[srcPerm[i] * sd + d];
    std::vector<double> upChk((long)nn * uc, 0.0), upEqu((long)nn * ue, 0.0);
    std::vector<double> dnChk((long)nn * dc, 0.0), dnEqu((long)nn * de, 0.0);
    std::vector<int> byDepth[64];
    int maxd = 0;
    for (int i = 0; i < nn; i++) {
      byDepth[nodes[i].depth].push_back(i);
      maxd = std::max(maxd, nodes[i].depth);
    }
    std::vector<double> pos;
    // 3. upward, :557-595 (bottom-up = decreasing node index; with more than
    // one thread the same node set runs depth by depth)
    if (stages & 1) {
      for (int dpt = maxd; dpt >= 0; dpt--) {
        const std::vector<int>& lv = byDepth[dpt];
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) private(pos)
        for (long ii = (long)lv.size() - 1; ii >= 0; ii--) {
          int g = lv[ii];
          const Node& nd = nodes[g];
          if (!(nd.tag & CBTR)) continue;
          double* chk = &upChk[(long)g * uc];
          if (terminal(g)) {  // S2M, fmm3d_mpi.cpp:124-137
            loc_pos(1, g, pos);
            direct_accum(ktype, coefs, nd.srcNum, &srcPos[3L * nd.srcBeg], &srcNor[3L * nd.srcBeg],
                         &den[(long)nd.srcBeg * sd], nUC, pos.data(), chk);
          } else {  // M2M
            for (int o = 0; o < 8; o++) {
              int chi = nd.chd + o;
              if (nodes[chi].tag & CBTR)
                upwEqu2UpwChk(nodes[chi].depth + rootLevel, o, &upEqu[(long)chi * ue], chk);
            }
          }
          upwChk2UpwEqu(nd.depth + rootLevel, chk, &upEqu[(long)g * ue]);
        }
      }
    }
    // U-list, :773-785
    if (stages & 2) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
      for (int g = nn - 1; g >= 0; g--) {
        const Node& nd = nodes[g];
        if (!(nd.tag & EVTR) || !terminal(g)) continue;
        for (int v : nd.U) {
          const Node& sn = nodes[v];
          direct_accum(ktype, coefs, sn.srcNum, &srcPos[3L * sn.srcBeg], &srcNor[3L * sn.srcBeg],
                       &den[(long)sn.srcBeg * sd], nd.trgNum, &trgPos[3L * nd.trgBeg],
                       &val[(long)nd.trgBeg * td]);
        }
      }
    }
    // V-list, :1015-1051 (source spectra computed once per source node)
    if (stages & 4) {
      std::vector<int> effIdx(nn, -1);
      std::vector<int> srcs;
      for (int g = 0; g < nn; g++)
        if (nodes[g].tag & EVTR)
          for (int v : nodes[g].V)
            if (effIdx[v] < 0) { effIdx[v] = (int)srcs.size(); srcs.push_back(v); }
      std::vector<cplx> effDen((long)srcs.size() * nEff * sdm);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
      for (long s = 0; s < (long)srcs.size(); s++) {
        int v = srcs[s];
        plnDen2EffDen(nodes[v].depth + rootLevel, &upEqu[(long)v * ue], &effDen[s * nEff * sdm]);
      }
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
      for (int g = nn - 1; g >= 0; g--) {
        const Node& nd = nodes[g];
        if (!(nd.tag & EVTR) || nd.V.empty()) continue;
        double c[3];
        center(g, c);
        double D = 2.0 * radius(g);
        std::vector<cplx> effVal((long)nEff * tdm, cplx(0, 0));
        for (int v : nd.V) {
          double vc[3];
          center(v, vc);
          int idx[3];
          for (int d = 0; d < 3; d++) idx[d] = int(std::floor((vc[d] - c[d]) / D + 0.5));
          upwEqu2DwnChk(idx, &effDen[(long)effIdx[v] * nEff * sdm], effVal.data());
        }
        effVal2PlnVal(effVal.data(), &dnChk[(long)g * dc]);
      }
    }
    // W-list, :1134-1175
    if (stages & 8) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) private(pos)
      for (int g = 0; g < nn; g++) {
        const Node& nd = nodes[g];
        if (!(nd.tag & EVTR) || !terminal(g)) continue;
        for (int w : nd.W) {
          const Node& sn = nodes[w];
          if (sn.glbSrcExaNum > 0 && (long)sn.srcNum * sd < ue) {  // S2T
            direct_accum(ktype, coefs, sn.srcNum, &srcPos[3L * sn.srcBeg], &srcNor[3L * sn.srcBeg],
                         &den[(long)sn.srcBeg * sd], nd.trgNum, &trgPos[3L * nd.trgBeg],
                         &val[(long)nd.trgBeg * td]);
          } else {  // M2T, fmm3d_mpi.cpp:208-249
            loc_pos(0, w, pos);
            direct_accum(mmtype, coefs, nUE, pos.data(), pos.data(), &upEqu[(long)w * ue], nd.trgNum,
                         &trgPos[3L * nd.trgBeg], &val[(long)nd.trgBeg * td]);
          }
        }
      }
    }
    // X-list, :1241-1257
    if (stages & 16) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) private(pos)
      for (int g = 0; g < nn; g++) {
        const Node& nd = nodes[g];
        if (!(nd.tag & EVTR)) continue;
        for (int x : nd.X) {
          const Node& sn = nodes[x];
          if (terminal(g) && (long)nd.trgNum * td < dc) {  // S2T
            direct_accum(ktype, coefs, sn.srcNum, &srcPos[3L * sn.srcBeg], &srcNor[3L * sn.srcBeg],
                         &den[(long)sn.srcBeg * sd], nd.trgNum, &trgPos[3L * nd.trgBeg],
                         &val[(long)nd.trgBeg * td]);
          } else {  // S2L, fmm3d_mpi.cpp:142-154
            loc_pos(3, g, pos);
            direct_accum(ktype, coefs, sn.srcNum, &srcPos[3L * sn.srcBeg], &srcNor[3L * sn.srcBeg],
                         &den[(long)sn.srcBeg * sd], nDC, pos.data(), &dnChk[(long)g * dc]);
          }
        }
      }
    }
    // downward, :1368-1438 (top-down = increasing node index)
    if (stages & 32) {
      for (int dpt = 0; dpt <= maxd; dpt++) {
        const std::vector<int>& lv = byDepth[dpt];
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) private(pos)
        for (long ii = 0; ii < (long)lv.size(); ii++) {
          int g = lv[ii];
          const Node& nd = nodes[g];
          if (!(nd.tag & EVTR)) continue;
          if (nd.depth >= 3) {
            int p = nd.par;
            int o = (nd.path[0] - 2 * nodes[p].path[0]) * 4 + (nd.path[1] - 2 * nodes[p].path[1]) * 2 +
                    (nd.path[2] - 2 * nodes[p].path[2]);
            dwnEqu2DwnChk(nodes[p].depth + rootLevel, o, &dnEqu[(long)p * de], &dnChk[(long)g * dc]);
          }
          if (nd.depth >= 2) dwnChk2DwnEqu(nd.depth + rootLevel, &dnChk[(long)g * dc], &dnEqu[(long)g * de]);
          if (terminal(g)) {  // L2T, fmm3d_mpi.cpp:159-202
            loc_pos(2, g, pos);
            direct_accum(mmtype, coefs, nDE, pos.data(), pos.data(), &dnEqu[(long)g * de], nd.trgNum,
                         &trgPos[3L * nd.trgBeg], &val[(long)nd.trgBeg * td]);
          }
        }
      }
    }
    // 8. write values in the caller's order, :1492-1508
    for (long i = 0; i < nt * td; i++) valOut[i] = 0.0;
    for (long i = 0; i < nt; i++)
      for (int d = 0; d < td; d++) valOut[trgPerm[i] * td + d] = val[i * td + d];
  }
};

}  // namespace orc

using namespace orc;

// ---------------------------------------------------------------- C entry points
extern "C" {

int orc_src_dof(int kt) { return src_dof(kt); }
int orc_trg_dof(int kt) { return trg_dof(kt); }
int orc_mm_type(int kt) { return knl_mm_type(kt); }

void* orc_create(int kt, const double* coefs, int np, int ptsMax, int maxLevel, const double* ctr,
                 int rootLevel, int nthreads) {
  if (knl_mm_type(kt) < 0 || np < 2 || ptsMax < 1 || maxLevel < 1) return nullptr;
  Oracle* o = new Oracle();
  o->ktype = kt;
  o->mmtype = knl_mm_type(kt);
  o->coefs[0] = coefs ? coefs[0] : 1.0;
  o->coefs[1] = coefs ? coefs[1] : 0.25;
  o->np = np; o->ptsMax = ptsMax; o->maxLevel = maxLevel; o->rootLevel = rootLevel;
  o->nthreads = nthreads < 1 ? 1 : nthreads;
  for (int d = 0; d < 3; d++) o->ctr[d] = ctr ? ctr[d] : 0.5;
  o->sd = src_dof(kt); o->td = trg_dof(kt);
  o->sdm = src_dof(o->mmtype); o->tdm = trg_dof(o->mmtype);
  hom_deg(o->mmtype, o->deg);
  o->build_operators();
  return o;
}

void orc_destroy(void* h) { delete (Oracle*)h; }

int orc_setup(void* h, long ns, const double* src, const double* nrm, long nt, const double* trg) {
  Oracle* o = (Oracle*)h;
  o->setup(ns, src, nrm, nt, trg);
  return 0;
}

// One V-list interaction at level l through the oracle's M2L helpers: UE
// density den (|UE| srcDOF values) -> DC check values accumulated into val
// (|DC| trgDOF values), translation id tid (0..315).
int orc_m2l_single(void* h, int l, int tid, const double* den, double* val) {
  Oracle* o = (Oracle*)h;
  int idx[3] = {0, 0, 0};
  bool found = false;
  for (int t = 0; t < 343 && !found; t++)
    if (o->trans_id[t / 49][(t / 7) % 7][t % 7] == tid) {
      idx[0] = t / 49 - 3;
      idx[1] = (t / 7) % 7 - 3;
      idx[2] = t % 7 - 3;
      found = true;
    }
  if (!found) return -1;
  std::vector<cplx> effDen((long)o->nEff * o->sdm), effVal((long)o->nEff * o->tdm, cplx(0.0, 0.0));
  o->plnDen2EffDen(l, den, effDen.data());
  o->upwEqu2DwnChk(idx, effDen.data(), effVal.data());
  o->effVal2PlnVal(effVal.data(), val);
  return 0;
}

int orc_set_gemv_order(void* h, int order) {
  ((Oracle*)h)->gemvOrder = order & 15;
  return 0;
}

int orc_evaluate(void* h, const double* den, double* val, int stages) {
  ((Oracle*)h)->evaluate(den, val, stages);
  return 0;
}

// check(): dense FP64 sum over all sources at the given points
// (fmm3d_check_mpi.cpp:122-131); out is [nchk][trgDOF].
int orc_dense(int kt, const double* coefs, long ns, const double* src, const double* nrm,
              const double* den, long nchk, const double* pos, double* out, int nthreads) {
  double cf[2] = {coefs ? coefs[0] : 1.0, coefs ? coefs[1] : 0.25};
  const int td = trg_dof(kt);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads < 1 ? 1 : nthreads)
  for (long i = 0; i < nchk; i++) {
    for (int t = 0; t < td; t++) out[i * td + t] = 0.0;
    direct_accum(kt, cf, (int)ns, src, nrm, den, 1, pos + 3 * i, out + i * td);
  }
  return 0;
}

long orc_num_nodes(void* h) { return (long)((Oracle*)h)->nodes.size(); }

// per node: depth, path[3], par, chd, tag, srcCount, trgCount, leaf srcBeg/trgBeg
int orc_nodes(void* h, int* out /* [nn][11] */) {
  Oracle* o = (Oracle*)h;
  for (size_t i = 0; i < o->nodes.size(); i++) {
    const Node& n = o->nodes[i];
    int* r = out + 11 * i;
    r[0] = n.depth; r[1] = n.path[0]; r[2] = n.path[1]; r[3] = n.path[2];
    r[4] = n.par; r[5] = n.chd; r[6] = n.tag; r[7] = n.srcCount; r[8] = n.trgCount;
    r[9] = n.srcBeg; r[10] = n.trgBeg;
  }
  return 0;
}

// which: 0 U, 1 V, 2 W, 3 X.  ptr has nn+1 entries; idx may be null to size.
long orc_lists(void* h, int which, long* ptr, int* idx) {
  Oracle* o = (Oracle*)h;
  long tot = 0;
  for (size_t i = 0; i < o->nodes.size(); i++) {
    const Node& n = o->nodes[i];
    const std::vector<int>& L = which == 0 ? n.U : which == 1 ? n.V : which == 2 ? n.W : n.X;
    if (ptr) ptr[i] = tot;
    if (idx) for (size_t k = 0; k < L.size(); k++) idx[tot + k] = L[k];
    tot += (long)L.size();
  }
  if (ptr) ptr[o->nodes.size()] = tot;
  return tot;
}

// leaf-order permutations (leaf-order position -> caller index)
int orc_perms(void* h, long* srcPerm, long* trgPerm) {
  Oracle* o = (Oracle*)h;
  if (srcPerm) std::copy(o->srcPerm.begin(), o->srcPerm.end(), srcPerm);
  if (trgPerm) std::copy(o->trgPerm.begin(), o->trgPerm.end(), trgPerm);
  return 0;
}

// Operator tables.  which: 0 UC2UE pinv, 1 UE2UC (idx 0..7), 2 DC2DE pinv,
// 3 DE2DC (idx 0..7), 4 UE2DC spectrum (idx 0..315, complex as 2 doubles).
// Matrices are column-major like the reference NumMat.  Returns the number of
// doubles; a null buffer only sizes.
long orc_operator(void* h, int which, int idx, double* get, const double* set) {
  Oracle* o = (Oracle*)h;
  std::vector<double>* m = nullptr;
  if (which == 0) m = &o->uc2ue;
  else if (which == 1 && idx >= 0 && idx < 8) m = &o->ue2uc[idx];
  else if (which == 2) m = &o->dc2de;
  else if (which == 3 && idx >= 0 && idx < 8) m = &o->de2dc[idx];
  if (m) {
    if (get) std::copy(m->begin(), m->end(), get);
    if (set) std::copy(set, set + m->size(), m->begin());
    return (long)m->size();
  }
  if (which == 4 && idx >= 0 && idx < 316) {
    std::vector<cplx>& c = o->ue2dc[idx];
    if (get) std::memcpy(get, c.data(), sizeof(cplx) * c.size());
    if (set) std::memcpy((void*)c.data(), set, sizeof(cplx) * c.size());
    return 2L * (long)c.size();
  }
  return -1;
}

// sizes: nUE nUC nDE nDC nReg nEff
int orc_sizes(void* h, int* out) {
  Oracle* o = (Oracle*)h;
  out[0] = o->nUE; out[1] = o->nUC; out[2] = o->nDE; out[3] = o->nDC; out[4] = o->nReg; out[5] = o->nEff;
  return 0;
}

// stand-alone pieces for unit tests
int orc_kernel_matrix(int kt, const double* coefs, int ns, const double* src, const double* nrm, int nt,
                      const double* trg, double* out) {
  double cf[2] = {coefs ? coefs[0] : 1.0, coefs ? coefs[1] : 0.25};
  kernel_matrix(kt, cf, ns, src, nrm, nt, trg, out);
  return 0;
}
int orc_pinv(int m, int n, const double* A, double eps, double* R) {
  pinv(m, n, A, eps, R);
  return 0;
}
int orc_rfft3(int n, int howmany, const double* in, double* out) {
  rfft3(n, howmany, in, (cplx*)out);
  return 0;
}
int orc_irfft3(int n, int howmany, const double* in, double* out) {
  irfft3(n, howmany, (const cplx*)in, out);
  return 0;
}
int orc_sampos(int np, double R, double* out) {
  std::vector<double> p;
  sam_pos(np, R, p);
  if (out) std::copy(p.begin(), p.end(), out);
  return (int)p.size() / 3;
}
int orc_regpos(int np, double R, double* out) {
  std::vector<double> p;
  reg_pos(np, R, p);
  if (out) std::copy(p.begin(), p.end(), out);
  return (int)p.size() / 3;
}

}  // extern "C"
