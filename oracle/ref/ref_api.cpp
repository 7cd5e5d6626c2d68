// ref_api.cpp -- plain C entry points over the reference's OWN kernel and
// operator code (fmm3d_mpi/kernel3d_mpi.cpp, fmm3d_mpi/matmgnt3d_mpi.cpp,
// common/vecmatop.cpp, common/svdrep.cpp, compiled unchanged from the
// reference tree by oracle/ref/Makefile), so that the tests can pin the
// oracle's restatement against it.  Test infrastructure only: nothing in the
// product loads this library.
//
// Index conventions are the oracle's (oracle/kifmm_oracle.cpp orc_operator):
// octant o = 4a + 2b + c <-> Index3(a, b, c); translation id t counts the
// offsets (i1, i2, i3) in [-3, 3]^3 outside [-1, 1]^3 with i3 fastest, as
// fmm3d_eval_mpi.cpp:841-849 enumerates them.
#include <cstring>
#include <vector>

#include "fmm3d_mpi/kernel3d_mpi.hpp"
#include "fmm3d_mpi/matmgnt3d_mpi.hpp"

extern "C" {

// Kernel3d_MPI::buildKnlIntCtx (kernel3d_mpi.cpp:142-466): the dense block
// (nt*trgDOF) x (ns*srcDOF), column-major, into out.  Positions and normals
// are interleaved xyz (the reference's 3 x n column-major DblNumMat).
int fmmg_ref_kernel_matrix(int kt, const double* coefs, int ns, const double* src, const double* nrm, int nt,
                           const double* trg, double* out) {
  std::vector<double> cf(coefs, coefs + 2);
  Kernel3d_MPI knl(kt, cf);
  const int sd = knl.srcDOF(), td = knl.trgDOF();
  DblNumMat sp(3, ns), sn(3, ns), tp(3, nt), inter(nt * td, ns * sd);
  std::memcpy(sp.data(), src, sizeof(double) * 3 * ns);
  std::memcpy(sn.data(), nrm, sizeof(double) * 3 * ns);
  std::memcpy(tp.data(), trg, sizeof(double) * 3 * nt);
  const int e = knl.buildKnlIntCtx(sp, sn, tp, inter);
  if (e) return e;
  std::memcpy(out, inter.data(), sizeof(double) * (size_t)nt * td * ns * sd);
  return 0;
}

// MatMgnt3d_MPI::samPosCal / regPosCal (matmgnt3d_mpi.cpp:451-499): returns
// the number of points; out (3 doubles a point) may be NULL to size.
int fmmg_ref_sampos(int np, double R, double* out) {
  MatMgnt3d_MPI mm;
  DblNumMat pos;
  if (mm.samPosCal(np, R, pos)) return -1;
  if (out) std::memcpy(out, pos.data(), sizeof(double) * 3 * pos.n());
  return pos.n();
}

int fmmg_ref_regpos(int np, double R, double* out) {
  MatMgnt3d_MPI mm;
  DblNumMat pos;
  if (mm.regPosCal(np, R, pos)) return -1;
  if (out) std::memcpy(out, pos.data(), sizeof(double) * 3 * pos.n());
  return pos.n();
}

// The operator tables the reference's MatMgnt3d_MPI builds for the
// equivalent kernel kt and order np, at level 0 (the homogeneous kernels keep
// one table set).  which: 0 UC->UE pseudo-inverse, 1 UE->UC (octant idx),
// 2 DC->DE pseudo-inverse, 3 DE->DC (octant idx), 4 UE->DC translation
// spectrum (translation id idx; complex as pairs, the DOF pair fastest then
// the r2c frequency).  Each table is built by the reference's own *_dgemv
// call on a zero vector, then copied out.  Returns the number of doubles
// (out may be NULL to size), or -1.
long fmmg_ref_operator(int kt, const double* coefs, int np, int which, int idx, double* out) {
  std::vector<double> cf(coefs, coefs + 2);
  MatMgnt3d_MPI* mm = MatMgnt3d_MPI::getmmptr(Kernel3d_MPI(kt, cf), np);
  const int sd = mm->srcDOF(), td = mm->trgDOF();
  const DblNumMat* m = nullptr;
  if (which == 0) {
    DblNumVec chk(td * mm->samPos(MatMgnt3d_MPI::UC).n()), den(sd * mm->samPos(MatMgnt3d_MPI::UE).n());
    clear(chk);
    clear(den);
    if (mm->UpwChk2UpwEqu_dgemv(0, chk, den)) return -1;
    m = &mm->_upwChk2UpwEqu[0];
  } else if (which == 2) {
    DblNumVec chk(td * mm->samPos(MatMgnt3d_MPI::DC).n()), den(sd * mm->samPos(MatMgnt3d_MPI::DE).n());
    clear(chk);
    clear(den);
    if (mm->DwnChk2DwnEqu_dgemv(0, chk, den)) return -1;
    m = &mm->_dwnChk2DwnEqu[0];
  } else if ((which == 1 || which == 3) && idx >= 0 && idx < 8) {
    Index3 ii(idx >> 2, (idx >> 1) & 1, idx & 1);
    if (which == 1) {
      DblNumVec den(sd * mm->samPos(MatMgnt3d_MPI::UE).n()), chk(td * mm->samPos(MatMgnt3d_MPI::UC).n());
      clear(den);
      clear(chk);
      if (mm->UpwEqu2UpwChk_dgemv(0, ii, den, chk)) return -1;
      m = &mm->_upwEqu2UpwChk[0](ii(0), ii(1), ii(2));
    } else {
      DblNumVec den(sd * mm->samPos(MatMgnt3d_MPI::DE).n()), chk(td * mm->samPos(MatMgnt3d_MPI::DC).n());
      clear(den);
      clear(chk);
      if (mm->DwnEqu2DwnChk_dgemv(0, ii, den, chk)) return -1;
      m = &mm->_dwnEqu2DwnChk[0](ii(0), ii(1), ii(2));
    }
  } else if (which == 4 && idx >= 0 && idx < 316) {
    int cnt = 0, t1 = 0, t2 = 0, t3 = 0;
    for (int i1 = -3; i1 <= 3; i1++)
      for (int i2 = -3; i2 <= 3; i2++)
        for (int i3 = -3; i3 <= 3; i3++)
          if (std::abs(i1) > 1 || std::abs(i2) > 1 || std::abs(i3) > 1) {
            if (cnt == idx) {
              t1 = i1;
              t2 = i2;
              t3 = i3;
            }
            cnt++;
          }
    Index3 ii(t1, t2, t3);
    DblNumVec effDen(mm->effDatSze(MatMgnt3d_MPI::UE)), effVal(mm->effDatSze(MatMgnt3d_MPI::DC));
    clear(effDen);
    clear(effVal);
    if (mm->UpwEqu2DwnChk_dgemv(0, ii, effDen, effVal)) return -1;
    m = &mm->_upwEqu2DwnChk[0](t1, t2, t3);
  }
  if (!m) return -1;
  const long cntD = (long)m->m() * m->n();
  if (out) std::memcpy(out, m->data(), sizeof(double) * cntD);
  return cntD;
}

// One V-list interaction through the reference's own pipeline at level l:
// plnDen2EffDen (scale, embed in the (2np)^3 grid, r2c FFT),
// UpwEqu2DwnChk_dgemv (the Hadamard product with translation idx), and
// effVal2PlnVal (c2r FFT, gather the DC surface), matmgnt3d_mpi.cpp:276-431.
// den has |UE| * srcDOF values, val receives |DC| * trgDOF (accumulated).
int fmmg_ref_m2l(int kt, const double* coefs, int np, int l, int idx, const double* den, double* val) {
  std::vector<double> cf(coefs, coefs + 2);
  MatMgnt3d_MPI* mm = MatMgnt3d_MPI::getmmptr(Kernel3d_MPI(kt, cf), np);
  const int sd = mm->srcDOF(), td = mm->trgDOF();
  int cnt = 0, t[3] = {0, 0, 0};
  for (int i1 = -3; i1 <= 3; i1++)
    for (int i2 = -3; i2 <= 3; i2++)
      for (int i3 = -3; i3 <= 3; i3++)
        if (std::abs(i1) > 1 || std::abs(i2) > 1 || std::abs(i3) > 1) {
          if (cnt == idx) {
            t[0] = i1;
            t[1] = i2;
            t[2] = i3;
          }
          cnt++;
        }
  DblNumVec plnDen(sd * mm->samPos(MatMgnt3d_MPI::UE).n()), plnVal(td * mm->samPos(MatMgnt3d_MPI::DC).n());
  std::memcpy(plnDen.data(), den, sizeof(double) * plnDen.m());
  std::memcpy(plnVal.data(), val, sizeof(double) * plnVal.m());
  DblNumVec effDen(mm->effDatSze(MatMgnt3d_MPI::UE)), effVal(mm->effDatSze(MatMgnt3d_MPI::DC));
  clear(effDen);
  clear(effVal);
  if (mm->plnDen2EffDen(l, plnDen, effDen)) return -1;
  if (mm->UpwEqu2DwnChk_dgemv(l, Index3(t[0], t[1], t[2]), effDen, effVal)) return -1;
  if (mm->effVal2PlnVal(l, effVal, plnVal)) return -1;
  std::memcpy(val, plnVal.data(), sizeof(double) * plnVal.m());
  return 0;
}

}  // extern "C"
