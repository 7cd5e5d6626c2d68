// fmmg_fmm3d.hpp -- a C++ class with the member names and meaning of the
// reference FMM3d_MPI (fmm3d_mpi/fmm3d_mpi.hpp:36-249, knlmat3d_mpi.hpp:40-70),
// single rank, no PETSc: std::vector<double> replaces Vec.  Header-only over
// the C ABI of fmmg.h.
//
//   fmmg::FMM3d fmm;                      // FMM3d_MPI("fmm3d_")
//   fmm.srcPos() = ...; fmm.srcNor() = ...; fmm.trgPos() = ...;   // xyz interleaved
//   fmm.knl() = fmmg::Kernel3d(111, {1.0, 0.25});
//   fmm.ctr() = {0.5, 0.5, 0.5}; fmm.rootLevel() = 1;
//   fmm.np() = 6; fmm.ptsMax() = 64; fmm.maxLevel() = 30;   // -fmm3d_np, -fmm3d_let3d_*
//   fmm.setup();                          // FMM3d_MPI::setup()
//   fmm.evaluate(srcDen, trgVal);         // FMM3d_MPI::evaluate(Vec, Vec)
//   fmm.check(srcDen, trgVal, 1000, rerr);// FMM3d_MPI::check(...)
//
// Differences from the reference, by design: the caller's vectors are not
// replaced by redistributed ones in setup() (at one rank the order is the
// input order anyway), and every method returns the fmmg_status code (0 = OK)
// instead of a PETSc error; lastError() gives the message.
#pragma once

#include <array>
#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "fmmg.h"

namespace fmmg {

// Kernel3d_MPI{kernelType, coefs} (fmm3d_mpi/kernel3d_mpi.hpp:81-125)
struct Kernel3d {
  int type = FMMG_KNL_LAP_S_U;
  std::vector<double> coefs{1.0, 0.25};
  Kernel3d() = default;
  Kernel3d(int t, std::vector<double> c) : type(t), coefs(std::move(c)) {}
  int& kernelType() { return type; }
  int srcDOF() const { return type == 111 || type == 121 ? 1 : 3; }
  int trgDOF() const { return type == 111 || type == 121 || type == 312 || type == 322 ? 1 : 3; }
};

class FMM3d {
 public:
  FMM3d() {
    fmmg_default_options(&opt_);
    made_ = opt_;
  }
  ~FMM3d() { fmmg_destroy(h_); }
  FMM3d(const FMM3d&) = delete;
  FMM3d& operator=(const FMM3d&) = delete;

  std::vector<double>& srcPos() { return src_; }
  std::vector<double>& srcNor() { return nrm_; }
  std::vector<double>& trgPos() { return trg_; }
  Kernel3d& knl() { return knl_; }
  std::array<double, 3>& ctr() { return ctr_; }
  int& rootLevel() { return opt_.root_level; }
  int& np() { return opt_.np; }
  int& ptsMax() { return opt_.pts_max; }
  int& maxLevel() { return opt_.max_level; }
  int& device() { return opt_.device; }
  int srcDOF() const { return knl_.srcDOF(); }
  int trgDOF() const { return knl_.trgDOF(); }
  const char* lastError() const { return fmmg_last_error(h_); }
  fmmg_handle* handle() { return h_; }

  // FMM3d_MPI::setup(): tree, lists, operators, device upload.  Called again
  // with the same kernel and options (points that moved), the handle is set
  // up again in place: it keeps its operator tables and device context.
  int setup() {
    opt_.kernel_type = knl_.type;
    opt_.coefs[0] = knl_.coefs.size() > 0 ? knl_.coefs[0] : 1.0;
    opt_.coefs[1] = knl_.coefs.size() > 1 ? knl_.coefs[1] : 0.25;
    for (int d = 0; d < 3; d++) opt_.ctr[d] = ctr_[d];
    if (!h_ || !same_options(opt_, made_)) {
      fmmg_destroy(h_);
      h_ = nullptr;
      fmmg_status s = fmmg_create(&opt_, &h_);
      if (s != FMMG_OK) return s;
      made_ = opt_;
    }
    if (src_.size() % 3 || trg_.size() % 3) return FMMG_INVALID_ARG;
    return fmmg_setup(h_, (int64_t)src_.size() / 3, src_.data(), nrm_.empty() ? nullptr : nrm_.data(),
                      (int64_t)trg_.size() / 3, trg_.data());
  }

  // FMM3d_MPI::evaluate(srcDen, trgVal): trgVal is overwritten
  int evaluate(const std::vector<double>& srcDen, std::vector<double>& trgVal) {
    if (srcDen.size() != src_.size() / 3 * srcDOF()) return FMMG_INVALID_ARG;
    trgVal.assign(trg_.size() / 3 * trgDOF(), 0.0);
    return fmmg_evaluate(h_, srcDen.data(), trgVal.data());
  }

  // FMM3d_MPI::check(srcDen, trgVal, numChk, rerr): relative L2 error at
  // numChk random targets against the dense sum (all targets if numChk >= n)
  int check(const std::vector<double>& srcDen, const std::vector<double>& trgVal, int64_t numChk, double& rerr,
            unsigned seed = 1) {
    const int64_t nt = (int64_t)trg_.size() / 3;
    std::vector<int64_t> idx;
    if (numChk >= nt) {
      for (int64_t k = 0; k < nt; k++) idx.push_back(k);
    } else {
      std::mt19937_64 g(seed);
      std::uniform_int_distribution<int64_t> u(0, nt - 1);
      for (int64_t k = 0; k < numChk; k++) idx.push_back(u(g));
    }
    double maxAbs = 0;
    return fmmg_check(h_, srcDen.data(), trgVal.data(), (int64_t)idx.size(), idx.data(), &rerr, &maxAbs, nullptr);
  }

 private:
  static bool same_options(const fmmg_options& a, const fmmg_options& b) {
    return a.kernel_type == b.kernel_type && a.coefs[0] == b.coefs[0] && a.coefs[1] == b.coefs[1] &&
           a.np == b.np && a.pts_max == b.pts_max && a.max_level == b.max_level && a.ctr[0] == b.ctr[0] &&
           a.ctr[1] == b.ctr[1] && a.ctr[2] == b.ctr[2] && a.root_level == b.root_level && a.device == b.device &&
           a.stream == b.stream;
  }
  fmmg_options opt_;
  fmmg_options made_;  // the options h_ was created with
  fmmg_handle* h_ = nullptr;
  Kernel3d knl_;
  std::array<double, 3> ctr_{0.5, 0.5, 0.5};
  std::vector<double> src_, nrm_, trg_;
};

}  // namespace fmmg
