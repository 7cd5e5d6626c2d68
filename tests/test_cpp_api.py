"""The C++ FMM3d class (include/fmmg_fmm3d.hpp) compiles against libfmmg.so and
drives the reference's setup()/evaluate()/check() sequence."""
import os
import subprocess

import pytest

import fmmg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <random>
#include "fmmg_fmm3d.hpp"
int main(int argc, char** argv) {
  int device = argc > 1 ? atoi(argv[1]) : 0;
  fmmg::FMM3d fmm;
  std::mt19937_64 g(7);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  const int n = 3000;
  for (int i = 0; i < 3 * n; i++) fmm.srcPos().push_back(u(g));
  fmm.trgPos() = fmm.srcPos();
  fmm.knl() = fmmg::Kernel3d(111, {1.0, 0.25});
  fmm.np() = 4; fmm.ptsMax() = 40; fmm.device() = device;
  int s = fmm.setup();
  if (s) { printf("setup %d %s\n", s, fmm.lastError()); return 1; }
  std::vector<double> den(n), val;
  for (auto& d : den) d = u(g) * 2 - 1;
  // the points move: the same object set up again (same options: the handle
  // is kept), then with another order (a new handle)
  for (int pass = 0; pass < 3; pass++) {
    if (pass > 0) {
      for (auto& x : fmm.srcPos()) x = 0.9 * x + 0.05;
      fmm.trgPos() = fmm.srcPos();
      if (pass == 2) fmm.np() = 5;
      s = fmm.setup();
      if (s) { printf("setup again %d %s\n", s, fmm.lastError()); return 5; }
    }
    s = fmm.evaluate(den, val);
    if (device < 0) {
      if (s != FMMG_STATE) { printf("evaluate status %d\n", s); return 2; }
      continue;
    }
    if (s) { printf("evaluate %d %s\n", s, fmm.lastError()); return 3; }
    double rerr = 1;
    s = fmm.check(den, val, 500, rerr);
    printf("rerr %.3e\n", rerr);
    if (s != 0 || rerr >= 1e-3) return 4;
  }
  return 0;
}
"""


def _build(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    libdir = os.path.dirname(fmmg.LIB_PATH)
    subprocess.check_call(["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src),
                           "-L", libdir, "-lfmmg", "-Wl,-rpath," + libdir, "-o", str(exe)])
    return exe


def test_cpp_class_host_plan(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), "-1"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_class_evaluate_and_check(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), "0"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
