"""A compiled C++ caller of the C ABI, linked against libfpe_engine.so.

The program wraps the reference's 16-symbol C interface the way a C++ user of
the reference does (an owning pipeline class that throws when create returns
NULL and converts every result struct to std::vector, freeing it with the
matching fpe_compute_free_* call; reference cpp/include/fpe_compute.hpp:38-262
and cpp/examples/demo.cpp), written here for this test.  The CPU test builds
and links it; the GPU test runs it and checks the one-shot prices and Greeks
against the reference README's table (README.md:380-392) and the stepwise
prices and Greeks against the CPU oracle.
"""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "fpe_option_b200")

PROGRAM = r"""
#include <cstdio>
#include <stdexcept>
#include <vector>
#include "fpe_engine.h"

namespace {

std::vector<double> take(FpeVecResult& r) {
  std::vector<double> v(r.data, r.data + (r.len > 0 ? r.len : 0));
  fpe_compute_free_vec(&r);
  return v;
}

struct Greeks { std::vector<double> delta, gamma, vega; };

// Owns one stepwise pipeline; the library allocates every result and the
// matching free call releases it.
class Pipeline {
 public:
  Pipeline(double kappa, double theta, double sigma, double rho, double r, double T, double S0, double V0,
           int n_s, int n_v, double barrier, int type, int num_insert, double s_min, double s_max)
      : h_(fpe_compute_create(kappa, theta, sigma, rho, r, T, S0, V0, n_s, n_v, barrier, type, num_insert,
                              s_min, s_max)) {
    if (!h_) throw std::runtime_error("fpe_compute_create returned NULL");
  }
  ~Pipeline() { fpe_compute_destroy(h_); }
  Pipeline(const Pipeline&) = delete;
  Pipeline& operator=(const Pipeline&) = delete;

  std::vector<double> price(const std::vector<double>& K) {
    FpeVecResult r;
    fpe_compute_price(h_, K.data(), int32_t(K.size()), &r);
    return take(r);
  }
  Greeks greeks(const std::vector<double>& K) {
    FpeGreeksResult r;
    fpe_compute_greeks(h_, K.data(), int32_t(K.size()), 0.0, 0.0, &r);
    Greeks g;
    g.delta.assign(r.delta, r.delta + r.len);
    g.gamma.assign(r.gamma, r.gamma + r.len);
    g.vega.assign(r.vega, r.vega + r.len);
    fpe_compute_free_greeks(&r);
    return g;
  }
  size_t knots() {
    FpeVec2Result r;
    fpe_compute_knots(h_, &r);
    const size_t n = size_t(r.s_len) + size_t(r.v_len);
    fpe_compute_free_vec2(&r);
    return n;
  }
  size_t pdf_points() {
    FpeMatResult r;
    fpe_compute_pdf(h_, &r);
    const size_t n = size_t(r.n_rows) * size_t(r.n_cols);
    fpe_compute_free_mat(&r);
    return n;
  }

 private:
  FpeCompute* h_;
};

void print_list(const char* key, const std::vector<double>& v, bool last = false) {
  std::printf("\"%s\": [", key);
  for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i]);
  std::printf("]%s\n", last ? "" : ",");
}

}  // namespace

int main() {
  const std::vector<double> K = {80.0, 90.0, 100.0};
  FpeOneshotResult one;
  fpe_price_oneshot(1.2, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, 0.1, K.data(), 3, 0.0, 8, 38, 38, 50, 0.0, 150.0, &one);
  if (one.len != 3) return 2;
  std::printf("{\n");
  print_list("oneshot_price", std::vector<double>(one.price, one.price + 3));
  print_list("oneshot_delta", std::vector<double>(one.delta, one.delta + 3));
  print_list("oneshot_gamma", std::vector<double>(one.gamma, one.gamma + 3));
  print_list("oneshot_vega", std::vector<double>(one.vega, one.vega + 3));
  fpe_compute_free_oneshot(&one);
  bool threw = false;
  try {
    Pipeline bad(-1.0, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, 0.1, 10, 10, 0.0, 8, 50, 0.0, 150.0);
  } catch (const std::runtime_error&) {
    threw = true;
  }
  Pipeline p(1.2, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, 0.1, 12, 12, 50.0, 2, 50, 0.0, 150.0);
  const std::vector<double> Kc = {56.0, 62.0};
  print_list("compute_price", p.price(Kc));
  const Greeks g = p.greeks(Kc);
  print_list("compute_delta", g.delta);
  print_list("compute_gamma", g.gamma);
  print_list("compute_vega", g.vega);
  std::printf("\"knots\": %zu, \"pdf_points\": %zu, \"invalid_threw\": %s\n}\n", p.knots(), p.pdf_points(),
              threw ? "true" : "false");
  return 0;
}
"""


def _build(tmp_path):
    from fpe_option_b200 import build

    build.build_library()
    src = tmp_path / "caller.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", LIBDIR, "-lfpe_engine", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_cpp_caller_builds_and_links(tmp_path):
    exe = _build(tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_cpp_caller_runs(tmp_path, engine, oracle):
    exe = _build(tmp_path)
    out = json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    # README.md:380-392, printed to 6 decimals
    np.testing.assert_allclose(out["oneshot_price"], [0.966276, 0.280919, 0.078883], atol=6e-7)
    np.testing.assert_allclose(out["oneshot_delta"], [0.175855, 0.060298, 0.018875], atol=6e-7)
    np.testing.assert_allclose(out["oneshot_gamma"], [0.017766, 0.009270, 0.002742], atol=6e-7)
    np.testing.assert_allclose(out["oneshot_vega"], [14.057144, 6.197252, 2.283113], atol=6e-6)
    assert out["invalid_threw"] is True
    assert out["knots"] > 0 and out["pdf_points"] > 0
    H = (1.2, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, 0.1)
    pipe = oracle.Pipeline(*H, n_s=12, n_v=12, barrier=50.0, option_type=2, s_max=150.0,
                           opt=oracle.options(num_insert=50))
    np.testing.assert_allclose(out["compute_price"], pipe.price_at([56.0, 62.0]), rtol=1e-9)
    d, g, v = pipe.greeks([56.0, 62.0])
    np.testing.assert_allclose(out["compute_delta"], d, rtol=1e-7, atol=1e-10)
    np.testing.assert_allclose(out["compute_gamma"], g, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(out["compute_vega"], v, rtol=1e-7, atol=1e-10)
