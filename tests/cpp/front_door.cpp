// The reference's C++ call sequence through pbbfmm3d_b200.hpp:
//   kernel_X Atree(...); Atree.buildFMMTree();
//   H2_3D_Compute<kernel_X>(Atree, target, source, weight, nCols, output);
// checked against a float64 direct sum on sampled targets.  Exit 0 and
// "OK" on success.  Usage: front_door [--no-run]  (--no-run: construct
// nothing, only proves the program compiles and links).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>

#include "pbbfmm3d_b200.hpp"

namespace fmm = pbbfmm3d_b200;

// the reference's own point type, as a caller would have it
struct vector3 {
  double x, y, z;
};

static double direct_rel_err(const std::vector<vector3>& T, const std::vector<vector3>& S,
                             const std::vector<double>& w, int C, const std::vector<double>& out,
                             double (*k)(double)) {
  double num = 0, den = 0;
  for (size_t i = 0; i < T.size(); i += 37)
    for (int c = 0; c < C; ++c) {
      double acc = 0;
      for (size_t j = 0; j < S.size(); ++j) {
        const double dx = S[j].x - T[i].x, dy = S[j].y - T[i].y, dz = S[j].z - T[i].z;
        const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
        const double kv = k(r);
        if (std::isfinite(kv)) acc += kv * w[c * S.size() + j];
      }
      const double d = out[c * T.size() + i] - acc;
      num += d * d;
      den += acc * acc;
    }
  return std::sqrt(num / den);
}

static double lap(double r) { return 1.0 / r; }
static double expcov(double r) { return std::exp(-r / 0.3); }

int main(int argc, char** argv) {
  if (argc > 1 && !std::strcmp(argv[1], "--no-run")) {
    std::printf("linked %s\n", pbbfmm_version());
    return 0;
  }
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> u(-0.5, 0.5);
  const int N = 4000;
  std::vector<vector3> pts(N);
  for (auto& p : pts) p = {u(rng), u(rng), u(rng)};
  try {
    // Laplacian, Chebyshev, FP64, one column (the reference's example shape)
    fmm::kernel_Laplacian t1(1.0, 4, 4, 1e-5, 1);
    t1.buildFMMTree();
    std::vector<double> w1(N), o1(N, 0.0);
    for (auto& v : w1) v = u(rng) + 0.5;
    fmm::H2_3D_Compute(t1, pts, pts, w1, 1, o1);
    const double e1 = direct_rel_err(pts, pts, w1, 1, o1, lap);
    // the same tree in mixed precision: Chebyshev M2L on the tensor cores
    t1.set_precision(PBBFMM_PREC_MIXED);
    const bool on_tc = t1.tensor_core_m2l() == PBBFMM_TC_F16;
    std::vector<double> o1m(N, 0.0);
    fmm::H2_3D_Compute(t1, pts, pts, w1, 1, o1m);
    const double e1m = direct_rel_err(pts, pts, w1, 1, o1m, lap);
    // exp(-r/0.3), uniform interpolation with FFT M2L, mixed precision, 3 columns
    fmm::kernel_ExpCov t2(1.0, 4, 5, 1e-5, 0, 0.3);
    t2.buildFMMTree();
    t2.set_precision(PBBFMM_PREC_MIXED);
    std::vector<double> w2(3 * N), o2(3 * N, 0.0);
    for (auto& v : w2) v = u(rng);
    fmm::H2_3D_Compute(t2, pts, pts, w2, 3, o2);
    const double e2 = direct_rel_err(pts, pts, w2, 3, o2, expcov);
    // errors come back as exceptions, not exits
    bool threw = false;
    try {
      fmm::kernel_Laplacian bad(1.0, 1, 4, 1e-5, 1);  // tree_level < 2
    } catch (const fmm::Error& e) {
      threw = e.status == PBBFMM_ERR_ARG;
    }
    std::printf(
        "laplace_cheb rel %.3e  laplace_cheb_mixed (tensor cores %d) rel %.3e  "
        "expcov_unif_mixed rel %.3e  bad-args threw %d\n",
        e1, (int)on_tc, e1m, e2, (int)threw);
    if (e1 < 1e-4 && on_tc && e1m < 1e-4 && e2 < 1e-4 && threw) {
      std::printf("OK\n");
      return 0;
    }
    return 1;
  } catch (const std::exception& e) {
    std::printf("error: %s\n", e.what());
    return 2;
  }
}
