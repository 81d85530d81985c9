// Command-line driver around the UNMODIFIED reference PBBFMM3D matvec
// (test infrastructure only; built by oracle/ref/Makefile into oracle/_ref/).
//
// It does what the reference examples do (examples/binary_file_standard_kernel.cpp:
// read inputs, `kernel_X Atree(L, level, order, eps, cheb); Atree.buildFMMTree();
// H2_3D_Compute<kernel_X> compute(Atree, target, source, weight, nCols, output);`)
// but takes every parameter from the command line and writes the output as raw
// float64 (column-major Nf x nCols, the layout of include/compute.hpp:747).
//
// Kernels beyond src/kernel_Types.cpp are added the way the reference README
// documents user kernels (subclass H2_3D_Tree, define SetKernelProperty and
// EvaluateKernel; README.md:178-227).  Their kernelType strings encode the
// parameter so the operator cache (src/H2_3D_Tree.cpp:84-91) is never stale.
//
// Timing: the reference cannot reuse a tree for a second compute (the per-call
// node state is never reset, include/compute.hpp:1176-1179, 1094-1099), so
// --repeat R rebuilds the tree before every compute, as app/fmm.hpp:80-82 does,
// and times only the H2_3D_Compute constructor with omp_get_wtime.
#include "bbfmm3d.hpp"

#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

class kernel_ExpCov : public H2_3D_Tree {  // exp(-r / ell)
 public:
  double ell;
  kernel_ExpCov(double L, int lv, int n, double eps, int cheb, double ell_)
      : H2_3D_Tree(L, lv, n, eps, cheb), ell(ell_) {}
  void SetKernelProperty() override {
    homogen = 0;
    symmetry = 1;
    char buf[32];
    snprintf(buf, sizeof buf, "ExpCov%g", ell);
    kernelType = buf;
  }
  double EvaluateKernel(const vector3& t, const vector3& s) override {
    double dx = s.x - t.x, dy = s.y - t.y, dz = s.z - t.z;
    return exp(-sqrt(dx * dx + dy * dy + dz * dz) / ell);
  }
};

class kernel_GaussSigma : public H2_3D_Tree {  // exp(-r^2 / (2 sigma^2))
 public:
  double sigma;
  kernel_GaussSigma(double L, int lv, int n, double eps, int cheb, double s)
      : H2_3D_Tree(L, lv, n, eps, cheb), sigma(s) {}
  void SetKernelProperty() override {
    homogen = 0;
    symmetry = 1;
    char buf[32];
    snprintf(buf, sizeof buf, "GaussS%g", sigma);
    kernelType = buf;
  }
  double EvaluateKernel(const vector3& t, const vector3& s) override {
    double dx = s.x - t.x, dy = s.y - t.y, dz = s.z - t.z;
    return exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * sigma * sigma));
  }
};

class kernel_AnisoExp : public H2_3D_Tree {  // python/mykernel_python.hpp:10-18
 public:
  kernel_AnisoExp(double L, int lv, int n, double eps, int cheb)
      : H2_3D_Tree(L, lv, n, eps, cheb) {}
  void SetKernelProperty() override {
    homogen = 0;
    symmetry = 1;
    kernelType = "AnisoExp";
  }
  double EvaluateKernel(const vector3& t, const vector3& s) override {
    double dx = s.x - t.x, dy = s.y - t.y, dz = s.z - t.z;
    double r = sqrt(dx * dx / 100. + dy * dy / 100. + dz * dz / 2.25);
    return 0.75 * exp(-r);
  }
};

// The softened Laplacian 1/sqrt(r^2 + delta^2): a kernel outside the
// library's built-in set, used to check user-defined device kernels.
class kernel_SoftLap : public H2_3D_Tree {
 public:
  double delta;
  kernel_SoftLap(double L, int lv, int n, double eps, int cheb, double d)
      : H2_3D_Tree(L, lv, n, eps, cheb), delta(d) {}
  void SetKernelProperty() override {
    homogen = 0;
    symmetry = 1;
    char buf[32];
    snprintf(buf, sizeof buf, "SoftLap%g", delta);
    kernelType = buf;
  }
  double EvaluateKernel(const vector3& t, const vector3& s) override {
    double dx = s.x - t.x, dy = s.y - t.y, dz = s.z - t.z;
    return 1. / sqrt(dx * dx + dy * dy + dz * dz + delta * delta);
  }
};

struct Args {
  std::string kernel = "Laplacian";
  double param = 0.0;
  double L = 1.0;
  int level = 3, order = 4, cheb = 1, ncols = 1, nf = 0, ns = 0, repeat = 1;
  double eps = 1e-5;
  std::string target, source, weight, out, workdir = ".", timing;
};

void die(const char* msg) {
  fprintf(stderr, "ref_fmm: %s\n", msg);
  exit(2);
}

std::string absolute(const std::string& p) {
  if (p.empty() || p[0] == '/') return p;
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd)) die("getcwd failed");
  return std::string(cwd) + "/" + p;
}

void read_points(const std::string& f, std::vector<vector3>& v, int n) {
  // column-wise layout: all x, then all y, then all z (README.md:318-351)
  FILE* fp = fopen(f.c_str(), "rb");
  if (!fp) die(("cannot open " + f).c_str());
  std::vector<double> buf(3 * (size_t)n);
  if (fread(buf.data(), sizeof(double), buf.size(), fp) != buf.size()) die("short read (points)");
  fclose(fp);
  v.resize(n);
  for (int i = 0; i < n; ++i) v[i] = vector3(buf[i], buf[n + i], buf[2 * (size_t)n + i]);
}

void read_doubles(const std::string& f, std::vector<double>& v, size_t n) {
  FILE* fp = fopen(f.c_str(), "rb");
  if (!fp) die(("cannot open " + f).c_str());
  v.resize(n);
  if (fread(v.data(), sizeof(double), n, fp) != n) die("short read (weights)");
  fclose(fp);
}

template <typename T, typename Make>
void run(const Args& a, Make make, const std::vector<vector3>& target,
         const std::vector<vector3>& source, std::vector<double>& weight,
         std::vector<double>& output, std::vector<double>& times, double& tpre) {
  for (int rep = 0; rep < a.repeat; ++rep) {
    std::vector<double> out(output.size(), 0.0);
    double t0 = omp_get_wtime();
    T* tree = make();
    tree->buildFMMTree();
    double t1 = omp_get_wtime();
    {
      H2_3D_Compute<T> compute(*tree, target, source, weight, a.ncols, out);
    }
    double t2 = omp_get_wtime();
    if (rep == 0) {
      output = out;
      tpre = t1 - t0;
    }
    times.push_back(t2 - t1);
    delete tree;
  }
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; ++i) {
    std::string k = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) die(("missing value for " + k).c_str());
      return argv[++i];
    };
    if (k == "--kernel") a.kernel = next();
    else if (k == "--param") a.param = atof(next());
    else if (k == "--L") a.L = atof(next());
    else if (k == "--level") a.level = atoi(next());
    else if (k == "--order") a.order = atoi(next());
    else if (k == "--eps") a.eps = atof(next());
    else if (k == "--cheb") a.cheb = atoi(next());
    else if (k == "--ncols") a.ncols = atoi(next());
    else if (k == "--nf") a.nf = atoi(next());
    else if (k == "--ns") a.ns = atoi(next());
    else if (k == "--target") a.target = absolute(next());
    else if (k == "--source") a.source = absolute(next());
    else if (k == "--weight") a.weight = absolute(next());
    else if (k == "--out") a.out = absolute(next());
    else if (k == "--timing") a.timing = absolute(next());
    else if (k == "--workdir") a.workdir = absolute(next());
    else if (k == "--repeat") a.repeat = atoi(next());
    else die(("unknown flag " + k).c_str());
  }
  if (a.nf <= 0 || a.target.empty() || a.weight.empty() || a.out.empty()) die("need --nf --target --weight --out");
  if (a.source.empty()) {
    a.source = a.target;
    a.ns = a.nf;
  }
  std::vector<vector3> target, source;
  std::vector<double> weight;
  read_points(a.target, target, a.nf);
  read_points(a.source, source, a.ns);
  read_doubles(a.weight, weight, (size_t)a.ns * a.ncols);
  std::vector<double> output((size_t)a.nf * a.ncols, 0.0);

  // The reference reads and writes its operator cache at ./../output/
  // (src/H2_3D_Tree.cpp:84-91), so run from <workdir>/exec.
  mkdir(a.workdir.c_str(), 0755);
  mkdir((a.workdir + "/exec").c_str(), 0755);
  mkdir((a.workdir + "/output").c_str(), 0755);
  if (chdir((a.workdir + "/exec").c_str()) != 0) die("chdir workdir failed");

  std::vector<double> times;
  double tpre = 0.0;
  const double L = a.L, eps = a.eps, prm = a.param;
  const int lv = a.level, n = a.order, ch = a.cheb;
#define RUN_BUILTIN(NAME, CLS)                                                      \
  else if (a.kernel == NAME) run<CLS>(                                              \
      a, [&]() { return new CLS(L, lv, n, eps, ch); }, target, source, weight, output, \
      times, tpre);
  if (false) {
  }
  RUN_BUILTIN("Laplacian", kernel_Laplacian)
  RUN_BUILTIN("OneOverR2", kernel_OneOverR2)
  RUN_BUILTIN("OneOverR4", kernel_OneOverR4)
  RUN_BUILTIN("Gaussian", kernel_Gaussian)
  RUN_BUILTIN("Logarithm", kernel_Logarithm)
  RUN_BUILTIN("Quadric", kernel_Quadric)
  RUN_BUILTIN("InverseQuadric", kernel_InverseQuadric)
  RUN_BUILTIN("ThinPlateSpline", kernel_ThinPlateSpline)
  RUN_BUILTIN("AnisoExp", kernel_AnisoExp)
  else if (a.kernel == "ExpCov") run<kernel_ExpCov>(
      a, [&]() { return new kernel_ExpCov(L, lv, n, eps, ch, prm); }, target, source, weight,
      output, times, tpre);
  else if (a.kernel == "GaussSigma") run<kernel_GaussSigma>(
      a, [&]() { return new kernel_GaussSigma(L, lv, n, eps, ch, prm); }, target, source,
      weight, output, times, tpre);
  else if (a.kernel == "SoftLap") run<kernel_SoftLap>(
      a, [&]() { return new kernel_SoftLap(L, lv, n, eps, ch, prm); }, target, source, weight,
      output, times, tpre);
  else die(("unknown kernel " + a.kernel).c_str());
#undef RUN_BUILTIN

  FILE* fp = fopen(a.out.c_str(), "wb");
  if (!fp) die("cannot open output");
  fwrite(output.data(), sizeof(double), output.size(), fp);
  fclose(fp);
  if (!a.timing.empty()) {
    FILE* ft = fopen(a.timing.c_str(), "w");
    if (!ft) die("cannot open timing file");
    fprintf(ft, "{\"threads\": %d, \"precompute_s\": %.9g, \"matvec_s\": [", omp_get_max_threads(), tpre);
    for (size_t i = 0; i < times.size(); ++i) fprintf(ft, "%s%.9g", i ? ", " : "", times[i]);
    fprintf(ft, "]}\n");
    fclose(ft);
  }
  return 0;
}
