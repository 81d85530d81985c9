// Host-side (float64) operator precompute: the buildFMMTree() half of the
// reference (src/H2_3D_Tree.cpp:40-239, 251-648, 715-909), restated.
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace pbbfmm {

struct KernelSpec {
  int id = 0;
  double param[4] = {0, 0, 0, 0};
  double homogen = 0;  // as set by SetKernelProperty (before the negation)
  int symmetry = 1;
  // user-defined kernel (id PBBFMM_KERNEL_USER): its kernelType and its
  // EvaluateKernel(target, source) on the host
  std::string user_type;
  double (*user_eval)(const double*, const double*, void*) = nullptr;
  void* user_ctx = nullptr;
};

// Kernel metadata of the built-in kernels (src/kernel_Types.cpp).
KernelSpec kernel_spec(int id, const double* param);
// kernelType string used for the cache file names (src/H2_3D_Tree.cpp:84-91).
std::string kernel_type_name(const KernelSpec& k);
double eval_kernel_host(const KernelSpec& k, const double t[3], const double s[3]);

struct Weights {
  int n = 0;
  std::vector<double> Tkz, Kweights, Cweights;  // n*n, n^3, 2n^2
  int Ktable[343];
};
// ComputeWeights, src/H2_3D_Tree.cpp:715-826.
Weights compute_weights(int n, int cheb);

struct Operators {
  int cheb = 1;
  int n = 0;
  int rf = 0, rs = 0;  // SVD cutoffs (uniform: n^3)
  int nlev = 1;        // 1 if homogeneous else tree_level - 1
  // Chebyshev (reference layout, FMMReadMatrices src/H2_3D_Tree.cpp:186-239)
  std::vector<double> K, U, VT;
  // Uniform: real kernel stencils nlev x 316 x (2n-1)^3 (MatM2L before its FFT,
  // src/H2_3D_Tree.cpp:599-631) -- the device derives its spectra from these.
  std::vector<double> stencil;
};

bool is_homogeneous(double homogen);  // IsHomoKernel, src/H2_3D_Tree.cpp:134-136

// Full precompute (StartPrecompute / ComputeKernelCheb / ComputeKernelUnif).
int precompute_operators(const KernelSpec& k, int n, int cheb, double box, int tree_level,
                         double eps, const Weights& w, Operators* ops, std::string* err);

// Reference cache files (<dir>/<type>{Cheb,Unif}{K,U,V}<n>.bin).
// Returns 0 if read, 1 if absent/stale (PrecomputeAvailable), <0 on error.
int read_cache(const std::string& dir, const KernelSpec& k, int n, int cheb, double box,
               int tree_level, Operators* ops, std::string* err);
int write_cache(const std::string& dir, const KernelSpec& k, int n, int cheb, double box,
                int tree_level, const Operators& ops, std::string* err);

// Uniform: FFTW-halfcomplex R2HC spectra of length P <-> real stencils.
void stencils_to_halfcomplex(const std::vector<double>& st, int P, std::vector<double>* hc);
void halfcomplex_to_stencils(const std::vector<double>& hc, int P, std::vector<double>* st);

// Thin SVD helpers (exposed for tests): singular values (descending) and
// right singular vectors (n x n, column-major) of a tall m x n matrix.
void svd_tall_right(const double* A, int64_t m, int n, std::vector<double>* sigma,
                    std::vector<double>* V);

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)>& body);

}  // namespace pbbfmm
