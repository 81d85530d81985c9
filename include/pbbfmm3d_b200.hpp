/* C++ front door of pbbfmm3d_b200: the reference's object model over the C ABI.
 *
 * Replaces, for a C++ caller of PBBFMM3D:
 *   kernel_X Atree(L, tree_level, interpolation_order, epsilon, use_chebyshev);
 *       (src/H2_3D_Tree.cpp:12-38, include/kernel_Types.hpp)
 *   Atree.buildFMMTree();                            (src/H2_3D_Tree.cpp:40-66)
 *   H2_3D_Compute<kernel_X>(Atree, target, source, weight, nCols, output);
 *       (include/compute.hpp:67-149; output is accumulated into)
 * with the same argument meaning and layouts: points are 3-double AoS records
 * (the reference's vector3), weight[col*Ns + i] and output[col*Nf + i]
 * column-major.  Failures throw pbbfmm3d_b200::Error (the reference asserts
 * or exits).  Header-only; link with -lpbbfmm3d_b200.
 *
 * Kernels are the library's compiled-in functors: the reference's built-ins
 * plus exp(-r/l) (kernel_ExpCov), exp(-r^2/2s^2) (kernel_GaussSigma) and the
 * anisotropic exponential of the reference's python example (kernel_AnisoExp).
 * User-defined kernels (the reference's subclasses with SetKernelProperty and
 * EvaluateKernel) are __device__ functors: include/pbbfmm3d_b200_kernel.cuh.
 */
#ifndef PBBFMM3D_B200_HPP
#define PBBFMM3D_B200_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pbbfmm3d_b200.h"

namespace pbbfmm3d_b200 {

struct Error : std::runtime_error {
  int status;
  Error(int rc, const std::string& what) : std::runtime_error(what), status(rc) {}
};

inline void check(int rc) {
  if (rc != PBBFMM_OK) throw Error(rc, pbbfmm_last_error());
}

// The reference's vector3: three doubles.
struct vector3 {
  double x, y, z;
};

class H2_3D_Tree {
 public:
  H2_3D_Tree(double L, int tree_level, int interpolation_order, double epsilon,
             int use_chebyshev, int kernel, double p0 = 0.0, int device = 0) {
    pbbfmm_tree_params p{};
    p.L = L;
    p.tree_level = tree_level;
    p.interpolation_order = interpolation_order;
    p.epsilon = epsilon;
    p.use_chebyshev = use_chebyshev;
    p.kernel = kernel;
    p.kernel_param[0] = p0;
    check(pbbfmm_tree_create(&p, device, &h_));
  }
  virtual ~H2_3D_Tree() { pbbfmm_tree_destroy(h_); }
  H2_3D_Tree(const H2_3D_Tree&) = delete;
  H2_3D_Tree& operator=(const H2_3D_Tree&) = delete;

  // Operator precompute (or the reference-format cache in cache_dir).
  void buildFMMTree(const char* cache_dir = nullptr) { check(pbbfmm_tree_build(live(), cache_dir)); }
  // PBBFMM_PREC_FP64 (default) or PBBFMM_PREC_MIXED.
  void set_precision(int precision) { check(pbbfmm_set_precision(live(), precision)); }
  // Mixed Chebyshev M2L operands: PBBFMM_TC_F16 (default), PBBFMM_TC_TF32, or
  // PBBFMM_TC_OFF for the CUDA cores; tensor_core_m2l() reports the one in use.
  void set_tensor_cores(int mode) { check(pbbfmm_set_tensor_cores(live(), mode)); }
  int tensor_core_m2l() const { return pbbfmm_tensor_core_m2l(h_); }
  pbbfmm_tree* handle() const { return h_; }

 protected:
  // For trees whose kernel is known only at buildFMMTree (user kernels, whose
  // SetKernelProperty runs there as in the reference): parameters are kept
  // and the library tree is created later by adopt().
  struct deferred {};
  H2_3D_Tree(deferred, double L, int tree_level, int interpolation_order, double epsilon,
             int use_chebyshev, int device)
      : device_(device) {
    params_.L = L;
    params_.tree_level = tree_level;
    params_.interpolation_order = interpolation_order;
    params_.epsilon = epsilon;
    params_.use_chebyshev = use_chebyshev;
  }
  void adopt(pbbfmm_tree* h) {
    if (h_) pbbfmm_tree_destroy(h_);
    h_ = h;
  }
  pbbfmm_tree* live() const {
    if (!h_) throw Error(PBBFMM_ERR_STATE, "call buildFMMTree() first");
    return h_;
  }
  pbbfmm_tree_params params_{};
  int device_ = 0;

 private:
  pbbfmm_tree* h_ = nullptr;
};

#define PBBFMM3D_B200_KERNEL_CLASS(NAME, ID)                                                  \
  class NAME : public H2_3D_Tree {                                                           \
   public:                                                                                   \
    NAME(double L, int tree_level, int interpolation_order, double epsilon,                 \
         int use_chebyshev, int device = 0)                                                  \
        : H2_3D_Tree(L, tree_level, interpolation_order, epsilon, use_chebyshev, ID, 0.0,    \
                     device) {}                                                              \
  };
PBBFMM3D_B200_KERNEL_CLASS(kernel_Laplacian, PBBFMM_KERNEL_LAPLACIAN)
PBBFMM3D_B200_KERNEL_CLASS(kernel_OneOverR2, PBBFMM_KERNEL_ONEOVERR2)
PBBFMM3D_B200_KERNEL_CLASS(kernel_OneOverR4, PBBFMM_KERNEL_ONEOVERR4)
PBBFMM3D_B200_KERNEL_CLASS(kernel_Gaussian, PBBFMM_KERNEL_GAUSSIAN)
PBBFMM3D_B200_KERNEL_CLASS(kernel_Logarithm, PBBFMM_KERNEL_LOGARITHM)
PBBFMM3D_B200_KERNEL_CLASS(kernel_Quadric, PBBFMM_KERNEL_QUADRIC)
PBBFMM3D_B200_KERNEL_CLASS(kernel_InverseQuadric, PBBFMM_KERNEL_INVQUADRIC)
PBBFMM3D_B200_KERNEL_CLASS(kernel_ThinPlateSpline, PBBFMM_KERNEL_THINPLATESPLINE)
PBBFMM3D_B200_KERNEL_CLASS(kernel_AnisoExp, PBBFMM_KERNEL_ANISOEXP)
#undef PBBFMM3D_B200_KERNEL_CLASS

// exp(-r / ell)
class kernel_ExpCov : public H2_3D_Tree {
 public:
  kernel_ExpCov(double L, int tree_level, int interpolation_order, double epsilon,
                int use_chebyshev, double ell, int device = 0)
      : H2_3D_Tree(L, tree_level, interpolation_order, epsilon, use_chebyshev,
                   PBBFMM_KERNEL_EXPCOV, ell, device) {}
};
// exp(-r^2 / (2 sigma^2))
class kernel_GaussSigma : public H2_3D_Tree {
 public:
  kernel_GaussSigma(double L, int tree_level, int interpolation_order, double epsilon,
                    int use_chebyshev, double sigma, int device = 0)
      : H2_3D_Tree(L, tree_level, interpolation_order, epsilon, use_chebyshev,
                   PBBFMM_KERNEL_GAUSSSIGMA, sigma, device) {}
};

// output += K(target, source) * weight, on the tree's GPU (host buffers in and
// out, synchronous).  V3 is any record of three doubles (this header's
// vector3 or the reference's).
template <class T, class V3>
void H2_3D_Compute(T& tree, const std::vector<V3>& target, const std::vector<V3>& source,
                   const std::vector<double>& weight, int nCols, std::vector<double>& output) {
  static_assert(sizeof(V3) == 3 * sizeof(double), "points must be three doubles");
  const int64_t Nf = (int64_t)target.size(), Ns = (int64_t)source.size();
  if (nCols < 1 || (int64_t)weight.size() < Ns * nCols || (int64_t)output.size() < Nf * nCols)
    throw Error(PBBFMM_ERR_ARG, "weight must hold Ns*nCols and output Nf*nCols values");
  check(pbbfmm_compute(tree.handle(), reinterpret_cast<const double*>(target.data()), Nf,
                       reinterpret_cast<const double*>(source.data()), Ns, weight.data(), nCols,
                       output.data()));
}

}  // namespace pbbfmm3d_b200

#endif  // PBBFMM3D_B200_HPP
