/*
 * pbbfmm3d_b200 -- user-defined kernels as __device__ functors (compile with
 * nvcc for sm_100a; link with -lpbbfmm3d_b200).
 *
 * The reference's user kernel (README.md:178-227) is a subclass of
 * H2_3D_Tree with SetKernelProperty() and a virtual EvaluateKernel(target,
 * source).  The same class, written for this library:
 *
 *   #include "pbbfmm3d_b200_kernel.cuh"
 *   using namespace pbbfmm3d_b200;
 *
 *   class myKernel : public H2_3D_Tree_device<myKernel> {
 *    public:
 *     using H2_3D_Tree_device::H2_3D_Tree_device;  // (L, tree_level, order, eps, cheb[, device])
 *     void SetKernelProperty() {
 *       homogen = -1;
 *       symmetry = 1;
 *       kernelType = "myKernel";
 *     }
 *     template <typename R>
 *     __host__ __device__ static R EvaluateKernel(const vec3<R>& targetpos,
 *                                                 const vec3<R>& sourcepos) {
 *       vec3<R> diff;
 *       diff.x = sourcepos.x - targetpos.x;
 *       diff.y = sourcepos.y - targetpos.y;
 *       diff.z = sourcepos.z - targetpos.z;
 *       return R(1) / sqrt(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
 *     }
 *   };
 *
 *   myKernel Atree(L, tree_level, interpolation_order, epsilon, use_chebyshev);
 *   Atree.buildFMMTree();
 *   H2_3D_Compute<myKernel>(Atree, target, source, weight, nCols, output);
 *
 * Differences from the reference's class: EvaluateKernel is a static
 * __host__ __device__ template over the real type R (double on the host and
 * on the float64 GPU path, float on the mixed path's near field), taking
 * vec3<R>.  As in the reference, SetKernelProperty runs in buildFMMTree and
 * the kernel must depend on sourcepos - targetpos only (the far-field
 * operators are precomputed per offset); a singular value (+inf) is taken as
 * 0.  On the GPU the kernel is evaluated at targetpos = (0, 0, 0) and
 * sourcepos = the source's offset from the target.  EvaluateKernel must be
 * thread-safe on the host (the operator precompute runs on several threads).
 *
 * Optional, for the adjoint's position gradients:
 *   template <typename R>
 *   __host__ __device__ static R EvaluateKernelGradient(const vec3<R>& targetpos,
 *                                                       const vec3<R>& sourcepos, R* g);
 * returning K and setting g[0..2] = dK/d(sourcepos) (0 at coincident points).
 * Without it, the adjoint's gradients with respect to positions return
 * PBBFMM_ERR_UNSUPPORTED (dL/dweight works).
 *
 * This header instantiates the library's leaf kernels (L2P + P2P,
 * pbbfmm3d_b200_leaf.cuh) for the class and hands them to the library
 * through pbbfmm_tree_create_user (pbbfmm3d_b200.h).  Every other phase of a
 * compute is independent of the kernel once its operators exist.
 */
#ifndef PBBFMM3D_B200_KERNEL_CUH
#define PBBFMM3D_B200_KERNEL_CUH

#include <string>
#include <type_traits>
#include <utility>

#include "pbbfmm3d_b200.hpp"
#include "pbbfmm3d_b200_leaf.cuh"

namespace pbbfmm3d_b200 {

template <typename R>
struct vec3 {
  R x, y, z;
};

namespace detail {

template <class D, class = void>
struct has_kernel_gradient : std::false_type {};
template <class D>
struct has_kernel_gradient<
    D, decltype((void)D::template EvaluateKernelGradient<double>(
           std::declval<const vec3<double>&>(), std::declval<const vec3<double>&>(),
           std::declval<double*>()))> : std::true_type {};

// The library's kernel-functor interface over a user class D.
template <class D>
struct DeviceFunctor {
  static constexpr bool has_gradient = has_kernel_gradient<D>::value;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    const vec3<T> t{T(0), T(0), T(0)}, s{dx, dy, dz};
    return D::template EvaluateKernel<T>(t, s);
  }
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double*, T* g) {
    const vec3<T> t{T(0), T(0), T(0)}, s{dx, dy, dz};
    return D::template EvaluateKernelGradient<T>(t, s, g);
  }
};

template <class D>
double evaluate_host(const double* t, const double* s, void*) {
  const vec3<double> tp{t[0], t[1], t[2]}, sp{s[0], s[1], s[2]};
  return D::template EvaluateKernel<double>(tp, sp);
}

template <class D>
int launch_leaf(const pbbfmm_leaf_args* a, void* stream) {
  return pbbfmm::launch_leaf_kernels<DeviceFunctor<D>>(*a, static_cast<cudaStream_t>(stream));
}

}  // namespace detail

// Base of a user kernel class (CRTP): the reference's H2_3D_Tree with a
// user-defined kernel.  Derived provides SetKernelProperty() (setting
// homogen, symmetry, kernelType) and the static EvaluateKernel<R> template.
template <class Derived>
class H2_3D_Tree_device : public H2_3D_Tree {
 public:
  H2_3D_Tree_device(double L, int tree_level, int interpolation_order, double epsilon,
                    int use_chebyshev, int device = 0)
      : H2_3D_Tree(deferred{}, L, tree_level, interpolation_order, epsilon, use_chebyshev,
                   device) {}

  // SetKernelProperty, then the tree and its operators (src/H2_3D_Tree.cpp:
  // 40-66); cache_dir reads / writes operator files named by kernelType.
  void buildFMMTree(const char* cache_dir = nullptr) {
    static_cast<Derived*>(this)->SetKernelProperty();
    pbbfmm_user_kernel k{};
    k.kernel_type = kernelType.c_str();
    k.homogen = homogen;
    k.symmetry = symmetry;
    k.evaluate = &detail::evaluate_host<Derived>;
    k.launch_leaf = &detail::launch_leaf<Derived>;
    k.has_gradient = detail::has_kernel_gradient<Derived>::value ? 1 : 0;
    k.ctx = nullptr;
    pbbfmm_tree* h = nullptr;
    check(pbbfmm_tree_create_user(&params_, &k, device_, &h));
    adopt(h);
    H2_3D_Tree::buildFMMTree(cache_dir);
  }

 protected:
  double homogen = 0;   // degree of homogeneity (0: not homogeneous)
  int symmetry = 1;     // 1 symmetric, -1 antisymmetric, 0 neither
  std::string kernelType = "myKernel";
};

}  // namespace pbbfmm3d_b200

#endif  // PBBFMM3D_B200_KERNEL_CUH
