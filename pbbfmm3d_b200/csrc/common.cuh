// Shared device utilities: the built-in kernel functors, dispatch helpers,
// complex types and asynchronous copies (Morton codes, the interpolation basis
// and the leaf kernels are in include/pbbfmm3d_b200_leaf.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pbbfmm3d_b200.h"
#include "../../include/pbbfmm3d_b200_leaf.cuh"

namespace pbbfmm {

// ------------------------------------------------------------ kernels
// K(t, s) with d = s - t, the arithmetic of src/kernel_Types.cpp (float64;
// the 1/r^k kernels use the reciprocal square root functions).
// 1/sqrt(r2), +inf at 0: rsqrtf in float32 (a few ulp), rsqrt in float64.
__device__ __forceinline__ float inv_sqrt(float r2) { return rsqrtf(r2); }
__device__ __forceinline__ double inv_sqrt(double r2) { return rsqrt(r2); }

template <int KID>
struct Kern;

template <>
struct Kern<PBBFMM_KERNEL_LAPLACIAN> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    return inv_sqrt(dx * dx + dy * dy + dz * dz);
  }
  template <typename T>
  __device__ static T eval_r2(T r2, const double*) {
    return inv_sqrt(r2);
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T r2 = dx * dx + dy * dy + dz * dz, ri = inv_sqrt(r2);
    const T f = r2 > T(0) ? -ri * ri * ri : T(0);
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return ri;
  }
};
template <>
struct Kern<PBBFMM_KERNEL_ONEOVERR2> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    T ri = inv_sqrt(dx * dx + dy * dy + dz * dz);
    return ri * ri;
  }
  template <typename T>
  __device__ static T eval_r2(T r2, const double*) {
    T ri = inv_sqrt(r2);
    return ri * ri;
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T r2 = dx * dx + dy * dy + dz * dz, ri2 = T(1) / r2;
    const T f = r2 > T(0) ? T(-2) * ri2 * ri2 : T(0);
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return ri2;
  }
};
template <>
struct Kern<PBBFMM_KERNEL_ONEOVERR4> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    T ri = inv_sqrt(dx * dx + dy * dy + dz * dz);
    return ri * ri * ri * ri;
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T r2 = dx * dx + dy * dy + dz * dz, ri2 = T(1) / r2;
    const T f = r2 > T(0) ? T(-4) * ri2 * ri2 * ri2 : T(0);
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return ri2 * ri2;
  }
};
template <>
struct Kern<PBBFMM_KERNEL_GAUSSIAN> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    T r = sqrt(dx * dx + dy * dy + dz * dz);
    return exp(-r * r);
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T k = eval(dx, dy, dz, p), f = T(-2) * k;
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return k;
  }
};
template <>
struct Kern<PBBFMM_KERNEL_LOGARITHM> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    T r2 = dx * dx + dy * dy + dz * dz;
    return r2 == T(0) ? T(0) : T(0.5) * log(r2);
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T r2 = dx * dx + dy * dy + dz * dz;
    const T f = r2 > T(0) ? T(1) / r2 : T(0);
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return eval(dx, dy, dz, p);
  }
};
template <>
struct Kern<PBBFMM_KERNEL_QUADRIC> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    return T(1) + (dx * dx + dy * dy + dz * dz);
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    g[0] = T(2) * dx, g[1] = T(2) * dy, g[2] = T(2) * dz;
    return eval(dx, dy, dz, p);
  }
};
template <>
struct Kern<PBBFMM_KERNEL_INVQUADRIC> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    return T(1) / (T(1) + (dx * dx + dy * dy + dz * dz));
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T q = eval(dx, dy, dz, p), f = T(-2) * q * q;
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return q;
  }
};
template <>
struct Kern<PBBFMM_KERNEL_THINPLATESPLINE> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    T r2 = dx * dx + dy * dy + dz * dz;
    return r2 == T(0) ? T(0) : T(0.5) * r2 * log(r2);
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T r2 = dx * dx + dy * dy + dz * dz;
    const T f = r2 > T(0) ? log(r2) + T(1) : T(0);
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return eval(dx, dy, dz, p);
  }
};
template <>
struct Kern<PBBFMM_KERNEL_EXPCOV> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double* p) {
    return exp(-sqrt(dx * dx + dy * dy + dz * dz) / T(p[0]));
  }
  template <typename T>
  __device__ static T eval_r2(T r2, const double* p) {
    return exp(-sqrt(r2) / T(p[0]));
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T r = sqrt(dx * dx + dy * dy + dz * dz), k = exp(-r / T(p[0]));
    const T f = r > T(0) ? -k / (T(p[0]) * r) : T(0);
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return k;
  }
};
template <>
struct Kern<PBBFMM_KERNEL_GAUSSSIGMA> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double* p) {
    return exp(-(dx * dx + dy * dy + dz * dz) / (T(2) * T(p[0]) * T(p[0])));
  }
  template <typename T>
  __device__ static T eval_r2(T r2, const double* p) {
    return exp(-r2 / (T(2) * T(p[0]) * T(p[0])));
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T s2 = T(2) * T(p[0]) * T(p[0]);
    const T k = exp(-(dx * dx + dy * dy + dz * dz) / s2), f = T(-2) * k / s2;
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return k;
  }
};
template <>
struct Kern<PBBFMM_KERNEL_ANISOEXP> {
  static constexpr bool has_gradient = true;
  template <typename T>
  __device__ static T eval(T dx, T dy, T dz, const double*) {
    return T(0.75) * exp(-sqrt(dx * dx / T(100) + dy * dy / T(100) + dz * dz / T(2.25)));
  }
  // value, and g = dK/dd (the gradient with respect to the target is -g); g = 0 at d = 0
  template <typename T>
  __device__ static T grad(T dx, T dy, T dz, const double* p, T* g) {
    const T q = sqrt(dx * dx / T(100) + dy * dy / T(100) + dz * dz / T(2.25));
    const T k = T(0.75) * exp(-q), f = q > T(0) ? -k / q : T(0);
    g[0] = f * dx / T(100), g[1] = f * dy / T(100), g[2] = f * dz / T(2.25);
    return k;
  }
};

// Run `f.template operator()<Kern<K>>()` for the runtime kernel id.
template <typename F>
inline int dispatch_kernel(int kid, F&& f) {
  switch (kid) {
    case PBBFMM_KERNEL_LAPLACIAN: return f.template run<Kern<PBBFMM_KERNEL_LAPLACIAN>>();
    case PBBFMM_KERNEL_ONEOVERR2: return f.template run<Kern<PBBFMM_KERNEL_ONEOVERR2>>();
    case PBBFMM_KERNEL_ONEOVERR4: return f.template run<Kern<PBBFMM_KERNEL_ONEOVERR4>>();
    case PBBFMM_KERNEL_GAUSSIAN: return f.template run<Kern<PBBFMM_KERNEL_GAUSSIAN>>();
    case PBBFMM_KERNEL_LOGARITHM: return f.template run<Kern<PBBFMM_KERNEL_LOGARITHM>>();
    case PBBFMM_KERNEL_QUADRIC: return f.template run<Kern<PBBFMM_KERNEL_QUADRIC>>();
    case PBBFMM_KERNEL_INVQUADRIC: return f.template run<Kern<PBBFMM_KERNEL_INVQUADRIC>>();
    case PBBFMM_KERNEL_THINPLATESPLINE:
      return f.template run<Kern<PBBFMM_KERNEL_THINPLATESPLINE>>();
    case PBBFMM_KERNEL_EXPCOV: return f.template run<Kern<PBBFMM_KERNEL_EXPCOV>>();
    case PBBFMM_KERNEL_GAUSSSIGMA: return f.template run<Kern<PBBFMM_KERNEL_GAUSSSIGMA>>();
    case PBBFMM_KERNEL_ANISOEXP: return f.template run<Kern<PBBFMM_KERNEL_ANISOEXP>>();
    default: return PBBFMM_ERR_ARG;
  }
}

// ------------------------------------------------------------ real types
// Every phase runs in float64 (PBBFMM_PREC_FP64) or float32 (the mixed path).
template <typename T>
struct Cplx;
template <>
struct Cplx<double> {
  using type = double2;
};
template <>
struct Cplx<float> {
  using type = float2;
};
template <typename T>
using cplx_t = typename Cplx<T>::type;
template <typename T>
__host__ __device__ __forceinline__ cplx_t<T> make_cplx(T re, T im) {
  cplx_t<T> v;
  v.x = re;
  v.y = im;
  return v;
}

// ------------------------------------------------------------ async copies
// 16-byte global -> shared copy that bypasses registers (cp.async, L2 only);
// src_bytes = 0 zero-fills the destination without reading `src` (which must
// still be a valid address).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src),
               "r"(src_bytes)
               : "memory");
}
// 8-byte copy with zero-fill (src_bytes 0 or 8), through L1.
__device__ __forceinline__ void cp_async8z(void* smem_dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(src_bytes)
               : "memory");
}
// Copy one complex value (double2: 16 bytes, float2: 8 bytes), zero-filled
// when `ok` is false.
template <typename C2>
__device__ __forceinline__ void cp_async_cplx(C2* smem_dst, const C2* src, bool ok) {
  if (sizeof(C2) == 16)
    cp_async16(smem_dst, src, ok ? 16 : 0);
  else
    cp_async8z(smem_dst, src, ok ? 8 : 0);
}

// 8-byte variant (through L1), for arrays without 16-byte alignment.
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
// One element (4 or 8 bytes), zero-filled when !ok (src must stay a valid address).
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
                 "r"(ok ? 8 : 0)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src),
                 "r"(ok ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Run `f.template run<N>()` for the runtime interpolation order N (2..10).
template <typename F>
inline int dispatch_order(int n, F&& f) {
  switch (n) {
    case 2: return f.template run<2>();
    case 3: return f.template run<3>();
    case 4: return f.template run<4>();
    case 5: return f.template run<5>();
    case 6: return f.template run<6>();
    case 7: return f.template run<7>();
    case 8: return f.template run<8>();
    case 9: return f.template run<9>();
    case 10: return f.template run<10>();
    default: return PBBFMM_ERR_ARG;
  }
}

}  // namespace pbbfmm
