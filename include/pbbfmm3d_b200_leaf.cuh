/*
 * pbbfmm3d_b200 -- device code shared by the library and by translation units
 * that instantiate the leaf phase for their own kernel functor.
 *
 * Holds the Morton codes of the leaf numbering, the interpolation basis, the
 * compensated sums, and the leaf-phase kernels (L2P + P2P + scatter to the
 * output, reference include/compute.hpp:591-785) templated on the kernel
 * functor KF, with their launcher launch_leaf_kernels<KF>().  The library
 * instantiates them for its built-in kernels; include/pbbfmm3d_b200_kernel.cuh
 * instantiates them for a user's kernel.  Everything the kernels read comes
 * in a pbbfmm_leaf_args (include/pbbfmm3d_b200.h).
 *
 * A kernel functor KF provides
 *   template <typename T> __device__ static T eval(T dx, T dy, T dz, const double* p);
 * the kernel K(t, s) at d = s - t (p: up to four parameters), +inf where it
 * is singular (set to 0, as the reference does, include/compute.hpp:767); and
 * for the gradient passes (adjoint with position gradients) also
 *   template <typename T> __device__ static T grad(T dx, T dy, T dz, const double* p, T* g);
 * returning K and setting g = dK/dd (0 at d = 0), with
 *   static constexpr bool has_gradient = true;
 * Requires nvcc.
 */
#ifndef PBBFMM3D_B200_LEAF_CUH
#define PBBFMM3D_B200_LEAF_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "pbbfmm3d_b200.h"

namespace pbbfmm {

constexpr int kMaxOrder = 10;

// ------------------------------------------------------------ Morton codes
// Leaf index of the reference: sum_l j_l 8^(L-1-l), j = 4 bx + 2 by + bz
// (src/H2_3D_Tree.cpp:939-971) -- x in the most significant bit of each
// octal digit.  Coordinate bit k sits at bit 3k+2 (x), 3k+1 (y), 3k (z).
__host__ __device__ inline uint32_t spread3(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x030000ff;
  v = (v | (v << 8)) & 0x0300f00f;
  v = (v | (v << 4)) & 0x030c30c3;
  v = (v | (v << 2)) & 0x09249249;
  return v;
}
__host__ __device__ inline uint32_t compact3(uint32_t v) {
  v &= 0x09249249;
  v = (v | (v >> 2)) & 0x030c30c3;
  v = (v | (v >> 4)) & 0x0300f00f;
  v = (v | (v >> 8)) & 0x030000ff;
  v = (v | (v >> 16)) & 0x000003ff;
  return v;
}
__host__ __device__ inline uint32_t morton_encode(int x, int y, int z) {
  return (spread3((uint32_t)x) << 2) | (spread3((uint32_t)y) << 1) | spread3((uint32_t)z);
}
__host__ __device__ inline void morton_decode(uint32_t m, int* x, int* y, int* z) {
  *x = (int)compact3(m >> 2);
  *y = (int)compact3(m >> 1);
  *z = (int)compact3(m);
}

// Compensated (Kahan) sum: s holds the sum, c the running low-order error.
template <typename T>
struct Kahan {
  T s = 0, c = 0;
  __device__ __forceinline__ void add(T x) {
    const T y = x - c;
    const T t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// ------------------------------------------------------------ basis
// S_m(x) per coordinate (ComputeSn, src/H2_3D_Tree.cpp:830-892).
// Chebyshev: (2/n) * Clenshaw sum of T_k(node_m) T_k(x); uniform: Lagrange.
template <typename T>
__device__ __forceinline__ T basis_one(int n, int cheb, T x, const T* Tkz, int m) {
  if (cheb) {
    const T* Tk = Tkz + m * n;
    T d0 = 0, d1 = 0, d2;
    for (int j = n - 1; j > 0; j--) {
      d2 = d0;
      d0 = T(2) * x * d0 - d1 + Tk[j];
      d1 = d2;
    }
    return (T(2) / T(n)) * (x * d0 - d1 + T(0.5) * Tk[0]);
  }
  T num = 1, den = 1;
  for (int j = 0; j < n; j++)
    if (m != j) {
      num *= x - (T(1) - T(2) * T(j) / T(n - 1));
      den *= T(-2) * (T(m) - T(j)) / T(n - 1);
    }
  return num / den;
}

// dS_m/dx on [-1, 1].  Chebyshev: S_m(x) = (2/n) (1/2 + sum_{k>=1} T_k(x_m)
// T_k(x)), so S_m'(x) = (2/n) sum_{k>=1} T_k(x_m) k U_{k-1}(x) with U the
// Chebyshev polynomials of the second kind.  Uniform: the derivative of the
// Lagrange polynomial, sum over i != m of prod_{j != m, i} (x - x_j) / den.
template <typename T>
__device__ __forceinline__ T basis_deriv(int n, int cheb, T x, const T* Tkz, int m) {
  if (cheb) {
    const T* Tk = Tkz + m * n;
    T u0 = 1, u1 = T(2) * x, s = 0;  // U_{k-1}, U_k
    for (int k = 1; k < n; ++k) {
      s += Tk[k] * T(k) * u0;
      const T u2 = T(2) * x * u1 - u0;
      u0 = u1;
      u1 = u2;
    }
    return (T(2) / T(n)) * s;
  }
  T den = 1;
  for (int j = 0; j < n; j++)
    if (m != j) den *= T(-2) * (T(m) - T(j)) / T(n - 1);
  T sum = 0;
  for (int i = 0; i < n; ++i) {
    if (i == m) continue;
    T prod = 1;
    for (int j = 0; j < n; ++j)
      if (j != m && j != i) prod *= x - (T(1) - T(2) * T(j) / T(n - 1));
    sum += prod;
  }
  return sum / den;
}

// out[m * stride] = S_m(x), m < n
template <typename T>
__device__ __forceinline__ void basis_all(int n, int cheb, T x, const T* Tkz, T* out,
                                          int stride = 1) {
  for (int m = 0; m < n; ++m) out[m * stride] = basis_one<T>(n, cheb, x, Tkz, m);
}

// Centre of cell m of level l (the reference's +-quarter-length steps from
// the root, src/H2_3D_Tree.cpp:927-961, in the same rounding).
__device__ __forceinline__ void cell_center_d(uint32_t m, int l, double box, double* c) {
  int x, y, z;
  morton_decode(m, &x, &y, &z);
  double cx = 0, cy = 0, cz = 0, len = box;
  for (int i = l - 1; i >= 0; --i) {
    const double q = 0.25 * len;
    cx = ((x >> i) & 1) ? __dadd_rn(cx, q) : __dsub_rn(cx, q);
    cy = ((y >> i) & 1) ? __dadd_rn(cy, q) : __dsub_rn(cy, q);
    cz = ((z >> i) & 1) ? __dadd_rn(cz, q) : __dsub_rn(cz, q);
    len = 0.5 * len;
  }
  c[0] = cx;
  c[1] = cy;
  c[2] = cz;
}

// Leaf phase (L2P + P2P): one warp per nonempty target leaf.  Dense leaves
// (kLaneLeafMin targets or more): one lane per target, 32 targets per pass;
// the sources of the 27 neighbour leaves are staged through a per-warp
// shared-memory tile of 32 (coalesced loads) that every lane sweeps by
// broadcast reads, and the far field evaluates the n^3 local coefficients
// (broadcast loads) against the lane's own basis.  Sparse leaves: one target
// at a time, lanes over its sources and coefficients, warp shuffle reduction.
// Reference: Local2Particle / DirectInteractions, include/compute.hpp:692-778.
constexpr int kLeafWarps = 4;
constexpr int kLeafCols = 8;  // columns per pass (registers)
constexpr int kLaneLeafMin = 12;  // leaves with fewer targets take the warp-per-target path
// resident CTAs per SM the dense-leaf kernel is compiled for: the float32
// one-column kernel fits 64 registers (32 warps per SM, latency hiding for
// the gathers); the others keep 128
template <typename T, int KC>
constexpr int kLeafBlocks = sizeof(T) == 4 && KC == 1 ? 8 : 4;
// the sparse-leaf kernel: float32 at 6 CTAs per SM for any column count
template <typename T>
constexpr int kSparseBlocks = sizeof(T) == 4 ? 6 : 4;

// Packed float32 pairs (two lanes of arithmetic per instruction, sm_100):
// a pair is a 64-bit register holding (first, second).
__device__ __forceinline__ unsigned long long f2_pack(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// Kernels that are functions of r^2 may provide eval_r2(r2, params); the
// packed pair loop then forms r^2 with packed arithmetic as well.
template <class KF, class = void>
struct HasEvalR2 : std::false_type {};
template <class KF>
struct HasEvalR2<KF, decltype((void)KF::template eval_r2<float>(0.f, nullptr))> : std::true_type {};

// pre[q] = the number of sources in neighbour slots < q (q = 0..27), from
// lane q's count (lanes 27..31 hold 0): a warp scan.
__device__ __forceinline__ void neighbour_prefix(int cnt, int lane, int* pre) {
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane < 27) pre[lane] = incl - cnt;
  if (lane == 26) pre[27] = incl;
}

// Source coordinates relative to the target leaf's centre.  float (mixed
// path): hi = float(d), lo = float(d - hi), so that differences of nearby
// points keep ~48 bits; double: the offsets themselves.
template <typename T>
struct RelPos;
template <>
struct RelPos<float> {
  float h[3], l[3];
  __device__ void set(double dx, double dy, double dz) {
    h[0] = (float)dx, h[1] = (float)dy, h[2] = (float)dz;
    l[0] = (float)(dx - h[0]), l[1] = (float)(dy - h[1]), l[2] = (float)(dz - h[2]);
  }
  // source minus target
  __device__ void diff(const float4& sh, const float4& sl, float* d) const {
    d[0] = (sh.x - h[0]) + (sl.x - l[0]);
    d[1] = (sh.y - h[1]) + (sl.y - l[1]);
    d[2] = (sh.z - h[2]) + (sl.z - l[2]);
  }
};
template <>
struct RelPos<double> {
  double h[3];
  __device__ void set(double dx, double dy, double dz) { h[0] = dx, h[1] = dy, h[2] = dz; }
  __device__ void diff(const double4& sh, const double4&, double* d) const {
    d[0] = sh.x - h[0];
    d[1] = sh.y - h[1];
    d[2] = sh.z - h[2];
  }
};
template <typename T>
using vec4_t = typename std::conditional<sizeof(T) == 4, float4, double4>::type;

// Running sum of the float64 path (plain; the mixed path uses Kahan<float>).
template <typename T>
struct PlainSum {
  T s = 0;
  __device__ __forceinline__ void add(T x) { s += x; }
  __device__ __forceinline__ double value() const { return (double)s; }
};
template <typename T>
using LeafAcc = typename std::conditional<sizeof(T) == 4, Kahan<T>, PlainSum<T>>::type;

// Dense leaves (at least kLaneLeafMin targets): warp = one 32-target chunk,
// one target per lane, sources through shared-memory tiles of 32.
// T = float (mixed path): kernel values, interpolation and per-tile partial
// sums in float32, each lane's running sums compensated (Kahan), the output
// update in float64.  T = double: everything in float64.
template <class KF, typename T, int KC>
__global__ void __launch_bounds__(32 * kLeafWarps, kLeafBlocks<T, KC>)
    k_leaf(const int* __restrict__ leaves, int nleaves, const int* __restrict__ part_count,
           const int* __restrict__ chunk_prefix, const int* __restrict__ tstart,
           const int* __restrict__ sstart, const int* __restrict__ tperm,
           const double* __restrict__ tpos, const double* __restrict__ spos,
           const double* __restrict__ wsorted, int Nf, int Ns, int C,
           const T* __restrict__ F_L, int n, int cheb, const T* __restrict__ Tkz_g,
           double box, int L, const double* __restrict__ kparam_g, double* __restrict__ out) {
  constexpr bool kMixed = sizeof(T) == 4;
  using V4 = vec4_t<T>;
  __shared__ T sTkz[kMaxOrder * kMaxOrder];
  __shared__ double kp[4];
  __shared__ int s_nb[kLeafWarps][27][2];  // neighbour source ranges
  __shared__ int s_pre[kLeafWarps][28];    // exclusive prefix of their lengths
  __shared__ V4 s_sh[kLeafWarps][32];               // staged sources: position (hi)
  __shared__ V4 s_sl[kLeafWarps][kMixed ? 32 : 1];  // position (lo), mixed path
  __shared__ T s_w[kLeafWarps][32][KC];             // staged weights
  __shared__ T s_F[kLeafWarps][KC * 32];            // staged local coefficients (L2P)
  // basis values of each lane's target, [warp][dim][m < n][lane] (dynamic, sized by n)
  extern __shared__ __align__(16) unsigned char leaf_dyn[];
  T* s_bw = reinterpret_cast<T*>(leaf_dyn) + (threadIdx.x >> 5) * 3 * n * 32;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTkz[i] = Tkz_g[i];
  if (threadIdx.x < 4) kp[threadIdx.x] = kparam_g[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int wid = blockIdx.x * kLeafWarps + wl;
  // leaves are partitioned: the dense ones first, the sparse ones after;
  // warp = one 32-target chunk of a dense leaf, chunk_prefix[i] the first
  // chunk of dense leaf i (exclusive scan), chunk_prefix[nd] the total
  const int nd = *part_count;
  if (wid >= chunk_prefix[nd]) return;
  int lo = 0, hi = nd - 1;
  while (lo < hi) {  // last i with chunk_prefix[i] <= wid
    const int mid = (lo + hi + 1) >> 1;
    if (chunk_prefix[mid] <= wid) lo = mid;
    else hi = mid - 1;
  }
  const int leaf = leaves[lo];
  const int te = tstart[leaf + 1];
  const int tc0 = tstart[leaf] + 32 * (wid - chunk_prefix[lo]);
  const int n3 = n * n * n;
  double c[3];
  cell_center_d((uint32_t)leaf, L, box, c);
  double len = box;
  for (int i = 0; i < L; ++i) len = 0.5 * len;
  const double ihalfL = 2. / len;
  int ax, ay, az;
  morton_decode((uint32_t)leaf, &ax, &ay, &az);
  const int nside = 1 << L;
  // neighbour source ranges, slot 9(x+1)+3(y+1)+(z+1)
  int nb_cnt = 0;
  if (lane < 27) {
    const int q = lane;
    const int bx = ax + q / 9 - 1, by = ay + (q / 3) % 3 - 1, bz = az + q % 3 - 1;
    int a = 0, e = 0;
    if (bx >= 0 && by >= 0 && bz >= 0 && bx < nside && by < nside && bz < nside) {
      const uint32_t bm = morton_encode(bx, by, bz);
      a = sstart[bm];
      e = sstart[bm + 1];
    }
    s_nb[wl][q][0] = a;
    s_nb[wl][q][1] = e;
    nb_cnt = e - a;
  }
  __syncwarp();
  neighbour_prefix(nb_cnt, lane, s_pre[wl]);
  __syncwarp();
  const int nsrc_total = s_pre[wl][27];
  for (int c0 = 0; c0 < C; c0 += KC) {
    const int cg = min(KC, C - c0);
    for (int t0 = tc0; t0 < te && t0 < tc0 + 32; t0 += 32) {  // this warp's chunk
      const int i = t0 + lane;
      const bool active = i < te;
      double x = c[0], y = c[1], z = c[2];
      if (active) x = tpos[i], y = tpos[(int64_t)Nf + i], z = tpos[2 * (int64_t)Nf + i];
      RelPos<T> tp;
      tp.set(x - c[0], y - c[1], z - c[2]);
      LeafAcc<T> acc[KC];
      // far field: phi += sum_l F[l] Sx[l1] Sy[l2] Sz[l3].  The leaf's
      // coefficients are staged 32 at a time (coalesced loads, one round
      // trip per chunk) and read by broadcast; every lane takes part,
      // inactive ones on the leaf centre, writing nothing.
      {
        T* b = s_bw + lane;  // b[(d n + m) 32]: conflict-free, no local memory
        for (int m = 0; m < n; ++m) {
          b[m * 32] = basis_one<T>(n, cheb, (T)(ihalfL * (x - c[0])), sTkz, m);
          b[(n + m) * 32] = basis_one<T>(n, cheb, (T)(ihalfL * (y - c[1])), sTkz, m);
          b[(2 * n + m) * 32] = basis_one<T>(n, cheb, (T)(ihalfL * (z - c[2])), sTkz, m);
        }
        const T* Fl = F_L + ((int64_t)leaf * C + c0) * n3;
        T* sF = s_F[wl];
        int l1 = 0, l2 = 0, l3 = 0;
        T b12 = b[0] * b[n * 32];
        for (int l0 = 0; l0 < n3; l0 += 32) {
          __syncwarp();
          if (l0 + lane < n3) {
#pragma unroll
            for (int cc = 0; cc < KC; ++cc)
              sF[cc * 32 + lane] = cc < cg ? Fl[cc * n3 + l0 + lane] : T(0);
          }
          __syncwarp();
          const int mm = min(32, n3 - l0);
          for (int jj = 0; jj < mm; ++jj) {
            const T v = b12 * b[(2 * n + l3) * 32];
#pragma unroll
            for (int cc = 0; cc < KC; ++cc)
              if (cc < cg) acc[cc].add(sF[cc * 32 + jj] * v);
            if (++l3 == n) {
              l3 = 0;
              if (++l2 == n) l2 = 0, ++l1;
              if (l1 < n) b12 = b[l1 * 32] * b[(n + l2) * 32];
            }
          }
        }
      }
      // near field: the 27 neighbours' source ranges, concatenated, in tiles of 32
      int q = 0;
      if constexpr (kMixed && KC == 1) {
        // float32, one column: two sources per step in packed f32x2
        // arithmetic.  The tile is staged as source pairs: per pair p,
        // (x_hi, y_hi) and (z_hi, w) of sources 2p and 2p + 1 interleaved,
        // then (x_lo, y_lo) and z_lo; an odd tile ends with a far, weightless
        // dummy source (finite kernel value times 0).
        float* P01 = reinterpret_cast<float*>(&s_sh[wl][0]);  // [16][4] | [16][4]
        float* P23 = reinterpret_cast<float*>(&s_sl[wl][0]);  // [16][4] | [16][2]
        const unsigned long long ntxh = f2_pack(-tp.h[0], -tp.h[0]), ntyh = f2_pack(-tp.h[1], -tp.h[1]),
                                 ntzh = f2_pack(-tp.h[2], -tp.h[2]), ntxl = f2_pack(-tp.l[0], -tp.l[0]),
                                 ntyl = f2_pack(-tp.l[1], -tp.l[1]), ntzl = f2_pack(-tp.l[2], -tp.l[2]);
        for (int v0 = 0; v0 < nsrc_total; v0 += 32) {
          const int v = v0 + lane, pr = lane >> 1, e = lane & 1;
          float xh = 1.0e3f, yh = 0.f, zh = 0.f, xl = 0.f, yl = 0.f, zl = 0.f, wv = 0.f;
          if (v < nsrc_total) {
            while (v >= s_pre[wl][q + 1]) ++q;
            const int j = s_nb[wl][q][0] + (v - s_pre[wl][q]);
            RelPos<T> sp;
            sp.set(spos[j] - c[0], spos[(int64_t)Ns + j] - c[1], spos[2 * (int64_t)Ns + j] - c[2]);
            xh = sp.h[0], yh = sp.h[1], zh = sp.h[2], xl = sp.l[0], yl = sp.l[1], zl = sp.l[2];
            wv = (float)wsorted[(int64_t)j * C + c0];
          }
          P01[4 * pr + e] = xh;
          P01[4 * pr + 2 + e] = yh;
          P01[64 + 4 * pr + e] = zh;
          P01[64 + 4 * pr + 2 + e] = wv;
          P23[4 * pr + e] = xl;
          P23[4 * pr + 2 + e] = yl;
          P23[64 + 2 * pr + e] = zl;
          __syncwarp();
          if (active) {
            const int np = (min(32, nsrc_total - v0) + 1) >> 1;
            unsigned long long part2 = 0ull;  // (0.f, 0.f)
#pragma unroll 4
            for (int pp = 0; pp < np; ++pp) {
              const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(P01 + 4 * pp);
              const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(P01 + 64 + 4 * pp);
              const ulonglong2 cl = *reinterpret_cast<const ulonglong2*>(P23 + 4 * pp);
              const unsigned long long zl2 = *reinterpret_cast<const unsigned long long*>(P23 + 64 + 2 * pp);
              const unsigned long long dx = f2_add(f2_add(a.x, ntxh), f2_add(cl.x, ntxl));
              const unsigned long long dy = f2_add(f2_add(a.y, ntyh), f2_add(cl.y, ntyl));
              const unsigned long long dz = f2_add(f2_add(b.x, ntzh), f2_add(zl2, ntzl));
              float k0, k1;
              if constexpr (HasEvalR2<KF>::value) {
                const unsigned long long r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx)));
                float r0, r1;
                f2_unpack(r2, r0, r1);
                k0 = KF::template eval_r2<float>(r0, kp);
                k1 = KF::template eval_r2<float>(r1, kp);
              } else {
                float x0, x1, y0, y1, z0, z1;
                f2_unpack(dx, x0, x1);
                f2_unpack(dy, y0, y1);
                f2_unpack(dz, z0, z1);
                k0 = KF::template eval<float>(x0, y0, z0, kp);
                k1 = KF::template eval<float>(x1, y1, z1, kp);
              }
              if (isinf(k0)) k0 = 0;  // coincident points (include/compute.hpp:767)
              if (isinf(k1)) k1 = 0;
              part2 = f2_fma(f2_pack(k0, k1), b.y, part2);
            }
            float p0, p1;
            f2_unpack(part2, p0, p1);
            acc[0].add(p0 + p1);
          }
          __syncwarp();
        }
      } else {
      for (int v0 = 0; v0 < nsrc_total; v0 += 32) {
        const int v = v0 + lane;
        if (v < nsrc_total) {
          while (v >= s_pre[wl][q + 1]) ++q;
          const int j = s_nb[wl][q][0] + (v - s_pre[wl][q]);
          RelPos<T> sp;
          sp.set(spos[j] - c[0], spos[(int64_t)Ns + j] - c[1], spos[2 * (int64_t)Ns + j] - c[2]);
          V4 h;
          h.x = sp.h[0], h.y = sp.h[1], h.z = sp.h[2], h.w = 0;
          s_sh[wl][lane] = h;
          if constexpr (kMixed) {
            V4 lo;
            lo.x = sp.l[0], lo.y = sp.l[1], lo.z = sp.l[2], lo.w = 0;
            s_sl[wl][lane] = lo;
          }
          const double* wj = wsorted + (int64_t)j * C + c0;
#pragma unroll
          for (int cc = 0; cc < KC; ++cc) s_w[wl][lane][cc] = cc < cg ? (T)wj[cc] : T(0);
        }
        __syncwarp();
        if (active) {
          const int m = min(32, nsrc_total - v0);
          T part[KC];
#pragma unroll
          for (int cc = 0; cc < KC; ++cc) part[cc] = 0;
#pragma unroll 4
          for (int jj = 0; jj < m; ++jj) {
            T d[3];
            tp.diff(s_sh[wl][jj], s_sl[wl][kMixed ? jj : 0], d);
            T kv = KF::template eval<T>(d[0], d[1], d[2], kp);
            if (isinf(kv)) kv = 0;  // coincident points (include/compute.hpp:767)
#pragma unroll
            for (int cc = 0; cc < KC; ++cc)
              if (cc < cg) part[cc] = fma(kv, s_w[wl][jj][cc], part[cc]);
          }
#pragma unroll
          for (int cc = 0; cc < KC; ++cc)
            if (cc < cg) acc[cc].add(part[cc]);
        }
        __syncwarp();
      }
      }
      if (active) {
        const int64_t oi = tperm[i];
#pragma unroll
        for (int cc = 0; cc < KC; ++cc)
          if (cc < cg) out[(int64_t)(c0 + cc) * Nf + oi] += (double)acc[cc].value();
      }
    }
  }
}

// Sparse leaves (fewer than kLaneLeafMin targets): one warp per leaf, all its
// targets at once, their positions and basis values computed once.  With few
// (target, column) pairs (up to TA targets) the lanes run over the sources
// of the 27 neighbour leaves and over the local coefficients, every lane
// holds every pair's partial sum, and one warp reduction per pair ends the
// leaf.  Otherwise the warp stages the sources 32 at a time in shared memory
// (positions relative to the leaf centre and the weights of KC columns),
// evaluates the kernel once per (target, source) pair with the lanes over
// sources, and lane (t, c) -- target group member t, column c -- accumulates
// its targets' sums over the tile from shared memory; its far field (L2P)
// reads the leaf's local coefficients of column c against its target's basis.
// T = float (mixed path): kernel values and per-tile partial sums in float32,
// running sums compensated (Kahan), output update in float64.
template <class KF, typename T, int KC>
__global__ void __launch_bounds__(32 * kLeafWarps, kSparseBlocks<T>)
    k_leaf_sparse(const int* __restrict__ leaves, int nleaves, const int* __restrict__ part_count,
                  const int* __restrict__ tstart, const int* __restrict__ sstart,
                  const int* __restrict__ tperm, const double* __restrict__ tpos,
                  const double* __restrict__ spos, const double* __restrict__ wsorted, int Nf,
                  int Ns, int C, const T* __restrict__ F_L, int n, int cheb,
                  const T* __restrict__ Tkz_g, double box, int L,
                  const double* __restrict__ kparam_g, double* __restrict__ out) {
  constexpr bool kMixed = sizeof(T) == 4;
  constexpr int kMaxT = kLaneLeafMin - 1;             // targets of a sparse leaf
  constexpr int G = KC == 1 ? kMaxT : 32 / KC;        // targets per lane group
  // up to TA targets: every (target, column) sum in each lane instead (one
  // column only: with several, the per-lane sums and reductions cost more
  // than the idle lanes of a short group)
  constexpr int TA = KC == 1 ? kMaxT : 0;
  static_assert(G * KC <= 32, "a lane group fits the warp");
  using V4 = vec4_t<T>;
  __shared__ T sTkz[kMaxOrder * kMaxOrder];
  __shared__ double kp[4];
  __shared__ int s_nb[kLeafWarps][27][2];
  __shared__ int s_pre[kLeafWarps][28];
  __shared__ V4 s_th[kLeafWarps][kMaxT], s_tl[kLeafWarps][kMaxT];  // targets (hi, lo)
  __shared__ T s_b[kLeafWarps][kMaxT][3 * kMaxOrder];              // their basis values
  __shared__ V4 s_sh[kLeafWarps][32], s_sl[kLeafWarps][kMixed ? 32 : 1];  // source tile
  __shared__ T s_w[kLeafWarps][32][KC];                            // its weights
  // kernel values [target][source], or basis products [target][coefficient]
  // (rows padded to 33: lanes of different targets read different banks)
  __shared__ T s_k[kLeafWarps][kMaxT][33];
  __shared__ T s_F[kLeafWarps][KC * 33];  // staged local coefficients [column][coefficient]
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTkz[i] = Tkz_g[i];
  if (threadIdx.x < 4) kp[threadIdx.x] = kparam_g[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int wid = blockIdx.x * kLeafWarps + wl;
  const int nd = *part_count;  // dense leaves come first in the list
  if (wid >= nleaves - nd) return;
  const int leaf = leaves[nd + wid];
  const int ta = tstart[leaf], te = tstart[leaf + 1], nt = te - ta;
  if (nt >= kLaneLeafMin || nt <= 0) return;  // (dense leaves run elsewhere)
  const int n3 = n * n * n;
  double c[3];
  cell_center_d((uint32_t)leaf, L, box, c);
  double len = box;
  for (int i = 0; i < L; ++i) len = 0.5 * len;
  const double ihalfL = 2. / len;
  int ax, ay, az;
  morton_decode((uint32_t)leaf, &ax, &ay, &az);
  const int nside = 1 << L;
  int nb_cnt = 0;
  if (lane < 27) {
    const int q = lane;
    const int bx = ax + q / 9 - 1, by = ay + (q / 3) % 3 - 1, bz = az + q % 3 - 1;
    int a = 0, e = 0;
    if (bx >= 0 && by >= 0 && bz >= 0 && bx < nside && by < nside && bz < nside) {
      const uint32_t bm = morton_encode(bx, by, bz);
      a = sstart[bm];
      e = sstart[bm + 1];
    }
    s_nb[wl][q][0] = a;
    s_nb[wl][q][1] = e;
    nb_cnt = e - a;
  }
  // the targets, relative to the leaf centre, and their basis values
  if (lane < nt) {
    const int i = ta + lane;
    const double x = tpos[i], y = tpos[(int64_t)Nf + i], z = tpos[2 * (int64_t)Nf + i];
    RelPos<T> tp;
    tp.set(x - c[0], y - c[1], z - c[2]);
    V4 h, l;
    h.x = tp.h[0], h.y = tp.h[1], h.z = tp.h[2], h.w = 0;
    l.x = 0, l.y = 0, l.z = 0, l.w = 0;
    if constexpr (kMixed) l.x = tp.l[0], l.y = tp.l[1], l.z = tp.l[2];
    s_th[wl][lane] = h;
    s_tl[wl][lane] = l;
  }
  for (int idx = lane; idx < nt * 3 * n; idx += 32) {
    const int t = idx / (3 * n), d = (idx / n) % 3, m = idx % n;
    const int i = ta + t;
    const double xd = tpos[(int64_t)d * Nf + i];
    s_b[wl][t][d * n + m] = basis_one<T>(n, cheb, (T)(ihalfL * (xd - c[d])), sTkz, m);
  }
  __syncwarp();
  neighbour_prefix(nb_cnt, lane, s_pre[wl]);
  __syncwarp();
  const int nsrc_total = s_pre[wl][27];
  const int tl = lane / KC, cl = lane % KC;  // this lane's target-group member and column
  for (int c0 = 0; c0 < C; c0 += KC) {
    const int kce = min(KC, C - c0);  // columns of this pass
    if constexpr (TA > 0) {
    if (nt <= TA) {
      // Few (target, column) pairs: lanes over sources (and over the
      // coefficients), every pair's sum in each lane, one warp reduction
      // per pair at the end.
      LeafAcc<T> acc[TA][KC];
      // the coefficients four per lane at a time, their loads issued together
      for (int l0 = lane; l0 < n3; l0 += 128) {
        T fv[4][KC];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int l = l0 + 32 * r;
#pragma unroll
          for (int cc = 0; cc < KC; ++cc)
            fv[r][cc] = (l < n3 && cc < kce) ? F_L[((int64_t)leaf * C + c0 + cc) * n3 + l] : T(0);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int l = l0 + 32 * r;
          if (l >= n3) break;
          const int l1 = l / (n * n), l2 = (l / n) % n, l3 = l % n;
#pragma unroll
          for (int t = 0; t < TA; ++t)
            if (t < nt) {
              const T* b = s_b[wl][t];
              const T v = b[l1] * b[n + l2] * b[2 * n + l3];
#pragma unroll
              for (int cc = 0; cc < KC; ++cc)
                if (cc < kce) acc[t][cc].add(fv[r][cc] * v);
            }
        }
      }
      int q = 0;
      for (int v = lane; v < nsrc_total; v += 32) {
        while (v >= s_pre[wl][q + 1]) ++q;
        const int j = s_nb[wl][q][0] + (v - s_pre[wl][q]);
        RelPos<T> sp;
        sp.set(spos[j] - c[0], spos[(int64_t)Ns + j] - c[1], spos[2 * (int64_t)Ns + j] - c[2]);
        V4 sh, sl;
        sh.x = sp.h[0], sh.y = sp.h[1], sh.z = sp.h[2], sh.w = 0;
        sl.x = 0, sl.y = 0, sl.z = 0, sl.w = 0;
        if constexpr (kMixed) sl.x = sp.l[0], sl.y = sp.l[1], sl.z = sp.l[2];
        T w[KC];
        const double* wj = wsorted + (int64_t)j * C + c0;
#pragma unroll
        for (int cc = 0; cc < KC; ++cc) w[cc] = cc < kce ? (T)wj[cc] : T(0);
#pragma unroll
        for (int t = 0; t < TA; ++t)
          if (t < nt) {
            RelPos<T> tp;
            const V4 th = s_th[wl][t];
            tp.h[0] = th.x, tp.h[1] = th.y, tp.h[2] = th.z;
            if constexpr (kMixed) {
              const V4 tlo = s_tl[wl][t];
              tp.l[0] = tlo.x, tp.l[1] = tlo.y, tp.l[2] = tlo.z;
            }
            T d[3];
            tp.diff(sh, sl, d);
            T kv = KF::template eval<T>(d[0], d[1], d[2], kp);
            if (isinf(kv)) kv = 0;  // coincident points (include/compute.hpp:767)
#pragma unroll
            for (int cc = 0; cc < KC; ++cc)
              if (cc < kce) acc[t][cc].add(kv * w[cc]);
          }
      }
#pragma unroll
      for (int t = 0; t < TA; ++t)
#pragma unroll
        for (int cc = 0; cc < KC; ++cc) {
          if (t >= nt || cc >= kce) continue;  // uniform over the warp
          double v = acc[t][cc].value();
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) out[(int64_t)(c0 + cc) * Nf + tperm[ta + t]] += v;
        }
      continue;
    }
    }
    // Many pairs: the targets in groups of G; for each group, lane (t, c)
    // owns group member t and column c, the sources are staged 32 at a time
    // and the kernel is evaluated once per (target, source) pair.  Groups run
    // one after the other (a loop, not unrolled: one accumulator, little
    // code), so the warp keeps few registers and a small instruction
    // footprint.
    const bool col_ok = tl < G && c0 + cl < C;
#pragma unroll 1
    for (int g0 = 0; g0 < nt; g0 += G) {
      const int gn = min(G, nt - g0);  // targets of this group
      const int t = g0 + tl;           // this lane's target
      const bool mine = col_ok && tl < gn;
      LeafAcc<T> acc;
      // far field: phi += sum_l F[l] Sx[l1] Sy[l2] Sz[l3], 32 coefficients at
      // a time: lanes over coefficients load the KC columns (coalesced) and
      // form the group's basis products, then lane (t, c) sums the chunk
      for (int l0 = 0; l0 < n3; l0 += 32) {
        const int l = l0 + lane, mm = min(32, n3 - l0);
        __syncwarp();
        if (l < n3) {
          const int l1 = l / (n * n), l2 = (l / n) % n, l3 = l % n;
#pragma unroll
          for (int cc = 0; cc < KC; ++cc)
            s_F[wl][cc * 33 + lane] =
                cc < kce ? F_L[((int64_t)leaf * C + c0 + cc) * n3 + l] : T(0);
          for (int u = 0; u < gn; ++u) {
            const T* bb = s_b[wl][g0 + u];
            s_k[wl][u][lane] = bb[l1] * bb[n + l2] * bb[2 * n + l3];
          }
        }
        __syncwarp();
        if (mine) {
          T part = 0;
          for (int jj = 0; jj < mm; ++jj) part = fma(s_F[wl][cl * 33 + jj], s_k[wl][tl][jj], part);
          acc.add(part);
        }
      }
      // near field: the neighbours' sources in tiles of 32
      int q = 0;
      for (int v0 = 0; v0 < nsrc_total; v0 += 32) {
        const int v = v0 + lane, m = min(32, nsrc_total - v0);
        __syncwarp();
        if (v < nsrc_total) {
          while (v >= s_pre[wl][q + 1]) ++q;
          const int j = s_nb[wl][q][0] + (v - s_pre[wl][q]);
          RelPos<T> sp;
          sp.set(spos[j] - c[0], spos[(int64_t)Ns + j] - c[1], spos[2 * (int64_t)Ns + j] - c[2]);
          V4 h;
          h.x = sp.h[0], h.y = sp.h[1], h.z = sp.h[2], h.w = 0;
          s_sh[wl][lane] = h;
          if constexpr (kMixed) {
            V4 lo;
            lo.x = sp.l[0], lo.y = sp.l[1], lo.z = sp.l[2], lo.w = 0;
            s_sl[wl][lane] = lo;
          }
          const double* wj = wsorted + (int64_t)j * C + c0;
#pragma unroll
          for (int cc = 0; cc < KC; ++cc) s_w[wl][lane][cc] = c0 + cc < C ? (T)wj[cc] : T(0);
        }
        __syncwarp();
        // kernel values: lanes over the tile's sources, one target at a time
        if (lane < m) {
          const V4 sh = s_sh[wl][lane];
          const V4 sl = s_sl[wl][kMixed ? lane : 0];
          for (int u = 0; u < gn; ++u) {
            RelPos<T> tp;
            const V4 th = s_th[wl][g0 + u];
            tp.h[0] = th.x, tp.h[1] = th.y, tp.h[2] = th.z;
            if constexpr (kMixed) {
              const V4 tlo = s_tl[wl][g0 + u];
              tp.l[0] = tlo.x, tp.l[1] = tlo.y, tp.l[2] = tlo.z;
            }
            T d[3];
            tp.diff(sh, sl, d);
            T kv = KF::template eval<T>(d[0], d[1], d[2], kp);
            if (isinf(kv)) kv = 0;  // coincident points (include/compute.hpp:767)
            s_k[wl][u][lane] = kv;
          }
        }
        __syncwarp();
        // sums over the tile: lane (t, c)
        if (mine) {
          T part = 0;
          for (int jj = 0; jj < m; ++jj) part = fma(s_k[wl][tl][jj], s_w[wl][jj][cl], part);
          acc.add(part);
        }
      }
      if (mine) out[(int64_t)(c0 + cl) * Nf + tperm[ta + t]] += (double)acc.value();
    }
  }
}

// Gradient leaf phase (adjoint and position gradients): for each target x
// and column c, phi_c(x) = sum_l F_lc S_l(x) + sum_j w_jc K(x, y_j) and its
// gradient, from the differentiated interpolation basis (chain factor
// 2 / cell length) and the kernel gradient.  grad_out[i*3 + d] gets
// sum_c contract[c*Nf + i] d phi_c / d x_d; out[c*Nf + i] gets phi_c when
// non-null.  One warp per target leaf, one target at a time, lanes over its
// sources and coefficients.
constexpr int kGradCols = 4;  // columns per pass (4 accumulators each)

template <class KF, typename T>
__global__ void __launch_bounds__(32 * kLeafWarps)
    k_leaf_grad(const int* __restrict__ leaves, int nleaves, const int* __restrict__ tstart,
                const int* __restrict__ sstart, const int* __restrict__ tperm,
                const double* __restrict__ tpos, const double* __restrict__ spos,
                const double* __restrict__ wsorted, int Nf, int Ns, int C,
                const T* __restrict__ F_L, int n, int cheb, const T* __restrict__ Tkz_g,
                double box, int L, const double* __restrict__ kparam_g, double* __restrict__ out,
                const double* __restrict__ contract, double* __restrict__ grad_out) {
  __shared__ T sTkz[kMaxOrder * kMaxOrder];
  __shared__ double kp[4];
  __shared__ int s_nb[kLeafWarps][27][2];
  __shared__ int s_pre[kLeafWarps][28];
  __shared__ T s_b[kLeafWarps][6 * kMaxOrder];  // S_m per dimension, then dS_m/dx
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTkz[i] = Tkz_g[i];
  if (threadIdx.x < 4) kp[threadIdx.x] = kparam_g[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int wid = blockIdx.x * kLeafWarps + wl;
  if (wid >= nleaves) return;
  const int leaf = leaves[wid];
  const int ta = tstart[leaf], te = tstart[leaf + 1];
  const int n3 = n * n * n;
  double c[3];
  cell_center_d((uint32_t)leaf, L, box, c);
  double len = box;
  for (int i = 0; i < L; ++i) len = 0.5 * len;
  const double ihalfL = 2. / len;
  int ax, ay, az;
  morton_decode((uint32_t)leaf, &ax, &ay, &az);
  const int nside = 1 << L;
  int nb_cnt = 0;
  if (lane < 27) {
    const int q = lane;
    const int bx = ax + q / 9 - 1, by = ay + (q / 3) % 3 - 1, bz = az + q % 3 - 1;
    int a = 0, e = 0;
    if (bx >= 0 && by >= 0 && bz >= 0 && bx < nside && by < nside && bz < nside) {
      const uint32_t bm = morton_encode(bx, by, bz);
      a = sstart[bm];
      e = sstart[bm + 1];
    }
    s_nb[wl][q][0] = a;
    s_nb[wl][q][1] = e;
    nb_cnt = e - a;
  }
  __syncwarp();
  neighbour_prefix(nb_cnt, lane, s_pre[wl]);
  __syncwarp();
  const int nsrc_total = s_pre[wl][27];
  const T* Sb = s_b[wl];
  const T* Db = s_b[wl] + 3 * n;
  for (int c0 = 0; c0 < C; c0 += kGradCols) {
    const int cg = min(kGradCols, C - c0);
    for (int i = ta; i < te; ++i) {
      const double x = tpos[i], y = tpos[(int64_t)Nf + i], z = tpos[2 * (int64_t)Nf + i];
      __syncwarp();
      if (lane < 3 * n) {
        const int d = lane / n, mm = lane % n;
        const T u = (T)(ihalfL * ((d == 0 ? x : d == 1 ? y : z) - c[d]));
        s_b[wl][d * n + mm] = basis_one<T>(n, cheb, u, sTkz, mm);
        s_b[wl][3 * n + d * n + mm] = basis_deriv<T>(n, cheb, u, sTkz, mm) * (T)ihalfL;
      }
      __syncwarp();
      LeafAcc<T> v[kGradCols], g[kGradCols][3];
      const T* Fl = F_L + ((int64_t)leaf * C + c0) * n3;
      for (int l = lane; l < n3; l += 32) {
        const int l1 = l / (n * n), l2 = (l / n) % n, l3 = l % n;
        const T b1 = Sb[l1], b2 = Sb[n + l2], b3 = Sb[2 * n + l3];
        const T e0 = Db[l1] * b2 * b3, e1 = b1 * Db[n + l2] * b3, e2 = b1 * b2 * Db[2 * n + l3];
        const T val = b1 * b2 * b3;
#pragma unroll
        for (int cc = 0; cc < kGradCols; ++cc)
          if (cc < cg) {
            const T f = Fl[cc * n3 + l];
            v[cc].add(f * val);
            g[cc][0].add(f * e0);
            g[cc][1].add(f * e1);
            g[cc][2].add(f * e2);
          }
      }
      int q = 0;
      for (int vv = lane; vv < nsrc_total; vv += 32) {
        while (vv >= s_pre[wl][q + 1]) ++q;
        const int j = s_nb[wl][q][0] + (vv - s_pre[wl][q]);
        const T dx = (T)(spos[j] - x), dy = (T)(spos[(int64_t)Ns + j] - y),
                dz = (T)(spos[2 * (int64_t)Ns + j] - z);
        T gk[3];
        T kv = KF::template grad<T>(dx, dy, dz, kp, gk);
        if (isinf(kv)) kv = 0;  // coincident points (include/compute.hpp:767)
        const double* wj = wsorted + (int64_t)j * C + c0;
#pragma unroll
        for (int cc = 0; cc < kGradCols; ++cc)
          if (cc < cg) {
            const T w = (T)wj[cc];
            v[cc].add(kv * w);
            // d K(x, y_j) / d x = -dK/dd with d = y_j - x
            g[cc][0].add(-gk[0] * w);
            g[cc][1].add(-gk[1] * w);
            g[cc][2].add(-gk[2] * w);
          }
      }
      double tv[kGradCols], tg[kGradCols][3];
#pragma unroll
      for (int cc = 0; cc < kGradCols; ++cc) {
        double a = v[cc].value(), b0 = g[cc][0].value(), b1 = g[cc][1].value(),
               b2 = g[cc][2].value();
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          a += __shfl_xor_sync(0xffffffffu, a, o);
          b0 += __shfl_xor_sync(0xffffffffu, b0, o);
          b1 += __shfl_xor_sync(0xffffffffu, b1, o);
          b2 += __shfl_xor_sync(0xffffffffu, b2, o);
        }
        tv[cc] = a, tg[cc][0] = b0, tg[cc][1] = b1, tg[cc][2] = b2;
      }
      if (lane == 0) {
        const int64_t oi = tperm[i];
        double gs[3] = {0, 0, 0};
#pragma unroll
        for (int cc = 0; cc < kGradCols; ++cc)
          if (cc < cg) {
            if (out) out[(int64_t)(c0 + cc) * Nf + oi] += tv[cc];
            if (grad_out) {
              const double wc = contract[(int64_t)(c0 + cc) * Nf + oi];
              gs[0] += wc * tg[cc][0], gs[1] += wc * tg[cc][1], gs[2] += wc * tg[cc][2];
            }
          }
        if (grad_out)
          for (int d = 0; d < 3; ++d) grad_out[oi * 3 + d] += gs[d];
      }
    }
  }
}

// Whether a kernel functor provides the gradient (KF::has_gradient).
template <class KF, class = void>
struct kf_has_gradient : std::false_type {};
template <class KF>
struct kf_has_gradient<KF, typename std::enable_if<KF::has_gradient>::type> : std::true_type {};

template <class KF, typename T>
inline int launch_leaf_kernels_t(const pbbfmm_leaf_args& a, cudaStream_t st) {
  const T* F = static_cast<const T*>(a.F_leaf);
  const T* Tkz = static_cast<const T*>(a.Tkz);
  if (a.gradient) {
    if constexpr (kf_has_gradient<KF>::value) {
      k_leaf_grad<KF, T><<<(a.nleaves + kLeafWarps - 1) / kLeafWarps, 32 * kLeafWarps, 0, st>>>(
          a.leaves, a.nleaves, a.tstart, a.sstart, a.tperm, a.tpos, a.spos, a.wsorted, a.Nf, a.Ns,
          a.C, F, a.n, a.cheb, Tkz, a.box, a.L, a.kparam, a.out, a.contract, a.grad_out);
      return (int)cudaGetLastError();
    } else {
      return -1;  // no gradient: the caller reports PBBFMM_ERR_UNSUPPORTED
    }
  }
  // dense leaves (32-target chunks, one warp each), then the sparse ones; one
  // column: registers for one, otherwise columns in passes of kLeafCols
  const size_t dyn = sizeof(T) * kLeafWarps * 3 * a.n * 32;
  for (int dense = 1; dense >= 0; --dense) {
    if (dense) {
      auto kern = a.C == 1 ? k_leaf<KF, T, 1> : k_leaf<KF, T, kLeafCols>;
      kern<<<(unsigned)((a.max_chunks + kLeafWarps - 1) / kLeafWarps), 32 * kLeafWarps, dyn, st>>>(
          a.leaves, a.nleaves, a.ndense, a.chunk_prefix, a.tstart, a.sstart, a.tperm, a.tpos,
          a.spos, a.wsorted, a.Nf, a.Ns, a.C, F, a.n, a.cheb, Tkz, a.box, a.L, a.kparam, a.out);
    } else {
      auto kern = a.C == 1 ? k_leaf_sparse<KF, T, 1> : k_leaf_sparse<KF, T, kLeafCols>;
      kern<<<(unsigned)((a.nleaves + kLeafWarps - 1) / kLeafWarps), 32 * kLeafWarps, 0, st>>>(
          a.leaves, a.nleaves, a.ndense, a.tstart, a.sstart, a.tperm, a.tpos, a.spos, a.wsorted,
          a.Nf, a.Ns, a.C, F, a.n, a.cheb, Tkz, a.box, a.L, a.kparam, a.out);
    }
    if (const cudaError_t e = cudaGetLastError()) return (int)e;
  }
  return 0;
}

// Launch the leaf phase described by `a` for the kernel functor KF on
// `stream`: 0 on success, a cudaError_t code if a launch failed, -1 when a
// gradient pass is asked of a functor without gradient.  Launches 2 kernels
// (values) or 1 (gradient).
template <class KF>
inline int launch_leaf_kernels(const pbbfmm_leaf_args& a, cudaStream_t st) {
  return a.precision == PBBFMM_PREC_FP64 ? launch_leaf_kernels_t<KF, double>(a, st)
                                         : launch_leaf_kernels_t<KF, float>(a, st);
}

}  // namespace pbbfmm

#endif  // PBBFMM3D_B200_LEAF_CUH
