// Uniform-grid far field in float64: FFT of the padded moments, the
// frequency-domain M2L, and the inverse FFT to local coefficients.
//
// Reference: UpwardPass padding + R2HC (include/compute.hpp:337-372),
// FarFieldInteractions / FrequencyProduct / HC2R (include/compute.hpp:
// 488-544, 930-943) and the stencils of ComputeKernelUnif
// (src/H2_3D_Tree.cpp:585-648).
//
// The reference embeds the n^3 moments in a length-(2n-1)^3 vector at offset
// (P-1)/2 and uses a 1-D circular correlation of length P; because the offset
// digits never carry, that equals the 3-D Toeplitz product
//     y[a] = sum_b A[n-1+b-a] x[b],   a, b in [0,n)^3,  A the (2n-1)^3 stencil,
// which is what runs here, as a 3-D real DFT on the m^3 grid (m = 2n-1):
// x placed at grid position b, y read at grid position (a + n) mod m, and
// the operator spectra stored as conj(DFT3(A)).  Only the k3 < n half of each
// spectrum is kept (Hermitian symmetry), nk = m*m*n complex values per cell
// and column.  Same sums as the reference, different rounding.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "fmm.cuh"

namespace pbbfmm {

// ----------------------------------------------------------------- FFT
// Each thread computes one whole 1-D transform of a stage: its n (or m)
// inputs are read once from shared memory and every output is accumulated in
// registers, with the loops fully unrolled so that every twiddle index
// (k l mod m) is a compile-time constant into the __constant__ tables below
// (constant-bank operands of the FMAs, no loads).

// cos / sin of 2 pi j / m for m = 2n - 1, n = 2..kMaxOrder, back to back.
constexpr int kTwTotal = kMaxOrder * kMaxOrder - 1;  // sum_{n=2}^{N} (2n - 1)
__host__ __device__ constexpr int tw_off(int n) { return n <= 2 ? 0 : tw_off(n - 1) + 2 * n - 3; }
__constant__ double c_tw_cos_d[kTwTotal];
__constant__ double c_tw_sin_d[kTwTotal];
__constant__ float c_tw_cos_f[kTwTotal];
__constant__ float c_tw_sin_f[kTwTotal];

template <int n, typename T>
struct Tw {
  static constexpr int m = 2 * n - 1, off = tw_off(n);
  static __device__ __forceinline__ T c(int j) {
    if constexpr (sizeof(T) == 8) return c_tw_cos_d[off + j];
    else return c_tw_cos_f[off + j];
  }
  static __device__ __forceinline__ T s(int j) {
    if constexpr (sizeof(T) == 8) return c_tw_sin_d[off + j];
    else return c_tw_sin_f[off + j];
  }
};

// Fill the tables on the current device (once per device).
int init_fft_twiddles() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  PB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && done[dev]) return PBBFMM_OK;
  double cd[kTwTotal], sd[kTwTotal];
  float cf[kTwTotal], sf[kTwTotal];
  for (int n = 2; n <= kMaxOrder; ++n) {
    const int m = 2 * n - 1;
    for (int j = 0; j < m; ++j) {
      cd[tw_off(n) + j] = cos(2.0 * M_PI * j / m);
      sd[tw_off(n) + j] = sin(2.0 * M_PI * j / m);
      cf[tw_off(n) + j] = (float)cd[tw_off(n) + j];
      sf[tw_off(n) + j] = (float)sd[tw_off(n) + j];
    }
  }
  PB_CUDA(cudaMemcpyToSymbol(c_tw_cos_d, cd, sizeof(cd)));
  PB_CUDA(cudaMemcpyToSymbol(c_tw_sin_d, sd, sizeof(sd)));
  PB_CUDA(cudaMemcpyToSymbol(c_tw_cos_f, cf, sizeof(cf)));
  PB_CUDA(cudaMemcpyToSymbol(c_tw_sin_f, sf, sizeof(sf)));
  if (dev < 64) done[dev] = true;
  return PBBFMM_OK;
}

// Length-9 transforms (order 5) by one radix-3 step, with l = b + 3a:
//   forward, 5 inputs:  X[k] = U0[k%3] + w^k U1[k%3] + w^2k v2,
//     U0[j] = v0 + v3 w^3j, U1[j] = v1 + v4 w^3j;
//   inverse, 9 inputs:  X[t] = sum_b w^-bt V_b[t%3], V_b[j] = sum_a v[b+3a] w^-3aj,
// for w = e^{-2 pi i / 9}; about half the multiply-adds of the direct sums.
// (a + ib) w^j = (a c + b s) + i (b c - a s), (a + ib) w^-j = (a c - b s) + i (b c + a s).
template <int n, typename T>
__device__ __forceinline__ cplx_t<T> mul_w(cplx_t<T> x, int j) {
  using W = Tw<n, T>;
  return make_cplx<T>(fma(x.x, W::c(j), x.y * W::s(j)), fma(x.y, W::c(j), -x.x * W::s(j)));
}
template <int n, typename T>
__device__ __forceinline__ cplx_t<T> mul_wc(cplx_t<T> x, int j) {
  using W = Tw<n, T>;
  return make_cplx<T>(fma(x.x, W::c(j), -x.y * W::s(j)), fma(x.y, W::c(j), x.x * W::s(j)));
}
// forward 5 -> 9, out(k, X[k]) for k = 0..8
template <int n, typename T, class Out>
__device__ __forceinline__ void dft_5_to_9(const cplx_t<T>* v, Out out) {
  static_assert(2 * n - 1 == 9, "length-9 transform");
  using W = Tw<n, T>;
  cplx_t<T> u0[3], u1[3];
  u0[0] = make_cplx<T>(v[0].x + v[3].x, v[0].y + v[3].y);
  u1[0] = make_cplx<T>(v[1].x + v[4].x, v[1].y + v[4].y);
#pragma unroll
  for (int j = 1; j < 3; ++j) {
    const cplx_t<T> a = mul_w<n, T>(v[3], 3 * j), b = mul_w<n, T>(v[4], 3 * j);
    u0[j] = make_cplx<T>(v[0].x + a.x, v[0].y + a.y);
    u1[j] = make_cplx<T>(v[1].x + b.x, v[1].y + b.y);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const cplx_t<T> a = u0[k % 3], b = u1[k % 3], c = v[2];
    const int j1 = k, j2 = (2 * k) % 9;
    T re = fma(c.x, W::c(j2), fma(c.y, W::s(j2), a.x));
    re = fma(b.x, W::c(j1), fma(b.y, W::s(j1), re));
    T im = fma(c.y, W::c(j2), fma(-c.x, W::s(j2), a.y));
    im = fma(b.y, W::c(j1), fma(-b.x, W::s(j1), im));
    out(k, make_cplx<T>(re, im));
  }
}
// inverse 9 -> 5 at t = (a + 5) mod 9, out(a, X[t]) for a = 0..4
template <int n, typename T, class Out>
__device__ __forceinline__ void idft_9_to_5(const cplx_t<T>* v, Out out) {
  static_assert(2 * n - 1 == 9, "length-9 transform");
  using W = Tw<n, T>;
  cplx_t<T> vb[3][3];  // [b][j]
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const cplx_t<T> x0 = v[b], x1 = v[b + 3], x2 = v[b + 6];
    vb[b][0] = make_cplx<T>(x0.x + x1.x + x2.x, x0.y + x1.y + x2.y);
#pragma unroll
    for (int j = 1; j < 3; ++j) {
      const cplx_t<T> p = mul_wc<n, T>(x1, 3 * j), q = mul_wc<n, T>(x2, (6 * j) % 9);
      vb[b][j] = make_cplx<T>(x0.x + p.x + q.x, x0.y + p.y + q.y);
    }
  }
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const int t = (a + 5) % 9, j = t % 3;
    const cplx_t<T> y0 = vb[0][j], y1 = vb[1][j], y2 = vb[2][j];
    const int j1 = t, j2 = (2 * t) % 9;
    T re = fma(y2.x, W::c(j2), fma(-y2.y, W::s(j2), y0.x));
    re = fma(y1.x, W::c(j1), fma(-y1.y, W::s(j1), re));
    T im = fma(y2.y, W::c(j2), fma(y2.x, W::s(j2), y0.y));
    im = fma(y1.y, W::c(j1), fma(y1.x, W::s(j1), im));
    out(a, make_cplx<T>(re, im));
  }
}

// Spectra of a level are stored frequency-major: X[(k * ncells + cell) * C + col]
// (ncells = 8^level), so that one frequency plane of a level is contiguous.

// Forward: CTAs loop over the nonempty source cells (cells[0..ncl)), columns
// in groups of CG.  With amax (float path, levels of the tensor-core MAC), a
// bound on |re| and |im| of the spectra per (k23, column mod 8), over the
// level's cells and k1, as float bits: the sum of |re| + |im| of the last
// transform's n inputs (a bound on every one of its m outputs), per CTA in
// shared memory, then one atomicMax per slot into amax[k23][8] (zeroed by
// the caller).
// w = e^{-2 pi i / m}; (a + ib) w^j = (a c + b s) + i (b c - a s).
template <int n, typename T>
__global__ void k_fft_fwd(const int* __restrict__ cells, int ncl, const T* __restrict__ S_l,
                          cplx_t<T>* __restrict__ X_l, int64_t ncells, int C, int CG,
                          const T* __restrict__ twid, unsigned* __restrict__ amax) {
  using C2 = cplx_t<T>;
  using W = Tw<n, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  constexpr int m = 2 * n - 1, n2 = n * n, n3 = n2 * n, ny = n * m * n;
  const int sin_stride = (CG * n3 + 3) & ~3;
  T* sin_buf = sm + 2 * m;                      // 2 x CG * n3 real moments (double-buffered)
  C2* Z = (C2*)(sin_buf + 2 * sin_stride);      // CG * n * n * n   (l1, l2, k3)
  C2* Y = Z + CG * n3;                         // CG * n * m * n   (l1, k2, k3)
  unsigned* s_amax = reinterpret_cast<unsigned*>(Y + CG * ny);  // [m n][8]
  (void)twid;
  const int tid = threadIdx.x, bd = blockDim.x;
  if (amax)
    for (int i = tid; i < m * n * 8; i += bd) s_amax[i] = 0u;
  // work units (cell, column group) of this CTA in order; each unit's moments
  // are copied (cp.async) into the other buffer while the previous unit is
  // transformed
  const int ngrp = (C + CG - 1) / CG;
  auto fetch = [&](int u, int buf) {
    const int ci = blockIdx.x + (u / ngrp) * gridDim.x;
    if (ci < ncl) {
      const int c0 = (u % ngrp) * CG, cg = min(CG, C - c0);
      const T* src = S_l + ((int64_t)cells[ci] * C + c0) * n3;
      T* dst = sin_buf + buf * sin_stride;
      for (int i = tid; i < cg * n3; i += bd) cp_async_elem(dst + i, src + i, true);
    }
    cp_async_commit();
  };
  int unit = 0;
  fetch(0, 0);
  for (int ci = blockIdx.x; ci < ncl; ci += gridDim.x) {
  const int cell = cells[ci];
  for (int c0 = 0; c0 < C; c0 += CG, ++unit) {
    const int cg = min(CG, C - c0);
    __syncthreads();  // the previous unit's readers of the other buffer are done
    fetch(unit + 1, (unit + 1) & 1);
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    __syncthreads();
    const T* sin_ = sin_buf + (unit & 1) * sin_stride;
    // z: Z[c][l1][l2][k3] = sum_l3 S[c][l1][l2][l3] w^(k3 l3), real input
    for (int job = tid; job < cg * n2; job += bd) {
      const T* s = sin_ + job * n;
      T x[n];
#pragma unroll
      for (int l = 0; l < n; ++l) x[l] = s[l];
      C2* z = Z + job * n;
#pragma unroll
      for (int k = 0; k < n; ++k) {
        T re = 0, im = 0;
#pragma unroll
        for (int l = 0; l < n; ++l) {
          re = fma(x[l], W::c((k * l) % m), re);
          im = fma(-x[l], W::s((k * l) % m), im);
        }
        z[k] = make_cplx<T>(re, im);
      }
    }
    __syncthreads();
    // y: Y[c][l1][k2][k3] = sum_l2 Z[c][l1][l2][k3] w^(k2 l2); job (c, l1, k3)
    for (int job = tid; job < cg * n2; job += bd) {
      const int k3 = job % n, l1 = (job / n) % n, cc = job / n2;
      const C2* z = Z + cc * n3 + l1 * n2 + k3;
      C2 v[n];
#pragma unroll
      for (int l = 0; l < n; ++l) v[l] = z[l * n];
      C2* y = Y + cc * ny + l1 * m * n + k3;
      if constexpr (m == 9) {
        dft_5_to_9<n, T>(v, [&](int k, C2 r) { y[k * n] = r; });
      } else {
#pragma unroll
        for (int k = 0; k < m; ++k) {
          T re = 0, im = 0;
#pragma unroll
          for (int l = 0; l < n; ++l) {
            const T c = W::c((k * l) % m), s = W::s((k * l) % m);
            re = fma(v[l].x, c, fma(v[l].y, s, re));
            im = fma(v[l].y, c, fma(-v[l].x, s, im));
          }
          y[k * n] = make_cplx<T>(re, im);
        }
      }
    }
    __syncthreads();
    // x: X[k1][k2][k3][c] = sum_l1 Y[c][l1][k2][k3] w^(k1 l1); job (k23, c), c fastest
    for (int job = tid; job < cg * m * n; job += bd) {
      const int cc = job % cg, k23 = job / cg;
      const C2* y = Y + cc * ny + k23;
      C2 v[n];
#pragma unroll
      for (int l = 0; l < n; ++l) v[l] = y[l * m * n];
      C2* out = X_l + ((int64_t)k23 * ncells + cell) * C + c0 + cc;
      if constexpr (sizeof(T) == 4) {
        if (amax) {  // |X_k1| <= sum_l |v_l| <= sum_l (|re| + |im|) for every k1
          float bnd = 0.f;
#pragma unroll
          for (int l = 0; l < n; ++l) bnd += fabsf(v[l].x) + fabsf(v[l].y);
          atomicMax(&s_amax[k23 * 8 + ((c0 + cc) & 7)], __float_as_uint(bnd));
        }
      }
      const int64_t kstride = (int64_t)m * n * ncells * C;
      if constexpr (m == 9) {
        dft_5_to_9<n, T>(v, [&](int k, C2 r) { out[k * kstride] = r; });
      } else {
#pragma unroll
        for (int k = 0; k < m; ++k) {
          T re = 0, im = 0;
#pragma unroll
          for (int l = 0; l < n; ++l) {
            const T c = W::c((k * l) % m), s = W::s((k * l) % m);
            re = fma(v[l].x, c, fma(v[l].y, s, re));
            im = fma(v[l].y, c, fma(-v[l].x, s, im));
          }
          out[k * kstride] = make_cplx<T>(re, im);
        }
      }
    }
  }
  }
  cp_async_wait_all();  // the (empty) prefetch past the last unit
  if (amax) {
    __syncthreads();
    for (int i = tid; i < m * n * 8; i += bd)
      if (s_amax[i]) atomicMax(&amax[i], s_amax[i]);
  }
}

// Inverse: one CTA per nonempty target cell.  F = scale * IDFT(Y)/P at grid
// positions (a + n) mod m; (a + ib) e^{+2 pi i j / m} = (a c - b s) + i (b c + a s).
template <int n, typename T>
__global__ void k_fft_inv(const int* __restrict__ cells, const cplx_t<T>* __restrict__ Y_l,
                          T* __restrict__ F_l, int64_t ncells, int C, int CG,
                          const T* __restrict__ twid, T invP, T scale) {
  using C2 = cplx_t<T>;
  using W = Tw<n, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  constexpr int m = 2 * n - 1, n2 = n * n, n3 = n2 * n, nk = m * m * n, ng = n * m * n;
  C2* Yh = (C2*)(sm + ((2 * m + 3) & ~3));  // CG * nk   (k1, k2, k3)
  C2* G = Yh + CG * nk;                     // CG * n*m*n (a1, k2, k3)
  C2* H = G + CG * ng;                      // CG * n3    (a1, a2, k3)
  (void)twid;
  const int cell = cells[blockIdx.x];
  const int tid = threadIdx.x, bd = blockDim.x;
  for (int c0 = 0; c0 < C; c0 += CG) {
    const int cg = min(CG, C - c0);
    __syncthreads();
    for (int i = tid; i < cg * nk; i += bd) {
      const int k = i / cg, cc = i % cg;
      cp_async_cplx(&Yh[cc * nk + k], &Y_l[((int64_t)k * ncells + cell) * C + c0 + cc], true);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    // x: G[c][a1][k2][k3] = sum_k1 Yh[c][k1][k2][k3] e^{+2 pi i k1 t1 / m}; job (c, k23)
    for (int job = tid; job < cg * m * n; job += bd) {
      const int k23 = job % (m * n), cc = job / (m * n);
      const C2* y = Yh + cc * nk + k23;
      C2 v[m];
#pragma unroll
      for (int k = 0; k < m; ++k) v[k] = y[k * m * n];
      C2* g = G + cc * ng + k23;
      if constexpr (m == 9) {
        idft_9_to_5<n, T>(v, [&](int a, C2 r) { g[a * m * n] = r; });
      } else {
#pragma unroll
        for (int a = 0; a < n; ++a) {
          const int t = (a + n) % m;
          T re = 0, im = 0;
#pragma unroll
          for (int k = 0; k < m; ++k) {
            const T c = W::c((k * t) % m), s = W::s((k * t) % m);
            re = fma(v[k].x, c, fma(-v[k].y, s, re));
            im = fma(v[k].y, c, fma(v[k].x, s, im));
          }
          g[a * m * n] = make_cplx<T>(re, im);
        }
      }
    }
    __syncthreads();
    // y: H[c][a1][a2][k3] = sum_k2 G[c][a1][k2][k3] e^{+2 pi i k2 t2 / m}; job (c, a1, k3)
    for (int job = tid; job < cg * n2; job += bd) {
      const int k3 = job % n, a1 = (job / n) % n, cc = job / n2;
      const C2* g = G + cc * ng + a1 * m * n + k3;
      C2 v[m];
#pragma unroll
      for (int k = 0; k < m; ++k) v[k] = g[k * n];
      C2* h = H + cc * n3 + a1 * n2 + k3;
      if constexpr (m == 9) {
        idft_9_to_5<n, T>(v, [&](int a, C2 r) { h[a * n] = r; });
      } else {
#pragma unroll
        for (int a = 0; a < n; ++a) {
          const int t = (a + n) % m;
          T re = 0, im = 0;
#pragma unroll
          for (int k = 0; k < m; ++k) {
            const T c = W::c((k * t) % m), s = W::s((k * t) % m);
            re = fma(v[k].x, c, fma(-v[k].y, s, re));
            im = fma(v[k].y, c, fma(v[k].x, s, im));
          }
          h[a * n] = make_cplx<T>(re, im);
        }
      }
    }
    __syncthreads();
    // z (complex to real over the Hermitian half):
    // out = Re H[..][0] + 2 sum_{k3>=1} Re(H[..][k3] e^{+2 pi i k3 t3 / m}); job (c, a1, a2)
    for (int job = tid; job < cg * n2; job += bd) {
      const C2* h = H + job * n;
      C2 v[n];
#pragma unroll
      for (int k = 0; k < n; ++k) v[k] = h[k];
      T* out = F_l + ((int64_t)cell * C + c0) * n3 + job * n;
#pragma unroll
      for (int a = 0; a < n; ++a) {
        const int t = (a + n) % m;
        T acc = v[0].x;
#pragma unroll
        for (int k = 1; k < n; ++k)
          acc = fma(T(2), fma(v[k].x, W::c((k * t) % m), -v[k].y * W::s((k * t) % m)), acc);
        out[a] = scale * (acc * invP);
      }
    }
  }
}

// ----------------------------------------------------------------- MAC
// One CTA per (block of PBX x 2 x 2 parents = 2PBX x 4 x 4 targets,
// frequency chunk), the frequency chunk varying slowest in the grid so that
// resident CTAs work on the same frequency plane (one plane of level 6 is
// 33.5 MB and stays in L2 while its halo reuse is served).  Threads =
// (parent, kc, col); each thread accumulates the 8 children of its parent for
// one frequency and one column, sweeping the 6x6x6 children of the parent's
// neighbours, staged in shared memory for the whole block ((2PBX+4) x 8 x 8
// cells).  The (child, source) interaction pattern and the operator index are
// compile-time constants; each complex accumulator is split over four
// independent FMA chains.
//
// Per level, halo[b*stride + r] holds the source cell of region slot r of
// parent block b (or -1: outside the domain or no sources), followed by the
// target cell of each block slot (or -1).

template <int PBX>
struct MacGeom {
  static constexpr int RX = 2 * PBX + 4;       // region extent in x (y, z: 8)
  static constexpr int RC = RX * 64;           // region cells
  static constexpr int TC = 2 * PBX * 16;      // target cells of a block
  static constexpr int STRIDE = RC + TC;       // halo table entries per block
  static constexpr int NPAR = PBX * 4;         // parents per block
};

template <int PBX>
__global__ void k_halo_tables(const int* __restrict__ sstart, const int* __restrict__ tstart,
                              int span, int lev, int* __restrict__ halo) {
  using G = MacGeom<PBX>;
  const int nby = 1 << (lev - 2), nbx = (1 << (lev - 1)) / PBX;  // blocks per dim
  const int b = blockIdx.x;
  const int bx = b / (nby * nby), by = (b / nby) % nby, bz = b % nby;
  const int nside = 1 << lev;
  for (int r = threadIdx.x; r < G::STRIDE; r += blockDim.x) {
    int v = -1;
    if (r < G::RC) {
      const int x = 2 * PBX * bx - 2 + (r >> 6), y = 4 * by - 2 + ((r >> 3) & 7),
                z = 4 * bz - 2 + (r & 7);
      if (x >= 0 && y >= 0 && z >= 0 && x < nside && y < nside && z < nside) {
        const uint32_t cm = morton_encode(x, y, z);
        if (sstart[(int64_t)(cm + 1) * span] > sstart[(int64_t)cm * span]) v = (int)cm;
      }
    } else {
      const int q = r - G::RC;
      const uint32_t cm =
          morton_encode(2 * PBX * bx + (q >> 4), 4 * by + ((q >> 2) & 3), 4 * bz + (q & 3));
      if (tstart[(int64_t)(cm + 1) * span] > tstart[(int64_t)cm * span]) v = (int)cm;
    }
    halo[(int64_t)b * G::STRIDE + r] = v;
  }
  (void)nbx;
}

// One sx slab of the MAC: the 6 x 6 (sy, sz) sources of the slab against
// the 8 children.  F0 / F1: children with tx = 0 / 1 are far in x at this sx
// (|sx - 2 - tx| > 1), so every interaction test is a compile-time constant.
template <bool F0, bool F1, int RS, typename C2, typename T>
__device__ __forceinline__ void mac_slab(const C2* __restrict__ rrow, const C2* __restrict__ orow,
                                         int py, int pz, T* ar, T* br, T* ai, T* bi) {
#pragma unroll
  for (int sy = 0; sy < 6; ++sy)
#pragma unroll
    for (int sz = 0; sz < 6; ++sz) {
      const int r = ((2 * py + sy) << 3) | (2 * pz + sz);
      const C2 xv = rrow[r * RS];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int tx = (t >> 2) & 1;
        const int oy = sy - 2 - ((t >> 1) & 1);
        const int oz = sz - 2 - (t & 1);
        const bool far_yz = oy > 1 || oy < -1 || oz > 1 || oz < -1;
        if (far_yz || (tx ? F1 : F0)) {
          const C2 a = orow[-49 * tx + 7 * (oy + 3) + (oz + 3)];
          ar[t] = fma(a.x, xv.x, ar[t]);
          br[t] = fma(-a.y, xv.y, br[t]);
          ai[t] = fma(a.x, xv.y, ai[t]);
          bi[t] = fma(a.y, xv.x, bi[t]);
        }
      }
    }
}

template <int PBX, int KC, int CG, typename T>
__global__ void __launch_bounds__(4 * PBX * KC * CG)
    k_m2l_unif_mac(const cplx_t<T>* __restrict__ X_l, cplx_t<T>* __restrict__ Y_l,
                   const cplx_t<T>* __restrict__ op,  // nk x 343 for this level
                   const int* __restrict__ halo, int64_t ncells, int C, int nk) {
  using G = MacGeom<PBX>;
  using C2 = cplx_t<T>;
  constexpr int NT = G::NPAR * KC * CG;
  constexpr int RC = G::RC;
  extern __shared__ __align__(16) unsigned char smraw[];
  C2* reg = reinterpret_cast<C2*>(smraw);  // RC x KC x CG
  C2* sop = reg + RC * KC * CG;            // KC x 343
  int* s_src = (int*)(sop + KC * 343);  // RC source cells, then TC target cells
  int* s_tgt = s_src + RC;
  const int tid = threadIdx.x;
  const int cc = tid % CG, kc = (tid / CG) % KC, p = tid / (CG * KC);
  const int px = p >> 2, py = (p >> 1) & 1, pz = p & 1;
  const int* hb = halo + (int64_t)blockIdx.x * G::STRIDE;
  int mine = 0;
  for (int r = tid; r < G::STRIDE; r += NT) {
    const int v = hb[r];
    s_src[r] = v;
    if (r >= RC) mine |= v >= 0;
  }
  if (!__syncthreads_or(mine)) return;
  const int k0 = blockIdx.y * KC;
  const int c0 = blockIdx.z * CG;
  // stage the source halo for frequencies k0..k0+KC-1 and columns
  // c0..c0+CG-1 with asynchronous copies (all in flight at once; empty or
  // out-of-domain cells are zero-filled)
  for (int i = tid; i < RC * KC * CG; i += NT) {
    const int r = i / (KC * CG), q = i % (KC * CG), kk = q / CG, c = q % CG;
    const int src = s_src[r];
    const bool ok = src >= 0 && k0 + kk < nk && c0 + c < C;
    const C2* g = ok ? &X_l[((int64_t)(k0 + kk) * ncells + src) * C + c0 + c] : X_l;
    cp_async_cplx(&reg[i], g, ok);
  }
  for (int i = tid; i < KC * 343; i += NT) {
    const int kk = i / 343, e = i % 343;
    const bool ok = k0 + kk < nk;
    cp_async_cplx(&sop[i], ok ? &op[(int64_t)(k0 + kk) * 343 + e] : op, ok);
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  T ar[8], br[8], ai[8], bi[8];  // re = ar + br, im = ai + bi
#pragma unroll
  for (int t = 0; t < 8; ++t) ar[t] = br[t] = ai[t] = bi[t] = T(0);
  const C2* myop = sop + kc * 343;
  // sx runs as a loop.  float64: the body for each sx is one of four
  // compile-time specialisations (whether the children with tx = 0 / 1 are
  // far in x at this sx), so no interaction test is left to run time (9 %
  // faster than the predicated body).  float32: one predicated body; the
  // four specialisations were 20 % slower there, the larger code costing
  // more than the predicated-off FMAs it saves.
#pragma unroll 1
  for (int sx = 0; sx < 6; ++sx) {
    const C2* rrow = reg + (((2 * px + sx) << 6) * KC + kc) * CG + cc;
    const C2* orow = myop + 49 * (sx + 1);  // lex of ox + 3 = sx + 1 - tx
    if constexpr (sizeof(T) == 8) {
      if (sx == 0 || sx == 5)
        mac_slab<true, true, KC * CG>(rrow, orow, py, pz, ar, br, ai, bi);
      else if (sx == 1)
        mac_slab<false, true, KC * CG>(rrow, orow, py, pz, ar, br, ai, bi);
      else if (sx == 4)
        mac_slab<true, false, KC * CG>(rrow, orow, py, pz, ar, br, ai, bi);
      else
        mac_slab<false, false, KC * CG>(rrow, orow, py, pz, ar, br, ai, bi);
    } else {
#pragma unroll
      for (int sy = 0; sy < 6; ++sy)
#pragma unroll
        for (int sz = 0; sz < 6; ++sz) {
          const int r = ((2 * py + sy) << 3) | (2 * pz + sz);
          const C2 xv = rrow[r * KC * CG];
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            const int tx = (t >> 2) & 1;
            const int oy = sy - 2 - ((t >> 1) & 1);
            const int oz = sz - 2 - (t & 1);
            const int ox = sx - 2 - tx;
            const bool far_yz = oy > 1 || oy < -1 || oz > 1 || oz < -1;
            if (far_yz || ox > 1 || ox < -1) {
              const C2 a = orow[-49 * tx + 7 * (oy + 3) + (oz + 3)];
              ar[t] = fma(a.x, xv.x, ar[t]);
              br[t] = fma(-a.y, xv.y, br[t]);
              ai[t] = fma(a.x, xv.y, ai[t]);
              bi[t] = fma(a.y, xv.x, bi[t]);
            }
          }
        }
    }
  }
  if (k0 + kc < nk && c0 + cc < C) {
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int q = ((2 * px + ((t >> 2) & 1)) << 4) | ((2 * py + ((t >> 1) & 1)) << 2) |
                    (2 * pz + (t & 1));
      const int cm = s_tgt[q];
      if (cm >= 0)
        Y_l[((int64_t)(k0 + kc) * ncells + cm) * C + c0 + cc] =
            make_cplx<T>(ar[t] + br[t], ai[t] + bi[t]);
    }
  }
}

template <int PBX, int KC, int CG, typename T>
static int launch_mac(const cplx_t<T>* X, cplx_t<T>* Y, const cplx_t<T>* op, int* halo,
                      const int* sstart, const int* tstart, int span, int lev, int C, int nk,
                      cudaStream_t st) {
  using G = MacGeom<PBX>;
  const int nby = 1 << (lev - 2), nbx = (1 << (lev - 1)) / PBX;
  const int nblk = nbx * nby * nby;
  k_halo_tables<PBX><<<nblk, 256, 0, st>>>(sstart, tstart, span, lev, halo);
  PB_LAUNCH("halo_tables");
  dim3 g((unsigned)nblk, (unsigned)((nk + KC - 1) / KC), (unsigned)((C + CG - 1) / CG));
  const size_t smem =
      sizeof(cplx_t<T>) * (G::RC * KC * CG + KC * 343) + sizeof(int) * G::STRIDE;
  PB_CUDA(cudaFuncSetAttribute(k_m2l_unif_mac<PBX, KC, CG, T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_m2l_unif_mac<PBX, KC, CG, T><<<g, G::NPAR * KC * CG, smem, st>>>(X, Y, op, halo,
                                                                     cells_at(lev), C, nk);
  PB_LAUNCH("m2l_unif_mac");
  return PBBFMM_OK;
}

template <int PBX, typename T>
static int launch_mac_cols(const cplx_t<T>* X, cplx_t<T>* Y, const cplx_t<T>* op, int* halo,
                           const int* sstart, const int* tstart, int span, int lev, int C, int nk,
                           cudaStream_t st) {
  if (C >= 8)
    return launch_mac<PBX, 1, 8, T>(X, Y, op, halo, sstart, tstart, span, lev, C, nk, st);
  if (C >= 4)
    return launch_mac<PBX, 2, 4, T>(X, Y, op, halo, sstart, tstart, span, lev, C, nk, st);
  if (C >= 2)
    return launch_mac<PBX, 4, 2, T>(X, Y, op, halo, sstart, tstart, span, lev, C, nk, st);
  return launch_mac<PBX, 8, 1, T>(X, Y, op, halo, sstart, tstart, span, lev, C, nk, st);
}

template <typename T>
struct FftLaunch {
  pbbfmm_tree* t;
  int C, CGf, CGi;
  size_t smem_f, smem_i;
  double invP;
  cudaStream_t st;
  int level = 2;
  bool inverse = false;
  double scale = 1.0;
  unsigned* amax = nullptr;  // forward: spectra maxima of the level (tensor-core MAC)
  template <int N>
  int run() {
    const int n3 = N * N * N, nk = (2 * N - 1) * (2 * N - 1) * N;
    Workspace& ws = t->ws;
    const int* lists = ws.lists.as<int>();
    const int64_t perS = (int64_t)C * n3, perX = (int64_t)nk * C;
    const int l = level;
    const T* twid = sizeof(T) == 8 ? (const T*)t->d_twid : (const T*)t->f_twid;
    if (!inverse) {
      PB_CUDA(cudaFuncSetAttribute(k_fft_fwd<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem_f));
      // CTAs loop over the cells: as many as fit on the GPU at once
      int per_sm = 1, dev = 0, nsm = 148;
      PB_CUDA(cudaGetDevice(&dev));
      PB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
      PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fft_fwd<N, T>, 128, smem_f));
      const int ncl = t->lists.nsrc[l];
      const int grid = std::max(1, std::min(ncl, std::max(1, per_sm) * nsm));
      k_fft_fwd<N, T><<<grid, 128, smem_f, st>>>(
          lists + t->lists.src_off[l], ncl, ws.S.as<T>() + level_offset(l, perS),
          ws.proxy.as<cplx_t<T>>() + level_offset(l, perX), cells_at(l), C, CGf, twid, amax);
      PB_LAUNCH("fft_fwd");
    } else {
      PB_CUDA(cudaFuncSetAttribute(k_fft_inv<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem_i));
      k_fft_inv<N, T><<<t->lists.ntgt[l], 128, smem_i, st>>>(
          lists + t->lists.tgt_off[l], ws.pf.as<cplx_t<T>>() + level_offset(l, perX),
          ws.F.as<T>() + level_offset(l, perS), cells_at(l), C, CGi, twid, (T)invP, (T)scale);
      PB_LAUNCH("fft_inv");
    }
    return PBBFMM_OK;
  }
};

template <typename T>
static int run_m2l_unif_t(pbbfmm_tree* t, int C, cudaStream_t st) {
  if (int rc = init_fft_twiddles()) return rc;
  using C2 = cplx_t<T>;
  const int L = t->p.tree_level, n = t->n, m = t->m, n3 = t->n3, nk = t->nk;
  Workspace& ws = t->ws;
  C2* X = ws.proxy.as<C2>();
  C2* Y = ws.pf.as<C2>();
  const int* sstart = ws.sstart.as<int>();
  const int* tstart = ws.tstart.as<int>();
  const int64_t perX = (int64_t)nk * C;
  const double invP = 1.0 / (double)(m * m * m);
  const int ts = (int)sizeof(T);
  // forward transforms of all nonempty source cells, levels 2..L
  const int fwd_col = n3 * ts + n3 * 2 * ts + n * m * n * 2 * ts;
  const int CGf = max(1, min(C, 60000 / fwd_col));
  const size_t smem_f = (size_t)ts * (2 * m + 2 * ((CGf * n3 + 3) & ~3)) +
                        (size_t)2 * ts * (CGf * n3 + CGf * n * m * n) + (size_t)4 * m * n * 8;
  const int inv_col = (nk + n * m * n + n3) * 2 * ts;
  const int CGi = max(1, min(C, 60000 / inv_col));
  const size_t smem_i = (size_t)ts * ((2 * m + 3) & ~3) +
                        (size_t)2 * ts * (CGi * nk + CGi * n * m * n + CGi * n3);
  FftLaunch<T> fl{t, C, CGf, CGi, smem_f, smem_i, invP, st};
  // spectra maxima per level for the tensor-core MAC's scaling (float path)
  const size_t amax_per = (size_t)m * n * 8;
  bool any_tc = false;
  for (int l = 2; l <= L; ++l) any_tc |= sizeof(T) == 4 && unif_tc_eligible(t, l, C);
  if (any_tc) {
    if (int rc_ = grow(ws.amax, (size_t)(L + 1) * amax_per * sizeof(unsigned))) return rc_;
    PB_CUDA(cudaMemsetAsync(ws.amax.p, 0, (size_t)(L + 1) * amax_per * sizeof(unsigned), st));
  }
  auto amax_at = [&](int l) -> unsigned* {
    return sizeof(T) == 4 && unif_tc_eligible(t, l, C) ? ws.amax.as<unsigned>() + l * amax_per
                                                       : nullptr;
  };
  for (int l = 2; l <= L; ++l) {
    if (t->lists.nsrc[l] == 0) continue;
    if (int rc_ = kt_begin(t, KS_FFT_FWD, st)) return rc_;
    fl.level = l;
    fl.inverse = false;
    fl.amax = amax_at(l);
    if (int rc_ = dispatch_order(n, fl)) return rc_;
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  int* halo = ws.halo.as<int>();
  const OpsView<T> ov = ops_view<T>(t);
  for (int l = 2; l <= L; ++l) {
    if (t->lists.ntgt[l] == 0) continue;
    const int lvl = t->homog ? 0 : l - 2;
    const C2* op = ov.op + (int64_t)lvl * nk * 343;
    const int span = (int)cells_at(L - l);
    int rc;
    if ((rc = kt_begin(t, KS_MAC, st))) return rc;
    const C2* Xl = X + level_offset(l, perX);
    C2* Yl = Y + level_offset(l, perX);
    // float32, 16 parents per side or more, columns in groups of 8: the
    // tensor cores (m2l_unif_tc.cu); otherwise 4x2x2 parent blocks on the
    // CUDA cores from level 3 up (level 2 has 2 parents per side)
    if (sizeof(T) == 4 && unif_tc_eligible(t, l, C))
      rc = run_m2l_unif_tc_level(t, C, l, lvl, reinterpret_cast<const float2*>(Xl),
                                 reinterpret_cast<float2*>(Yl), amax_at(l), st);
    else if (l >= 3)
      rc = launch_mac_cols<4, T>(Xl, Yl, op, halo, sstart, tstart, span, l, C, nk, st);
    else
      rc = launch_mac_cols<2, T>(Xl, Yl, op, halo, sstart, tstart, span, l, C, nk, st);
    if (rc) return rc;
    if ((rc = kt_end(t, st))) return rc;
    double len = t->p.L;
    for (int i = 0; i < l; ++i) len = 0.5 * len;
    const double scale = pow(1.0 / len, t->homogen_neg);
    if (int rc_ = kt_begin(t, KS_FFT_INV, st)) return rc_;
    fl.level = l;
    fl.inverse = true;
    fl.scale = scale;
    if (int rc_ = dispatch_order(n, fl)) return rc_;
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  return PBBFMM_OK;
}

int run_m2l_unif(pbbfmm_tree* t, int C, cudaStream_t st) {
  return t->cur_prec == PBBFMM_PREC_FP64 ? run_m2l_unif_t<double>(t, C, st)
                                         : run_m2l_unif_t<float>(t, C, st);
}

}  // namespace pbbfmm
