// Downward pass (L2L) and the leaf phase (L2P + P2P + scatter to output).
//
// Reference: DownwardPass / Local2Local (include/compute.hpp:552-587,
// 799-878) and NearFieldInteractions (include/compute.hpp:591-749) with
// EvaluateField / EvaluateField_self (:761-785).  The reference's P2P uses
// the kernel's symmetry to update both leaves of a pair under an OpenMP
// critical section; here each target point gathers from its 27 neighbour
// leaves (no atomics, no symmetry assumption, sources may differ from
// targets), and the far-field interpolation, the near-field sum and the
// scatter to the caller's output are one kernel.
#include <cub/cub.cuh>

#include <type_traits>

#include "fmm.cuh"

namespace pbbfmm {

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

// L2L, one warp per nonempty target parent and column: the parent's local
// coefficients are staged once and pushed through the x, y and z passes for
// each nonempty child, which is updated in place (F_child += ...).
template <int N>
struct L2LCfg {
  static constexpr int n3 = N * N * N;
  static constexpr int per_warp = 3 * n3;  // parent + two pass buffers (elements)
  static constexpr int warps = 8;
};

template <int N, typename T>
__global__ void __launch_bounds__(32 * L2LCfg<N>::warps)
    k_l2l(const int* __restrict__ parents, int npar, const int* __restrict__ tstart,
          int span_child, const T* __restrict__ Fpar, T* __restrict__ Fch, int C,
          const T* __restrict__ Cw_g) {
  using G = L2LCfg<N>;
  constexpr int n2 = N * N, n3 = G::n3;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* smd = reinterpret_cast<T*>(smraw);
  __shared__ T sCw[2 * N * N];
  for (int i = threadIdx.x; i < 2 * n2; i += blockDim.x) sCw[i] = Cw_g[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int task = blockIdx.x * G::warps + wl;
  if (task >= npar * C) return;
  const int par = parents[task / C], col = task % C;
  T* sp = smd + wl * G::per_warp;
  T* b0 = sp + n3;
  T* b1 = b0 + n3;
  const T* src = Fpar + ((int64_t)par * C + col) * n3;
  for (int i = lane; i < n3; i += 32) sp[i] = src[i];
  __syncwarp();
  for (int ch = 0; ch < 8; ++ch) {
    const int cell = par * 8 + ch;
    const int64_t a = (int64_t)cell * span_child, b = (int64_t)(cell + 1) * span_child;
    if (tstart[b] == tstart[a]) continue;  // child without targets
    const T* wx = sCw + (((ch >> 2) & 1) ? n2 : 0);
    const T* wy = sCw + (((ch >> 1) & 1) ? n2 : 0);
    const T* wz = sCw + ((ch & 1) ? n2 : 0);
    // x: Fx[l1 n2 + l2 n + l3] = sum_k F[k n2 + l2 n + l3] wx[l1 + k n]
    for (int i = lane; i < n3; i += 32) {
      const int l1 = i / n2, rem = i % n2;
      T v = 0;
#pragma unroll
      for (int k = 0; k < N; ++k) v += sp[k * n2 + rem] * wx[l1 + k * N];
      b0[i] = v;
    }
    __syncwarp();
    // y: Fy[l1 n2 + l2 n + l3] = sum_k Fx[l1 n2 + k n + l3] wy[l2 + k n]
    for (int i = lane; i < n3; i += 32) {
      const int l1 = i / n2, l2 = (i / N) % N, l3 = i % N;
      T v = 0;
#pragma unroll
      for (int k = 0; k < N; ++k) v += b0[l1 * n2 + k * N + l3] * wy[l2 + k * N];
      b1[i] = v;
    }
    __syncwarp();
    // z: Fchild[l1 n + l3] += sum_k Fy[l1 n + k] wz[l3 + k n]   (l1 over n^2)
    T* dst = Fch + ((int64_t)cell * C + col) * n3;
    for (int i = lane; i < n3; i += 32) {
      const int l1 = i / N, l3 = i % N;
      T v = 0;
#pragma unroll
      for (int k = 0; k < N; ++k) v += b1[l1 * N + k] * wz[l3 + k * N];
      dst[i] += v;
    }
    __syncwarp();
  }
}

template <typename T>
struct L2LLaunch {
  pbbfmm_tree* t;
  int C, l;  // child level
  cudaStream_t st;
  template <int N>
  int run() {
    using G = L2LCfg<N>;
    const int L = t->p.tree_level;
    Workspace& ws = t->ws;
    const int64_t per = (int64_t)C * G::n3;
    const int np = t->lists.ntgt[l - 1];
    const int64_t tasks = (int64_t)np * C;
    const size_t smem = sizeof(T) * G::per_warp * G::warps;
    PB_CUDA(cudaFuncSetAttribute(k_l2l<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_l2l<N, T><<<(unsigned)((tasks + G::warps - 1) / G::warps), 32 * G::warps, smem, st>>>(
        ws.lists.as<int>() + t->lists.tgt_off[l - 1], np, ws.tstart.as<int>(),
        (int)cells_at(L - l), ws.F.as<T>() + level_offset(l - 1, per),
        ws.F.as<T>() + level_offset(l, per), C, ops_view<T>(t).Cw);
    PB_LAUNCH("l2l");
    return PBBFMM_OK;
  }
};

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

// T = float (mixed path): kernel values, interpolation and per-tile partial
// sums in float32, each lane's running sums compensated (Kahan), the output
// update in float64.  T = double: everything in float64.
template <class KF, typename T, int KC, bool DENSE>
__global__ void __launch_bounds__(32 * kLeafWarps, DENSE ? 4 : 6)
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
  __shared__ V4 s_sh[kLeafWarps][DENSE ? 32 : 1];              // staged sources: position (hi)
  __shared__ V4 s_sl[kLeafWarps][DENSE && kMixed ? 32 : 1];    // position (lo), mixed path
  __shared__ T s_w[kLeafWarps][DENSE ? 32 : 1][KC];            // staged weights
  // basis values of each lane's target, [warp][dim][m < n][lane] (dynamic, sized by n)
  extern __shared__ __align__(16) unsigned char leaf_dyn[];
  T* s_bw = reinterpret_cast<T*>(leaf_dyn) + (threadIdx.x >> 5) * 3 * n * 32;
  __shared__ T s_bs[kLeafWarps][DENSE ? 1 : 3 * kMaxOrder];  // sparse path: the warp's target
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTkz[i] = Tkz_g[i];
  if (threadIdx.x < 4) kp[threadIdx.x] = kparam_g[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int wid = blockIdx.x * kLeafWarps + wl;
  // leaves are partitioned: the dense ones first, the sparse ones after
  const int nd = *part_count;
  int leaf, ta, te, tc0 = 0;
  if constexpr (DENSE) {
    // warp = one 32-target chunk of a dense leaf; chunk_prefix[i] is the first
    // chunk of dense leaf i (exclusive scan), chunk_prefix[nd] the total
    if (wid >= chunk_prefix[nd]) return;
    int lo = 0, hi = nd - 1;
    while (lo < hi) {  // last i with chunk_prefix[i] <= wid
      const int mid = (lo + hi + 1) >> 1;
      if (chunk_prefix[mid] <= wid) lo = mid;
      else hi = mid - 1;
    }
    leaf = leaves[lo];
    ta = tstart[leaf];
    te = tstart[leaf + 1];
    tc0 = ta + 32 * (wid - chunk_prefix[lo]);
  } else {
    if (wid >= nleaves - nd) return;
    leaf = leaves[nd + wid];
    ta = tstart[leaf];
    te = tstart[leaf + 1];
  }
  if ((te - ta >= kLaneLeafMin) != DENSE) return;  // the other instantiation's leaf
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
  }
  __syncwarp();
  if (lane == 0) {
    int acc = 0;
    for (int q = 0; q < 27; ++q) {
      s_pre[wl][q] = acc;
      acc += s_nb[wl][q][1] - s_nb[wl][q][0];
    }
    s_pre[wl][27] = acc;
  }
  __syncwarp();
  const int nsrc_total = s_pre[wl][27];
  if constexpr (!DENSE) {
    // Sparse leaf: one target at a time, lanes over its sources and over the
    // n^3 local coefficients, warp-reduced in float64.
    for (int c0 = 0; c0 < C; c0 += KC) {
      const int cg = min(KC, C - c0);
      for (int i = ta; i < te; ++i) {
        const double x = tpos[i], y = tpos[(int64_t)Nf + i], z = tpos[2 * (int64_t)Nf + i];
        LeafAcc<T> acc[KC];
        __syncwarp();
        if (lane < 3 * n) {
          const int d = lane / n, mm = lane % n;
          const T u = (T)(ihalfL * ((d == 0 ? x : d == 1 ? y : z) - c[d]));
          s_bs[wl][d * n + mm] = basis_one<T>(n, cheb, u, sTkz, mm);
        }
        __syncwarp();
        const T* Fl = F_L + ((int64_t)leaf * C + c0) * n3;
        for (int l = lane; l < n3; l += 32) {
          const int l1 = l / (n * n), l2 = (l / n) % n, l3 = l % n;
          const T v = s_bs[wl][l1] * s_bs[wl][n + l2] * s_bs[wl][2 * n + l3];
#pragma unroll
          for (int cc = 0; cc < KC; ++cc)
            if (cc < cg) acc[cc].add(Fl[cc * n3 + l] * v);
        }
        int q = 0;
        for (int v = lane; v < nsrc_total; v += 32) {
          while (v >= s_pre[wl][q + 1]) ++q;
          const int j = s_nb[wl][q][0] + (v - s_pre[wl][q]);
          const T dx = (T)(spos[j] - x), dy = (T)(spos[(int64_t)Ns + j] - y),
                  dz = (T)(spos[2 * (int64_t)Ns + j] - z);
          T kv = KF::template eval<T>(dx, dy, dz, kp);
          if (isinf(kv)) kv = 0;  // coincident points (include/compute.hpp:767)
          const double* wj = wsorted + (int64_t)j * C + c0;
#pragma unroll
          for (int cc = 0; cc < KC; ++cc)
            if (cc < cg) acc[cc].add(kv * (T)wj[cc]);
        }
        double tot[KC];
#pragma unroll
        for (int cc = 0; cc < KC; ++cc) {
          double v = acc[cc].value();
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          tot[cc] = v;
        }
        if (lane == 0) {
          const int64_t oi = tperm[i];
#pragma unroll
          for (int cc = 0; cc < KC; ++cc)
            if (cc < cg) out[(int64_t)(c0 + cc) * Nf + oi] += tot[cc];
        }
      }
    }
  } else {
  // Dense leaf: one target per lane, sources through shared-memory tiles.
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
      // far field: phi += sum_l F[l] Sx[l1] Sy[l2] Sz[l3]
      if (active) {
        T* b = s_bw + lane;  // b[(d n + m) 32]: conflict-free, no local memory
        for (int m = 0; m < n; ++m) {
          b[m * 32] = basis_one<T>(n, cheb, (T)(ihalfL * (x - c[0])), sTkz, m);
          b[(n + m) * 32] = basis_one<T>(n, cheb, (T)(ihalfL * (y - c[1])), sTkz, m);
          b[(2 * n + m) * 32] = basis_one<T>(n, cheb, (T)(ihalfL * (z - c[2])), sTkz, m);
        }
        const T* Fl = F_L + ((int64_t)leaf * C + c0) * n3;
        int l = 0;
        for (int l1 = 0; l1 < n; ++l1)
          for (int l2 = 0; l2 < n; ++l2) {
            const T b12 = b[l1 * 32] * b[(n + l2) * 32];
            for (int l3 = 0; l3 < n; ++l3, ++l) {
              const T v = b12 * b[(2 * n + l3) * 32];
#pragma unroll
              for (int cc = 0; cc < KC; ++cc)
                if (cc < cg) acc[cc].add(Fl[cc * n3 + l] * v);
            }
          }
      }
      // near field: the 27 neighbours' source ranges, concatenated, in tiles of 32
      int q = 0;
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
      if (active) {
        const int64_t oi = tperm[i];
#pragma unroll
        for (int cc = 0; cc < KC; ++cc)
          if (cc < cg) out[(int64_t)(c0 + cc) * Nf + oi] += (double)acc[cc].value();
      }
    }
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
  }
  __syncwarp();
  if (lane == 0) {
    int acc = 0;
    for (int q = 0; q < 27; ++q) {
      s_pre[wl][q] = acc;
      acc += s_nb[wl][q][1] - s_nb[wl][q][0];
    }
    s_pre[wl][27] = acc;
  }
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

template <typename T>
struct LeafGradLaunch {
  pbbfmm_tree* t;
  int64_t Nf, Ns;
  int C;
  double* out;
  cudaStream_t st;
  const double* kparam;
  template <class KF>
  int run() {
    const int L = t->p.tree_level;
    const int nl = t->lists.ntgt[L];
    if (nl == 0) return PBBFMM_OK;
    Workspace& ws = t->ws;
    const int64_t perS = (int64_t)C * t->n3;
    if (int rc_ = kt_begin(t, KS_LEAF, st)) return rc_;
    k_leaf_grad<KF, T><<<(nl + kLeafWarps - 1) / kLeafWarps, 32 * kLeafWarps, 0, st>>>(
        ws.lists.as<int>() + t->lists.tgt_off[L], nl, ws.tstart.as<int>(), ws.sstart.as<int>(),
        ws.tperm.as<int>(), ws.tpos.as<double>(), ws.spos.as<double>(), ws.wsorted.as<double>(),
        (int)Nf, (int)Ns, C, ws.F.as<T>() + level_offset(L, perS), t->n, t->p.use_chebyshev,
        ops_view<T>(t).Tkz, t->p.L, L, kparam, t->gl.values ? out : nullptr, t->gl.contract,
        t->gl.grad_out);
    PB_LAUNCH("leaf_grad");
    return kt_end(t, st);
  }
};

// counts[i] = 32-target chunks of dense leaf i (i < *nsel), 0 otherwise (i <= nl)
__global__ void k_chunk_counts(const int* __restrict__ part, const int* __restrict__ nsel, int nl,
                               const int* __restrict__ tstart, int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nl) return;
  int c = 0;
  if (i < *nsel) {
    const int leaf = part[i];
    c = (tstart[leaf + 1] - tstart[leaf] + 31) / 32;
  }
  counts[i] = c;
}

struct DenseLeaf {
  const int* tstart;
  __host__ __device__ bool operator()(int leaf) const {
    return tstart[leaf + 1] - tstart[leaf] >= kLaneLeafMin;
  }
};

template <typename T>
struct LeafLaunch {
  pbbfmm_tree* t;
  int64_t Nf, Ns;
  int C;
  double* out;
  cudaStream_t st;
  const double* kparam;
  template <class KF>
  int run() {
    const int L = t->p.tree_level;
    const int nl = t->lists.ntgt[L];
    if (nl == 0) return PBBFMM_OK;
    Workspace& ws = t->ws;
    const int64_t perS = (int64_t)C * t->n3;
    if (int rc_ = kt_begin(t, KS_LEAF, st)) return rc_;
    const size_t dyn = sizeof(T) * kLeafWarps * 3 * t->n * 32;
    // partition the leaves (dense first) so that each launch's active warps
    // are packed into the first CTAs of its grid
    const int* leaves = ws.lists.as<int>() + t->lists.tgt_off[L];
    if (int rc_ = grow(ws.leafpart, sizeof(int) * 3 * ((size_t)nl + 1))) return rc_;
    int* part = ws.leafpart.as<int>();
    int* nsel = part + nl;
    size_t tb = 0;
    DenseLeaf pred{ws.tstart.as<int>()};
    PB_CUDA(cub::DevicePartition::If(nullptr, tb, leaves, part, nsel, nl, pred, st));
    if (int rc_ = grow(ws.cub_temp, tb)) return rc_;
    tb = ws.cub_temp.cap;
    PB_CUDA(cub::DevicePartition::If(ws.cub_temp.p, tb, leaves, part, nsel, nl, pred, st));
    count_launches(2);
    // 32-target chunks of the dense leaves, exclusive scan -> one warp each
    int* chunks = part + nl + 1;  // nl + 1 counts, then nl + 1 prefixes
    int* prefix = chunks + nl + 1;
    k_chunk_counts<<<(unsigned)((nl + 1 + 255) / 256), 256, 0, st>>>(part, nsel, nl,
                                                                   ws.tstart.as<int>(), chunks);
    PB_LAUNCH("leaf_chunks");
    size_t tb2 = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, chunks, prefix, nl + 1, st));
    if (int rc_ = grow(ws.cub_temp, tb2)) return rc_;
    tb2 = ws.cub_temp.cap;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(ws.cub_temp.p, tb2, chunks, prefix, nl + 1, st));
    count_launches(2);
    // upper bound of the chunk count: Nf / 32 + one partial chunk per dense
    // leaf (at most Nf / kLaneLeafMin of them)
    const int64_t max_chunks = Nf / 32 + (nl < Nf / kLaneLeafMin ? nl : Nf / kLaneLeafMin) + 1;
    // one column: registers for one; otherwise columns in passes of kLeafCols.
    for (int dense = 1; dense >= 0; --dense) {
      auto kern = C == 1 ? (dense ? k_leaf<KF, T, 1, true> : k_leaf<KF, T, 1, false>)
                         : (dense ? k_leaf<KF, T, kLeafCols, true> : k_leaf<KF, T, kLeafCols, false>);
      const int64_t warps = dense ? max_chunks : nl;
      kern<<<(unsigned)((warps + kLeafWarps - 1) / kLeafWarps), 32 * kLeafWarps, dense ? dyn : 0,
             st>>>(part, nl, nsel, prefix, ws.tstart.as<int>(), ws.sstart.as<int>(),
          ws.tperm.as<int>(), ws.tpos.as<double>(), ws.spos.as<double>(), ws.wsorted.as<double>(),
          (int)Nf, (int)Ns, C, ws.F.as<T>() + level_offset(L, perS), t->n, t->p.use_chebyshev,
          ops_view<T>(t).Tkz, t->p.L, L, kparam, out);
      PB_LAUNCH("leaf");
    }
    if (int rc_ = kt_end(t, st)) return rc_;
    return PBBFMM_OK;
  }
};

template <typename T>
static int run_downward_t(pbbfmm_tree* t, int C, cudaStream_t st) {
  const int L = t->p.tree_level;
  // level-2 locals have no parent contribution (levels 0 and 1 carry none)
  for (int l = 3; l <= L; ++l) {
    if (t->lists.ntgt[l - 1] == 0) continue;
    if (int rc_ = kt_begin(t, KS_L2L, st)) return rc_;
    L2LLaunch<T> ll{t, C, l, st};
    if (int rc_ = dispatch_order(t->n, ll)) return rc_;
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  return PBBFMM_OK;
}

int run_downward(pbbfmm_tree* t, int C, cudaStream_t st) {
  return t->cur_prec == PBBFMM_PREC_FP64 ? run_downward_t<double>(t, C, st)
                                         : run_downward_t<float>(t, C, st);
}

int run_leaves(pbbfmm_tree* t, int64_t Nf, int64_t Ns, int C, double* d_out, cudaStream_t st) {
  if (t->gl.on) {
    if (t->cur_prec == PBBFMM_PREC_FP64) {
      LeafGradLaunch<double> ll{t, Nf, Ns, C, d_out, st, t->d_kparam};
      return dispatch_kernel(t->p.kernel, ll);
    }
    LeafGradLaunch<float> ll{t, Nf, Ns, C, d_out, st, t->d_kparam};
    return dispatch_kernel(t->p.kernel, ll);
  }
  if (t->cur_prec == PBBFMM_PREC_FP64) {
    LeafLaunch<double> ll{t, Nf, Ns, C, d_out, st, t->d_kparam};
    return dispatch_kernel(t->p.kernel, ll);
  }
  LeafLaunch<float> ll{t, Nf, Ns, C, d_out, st, t->d_kparam};
  return dispatch_kernel(t->p.kernel, ll);
}

}  // namespace pbbfmm
