// Upward pass: P2M at the leaves and M2M up to level 2.
//
// Reference: UpwardPass (include/compute.hpp:225-333) and Moment2Moment
// (include/compute.hpp:957-1034).  The reference recurses over a pointer
// tree with OpenMP tasks and lets children add into the parent concurrently
// (a data race); here every level is one launch, one CTA per nonempty cell,
// and each parent gathers its children in a fixed order (deterministic).
//
// Layout: moments of level l live at S + level_offset(l, C*n3), cell-major,
// S[(cell*C + col)*n3 + (l1*n + l2)*n + l3] as in the reference's sourceval.
#include "fmm.cuh"

namespace pbbfmm {

// Centre of cell m at level l, by the reference's +-quarter steps
// (src/H2_3D_Tree.cpp:927-961) -- identical FP64 operations.
__device__ __forceinline__ void cell_center(uint32_t m, int l, double box, double* c) {
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

constexpr int kP2MChunk = 32;  // points per pass (one per lane)
constexpr int kP2MCols = 8;    // columns per pass
// warps per CTA: static shared memory (basis + weights) stays under 48 KB
template <int N, typename T>
constexpr int p2m_warps() {
  return (3 * N * (kP2MChunk + 1) + kP2MChunk * kP2MCols) * (int)sizeof(T) * 8 <= 40 * 1024 ? 8 : 4;
}

// One warp per nonempty source leaf.  Lanes first evaluate the basis of up to
// 32 points (one point each) and stage their weights, then each lane owns
// tasks (column, l1, l2) and sums the N outputs l3 of a task over the staged
// points in point order.  Leaves with more than 32 points accumulate chunk by
// chunk in the output array (each output has a single owner lane).
// T = float (mixed path): the basis is evaluated from float64 leaf-relative
// coordinates, each chunk of up to 32 points is summed in float32 and added to
// the running value in float64.
template <int N, typename T, int kP2MWarps = p2m_warps<N, T>()>
__global__ void __launch_bounds__(32 * kP2MWarps)
    k_p2m(const int* __restrict__ leaves, int nleaves, const int* __restrict__ sstart,
          const double* __restrict__ spos, int Ns, const double* __restrict__ wsorted, int C,
          int cheb, const T* __restrict__ Tkz_g, double box, int L, T* __restrict__ S_L) {
  constexpr int n3 = N * N * N;
  constexpr bool kKahan = sizeof(T) == 4;
  __shared__ T sTkz[N * N];
  // basis values [dim][m][point], rows padded to 33 so that lanes reading
  // different m of one point hit different banks
  __shared__ T sB[kP2MWarps][3][N][kP2MChunk + 1];
  __shared__ T sW[kP2MWarps][kP2MChunk][kP2MCols];
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) sTkz[i] = Tkz_g[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int wid = blockIdx.x * kP2MWarps + wl;
  if (wid >= nleaves) return;
  const int leaf = leaves[wid];
  const int a = sstart[leaf], e = sstart[leaf + 1];
  double c[3];
  cell_center((uint32_t)leaf, L, box, c);
  double len = box;
  for (int i = 0; i < L; ++i) len = 0.5 * len;
  const double ihalfL = 2. / len;
  for (int c0 = 0; c0 < C; c0 += kP2MCols) {
    const int cg = min(kP2MCols, C - c0);
    T* Sout = S_L + ((int64_t)leaf * C + c0) * n3;
    for (int p0 = a; p0 < e; p0 += kP2MChunk) {
      const int cnt = min(kP2MChunk, e - p0);
      __syncwarp();
      if (lane < cnt) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const T q = (T)(ihalfL * (spos[(int64_t)d * Ns + p0 + lane] - c[d]));
#pragma unroll
          for (int m = 0; m < N; ++m) sB[wl][d][m][lane] = basis_one<T>(N, cheb, q, sTkz, m);
        }
        for (int cc = 0; cc < cg; ++cc)
          sW[wl][lane][cc] = (T)wsorted[(int64_t)(p0 + lane) * C + c0 + cc];
      }
      __syncwarp();
      // lane task (column, l1, l2): the N outputs l3 = 0..N-1 at once, the
      // weight x basis product over (l1, l2) formed once per point
      for (int task = lane; task < cg * N * N; task += 32) {
        const int cc = task / (N * N), l12 = task % (N * N), l1 = l12 / N, l2 = l12 % N;
        T part[N];
#pragma unroll
        for (int l3 = 0; l3 < N; ++l3) part[l3] = 0;
        for (int j = 0; j < cnt; ++j) {
          const T t = sW[wl][j][cc] * sB[wl][0][l1][j] * sB[wl][1][l2][j];
#pragma unroll
          for (int l3 = 0; l3 < N; ++l3) part[l3] = fma(t, sB[wl][2][l3][j], part[l3]);
        }
        T* o = Sout + cc * n3 + l12 * N;
#pragma unroll
        for (int l3 = 0; l3 < N; ++l3) {
          if (kKahan) {  // the chunk's float32 sum added to the float64 running value
            o[l3] = (T)(p0 == a ? (double)part[l3] : (double)o[l3] + (double)part[l3]);
          } else {
            o[l3] = p0 == a ? part[l3] : o[l3] + part[l3];
          }
        }
      }
    }
  }
}

template <typename T>
struct P2MLaunch {
  pbbfmm_tree* t;
  int C;
  cudaStream_t st;
  template <int N>
  int run() {
    const int L = t->p.tree_level;
    Workspace& ws = t->ws;
    const int nl = t->lists.nsrc[L];
    constexpr int W = p2m_warps<N, T>();
    const OpsView<T> ov = ops_view<T>(t);
    k_p2m<N, T><<<(nl + W - 1) / W, 32 * W, 0, st>>>(
        ws.lists.as<int>() + t->lists.src_off[L], nl, ws.sstart.as<int>(), ws.spos.as<double>(),
        (int)t->last_Ns, ws.wsorted.as<double>(), C, t->p.use_chebyshev, ov.Tkz, t->p.L, L,
        ws.S.as<T>() + level_offset(L, (int64_t)C * N * N * N));
    PB_LAUNCH("p2m");
    return PBBFMM_OK;
  }
};

// M2M, one warp per nonempty parent and column: the column's moments of all
// nonempty children are staged in the warp's shared slice (cp.async), then
// each child goes through the z, y and x passes and is added to the parent
// (children in order 0..7, as the reference accumulates them).
template <int N, typename T>
struct M2MCfg {
  static constexpr int n3 = N * N * N;
  static constexpr int per_warp = 8 * n3 + 2 * n3;  // children + two pass buffers (elements)
  static constexpr int warps = (per_warp * (int)sizeof(T) * 4 <= 96 * 1024) ? 4 : 1;
};

template <int N, typename T>
__global__ void __launch_bounds__(32 * M2MCfg<N, T>::warps)
    k_m2m(const int* __restrict__ parents, int npar, const int* __restrict__ sstart,
          int span_child, const T* __restrict__ Schild, T* __restrict__ Spar, int C,
          const T* __restrict__ Cw_g) {
  using G = M2MCfg<N, T>;
  constexpr int n2 = N * N, n3 = G::n3;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* smd = reinterpret_cast<T*>(smraw);
  __shared__ T sCw[2 * N * N];
  for (int i = threadIdx.x; i < 2 * n2; i += blockDim.x) sCw[i] = Cw_g[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int task = blockIdx.x * G::warps + wl;  // (parent, column)
  if (task >= npar * C) return;
  const int par = parents[task / C], col = task % C;
  T* sch = smd + wl * G::per_warp;  // 8 x n3
  T* b0 = sch + 8 * n3;
  T* b1 = b0 + n3;
  // which children hold sources: lanes 0..8 read the 9 leaf-range bounds at
  // once; then (float32, orders up to 6) every child's moments are loaded
  // with all loads in flight (an empty child's moments are never read)
  int bound = 0;
  if (lane <= 8) bound = sstart[(int64_t)(par * 8 + lane) * span_child];
  unsigned present = 0;
#pragma unroll
  for (int ch = 0; ch < 8; ++ch)
    present |= (__shfl_sync(0xffffffffu, bound, ch + 1) != __shfl_sync(0xffffffffu, bound, ch))
                   ? 1u << ch : 0u;
  constexpr int PER = (n3 + 31) / 32;
  if constexpr (N > 6 || sizeof(T) == 8) {
    for (int ch = 0; ch < 8; ++ch) {
      if (!((present >> ch) & 1)) continue;
      const T* src = Schild + ((int64_t)(par * 8 + ch) * C + col) * n3;
      for (int i = lane; i < n3; i += 32) sch[ch * n3 + i] = src[i];
    }
  } else {
    T v[8][PER];
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      const T* src = Schild + ((int64_t)(par * 8 + ch) * C + col) * n3;
#pragma unroll
      for (int r = 0; r < PER; ++r) {
        const int i = lane + 32 * r;
        v[ch][r] = ((present >> ch) & 1) && i < n3 ? src[i] : T(0);
      }
    }
#pragma unroll
    for (int ch = 0; ch < 8; ++ch)
#pragma unroll
      for (int r = 0; r < PER; ++r) {
        const int i = lane + 32 * r;
        if (i < n3) sch[ch * n3 + i] = v[ch][r];
      }
  }
  __syncwarp();
  // Orders up to 6 (float32) or 5 (float64): each pass as row tasks, a lane
  // loading the N inputs of one 1-D transform once and forming its N outputs
  // (the operator rows read by broadcast).  Higher orders (registers):
  // element tasks, one output per lane and pass.
  if constexpr (N <= (sizeof(T) == 4 ? 6 : 5)) {
  constexpr int TPL = (n2 + 31) / 32;  // x-pass tasks per lane
  T acc[TPL][N];
#pragma unroll
  for (int t = 0; t < TPL; ++t)
#pragma unroll
    for (int l = 0; l < N; ++l) acc[t][l] = 0;
  for (int ch = 0; ch < 8; ++ch) {
    if (!((present >> ch) & 1)) continue;
    const T* wx = sCw + (((ch >> 2) & 1) ? n2 : 0);
    const T* wy = sCw + (((ch >> 1) & 1) ? n2 : 0);
    const T* wz = sCw + ((ch & 1) ? n2 : 0);
    const T* sc = sch + ch * n3;
    // z: Sz[r n + l3] = sum_k S[r n + k] wz[l3 n + k]   (row r over n^2)
    for (int r = lane; r < n2; r += 32) {
      T x[N];
#pragma unroll
      for (int k = 0; k < N; ++k) x[k] = sc[r * N + k];
#pragma unroll
      for (int l3 = 0; l3 < N; ++l3) {
        T v = 0;
#pragma unroll
        for (int k = 0; k < N; ++k) v = fma(x[k], wz[l3 * N + k], v);
        b0[r * N + l3] = v;
      }
    }
    __syncwarp();
    // y: Sy[l1 n2 + l2 n + l3] = sum_k Sz[l1 n2 + k n + l3] wy[l2 n + k]   (task (l1, l3))
    for (int q = lane; q < n2; q += 32) {
      const int l1 = q / N, l3 = q % N;
      T x[N];
#pragma unroll
      for (int k = 0; k < N; ++k) x[k] = b0[l1 * n2 + k * N + l3];
#pragma unroll
      for (int l2 = 0; l2 < N; ++l2) {
        T v = 0;
#pragma unroll
        for (int k = 0; k < N; ++k) v = fma(x[k], wy[l2 * N + k], v);
        b1[l1 * n2 + l2 * N + l3] = v;
      }
    }
    __syncwarp();
    // x: SS[l1 n2 + rem] += sum_k Sy[k n2 + rem] wx[l1 n + k]   (task rem)
#pragma unroll
    for (int t = 0; t < TPL; ++t) {
      const int rem = lane + 32 * t;
      if (rem < n2) {
        T x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = b1[k * n2 + rem];
#pragma unroll
        for (int l1 = 0; l1 < N; ++l1) {
          T v = acc[t][l1];
#pragma unroll
          for (int k = 0; k < N; ++k) v = fma(x[k], wx[l1 * N + k], v);
          acc[t][l1] = v;
        }
      }
    }
    __syncwarp();
  }
  T* dst = Spar + ((int64_t)par * C + col) * n3;
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    const int rem = lane + 32 * t;
    if (rem < n2)
#pragma unroll
      for (int l1 = 0; l1 < N; ++l1) dst[l1 * n2 + rem] = acc[t][l1];
  }
  } else {
  constexpr int PER = (n3 + 31) / 32;
  T acc[PER];
#pragma unroll
  for (int r = 0; r < PER; ++r) acc[r] = 0;
  for (int ch = 0; ch < 8; ++ch) {
    if (!((present >> ch) & 1)) continue;
    const T* wx = sCw + (((ch >> 2) & 1) ? n2 : 0);
    const T* wy = sCw + (((ch >> 1) & 1) ? n2 : 0);
    const T* wz = sCw + ((ch & 1) ? n2 : 0);
    const T* sc = sch + ch * n3;
    // z: Sz[l1*n + l3] = sum_k S[l1*n + k] wz[l3*n + k]   (l1 over n^2)
    for (int i = lane; i < n3; i += 32) {
      const int l1 = i / N, l3 = i % N;
      T v = 0;
#pragma unroll
      for (int k = 0; k < N; ++k) v += sc[l1 * N + k] * wz[l3 * N + k];
      b0[i] = v;
    }
    __syncwarp();
    // y: Sy[l1 n2 + l2 n + l3] = sum_k Sz[l1 n2 + k n + l3] wy[l2 n + k]
    for (int i = lane; i < n3; i += 32) {
      const int l1 = i / n2, l2 = (i / N) % N, l3 = i % N;
      T v = 0;
#pragma unroll
      for (int k = 0; k < N; ++k) v += b0[l1 * n2 + k * N + l3] * wy[l2 * N + k];
      b1[i] = v;
    }
    __syncwarp();
    // x: SS[l1 n2 + l2 n + l3] = sum_k Sy[k n2 + l2 n + l3] wx[l1 n + k]
#pragma unroll
    for (int r = 0; r < PER; ++r) {
      const int i = lane + 32 * r;
      if (i < n3) {
        const int l1 = i / n2, rem = i % n2;
        T v = 0;
#pragma unroll
        for (int k = 0; k < N; ++k) v += b1[k * n2 + rem] * wx[l1 * N + k];
        acc[r] += v;
      }
    }
    __syncwarp();
  }
  T* dst = Spar + ((int64_t)par * C + col) * n3;
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int i = lane + 32 * r;
    if (i < n3) dst[i] = acc[r];
  }
  }
}

template <typename T>
struct M2MLaunch {
  pbbfmm_tree* t;
  int C, l;
  cudaStream_t st;
  template <int N>
  int run() {
    using G = M2MCfg<N, T>;
    const int L = t->p.tree_level;
    Workspace& ws = t->ws;
    const int64_t per = (int64_t)C * G::n3;
    const int np = t->lists.nsrc[l];
    const int64_t tasks = (int64_t)np * C;
    const size_t smem = sizeof(T) * G::per_warp * G::warps;
    PB_CUDA(cudaFuncSetAttribute(k_m2m<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_m2m<N, T><<<(unsigned)((tasks + G::warps - 1) / G::warps), 32 * G::warps, smem, st>>>(
        ws.lists.as<int>() + t->lists.src_off[l], np, ws.sstart.as<int>(), (int)cells_at(L - l - 1),
        ws.S.as<T>() + level_offset(l + 1, per), ws.S.as<T>() + level_offset(l, per), C,
        ops_view<T>(t).Cw);
    PB_LAUNCH("m2m");
    return PBBFMM_OK;
  }
};

template <typename T>
static int run_upward_t(pbbfmm_tree* t, int C, cudaStream_t st) {
  const int L = t->p.tree_level, n = t->n;
  if (t->lists.nsrc[L] > 0) {
    if (int rc_ = kt_begin(t, KS_P2M, st)) return rc_;
    P2MLaunch<T> pl{t, C, st};
    if (int rc_ = dispatch_order(n, pl)) return rc_;
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  for (int l = L - 1; l >= 2; --l) {
    if (t->lists.nsrc[l] == 0) continue;
    if (int rc_ = kt_begin(t, KS_M2M, st)) return rc_;
    M2MLaunch<T> ml{t, C, l, st};
    if (int rc_ = dispatch_order(n, ml)) return rc_;
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  return PBBFMM_OK;
}

int run_upward(pbbfmm_tree* t, int C, cudaStream_t st) {
  return t->cur_prec == PBBFMM_PREC_FP64 ? run_upward_t<double>(t, C, st)
                                         : run_upward_t<float>(t, C, st);
}

}  // namespace pbbfmm
