// Chebyshev far field in float64: the M2L pre-transform (proxy = VT (Kw o S)),
// the SVD-compressed M2L over interaction lists, and the post-transform
// (F = scale * Kw o (U Pf)).
//
// Reference: UpwardPass tail (include/compute.hpp:373-396), FarFieldInteractions
// (include/compute.hpp:402-508) and Moment2Local (include/compute.hpp:881-914).
// The reference runs one r_f x r_s x nCols dgemm per (target, source) pair;
// here the targets of one level that share their position in the parent
// (child type) share the same 189 offsets, so a tile of such targets walks
// the 189 operators E_i once and multiplies each by the gathered proxies of
// the tile -- one accumulated GEMM with K = 189 * r_s per tile.
#include <type_traits>

#include "fmm.cuh"

namespace pbbfmm {

constexpr int GBM = 64, GBN = 64, GBK = 16, GTM = 4, GTN = 4;
constexpr int kGemmThreads = (GBM / GTM) * (GBN / GTN);  // 256

// Out(:, j) = alpha * oscale o (A * (bscale o B(:, j))), A col-major M x K,
// column j = (cells[j / C], j % C); B columns are K-contiguous, Out columns
// M-contiguous, both indexed by (cell * C + col).
template <typename T>
__global__ void __launch_bounds__(kGemmThreads)
    k_colgemm(int M, int K, const T* __restrict__ A, const int* __restrict__ cells, int ncols,
              int C, const T* __restrict__ B, const T* __restrict__ bscale, T* __restrict__ Out,
              const T* __restrict__ oscale, T alpha) {
  __shared__ T As[GBK][GBM];
  __shared__ T Bs[GBK][GBN];
  __shared__ int64_t colbase[GBN];
  const int tid = threadIdx.x;
  const int tx = tid % (GBN / GTN), ty = tid / (GBN / GTN);
  const int m0 = blockIdx.y * GBM, j0 = blockIdx.x * GBN;
  if (tid < GBN) {
    int j = j0 + tid;
    colbase[tid] = j < ncols ? (int64_t)cells[j / C] * C + j % C : -1;
  }
  T acc[GTM][GTN];
#pragma unroll
  for (int i = 0; i < GTM; ++i)
#pragma unroll
    for (int j = 0; j < GTN; ++j) acc[i][j] = 0;
  __syncthreads();
  for (int k0 = 0; k0 < K; k0 += GBK) {
#pragma unroll
    for (int r = 0; r < (GBM * GBK) / kGemmThreads; ++r) {
      const int e = tid + r * kGemmThreads, mm = e % GBM, kk = e / GBM;
      const int gm = m0 + mm, gk = k0 + kk;
      As[kk][mm] = (gm < M && gk < K) ? A[gm + (int64_t)M * gk] : T(0);
    }
#pragma unroll
    for (int r = 0; r < (GBN * GBK) / kGemmThreads; ++r) {
      const int e = tid + r * kGemmThreads, kk = e % GBK, jj = e / GBK;
      const int gk = k0 + kk;
      const int64_t cb = colbase[jj];
      T v = 0;
      if (cb >= 0 && gk < K) {
        v = B[cb * K + gk];
        if (bscale) v = v * bscale[gk];
      }
      Bs[kk][jj] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK; ++kk) {
      T a[GTM], b[GTN];
#pragma unroll
      for (int i = 0; i < GTM; ++i) a[i] = As[kk][ty * GTM + i];
#pragma unroll
      for (int j = 0; j < GTN; ++j) b[j] = Bs[kk][tx * GTN + j];
#pragma unroll
      for (int i = 0; i < GTM; ++i)
#pragma unroll
        for (int j = 0; j < GTN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < GTN; ++j) {
    const int64_t cb = colbase[tx * GTN + j];
    if (cb < 0) continue;
#pragma unroll
    for (int i = 0; i < GTM; ++i) {
      const int gm = m0 + ty * GTM + i;
      if (gm >= M) continue;
      T v = alpha * acc[i][j];
      if (oscale) v = v * oscale[gm];
      Out[cb * M + gm] = v;
    }
  }
}

struct TypeTiles {
  int start[9];  // first tile of each type; start[8] = total tiles
  int first[8];  // first list position of each type
  int count[8];  // targets of each type
};

// M2L for one level.  Grid: (tiles over all types, M-tiles).  A tile holds
// up to GBN / C targets of one child type; columns are (target, col).
template <typename T>
__global__ void __launch_bounds__(kGemmThreads)
    k_m2l_cheb(int rf, int rs, const T* __restrict__ E, const int* __restrict__ typed,
               TypeTiles tt, int C, int lev, const int* __restrict__ sstart, int span,
               const int* __restrict__ offs, const T* __restrict__ proxy, T* __restrict__ pf) {
  __shared__ T As[GBK][GBM];
  __shared__ T Bs[GBK][GBN];
  __shared__ int s_tx[GBN], s_ty[GBN], s_tz[GBN];
  __shared__ int64_t s_src[GBN];  // proxy column base of the source, or -1
  __shared__ int s_tcell[GBN];
  const int tid = threadIdx.x;
  const int tx = tid % (GBN / GTN), ty = tid / (GBN / GTN);
  const int m0 = blockIdx.y * GBM;
  int type = 0;
  while (type < 7 && (int)blockIdx.x >= tt.start[type + 1]) ++type;
  const int per_tile = GBN / C;
  const int tfirst = (blockIdx.x - tt.start[type]) * per_tile;
  const int ntile = min(per_tile, tt.count[type] - tfirst);
  if (tid < GBN) {
    const int tt_i = tid / C;
    if (tid < per_tile * C && tt_i < ntile) {
      const int cell = typed[tt.first[type] + tfirst + tt_i];
      int x, y, z;
      morton_decode((uint32_t)cell, &x, &y, &z);
      s_tx[tid] = x;
      s_ty[tid] = y;
      s_tz[tid] = z;
      s_tcell[tid] = cell;
    } else {
      s_tcell[tid] = -1;
    }
  }
  const int nside = 1 << lev;
  T acc[GTM][GTN];
#pragma unroll
  for (int i = 0; i < GTM; ++i)
#pragma unroll
    for (int j = 0; j < GTN; ++j) acc[i][j] = 0;
  const int* my_offs = offs + type * 189 * 4;
  for (int o = 0; o < 189; ++o) {
    const int ox = my_offs[4 * o + 0], oy = my_offs[4 * o + 1], oz = my_offs[4 * o + 2];
    const int opi = my_offs[4 * o + 3];
    __syncthreads();
    int any = 0;
    if (tid < GBN) {
      int64_t src = -1;
      if (s_tcell[tid] >= 0) {
        const int bx = s_tx[tid] + ox, by = s_ty[tid] + oy, bz = s_tz[tid] + oz;
        if (bx >= 0 && by >= 0 && bz >= 0 && bx < nside && by < nside && bz < nside) {
          const uint32_t bm = morton_encode(bx, by, bz);
          if (sstart[(int64_t)(bm + 1) * span] > sstart[(int64_t)bm * span])
            src = ((int64_t)bm * C + tid % C) * rs;
        }
      }
      s_src[tid] = src;
      any = src >= 0;
    }
    if (!__syncthreads_or(any)) continue;
    const T* Eo = E + (int64_t)opi * rf * rs;
    for (int k0 = 0; k0 < rs; k0 += GBK) {
#pragma unroll
      for (int r = 0; r < (GBM * GBK) / kGemmThreads; ++r) {
        const int e = tid + r * kGemmThreads, mm = e % GBM, kk = e / GBM;
        const int gm = m0 + mm, gk = k0 + kk;
        As[kk][mm] = (gm < rf && gk < rs) ? Eo[gm + (int64_t)rf * gk] : T(0);
      }
#pragma unroll
      for (int r = 0; r < (GBN * GBK) / kGemmThreads; ++r) {
        const int e = tid + r * kGemmThreads, kk = e % GBK, jj = e / GBK;
        const int gk = k0 + kk;
        const int64_t sb = s_src[jj];
        Bs[kk][jj] = (sb >= 0 && gk < rs) ? proxy[sb + gk] : T(0);
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < GBK; ++kk) {
        T a[GTM], b[GTN];
#pragma unroll
        for (int i = 0; i < GTM; ++i) a[i] = As[kk][ty * GTM + i];
#pragma unroll
        for (int j = 0; j < GTN; ++j) b[j] = Bs[kk][tx * GTN + j];
#pragma unroll
        for (int i = 0; i < GTM; ++i)
#pragma unroll
          for (int j = 0; j < GTN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < GTN; ++j) {
    const int jj = tx * GTN + j;
    const int cell = s_tcell[jj];
    if (cell < 0) continue;
#pragma unroll
    for (int i = 0; i < GTM; ++i) {
      const int gm = m0 + ty * GTM + i;
      if (gm < rf) pf[((int64_t)cell * C + jj % C) * rf + gm] = acc[i][j];
    }
  }
}

template <typename T>
static int run_m2l_cheb_t(pbbfmm_tree* t, int C, cudaStream_t st) {
  const int L = t->p.tree_level, n3 = t->n3;
  const int rf = t->ops.rf, rs = t->ops.rs;
  Workspace& ws = t->ws;
  const int* lists = ws.lists.as<int>();
  const T* S = ws.S.as<T>();
  T* F = ws.F.as<T>();
  T* proxy = ws.proxy.as<T>();
  T* pf = ws.pf.as<T>();
  const OpsView<T> ov = ops_view<T>(t);
  const int* sstart = ws.sstart.as<int>();
  if (C > GBN) {
    set_error("nCols above 64 must be split by the caller");
    return PBBFMM_ERR_UNSUPPORTED;
  }
  for (int l = 2; l <= L; ++l) {
    const int lvl = t->homog ? 0 : l - 2;
    // proxy = VT_lvl * (Kw o S) for nonempty source cells
    const int ns = t->lists.nsrc[l];
    if (ns > 0) {
      dim3 g((unsigned)((ns * (int64_t)C + GBN - 1) / GBN), (unsigned)((rs + GBM - 1) / GBM));
      if (int rc_ = kt_begin(t, KS_M2L_PRE, st)) return rc_;
      k_colgemm<T><<<g, kGemmThreads, 0, st>>>(rs, n3, ov.VT + (int64_t)lvl * rs * n3,
                                            lists + t->lists.src_off[l], ns * C, C,
                                            S + level_offset(l, (int64_t)C * n3), ov.Kw,
                                            proxy + level_offset(l, (int64_t)C * rs), nullptr,
                                            T(1));
      PB_LAUNCH("m2l_pre");
      if (int rc_ = kt_end(t, st)) return rc_;
    }
  }
  for (int l = 2; l <= L; ++l) {
    const int lvl = t->homog ? 0 : l - 2;
    const int nt = t->lists.ntgt[l];
    if (nt == 0) continue;
    bool on_tc = false;  // float path: tcgen05 3xTF32 kernel when rf fits TMEM
    if constexpr (std::is_same<T, float>::value) {
      if (tc_eligible(t)) {
        if (int rc_ = run_m2l_cheb_tc_level(t, C, l, lvl, proxy + level_offset(l, (int64_t)C * rs),
                                            pf + level_offset(l, (int64_t)C * rf), st))
          return rc_;
        on_tc = true;
      }
    }
    TypeTiles tt;
    const int per_tile = GBN / C;
    int tiles = 0;
    for (int ty = 0; ty < 8; ++ty) {
      tt.start[ty] = tiles;
      tt.first[ty] = t->lists.ntyp[l][ty];
      tt.count[ty] = t->lists.ntyp[l][ty + 1] - t->lists.ntyp[l][ty];
      tiles += (tt.count[ty] + per_tile - 1) / per_tile;
    }
    tt.start[8] = tiles;
    if (tiles > 0 && !on_tc) {
      dim3 g((unsigned)tiles, (unsigned)((rf + GBM - 1) / GBM));
      if (int rc_ = kt_begin(t, KS_M2L, st)) return rc_;
      k_m2l_cheb<T><<<g, kGemmThreads, 0, st>>>(
          rf, rs, ov.E + (int64_t)lvl * 316 * rf * rs, lists + t->lists.typ_off[l], tt, C, l,
          sstart, (int)cells_at(L - l), t->d_offs, proxy + level_offset(l, (int64_t)C * rs),
          pf + level_offset(l, (int64_t)C * rf));
      PB_LAUNCH("m2l_cheb");
      if (int rc_ = kt_end(t, st)) return rc_;
    }
    // F = scale * Kw o (U_lvl * Pf)
    double len = t->p.L;
    for (int i = 0; i < l; ++i) len = 0.5 * len;
    const double scale = pow(1.0 / len, t->homogen_neg);
    dim3 g2((unsigned)((nt * (int64_t)C + GBN - 1) / GBN), (unsigned)((n3 + GBM - 1) / GBM));
    if (int rc_ = kt_begin(t, KS_M2L_POST, st)) return rc_;
    k_colgemm<T><<<g2, kGemmThreads, 0, st>>>(n3, rf, ov.U + (int64_t)lvl * n3 * rf,
                                           lists + t->lists.tgt_off[l], nt * C, C,
                                           pf + level_offset(l, (int64_t)C * rf), nullptr,
                                           F + level_offset(l, (int64_t)C * n3), ov.Kw,
                                           (T)scale);
    PB_LAUNCH("m2l_post");
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  return PBBFMM_OK;
}

int run_m2l_cheb(pbbfmm_tree* t, int C, cudaStream_t st) {
  return t->cur_prec == PBBFMM_PREC_FP64 ? run_m2l_cheb_t<double>(t, C, st)
                                         : run_m2l_cheb_t<float>(t, C, st);
}

}  // namespace pbbfmm
