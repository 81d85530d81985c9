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

// M2L for one level on the CUDA cores (float64 path; also the float32 path
// when r_f exceeds the tensor-core tile).  A CTA owns 128 (target, column)
// rows of one child type and 128 rows of r_f, and walks the offsets where
// some row of the tile has a source.  Per offset only the rows with a source
// take part: they are compacted (in tile-row order) into chunks of 16, so
// that a tile whose targets have few sources at an offset (sparse cells at
// the deepest levels of a clustered tree) multiplies 16-row chunks instead
// of all 128 rows.  For each offset and r_s in steps of 16, the gathered
// proxies of the compacted rows (A, up to 128 x 16) and the operator (B,
// 128 x 16) are staged in double-buffered shared memory (cp.async, element-
// wise so the A tile is stored transposed).  Each thread accumulates a
// c x 8 block of the offset's product in registers (compacted rows ty + 16 i,
// i < c chunks; columns tx + 16 j), then adds it into the tile's running sum
// in shared memory under the rows' target positions.  Every row of the tile
// appears at most once per offset, the offsets are taken in a fixed order,
// and a block barrier separates the adds of consecutive offsets, so the
// result is deterministic.
constexpr int CG_M = 128, CG_N = 128, CG_K = 16, CG_THREADS = 256;
constexpr int CG_NS = 2;           // stages: loads run one K step ahead
constexpr int CG_SLOTS = 3;        // compacted row lists in flight (see lookup)
constexpr int CG_APAD = CG_M + 1;  // A rows padded: conflict-free transposed stores

// stages (A and B) and the running sum [CG_M][CG_N]; the float64 instance
// takes 192 KB (two 16-deep stages next to the 128 KB running sum)
template <typename T>
__host__ __device__ constexpr size_t cg_smem_bytes() {
  return sizeof(T) * (CG_NS * CG_K * (CG_APAD + CG_N) + (size_t)CG_M * CG_N);
}

// One K step of CG_K for the first NC chunks of compacted rows: thread
// (tx, ty) owns compacted rows ty + 16 i and columns tx + 16 j.
template <int NC, typename T>
__device__ __forceinline__ void cg_step(const T* __restrict__ as, const T* __restrict__ bs, int tx,
                                        int ty, T (&acc)[8][8]) {
#pragma unroll
  for (int kk = 0; kk < CG_K; ++kk) {
    T a[NC], b[8];
#pragma unroll
    for (int i = 0; i < NC; ++i) a[i] = as[kk * CG_APAD + ty + 16 * i];
#pragma unroll
    for (int j = 0; j < 8; ++j) b[j] = bs[kk * CG_N + tx + 16 * j];
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
}

template <typename T>
__global__ void __launch_bounds__(CG_THREADS, 1)
    k_m2l_cheb(int rf, int rs, const T* __restrict__ E, const int* __restrict__ typed,
               TypeTiles tt, int C, int lev, const int* __restrict__ sstart, int span,
               const int* __restrict__ offs, const T* __restrict__ proxy, T* __restrict__ pf) {
  extern __shared__ __align__(16) unsigned char cg_raw[];
  T* As = reinterpret_cast<T*>(cg_raw);         // [CG_NS][CG_K][CG_APAD]
  T* Bs = As + CG_NS * CG_K * CG_APAD;          // [CG_NS][CG_K][CG_N]
  T* Sum = Bs + CG_NS * CG_K * CG_N;            // [CG_M][CG_N] running sum by tile row
  // Compacted rows of valid offset q, in slot q % CG_SLOTS.  The lookup of
  // the offset that starts at iteration it + 1 runs at the top of iteration
  // it; with one K step per offset, offset q - 2's adds end in iteration
  // it - 1 and q - 3's in it - 2, behind iteration it - 1's block barrier:
  // three slots never overwrite rows that a thread may still be adding.
  __shared__ long long s_src[CG_SLOTS][CG_M];   // compacted row j: proxy row offset of its source
  __shared__ uint8_t s_row[CG_SLOTS][CG_M];     // compacted row j: its tile row
  __shared__ int s_wcnt[CG_SLOTS][4];           // rows with a source per lookup warp
  __shared__ int s_cell[CG_M], s_xyz[CG_M];
  __shared__ uint32_t s_valid[6];
  __shared__ int4 s_off[189];
  __shared__ int s_nvalid;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tx = tid & 15, ty = tid >> 4;
  const int n0 = blockIdx.y * CG_N;
  int type = 0, tstart = 0, tlist = 0, tcount = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if ((int)blockIdx.x >= tt.start[i]) {
      type = i;
      tstart = tt.start[i];
      tlist = tt.first[i];
      tcount = tt.count[i];
    }
  const int per_tile = CG_M / C;
  const int tfirst = (blockIdx.x - tstart) * per_tile;
  const int ntile = min(per_tile, tcount - tfirst);
  const int nside = 1 << lev;
  const int* my_offs = offs + type * 189 * 4;
  if (tid < CG_M) {
    const int cell = (tid < per_tile * C && tid / C < ntile) ? typed[tlist + tfirst + tid / C] : -1;
    int x = 0, y = 0, z = 0;
    if (cell >= 0) morton_decode((uint32_t)cell, &x, &y, &z);
    s_cell[tid] = cell;
    s_xyz[tid] = (x << 20) | (y << 10) | z;
  }
  if (tid < 6) s_valid[tid] = 0;
  for (int i = tid; i < CG_M * CG_N; i += CG_THREADS) Sum[i] = T(0);
  __syncthreads();
  if (tid < CG_M && s_cell[tid] >= 0 && tid % C == 0) {
    const int x = s_xyz[tid] >> 20, y = (s_xyz[tid] >> 10) & 1023, z = s_xyz[tid] & 1023;
    for (int o = 0; o < 189; ++o) {
      const int bx = x + my_offs[4 * o], by = y + my_offs[4 * o + 1], bz = z + my_offs[4 * o + 2];
      if (bx < 0 || by < 0 || bz < 0 || bx >= nside || by >= nside || bz >= nside) continue;
      const uint32_t bm = morton_encode(bx, by, bz);
      if (sstart[(int64_t)(bm + 1) * span] > sstart[(int64_t)bm * span])
        atomicOr(&s_valid[o >> 5], 1u << (o & 31));
    }
  }
  __syncthreads();
  if (tid == 0) {
    int nv = 0;
    for (int o = 0; o < 189; ++o)
      if ((s_valid[o >> 5] >> (o & 31)) & 1)
        s_off[nv++] = make_int4(my_offs[4 * o], my_offs[4 * o + 1], my_offs[4 * o + 2],
                                my_offs[4 * o + 3]);
    s_nvalid = nv;
  }
  __syncthreads();
  const int nvalid = s_nvalid;
  const int kchunks = (rs + CG_K - 1) / CG_K;
  const int niter = nvalid * kchunks;
  // The rows of the tile that have a source at valid offset q, compacted in
  // row order into slot q % CG_SLOTS; warps 0-3 (one row per thread), with a
  // barrier of their own between the per-warp counts and the writes.
  auto lookup = [&](int q) {
    if (tid >= CG_M) return;
    const int sl = q % CG_SLOTS;
    long long r = -1;
    const int cell = s_cell[tid];
    if (cell >= 0) {
      const int4 o = s_off[q];
      const int x = (s_xyz[tid] >> 20) + o.x, y = ((s_xyz[tid] >> 10) & 1023) + o.y,
                z = (s_xyz[tid] & 1023) + o.z;
      if (x >= 0 && y >= 0 && z >= 0 && x < nside && y < nside && z < nside) {
        const uint32_t bm = morton_encode(x, y, z);
        if (sstart[(int64_t)(bm + 1) * span] > sstart[(int64_t)bm * span])
          r = ((long long)bm * C + tid % C) * rs;
      }
    }
    const unsigned has = __ballot_sync(0xffffffffu, r >= 0);
    if (lane == 0) s_wcnt[sl][warp] = __popc(has);
    asm volatile("bar.sync 1, 128;\n" ::: "memory");
    int base = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) base += k < warp ? s_wcnt[sl][k] : 0;
    if (r >= 0) {
      const int j = base + __popc(has & ((1u << lane) - 1u));
      s_src[sl][j] = r;
      s_row[sl][j] = (uint8_t)tid;
    }
  };
  auto rows_at = [&](int q) {
    const int sl = q % CG_SLOTS;
    return s_wcnt[sl][0] + s_wcnt[sl][1] + s_wcnt[sl][2] + s_wcnt[sl][3];
  };
  // iteration j (offset q = j / kchunks, K chunk j % kchunks) into stage j % CG_NS
  auto load = [&](int j) {
    const int q = j / kchunks, k0 = (j - q * kchunks) * CG_K, st = j % CG_NS;
    const int m_o = rows_at(q);
    const int nr = (m_o + 15) & ~15;  // compacted rows, whole chunks (zero-filled)
    const long long* src = s_src[q % CG_SLOTS];
    T* as = As + st * CG_K * CG_APAD;
    T* bs = Bs + st * CG_K * CG_N;
    for (int e = tid; e < nr * CG_K; e += CG_THREADS) {
      const int m = e / CG_K, kk = e - m * CG_K;
      const long long r = m < m_o ? src[m] : -1;
      const bool ok = r >= 0 && k0 + kk < rs;
      cp_async_elem(as + kk * CG_APAD + m, proxy + (ok ? r + k0 + kk : 0), ok);
    }
    const T* Eo = E + (int64_t)s_off[q].w * rf * rs;
    for (int e = tid; e < CG_N * CG_K; e += CG_THREADS) {
      const int kk = e / CG_N, nn = e - kk * CG_N;
      const bool ok = n0 + nn < rf && k0 + kk < rs;
      cp_async_elem(bs + kk * CG_N + nn, Eo + (ok ? (int64_t)(n0 + nn) + (int64_t)rf * (k0 + kk) : 0),
                    ok);
    }
    cp_async_commit();
  };
  T acc[8][8];  // the current offset's product, compacted rows ty + 16 i
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0;
  // prologue: the first iteration's rows and loads
  if (niter > 0) lookup(0);
  __syncthreads();
  if (niter > 0) load(0);
  for (int it = 0; it < niter; ++it) {
    const int q = it / kchunks;
    // the rows of the offset that starts at iteration it + 1
    if (it + 1 < niter && (it + 1) % kchunks == 0) lookup((it + 1) / kchunks);
    cp_async_wait_all();
    __syncthreads();
    if (it + 1 < niter) load(it + 1);
    const T* as = As + (it % CG_NS) * CG_K * CG_APAD;
    const T* bs = Bs + (it % CG_NS) * CG_K * CG_N;
    const int m_o = rows_at(q);
    switch ((m_o + 15) >> 4) {  // uniform: chunks of 16 compacted rows
      case 1: cg_step<1>(as, bs, tx, ty, acc); break;
      case 2: cg_step<2>(as, bs, tx, ty, acc); break;
      case 3: cg_step<3>(as, bs, tx, ty, acc); break;
      case 4: cg_step<4>(as, bs, tx, ty, acc); break;
      case 5: cg_step<5>(as, bs, tx, ty, acc); break;
      case 6: cg_step<6>(as, bs, tx, ty, acc); break;
      case 7: cg_step<7>(as, bs, tx, ty, acc); break;
      default: cg_step<8>(as, bs, tx, ty, acc); break;
    }
    if ((it + 1) % kchunks == 0) {
      // the offset is complete: add its rows into the running sum by tile row
      const uint8_t* rows = s_row[q % CG_SLOTS];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int j = ty + 16 * i;
        if (j < m_o) {
          T* srow = Sum + (int)rows[j] * CG_N;
#pragma unroll
          for (int c = 0; c < 8; ++c) srow[tx + 16 * c] += acc[i][c];
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[i][c] = 0;
      }
    }
  }
  __syncthreads();
  const int ncol = min(CG_N, rf - n0);
  for (int e = tid; e < CG_M * CG_N; e += CG_THREADS) {
    const int m = e / CG_N, n = e - m * CG_N;
    const int cell = s_cell[m];
    if (cell < 0 || n >= ncol) continue;
    pf[((int64_t)cell * C + m % C) * rf + n0 + n] = Sum[m * CG_N + n];
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
      bool pre_tc = false;  // float path: tcgen05 (scaled F16 hi / lo) when W fits
      if constexpr (std::is_same<T, float>::value) {
        if (colgemm_tc_eligible(t, false)) {
          if (int rc_ = run_colgemm_tc(t, false, lvl, lists + t->lists.src_off[l], ns * C, C,
                                       S + level_offset(l, (int64_t)C * n3),
                                       proxy + level_offset(l, (int64_t)C * rs), 1.f, st))
            return rc_;
          pre_tc = true;
        }
      }
      if (!pre_tc) {
        k_colgemm<T><<<g, kGemmThreads, 0, st>>>(rs, n3, ov.VT + (int64_t)lvl * rs * n3,
                                              lists + t->lists.src_off[l], ns * C, C,
                                              S + level_offset(l, (int64_t)C * n3), ov.Kw,
                                              proxy + level_offset(l, (int64_t)C * rs), nullptr,
                                              T(1));
        PB_LAUNCH("m2l_pre");
      }
      if (int rc_ = kt_end(t, st)) return rc_;
    }
  }
  for (int l = 2; l <= L; ++l) {
    const int lvl = t->homog ? 0 : l - 2;
    const int nt = t->lists.ntgt[l];
    if (nt == 0) continue;
    bool on_tc = false;  // float path: the tcgen05 kernel (split F16 or TF32) when rf fits TMEM
    if constexpr (std::is_same<T, float>::value) {
      if (tc_eligible(t)) {
        if (int rc_ = run_m2l_cheb_tc_level(t, C, l, lvl, proxy + level_offset(l, (int64_t)C * rs),
                                            pf + level_offset(l, (int64_t)C * rf), st))
          return rc_;
        on_tc = true;
      }
    }
    TypeTiles tt;
    const int per_tile = CG_M / C;
    int tiles = 0;
    for (int ty = 0; ty < 8; ++ty) {
      tt.start[ty] = tiles;
      tt.first[ty] = t->lists.ntyp[l][ty];
      tt.count[ty] = t->lists.ntyp[l][ty + 1] - t->lists.ntyp[l][ty];
      tiles += (tt.count[ty] + per_tile - 1) / per_tile;
    }
    tt.start[8] = tiles;
    if (tiles > 0 && !on_tc) {
      dim3 g((unsigned)tiles, (unsigned)((rf + CG_N - 1) / CG_N));
      PB_CUDA(cudaFuncSetAttribute(k_m2l_cheb<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)cg_smem_bytes<T>()));
      if (int rc_ = kt_begin(t, KS_M2L, st)) return rc_;
      k_m2l_cheb<T><<<g, CG_THREADS, cg_smem_bytes<T>(), st>>>(
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
    bool post_tc = false;
    if constexpr (std::is_same<T, float>::value) {
      if (colgemm_tc_eligible(t, true)) {
        if (int rc_ = run_colgemm_tc(t, true, lvl, lists + t->lists.tgt_off[l], nt * C, C,
                                     pf + level_offset(l, (int64_t)C * rf),
                                     F + level_offset(l, (int64_t)C * n3), (float)scale, st))
          return rc_;
        post_tc = true;
      }
    }
    if (!post_tc) {
      k_colgemm<T><<<g2, kGemmThreads, 0, st>>>(n3, rf, ov.U + (int64_t)lvl * n3 * rf,
                                             lists + t->lists.tgt_off[l], nt * C, C,
                                             pf + level_offset(l, (int64_t)C * rf), nullptr,
                                             F + level_offset(l, (int64_t)C * n3), ov.Kw,
                                             (T)scale);
      PB_LAUNCH("m2l_post");
    }
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  return PBBFMM_OK;
}

int run_m2l_cheb(pbbfmm_tree* t, int C, cudaStream_t st) {
  return t->cur_prec == PBBFMM_PREC_FP64 ? run_m2l_cheb_t<double>(t, C, st)
                                         : run_m2l_cheb_t<float>(t, C, st);
}

}  // namespace pbbfmm
