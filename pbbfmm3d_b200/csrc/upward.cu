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

constexpr int kP2MThreads = 256;
constexpr int kP2MChunk = 32;
constexpr int kMaxOut = 4;  // outputs per thread per column group (<= 1024 / 256)

// One CTA per nonempty source leaf.
__global__ void __launch_bounds__(kP2MThreads)
    k_p2m(const int* __restrict__ leaves, const int* __restrict__ sstart,
          const double* __restrict__ spos, int Ns, const double* __restrict__ wsorted, int C,
          int n, int cheb, const double* __restrict__ Tkz_g, double box, int L,
          double* __restrict__ S_L) {
  extern __shared__ double sm[];
  double* sTkz = sm;                               // n*n
  double* sB = sTkz + n * n;                       // 3 x n x chunk basis values
  double* sW = sB + 3 * n * kP2MChunk;             // chunk x C weights
  const int leaf = leaves[blockIdx.x];
  const int a = sstart[leaf], e = sstart[leaf + 1];
  const int n3 = n * n * n;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTkz[i] = Tkz_g[i];
  double c[3];
  cell_center((uint32_t)leaf, L, box, c);
  double len = box;
  for (int i = 0; i < L; ++i) len = 0.5 * len;
  const double ihalfL = 2. / len;
  const int CG = max(1, min(C, (kP2MThreads * kMaxOut) / n3));
  for (int c0 = 0; c0 < C; c0 += CG) {
    const int cg = min(CG, C - c0);
    double acc[kMaxOut];
#pragma unroll
    for (int r = 0; r < kMaxOut; ++r) acc[r] = 0;
    for (int p0 = a; p0 < e; p0 += kP2MChunk) {
      const int cnt = min(kP2MChunk, e - p0);
      __syncthreads();
      if (threadIdx.x < 3 * cnt) {
        const int j = threadIdx.x % cnt, d = threadIdx.x / cnt;
        const double q = ihalfL * (spos[(int64_t)d * Ns + p0 + j] - c[d]);
        basis_all<double>(n, cheb, q, sTkz, sB + (d * n) * kP2MChunk + j, kP2MChunk);
      }
      for (int i = threadIdx.x; i < cnt * cg; i += blockDim.x) {
        const int j = i / cg, cc = i % cg;
        sW[j * CG + cc] = wsorted[(int64_t)(p0 + j) * C + c0 + cc];
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < kMaxOut; ++r) {
        const int o = threadIdx.x + r * kP2MThreads;
        if (o < cg * n3) {
          const int cc = o / n3, l = o % n3;
          const int l1 = l / (n * n), l2 = (l / n) % n, l3 = l % n;
          const double* bx = sB + (0 * n + l1) * kP2MChunk;
          const double* by = sB + (1 * n + l2) * kP2MChunk;
          const double* bz = sB + (2 * n + l3) * kP2MChunk;
          double s = acc[r];
          for (int j = 0; j < cnt; ++j) s += sW[j * CG + cc] * bx[j] * by[j] * bz[j];
          acc[r] = s;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kMaxOut; ++r) {
      const int o = threadIdx.x + r * kP2MThreads;
      if (o < cg * n3) {
        const int cc = o / n3, l = o % n3;
        S_L[((int64_t)leaf * C + c0 + cc) * n3 + l] = acc[r];
      }
    }
  }
}

constexpr int kM2MThreads = 128;
constexpr int kM2MGroup = 1024;  // values per smem buffer

// One CTA per nonempty parent at level l; children at level l+1.
__global__ void __launch_bounds__(kM2MThreads)
    k_m2m(const int* __restrict__ parents, const int* __restrict__ sstart, int span_child,
          const double* __restrict__ Schild, double* __restrict__ Spar, int C, int n,
          const double* __restrict__ Cw_g) {
  __shared__ double sCw[2 * kMaxOrder * kMaxOrder];
  __shared__ double b0[kM2MGroup], b1[kM2MGroup], acc[kM2MGroup];
  const int n2 = n * n, n3 = n2 * n;
  for (int i = threadIdx.x; i < 2 * n2; i += blockDim.x) sCw[i] = Cw_g[i];
  const int par = parents[blockIdx.x];
  const int CG = max(1, min(C, kM2MGroup / n3));
  for (int c0 = 0; c0 < C; c0 += CG) {
    const int cg = min(CG, C - c0);
    const int tot = cg * n3;
    __syncthreads();
    for (int i = threadIdx.x; i < tot; i += blockDim.x) acc[i] = 0;
    for (int ch = 0; ch < 8; ++ch) {
      const int cell = par * 8 + ch;
      const int64_t a = (int64_t)cell * span_child, b = (int64_t)(cell + 1) * span_child;
      if (sstart[b] == sstart[a]) continue;  // empty child: no moments
      const double* wx = sCw + (((ch >> 2) & 1) ? n2 : 0);
      const double* wy = sCw + (((ch >> 1) & 1) ? n2 : 0);
      const double* wz = sCw + ((ch & 1) ? n2 : 0);
      __syncthreads();
      for (int i = threadIdx.x; i < tot; i += blockDim.x)
        b0[i] = Schild[((int64_t)cell * C + c0) * n3 + i];
      __syncthreads();
      // z: Sz[l1*n + l3] = sum_k S[l1*n + k] wz[l3*n + k]   (l1 over n^2)
      for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int cc = i / n3, r = i % n3, l1 = r / n, l3 = r % n;
        const double* s = b0 + cc * n3 + l1 * n;
        double v = 0;
        for (int k = 0; k < n; ++k) v += s[k] * wz[l3 * n + k];
        b1[i] = v;
      }
      __syncthreads();
      // y: Sy[l1 n2 + l2 n + l3] = sum_k Sz[l1 n2 + k n + l3] wy[l2 n + k]
      for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int cc = i / n3, r = i % n3, l1 = r / n2, l2 = (r / n) % n, l3 = r % n;
        const double* s = b1 + cc * n3 + l1 * n2 + l3;
        double v = 0;
        for (int k = 0; k < n; ++k) v += s[k * n] * wy[l2 * n + k];
        b0[i] = v;
      }
      __syncthreads();
      // x: SS[l1 n2 + l2 n + l3] = sum_k Sy[k n2 + l2 n + l3] wx[l1 n + k]
      for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int cc = i / n3, r = i % n3, l1 = r / n2, rem = r % n2;
        const double* s = b0 + cc * n3 + rem;
        double v = 0;
        for (int k = 0; k < n; ++k) v += s[k * n2] * wx[l1 * n + k];
        acc[i] += v;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tot; i += blockDim.x)
      Spar[((int64_t)par * C + c0) * n3 + i] = acc[i];
  }
}

int run_upward(pbbfmm_tree* t, int C, cudaStream_t st) {
  const int L = t->p.tree_level, n = t->n, n3 = t->n3;
  Workspace& ws = t->ws;
  const int* lists = ws.lists.as<int>();
  double* S = ws.S.as<double>();
  const int* sstart = ws.sstart.as<int>();
  const int64_t per = (int64_t)C * n3;
  if (t->lists.nsrc[L] > 0) {
    size_t smem = sizeof(double) * (n * n + 3 * n * kP2MChunk + kP2MChunk * C);
    if (int rc_ = kt_begin(t, KS_P2M, st)) return rc_;
    k_p2m<<<t->lists.nsrc[L], kP2MThreads, smem, st>>>(
        lists + t->lists.src_off[L], sstart, ws.spos.as<double>(), (int)t->last_Ns,
        ws.wsorted.as<double>(), C, n, t->p.use_chebyshev, t->d_Tkz, t->p.L, L,
        S + level_offset(L, per));
    PB_LAUNCH("p2m");
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  for (int l = L - 1; l >= 2; --l) {
    if (t->lists.nsrc[l] == 0) continue;
    if (int rc_ = kt_begin(t, KS_M2M, st)) return rc_;
    k_m2m<<<t->lists.nsrc[l], kM2MThreads, 0, st>>>(
        lists + t->lists.src_off[l], sstart, (int)cells_at(L - l - 1), S + level_offset(l + 1, per),
        S + level_offset(l, per), C, n, t->d_Cw);
    PB_LAUNCH("m2m");
    if (int rc_ = kt_end(t, st)) return rc_;
  }
  return PBBFMM_OK;
}

}  // namespace pbbfmm
