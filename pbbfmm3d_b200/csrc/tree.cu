// Point binning on the GPU: recentring, bit-exact leaf keys, stable sort,
// leaf ranges and per-level lists of nonempty cells.
//
// Reference: H2_3D_Compute ctor recentring (include/compute.hpp:92-131) and
// DistributeFieldPoints (include/compute.hpp:1127-1203) over the octree of
// BuildFMMHierarchy (src/H2_3D_Tree.cpp:917-977).  The reference walks a
// pointer tree and compares each point against FP64 cell centres built by
// repeated +-quarter-length steps; here the same comparisons run per point on
// the device, producing the same Morton leaf index, and a stable radix sort
// keeps the reference's within-leaf order (original index order).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include "fmm.cuh"

namespace pbbfmm {

constexpr int kBBoxBlocks = 296;
constexpr int kBBoxThreads = 256;

__global__ void k_bbox_partial(const double* __restrict__ p, int64_t N, double* __restrict__ part) {
  double mn[3] = {1e32, 1e32, 1e32}, mx[3] = {-1e32, -1e32, -1e32};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double v = p[3 * i + d];
      mn[d] = v < mn[d] ? v : mn[d];
      mx[d] = mx[d] < v ? v : mx[d];
    }
  }
  __shared__ double s[6][kBBoxThreads / 32];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      double a = __shfl_down_sync(0xffffffffu, mn[d], o);
      double b = __shfl_down_sync(0xffffffffu, mx[d], o);
      mn[d] = a < mn[d] ? a : mn[d];
      mx[d] = mx[d] < b ? b : mx[d];
    }
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int d = 0; d < 3; ++d) {
      s[d][w] = mn[d];
      s[3 + d][w] = mx[d];
    }
  __syncthreads();
  if (threadIdx.x < 3) {
    int d = threadIdx.x;
    double a = s[d][0], b = s[3 + d][0];
    for (int j = 1; j < kBBoxThreads / 32; ++j) {
      a = s[d][j] < a ? s[d][j] : a;
      b = b < s[3 + d][j] ? s[3 + d][j] : b;
    }
    part[blockIdx.x * 6 + d] = a;
    part[blockIdx.x * 6 + 3 + d] = b;
  }
}

__global__ void k_bbox_final(const double* __restrict__ part, int nb, double* __restrict__ ctr) {
  if (threadIdx.x < 3) {
    int d = threadIdx.x;
    double a = 1e32, b = -1e32;
    for (int j = 0; j < nb; ++j) {
      a = part[j * 6 + d] < a ? part[j * 6 + d] : a;
      b = b < part[j * 6 + 3 + d] ? part[j * 6 + 3 + d] : b;
    }
    ctr[d] = 0.5 * (a + b);  // include/compute.hpp:108-111
  }
}

// Leaf key by the reference's comparison descent.
__global__ void k_keys(const double* __restrict__ p, int64_t N, const double* __restrict__ ctr,
                       double box, int L, uint32_t* __restrict__ key, int* __restrict__ idx) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double qx = p[3 * i + 0] - ctr[0];
  const double qy = p[3 * i + 1] - ctr[1];
  const double qz = p[3 * i + 2] - ctr[2];
  double cx = 0, cy = 0, cz = 0, len = box;
  uint32_t k = 0;
  for (int lev = 0; lev < L; ++lev) {
    const int bx = !(qx < cx), by = !(qy < cy), bz = !(qz < cz);
    k = k * 8u + (uint32_t)(4 * bx + 2 * by + bz);
    const double q = 0.25 * len;
    cx = bx ? __dadd_rn(cx, q) : __dsub_rn(cx, q);
    cy = by ? __dadd_rn(cy, q) : __dsub_rn(cy, q);
    cz = bz ? __dadd_rn(cz, q) : __dsub_rn(cz, q);
    len = 0.5 * len;
  }
  key[i] = k;
  idx[i] = (int)i;
}

// start[k] = first sorted position with key >= k, k in [0, nleaf].
__global__ void k_leaf_start(const uint32_t* __restrict__ ks, int N, int64_t nleaf,
                             int* __restrict__ start) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k > nleaf) return;
  int lo = 0, hi = N;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if ((int64_t)ks[mid] < k)
      lo = mid + 1;
    else
      hi = mid;
  }
  start[k] = lo;
}

__global__ void k_gather_pos(const double* __restrict__ p, const int* __restrict__ perm, int N,
                             const double* __restrict__ ctr, double* __restrict__ soa) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int j = perm[i];
#pragma unroll
  for (int d = 0; d < 3; ++d) soa[(int64_t)d * N + i] = p[3 * (int64_t)j + d] - ctr[d];
}

__global__ void k_gather_w(const double* __restrict__ w, const int* __restrict__ perm, int Ns,
                           int C, double* __restrict__ ws) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)Ns * C) return;
  int j = (int)(t / C), c = (int)(t % C);
  ws[t] = w[(int64_t)c * Ns + perm[j]];
}

struct NonEmpty {
  const int* start;
  int span_shift;  // 3 * (L - l)
  __host__ __device__ bool operator()(int cell) const {
    int64_t a = (int64_t)cell << span_shift, b = (int64_t)(cell + 1) << span_shift;
    return start[b] > start[a];
  }
};

// virtual index v -> cell 8*(v % npar) + v / npar, so selection is ordered by
// (child type, parent Morton index)
struct TypedCell {
  int npar;
  __host__ __device__ int operator()(int v) const { return 8 * (v % npar) + v / npar; }
};

__global__ void k_type_bounds(const int* __restrict__ list, const int* __restrict__ count,
                              int* __restrict__ bounds) {
  int t = threadIdx.x;
  if (t > 8) return;
  int n = *count;
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if ((list[mid] & 7) < t)
      lo = mid + 1;
    else
      hi = mid;
  }
  bounds[t] = lo;
}

int run_binning(pbbfmm_tree* t, const double* d_tgt, int64_t Nf, const double* d_src, int64_t Ns,
                const double* d_w, int C, cudaStream_t st) {
  Workspace& ws = t->ws;
  const int L = t->p.tree_level;
  const int64_t nleaf = cells_at(L);
  const int64_t Nmax = Nf > Ns ? Nf : Ns;

  // CUB scratch: radix sort of Nmax keys and selection over 8^L cells
  size_t sort_bytes = 0, sel_bytes = 0;
  PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint32_t*)nullptr,
                                          (uint32_t*)nullptr, (const int*)nullptr, (int*)nullptr,
                                          (int)Nmax, 0, 3 * L, st));
  size_t sel2_bytes = 0;
  {
    NonEmpty pred{nullptr, 0};
    thrust::counting_iterator<int> it(0);
    PB_CUDA(cub::DeviceSelect::If(nullptr, sel_bytes, it, (int*)nullptr, (int*)nullptr,
                                  (int)nleaf, pred, st));
    auto tit = thrust::make_transform_iterator(it, TypedCell{(int)(nleaf / 8)});
    PB_CUDA(cub::DeviceSelect::If(nullptr, sel2_bytes, tit, (int*)nullptr, (int*)nullptr,
                                  (int)nleaf, pred, st));
  }
  size_t cub_need = sort_bytes > sel_bytes ? sort_bytes : sel_bytes;
  cub_need = cub_need > sel2_bytes ? cub_need : sel2_bytes;

  int64_t list_need = 0;
  for (int l = 2; l <= L; ++l) {
    int64_t nc = cells_at(l);
    list_need += (nc < Ns ? nc : Ns) + 2 * (nc < Nf ? nc : Nf);
  }
  int rc;
  if ((rc = grow(ws.bbox_part, 8 * 6 * kBBoxBlocks))) return rc;
  if ((rc = grow(ws.ctr, 8 * 4))) return rc;
  if ((rc = grow(ws.key, 4 * Nmax))) return rc;
  if ((rc = grow(ws.key_sorted, 4 * Nmax))) return rc;
  if ((rc = grow(ws.idx, 4 * Nmax))) return rc;
  if ((rc = grow(ws.tperm, 4 * Nf))) return rc;
  if ((rc = grow(ws.sperm, 4 * Ns))) return rc;
  if ((rc = grow(ws.tstart, 4 * (nleaf + 1)))) return rc;
  if ((rc = grow(ws.sstart, 4 * (nleaf + 1)))) return rc;
  if ((rc = grow(ws.tpos, 8 * 3 * Nf))) return rc;
  if ((rc = grow(ws.spos, 8 * 3 * Ns))) return rc;
  if ((rc = grow(ws.wsorted, 8 * Ns * (int64_t)C))) return rc;
  if ((rc = grow(ws.cub_temp, cub_need))) return rc;
  if ((rc = grow(ws.lists, 4 * (list_need + 16)))) return rc;
  if ((rc = grow(ws.dcounts, 4 * (kMaxLevel + 1) * 12))) return rc;
  double* ctr = ws.ctr.as<double>();
  uint32_t* key = ws.key.as<uint32_t>();
  uint32_t* key_sorted = ws.key_sorted.as<uint32_t>();
  int* idx = ws.idx.as<int>();
  int* lists = ws.lists.as<int>();

  // recentre on the target bounding box (an adjoint pass keeps the forward
  // targets' box, given by bbox_pts)
  const double* bpts = t->bbox_pts ? t->bbox_pts : d_tgt;
  const int64_t bn = t->bbox_pts ? t->bbox_n : Nf;
  k_bbox_partial<<<kBBoxBlocks, kBBoxThreads, 0, st>>>(bpts, bn, ws.bbox_part.as<double>());
  k_bbox_final<<<1, 32, 0, st>>>(ws.bbox_part.as<double>(), kBBoxBlocks, ctr);
  PB_LAUNCH_N("bbox", 2);

  auto bin_set = [&](const double* pts, int64_t N, int* perm, int* start) -> int {
    if (N > 0) {
      k_keys<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(pts, N, ctr, t->p.L, L, key, idx);
      PB_LAUNCH("keys");
      size_t bytes = ws.cub_temp.cap;
      PB_CUDA(cub::DeviceRadixSort::SortPairs(ws.cub_temp.p, bytes, key, key_sorted, idx, perm,
                                              (int)N, 0, 3 * L, st));
      // onesweep: one histogram pass plus one pass per 8-bit digit
      count_launches(1 + (3 * L + 7) / 8);
    }
    k_leaf_start<<<(unsigned)((nleaf + 1 + 255) / 256), 256, 0, st>>>(key_sorted, (int)N, nleaf,
                                                                      start);
    PB_LAUNCH("leaf_start");
    return PBBFMM_OK;
  };
  if ((rc = bin_set(d_tgt, Nf, ws.tperm.as<int>(), ws.tstart.as<int>()))) return rc;
  if (Nf > 0) {
    k_gather_pos<<<(unsigned)((Nf + 255) / 256), 256, 0, st>>>(d_tgt, ws.tperm.as<int>(), (int)Nf,
                                                               ctr, ws.tpos.as<double>());
    PB_LAUNCH("gather_tpos");
  }
  if ((rc = bin_set(d_src, Ns, ws.sperm.as<int>(), ws.sstart.as<int>()))) return rc;
  if (Ns > 0) {
    k_gather_pos<<<(unsigned)((Ns + 255) / 256), 256, 0, st>>>(d_src, ws.sperm.as<int>(), (int)Ns,
                                                               ctr, ws.spos.as<double>());
    int64_t tot = Ns * (int64_t)C;
    k_gather_w<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d_w, ws.sperm.as<int>(), (int)Ns, C,
                                                              ws.wsorted.as<double>());
    PB_LAUNCH_N("gather_src", 2);
  }

  // nonempty-cell lists for levels 2..L
  LevelLists& LL = t->lists;
  int64_t off = 0;
  int* cnt = ws.dcounts.as<int>();  // [l][0]=nsrc [l][1]=ntgt [l][2]=ntyp [l][3..11] type bounds
  for (int l = 2; l <= L; ++l) {
    const int64_t nc = cells_at(l);
    const int shift = 3 * (L - l);
    thrust::counting_iterator<int> it(0);
    size_t bytes;
    LL.src_off[l] = off;
    bytes = ws.cub_temp.cap;
    PB_CUDA(cub::DeviceSelect::If(ws.cub_temp.p, bytes, it, lists + off, cnt + 12 * l + 0,
                                  (int)nc, NonEmpty{ws.sstart.as<int>(), shift}, st));
    off += (nc < Ns ? nc : Ns);
    LL.tgt_off[l] = off;
    bytes = ws.cub_temp.cap;
    PB_CUDA(cub::DeviceSelect::If(ws.cub_temp.p, bytes, it, lists + off, cnt + 12 * l + 1,
                                  (int)nc, NonEmpty{ws.tstart.as<int>(), shift}, st));
    off += (nc < Nf ? nc : Nf);
    LL.typ_off[l] = off;
    bytes = ws.cub_temp.cap;
    auto tit = thrust::make_transform_iterator(it, TypedCell{(int)(nc / 8)});
    PB_CUDA(cub::DeviceSelect::If(ws.cub_temp.p, bytes, tit, lists + off, cnt + 12 * l + 2,
                                  (int)nc, NonEmpty{ws.tstart.as<int>(), shift}, st));
    count_launches(3 * 2);  // three DeviceSelect calls: init + scan kernels each
    k_type_bounds<<<1, 32, 0, st>>>(lists + off, cnt + 12 * l + 2, cnt + 12 * l + 3);
    PB_LAUNCH("type_bounds");
    off += (nc < Nf ? nc : Nf);
  }
  int hc[(kMaxLevel + 1) * 12];
  PB_CUDA(cudaMemcpyAsync(hc, ws.dcounts.p, sizeof(int) * 12 * (L + 1), cudaMemcpyDeviceToHost, st));
  PB_CUDA(cudaStreamSynchronize(st));
  for (int l = 2; l <= L; ++l) {
    LL.nsrc[l] = hc[12 * l + 0];
    LL.ntgt[l] = hc[12 * l + 1];
    for (int k = 0; k < 9; ++k) LL.ntyp[l][k] = hc[12 * l + 3 + k];
  }
  return PBBFMM_OK;
}

}  // namespace pbbfmm
