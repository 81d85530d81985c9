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
  // which children hold targets (lanes 0..8 read the 9 leaf-range bounds at
  // once)
  int bound = 0;
  if (lane <= 8) bound = tstart[(int64_t)(par * 8 + lane) * span_child];
  unsigned present = 0;
#pragma unroll
  for (int ch = 0; ch < 8; ++ch)
    present |= (__shfl_sync(0xffffffffu, bound, ch + 1) != __shfl_sync(0xffffffffu, bound, ch))
                   ? 1u << ch : 0u;
  constexpr int PER = (n3 + 31) / 32;
  constexpr bool kRows = N <= (sizeof(T) == 4 ? 6 : 5);  // passes as row tasks
  constexpr bool kBatch = sizeof(T) == 4 && N <= 5;
  constexpr int TPL = (n2 + 31) / 32;                    // row tasks per lane
  if constexpr (kRows) {
    // Each pass as row tasks: a lane loads the N inputs of one 1-D transform
    // once and forms its N outputs (operator rows read by broadcast).  The
    // z pass of task r updates the child's coefficients r n .. r n + n-1,
    // read up front for all children (kBatch) so those loads are in flight
    // together.
    T cur[kBatch ? 8 : 1][kBatch ? TPL : 1][kBatch ? N : 1];
    if constexpr (kBatch) {
#pragma unroll
      for (int ch = 0; ch < 8; ++ch) {
        const T* d = Fch + ((int64_t)(par * 8 + ch) * C + col) * n3;
#pragma unroll
        for (int t = 0; t < TPL; ++t) {
          const int r = lane + 32 * t;
#pragma unroll
          for (int l3 = 0; l3 < N; ++l3)
            cur[ch][t][l3] = ((present >> ch) & 1) && r < n2 ? d[r * N + l3] : T(0);
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      const int cell = par * 8 + ch;
      if (!((present >> ch) & 1)) continue;  // child without targets
      const T* wx = sCw + (((ch >> 2) & 1) ? n2 : 0);
      const T* wy = sCw + (((ch >> 1) & 1) ? n2 : 0);
      const T* wz = sCw + ((ch & 1) ? n2 : 0);
      // x: Fx[l1 n2 + rem] = sum_k F[k n2 + rem] wx[l1 + k n]   (task rem)
      for (int q = lane; q < n2; q += 32) {
        T x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = sp[k * n2 + q];
#pragma unroll
        for (int l1 = 0; l1 < N; ++l1) {
          T v = 0;
#pragma unroll
          for (int k = 0; k < N; ++k) v = fma(x[k], wx[l1 + k * N], v);
          b0[l1 * n2 + q] = v;
        }
      }
      __syncwarp();
      // y: Fy[l1 n2 + l2 n + l3] = sum_k Fx[l1 n2 + k n + l3] wy[l2 + k n]   (task (l1, l3))
      for (int q = lane; q < n2; q += 32) {
        const int l1 = q / N, l3 = q % N;
        T x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = b0[l1 * n2 + k * N + l3];
#pragma unroll
        for (int l2 = 0; l2 < N; ++l2) {
          T v = 0;
#pragma unroll
          for (int k = 0; k < N; ++k) v = fma(x[k], wy[l2 + k * N], v);
          b1[l1 * n2 + l2 * N + l3] = v;
        }
      }
      __syncwarp();
      // z: Fchild[r n + l3] += sum_k Fy[r n + k] wz[l3 + k n]   (task row r over n^2)
      T* dst = Fch + ((int64_t)cell * C + col) * n3;
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        const int r = lane + 32 * t;
        if (r < n2) {
          T x[N];
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = b1[r * N + k];
#pragma unroll
          for (int l3 = 0; l3 < N; ++l3) {
            T v = 0;
#pragma unroll
            for (int k = 0; k < N; ++k) v = fma(x[k], wz[l3 + k * N], v);
            if constexpr (kBatch) dst[r * N + l3] = cur[ch][t][l3] + v;
            else dst[r * N + l3] += v;
          }
        }
      }
      __syncwarp();
    }
  } else {
    __syncwarp();
    for (int ch = 0; ch < 8; ++ch) {
      const int cell = par * 8 + ch;
      if (!((present >> ch) & 1)) continue;  // child without targets
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
  (void)PER;
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

// The leaf kernels' arguments for this compute.  Potentials: the leaves are
// partitioned dense-first and the dense leaves' 32-target chunks counted and
// scanned (so that each launch's active warps are packed into the first CTAs
// of its grid).  Gradients: all leaves, one warp each.
static int prepare_leaf_args(pbbfmm_tree* t, int64_t Nf, int64_t Ns, int C, double* out,
                             cudaStream_t st, pbbfmm_leaf_args* a) {
  const int L = t->p.tree_level;
  const int nl = t->lists.ntgt[L];
  Workspace& ws = t->ws;
  const bool f64 = t->cur_prec == PBBFMM_PREC_FP64;
  const int64_t perS = (int64_t)C * t->n3;
  *a = pbbfmm_leaf_args{};
  a->precision = t->cur_prec;
  a->gradient = t->gl.on ? 1 : 0;
  a->leaves = ws.lists.as<int>() + t->lists.tgt_off[L];
  a->nleaves = nl;
  a->tstart = ws.tstart.as<int>();
  a->sstart = ws.sstart.as<int>();
  a->tperm = ws.tperm.as<int>();
  a->tpos = ws.tpos.as<double>();
  a->spos = ws.spos.as<double>();
  a->wsorted = ws.wsorted.as<double>();
  a->Nf = (int)Nf;
  a->Ns = (int)Ns;
  a->C = C;
  a->F_leaf = f64 ? (const void*)(ws.F.as<double>() + level_offset(L, perS))
                  : (const void*)(ws.F.as<float>() + level_offset(L, perS));
  a->n = t->n;
  a->cheb = t->p.use_chebyshev;
  a->Tkz = f64 ? (const void*)t->d_Tkz : (const void*)t->f_Tkz;
  a->box = t->p.L;
  a->L = L;
  a->kparam = t->d_kparam;
  if (t->gl.on) {
    a->out = t->gl.values ? out : nullptr;
    a->contract = t->gl.contract;
    a->grad_out = t->gl.grad_out;
    return PBBFMM_OK;
  }
  a->out = out;
  if (int rc_ = grow(ws.leafpart, sizeof(int) * 3 * ((size_t)nl + 1))) return rc_;
  int* part = ws.leafpart.as<int>();
  int* nsel = part + nl;
  size_t tb = 0;
  DenseLeaf pred{ws.tstart.as<int>()};
  PB_CUDA(cub::DevicePartition::If(nullptr, tb, a->leaves, part, nsel, nl, pred, st));
  if (int rc_ = grow(ws.cub_temp, tb)) return rc_;
  tb = ws.cub_temp.cap;
  PB_CUDA(cub::DevicePartition::If(ws.cub_temp.p, tb, a->leaves, part, nsel, nl, pred, st));
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
  a->leaves = part;
  a->ndense = nsel;
  a->chunk_prefix = prefix;
  // upper bound of the chunk count: Nf / 32 + one partial chunk per dense
  // leaf (at most Nf / kLaneLeafMin of them)
  a->max_chunks = Nf / 32 + (nl < Nf / kLaneLeafMin ? nl : Nf / kLaneLeafMin) + 1;
  return PBBFMM_OK;
}

// Status of a leaf launcher's return value (0, a cudaError_t code, or -1 for
// a gradient pass of a kernel without gradient).
static int leaf_status(int r) {
  if (r == 0) return PBBFMM_OK;
  if (r < 0) {
    set_error("this kernel has no gradient: position gradients are not available");
    return PBBFMM_ERR_UNSUPPORTED;
  }
  return cuda_status((cudaError_t)r, "leaf kernels");
}

struct LeafBuiltin {
  const pbbfmm_leaf_args* a;
  cudaStream_t st;
  template <class KF>
  int run() {
    return leaf_status(launch_leaf_kernels<KF>(*a, st));
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
  if (t->lists.ntgt[t->p.tree_level] == 0) return PBBFMM_OK;
  pbbfmm_leaf_args a;
  if (int rc = kt_begin(t, KS_LEAF, st)) return rc;
  if (int rc = prepare_leaf_args(t, Nf, Ns, C, d_out, st, &a)) return rc;
  int rc;
  if (t->p.kernel == PBBFMM_KERNEL_USER) {
    if (a.gradient && !t->user.has_gradient) return leaf_status(-1);
    rc = leaf_status(t->user.launch_leaf(&a, (void*)st));
  } else {
    LeafBuiltin lb{&a, st};
    rc = dispatch_kernel(t->p.kernel, lb);
  }
  if (rc) return rc;
  count_launches(a.gradient ? 1 : 2);
  return kt_end(t, st);
}

}  // namespace pbbfmm
