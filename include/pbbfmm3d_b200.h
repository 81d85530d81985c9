/*
 * pbbfmm3d_b200 — C ABI of the B200-native black-box FMM matvec.
 *
 * This is the drop-in boundary for PBBFMM3D's matvec hot path
 * (H2_3D_Compute<T>, include/compute.hpp:67-149 of the reference).  Plain
 * pointers and sizes only; every call returns a status code (never exits)
 * and pbbfmm_last_error() describes the most recent failure on this thread.
 *
 * Object model, one-to-one with the reference:
 *   pbbfmm_tree_create   <- H2_3D_Tree(L, tree_level, order, eps, use_chebyshev)
 *                           + SetKernelProperty()   (src/H2_3D_Tree.cpp:12-38,
 *                           src/kernel_Types.cpp)
 *   pbbfmm_tree_build    <- buildFMMTree()          (src/H2_3D_Tree.cpp:40-66)
 *   pbbfmm_compute       <- H2_3D_Compute<T>(tree, target, source, weight,
 *                           nCols, output)           (include/compute.hpp:67)
 * A tree is built once and can then serve any number of computes (the
 * reference cannot be reused; here geometry and operators are cached on the
 * device and points are re-binned on every call).
 *
 * Layouts (as in the reference): points are xyz AoS float64 (vector3,
 * include/bbfmm.h:29-39); weight is column-major Ns x nCols
 * (weight[col*Ns + i]); output is column-major Nf x nCols and is ACCUMULATED
 * into (include/compute.hpp:747).  Sources and targets may differ.
 */
#ifndef PBBFMM3D_B200_H
#define PBBFMM3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PBBFMM_OK 0
#define PBBFMM_ERR_ARG 1         /* bad argument (size, order, level, pointer) */
#define PBBFMM_ERR_CUDA 2        /* CUDA runtime / launch error                */
#define PBBFMM_ERR_ALLOC 3       /* device or host allocation failed           */
#define PBBFMM_ERR_STATE 4       /* call out of order (e.g. compute before build) */
#define PBBFMM_ERR_IO 5          /* operator cache file unreadable / malformed */
#define PBBFMM_ERR_UNSUPPORTED 6 /* combination not implemented                */
#define PBBFMM_ERR_NUMERIC 7     /* non-finite input detected                  */
#define PBBFMM_ERR_TIMEOUT 8     /* a bounded device wait ran out (output invalid) */

/* ---- built-in kernels (src/kernel_Types.cpp; the last three are the user
 * kernels of the reference's examples and python binding) ---- */
#define PBBFMM_KERNEL_LAPLACIAN 0       /* 1/r            homogen -1 */
#define PBBFMM_KERNEL_ONEOVERR2 1       /* 1/r^2          homogen -2 */
#define PBBFMM_KERNEL_ONEOVERR4 2       /* 1/r^4          homogen -4 */
#define PBBFMM_KERNEL_GAUSSIAN 3        /* exp(-r^2)                 */
#define PBBFMM_KERNEL_LOGARITHM 4       /* 0.5 log(r^2)              */
#define PBBFMM_KERNEL_QUADRIC 5         /* 1 + r^2                   */
#define PBBFMM_KERNEL_INVQUADRIC 6      /* 1 / (1 + r^2)             */
#define PBBFMM_KERNEL_THINPLATESPLINE 7 /* 0.5 r^2 log(r^2)          */
#define PBBFMM_KERNEL_EXPCOV 8          /* exp(-r / p0)              */
#define PBBFMM_KERNEL_GAUSSSIGMA 9      /* exp(-r^2 / (2 p0^2))      */
#define PBBFMM_KERNEL_ANISOEXP 10       /* 0.75 exp(-sqrt(dx^2/100 + dy^2/100 + dz^2/2.25)) */
#define PBBFMM_KERNEL_COUNT 11

/* ---- precision modes ---- */
#define PBBFMM_PREC_FP64 0  /* every phase in float64 (the plain GPU path)  */
#define PBBFMM_PREC_MIXED 1 /* tensor-core split-precision M2L, FP32 Kahan
                               interpolation and near field                  */

typedef struct pbbfmm_tree pbbfmm_tree;

typedef struct {
  double L;                /* side of the cubic computational box           */
  int tree_level;          /* number of levels below the root               */
  int interpolation_order; /* n, nodes per dimension (2..10)                */
  double epsilon;          /* SVD truncation tolerance (Chebyshev)          */
  int use_chebyshev;       /* 1: Chebyshev + SVD M2L, 0: uniform + FFT M2L  */
  int kernel;              /* PBBFMM_KERNEL_*                               */
  double kernel_param[4];  /* kernel parameters (p0 = length scale)         */
} pbbfmm_tree_params;

/* H2_3D_Tree constructor + SetKernelProperty (src/H2_3D_Tree.cpp:12-38).
 * Selects the CUDA device; nothing is computed yet.  device = -1 makes a
 * host-only tree: buildFMMTree's float64 precompute and the operator
 * accessors work without a GPU, computes return PBBFMM_ERR_STATE. */
int pbbfmm_tree_create(const pbbfmm_tree_params *params, int device, pbbfmm_tree **tree);

/* ---- user-defined kernels ----
 * The reference's user kernels subclass H2_3D_Tree and define
 * SetKernelProperty (homogen, symmetry, kernelType) and
 * EvaluateKernel(target, source) (README.md:178-227, include/H2_3D_Tree.hpp:
 * 93-95).  Here a user kernel is a __device__ functor compiled by the user's
 * nvcc: include/pbbfmm3d_b200_kernel.cuh turns a class with a
 * __host__ __device__ EvaluateKernel into a pbbfmm_user_kernel whose
 * launch_leaf instantiates this library's leaf kernels (L2P + P2P,
 * include/pbbfmm3d_b200_leaf.cuh) for it.  Everything else in a compute is
 * kernel-independent once the operators exist. */

/* Everything the leaf-phase kernels read, prepared by the library for one
 * compute (device pointers unless noted). */
typedef struct {
  int precision;             /* PBBFMM_PREC_FP64: F_leaf / Tkz are double; MIXED: float */
  int gradient;              /* 0: potentials (L2P + P2P);  1: potentials and gradients */
  const int *leaves;         /* nonempty target leaves (values: dense ones first) */
  int nleaves;
  const int *ndense;         /* values: number of dense leaves (device scalar) */
  const int *chunk_prefix;   /* values: first 32-target chunk of each dense leaf */
  int64_t max_chunks;        /* values: upper bound of the dense chunks (host) */
  const int *tstart, *sstart;  /* leaf offsets of the sorted targets / sources */
  const int *tperm;            /* sorted target -> original index */
  const double *tpos, *spos;   /* recentred sorted positions, SoA 3 x N */
  const double *wsorted;       /* sorted weights, point-major [j][col] */
  int Nf, Ns, C;
  const void *F_leaf;        /* leaf-level local coefficients [cell][col][n^3] */
  int n, cheb;               /* interpolation order, 1 = Chebyshev */
  const void *Tkz;           /* Chebyshev polynomial table n x n */
  double box;                /* side of the computational box (host) */
  int L;                     /* tree level (host) */
  const double *kparam;      /* 4 kernel parameters */
  double *out;               /* output [col * Nf + i] += potentials (may be NULL in gradient mode) */
  const double *contract;    /* gradient: weights of each target's gradient [col * Nf + i] */
  double *grad_out;          /* gradient: [i * 3 + d] += sum_col contract * d phi / d x_d */
} pbbfmm_leaf_args;

typedef struct {
  const char *kernel_type; /* kernelType: names the operator-cache files */
  double homogen;          /* degree of homogeneity as SetKernelProperty sets it (0: none) */
  int symmetry;            /* 1 symmetric, -1 antisymmetric, 0 neither */
  /* EvaluateKernel(target, source) in float64 on the host: the operator
   * precompute (src/H2_3D_Tree.cpp:251-648) */
  double (*evaluate)(const double *target, const double *source, void *ctx);
  /* the leaf kernels instantiated for the device functor, launched on
   * `stream` (a cudaStream_t): 0, a cudaError_t code, or -1 when a gradient
   * pass is asked of a kernel without a gradient */
  int (*launch_leaf)(const pbbfmm_leaf_args *args, void *stream);
  int has_gradient;        /* launch_leaf supports gradient mode */
  void *ctx;               /* passed to evaluate */
} pbbfmm_user_kernel;

#define PBBFMM_KERNEL_USER 64

/* A tree over a user-defined kernel (the constructor + SetKernelProperty of
 * a user subclass of H2_3D_Tree).  params->kernel and kernel_param are
 * ignored; *kernel is copied (kernel_type included) and its functions must
 * stay valid for the tree's lifetime. */
int pbbfmm_tree_create_user(const pbbfmm_tree_params *params, const pbbfmm_user_kernel *kernel,
                            int device, pbbfmm_tree **tree);

/* buildFMMTree (src/H2_3D_Tree.cpp:40-66): computes the interpolation
 * weights and the M2L operators in float64 on the host and uploads them.
 * If cache_dir is non-NULL, operator files in the reference's format and
 * naming (<cache_dir>/<kernelType>{Cheb,Unif}{K,U,V}<n>.bin,
 * src/H2_3D_Tree.cpp:84-91) are read when present and valid
 * (PrecomputeAvailable, :102-132) and written otherwise. */
int pbbfmm_tree_build(pbbfmm_tree *tree, const char *cache_dir);

/* Install M2L operators directly, in the layout FMMReadMatrices returns
 * (src/H2_3D_Tree.cpp:186-239): Chebyshev K = nlev x 316 x (rf x rs),
 * U = nlev x (n^3 x rf), VT = nlev x (rs x n^3), all column-major; uniform
 * K = nlev x 316 x (2n-1)^3 FFTW halfcomplex spectra, U/VT ignored.
 * nlev = 1 for homogeneous kernels, tree_level - 1 otherwise.  Replaces
 * pbbfmm_tree_build's precompute (the weights are still computed). */
int pbbfmm_tree_set_operators(pbbfmm_tree *tree, int rf, int rs, int nlev, const double *K,
                              const double *U, const double *VT);

/* Copy the tree's operators out in the same layout (NULL pointers query the
 * sizes: *rf, *rs, *nlev are always written). */
int pbbfmm_tree_get_operators(const pbbfmm_tree *tree, int *rf, int *rs, int *nlev, double *K,
                              double *U, double *VT);

int pbbfmm_tree_destroy(pbbfmm_tree *tree);

/* H2_3D_Compute<T>(tree, target, source, weight, nCols, output)
 * (include/compute.hpp:67-149).  HOST buffers; copies in, runs on the tree's
 * device, copies out and synchronises.  output += K * weight. */
int pbbfmm_compute(pbbfmm_tree *tree, const double *target, int64_t Nf, const double *source,
                   int64_t Ns, const double *weight, int nCols, double *output);

/* Same, on DEVICE buffers, asynchronous on `stream` (a cudaStream_t; NULL =
 * legacy default stream).  precision: PBBFMM_PREC_*. */
int pbbfmm_compute_device(pbbfmm_tree *tree, const double *d_target, int64_t Nf,
                          const double *d_source, int64_t Ns, const double *d_weight, int nCols,
                          double *d_output, int precision, void *stream);

/* Adjoint of the matvec f = K(target, source) w, for a loss L with upstream
 * gradient g = dL/df (Nf x nCols, column-major, device).  No counterpart in
 * the reference, which has no derivatives; its transposed product is the
 * reference's H2_3D_Compute with sources and targets swapped.  Each output is
 * accumulated into when non-NULL:
 *   d_grad_weight (Ns x nCols) += K^T g, the exact transpose of this tree's
 *       FMM (same box, same interaction lists, transposed operators);
 *   d_grad_source (Ns x 3, xyz AoS) += dL/dy_j = sum_c w_jc grad_y phi_c(y_j),
 *       phi = K^T g, through the differentiated interpolation basis and the
 *       kernel gradient (needs d_weight);
 *   d_grad_target (Nf x 3, xyz AoS) += dL/dx_i = sum_c g_ic grad_x f_c(x_i)
 *       (needs d_weight).
 * Asynchronous on `stream`; precision: PBBFMM_PREC_*. */
int pbbfmm_compute_adjoint_device(pbbfmm_tree *tree, const double *d_target, int64_t Nf,
                                  const double *d_source, int64_t Ns, const double *d_weight,
                                  const double *d_g, int nCols, double *d_grad_weight,
                                  double *d_grad_source, double *d_grad_target, int precision,
                                  void *stream);

/* Precision used by pbbfmm_compute (default PBBFMM_PREC_FP64). */
int pbbfmm_set_precision(pbbfmm_tree *tree, int precision);

/* Chebyshev M2L of the mixed path on the tensor cores (tcgen05, split
 * precision hi + lo with three products and float32 accumulation; default on).
 * mode: PBBFMM_TC_F16 (default): F16 hi / lo parts of power-of-two scaled
 *       proxies and operators (kind::f16);
 *       PBBFMM_TC_TF32: TF32 hi / lo parts (kind::tf32, "3xTF32");
 *       PBBFMM_TC_OFF: the CUDA-core float32 kernel instead.
 * (1 still means "on"; it is PBBFMM_TC_F16.)  No reference counterpart: the
 * reference has one CPU path.  pbbfmm_tensor_core_m2l returns the format a
 * mixed Chebyshev compute of this tree runs with (PBBFMM_TC_F16 or
 * PBBFMM_TC_TF32), or PBBFMM_TC_OFF when it runs on the CUDA cores (disabled,
 * operators not loaded, or r_f > 256).
 * If a tensor-core wait ever times out (about 1 s), that compute's output is
 * invalid and the next compute entry returns PBBFMM_ERR_TIMEOUT once. */
#define PBBFMM_TC_OFF 0
#define PBBFMM_TC_F16 1
#define PBBFMM_TC_TF32 2
int pbbfmm_set_tensor_cores(pbbfmm_tree *tree, int mode);
int pbbfmm_tensor_core_m2l(const pbbfmm_tree *tree);

/* Test access to the timeout path (no reference counterpart).  Sets the poll
 * limit of the tensor-core Chebyshev M2L's pipeline waits on `device` (-1:
 * the current device); polls <= 0 restores the default (about a second).
 * With a limit of a few polls those waits run out, the kernel stops, waits
 * with the full bound for the copies and MMAs it has already issued, frees
 * its TMEM and reports through the timeout flag: the compute returns
 * PBBFMM_ERR_TIMEOUT (pbbfmm_compute leaves the output untouched) and the
 * next compute runs normally once the limit is restored. */
int pbbfmm_debug_set_pipeline_wait_limit(int device, long long polls);

/* Per-phase device times (ms) of the last compute, when timing is enabled
 * with pbbfmm_set_timing(tree, 1).  names: comma-separated phase names. */
int pbbfmm_set_timing(pbbfmm_tree *tree, int enable);
int pbbfmm_get_phase_times(const pbbfmm_tree *tree, float *ms, int max_phases, int *nphases,
                           const char **names);

/* Per-kernel device times: with timing enabled, every launch of a compute
 * is bracketed by CUDA events on its stream.  Slots (names, comma-separated):
 * binning, p2m, m2m, m2l_pre, m2l, m2l_post, fft_fwd, m2l_mac, fft_inv,
 * l2l, leaf, m2l_split.  ms / launches are summed since the last reset. */
int pbbfmm_reset_kernel_times(pbbfmm_tree *tree);
int pbbfmm_get_kernel_times(pbbfmm_tree *tree, float *ms, int *launches, int max_slots,
                            int *nslots, const char **names);

/* Measured float64 (precision 0) or float32 (1) FMA throughput of `device`
 * in TFLOP/s (2 flops per FMA): the peak the CUDA-core kernels are held to;
 * precision 2: float32 reciprocal square roots (the special-function pipe)
 * in 1e12 per second. */
int pbbfmm_measure_fma_peak(int device, int precision, double *tflops);

/* Debug/test access to device arrays of the last compute (all as float64):
 * what = 0 moments S of `level` (8^level x nCols x n^3, cell-major; only
 * nonempty source cells are defined), 1 locals F after L2L (nonempty target
 * cells), 2 target leaf offsets (8^L + 1), 3 target sort permutation (Nf),
 * 4 source leaf offsets, 5 source sort permutation (Ns).
 * Writes at most `count` doubles; *written gets the full size. */
int pbbfmm_debug_copy(pbbfmm_tree *tree, int what, int level, double *host, int64_t count,
                      int64_t *written);

/* Interpolation weights of the tree (ComputeWeights, src/H2_3D_Tree.cpp:715-826):
 * Tkz n*n, Kweights n^3, Cweights 2n^2, Ktable 343 (any pointer may be NULL). */
int pbbfmm_tree_get_weights(const pbbfmm_tree *tree, double *Tkz, double *Kweights,
                            double *Cweights, int *Ktable);

/* Leaf binning that allocates nothing.  No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc, e.g. a process whose device
 * memory is reserved up front by another allocator, or a deployment that
 * forbids allocation after start-up to keep its footprint fixed.
 *
 * For the N points at d_points (xyz AoS float64, device) it does the binning
 * step of the matvec: recentring on the points' bounding box (*d_center gets
 * the shift if non-NULL), the reference's leaf assignment on a tree of
 * `tree_level` levels and side `box`, and a stable sort by leaf: d_perm[i] is
 * the original index of the i-th point in leaf order (N ints), d_leaf_start
 * the first sorted position of every leaf (8^tree_level + 1 ints).  Same
 * results as the binning inside pbbfmm_compute_device.
 *
 * All scratch lives in one fixed device array inside this library (about
 * 18 MB, held on every GPU that loads the library until the process exits),
 * so N may not exceed PBBFMM_NOALLOC_MAX_POINTS (larger N returns
 * PBBFMM_ERR_ARG).  The first call on each device looks up the array's device
 * address; make that first call before any stream capture.  Calls share the
 * array: calls that overlap on the GPU (other streams, other host threads)
 * race on it.  Runs on the current device, asynchronously on `stream`. */
#define PBBFMM_NOALLOC_MAX_POINTS 524288
int pbbfmm_bin_points_noalloc(const double *d_points, int64_t N, double box, int tree_level,
                              int *d_perm, int *d_leaf_start, double *d_center, void *stream);

const char *pbbfmm_last_error(void);
const char *pbbfmm_version(void);

/* Number of CUDA kernel launches this library has issued in this process
 * (including the kernels of the CUB sort/select calls it makes). */
long long pbbfmm_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* PBBFMM3D_B200_H */
