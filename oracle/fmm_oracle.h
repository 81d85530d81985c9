/*
 * CPU restatement of the PBBFMM3D matvec (H2_3D_Compute<T>, include/compute.hpp)
 * used ONLY as a test oracle / CPU baseline checker.  Plain C, FP64.
 *
 * Parity status: pinned against the unmodified reference built from its own
 * sources (oracle/ref, outputs in oracle/_ref) and against the golden vectors
 * committed under tests/golden/ that the reference produced.
 *
 * Differences from the reference, all deliberate:
 *   - sources and targets are binned separately, so S != T is handled (the
 *     reference bins only targets and reuses that list for sources,
 *     include/compute.hpp:1191-1196); for S == T the results agree to rounding.
 *   - P2P evaluates K for every (target leaf, neighbour leaf) pair instead of
 *     the symmetric half (include/compute.hpp:680-690): same sums, different
 *     rounding order.
 *   - the tree is rebuilt implicitly on every call (the reference cannot be
 *     reused, include/compute.hpp:1176-1179).
 */
#ifndef PBBFMM3D_ORACLE_H
#define PBBFMM3D_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kernel ids shared with the product's C-ABI (include/pbbfmm3d_b200.h) */
enum {
  ORC_K_LAPLACIAN = 0,      /* 1/r            src/kernel_Types.cpp:7-28   */
  ORC_K_ONEOVERR2 = 1,      /* 1/r^2          src/kernel_Types.cpp:101-120 */
  ORC_K_ONEOVERR4 = 2,      /* 1/r^4          src/kernel_Types.cpp:34-53  */
  ORC_K_GAUSSIAN = 3,       /* exp(-r^2)      src/kernel_Types.cpp:56-74  */
  ORC_K_LOGARITHM = 4,      /* 0.5 log r^2    src/kernel_Types.cpp:77-99  */
  ORC_K_QUADRIC = 5,        /* 1 + r^2        src/kernel_Types.cpp:123-138 */
  ORC_K_INVQUADRIC = 6,     /* 1/(1 + r^2)    src/kernel_Types.cpp:140-155 */
  ORC_K_THINPLATE = 7,      /* 0.5 r^2 log r^2 src/kernel_Types.cpp:157-178 */
  ORC_K_EXPCOV = 8,         /* exp(-r/p0)     user kernel                 */
  ORC_K_GAUSSSIGMA = 9,     /* exp(-r^2/(2 p0^2)) user kernel             */
  ORC_K_ANISOEXP = 10       /* python/mykernel_python.hpp:10-18           */
};

typedef struct {
  int n;            /* interpolation order                              */
  int L;            /* tree_level                                        */
  double box;       /* box side length L of H2_3D_Tree                   */
  int cheb;         /* use_chebyshev                                     */
  int kernel;       /* ORC_K_*                                           */
  double kparam[4];
  double homogen;   /* as set by SetKernelProperty (before negation)     */
  int rf, rs;       /* SVD cutoffs (Chebyshev); ignored for uniform      */
  int nlev_ops;     /* operator levels: 1 (homogeneous) or L-1           */
  const double *K;  /* Cheb: nlev*316*rf*rs, Unif: nlev*316*(2n-1)^3     */
  const double *U;  /* Cheb: nlev*n^3*rf (col-major n^3 x rf)            */
  const double *VT; /* Cheb: nlev*rs*n^3 (col-major rs x n^3)            */
} orc_params;

double orc_kernel(int kernel, const double *kparam, const double t[3], const double s[3]);

/* ComputeWeights (src/H2_3D_Tree.cpp:715-826): Tkz n*n, Kweights n^3,
 * Cweights 2n^2, Ktable 343. */
void orc_compute_weights(int n, int cheb, double *Tkz, double *Kweights, double *Cweights,
                         int *Ktable);

/* Full matvec, output ACCUMULATED like the reference (compute.hpp:747).
 * tgt/src AoS xyz, w column-major Ns x C, out column-major Nf x C.
 * Returns 0 on success. */
int orc_matvec(const orc_params *p, const double *tgt, int64_t Nf, const double *src, int64_t Ns,
               const double *w, int C, double *out);

/* After orc_matvec: copy a dense per-level array of the last call.
 * what: 0 = moments S (8^lvl * C * n^3), 1 = local F after L2L (same size),
 * 2 = target leaf key per point (Nf int64 as double), 3 = source leaf key.
 * Returns number of doubles written (or needed if out == NULL). */
int64_t orc_dump(int what, int level, double *out);

/* Direct sum on rows [0, nrows) of the targets (include/test.hpp:19-34,
 * inf -> 0), out column-major nrows x C (overwritten). */
void orc_direct(int kernel, const double *kparam, const double *tgt, int64_t nrows,
                const double *src, int64_t Ns, const double *w, int C, double *out);

/* Direct sum on an explicit list of target rows. */
void orc_direct_rows(int kernel, const double *kparam, const double *tgt, const int64_t *rows,
                     int64_t nrows, const double *src, int64_t Ns, const double *w, int C,
                     double *out);

#ifdef __cplusplus
}
#endif
#endif
