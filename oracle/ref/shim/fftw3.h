/*
 * FFTW3-API shim used only to compile the reference PBBFMM3D sources as a
 * CPU oracle (test infrastructure; never linked into the product).
 *
 * The reference calls exactly these entry points (include/compute.hpp:348-371,
 * 517-529; src/H2_3D_Tree.cpp:593-647): fftw_plan_r2r_1d with FFTW_R2HC /
 * FFTW_HC2R, fftw_execute, fftw_destroy_plan, fftw_alloc_real, fftw_free.
 * FFTW 3.3.8 itself is not vendored in the reference, so this restates FFTW's
 * published real-to-halfcomplex convention:
 *   R2HC: X_k = sum_j x_j exp(-2 pi i j k / n), stored as
 *         out[k] = Re X_k (0 <= k <= n/2), out[n-k] = Im X_k (0 < k < (n+1)/2)
 *   HC2R: the unnormalised inverse (sign +) of a halfcomplex input.
 * Any exact real DFT in this convention reproduces the reference to rounding.
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { FFTW_R2HC = 0, FFTW_HC2R = 1 } fftw_r2r_kind;
#define FFTW_ESTIMATE (1U << 6)

typedef struct oracle_fftw_plan_s *fftw_plan;

fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
double *fftw_alloc_real(size_t n);
void fftw_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
