/*
 * Sequential, lock-free dgemm_ / ddot_ for the reference CPU oracle (test
 * infrastructure only).  The reference calls these from inside OpenMP
 * parallel regions (include/compute.hpp:394, 483/913, 502, 687-699, 831-1028);
 * a pthread BLAS serialises those calls, so the oracle supplies its own
 * reentrant column-major versions with the standard Fortran-77 LP64 ABI.
 * LAPACK's dgesvd_ (operator precompute only, src/H2_3D_Tree.cpp:400, 471)
 * still comes from a real LAPACK library at link time.
 */
#include <stddef.h>

static int is_t(const char *c) { return *c == 't' || *c == 'T' || *c == 'c' || *c == 'C'; }

void dgemm_(char *transa, char *transb, int *pm, int *pn, int *pk, double *palpha,
            double *A, int *plda, double *B, int *pldb, double *pbeta, double *C,
            int *pldc) {
  const int m = *pm, n = *pn, k = *pk, lda = *plda, ldb = *pldb, ldc = *pldc;
  const double alpha = *palpha, beta = *pbeta;
  const int ta = is_t(transa), tb = is_t(transb);
  for (int j = 0; j < n; ++j) {
    double *c = C + (size_t)j * ldc;
    if (beta == 0.0) {
      for (int i = 0; i < m; ++i) c[i] = 0.0;
    } else if (beta != 1.0) {
      for (int i = 0; i < m; ++i) c[i] *= beta;
    }
    if (alpha == 0.0) continue;
    if (!ta) {
      /* C(:,j) += alpha * sum_p A(:,p) * op(B)(p,j) */
      for (int p = 0; p < k; ++p) {
        double b = tb ? B[(size_t)p * ldb + j] : B[(size_t)j * ldb + p];
        double s = alpha * b;
        if (s == 0.0) continue;
        const double *a = A + (size_t)p * lda;
        for (int i = 0; i < m; ++i) c[i] += s * a[i];
      }
    } else {
      /* C(i,j) += alpha * sum_p A(p,i) * op(B)(p,j) */
      for (int i = 0; i < m; ++i) {
        const double *a = A + (size_t)i * lda;
        double acc = 0.0;
        if (!tb) {
          const double *b = B + (size_t)j * ldb;
          for (int p = 0; p < k; ++p) acc += a[p] * b[p];
        } else {
          for (int p = 0; p < k; ++p) acc += a[p] * B[(size_t)p * ldb + j];
        }
        c[i] += alpha * acc;
      }
    }
  }
}

double ddot_(int *pn, double *x, int *pincx, double *y, int *pincy) {
  const int n = *pn, incx = *pincx, incy = *pincy;
  double acc = 0.0;
  for (int i = 0; i < n; ++i) acc += x[(long)i * incx] * y[(long)i * incy];
  return acc;
}
