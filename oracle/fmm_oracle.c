/*
 * CPU restatement of the PBBFMM3D matvec (test oracle only; see fmm_oracle.h).
 * Every phase cites the reference lines it restates.  FP64 throughout; the
 * FFT of the uniform path reuses the oracle's FFTW-API shim (ref/shim).
 */
#include "fmm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ref/shim/fftw3.h"

/* ------------------------------------------------------------------ kernels */

double orc_kernel(int kernel, const double *kp, const double t[3], const double s[3]) {
  /* src/kernel_Types.cpp: diff = source - target in every kernel */
  const double dx = s[0] - t[0], dy = s[1] - t[1], dz = s[2] - t[2];
  switch (kernel) {
    case ORC_K_LAPLACIAN: {
      double rinv = 1. / sqrt(dx * dx + dy * dy + dz * dz);
      return rinv;
    }
    case ORC_K_ONEOVERR2: {
      double rinv = 1. / sqrt(dx * dx + dy * dy + dz * dz);
      return rinv * rinv;
    }
    case ORC_K_ONEOVERR4: {
      double rinv = 1. / sqrt(dx * dx + dy * dy + dz * dz);
      return rinv * rinv * rinv * rinv;
    }
    case ORC_K_GAUSSIAN: {
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      return exp(-r * r);
    }
    case ORC_K_LOGARITHM: {
      double r2 = dx * dx + dy * dy + dz * dz;
      return r2 == 0 ? 0 : 0.5 * log(r2);
    }
    case ORC_K_QUADRIC: {
      double r2 = dx * dx + dy * dy + dz * dz;
      return 1.0 + r2;
    }
    case ORC_K_INVQUADRIC: {
      double r2 = dx * dx + dy * dy + dz * dz;
      return 1.0 / (1.0 + r2);
    }
    case ORC_K_THINPLATE: {
      double r2 = dx * dx + dy * dy + dz * dz;
      return r2 == 0 ? 0 : 0.5 * r2 * log(r2);
    }
    case ORC_K_EXPCOV:
      return exp(-sqrt(dx * dx + dy * dy + dz * dz) / kp[0]);
    case ORC_K_GAUSSSIGMA:
      return exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * kp[0] * kp[0]));
    case ORC_K_ANISOEXP: {
      double r = sqrt(dx * dx / 100. + dy * dy / 100. + dz * dz / 2.25);
      return 0.75 * exp(-r);
    }
    default:
      return NAN;
  }
}

/* ------------------------------------------------------- interpolation basis */

/* ClenshawSum, src/H2_3D_Tree.cpp:869-879 */
static double clenshaw(int n, double x, const double *Tk) {
  double d0 = 0, d1 = 0, d2;
  for (int j = n - 1; j > 0; j--) {
    d2 = d0;
    d0 = 2.0 * x * d0 - d1 + Tk[j];
    d1 = d2;
  }
  return x * d0 - d1 + 0.5 * Tk[0];
}

/* LagrangeWeight, src/H2_3D_Tree.cpp:882-892 */
static double lagrange(int n, double x, int m) {
  double num = 1., denom = 1.;
  for (int j = 0; j < n; j++) {
    if (m != j) {
      num *= x - (1 - 2 * (double)j / (double)(n - 1));
      denom *= -2 * ((double)m - (double)j) / (double)(n - 1);
    }
  }
  return num / denom;
}

/* S_m(x) for one coordinate, ComputeSn src/H2_3D_Tree.cpp:830-866 */
static double sn1(int n, int cheb, const double *Tkz, int m, double x) {
  if (cheb) return (2. / n) * clenshaw(n, x, Tkz + m * n);
  return lagrange(n, x, m);
}

void orc_compute_weights(int n, int cheb, double *Tkz, double *Kweights, double *Cweights,
                         int *Ktable) {
  /* Ktable, src/H2_3D_Tree.cpp:731-747 */
  for (int i = 0; i < 343; i++) Ktable[i] = -1;
  int ncell = 0, ninteract = 0;
  for (int l1 = -3; l1 < 4; l1++)
    for (int l2 = -3; l2 < 4; l2++)
      for (int l3 = -3; l3 < 4; l3++) {
        if (abs(l1) > 1 || abs(l2) > 1 || abs(l3) > 1) Ktable[ncell] = ninteract++;
        ncell++;
      }
  /* GridPos1d(0, 1.0, ...), src/H2_3D_Tree.cpp:657-670 */
  double nodes[64];
  for (int m = 0; m < n; m++)
    nodes[m] = cheb ? cos(M_PI * ((double)m + 0.5) / (double)n) * 1.0
                    : 1 - 2 * (double)m / ((double)(n - 1)) * 1.0;
  /* Tkz via ComputeTk, src/H2_3D_Tree.cpp:750-757, 901-909 */
  for (int m = 0; m < n; m++) {
    double vec[64];
    vec[0] = 1;
    vec[1] = nodes[m];
    for (int k = 2; k < n; k++) vec[k] = 2.0 * nodes[m] * vec[k - 1] - vec[k - 2];
    for (int k = 0; k < n; k++) Tkz[m * n + k] = vec[k];
  }
  /* Kweights, src/H2_3D_Tree.cpp:759-772 (uniform: unused, set to 1) */
  int count = 0;
  for (int l1 = 0; l1 < n; l1++) {
    double tmp1 = 1. / sqrt(1 - nodes[l1] * nodes[l1]);
    for (int l2 = 0; l2 < n; l2++) {
      double tmp2 = tmp1 / sqrt(1 - nodes[l2] * nodes[l2]);
      for (int l3 = 0; l3 < n; l3++) {
        Kweights[count++] = cheb ? tmp2 / sqrt(1 - nodes[l3] * nodes[l3]) : 1.0;
      }
    }
  }
  /* Cweights: S_{l1} at child nodes, src/H2_3D_Tree.cpp:774-819 */
  for (int l1 = 0; l1 < n; l1++)
    for (int l2 = 0; l2 < n; l2++) {
      double zlo = nodes[l2] * .5 + (-0.5) * 1.0;
      double zhi = nodes[l2] * .5 + 0.5 * 1.0;
      Cweights[l1 * n + l2] = sn1(n, cheb, Tkz, l1, zlo);
      Cweights[n * n + l1 * n + l2] = sn1(n, cheb, Tkz, l1, zhi);
    }
}

/* ----------------------------------------------------------- last-call state */

static struct {
  int L, n, C;
  double **S;  /* per level, dense 8^l * C * n3 */
  double **F;
  double *tkey, *skey;
  int64_t Nf, Ns;
} g_last;

static void free_last(void) {
  if (g_last.S) {
    for (int l = 0; l <= g_last.L; l++) {
      free(g_last.S[l]);
      free(g_last.F[l]);
    }
  }
  free(g_last.S);
  free(g_last.F);
  free(g_last.tkey);
  free(g_last.skey);
  memset(&g_last, 0, sizeof g_last);
}

int64_t orc_dump(int what, int level, double *out) {
  if (what == 0 || what == 1) {
    if (!g_last.S || level < 0 || level > g_last.L) return -1;
    int64_t n3 = (int64_t)g_last.n * g_last.n * g_last.n;
    int64_t cnt = ((int64_t)1 << (3 * level)) * g_last.C * n3;
    double *src = what == 0 ? g_last.S[level] : g_last.F[level];
    if (!src) return -1;
    if (out) memcpy(out, src, sizeof(double) * (size_t)cnt);
    return cnt;
  }
  if (what == 2 || what == 3) {
    double *src = what == 2 ? g_last.tkey : g_last.skey;
    int64_t cnt = what == 2 ? g_last.Nf : g_last.Ns;
    if (!src) return -1;
    if (out) memcpy(out, src, sizeof(double) * (size_t)cnt);
    return cnt;
  }
  return -1;
}

/* ------------------------------------------------------------------- matvec */

typedef struct {
  int64_t *start; /* nleaf+1 */
  int64_t *perm;  /* sorted point index */
} bins_t;

/* DistributeFieldPoints descent, include/compute.hpp:1137-1188, with the
 * centres of BuildFMMHierarchy, src/H2_3D_Tree.cpp:925-971. */
static int64_t leaf_key(const double q[3], double box, int L) {
  double cx = 0, cy = 0, cz = 0, len = box;
  int64_t key = 0;
  for (int lev = 0; lev < L; lev++) {
    int bx = !(q[0] < cx), by = !(q[1] < cy), bz = !(q[2] < cz);
    key = key * 8 + (4 * bx + 2 * by + bz);
    double quarter = 0.25 * len;
    cx = bx ? cx + quarter : cx - quarter;
    cy = by ? cy + quarter : cy - quarter;
    cz = bz ? cz + quarter : cz - quarter;
    len = 0.5 * len;
  }
  return key;
}

static void bin_points(const double *pts, int64_t N, double box, int L, double *keys_out,
                       bins_t *b) {
  int64_t nleaf = (int64_t)1 << (3 * L);
  int64_t *key = (int64_t *)malloc(sizeof(int64_t) * (size_t)(N ? N : 1));
  b->start = (int64_t *)calloc((size_t)nleaf + 1, sizeof(int64_t));
  b->perm = (int64_t *)malloc(sizeof(int64_t) * (size_t)(N ? N : 1));
  for (int64_t i = 0; i < N; i++) {
    key[i] = leaf_key(pts + 3 * i, box, L);
    keys_out[i] = (double)key[i];
    b->start[key[i] + 1]++;
  }
  for (int64_t k = 0; k < nleaf; k++) b->start[k + 1] += b->start[k];
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)nleaf);
  memcpy(fill, b->start, sizeof(int64_t) * (size_t)nleaf);
  for (int64_t i = 0; i < N; i++) b->perm[fill[key[i]]++] = i; /* stable */
  free(fill);
  free(key);
}

static inline int64_t cell_count(const bins_t *b, int L, int l, int64_t m) {
  int64_t span = (int64_t)1 << (3 * (L - l));
  return b->start[(m + 1) * span] - b->start[m * span];
}

static inline void morton_decode(int64_t m, int l, int *x, int *y, int *z) {
  int xx = 0, yy = 0, zz = 0;
  for (int i = 0; i < l; i++) {
    int j = (int)((m >> (3 * i)) & 7);
    xx |= ((j >> 2) & 1) << i;
    yy |= ((j >> 1) & 1) << i;
    zz |= (j & 1) << i;
  }
  *x = xx;
  *y = yy;
  *z = zz;
}

static inline int64_t morton_encode(int x, int y, int z, int l) {
  int64_t m = 0;
  for (int i = l - 1; i >= 0; i--) {
    int j = (((x >> i) & 1) << 2) | (((y >> i) & 1) << 1) | ((z >> i) & 1);
    m = m * 8 + j;
  }
  return m;
}

/* M2M, include/compute.hpp:957-1034: SS = (Cx (x) Cy (x) Cz) Schild, applied
 * z, then y, then x, child bits choosing the Cweights half. */
static void m2m(int n, int C, int child, const double *Cw, const double *Sc, double *SS) {
  int n2 = n * n, n3 = n2 * n;
  int bx = (child >> 2) & 1, by = (child >> 1) & 1, bz = child & 1;
  const double *wz = Cw + (bz ? n2 : 0), *wy = Cw + (by ? n2 : 0), *wx = Cw + (bx ? n2 : 0);
  double *Sz = (double *)malloc(sizeof(double) * n3), *Sy = (double *)malloc(sizeof(double) * n3);
  for (int col = 0; col < C; col++) {
    const double *s = Sc + (size_t)col * n3;
    for (int l1 = 0; l1 < n2; l1++)
      for (int l3 = 0; l3 < n; l3++) {
        double acc = 0;
        for (int k = 0; k < n; k++) acc += s[l1 * n + k] * wz[l3 * n + k];
        Sz[l1 * n + l3] = acc;
      }
    for (int l1 = 0; l1 < n; l1++)
      for (int l2 = 0; l2 < n; l2++)
        for (int l3 = 0; l3 < n; l3++) {
          double acc = 0;
          for (int k = 0; k < n; k++) acc += Sz[l1 * n2 + k * n + l3] * wy[l2 * n + k];
          Sy[l1 * n2 + l2 * n + l3] = acc;
        }
    for (int l1 = 0; l1 < n; l1++)
      for (int l2 = 0; l2 < n; l2++)
        for (int l3 = 0; l3 < n; l3++) {
          double acc = 0;
          for (int k = 0; k < n; k++) acc += Sy[k * n2 + l2 * n + l3] * wx[l1 * n + k];
          SS[(size_t)col * n3 + l1 * n2 + l2 * n + l3] = acc;
        }
  }
  free(Sz);
  free(Sy);
}

/* L2L, include/compute.hpp:799-878: Fchild += (Cx^T (x) Cy^T (x) Cz^T) F, x first. */
static void l2l(int n, int C, int child, const double *Cw, const double *F, double *Fc) {
  int n2 = n * n, n3 = n2 * n;
  int bx = (child >> 2) & 1, by = (child >> 1) & 1, bz = child & 1;
  const double *wx = Cw + (bx ? n2 : 0), *wy = Cw + (by ? n2 : 0), *wz = Cw + (bz ? n2 : 0);
  double *Fx = (double *)malloc(sizeof(double) * n3), *Fy = (double *)malloc(sizeof(double) * n3);
  for (int col = 0; col < C; col++) {
    const double *f = F + (size_t)col * n3;
    for (int l1 = 0; l1 < n; l1++)
      for (int l2 = 0; l2 < n; l2++)
        for (int l3 = 0; l3 < n; l3++) {
          double acc = 0;
          for (int k = 0; k < n; k++) acc += f[k * n2 + l2 * n + l3] * wx[l1 + k * n];
          Fx[l1 * n2 + l2 * n + l3] = acc;
        }
    for (int l1 = 0; l1 < n; l1++)
      for (int l2 = 0; l2 < n; l2++)
        for (int l3 = 0; l3 < n; l3++) {
          double acc = 0;
          for (int k = 0; k < n; k++) acc += Fx[l1 * n2 + k * n + l3] * wy[l2 + k * n];
          Fy[l1 * n2 + l2 * n + l3] = acc;
        }
    for (int l1 = 0; l1 < n2; l1++)
      for (int l3 = 0; l3 < n; l3++) {
        double acc = 0;
        for (int k = 0; k < n; k++) acc += Fy[l1 * n + k] * wz[l3 + k * n];
        Fc[(size_t)col * n3 + l1 * n + l3] += acc;
      }
  }
  free(Fx);
  free(Fy);
}

/* FrequencyProduct, include/compute.hpp:930-943 (res += conj(A) * x, halfcomplex) */
static void freq_product(int N, const double *A, const double *x, double *res) {
  res[0] += A[0] * x[0];
  for (int i = 1; i < N; i++) {
    if (i < (N + 1) / 2)
      res[i] += A[i] * x[i] + A[N - i] * x[N - i];
    else
      res[i] += A[N - i] * x[i] - A[i] * x[N - i];
  }
  if (N % 2 == 0) res[N / 2] += A[N / 2] * x[N / 2];
}

int orc_matvec(const orc_params *p, const double *tgt, int64_t Nf, const double *src, int64_t Ns,
               const double *w, int C, double *out) {
  const int n = p->n, L = p->L, cheb = p->cheb;
  if (n < 2 || n > 32 || L < 2 || L > 9 || C < 1) return 1;
  const int n2 = n * n, n3 = n2 * n;
  const int homog = fabs(p->homogen) > 0.1; /* IsHomoKernel, src/H2_3D_Tree.cpp:134-136 */
  const double homogen_neg = -p->homogen;   /* buildFMMTree negates, src/H2_3D_Tree.cpp:45 */
  const int m = 2 * n - 1, P = m * m * m, halfSize = P / 2;
  const int rf = cheb ? p->rf : n3, rs = cheb ? p->rs : n3;

  double Tkz[32 * 32], *Kw = (double *)malloc(sizeof(double) * n3), Cw[2 * 32 * 32];
  int Ktable[343];
  orc_compute_weights(n, cheb, Tkz, Kw, Cw, Ktable);

  free_last();
  g_last.L = L;
  g_last.n = n;
  g_last.C = C;
  g_last.Nf = Nf;
  g_last.Ns = Ns;

  /* recentre on the target bounding box, include/compute.hpp:92-131 */
  double xmin[3] = {1e32, 1e32, 1e32}, xmax[3] = {-1e32, -1e32, -1e32};
  for (int64_t i = 0; i < Nf; i++)
    for (int d = 0; d < 3; d++) {
      double v = tgt[3 * i + d];
      xmin[d] = (v < xmin[d]) ? v : xmin[d];
      xmax[d] = (xmax[d] < v) ? v : xmax[d];
    }
  double ctr[3];
  for (int d = 0; d < 3; d++) ctr[d] = 0.5 * (xmin[d] + xmax[d]);
  double *T = (double *)malloc(sizeof(double) * 3 * (size_t)(Nf ? Nf : 1));
  double *S = (double *)malloc(sizeof(double) * 3 * (size_t)(Ns ? Ns : 1));
  for (int64_t i = 0; i < Nf; i++)
    for (int d = 0; d < 3; d++) T[3 * i + d] = tgt[3 * i + d] - ctr[d];
  for (int64_t i = 0; i < Ns; i++)
    for (int d = 0; d < 3; d++) S[3 * i + d] = src[3 * i + d] - ctr[d];

  bins_t bt, bs;
  g_last.tkey = (double *)malloc(sizeof(double) * (size_t)(Nf ? Nf : 1));
  g_last.skey = (double *)malloc(sizeof(double) * (size_t)(Ns ? Ns : 1));
  bin_points(T, Nf, p->box, L, g_last.tkey, &bt);
  bin_points(S, Ns, p->box, L, g_last.skey, &bs);

  /* cell centres and lengths per level, src/H2_3D_Tree.cpp:925-966 */
  double **cen = (double **)calloc((size_t)L + 1, sizeof(double *));
  double *len = (double *)malloc(sizeof(double) * (L + 1));
  len[0] = p->box;
  cen[0] = (double *)calloc(3, sizeof(double));
  for (int l = 0; l < L; l++) {
    int64_t nc = (int64_t)1 << (3 * l);
    cen[l + 1] = (double *)malloc(sizeof(double) * 3 * (size_t)nc * 8);
    double quarter = 0.25 * len[l];
    for (int64_t c = 0; c < nc; c++)
      for (int j = 0; j < 8; j++) {
        int b[3] = {(j >> 2) & 1, (j >> 1) & 1, j & 1};
        for (int d = 0; d < 3; d++)
          cen[l + 1][3 * (c * 8 + j) + d] =
              b[d] ? cen[l][3 * c + d] + quarter : cen[l][3 * c + d] - quarter;
      }
    len[l + 1] = 0.5 * len[l];
  }

  g_last.S = (double **)calloc((size_t)L + 1, sizeof(double *));
  g_last.F = (double **)calloc((size_t)L + 1, sizeof(double *));
  double **proxy = (double **)calloc((size_t)L + 1, sizeof(double *));
  for (int l = 2; l <= L; l++) {
    size_t nc = (size_t)1 << (3 * l);
    g_last.S[l] = (double *)calloc(nc * C * n3, sizeof(double));
    g_last.F[l] = (double *)calloc(nc * C * n3, sizeof(double));
    proxy[l] = (double *)calloc(nc * C * (size_t)(cheb ? rs : P), sizeof(double));
  }

  /* P2M at the leaves, include/compute.hpp:287-333 */
  {
    const double ihalfL = 2. / len[L];
    int64_t nleaf = (int64_t)1 << (3 * L);
    for (int64_t c = 0; c < nleaf; c++) {
      int64_t a = bs.start[c], e = bs.start[c + 1], cnt = e - a;
      if (cnt == 0) continue;
      double *Sn = (double *)malloc(sizeof(double) * 3 * n * (size_t)cnt);
      for (int64_t j = 0; j < cnt; j++) {
        int64_t k = bs.perm[a + j];
        double q[3];
        for (int d = 0; d < 3; d++) q[d] = ihalfL * (S[3 * k + d] - cen[L][3 * c + d]);
        for (int mm = 0; mm < n; mm++)
          for (int d = 0; d < 3; d++) Sn[(mm * cnt + j) * 3 + d] = sn1(n, cheb, Tkz, mm, q[d]);
      }
      double *Sl = g_last.S[L] + (size_t)c * C * n3;
      for (int col = 0; col < C; col++) {
        int l = 0;
        for (int l1 = 0; l1 < n; l1++)
          for (int l2 = 0; l2 < n; l2++)
            for (int l3 = 0; l3 < n; l3++) {
              double sum = 0;
              for (int64_t j = 0; j < cnt; j++) {
                int64_t k = bs.perm[a + j];
                sum += w[(size_t)col * Ns + k] * Sn[(l1 * cnt + j) * 3 + 0] *
                       Sn[(l2 * cnt + j) * 3 + 1] * Sn[(l3 * cnt + j) * 3 + 2];
              }
              Sl[(size_t)n3 * col + l] = sum;
              l++;
            }
      }
      free(Sn);
    }
  }

  /* M2M upward to level 2, include/compute.hpp:234-283 */
  {
    double *SS = (double *)malloc(sizeof(double) * (size_t)C * n3);
    for (int l = L - 1; l >= 2; l--) {
      int64_t nc = (int64_t)1 << (3 * l);
      for (int64_t c = 0; c < nc; c++) {
        if (cell_count(&bs, L, l, c) == 0) continue;
        double *Sp = g_last.S[l] + (size_t)c * C * n3;
        for (int i = 0; i < 8; i++) {
          int64_t ch = c * 8 + i;
          if (cell_count(&bs, L, l + 1, ch) == 0) continue;
          m2m(n, C, i, Cw, g_last.S[l + 1] + (size_t)ch * C * n3, SS);
          for (int t = 0; t < C * n3; t++) Sp[t] += SS[t];
        }
      }
    }
    free(SS);
  }

  /* M2L pre-transform, include/compute.hpp:337-396 */
  for (int l = 2; l <= L; l++) {
    int64_t nc = (int64_t)1 << (3 * l);
    int lvl = homog ? 0 : l - 2;
    for (int64_t c = 0; c < nc; c++) {
      if (cell_count(&bs, L, l, c) == 0) continue;
      const double *x = g_last.S[l] + (size_t)c * C * n3;
      if (cheb) {
        const double *VT = p->VT + (size_t)lvl * rs * n3;
        double *px = proxy[l] + (size_t)c * C * rs;
        for (int col = 0; col < C; col++)
          for (int r = 0; r < rs; r++) {
            double acc = 0;
            for (int t = 0; t < n3; t++) acc += VT[r + (size_t)rs * t] * (x[col * n3 + t] * Kw[t]);
            px[(size_t)col * rs + r] = acc;
          }
      } else {
        double *padx = (double *)calloc((size_t)P * C, sizeof(double));
        for (int col = 0; col < C; col++)
          for (int i = 0; i < n3; i++) {
            int l3 = i % n, l1 = i / n2, l2 = i / n % n;
            padx[(size_t)col * P + halfSize + l1 * m * m + l2 * m + l3] = x[col * n3 + i];
          }
        double *fre = proxy[l] + (size_t)c * C * P;
        for (int col = 0; col < C; col++) {
          fftw_plan pl = fftw_plan_r2r_1d(P, padx + (size_t)col * P, fre + (size_t)col * P,
                                          FFTW_R2HC, FFTW_ESTIMATE);
          fftw_execute(pl);
          fftw_destroy_plan(pl);
        }
        free(padx);
      }
    }
  }

  /* M2L, include/compute.hpp:402-549; list order from InteractionList,
   * include/compute.hpp:1062-1106 (parent-neighbour slot, then child j). */
  {
    const size_t matSize = cheb ? (size_t)rf : (size_t)P;
    double *acc = (double *)malloc(sizeof(double) * matSize * C);
    double *ff = (double *)malloc(sizeof(double) * matSize * C);
    double *res = (double *)malloc(sizeof(double) * (size_t)P * C);
    for (int l = 2; l <= L; l++) {
      int64_t nc = (int64_t)1 << (3 * l);
      int npar = 1 << (l - 1);
      int lvl = homog ? 0 : l - 2;
      double scale = pow(1.0 / len[l], homogen_neg);
      for (int64_t c = 0; c < nc; c++) {
        if (cell_count(&bt, L, l, c) == 0) continue;
        int ax, ay, az;
        morton_decode(c, l, &ax, &ay, &az);
        int qx = ax >> 1, qy = ay >> 1, qz = az >> 1;
        memset(acc, 0, sizeof(double) * matSize * C);
        for (int dx = -1; dx <= 1; dx++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dz = -1; dz <= 1; dz++) {
              int px = qx + dx, py = qy + dy, pz = qz + dz;
              if (px < 0 || py < 0 || pz < 0 || px >= npar || py >= npar || pz >= npar) continue;
              int64_t pm = morton_encode(px, py, pz, l - 1);
              if (cell_count(&bs, L, l - 1, pm) == 0) continue;
              for (int j = 0; j < 8; j++) {
                int64_t bm = pm * 8 + j;
                if (cell_count(&bs, L, l, bm) == 0) continue;
                int bx = 2 * px + ((j >> 2) & 1), by = 2 * py + ((j >> 1) & 1),
                    bz = 2 * pz + (j & 1);
                int ox = bx - ax, oy = by - ay, oz = bz - az;
                if (abs(ox) <= 1 && abs(oy) <= 1 && abs(oz) <= 1) continue; /* neighbour */
                int idx = Ktable[49 * (ox + 3) + 7 * (oy + 3) + (oz + 3)];
                if (cheb) {
                  const double *E =
                      p->K + (size_t)lvl * 316 * rf * rs + (size_t)idx * rf * rs;
                  const double *pb = proxy[l] + (size_t)bm * C * rs;
                  for (int col = 0; col < C; col++)
                    for (int r = 0; r < rf; r++) {
                      double s = 0;
                      for (int k = 0; k < rs; k++) s += E[r + (size_t)rf * k] * pb[col * rs + k];
                      ff[(size_t)col * rf + r] = s;
                    }
                  for (size_t t = 0; t < (size_t)rf * C; t++) acc[t] += ff[t];
                } else {
                  const double *A = p->K + (size_t)lvl * 316 * P + (size_t)idx * P;
                  memset(ff, 0, sizeof(double) * (size_t)P * C);
                  for (int col = 0; col < C; col++)
                    freq_product(P, A, proxy[l] + (size_t)bm * C * P + (size_t)col * P,
                                 ff + (size_t)col * P);
                  for (size_t t = 0; t < (size_t)P * C; t++) acc[t] += ff[t];
                }
              }
            }
        double *F = g_last.F[l] + (size_t)c * C * n3;
        if (cheb) {
          const double *U = p->U + (size_t)lvl * n3 * rf;
          for (int col = 0; col < C; col++)
            for (int i = 0; i < n3; i++) {
              double s = 0;
              for (int k = 0; k < rf; k++) s += U[i + (size_t)n3 * k] * acc[col * rf + k];
              F[col * n3 + i] += (scale * s) * Kw[i];
            }
        } else {
          for (int col = 0; col < C; col++) {
            fftw_plan pl = fftw_plan_r2r_1d(P, acc + (size_t)col * P, res + (size_t)col * P,
                                            FFTW_HC2R, FFTW_ESTIMATE);
            fftw_execute(pl);
            fftw_destroy_plan(pl);
          }
          for (int col = 0; col < C; col++)
            for (int i = 0; i < n3; i++) {
              int l3 = i % n, l1 = i / n2, l2 = i / n % n;
              double pf = res[(size_t)col * P + l1 * m * m + l2 * m + l3] / P;
              F[col * n3 + i] += scale * pf;
            }
        }
      }
    }
    free(acc);
    free(ff);
    free(res);
  }

  /* L2L downward, include/compute.hpp:552-587 (levels < 2 carry zeros) */
  for (int l = 3; l <= L; l++) {
    int64_t nc = (int64_t)1 << (3 * l);
    for (int64_t c = 0; c < nc; c++) {
      if (cell_count(&bt, L, l, c) == 0) continue;
      l2l(n, C, (int)(c & 7), Cw, g_last.F[l - 1] + (size_t)(c >> 3) * C * n3,
          g_last.F[l] + (size_t)c * C * n3);
    }
  }

  /* L2P + P2P + scatter, include/compute.hpp:591-749 */
  {
    const double ihalfL = 2. / len[L];
    int64_t nleaf = (int64_t)1 << (3 * L);
    int nside = 1 << L;
    double *phi = (double *)malloc(sizeof(double) * (size_t)C);
    for (int64_t c = 0; c < nleaf; c++) {
      int64_t a = bt.start[c], e = bt.start[c + 1];
      if (e == a) continue;
      int ax, ay, az;
      morton_decode(c, L, &ax, &ay, &az);
      const double *F = g_last.F[L] + (size_t)c * C * n3;
      for (int64_t ii = a; ii < e; ii++) {
        int64_t i = bt.perm[ii];
        double q[3], Sf[3][32];
        for (int d = 0; d < 3; d++) q[d] = ihalfL * (T[3 * i + d] - cen[L][3 * c + d]);
        for (int mm = 0; mm < n; mm++)
          for (int d = 0; d < 3; d++) Sf[d][mm] = sn1(n, cheb, Tkz, mm, q[d]);
        for (int col = 0; col < C; col++) {
          int l = 0;
          double sum = 0;
          for (int l1 = 0; l1 < n; l1++) {
            double tmp1 = Sf[0][l1];
            for (int l2 = 0; l2 < n; l2++) {
              double tmp2 = tmp1 * Sf[1][l2];
              for (int l3 = 0; l3 < n; l3++) {
                sum += F[col * n3 + l] * tmp2 * Sf[2][l3];
                l += 1;
              }
            }
          }
          phi[col] = sum;
        }
        /* P2P over the 27 neighbour leaves, index 9(x+1)+3(y+1)+(z+1) */
        for (int dx = -1; dx <= 1; dx++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dz = -1; dz <= 1; dz++) {
              int bx = ax + dx, by = ay + dy, bz = az + dz;
              if (bx < 0 || by < 0 || bz < 0 || bx >= nside || by >= nside || bz >= nside) continue;
              int64_t bm = morton_encode(bx, by, bz, L);
              for (int64_t jj = bs.start[bm]; jj < bs.start[bm + 1]; jj++) {
                int64_t j = bs.perm[jj];
                double kv = orc_kernel(p->kernel, p->kparam, tgt + 3 * i, src + 3 * j);
                if (isinf(kv)) kv = 0;
                for (int col = 0; col < C; col++) phi[col] += kv * w[(size_t)col * Ns + j];
              }
            }
        for (int col = 0; col < C; col++) out[(size_t)col * Nf + i] += phi[col];
      }
    }
    free(phi);
  }

  for (int l = 0; l <= L; l++) {
    free(cen[l]);
    free(proxy[l]);
  }
  free(cen);
  free(proxy);
  free(len);
  free(T);
  free(S);
  free(Kw);
  free(bt.start);
  free(bt.perm);
  free(bs.start);
  free(bs.perm);
  return 0;
}

/* ------------------------------------------------------------- direct sums */

void orc_direct_rows(int kernel, const double *kparam, const double *tgt, const int64_t *rows,
                     int64_t nrows, const double *src, int64_t Ns, const double *w, int C,
                     double *out) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t r = 0; r < nrows; r++) {
    int64_t i = rows ? rows[r] : r;
    for (int col = 0; col < C; col++) out[(size_t)col * nrows + r] = 0;
    for (int64_t j = 0; j < Ns; j++) {
      double v = orc_kernel(kernel, kparam, tgt + 3 * i, src + 3 * j);
      if (isinf(v)) v = 0;
      for (int col = 0; col < C; col++) out[(size_t)col * nrows + r] += v * w[(size_t)col * Ns + j];
    }
  }
}

void orc_direct(int kernel, const double *kparam, const double *tgt, int64_t nrows,
                const double *src, int64_t Ns, const double *w, int C, double *out) {
  orc_direct_rows(kernel, kparam, tgt, NULL, nrows, src, Ns, w, C, out);
}
