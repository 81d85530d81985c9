// Host-side float64 operator precompute, restating the reference's
// buildFMMTree() (src/H2_3D_Tree.cpp).  Runs once per tree; the device path
// only consumes its outputs.
#include "precompute.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>

#include "../../include/pbbfmm3d_b200.h"

namespace pbbfmm {

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)>& body) {
  if (n <= 0) return;
  unsigned hw = std::thread::hardware_concurrency();
  int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw ? hw : 1, 64));
  nt = std::min(nt, n);
  if (nt == 1) {
    body(0, n);
    return;
  }
  std::vector<std::thread> th;
  int64_t chunk = (n + nt - 1) / nt;
  for (int64_t t = 0; t < nt; ++t) {
    int64_t a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back([&body, a, b]() { body(a, b); });
  }
  for (auto& x : th) x.join();
}

// ------------------------------------------------------------------ kernels

KernelSpec kernel_spec(int id, const double* param) {
  KernelSpec k;
  k.id = id;
  if (param)
    for (int i = 0; i < 4; ++i) k.param[i] = param[i];
  switch (id) {  // SetKernelProperty, src/kernel_Types.cpp
    case PBBFMM_KERNEL_LAPLACIAN: k.homogen = -1; break;
    case PBBFMM_KERNEL_ONEOVERR2: k.homogen = -2; break;
    case PBBFMM_KERNEL_ONEOVERR4: k.homogen = -4; break;
    default: k.homogen = 0; break;
  }
  k.symmetry = 1;
  return k;
}

std::string kernel_type_name(const KernelSpec& k) {
  char buf[40];
  switch (k.id) {
    case PBBFMM_KERNEL_LAPLACIAN: return "Laplacian";
    case PBBFMM_KERNEL_ONEOVERR2: return "OneOverR2";
    case PBBFMM_KERNEL_ONEOVERR4: return "OneOverR4";
    case PBBFMM_KERNEL_GAUSSIAN: return "Gaussian";
    case PBBFMM_KERNEL_LOGARITHM: return "Logarithm";
    case PBBFMM_KERNEL_QUADRIC: return "Quadric";
    case PBBFMM_KERNEL_INVQUADRIC: return "InverseQuadric";
    case PBBFMM_KERNEL_THINPLATESPLINE: return "ThinPlateSpline";
    case PBBFMM_KERNEL_EXPCOV: snprintf(buf, sizeof buf, "ExpCov%g", k.param[0]); return buf;
    case PBBFMM_KERNEL_GAUSSSIGMA: snprintf(buf, sizeof buf, "GaussS%g", k.param[0]); return buf;
    case PBBFMM_KERNEL_ANISOEXP: return "AnisoExp";
    case PBBFMM_KERNEL_USER: return k.user_type;
    default: return "Unknown";
  }
}

double eval_kernel_host(const KernelSpec& k, const double t[3], const double s[3]) {
  if (k.id == PBBFMM_KERNEL_USER) return k.user_eval(t, s, k.user_ctx);
  const double dx = s[0] - t[0], dy = s[1] - t[1], dz = s[2] - t[2];
  switch (k.id) {
    case PBBFMM_KERNEL_LAPLACIAN: return 1. / sqrt(dx * dx + dy * dy + dz * dz);
    case PBBFMM_KERNEL_ONEOVERR2: {
      double ri = 1. / sqrt(dx * dx + dy * dy + dz * dz);
      return ri * ri;
    }
    case PBBFMM_KERNEL_ONEOVERR4: {
      double ri = 1. / sqrt(dx * dx + dy * dy + dz * dz);
      return ri * ri * ri * ri;
    }
    case PBBFMM_KERNEL_GAUSSIAN: {
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      return exp(-r * r);
    }
    case PBBFMM_KERNEL_LOGARITHM: {
      double r2 = dx * dx + dy * dy + dz * dz;
      return r2 == 0 ? 0 : 0.5 * log(r2);
    }
    case PBBFMM_KERNEL_QUADRIC: return 1.0 + (dx * dx + dy * dy + dz * dz);
    case PBBFMM_KERNEL_INVQUADRIC: return 1.0 / (1.0 + (dx * dx + dy * dy + dz * dz));
    case PBBFMM_KERNEL_THINPLATESPLINE: {
      double r2 = dx * dx + dy * dy + dz * dz;
      return r2 == 0 ? 0 : 0.5 * r2 * log(r2);
    }
    case PBBFMM_KERNEL_EXPCOV: return exp(-sqrt(dx * dx + dy * dy + dz * dz) / k.param[0]);
    case PBBFMM_KERNEL_GAUSSSIGMA:
      return exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * k.param[0] * k.param[0]));
    case PBBFMM_KERNEL_ANISOEXP:
      return 0.75 * exp(-sqrt(dx * dx / 100. + dy * dy / 100. + dz * dz / 2.25));
    default: return NAN;
  }
}

bool is_homogeneous(double homogen) { return fabs(homogen) > 1e-1; }

// ------------------------------------------------------------------ weights

static double clenshaw(int n, double x, const double* Tk) {  // src/H2_3D_Tree.cpp:869-879
  double d0 = 0, d1 = 0, d2;
  for (int j = n - 1; j > 0; j--) {
    d2 = d0;
    d0 = 2.0 * x * d0 - d1 + Tk[j];
    d1 = d2;
  }
  return x * d0 - d1 + 0.5 * Tk[0];
}

static double lagrange(int n, double x, int m) {  // src/H2_3D_Tree.cpp:882-892
  double num = 1., den = 1.;
  for (int j = 0; j < n; j++)
    if (m != j) {
      num *= x - (1 - 2 * (double)j / (double)(n - 1));
      den *= -2 * ((double)m - (double)j) / (double)(n - 1);
    }
  return num / den;
}

Weights compute_weights(int n, int cheb) {
  Weights w;
  w.n = n;
  w.Tkz.assign(n * n, 0);
  w.Kweights.assign(n * n * n, 1.0);
  w.Cweights.assign(2 * n * n, 0);
  for (int i = 0; i < 343; i++) w.Ktable[i] = -1;
  int ncell = 0, ninteract = 0;
  for (int l1 = -3; l1 < 4; l1++)
    for (int l2 = -3; l2 < 4; l2++)
      for (int l3 = -3; l3 < 4; l3++) {
        if (abs(l1) > 1 || abs(l2) > 1 || abs(l3) > 1) w.Ktable[ncell] = ninteract++;
        ncell++;
      }
  std::vector<double> nodes(n);
  for (int m = 0; m < n; m++)  // GridPos1d(0, 1.0, ...), src/H2_3D_Tree.cpp:657-670
    nodes[m] = cheb ? cos(M_PI * ((double)m + 0.5) / (double)n) * 1.0
                    : 1 - 2 * (double)m / ((double)(n - 1)) * 1.0;
  for (int m = 0; m < n; m++) {  // ComputeTk, src/H2_3D_Tree.cpp:901-909
    std::vector<double> v(std::max(n, 2));
    v[0] = 1;
    v[1] = nodes[m];
    for (int k = 2; k < n; k++) v[k] = 2.0 * nodes[m] * v[k - 1] - v[k - 2];
    for (int k = 0; k < n; k++) w.Tkz[m * n + k] = v[k];
  }
  if (cheb) {  // src/H2_3D_Tree.cpp:759-772
    int c = 0;
    for (int l1 = 0; l1 < n; l1++) {
      double t1 = 1. / sqrt(1 - nodes[l1] * nodes[l1]);
      for (int l2 = 0; l2 < n; l2++) {
        double t2 = t1 / sqrt(1 - nodes[l2] * nodes[l2]);
        for (int l3 = 0; l3 < n; l3++) w.Kweights[c++] = t2 / sqrt(1 - nodes[l3] * nodes[l3]);
      }
    }
  }
  auto S = [&](int m, double x) {
    return cheb ? (2. / n) * clenshaw(n, x, &w.Tkz[m * n]) : lagrange(n, x, m);
  };
  for (int l1 = 0; l1 < n; l1++)  // src/H2_3D_Tree.cpp:774-819
    for (int l2 = 0; l2 < n; l2++) {
      w.Cweights[l1 * n + l2] = S(l1, nodes[l2] * .5 + (-0.5) * 1.0);
      w.Cweights[n * n + l1 * n + l2] = S(l1, nodes[l2] * .5 + 0.5 * 1.0);
    }
  return w;
}

// --------------------------------------------------------------------- SVD

// Householder QR of a tall column-major m x n matrix (in place); returns the
// n x n upper-triangular R (column-major).  Blocked: a panel of kQrPanel
// columns is factored column by column, then applied to the trailing
// columns at once in compact WY form, A2 -= V T^T V^T A2, with both products
// parallel over row blocks (the matrix is streamed twice per panel instead
// of once per column).
constexpr int kQrPanel = 32;
static std::vector<double> householder_r(std::vector<double>& A, int64_t m, int n) {
  std::vector<double> R((size_t)n * n, 0.0);
  std::vector<double> tau(n, 0.0);
  constexpr int64_t kRows = 2048;  // row block of the parallel products
  const int64_t nrb = (m + kRows - 1) / kRows;
  for (int j0 = 0; j0 < n; j0 += kQrPanel) {
    const int b = std::min(kQrPanel, n - j0);
    // panel: reflector j stored in column j, rows j..m-1 (v_j[j] kept in a[j])
    for (int j = j0; j < j0 + b; ++j) {
      double* a = &A[(size_t)j * m];
      double nrm2 = 0;
      for (int64_t i = j; i < m; ++i) nrm2 += a[i] * a[i];
      const double nrm = sqrt(nrm2);
      const double alpha = a[j] > 0 ? -nrm : nrm;
      const double v0 = a[j] - alpha;
      const double vv = nrm2 - a[j] * a[j] + v0 * v0;
      R[(size_t)j * n + j] = alpha;
      a[j] = v0;
      tau[j] = vv == 0 ? 0.0 : 2.0 / vv;
      if (tau[j] == 0.0) continue;
      const int nc = j0 + b - j - 1;  // remaining panel columns
      parallel_for(nc, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; ++c) {
          double* bc = &A[(size_t)(j + 1 + c) * m];
          double d = 0;
          for (int64_t i = j; i < m; ++i) d += a[i] * bc[i];
          d *= tau[j];
          for (int64_t i = j; i < m; ++i) bc[i] -= d * a[i];
        }
      });
    }
    for (int j = j0; j < j0 + b; ++j)
      for (int c = j + 1; c < j0 + b; ++c) R[(size_t)c * n + j] = A[(size_t)c * m + j];
    const int nt = n - j0 - b;  // trailing columns
    if (nt > 0) {
      // T (b x b, upper triangular): H_j0 ... H_j0+b-1 = I - V T V^T
      std::vector<double> T((size_t)b * b, 0.0), vtv((size_t)b * b, 0.0);
      parallel_for(b, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k)
          for (int l = 0; l < k; ++l) {
            // v_l^T v_k over rows >= j0 + k (v_k is zero above its diagonal)
            const double* vl = &A[(size_t)(j0 + l) * m];
            const double* vk = &A[(size_t)(j0 + k) * m];
            double d = 0;
            for (int64_t i = j0 + k; i < m; ++i) d += vl[i] * vk[i];
            vtv[(size_t)l * b + k] = d;
          }
      });
      for (int k = 0; k < b; ++k) {
        T[(size_t)k * b + k] = tau[j0 + k];
        for (int r = 0; r < k; ++r) {
          double acc = 0;
          for (int l = r; l < k; ++l) acc += T[(size_t)l * b + r] * vtv[(size_t)l * b + k];
          T[(size_t)k * b + r] = -tau[j0 + k] * acc;
        }
      }
      // W = V^T A2 (b x nt): partial sums per row block, then summed in order
      std::vector<double> Wp((size_t)nrb * b * nt, 0.0);
      parallel_for(nrb, [&](int64_t r0, int64_t r1) {
        for (int64_t rb = r0; rb < r1; ++rb) {
          const int64_t i0 = std::max<int64_t>(rb * kRows, j0), i1 = std::min(m, (rb + 1) * kRows);
          double* W = &Wp[(size_t)rb * b * nt];
          for (int c = 0; c < nt; ++c) {
            const double* ac = &A[(size_t)(j0 + b + c) * m];
            for (int k = 0; k < b; ++k) {
              const double* vk = &A[(size_t)(j0 + k) * m];
              const int64_t lo = std::max<int64_t>(i0, j0 + k);
              double d = 0;
              for (int64_t i = lo; i < i1; ++i) d += vk[i] * ac[i];
              W[(size_t)c * b + k] = d;
            }
          }
        }
      });
      std::vector<double> W((size_t)b * nt, 0.0), W2((size_t)b * nt, 0.0);
      for (int64_t rb = 0; rb < nrb; ++rb)
        for (size_t e = 0; e < W.size(); ++e) W[e] += Wp[(size_t)rb * b * nt + e];
      // W2 = T^T W
      for (int c = 0; c < nt; ++c)
        for (int k = 0; k < b; ++k) {
          double acc = 0;
          for (int r = 0; r <= k; ++r) acc += T[(size_t)k * b + r] * W[(size_t)c * b + r];
          W2[(size_t)c * b + k] = acc;
        }
      // A2 -= V W2, parallel over row blocks
      parallel_for(nrb, [&](int64_t r0, int64_t r1) {
        for (int64_t rb = r0; rb < r1; ++rb) {
          const int64_t i0 = std::max<int64_t>(rb * kRows, j0), i1 = std::min(m, (rb + 1) * kRows);
          for (int c = 0; c < nt; ++c) {
            double* ac = &A[(size_t)(j0 + b + c) * m];
            for (int k = 0; k < b; ++k) {
              const double* vk = &A[(size_t)(j0 + k) * m];
              const double w = W2[(size_t)c * b + k];
              const int64_t lo = std::max<int64_t>(i0, j0 + k);
              for (int64_t i = lo; i < i1; ++i) ac[i] -= vk[i] * w;
            }
          }
        }
      });
    }
    // the trailing columns' rows j0..j0+b-1 are final: the panel's part of R
    for (int j = j0; j < j0 + b; ++j)
      for (int c = j0 + b; c < n; ++c) R[(size_t)c * n + j] = A[(size_t)c * m + j];
  }
  return R;
}

// One-sided (Hestenes) Jacobi on a square column-major n x n matrix B:
// B W = U Sigma.  Returns sigma (descending) and W (columns permuted to match).
// Each sweep runs the n(n-1)/2 column pairs as rounds of disjoint pairs (a
// round-robin tournament over n rounded up to even; the extra player sits
// out), the pairs of a round spread over a fixed set of threads that meet at
// a barrier after every round; the order of the rounds and the rotations are
// the same on every run.
static void jacobi_svd(std::vector<double> B, int n, std::vector<double>* sigma,
                       std::vector<double>* W) {
  std::vector<double> V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  const int np = n + (n & 1);
  unsigned hw = std::thread::hardware_concurrency();
  const int nth = std::max(1, std::min<int>(hw ? (int)hw : 1, std::min(32, np / 2)));
  // sense-reversing spin barrier
  std::atomic<int> count(0), sense(0);
  auto barrier = [&](int& local) {
    local ^= 1;
    if (count.fetch_add(1) + 1 == nth) {
      count.store(0);
      sense.store(local);
    } else {
      while (sense.load() != local) std::this_thread::yield();
    }
  };
  std::atomic<int> rot_flag[2];
  rot_flag[0].store(0);
  rot_flag[1].store(0);
  auto work = [&](int tid) {
    int local = 0;
    std::vector<int> ring(np);
    for (int i = 0; i < np; ++i) ring[i] = i;
    for (int sweep = 0; sweep < 80; ++sweep) {
      std::atomic<int>& rot = rot_flag[sweep & 1];
      for (int round = 0; round < np - 1; ++round) {
        for (int i = tid; i < np / 2; i += nth) {
          int p = ring[i], q = ring[np - 1 - i];
          if (p > q) std::swap(p, q);
          if (q >= n) continue;
          double* bp = &B[(size_t)p * n];
          double* bq = &B[(size_t)q * n];
          double a = 0, b = 0, g = 0;
          for (int k = 0; k < n; ++k) {
            a += bp[k] * bp[k];
            b += bq[k] * bq[k];
            g += bp[k] * bq[k];
          }
          if (fabs(g) <= 1e-15 * sqrt(a * b) || g == 0) continue;
          rot.store(1, std::memory_order_relaxed);
          const double zeta = (b - a) / (2 * g);
          const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1 + zeta * zeta));
          const double c = 1 / sqrt(1 + t * t), s = c * t;
          for (int k = 0; k < n; ++k) {
            const double x = bp[k], y = bq[k];
            bp[k] = c * x - s * y;
            bq[k] = s * x + c * y;
          }
          double* vp = &V[(size_t)p * n];
          double* vq = &V[(size_t)q * n];
          for (int k = 0; k < n; ++k) {
            const double x = vp[k], y = vq[k];
            vp[k] = c * x - s * y;
            vq[k] = s * x + c * y;
          }
        }
        std::rotate(ring.begin() + 1, ring.end() - 1, ring.end());  // player 0 stays
        barrier(local);
      }
      const bool more = rot.load() != 0;
      barrier(local);  // every thread has read this sweep's flag
      if (tid == 0) rot_flag[(sweep + 1) & 1].store(0);
      barrier(local);
      if (!more) break;
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nth; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  std::vector<double> sv(n);
  for (int j = 0; j < n; ++j) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += B[(size_t)j * n + i] * B[(size_t)j * n + i];
    sv[j] = sqrt(s);
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return sv[x] > sv[y]; });
  sigma->resize(n);
  W->resize((size_t)n * n);
  for (int j = 0; j < n; ++j) {
    (*sigma)[j] = sv[ord[j]];
    memcpy(&(*W)[(size_t)j * n], &V[(size_t)ord[j] * n], sizeof(double) * n);
  }
}

void svd_tall_right(const double* A, int64_t m, int n, std::vector<double>* sigma,
                    std::vector<double>* V) {
  std::vector<double> work(A, A + (size_t)m * n);
  std::vector<double> R = householder_r(work, m, n);
  jacobi_svd(std::move(R), n, sigma, V);
}

// Number of singular values kept (src/H2_3D_Tree.cpp:406-421, 474-491).
static int svd_cutoff(const std::vector<double>& s, double eps) {
  int N = (int)s.size();
  double sumsqr = 0;
  for (int i = N - 1; i >= 0; --i) sumsqr += s[i] * s[i];
  double sum = 0, epsqr = sumsqr * eps * eps;
  int cut = N;
  for (int i = N - 1; i >= 0; --i) {
    sum += s[i] * s[i];
    if (sum < epsqr)
      --cut;
    else
      break;
  }
  return cut;
}

// ------------------------------------------------------------- Chebyshev M2L

// One level of ComputeKernelCheb (src/H2_3D_Tree.cpp:251-575).  On the first
// level the cutoffs are chosen; later levels reuse them.
static void cheb_level(const KernelSpec& k, int n, double eps, double boxLen,
                       const std::vector<double>& Kw, bool first, int* rf, int* rs,
                       double* Uout, double* VTout, double* Eout) {
  const int n3 = n * n * n;
  const size_t n6 = (size_t)n3 * n3;
  std::vector<double> nodes(n);
  for (int m = 0; m < n; m++) nodes[m] = cos(M_PI * ((double)m + 0.5) / (double)n) * 1.0;
  std::vector<double> tpos(3 * (size_t)n3);
  {
    int c = 0;
    for (int l1 = 0; l1 < n; l1++)
      for (int l2 = 0; l2 < n; l2++)
        for (int l3 = 0; l3 < n; l3++, c++) {
          tpos[3 * c + 0] = 0.5 * nodes[l1] * boxLen;
          tpos[3 * c + 1] = 0.5 * nodes[l2] * boxLen;
          tpos[3 * c + 2] = 0.5 * nodes[l3] * boxLen;
        }
  }
  // 316 weighted blocks; symmetric kernels evaluate half and mirror
  // (src/H2_3D_Tree.cpp:299-365)
  std::vector<double> K0(316 * n6);
  const int symm = k.symmetry;
  const int symmNum = 158 * (2 - abs(symm));
  std::vector<int> offs;
  for (int k1 = -3; k1 < 4; k1++)
    for (int k2 = -3; k2 < 4; k2++)
      for (int k3 = -3; k3 < 4; k3++)
        if (abs(k1) > 1 || abs(k2) > 1 || abs(k3) > 1) {
          offs.push_back(k1);
          offs.push_back(k2);
          offs.push_back(k3);
        }
  parallel_for(316, [&](int64_t c0, int64_t c1) {
    std::vector<double> spos(3 * (size_t)n3);
    for (int64_t c = c0; c < c1; ++c) {
      if (c >= symmNum) continue;
      int k1 = offs[3 * c], k2 = offs[3 * c + 1], k3 = offs[3 * c + 2];
      for (int l1 = 0; l1 < n; l1++)
        for (int l2 = 0; l2 < n; l2++)
          for (int l3 = 0; l3 < n; l3++) {
            int ind = l3 + l2 * n + l1 * n * n;
            spos[3 * ind + 0] = (k1 + 0.5 * nodes[l1]) * boxLen;
            spos[3 * ind + 1] = (k2 + 0.5 * nodes[l2]) * boxLen;
            spos[3 * ind + 2] = (k3 + 0.5 * nodes[l3]) * boxLen;
          }
      double* blk = &K0[(size_t)c * n6];
      for (int j = 0; j < n3; ++j)
        for (int i = 0; i < n3; ++i)
          blk[i + (size_t)n3 * j] =
              eval_kernel_host(k, &tpos[3 * i], &spos[3 * j]) / (Kw[j] * Kw[i]);
    }
  });
  if (symm) {
    for (int c = symmNum; c < 316; ++c)
      for (int col = 0; col < n3; col++)
        for (int row = 0; row < n3; row++)
          K0[(size_t)c * n6 + (size_t)row * n3 + col] =
              symm * K0[(size_t)(315 - c) * n6 + (size_t)col * n3 + row];
  }
  // fat SVD (left vectors of n3 x 316n3) = right vectors of its transpose
  std::vector<double> T((size_t)316 * n6);
  parallel_for(316, [&](int64_t c0, int64_t c1) {
    for (int64_t c = c0; c < c1; ++c)
      for (int i = 0; i < n3; ++i)
        for (int j = 0; j < n3; ++j)
          T[(size_t)i * 316 * n3 + (size_t)c * n3 + j] = K0[(size_t)c * n6 + i + (size_t)n3 * j];
  });
  std::vector<double> sig, Ufull;
  svd_tall_right(T.data(), (int64_t)316 * n3, n3, &sig, &Ufull);
  if (first) *rf = svd_cutoff(sig, eps);
  // thin SVD: vertical stack of the blocks
  parallel_for(316, [&](int64_t c0, int64_t c1) {
    for (int64_t c = c0; c < c1; ++c)
      for (int j = 0; j < n3; ++j)
        for (int i = 0; i < n3; ++i)
          T[(size_t)j * 316 * n3 + (size_t)c * n3 + i] = K0[(size_t)c * n6 + i + (size_t)n3 * j];
  });
  std::vector<double> sig2, Vfull;
  svd_tall_right(T.data(), (int64_t)316 * n3, n3, &sig2, &Vfull);
  if (first) *rs = svd_cutoff(sig2, eps);
  const int f = *rf, s = *rs;
  for (int r = 0; r < f; ++r)
    for (int i = 0; i < n3; ++i) Uout[i + (size_t)n3 * r] = Ufull[(size_t)r * n3 + i];
  for (int j = 0; j < n3; ++j)
    for (int r = 0; r < s; ++r) VTout[r + (size_t)s * j] = Vfull[(size_t)r * n3 + j];
  // E_c = U^T K_c V  (src/H2_3D_Tree.cpp:518-556)
  parallel_for(316, [&](int64_t c0, int64_t c1) {
    std::vector<double> KV((size_t)n3 * s);
    for (int64_t c = c0; c < c1; ++c) {
      const double* blk = &K0[(size_t)c * n6];
      // KV = K_c V, column by column as axpys over the contiguous columns of K_c
      for (int b = 0; b < s; ++b) {
        double* kv = &KV[(size_t)n3 * b];
        for (int i = 0; i < n3; ++i) kv[i] = 0;
        for (int j = 0; j < n3; ++j) {
          const double v = Vfull[(size_t)b * n3 + j];
          const double* col = blk + (size_t)n3 * j;
          for (int i = 0; i < n3; ++i) kv[i] += col[i] * v;
        }
      }
      double* E = Eout + (size_t)c * f * s;
      for (int b = 0; b < s; ++b)
        for (int a = 0; a < f; ++a) {
          double acc = 0;
          for (int i = 0; i < n3; ++i) acc += Uout[i + (size_t)n3 * a] * KV[i + (size_t)n3 * b];
          E[a + (size_t)f * b] = acc;
        }
    }
  });
}

// ---------------------------------------------------------- uniform M2L

// Kernel stencils of ComputeKernelUnif (src/H2_3D_Tree.cpp:585-631) for one
// level, before the FFT: 316 x (2n-1)^3.
static void unif_level(const KernelSpec& k, int n, double len, double* out) {
  const int m = 2 * n - 1, P = m * m * m;
  std::vector<double> nodes(n);
  for (int i = 0; i < n; i++)  // GridPos1d, src/H2_3D_Tree.cpp:668-669
    nodes[i] = 1 - 2 * (double)i / ((double)(n - 1)) * (len * (1 + 0.0));
  auto pos = [&](int idx, double* t, double* s) {  // GetPosition, :677-687
    if (idx < n) {
      *t = nodes[n - 1] / 2;
      *s = nodes[idx] / 2;
    } else {
      *t = nodes[2 * (n - 1) - idx] / 2;
      *s = nodes[n - 1] / 2;
    }
  };
  int c = 0;
  for (int k1 = -3; k1 < 4; k1++)
    for (int k2 = -3; k2 < 4; k2++)
      for (int k3 = -3; k3 < 4; k3++) {
        if (!(abs(k1) > 1 || abs(k2) > 1 || abs(k3) > 1)) continue;
        double* dst = out + (size_t)c * P;
        int cnt = 0;
        double t[3], s[3];
        for (int l1 = 0; l1 < m; l1++) {
          pos(l1, &t[0], &s[0]);
          s[0] += (double)k1 * len;
          for (int l2 = 0; l2 < m; l2++) {
            pos(l2, &t[1], &s[1]);
            s[1] += (double)k2 * len;
            for (int l3 = 0; l3 < m; l3++, cnt++) {
              pos(l3, &t[2], &s[2]);
              s[2] += (double)k3 * len;
              dst[cnt] = eval_kernel_host(k, t, s);
            }
          }
        }
        ++c;
      }
}

void stencils_to_halfcomplex(const std::vector<double>& st, int P, std::vector<double>* hc) {
  const size_t nb = st.size() / P;
  hc->assign(st.size(), 0.0);
  std::vector<double> cs(P), sn(P);
  for (int i = 0; i < P; ++i) {
    cs[i] = cos(2.0 * M_PI * i / P);
    sn[i] = sin(2.0 * M_PI * i / P);
  }
  parallel_for((int64_t)nb, [&](int64_t b0, int64_t b1) {
    for (int64_t b = b0; b < b1; ++b) {
      const double* x = &st[(size_t)b * P];
      double* y = &(*hc)[(size_t)b * P];
      for (int k = 0; k <= P / 2; ++k) {
        double re = 0, im = 0;
        int64_t e = 0;
        for (int j = 0; j < P; ++j) {
          re += x[j] * cs[e];
          im -= x[j] * sn[e];
          e += k;
          if (e >= P) e -= P;
        }
        y[k] = re;
        if (k > 0 && k < (P + 1) / 2) y[P - k] = im;
      }
    }
  });
}

void halfcomplex_to_stencils(const std::vector<double>& hc, int P, std::vector<double>* st) {
  const size_t nb = hc.size() / P;
  st->assign(hc.size(), 0.0);
  std::vector<double> cs(P), sn(P);
  for (int i = 0; i < P; ++i) {
    cs[i] = cos(2.0 * M_PI * i / P);
    sn[i] = sin(2.0 * M_PI * i / P);
  }
  parallel_for((int64_t)nb, [&](int64_t b0, int64_t b1) {
    for (int64_t b = b0; b < b1; ++b) {
      const double* y = &hc[(size_t)b * P];
      double* x = &(*st)[(size_t)b * P];
      for (int j = 0; j < P; ++j) {
        double acc = y[0];
        int64_t e = j;
        for (int k = 1; k < (P + 1) / 2; ++k) {
          acc += 2.0 * (y[k] * cs[e] - y[P - k] * sn[e]);
          e += j;
          if (e >= P) e -= P;
        }
        if (P % 2 == 0) acc += y[P / 2] * ((j % 2) ? -1.0 : 1.0);
        x[j] = acc / P;
      }
    }
  });
}

// --------------------------------------------------------------- top level

int precompute_operators(const KernelSpec& k, int n, int cheb, double box, int tree_level,
                         double eps, const Weights& w, Operators* ops, std::string* err) {
  ops->cheb = cheb;
  ops->n = n;
  const bool homog = is_homogeneous(k.homogen);
  ops->nlev = homog ? 1 : tree_level - 1;
  const int n3 = n * n * n;
  // homogeneous: unit cell; otherwise levels 2..L at box/4, box/8, ...
  // (StartPrecompute, src/H2_3D_Tree.cpp:147-160)
  std::vector<double> lens;
  if (homog) {
    lens.push_back(1.0);
  } else {
    double b = box / 4;
    for (int j = 2; j <= tree_level; j++) {
      lens.push_back(b);
      b /= 2;
    }
  }
  if (cheb) {
    int rf = n3, rs = n3;
    std::vector<std::vector<double>> U(ops->nlev), VT(ops->nlev), E(ops->nlev);
    for (int l = 0; l < ops->nlev; ++l) {
      std::vector<double> Ut((size_t)n3 * n3), VTt((size_t)n3 * n3),
          Et((size_t)316 * n3 * n3);
      cheb_level(k, n, eps, lens[l], w.Kweights, l == 0, &rf, &rs, Ut.data(), VTt.data(),
                 Et.data());
      Ut.resize((size_t)n3 * rf);
      VTt.resize((size_t)rs * n3);
      Et.resize((size_t)316 * rf * rs);
      U[l].swap(Ut);
      VT[l].swap(VTt);
      E[l].swap(Et);
    }
    ops->rf = rf;
    ops->rs = rs;
    ops->K.clear();
    ops->U.clear();
    ops->VT.clear();
    for (int l = 0; l < ops->nlev; ++l) {
      ops->K.insert(ops->K.end(), E[l].begin(), E[l].end());
      ops->U.insert(ops->U.end(), U[l].begin(), U[l].end());
      ops->VT.insert(ops->VT.end(), VT[l].begin(), VT[l].end());
    }
  } else {
    const int m = 2 * n - 1, P = m * m * m;
    ops->rf = ops->rs = n3;
    ops->stencil.assign((size_t)ops->nlev * 316 * P, 0.0);
    for (int l = 0; l < ops->nlev; ++l) unif_level(k, n, lens[l], &ops->stencil[(size_t)l * 316 * P]);
  }
  (void)err;
  return 0;
}

// ------------------------------------------------------------ cache files

static std::string cache_name(const std::string& dir, const KernelSpec& k, int n, int cheb,
                              char which) {
  char buf[64];
  snprintf(buf, sizeof buf, "%s%c%d.bin", cheb ? "Cheb" : "Unif", which, n);
  return dir + "/" + kernel_type_name(k) + buf;
}

static long file_size(FILE* f) {
  long cur = ftell(f);
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, cur, SEEK_SET);
  return sz;
}

int read_cache(const std::string& dir, const KernelSpec& k, int n, int cheb, double box,
               int tree_level, Operators* ops, std::string* err) {
  const bool homog = is_homogeneous(k.homogen);
  const int nlev = homog ? 1 : tree_level - 1;
  const int n3 = n * n * n;
  std::string kf = cache_name(dir, k, n, cheb, 'K');
  FILE* fK = fopen(kf.c_str(), "rb");
  if (!fK) return 1;
  double len_file = 0;
  int lvl_file = 0;
  bool ok = fread(&len_file, sizeof(double), 1, fK) == 1 && fread(&lvl_file, sizeof(int), 1, fK) == 1;
  // PrecomputeAvailable, src/H2_3D_Tree.cpp:115-122
  if (ok && !homog && (lvl_file != tree_level || fabs(len_file - box) >= 1e-6)) {
    fclose(fK);
    return 1;
  }
  if (!ok) {
    fclose(fK);
    *err = "truncated operator file " + kf;
    return -1;
  }
  ops->cheb = cheb;
  ops->n = n;
  ops->nlev = nlev;
  if (cheb) {
    FILE* fU = fopen(cache_name(dir, k, n, cheb, 'U').c_str(), "rb");
    FILE* fV = fopen(cache_name(dir, k, n, cheb, 'V').c_str(), "rb");
    if (!fU || !fV) {
      if (fU) fclose(fU);
      if (fV) fclose(fV);
      fclose(fK);
      return 1;
    }
    int rf = 0, rs = 0;
    bool good = fread(&rf, sizeof(int), 1, fU) == 1 && fread(&rs, sizeof(int), 1, fV) == 1 &&
                rf > 0 && rf <= n3 && rs > 0 && rs <= n3;
    size_t nU = (size_t)n3 * rf * nlev, nV = (size_t)n3 * rs * nlev,
           nK = (size_t)316 * rf * rs * nlev;
    good = good && file_size(fU) >= (long)(4 + 8 * nU) && file_size(fV) >= (long)(4 + 8 * nV) &&
           file_size(fK) >= (long)(12 + 8 * nK);
    if (good) {
      ops->U.resize(nU);
      ops->VT.resize(nV);
      ops->K.resize(nK);
      good = fread(ops->U.data(), 8, nU, fU) == nU && fread(ops->VT.data(), 8, nV, fV) == nV &&
             fread(ops->K.data(), 8, nK, fK) == nK;
    }
    fclose(fU);
    fclose(fV);
    fclose(fK);
    if (!good) {
      *err = "malformed Chebyshev operator files in " + dir;
      return -1;
    }
    ops->rf = rf;
    ops->rs = rs;
    return 0;
  }
  const int m = 2 * n - 1, P = m * m * m;
  size_t nK = (size_t)316 * P * nlev;
  bool good = file_size(fK) >= (long)(12 + 8 * nK);
  std::vector<double> hc(nK);
  if (good) good = fread(hc.data(), 8, nK, fK) == nK;
  fclose(fK);
  if (!good) {
    *err = "malformed uniform operator file " + kf;
    return -1;
  }
  ops->rf = ops->rs = n3;
  halfcomplex_to_stencils(hc, P, &ops->stencil);
  return 0;
}

int write_cache(const std::string& dir, const KernelSpec& k, int n, int cheb, double box,
                int tree_level, const Operators& ops, std::string* err) {
  std::string kf = cache_name(dir, k, n, cheb, 'K');
  FILE* fK = fopen(kf.c_str(), "wb");
  if (!fK) {
    *err = "cannot write " + kf;
    return -1;
  }
  fwrite(&box, sizeof(double), 1, fK);
  fwrite(&tree_level, sizeof(int), 1, fK);
  if (cheb) {
    fwrite(ops.K.data(), 8, ops.K.size(), fK);
    fclose(fK);
    FILE* fU = fopen(cache_name(dir, k, n, cheb, 'U').c_str(), "wb");
    FILE* fV = fopen(cache_name(dir, k, n, cheb, 'V').c_str(), "wb");
    if (!fU || !fV) {
      if (fU) fclose(fU);
      if (fV) fclose(fV);
      *err = "cannot write U/V operator files in " + dir;
      return -1;
    }
    fwrite(&ops.rf, sizeof(int), 1, fU);
    fwrite(ops.U.data(), 8, ops.U.size(), fU);
    fwrite(&ops.rs, sizeof(int), 1, fV);
    fwrite(ops.VT.data(), 8, ops.VT.size(), fV);
    fclose(fU);
    fclose(fV);
    return 0;
  }
  const int m = 2 * n - 1, P = m * m * m;
  std::vector<double> hc;
  stencils_to_halfcomplex(ops.stencil, P, &hc);
  fwrite(hc.data(), 8, hc.size(), fK);
  fclose(fK);
  return 0;
}

}  // namespace pbbfmm
