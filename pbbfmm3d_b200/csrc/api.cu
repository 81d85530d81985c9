// C ABI (include/pbbfmm3d_b200.h): tree lifecycle, operator upload, the
// per-call workspace and the phase sequence of one matvec.
//
// Phase order follows H2_3D_Compute (include/compute.hpp:140-222):
// distribute (binning) -> upward (P2M, M2M) -> far field (M2L with its pre-
// and post-transforms) -> downward (L2L) -> near field (L2P, P2P, scatter).
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <string>
#include <thread>
#include <utility>

#include "fmm.cuh"

namespace pbbfmm {

static thread_local std::string g_err;
static std::atomic<long long> g_launches{0};

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

const char* const kSlotNames =
    "binning,p2m,m2m,m2l_pre,m2l,m2l_post,fft_fwd,m2l_mac,fft_inv,l2l,leaf,m2l_split";

int kt_begin(pbbfmm_tree* t, int slot, cudaStream_t st) {
  if (!t->timing) return PBBFMM_OK;
  if (t->kused + 2 > t->kev.size()) {
    for (int i = 0; i < 64; ++i) {
      cudaEvent_t e;
      PB_CUDA(cudaEventCreate(&e));
      t->kev.push_back(e);
    }
    t->kslot.resize(t->kev.size() / 2 + 1);
  }
  t->kslot[t->kused / 2] = slot;
  PB_CUDA(cudaEventRecord(t->kev[t->kused], st));
  t->kused += 1;
  return PBBFMM_OK;
}

int kt_end(pbbfmm_tree* t, cudaStream_t st) {
  if (!t->timing) return PBBFMM_OK;
  PB_CUDA(cudaEventRecord(t->kev[t->kused], st));
  t->kused += 1;
  return PBBFMM_OK;
}

void set_error(const std::string& msg) { g_err = msg; }

int cuda_status(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return PBBFMM_ERR_ALLOC;
  return PBBFMM_ERR_CUDA;
}

int grow(DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.p && b.cap >= bytes) return PBBFMM_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    set_error("device allocation of " + std::to_string(bytes) + " bytes failed: " +
              cudaGetErrorString(e));
    return PBBFMM_ERR_ALLOC;
  }
  b.cap = bytes;
  return PBBFMM_OK;
}

void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

static int upload(double** dst, const double* src, size_t count) {
  if (*dst) cudaFree(*dst);
  *dst = nullptr;
  if (count == 0) return PBBFMM_OK;
  PB_CUDA(cudaMalloc(dst, count * sizeof(double)));
  PB_CUDA(cudaMemcpy(*dst, src, count * sizeof(double), cudaMemcpyHostToDevice));
  return PBBFMM_OK;
}

// float32 copy (rounded once from the float64 tables) for the mixed path
static int upload_f32(float** dst, const double* src, size_t count) {
  if (*dst) cudaFree(*dst);
  *dst = nullptr;
  if (count == 0) return PBBFMM_OK;
  std::vector<float> h(src, src + count);
  PB_CUDA(cudaMalloc(dst, count * sizeof(float)));
  PB_CUDA(cudaMemcpy(*dst, h.data(), count * sizeof(float), cudaMemcpyHostToDevice));
  return PBBFMM_OK;
}

// float32 value rounded to TF32 (10 explicit mantissa bits), to nearest with
// ties away from zero -- the rounding of cvt.rna.tf32.f32.
static float tf32_round(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  u = (u + 0x1000u) & 0xffffe000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

static void free_tc_ops(TcOps* o) {
  void* b[] = {o->eth, o->etl, o->eh16, o->el16, o->eexp, o->vth, o->vtl, o->uh, o->ul};
  for (void* p : b)
    if (p) cudaFree(p);
  *o = TcOps{};
}

template <typename V>
static int upload_vec(V** dst, const std::vector<V>& h) {
  PB_CUDA(cudaMalloc(dst, h.size() * sizeof(V)));
  PB_CUDA(cudaMemcpy(*dst, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice));
  return PBBFMM_OK;
}

// Operands of the tensor-core Chebyshev M2L (both formats, see TcOps): for
// each level and operator o, E_o^T as NP rows (row f holds E_o[f][s], s < rs),
// zero padded,
//   TF32: hi = tf32(x), lo = tf32(x - hi) of x = float(E);
//   F16 : x = float(E) 2^e with e such that max |x| lies in [2^14, 2^15)
//         (e = 0 for a zero operator), hi = fp16(x), lo = fp16(x - hi).
// K: nlev x 316 column-major rf x rs blocks.  Leaves everything null when NP
// exceeds the tensor-core limit (the float path then uses the CUDA-core
// kernel).
static int upload_tc_split(const double* K, int nlev, int rf, int rs, TcOps* o) {
  free_tc_ops(o);
  const int NP = (rf + 15) / 16 * 16, KP = (rs + 31) / 32 * 32, KP16 = (rs + 63) / 64 * 64;
  o->np = NP;
  o->kp = KP;
  o->kp16 = KP16;
  if (NP > kTcMaxN) return PBBFMM_OK;
  const size_t total = (size_t)nlev * 316 * NP * KP, total16 = (size_t)nlev * 316 * NP * KP16;
  std::vector<float> hi(total, 0.f), lo(total, 0.f);
  std::vector<uint16_t> hi16(total16, 0), lo16(total16, 0);
  std::vector<int> ex((size_t)nlev * 316, 0);
  parallel_for((int64_t)nlev * 316, [&](int64_t b0, int64_t b1) {
    for (int64_t b = b0; b < b1; ++b) {
      const double* E = K + (size_t)b * rf * rs;
      float* h = hi.data() + (size_t)b * NP * KP;
      float* l = lo.data() + (size_t)b * NP * KP;
      float m = 0.f;
      for (int f = 0; f < rf; ++f)
        for (int s = 0; s < rs; ++s) {
          const float x = (float)E[f + (size_t)rf * s];
          const float xh = tf32_round(x);
          h[(size_t)f * KP + s] = xh;
          l[(size_t)f * KP + s] = tf32_round(x - xh);
          m = std::max(m, std::fabs(x));
        }
      int e = 0;
      if (m > 0.f) {
        int k2;
        std::frexp(m, &k2);
        e = 15 - k2;
      }
      ex[b] = e;
      uint16_t* h16 = hi16.data() + (size_t)b * NP * KP16;
      uint16_t* l16 = lo16.data() + (size_t)b * NP * KP16;
      for (int f = 0; f < rf; ++f)
        for (int s = 0; s < rs; ++s) {
          const float x = std::ldexp((float)E[f + (size_t)rf * s], e);
          const __half xh = __float2half_rn(x);
          const __half xl = __float2half_rn(x - __half2float(xh));
          memcpy(&h16[(size_t)f * KP16 + s], &xh, 2);
          memcpy(&l16[(size_t)f * KP16 + s], &xl, 2);
        }
    }
  });
  int rc;
  if ((rc = upload_vec(&o->eth, hi)) || (rc = upload_vec(&o->etl, lo)) ||
      (rc = upload_vec(&o->eh16, hi16)) || (rc = upload_vec(&o->el16, lo16)) ||
      (rc = upload_vec(&o->eexp, ex)))
    return rc;
  return PBBFMM_OK;
}

// Scaled F16 hi / lo rows of a level's matrix W (rows x cols, read through
// at(level, m, k)), [level][mp][kp] zero padded; exp[level] makes max |W|
// 2^exp lie in [2^14, 2^15).
template <typename At>
static void split_f16_rows(int nlev, int rows, int cols, int mp, int kp, At at,
                           std::vector<uint16_t>* hi, std::vector<uint16_t>* lo, int* exps) {
  hi->assign((size_t)nlev * mp * kp, 0);
  lo->assign((size_t)nlev * mp * kp, 0);
  for (int lv = 0; lv < nlev; ++lv) {
    float m = 0.f;
    for (int r = 0; r < rows; ++r)
      for (int k = 0; k < cols; ++k) m = std::max(m, std::fabs((float)at(lv, r, k)));
    int e = 0;
    if (m > 0.f) {
      int k2;
      std::frexp(m, &k2);
      e = 15 - k2;
    }
    exps[lv] = e;
    for (int r = 0; r < rows; ++r)
      for (int k = 0; k < cols; ++k) {
        const float x = std::ldexp((float)at(lv, r, k), e);
        const __half xh = __float2half_rn(x);
        const __half xl = __float2half_rn(x - __half2float(xh));
        const size_t i = ((size_t)lv * mp + r) * kp + k;
        memcpy(&(*hi)[i], &xh, 2);
        memcpy(&(*lo)[i], &xl, 2);
      }
  }
}

// The M2L pre / post transforms' matrices for the tensor cores (see TcOps):
// VT (column-major rs x n3 per level) and U (column-major n3 x rf per level).
static int upload_tc_uvt(const double* U, const double* VT, int nlev, int n3, int rf, int rs,
                         TcOps* o) {
  if (nlev > 32) return PBBFMM_OK;  // more levels than the exponent tables: CUDA cores
  // rows padded to 16, or to 32 above 256 (two MMAs of mp / 2, each a
  // multiple of 16)
  auto pad_rows = [](int r) { return r <= 256 ? (r + 15) / 16 * 16 : (r + 31) / 32 * 32; };
  o->vt_mp = pad_rows(rs);
  o->vt_kp = (n3 + 63) / 64 * 64;
  o->u_mp = pad_rows(n3);
  o->u_kp = (rf + 63) / 64 * 64;
  std::vector<uint16_t> h, l;
  int rc;
  if (o->vt_mp <= 512) {
    split_f16_rows(nlev, rs, n3, o->vt_mp, o->vt_kp,
                   [&](int lv, int m, int k) { return VT[(size_t)lv * rs * n3 + m + (size_t)rs * k]; },
                   &h, &l, o->vt_exp);
    if ((rc = upload_vec(&o->vth, h)) || (rc = upload_vec(&o->vtl, l))) return rc;
  }
  if (o->u_mp <= 512) {
    split_f16_rows(nlev, n3, rf, o->u_mp, o->u_kp,
                   [&](int lv, int m, int k) { return U[(size_t)lv * n3 * rf + m + (size_t)n3 * k]; },
                   &h, &l, o->u_exp);
    if ((rc = upload_vec(&o->uh, h)) || (rc = upload_vec(&o->ul, l))) return rc;
  }
  return PBBFMM_OK;
}

static int upload_tc_operators(pbbfmm_tree* t) {
  if (int rc = upload_tc_split(t->ops.K.data(), t->ops.nlev, t->ops.rf, t->ops.rs, &t->tc))
    return rc;
  if (int rc = upload_tc_uvt(t->ops.U.data(), t->ops.VT.data(), t->ops.nlev, t->n3, t->ops.rf,
                             t->ops.rs, &t->tc))
    return rc;
  return PBBFMM_OK;
}

// The timeout flag of the tensor-core kernels (mapped pinned memory), for
// every tree that computes: the Chebyshev and the uniform M2L both have
// tensor-core kernels that report through it.
static int ensure_tc_err_flag(pbbfmm_tree* t) {
  if (!t->h_tc_err) {
    PB_CUDA(cudaHostAlloc(&t->h_tc_err, sizeof(int), cudaHostAllocMapped));
    *t->h_tc_err = 0;
    PB_CUDA(cudaHostGetDevicePointer(&t->d_tc_err, t->h_tc_err, 0));
  }
  return PBBFMM_OK;
}

// conj(DFT3(stencil)) for k3 < n, stored [lvl][k][lex 343] complex; the 27
// inner (near-field) slots stay zero.  k = (k1*m + k2)*n + k3.
void unif_spectra(int n, const std::vector<double>& stencil, int nlev, std::vector<double>* op) {
  const int m = 2 * n - 1, P = m * m * m, nk = m * m * n;
  op->assign((size_t)nlev * nk * 343 * 2, 0.0);
  std::vector<int> lex;
  for (int a = -3; a < 4; ++a)
    for (int b = -3; b < 4; ++b)
      for (int c = -3; c < 4; ++c)
        if (abs(a) > 1 || abs(b) > 1 || abs(c) > 1) lex.push_back(49 * (a + 3) + 7 * (b + 3) + (c + 3));
  std::vector<double> cs(m), sn(m);
  for (int j = 0; j < m; ++j) {
    cs[j] = cos(2.0 * M_PI * j / m);
    sn[j] = sin(2.0 * M_PI * j / m);
  }
  parallel_for((int64_t)nlev * 316, [&](int64_t b0, int64_t b1) {
    std::vector<double> zr((size_t)m * m * n), zi((size_t)m * m * n), yr((size_t)m * m * n),
        yi((size_t)m * m * n);
    for (int64_t b = b0; b < b1; ++b) {
      const int lvl = (int)(b / 316), i = (int)(b % 316);
      const double* A = &stencil[((size_t)lvl * 316 + i) * P];
      // along d3 (real input), keep k3 < n
      for (int d1 = 0; d1 < m; ++d1)
        for (int d2 = 0; d2 < m; ++d2)
          for (int k3 = 0; k3 < n; ++k3) {
            double re = 0, im = 0;
            for (int d3 = 0; d3 < m; ++d3) {
              const int e = (k3 * d3) % m;
              const double v = A[(d1 * m + d2) * m + d3];
              re += v * cs[e];
              im -= v * sn[e];
            }
            zr[(d1 * m + d2) * n + k3] = re;
            zi[(d1 * m + d2) * n + k3] = im;
          }
      // along d2
      for (int d1 = 0; d1 < m; ++d1)
        for (int k2 = 0; k2 < m; ++k2)
          for (int k3 = 0; k3 < n; ++k3) {
            double re = 0, im = 0;
            for (int d2 = 0; d2 < m; ++d2) {
              const int e = (k2 * d2) % m;
              const double xr = zr[(d1 * m + d2) * n + k3], xi = zi[(d1 * m + d2) * n + k3];
              re += xr * cs[e] + xi * sn[e];
              im += xi * cs[e] - xr * sn[e];
            }
            yr[(d1 * m + k2) * n + k3] = re;
            yi[(d1 * m + k2) * n + k3] = im;
          }
      // along d1, conjugate, store
      for (int k1 = 0; k1 < m; ++k1)
        for (int k2 = 0; k2 < m; ++k2)
          for (int k3 = 0; k3 < n; ++k3) {
            double re = 0, im = 0;
            for (int d1 = 0; d1 < m; ++d1) {
              const int e = (k1 * d1) % m;
              const double xr = yr[(d1 * m + k2) * n + k3], xi = yi[(d1 * m + k2) * n + k3];
              re += xr * cs[e] + xi * sn[e];
              im += xi * cs[e] - xr * sn[e];
            }
            const size_t k = ((size_t)k1 * m + k2) * n + k3;
            double* dst = &(*op)[(((size_t)lvl * nk + k) * 343 + lex[i]) * 2];
            dst[0] = re;
            dst[1] = -im;
          }
    }
  });
}

// 189 interaction offsets per child type, in the order InteractionList
// visits them (parent-neighbour slot 9(x+1)+3(y+1)+(z+1), then child j;
// include/compute.hpp:1062-1106), with their operator index (Ktable).
static std::vector<int> m2l_offsets(const int* Ktable) {
  std::vector<int> offs;
  for (int t = 0; t < 8; ++t) {
    const int tx = (t >> 2) & 1, ty = (t >> 1) & 1, tz = t & 1;
    int cnt = 0;
    for (int px = -1; px <= 1; ++px)
      for (int py = -1; py <= 1; ++py)
        for (int pz = -1; pz <= 1; ++pz)
          for (int j = 0; j < 8; ++j) {
            const int ox = 2 * px + ((j >> 2) & 1) - tx, oy = 2 * py + ((j >> 1) & 1) - ty,
                      oz = 2 * pz + (j & 1) - tz;
            if (abs(ox) <= 1 && abs(oy) <= 1 && abs(oz) <= 1) continue;
            offs.push_back(ox);
            offs.push_back(oy);
            offs.push_back(oz);
            offs.push_back(Ktable[49 * (ox + 3) + 7 * (oy + 3) + (oz + 3)]);
            ++cnt;
          }
    (void)cnt;
  }
  return offs;
}

static void free_adjoint_ops(pbbfmm_tree* t) {
  double** d[] = {&t->adj.E, &t->adj.U, &t->adj.VT};
  for (double** b : d) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
  float** f[] = {&t->adj.fE, &t->adj.fU, &t->adj.fVT};
  for (float** b : f) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
  free_tc_ops(&t->adj.tc);
  t->adj_ready = false;
}

// Transposed Chebyshev operators for the adjoint pass (reference operator
// layout: E_p column-major rf x rs, U column-major n^3 x rf, VT column-major
// rs x n^3): U' = VT^T, VT' = U^T and E'_p = E_q^T where q is the operator of
// the opposite offset, since the pair (s <- t) has offset -(t <- s).
static int build_adjoint_ops(pbbfmm_tree* t) {
  free_adjoint_ops(t);
  const int rf = t->ops.rf, rs = t->ops.rs, nlev = t->ops.nlev, n3 = t->n3;
  std::vector<double> E((size_t)nlev * 316 * rf * rs), U((size_t)nlev * n3 * rs),
      VT((size_t)nlev * rf * n3);
  std::vector<int> neg(316, -1);
  for (int a = -3; a <= 3; ++a)
    for (int b = -3; b <= 3; ++b)
      for (int c = -3; c <= 3; ++c) {
        const int p = t->w.Ktable[49 * (a + 3) + 7 * (b + 3) + (c + 3)];
        const int q = t->w.Ktable[49 * (3 - a) + 7 * (3 - b) + (3 - c)];
        if (p >= 0) neg[p] = q;
      }
  for (int p = 0; p < 316; ++p)
    if (neg[p] < 0) {
      set_error("operator table has no opposite offset");
      return PBBFMM_ERR_STATE;
    }
  for (int lv = 0; lv < nlev; ++lv) {
    for (int p = 0; p < 316; ++p) {
      const double* Eq = t->ops.K.data() + ((size_t)lv * 316 + neg[p]) * rf * rs;
      double* Ep = E.data() + ((size_t)lv * 316 + p) * rf * rs;  // rs x rf column-major
      for (int i = 0; i < rs; ++i)
        for (int j = 0; j < rf; ++j) Ep[i + (size_t)rs * j] = Eq[j + (size_t)rf * i];
    }
    const double* Ul = t->ops.U.data() + (size_t)lv * n3 * rf;
    const double* Vl = t->ops.VT.data() + (size_t)lv * rs * n3;
    for (int l = 0; l < n3; ++l) {
      for (int s2 = 0; s2 < rs; ++s2) U[(size_t)lv * n3 * rs + l + (size_t)n3 * s2] = Vl[s2 + (size_t)rs * l];
      for (int f = 0; f < rf; ++f) VT[(size_t)lv * rf * n3 + f + (size_t)rf * l] = Ul[l + (size_t)n3 * f];
    }
  }
  int rc;
  if ((rc = upload(&t->adj.E, E.data(), E.size()))) return rc;
  if ((rc = upload(&t->adj.U, U.data(), U.size()))) return rc;
  if ((rc = upload(&t->adj.VT, VT.data(), VT.size()))) return rc;
  if ((rc = upload_f32(&t->adj.fE, E.data(), E.size()))) return rc;
  if ((rc = upload_f32(&t->adj.fU, U.data(), U.size()))) return rc;
  if ((rc = upload_f32(&t->adj.fVT, VT.data(), VT.size()))) return rc;
  if ((rc = upload_tc_split(E.data(), nlev, rs, rf, &t->adj.tc))) return rc;
  // adjoint: U' (n3 x rs) = VT^T and VT' (rf x n3) = U^T, so r_f' = rs, r_s' = rf
  if ((rc = upload_tc_uvt(U.data(), VT.data(), nlev, n3, rs, rf, &t->adj.tc))) return rc;
  t->adj.rf = rs;
  t->adj.rs = rf;
  t->adj_ready = true;
  return PBBFMM_OK;
}

// Exchange the forward and adjoint Chebyshev operator sets (an involution).
static void swap_adjoint_ops(pbbfmm_tree* t) {
  std::swap(t->d_E, t->adj.E);
  std::swap(t->d_U, t->adj.U);
  std::swap(t->d_VT, t->adj.VT);
  std::swap(t->f_E, t->adj.fE);
  std::swap(t->f_U, t->adj.fU);
  std::swap(t->f_VT, t->adj.fVT);
  std::swap(t->tc, t->adj.tc);
  std::swap(t->ops.rf, t->adj.rf);
  std::swap(t->ops.rs, t->adj.rs);
}

static int upload_operators(pbbfmm_tree* t) {
  if (t->device < 0) {
    t->ops_ready = true;
    return PBBFMM_OK;
  }
  PB_CUDA(cudaSetDevice(t->device));
  free_adjoint_ops(t);  // rebuilt from the new operators on the next adjoint
  int rc;
  if ((rc = ensure_tc_err_flag(t))) return rc;
  if (t->p.use_chebyshev) {
    if ((rc = upload(&t->d_E, t->ops.K.data(), t->ops.K.size()))) return rc;
    if ((rc = upload(&t->d_U, t->ops.U.data(), t->ops.U.size()))) return rc;
    if ((rc = upload(&t->d_VT, t->ops.VT.data(), t->ops.VT.size()))) return rc;
    if ((rc = upload_f32(&t->f_E, t->ops.K.data(), t->ops.K.size()))) return rc;
    if ((rc = upload_f32(&t->f_U, t->ops.U.data(), t->ops.U.size()))) return rc;
    if ((rc = upload_f32(&t->f_VT, t->ops.VT.data(), t->ops.VT.size()))) return rc;
    if ((rc = upload_tc_operators(t))) return rc;
  } else {
    std::vector<double> op;
    unif_spectra(t->n, t->ops.stencil, t->ops.nlev, &op);
    if ((rc = upload(&t->d_op, op.data(), op.size()))) return rc;
    if ((rc = upload_f32(&t->f_op, op.data(), op.size()))) return rc;
    std::vector<uint16_t> tiles;
    std::vector<int> bexp;
    unif_tc_tiles(t->n, op, t->ops.nlev, &tiles, &bexp);
    if (t->f_unif_tiles) cudaFree(t->f_unif_tiles);
    if (t->f_unif_bexp) cudaFree(t->f_unif_bexp);
    t->f_unif_tiles = nullptr;
    t->f_unif_bexp = nullptr;
    if ((rc = upload_vec(&t->f_unif_tiles, tiles))) return rc;
    if ((rc = upload_vec(&t->f_unif_bexp, bexp))) return rc;
  }
  t->ops_ready = true;
  return PBBFMM_OK;
}

static void free_tree_device(pbbfmm_tree* t) {
  double** bufs[] = {&t->d_Tkz, &t->d_Kw, &t->d_Cw, &t->d_E,  &t->d_U,
                     &t->d_VT,  &t->d_op, &t->d_twid, &t->d_kparam};
  for (double** b : bufs) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
  float** fbufs[] = {&t->f_Tkz, &t->f_Kw, &t->f_Cw, &t->f_E,    &t->f_U,
                     &t->f_VT,  &t->f_op, &t->f_twid};
  for (float** b : fbufs) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
  if (t->f_unif_tiles) cudaFree(t->f_unif_tiles);
  if (t->f_unif_bexp) cudaFree(t->f_unif_bexp);
  t->f_unif_tiles = nullptr;
  t->f_unif_bexp = nullptr;
  if (t->d_offs) cudaFree(t->d_offs);
  t->d_offs = nullptr;
  free_tc_ops(&t->tc);
  if (t->h_tc_err) cudaFreeHost(t->h_tc_err);
  t->h_tc_err = t->d_tc_err = nullptr;
  free_adjoint_ops(t);
  Workspace& ws = t->ws;
  DevBuf* all[] = {&ws.bbox_part, &ws.ctr,   &ws.key,     &ws.key_sorted, &ws.idx,
                   &ws.tperm,     &ws.sperm, &ws.tstart,  &ws.sstart,     &ws.tpos,
                   &ws.spos,      &ws.wsorted, &ws.cub_temp, &ws.lists,    &ws.dcounts,
                   &ws.S,         &ws.F,     &ws.proxy,   &ws.pf,         &ws.io_tgt,
                   &ws.io_src,    &ws.io_w,  &ws.io_out, &ws.halo, &ws.tc_proxy, &ws.leafpart,
                   &ws.occ,       &ws.amax};
  for (DevBuf* b : all) release(*b);
  if (ws.h_in) cudaFreeHost(ws.h_in);
  if (ws.h_out) cudaFreeHost(ws.h_out);
  ws.h_in = ws.h_out = nullptr;
  ws.h_in_cap = ws.h_out_cap = 0;
  if (ws.io_stream) cudaStreamDestroy(ws.io_stream);
  ws.io_stream = nullptr;
  for (int i = 0; i < 16; ++i)
    if (t->ev[i]) {
      cudaEventDestroy(t->ev[i]);
      t->ev[i] = nullptr;
    }
  for (cudaEvent_t e : t->kev) cudaEventDestroy(e);
  t->kev.clear();
  t->kused = 0;
}

// A tensor-core M2L whose mbarrier wait timed out sets the mapped flag and
// leaves that compute's output invalid; the next entry on the host reports
// it (once).  Visible here after any synchronisation with the compute.
static int take_tc_timeout(pbbfmm_tree* t) {
  if (t->h_tc_err && *(volatile int*)t->h_tc_err) {
    *(volatile int*)t->h_tc_err = 0;
    set_error("tensor-core M2L: a wait for the tensor pipe timed out; that compute's output is "
              "invalid");
    return PBBFMM_ERR_TIMEOUT;
  }
  return PBBFMM_OK;
}

// ---- host staging of the host-buffer entry point
constexpr size_t kStageChunk = 16u << 20;

static int grow_pinned(void** p, size_t* cap, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (*p && *cap >= bytes) return PBBFMM_OK;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  PB_CUDA(cudaHostAlloc(p, bytes, cudaHostAllocDefault));
  *cap = bytes;
  return PBBFMM_OK;
}

static int host_threads(size_t bytes) {
  const unsigned hw = std::thread::hardware_concurrency();
  const size_t by_size = bytes / (1u << 20) + 1;  // about 1 MB per thread at least
  size_t n = hw ? (hw < 16 ? hw : 16) : 4;
  return (int)(n < by_size ? n : by_size);
}

// memcpy split over host threads (pageable source into pinned staging)
static void host_copy_mt(void* dst, const void* src, size_t bytes) {
  const int nt = host_threads(bytes);
  if (nt <= 1) {
    memcpy(dst, src, bytes);
    return;
  }
  std::vector<std::thread> th;
  const size_t per = (bytes + nt - 1) / nt;
  for (int i = 0; i < nt; ++i) {
    const size_t a = i * per, b = a + per < bytes ? a + per : bytes;
    if (a >= b) break;
    th.emplace_back([=] {
      memcpy(static_cast<unsigned char*>(dst) + a, static_cast<const unsigned char*>(src) + a, b - a);
    });
  }
  for (auto& x : th) x.join();
}

// dst[i] += src[i], split over host threads
static void host_add_mt(double* dst, const double* src, size_t n) {
  const int nt = host_threads(n * sizeof(double));
  auto add = [](double* d, const double* s, size_t a, size_t b) {
    for (size_t i = a; i < b; ++i) d[i] += s[i];
  };
  if (nt <= 1) {
    add(dst, src, 0, n);
    return;
  }
  std::vector<std::thread> th;
  const size_t per = (n + nt - 1) / nt;
  for (int i = 0; i < nt; ++i) {
    const size_t a = i * per, b = a + per < n ? a + per : n;
    if (a >= b) break;
    th.emplace_back(add, dst, src, a, b);
  }
  for (auto& x : th) x.join();
}

static const char* kPhaseNames = "binning,upward,far_field,downward,near_field";
constexpr int kNumPhases = 5;

static int compute_chunk(pbbfmm_tree* t, const double* d_tgt, int64_t Nf, const double* d_src,
                         int64_t Ns, const double* d_w, int C, double* d_out, int precision,
                         cudaStream_t st) {
  const int L = t->p.tree_level, n3 = t->n3;
  Workspace& ws = t->ws;
  int rc;
  if (t->timing) PB_CUDA(cudaEventRecord(t->ev[0], st));
  t->last_Nf = Nf;
  t->last_Ns = Ns;
  t->last_C = C;
  t->cur_prec = precision;
  if ((rc = kt_begin(t, KS_BINNING, st))) return rc;
  if ((rc = run_binning(t, d_tgt, Nf, d_src, Ns, d_w, C, st))) return rc;
  if ((rc = kt_end(t, st))) return rc;
  if (t->timing) PB_CUDA(cudaEventRecord(t->ev[1], st));
  const int64_t perS = (int64_t)C * n3;
  // coefficient arrays in the precision of the pass (float32 on the mixed path)
  const size_t es = precision == PBBFMM_PREC_FP64 ? sizeof(double) : sizeof(float);
  if ((rc = grow(ws.S, es * level_total(L, perS)))) return rc;
  if ((rc = grow(ws.F, es * level_total(L, perS)))) return rc;
  if (t->p.use_chebyshev) {
    if ((rc = grow(ws.proxy, es * level_total(L, (int64_t)C * t->ops.rs)))) return rc;
    if ((rc = grow(ws.pf, es * level_total(L, (int64_t)C * t->ops.rf)))) return rc;
  } else {
    if ((rc = grow(ws.proxy, 2 * es * level_total(L, (int64_t)C * t->nk)))) return rc;
    if ((rc = grow(ws.pf, 2 * es * level_total(L, (int64_t)C * t->nk)))) return rc;
    // halo tables: at most 8^(L-2) parent blocks x (region + target) entries
    if ((rc = grow(ws.halo, sizeof(int) * 576 * cells_at(L - 2)))) return rc;
  }
  if ((rc = run_upward(t, C, st))) return rc;
  if (t->timing) PB_CUDA(cudaEventRecord(t->ev[2], st));
  if (t->p.use_chebyshev)
    rc = run_m2l_cheb(t, C, st);
  else
    rc = run_m2l_unif(t, C, st);
  if (rc) return rc;
  if (t->timing) PB_CUDA(cudaEventRecord(t->ev[3], st));
  if ((rc = run_downward(t, C, st))) return rc;
  if (t->timing) PB_CUDA(cudaEventRecord(t->ev[4], st));
  if ((rc = run_leaves(t, Nf, Ns, C, d_out, st))) return rc;
  if (t->timing) PB_CUDA(cudaEventRecord(t->ev[5], st));
  t->have_last = true;
  return PBBFMM_OK;
}

}  // namespace pbbfmm

using namespace pbbfmm;

extern "C" {

const char* pbbfmm_last_error(void) { return g_err.c_str(); }
const char* pbbfmm_version(void) { return "pbbfmm3d_b200 0.1 (sm_100a)"; }

long long pbbfmm_launch_count(void) { return g_launches.load(); }

static int create_tree(const pbbfmm_tree_params* params, const pbbfmm_user_kernel* uk,
                       int device, pbbfmm_tree** out) {
  if (!params || !out) {
    set_error("null argument");
    return PBBFMM_ERR_ARG;
  }
  *out = nullptr;
  pbbfmm_tree_params p = *params;
  if (uk) {
    p.kernel = PBBFMM_KERNEL_USER;
    for (double& x : p.kernel_param) x = 0.0;
  }
  if (!(p.L > 0) || !std::isfinite(p.L)) {
    set_error("box length L must be positive");
    return PBBFMM_ERR_ARG;
  }
  if (p.tree_level < 2 || p.tree_level > kMaxLevel) {
    set_error("tree_level must be in [2, 10]");
    return PBBFMM_ERR_ARG;
  }
  if (p.interpolation_order < 2 || p.interpolation_order > kMaxOrder) {
    set_error("interpolation_order must be in [2, 10]");
    return PBBFMM_ERR_ARG;
  }
  if (!uk && (p.kernel < 0 || p.kernel >= PBBFMM_KERNEL_COUNT)) {
    set_error("unknown kernel id");
    return PBBFMM_ERR_ARG;
  }
  if (uk && (!uk->evaluate || !uk->launch_leaf || !uk->kernel_type || !uk->kernel_type[0] ||
             uk->symmetry < -1 || uk->symmetry > 1 || !std::isfinite(uk->homogen))) {
    set_error("user kernel needs evaluate, launch_leaf, a kernel_type name, symmetry in "
              "{-1, 0, 1} and a finite homogen");
    return PBBFMM_ERR_ARG;
  }
  if (p.use_chebyshev && !(p.epsilon > 0)) {
    set_error("epsilon must be positive");
    return PBBFMM_ERR_ARG;
  }
  if ((p.kernel == PBBFMM_KERNEL_EXPCOV || p.kernel == PBBFMM_KERNEL_GAUSSSIGMA) &&
      !(p.kernel_param[0] > 0)) {
    set_error("kernel_param[0] (length scale) must be positive");
    return PBBFMM_ERR_ARG;
  }
  if (device >= 0) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      set_error("no CUDA device available");
      return PBBFMM_ERR_CUDA;
    }
    if (device >= ndev) {
      set_error("device index out of range");
      return PBBFMM_ERR_ARG;
    }
    PB_CUDA(cudaSetDevice(device));
  }
  pbbfmm_tree* t = new pbbfmm_tree();
  t->p = p;
  t->device = device;
  t->kspec = kernel_spec(p.kernel, p.kernel_param);
  if (uk) {  // SetKernelProperty of the user's subclass
    t->user = *uk;
    t->kspec.homogen = uk->homogen;
    t->kspec.symmetry = uk->symmetry;
    t->kspec.user_type = uk->kernel_type;
    t->kspec.user_eval = uk->evaluate;
    t->kspec.user_ctx = uk->ctx;
    t->user.kernel_type = nullptr;  // the copy in kspec.user_type is the one used
  }
  t->n = p.interpolation_order;
  t->n3 = t->n * t->n * t->n;
  t->m = 2 * t->n - 1;
  t->nk = t->m * t->m * t->n;
  t->homog = is_homogeneous(t->kspec.homogen);
  t->homogen_neg = -t->kspec.homogen;  // src/H2_3D_Tree.cpp:45
  t->w = compute_weights(t->n, p.use_chebyshev);
  t->weights_ready = true;
  if (device < 0) {  // host-only tree: precompute and operator access, no compute
    *out = t;
    return PBBFMM_OK;
  }
  int rc;
  if ((rc = upload(&t->d_Tkz, t->w.Tkz.data(), t->w.Tkz.size())) ||
      (rc = upload(&t->d_Kw, t->w.Kweights.data(), t->w.Kweights.size())) ||
      (rc = upload(&t->d_Cw, t->w.Cweights.data(), t->w.Cweights.size())) ||
      (rc = upload(&t->d_kparam, t->kspec.param, 4)) ||
      (rc = upload_f32(&t->f_Tkz, t->w.Tkz.data(), t->w.Tkz.size())) ||
      (rc = upload_f32(&t->f_Kw, t->w.Kweights.data(), t->w.Kweights.size())) ||
      (rc = upload_f32(&t->f_Cw, t->w.Cweights.data(), t->w.Cweights.size()))) {
    free_tree_device(t);
    delete t;
    return rc;
  }
  {
    std::vector<double> tw(2 * t->m);
    for (int j = 0; j < t->m; ++j) {
      tw[j] = cos(2.0 * M_PI * j / t->m);
      tw[t->m + j] = sin(2.0 * M_PI * j / t->m);
    }
    if ((rc = upload(&t->d_twid, tw.data(), tw.size())) ||
        (rc = upload_f32(&t->f_twid, tw.data(), tw.size()))) {
      free_tree_device(t);
      delete t;
      return rc;
    }
    std::vector<int> offs = m2l_offsets(t->w.Ktable);
    cudaError_t e = cudaMalloc(&t->d_offs, offs.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(t->d_offs, offs.data(), offs.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      rc = cuda_status(e, "upload offsets");
      free_tree_device(t);
      delete t;
      return rc;
    }
  }
  *out = t;
  return PBBFMM_OK;
}

int pbbfmm_tree_create(const pbbfmm_tree_params* params, int device, pbbfmm_tree** out) {
  return create_tree(params, nullptr, device, out);
}

int pbbfmm_tree_create_user(const pbbfmm_tree_params* params, const pbbfmm_user_kernel* kernel,
                            int device, pbbfmm_tree** out) {
  if (!kernel) {
    set_error("null user kernel");
    return PBBFMM_ERR_ARG;
  }
  return create_tree(params, kernel, device, out);
}

int pbbfmm_tree_build(pbbfmm_tree* t, const char* cache_dir) {
  if (!t) {
    set_error("null tree");
    return PBBFMM_ERR_ARG;
  }
  std::string err;
  const pbbfmm_tree_params& p = t->p;
  bool have = false;
  if (cache_dir) {
    int r = read_cache(cache_dir, t->kspec, t->n, p.use_chebyshev, p.L, p.tree_level, &t->ops, &err);
    if (r < 0) {
      set_error(err);
      return PBBFMM_ERR_IO;
    }
    have = (r == 0);
  }
  if (!have) {
    if (precompute_operators(t->kspec, t->n, p.use_chebyshev, p.L, p.tree_level, p.epsilon, t->w,
                             &t->ops, &err)) {
      set_error(err);
      return PBBFMM_ERR_ARG;
    }
    if (cache_dir && write_cache(cache_dir, t->kspec, t->n, p.use_chebyshev, p.L, p.tree_level,
                                 t->ops, &err)) {
      set_error(err);
      return PBBFMM_ERR_IO;
    }
  }
  return upload_operators(t);
}

int pbbfmm_tree_set_operators(pbbfmm_tree* t, int rf, int rs, int nlev, const double* K,
                              const double* U, const double* VT) {
  if (!t || !K) {
    set_error("null argument");
    return PBBFMM_ERR_ARG;
  }
  const int n3 = t->n3;
  const int want = t->homog ? 1 : t->p.tree_level - 1;
  if (nlev != want) {
    set_error("nlev must be " + std::to_string(want) + " for this kernel and tree_level");
    return PBBFMM_ERR_ARG;
  }
  t->ops.cheb = t->p.use_chebyshev;
  t->ops.n = t->n;
  t->ops.nlev = nlev;
  if (t->p.use_chebyshev) {
    if (!U || !VT || rf < 1 || rf > n3 || rs < 1 || rs > n3) {
      set_error("Chebyshev operators need U, VT and 1 <= rf, rs <= n^3");
      return PBBFMM_ERR_ARG;
    }
    t->ops.rf = rf;
    t->ops.rs = rs;
    t->ops.K.assign(K, K + (size_t)nlev * 316 * rf * rs);
    t->ops.U.assign(U, U + (size_t)nlev * n3 * rf);
    t->ops.VT.assign(VT, VT + (size_t)nlev * rs * n3);
  } else {
    const int P = t->m * t->m * t->m;
    t->ops.rf = t->ops.rs = n3;
    std::vector<double> hc(K, K + (size_t)nlev * 316 * P);
    halfcomplex_to_stencils(hc, P, &t->ops.stencil);
  }
  return upload_operators(t);
}

int pbbfmm_tree_get_operators(const pbbfmm_tree* t, int* rf, int* rs, int* nlev, double* K,
                              double* U, double* VT) {
  if (!t || !t->ops_ready) {
    set_error("tree has no operators (call pbbfmm_tree_build)");
    return PBBFMM_ERR_STATE;
  }
  if (rf) *rf = t->ops.rf;
  if (rs) *rs = t->ops.rs;
  if (nlev) *nlev = t->ops.nlev;
  if (t->p.use_chebyshev) {
    if (K) memcpy(K, t->ops.K.data(), t->ops.K.size() * sizeof(double));
    if (U) memcpy(U, t->ops.U.data(), t->ops.U.size() * sizeof(double));
    if (VT) memcpy(VT, t->ops.VT.data(), t->ops.VT.size() * sizeof(double));
  } else if (K) {
    std::vector<double> hc;
    stencils_to_halfcomplex(t->ops.stencil, t->m * t->m * t->m, &hc);
    memcpy(K, hc.data(), hc.size() * sizeof(double));
  }
  return PBBFMM_OK;
}

int pbbfmm_tree_get_weights(const pbbfmm_tree* t, double* Tkz, double* Kweights, double* Cweights,
                            int* Ktable) {
  if (!t) {
    set_error("null tree");
    return PBBFMM_ERR_ARG;
  }
  if (Tkz) memcpy(Tkz, t->w.Tkz.data(), t->w.Tkz.size() * sizeof(double));
  if (Kweights) memcpy(Kweights, t->w.Kweights.data(), t->w.Kweights.size() * sizeof(double));
  if (Cweights) memcpy(Cweights, t->w.Cweights.data(), t->w.Cweights.size() * sizeof(double));
  if (Ktable) memcpy(Ktable, t->w.Ktable, sizeof(int) * 343);
  return PBBFMM_OK;
}

int pbbfmm_tree_destroy(pbbfmm_tree* t) {
  if (!t) return PBBFMM_OK;
  if (t->device >= 0) {
    cudaSetDevice(t->device);
    free_tree_device(t);
  }
  delete t;
  return PBBFMM_OK;
}

int pbbfmm_set_precision(pbbfmm_tree* t, int precision) {
  if (!t || (precision != PBBFMM_PREC_FP64 && precision != PBBFMM_PREC_MIXED)) {
    set_error("bad precision mode");
    return PBBFMM_ERR_ARG;
  }
  t->precision = precision;
  return PBBFMM_OK;
}

int pbbfmm_set_timing(pbbfmm_tree* t, int enable) {
  if (!t || t->device < 0) return PBBFMM_ERR_ARG;
  PB_CUDA(cudaSetDevice(t->device));
  if (enable && !t->ev[0])
    for (int i = 0; i <= kNumPhases; ++i) PB_CUDA(cudaEventCreate(&t->ev[i]));
  t->timing = enable != 0;
  return PBBFMM_OK;
}

int pbbfmm_reset_kernel_times(pbbfmm_tree* t) {
  if (!t) return PBBFMM_ERR_ARG;
  t->kused = 0;
  return PBBFMM_OK;
}

int pbbfmm_get_kernel_times(pbbfmm_tree* t, float* ms, int* launches, int max_slots, int* nslots,
                            const char** names) {
  if (!t || t->device < 0) return PBBFMM_ERR_ARG;
  if (names) *names = kSlotNames;
  if (nslots) *nslots = KS_COUNT;
  for (int i = 0; i < max_slots && i < KS_COUNT; ++i) {
    if (ms) ms[i] = 0;
    if (launches) launches[i] = 0;
  }
  PB_CUDA(cudaSetDevice(t->device));
  for (size_t k = 0; k + 1 < t->kused; k += 2) {
    float v = 0;
    PB_CUDA(cudaEventSynchronize(t->kev[k + 1]));
    PB_CUDA(cudaEventElapsedTime(&v, t->kev[k], t->kev[k + 1]));
    const int slot = t->kslot[k / 2];
    if (slot < max_slots) {
      if (ms) ms[slot] += v;
      if (launches) launches[slot] += 1;
    }
  }
  return PBBFMM_OK;
}

int pbbfmm_get_phase_times(const pbbfmm_tree* t, float* ms, int max_phases, int* nphases,
                           const char** names) {
  if (!t) return PBBFMM_ERR_ARG;
  if (names) *names = kPhaseNames;
  if (nphases) *nphases = kNumPhases;
  if (!t->timing || !t->have_last) {
    set_error("timing not enabled or no compute yet");
    return PBBFMM_ERR_STATE;
  }
  for (int i = 0; i < kNumPhases && i < max_phases; ++i) {
    PB_CUDA(cudaEventSynchronize(t->ev[i + 1]));
    PB_CUDA(cudaEventElapsedTime(&ms[i], t->ev[i], t->ev[i + 1]));
  }
  return PBBFMM_OK;
}

int pbbfmm_compute_device(pbbfmm_tree* t, const double* d_target, int64_t Nf,
                          const double* d_source, int64_t Ns, const double* d_weight, int nCols,
                          double* d_output, int precision, void* stream) {
  if (!t) {
    set_error("null tree");
    return PBBFMM_ERR_ARG;
  }
  if (!t->ops_ready) {
    set_error("tree operators missing: call pbbfmm_tree_build first");
    return PBBFMM_ERR_STATE;
  }
  if (t->device < 0) {
    set_error("host-only tree (device -1) cannot compute");
    return PBBFMM_ERR_STATE;
  }
  if (Nf < 0 || Ns < 0 || nCols < 1 || Nf > INT32_MAX || Ns > INT32_MAX) {
    set_error("bad sizes (0 <= Nf, Ns < 2^31, nCols >= 1)");
    return PBBFMM_ERR_ARG;
  }
  if ((Nf > 0 && (!d_target || !d_output)) || (Ns > 0 && (!d_source || !d_weight))) {
    set_error("null data pointer");
    return PBBFMM_ERR_ARG;
  }
  if (precision != PBBFMM_PREC_FP64 && precision != PBBFMM_PREC_MIXED) {
    set_error("bad precision mode");
    return PBBFMM_ERR_ARG;
  }
  if (int rc = take_tc_timeout(t)) return rc;
  if (Nf == 0) return PBBFMM_OK;
  PB_CUDA(cudaSetDevice(t->device));
  cudaStream_t st = (cudaStream_t)stream;
  // Right-hand sides run in blocks of at most 64 columns (the Chebyshev M2L
  // tile width; it also bounds the per-CTA shared memory of P2M); weights
  // and outputs are column-major, so a block is a contiguous slice of each.
  const int cmax = 64;
  for (int c0 = 0; c0 < nCols; c0 += cmax) {
    const int cc = nCols - c0 < cmax ? nCols - c0 : cmax;
    int rc = compute_chunk(t, d_target, Nf, d_source, Ns, d_weight + (int64_t)c0 * Ns, cc,
                           d_output + (int64_t)c0 * Nf, precision, st);
    if (rc) return rc;
  }
  return PBBFMM_OK;
}

// Restores the forward configuration of a tree after an adjoint or gradient
// pass, on every exit path.
struct PassGuard {
  pbbfmm_tree* t;
  bool swapped = false;
  ~PassGuard() {
    if (swapped) swap_adjoint_ops(t);
    t->bbox_pts = nullptr;
    t->bbox_n = 0;
    t->gl = pbbfmm_tree::GradLeaf{};
  }
};

int pbbfmm_compute_adjoint_device(pbbfmm_tree* t, const double* d_target, int64_t Nf,
                                  const double* d_source, int64_t Ns, const double* d_weight,
                                  const double* d_g, int nCols, double* d_grad_weight,
                                  double* d_grad_source, double* d_grad_target, int precision,
                                  void* stream) {
  if (!t) {
    set_error("null tree");
    return PBBFMM_ERR_ARG;
  }
  if (!t->ops_ready || t->device < 0) {
    set_error("tree cannot compute: host-only or operators missing");
    return PBBFMM_ERR_STATE;
  }
  if (Nf < 0 || Ns < 0 || nCols < 1 || Nf > INT32_MAX || Ns > INT32_MAX) {
    set_error("bad sizes (0 <= Nf, Ns < 2^31, nCols >= 1)");
    return PBBFMM_ERR_ARG;
  }
  if (precision != PBBFMM_PREC_FP64 && precision != PBBFMM_PREC_MIXED) {
    set_error("bad precision mode");
    return PBBFMM_ERR_ARG;
  }
  if (Nf > 0 && Ns > 0 &&
      (!d_target || !d_source || !d_g || ((d_grad_source || d_grad_target) && !d_weight))) {
    set_error("null data pointer (gradients with respect to positions need the weights)");
    return PBBFMM_ERR_ARG;
  }
  if (int rc = take_tc_timeout(t)) return rc;
  if (Nf == 0 || Ns == 0) return PBBFMM_OK;
  PB_CUDA(cudaSetDevice(t->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int cmax = 64;
  if (d_grad_weight || d_grad_source) {
    // Transposed pass on the forward tree: the sources become targets, the
    // targets sources carrying g, the box stays the forward targets' one.
    PassGuard guard{t};
    if (t->p.use_chebyshev) {
      if (!t->adj_ready)
        if (int rc = build_adjoint_ops(t)) return rc;
      swap_adjoint_ops(t);
      guard.swapped = true;
    }
    t->bbox_pts = d_target;
    t->bbox_n = Nf;
    for (int c0 = 0; c0 < nCols; c0 += cmax) {
      const int cc = nCols - c0 < cmax ? nCols - c0 : cmax;
      t->gl = pbbfmm_tree::GradLeaf{};
      if (d_grad_source) {
        t->gl.on = true;
        t->gl.contract = d_weight + (int64_t)c0 * Ns;
        t->gl.grad_out = d_grad_source;
        t->gl.values = d_grad_weight != nullptr;
      }
      int rc = compute_chunk(t, d_source, Ns, d_target, Nf, d_g + (int64_t)c0 * Nf, cc,
                             d_grad_weight ? d_grad_weight + (int64_t)c0 * Ns : nullptr,
                             precision, st);
      if (rc) return rc;
    }
  }
  if (d_grad_target) {
    // forward pass whose leaf phase evaluates the potentials' gradients at the
    // targets, contracted with g
    PassGuard guard{t};
    for (int c0 = 0; c0 < nCols; c0 += cmax) {
      const int cc = nCols - c0 < cmax ? nCols - c0 : cmax;
      t->gl = pbbfmm_tree::GradLeaf{};
      t->gl.on = true;
      t->gl.contract = d_g + (int64_t)c0 * Nf;
      t->gl.grad_out = d_grad_target;
      t->gl.values = false;
      int rc = compute_chunk(t, d_target, Nf, d_source, Ns, d_weight + (int64_t)c0 * Ns, cc,
                             nullptr, precision, st);
      if (rc) return rc;
    }
  }
  return PBBFMM_OK;
}

int pbbfmm_compute(pbbfmm_tree* t, const double* target, int64_t Nf, const double* source,
                   int64_t Ns, const double* weight, int nCols, double* output) {
  if (!t) {
    set_error("null tree");
    return PBBFMM_ERR_ARG;
  }
  if (Nf < 0 || Ns < 0 || nCols < 1) {
    set_error("bad sizes");
    return PBBFMM_ERR_ARG;
  }
  if ((Nf > 0 && (!target || !output)) || (Ns > 0 && (!source || !weight))) {
    set_error("null data pointer");
    return PBBFMM_ERR_ARG;
  }
  if (Nf == 0) return PBBFMM_OK;
  if (t->device < 0 || !t->ops_ready) {
    set_error("tree cannot compute: host-only or operators missing");
    return PBBFMM_ERR_STATE;
  }
  PB_CUDA(cudaSetDevice(t->device));
  Workspace& ws = t->ws;
  int rc;
  if (!ws.io_stream) PB_CUDA(cudaStreamCreateWithFlags(&ws.io_stream, cudaStreamNonBlocking));
  cudaStream_t st = ws.io_stream;
  // Every exit waits for the stream: no copy queued here may still read the
  // pinned staging (which the next call overwrites) or write the caller's
  // result after this call returns.  On success the stream is already idle.
  struct StreamDrain {
    cudaStream_t s;
    ~StreamDrain() { cudaStreamSynchronize(s); }
  } drain{st};
  const bool same = (source == target && Ns == Nf);
  const size_t bt = sizeof(double) * 3 * Nf, bs = same ? 0 : sizeof(double) * 3 * Ns;
  const size_t bw = sizeof(double) * (size_t)Ns * nCols, bo = sizeof(double) * (size_t)Nf * nCols;
  if ((rc = grow(ws.io_tgt, bt))) return rc;
  if (!same && (rc = grow(ws.io_src, bs ? bs : 16))) return rc;
  if ((rc = grow(ws.io_w, bw ? bw : 16))) return rc;
  if ((rc = grow(ws.io_out, bo))) return rc;
  if ((rc = grow_pinned(&ws.h_in, &ws.h_in_cap, bt + bs + bw))) return rc;
  if ((rc = grow_pinned(&ws.h_out, &ws.h_out_cap, bo))) return rc;
  double* dt = ws.io_tgt.as<double>();
  double* ds = same ? dt : ws.io_src.as<double>();
  // inputs: multithreaded copy into pinned staging, chunk by chunk, each
  // chunk's DMA overlapping the next chunk's host copy
  unsigned char* hin = static_cast<unsigned char*>(ws.h_in);
  struct Seg {
    const void* src;
    void* dev;
    size_t bytes;
  } segs[3] = {{target, dt, bt}, {source, ds, bs}, {weight, ws.io_w.p, bw}};
  size_t off = 0;
  for (const Seg& g : segs)
    for (size_t c = 0; c < g.bytes; c += kStageChunk) {
      const size_t n = g.bytes - c < kStageChunk ? g.bytes - c : kStageChunk;
      host_copy_mt(hin + off, static_cast<const unsigned char*>(g.src) + c, n);
      PB_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(g.dev) + c, hin + off, n,
                              cudaMemcpyHostToDevice, st));
      off += n;
    }
  // the result comes back into a zeroed buffer and is added to the caller's
  // output on the host (accumulate semantics without uploading the output)
  PB_CUDA(cudaMemsetAsync(ws.io_out.p, 0, bo, st));
  rc = pbbfmm_compute_device(t, dt, Nf, ds, Ns, ws.io_w.as<double>(), nCols,
                             ws.io_out.as<double>(), t->precision, st);
  if (rc) return rc;
  double* hout = static_cast<double*>(ws.h_out);
  const size_t chunk_d = kStageChunk / sizeof(double);
  const size_t total_d = (size_t)Nf * nCols;
  std::vector<cudaEvent_t> evs;
  for (size_t c = 0; c < total_d; c += chunk_d) {
    const size_t n = total_d - c < chunk_d ? total_d - c : chunk_d;
    PB_CUDA(cudaMemcpyAsync(hout + c, ws.io_out.as<double>() + c, n * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
    cudaEvent_t e;
    PB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    PB_CUDA(cudaEventRecord(e, st));
    evs.push_back(e);
  }
  int status = PBBFMM_OK;
  size_t k = 0;
  for (size_t c = 0; c < total_d; c += chunk_d, ++k) {
    const size_t n = total_d - c < chunk_d ? total_d - c : chunk_d;
    cudaError_t e = cudaEventSynchronize(evs[k]);
    if (e != cudaSuccess && status == PBBFMM_OK) status = cuda_status(e, "result copy");
    // The compute's kernels finished before the first result chunk landed,
    // so a timed-out tensor-core wait has set its flag by now: nothing is
    // added to the caller's output from an invalid compute.
    if (k == 0 && status == PBBFMM_OK) status = take_tc_timeout(t);
    if (status == PBBFMM_OK) host_add_mt(output + c, hout + c, n);
  }
  for (cudaEvent_t e : evs) cudaEventDestroy(e);
  return status;
}

int pbbfmm_set_tensor_cores(pbbfmm_tree* t, int mode) {
  if (!t) {
    set_error("null tree");
    return PBBFMM_ERR_ARG;
  }
  if (mode != PBBFMM_TC_OFF && mode != PBBFMM_TC_F16 && mode != PBBFMM_TC_TF32) {
    set_error("tensor-core mode must be PBBFMM_TC_OFF, PBBFMM_TC_F16 or PBBFMM_TC_TF32");
    return PBBFMM_ERR_ARG;
  }
  t->use_tc = mode != PBBFMM_TC_OFF;
  if (mode != PBBFMM_TC_OFF) t->tc_fmt = mode;
  return PBBFMM_OK;
}

int pbbfmm_tensor_core_m2l(const pbbfmm_tree* t) {
  return t && tc_eligible(t) ? t->tc_fmt : PBBFMM_TC_OFF;
}

int pbbfmm_debug_copy(pbbfmm_tree* t, int what, int level, double* host, int64_t count,
                      int64_t* written) {
  if (!t || !t->have_last || t->device < 0) {
    set_error("no compute to inspect");
    return PBBFMM_ERR_STATE;
  }
  PB_CUDA(cudaSetDevice(t->device));
  PB_CUDA(cudaDeviceSynchronize());
  const int L = t->p.tree_level;
  const int C = t->last_C;
  std::vector<int> tmp;
  const double* src = nullptr;
  int64_t total = 0;
  if (what == 0 || what == 1) {
    if (level < 2 || level > L) {
      set_error("level must be in [2, tree_level]");
      return PBBFMM_ERR_ARG;
    }
    const int64_t per = (int64_t)C * t->n3;
    total = cells_at(level) * per;
    if (t->cur_prec != PBBFMM_PREC_FP64) {  // mixed path: float32 arrays, widened here
      const float* fs =
          (what == 0 ? t->ws.S.as<float>() : t->ws.F.as<float>()) + level_offset(level, per);
      const int64_t nc = count < total ? count : total;
      std::vector<float> tmpf(nc > 0 ? nc : 1);
      if (host && nc > 0) {
        PB_CUDA(cudaMemcpy(tmpf.data(), fs, sizeof(float) * nc, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < nc; ++i) host[i] = tmpf[i];
      }
      if (written) *written = total;
      return PBBFMM_OK;
    }
    src = (what == 0 ? t->ws.S.as<double>() : t->ws.F.as<double>()) + level_offset(level, per);
  } else if (what >= 2 && what <= 5) {
    const int* p = nullptr;
    if (what == 2) {
      p = t->ws.tstart.as<int>();
      total = cells_at(L) + 1;
    } else if (what == 3) {
      p = t->ws.tperm.as<int>();
      total = t->last_Nf;
    } else if (what == 4) {
      p = t->ws.sstart.as<int>();
      total = cells_at(L) + 1;
    } else {
      p = t->ws.sperm.as<int>();
      total = t->last_Ns;
    }
    tmp.resize(total);
    PB_CUDA(cudaMemcpy(tmp.data(), p, sizeof(int) * total, cudaMemcpyDeviceToHost));
    int64_t nc = count < total ? count : total;
    for (int64_t i = 0; i < nc; ++i) host[i] = tmp[i];
    if (written) *written = total;
    return PBBFMM_OK;
  } else {
    set_error("unknown debug array");
    return PBBFMM_ERR_ARG;
  }
  if (written) *written = total;
  int64_t nc = count < total ? count : total;
  if (host && nc > 0) PB_CUDA(cudaMemcpy(host, src, sizeof(double) * nc, cudaMemcpyDeviceToHost));
  return PBBFMM_OK;
}

}  // extern "C"
