// Internal state of a tree (the C-ABI's opaque pbbfmm_tree) and the launch
// entry points of each phase.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "precompute.h"

namespace pbbfmm {

constexpr int kMaxLevel = 10;

// Grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};
int grow(DevBuf& b, size_t bytes);  // PBBFMM_OK or PBBFMM_ERR_ALLOC
void release(DevBuf& b);

// Device arrays of one compute, grown on demand and kept by the tree.
struct Workspace {
  // binning
  DevBuf bbox_part;  // 6 doubles per reduction block
  DevBuf ctr;        // 3 doubles: recentring shift
  DevBuf key, key_sorted, idx;  // max(Nf, Ns)
  DevBuf tperm, sperm;          // sorted position -> original index
  DevBuf tstart, sstart;        // nleaf + 1 leaf offsets
  DevBuf tpos, spos;            // SoA 3 x N, recentred, sorted
  DevBuf wsorted;               // Ns x C, point-major
  DevBuf cub_temp;
  DevBuf lists;    // nonempty-cell lists, back to back
  DevBuf dcounts;  // device-side counts of the lists
  // per-level coefficient arrays (levels 2..L)
  DevBuf S;      // moments      sum_l 8^l * C * n3
  DevBuf F;      // locals       sum_l 8^l * C * n3
  DevBuf proxy;  // Cheb: sum_l 8^l * C * rs ;  Unif: spectra sum_l 8^l * nk * C (complex)
  DevBuf pf;     // Cheb: sum_l 8^l * C * rf ;  Unif: accumulated spectra
  DevBuf halo;   // Unif M2L: per parent block 512 halo + 64 target cells
  DevBuf tc_proxy;  // tensor-core Cheb M2L: hi then lo proxies of one level (+ F16 exponents)
  DevBuf leafpart;  // leaf phase: target leaves partitioned dense-first, then their count
  DevBuf occ;       // tensor-core uniform M2L: per-cell source / target occupancy of a level
  DevBuf amax;      // tensor-core uniform M2L: per level, largest |spectra| per (k23, column mod 8)
  // staging for the host-pointer entry point
  DevBuf io_tgt, io_src, io_w, io_out;
  // pinned host staging of the host-buffer entry point (cudaHostAlloc)
  void* h_in = nullptr;
  size_t h_in_cap = 0;
  void* h_out = nullptr;
  size_t h_out_cap = 0;
  cudaStream_t io_stream = nullptr;  // the host entry's stream (created on first use)
};

struct LevelLists {
  // offsets into Workspace::lists and counts (host copies after binning)
  int64_t src_off[kMaxLevel + 1];   // nonempty source cells, Morton order
  int64_t tgt_off[kMaxLevel + 1];   // nonempty target cells, Morton order
  int64_t typ_off[kMaxLevel + 1];   // nonempty target cells ordered (child type, parent)
  int nsrc[kMaxLevel + 1];
  int ntgt[kMaxLevel + 1];
  int ntyp[kMaxLevel + 1][9];       // type boundaries within the typed list
};

// Operands of the tensor-core Chebyshev M2L: for each level and operator o,
// E_o^T as np rows (rf padded to 16), split hi / lo, zero padded:
//   TF32: rows of kp floats (rs padded to 32);
//   F16 : rows of kp16 halves (rs padded to 64), each operator scaled by
//         2^eexp[lvl * 316 + o].
// Null when np exceeds the tensor-core limit.
struct TcOps {
  float* eth = nullptr;
  float* etl = nullptr;
  uint16_t* eh16 = nullptr;
  uint16_t* el16 = nullptr;
  int* eexp = nullptr;
  int np = 0, kp = 0, kp16 = 0;
  // M2L pre / post transforms on the tensor cores: W = VT (rs x n^3) and
  // U (n^3 x r_f) as [level][mp][kp] F16 hi / lo rows (row m holds W[m][k]
  // over k, zero padded; mp = rows padded to 16 (32 above 256), kp = K
  // padded to 64), each level's matrix scaled by 2^exp[level].  Null when mp
  // exceeds 512.
  uint16_t *vth = nullptr, *vtl = nullptr, *uh = nullptr, *ul = nullptr;
  int vt_mp = 0, vt_kp = 0, u_mp = 0, u_kp = 0;
  int vt_exp[32] = {}, u_exp[32] = {};
};

}  // namespace pbbfmm

struct pbbfmm_tree {
  pbbfmm_tree_params p{};
  pbbfmm::KernelSpec kspec;
  pbbfmm_user_kernel user{};  // user-defined kernel (p.kernel == PBBFMM_KERNEL_USER)
  pbbfmm::Weights w;
  pbbfmm::Operators ops;
  int device = 0;
  bool weights_ready = false;
  bool ops_ready = false;
  int precision = PBBFMM_PREC_FP64;
  int n = 0, n3 = 0, m = 0, nk = 0;  // order, n^3, 2n-1, complex spectrum size m*m*n
  bool homog = false;
  double homogen_neg = 0;
  // device operators
  double* d_Tkz = nullptr;
  double* d_Kw = nullptr;
  double* d_Cw = nullptr;
  double* d_E = nullptr;   // Cheb: nlev x 316 x rf x rs (col-major blocks)
  double* d_U = nullptr;   // Cheb: nlev x n3 x rf
  double* d_VT = nullptr;  // Cheb: nlev x rs x n3
  double* d_op = nullptr;  // Unif: nlev x 343 x nk complex (lex-indexed, inner 27 zero)
  int* d_offs = nullptr;   // Cheb M2L: 8 types x 189 x 4 (ox, oy, oz, op index)
  double* d_twid = nullptr;  // Unif: cos/sin of 2 pi j / m, j < m
  double* d_kparam = nullptr;  // 4 kernel parameters
  // float32 copies of the weights and operators for the mixed path
  float* f_Tkz = nullptr;
  float* f_Kw = nullptr;
  float* f_Cw = nullptr;
  float* f_E = nullptr;
  float* f_U = nullptr;
  float* f_VT = nullptr;
  float* f_op = nullptr;  // nlev x nk x 343 complex (float2)
  // tensor-core uniform M2L: per level and frequency the operator tiles of
  // the block product (m2l_unif_tc.cu), scaled F16 hi / lo, and their
  // power-of-two exponents
  uint16_t* f_unif_tiles = nullptr;
  int* f_unif_bexp = nullptr;
  float* f_twid = nullptr;
  // tensor-core Chebyshev M2L (mixed path); tc_fmt: PBBFMM_TC_F16 (scaled
  // F16 operands, default) or PBBFMM_TC_TF32
  bool use_tc = true;
  int tc_fmt = PBBFMM_TC_F16;
  pbbfmm::TcOps tc;
  int* h_tc_err = nullptr;  // mapped pinned flag: a tensor-core wait timed out
  int* d_tc_err = nullptr;  // its device address
  // Adjoint (transposed) Chebyshev operators: U' = VT^T, E'_p = E_{-p}^T,
  // VT' = U^T, so r_f' = r_s and r_s' = r_f.  Swapped with the forward set
  // (swap_adjoint_ops) for the duration of an adjoint pass.
  struct OpSet {
    double *E = nullptr, *U = nullptr, *VT = nullptr;
    float *fE = nullptr, *fU = nullptr, *fVT = nullptr;
    pbbfmm::TcOps tc;
    int rf = 0, rs = 0;
  } adj;
  bool adj_ready = false;
  // pass settings (set by the adjoint / gradient entry points, cleared after)
  const double* bbox_pts = nullptr;  // recentre on these points instead of the targets
  int64_t bbox_n = 0;
  struct GradLeaf {
    bool on = false;
    const double* contract = nullptr;  // [col * Nf + i]: weights of each target's gradient
    double* grad_out = nullptr;        // [i * 3 + d] += sum_col contract * d phi_col / d x_d
    bool values = true;                // also add the potentials to the compute's output
  } gl;
  int cur_prec = PBBFMM_PREC_FP64;  // precision of the compute in flight
  pbbfmm::Workspace ws;
  pbbfmm::LevelLists lists;
  // last compute (debug access)
  int last_C = 0;
  int64_t last_Nf = 0, last_Ns = 0;
  bool have_last = false;
  // timing
  bool timing = false;
  cudaEvent_t ev[16] = {};
  int nev = 0;
  float phase_ms[16] = {};
  int nphase = 0;
  // per-kernel event pairs of the computes since the last reset (timing on)
  std::vector<cudaEvent_t> kev;
  std::vector<int> kslot;  // slot of each event pair
  size_t kused = 0;
};

namespace pbbfmm {

// Device operators in the precision of a compute.
template <typename T>
struct OpsView {
  const T* Tkz;
  const T* Kw;
  const T* Cw;
  const T* E;
  const T* U;
  const T* VT;
  const cplx_t<T>* op;
};
template <typename T>
inline OpsView<T> ops_view(const pbbfmm_tree* t);
template <>
inline OpsView<double> ops_view<double>(const pbbfmm_tree* t) {
  return {t->d_Tkz, t->d_Kw, t->d_Cw, t->d_E, t->d_U, t->d_VT, (const double2*)t->d_op};
}
template <>
inline OpsView<float> ops_view<float>(const pbbfmm_tree* t) {
  return {t->f_Tkz, t->f_Kw, t->f_Cw, t->f_E, t->f_U, t->f_VT, (const float2*)t->f_op};
}

// level geometry
inline int64_t cells_at(int l) { return (int64_t)1 << (3 * l); }
// element offset of level l in an array holding `per_cell` values per cell for levels 2..L
inline int64_t level_offset(int l, int64_t per_cell) {
  int64_t off = 0;
  for (int j = 2; j < l; ++j) off += cells_at(j) * per_cell;
  return off;
}
inline int64_t level_total(int L, int64_t per_cell) { return level_offset(L + 1, per_cell); }

// ---- phase launchers (return PBBFMM_* status; errors via last_error) ----
int run_binning(pbbfmm_tree* t, const double* d_tgt, int64_t Nf, const double* d_src, int64_t Ns,
                const double* d_w, int C, cudaStream_t st);
int run_upward(pbbfmm_tree* t, int C, cudaStream_t st);
int run_m2l_cheb(pbbfmm_tree* t, int C, cudaStream_t st);
// tensor-core Chebyshev M2L (float path): N = rf padded to 16 must fit TMEM
constexpr int kTcMaxN = 256;
bool tc_eligible(const pbbfmm_tree* t);
// M2L pre (post = false: proxy = VT (Kw o S)) or post (post = true:
// F = alpha Kw o (U Pf)) transform of level l on the tensor cores, for the
// ncols = (cells x C) columns listed; false from colgemm_tc_eligible when the
// CUDA-core kernel must run instead.
bool colgemm_tc_eligible(const pbbfmm_tree* t, bool post);
int run_colgemm_tc(pbbfmm_tree* t, bool post, int lvl, const int* cells, int ncols, int C,
                   const float* X, float* Out, float alpha, cudaStream_t st);
int run_m2l_cheb_tc_level(pbbfmm_tree* t, int C, int l, int lvl, const float* proxy, float* pf,
                          cudaStream_t st);
int run_m2l_unif(pbbfmm_tree* t, int C, cudaStream_t st);
// tensor-core uniform M2L (float path): levels with >= 16 parents per side,
// columns in groups of 8
bool unif_tc_eligible(const pbbfmm_tree* t, int l, int C);
int run_m2l_unif_tc_level(pbbfmm_tree* t, int C, int l, int lvl, const float2* X, float2* Y,
                          const uint32_t* amax, cudaStream_t st);
void unif_tc_tiles(int n, const std::vector<double>& op, int nlev, std::vector<uint16_t>* tiles,
                   std::vector<int>* bexp);
int set_unif_tc_wait_limit(long long polls);
int run_downward(pbbfmm_tree* t, int C, cudaStream_t st);
int run_leaves(pbbfmm_tree* t, int64_t Nf, int64_t Ns, int C, double* d_out, cudaStream_t st);
// operator spectra for the uniform path (host, float64) from the stencils
void unif_spectra(int n, const std::vector<double>& stencil, int nlev, std::vector<double>* op);

// Kernel timer slots (pbbfmm_get_kernel_times).
enum KSlot {
  KS_BINNING = 0, KS_P2M, KS_M2M, KS_M2L_PRE, KS_M2L, KS_M2L_POST, KS_FFT_FWD, KS_MAC, KS_FFT_INV,
  KS_L2L, KS_LEAF, KS_M2L_SPLIT, KS_COUNT
};
extern const char* const kSlotNames;
// Record an event before / after a launch when timing is enabled.
int kt_begin(pbbfmm_tree* t, int slot, cudaStream_t st);
int kt_end(pbbfmm_tree* t, cudaStream_t st);

void set_error(const std::string& msg);
int cuda_status(cudaError_t e, const char* what);

#define PB_CUDA(call)                                              \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return ::pbbfmm::cuda_status(e_, #call); \
  } while (0)
// Kernel launches issued by this library (CUB calls count their internal
// launches: see count_launches at the CUB call sites).
void count_launches(int n);
#define PB_LAUNCH_N(what, n)                                               \
  do {                                                                     \
    ::pbbfmm::count_launches(n);                                           \
    cudaError_t e_ = cudaGetLastError();                                   \
    if (e_ != cudaSuccess) return ::pbbfmm::cuda_status(e_, what);         \
  } while (0)
#define PB_LAUNCH(what) PB_LAUNCH_N(what, 1)

}  // namespace pbbfmm
