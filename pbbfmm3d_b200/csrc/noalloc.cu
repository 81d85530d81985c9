// Leaf binning that allocates nothing.
//
// Some callers cannot call cudaMalloc: for example a process whose device
// memory is reserved up front by another allocator (a framework's caching
// allocator or a pool sized to the whole GPU), or a deployment that forbids
// allocation after start-up so that its memory footprint is fixed and known in
// advance.  pbbfmm_bin_points_noalloc gives them the binning step of the
// matvec -- recentring, the reference's leaf assignment and a stable sort by
// leaf -- with every scratch byte in one file-scope device array of fixed size
// (kNoAllocScratchBytes below, for at most PBBFMM_NOALLOC_MAX_POINTS points).
// Each GPU that loads this library holds that array until the process exits.
//
// The array's name is only a host-side stand-in for the device symbol, so the
// host looks up its device address once per device with
// cudaGetSymbolAddress (on the entry point's first call on that device) and
// passes the pointer to the kernels.  All calls share the array and it keeps
// the last call's contents; calls that overlap on the GPU (different streams,
// or different host threads on the same device) race on it.
#include <cub/cub.cuh>

#include <mutex>

#include "fmm.cuh"

namespace pbbfmm {

// The matvec's own binning kernels (tree.cu), launched here unchanged on the
// scratch array instead of the tree's workspace.
constexpr int kBBoxBlocks = 296;
constexpr int kBBoxThreads = 256;
__global__ void k_bbox_partial(const double* __restrict__ p, int64_t N, double* __restrict__ part);
__global__ void k_bbox_final(const double* __restrict__ part, int nb, double* __restrict__ ctr);
__global__ void k_keys(const double* __restrict__ p, int64_t N, const double* __restrict__ ctr,
                       double box, int L, uint32_t* __restrict__ key, int* __restrict__ idx);
__global__ void k_leaf_start(const uint32_t* __restrict__ ks, int N, int64_t nleaf,
                             int* __restrict__ start);

// Scratch layout (bytes): bbox partials | centre | keys | sorted keys |
// indices | CUB temporary storage.
constexpr int64_t kNoAllocMax = PBBFMM_NOALLOC_MAX_POINTS;
constexpr size_t kPartBytes = 8 * 6 * kBBoxBlocks;
constexpr size_t kCtrBytes = 256;
constexpr size_t kArrBytes = 4 * (size_t)kNoAllocMax;
constexpr size_t kCubBytes = 12u << 20;
constexpr size_t kNoAllocScratchBytes = kPartBytes + kCtrBytes + 3 * kArrBytes + kCubBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once).
int noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device index out of range for the allocation-free entry point");
    return PBBFMM_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(noalloc scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return PBBFMM_OK;
}
}  // namespace

}  // namespace pbbfmm

using namespace pbbfmm;

extern "C" int pbbfmm_bin_points_noalloc(const double* d_points, int64_t N, double box,
                                         int tree_level, int* d_perm, int* d_leaf_start,
                                         double* d_center, void* stream) {
  if (N < 0 || N > kNoAllocMax) {
    set_error("pbbfmm_bin_points_noalloc: N must be in [0, " + std::to_string(kNoAllocMax) +
              "] (the fixed scratch array holds at most that many points)");
    return PBBFMM_ERR_ARG;
  }
  if (tree_level < 1 || tree_level > kMaxLevel || !(box > 0)) {
    set_error("pbbfmm_bin_points_noalloc: tree_level must be in [1, 10] and box > 0");
    return PBBFMM_ERR_ARG;
  }
  if ((N > 0 && (!d_points || !d_perm)) || !d_leaf_start) {
    set_error("pbbfmm_bin_points_noalloc: null pointer");
    return PBBFMM_ERR_ARG;
  }
  int dev = 0;
  PB_CUDA(cudaGetDevice(&dev));
  unsigned char* base = nullptr;
  if (int rc = noalloc_scratch(dev, &base)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  double* part = reinterpret_cast<double*>(base);
  double* ctr = reinterpret_cast<double*>(base + kPartBytes);
  uint32_t* key = reinterpret_cast<uint32_t*>(base + kPartBytes + kCtrBytes);
  uint32_t* key_sorted = reinterpret_cast<uint32_t*>(base + kPartBytes + kCtrBytes + kArrBytes);
  int* idx = reinterpret_cast<int*>(base + kPartBytes + kCtrBytes + 2 * kArrBytes);
  void* cub_temp = base + kPartBytes + kCtrBytes + 3 * kArrBytes;
  const int L = tree_level;
  const int64_t nleaf = cells_at(L);
  if (N > 0) {
    size_t need = 0;
    PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, key, key_sorted, idx, d_perm, (int)N, 0,
                                            3 * L, st));
    if (need > kCubBytes) {
      set_error("pbbfmm_bin_points_noalloc: sort scratch exceeds the fixed array");
      return PBBFMM_ERR_UNSUPPORTED;
    }
    // every scratch word read below is written first in this call, so the
    // previous call's contents never leak into this one
    k_bbox_partial<<<kBBoxBlocks, kBBoxThreads, 0, st>>>(d_points, N, part);
    k_bbox_final<<<1, 32, 0, st>>>(part, kBBoxBlocks, ctr);
    PB_LAUNCH_N("noalloc bbox", 2);
    k_keys<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(d_points, N, ctr, box, L, key, idx);
    PB_LAUNCH("noalloc keys");
    size_t bytes = kCubBytes;
    PB_CUDA(cub::DeviceRadixSort::SortPairs(cub_temp, bytes, key, key_sorted, idx, d_perm, (int)N,
                                            0, 3 * L, st));
    count_launches(1 + (3 * L + 7) / 8);
    if (d_center) PB_CUDA(cudaMemcpyAsync(d_center, ctr, 3 * sizeof(double),
                                          cudaMemcpyDeviceToDevice, st));
  }
  k_leaf_start<<<(unsigned)((nleaf + 1 + 255) / 256), 256, 0, st>>>(key_sorted, (int)N, nleaf,
                                                                    d_leaf_start);
  PB_LAUNCH("noalloc leaf_start");
  return PBBFMM_OK;
}
