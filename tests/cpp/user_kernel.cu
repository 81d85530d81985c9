// A user-defined kernel in the reference's style (README.md:178-227: a
// subclass with SetKernelProperty and EvaluateKernel), written as a
// __host__ __device__ functor for pbbfmm3d_b200 and run through the C++ front
// door: Atree.buildFMMTree(cache_dir); H2_3D_Compute<mySoftened>(...).
//
// The kernel is the softened Laplacian 1/sqrt(r^2 + delta^2), delta = 0.05
// (not homogeneous: one operator set per level; symmetric), kernelType
// "SoftLap0.05" -- the same class the reference test driver compiles.
//
// Usage: user_kernel <points.bin> <weight.bin> N nCols level order eps cheb
//                    <cache_dir> <out64.bin> <out32.bin> [grad.bin]
//        user_kernel --no-run
// points: N x 3 float64 (xyz records); weight: column-major N x nCols.
// Sources = targets.  Writes the float64 and the mixed-precision outputs,
// and with grad.bin the adjoint's dL/d(source) for g = weight (float64).
// Exit 0 and "OK" on success.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pbbfmm3d_b200_kernel.cuh"

using namespace pbbfmm3d_b200;

class mySoftened : public H2_3D_Tree_device<mySoftened> {
 public:
  using H2_3D_Tree_device::H2_3D_Tree_device;
  void SetKernelProperty() {
    homogen = 0;
    symmetry = 1;
    kernelType = "SoftLap0.05";
  }
  template <typename R>
  __host__ __device__ static R EvaluateKernel(const vec3<R>& targetpos, const vec3<R>& sourcepos) {
    vec3<R> diff;
    diff.x = sourcepos.x - targetpos.x;
    diff.y = sourcepos.y - targetpos.y;
    diff.z = sourcepos.z - targetpos.z;
    return R(1) / sqrt(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z + R(0.05) * R(0.05));
  }
  // dK/d(sourcepos) = -diff / (r^2 + delta^2)^(3/2)
  template <typename R>
  __host__ __device__ static R EvaluateKernelGradient(const vec3<R>& targetpos,
                                                      const vec3<R>& sourcepos, R* g) {
    const R dx = sourcepos.x - targetpos.x, dy = sourcepos.y - targetpos.y,
            dz = sourcepos.z - targetpos.z;
    const R k = R(1) / sqrt(dx * dx + dy * dy + dz * dz + R(0.05) * R(0.05));
    const R f = -k * k * k;
    g[0] = f * dx, g[1] = f * dy, g[2] = f * dz;
    return k;
  }
};

static std::vector<double> read_file(const char* path, size_t count) {
  std::vector<double> v(count);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(double), count, f) != count) {
    std::fprintf(stderr, "cannot read %s\n", path);
    std::exit(2);
  }
  std::fclose(f);
  return v;
}

static void write_file(const char* path, const std::vector<double>& v) {
  FILE* f = std::fopen(path, "wb");
  if (!f || std::fwrite(v.data(), sizeof(double), v.size(), f) != v.size()) {
    std::fprintf(stderr, "cannot write %s\n", path);
    std::exit(2);
  }
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc > 1 && !std::strcmp(argv[1], "--no-run")) {
    std::printf("linked %s\n", pbbfmm_version());
    return 0;
  }
  if (argc < 12) {
    std::fprintf(stderr, "usage: see the file header\n");
    return 2;
  }
  const size_t N = std::strtoull(argv[3], nullptr, 10);
  const int C = std::atoi(argv[4]), level = std::atoi(argv[5]), order = std::atoi(argv[6]);
  const double eps = std::atof(argv[7]);
  const int cheb = std::atoi(argv[8]);
  const std::vector<double> pts = read_file(argv[1], 3 * N);
  const std::vector<double> w = read_file(argv[2], N * C);
  std::vector<vec3<double>> points(N);
  for (size_t i = 0; i < N; ++i) points[i] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  try {
    mySoftened Atree(1.0, level, order, eps, cheb);
    Atree.buildFMMTree(argv[9]);  // the reference's operator files, named by kernelType
    std::vector<double> out64(N * C, 0.0), out32(N * C, 0.0);
    H2_3D_Compute<mySoftened>(Atree, points, points, w, C, out64);
    Atree.set_precision(PBBFMM_PREC_MIXED);
    H2_3D_Compute<mySoftened>(Atree, points, points, w, C, out32);
    write_file(argv[10], out64);
    write_file(argv[11], out32);
    if (argc > 12) {  // adjoint through the C ABI: dL/d(source) with g = weight
      double *d_p, *d_w, *d_g;
      cudaMalloc(&d_p, 3 * N * sizeof(double));
      cudaMalloc(&d_w, N * C * sizeof(double));
      cudaMalloc(&d_g, 3 * N * sizeof(double));
      cudaMemcpy(d_p, pts.data(), 3 * N * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(d_w, w.data(), N * C * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemset(d_g, 0, 3 * N * sizeof(double));
      check(pbbfmm_compute_adjoint_device(Atree.handle(), d_p, (int64_t)N, d_p, (int64_t)N, d_w,
                                          d_w, C, nullptr, d_g, nullptr, PBBFMM_PREC_FP64,
                                          nullptr));
      std::vector<double> grad(3 * N);
      if (cudaMemcpy(grad.data(), d_g, 3 * N * sizeof(double), cudaMemcpyDeviceToHost) !=
          cudaSuccess) {
        std::fprintf(stderr, "copy failed\n");
        return 1;
      }
      cudaFree(d_p);
      cudaFree(d_w);
      cudaFree(d_g);
      write_file(argv[12], grad);
    }
  } catch (const Error& e) {
    std::fprintf(stderr, "pbbfmm3d_b200 error %d: %s\n", e.status, e.what());
    return 1;
  }
  std::printf("OK\n");
  return 0;
}
