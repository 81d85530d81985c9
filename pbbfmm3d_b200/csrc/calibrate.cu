// Throughput calibration for the roofline of the CUDA-core (non-tensor)
// kernels: a dependent-chain-free FMA loop on every SM, timed with CUDA
// events.  The driver-measured peaks cover HBM copy and bf16 tensor GEMMs;
// the frequency-domain M2L runs on the float64 / float32 FMA pipes, whose
// peak is measured here the same way (best of a few runs).
#include "fmm.cuh"

namespace pbbfmm {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T* out, int iters, T a, T b) {
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5,
    x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-12345.678)) out[0] = s;  // keeps the loop alive
}

// The special-function pipe: float32 reciprocal square roots (rsqrtf), the
// 1/r kernels' near-field step, 8 independent chains per thread.
__global__ void __launch_bounds__(256) k_rsqrt_peak(float* out, int iters, float b) {
  float x0 = threadIdx.x + 1.f, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4,
        x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      x0 = rsqrtf(x0 + b); x1 = rsqrtf(x1 + b); x2 = rsqrtf(x2 + b); x3 = rsqrtf(x3 + b);
      x4 = rsqrtf(x4 + b); x5 = rsqrtf(x5 + b); x6 = rsqrtf(x6 + b); x7 = rsqrtf(x7 + b);
    }
  }
  const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == -12345.678f) out[0] = s;  // keeps the loop alive
}

template <typename T, bool RSQRT = false>
static int measure(int device, double* tflops) {
  PB_CUDA(cudaSetDevice(device));
  int sms = 0;
  PB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  T* out = nullptr;
  PB_CUDA(cudaMalloc(&out, sizeof(T)));
  cudaEvent_t e0, e1;
  PB_CUDA(cudaEventCreate(&e0));
  PB_CUDA(cudaEventCreate(&e1));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  double best = 0;
  for (int rep = 0; rep < 4; ++rep) {
    PB_CUDA(cudaEventRecord(e0));
    if constexpr (RSQRT)
      k_rsqrt_peak<<<blocks, threads>>>(reinterpret_cast<float*>(out), iters / 4, 1.f);
    else
      k_fma_peak<T><<<blocks, threads>>>(out, iters, T(0.999999), T(1e-7));
    PB_CUDA(cudaEventRecord(e1));
    PB_CUDA(cudaEventSynchronize(e1));
    PB_LAUNCH("fma_peak");
    float ms = 0;
    PB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    // FMA: 2 flops each; rsqrt: one operation each (a quarter of the iterations)
    const double flops = RSQRT ? 8.0 * 16 * (double)(iters / 4) * blocks * threads
                               : 2.0 * 8 * 16 * (double)iters * blocks * threads;
    const double tf = flops / (ms * 1e-3) / 1e12;
    if (rep > 0 && tf > best) best = tf;  // first run is warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = best;
  return PBBFMM_OK;
}

}  // namespace pbbfmm

extern "C" int pbbfmm_measure_fma_peak(int device, int precision, double* tflops) {
  if (!tflops) return PBBFMM_ERR_ARG;
  if (precision == 2) return pbbfmm::measure<float, true>(device, tflops);
  return precision == PBBFMM_PREC_FP64 ? pbbfmm::measure<double>(device, tflops)
                                       : pbbfmm::measure<float>(device, tflops);
}
