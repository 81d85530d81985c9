// Device helpers of the tensor-core kernels (sm_100a): shared-memory
// matrix and instruction descriptors of tcgen05.mma, bounded mbarrier waits,
// TMA / bulk copies without multicast, TMEM loads and stores, and exact
// power-of-two scaling.  Descriptor fields follow the sm100 formats as the
// vendored CUTLASS cute/arch/mma_sm100_desc.hpp lays them out.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace pbbfmm {

constexpr long long kWaitCycles = 2000000000ll;  // about 1 s of SM clock
constexpr long long kWaitIters = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major SWIZZLE_128B shared-memory matrix descriptor (sm100 format:
// start>>4 in [0,14), LBO>>4 in [16,30) (unused for this layout, 1), SBO>>4 in
// [32,46) = 1024 bytes between 8-row groups, version 1 in [46,48), layout
// type 2 = SWIZZLE_128B in [61,64)).  Tile bases are 1024-byte aligned; a K
// step of 8 float32 inside the 128-byte row advances the start by 32 bytes.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor for kind::tf32: D float32 (bits 4-5 = 1), A and B
// TF32 (bits 7-9, 10-12 = 2), both K-major, N>>3 in bits 17-22, M>>4 in 24-28.
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}
// kind::f16 with A and B F16 (format 0 in bits 7-9, 10-12), D float32.
__host__ __device__ constexpr uint32_t f16_idesc(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of (row r, 16-byte chunk j) in a K-major SWIZZLE_128B tile.
__device__ __forceinline__ uint32_t sw128_off(int r, int j) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t a, int parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}

// try_wait that may suspend the thread (not issuing) for up to `ns`
// nanoseconds while the phase is incomplete; it returns as soon as the phase
// completes.
__device__ __forceinline__ bool mbar_try_sleep(uint32_t a, int parity, uint32_t ns) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(a), "r"(parity), "r"(ns)
      : "memory");
  return done != 0;
}

// mbar_wait with suspending polls (see mbar_try_sleep): for waiters that
// share their SM sub-partition with warps doing work.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, int parity,
                                                const volatile int* abort,
                                                long long iters = kWaitIters) {
  const uint32_t a = smem_u32(bar);
  if (mbar_try(a, parity)) return true;
  const long long t0 = clock64();
  // (a poll limit below 1024, a test's forced timeout, polls without suspending)
  const uint32_t ns = iters >= 1024 ? 20000u : 0u;
  for (long long it = 0; it < iters; ++it) {
    if (ns ? mbar_try_sleep(a, parity, ns) : mbar_try(a, parity)) return true;
    if ((it & 15) == 15 && ((abort && *abort) || clock64() - t0 > kWaitCycles)) return false;
  }
  return false;
}

// Wait for the completion of the phase with parity `parity`; false after
// about a second of SM clock (or kWaitIters polls) without it, or once *abort
// is set (abort may be null).  The first poll reads no clock: a wait that is
// already satisfied costs one try_wait.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, int parity, const volatile int* abort,
                                          long long iters = kWaitIters) {
  const uint32_t a = smem_u32(bar);
  if (mbar_try(a, parity)) return true;
  const long long t0 = clock64();
  for (long long it = 0; it < iters; ++it) {
    if (mbar_try(a, parity)) return true;
    if ((it & 255) == 255 && ((abort && *abort) || clock64() - t0 > kWaitCycles)) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Arrive on `bar` and add `bytes` to the transaction count it waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// 2-D tiled TMA load (no multicast) into this CTA's shared memory, completing
// `bytes` of the transaction count of `bar`; x (the innermost coordinate)
// is a multiple of 32 floats (128 bytes).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4}], [%2];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Arrive on `bar` once every cp.async issued so far by this thread has
// landed (the barrier's expected count includes this arrival).
__device__ __forceinline__ void cp_async_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                           uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive on `bar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 16 consecutive float32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive float32 columns of this thread's TMEM lane, loaded and waited
// for in one asm statement (so that no use of r can precede the wait).
__device__ __forceinline__ void tc_ld16_wait(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

// Store 16 consecutive float32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_st16(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};\n" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}
__device__ __forceinline__ void tc_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
}

// 2^k as a float, exactly, for k in [-149, 127].
__device__ __forceinline__ float exp2i(int k) {
  return k >= -126 ? __int_as_float((k + 127) << 23) : __int_as_float(1 << (k + 149));
}

// x 2^k with every step an exact power-of-two product: k is split into
// factors inside the float exponent range, so the result is exact whenever
// it is a normal number (whatever k), and correctly rounded otherwise.
__device__ __forceinline__ float scale2(float x, int k) {
  k = min(max(k, -400), 400);
  while (k > 127) {
    x *= exp2i(127);
    k -= 127;
  }
  while (k < -126) {
    x *= exp2i(-126);
    k += 126;
  }
  return x * exp2i(k);
}

// k2 with |x| in [2^(k2-1), 2^k2) for finite x != 0 (frexp's exponent).
__device__ __forceinline__ int exponent_of(float x) {
  const uint32_t b = __float_as_uint(x) & 0x7fffffffu;
  if (b >= 0x00800000u) return (int)(b >> 23) - 126;
  return 32 - __clz(b) - 149;  // subnormal: b 2^-149, b in [2^(j-1), 2^j)
}

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}


}  // namespace pbbfmm

namespace pbbfmm {

// K-major SWIZZLE_NONE ("interleaved") shared-memory matrix descriptor:
// 8-row x 16-byte core matrices, rows 16 bytes apart inside one; lbo = bytes
// between the two K-adjacent core matrices an instruction reads, sbo = bytes
// between 8-row groups along M / N (start, LBO, SBO in 16-byte units, version
// 1 in bits [46,48), layout type 0).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Bulk copy (no multicast) of `bytes` (a multiple of 16, both addresses
// 16-byte aligned) from global into this CTA's shared memory, completing on
// the transaction count of `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace pbbfmm

namespace pbbfmm {

// 64 consecutive float32 columns of this thread's TMEM lane, loaded and
// waited for in one asm statement (so that no use of r can precede the wait).
__device__ __forceinline__ void tc_ld64_wait(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(taddr)
      : "memory");
}

}  // namespace pbbfmm
