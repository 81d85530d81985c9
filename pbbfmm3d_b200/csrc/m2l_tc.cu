// Chebyshev M2L of the mixed-precision path on the 5th-generation tensor
// cores (tcgen05 with TMEM accumulators), in split precision:
//     D += A_lo B_hi + A_hi B_lo + A_hi B_hi,
// with x = hi + lo, accumulated in float32.  Two operand formats:
//   F16  (default): x scaled by a power of two 2^e (one e per proxy row and
//        one per operator, so that the largest magnitude lies in
//        [2^14, 2^15)), hi = fp16(x 2^e), lo = fp16(x 2^e - hi);
//        kind::f16, K = 16 per instruction.  Elements down to 2^-17 of their
//        row's largest keep 22 significant bits; smaller ones an absolute
//        error below 2^-39 of it.  Each offset's accumulator is unscaled by
//        2^-(e_row + e_op) (exact) when it is drained.
//   TF32: hi = tf32(x), lo = tf32(x - hi); kind::tf32, K = 8 per instruction.
// Either way the dropped A_lo B_lo term and the splitting leave a relative
// error near 2^-21 per product.  F16 moves half the bytes and issues half the
// instructions per useful product.  The float32 accumulation inside the
// tensor pipe loses about one unit in the last place per accumulation step,
// so accumulators are drained into a running sum every few offsets (every
// offset for F16, see `group`), which keeps the result within ~1e-6 of float64.
//
// Same product as k_m2l_cheb (reference: FarFieldInteractions / Moment2Local,
// include/compute.hpp:402-508 and 881-914): for a tile of targets of one
// level that share their child type, D[(target, col)][f] = sum over the 189
// offsets o of sum_s proxy_{target+o}[col][s] E_o[f][s].
//
//   M = 128 rows (target, col) of one child type,  N = rf padded to 16,
//   K = (offsets with a source in the tile) x (rs padded to 32).
//
// Operands are K-major, 128-byte-swizzled tiles (rows of 128 bytes: 32 TF32 or
// 64 F16 values; groups of 8 rows 1024 bytes apart), A filled with cp.async
// (zero-fill for absent sources) and B by TMA, in NST stages.  Every wait is bounded: on timeout the kernel sets
// *err, waits (bounded) for its last MMAs, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "fmm.cuh"
#include "tcgen05.cuh"

namespace pbbfmm {

constexpr int TC_M = 128;
constexpr int TC_ROWB = 128;       // bytes of K per stage: one 128-byte swizzle row
constexpr int TC_PRODUCERS = 128;  // warps 0-3: operand loads
constexpr int TC_MMA_WARP = 4;     // warp 4: TMEM allocation, MMA issue (one thread)
constexpr int TC_THREADS = 288;    // + warps 5-8: accumulator drains
constexpr int TC_TMEM_COLS = 512;  // columns allocated (accumulators and running sum)
// Poll limit of the M2L kernel's pipeline waits (stage and accumulator
// barriers inside its main loops), per device; kWaitIters unless a test
// lowers it through pbbfmm_debug_set_pipeline_wait_limit to make those waits
// run out.  The waits for committed copies and MMAs before a CTA exits always
// keep the full bound.
__device__ long long g_pipe_wait_iters = kWaitIters;

struct TcTiles {
  int start[9];  // first tile of each child type; start[8] = total tiles
  int first[8];  // first list position of each type
  int count[8];  // targets of each type
};

// Stage layout: A_hi 16 KB | A_lo 16 KB | B_hi NP*128 | B_lo NP*128, each
// part 1024-byte aligned (NP is a multiple of 16).
__host__ __device__ constexpr int tc_stage_bytes(int NP) { return 2 * 16384 + 2 * NP * 128; }
__host__ __device__ constexpr int tc_smem_bytes(int NP, int nst) {
  return nst * tc_stage_bytes(NP) + 1024;
}

// TMEM columns (512 allocated): accumulator b at b * stride.  With the
// running sum in registers (N <= TC_REG_SUM) four accumulators take turns;
// otherwise two, and when a third region fits (N <= 160) a running sum at
// 2 * stride that the drains update inside TMEM, so that pf is written once;
// beyond that drains add into pf.
__host__ __device__ constexpr int tc_acc_stride(int NP) { return NP <= 160 ? (NP + 31) / 32 * 32 : 256; }
__host__ __device__ constexpr bool tc_sum_in_tmem(int NP) { return NP <= 160; }
// Up to this many columns the running sum lives in the drain threads'
// registers (the CTA is alone on its SM, so they cost no occupancy).
constexpr int TC_REG_SUM = 128;

// One CTA per tile of 128 (target, col) rows of one child type; NST stages.
//   tm_eh, tm_el : [nlev][316][NP] rows of hi / lo of E_o^T (row f holds
//                  E_o[f][s] over s), zero padded to rowb bytes
//   Ph, Pl : proxy hi / lo, row (cell * C + col) of rowb bytes, zero padded
//   pexp   : F16 only: the scale exponent of each proxy row (read for
//            nonempty source cells only, like Ph / Pl)
//   eexp   : F16 only: the scale exponent of each operator of this level
//   pf     : output rows (cell * C + col) of rf floats
// Warp roles:
//   warps 0-3  producers: each warp gathers its 32 rows of A with cp.async and
//              signals the stage's full barrier when its copies land
//              (cp.async.mbarrier.arrive); thread 0 also loads B (the
//              operator tile, hi and lo) with two TMA copies;
//   warp 4     allocates TMEM; one thread waits for full stages, issues the
//              MMAs and commits them to the stage's empty barrier;
//   warps 5-8  drain accumulators into the running sum (TMEM lane quadrant
//              warp % 4).
// NACC TMEM accumulators (four with the register running sum, else two) take
// turns, one per group of `group` consecutive offsets, so every float32
// accumulation chain inside the tensor pipe spans at most `group` offsets;
// an accumulator is reused NACC groups later, once drained (the commit that
// releases a group's accumulator to the drains arrives well after its MMAs
// are issued, so two accumulators left the MMA thread waiting for drains).
//   s_full[s]  : 128 producer arrivals, one per thread, when its copies land
//   s_tfull[s] : the operator tile's TMA bytes (thread 0's expect_tx)
//   s_empty[s] : MMAs reading stage s done (tcgen05.commit)
//   s_accf[b]  : MMAs of accumulator b's group done (tcgen05.commit)
//   s_acce[b]  : accumulator b drained (128 drainer arrivals)
template <int NST, bool F16, bool RSUM>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_m2l_cheb_tc(int rf, int NP, int rowb, const __grid_constant__ CUtensorMap tm_eh,
                  const __grid_constant__ CUtensorMap tm_el, int lvl,
                  const int* __restrict__ typed, TcTiles tt, int C,
                  int lev, const int* __restrict__ sstart, int span, const int* __restrict__ offs,
                  const unsigned char* __restrict__ Ph, const unsigned char* __restrict__ Pl,
                  const int* __restrict__ pexp, const int* __restrict__ eexp,
                  float* __restrict__ pf, int group, int* __restrict__ err) {
  extern __shared__ unsigned char smraw[];
  const int bbytes = NP * 128;
  const int stage_bytes = tc_stage_bytes(NP);
  unsigned char* base = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);
  constexpr int NACC = RSUM ? 4 : 2;  // TMEM accumulators (4 x 128 columns at most)
  __shared__ uint64_t s_full[NST], s_tfull[NST], s_empty[NST], s_accf[NACC], s_acce[NACC];
  __shared__ uint32_t s_tmem;
  __shared__ int s_cell[TC_M];     // target cell of each row, or -1
  __shared__ int s_xyz[TC_M];      // target coordinates, x << 20 | y << 10 | z
  __shared__ uint32_t s_valid[6];  // bit o: some target of the tile has a source at offset o
  __shared__ uint32_t s_tmask[TC_M][6];  // per target of the tile: bit o = source at offset o
  __shared__ int4 s_off[189];      // valid offsets: (ox, oy, oz, operator index)
  __shared__ uint8_t s_oidx[189];  // valid offset q: its index o in the type's list
  __shared__ int s_oexp[189];      // F16: valid offset q: its operator's scale exponent
  __shared__ int s_nvalid;
  __shared__ int s_abort_flag;
  volatile int* s_abort = &s_abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long piters = g_pipe_wait_iters;  // poll limit of the pipeline waits

  // child type of this tile (unrolled so the parameter arrays stay in registers)
  int type = 0, tstart = 0, tlist = 0, tcount = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if ((int)blockIdx.x >= tt.start[i]) {
      type = i;
      tstart = tt.start[i];
      tlist = tt.first[i];
      tcount = tt.count[i];
    }
  const int per_tile = TC_M / C;
  const int tfirst = (blockIdx.x - tstart) * per_tile;
  const int ntile = min(per_tile, tcount - tfirst);
  const int nside = 1 << lev;
  const int* my_offs = offs + type * 189 * 4;

  if (tid < TC_M) {
    const int cell = (tid < per_tile * C && tid / C < ntile) ? typed[tlist + tfirst + tid / C] : -1;
    int x = 0, y = 0, z = 0;
    if (cell >= 0) morton_decode((uint32_t)cell, &x, &y, &z);
    s_cell[tid] = cell;
    s_xyz[tid] = (x << 20) | (y << 10) | z;
  }
  if (tid < 6) s_valid[tid] = 0;
  for (int i = tid; i < TC_M * 6; i += TC_THREADS) (&s_tmask[0][0])[i] = 0;
  if (warp == TC_MMA_WARP) {  // 128 lanes x 512 float32 columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < NST; ++i) {
      mbar_init(&s_full[i], TC_PRODUCERS);
      mbar_init(&s_tfull[i], 1);
      mbar_init(&s_empty[i], 1);
    }
    for (int b = 0; b < NACC; ++b) {
      mbar_init(&s_accf[b], 1);
      mbar_init(&s_acce[b], TC_M);
    }
    s_abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  // which (target, offset) pairs of the tile have a source cell: all threads,
  // one pair per item, independent loads
#pragma unroll 4
  for (int i = tid; i < ntile * 189; i += TC_THREADS) {
    const int tg = i / 189, o = i - tg * 189;
    const int xyz = s_xyz[tg * C];
    const int bx = (xyz >> 20) + my_offs[4 * o], by = ((xyz >> 10) & 1023) + my_offs[4 * o + 1],
              bz = (xyz & 1023) + my_offs[4 * o + 2];
    if (bx < 0 || by < 0 || bz < 0 || bx >= nside || by >= nside || bz >= nside) continue;
    const uint32_t bm = morton_encode(bx, by, bz);
    if (sstart[(int64_t)(bm + 1) * span] > sstart[(int64_t)bm * span]) {
      atomicOr(&s_tmask[tg][o >> 5], 1u << (o & 31));
      atomicOr(&s_valid[o >> 5], 1u << (o & 31));
    }
  }
  __syncthreads();
  if (tid == 0) {
    int nv = 0;
    for (int o = 0; o < 189; ++o)
      if ((s_valid[o >> 5] >> (o & 31)) & 1) {
        s_oidx[nv] = (uint8_t)o;
        s_off[nv++] = make_int4(my_offs[4 * o], my_offs[4 * o + 1], my_offs[4 * o + 2],
                                my_offs[4 * o + 3]);
      }
    s_nvalid = nv;
  }
  __syncthreads();
  if constexpr (F16)
    for (int q = tid; q < s_nvalid; q += TC_THREADS) s_oexp[q] = eexp[s_off[q].w];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int nvalid = s_nvalid;
  const int kchunks = rowb / TC_ROWB;
  const int niter = nvalid * kchunks;
  const int group_iters = max(group, 1) * kchunks;
  const int ngroups = (niter + group_iters - 1) / group_iters;

  if (warp < TC_PRODUCERS / 32) {
    // ---------------------------------------------------------------- producers
    // Lane l copies 16-byte chunk (l & 7) of rows 4 warp + (l >> 3) + 16 i of
    // A (i < 8) and B (i < NP / 16): four 128-byte rows per warp instruction.
    // Lane l also owns A row 4 warp + (l & 3) + 16 (l >> 2): it finds that
    // row's source once per offset (from the tile's source mask: no global
    // load) and the lanes copying the row fetch the result by shuffle.
    const int own = 4 * warp + (lane & 3) + 16 * (lane >> 2);
    const int ocell = s_cell[own], ocol = own % C, otg = own / C;
    const int ox = s_xyz[own] >> 20, oy = (s_xyz[own] >> 10) & 1023, oz = s_xyz[own] & 1023;
    const int ch = lane & 7, r0 = 4 * warp + (lane >> 3);
    const uint32_t soff0 = sw128_off(r0, ch);  // row r0 + 16 i lies 2048 i bytes further
    int cur_q = -1;
    long long cur_row = -1;  // this lane's own row: source row offset or -1
    int tma_last[NST];       // thread 0: last iteration whose TMA went into each stage
#pragma unroll
    for (int i = 0; i < NST; ++i) tma_last[i] = -1;
    for (int j = 0; j < niter; ++j) {
      const int s = j % NST;
      // warp-uniform: the shuffles below are warp-collective
      if (j >= NST &&
          !__all_sync(0xffffffffu, mbar_wait_sleep(&s_empty[s], (j / NST - 1) & 1, s_abort, piters))) {
        *s_abort = 1;
        break;
      }
      const int q = j / kchunks, kc = j - q * kchunks;
      if (q != cur_q) {
        const int o = s_oidx[q];
        cur_row = -1;
        if (ocell >= 0 && ((s_tmask[otg][o >> 5] >> (o & 31)) & 1)) {
          const int4 d = s_off[q];
          cur_row = ((long long)morton_encode(ox + d.x, oy + d.y, oz + d.z) * C + ocol) * rowb;
        }
        cur_q = q;
      }
      unsigned char* st = base + s * stage_bytes;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const long long rr = __shfl_sync(0xffffffffu, cur_row, (lane >> 3) | (i << 2));
        const bool ok = rr >= 0;
        const int64_t off = ok ? rr + kc * TC_ROWB + 16 * ch : 0;
        cp_async16(st + soff0 + 2048 * i, Ph + off, ok ? 16 : 0);
        cp_async16(st + 16384 + soff0 + 2048 * i, Pl + off, ok ? 16 : 0);
      }
      if (tid == 0) {
        // the operator tile (NP rows x 128 bytes, hi and lo) by TMA; x in
        // elements: 64 per 128 bytes for F16, 32 for TF32
        const int y = (lvl * 316 + s_off[q].w) * NP;
        const int x = kc * (F16 ? 64 : 32);
        mbar_arrive_expect_tx(&s_tfull[s], 2u * NP * 128u);
        tma_load_2d(st + 32768, &tm_eh, x, y, &s_tfull[s]);
        tma_load_2d(st + 32768 + bbytes, &tm_el, x, y, &s_tfull[s]);
        tma_last[s] = j;
      }
      cp_async_arrive(&s_full[s]);
    }
    cp_async_wait_all();
    // no TMA may still be writing when the CTA ends: wait (bounded) for the
    // last load issued into each stage
    if (tid == 0)
      for (int s2 = 0; s2 < NST; ++s2)
        if (tma_last[s2] >= 0 && !mbar_wait(&s_tfull[s2], (tma_last[s2] / NST) & 1, nullptr))
          *s_abort = 1;
  } else if (warp == TC_MMA_WARP) {
    // ---------------------------------------------------------------- MMA issue
    if (lane == 0) {
      const uint32_t idesc = F16 ? f16_idesc(TC_M, NP) : tf32_idesc(TC_M, NP);
      const int astride = tc_acc_stride(NP);
      int last = -1;  // last iteration whose MMAs were committed
      for (int it = 0; it < niter; ++it) {
        const int s = it % NST;
        const int g = it / group_iters;
        const bool fresh = it == g * group_iters;
        // accumulator g % NACC is free once the drain of group g - NACC is done
        const int ab = g % NACC;
        if (fresh && g >= NACC &&
            !mbar_wait_sleep(&s_acce[ab], ((g - NACC) / NACC) & 1, s_abort, piters)) {
          *s_abort = 1;
          break;
        }
        if (!mbar_wait_sleep(&s_full[s], (it / NST) & 1, s_abort, piters) ||
            !mbar_wait_sleep(&s_tfull[s], (it / NST) & 1, s_abort, piters)) {
          *s_abort = 1;
          break;
        }
        fence_async_smem();  // the producers' copies, seen through the barrier, to the async proxy
        tc_fence_after();
        const uint32_t a_hi = smem_u32(base + s * stage_bytes), a_lo = a_hi + 16384;
        const uint32_t b_hi = a_hi + 32768, b_lo = b_hi + bbytes;
        const uint32_t d = tmem + (uint32_t)(ab * astride);
        // four K steps of 32 bytes (16 F16 or 8 TF32 values) per 128-byte row
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t off = k * 32;
          if constexpr (F16) {
            tc_mma_f16(d, sw128_desc(a_lo + off), sw128_desc(b_hi + off), idesc,
                       (fresh && k == 0) ? 0u : 1u);
            tc_mma_f16(d, sw128_desc(a_hi + off), sw128_desc(b_lo + off), idesc, 1u);
            tc_mma_f16(d, sw128_desc(a_hi + off), sw128_desc(b_hi + off), idesc, 1u);
          } else {
            tc_mma_tf32(d, sw128_desc(a_lo + off), sw128_desc(b_hi + off), idesc,
                        (fresh && k == 0) ? 0u : 1u);
            tc_mma_tf32(d, sw128_desc(a_hi + off), sw128_desc(b_lo + off), idesc, 1u);
            tc_mma_tf32(d, sw128_desc(a_hi + off), sw128_desc(b_hi + off), idesc, 1u);
          }
        }
        tc_commit(&s_empty[s]);
        if (it + 1 == niter || it + 1 == (g + 1) * group_iters) tc_commit(&s_accf[ab]);
        last = it;
      }
      // Before the TMEM is freed: MMAs complete in order, so the last commit
      // covers all of them (waited for even after an abort, still bounded).
      if (last >= 0 && !mbar_wait(&s_empty[last % NST], (last / NST) & 1, nullptr)) *s_abort = 1;
    }
    __syncwarp();
  } else {
    // ---------------------------------------------------------------- drainers
    const int row = 32 * (warp & 3) + lane;  // TMEM lane quadrant of this warp
    const int cell = s_cell[row];
    float* dst = cell >= 0 ? pf + ((int64_t)cell * C + row % C) * rf : nullptr;
    const uint32_t lane_base = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const int astride = tc_acc_stride(NP);
    const bool tsum = tc_sum_in_tmem(NP);
    const uint32_t sum_base = lane_base + (uint32_t)(2 * astride);
    // F16 (one offset per group): the unscaling exponent of this row at offset
    // q is e_op + e_row of its source.  The row's exponent is loaded two
    // offsets ahead, unconditionally (index 0 when the row has no source at q,
    // the flag then marks it unused), so that no instruction waits for the
    // load before the offset's drain.
    const int rcol = row % C;
    const int rx = s_xyz[row] >> 20, ry = (s_xyz[row] >> 10) & 1023, rz = s_xyz[row] & 1023;
    const int rtg = row / C;
    auto has_src = [&](int q) -> bool {
      if (!F16 || q >= nvalid || cell < 0) return false;
      const int oi = s_oidx[q];
      return (s_tmask[rtg][oi >> 5] >> (oi & 31)) & 1;
    };
    auto src_row = [&](int q, bool ok) -> int64_t {
      if (!ok) return 0;
      const int4 o = s_off[q];
      return (int64_t)morton_encode(rx + o.x, ry + o.y, rz + o.z) * C + rcol;
    };
    bool v1 = has_src(0), v2 = has_src(1);
    int x1 = F16 ? pexp[src_row(0, v1)] : 0, x2 = F16 && nvalid > 1 ? pexp[src_row(1, v2)] : 0;
    float rsum[RSUM ? TC_REG_SUM : 1];  // running sum (RSUM: NP <= TC_REG_SUM)
#pragma unroll
    for (int i = 0; i < (RSUM ? TC_REG_SUM : 1); ++i) rsum[i] = 0.f;
    for (int g = 0; g < ngroups; ++g) {
      const int b = g % NACC;
      // the unscaling 2^-e, e = e_op + e_row, as two exact powers of two
      // 2^-e1 2^-e2 with e1 in [-126, 126] (a normal number) and the rest in
      // e2 (normal or subnormal): a sum beyond one float's exponent range
      // still scales correctly as long as the result itself is a normal
      // number; rows without a source are zero (any scale)
      const int e = v1 ? s_oexp[g] + min(max(x1, -256), 256) : 0;
      const int e1 = min(max(e, -126), 126), e2 = min(max(e - e1, -126), 149);
      const float sc = __int_as_float((127 - e1) << 23);
      const float sc2 = e2 <= 126 ? __int_as_float((127 - e2) << 23) : __int_as_float(1 << (149 - e2));
      v1 = v2;
      x1 = x2;
      v2 = has_src(g + 2);
      if (F16 && g + 2 < nvalid) x2 = pexp[src_row(g + 2, v2)];
      // warp-uniform: the TMEM loads below are warp-collective
      if (!__all_sync(0xffffffffu, mbar_wait_sleep(&s_accf[b], (g / NACC) & 1, s_abort, piters))) {
        *s_abort = 1;
        break;
      }
      tc_fence_after();
      if constexpr (RSUM) {
        // batches of 16 columns (one wait each) added into the register sum;
        // the accumulator is released once its last batch is in registers
#pragma unroll
        for (int c = 0; c < TC_REG_SUM / 16; ++c) {
          if (c * 16 >= NP) break;
          uint32_t r[16];
          tc_ld16_wait(lane_base + (uint32_t)(b * astride + c * 16), r);
          if ((c + 1) * 16 >= NP) {
            tc_fence_before();
            mbar_arrive(&s_acce[b]);
          }
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float x = __uint_as_float(r[i]);
            rsum[c * 16 + i] = F16 ? fmaf(x * sc, sc2, rsum[c * 16 + i]) : rsum[c * 16 + i] + x;
          }
        }
        continue;
      } else {
      const bool final_group = g + 1 == ngroups;
      float v[16], u[16];
      for (int n0 = 0; n0 < NP; n0 += 16) {
        tc_ld16(lane_base + (uint32_t)(b * astride + n0), v);
        if constexpr (F16) {
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] = v[i] * sc * sc2;  // exact unless the result is subnormal
        }
        if (tsum) {
          if (g > 0) {
            tc_ld16(sum_base + (uint32_t)n0, u);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] += u[i];
          }
          if (!final_group) {
            tc_st16(sum_base + (uint32_t)n0, v);
          } else if (dst) {
#pragma unroll
            for (int i = 0; i < 16; ++i)
              if (n0 + i < rf) dst[n0 + i] = v[i];
          }
        } else if (dst) {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (n0 + i < rf) dst[n0 + i] = g == 0 ? v[i] : dst[n0 + i] + v[i];
        }
      }
      if (tsum && !final_group) tc_wait_st();
      tc_fence_before();
      mbar_arrive(&s_acce[b]);
      }
    }
    if constexpr (RSUM) {
      if (dst)
#pragma unroll
        for (int i = 0; i < TC_REG_SUM; ++i)
          if (i < rf) dst[i] = rsum[i];
    } else if (ngroups == 0 && dst) {  // no source in any interaction list of the tile
      for (int n = 0; n < rf; ++n) dst[n] = 0.f;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *s_abort && err) atomicExch(err, 1);
  if (warp == TC_MMA_WARP) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(TC_TMEM_COLS)
                 : "memory");
  }
}

// Split the proxies of the listed source cells into TF32 hi / lo rows of KP
// floats (zero padded from rs): thread per (row, k).  (TF32 operands.)
__global__ void k_split_proxy(const int* __restrict__ cells, int64_t nrows, int C, int rs, int KP,
                              const float* __restrict__ proxy, float* __restrict__ ph,
                              float* __restrict__ pl) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nrows * KP) return;
  const int64_t r = e / KP;
  const int k = (int)(e - r * KP);
  const int64_t row = (int64_t)cells[r / C] * C + r % C;
  const float v = k < rs ? proxy[row * rs + k] : 0.f;
  const float h = to_tf32(v);
  ph[row * KP + k] = h;
  pl[row * KP + k] = to_tf32(v - h);
}

// F16 operands: split the proxies of the listed source cells into scaled F16
// hi / lo rows of KP values (zero padded from rs) and the row's exponent e,
// chosen so that the row's largest |x| 2^e lies in [2^14, 2^15) (e = 0 for a
// zero row): one warp per row.
__global__ void k_split_proxy_f16(const int* __restrict__ cells, int64_t nrows, int C, int rs,
                                  int KP, const float* __restrict__ proxy, __half* __restrict__ ph,
                                  __half* __restrict__ pl, int* __restrict__ pexp) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= nrows) return;  // uniform over the warp
  const int64_t row = (int64_t)cells[r / C] * C + r % C;
  const float* x = proxy + row * rs;
  float m = 0.f;
  for (int k = lane; k < rs; k += 32) m = fmaxf(m, fabsf(x[k]));
#pragma unroll
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int e = m > 0.f ? 15 - exponent_of(m) : 0;  // m in [2^(k2-1), 2^k2)
  for (int k = lane; k < KP; k += 32) {
    const float v = k < rs ? scale2(x[k], e) : 0.f;
    const __half h = __float2half_rn(v);
    ph[row * KP + k] = h;
    pl[row * KP + k] = __float2half_rn(v - __half2float(h));
  }
  if (lane == 0) pexp[row] = e;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links no driver library).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map over an operator half (rows of KP values, nrows rows): boxes of
// NP rows x 128 bytes (32 TF32 or 64 F16 values), 128-byte swizzle (the
// layout the MMA descriptors read).
static int operator_tensor_map(CUtensorMap* m, const void* base, bool f16, int NP, int KP,
                               int64_t nrows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return PBBFMM_ERR_CUDA;
  }
  const int esize = f16 ? 2 : 4;
  const cuuint64_t dims[2] = {(cuuint64_t)KP, (cuuint64_t)nrows};
  const cuuint64_t strides[1] = {(cuuint64_t)KP * esize};
  const cuuint32_t box[2] = {(cuuint32_t)(TC_ROWB / esize), (cuuint32_t)NP};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(m, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, const_cast<void*>(base), dims,
                         strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for the tensor-core operator tiles");
    return PBBFMM_ERR_CUDA;
  }
  return PBBFMM_OK;
}

// Offsets per TMEM accumulation chain (PBBFMM_TC_GROUP overrides the TF32
// default): one offset when the running sum stays in TMEM (drains then cost
// nothing measurable), four when drains add into pf in global memory.  F16
// operands always drain every offset (each has its own scale).
static int tc_group(int NP, bool f16) {
  if (f16) return 1;
  const char* e = getenv("PBBFMM_TC_GROUP");
  const int g = e ? atoi(e) : (tc_sum_in_tmem(NP) ? 1 : 4);
  return g < 1 ? 1 : (g > 189 ? 189 : g);
}

bool tc_eligible(const pbbfmm_tree* t) {
  return t->p.use_chebyshev && t->use_tc && t->tc.eth && t->tc.eh16 && t->tc.np > 0 &&
         t->tc.np <= kTcMaxN;
}

template <int NST, bool F16, bool RSUM>
static int launch_tc(const pbbfmm_tree* t, unsigned tiles, int smem, int rf, int NP, int rowb,
                     const CUtensorMap& tm_h, const CUtensorMap& tm_l, int lvl, const int* typed,
                     const TcTiles& tt, int C, int l, int span, const unsigned char* ph,
                     const unsigned char* pl, const int* pexp, float* pf, cudaStream_t st) {
  PB_CUDA(cudaFuncSetAttribute(k_m2l_cheb_tc<NST, F16, RSUM>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_m2l_cheb_tc<NST, F16, RSUM><<<tiles, TC_THREADS, smem, st>>>(
      rf, NP, rowb, tm_h, tm_l, lvl, typed, tt, C, l, t->ws.sstart.as<int>(), span, t->d_offs,
      ph, pl, pexp, t->tc.eexp + (int64_t)lvl * 316, pf, tc_group(NP, F16), t->d_tc_err);
  PB_LAUNCH("m2l_cheb_tc");
  return PBBFMM_OK;
}

// Level l of the tensor-core M2L: split the proxies, then the MMA kernel.
// proxy / pf are the level's float arrays (rows cell * C + col).
int run_m2l_cheb_tc_level(pbbfmm_tree* t, int C, int l, int lvl, const float* proxy, float* pf,
                          cudaStream_t st) {
  const int L = t->p.tree_level, rf = t->ops.rf, rs = t->ops.rs;
  const bool f16 = t->tc_fmt == PBBFMM_TC_F16;
  const int NP = t->tc.np, KP = f16 ? t->tc.kp16 : t->tc.kp, esize = f16 ? 2 : 4;
  const int rowb = KP * esize;  // a multiple of 128
  Workspace& ws = t->ws;
  const int* lists = ws.lists.as<int>();
  if (C > TC_M) {
    set_error("tensor-core M2L takes at most 128 columns per block");
    return PBBFMM_ERR_UNSUPPORTED;
  }
  // hi rows | lo rows | (F16) row exponents, every cell of the level
  const int64_t rows = cells_at(l) * C, pbytes = rows * rowb;
  if (int rc = grow(ws.tc_proxy, 2 * pbytes + (f16 ? rows * (int64_t)sizeof(int) : 0))) return rc;
  unsigned char* ph = ws.tc_proxy.as<unsigned char>();
  unsigned char* pl = ph + pbytes;
  int* pexp = f16 ? reinterpret_cast<int*>(pl + pbytes) : nullptr;
  const int ns = t->lists.nsrc[l];
  if (ns > 0) {
    const int64_t nrows = (int64_t)ns * C;
    if (int rc = kt_begin(t, KS_M2L_SPLIT, st)) return rc;
    if (f16)
      k_split_proxy_f16<<<(unsigned)((nrows * 32 + 255) / 256), 256, 0, st>>>(
          lists + t->lists.src_off[l], nrows, C, rs, KP, proxy, reinterpret_cast<__half*>(ph),
          reinterpret_cast<__half*>(pl), pexp);
    else
      k_split_proxy<<<(unsigned)((nrows * KP + 255) / 256), 256, 0, st>>>(
          lists + t->lists.src_off[l], nrows, C, rs, KP, proxy, reinterpret_cast<float*>(ph),
          reinterpret_cast<float*>(pl));
    PB_LAUNCH("m2l_split");
    if (int rc = kt_end(t, st)) return rc;
  }
  TcTiles tt;
  const int per_tile = TC_M / C;
  int tiles = 0;
  for (int ty = 0; ty < 8; ++ty) {
    tt.start[ty] = tiles;
    tt.first[ty] = t->lists.ntyp[l][ty];
    tt.count[ty] = t->lists.ntyp[l][ty + 1] - t->lists.ntyp[l][ty];
    tiles += (tt.count[ty] + per_tile - 1) / per_tile;
  }
  tt.start[8] = tiles;
  if (tiles == 0) return PBBFMM_OK;
  // three stages when they fit in shared memory next to the static arrays
  const int nst = tc_smem_bytes(NP, 3) + 8192 <= 232448 ? 3 : 2;
  const int smem = tc_smem_bytes(NP, nst);
  CUtensorMap tm_h, tm_l;
  const int64_t nrows = (int64_t)t->ops.nlev * 316 * NP;
  const void* eh = f16 ? (const void*)t->tc.eh16 : (const void*)t->tc.eth;
  const void* el = f16 ? (const void*)t->tc.el16 : (const void*)t->tc.etl;
  if (int rc = operator_tensor_map(&tm_h, eh, f16, NP, KP, nrows)) return rc;
  if (int rc = operator_tensor_map(&tm_l, el, f16, NP, KP, nrows)) return rc;
  if (int rc = kt_begin(t, KS_M2L, st)) return rc;
  const int* typed = lists + t->lists.typ_off[l];
  const int span = (int)cells_at(L - l);
  // register running sum up to TC_REG_SUM columns (three stages always fit there)
  const bool rsum = NP <= TC_REG_SUM && nst == 3;
#define PB_TC_LAUNCH(NSTV, F, R)                                                              \
  launch_tc<NSTV, F, R>(t, tiles, smem, rf, NP, rowb, tm_h, tm_l, lvl, typed, tt, C, l, span, \
                        ph, pl, pexp, pf, st)
  int rc;
  if (f16)
    rc = rsum ? PB_TC_LAUNCH(3, true, true)
              : (nst == 3 ? PB_TC_LAUNCH(3, true, false) : PB_TC_LAUNCH(2, true, false));
  else
    rc = rsum ? PB_TC_LAUNCH(3, false, true)
              : (nst == 3 ? PB_TC_LAUNCH(3, false, false) : PB_TC_LAUNCH(2, false, false));
#undef PB_TC_LAUNCH
  if (rc) return rc;
  return kt_end(t, st);
}

// ------------------------------------------------------------------------
// M2L pre / post transforms on the tensor cores, same split as the F16 M2L:
//   Out[row_n][m] = alpha oscale[m] sum_k W[m][k] bscale[k] X[row_n][k],  m < M,
// for the columns n < ncols, row_n = cells[n / C] * C + n % C (reference:
// UpwardPass tail, include/compute.hpp:373-396, and the Moment2Local
// post-transform, include/compute.hpp:881-914).  One CTA of 128 threads per
// 128 columns; thread t owns column n = 128 blockIdx.x + t:
//   A = its row of X (times bscale), scaled by its own power of two and split
//       into F16 hi / lo, written to shared memory (SW128 K-major) one K chunk
//       of 64 at a time;
//   B = W (mp rows, pre-split with one exponent per level), by TMA;
//   D[n][m] (128 lanes x mp columns, TMEM) accumulates three products per
//       K step; thread t drains lane t, unscales and writes row_n of Out.
// Chunks run one after another (one stage); two CTAs share an SM (one when
// mp > 256: then each product is two MMAs of N = mp / 2 and the CTA holds all
// 512 TMEM columns).  When
// mp <= 128 each chunk's accumulator is drained into a register sum (the
// tensor pipe's float32 accumulation loses about one ulp per step, so chains
// stay 12 steps long); otherwise the chunks accumulate in TMEM.
constexpr int CG_TC_THREADS = 128;

template <bool BSCALE, bool OSCALE>
__global__ void __launch_bounds__(CG_TC_THREADS, 1)
    k_colgemm_tc(int M, int mp, int K, int kp, const __grid_constant__ CUtensorMap tm_wh,
                 const __grid_constant__ CUtensorMap tm_wl, int wrow0, int wexp,
                 const int* __restrict__ cells, int ncols, int C, const float* __restrict__ X,
                 const float* __restrict__ bscale, float* __restrict__ Out,
                 const float* __restrict__ oscale, float alpha, int* __restrict__ err) {
  extern __shared__ unsigned char smraw[];
  unsigned char* base = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);
  const int nh = mp > 256 ? 2 : 1;             // MMAs (and TMA boxes) per product
  const int hn = mp / nh;                      // their N (a multiple of 16)
  const uint32_t tcols = mp > 256 ? 512 : 256;  // TMEM columns
  unsigned char* a_hi = base;
  unsigned char* a_lo = base + 16384;
  unsigned char* b_hi = base + 32768;
  unsigned char* b_lo = b_hi + mp * 128;
  __shared__ uint64_t s_tma, s_mma;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int n = blockIdx.x * CG_TC_THREADS + tid;
  const bool valid = n < ncols;
  const int64_t row = valid ? (int64_t)cells[n / C] * C + n % C : 0;
  const float* xr = X + row * K;
  // 16-byte loads when rows (K floats, from 16-byte aligned level bases) are
  // 16-byte aligned
  const bool vec4 = (K & 3) == 0;
  // this column's exponent: max |bscale x| 2^e in [2^14, 2^15)
  float mx = 0.f;
  if (valid) {
    if (vec4) {
      const float4* x4 = reinterpret_cast<const float4*>(xr);
#pragma unroll 4
      for (int k4 = 0; k4 < K / 4; ++k4) {
        float4 v = x4[k4];
        if (BSCALE) {
          const float4 b = reinterpret_cast<const float4*>(bscale)[k4];
          v.x *= b.x, v.y *= b.y, v.z *= b.z, v.w *= b.w;
        }
        mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
      }
    } else {
      for (int k = 0; k < K; ++k) mx = fmaxf(mx, fabsf(BSCALE ? xr[k] * bscale[k] : xr[k]));
    }
  }
  const int e = mx > 0.f ? 15 - exponent_of(mx) : 0;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&s_tma, 1);
    mbar_init(&s_mma, 1);
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t idesc = f16_idesc(TC_M, hn);
  const int nchunks = kp / 64;
  const bool rdrain = mp <= 128;  // uniform
  const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
  float racc[128];  // register sum of the drained chunks (rdrain)
#pragma unroll
  for (int i = 0; i < 128; ++i) racc[i] = 0.f;
  int last_tma = -1;  // thread 0: the last chunk whose TMA was issued
  for (int c = 0; c < nchunks; ++c) {
    // A chunk: this column's 64 values (zero past K), scaled and split
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t h[4], l[4];
      float v8[8];
      const int kb = c * 64 + j * 8;
      if (vec4) {  // two 16-byte loads; a block of 4 lies wholly below or above K
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int k = kb + 4 * q;
          float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
          if (valid && k < K) {
            x = *reinterpret_cast<const float4*>(xr + k);
            if (BSCALE) {
              const float4 b = *reinterpret_cast<const float4*>(bscale + k);
              x.x *= b.x, x.y *= b.y, x.z *= b.z, x.w *= b.w;
            }
          }
          v8[4 * q] = scale2(x.x, e), v8[4 * q + 1] = scale2(x.y, e);
          v8[4 * q + 2] = scale2(x.z, e), v8[4 * q + 3] = scale2(x.w, e);
        }
      } else {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = kb + u;
          v8[u] = (valid && k < K) ? scale2(BSCALE ? xr[k] * bscale[k] : xr[k], e) : 0.f;
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float v[2] = {v8[2 * i], v8[2 * i + 1]};
        const __half2 vh = __floats2half2_rn(v[0], v[1]);
        const float2 vf = __half22float2(vh);
        const __half2 vl = __floats2half2_rn(v[0] - vf.x, v[1] - vf.y);
        h[i] = *reinterpret_cast<const uint32_t*>(&vh);
        l[i] = *reinterpret_cast<const uint32_t*>(&vl);
      }
      *reinterpret_cast<uint4*>(a_hi + sw128_off(tid, j)) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(a_lo + sw128_off(tid, j)) = make_uint4(l[0], l[1], l[2], l[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // to the tensor pipe
    if (tid == 0) {
      mbar_arrive_expect_tx(&s_tma, 2u * (uint32_t)mp * 128u);
      for (int h = 0; h < nh; ++h) {  // boxes of hn rows
        tma_load_2d(b_hi + h * hn * 128, &tm_wh, c * 64, wrow0 + h * hn, &s_tma);
        tma_load_2d(b_lo + h * hn * 128, &tm_wl, c * 64, wrow0 + h * hn, &s_tma);
      }
      last_tma = c;
    }
    __syncthreads();
    if (tid == 0) {
      if (mbar_wait(&s_tma, c & 1, nullptr)) {
        tc_fence_after();
        const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
        const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
        for (int h = 0; h < nh; ++h) {  // D columns [h hn, (h + 1) hn)
          const uint32_t d = tmem + (uint32_t)(h * hn), bo = (uint32_t)(h * hn * 128);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint32_t off = k * 32;
            tc_mma_f16(d, sw128_desc(al + off), sw128_desc(bh + bo + off), idesc,
                       ((c > 0 && !rdrain) || k > 0) ? 1u : 0u);
            tc_mma_f16(d, sw128_desc(ah + off), sw128_desc(bl + bo + off), idesc, 1u);
            tc_mma_f16(d, sw128_desc(ah + off), sw128_desc(bh + bo + off), idesc, 1u);
          }
        }
        tc_commit(&s_mma);
      } else {
        s_fail = 1;
        mbar_arrive(&s_mma);  // release the others; the result is not used
      }
    }
    // the chunk's MMAs (or the failure) before its shared memory is rewritten
    if (!mbar_wait(&s_mma, c & 1, nullptr)) s_fail = 1;
    __syncthreads();
    if (s_fail) break;
    if (rdrain) {
      // all lanes (warp-collective loads); done before the next chunk's MMAs
      // are issued (the barrier at the top of the next chunk orders them)
      tc_fence_after();
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (q * 16 >= mp) break;
        uint32_t r[16];
        tc_ld16_wait(lane_base + (uint32_t)(q * 16), r);
#pragma unroll
        for (int i = 0; i < 16; ++i) racc[q * 16 + i] += __uint_as_float(r[i]);
      }
      tc_fence_before();
    }
  }
  if (s_fail) {
    // no copy or MMA may still be running when the CTA ends: wait (bounded)
    // once more for the last chunk's
    if (tid == 0 && last_tma >= 0) {
      mbar_wait(&s_tma, last_tma & 1, nullptr);
      mbar_wait(&s_mma, last_tma & 1, nullptr);
    }
    if (tid == 0 && err) atomicExch(err, 1);
  } else {
    // every lane of the warp takes part in the (warp-collective) TMEM loads;
    // only valid columns store
    tc_fence_after();
    // the unscaling 2^-(e + wexp) as two exact power-of-two factors applied
    // one after the other (never multiplied together, which could leave the
    // float range although the result lies inside it), then alpha
    const int kt = -(e + wexp), k1 = min(max(kt, -126), 127), k2 = min(max(kt - k1, -149), 127);
    const float sc = exp2i(k1), sc2 = exp2i(k2);
    float* o = valid ? Out + row * M : nullptr;
    if (rdrain) {
      if (o) {
#pragma unroll
        for (int m = 0; m < 128; ++m)
          if (m < M) o[m] = racc[m] * sc * sc2 * alpha * (OSCALE ? oscale[m] : 1.f);
      }
    } else {
      for (int m0 = 0; m0 < mp; m0 += 16) {
        uint32_t r[16];
        tc_ld16_wait(lane_base + (uint32_t)m0, r);
        if (o) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int m = m0 + i;
            if (m < M) o[m] = __uint_as_float(r[i]) * sc * sc2 * alpha * (OSCALE ? oscale[m] : 1.f);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(tcols)
                 : "memory");
  }
}

// Tensor cores when the output width fits two MMAs (mp <= 512) and no TMEM
// accumulation chain is longer than two K chunks (24 steps): either the
// chunks are drained into registers (mp <= 128) or there are at most two
// (K <= 128).  Longer chains would add ~1e-6 of accumulation error.
bool colgemm_tc_eligible(const pbbfmm_tree* t, bool post) {
  if (!t->p.use_chebyshev || !t->use_tc || t->ops.nlev > 32) return false;
  const TcOps& o = t->tc;
  const int mp = post ? o.u_mp : o.vt_mp, kp = post ? o.u_kp : o.vt_kp;
  if (!(post ? o.uh : o.vth) || mp > 512) return false;
  return mp <= 128 || kp <= 128;
}

int run_colgemm_tc(pbbfmm_tree* t, bool post, int lvl, const int* cells, int ncols, int C,
                   const float* X, float* Out, float alpha, cudaStream_t st) {
  if (ncols <= 0) return PBBFMM_OK;
  const TcOps& o = t->tc;
  const int M = post ? t->n3 : t->ops.rs, K = post ? t->ops.rf : t->n3;
  const int mp = post ? o.u_mp : o.vt_mp, kp = post ? o.u_kp : o.vt_kp;
  const uint16_t* wh = post ? o.uh : o.vth;
  const uint16_t* wl = post ? o.ul : o.vtl;
  const int wexp = post ? o.u_exp[lvl] : o.vt_exp[lvl];
  CUtensorMap tm_h, tm_l;
  const int64_t nrows = (int64_t)t->ops.nlev * mp;
  const int hn = mp > 256 ? mp / 2 : mp;  // rows per TMA box
  if (int rc = operator_tensor_map(&tm_h, wh, true, hn, kp, nrows)) return rc;
  if (int rc = operator_tensor_map(&tm_l, wl, true, hn, kp, nrows)) return rc;
  // at least 78 KB (114 KB when a CTA takes all 512 TMEM columns), so that
  // the CTAs sharing an SM always find their TMEM columns free and no
  // allocation waits for another CTA
  const int smem = std::max(32768 + 2 * mp * 128 + 1024, (mp > 256 ? 114 : 78) * 1024);
  const unsigned grid = (unsigned)((ncols + CG_TC_THREADS - 1) / CG_TC_THREADS);
  const float* Kw = t->f_Kw;
  if (post) {
    PB_CUDA(cudaFuncSetAttribute(k_colgemm_tc<false, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_colgemm_tc<false, true><<<grid, CG_TC_THREADS, smem, st>>>(
        M, mp, K, kp, tm_h, tm_l, lvl * mp, wexp, cells, ncols, C, X, nullptr, Out, Kw, alpha,
        t->d_tc_err);
  } else {
    PB_CUDA(cudaFuncSetAttribute(k_colgemm_tc<true, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_colgemm_tc<true, false><<<grid, CG_TC_THREADS, smem, st>>>(
        M, mp, K, kp, tm_h, tm_l, lvl * mp, wexp, cells, ncols, C, X, Kw, Out, nullptr, alpha,
        t->d_tc_err);
  }
  PB_LAUNCH(post ? "m2l_post_tc" : "m2l_pre_tc");
  return PBBFMM_OK;
}


}  // namespace pbbfmm

extern "C" int pbbfmm_debug_set_pipeline_wait_limit(int device, long long polls) {
  using namespace pbbfmm;
  int cur = 0;
  PB_CUDA(cudaGetDevice(&cur));
  if (device >= 0 && device != cur) PB_CUDA(cudaSetDevice(device));
  const long long v = polls > 0 ? polls : kWaitIters;
  const cudaError_t e = cudaMemcpyToSymbol(g_pipe_wait_iters, &v, sizeof(v));
  const int rc = e == cudaSuccess ? set_unif_tc_wait_limit(v) : PBBFMM_OK;
  if (device >= 0 && device != cur) cudaSetDevice(cur);
  if (e != cudaSuccess) return cuda_status(e, "set pipeline wait limit");
  return rc;
}
