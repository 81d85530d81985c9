// Frequency-domain M2L of the uniform path on the tensor cores (mixed
// precision), for levels with at least 16 parents per side and column groups
// of 8.
//
// Reference: FarFieldInteractions / FrequencyProduct, include/compute.hpp:
// 488-544 and 930-943: for each frequency k, each target child t of a parent
// P accumulates E_k[o] x_k(s) over the source children s of P's 27
// neighbour parents whose offset o (in child widths) is far.  Written per
// parent offset D in {-1, 0, 1}^3 this is a block product
//     y_k(P)[t] += sum_s B_{k,D}[t][s] x_k(P + D)[s],
// with B_{k,D} an 8 x 8 complex block that is zero where (t, s) are near
// neighbours.  In real form (x = re + i im) the block is 16 x 16, and the
// whole step is a GEMM whose rows are (parent, column) pairs.
//
// Tiling.  A CTA owns 8 target lines of 16 parents (z-lines at x = bx,
// y = y0..y0+7, z = z0..z0+15) and a chunk of frequencies.  For a frequency
// it walks the 3 x 10 source lines (x = bx-1..bx+1, y = y0-1..y0+8) of 18
// parents (z0-1..z0+16).  A source line is staged in shared memory as the
// A operand, 144 rows (z, column) x K = 16 (child, re/im), split into F16 hi
// and lo parts; a window of 128 of its rows, shifted by D_z parents, lines up
// with the rows of the target lines.  The operator tiles B for one D_x and D_z
// stack the three D_y in N (96 rows: D_y x (hi, lo) x (child, re/im)), so one
// MMA serves the three target lines y - D_y at once; their TMEM accumulators
// (32 columns per line: the products with B hi, then with B lo) are adjacent.
// Each (line, D_z) issues two tcgen05.mma kind::f16 (A hi and A lo, K = 16):
// D = A_hi B + A_lo B = (A_hi + A_lo)(B_hi + B_lo), accumulated in float32.
//
// Scaling.  F16 holds 11 significant bits between 2^-14 and 2^16, so both
// operands are scaled by powers of two before the split: the spectra of
// column c at frequencies (k1, k23) by 2^sA(k23, c mod 8), with sA chosen from
// a bound on their magnitude over the level's cells and k1 (recorded by the
// forward FFT, within a small factor of the largest) so that it lies in
// [2^14, 2^15); the operator tiles of a frequency by 2^sB(k) from their
// largest entry.  hi = fp16(x 2^s), lo = fp16(x 2^s - hi)
// keep 22 significant bits for values down to 2^-17 of the scale's maximum
// and an absolute error below 2^-39 of it for smaller ones.  A TMEM row holds
// one column only (source and target rows share the column), so one factor
// 2^-(sA + sB) per drained row and frequency undoes the scaling exactly.
//
// Roles (448 threads): warps 0-8 produce the A operand, one (K plane, row)
// task per thread: each thread loads its four spectra values and the
// children's occupancy into a register ring six lines ahead (so the loads of
// several lines are in flight), then scales, splits and stores them into an
// A stage; thread 0 also loads each frequency's operator tiles by a bulk
// copy.  One thread of warp 9 issues the MMAs; warps 10-13 drain the
// accumulators (two TMEM sets, alternating by frequency), write the target
// spectra and zero the accumulators.  Producer warps run on their own,
// ordered by mbarriers only (no block-wide barrier per line).  Every wait is
// bounded; on timeout the kernel sets *err, waits (bounded) for its issued
// copies and MMAs, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "fmm.cuh"
#include "tcgen05.cuh"

namespace pbbfmm {

constexpr int UT_BY = 8;                   // target lines per CTA (along y)
constexpr int UT_LINE = 16;                // parents per target line (along z)
constexpr int UT_SRCZ = UT_LINE + 2;       // parents per source line
constexpr int UT_ROWS = UT_SRCZ * 8;       // A rows of a source line: (z, column)
constexpr int UT_SRC_LINES = 3 * (UT_BY + 2);  // source lines per frequency
constexpr int UT_APLANE = UT_ROWS * 16;    // bytes of one K core plane (8 F16) of A
constexpr int UT_APART = 2 * UT_APLANE;    // hi or lo part of a stage (K = 16)
constexpr int UT_ASTAGE = 2 * UT_APART;
constexpr int UT_NST = 8;                  // A stages
constexpr int UT_RING = 6;                 // lines whose loads run ahead of the split (registers)
constexpr int UT_BROWS = 96;               // B rows of one (D_x, D_z) tile
constexpr int UT_BPLANE = UT_BROWS * 16;
constexpr int UT_BTILE = 2 * UT_BPLANE;
constexpr int UT_BFREQ = 9 * UT_BTILE;     // operator tiles of one frequency (bytes)
constexpr int UT_PWARPS = 9;               // producer warps: one task per thread
constexpr int UT_PRODUCERS = 32 * UT_PWARPS;
// Warp roles: producers 0-8, the MMA warp 9, drains 10-13.  (Moving the MMA
// warp to an SM sub-partition of its own, with the producers on the other
// three, measured 3 % slower.)
constexpr int UT_THREADS = 14 * 32;
constexpr int UT_MMA_WARP = 9;
constexpr int UT_DRAIN0 = 10 * 32;  // the drain thread that waits and signals
enum { UT_PRODUCER = 0, UT_MMA = 1, UT_DRAIN = 2, UT_IDLE = 3 };
__device__ __forceinline__ int ut_role(int warp, int* pidx) {
  *pidx = warp;
  return warp < UT_PWARPS ? UT_PRODUCER : warp == UT_MMA_WARP ? UT_MMA : UT_DRAIN;
}
constexpr int UT_TMEM_COLS = 512;          // two sets of UT_BY x 32 columns
constexpr int UT_SMEM = UT_NST * UT_ASTAGE + 2 * UT_BFREQ + 1024;
static_assert(2 * UT_BY * 32 == UT_TMEM_COLS, "two accumulator sets fill the TMEM");
static_assert(UT_PRODUCERS == 2 * UT_ROWS, "one split task (K plane, row) per producer thread");
static_assert(UT_SMEM <= 232448, "shared memory of one CTA");

// F16 values (uint16 bit patterns) of the operator tiles per (level, frequency).
constexpr int kUnifTcTileHalves = UT_BFREQ / 2;

// Poll limit of the pipeline waits (see g_pipe_wait_iters in m2l_tc.cu).
__device__ long long g_unif_wait_iters = kWaitIters;

// Barrier among the `n` threads of a role group (named barrier `id`).
__device__ __forceinline__ void group_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}

// OR of `v` over the 128 drain threads (warps 9-12, named barrier 2).
__device__ __forceinline__ bool drains_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, 2, 128, q;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

// 2^s as a float with s = 15 - e for the largest magnitude m = 2^(e-1).. of
// a spectra scale slot (float bits, 0 if every value is zero), so that
// m 2^s lies in [2^14, 2^15); s clamped to the float exponent range.
__device__ __forceinline__ int unif_scale_exp(uint32_t mbits) {
  if (mbits == 0u || (mbits & 0x7f800000u) == 0x7f800000u) return 0;
  return max(-126, min(127, 15 - exponent_of(__uint_as_float(mbits))));
}

__global__ void k_occupancy(const int* __restrict__ start, int span, int64_t ncells,
                            uint8_t* __restrict__ occ) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < ncells) occ[c] = start[(c + 1) * span] > start[c * span] ? 1 : 0;
}

struct UnifTcArgs {
  const float2* X;       // level spectra [k][cell][C]
  float2* Y;             // level target spectra [k][cell][C]
  const uint16_t* tiles;  // [nk][kUnifTcTileHalves] operator tiles of this level (F16)
  const int* bexp;        // [nk] exponent sB of each frequency's tiles
  const uint32_t* amax;   // [nk23][8] largest |spectra| (float bits) per (k23, column mod 8)
  const uint8_t* socc;   // [cell] source cell nonempty
  const uint8_t* tocc;   // [cell] target cell nonempty
  int lev;               // cells 2^lev per side, parents S = 2^(lev-1)
  int C, c0;             // columns of the arrays; first of this group of 8
  int nk, nk23, kchunk, nchunks, nblocks;  // frequencies k = k1 nk23 + k23
  int* err;
};

__device__ __forceinline__ void ut_block(int b, int S, int* bx, int* y0, int* z0) {
  const int nyb = S / UT_BY, nzb = S / UT_LINE;
  *bx = b / (nyb * nzb);
  const int r = b % (nyb * nzb);
  *y0 = (r / nzb) * UT_BY;
  *z0 = (r % nzb) * UT_LINE;
}

__global__ void __launch_bounds__(UT_THREADS, 1) k_m2l_unif_tc(const UnifTcArgs a) {
  extern __shared__ unsigned char smraw[];
  unsigned char* base = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);
  unsigned char* astage = base;                               // UT_NST x (hi | lo)
  unsigned char* bbuf = astage + UT_NST * UT_ASTAGE;          // 2 x operator tiles
  __shared__ uint64_t s_full[UT_NST], s_empty[UT_NST], s_bfull[2], s_bempty[2], s_accf[2],
      s_acce[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_nz[UT_NST];  // stage s holds a nonempty line: its line number + 1
  __shared__ int s_abort_flag;
  volatile int* s_abort = &s_abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int pidx = 0;
  const int role = ut_role(warp, &pidx);
  const long long piters = g_unif_wait_iters;
  const int S = 1 << (a.lev - 1);
  const int64_t ncells = (int64_t)1 << (3 * a.lev);
  const int nitems = a.nblocks * a.nchunks;

  if (role == UT_MMA) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(UT_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < UT_NST; ++i) {
      mbar_init(&s_full[i], UT_PWARPS);  // one arrival per producer warp
      mbar_init(&s_empty[i], 1);         // the MMA commit
      s_nz[i] = 0;
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s_bfull[i], 1);
      mbar_init(&s_bempty[i], 1);
      mbar_init(&s_accf[i], 1);
      mbar_init(&s_acce[i], 1);
    }
    s_abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  // the drain warps zero both accumulator sets before the first MMA
  if (role == UT_DRAIN) {
    const uint32_t lb = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const float z[16] = {};
    for (int c = 0; c < UT_TMEM_COLS; c += 16) tc_st16(lb + (uint32_t)c, z);
    tc_wait_st();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  // The source lines of every frequency of every work item, in the order the
  // MMA thread consumes them: item (block, frequency chunk) round robin over
  // the CTAs, then frequency, then line.
  struct Pos {
    int item, k, sl;
  };
  auto first_k = [&](int item) { return (item / a.nblocks) * a.kchunk; };
  auto end_k = [&](int item) { return min(a.nk, (item / a.nblocks + 1) * a.kchunk); };
  auto advance = [&](Pos& p) {
    if (++p.sl == UT_SRC_LINES) {
      p.sl = 0;
      if (++p.k == end_k(p.item)) {
        p.item += gridDim.x;
        if (p.item < nitems) p.k = first_k(p.item);
      }
    }
  };
  if (role == UT_PRODUCER) {
    // ------------------------------------------------------------ producers
    // Thread ptid's task: K plane kc = ptid / 144 (the children 4 kc ..
    // 4 kc + 3) and row = ptid % 144 = (zpos, column) of every source line.
    // Its four spectra values (8 bytes each; a warp's loads cover four
    // parents x 64 contiguous bytes per child) and the children's occupancy
    // are loaded into registers UT_RING lines ahead of their split, so the
    // loads of several lines are in flight while the warp converts one.
    // Each producer warp runs on its own, ordered by mbarriers: a line is
    // stored once the MMAs of the stage's previous line completed
    // (s_empty), and the MMA thread starts once every warp stored its part
    // (s_full).
    const int ptid = pidx * 32 + lane;
    const int t_kc = ptid / UT_ROWS, t_row = ptid - t_kc * UT_ROWS;
    const int t_z = t_row >> 3, t_col = t_row & 7;
    const int split_dst = t_kc * UT_APLANE + t_row * 16;
    struct Slot {
      float2 v[4];    // children 4 kc + e, column c0 + t_col
      uint32_t occ;   // their occupancy bytes (0 outside the domain)
      uint32_t amax;  // the spectra bound of (k23, t_col)
    };
    Slot ring[UT_RING];
    Pos lp{(int)blockIdx.x, 0, 0};  // the next line to load
    if (lp.item < nitems) lp.k = first_k(lp.item);
    int item_ctx = -1, bx = 0, y0 = 0, k_ctx = -1;
    uint32_t zsp = 0xffffffffu;
    const uint32_t* amax_k = a.amax;
    auto load = [&](Slot& r) {
      if (lp.item != item_ctx) {
        int z0;
        item_ctx = lp.item;
        ut_block(lp.item % a.nblocks, S, &bx, &y0, &z0);
        const int z = z0 - 1 + t_z;
        zsp = (z >= 0 && z < S) ? spread3((uint32_t)z) : 0xffffffffu;
      }
      const int xs = bx + lp.sl / (UT_BY + 2) - 1, ys = y0 + lp.sl % (UT_BY + 2) - 1;
      const bool in = xs >= 0 && xs < S && ys >= 0 && ys < S && zsp != 0xffffffffu;
      if (lp.k != k_ctx) {
        k_ctx = lp.k;
        amax_k = a.amax + 8 * (lp.k % a.nk23) + t_col;
      }
      r.amax = __ldg(amax_k);
      r.occ = 0;
      if (in) {
        const int64_t cell =
            8 * (int64_t)((spread3((uint32_t)xs) << 2) | (spread3((uint32_t)ys) << 1) | zsp) +
            4 * t_kc;
        r.occ = __ldg(reinterpret_cast<const uint32_t*>(a.socc + cell));
        const float2* src = a.X + ((int64_t)lp.k * ncells + cell) * a.C + a.c0 + t_col;
#pragma unroll
        for (int e = 0; e < 4; ++e) r.v[e] = __ldg(src + (int64_t)e * a.C);
      }
      advance(lp);
    };
    // operator tiles: frequency f goes to buffer f % 2; the load for f + 1 is
    // issued by thread 0 in the middle of frequency f (the MMAs of f - 1,
    // the buffer's previous user, are issued by then)
    Pos bnext{(int)blockIdx.x, 0, 0};
    if (bnext.item < nitems) bnext.k = first_k(bnext.item);
    int bissued = 0, last_b = -1;
    auto load_b = [&]() -> bool {  // ptid 0 only
      if (bnext.item >= nitems) return true;
      const int fb = bissued & 1;
      if (bissued >= 2 && !mbar_wait(&s_bempty[fb], ((bissued - 2) >> 1) & 1, s_abort, piters))
        return false;
      mbar_arrive_expect_tx(&s_bfull[fb], UT_BFREQ);
      bulk_load(bbuf + fb * UT_BFREQ, a.tiles + (int64_t)bnext.k * kUnifTcTileHalves, UT_BFREQ,
                &s_bfull[fb]);
      last_b = bissued++;
      if (++bnext.k == end_k(bnext.item)) {
        bnext.item += gridDim.x;
        if (bnext.item < nitems) bnext.k = first_k(bnext.item);
      }
      return true;
    };
    bool fail = false;
    if (ptid == 0) fail = !load_b();
#pragma unroll
    for (int d = 0; d < UT_RING; ++d)
      if (lp.item < nitems) load(ring[d]);
    Pos cur{(int)blockIdx.x, 0, 0};  // the line to store
    if (cur.item < nitems) cur.k = first_k(cur.item);
    int li = 0;
    while (cur.item < nitems && !fail) {
#pragma unroll
      for (int d = 0; d < UT_RING; ++d) {
        if (cur.item >= nitems) break;
        if (ptid == 0 && cur.sl == UT_SRC_LINES / 2 && !load_b()) fail = true;
        const int s = li % UT_NST;
        if (!fail && li >= UT_NST &&
            !mbar_wait_sleep(&s_empty[s], (li / UT_NST - 1) & 1, s_abort, piters))
          fail = true;
        if (__any_sync(0xffffffffu, fail)) {
          fail = true;
          break;
        }
        // scaled split into the A layout, zero for empty cells and parents
        // outside the domain; a warp's stores fill 32 consecutive 16-byte
        // rows of one K plane
        {
          const Slot& r = ring[d];
          const float sc = exp2i(unif_scale_exp(r.amax));
          uint32_t h[4], l[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {  // child 4 kc + e: (re, im)
            const bool ok = (r.occ >> (8 * e)) & 0xffu;
            const float x0 = ok ? r.v[e].x * sc : 0.f, x1 = ok ? r.v[e].y * sc : 0.f;
            const __half2 hh = __floats2half2_rn(x0, x1);
            const float2 hf = __half22float2(hh);
            const __half2 ll = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
            h[e] = *reinterpret_cast<const uint32_t*>(&hh);
            l[e] = *reinterpret_cast<const uint32_t*>(&ll);
          }
          unsigned char* ahi = astage + s * UT_ASTAGE;
          *reinterpret_cast<uint4*>(ahi + split_dst) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4*>(ahi + UT_APART + split_dst) =
              make_uint4(l[0], l[1], l[2], l[3]);
          if (r.occ) s_nz[s] = li + 1;
        }
        fence_async_smem();  // this thread's generic-proxy stores, to the tensor pipe
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_full[s]);
        if (lp.item < nitems) load(ring[d]);
        advance(cur);
        ++li;
      }
    }
    if (fail) *s_abort = 1;
    // no bulk copy may still be writing when the CTA ends
    if (ptid == 0 && last_b >= 0 &&
        !mbar_wait(&s_bfull[last_b & 1], (last_b >> 1) & 1, nullptr))
      *s_abort = 1;
  } else if (role == UT_MMA) {
    // ------------------------------------------------------------ MMA issue
    if (lane == 0) {
      int fi = 0, li = 0;
      bool committed = false;
      bool stop = false;
      for (int item = blockIdx.x; item < nitems && !stop; item += gridDim.x) {
        const int k0 = (item / a.nblocks) * a.kchunk, k1 = min(a.nk, k0 + a.kchunk);
        for (int k = k0; k < k1 && !stop; ++k, ++fi) {
          const int fb = fi & 1;
          if (!mbar_wait_sleep(&s_bfull[fb], (fi >> 1) & 1, s_abort, piters) ||
              (fi >= 2 && !mbar_wait_sleep(&s_acce[fb], ((fi - 2) >> 1) & 1, s_abort, piters))) {
            *s_abort = 1;
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t bb = smem_u32(bbuf + fb * UT_BFREQ);
          const uint32_t dset = tmem + (uint32_t)(fb * UT_BY * 32);
          for (int sl = 0; sl < UT_SRC_LINES; ++sl, ++li) {
            const int s = li % UT_NST;
            if (!mbar_wait_sleep(&s_full[s], (li / UT_NST) & 1, s_abort, piters)) {
              *s_abort = 1;
              stop = true;
              break;
            }
            tc_fence_after();
            if (s_nz[s] == li + 1) {
              const int dxi = sl / (UT_BY + 2), sy = sl % (UT_BY + 2) - 1;
              const int ty_lo = max(0, sy - 1), ty_hi = min(UT_BY - 1, sy + 1);
              const int dyi_lo = ty_lo - sy + 1, nl = ty_hi - ty_lo + 1;
              const uint32_t idesc = f16_idesc(128, 32 * nl);
              const uint32_t d = dset + (uint32_t)(32 * ty_lo);
              // descriptors of the line's first A and B tiles; the others
              // differ only in their start address (16-byte units, no carry:
              // shared memory is below 256 KB), by compile-time offsets
              const uint64_t a0 = kmajor_desc(smem_u32(astage + s * UT_ASTAGE), UT_APLANE, 128);
              const uint64_t b0 =
                  kmajor_desc(bb + (uint32_t)(dxi * 3 * UT_BTILE + dyi_lo * 32 * 16), UT_BPLANE, 128);
#pragma unroll
              for (int dzi = 0; dzi < 3; ++dzi) {
                // A window D_z + 1 parents down
                const uint64_t ah = a0 + ((dzi * 8 * 16) >> 4);
                const uint64_t bd = b0 + ((dzi * UT_BTILE) >> 4);
                tc_mma_f16(d, ah, bd, idesc, 1u);
                tc_mma_f16(d, ah + (UT_APART >> 4), bd, idesc, 1u);
              }
            }
            tc_commit(&s_empty[s]);
            committed = true;
          }
          if (stop) break;
          tc_commit(&s_accf[fb]);
          tc_commit(&s_bempty[fb]);
        }
      }
      // MMAs complete in order: the last stage commit covers all of them
      if (committed && !mbar_wait(&s_empty[(li - 1) % UT_NST], ((li - 1) / UT_NST) & 1, nullptr))
        *s_abort = 1;
    }
    __syncwarp();
  } else if (role == UT_DRAIN) {
    // ------------------------------------------------------------ drains
    const int row = 32 * (warp & 3) + lane;  // TMEM lane: (z, column) of the target lines
    const int tz = row >> 3, col = row & 7;
    const uint32_t lb = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const float zero[16] = {};
    int fi = 0;
    bool stop = false;
    for (int item = blockIdx.x; item < nitems && !stop; item += gridDim.x) {
      int bx, y0, z0;
      ut_block(item % a.nblocks, S, &bx, &y0, &z0);
      const int k0 = (item / a.nblocks) * a.kchunk, k1 = min(a.nk, k0 + a.kchunk);
      for (int k = k0; k < k1; ++k, ++fi) {
        const int fb = fi & 1;
        // one thread waits for the accumulators; the barrier-with-reduction
        // releases the other drain threads (uniformly: the TMEM loads below
        // are warp-collective)
        bool bad = false;
        if (tid == UT_DRAIN0 && !mbar_wait_sleep(&s_accf[fb], (fi >> 1) & 1, s_abort, piters))
          bad = true;
        if (drains_any(bad)) {
          *s_abort = 1;
          stop = true;
          break;
        }
        tc_fence_after();
        // undo the scaling of this row's column and of the frequency's tiles
        const float ua = exp2i(-unif_scale_exp(__ldg(a.amax + 8 * (k % a.nk23) + col)));
        const float ub = exp2i(-__ldg(a.bexp + k));
        for (int ty = 0; ty < UT_BY; ++ty) {
          const uint32_t ta = lb + (uint32_t)(fb * UT_BY * 32 + 32 * ty);
          uint32_t h[16], l[16];
          tc_ld16_wait(ta, h);
          tc_ld16_wait(ta + 16, l);
          tc_st16(ta, zero);
          tc_st16(ta + 16, zero);
          const int64_t p = morton_encode(bx, y0 + ty, z0 + tz);
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            const int64_t cell = 8 * p + t;
            if (a.tocc[cell])
              a.Y[((int64_t)k * ncells + cell) * a.C + a.c0 + col] = make_float2(
                  (__uint_as_float(h[2 * t]) + __uint_as_float(l[2 * t])) * ua * ub,
                  (__uint_as_float(h[2 * t + 1]) + __uint_as_float(l[2 * t + 1])) * ua * ub);
          }
        }
        tc_wait_st();
        tc_fence_before();
        group_sync(2, 128);  // every drain thread's loads and stores
        if (tid == UT_DRAIN0) mbar_arrive(&s_acce[fb]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *s_abort && a.err) atomicExch(a.err, 1);
  if (role == UT_MMA) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(UT_TMEM_COLS)
                 : "memory");
  }
}

// Operator tiles of the tensor-core MAC from the spectra op[lvl][k][343]
// (complex, lex-indexed offsets, inner 27 zero): for each level and frequency
// nine tiles (D_x, D_z), each [kcore 2][row 96][8 halves], row = 32 dyi +
// 16 part + 2 t + ri_out (D_y = 1 - dyi; part 0: F16 hi, 1: lo), element
// K = 8 kcore + e = 2 s + ri_in, value the real form of E[o] with
// o = 2 D + bits(s) - bits(t):  (re, re) = a, (im, re) = -b, (re, im) = b,
// (im, im) = a for E = a + i b, zero where o is near; every value of a
// frequency scaled by 2^sB (bexp), sB putting the largest in [2^14, 2^15).
void unif_tc_tiles(int n, const std::vector<double>& op, int nlev, std::vector<uint16_t>* tiles,
                   std::vector<int>* bexp) {
  const int m = 2 * n - 1, nk = m * m * n;
  tiles->assign((size_t)nlev * nk * kUnifTcTileHalves, 0);
  bexp->assign((size_t)nlev * nk, 0);
  parallel_for((int64_t)nlev * nk, [&](int64_t b0, int64_t b1) {
    std::vector<float> val(UT_BFREQ / 4);  // float32 values of the hi slots, tile order
    for (int64_t b = b0; b < b1; ++b) {
      const double* E = &op[(size_t)b * 343 * 2];
      float vmax = 0.f;
      for (int tile = 0; tile < 9; ++tile) {
        const int dxi = tile / 3, dzi = tile % 3;
        for (int row = 0; row < UT_BROWS; ++row) {
          const int dyi = row / 32, part = (row / 16) & 1, t = (row & 15) >> 1, ro = row & 1;
          if (part) continue;
          const int D[3] = {dxi - 1, 1 - dyi, dzi - 1};
          for (int kk = 0; kk < 16; ++kk) {
            const int s = kk >> 1, ri = kk & 1;
            int o[3], far = 0;
            for (int d = 0; d < 3; ++d) {
              o[d] = 2 * D[d] + ((s >> (2 - d)) & 1) - ((t >> (2 - d)) & 1);
              far |= o[d] > 1 || o[d] < -1;
            }
            float v = 0.f;
            if (far) {
              const int lex = 49 * (o[0] + 3) + 7 * (o[1] + 3) + (o[2] + 3);
              const double re = E[2 * lex], im = E[2 * lex + 1];
              v = (float)(ri == ro ? re : (ri ? -im : im));
            }
            val[(size_t)(tile * 48 + dyi * 16 + (row & 15)) * 16 + kk] = v;
            vmax = std::max(vmax, std::fabs(v));
          }
        }
      }
      int e = 0;
      if (vmax > 0.f && std::isfinite(vmax)) {
        int k2;
        std::frexp(vmax, &k2);
        e = std::max(-126, std::min(127, 15 - k2));
      }
      (*bexp)[b] = e;
      uint16_t* dst = tiles->data() + (size_t)b * kUnifTcTileHalves;
      for (int tile = 0; tile < 9; ++tile)
        for (int row = 0; row < UT_BROWS; ++row) {
          const int dyi = row / 32, part = (row / 16) & 1;
          for (int kk = 0; kk < 16; ++kk) {
            const float x = std::ldexp(val[(size_t)(tile * 48 + dyi * 16 + (row & 15)) * 16 + kk], e);
            const __half xh = __float2half_rn(x);
            const __half xv = part ? __float2half_rn(x - __half2float(xh)) : xh;
            memcpy(&dst[tile * (UT_BTILE / 2) + (kk >> 3) * (UT_BPLANE / 2) + row * 8 + (kk & 7)],
                   &xv, 2);
          }
        }
    }
  });
}

bool unif_tc_eligible(const pbbfmm_tree* t, int l, int C) {
  return t->use_tc && t->f_unif_tiles && t->f_unif_bexp && (C % 8) == 0 && l >= 5 && l <= 10;
}

// Level l of the tensor-core MAC (after the forward FFTs): Y = sum_D B X for
// every column group of 8.
int run_m2l_unif_tc_level(pbbfmm_tree* t, int C, int l, int lvl, const float2* X, float2* Y,
                          const uint32_t* amax, cudaStream_t st) {
  if (!t->d_tc_err) {
    set_error("tensor-core uniform M2L: the tree has no timeout flag");
    return PBBFMM_ERR_STATE;
  }
  PB_CUDA(cudaFuncSetAttribute(k_m2l_unif_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               UT_SMEM));
  const int L = t->p.tree_level, nk = t->nk;
  const int64_t ncells = cells_at(l);
  Workspace& ws = t->ws;
  if (int rc = grow(ws.occ, 2 * (size_t)ncells)) return rc;
  uint8_t* socc = ws.occ.as<uint8_t>();
  uint8_t* tocc = socc + ncells;
  const int span = (int)cells_at(L - l);
  const unsigned g = (unsigned)((ncells + 255) / 256);
  k_occupancy<<<g, 256, 0, st>>>(ws.sstart.as<int>(), span, ncells, socc);
  PB_LAUNCH("occupancy");
  k_occupancy<<<g, 256, 0, st>>>(ws.tstart.as<int>(), span, ncells, tocc);
  PB_LAUNCH("occupancy");
  const int S = 1 << (l - 1);
  UnifTcArgs a{};
  a.X = X;
  a.Y = Y;
  a.tiles = t->f_unif_tiles + (size_t)lvl * nk * kUnifTcTileHalves;
  a.bexp = t->f_unif_bexp + (size_t)lvl * nk;
  a.amax = amax;
  a.nk23 = (2 * t->n - 1) * t->n;
  a.socc = socc;
  a.tocc = tocc;
  a.lev = l;
  a.C = C;
  a.nk = nk;
  a.nblocks = S * (S / UT_BY) * (S / UT_LINE);
  int dev = 0, nsm = 148;
  PB_CUDA(cudaGetDevice(&dev));
  PB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  // frequency chunks: about 16 work items per SM (the line pipeline runs on
  // across items, so short items cost nothing; many of them balance the SMs)
  a.nchunks = std::max(1, std::min(nk, (16 * nsm + a.nblocks - 1) / a.nblocks));
  a.kchunk = (nk + a.nchunks - 1) / a.nchunks;
  a.nchunks = (nk + a.kchunk - 1) / a.kchunk;
  a.err = t->d_tc_err;
  const unsigned grid = (unsigned)std::min(a.nblocks * a.nchunks, nsm);
  for (int c0 = 0; c0 < C; c0 += 8) {
    a.c0 = c0;
    k_m2l_unif_tc<<<grid, UT_THREADS, UT_SMEM, st>>>(a);
    PB_LAUNCH("m2l_unif_tc");
  }
  return PBBFMM_OK;
}

int set_unif_tc_wait_limit(long long polls) {
  PB_CUDA(cudaMemcpyToSymbol(g_unif_wait_iters, &polls, sizeof(polls)));
  return PBBFMM_OK;
}

}  // namespace pbbfmm


