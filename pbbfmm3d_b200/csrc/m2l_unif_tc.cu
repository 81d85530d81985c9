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
// A operand, 144 rows (z, column) x K = 16 (child, re/im), split into TF32 hi
// and lo parts; a window of 128 of its rows, shifted by D_z parents, lines up
// with the rows of the target lines.  The operator tiles B for one D_x and D_z
// stack the three D_y in N (96 rows: D_y x (hi, lo) x (child, re/im)), so one
// MMA serves the three target lines y - D_y at once; their TMEM accumulators
// (32 columns per line: the products with B hi, then with B lo) are adjacent.
// Each (line, D_x, D_z) issues four tcgen05.mma kind::tf32 (A hi and A lo, K
// in two steps of 8); D = A_hi B + A_lo B = (A_hi + A_lo)(B_hi + B_lo), i.e.
// float32 operands at about 2^-21 relative error per product (3xTF32 plus
// the lo x lo term), accumulated in float32.
//
// Roles (416 threads): warps 0-7 stage source lines (cp.async of the raw
// float32 spectra, zero-filled for empty or out-of-domain cells, then a split
// into the hi / lo A layout) and load each frequency's operator tiles by a
// bulk copy; one thread of warp 8 issues the MMAs; warps 9-12 drain the
// accumulators (two TMEM sets, alternating by frequency), write the target
// spectra and zero the accumulators.  Every wait is bounded; on timeout the
// kernel sets *err, waits (bounded) for its issued copies and MMAs, frees its
// TMEM and returns.
#include <cuda.h>

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
constexpr int UT_APLANE = UT_ROWS * 16;    // bytes of one K core plane of A
constexpr int UT_APART = 4 * UT_APLANE;    // hi or lo part of a stage (K = 16 floats)
constexpr int UT_ASTAGE = 2 * UT_APART;
constexpr int UT_NST = 3;                  // A stages
constexpr int UT_RAWZ = 576;               // bytes per parent in a raw line (512 + bank padding)
constexpr int UT_RAWLINE = UT_SRCZ * UT_RAWZ;  // raw float32 spectra of one source line
constexpr int UT_PREFETCH = 4;             // lines whose raw copies run ahead of the split
constexpr int UT_NRAW = UT_PREFETCH + 2;   // raw slots
constexpr int UT_BROWS = 96;               // B rows of one (D_x, D_z) tile
constexpr int UT_BPLANE = UT_BROWS * 16;
constexpr int UT_BTILE = 4 * UT_BPLANE;
constexpr int UT_BFREQ = 9 * UT_BTILE;     // operator tiles of one frequency (bytes)
constexpr int UT_PRODUCERS = 256;          // warps 0-7
constexpr int UT_MMA_WARP = UT_PRODUCERS / 32;  // warp 8
constexpr int UT_DRAIN0 = UT_PRODUCERS + 32;    // first drain thread (warps 9-12)
constexpr int UT_THREADS = UT_DRAIN0 + 128;
constexpr int UT_TMEM_COLS = 512;          // two sets of UT_BY x 32 columns
constexpr int UT_SMEM = UT_NST * UT_ASTAGE + UT_NRAW * UT_RAWLINE + 2 * UT_BFREQ + 1024;
static_assert(2 * UT_BY * 32 == UT_TMEM_COLS, "two accumulator sets fill the TMEM");
static_assert(UT_SMEM <= 232448, "shared memory of one CTA");

// Floats of the operator tiles per (level, frequency).
constexpr int kUnifTcTileFloats = UT_BFREQ / 4;

// Poll limit of the pipeline waits (see g_pipe_wait_iters in m2l_tc.cu).
__device__ long long g_unif_wait_iters = kWaitIters;

// OR of `v` over the 256 producer threads (warps 0-7), which also acts as
// their barrier (named barrier 1): every producer executes the same sequence
// of these, so none waits for a thread that has left.
__device__ __forceinline__ bool producers_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, 1, 256, q;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

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

// x rounded to TF32 (10 explicit mantissa bits), to nearest with ties away
// from zero, by integer operations on its bits: the value cvt.rna.tf32.f32
// gives for finite x (no conversion instruction on the producers' path).
__device__ __forceinline__ float tf32_rna_bits(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
}

__global__ void k_occupancy(const int* __restrict__ start, int span, int64_t ncells,
                            uint8_t* __restrict__ occ) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < ncells) occ[c] = start[(c + 1) * span] > start[c * span] ? 1 : 0;
}

struct UnifTcArgs {
  const float2* X;       // level spectra [k][cell][C]
  float2* Y;             // level target spectra [k][cell][C]
  const float* tiles;    // [nk][kUnifTcTileFloats] operator tiles of this level
  const uint8_t* socc;   // [cell] source cell nonempty
  const uint8_t* tocc;   // [cell] target cell nonempty
  int lev;               // cells 2^lev per side, parents S = 2^(lev-1)
  int C, c0;             // columns of the arrays; first of this group of 8
  int nk, kchunk, nchunks, nblocks;
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
  unsigned char* raw = astage + UT_NST * UT_ASTAGE;           // UT_NRAW raw lines
  unsigned char* bbuf = raw + UT_NRAW * UT_RAWLINE;           // 2 x operator tiles
  __shared__ uint64_t s_full[UT_NST], s_empty[UT_NST], s_bfull[2], s_bempty[2], s_accf[2],
      s_acce[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_nz[UT_NST];  // stage s holds a nonempty line: its line number + 1
  __shared__ int s_abort_flag;
  volatile int* s_abort = &s_abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long piters = g_unif_wait_iters;
  const int S = 1 << (a.lev - 1);
  const int64_t ncells = (int64_t)1 << (3 * a.lev);
  const int nitems = a.nblocks * a.nchunks;

  if (warp == UT_MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(UT_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < UT_NST; ++i) {
      mbar_init(&s_full[i], 1);
      mbar_init(&s_empty[i], 1);
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
  if (warp > UT_MMA_WARP) {
    const uint32_t lb = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const float z[16] = {};
    for (int c = 0; c < UT_TMEM_COLS; c += 16) tc_st16(lb + (uint32_t)c, z);
    tc_wait_st();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  if (warp < UT_MMA_WARP) {
    // ------------------------------------------------------------ producers
    // The source lines of every frequency of every work item, in the order
    // the MMA thread consumes them: item (block, frequency chunk) round robin
    // over the CTAs, then frequency, then line.
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
    const int ptid = tid;
    // This thread's split tasks t = ptid + 256 i: K plane kc = t / 144 and
    // row = t % 144 = (zpos, column); byte offsets in the raw line and in
    // one part of an A stage (-1: no task)
    constexpr int kSplit = (4 * UT_ROWS + UT_PRODUCERS - 1) / UT_PRODUCERS;
    int split_src[kSplit], split_dst[kSplit];
#pragma unroll
    for (int i = 0; i < kSplit; ++i) {
      const int t = ptid + i * UT_PRODUCERS;
      const int kc = t / UT_ROWS, row = t - kc * UT_ROWS;
      split_src[i] = t < 4 * UT_ROWS ? (row >> 3) * UT_RAWZ + (2 * kc) * 64 + (row & 7) * 8 : -1;
      split_dst[i] = kc * UT_APLANE + row * 16;
    }
    // This thread's raw chunks: q_i = ptid + 256 i (16 bytes each): parent
    // zpos = q / 32, child j = (q / 4) % 8, columns 2 (q % 4) and 2 (q % 4) + 1.
    // The z part of their Morton codes is fixed per work item.
    constexpr int kPer = (UT_SRCZ * 32 + UT_PRODUCERS - 1) / UT_PRODUCERS;
    int item_ctx = -1, bx = 0, y0 = 0, z0 = 0;
    uint32_t zsp[kPer];
    auto set_item = [&](int item) {
      if (item == item_ctx) return;
      item_ctx = item;
      ut_block(item % a.nblocks, S, &bx, &y0, &z0);
#pragma unroll
      for (int i = 0; i < kPer; ++i) {
        const int q = ptid + i * UT_PRODUCERS;
        const int z = z0 - 1 + (q >> 5);
        zsp[i] = (q < UT_SRCZ * 32 && z >= 0 && z < S) ? spread3((uint32_t)z) : 0xffffffffu;
      }
    };
    // A line whose copies are about to be issued: its cells and their
    // occupancy, loaded one iteration before the copies need them.
    struct Pending {
      int64_t cell[kPer];
      uint8_t occ[kPer];
      int k;
    };
    auto prepare = [&](const Pos& p, Pending& L) {
      set_item(p.item);
      const int xs = bx + p.sl / (UT_BY + 2) - 1, ys = y0 + p.sl % (UT_BY + 2) - 1;
      const bool in = xs >= 0 && xs < S && ys >= 0 && ys < S;
      const uint32_t xy = in ? (spread3((uint32_t)xs) << 2) | (spread3((uint32_t)ys) << 1) : 0u;
#pragma unroll
      for (int i = 0; i < kPer; ++i) {
        const int q = ptid + i * UT_PRODUCERS;
        L.cell[i] = (in && zsp[i] != 0xffffffffu) ? 8 * (int64_t)(xy | zsp[i]) + ((q >> 2) & 7) : -1;
        L.occ[i] = L.cell[i] >= 0 ? a.socc[L.cell[i]] : 0;
      }
      L.k = p.k;
    };
    // raw copies (cp.async) of a prepared line into raw slot `slot`, zero for
    // empty or out-of-domain cells; parent rows UT_RAWZ bytes apart
    auto issue = [&](const Pending& L, int slot) -> bool {
      unsigned char* dst = raw + slot * UT_RAWLINE;
      const float2* xk = a.X + (int64_t)L.k * ncells * a.C + a.c0;
      bool any = false;
#pragma unroll
      for (int i = 0; i < kPer; ++i) {
        const int q = ptid + i * UT_PRODUCERS;
        if (q < UT_SRCZ * 32) {
          const bool ok = L.occ[i] != 0;
          any |= ok;
          cp_async16(dst + (q >> 5) * UT_RAWZ + (q & 31) * 16,
                     ok ? xk + L.cell[i] * a.C + 2 * (q & 3) : a.X, ok ? 16 : 0);
        }
      }
      return any;
    };
    Pos cur{(int)blockIdx.x, 0, 0};
    if (cur.item < nitems) cur.k = first_k(cur.item);
    // prefetch: the raw copies run UT_PREFETCH lines ahead of the split, in
    // UT_PREFETCH + 2 slots (a slot is rewritten two iterations after its
    // split, so one barrier per line orders the reuse)
    Pos pf = cur;
    Pending L;
    bool have = pf.item < nitems;
    if (have) prepare(pf, L);
    int issued = 0;
    uint32_t anymask = 0;  // bit r: this thread's chunks of the line in raw slot r hold data
    auto issue_next = [&]() {
      if (have) {
        const int slot = issued % UT_NRAW;
        anymask = (anymask & ~(1u << slot)) | ((issue(L, slot) ? 1u : 0u) << slot);
        ++issued;
        advance(pf);
        have = pf.item < nitems;
        if (have) prepare(pf, L);
      }
      cp_async_commit();  // (possibly empty) keeps one group per line
    };
    for (int i = 0; i < UT_PREFETCH; ++i) issue_next();
    // operator tiles: frequency f goes to buffer f % 2; the load for f + 1 is
    // issued in the middle of frequency f (the MMAs of f - 1, the buffer's
    // previous user, are issued by then)
    Pos bnext = cur;  // the frequency whose tiles are loaded next
    int fi = 0, li = 0, bissued = 0, last_b = -1;
    auto load_b = [&]() -> bool {  // ptid 0 only
      if (bnext.item >= nitems) return true;
      const int fb = bissued & 1;
      if (bissued >= 2 && !mbar_wait(&s_bempty[fb], ((bissued - 2) >> 1) & 1, s_abort, piters))
        return false;
      mbar_arrive_expect_tx(&s_bfull[fb], UT_BFREQ);
      bulk_load(bbuf + fb * UT_BFREQ, a.tiles + (int64_t)bnext.k * kUnifTcTileFloats, UT_BFREQ,
                &s_bfull[fb]);
      last_b = bissued++;
      // the following frequency
      if (++bnext.k == end_k(bnext.item)) {
        bnext.item += gridDim.x;
        if (bnext.item < nitems) bnext.k = first_k(bnext.item);
      }
      return true;
    };
    bool fail = false;
    if (ptid == 0 && cur.item < nitems) fail = !load_b();
    for (; cur.item < nitems; advance(cur)) {
      if (ptid == 0 && cur.sl == UT_SRC_LINES / 2 && !fail) fail = !load_b();
      issue_next();
      asm volatile("cp.async.wait_group %0;\n" ::"n"(UT_PREFETCH) : "memory");
      const int s = li % UT_NST;
      // one thread waits for the stage (its MMAs of UT_NST lines ago); the
      // barrier-with-reduction then releases every producer, makes the raw
      // line complete for all of them, and lets all leave together on failure
      if (ptid == 0 && li >= UT_NST &&
          !mbar_wait(&s_empty[s], (li / UT_NST - 1) & 1, s_abort, piters))
        fail = true;
      if (producers_any(fail)) {
        *s_abort = 1;
        break;
      }
      // split into the A layout: task t = (kc, row), row = (zpos, column);
      // a warp's stores fill 32 consecutive 16-byte rows of one K plane
      const unsigned char* rl = raw + (li % UT_NRAW) * UT_RAWLINE;
      unsigned char* ahi = astage + s * UT_ASTAGE;
      unsigned char* alo = ahi + UT_APART;
#pragma unroll
      for (int i = 0; i < kSplit; ++i) {
        if (split_src[i] >= 0) {
          const unsigned char* src = rl + split_src[i];
          const float2 u = *reinterpret_cast<const float2*>(src);
          const float2 v = *reinterpret_cast<const float2*>(src + 64);
          const float r[4] = {u.x, u.y, v.x, v.y};
          float h[4], l[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            h[e] = tf32_rna_bits(r[e]);
            l[e] = tf32_rna_bits(r[e] - h[e]);
          }
          *reinterpret_cast<float4*>(ahi + split_dst[i]) = make_float4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<float4*>(alo + split_dst[i]) = make_float4(l[0], l[1], l[2], l[3]);
        }
      }
      if ((anymask >> (li % UT_NRAW)) & 1u) s_nz[s] = li + 1;
      fence_async_smem();  // this thread's generic-proxy stores, to the tensor pipe
      group_sync(1, UT_PRODUCERS);  // every producer's stores and fence
      if (ptid == 0) mbar_arrive(&s_full[s]);
      ++li;
      if (cur.sl == UT_SRC_LINES - 1) ++fi;
    }
    cp_async_wait_all();
    // no bulk copy may still be writing when the CTA ends
    if (ptid == 0 && last_b >= 0 &&
        !mbar_wait(&s_bfull[last_b & 1], (last_b >> 1) & 1, nullptr))
      *s_abort = 1;
    (void)fi;
  } else if (warp == UT_MMA_WARP) {
    // ------------------------------------------------------------ MMA issue
    if (lane == 0) {
      int fi = 0, li = 0;
      bool committed = false;
      bool stop = false;
      for (int item = blockIdx.x; item < nitems && !stop; item += gridDim.x) {
        const int k0 = (item / a.nblocks) * a.kchunk, k1 = min(a.nk, k0 + a.kchunk);
        for (int k = k0; k < k1 && !stop; ++k, ++fi) {
          const int fb = fi & 1;
          if (!mbar_wait(&s_bfull[fb], (fi >> 1) & 1, s_abort, piters) ||
              (fi >= 2 && !mbar_wait(&s_acce[fb], ((fi - 2) >> 1) & 1, s_abort, piters))) {
            *s_abort = 1;
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t bb = smem_u32(bbuf + fb * UT_BFREQ);
          const uint32_t dset = tmem + (uint32_t)(fb * UT_BY * 32);
          for (int sl = 0; sl < UT_SRC_LINES; ++sl, ++li) {
            const int s = li % UT_NST;
            if (!mbar_wait(&s_full[s], (li / UT_NST) & 1, s_abort, piters)) {
              *s_abort = 1;
              stop = true;
              break;
            }
            tc_fence_after();
            if (s_nz[s] == li + 1) {
              const int dxi = sl / (UT_BY + 2), sy = sl % (UT_BY + 2) - 1;
              const int ty_lo = max(0, sy - 1), ty_hi = min(UT_BY - 1, sy + 1);
              const int dyi_lo = ty_lo - sy + 1, nl = ty_hi - ty_lo + 1;
              const uint32_t idesc = tf32_idesc(128, 32 * nl);
              const uint32_t d = dset + (uint32_t)(32 * ty_lo);
              // descriptors of the line's first A and B tiles; the others
              // differ only in their start address (16-byte units, no carry:
              // shared memory is below 256 KB), by compile-time offsets
              const uint64_t a0 = kmajor_desc(smem_u32(astage + s * UT_ASTAGE), UT_APLANE, 128);
              const uint64_t b0 =
                  kmajor_desc(bb + (uint32_t)(dxi * 3 * UT_BTILE + dyi_lo * 32 * 16), UT_BPLANE, 128);
#pragma unroll
              for (int dzi = 0; dzi < 3; ++dzi)
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                  // A window D_z + 1 parents down; K step ks = planes 2 ks, 2 ks + 1
                  const uint64_t ah = a0 + ((dzi * 8 * 16 + ks * 2 * UT_APLANE) >> 4);
                  const uint64_t bd = b0 + ((dzi * UT_BTILE + ks * 2 * UT_BPLANE) >> 4);
                  tc_mma_tf32(d, ah, bd, idesc, 1u);
                  tc_mma_tf32(d, ah + (UT_APART >> 4), bd, idesc, 1u);
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
  } else {
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
        if (tid == UT_DRAIN0 && !mbar_wait(&s_accf[fb], (fi >> 1) & 1, s_abort, piters)) bad = true;
        if (drains_any(bad)) {
          *s_abort = 1;
          stop = true;
          break;
        }
        tc_fence_after();
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
              a.Y[((int64_t)k * ncells + cell) * a.C + a.c0 + col] =
                  make_float2(__uint_as_float(h[2 * t]) + __uint_as_float(l[2 * t]),
                              __uint_as_float(h[2 * t + 1]) + __uint_as_float(l[2 * t + 1]));
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
  if (warp == UT_MMA_WARP) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(UT_TMEM_COLS)
                 : "memory");
  }
}

// Operator tiles of the tensor-core MAC from the spectra op[lvl][k][343]
// (complex, lex-indexed offsets, inner 27 zero): for each level and frequency
// nine tiles (D_x, D_z), each [kcore 4][row 96][4 floats], row = 32 dyi +
// 16 part + 2 t + ri_out (D_y = 1 - dyi; part 0: TF32 hi, 1: lo), element
// K = 4 kcore + e = 2 s + ri_in, value the real form of E[o] with
// o = 2 D + bits(s) - bits(t):  (re, re) = a, (im, re) = -b, (re, im) = b,
// (im, im) = a for E = a + i b, zero where o is near.
void unif_tc_tiles(int n, const std::vector<double>& op, int nlev, std::vector<float>* tiles) {
  const int m = 2 * n - 1, nk = m * m * n;
  tiles->assign((size_t)nlev * nk * kUnifTcTileFloats, 0.f);
  auto tf32r = [](float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u = (u + 0x1000u) & 0xffffe000u;  // to nearest, ties away (cvt.rna.tf32.f32)
    float r;
    memcpy(&r, &u, 4);
    return r;
  };
  parallel_for((int64_t)nlev * nk, [&](int64_t b0, int64_t b1) {
    for (int64_t b = b0; b < b1; ++b) {
      const double* E = &op[(size_t)b * 343 * 2];
      float* dst = tiles->data() + (size_t)b * kUnifTcTileFloats;
      for (int dxi = 0; dxi < 3; ++dxi)
        for (int dzi = 0; dzi < 3; ++dzi) {
          float* tile = dst + (dxi * 3 + dzi) * (UT_BTILE / 4);
          for (int row = 0; row < UT_BROWS; ++row) {
            const int dyi = row / 32, part = (row / 16) & 1, t = (row & 15) >> 1, ro = row & 1;
            const int D[3] = {dxi - 1, 1 - dyi, dzi - 1};
            for (int kk = 0; kk < 16; ++kk) {
              const int s = kk >> 1, ri = kk & 1;
              int o[3], far = 0;
              for (int d = 0; d < 3; ++d) {
                o[d] = 2 * D[d] + ((s >> (2 - d)) & 1) - ((t >> (2 - d)) & 1);
                far |= o[d] > 1 || o[d] < -1;
              }
              double v = 0;
              if (far) {
                const int lex = 49 * (o[0] + 3) + 7 * (o[1] + 3) + (o[2] + 3);
                const double re = E[2 * lex], im = E[2 * lex + 1];
                v = ri == ro ? re : (ri ? -im : im);
              }
              const float hi = tf32r((float)v), lo = tf32r((float)v - hi);
              tile[((kk >> 2) * UT_BROWS + row) * 4 + (kk & 3)] = part ? lo : hi;
            }
          }
        }
    }
  });
}

bool unif_tc_eligible(const pbbfmm_tree* t, int l, int C) {
  return t->use_tc && t->f_unif_tiles && (C % 8) == 0 && l >= 5 && l <= 10;
}

// Level l of the tensor-core MAC (after the forward FFTs): Y = sum_D B X for
// every column group of 8.
int run_m2l_unif_tc_level(pbbfmm_tree* t, int C, int l, int lvl, const float2* X, float2* Y,
                          cudaStream_t st) {
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
  a.tiles = t->f_unif_tiles + (size_t)lvl * nk * kUnifTcTileFloats;
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


