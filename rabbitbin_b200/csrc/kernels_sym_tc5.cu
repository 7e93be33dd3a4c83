// Symmetric all-pairs pass, part 1: the abundance prefilter on the
// 5th-generation tensor cores, hand-written for sm_100a.
//
// The abundance prune of the fused path (unit_dot_f(U_i, U_j) >= eps,
// src/impl/rb_graph.cpp:501-1356, the order of src/rabbitbin.cpp:754-796) is
// a threshold on the products of the unit rank rows.  Their FP16 copies, padded
// to 64 halves (one 128-byte swizzle atom), are multiplied here with
// tcgen05.mma kind::f16 (FP32 accumulation in TMEM); every pair whose product
// reaches lo16 = eps - 2.5e-3 (the bound that makes the FP16 prune exact, see
// prefilter_bands; here lo16 rounded down to FP16) is a candidate, and only
// candidates reach the exact check and the register compare of part 2
// (k_sym_check, kernels_allpairs.cu).  The threshold rides in the MMA as a
// bias column (row side 1.0, column side -lo16 in the last half, free for
// S < 64), so a candidate is a product whose sign bit is clear; byte permutes
// gather the sign bits of 32 products into one mask.
//
// Work: items (128-row block rb, 256-column tile ct) of the pairs i < j with j
// in a column window [jlo, jhi) (the whole upper triangle, or the columns of
// one input chunk while later chunks are still being copied in; ct from the
// tile holding the block's first row, or the window's first tile, on), each
// CTA (one per SM) a contiguous range of them in row-block order.  Warp 0 issues the TMA loads
// (the row block's 128 rows once per block into a 2-deep ring, each column
// tile's 256 rows into a 4-deep ring), warp 1 allocates TMEM (two 256-column
// accumulators, so an item's MMAs run while the epilogue reads the previous
// item) and issues 4 MMAs of K = 16 per item, warps 2-17 are the epilogue: a
// thread takes one row and 64 of the tile's columns, keeps the pairs j > i
// with j in the window and a product of at least lo16 (a contig without
// abundance has a zero unit row, so it never gets there; part 2 checks the
// flags), and appends them to its 32-row block's candidate list (entry
// r << 27 | j, r the row within the block) with one atomic per warp and item.
// A block's list has the capacity the host gave it; the count goes on past it,
// so a pass that overflows is rerun with exact capacities.
//
// Every mbarrier wait is bounded (2 s of %globaltimer); a wait that runs out
// records an error code for the host and the CTA stops issuing work, waits
// (bounded) for its own copies and MMAs in flight, frees its TMEM and returns.
// No TMA load uses cluster multicast.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "rbg_internal.h"
#include "tc05.cuh"

namespace rbg {
namespace {

using namespace tc05;

constexpr int kPM = 128;                       // rows per item (UMMA M)
constexpr int kPN = 256;                       // columns per item (UMMA N)
constexpr int kPK = 64;                        // halves per padded unit row (128 bytes)
constexpr int kPStages = 4;                    // column-tile ring
constexpr int kPEpiWarps = 16;
constexpr int kPThreads = (2 + kPEpiWarps) * 32;
constexpr int kABytes = kPM * kPK * 2;         // 16 KB
constexpr int kBBytes = kPN * kPK * 2;         // 32 KB
constexpr unsigned FULL = 0xffffffffu;
// D f32 (bits 4-5 = 1), A and B f16 (0), both K-major, N >> 3 at bits 17-22,
// M >> 4 at bits 24-28
constexpr uint32_t kIdescF16 =
    (1u << 4) | ((uint32_t)(kPN >> 3) << 17) | ((uint32_t)(kPM >> 4) << 24);

struct PfArgs {
  int jlo, jhi;           // pairs i < j with j in [jlo, jhi) (rows [0, jhi))
  int ct_lo;              // first column tile: jlo / 256
  const int32_t *item0;   // [RB + 1] first item of each 128-row block
  int RB, NT, items;      // row blocks below jhi, column tiles below jhi, items
  uint32_t *cand;         // block b's entries at cand + coff[b], coff[b + 1] - coff[b] of them
  const int64_t *coff;    // [B32 + 1]
  int32_t *ccnt;          // [B32] entries found (counted on past the capacity)
  int *overflow;          // set when a block's entries outgrow its capacity
  unsigned long long *stats;   // [0] += pairs evaluated
  int *err;               // set when a bounded wait runs out
};

__device__ __forceinline__ void mma_f16(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dt), "l"(ad), "l"(bd), "r"(kIdescF16), "r"(acc));
}

// Named barrier 1 of the epilogue warps; returns the OR of every thread's flag.
__device__ __forceinline__ uint32_t pf_barrier_or(uint32_t flag) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "barrier.cta.red.or.pred po, 1, %2, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(out)
      : "r"(flag), "n"(kPEpiWarps * 32)
      : "memory");
  return out;
}

// Item it -> (row block rb, column tile ct); the next item in order.
struct ItemWalk {
  int rb, ct;
  __device__ void start(const PfArgs &A, int it) {
    int lo = 0, hi = A.RB - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (A.item0[mid] <= it) lo = mid; else hi = mid - 1;
    }
    rb = lo;
    ct = max((kPM * rb) / kPN, A.ct_lo) + (it - A.item0[rb]);
  }
  __device__ void next(const PfArgs &A) {
    if (++ct == A.NT) {
      ++rb;
      ct = max((kPM * rb) / kPN, A.ct_lo);
    }
  }
};

__global__ void __launch_bounds__(kPThreads, 1)
k_sym_prefilter(const __grid_constant__ CUtensorMap tmapA, const __grid_constant__ CUtensorMap tmapB,
                const PfArgs A) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *sa = base;                                  // [2][kABytes]
  uint8_t *sb = base + 2 * kABytes;                    // [kPStages][kBBytes]
  uint64_t *bars = (uint64_t *)(sb + kPStages * kBBytes);
  // bars: fullA[2], emptyA[2], full[S], empty[S], tfull[2], tempty[2], mdone
  uint32_t *tmem_slot = (uint32_t *)(bars + 4 + 2 * kPStages + 5);
  int *abort_flag = (int *)(tmem_slot + 4);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int it0 = (int)((int64_t)blockIdx.x * A.items / gridDim.x);
  const int it1 = (int)((int64_t)(blockIdx.x + 1) * A.items / gridDim.x);
  const uint32_t b0 = smem_u32(bars);
  auto fullA = [&](int i) { return b0 + 8u * i; };
  auto emptyA = [&](int i) { return b0 + 8u * (2 + i); };
  auto full = [&](int s) { return b0 + 8u * (4 + s); };
  auto empty = [&](int s) { return b0 + 8u * (4 + kPStages + s); };
  auto tfull = [&](int i) { return b0 + 8u * (4 + 2 * kPStages + i); };
  auto tempty = [&](int i) { return b0 + 8u * (6 + 2 * kPStages + i); };
  const uint32_t mdone = b0 + 8u * (8 + 2 * kPStages);

  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(fullA(i), 1);
      mbar_init(emptyA(i), 1);
      mbar_init(tfull(i), 1);
      mbar_init(tempty(i), kPEpiWarps * 32);
    }
    for (int s = 0; s < kPStages; ++s) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    mbar_init(mdone, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {                                      // TMEM: two 256-column accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;"
                 ::"r"(smem_u32(tmem_slot)) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tbase = *tmem_slot;

  if (it0 < it1 && warp == 0) {
    // ── TMA producer ──
    if (lane == 0) {
      ItemWalk w;
      w.start(A, it0);
      int arb = -1, an = 0;                             // row block in the A ring, A loads
      int s = 0;
      uint32_t ph = 0, issued = 0, last_ph = 0;         // B ring state (bit s: stage s)
      uint32_t a_issued = 0, a_last = 0;                // A ring state (bit i: buffer i)
      bool ok = true;
      for (int it = it0; it < it1 && ok; ++it, w.next(A)) {
        if (w.rb != arb) {
          const int ai = an & 1;
          const uint32_t aph = (uint32_t)(an >> 1) & 1u;
          if (!mbar_wait(emptyA(ai), aph ^ 1u, A.err, 11) || *(volatile int *)abort_flag) {
            ok = false;
            break;
          }
          mbar_expect_tx(fullA(ai), kABytes);
          tma_load(smem_u32(sa + ai * kABytes), &tmapA, 0, kPM * w.rb, fullA(ai));
          a_issued |= 1u << ai;
          a_last = (a_last & ~(1u << ai)) | (aph << ai);
          arb = w.rb;
          ++an;
        }
        if (!mbar_wait(empty(s), ph ^ 1u, A.err, 12) || *(volatile int *)abort_flag) {
          ok = false;
          break;
        }
        const uint32_t dst = smem_u32(sb + (size_t)s * kBBytes);
        mbar_expect_tx(full(s), kBBytes);
        tma_load(dst, &tmapB, 0, kPN * w.ct, full(s));
        tma_load(dst + kBBytes / 2, &tmapB, 0, kPN * w.ct + kPN / 2, full(s));
        issued |= 1u << s;
        last_ph = (last_ph & ~(1u << s)) | (ph << s);
        if (++s == kPStages) { s = 0; ph ^= 1u; }
      }
      if (!ok) *(volatile int *)abort_flag = 1;
      // copies in flight land before the CTA leaves
      for (int t = 0; t < kPStages; ++t)
        if ((issued >> t) & 1u) mbar_wait(full(t), (last_ph >> t) & 1u, A.err, 13);
      for (int t = 0; t < 2; ++t)
        if ((a_issued >> t) & 1u) mbar_wait(fullA(t), (a_last >> t) & 1u, A.err, 14);
    }
  } else if (it0 < it1 && warp == 1) {
    // ── MMA issuer ──
    if (lane == 0) {
      ItemWalk w;
      w.start(A, it0);
      int arb = -1, an = 0, ai = 0;
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      int k = 0;
      for (int it = it0; it < it1 && ok; ++it, ++k) {
        if (w.rb != arb) {
          ai = an & 1;
          if (!mbar_wait(fullA(ai), (uint32_t)(an >> 1) & 1u, A.err, 15) ||
              *(volatile int *)abort_flag) {
            ok = false;
            break;
          }
          arb = w.rb;
          ++an;
        }
        const int tb = k & 1;
        if (!mbar_wait(tempty(tb), ((uint32_t)(k >> 1) & 1u) ^ 1u, A.err, 16) ||
            !mbar_wait(full(s), ph, A.err, 17) || *(volatile int *)abort_flag) {
          ok = false;
          break;
        }
        fence_after();
        const uint64_t da = sdesc128(smem_u32(sa + ai * kABytes));
        const uint64_t db = sdesc128(smem_u32(sb + (size_t)s * kBBytes));
#pragma unroll
        for (int kk = 0; kk < kPK / 16; ++kk)           // K = 16 halves (32 bytes) a step
          mma_f16(tbase + (uint32_t)(tb * kPN), da + 2 * kk, db + 2 * kk, kk ? 1u : 0u);
        mma_commit(empty(s));                           // the column tile is free
        mma_commit(tfull(tb));                          // the products are in TMEM
        w.next(A);
        if (it + 1 == it1 || w.rb != arb) mma_commit(emptyA(ai));   // the row block is done
        if (++s == kPStages) { s = 0; ph ^= 1u; }
      }
      if (!ok) *(volatile int *)abort_flag = 1;
      mma_commit(mdone);                                // every MMA issued has finished
      mbar_wait(mdone, 0, A.err, 18);
    }
  } else if (it0 < it1) {
    // ── epilogue: thread = (row, 64 columns of the tile) ──
    const int e = warp - 2;                             // 0..15
    const int q = warp & 3;                             // TMEM lane quarter of this warp
    const int p = e >> 2;                               // columns [64 p, 64 p + 64)
    const int jlo = A.jlo, jhi = A.jhi;
    ItemWalk w;
    w.start(A, it0);
    unsigned long long npref = 0;
    int k = 0;
    for (int it = it0; it < it1; ++it, ++k, w.next(A)) {
      const int tb = k & 1;
      uint32_t bad = mbar_wait(tfull(tb), (uint32_t)(k >> 1) & 1u, A.err, 19) ? 0u : 1u;
      if (*(volatile int *)abort_flag) bad = 1u;
      if (pf_barrier_or(bad)) {                         // one decision for all epilogue threads
        *(volatile int *)abort_flag = 1;
        break;
      }
      fence_after();
      uint32_t v0[32], v1[32];
      const uint32_t ta = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(tb * kPN + p * 64);
      tmem_ld32(ta, v0);
      tmem_ld32(ta + 32, v1);
      tmem_wait_ld();
      fence_before();
      mbar_arrive(tempty(tb));                          // the accumulator is free again
      const int row0w = kPM * w.rb + 32 * q;            // the warp's 32 rows
      const int row = row0w + lane;
      // Masks in "gather order": bit 8 q + k stands for column t = 4 k + q of
      // the 32-column chunk (the order the byte permutes below produce).
      uint32_t cm[2];
      int cnt = 0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t(&v)[32] = h ? v1 : v0;
        const int j0 = kPN * w.ct + 64 * p + 32 * h;
        // valid columns: i < j, jlo <= j < jhi (the warp-uniform interior case first)
        uint32_t valid;
        if (j0 > row0w + 31 && j0 >= jlo && j0 + 32 <= jhi && row0w + 31 < jhi) {
          valid = ~0u;
          npref += 32;
        } else {
          const int tl = max(row - j0 + 1, jlo - j0);     // first valid t
          const int dh = jhi - j0;                        // t < dh
          uint32_t vt = tl <= 0 ? ~0u : (tl >= 32 ? 0u : (~0u << tl));
          vt &= dh >= 32 ? ~0u : (dh <= 0 ? 0u : ((1u << dh) - 1u));
          if (row >= jhi) vt = 0u;
          npref += (unsigned)__popc(vt);
          valid = 0;
#pragma unroll
          for (int kk = 0; kk < 8; ++kk)                  // t = 4 kk + q -> bit 8 q + kk
            valid |= ((((vt >> (4 * kk)) & 0xFu) * 0x00204081u) & 0x01010101u) << kk;
        }
        // The MMA carried the threshold as a bias column (product - lo16): a
        // candidate's sign bit is clear.  Top bytes of four products per word.
        uint32_t sg = 0;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
          const uint32_t lo2 = __byte_perm(v[4 * kk], v[4 * kk + 1], 0x0073u);
          const uint32_t hi2 = __byte_perm(v[4 * kk + 2], v[4 * kk + 3], 0x0073u);
          const uint32_t g = __byte_perm(lo2, hi2, 0x5410u);
          sg |= ((g >> 7) & 0x01010101u) << kk;
        }
        cm[h] = ~sg & valid;
        cnt += __popc(cm[h]);
      }
      // one slot range per warp and item in the 32-row block's list
      int incl = cnt;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, d);
        if (lane >= d) incl += t;
      }
      const int total = __shfl_sync(FULL, incl, 31);
      if (total) {
        const int blk = row0w >> 5;
        int bpos = 0;
        if (lane == 0) bpos = atomicAdd(A.ccnt + blk, total);
        bpos = __shfl_sync(FULL, bpos, 0);
        const int64_t off = A.coff[blk];
        const int64_t cap = A.coff[blk + 1] - off;
        int64_t pos = (int64_t)bpos + incl - cnt;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t j0 = (uint32_t)(kPN * w.ct + 64 * p + 32 * h);
          uint32_t m = cm[h];
          while (m) {
            const int bit = __ffs(m) - 1;
            m &= m - 1;
            const int t = 4 * (bit & 7) + (bit >> 3);
            if (pos < cap) A.cand[off + pos] = ((uint32_t)lane << 27) | (j0 + (uint32_t)t);
            ++pos;
          }
        }
        if (lane == 0 && (int64_t)bpos + total > cap) atomicExch(A.overflow, 1);
      }
    }
    npref = __reduce_add_sync(FULL, (unsigned)npref);
    if (lane == 0 && npref && A.stats) atomicAdd(A.stats, npref);
  }
  __syncthreads();
  fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase) : "memory");
}

size_t pf_smem() {
  return 1024 + 2 * (size_t)kABytes + (size_t)kPStages * kBBytes + (4 + 2 * kPStages + 5) * 8 +
         16 + 16;
}

// unit16 rows (Kp halves) -> two [n][64] copies, zero padded, with the
// threshold as a bias column in the last half (S < 64 leaves it free): the row
// side (A) holds 1.0 there and the column side (B) -lo16', lo16' the largest
// FP16 value not above lo16, so each product comes out of the MMA as
// U_i . U_j - lo16'.
__global__ void k_pad_unit16(const uint16_t *__restrict__ u, int Kp, int64_t n, float lo16,
                             uint16_t *__restrict__ outA, uint16_t *__restrict__ outB) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   // one half each
  if (i >= n * kPK) return;
  const int64_t r = i / kPK;
  const int k = (int)(i - r * kPK);
  uint16_t a = k < Kp ? u[r * Kp + k] : (uint16_t)0, b = a;
  if (k == kPK - 1) {
    a = __half_as_ushort(__float2half_rn(1.0f));
    b = __half_as_ushort(__hneg(__float2half_rd(lo16)));
  }
  outA[i] = a;
  outB[i] = b;
}

// Exclusive prefix sums of one CTA (1024 threads) over v(0 .. count-1) into
// out[0 .. count]; v(k) a value the caller's functor gives.
template <class F, class T>
__device__ void block_scan_into(int64_t count, F v, T *out) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t per = (count + 1023) / 1024;
  const int64_t a = min(count, t * per), b = min(count, a + per);
  int64_t sum = 0;
  for (int64_t k = a; k < b; ++k) sum += v(k);
  part[t] = sum;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int64_t add = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += add;
    __syncthreads();
  }
  int64_t run = t ? part[t - 1] : 0;
  for (int64_t k = a; k < b; ++k) {
    out[k] = (T)run;
    run += v(k);
  }
  if (t == 1023) out[count] = (T)part[1023];
}

// List offsets of the 32-row blocks: capacities from the kept fraction
// (32 (n - 32 b) pairs x frac + 256, rounded up to 32) or given ones.
__global__ void k_tc5_coff(int64_t n, double frac, const int64_t *caps, int64_t *coff) {
  const int64_t B32 = (n + 31) / 32;
  block_scan_into(B32, [&](int64_t b) -> int64_t {
    if (caps) return caps[b];
    const double pairs = 32.0 * (double)max((int64_t)0, n - 32 * b);
    return (((int64_t)(pairs * frac) + 256 + 31) & ~(int64_t)31);
  }, coff);
}

// Item table of a pass (see sym_tc5_items).
__global__ void k_tc5_items(int RB, int NT, int ct_lo, int32_t *item0) {
  block_scan_into((int64_t)RB, [&](int64_t rb) -> int64_t {
    return (int64_t)max(0, NT - max((kPM * (int)rb) / kPN, ct_lo));
  }, item0);
}

}  // namespace

// Items (128-row block, 256-column tile) of the pairs i < j with j in
// [cb, ce): row blocks below ce, column tiles from cb / 256 (and from the
// tile of the block's first row) below ce; item0[rb] = the first item of row
// block rb, item0[RB] = the total.
int sym_tc5_items(int64_t cb, int64_t ce, int *RB, int *NT) {
  *RB = (int)((ce + kPM - 1) / kPM);
  *NT = (int)((ce + kPN - 1) / kPN);
  const int ct_lo = (int)(cb / kPN);
  int tot = 0;
  for (int rb = 0; rb < *RB; ++rb) tot += std::max(0, *NT - std::max((kPM * rb) / kPN, ct_lo));
  return tot;
}

// Total list capacity of the frac-based capacities (the arithmetic of k_tc5_coff).
int64_t tc5_capacity(int64_t n, double frac) {
  int64_t tot = 0;
  for (int64_t b = 0; b < (n + 31) / 32; ++b) {
    const double pairs = 32.0 * (double)std::max<int64_t>(0, n - 32 * b);
    tot += ((int64_t)(pairs * frac) + 256 + 31) & ~(int64_t)31;
  }
  return tot;
}

void launch_tc5_coff(int64_t n, double frac, const int64_t *caps, int64_t *coff, cudaStream_t s) {
  k_tc5_coff<<<1, 1024, 0, s>>>(n, frac, caps, coff);
}

void launch_tc5_items(int64_t cb, int64_t ce, int32_t *item0, cudaStream_t s) {
  const int RB = (int)((ce + kPM - 1) / kPM), NT = (int)((ce + kPN - 1) / kPN);
  k_tc5_items<<<1, 1024, 0, s>>>(RB, NT, (int)(cb / kPN), item0);
}

void launch_pad_unit16(const GraphArgs &g, float lo16, uint16_t *u16p, cudaStream_t s) {
  const int64_t nh = g.n * kPK;
  if (nh > 0)
    k_pad_unit16<<<(unsigned)((nh + 255) / 256), 256, 0, s>>>(g.unit16, g.Kp, g.n, lo16, u16p,
                                                              u16p + nh);
}

int launch_sym_prefilter(const GraphArgs &g, const uint16_t *u16p, int64_t cb, int64_t ce,
                         const int32_t *item0, int RB, int NT, int items, uint32_t *cand,
                         const int64_t *coff, int32_t *ccnt, int *overflow, int *err, int sms,
                         cudaStream_t s, const char **why) {
  if (g.n == 0 || items == 0) return RBG_OK;
  auto enc = encode_fn();
  if (!enc) {
    *why = "cuTensorMapEncodeTiled is not available";
    return RBG_ERR_CUDA;
  }
  if (g.Kp > kPK || g.S >= kPK || g.n >= ((int64_t)1 << 27) || ((uintptr_t)u16p & 15u) != 0 ||
      cb < 0 || ce > g.n || cb >= ce) {
    *why = "prefilter operand layout";
    return RBG_ERR_ARG;
  }
  CUtensorMap map[2];
  std::memset(map, 0, sizeof(map));
  const cuuint64_t dims[2] = {(cuuint64_t)kPK, (cuuint64_t)g.n};
  const cuuint64_t strides[1] = {(cuuint64_t)kPK * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kPK, (cuuint32_t)kPM};
  const cuuint32_t estr[2] = {1, 1};
  for (int side = 0; side < 2; ++side) {       // rows (A), then columns (B)
    const CUresult r = enc(&map[side], CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
                           (void *)(u16p + (size_t)side * g.n * kPK), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      *why = "cuTensorMapEncodeTiled failed";
      return RBG_ERR_CUDA;
    }
  }
  PfArgs A;
  A.jlo = (int)cb;
  A.jhi = (int)ce;
  A.ct_lo = (int)(cb / kPN);
  A.item0 = item0;
  A.RB = RB;
  A.NT = NT;
  A.items = items;
  A.cand = cand;
  A.coff = coff;
  A.ccnt = ccnt;
  A.overflow = overflow;
  A.stats = g.stats;
  A.err = err;
  cudaError_t e = cudaSuccess;
  {
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    e = cudaFuncSetAttribute(k_sym_prefilter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)pf_smem());
  }
  if (e == cudaSuccess) {
    const int grid = std::max(1, std::min(sms, items));
    k_sym_prefilter<<<grid, kPThreads, pf_smem(), s>>>(map[0], map[1], A);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    *why = cudaGetErrorString(e);
    return RBG_ERR_CUDA;
  }
  return RBG_OK;
}

}  // namespace rbg
