// Dense regime on the 5th-generation tensor cores, hand-written for sm_100a.
//
// The register-match count of contigs i and j (pmh_match_count16,
// src/rabbitbin.cpp:1261-1293: registers with equal nonzero codes) is the dot
// product X_i . X_j of their binary one-hot rows over the (register, code)
// pairs that occur in the assembly (kernels_onehot.cu builds X).  The small
// path (build_graph_allpairs, src/impl/rb_graph.cpp:7-72) needs every pair's
// count, so the counts are one int8 contraction X X^T, computed here with
// tcgen05.mma kind::i8 into TMEM and consumed in the same kernel: no count
// matrix is written to memory.
//
// CTA tile: 256 rows x 256 columns = two UMMA 128x256 accumulators (A rows
// 0-127 and 128-255 against the same B columns), which fill the 512 TMEM
// columns of the SM.  The one-hot width is walked in chunks of 128 bytes (one
// 128-byte swizzle atom): TMA brings the chunk of the 256 A rows and the 256
// B rows (64 KB) into a 3-stage shared-memory ring.  Warp 0 issues the TMA
// loads, warp 1 allocates TMEM and issues the MMAs (4 K-steps of 32 per
// chunk per accumulator), warps 2-17 are the epilogue: each thread owns one
// row and one 128-column half of the tile, reads its 128 counts from TMEM in
// one load as 16-bit values (tcgen05.ld 32x32b .pack::16b; the counts are at
// most m < 4096), frees TMEM for the next tile's MMAs at once, and then keeps
// the row maxima and appends the candidates above the admission floor to its
// own list in global memory while the next tile's MMAs run.
//
// List keys are 32 bits: rank << 20 | (0xFFFFF - j), where rank is the dense
// rank of the pair's similarity among the distinct values of the similarity
// table (k_sv_rank; the table is non-decreasing in the count).  Their order is
// the order of the similarity keys (similarity bits << 32 | ~j) the other
// dense kernels rank by, ties in the similarity included, for j < 2^20.  A
// list holds up to 1024 keys; with room for every column of its group no cut
// ever runs in the kernel, otherwise a list that reaches its capacity is cut
// to the K best by the warp together (select_topk32), which raises its
// threshold.
//
// Work split: the CTAs form a GR x GC grid; CTA (a, b) takes the row blocks
// a, a + GR, ... and, in each, the column tiles of column group b, so at any
// moment GR row blocks and GC column tiles are in use (their operands stay in
// L2).  Each (row, column group, half) has its own list: k_merge_onehot then
// selects a row's top-K from its 2 GC lists and writes the similarity keys,
// exactly what the other dense kernels produce (top-K keys over the
// candidates above the admission floor, maxima over all other contigs and
// over the candidates).
//
// Every wait on an mbarrier is bounded (2 s of %globaltimer); a wait that
// runs out records an error code for the host and the CTA stops issuing work,
// waits (bounded) for its own copies and MMAs in flight, frees its TMEM and
// returns.  No TMA load uses cluster multicast.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "rbg_internal.h"
#include "select_topk.cuh"
#include "tc05.cuh"

namespace rbg {
namespace {

using namespace tc05;

constexpr int kTM = 256;                      // rows per CTA tile
constexpr int kTN = 256;                      // columns per CTA tile
constexpr int kKC = 128;                      // one-hot bytes per stage (one swizzle atom)
constexpr int kStages = 3;
constexpr int kHalfBytes = 128 * kKC;         // one 128-row operand block: 16 KB
constexpr int kStageBytes = (kTM + kTN) * kKC;   // 64 KB
constexpr int kEpiWarps = 16;
constexpr int kCapW32 = 32;                   // list capacity: 32 * kCapW32 keys
constexpr int kThreads = (2 + kEpiWarps) * 32;
constexpr unsigned FULL = 0xffffffffu;

// instruction descriptor: D s32 (bits 4-5 = 2), A and B unsigned 8-bit (bits
// 7-9, 10-12 = 0), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22,
// M >> 4 at bits 24-28
constexpr uint32_t kIdesc = (2u << 4) | ((uint32_t)(kTN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

struct OhArgs {
  GraphArgs g;
  int64_t rows;          // rows scored: [g.row_lo, g.row_lo + rows)
  int nkc;               // one-hot chunks of 128 bytes
  int RB, NT;            // 256-row blocks, 256-column tiles
  int GR, GC;            // CTA grid: row groups x column groups
  uint32_t *cand;        // [rows32 x 2 GC x 32] lists of cap keys
  int cap;               // keys per list (multiple of 32, <= 1024, >= K + 136)
  int32_t *cand_cnt;     // [rows32 x 2 GC x 32]
  const uint32_t *tab;   // rank[m + 1], value[m + 1], admission count, count-key flag
  int *err;              // set when a bounded wait runs out
};

__device__ __forceinline__ void mma_i8(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dt), "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
}

// 128 consecutive TMEM columns of this warp's 32 lanes as 16-bit values, two
// per register (column 2k in the low half of v[k]); the counts are below 2^16.
__device__ __forceinline__ void tmem_ld128_pack16(uint32_t taddr, uint32_t (&v)[64]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.pack::16b.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Named barrier 1 of the epilogue warps; returns the OR of every thread's flag.
__device__ __forceinline__ uint32_t epi_barrier_or(uint32_t flag) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "barrier.cta.red.or.pred po, 1, %2, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(out)
      : "r"(flag), "n"(kEpiWarps * 32)
      : "memory");
  return out;
}

// Smallest count whose similarity rank is at least R (rank is non-decreasing).
__device__ __forceinline__ uint32_t rank_floor(const uint16_t *rank, int m, uint32_t R) {
  int lo = 0, up = m + 1;
  while (lo < up) {
    const int mid = (lo + up) >> 1;
    if (rank[mid] >= R) up = mid; else lo = mid + 1;
  }
  return (uint32_t)max(lo, 1);
}

// The tiles of CTA (a, b): row blocks a, a + GR, ...; columns tiles
// [c0, c1) of column group b.
__device__ __forceinline__ void col_range(const OhArgs &A, int b, int &c0, int &c1) {
  c0 = (int)((int64_t)b * A.NT / A.GC);
  c1 = (int)((int64_t)(b + 1) * A.NT / A.GC);
}

__global__ void __launch_bounds__(kThreads, 1)
k_onehot_mma(const __grid_constant__ CUtensorMap tmap, const OhArgs A) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte aligned stage ring (the swizzle pattern follows address bits)
  uint8_t *ring = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *bars = (uint64_t *)(ring + kStages * kStageBytes);
  // bars: full[kStages], empty[kStages], tmem_full, tmem_empty, mma_done
  uint32_t *tmem_slot = (uint32_t *)(bars + 2 * kStages + 3);
  uint32_t *nzw = tmem_slot + 4;               // [2][8] candidate-flag words of a tile
  int *abort_flag = (int *)(nzw + 16);
  uint16_t *rank = (uint16_t *)(abort_flag + 4);   // [m + 1] similarity rank of a count
  // [11][512] staged keys of the epilogue threads (slot k of thread t at k * 512 + t)
  uint32_t *stage = (uint32_t *)(((uintptr_t)(rank + A.g.m + 1) + 15) & ~(uintptr_t)15);

  const GraphArgs &g = A.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = blockIdx.x / A.GC, b = blockIdx.x % A.GC;
  int c0, c1;
  col_range(A, b, c0, c1);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kStages + s); };
  const uint32_t tfull = bar0 + 8u * (2 * kStages), tempty = tfull + 8u, mdone = tfull + 16u;

  for (int i = threadIdx.x; i <= g.m; i += kThreads) rank[i] = (uint16_t)A.tab[i];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(tfull, 1);
    mbar_init(tempty, kEpiWarps * 32);
    mbar_init(mdone, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {                               // TMEM: all 512 columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;"
                 ::"r"(smem_u32(tmem_slot)) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tbase = *tmem_slot;
  const int nrb = (A.RB - a + A.GR - 1) / A.GR;  // row blocks of this CTA

  if (warp == 0) {
    // ── TMA producer ──
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t issued = 0;                       // bit s: stage s holds an issued load
      uint32_t last_ph = 0;                      // bit s: phase of its last load
      bool ok = true;
      for (int r = 0; r < nrb && ok; ++r) {
        const int y_a = (int)(g.row_lo + (int64_t)(a + r * A.GR) * kTM);
        for (int ct = c0; ct < c1 && ok; ++ct) {
          for (int kc = 0; kc < A.nkc; ++kc) {
            if (!mbar_wait(empty_bar(s), ph ^ 1u, A.err, 1) || *(volatile int *)abort_flag) {
              ok = false;
              *(volatile int *)abort_flag = 1;
              break;
            }
            const uint32_t dst = smem_u32(ring + (size_t)s * kStageBytes);
            mbar_expect_tx(full_bar(s), kStageBytes);
            tma_load(dst, &tmap, kc * kKC, y_a, full_bar(s));
            tma_load(dst + 2 * kHalfBytes, &tmap, kc * kKC, ct * kTN, full_bar(s));
            issued |= 1u << s;
            last_ph = (last_ph & ~(1u << s)) | (ph << s);
            if (++s == kStages) { s = 0; ph ^= 1u; }
          }
        }
      }
      // copies in flight land before the CTA leaves (already true when the
      // MMAs consumed them)
      for (int t = 0; t < kStages; ++t)
        if ((issued >> t) & 1u) mbar_wait(full_bar(t), (last_ph >> t) & 1u, A.err, 2);
    }
  } else if (warp == 1) {
    // ── MMA issuer ──
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0, tph = 0;
      bool ok = true;
      for (int r = 0; r < nrb && ok; ++r) {
        for (int ct = c0; ct < c1 && ok; ++ct) {
          if (!mbar_wait(tempty, tph ^ 1u, A.err, 3) || *(volatile int *)abort_flag) {
            ok = false;
            *(volatile int *)abort_flag = 1;
            break;
          }
          fence_after();
          for (int kc = 0; kc < A.nkc; ++kc) {
            if (!mbar_wait(full_bar(s), ph, A.err, 4) || *(volatile int *)abort_flag) {
              ok = false;
              *(volatile int *)abort_flag = 1;
              break;
            }
            fence_after();
            const uint32_t st = smem_u32(ring + (size_t)s * kStageBytes);
            const uint64_t da0 = sdesc128(st), da1 = sdesc128(st + kHalfBytes),
                           db = sdesc128(st + 2 * kHalfBytes);
#pragma unroll
            for (int k = 0; k < kKC / 32; ++k) {
              const uint32_t acc = (kc | k) ? 1u : 0u;
              // +32 bytes of K per step: +2 in the descriptor's 16-byte units
              mma_i8(tbase, da0 + 2 * k, db + 2 * k, acc);
              mma_i8(tbase + kTN, da1 + 2 * k, db + 2 * k, acc);
            }
            mma_commit(empty_bar(s));            // the stage is free once these finish
            if (++s == kStages) { s = 0; ph ^= 1u; }
          }
          if (!ok) break;
          mma_commit(tfull);                     // the tile's counts are in TMEM
          tph ^= 1u;
        }
      }
      mma_commit(mdone);                         // every MMA issued has finished
      mbar_wait(mdone, 0, A.err, 5);
    }
  } else {
    // ── epilogue: thread = (row, column half of the tile) ──
    const int e = warp - 2;                      // 0..15
    const int q = warp & 3;                      // TMEM lane quarter of this warp
    const int half = (e >> 2) & 1;               // accumulator 0 or 1
    const int ch = e >> 3;                       // columns [128 ch, 128 ch + 128) of the tile
    const int K = g.K, m = g.m;
    const int n = (int)g.n;                      // < 2^20 (onehot_mma_fits)
    const int P = 2 * A.GC;                      // lists per row: column group x half
    const uint32_t cf = max(A.tab[2 * (m + 1)], 1u);   // counts above the floor
    const bool ident = A.tab[2 * (m + 1) + 1] != 0u;    // keys carry the count
    // Keys go to the list eight at a time (two 16-byte stores): they are staged
    // in shared memory first (up to 11 per thread).  fill (keys in the list)
    // stays a multiple of 8 except after the row's last drain.
    uint32_t *stg = stage + (threadIdx.x - 64);
    uint32_t tph = 0;
    int tcount = 0;
    bool ok = true;
    for (int r = 0; r < nrb && ok; ++r) {
      const int rb = a + r * A.GR;
      const int li = rb * kTM + half * 128 + q * 32 + lane;   // local row
      const int i = (int)g.row_lo + li;
      const bool valid_row = li < A.rows;
      const uint32_t nz_i = valid_row ? g.anynz[i] : 0u;
      uint32_t *buf = nullptr;
      size_t slot = 0;
      if (valid_row) {
        slot = ((size_t)(li >> 5) * P + 2 * b + ch) * 32 + (size_t)(li & 31);
        buf = A.cand + slot * (size_t)A.cap;
      }
      int fill = 0, qn = 0;                      // keys in the list, staged keys
      auto push = [&](uint32_t key) {
        stg[qn * 512] = key;
        ++qn;
      };
      // after every 4 candidates (at most 11 staged): 8 keys to the list
      auto flush = [&]() {
        if (qn >= 8) {
          const uint4 lo = make_uint4(stg[0], stg[512], stg[1024], stg[1536]);
          const uint4 hi = make_uint4(stg[2048], stg[2560], stg[3072], stg[3584]);
          *reinterpret_cast<uint4 *>(buf + fill) = lo;
          *reinterpret_cast<uint4 *>(buf + fill + 4) = hi;
          fill += 8;
          qn -= 8;
          for (int k = 0; k < qn; ++k) stg[k * 512] = stg[(k + 8) * 512];
        }
      };
      auto drain = [&]() {
        for (int k = 0; k < qn; ++k) buf[fill + k] = stg[k * 512];
        fill += qn;
        qn = 0;
      };
      uint32_t thr = 0;                          // after a cut: keys <= thr are out
      uint32_t cthr = cf;
      uint32_t mx_a = 0, mx_c = 0;
      for (int ct = c0; ct < c1; ++ct, ++tcount) {
        // candidate flags of the tile's columns (anynz), one word per warp of the first 8
        if (e < kTN / 32) {
          const int j = ct * kTN + e * 32 + lane;
          const unsigned w = __ballot_sync(FULL, j < n && g.anynz[j]);
          if (lane == 0) nzw[(tcount & 1) * 8 + e] = w;
        }
        uint32_t bad = mbar_wait(tfull, tph, A.err, 6) ? 0u : 1u;
        if (*(volatile int *)abort_flag) bad = 1u;
        // one decision for all epilogue threads (they meet at this barrier every tile)
        bad = epi_barrier_or(bad);
        if (bad) {
          ok = false;
          *(volatile int *)abort_flag = 1;
          break;
        }
        fence_after();
        const uint32_t *nzt = nzw + (tcount & 1) * 8 + ch * 4;
        uint32_t pk[64];                         // the 128 counts, two per register
        tmem_ld128_pack16(tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(half * kTN + ch * 128),
                          pk);
        fence_before();
        mbar_arrive(tempty);                     // TMEM is free for the next tile's MMAs
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int j0 = ct * kTN + ch * 128 + c * 32;
          // valid columns: j < n and j != i; candidates: valid and (nz_i or nz_j)
          uint32_t vm = ~0u;
          if (j0 + 32 > n) vm = (n <= j0) ? 0u : (~0u >> (32 - (n - j0)));
          if (i >= j0 && i < j0 + 32) vm &= ~(1u << (i - j0));
          if (!valid_row) vm = 0u;
          const uint32_t cm = vm & (nz_i ? ~0u : nzt[c]);
          bool hit = false;
          const bool full = __all_sync(FULL, vm == ~0u && cm == ~0u);   // warp-uniform
          if (full) {
            // both halves at once: maximum and the test against the count threshold
            uint32_t m2 = 0, h2 = 0;
            const uint32_t c2 = cthr * 0x10001u;  // cthr <= m + 1 < 2^16
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              m2 = __vmaxu2(m2, pk[c * 16 + k]);
              h2 |= __vcmpgeu2(pk[c * 16 + k], c2);
            }
            const uint32_t cmx = max(m2 & 0xFFFFu, m2 >> 16);
            mx_a = max(mx_a, cmx);
            mx_c = max(mx_c, cmx);
            hit = h2 != 0u;
          } else {
#pragma unroll
            for (int t = 0; t < 32; ++t) {
              const uint32_t v = (pk[c * 16 + (t >> 1)] >> (16 * (t & 1))) & 0xFFFFu;
              const uint32_t va = ((vm >> t) & 1u) ? v : 0u;
              const uint32_t vc = ((cm >> t) & 1u) ? v : 0u;
              mx_a = max(mx_a, va);
              mx_c = max(mx_c, vc);
              hit |= vc >= cthr;
            }
          }
          if (hit) {
            const uint32_t jr = 0xFFFFFu - (uint32_t)j0;
            if (ident && full) {                 // the common case: count keys, every column
#pragma unroll
              for (int t = 0; t < 32; ++t) {
                const uint32_t v = (pk[c * 16 + (t >> 1)] >> (16 * (t & 1))) & 0xFFFFu;
                const uint32_t key = (v << 20) + (jr - (uint32_t)t);
                if (v >= cthr && key > thr) push(key);
                if ((t & 3) == 3) flush();
              }
            } else {
#pragma unroll
              for (int t = 0; t < 32; ++t) {
                const uint32_t v = (pk[c * 16 + (t >> 1)] >> (16 * (t & 1))) & 0xFFFFu;
                if (((cm >> t) & 1u) && v >= cthr) {
                  const uint32_t key = ((ident ? v : (uint32_t)rank[v]) << 20) | (jr - (uint32_t)t);
                  if (key > thr) push(key);
                }
                if ((t & 3) == 3) flush();
              }
            }
          }
        }
        // lists that could not take another tile (128 keys) are cut to the K best
        unsigned need = __ballot_sync(FULL, fill + qn > A.cap - 128);
        if ((need >> lane) & 1u) drain();
        while (need) {
          const int L = __ffs(need) - 1;
          need &= need - 1;
          uint32_t *lb = (uint32_t *)__shfl_sync(FULL, (unsigned long long)buf, L);
          const int lc = __shfl_sync(FULL, fill, L);
          __syncwarp();
          const uint32_t t = select_topk32<kCapW32>(lb, lc, K);
          if (lane == L) {
            thr = t;
            fill = (K + 7) & ~7;                 // zero keys pad to a multiple of 8
            for (int k = K; k < fill; ++k) buf[k] = 0u;
            cthr = ident ? max(t >> 20, 1u) : rank_floor(rank, m, t >> 20);
          }
        }
        tph ^= 1u;
      }
      if (!ok) break;
      // this half's list of the column group (cut by the merge), the maxima
      drain();
      if (valid_row) {
        A.cand_cnt[slot] = fill;
        if (mx_a) atomicMax(g.maxcnt_all + i, mx_a);
        if (mx_c) atomicMax(g.maxcnt_cand + i, mx_c);
      }
      if (b == 0 && ch == 0 && g.stats) {        // every other contig, once per row
        const unsigned vr = __ballot_sync(FULL, valid_row);
        if (lane == 0 && vr)
          atomicAdd(g.stats + 1, (unsigned long long)__popc(vr) * (unsigned long long)(n - 1));
      }
    }
  }
  __syncthreads();
  fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase) : "memory");
}

size_t oh_smem(int m) {
  return 1024 + (size_t)kStages * kStageBytes + (2 * kStages + 3) * 8 + 16 + 64 + 16 +
         (size_t)(m + 1) * 2 + 16 + (size_t)11 * kEpiWarps * 32 * 4;
}

// One warp: rank[c] = distinct similarity values below sv[c] (sv is
// non-decreasing in the count), value[rank] = sv bits, the admission count
// (the first count whose similarity is above the floor; m + 1 when none is)
// and the flag of the common case where the similarity strictly increases
// from the admission count on: keys then carry the count instead of the rank
// (the same order) and value[] is indexed by the count.
// tab: rank at [0, m], value at [m + 1, 2m + 1], admission count at 2m + 2,
// the flag at 2m + 3.
__global__ void k_sv_rank(const uint32_t *__restrict__ sv, int m, uint32_t fbits,
                          uint32_t *__restrict__ tab) {
  const int lane = threadIdx.x;
  const int n1 = m + 1, per = (n1 + 31) / 32;
  const int a = min(lane * per, n1), b = min(a + per, n1);
  int ch = 0;
  uint32_t first = (uint32_t)n1;
  for (int c = a; c < b; ++c) {
    const uint32_t x = sv[c];
    if (c > 0 && x != sv[c - 1]) ++ch;
    if (first == (uint32_t)n1 && x > fbits) first = (uint32_t)c;
  }
  int inc = ch;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int t = __shfl_up_sync(FULL, inc, d);
    if (lane >= d) inc += t;
  }
  uint32_t r = (uint32_t)(inc - ch);
  for (int c = a; c < b; ++c) {
    const uint32_t x = sv[c];
    if (c > 0 && x != sv[c - 1]) ++r;
    tab[c] = r;
    tab[n1 + r] = x;                             // equal values for equal ranks
  }
  first = __reduce_min_sync(FULL, first);
  __syncwarp();
  // the similarity strictly increases from the admission count on: the count
  // itself orders the keys, and value[] is indexed by the count
  const bool ident = first < (uint32_t)n1 && tab[m] - tab[first] == (uint32_t)m - first;
  if (ident) {
    __syncwarp();
    for (int c = a; c < b; ++c) tab[n1 + c] = sv[c];
  }
  if (lane == 0) {
    tab[2 * n1] = first;
    tab[2 * n1 + 1] = ident ? 1u : 0u;
  }
}

// Warp per row: the K best of the row's P lists of 32-bit keys (list of row
// r, list s at ((r/32 * P + s) * 32 + r%32) * cap), 32 keys a step into a
// 1024-key shared buffer that select_topk32 cuts to K when it could not take
// another step; after the first cut only keys above the K-th best so far are
// kept.  The kept keys leave as similarity keys (similarity bits << 32 | ~j).
constexpr int kOmWarps = 8;
constexpr int kOmBuf = 32 * kCapW32;
constexpr int kOmDepth = 8;                    // steps of 32 keys loaded ahead

__global__ void __launch_bounds__(kOmWarps * 32)
k_merge_onehot(GraphArgs g, const uint32_t *__restrict__ cand, const int32_t *__restrict__ cnt,
               int cap, int P, const uint32_t *__restrict__ tab, int64_t rows) {
  __shared__ uint32_t mk[kOmWarps][kOmBuf];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t q = (int64_t)blockIdx.x * kOmWarps + wib;
  if (q >= rows) return;
  const int64_t row = g.row_lo + q;
  const int K = g.K;
  uint32_t *keys = mk[wib];
  const size_t br0 = (size_t)(q >> 5) * P * 32 + (size_t)(q & 31);
  const int cl = lane < P ? cnt[br0 + (size_t)lane * 32] : 0;    // P <= 32
  const unsigned below = (1u << lane) - 1u;
  int fill = 0;
  uint32_t thr = 0;
  for (int s = 0; s < P; ++s) {
    const int c = __shfl_sync(FULL, cl, s);
    const uint32_t *src = cand + (br0 + (size_t)s * 32) * cap;
    for (int i0 = 0; i0 < c; i0 += 32 * kOmDepth) {
      uint32_t kv[kOmDepth];                     // the loads of several steps in flight
#pragma unroll
      for (int u = 0; u < kOmDepth; ++u) {
        const int i = i0 + 32 * u + lane;
        kv[u] = i < c ? __ldg(src + i) : 0u;
      }
#pragma unroll
      for (int u = 0; u < kOmDepth; ++u) {
        const bool take = kv[u] > thr;
        const unsigned m = __ballot_sync(FULL, take);
        if (take) keys[fill + __popc(m & below)] = kv[u];
        fill += __popc(m);
        __syncwarp();
        if (fill > kOmBuf - 32) {
          thr = select_topk32<kCapW32>(keys, fill, K);
          fill = K;
        }
      }
    }
  }
  if (fill > K) {
    select_topk32<kCapW32>(keys, fill, K);
    fill = K;
  }
  const uint32_t *value = tab + g.m + 1;
  for (int i = lane; i < fill; i += 32) {
    const uint32_t key = keys[i];
    const uint32_t j = 0xFFFFFu - (key & 0xFFFFFu);
    g.topk[row * K + i] = ((uint64_t)__ldg(value + (key >> 20)) << 32) | (uint64_t)(~j);
  }
  if (lane == 0) g.topk_cnt[row] = fill;
}

}  // namespace

bool onehot_mma_fits(int64_t n, int m) { return n < ((int64_t)1 << 20) && m < 4096; }

// Keys per (row, column group, half) list: every column the list covers (no
// cut in the kernel) up to 1024, and at least K + 136 so that a tile's 128
// columns always fit after a cut to K (padded to a multiple of 8).  cap_max
// (> 0) lowers it, down to that floor.
int onehot_mma_cap(int64_t n, int GC, int K, int cap_max) {
  const int64_t NT = (n + 255) / 256;
  const int64_t cols = std::min<int64_t>(n, (NT + GC - 1) / GC * 128);
  int cap = (int)std::min<int64_t>(32 * kCapW32, (cols + 136 + 31) / 32 * 32);
  if (cap_max > 0) cap = std::min(cap, cap_max);
  return std::max(cap, (K + 136 + 31) & ~31);
}

// GR x GC CTA grid for RB row blocks and NT column tiles on `sms` SMs: the
// split with the smallest largest share of tiles, then the fewest column
// groups (fewer lists per row), then the fewest CTAs.
void onehot_mma_grid(int RB, int NT, int sms, int *GR, int *GC) {
  int bestR = 1, bestC = 1;
  int64_t best = INT64_MAX;
  for (int gr = 1; gr <= std::min(RB, sms); ++gr)
    for (int gc = 1; gc <= std::min(NT, std::min(16, sms / gr)); ++gc) {
      const int64_t load = (int64_t)((RB + gr - 1) / gr) * ((NT + gc - 1) / gc);
      if (load < best || (load == best && (gc < bestC || (gc == bestC && gr * gc < bestR * bestC)))) {
        best = load;
        bestR = gr;
        bestC = gc;
      }
    }
  *GR = bestR;
  *GC = bestC;
}

// X: [n][ldx] one-hot rows (ldx a multiple of 128, zero padded); the rows
// [g.row_lo, g.row_lo + rows) against every column, on a GR x GC CTA grid.
// cand/cand_cnt hold ceil(rows / 32) * 32 * 2 GC lists of cap keys (cand_cnt
// is zeroed here); tab [2m + 4] receives the rank tables.  The three launches:
// ranks, counts and lists, top-K per row.  Returns RBG_OK or a status with
// *why set.
int launch_onehot_mma(const GraphArgs &g, const int8_t *X, int64_t ldx, int64_t rows,
                      uint32_t *cand, int cap, int32_t *cand_cnt, uint32_t *tab, int *err, int GR,
                      int GC, cudaStream_t s, const char **why) {
  auto enc = encode_fn();
  if (!enc) {
    *why = "cuTensorMapEncodeTiled is not available";
    return RBG_ERR_CUDA;
  }
  if (ldx % kKC != 0 || ((uintptr_t)X & 15u) != 0 || !onehot_mma_fits(g.n, g.m) || GC > 16 ||
      g.K < 1 || g.K > 448 || cap > 32 * kCapW32 || cap < g.K + 136 || cap % 32 != 0) {
    *why = "one-hot operand layout";
    return RBG_ERR_ARG;
  }
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  const cuuint64_t dims[2] = {(cuuint64_t)ldx, (cuuint64_t)g.n};
  const cuuint64_t strides[1] = {(cuuint64_t)ldx};
  const cuuint32_t box[2] = {(cuuint32_t)kKC, (cuuint32_t)kTM};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)X, dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    *why = "cuTensorMapEncodeTiled failed";
    return RBG_ERR_CUDA;
  }
  OhArgs A;
  A.g = g;
  A.rows = rows;
  A.nkc = (int)(ldx / kKC);
  A.RB = (int)((rows + kTM - 1) / kTM);
  A.NT = (int)((g.n + kTN - 1) / kTN);
  A.GR = GR;
  A.GC = GC;
  A.cand = cand;
  A.cap = cap;
  A.cand_cnt = cand_cnt;
  A.tab = tab;
  A.err = err;
  const size_t nslots = (size_t)((rows + 31) / 32) * 32 * 2 * GC;
  cudaError_t e = cudaMemsetAsync(cand_cnt, 0, nslots * sizeof(int32_t), s);
  if (e == cudaSuccess) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    e = cudaFuncSetAttribute(k_onehot_mma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)oh_smem(4096));
  }
  if (e == cudaSuccess) {
    k_sv_rank<<<1, 32, 0, s>>>(g.sv_bits, g.m, (uint32_t)(g.key_floor >> 32), tab);
    k_onehot_mma<<<GR * GC, kThreads, oh_smem(g.m), s>>>(map, A);
    if (rows > 0)
      k_merge_onehot<<<(unsigned)((rows + kOmWarps - 1) / kOmWarps), kOmWarps * 32, 0, s>>>(
          g, cand, cand_cnt, cap, 2 * GC, tab, rows);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    *why = cudaGetErrorString(e);
    return RBG_ERR_CUDA;
  }
  return RBG_OK;
}

}  // namespace rbg
