// All-pairs pass: per row top-K of (similarity, id) keys plus the row maxima
// the calibration reads, over full rows (every ordered pair i != j).
//
// A work item is a block of 32 rows (lane = row) against kWarps column slices,
// one warp per slice; the plain launch maps items to the grid, the batch form
// runs a persistent kernel that pulls (assembly, row block, slice group)
// items from a device counter.  Each row keeps its candidate keys in a
// private global buffer per slice (L2-resident) with the admission threshold
// and fill count in shared memory; when a buffer fills, the owning warp
// selects the K best in registers (radix search of the K-th largest key) and
// raises the threshold to it.  A merge pass then keeps the K best over the
// slices.
//
// Two regimes:
//  * dense (no abundance prune: the N <= 25000 path, S <= 2, RABBIT_NO_ABDFIRST):
//    every pair's register-match count, 4 columns per step over 8-bit code
//    words (row words from shared memory, column words staged by cp.async);
//  * sparse (the abundance-first prune of the fused path): tensor-core FP16
//    products of the unit rows prune almost every pair under a rigorous error
//    bound; the few left are decided by an FP32 chain with its own band and
//    then the AVX-512 order of unit_dot_f exactly.  Survivors queue per warp
//    and are counted by the whole warp, one survivor at a time.
//
// Compiled with -fmad=false; __fmaf_rn marks every fused operation.
#include <algorithm>
#include <cstdint>
#include <cuda_fp16.h>

#include "rbg_internal.h"
#include "select_topk.cuh"

namespace rbg {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kWarps = 4;         // warps per CTA (independent)

// One 16-byte shared-memory load (a single 128-bit access: lanes reading
// consecutive 16-byte blocks take 4 wavefronts for the warp, where four 32-bit
// loads of the same blocks would conflict 4-way each).  Volatile, so it stays
// ordered after the cp.async waits and warp barriers around it.
__device__ __forceinline__ uint4 lds128(const void *p) {
  uint4 v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(a));
  return v;
}

// Row stride (floats) of the unit rows staged in shared memory: an odd number
// of 16-byte units, so lanes gathering rows of random indices spread over all
// eight 16-byte bank groups.
__host__ __device__ __forceinline__ int su_stride(int Su) {
  return ((Su >> 2) & 1) ? Su : Su + 4;
}

// 0x80 in each byte where a and b agree, 0 elsewhere: the low seven bits of
// each byte of a ^ b are tested by an add that cannot carry out of the byte,
// the top bit directly.
__device__ __forceinline__ uint32_t eq_mask(uint32_t a, uint32_t b) {
  const uint32_t x = a ^ b;
  const uint32_t t = (x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
  return ~(t | x) & 0x80808080u;
}
// acc + 128 x (number of equal bytes of two 16-byte blocks); the byte dot
// product with 0x01010101 sums the masks on the FMA pipe, beside the ALU
// work of the masks.
__device__ __forceinline__ uint32_t eq16(const uint4 a, const uint4 b, uint32_t acc) {
  acc = __dp4a(eq_mask(a.x, b.x), 0x01010101u, acc);
  acc = __dp4a(eq_mask(a.y, b.y), 0x01010101u, acc);
  acc = __dp4a(eq_mask(a.z, b.z), 0x01010101u, acc);
  return __dp4a(eq_mask(a.w, b.w), 0x01010101u, acc);
}

// unit_dot_f (src/rabbitbin.cpp:754-796) as an AVX-512 build evaluates it:
// element t feeds lane t % 16 of acc1 in the upper half of a full 32-element
// block, else of acc0 (the masked tail included); then acc0 + acc1 and the
// _mm512_reduce_add_ps tree (lanes i + i+8, i + i+4, i + i+2, 0 + 1).
template <int SMAX>
__device__ __forceinline__ float dot_avx512(const float (&a)[SMAX], const float *b, int S) {
  float acc0[16], acc1[16];
#pragma unroll
  for (int l = 0; l < 16; ++l) { acc0[l] = 0.f; acc1[l] = 0.f; }
  const int lim32 = S & ~31;
#pragma unroll
  for (int t = 0; t < SMAX; ++t) {
    if (t < S) {
      const float bt = __ldg(b + t);
      if ((t & 16) && t < lim32) acc1[t & 15] = __fmaf_rn(a[t], bt, acc1[t & 15]);
      else acc0[t & 15] = __fmaf_rn(a[t], bt, acc0[t & 15]);
    }
  }
  float v[16];
#pragma unroll
  for (int l = 0; l < 16; ++l) v[l] = lim32 ? __fadd_rn(acc0[l], acc1[l]) : acc0[l];
#pragma unroll
  for (int l = 0; l < 8; ++l) v[l] = __fadd_rn(v[l], v[l + 8]);
#pragma unroll
  for (int l = 0; l < 4; ++l) v[l] = __fadd_rn(v[l], v[l + 4]);
  v[0] = __fadd_rn(v[0], v[2]);
  v[1] = __fadd_rn(v[1], v[3]);
  return __fadd_rn(v[0], v[1]);
}

// 16-byte asynchronous global->shared copies (per lane), and their groups.
__device__ __forceinline__ void cp16(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

struct Warp {
  uint64_t *gbuf;     // [32 rows][cap] candidate keys of this warp's rows
  int *cnt;           // smem [32]
  uint64_t *thr;      // smem [32]
  uint32_t *mxc;      // smem [32]
  int cap, K;
};

// Compact every row of the warp whose buffer holds more than `limit` keys.
__device__ __forceinline__ void compact_full_rows(Warp &w, int limit) {
  const int lane = threadIdx.x & 31;
  unsigned full = __ballot_sync(FULL, w.cnt[lane] > limit);
  while (full) {
    const int r = __ffs(full) - 1;
    full &= full - 1;
    const uint64_t P = select_topk<false>(w.gbuf + (size_t)r * w.cap, w.cnt[r], w.K);
    if (lane == 0) { w.cnt[r] = w.K; w.thr[r] = P; }
    __syncwarp();
  }
}

// Register-match counts of up to 32 queued survivors, the warp working on one
// survivor at a time: row codes from shared memory (sA, [32][mpad]) and column
// codes as coalesced 16-byte loads, four survivors in flight.  Lane p ends
// with survivor p's count and admits it.
__device__ __forceinline__ void count_batch_coop(const GraphArgs &g, Warp &w, const int *q, int nq,
                                                 const unsigned char *sA) {
  const int lane = threadIdx.x & 31;
  const int m16 = g.mpad >> 4;
  uint32_t mine = 0;
  for (int p = 0; p < nq; p += 4) {
    const uint4 *ra[4], *cb[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const unsigned e = (unsigned)q[p + u < nq ? p + u : p];
      ra[u] = (const uint4 *)(sA + (size_t)(e >> 27) * g.mpad);
      cb[u] = (const uint4 *)(g.codesB + (int64_t)(e & 0x07FFFFFFu) * g.mpad);
    }
    uint32_t acc[4] = {0u, 0u, 0u, 0u};         // 128 x matches
    for (int t = lane; t < m16; t += 32) {
      uint4 b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) b[u] = __ldg(cb[u] + t);
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] = eq16(lds128(ra[u] + t), b[u], acc[u]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t c = __reduce_add_sync(FULL, acc[u]) >> 7;
      if (lane == p + u) mine = c;
    }
  }
  // Row maxima and admission.  The row state is this warp's own, so lanes of
  // the same row combine in registers and one of them writes: no shared-memory
  // atomics, which serialise when survivors share a row.
  const unsigned act = __ballot_sync(FULL, lane < nq);
  if (lane < nq) {
    const unsigned e = (unsigned)q[lane];
    const int r = (int)(e >> 27);
    const int64_t j = e & 0x07FFFFFFu;
    const unsigned grp = __match_any_sync(act, r);
    const uint32_t mx = __reduce_max_sync(grp, mine);
    const uint64_t key = ((uint64_t)__ldg(g.sv_bits + mine) << 32) | (uint64_t)(~(uint32_t)j);
    const bool adm = key > w.thr[r];
    const unsigned ag = grp & __ballot_sync(act, adm);
    const int base = w.cnt[r];
    if (adm) w.gbuf[(size_t)r * w.cap + base + __popc(ag & ((1u << lane) - 1u))] = key;
    __syncwarp(act);
    if (lane == __ffs(grp) - 1) {
      if (mx > w.mxc[r]) w.mxc[r] = mx;
      w.cnt[r] = base + __popc(ag);
    }
  }
  __syncwarp();
  compact_full_rows(w, w.cap - 32);
}

// Symmetric form of count_batch_coop: the same counts, then each survivor
// (i = row0 + r, j) raises both rows' maxima (row i through the warp's own
// state, row j by an atomic) and, when its similarity passes the admission
// floor, is appended once to the pair list with both rows' counts raised.
// grow0: the assembly's first row in the row space of the pair list.
template <int NF = 4>
__device__ __forceinline__ void count_batch_sym(const GraphArgs &g, const SymOut &o, uint32_t *mxc,
                                                int64_t row0, int64_t grow0, const int *q, int nq,
                                                const unsigned char *sA) {
  const int lane = threadIdx.x & 31;
  const int m16 = g.mpad >> 4;
  uint32_t mine = 0;
  for (int p = 0; p < nq; p += NF) {               // NF survivors' column codes in flight
    const uint4 *ra[NF], *cb[NF];
#pragma unroll
    for (int u = 0; u < NF; ++u) {
      const unsigned e = (unsigned)q[p + u < nq ? p + u : p];
      ra[u] = (const uint4 *)(sA + (size_t)(e >> 27) * g.mpad);
      cb[u] = (const uint4 *)(g.codesB + (int64_t)(e & 0x07FFFFFFu) * g.mpad);
    }
    uint32_t acc[NF];
#pragma unroll
    for (int u = 0; u < NF; ++u) acc[u] = 0u;
    for (int t = lane; t < m16; t += 32) {
      uint4 b[NF];
#pragma unroll
      for (int u = 0; u < NF; ++u) b[u] = __ldg(cb[u] + t);
#pragma unroll
      for (int u = 0; u < NF; ++u) acc[u] = eq16(lds128(ra[u] + t), b[u], acc[u]);
    }
#pragma unroll
    for (int u = 0; u < NF; ++u) {
      const uint32_t c = __reduce_add_sync(FULL, acc[u]) >> 7;
      if (lane == p + u) mine = c;
    }
  }
  const unsigned act = __ballot_sync(FULL, lane < nq);
  bool adm = false;
  int r = 0;
  uint32_t j = 0, svb = 0;
  if (lane < nq) {
    const unsigned e = (unsigned)q[lane];
    r = (int)(e >> 27);
    j = e & 0x07FFFFFFu;
    const unsigned grp = __match_any_sync(act, r);
    const uint32_t mx = __reduce_max_sync(grp, mine);
    if (lane == __ffs(grp) - 1 && mx > mxc[r]) mxc[r] = mx;
    if (mine) atomicMax(g.maxcnt_cand + j, mine);
    if (o.defer) {
      svb = mine;                        // converted once the similarity table exists
      adm = mine > 0;
    } else {
      svb = __ldg(g.sv_bits + mine);
      adm = svb > (uint32_t)(g.key_floor >> 32);
    }
  }
  const unsigned am = __ballot_sync(FULL, adm);
  if (am) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(o.npairs, (unsigned long long)__popc(am));
    base = __shfl_sync(FULL, base, 0);
    if (adm) {
      const unsigned long long pos = base + (unsigned)__popc(am & ((1u << lane) - 1u));
      if (pos < o.cap) {
        const uint32_t gi = (uint32_t)(grow0 + row0 + r), gj = (uint32_t)(grow0 + j);
        o.pairs[pos] = make_uint4(gi, gj, svb, (uint32_t)grow0);
        atomicAdd(o.rowcnt + gi, 1);
        atomicAdd(o.rowcnt + gj, 1);
      }
    }
  }
  __syncwarp();
}

// Dense regime: one work item = 32 rows (row block bx) x the column slices
// kWarps*by .. kWarps*by+3, one warp per slice.
__device__ __forceinline__ void dense_item(const GraphArgs &g, uint64_t *gbuf, int32_t *gcnt,
                                           int cap, int P, int64_t bx, int by,
                                           unsigned char *smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t n = g.n;
  const int64_t rhi = g.row_hi < 0 ? n : g.row_hi;
  const int64_t row0 = g.row_lo + bx * 32;
  const int64_t row = row0 + lane;
  const bool vrow = row < rhi;
  const int mw = g.mpad >> 2;
  const int mwq = ((mw + 27) & ~31) + 4;           // = 4 mod 32 words: conflict-free LDS.128
  const int slice = by * kWarps + warp;              // column slice of this warp
  const int64_t jb = n * slice / P, je = n * (slice + 1) / P;

  // shared: per-warp state, then the 32 row-code rows of the block
  unsigned char *ws = smem + (size_t)warp * 1024;
  uint64_t *thr = (uint64_t *)ws;                  // [32]
  int *cnt = (int *)(thr + 32);                    // [32]
  uint32_t *mxc = (uint32_t *)(cnt + 32);          // [32]
  uint32_t *sA = (uint32_t *)(smem + (size_t)kWarps * 1024);   // [32][mwq]

  thr[lane] = g.key_floor;
  cnt[lane] = 0;
  mxc[lane] = 0;
  const size_t bufrow = ((size_t)bx * P + slice) * 32;  // first buffer row of the warp
  Warp w{gbuf + bufrow * cap, cnt, thr, mxc, cap, g.K};
  const uint8_t nz_row = vrow ? g.anynz[row] : 0;
  unsigned n_pref = 0, n_cmp = 0;
  uint32_t mx_a = 0, mx_c = 0;

  for (int i = threadIdx.x; i < 32 * (mw >> 2); i += blockDim.x) {
    const int r = i / (mw >> 2), t = i - r * (mw >> 2);
    uint4 v = make_uint4(0, 0, 0, 0);
    if (row0 + r < n) v = __ldg((const uint4 *)(g.codesA + (row0 + r) * g.mpad) + t);
    *(uint4 *)(sA + r * mwq + 4 * t) = v;
  }
  __syncthreads();
  const uint32_t *ra = sA + lane * mwq;
  const int m4 = mw >> 2;
  // per-warp ring: 2 stages x 4 columns of B codes
  uint4 *ring = (uint4 *)(smem + (size_t)kWarps * 1024 + 32 * (size_t)mwq * 4) +
                (size_t)warp * 2 * 4 * m4;
  auto stage_cols = [&](int st, int64_t j0) {
    uint4 *dst = ring + (size_t)st * 4 * m4;
    for (int i = lane; i < 4 * m4; i += 32) {
      const int u = i / m4, t = i - u * m4;
      const int64_t j = j0 + u < je ? j0 + u : j0;
      cp16(dst + i, (const uint4 *)(g.codesB + j * g.mpad) + t);
    }
    cp_commit();
  };
  if (jb < je) stage_cols(0, jb);
  int st = 0;
  for (int64_t j0 = jb; j0 < je; j0 += 4, st ^= 1) {
    if (j0 + 4 < je) stage_cols(st ^ 1, j0 + 4); else cp_commit();
    cp_wait1();
    __syncwarp();
    const uint4 *c0 = ring + (size_t)st * 4 * m4;
    const uint4 *c1 = c0 + m4, *c2 = c1 + m4, *c3 = c2 + m4;
    uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;      // 128 x matches
#pragma unroll 2
    for (int t = 0; t < m4; ++t) {
      const uint4 a = lds128(ra + 4 * t);
      a0 = eq16(a, lds128(c0 + t), a0);
      a1 = eq16(a, lds128(c1 + t), a1);
      a2 = eq16(a, lds128(c2 + t), a2);
      a3 = eq16(a, lds128(c3 + t), a3);
    }
    const uint32_t cntq[4] = {a0 >> 7, a1 >> 7, a2 >> 7, a3 >> 7};
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int64_t j = j0 + t;
      const bool other = vrow && j < je && j != row;
      const bool cand = other && (nz_row | __ldg(g.anynz + (j < je ? j : jb)));
      const uint32_t c = cntq[t];
      if (other && c > mx_a) mx_a = c;
      if (cand && c > mx_c) mx_c = c;
      n_cmp += other;
      if (cand) {
        const uint64_t key = ((uint64_t)__ldg(g.sv_bits + c) << 32) | (uint64_t)(~(uint32_t)j);
        if (key > thr[lane]) w.gbuf[(size_t)lane * cap + cnt[lane]++] = key;
      }
    }
    __syncwarp();
    compact_full_rows(w, cap - 4);
  }
  if (g.stats) {
    const unsigned a = __reduce_add_sync(FULL, n_pref), b = __reduce_add_sync(FULL, n_cmp);
    if (lane == 0) {
      if (a) atomicAdd(g.stats, (unsigned long long)a);
      if (b) atomicAdd(g.stats + 1, (unsigned long long)b);
    }
  }
  __syncwarp();
  // this slice's K best of each row stay in the buffer for the merge
  compact_full_rows(w, g.K);
  gcnt[bufrow + lane] = cnt[lane];
  if (vrow) {
    if (mx_c) atomicMax(g.maxcnt_cand + row, mx_c);
    if (mx_a) atomicMax(g.maxcnt_all + row, mx_a);
  }
}

template <int SMAX>
__global__ void __launch_bounds__(kWarps * 32)
k_allpairs(GraphArgs g, uint64_t *gbuf, int32_t *gcnt, int cap, int P) {
  extern __shared__ __align__(16) unsigned char smem[];
  dense_item(g, gbuf, gcnt, cap, P, blockIdx.x, blockIdx.y, smem);
}

// ── sparse regime on the tensor cores ──────────────────────────────────────
// The abundance prune is a threshold on U·Uᵀ.  A warp multiplies its 32 rows
// (FP16 copies of the unit rank rows, A fragments kept in registers) with
// 8-column tiles of its column slice (FP16, staged in shared memory, B
// fragments by ldmatrix) using mma.sync m16n8k16 with FP32 accumulation.  For
// unit rows, |c16 - c_ref| <= 2^-10·Σ|a_k b_k| + 2^-24·(|a|_1+|b|_1) + K·2^-22
// + |c_ref - a·b| < 1.1e-3 (FP16 rounding of both inputs, accumulation,
// the reference's own FP32 error), so every pair with c16 < eps - kTcDelta is
// pruned exactly as the reference prunes it.  The rest are checked one per
// lane: FP32 chain with its own band, then the AVX-512 order inside the band.
constexpr float kTcDelta = 2.5e-3f;
constexpr int kTCT = 16;          // columns per staged tile
// check-queue ring entries per warp: at least 31 left over + 256 new ones
// (32 rows x 8 columns) of one step; not a power of two, indexed modulo
constexpr int kCQ = 320;
constexpr int kTcWs = 768;        // per-warp workspace: thresholds, counts, maxima, survivors

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void *p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ void ldsm_x2(uint32_t &r0, uint32_t &r1, const void *p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n"
               : "=r"(r0), "=r"(r1)
               : "r"(a));
}

// Exact prune decision for up to 32 queued candidates (lane = candidate),
// survivors appended to the counting queue.  RING: candidates in the check
// ring at head (modulo kCQ); otherwise a plain list from cq + head.
template <int SMAX, bool SYM, bool RING = true>
__device__ __forceinline__ void check_batch(const GraphArgs &g, Warp &w, const SymOut &o,
                                            int64_t grow0, const int *cq, unsigned head, int nq,
                                            int64_t row0, int *q, int &qn, float lo, float hi,
                                            unsigned long long &n_cmp, const float *sU,
                                            int SuP, const unsigned char *sA) {
  const int lane = threadIdx.x & 31;
  const bool act = lane < nq;
  const unsigned e = act ? (unsigned)cq[RING ? (head + lane) % kCQ : head + lane] : 0u;
  const int r = (int)(e >> 27);
  const int64_t j = e & 0x07FFFFFFu;
  const int64_t row = row0 + r;
  bool pass = false;
  if (act && j != row && (__ldg(g.anynz + row) | __ldg(g.anynz + j))) {
    const int Su = g.Su;
    const float4 *ua = (const float4 *)(sU + r * SuP);
    const float4 *ub = (const float4 *)(g.unit + j * Su);
    float ur[SMAX];
    float c1 = 0.f;
#pragma unroll
    for (int t4 = 0; t4 < SMAX; t4 += 4) {
      if (t4 < Su) {
        const float4 x = ua[t4 >> 2], y = __ldg(ub + (t4 >> 2));
        ur[t4] = x.x; ur[t4 + 1] = x.y; ur[t4 + 2] = x.z; ur[t4 + 3] = x.w;
        c1 = __fmaf_rn(x.x, y.x, c1);
        c1 = __fmaf_rn(x.y, y.y, c1);
        c1 = __fmaf_rn(x.z, y.z, c1);
        c1 = __fmaf_rn(x.w, y.w, c1);
      } else {
        ur[t4] = ur[t4 + 1] = ur[t4 + 2] = ur[t4 + 3] = 0.f;
      }
    }
    if (c1 >= hi) pass = true;
    else if (c1 >= lo) pass = !(dot_avx512<SMAX>(ur, g.unit + j * Su, g.S) < g.prefilter_eps);
  }
  const unsigned m = __ballot_sync(FULL, pass);
  if (pass) q[qn + __popc(m & ((1u << lane) - 1u))] = (int)(((unsigned)r << 27) | (unsigned)j);
  qn += __popc(m);
  __syncwarp();
  if (qn >= 32) {
    if constexpr (SYM) count_batch_sym<RING ? 4 : 8>(g, o, w.mxc, row0, grow0, q, 32, sA);
    else count_batch_coop(g, w, q, 32, sA);
    n_cmp += 1;
    if (lane + 32 < qn) q[lane] = q[lane + 32];
    __syncwarp();
    qn -= 32;
  }
}

// SYM: the warp's slice is a slice of columns [row0, n) instead of [0, n), the
// block's own rows only pair with later rows (j > i), and survivors go to the
// pair list (count_batch_sym) instead of the rows' candidate buffers.
template <int KS, int SMAX, bool SYM>
__device__ __forceinline__ void tc_item(const GraphArgs &g, uint64_t *gbuf, int32_t *gcnt,
                                        int cap, int P, float lo, float hi, float lo16,
                                        int64_t bx, int by, unsigned char *smem,
                                        const SymOut &o, int64_t grow0, int64_t cb = 0,
                                        int64_t ce = -1) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int64_t n = g.n;
  const int64_t row0 = (SYM ? 0 : g.row_lo) + bx * 32;
  const int slice = by * kWarps + warp;
  // columns [c_lo, c_hi); rows at or past row_end are never candidates
  const int64_t c_hi = (SYM && ce >= 0) ? ce : n;
  const int64_t row_end = SYM ? c_hi : (g.row_hi < 0 ? n : g.row_hi);
  const int64_t c_lo = SYM ? (row0 > cb ? row0 : cb) : 0;
  const int64_t span = c_hi > c_lo ? c_hi - c_lo : 0;
  const int64_t jb = c_lo + span * slice / P, je = c_lo + span * (slice + 1) / P;
  const int Kp = KS * 16;
  const int cstride = Kp * 2 + 16;                 // bytes per staged column (conflict-free ldmatrix)

  unsigned char *ws = smem + (size_t)warp * kTcWs;
  uint64_t *thr = (uint64_t *)ws;
  int *cnt = (int *)(thr + 32);
  uint32_t *mxc = (uint32_t *)(cnt + 32);
  int *q = (int *)(mxc + 32);                      // [64] survivors to count
  int *cq = (int *)(smem + (size_t)kWarps * kTcWs) + (size_t)warp * kCQ;     // check ring
  unsigned char *rings = smem + (size_t)kWarps * kTcWs + (size_t)kWarps * kCQ * 4;
  unsigned char *ring = rings + (size_t)warp * 2 * kTCT * cstride;
  // the block's 32 rows: register codes [32][mpad] and unit rows [32][Su]
  unsigned char *sA = rings + (size_t)kWarps * 2 * kTCT * cstride;
  float *sU = (float *)(sA + (size_t)32 * g.mpad);
  const int SuP = su_stride(g.Su);
  {
    const int m16 = g.mpad >> 4, s4 = g.Su >> 2;
    for (int i = threadIdx.x; i < 32 * m16; i += blockDim.x) {
      const int r = i / m16, t = i - r * m16;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (row0 + r < n) v = __ldg((const uint4 *)(g.codesA + (row0 + r) * g.mpad) + t);
      *((uint4 *)(sA + (size_t)r * g.mpad) + t) = v;
    }
    for (int i = threadIdx.x; i < 32 * s4; i += blockDim.x) {
      const int r = i / s4, t = i - r * s4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (row0 + r < n) v = __ldg((const float4 *)(g.unit + (row0 + r) * g.Su) + t);
      *((float4 *)(sU + (size_t)r * SuP) + t) = v;
    }
    __syncthreads();
  }
  thr[lane] = g.key_floor;
  cnt[lane] = 0;
  mxc[lane] = 0;
  const size_t bufrow = ((size_t)bx * P + slice) * 32;
  Warp w{SYM ? gbuf : gbuf + bufrow * cap, cnt, thr, mxc, cap, g.K};
  unsigned long long n_pref = 0, n_cmp = 0;

  // A fragments: rows mt*16 + gq (+8), k = ks*16 + 2*tq (+8)
  uint32_t af[2][KS][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int64_t ra = row0 + mt * 16 + gq, rb = ra + 8;
    const uint32_t *pa = (const uint32_t *)(g.unit16 + (ra < n ? ra : 0) * Kp);
    const uint32_t *pb = (const uint32_t *)(g.unit16 + (rb < n ? rb : 0) * Kp);
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      af[mt][ks][0] = ra < n ? __ldg(pa + ks * 8 + tq) : 0u;
      af[mt][ks][1] = rb < n ? __ldg(pb + ks * 8 + tq) : 0u;
      af[mt][ks][2] = ra < n ? __ldg(pa + ks * 8 + 4 + tq) : 0u;
      af[mt][ks][3] = rb < n ? __ldg(pb + ks * 8 + 4 + tq) : 0u;
    }
  }
  auto stage_cols = [&](int st, int64_t jt) {
    const int nc = (int)(je - jt < kTCT ? je - jt : kTCT);
    unsigned char *dst = ring + (size_t)st * kTCT * cstride;
    const int per = Kp / 8;                        // 16-byte chunks per column
    for (int i = lane; i < nc * per; i += 32) {
      const int c = i / per, t = i - c * per;
      cp16(dst + c * cstride + 16 * t, g.unit16 + (jt + c) * Kp + 8 * t);
    }
    cp_commit();
  };
  unsigned head = 0, tail = 0;                     // check ring
  int qn = 0;
  if (jb < je) stage_cols(0, jb);
  int st = 0;
  for (int64_t jt = jb; jt < je; jt += kTCT, st ^= 1) {
    if (jt + kTCT < je) stage_cols(st ^ 1, jt + kTCT); else cp_commit();
    const int nc = (int)(je - jt < kTCT ? je - jt : kTCT);
    cp_wait1();
    __syncwarp();
    const unsigned char *tile = ring + (size_t)st * kTCT * cstride;
    const bool interior = nc == kTCT && row0 + 32 <= row_end && (!SYM || jt >= row0 + 32);
    for (int c0 = 0; c0 < nc; c0 += 8) {
      float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
      // B fragments: ldmatrix rows = columns c0 + (lane & 7), k block by lane >> 3
      const unsigned char *bp = tile + (c0 + (lane & 7)) * cstride;
      if (KS == 1) {
        uint32_t b0, b1;
        ldsm_x2(b0, b1, bp + 16 * ((lane >> 3) & 1));
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) mma16816(acc[mt], af[mt][0], b0, b1);
      } else {
#pragma unroll
        for (int kp = 0; kp < KS; kp += 2) {
          uint32_t b[4];
          ldsm_x4(b, bp + 16 * (2 * kp + (lane >> 3)));
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            mma16816(acc[mt], af[mt][kp], b[0], b[1]);
            mma16816(acc[mt], af[mt][kp + 1], b[2], b[3]);
          }
        }
      }
      // candidates: value i of m-tile mt -> row mt*16 + gq + 8*(i>>1), column c0 + 2*tq + (i&1).
      // Away from the staged tile's end, the valid rows' end and the diagonal
      // (a warp-uniform test), the threshold alone decides.
      unsigned mk = 0;
      if (interior) {
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int i = 0; i < 4; ++i) mk |= (acc[mt][i] >= lo16 ? 1u : 0u) << (mt * 4 + i);
      } else {
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int rr = mt * 16 + gq + 8 * (i >> 1);
            const int cc = c0 + 2 * tq + (i & 1);
            if (acc[mt][i] >= lo16 && cc < nc && row0 + rr < row_end && (!SYM || jt + cc > row0 + rr))
              mk |= 1u << (mt * 4 + i);
          }
      }
      n_pref += 8;
      if (__any_sync(FULL, mk != 0)) {
        // each lane's slot: the candidates of the lanes below it, summed from
        // the bit planes of the per-lane counts (0..8: four votes) rather than
        // by a chain of dependent shuffles
        const unsigned cntl = (unsigned)__popc(mk), below = (1u << lane) - 1u;
        const unsigned v0 = __ballot_sync(FULL, cntl & 1u), v1 = __ballot_sync(FULL, cntl & 2u);
        const unsigned v2 = __ballot_sync(FULL, cntl & 4u), v3 = __ballot_sync(FULL, cntl & 8u);
        const int excl = __popc(v0 & below) + 2 * __popc(v1 & below) + 4 * __popc(v2 & below) +
                         8 * __popc(v3 & below);
        const int total = __popc(v0) + 2 * __popc(v1) + 4 * __popc(v2) + 8 * __popc(v3);
        unsigned pos = tail + (unsigned)excl;
        while (mk) {
          const int b = __ffs(mk) - 1;
          mk &= mk - 1;
          const int mt = b >> 2, i = b & 3;
          const int rr = mt * 16 + gq + 8 * (i >> 1);
          const int64_t jj = jt + c0 + 2 * tq + (i & 1);
          cq[pos % kCQ] = (int)(((unsigned)rr << 27) | (unsigned)jj);
          ++pos;
        }
        tail += (unsigned)total;
        __syncwarp();
        while (tail - head >= 32) {
          check_batch<SMAX, SYM>(g, w, o, grow0, cq, head, 32, row0, q, qn, lo, hi, n_cmp, sU, SuP, sA);
          head += 32;
        }
      }
    }
    __syncwarp();
  }
  while (tail != head) {
    const int nq = (int)(tail - head < 32 ? tail - head : 32);
    check_batch<SMAX, SYM>(g, w, o, grow0, cq, head, nq, row0, q, qn, lo, hi, n_cmp, sU, SuP, sA);
    head += (unsigned)nq;
  }
  if (qn > 0) {
    n_cmp += lane < qn;
    if constexpr (SYM) count_batch_sym(g, o, mxc, row0, grow0, q, qn, sA);
    else count_batch_coop(g, w, q, qn, sA);
  }
  if (g.stats) {
    // pairs evaluated: ordered pairs, or unordered ones in the symmetric pass
    const unsigned a = __reduce_add_sync(FULL, (unsigned)n_pref),
                   b = __reduce_add_sync(FULL, (unsigned)n_cmp);
    if (lane == 0) {
      if (a) atomicAdd(g.stats, (unsigned long long)a);
      if (b) atomicAdd(g.stats + 1, (unsigned long long)b);
    }
  }
  __syncwarp();
  if constexpr (!SYM) {
    compact_full_rows(w, g.K);
    gcnt[bufrow + lane] = cnt[lane];
  }
  const int64_t row = row0 + lane;
  if (row < n && mxc[lane]) atomicMax(g.maxcnt_cand + row, mxc[lane]);
}

template <int KS, int SMAX>
__global__ void __launch_bounds__(kWarps * 32)
k_allpairs_tc(GraphArgs g, uint64_t *gbuf, int32_t *gcnt, int cap, int P, float lo, float hi,
              float lo16) {
  extern __shared__ __align__(16) unsigned char smem[];
  tc_item<KS, SMAX, false>(g, gbuf, gcnt, cap, P, lo, hi, lo16, blockIdx.x, blockIdx.y, smem,
                           SymOut{}, 0);
}

// Symmetric pass: CTA x scores row block x and row block B-1-x (columns from
// the block's first row on), so every CTA's column work is about n + 32.
// With x0, xs: CTA x0 + blockIdx.x * xs of that layout (the share of one rank
// of a sharded assembly).
template <int KS, int SMAX>
__global__ void __launch_bounds__(kWarps * 32, KS == 2 ? 6 : 1)
k_allpairs_tc_sym(GraphArgs g, int P, float lo, float hi, float lo16, SymOut o, int x0, int xs) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int64_t B = (g.n + 31) / 32;
  const int64_t x = x0 + (int64_t)blockIdx.x * xs;
  const int64_t b1 = x, b2 = B - 1 - x;
  tc_item<KS, SMAX, true>(g, nullptr, nullptr, 0, P, lo, hi, lo16, b1, blockIdx.y, smem, o, 0);
  if (b2 > b1) {
    __syncthreads();
    tc_item<KS, SMAX, true>(g, nullptr, nullptr, 0, P, lo, hi, lo16, b2, blockIdx.y, smem, o, 0);
  }
}

// Window of the symmetric pass: CTA x scores row block x against the columns
// [max(cb, its first row), ce).
template <int KS, int SMAX>
__global__ void __launch_bounds__(kWarps * 32)
k_allpairs_tc_win(GraphArgs g, int P, float lo, float hi, float lo16, SymOut o, int64_t cb,
                  int64_t ce) {
  extern __shared__ __align__(16) unsigned char smem[];
  tc_item<KS, SMAX, true>(g, nullptr, nullptr, 0, P, lo, hi, lo16, blockIdx.x, blockIdx.y, smem, o,
                          0, cb, ce);
}

// Symmetric pass, part 2 (after k_sym_prefilter, kernels_sym_tc5.cu): a CTA
// takes 32-row block x and block B-1-x of the B blocks in play (as
// k_allpairs_tc_sym pairs them; gridDim.y CTAs share a pair's lists), with
// the block's register codes and unit rows in shared memory, and its warps work
// through the block's candidate list 32 entries at a time: the exact prune
// decision (check_batch), then the survivors' register compares and pair
// records (count_batch_sym), exactly as in the single-kernel pass.
template <int SMAX>
__device__ __forceinline__ void sym_check_block(const GraphArgs &g, const SymOut &o, float lo,
                                                float hi, const uint32_t *cand,
                                                const int64_t *coff, const int32_t *ccnt,
                                                int64_t bx, unsigned char *smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t n = g.n, row0 = bx * 32;
  unsigned char *ws = smem + (size_t)warp * kTcWs;
  uint64_t *thr = (uint64_t *)ws;
  int *cntw = (int *)(thr + 32);
  uint32_t *mxc = (uint32_t *)(cntw + 32);
  int *q = (int *)(mxc + 32);                      // [64] survivors to count
  unsigned char *sA = smem + (size_t)kWarps * kTcWs;
  float *sU = (float *)(sA + (size_t)32 * g.mpad);
  const int SuP = su_stride(g.Su);
  {
    const int m16 = g.mpad >> 4, s4 = g.Su >> 2;
    for (int i = threadIdx.x; i < 32 * m16; i += blockDim.x) {
      const int r = i / m16, t = i - r * m16;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (row0 + r < n) v = __ldg((const uint4 *)(g.codesA + (row0 + r) * g.mpad) + t);
      *((uint4 *)(sA + (size_t)r * g.mpad) + t) = v;
    }
    for (int i = threadIdx.x; i < 32 * s4; i += blockDim.x) {
      const int r = i / s4, t = i - r * s4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (row0 + r < n) v = __ldg((const float4 *)(g.unit + (row0 + r) * g.Su) + t);
      *((float4 *)(sU + (size_t)r * SuP) + t) = v;
    }
  }
  mxc[lane] = 0;
  __syncthreads();
  Warp w{nullptr, cntw, thr, mxc, 0, g.K};
  unsigned long long n_cmp = 0;
  int qn = 0;
  const int64_t off = coff[bx];
  const int cnt = (int)min((int64_t)ccnt[bx], coff[bx + 1] - off);
  const int *list = (const int *)(cand + off);
  // the gridDim.y CTAs of a block pair share its list
  for (int i0 = ((int)blockIdx.y * kWarps + warp) * 32; i0 < cnt;
       i0 += (int)gridDim.y * kWarps * 32)
    check_batch<SMAX, true, false>(g, w, o, 0, list, (unsigned)i0, min(32, cnt - i0), row0, q,
                                   qn, lo, hi, n_cmp, sU, SuP, sA);
  if (qn > 0) {
    n_cmp += lane < qn;
    count_batch_sym<8>(g, o, mxc, row0, 0, q, qn, sA);
  }
  if (g.stats) {
    const unsigned b = __reduce_add_sync(FULL, (unsigned)n_cmp);
    if (lane == 0 && b) atomicAdd(g.stats + 1, (unsigned long long)b);
  }
  __syncwarp();
  const int64_t row = row0 + lane;
  if (row < n && mxc[lane]) atomicMax(g.maxcnt_cand + row, mxc[lane]);
}

template <int SMAX>
__global__ void __launch_bounds__(kWarps * 32, SMAX == 32 ? 6 : 1)
k_sym_check(GraphArgs g, float lo, float hi, SymOut o, const uint32_t *cand,
            const int64_t *coff, const int32_t *ccnt, int64_t B) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int64_t b1 = blockIdx.x, b2 = B - 1 - b1;
  sym_check_block<SMAX>(g, o, lo, hi, cand, coff, ccnt, b1, smem);
  if (b2 > b1) {
    __syncthreads();
    sym_check_block<SMAX>(g, o, lo, hi, cand, coff, ccnt, b2, smem);
  }
}

// Persistent form over a batch: CTAs pull (assembly, row block, slice group)
// items from a device counter until the variant's items are exhausted.  The
// tensor-core variants run the symmetric pass (a row block's slices cover the
// columns from its first row on; items come in ascending row blocks, so the
// largest first).
template <int KS, int SMAX>
__global__ void __launch_bounds__(kWarps * 32)
k_allpairs_batch(const BatchAsm *B, const int32_t *list, const int64_t *item0s, int nv,
                 int64_t items, unsigned long long *next, SymOut o) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long s_item;
  for (;;) {
    __syncthreads();                     // the previous item is done with shared memory
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(next, 1ull);
    __syncthreads();
    const int64_t it = s_item;
    if (it >= items) return;
    int lo = 0, hi = nv - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(item0s + mid) <= it) lo = mid; else hi = mid - 1;
    }
    const BatchAsm &b = B[list[lo]];
    const GraphArgs g = b.g;
    const int G = b.P / kWarps;
    const int64_t local = it - item0s[lo];
    const int64_t bx = local / G;
    const int by = (int)(local - bx * G);
    if constexpr (KS == 0) dense_item(g, b.gbuf, b.gcnt, b.cap, b.P, bx, by, smem);
    else tc_item<KS, SMAX, true>(g, nullptr, nullptr, 0, b.P, b.lo, b.hi, b.lo16, bx, by, smem, o,
                                 b.row0);
  }
}

// Warp per row: the K best keys among the P slices' partial lists.  The lists
// stream through a 512-key shared buffer per warp; whenever it fills, the
// register radix select keeps its K best (K <= 448 leaves room to refill).
constexpr int kMergeWarps = 8;
constexpr int kMergeBuf = 32 * kCapW;       // 512 keys per warp

__device__ __forceinline__ void merge_row(const GraphArgs &g, const uint64_t *gbuf,
                                          const int32_t *gcnt, int cap, int P, int64_t row,
                                          uint64_t *keys) {
  const int lane = threadIdx.x & 31;
  const int K = g.K;
  const int64_t rb = (row - g.row_lo) >> 5, rl = (row - g.row_lo) & 31;
  const size_t br0 = (size_t)rb * P * 32 + rl;          // slice s: br0 + 32 s
  const int cl = lane < P ? gcnt[br0 + (size_t)lane * 32] : 0;   // P <= 32
  int fill = 0;
  for (int s = 0; s < P; ++s) {
    const int c = __shfl_sync(FULL, cl, s);
    const uint64_t *src = gbuf + (br0 + (size_t)s * 32) * cap;
    for (int i0 = 0; i0 < c;) {
      const int take = min(c - i0, kMergeBuf - fill);
      for (int i = lane; i < take; i += 32) keys[fill + i] = src[i0 + i];
      fill += take;
      i0 += take;
      __syncwarp();
      if (fill == kMergeBuf) {
        select_topk(keys, fill, K);
        fill = K;
      }
    }
  }
  if (fill > K) {
    select_topk(keys, fill, K);
    fill = K;
  }
  for (int i = lane; i < fill; i += 32) g.topk[row * K + i] = keys[i];
  if (lane == 0) g.topk_cnt[row] = fill;
}

__global__ void __launch_bounds__(kMergeWarps * 32)
k_merge_topk(GraphArgs g, const uint64_t *gbuf, const int32_t *gcnt, int cap, int P) {
  __shared__ uint64_t mk[kMergeWarps][kMergeBuf];
  const int wib = threadIdx.x >> 5;
  const int64_t row = g.row_lo + (int64_t)blockIdx.x * kMergeWarps + wib;
  if (row < (g.row_hi < 0 ? g.n : g.row_hi)) merge_row(g, gbuf, gcnt, cap, P, row, mk[wib]);
}

__global__ void __launch_bounds__(kMergeWarps * 32)
k_merge_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t r_begin, int64_t rows) {
  __shared__ uint64_t mk[kMergeWarps][kMergeBuf];
  const int wib = threadIdx.x >> 5;
  const int64_t r = r_begin + (int64_t)blockIdx.x * kMergeWarps + wib;
  if (r >= rows) return;
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(row0s + mid) <= r) lo = mid; else hi = mid - 1;
  }
  const BatchAsm &b = B[lo];
  if (b.variant != 0) return;          // top-K from the symmetric pass's pairs
  merge_row(b.g, b.gbuf, b.gcnt, b.cap, b.P, r - b.row0, mk[wib]);
}

// Admitted keys per row of a pair list gathered from several ranks (both ends).
__global__ void k_pair_rowcounts(const uint4 *__restrict__ pairs, unsigned long long np,
                                 int32_t *__restrict__ rowcnt) {
  for (unsigned long long p = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (unsigned long long)gridDim.x * blockDim.x) {
    const uint4 x = pairs[p];
    atomicAdd(rowcnt + x.x, 1);
    atomicAdd(rowcnt + x.y, 1);
  }
}

// out[i] = the largest of the W ranks' partial maxima (blocks of `stride`).
__global__ void k_max_blocks(const uint32_t *__restrict__ blocks, int W, int64_t stride,
                             int64_t n, uint32_t *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t v = 0;
    for (int r = 0; r < W; ++r) v = max(v, blocks[(int64_t)r * stride + i]);
    out[i] = v;
  }
}

// Row offsets of the admitted keys: exclusive scan of the per-row counts, one CTA.
__global__ void k_rows_scan(const int32_t *cnt, int64_t *off, int64_t n) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t per = (n + 1023) / 1024;
  const int64_t a = t * per, b = (a + per < n) ? a + per : n;
  int64_t s = 0;
  for (int64_t q = a; q < b; ++q) s += cnt[q];
  part[t] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int64_t add = (t >= d) ? part[t - d] : 0;
    __syncthreads();
    part[t] += add;
    __syncthreads();
  }
  int64_t run = (t > 0) ? part[t - 1] : 0;
  for (int64_t q = a; q < b; ++q) { off[q] = run; run += cnt[q]; }
  if (t == 1023) off[n] = part[1023];
}

// Both keys of every admitted pair into their rows' segments (grid-stride over
// the pairs written).  Positions count down from each row's end, so the row
// counts return to zero.
__global__ void k_scatter_pairs(SymOut o, const int64_t *off, uint64_t *keys,
                                const uint32_t *svtab) {
  const unsigned long long np = *o.npairs < o.cap ? *o.npairs : o.cap;
  for (unsigned long long p = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (unsigned long long)gridDim.x * blockDim.x) {
    const uint4 x = o.pairs[p];                 // ids in keys are the assembly's own
    const uint64_t hi = (uint64_t)(svtab ? __ldg(svtab + x.z) : x.z) << 32;
    const int64_t pi = off[x.x] + atomicSub(o.rowcnt + x.x, 1) - 1;
    keys[pi] = hi | (uint64_t)(~(x.y - x.w));
    const int64_t pj = off[x.y] + atomicSub(o.rowcnt + x.y, 1) - 1;
    keys[pj] = hi | (uint64_t)(~(x.x - x.w));
  }
}

// Warp per row: the K best keys of the row's segment (row space index gr,
// assembly row `row`), streamed through a 512-key shared buffer (the register
// radix select keeps the K best whenever it fills).
__device__ __forceinline__ void select_row(const GraphArgs &g, int64_t row, int64_t gr,
                                           const int64_t *off, const uint64_t *keys,
                                           uint64_t *buf) {
  const int lane = threadIdx.x & 31;
  const int K = g.K;
  const int64_t s0 = off[gr];
  const int64_t c = off[gr + 1] - s0;
  const uint64_t *src = keys + s0;
  if (c <= K) {
    for (int64_t i = lane; i < c; i += 32) g.topk[row * K + i] = src[i];
    if (lane == 0) g.topk_cnt[row] = (int32_t)c;
    return;
  }
  int fill = 0;
  for (int64_t i0 = 0; i0 < c;) {
    const int take = (int)(c - i0 < (int64_t)(kMergeBuf - fill) ? c - i0 : (int64_t)(kMergeBuf - fill));
    for (int i = lane; i < take; i += 32) buf[fill + i] = src[i0 + i];
    fill += take;
    i0 += take;
    __syncwarp();
    if (fill == kMergeBuf) {
      select_topk(buf, fill, K);
      fill = K;
    }
  }
  if (fill > K) {
    select_topk(buf, fill, K);
    fill = K;
  }
  for (int i = lane; i < fill; i += 32) g.topk[row * K + i] = buf[i];
  if (lane == 0) g.topk_cnt[row] = fill;
}

__global__ void __launch_bounds__(kMergeWarps * 32)
k_select_rows(GraphArgs g, const int64_t *off, const uint64_t *keys) {
  __shared__ uint64_t mk[kMergeWarps][kMergeBuf];
  const int wib = threadIdx.x >> 5;
  const int64_t row = (int64_t)blockIdx.x * kMergeWarps + wib;
  if (row < g.n) select_row(g, row, row, off, keys, mk[wib]);
}

__global__ void __launch_bounds__(kMergeWarps * 32)
k_select_rows_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                    const int64_t *off, const uint64_t *keys) {
  __shared__ uint64_t mk[kMergeWarps][kMergeBuf];
  const int wib = threadIdx.x >> 5;
  const int64_t r = (int64_t)blockIdx.x * kMergeWarps + wib;
  if (r >= rows) return;
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(row0s + mid) <= r) lo = mid; else hi = mid - 1;
  }
  const BatchAsm &b = B[lo];
  if (b.variant <= 0) return;          // dense: candidate buffers or the one-hot GEMM
  select_row(b.g, r - b.row0, r, off, keys, mk[wib]);
}

size_t dense_smem(int mpad) {
  const int mw = mpad >> 2;
  const int mwq = ((mw + 27) & ~31) + 4;
  return (size_t)kWarps * 1024 + 32 * (size_t)mwq * 4 + (size_t)kWarps * 2 * 4 * mpad;
}

size_t tc_smem(int KS, int mpad, int Su) {
  return (size_t)kWarps * kTcWs + (size_t)kWarps * kCQ * 4 +
         (size_t)kWarps * 2 * kTCT * (KS * 16 * 2 + 16) + (size_t)32 * mpad +
         (size_t)32 * su_stride(Su) * 4;
}

}  // namespace

int allpairs_cap(int K) { return (K + 64 + 31) & ~31; }

// Column slices per 32-row block: enough warps for several waves of the GPU,
// each slice at least 64 columns; a multiple of the CTA's warp count.
int allpairs_slices(int64_t n, int K) { return allpairs_slices_rows(n, n, K); }

int allpairs_slices_rows(int64_t rows, int64_t n, int K) {
  const int64_t blocks = (rows + 31) / 32;
  int64_t P = (4 * 148 * 48 + blocks - 1) / std::max<int64_t>(blocks, 1);
  P = std::min<int64_t>(P, std::max<int64_t>(n / 64, 1));
  P = std::max<int64_t>(P, 1);
  const int pmax = std::max(kWarps, std::min(32, (6400 / std::max(K, 1)) / kWarps * kWarps));
  P = std::min<int64_t>(P, pmax);
  return (int)(((P + kWarps - 1) / kWarps) * kWarps);
}

int64_t allpairs_items(int64_t n, int P) { return ((n + 31) / 32) * (P / kWarps); }

size_t allpairs_batch_smem(int variant, int mpad, int Su) {
  return variant == 0 ? dense_smem(mpad) : tc_smem(variant, mpad, Su);
}

void prefilter_bands(int S, float eps, float *lo, float *hi, float *lo16) {
  // band of the exact-safe prefilter: |chain - AVX-512 order| < delta
  const double e = (double)eps;
  const double delta = (double)(S + (S + 15) / 16 + 8) * ldexp(1.0, -23);
  float l = (float)(e - delta), h = (float)(e + delta);
  if ((double)l > e - delta) l = nextafterf(l, -INFINITY);
  if ((double)h < e + delta) h = nextafterf(h, INFINITY);
  *lo = l;
  *hi = h;
  *lo16 = (float)(e - (double)kTcDelta);
}

int allpairs_variant(const GraphArgs &g) {
  if (!g.prefilter) return 0;
  return g.Kp == 16 ? 1 : (g.Kp == 32 ? 2 : 4);   // the FP16 rows are KS * 16 halves wide
}

void launch_allpairs(const GraphArgs &g, uint64_t *gbuf, int32_t *gcnt, cudaStream_t s) {
  const int64_t rows = (g.row_hi < 0 ? g.n : g.row_hi) - g.row_lo;
  if (g.n == 0 || rows <= 0) return;
  const int cap = allpairs_cap(g.K);
  const int P = allpairs_slices_rows(rows, g.n, g.K);
  const dim3 grid((unsigned)((rows + 31) / 32), (unsigned)(P / kWarps));
  float lo, hi, lo16;
  prefilter_bands(g.S, g.prefilter_eps, &lo, &hi, &lo16);
  const int v = allpairs_variant(g);
  const size_t smem = allpairs_batch_smem(v, g.mpad, g.Su);
#define RBG_TC(KS, SM)                                                                        \
  do {                                                                                        \
    smem_cap_max((const void *)k_allpairs_tc<KS, SM>);                                        \
    k_allpairs_tc<KS, SM><<<grid, kWarps * 32, smem, s>>>(g, gbuf, gcnt, cap, P, lo, hi, lo16); \
  } while (0)
  if (v == 1) RBG_TC(1, 16);
  else if (v == 2) RBG_TC(2, 32);
  else if (v == 4) RBG_TC(4, 64);
  else {
    smem_cap_max((const void *)k_allpairs<4>);
    k_allpairs<4><<<grid, kWarps * 32, smem, s>>>(g, gbuf, gcnt, cap, P);
  }
#undef RBG_TC
  k_merge_topk<<<(unsigned)((rows + kMergeWarps - 1) / kMergeWarps), kMergeWarps * 32, 0, s>>>(
      g, gbuf, gcnt, cap, P);
}

void launch_pair_rowcounts(const uint4 *pairs, unsigned long long np, int32_t *rowcnt,
                           cudaStream_t s) {
  if (np == 0) return;
  k_pair_rowcounts<<<(unsigned)std::min<unsigned long long>((np + 255) / 256, 148 * 8), 256, 0,
                     s>>>(pairs, np, rowcnt);
}

void launch_max_blocks(const uint32_t *blocks, int W, int64_t stride, int64_t n, uint32_t *out,
                       cudaStream_t s) {
  if (n == 0) return;
  k_max_blocks<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(
      blocks, W, stride, n, out);
}

void launch_merge_topk(const GraphArgs &g, const uint64_t *gbuf, const int32_t *gcnt, int cap,
                       int P, cudaStream_t s) {
  const int64_t rows = (g.row_hi < 0 ? g.n : g.row_hi) - g.row_lo;
  if (rows <= 0) return;
  k_merge_topk<<<(unsigned)((rows + kMergeWarps - 1) / kMergeWarps), kMergeWarps * 32, 0, s>>>(
      g, gbuf, gcnt, cap, P);
}

void launch_sym_check(const GraphArgs &g, const SymOut &o, const uint32_t *cand,
                      const int64_t *coff, const int32_t *ccnt, int64_t B, cudaStream_t s) {
  if (g.n == 0 || B <= 0) return;
  float lo, hi, lo16;
  prefilter_bands(g.S, g.prefilter_eps, &lo, &hi, &lo16);
  const int v = allpairs_variant(g);
  const size_t smem = (size_t)kWarps * kTcWs + (size_t)32 * g.mpad +
                      (size_t)32 * su_stride(g.Su) * 4;
  // enough CTAs for six per SM: a block pair's list is split over gridDim.y CTAs
  const int64_t pairs = (B + 1) / 2;
  const unsigned gy =
      (unsigned)std::min<int64_t>(4, std::max<int64_t>(1, (6 * 148 + pairs - 1) / pairs));
  const dim3 grid((unsigned)pairs, gy);
#define RBG_SC(SM)                                                                        \
  do {                                                                                    \
    smem_cap_max((const void *)k_sym_check<SM>);                                          \
    k_sym_check<SM><<<grid, kWarps * 32, smem, s>>>(g, lo, hi, o, cand, coff, ccnt, B);   \
  } while (0)
  if (v == 1) RBG_SC(16);
  else if (v == 2) RBG_SC(32);
  else RBG_SC(64);
#undef RBG_SC
}

float prefilter_lo16(int S, float eps) {
  float lo, hi, lo16;
  prefilter_bands(S, eps, &lo, &hi, &lo16);
  return lo16;
}

void launch_allpairs_sym(const GraphArgs &g, const SymOut &o, cudaStream_t s, int x0, int xs) {
  if (g.n == 0) return;
  const int P = allpairs_slices(g.n, g.K);
  const int64_t B = (g.n + 31) / 32;
  const int64_t nx = (B + 1) / 2;                 // CTAs of the whole pass
  if (x0 >= nx) return;
  const dim3 grid((unsigned)((nx - x0 + xs - 1) / xs), (unsigned)(P / kWarps));
  float lo, hi, lo16;
  prefilter_bands(g.S, g.prefilter_eps, &lo, &hi, &lo16);
  const int v = allpairs_variant(g);
  const size_t smem = tc_smem(v, g.mpad, g.Su);
#define RBG_TS(KS, SM)                                                                        \
  do {                                                                                        \
    smem_cap_max((const void *)k_allpairs_tc_sym<KS, SM>);                                    \
    k_allpairs_tc_sym<KS, SM><<<grid, kWarps * 32, smem, s>>>(g, P, lo, hi, lo16, o, x0, xs); \
  } while (0)
  if (v == 1) RBG_TS(1, 16);
  else if (v == 2) RBG_TS(2, 32);
  else RBG_TS(4, 64);
#undef RBG_TS
}

void launch_allpairs_sym_window(const GraphArgs &g, const SymOut &o, int64_t cb, int64_t ce,
                                cudaStream_t s) {
  if (g.n == 0 || ce <= cb) return;
  // slices of about 1024 columns: a window is a fraction of the columns, and
  // every CTA stages its row block once
  const int Pfull = allpairs_slices(g.n, g.K);
  const int64_t want = (ce - cb) / 1024 / kWarps * kWarps;
  const int P = (int)std::max<int64_t>(kWarps, std::min<int64_t>(Pfull, want));
  const dim3 grid((unsigned)((ce + 31) / 32), (unsigned)(P / kWarps));
  float lo, hi, lo16;
  prefilter_bands(g.S, g.prefilter_eps, &lo, &hi, &lo16);
  const int v = allpairs_variant(g);
  const size_t smem = tc_smem(v, g.mpad, g.Su);
#define RBG_TW(KS, SM)                                                                        \
  do {                                                                                        \
    smem_cap_max((const void *)k_allpairs_tc_win<KS, SM>);                                    \
    k_allpairs_tc_win<KS, SM><<<grid, kWarps * 32, smem, s>>>(g, P, lo, hi, lo16, o, cb, ce); \
  } while (0)
  if (v == 1) RBG_TW(1, 16);
  else if (v == 2) RBG_TW(2, 32);
  else RBG_TW(4, 64);
#undef RBG_TW
}

void launch_rows_topk_counts(const GraphArgs &g, const SymOut &o, const uint32_t *svtab,
                             int64_t *rowoff, uint64_t *keys, cudaStream_t s) {
  if (g.n == 0) return;
  k_rows_scan<<<1, 1024, 0, s>>>(o.rowcnt, rowoff, g.n);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_scatter_pairs<<<(unsigned)(sms * 32), 256, 0, s>>>(o, rowoff, keys, svtab);
  k_select_rows<<<(unsigned)((g.n + kMergeWarps - 1) / kMergeWarps), kMergeWarps * 32, 0, s>>>(
      g, rowoff, keys);
}

void launch_rows_topk(const GraphArgs &g, const SymOut &o, int64_t *rowoff, uint64_t *keys,
                      cudaStream_t s) {
  if (g.n == 0) return;
  k_rows_scan<<<1, 1024, 0, s>>>(o.rowcnt, rowoff, g.n);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_scatter_pairs<<<(unsigned)(sms * 32), 256, 0, s>>>(o, rowoff, keys, nullptr);   // a few pairs per thread
  k_select_rows<<<(unsigned)((g.n + kMergeWarps - 1) / kMergeWarps), kMergeWarps * 32, 0, s>>>(
      g, rowoff, keys);
}

void launch_rows_topk_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                            const SymOut &o, int64_t *rowoff, uint64_t *keys, cudaStream_t s) {
  if (rows == 0) return;
  k_rows_scan<<<1, 1024, 0, s>>>(o.rowcnt, rowoff, rows);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_scatter_pairs<<<(unsigned)(sms * 32), 256, 0, s>>>(o, rowoff, keys, nullptr);
  k_select_rows_batch<<<(unsigned)((rows + kMergeWarps - 1) / kMergeWarps), kMergeWarps * 32, 0,
                        s>>>(B, row0s, nb, rows, rowoff, keys);
}

void launch_allpairs_batch(const BatchAsm *B, int variant, const int32_t *list,
                           const int64_t *item0s, int nv, int64_t items, size_t smem,
                           unsigned long long *next, const SymOut &o, cudaStream_t s) {
  if (items == 0 || nv == 0) return;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
#define RBG_PB(KS, SM)                                                                         \
  do {                                                                                         \
    smem_cap_max((const void *)k_allpairs_batch<KS, SM>);                                      \
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_allpairs_batch<KS, SM>,           \
                                                  kWarps * 32, smem);                          \
    const int64_t grid = std::min<int64_t>(items, (int64_t)std::max(per_sm, 1) * sms);         \
    k_allpairs_batch<KS, SM><<<(unsigned)grid, kWarps * 32, smem, s>>>(B, list, item0s, nv,    \
                                                                       items, next, o);        \
  } while (0)
  if (variant == 1) RBG_PB(1, 16);
  else if (variant == 2) RBG_PB(2, 32);
  else if (variant == 4) RBG_PB(4, 64);
  else RBG_PB(0, 4);
#undef RBG_PB
}

void launch_merge_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                        cudaStream_t s, int64_t r_begin) {
  if (rows <= r_begin) return;
  k_merge_batch<<<(unsigned)((rows - r_begin + kMergeWarps - 1) / kMergeWarps), kMergeWarps * 32,
                  0, s>>>(B, row0s, nb, r_begin, rows);
}

}  // namespace rbg
