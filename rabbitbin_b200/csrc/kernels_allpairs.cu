// All-pairs pass: per row top-K of (similarity, id) keys plus the row maxima
// the calibration reads, over full rows (every ordered pair i != j).
//
// Layout: lane = row, a warp owns 32 rows and streams every column j in
// order; column data (unit rank rows, 8-bit register codes) are read with
// warp-uniform 128-bit loads that the SM's L1 serves to all warps walking the
// same columns.  Nothing is shared across warps, so there is no CTA barrier.
// Each row keeps its candidate keys in a private global buffer (L2-resident)
// with the admission threshold and fill count in shared memory; when a buffer
// fills, the owning warp selects the K best in registers (radix search of the
// K-th largest key) and raises the threshold to it.
//
// Two regimes:
//  * dense (no abundance prune: the N <= 25000 path, S <= 2, RABBIT_NO_ABDFIRST):
//    every pair's register-match count, 4 columns per step over 8-bit code
//    words (row words from shared memory, column words uniform loads);
//  * sparse (the abundance-first prune of the fused path): a single FP32 FMA
//    chain decides the prune for almost every pair under a rigorous error bound
//    against the AVX-512 order of unit_dot_f; pairs inside the bound's band
//    evaluate that order exactly.  Survivors queue per warp and are counted 32
//    at a time, lane = survivor.
//
// Compiled with -fmad=false; __fmaf_rn marks every fused operation.
#include <cstdint>

#include "rbg_internal.h"

namespace rbg {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kWarps = 4;         // warps per CTA (independent)
constexpr int kCapW = 16;         // candidate buffer <= 32 * kCapW keys per row
constexpr int kQ = 64;            // survivor queue entries per warp

__device__ __forceinline__ uint32_t eq_bytes(uint32_t a, uint32_t b) {
  const uint32_t x = a ^ b;
  const uint32_t t = ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x;
  return (~t & 0x80808080u) >> 7;      // 0x01 in each equal byte
}
__device__ __forceinline__ uint32_t byte_sum(uint32_t acc) {
  const uint32_t t = (acc & 0x00FF00FFu) + ((acc >> 8) & 0x00FF00FFu);
  return (t & 0xFFFFu) + (t >> 16);
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

// Warp-cooperative: keep the K largest of the cnt unique keys in buf (global),
// in place; returns the K-th largest key (the new admission threshold).
__device__ uint64_t select_topk(uint64_t *buf, int cnt, int K) {
  const int lane = threadIdx.x & 31;
  uint64_t v[kCapW];
#pragma unroll
  for (int t = 0; t < kCapW; ++t) {
    const int i = t * 32 + lane;
    v[t] = i < cnt ? buf[i] : 0ull;
  }
  uint64_t P = 0;
  for (int bit = 63; bit >= 0; --bit) {
    const uint64_t c = P | (1ull << bit);
    int k = 0;
#pragma unroll
    for (int t = 0; t < kCapW; ++t) k += v[t] >= c;
    if ((int)__reduce_add_sync(FULL, (unsigned)k) >= K) P = c;
  }
  __syncwarp();
  int out = 0;
#pragma unroll
  for (int t = 0; t < kCapW; ++t) {
    const bool keep = v[t] >= P && v[t] != 0ull;
    const unsigned m = __ballot_sync(FULL, keep);
    if (keep) buf[out + __popc(m & ((1u << lane) - 1u))] = v[t];
    out += __popc(m);
  }
  __syncwarp();
  return P;
}

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
    const uint64_t P = select_topk(w.gbuf + (size_t)r * w.cap, w.cnt[r], w.K);
    if (lane == 0) { w.cnt[r] = w.K; w.thr[r] = P; }
    __syncwarp();
  }
}

// Register-match counts of up to 32 queued survivors (lane = survivor); the
// row codes and column codes both come through L1/L2.
__device__ __forceinline__ void count_batch(const GraphArgs &g, Warp &w, const int *q, int nq,
                                            int64_t row0) {
  const int lane = threadIdx.x & 31;
  const bool act = lane < nq;
  const unsigned e = act ? (unsigned)q[lane] : 0u;
  const int r = (int)(e >> 27);
  const int64_t j = e & 0x07FFFFFFu;
  if (act) {
    const uint4 *ra = (const uint4 *)(g.codesA + (row0 + r) * g.mpad);
    const uint4 *cb = (const uint4 *)(g.codesB + j * g.mpad);
    const int m4 = g.mpad >> 4;
    uint32_t cnt = 0;
    for (int w0 = 0; w0 < m4; w0 += 63) {
      const int w1 = (w0 + 63 < m4) ? w0 + 63 : m4;
      uint32_t acc = 0;
      for (int t = w0; t < w1; ++t) {
        const uint4 a = __ldg(ra + t), b = __ldg(cb + t);
        acc += eq_bytes(a.x, b.x) + eq_bytes(a.y, b.y) + eq_bytes(a.z, b.z) +
               eq_bytes(a.w, b.w);
      }
      cnt += byte_sum(acc);
    }
    atomicMax(&w.mxc[r], cnt);
    const uint64_t key = ((uint64_t)__ldg(g.sv_bits + cnt) << 32) | (uint64_t)(~(uint32_t)j);
    if (key > w.thr[r]) {
      const int p = atomicAdd(&w.cnt[r], 1);
      w.gbuf[(size_t)r * w.cap + p] = key;
    }
  }
  __syncwarp();
  compact_full_rows(w, w.cap - 32);
}

template <int SMAX, bool SPARSE>
__global__ void __launch_bounds__(kWarps * 32)
k_allpairs(GraphArgs g, uint64_t *gbuf, int cap, float lo, float hi) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t n = g.n;
  const int64_t row0 = ((int64_t)blockIdx.x * kWarps + warp) * 32;
  const int64_t row = row0 + lane;
  const bool vrow = row < n;
  const int S = g.S, Su = g.Su;
  const int mw = g.mpad >> 2;
  const int mwq = ((mw + 27) & ~31) + 4;           // = 4 mod 32 words: conflict-free LDS.128

  // per-warp shared state
  unsigned char *ws = smem + (size_t)warp * (SPARSE ? 1024 : (1024 + 32 * mwq * 4));
  uint64_t *thr = (uint64_t *)ws;                  // [32]
  int *cnt = (int *)(thr + 32);                    // [32]
  uint32_t *mxc = (uint32_t *)(cnt + 32);          // [32]
  uint32_t *mxa = mxc + 32;                        // [32]
  int *q = (int *)(mxa + 32);                      // [kQ]
  uint32_t *sA = (uint32_t *)(ws + 1024);          // dense: [32][mwq] row codes

  thr[lane] = 0;
  cnt[lane] = 0;
  mxc[lane] = 0;
  mxa[lane] = 0;
  Warp w{gbuf + (size_t)(row0 < n ? row0 : 0) * cap, cnt, thr, mxc, cap, g.K};
  const uint8_t nz_row = vrow ? g.anynz[row] : 0;
  unsigned long long n_pref = 0, n_cmp = 0;
  __syncwarp();

  if (!SPARSE) {
    for (int i = lane; i < 32 * (mw >> 2); i += 32) {
      const int r = i / (mw >> 2), t = i - r * (mw >> 2);
      uint4 v = make_uint4(0, 0, 0, 0);
      if (row0 + r < n) v = __ldg((const uint4 *)(g.codesA + (row0 + r) * g.mpad) + t);
      *(uint4 *)(sA + r * mwq + 4 * t) = v;
    }
    __syncwarp();
    const uint32_t *ra = sA + lane * mwq;
    uint32_t mx_a = 0, mx_c = 0;
    const int m4 = mw >> 2;
    for (int64_t j0 = 0; j0 < n; j0 += 4) {
      const int64_t j1 = j0 + 1 < n ? j0 + 1 : j0, j2 = j0 + 2 < n ? j0 + 2 : j0,
                    j3 = j0 + 3 < n ? j0 + 3 : j0;
      const uint4 *c0 = (const uint4 *)(g.codesB + j0 * g.mpad);
      const uint4 *c1 = (const uint4 *)(g.codesB + j1 * g.mpad);
      const uint4 *c2 = (const uint4 *)(g.codesB + j2 * g.mpad);
      const uint4 *c3 = (const uint4 *)(g.codesB + j3 * g.mpad);
      uint32_t cntq[4] = {0, 0, 0, 0};
      for (int t0 = 0; t0 < m4; t0 += 63) {
        const int t1 = t0 + 63 < m4 ? t0 + 63 : m4;
        uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll 2
        for (int t = t0; t < t1; ++t) {
          const uint4 a = *(const uint4 *)(ra + 4 * t);
          const uint4 b0 = __ldg(c0 + t), b1 = __ldg(c1 + t), b2 = __ldg(c2 + t),
                      b3 = __ldg(c3 + t);
          a0 += eq_bytes(a.x, b0.x) + eq_bytes(a.y, b0.y) + eq_bytes(a.z, b0.z) + eq_bytes(a.w, b0.w);
          a1 += eq_bytes(a.x, b1.x) + eq_bytes(a.y, b1.y) + eq_bytes(a.z, b1.z) + eq_bytes(a.w, b1.w);
          a2 += eq_bytes(a.x, b2.x) + eq_bytes(a.y, b2.y) + eq_bytes(a.z, b2.z) + eq_bytes(a.w, b2.w);
          a3 += eq_bytes(a.x, b3.x) + eq_bytes(a.y, b3.y) + eq_bytes(a.z, b3.z) + eq_bytes(a.w, b3.w);
        }
        cntq[0] += byte_sum(a0);
        cntq[1] += byte_sum(a1);
        cntq[2] += byte_sum(a2);
        cntq[3] += byte_sum(a3);
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int64_t j = j0 + t;
        const bool other = vrow && j < n && j != row;
        const bool cand = other && (nz_row | __ldg(g.anynz + (j < n ? j : 0)));
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
    mxa[lane] = mx_a;
    mxc[lane] = mx_c;
  } else {
    float ur[SMAX];
#pragma unroll
    for (int t = 0; t < SMAX; ++t) ur[t] = (vrow && t < Su) ? g.unit[row * Su + t] : 0.f;
    int qn = 0;
    for (int64_t j = 0; j < n; ++j) {
      const bool other = vrow && j != row;
      const bool cand = other && (nz_row | __ldg(g.anynz + j));
      const float4 *uj = (const float4 *)(g.unit + j * Su);
      float c1 = 0.f;
#pragma unroll
      for (int t4 = 0; t4 < SMAX; t4 += 4) {
        if (t4 < Su) {
          const float4 v = __ldg(uj + (t4 >> 2));
          c1 = __fmaf_rn(ur[t4 + 0], v.x, c1);
          c1 = __fmaf_rn(ur[t4 + 1], v.y, c1);
          c1 = __fmaf_rn(ur[t4 + 2], v.z, c1);
          c1 = __fmaf_rn(ur[t4 + 3], v.w, c1);
        }
      }
      n_pref += cand;
      bool pass = cand && c1 >= hi;
      const bool band = cand && c1 >= lo && c1 < hi;
      if (__any_sync(FULL, band)) {
        if (band) pass = !(dot_avx512<SMAX>(ur, g.unit + j * Su, S) < g.prefilter_eps);
      }
      const unsigned m = __ballot_sync(FULL, pass);
      if (m) {
        if (pass) q[qn + __popc(m & ((1u << lane) - 1u))] = (int)(((unsigned)lane << 27) | (unsigned)j);
        qn += __popc(m);
        __syncwarp();
        if (qn >= 32) {
          count_batch(g, w, q, 32, row0);
          n_cmp += 1;
          if (lane + 32 < qn) q[lane] = q[lane + 32];
          __syncwarp();
          qn -= 32;
        }
      }
    }
    if (qn > 0) {
      n_cmp += lane < qn;
      count_batch(g, w, q, qn, row0);
    }
  }
  if (g.stats) {
    if (n_pref) atomicAdd(g.stats, n_pref);
    if (n_cmp) atomicAdd(g.stats + 1, n_cmp);
  }
  __syncwarp();
  // the K best of each row, written unsorted
  compact_full_rows(w, g.K);
  if (vrow) {
    const int c = cnt[lane];
    for (int i = 0; i < c; ++i) g.topk[row * g.K + i] = w.gbuf[(size_t)lane * cap + i];
    g.topk_cnt[row] = c;
    g.maxcnt_cand[row] = mxc[lane];
    g.maxcnt_all[row] = mxa[lane];
  }
}

size_t allpairs_smem(int mpad, bool sparse) {
  const int mw = mpad >> 2;
  const int mwq = ((mw + 27) & ~31) + 4;
  return (size_t)kWarps * (sparse ? 1024 : (1024 + 32 * (size_t)mwq * 4));
}

}  // namespace

int allpairs_cap(int K) { return (K + 64 + 31) & ~31; }

void launch_allpairs(const GraphArgs &g, uint64_t *gbuf, cudaStream_t s) {
  if (g.n == 0) return;
  const int cap = allpairs_cap(g.K);
  const bool sparse = g.prefilter != 0;
  const size_t smem = allpairs_smem(g.mpad, sparse);
  const unsigned grid = (unsigned)((g.n + kWarps * 32 - 1) / (kWarps * 32));
  // band of the exact-safe prefilter: |chain - AVX-512 order| < delta
  const double eps = (double)g.prefilter_eps;
  const double delta = (double)(g.S + (g.S + 15) / 16 + 8) * ldexp(1.0, -23);
  float lo = (float)(eps - delta), hi = (float)(eps + delta);
  if ((double)lo > eps - delta) lo = nextafterf(lo, -INFINITY);
  if ((double)hi < eps + delta) hi = nextafterf(hi, INFINITY);
#define RBG_LAUNCH(SM, SP)                                                                   \
  do {                                                                                       \
    cudaFuncSetAttribute(k_allpairs<SM, SP>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                         (int)smem);                                                         \
    k_allpairs<SM, SP><<<grid, kWarps * 32, smem, s>>>(g, gbuf, cap, lo, hi);               \
  } while (0)
  if (sparse) {
    if (g.Su <= 16) RBG_LAUNCH(16, true);
    else if (g.Su <= 32) RBG_LAUNCH(32, true);
    else RBG_LAUNCH(64, true);
  } else {
    RBG_LAUNCH(4, false);
  }
#undef RBG_LAUNCH
}

}  // namespace rbg
