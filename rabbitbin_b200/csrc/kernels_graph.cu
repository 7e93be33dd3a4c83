// Graph stage kernels: unit rank rows, column norms, register-match counts,
// the all-pairs top-K pass, neighbour filtering / edge emission and edge
// weights.
//
// Compiled with -fmad=false.  Where the reference's release build computes a
// fused multiply-add (AVX-512 _mm512_fmadd_ps, or a GCC-contracted a*b+c) the
// code below calls __fmaf_rn / __fma_rn explicitly; everything else rounds
// operation by operation exactly as the reference does.
#include <cstdint>

#include "rbg_internal.h"

namespace rbg {
namespace {

constexpr unsigned FULL = 0xffffffffu;

// ── unit rank rows (src/rabbitbin.cpp:4867-4874 rank, :4972-4988 unit rows,
//    src/ranker.h:55-66 average ranks, src/impl/rb_abundance.cpp:94-114 anynz)
__global__ void k_unit_rows(GraphArgs g) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= g.n) return;
  const int S = g.S;
  float x[kMaxS], rk[kMaxS];
  for (int k = 0; k < S; ++k) x[k] = g.depth_raw[r * S + k];
  uint8_t nz = 1;
  if (g.has_depth) {
    nz = 0;
    if (S > 1) {
      for (int k = 0; k < S; ++k) {
        int less = 0, eq = 0;
        for (int l = 0; l < S; ++l) { less += x[l] < x[k]; eq += x[l] == x[k]; }
        // average rank of a tie group starting at sorted position `less`
        rk[k] = __fadd_rn((float)(2 * less + eq - 1) / 2.0f, 1.0f);
        if ((double)rk[k] > g.min_cv_d) nz = 1;
      }
    } else {
      for (int k = 0; k < S; ++k) if ((double)x[k] > g.min_cv_d) nz = 1;
    }
  }
  g.anynz[r] = nz;
  if (S <= 1) return;
  double mean = 0.0;
  for (int k = 0; k < S; ++k) mean = __dadd_rn(mean, (double)rk[k]);
  mean = mean / (double)S;
  double ss = 0.0;
  for (int k = 0; k < S; ++k) {
    const double d = __dsub_rn((double)rk[k], mean);
    ss = __dadd_rn(ss, __dmul_rn(d, d));
  }
  float *u = g.unit + r * S;
  if (ss > 0.0) {
    const double inv = 1.0 / __dsqrt_rn(ss);
    for (int k = 0; k < S; ++k)
      u[k] = __double2float_rn(__dmul_rn(__dsub_rn((double)rk[k], mean), inv));
  } else {
    for (int k = 0; k < S; ++k) u[k] = 0.0f;
  }
}

// Column norms of the raw depths, summed in row order
// (src/rabbitbin.cpp:4800-4806).
__global__ void k_colnorm(GraphArgs g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.S) return;
  double s = 0.0;
  for (int64_t r = 0; r < g.n; ++r) s = __dadd_rn(s, (double)g.depth_raw[r * g.S + i]);
  const double mean = s / (double)(g.n > 1 ? g.n : 1);
  g.colnorm[i] = (mean > 1e-12) ? 1.0 / mean : 0.0;
}

// Number of registers where two 8-bit code words agree (A side: 0 = unset,
// B side: 0xFF = unset, so unset never matches).
__device__ __forceinline__ uint32_t match4(uint32_t a, uint32_t b) {
  const uint32_t x = a ^ b;
  const uint32_t t = ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x;
  return __popc(~t & 0x80808080u);
}

__global__ void k_pair_counts(const uint8_t *__restrict__ A, const uint8_t *__restrict__ B,
                              int mpad, const int64_t *__restrict__ pairs, int np,
                              uint32_t *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const uint32_t *a = (const uint32_t *)(A + pairs[2 * p] * (int64_t)mpad);
  const uint32_t *b = (const uint32_t *)(B + pairs[2 * p + 1] * (int64_t)mpad);
  uint32_t c = 0;
  for (int w = 0; w < mpad / 4; ++w) c += match4(__ldg(a + w), __ldg(b + w));
  out[p] = c;
}

// unit_dot_f (src/rabbitbin.cpp:754-796) on an AVX-512 host: element t goes to
// lane t % 16 of accumulator acc1 when it lies in the second half of a full
// 32-element block, else of acc0; the masked tail joins acc0; the lanes are
// then reduced as _mm512_reduce_add_ps does (halves of 8, 4, 2, 1).
template <int SMAX>
__device__ __forceinline__ float unit_dot_avx512(const float (&a)[SMAX], const float *b,
                                                 int S) {
  float acc0[16], acc1[16];
#pragma unroll
  for (int l = 0; l < 16; ++l) { acc0[l] = 0.f; acc1[l] = 0.f; }
  const int lim32 = S & ~31;
#pragma unroll
  for (int t = 0; t < SMAX; ++t) {
    if (t < S) {
      if ((t & 16) && t < lim32) acc1[t & 15] = __fmaf_rn(a[t], b[t], acc1[t & 15]);
      else acc0[t & 15] = __fmaf_rn(a[t], b[t], acc0[t & 15]);
    }
  }
  float v[16];
  if (lim32 > 0) {
#pragma unroll
    for (int l = 0; l < 16; ++l) v[l] = __fadd_rn(acc0[l], acc1[l]);
  } else {
    // acc1 is all zeros: acc0 + 0 only differs in the sign of a zero lane
#pragma unroll
    for (int l = 0; l < 16; ++l) v[l] = acc0[l];
  }
#pragma unroll
  for (int l = 0; l < 8; ++l) v[l] = __fadd_rn(v[l], v[l + 8]);
#pragma unroll
  for (int l = 0; l < 4; ++l) v[l] = __fadd_rn(v[l], v[l + 4]);
  v[0] = __fadd_rn(v[0], v[2]);
  v[1] = __fadd_rn(v[1], v[3]);
  return __fadd_rn(v[0], v[1]);
}

// Bitonic sort, descending, of `len` (power of two) keys in shared memory by
// one warp.
__device__ void warp_sort_desc(uint64_t *keys, int len) {
  const int lane = threadIdx.x & 31;
  for (int size = 2; size <= len; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < len; i += 32) {
        const int j = i ^ stride;
        if (j > i) {
          const uint64_t a = keys[i], b = keys[j];
          const bool desc = ((i & size) == 0);
          if (desc ? (a < b) : (a > b)) { keys[i] = b; keys[j] = a; }
        }
      }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ int pow2_at_least(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

constexpr int kWarps = 8;       // warps per all-pairs CTA
constexpr int kColsPerWarp = 2; // columns a warp handles between CTA syncs
constexpr int kColWords = 8;    // column code words a lane keeps in registers

// Compact one row's candidate buffer: keep the K best keys (descending) and
// move the admission threshold up to the K-th best.
__device__ void compact_row(uint64_t *buf, int &cnt, uint64_t &thr, int K, int cap) {
  const int lane = threadIdx.x & 31;
  const int len = pow2_at_least(cnt > 1 ? cnt : 2);
  for (int i = cnt + lane; i < len; i += 32) buf[i] = 0;
  __syncwarp();
  warp_sort_desc(buf, len);
  if (cnt >= K) {
    thr = buf[K - 1];
    cnt = K;
  }
  __syncwarp();
}

// All-pairs pass over full rows.  CTA = 32 rows (lane = row) x 8 warps that
// walk the columns; per (row, column) pair: is_nz, the abundance-first float
// test, the register-match count (warp-cooperative, only for surviving pairs),
// the per-row maximum count and admission of the (similarity, id) key into the
// row's top-K buffer.  Sampled-row calibration and both graph paths are served
// from the per-row maxima and top-K lists this pass leaves behind.
template <int SMAX>
__global__ void __launch_bounds__(kWarps * 32)
k_allpairs(GraphArgs g, int cap, int small_path) {
  extern __shared__ uint64_t sh[];
  uint64_t *buf = sh;                                     // [32][cap]
  uint64_t *thr = buf + (size_t)kRowsPerCta * cap;        // [32]
  int *bcnt = (int *)(thr + kRowsPerCta);                 // [32]
  uint32_t *maxc = (uint32_t *)(bcnt + kRowsPerCta);      // [32]
  uint32_t *maxa = maxc + kRowsPerCta;                    // [32]
  int *need = (int *)(maxa + kRowsPerCta);                // [1]
  uint32_t *rowA = (uint32_t *)(need + 4);                // [32][mpad/4]

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t row0 = (int64_t)blockIdx.x * kRowsPerCta;
  const int64_t row = row0 + lane;
  const bool vrow = row < g.n;
  const int mw = g.mpad >> 2;
  const int S = g.S;
  const int K = g.K;

  for (int i = threadIdx.x; i < kRowsPerCta; i += blockDim.x) {
    thr[i] = 0; bcnt[i] = 0; maxc[i] = 0; maxa[i] = 0;
  }
  for (int i = threadIdx.x; i < kRowsPerCta * mw; i += blockDim.x) {
    const int r = i / mw, w = i - r * mw;
    rowA[i] = (row0 + r < g.n) ? __ldg((const uint32_t *)(g.codesA + (row0 + r) * g.mpad) + w) : 0u;
  }
  float ur[SMAX];
#pragma unroll
  for (int t = 0; t < SMAX; ++t) ur[t] = (vrow && t < S && g.prefilter) ? g.unit[row * S + t] : 0.f;
  const uint8_t nz_row = vrow ? g.anynz[row] : 0;
  __syncthreads();

  uint32_t my_maxc = 0, my_maxa = 0;
  unsigned long long n_pref = 0, n_cmp = 0;
  const int64_t step = (int64_t)kWarps * kColsPerWarp;
  for (int64_t j0 = 0; j0 < g.n; j0 += step) {
    for (int q = 0; q < kColsPerWarp; ++q) {
      const int64_t j = j0 + warp * kColsPerWarp + q;
      if (j >= g.n) break;
      const bool other = vrow && j != row;
      bool cand = other && (nz_row | __ldg(g.anynz + j));
      if (cand && g.prefilter) {
        float ub[SMAX];
        const float *uj = g.unit + j * S;
#pragma unroll
        for (int t = 0; t < SMAX; ++t) ub[t] = (t < S) ? __ldg(uj + t) : 0.f;
        const float c = unit_dot_avx512<SMAX>(ur, ub, S);
        ++n_pref;
        if (c < g.prefilter_eps) cand = false;
      }
      const bool count_it = small_path ? other : cand;
      uint32_t mask = __ballot_sync(FULL, count_it);
      if (mask == 0) continue;
      n_cmp += (count_it ? 1 : 0);
      // column j's B codes: lane holds words lane, lane+32, ...
      const uint32_t *cb = (const uint32_t *)(g.codesB + j * g.mpad);
      uint32_t colw[kColWords];
#pragma unroll
      for (int t = 0; t < kColWords; ++t) {
        const int w = lane + 32 * t;
        colw[t] = (w < mw) ? __ldg(cb + w) : 0xFFFFFFFFu;
      }
      uint32_t cnt = 0;
      while (mask) {
        const int r = __ffs(mask) - 1;
        mask &= mask - 1;
        const uint32_t *ra = rowA + r * mw;
        uint32_t part = 0;
#pragma unroll
        for (int t = 0; t < kColWords; ++t) {
          const int w = lane + 32 * t;
          if (w < mw) part += match4(ra[w], colw[t]);
        }
        for (int w = lane + 32 * kColWords; w < mw; w += 32)
          part += match4(ra[w], __ldg(cb + w));
        const uint32_t tot = __reduce_add_sync(FULL, part);
        if (lane == r) cnt = tot;
      }
      if (count_it) {
        if (small_path) my_maxa = cnt > my_maxa ? cnt : my_maxa;
        if (cand) {
          my_maxc = cnt > my_maxc ? cnt : my_maxc;
          const uint64_t key = ((uint64_t)__ldg(g.sv_bits + cnt) << 32) |
                               (uint64_t)(~(uint32_t)j);
          if (key > thr[lane]) {
            const int p = atomicAdd(&bcnt[lane], 1);
            buf[(size_t)lane * cap + p] = key;
          }
        }
      }
    }
    __syncthreads();
    // compact rows whose buffers could overflow before the next sync
    for (int r = warp; r < kRowsPerCta; r += kWarps) {
      int c = bcnt[r];
      if (c > cap - (int)step) {
        uint64_t t = thr[r];
        compact_row(buf + (size_t)r * cap, c, t, K, cap);
        if (lane == 0) { bcnt[r] = c; thr[r] = t; }
      }
    }
    __syncthreads();
  }
  atomicMax(&maxc[lane], my_maxc);
  atomicMax(&maxa[lane], my_maxa);
  if (g.stats) {
    if (n_pref) atomicAdd(g.stats, n_pref);
    if (n_cmp) atomicAdd(g.stats + 1, n_cmp);
  }
  __syncthreads();
  for (int r = warp; r < kRowsPerCta; r += kWarps) {
    const int64_t gr = row0 + r;
    if (gr >= g.n) continue;
    int c = bcnt[r];
    uint64_t t = thr[r];
    compact_row(buf + (size_t)r * cap, c, t, K, cap);
    const int keep = c < K ? c : K;
    for (int i = lane; i < keep; i += 32) g.topk[gr * K + i] = buf[(size_t)r * cap + i];
    if (lane == 0) {
      g.topk_cnt[gr] = keep;
      g.maxcnt_cand[gr] = maxc[r];
      g.maxcnt_all[gr] = maxa[r];
    }
  }
}

// ── neighbour lists: cut by the calibrated threshold, sorted by id ──────────
__global__ void k_sort_rows(EmitArgs e) {
  extern __shared__ uint64_t shk[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  if (i >= e.n) return;
  const int K = e.K;
  const int len = pow2_at_least(K > 32 ? K : 32);
  uint64_t *keys = shk + (size_t)wib * len;
  const int c = e.topk_cnt[i];
  // keep sv > cutoff; re-key as (id, sv bits) so an ascending sort orders ids
  for (int q = lane; q < len; q += 32) {
    uint64_t v = ~0ULL;
    if (q < c) {
      const uint64_t key = e.topk[i * K + q];
      const uint32_t svb = (uint32_t)(key >> 32);
      const float sv = __uint_as_float(svb);
      if ((double)sv > e.cutoff) v = ((uint64_t)(~(uint32_t)key) << 32) | svb;
    }
    keys[q] = ~v;   // descending sort of ~v = ascending sort of v
  }
  __syncwarp();
  warp_sort_desc(keys, len);
  int kept = 0;
  for (int q0 = 0; q0 < len; q0 += 32) {
    const int q = q0 + lane;
    const uint64_t v = ~keys[q];
    const bool ok = v != ~0ULL;
    if (ok) {
      e.nbr_sorted[i * K + q] = (uint32_t)(v >> 32);
      e.nbr_sv[i * K + q] = __uint_as_float((uint32_t)v);
    }
    kept += __popc(__ballot_sync(FULL, ok));
  }
  if (lane == 0) e.nbr_cnt[i] = kept;
}

__device__ __forceinline__ bool has_nbr(const uint32_t *ids, int cnt, uint32_t x) {
  int lo = 0, hi = cnt;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ids[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo < cnt && ids[lo] == x;
}

// Edges of row i: (i, j) for kept neighbours j > i; with the mutual filter
// (src/impl/rb_graph.cpp:1284-1348) i must also be a kept neighbour of j.
__global__ void k_count_edges(EmitArgs e) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= e.n) return;
  const int c = e.nbr_cnt[i];
  const uint32_t *ids = e.nbr_sorted + i * e.K;
  int cnt = 0;
  for (int q = 0; q < c; ++q) {
    const uint32_t j = ids[q];
    if ((int64_t)j <= i) continue;
    if (e.mutual && !e.small_path &&
        !has_nbr(e.nbr_sorted + (int64_t)j * e.K, e.nbr_cnt[j], (uint32_t)i)) continue;
    ++cnt;
  }
  e.row_edges[i] = cnt;
}

__global__ void k_scan(int32_t *v, int64_t n) {
  // exclusive scan of n counts into v[0..n], one CTA of 1024 threads
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t per = (n + 1023) / 1024;
  const int64_t a = t * per, b = (a + per < n) ? a + per : n;
  int64_t s = 0;
  for (int64_t q = a; q < b; ++q) s += v[q];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int64_t add = (t >= off) ? part[t - off] : 0;
    __syncthreads();
    part[t] += add;
    __syncthreads();
  }
  int64_t run = (t > 0) ? part[t - 1] : 0;
  for (int64_t q = a; q < b; ++q) { const int32_t x = v[q]; v[q] = (int32_t)run; run += x; }
  if (t == 1023) v[n] = (int32_t)part[1023];
}

__global__ void k_write_edges(EmitArgs e) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= e.n) return;
  const int c = e.nbr_cnt[i];
  const uint32_t *ids = e.nbr_sorted + i * e.K;
  int64_t o = e.row_edges[i];
  for (int q = 0; q < c; ++q) {
    const uint32_t j = ids[q];
    if ((int64_t)j <= i) continue;
    if (e.mutual && !e.small_path &&
        !has_nbr(e.nbr_sorted + (int64_t)j * e.K, e.nbr_cnt[j], (uint32_t)i)) continue;
    e.from[o] = (uint32_t)i;
    e.to[o] = j;
    e.scomp[o] = e.nbr_sv[i * e.K + q];
    ++o;
  }
}

// ── edge weights (src/rabbitbin.cpp:5482-5509, depth_edge_term :930-970) ───
// depth_corr_fast (:705-746) on an AVX-512 host: full 16-lane blocks in float
// (two accumulators over 32-element blocks), one horizontal reduction, then
// the remaining samples in double.
__device__ double depth_corr(const float *a, const float *b, int S) {
  float acc0[16], acc1[16];
#pragma unroll
  for (int l = 0; l < 16; ++l) { acc0[l] = 0.f; acc1[l] = 0.f; }
  int k = 0;
  for (; k + 32 <= S; k += 32)
    for (int l = 0; l < 16; ++l) {
      acc0[l] = __fmaf_rn(a[k + l], b[k + l], acc0[l]);
      acc1[l] = __fmaf_rn(a[k + 16 + l], b[k + 16 + l], acc1[l]);
    }
  for (; k + 16 <= S; k += 16)
    for (int l = 0; l < 16; ++l) acc0[l] = __fmaf_rn(a[k + l], b[k + l], acc0[l]);
  double s = 0.0;
  if (k > 0) {
    float v[16];
    for (int l = 0; l < 16; ++l) v[l] = __fadd_rn(acc0[l], acc1[l]);
    for (int l = 0; l < 8; ++l) v[l] = __fadd_rn(v[l], v[l + 8]);
    for (int l = 0; l < 4; ++l) v[l] = __fadd_rn(v[l], v[l + 4]);
    v[0] = __fadd_rn(v[0], v[2]);
    v[1] = __fadd_rn(v[1], v[3]);
    s = (double)__fadd_rn(v[0], v[1]);
  }
  for (; k < S; ++k) s = __dadd_rn(s, __dmul_rn((double)a[k], (double)b[k]));
  return s;
}

// cal_depth_wjac (src/rabbitbin.cpp:685-697)
__device__ double depth_wjac(const float *a, const float *b, int S, const double *cn) {
  double mn = 0.0, mx = 0.0;
  for (int i = 0; i < S; ++i) {
    double x = a[i], y = b[i];
    if (cn) { x = __dmul_rn(x, cn[i]); y = __dmul_rn(y, cn[i]); }
    if (x < y) { mn = __dadd_rn(mn, x); mx = __dadd_rn(mx, y); }
    else { mn = __dadd_rn(mn, y); mx = __dadd_rn(mx, x); }
  }
  if (mx <= 0.0) return 0.0;
  return mn / mx;
}

__global__ void k_edge_weights(WeightArgs w) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= w.n_edges) return;
  const float sc = w.scomp[e];
  if (w.S <= 0) {              // no depth file (src/rabbitbin.cpp:5532-5536)
    w.score[e] = (sc < w.min_edge) ? 0.0f : sc;
    return;
  }
  if (w.S == 1) { w.score[e] = sc; return; }
  const int64_t i = w.from[e], j = w.to[e];
  const int S = w.S;
  double dterm;
  bool ok = true;
  if (w.depth_sim == 1) {
    double wj = depth_wjac(w.depth_raw + i * S, w.depth_raw + j * S, S, w.colnorm);
    if (!isfinite(wj)) ok = false;
    else if (w.wjac_cut > 0.0 && wj < w.wjac_cut) ok = false;
    else {
      if (w.wjac_gate && w.neg_thr > -0.99) {
        const double corr = depth_corr(w.unit + i * S, w.unit + j * S, S);
        if (isfinite(corr) && corr < w.neg_thr) ok = false;
      }
      dterm = wj < 0.0 ? 0.0 : (wj > 1.0 ? 1.0 : wj);
    }
  } else {
    const double corr = depth_corr(w.unit + i * S, w.unit + j * S, S);
    if (!isfinite(corr)) ok = false;
    else if (w.neg_thr > -0.99 && corr < w.neg_thr) ok = false;
    else {
      const double cp = corr < 0.0 ? 0.0 : corr;
      dterm = cp;
      if (w.depth_sim == 2) {
        double wj = depth_wjac(w.depth_raw + i * S, w.depth_raw + j * S, S, w.colnorm);
        if (!isfinite(wj)) wj = 0.0;
        wj = wj < 0.0 ? 0.0 : (wj > 1.0 ? 1.0 : wj);
        if (w.depth_fuse == 1) dterm = cp < wj ? cp : wj;
        else if (w.depth_fuse == 2) dterm = __dmul_rn(cp, wj);
        else dterm = __dsqrt_rn(__dmul_rn(cp, wj));
      }
    }
  }
  if (!ok) { w.score[e] = 0.0f; return; }
  // w = a*sComp + (1-a)*dterm; the release build fuses the first product
  const double a = w.w_comp;
  const double s = (double)sc;
  double val = w.contract ? __fma_rn(a, s, __dmul_rn(1.0 - a, dterm))
                          : __dadd_rn(__dmul_rn(a, s), __dmul_rn(1.0 - a, dterm));
  if (!isfinite(val) || val < w.min_edge) val = 0.0;
  w.score[e] = (float)val;
}

}  // namespace

void launch_unit_rows(const GraphArgs &g, cudaStream_t s) {
  if (g.n == 0) return;
  k_unit_rows<<<(unsigned)((g.n + 127) / 128), 128, 0, s>>>(g);
}

void launch_colnorm(const GraphArgs &g, cudaStream_t s) {
  if (g.S == 0) return;
  k_colnorm<<<1, 64, 0, s>>>(g);
}

void launch_pair_counts(const uint8_t *A, const uint8_t *B, int mpad, int m,
                        const int64_t *pairs, int np, uint32_t *out, cudaStream_t s) {
  (void)m;
  if (np == 0) return;
  k_pair_counts<<<(np + 127) / 128, 128, 0, s>>>(A, B, mpad, pairs, np, out);
}

static size_t allpairs_smem(int cap, int mpad) {
  return (size_t)kRowsPerCta * cap * 8 + kRowsPerCta * 8 + kRowsPerCta * 4 * 3 + 16 +
         (size_t)kRowsPerCta * mpad;
}

int allpairs_cap(int K) {
  int c = 1;
  while (c < K + 2 * kWarps * kColsPerWarp) c <<= 1;
  return c;
}

void launch_allpairs(const GraphArgs &g, cudaStream_t s) {
  if (g.n == 0) return;
  const int cap = allpairs_cap(g.K);
  const size_t smem = allpairs_smem(cap, g.mpad);
  const unsigned grid = (unsigned)((g.n + kRowsPerCta - 1) / kRowsPerCta);
  if (g.S <= 16) {
    cudaFuncSetAttribute(k_allpairs<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_allpairs<16><<<grid, kWarps * 32, smem, s>>>(g, cap, g.small_path);
  } else if (g.S <= 32) {
    cudaFuncSetAttribute(k_allpairs<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_allpairs<32><<<grid, kWarps * 32, smem, s>>>(g, cap, g.small_path);
  } else {
    cudaFuncSetAttribute(k_allpairs<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_allpairs<64><<<grid, kWarps * 32, smem, s>>>(g, cap, g.small_path);
  }
}

void launch_sort_rows(const EmitArgs &e, cudaStream_t s) {
  if (e.n == 0) return;
  int len = 1;
  while (len < (e.K > 32 ? e.K : 32)) len <<= 1;
  const int warps = 4;
  k_sort_rows<<<(unsigned)((e.n + warps - 1) / warps), warps * 32,
                (size_t)warps * len * 8, s>>>(e);
}

void launch_count_edges(const EmitArgs &e, cudaStream_t s) {
  if (e.n == 0) return;
  k_count_edges<<<(unsigned)((e.n + 127) / 128), 128, 0, s>>>(e);
  k_scan<<<1, 1024, 0, s>>>(e.row_edges, e.n);
}

void launch_write_edges(const EmitArgs &e, cudaStream_t s) {
  if (e.n == 0) return;
  k_write_edges<<<(unsigned)((e.n + 127) / 128), 128, 0, s>>>(e);
}

void launch_edge_weights(const WeightArgs &w, cudaStream_t s) {
  if (w.n_edges == 0) return;
  k_edge_weights<<<(unsigned)((w.n_edges + 127) / 128), 128, 0, s>>>(w);
}

}  // namespace rbg
