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
  float *u = g.unit + r * g.Su;
  if (ss > 0.0) {
    const double inv = 1.0 / __dsqrt_rn(ss);
    for (int k = 0; k < S; ++k)
      u[k] = __double2float_rn(__dmul_rn(__dsub_rn((double)rk[k], mean), inv));
  } else {
    for (int k = 0; k < S; ++k) u[k] = 0.0f;
  }
  for (int k = S; k < g.Su; ++k) u[k] = 0.0f;
}

// Column norms of the raw depths, summed in row order
// (src/rabbitbin.cpp:4800-4806): one CTA stages row chunks in shared memory
// with coalesced loads; thread i < S adds its column sequentially.
__global__ void k_colnorm(GraphArgs g) {
  constexpr int CH = 128;
  __shared__ float chunk[CH * kMaxS];
  const int S = g.S, i = threadIdx.x;
  double s = 0.0;
  for (int64_t r0 = 0; r0 < g.n; r0 += CH) {
    const int rows = (int)((g.n - r0) < CH ? (g.n - r0) : CH);
    __syncthreads();
    for (int q = threadIdx.x; q < rows * S; q += blockDim.x) chunk[q] = g.depth_raw[r0 * S + q];
    __syncthreads();
    if (i < S)
      for (int r = 0; r < rows; ++r) s = __dadd_rn(s, (double)chunk[r * S + i]);
  }
  if (i < S) {
    const double mean = s / (double)(g.n > 1 ? g.n : 1);
    g.colnorm[i] = (mean > 1e-12) ? 1.0 / mean : 0.0;
  }
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
        const double corr = depth_corr(w.unit + i * w.Su, w.unit + j * w.Su, S);
        if (isfinite(corr) && corr < w.neg_thr) ok = false;
      }
      dterm = wj < 0.0 ? 0.0 : (wj > 1.0 ? 1.0 : wj);
    }
  } else {
    const double corr = depth_corr(w.unit + i * w.Su, w.unit + j * w.Su, S);
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
  k_colnorm<<<1, 256, 0, s>>>(g);
}

void launch_pair_counts(const uint8_t *A, const uint8_t *B, int mpad, int m,
                        const int64_t *pairs, int np, uint32_t *out, cudaStream_t s) {
  (void)m;
  if (np == 0) return;
  k_pair_counts<<<(np + 127) / 128, 128, 0, s>>>(A, B, mpad, pairs, np, out);
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
