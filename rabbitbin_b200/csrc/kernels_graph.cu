// Graph stage kernels: unit rank rows, column norms, register-match counts,
// the all-pairs top-K pass, neighbour filtering / edge emission and edge
// weights.
//
// Compiled with -fmad=false.  Where the reference's release build computes a
// fused multiply-add (AVX-512 _mm512_fmadd_ps, or a GCC-contracted a*b+c) the
// code below calls __fmaf_rn / __fma_rn explicitly; everything else rounds
// operation by operation exactly as the reference does.
#include <cstdint>
#include <cuda_fp16.h>

#include "rbg_internal.h"

namespace rbg {
namespace {

constexpr unsigned FULL = 0xffffffffu;

// Last assembly a with starts[a] <= x (starts ascending, starts[0] = 0).
__device__ __forceinline__ int find_asm(const int64_t *starts, int nb, int64_t x) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(starts + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ── unit rank rows (src/rabbitbin.cpp:4867-4874 rank, :4972-4988 unit rows,
//    src/ranker.h:55-66 average ranks, src/impl/rb_abundance.cpp:94-114 anynz)
// Warp per row, lane = sample (two samples per lane when S > 32).  The average
// rank of x_k is 1 + #{x_l < x_k} + (#{x_l == x_k} - 1) / 2, a half-integer, so
// the reference's sequential double sums of ranks and of squared deviations
// (multiples of 1/4, far below 2^53) are exact in any order: warp reductions
// give the same mean and ss.
__device__ __forceinline__ void unit_row(const GraphArgs &g, int64_t r) {
  const int lane = threadIdx.x & 31;
  const int S = g.S;
  const float *x = g.depth_raw + r * S;
  const float x0 = lane < S ? x[lane] : 0.f;
  const float x1 = lane + 32 < S ? x[lane + 32] : 0.f;
  float rk0 = 0.f, rk1 = 0.f;
  bool nz = !g.has_depth;
  if (g.has_depth) {
    if (S > 1) {
      int less0 = 0, eq0 = 0, less1 = 0, eq1 = 0;
      for (int l = 0; l < S; ++l) {
        const float xl = __shfl_sync(0xffffffffu, l < 32 ? x0 : x1, l & 31);
        less0 += xl < x0; eq0 += xl == x0;
        less1 += xl < x1; eq1 += xl == x1;
      }
      rk0 = __fadd_rn((float)(2 * less0 + eq0 - 1) / 2.0f, 1.0f);
      rk1 = __fadd_rn((float)(2 * less1 + eq1 - 1) / 2.0f, 1.0f);
      nz = (lane < S && (double)rk0 > g.min_cv_d) || (lane + 32 < S && (double)rk1 > g.min_cv_d);
    } else {
      nz = lane < S && (double)x0 > g.min_cv_d;
    }
    nz = __any_sync(0xffffffffu, nz);
  }
  if (lane == 0) g.anynz[r] = nz ? 1 : 0;
  if (S <= 1) return;
  double sum = (lane < S ? (double)rk0 : 0.0) + (lane + 32 < S ? (double)rk1 : 0.0);
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  const double mean = sum / (double)S;
  const double d0 = lane < S ? __dsub_rn((double)rk0, mean) : 0.0;
  const double d1 = lane + 32 < S ? __dsub_rn((double)rk1, mean) : 0.0;
  double ss = __dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1));
  for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
  float *u = g.unit + r * g.Su;
  const double inv = ss > 0.0 ? 1.0 / __dsqrt_rn(ss) : 0.0;
  const float f0 = (lane < S && ss > 0.0) ? __double2float_rn(__dmul_rn(d0, inv)) : 0.0f;
  const float f1 = (lane + 32 < S && ss > 0.0) ? __double2float_rn(__dmul_rn(d1, inv)) : 0.0f;
  if (lane < g.Su) u[lane] = f0;
  if (lane + 32 < g.Su) u[lane + 32] = f1;
  if (g.unit16) {
    uint16_t *h = g.unit16 + r * g.Kp;
    if (lane < g.Kp) h[lane] = __half_as_ushort(__float2half_rn(f0));
    if (lane + 32 < g.Kp) h[lane + 32] = __half_as_ushort(__float2half_rn(f1));
  }
}

__global__ void k_unit_rows(GraphArgs g) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (r >= g.n) return;
  unit_row(g, r);
}

__global__ void k_unit_rows_batch(const BatchAsm *B, const int64_t *row0s, int nb,
                                  int64_t r_begin, int64_t rows) {
  const int64_t r = r_begin + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (r >= rows) return;
  const int a = find_asm(row0s, nb, r);
  unit_row(B[a].g, r - B[a].row0);
}

// Column norms of the raw depths (src/rabbitbin.cpp:4800-4806): the reference
// sums each column in row order in double.  Fast path: if every value of a
// column is an integer multiple of 2^E (E = lowest set bit over its non-zero
// values) and sum|x| < 2^(52+E), every partial sum in any order is a multiple
// of 2^E below 2^(53+E) and so exact; the parallel sum then equals the
// sequential one.  Columns that fail the test are summed sequentially.
__device__ __forceinline__ int low_bit_exp(float x) {
  const uint32_t b = __float_as_uint(x) & 0x7FFFFFFFu;
  const int e = (int)(b >> 23);
  uint32_t mant = b & 0x7FFFFFu;
  int base;
  if (e == 0) base = -149;                       // subnormal: mant * 2^-149
  else { mant |= 0x800000u; base = e - 150; }    // mant * 2^(e-150)
  return base + __ffs(mant) - 1;
}

__device__ __forceinline__ void colsum_fast(const GraphArgs &g, double *acc, int blk, int nblk) {
  // acc layout per column i: [0] sum, [1] sum |x|, [2] (int) min exponent
  __shared__ double ssum[kMaxS], sabs[kMaxS];
  __shared__ int semin[kMaxS];
  const int S = g.S;
  for (int i = threadIdx.x; i < S; i += blockDim.x) { ssum[i] = 0.0; sabs[i] = 0.0; semin[i] = 1 << 20; }
  __syncthreads();
  const int64_t total = g.n * S;
  for (int64_t q = (int64_t)blk * blockDim.x + threadIdx.x; q < total;
       q += (int64_t)nblk * blockDim.x) {
    const float x = g.depth_raw[q];
    const int i = (int)(q % S);
    if (x != 0.0f) {
      atomicAdd(&ssum[i], (double)x);
      atomicAdd(&sabs[i], fabs((double)x));
      atomicMin(&semin[i], low_bit_exp(x));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    atomicAdd(&acc[3 * i], ssum[i]);
    atomicAdd(&acc[3 * i + 1], sabs[i]);
    atomicMin((int *)&acc[3 * i + 2], semin[i]);
  }
}

__global__ void k_colsum_fast(GraphArgs g, double *acc) { colsum_fast(g, acc, blockIdx.x, gridDim.x); }

__global__ void k_colsum_fast_batch(const BatchAsm *B) {
  const BatchAsm &b = B[blockIdx.y];
  if (b.colnorm_on && b.g.n > 0) colsum_fast(b.g, b.colacc, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ void colnorm_body(const GraphArgs &g, const double *acc) {
  constexpr int CH = 128;
  __shared__ float chunk[CH * kMaxS];
  __shared__ int need_seq;
  const int S = g.S, i = threadIdx.x;
  bool exact = false;
  double s = 0.0;
  if (i < S) {
    const int emin = *(const int *)&acc[3 * i + 2];
    const double sum_abs = acc[3 * i + 1];
    exact = (emin >= (1 << 20)) ||                                  // all zero
            (emin > -1000 && sum_abs < ldexp(1.0, 52 + emin));
    s = emin >= (1 << 20) ? 0.0 : acc[3 * i];
  }
  if (threadIdx.x == 0) need_seq = 0;
  __syncthreads();
  if (i < S && !exact) atomicOr(&need_seq, 1);
  __syncthreads();
  if (need_seq) {
    double sq = 0.0;
    for (int64_t r0 = 0; r0 < g.n; r0 += CH) {
      const int rows = (int)((g.n - r0) < CH ? (g.n - r0) : CH);
      __syncthreads();
      for (int q = threadIdx.x; q < rows * S; q += blockDim.x) chunk[q] = g.depth_raw[r0 * S + q];
      __syncthreads();
      if (i < S && !exact)
        for (int r = 0; r < rows; ++r) sq = __dadd_rn(sq, (double)chunk[r * S + i]);
    }
    if (i < S && !exact) s = sq;
  }
  if (i < S) {
    const double mean = s / (double)(g.n > 1 ? g.n : 1);
    g.colnorm[i] = (mean > 1e-12) ? 1.0 / mean : 0.0;
  }
}

__global__ void k_colnorm(GraphArgs g, const double *acc) { colnorm_body(g, acc); }

__global__ void k_colnorm_batch(const BatchAsm *B) {
  const BatchAsm &b = B[blockIdx.x];
  if (b.colnorm_on && b.g.n > 0) colnorm_body(b.g, b.colacc);
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

// b0 of every assembly of a batch (estimate_pmh_baseline,
// src/rabbitbin.cpp:1340-1369): register-match counts of its sampled pairs
// (local ids), then the element at index np/2 of their sorted list from a
// histogram of the counts (the float match fractions sort as the counts do),
// then the similarity table of pmh_sv_from_count (:1297-1305).
__global__ void k_pair_counts_batch(const BatchAsm *B, const int64_t *pair0s, int nb,
                                    int64_t p_begin, int64_t npairs,
                                    const int32_t *__restrict__ pairs, uint32_t *__restrict__ out) {
  const int64_t p = p_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const int a = find_asm(pair0s, nb, p);
  const GraphArgs &g = B[a].g;
  const uint32_t *x = (const uint32_t *)(g.codesA + (int64_t)pairs[2 * p] * g.mpad);
  const uint32_t *y = (const uint32_t *)(g.codesB + (int64_t)pairs[2 * p + 1] * g.mpad);
  uint32_t c = 0;
  for (int w = 0; w < g.mpad / 4; ++w) c += match4(__ldg(x + w), __ldg(y + w));
  out[p] = c;
}

// b0 = the count at index np/2 of the sorted sample counts (a histogram of
// the counts: the float match fractions sort as the counts do), then the
// similarity table of pmh_sv_from_count.  One CTA.
__device__ __forceinline__ void b0_body(const uint32_t *__restrict__ counts, int np, int m,
                                        bool base_on_in, float *b0_out, uint32_t *sv_out) {
  extern __shared__ int hist[];
  __shared__ int med;
  const bool on = base_on_in && np > 0;
  if (on) {
    for (int c = threadIdx.x; c <= m; c += blockDim.x) hist[c] = 0;
    __syncthreads();
    for (int q = threadIdx.x; q < np; q += blockDim.x) atomicAdd(&hist[counts[q]], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      int cum = 0, c = 0;
      for (; c < m; ++c) {
        cum += hist[c];
        if (cum > np / 2) break;
      }
      med = c;
    }
    __syncthreads();
  }
  const double inv_m = 1.0 / (double)m;
  const float b0f = on ? (float)__dmul_rn((double)(uint32_t)med, inv_m) : 0.0f;
  const double b0 = (double)b0f;
  if (threadIdx.x == 0) *b0_out = b0f;
  const double inv1mb0 = (b0 < 1.0) ? 1.0 / __dsub_rn(1.0, b0) : 1.0;
  for (int c = threadIdx.x; c <= m; c += blockDim.x) {
    double j = __dmul_rn((double)(uint32_t)c, inv_m);
    if (base_on_in && b0 > 0.0 && b0 < 1.0) {
      j = __dmul_rn(__dsub_rn(j, b0), inv1mb0);
      if (j < 0.0) j = 0.0;
    }
    if (j > 1.0 - 1e-6) j = 1.0 - 1e-6;
    sv_out[c] = __float_as_uint((float)j);
  }
}

__global__ void k_b0_batch(const BatchAsm *B, const uint32_t *__restrict__ counts) {
  const BatchAsm &b = B[blockIdx.x];
  b0_body(counts + b.pair0, b.np, b.g.m, b.base_on != 0, b.b0, b.sv_out);
}

__global__ void k_b0(const uint32_t *__restrict__ counts, int np, int m, float *b0_out,
                     uint32_t *sv_out) {
  b0_body(counts, np, m, true, b0_out, sv_out);
}

__host__ __device__ __forceinline__ int pow2_at_least(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Ascending bitonic sort of 32 R keys held in registers, element r * 32 + lane
// in v[r]: strides of 32 and more pair registers of the same lane, shorter
// strides pair lanes through shuffles.
template <int R>
__device__ __forceinline__ void warp_bitonic_asc(uint64_t (&v)[R]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32 * R; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int p = r ^ (stride >> 5);
          if (p > r) {
            const bool up = (((r * 32 + lane) & size) == 0);
            const uint64_t x = v[r], y = v[p];
            if ((x > y) == up) { v[r] = y; v[p] = x; }
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const uint64_t o = __shfl_xor_sync(FULL, v[r], stride);
          const bool up = (((r * 32 + lane) & size) == 0);
          const bool lower = (lane & stride) == 0;
          v[r] = (lower == up) ? (v[r] < o ? v[r] : o) : (v[r] < o ? o : v[r]);
        }
      }
    }
  }
}

// The first `len` (= 32 R) keys of buf, ascending, written out as ids and
// similarities; entries equal to ~0 are padding.
template <int R>
__device__ __forceinline__ void sort_kept(const EmitArgs &e, int64_t i, const uint64_t *buf) {
  const int lane = threadIdx.x & 31;
  uint64_t v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = buf[r * 32 + lane];
  warp_bitonic_asc<R>(v);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int q = r * 32 + lane;
    if (v[r] != ~0ULL) {
      e.nbr_sorted[i * e.K + q] = (uint32_t)(v[r] >> 32);
      e.nbr_sv[i * e.K + q] = __uint_as_float((uint32_t)v[r]);
    }
  }
}

// ── neighbour lists: cut by the calibrated threshold, sorted by id ──────────
// Keys above the cutoff are compacted into the warp's shared buffer as
// (id, sv bits), so an ascending sort orders ids; only the next power of two
// above their number is sorted, in registers.
__device__ __forceinline__ void sort_row(const EmitArgs &e, int64_t i, uint64_t *keys) {
  const int lane = threadIdx.x & 31;
  const int K = e.K;
  const int c = e.topk_cnt[i];
  int kept = 0;
  for (int q0 = 0; q0 < c; q0 += 32) {
    const int q = q0 + lane;
    bool ok = false;
    uint64_t v = 0;
    if (q < c) {
      const uint64_t key = e.topk[i * K + q];
      const uint32_t svb = (uint32_t)(key >> 32);
      ok = (double)__uint_as_float(svb) > e.cutoff;
      v = ((uint64_t)(~(uint32_t)key) << 32) | svb;
    }
    const unsigned m = __ballot_sync(FULL, ok);
    if (ok) keys[kept + __popc(m & ((1u << lane) - 1u))] = v;
    kept += __popc(m);
  }
  const int len = pow2_at_least(kept > 32 ? kept : 32);
  for (int q = kept + lane; q < len; q += 32) keys[q] = ~0ULL;
  __syncwarp();
  if (len <= 32) sort_kept<1>(e, i, keys);
  else if (len <= 64) sort_kept<2>(e, i, keys);
  else if (len <= 128) sort_kept<4>(e, i, keys);
  else if (len <= 256) sort_kept<8>(e, i, keys);
  else sort_kept<16>(e, i, keys);
  if (lane == 0) e.nbr_cnt[i] = kept;
  __syncwarp();
}

__global__ void k_sort_rows(EmitArgs e) {
  extern __shared__ uint64_t shk[];
  const int wib = threadIdx.x >> 5;
  const int64_t i = e.row_lo + (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  if (i >= (e.row_hi < 0 ? e.n : e.row_hi)) return;
  sort_row(e, i, shk + (size_t)wib * pow2_at_least(e.K > 32 ? e.K : 32));
}

__global__ void k_sort_rows_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                                  int maxlen) {
  extern __shared__ uint64_t shk[];
  const int wib = threadIdx.x >> 5;
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  if (r >= rows) return;
  const int a = find_asm(row0s, nb, r);
  sort_row(B[a].e, r - B[a].row0, shk + (size_t)wib * maxlen);
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
// Warp per row: lane q tests neighbour q (coalesced id reads, the searches in
// the partners' lists run side by side).
__device__ __forceinline__ bool edge_kept(const EmitArgs &e, int64_t i, uint32_t j) {
  if ((int64_t)j <= i) return false;
  return !(e.mutual && !e.small_path) ||
         has_nbr(e.nbr_sorted + (int64_t)j * e.K, e.nbr_cnt[j], (uint32_t)i);
}

__device__ __forceinline__ void count_edges_row(const EmitArgs &e, int64_t i) {
  const int lane = threadIdx.x & 31;
  const int c = e.nbr_cnt[i];
  const uint32_t *ids = e.nbr_sorted + i * e.K;
  int cnt = 0;
  const int kw = (e.K + 31) >> 5;
  for (int q0 = 0; q0 < c; q0 += 32) {
    const int q = q0 + lane;
    const bool ok = q < c && edge_kept(e, i, ids[q]);
    const unsigned m = __ballot_sync(FULL, ok);
    if (e.kept && lane == 0) e.kept[i * kw + (q0 >> 5)] = m;
    cnt += __popc(m);
  }
  if (lane == 0) e.row_edges[i] = cnt;
}

__global__ void k_count_edges(EmitArgs e) {
  const int64_t i = e.row_lo + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i < (e.row_hi < 0 ? e.n : e.row_hi)) count_edges_row(e, i);
}

__global__ void k_count_edges_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= rows) return;
  const int a = find_asm(row0s, nb, r);
  count_edges_row(B[a].e, r - B[a].row0);
}

// First edge of every assembly after the batch-wide scan of row_edges.
__global__ void k_edge0s(const int64_t *row0s, int nb, const int32_t *row_edges, int64_t *edge0s) {
  for (int a = threadIdx.x; a <= nb; a += blockDim.x) edge0s[a] = row_edges[row0s[a]];
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

__device__ __forceinline__ void write_edges_row(const EmitArgs &e, int64_t i) {
  const int lane = threadIdx.x & 31;
  const int c = e.nbr_cnt[i];
  const uint32_t *ids = e.nbr_sorted + i * e.K;
  int64_t o = e.row_edges[i];
  const int kw = (e.K + 31) >> 5;
  for (int q0 = 0; q0 < c; q0 += 32) {
    const int q = q0 + lane;
    const uint32_t j = q < c ? ids[q] : 0u;
    unsigned m;
    if (e.kept) {
      m = e.kept[i * kw + (q0 >> 5)];              // recorded by the edge count
    } else {
      m = __ballot_sync(FULL, q < c && edge_kept(e, i, j));
    }
    const bool ok = (m >> lane) & 1u;
    if (ok) {
      const int64_t at = o + __popc(m & ((1u << lane) - 1u));
      e.from[at] = (uint32_t)i;
      e.to[at] = j;
      e.scomp[at] = e.nbr_sv[i * e.K + q];
    }
    o += __popc(m);
  }
}

__global__ void k_write_edges(EmitArgs e) {
  const int64_t i = e.row_lo + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i < (e.row_hi < 0 ? e.n : e.row_hi)) write_edges_row(e, i);
}

__global__ void k_write_edges_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= rows) return;
  const int a = find_asm(row0s, nb, r);
  write_edges_row(B[a].e, r - B[a].row0);
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

__device__ __forceinline__ void edge_weight(const WeightArgs &w, int64_t e) {
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

__global__ void k_edge_weights(WeightArgs w) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < w.n_edges) edge_weight(w, e);
}

__global__ void k_edge_weights_batch(const BatchAsm *B, const int64_t *edge0s, int nb, int64_t edges) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= edges) return;
  edge_weight(B[find_asm(edge0s, nb, e)].w, e);
}

}  // namespace

void launch_unit_rows(const GraphArgs &g, cudaStream_t s) {
  if (g.n == 0) return;
  k_unit_rows<<<(unsigned)((g.n + 7) / 8), 256, 0, s>>>(g);   // warp per row
}

void launch_colnorm(const GraphArgs &g, double *acc, cudaStream_t s) {
  if (g.S == 0) return;
  // zeroed slots: the exponent minimum then starts at 0, a valid (conservative)
  // lower bound of every column's lowest set bit once values below 1 appear
  cudaMemsetAsync(acc, 0, 3 * sizeof(double) * g.S, s);
  k_colsum_fast<<<296, 256, 0, s>>>(g, acc);
  k_colnorm<<<1, 256, 0, s>>>(g, acc);
}

void launch_b0(const uint32_t *counts, int np, int m, float *b0_out, uint32_t *sv_out,
               cudaStream_t s) {
  k_b0<<<1, 256, (size_t)(m + 1) * sizeof(int), s>>>(counts, np, m, b0_out, sv_out);
}

void launch_pair_counts(const uint8_t *A, const uint8_t *B, int mpad, int m,
                        const int64_t *pairs, int np, uint32_t *out, cudaStream_t s) {
  (void)m;
  if (np == 0) return;
  k_pair_counts<<<(np + 127) / 128, 128, 0, s>>>(A, B, mpad, pairs, np, out);
}

void launch_sort_rows(const EmitArgs &e, cudaStream_t s) {
  const int64_t rows = (e.row_hi < 0 ? e.n : e.row_hi) - e.row_lo;
  if (rows <= 0) return;
  int len = 1;
  while (len < (e.K > 32 ? e.K : 32)) len <<= 1;
  const int warps = 4;
  k_sort_rows<<<(unsigned)((rows + warps - 1) / warps), warps * 32,
                (size_t)warps * len * 8, s>>>(e);
}

// Edge counts of the rows, then their exclusive scan in place (total at
// row_edges[row_hi]): the edges of row i start at row_edges[i].
void launch_count_edges(const EmitArgs &e, cudaStream_t s) {
  const int64_t rows = (e.row_hi < 0 ? e.n : e.row_hi) - e.row_lo;
  if (rows <= 0) return;
  k_count_edges<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(e);   // warp per row
  k_scan<<<1, 1024, 0, s>>>(e.row_edges + e.row_lo, rows);
}

void launch_write_edges(const EmitArgs &e, cudaStream_t s) {
  const int64_t rows = (e.row_hi < 0 ? e.n : e.row_hi) - e.row_lo;
  if (rows <= 0) return;
  k_write_edges<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(e);   // warp per row
}

void launch_edge_weights(const WeightArgs &w, cudaStream_t s) {
  if (w.n_edges == 0) return;
  k_edge_weights<<<(unsigned)((w.n_edges + 127) / 128), 128, 0, s>>>(w);
}

void launch_unit_rows_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                            cudaStream_t s, int64_t r_begin) {
  if (rows <= r_begin) return;
  k_unit_rows_batch<<<(unsigned)((rows - r_begin + 7) / 8), 256, 0, s>>>(B, row0s, nb, r_begin,
                                                                         rows);
}

void launch_colnorm_batch(const BatchAsm *B, int nb, int max_s, cudaStream_t s) {
  if (nb <= 0 || max_s <= 1) return;
  k_colsum_fast_batch<<<dim3(64, (unsigned)nb), 256, 0, s>>>(B);
  k_colnorm_batch<<<(unsigned)nb, 256, 0, s>>>(B);
}

void launch_b0_batch(const BatchAsm *B, const int64_t *pair0s, int nb, int64_t npairs,
                     const int32_t *pairs, uint32_t *counts, int max_m, cudaStream_t s) {
  launch_b0_batch_range(B, pair0s, nb, 0, npairs, pairs, counts, max_m, 0, nb, s);
}

void launch_b0_batch_range(const BatchAsm *B, const int64_t *pair0s, int nb, int64_t p_begin,
                           int64_t p_end, const int32_t *pairs, uint32_t *counts, int max_m,
                           int b_begin, int b_end, cudaStream_t s) {
  if (b_end <= b_begin) return;
  if (p_end > p_begin)
    k_pair_counts_batch<<<(unsigned)((p_end - p_begin + 127) / 128), 128, 0, s>>>(
        B, pair0s, nb, p_begin, p_end, pairs, counts);
  k_b0_batch<<<(unsigned)(b_end - b_begin), 256, (size_t)(max_m + 1) * sizeof(int), s>>>(
      B + b_begin, counts);
}

void launch_emit_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows, int max_k,
                       int32_t *row_edges, int64_t *edge0s, cudaStream_t s) {
  if (rows > 0) {
    const int len = pow2_at_least(max_k > 32 ? max_k : 32);
    const int warps = 4;
    k_sort_rows_batch<<<(unsigned)((rows + warps - 1) / warps), warps * 32,
                        (size_t)warps * len * 8, s>>>(B, row0s, nb, rows, len);
    k_count_edges_batch<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(B, row0s, nb, rows);
  }
  k_scan<<<1, 1024, 0, s>>>(row_edges, rows);
  k_edge0s<<<1, 256, 0, s>>>(row0s, nb, row_edges, edge0s);
}

void launch_write_edges_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                              cudaStream_t s) {
  if (rows == 0) return;
  k_write_edges_batch<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(B, row0s, nb, rows);
}

void launch_edge_weights_batch(const BatchAsm *B, const int64_t *edge0s, int nb, int64_t edges,
                               cudaStream_t s) {
  if (edges == 0) return;
  k_edge_weights_batch<<<(unsigned)((edges + 127) / 128), 128, 0, s>>>(B, edge0s, nb, edges);
}

}  // namespace rbg
