// FASTA ingest on the device (parse_fasta_mmap_parallel,
// src/rabbitbin.cpp:1890-2248): the file's bytes in HBM become the large and
// small contigs' sequences back to back, their lengths and name ranges.
//
//   1. positions of every '\n' and '>' (per-tile counts, a scan, a scatter);
//   2. record starts: a '>' starts a record when it is the first '>' of its
//      line (no '>' between it and the previous '\n'): the reference scans
//      for '>' from the end of each body, and a header's own later '>' bytes
//      are inside the header line it skips;
//   3. per record (thread): name = bytes > ' ' after the '>', header ends at
//      the next '\n' (none: the record and everything after it are dropped),
//      body = up to the next record start; single-line when the bytes after
//      its first '\n' are all '\n'/'\r' (its first line minus one trailing
//      '\r'), else every '\n'-separated segment minus one trailing '\r';
//   4. large (>= min_contig) and small (>= min_small) lengths scanned into
//      offsets; one CTA per record copies its segments.
#include <cstdint>

#include "rbg_internal.h"

namespace rbg {
namespace {

constexpr int kTile = 4096;               // bytes per CTA in the position passes
constexpr int kTileThreads = 256;         // 16 bytes per thread

__device__ __forceinline__ void count16(const uint4 v, int &nl, int &gt) {
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint32_t c = (w[k] >> (8 * b)) & 0xFFu;
      nl += c == '\n';
      gt += c == '>';
    }
}

// Bytes [t*16, t*16+16) of the tile; the input is padded to 16 bytes with
// zeros (never '\n' or '>').
__global__ void k_fasta_tile_counts(const uint4 *__restrict__ in, int64_t words, int *nl_cnt,
                                    int *gt_cnt) {
  __shared__ int s_nl[kTileThreads / 32], s_gt[kTileThreads / 32];
  const int64_t w = (int64_t)blockIdx.x * kTileThreads + threadIdx.x;
  int nl = 0, gt = 0;
  if (w < words) count16(__ldg(in + w), nl, gt);
  nl = __reduce_add_sync(0xffffffffu, nl);
  gt = __reduce_add_sync(0xffffffffu, gt);
  if ((threadIdx.x & 31) == 0) { s_nl[threadIdx.x >> 5] = nl; s_gt[threadIdx.x >> 5] = gt; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int a = 0, b = 0;
    for (int i = 0; i < kTileThreads / 32; ++i) { a += s_nl[i]; b += s_gt[i]; }
    nl_cnt[blockIdx.x] = a;
    gt_cnt[blockIdx.x] = b;
  }
}

// Exclusive scan of n counts in place (+ total at v[n]), one CTA.
__global__ void k_scan64(int64_t *v, int64_t n) {
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
  for (int64_t q = a; q < b; ++q) { const int64_t x = v[q]; v[q] = run; run += x; }
  if (t == 1023) v[n] = part[1023];
}

__global__ void k_widen(const int *in, int64_t *out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

// Positions of '\n' and '>' in file order (tile prefix offsets from k_scan64).
__global__ void k_fasta_scatter(const uint4 *__restrict__ in, int64_t words,
                                const int64_t *__restrict__ nl_base,
                                const int64_t *__restrict__ gt_base, int64_t *nl_pos,
                                int64_t *gt_pos) {
  __shared__ int s_nl[kTileThreads / 32 + 1], s_gt[kTileThreads / 32 + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t w = (int64_t)blockIdx.x * kTileThreads + threadIdx.x;
  uint4 v = make_uint4(0, 0, 0, 0);
  if (w < words) v = __ldg(in + w);
  int nl = 0, gt = 0;
  count16(v, nl, gt);
  // block-exclusive ranks: warp inclusive scans, then warp offsets
  int inl = nl, igt = gt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int a = __shfl_up_sync(0xffffffffu, inl, o), b = __shfl_up_sync(0xffffffffu, igt, o);
    if (lane >= o) { inl += a; igt += b; }
  }
  if (lane == 31) { s_nl[wid] = inl; s_gt[wid] = igt; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int a = 0, b = 0;
    for (int i = 0; i < kTileThreads / 32; ++i) {
      const int x = s_nl[i], y = s_gt[i];
      s_nl[i] = a; s_gt[i] = b;
      a += x; b += y;
    }
  }
  __syncthreads();
  int64_t pn = nl_base[blockIdx.x] + s_nl[wid] + inl - nl;
  int64_t pg = gt_base[blockIdx.x] + s_gt[wid] + igt - gt;
  const uint32_t wd[4] = {v.x, v.y, v.z, v.w};
  const int64_t base = w * 16;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint32_t c = (wd[k] >> (8 * b)) & 0xFFu;
      if (c == '\n') nl_pos[pn++] = base + 4 * k + b;
      if (c == '>') gt_pos[pg++] = base + 4 * k + b;
    }
}

// Number of entries of sorted a[0..n) that are < x.
__device__ __forceinline__ int64_t lower_count(const int64_t *a, int64_t n, int64_t x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// flag[i] = 1 when the i-th '>' is the first '>' of its line.
__global__ void k_fasta_starts(const int64_t *__restrict__ gt_pos, int64_t ngt,
                               const int64_t *__restrict__ nl_pos, int64_t nnl, int64_t *flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ngt) return;
  if (i == 0) { flag[i] = 1; return; }
  const int64_t q = gt_pos[i];
  const int64_t k = lower_count(nl_pos, nnl, q);        // newlines before q
  const int64_t prev_nl = k > 0 ? nl_pos[k - 1] : -1;
  flag[i] = gt_pos[i - 1] < prev_nl ? 1 : 0;
}

__global__ void k_fasta_compact(const int64_t *__restrict__ gt_pos, int64_t ngt,
                                const int64_t *__restrict__ rank, int64_t *rs) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ngt && rank[i + 1] != rank[i]) rs[rank[i]] = gt_pos[i];
}

// One record per thread: name range, body, length after newline removal and
// class (0 tiny, 1 small, 2 large, 3 no header newline: dropped, not counted).
__global__ void k_fasta_records(const uint8_t *__restrict__ in, int64_t F,
                                const int64_t *__restrict__ rs, int64_t nrs,
                                const int64_t *__restrict__ nl_pos, int64_t nnl,
                                int64_t min_contig, int64_t min_small, FastaRec *rec) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nrs) return;
  FastaRec r;
  const int64_t s = rs[k];
  int64_t ne = s + 1;
  while (ne < F && in[ne] > ' ') ++ne;
  r.name_start = s + 1;
  r.name_len = (int32_t)(ne - s - 1);
  const int64_t ih = lower_count(nl_pos, nnl, ne);          // the header's newline
  if (ih >= nnl) {
    r.cls = 3; r.single = 0; r.len = 0; r.b0 = r.b1 = 0; r.nl0 = r.nl1 = 0;
    rec[k] = r;
    return;
  }
  const int64_t b0 = nl_pos[ih] + 1;
  const int64_t b1 = k + 1 < nrs ? rs[k + 1] : F;
  const int64_t ie = lower_count(nl_pos, nnl, b1);           // newlines before b1
  r.b0 = b0;
  r.b1 = b1;
  r.nl0 = ih + 1;                                            // body newlines [nl0, nl1)
  r.nl1 = ie > ih + 1 ? ie : ih + 1;
  const int64_t first_nl = r.nl1 > r.nl0 ? nl_pos[r.nl0] : -1;
  bool single = true;
  if (first_nl >= 0)
    for (int64_t q = first_nl + 1; q < b1; ++q)
      if (in[q] != '\n' && in[q] != '\r') { single = false; break; }
  int64_t len = 0;
  if (single) {
    int64_t e = first_nl >= 0 ? first_nl : b1;
    if (e > b0 && in[e - 1] == '\r') --e;
    len = e - b0;
  } else {
    int64_t st = b0;
    for (int64_t i = r.nl0; i <= r.nl1; ++i) {
      const int64_t e = i < r.nl1 ? nl_pos[i] : b1;
      int64_t l = e - st;
      if (l > 0 && in[e - 1] == '\r') --l;
      len += l;
      st = e + 1;
    }
  }
  r.single = single ? 1 : 0;
  r.len = len;
  r.cls = len >= min_contig ? 2 : (len >= min_small ? 1 : 0);
  rec[k] = r;
}

// Per record: 1 / length when it is of class c, else 0 (scanned into output
// indices and byte offsets).
__global__ void k_fasta_class(const FastaRec *__restrict__ rec, int64_t nrs, int c,
                              int64_t *flag, int64_t *bytes) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nrs) return;
  const bool on = rec[k].cls == c;
  flag[k] = on ? 1 : 0;
  bytes[k] = on ? rec[k].len : 0;
}

// One CTA per record: copy its kept bytes (segments minus newlines and one
// trailing '\r' each) to its output slot; write its name range and length.
__global__ void k_fasta_copy(const uint8_t *__restrict__ in, const FastaRec *__restrict__ rec,
                             const int64_t *__restrict__ nl_pos, int c,
                             const int64_t *__restrict__ idx, const int64_t *__restrict__ off,
                             uint8_t *out, int64_t *out_off, int64_t *name_start,
                             int32_t *name_len) {
  const int64_t k = blockIdx.x;
  const FastaRec r = rec[k];
  if (r.cls != c) return;
  const int64_t o = idx[k];
  uint8_t *dst = out + off[k];
  if (threadIdx.x == 0) {
    out_off[o + 1] = off[k] + r.len;
    name_start[o] = r.name_start;
    name_len[o] = r.name_len;
    if (o == 0) out_off[0] = 0;
  }
  if (r.single) {
    for (int64_t q = threadIdx.x; q < r.len; q += blockDim.x) dst[q] = in[r.b0 + q];
    return;
  }
  int64_t st = r.b0, w = 0;
  for (int64_t i = r.nl0; i <= r.nl1; ++i) {
    const int64_t e = i < r.nl1 ? nl_pos[i] : r.b1;
    int64_t l = e - st;
    if (l > 0 && in[e - 1] == '\r') --l;
    for (int64_t q = threadIdx.x; q < l; q += blockDim.x) dst[w + q] = in[st + q];
    w += l;
    st = e + 1;
  }
}

}  // namespace

void launch_fasta_positions(const uint8_t *in, int64_t F, int *tile_nl, int *tile_gt,
                            int64_t *nl_base, int64_t *gt_base, cudaStream_t s) {
  const int64_t words = (F + 15) / 16;
  const int64_t tiles = (words + kTileThreads - 1) / kTileThreads;
  if (tiles == 0) return;
  k_fasta_tile_counts<<<(unsigned)tiles, kTileThreads, 0, s>>>((const uint4 *)in, words, tile_nl,
                                                              tile_gt);
  k_widen<<<(unsigned)((tiles + 255) / 256), 256, 0, s>>>(tile_nl, nl_base, tiles);
  k_widen<<<(unsigned)((tiles + 255) / 256), 256, 0, s>>>(tile_gt, gt_base, tiles);
  k_scan64<<<1, 1024, 0, s>>>(nl_base, tiles);
  k_scan64<<<1, 1024, 0, s>>>(gt_base, tiles);
}

void launch_fasta_scatter(const uint8_t *in, int64_t F, const int64_t *nl_base,
                          const int64_t *gt_base, int64_t *nl_pos, int64_t *gt_pos,
                          cudaStream_t s) {
  const int64_t words = (F + 15) / 16;
  const int64_t tiles = (words + kTileThreads - 1) / kTileThreads;
  if (tiles == 0) return;
  k_fasta_scatter<<<(unsigned)tiles, kTileThreads, 0, s>>>((const uint4 *)in, words, nl_base,
                                                          gt_base, nl_pos, gt_pos);
}

void launch_fasta_starts(const int64_t *gt_pos, int64_t ngt, const int64_t *nl_pos, int64_t nnl,
                         int64_t *flag, int64_t *rs, cudaStream_t s) {
  if (ngt == 0) return;
  k_fasta_starts<<<(unsigned)((ngt + 255) / 256), 256, 0, s>>>(gt_pos, ngt, nl_pos, nnl, flag);
  k_scan64<<<1, 1024, 0, s>>>(flag, ngt);
  k_fasta_compact<<<(unsigned)((ngt + 255) / 256), 256, 0, s>>>(gt_pos, ngt, flag, rs);
}

void launch_fasta_records(const uint8_t *in, int64_t F, const int64_t *rs, int64_t nrs,
                          const int64_t *nl_pos, int64_t nnl, int64_t min_contig,
                          int64_t min_small, FastaRec *rec, cudaStream_t s) {
  if (nrs == 0) return;
  k_fasta_records<<<(unsigned)((nrs + 127) / 128), 128, 0, s>>>(in, F, rs, nrs, nl_pos, nnl,
                                                               min_contig, min_small, rec);
}

void launch_fasta_class(const FastaRec *rec, int64_t nrs, int c, int64_t *flag, int64_t *bytes,
                        cudaStream_t s) {
  if (nrs == 0) return;
  k_fasta_class<<<(unsigned)((nrs + 255) / 256), 256, 0, s>>>(rec, nrs, c, flag, bytes);
  k_scan64<<<1, 1024, 0, s>>>(flag, nrs);
  k_scan64<<<1, 1024, 0, s>>>(bytes, nrs);
}

void launch_fasta_copy(const uint8_t *in, const FastaRec *rec, int64_t nrs, const int64_t *nl_pos,
                       int c, const int64_t *idx, const int64_t *off, uint8_t *out,
                       int64_t *out_off, int64_t *name_start, int32_t *name_len, cudaStream_t s) {
  if (nrs == 0) return;
  k_fasta_copy<<<(unsigned)nrs, 256, 0, s>>>(in, rec, nl_pos, c, idx, off, out, out_off,
                                            name_start, name_len);
}

}  // namespace rbg
