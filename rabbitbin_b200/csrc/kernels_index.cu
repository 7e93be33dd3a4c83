// Inverted-index candidate graph of the small path (RABBIT_GRAPH_INDEX=1).
//
// build_similarity_graph (src/impl/rb_graph.cpp:199-383) restricts each
// contig's neighbours to the contigs that share at least minCommon
// one-permutation sketch keys with it (KmerSketch::getKeys,
// src/rabbit_sketch.h:166-175), found through an inverted index of those keys
// (rabbit_invidx::InvertedIndex, src/rabbit_invidx.h:51-160); posting lists
// longer than max(256, N / 8) are skipped.  The candidates are visited in the
// order the traversal first meets them (keys in bucket order, each posting
// list in contig order), each scored with the graph similarity, and a
// max-edges heap ordered by CompareEdge keeps those above the cutoff, a new
// candidate entering a full heap only when its similarity is strictly larger
// than the heap top's.
//
// Here: the index is the (key, contig) pairs of every non-empty bucket sorted
// by key with a stable radix sort (so each posting list is in contig order,
// the order the reference's single-threaded index build gives), run-length
// encoded into unique keys, list lengths and offsets.  One CTA per row: its
// posting lists are walked by all warps, which count shared keys per contig
// and record each contig's first touch (bucket << 19 | position) in shared
// memory; warp 0 then walks the lists again in order, keeps each contig at its
// first touch if it shares enough keys, scores it (8-bit register codes: the
// graph similarity through the similarity table) and lane 0 runs the heap.
// The kept neighbours are written as the row's top-K keys, descending, for
// the small path's edge emission.
#include <cub/cub.cuh>

#include <cstdint>

#include "rbg_internal.h"

namespace rbg {
namespace {

constexpr int kIxThreads = 256;
constexpr unsigned FULL = 0xffffffffu;
constexpr int kPosBits = 19;          // first-touch code: bucket << 19 | list position

struct HeapItem {
  float sim;
  uint32_t id;
};

// CompareEdge (src/rabbitbin.h:418-429) as "a below b" in the max-heap the
// priority queue keeps: lower similarity first, then the larger id.
__device__ __forceinline__ bool heap_less(const HeapItem &a, const HeapItem &b) {
  if (a.sim != b.sim) return a.sim > b.sim;
  return a.id < b.id;
}

__device__ void heap_push(HeapItem *h, int &size, HeapItem x) {
  int i = size++;
  while (i > 0) {
    const int p = (i - 1) >> 1;
    if (!heap_less(h[p], x)) break;
    h[i] = h[p];
    i = p;
  }
  h[i] = x;
}

__device__ HeapItem heap_pop(HeapItem *h, int &size) {
  const HeapItem top = h[0];
  const HeapItem x = h[--size];
  int i = 0;
  for (;;) {
    const int l = 2 * i + 1;
    if (l >= size) break;
    const int r = l + 1;
    const int c = (r < size && heap_less(h[l], h[r])) ? r : l;
    if (!heap_less(x, h[c])) break;
    h[i] = h[c];
    i = c;
  }
  if (size > 0) h[i] = x;
  return top;
}

__device__ __forceinline__ int64_t find_key(const uint64_t *keys, int64_t nk, uint64_t key) {
  int64_t lo = 0, hi = nk;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  return (lo < nk && keys[lo] == key) ? lo : -1;
}

// Register-match count of rows i and j on the 8-bit codes (A side 0 unset,
// B side 0xFF unset), by the whole warp.
__device__ __forceinline__ uint32_t warp_match_count(const GraphArgs &g, int64_t i, int64_t j) {
  const int lane = threadIdx.x & 31;
  const uint4 *a = reinterpret_cast<const uint4 *>(g.codesA + i * g.mpad);
  const uint4 *b = reinterpret_cast<const uint4 *>(g.codesB + j * g.mpad);
  uint32_t cnt = 0;
  for (int q = lane; q < g.mpad / 16; q += 32) {
    const uint4 x = __ldg(a + q), y = __ldg(b + q);
    const uint32_t w[4] = {x.x ^ y.x, x.y ^ y.y, x.z ^ y.z, x.w ^ y.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const uint32_t z = ~(((w[t] & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | w[t]) & 0x80808080u;
      cnt += __popc(z);
    }
  }
  return __reduce_add_sync(FULL, cnt);
}

struct IndexArgs {
  GraphArgs g;
  const uint64_t *row_keys;      // [n][m] keys of every row (0 = empty bucket)
  const uint64_t *ukeys;         // [nk] unique keys, ascending
  const int32_t *ucount;         // [nk] posting-list lengths
  const int64_t *uoff;           // [nk] offsets into post
  const uint32_t *post;          // posting lists (contigs ascending in each)
  const int32_t *nk;             // number of unique keys (device)
  int64_t pl_cap;                // lists longer than this are skipped
  int32_t min_common;
  double cutoff;                 // simCutoff / 1000
};

__global__ void __launch_bounds__(kIxThreads)
k_index_rows(const IndexArgs A) {
  extern __shared__ uint32_t ix_smem[];
  const GraphArgs &g = A.g;
  const int64_t n = g.n;
  const int m = g.m, K = g.K;
  const int64_t nk = *A.nk;
  uint32_t *first = ix_smem;                            // [n] first touch
  uint32_t *isect = first + n;                          // [(n + 1) / 2] 16-bit counts
  HeapItem *heap = reinterpret_cast<HeapItem *>(isect + (n + 1) / 2 + 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    for (int64_t t = threadIdx.x; t < n; t += kIxThreads) first[t] = 0xFFFFFFFFu;
    for (int64_t t = threadIdx.x; t < (n + 1) / 2; t += kIxThreads) isect[t] = 0u;
    __syncthreads();
    const uint64_t *ks = A.row_keys + i * m;
    // ── collisions and first touches ──
    for (int r = warp; r < m; r += kIxThreads / 32) {
      const uint64_t key = ks[r];
      if (key == 0ull) continue;
      const int64_t u = find_key(A.ukeys, nk, key);
      if (u < 0) continue;
      const int32_t cnt = A.ucount[u];
      if (cnt > A.pl_cap) continue;
      const uint32_t *pl = A.post + A.uoff[u];
      for (int pos = lane; pos < cnt; pos += 32) {
        const uint32_t j = pl[pos];
        if (j == (uint32_t)i) continue;
        atomicAdd(isect + (j >> 1), 1u << (16 * (j & 1u)));
        atomicMin(first + j, ((uint32_t)r << kPosBits) | (uint32_t)pos);
      }
    }
    __syncthreads();
    // ── candidates in traversal order, scored, through the heap (warp 0) ──
    if (warp == 0) {
      int size = 0;
      const uint8_t nz_i = g.anynz[i];
      for (int r = 0; r < m; ++r) {
        const uint64_t key = ks[r];
        if (key == 0ull) continue;
        const int64_t u = find_key(A.ukeys, nk, key);
        if (u < 0) continue;
        const int32_t cnt = A.ucount[u];
        if (cnt > A.pl_cap) continue;
        const uint32_t *pl = A.post + A.uoff[u];
        for (int p0 = 0; p0 < cnt; p0 += 32) {
          const int pos = p0 + lane;
          uint32_t j = 0;
          bool take = false;
          if (pos < cnt) {
            j = pl[pos];
            if (j != (uint32_t)i && first[j] == (((uint32_t)r << kPosBits) | (uint32_t)pos)) {
              const uint32_t c = (isect[j >> 1] >> (16 * (j & 1u))) & 0xFFFFu;
              take = (int)c >= A.min_common && (nz_i | g.anynz[j]);
            }
          }
          unsigned mk = __ballot_sync(FULL, take);
          while (mk) {
            const int L = __ffs(mk) - 1;
            mk &= mk - 1;
            const uint32_t jj = __shfl_sync(FULL, j, L);
            const uint32_t c = warp_match_count(g, i, jj);
            if (lane == 0) {
              const float sim = __uint_as_float(__ldg(g.sv_bits + c));
              if ((double)sim > A.cutoff &&
                  (size < K || (size == K && sim > heap[0].sim))) {
                if (size == K) heap_pop(heap, size);
                heap_push(heap, size, HeapItem{sim, jj});
              }
            }
            size = __shfl_sync(FULL, size, 0);
          }
        }
      }
      // the kept neighbours as top-K keys, descending: pops come weakest first
      if (lane == 0) {
        const int kept = size;
        for (int t = kept - 1; t >= 0; --t) {
          const HeapItem x = heap_pop(heap, size);
          g.topk[i * K + t] = ((uint64_t)__float_as_uint(x.sim) << 32) | (uint64_t)(~x.id);
        }
        g.topk_cnt[i] = kept;
      }
    }
    __syncthreads();
  }
}

__global__ void k_index_pairs(const uint64_t *__restrict__ row_keys, int64_t total, int m,
                              uint32_t *__restrict__ contig) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x)
    contig[q] = (uint32_t)(q / m);
}

}  // namespace

size_t index_rows_smem(int64_t n, int K) {
  return (size_t)n * 4 + (size_t)((n + 1) / 2 + 1) * 4 + (size_t)K * sizeof(HeapItem) + 16;
}

// Sorted (key, contig) pairs -> unique keys, list lengths, offsets.  Scratch
// is sized by the caller from index_build_bytes.  Returns the number of
// unique keys (including the empty-bucket key 0, which the rows never look up).
size_t index_build_bytes(int64_t total) {
  size_t a = 0, b = 0, c = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                  (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)total);
  cub::DeviceRunLengthEncode::Encode(nullptr, b, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                     (int32_t *)nullptr, (int32_t *)nullptr, (int)total);
  cub::DeviceScan::ExclusiveSum(nullptr, c, (const int32_t *)nullptr, (int64_t *)nullptr,
                                (int)total);
  return std::max(a, std::max(b, c)) + 256;
}

int launch_index_build(const uint64_t *row_keys, int64_t n, int m, uint64_t *keys_sorted,
                       uint32_t *contig_in, uint32_t *post, uint64_t *ukeys, int32_t *ucount,
                       int64_t *uoff, int32_t *nruns_dev, void *scratch, size_t scratch_bytes,
                       cudaStream_t s) {
  const int64_t total = n * (int64_t)m;
  if (total == 0) return 0;
  k_index_pairs<<<(unsigned)std::min<int64_t>((total + 255) / 256, 148 * 16), 256, 0, s>>>(
      row_keys, total, m, contig_in);
  if (cudaMemsetAsync(ucount, 0, (size_t)total * sizeof(int32_t), s) != cudaSuccess) return -1;
  size_t sb = scratch_bytes;
  // stable: equal keys keep their contig order
  if (cub::DeviceRadixSort::SortPairs(scratch, sb, row_keys, keys_sorted, contig_in, post,
                                      (int)total, 0, 64, s) != cudaSuccess)
    return -1;
  sb = scratch_bytes;
  if (cub::DeviceRunLengthEncode::Encode(scratch, sb, keys_sorted, ukeys, ucount, nruns_dev,
                                         (int)total, s) != cudaSuccess)
    return -1;
  sb = scratch_bytes;
  if (cub::DeviceScan::ExclusiveSum(scratch, sb, ucount, uoff, (int)total, s) != cudaSuccess)
    return -1;
  return 0;
}

void launch_index_rows(const GraphArgs &g, const uint64_t *row_keys, const uint64_t *ukeys,
                       const int32_t *ucount, const int64_t *uoff, const uint32_t *post,
                       const int32_t *nk, int64_t pl_cap, int min_common, double cutoff, int sms,
                       cudaStream_t s) {
  if (g.n == 0) return;
  IndexArgs A;
  A.g = g;
  A.row_keys = row_keys;
  A.ukeys = ukeys;
  A.ucount = ucount;
  A.uoff = uoff;
  A.post = post;
  A.nk = nk;
  A.pl_cap = pl_cap;
  A.min_common = min_common;
  A.cutoff = cutoff;
  const size_t smem = index_rows_smem(g.n, g.K);
  smem_cap_max((const void *)k_index_rows);
  const int64_t grid = std::min<int64_t>(g.n, (int64_t)sms * 2);
  k_index_rows<<<(unsigned)grid, kIxThreads, smem, s>>>(A);
}

}  // namespace rbg
