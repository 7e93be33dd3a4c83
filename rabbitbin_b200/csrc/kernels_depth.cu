// BAM -> depth summariser, device side: per-record depth sums and the means
// matrix.  The host (bam.cpp) inflates the BGZF blocks, walks the records and
// hands each chunk of decompressed records over with one offset per record.
//
//   k_depth_reads   one thread per record: the reference's per-read rule
//                   (depth_record.cuh) and the sum into the record's contig.
//                   Records arrive sorted by contig, so a warp's records fall
//                   into a few contigs: lanes with the same contig are grouped
//                   (match_any), their bases summed in the warp, and one 64-bit
//                   atomic per group goes to HBM.
//   k_depth_means   one thread per (kept contig, column): the mean of
//                   src/rabbit_depth.cpp:1515-1534 (sum / (length - 2 edge)
//                   when the contig is longer than 2 edge + 1, values above
//                   1e6 clamped to 0).
#include <cuda_runtime.h>

#include "depth_record.cuh"
#include "rbg_internal.h"

namespace rbg {
namespace {

__global__ void __launch_bounds__(256) k_depth_reads(const uint8_t *__restrict__ buf,
                                                     const uint32_t *__restrict__ rec_off, int64_t nrec,
                                                     const uint32_t *__restrict__ target_len,
                                                     depth::Params P,
                                                     unsigned long long *__restrict__ sum,
                                                     unsigned long long *__restrict__ sum_u) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  depth::Outcome o{-1, 0u, false, false};
  if (i < nrec) {
    const uint8_t *rec = buf + rec_off[i];
    o = depth::depth_of_record(rec, depth::ld_u32(rec) + 4u, target_len, P);
  }
  const unsigned active = __ballot_sync(0xffffffffu, o.add);
  if (!o.add) return;
  const unsigned grp = __match_any_sync(active, o.tid);
  const int lane = threadIdx.x & 31;
  const bool leader = (__ffs(grp) - 1) == lane;
  // warp sums in 32 bits: every term below 2^26 keeps a 32-lane sum exact
  const bool small = __all_sync(grp, o.bases < (1u << 26));
  if (small) {
    const unsigned s = __reduce_add_sync(grp, o.bases);
    if (leader && s) atomicAdd(sum + o.tid, (unsigned long long)s);
    if (sum_u) {
      const unsigned su = __reduce_add_sync(grp, o.uniq ? o.bases : 0u);
      if (leader && su) atomicAdd(sum_u + o.tid, (unsigned long long)su);
    }
  } else {
    if (o.bases) atomicAdd(sum + o.tid, (unsigned long long)o.bases);
    if (sum_u && o.uniq && o.bases) atomicAdd(sum_u + o.tid, (unsigned long long)o.bases);
  }
}

// sums: [ncols][n_targets]; edge_of_col: the edge of each column's sample
__global__ void k_depth_means(const unsigned long long *__restrict__ sums, int64_t n_targets,
                              const int32_t *__restrict__ kept_tid, int64_t n_kept,
                              const uint32_t *__restrict__ target_len,
                              const int32_t *__restrict__ edge_of_col, int ncols,
                              float *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_kept * ncols) return;
  const int64_t row = i / ncols;
  const int col = (int)(i - row * ncols);
  const int32_t t = kept_tid[row];
  const int32_t edge = edge_of_col[col];
  const int32_t cl = (int32_t)target_len[t];
  const int32_t adj = (cl > 2 * edge + 1) ? (cl - 2 * edge) : cl;
  float m = adj > 2 ? (float)((double)sums[(int64_t)col * n_targets + t] / (double)adj) : 0.0f;
  if (m > 1000000.0f) m = 0.0f;
  out[i] = m;
}

}  // namespace

void launch_depth_reads(const uint8_t *buf, const uint32_t *rec_off, int64_t nrec,
                        const uint32_t *target_len, const depth::Params &P, unsigned long long *sum,
                        unsigned long long *sum_u, cudaStream_t s) {
  if (nrec <= 0) return;
  k_depth_reads<<<(unsigned)((nrec + 255) / 256), 256, 0, s>>>(buf, rec_off, nrec, target_len, P,
                                                              sum, sum_u);
}

void launch_depth_means(const unsigned long long *sums, int64_t n_targets, const int32_t *kept_tid,
                        int64_t n_kept, const uint32_t *target_len, const int32_t *edge_of_col,
                        int ncols, float *out, cudaStream_t s) {
  const int64_t tot = n_kept * ncols;
  if (tot <= 0) return;
  k_depth_means<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(sums, n_targets, kept_tid, n_kept,
                                                              target_len, edge_of_col, ncols, out);
}

}  // namespace rbg
