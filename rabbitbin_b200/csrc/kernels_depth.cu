// BAM -> depth summariser, device side: BGZF inflation, the record walk,
// per-record depth sums and the means matrix.  Two routes feed the sums:
// the device route (k_inflate, k_walk, k_scan_counts, k_depth_reads_dev) takes
// a chunk of compressed blocks; the host route (bam.cpp inflates and walks)
// hands over decompressed records with one offset per record (k_depth_reads).
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

#include <algorithm>
#include <cstdlib>

#include "depth_record.cuh"
#include "inflate.cuh"
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

// ── device BGZF path ─────────────────────────────────────────────────────
// One warp per BGZF block inflates it into its place in the chunk's output
// (inflate.cuh: the lanes decode in lockstep and copy together; the warp's
// Huffman tables in shared memory) and checks its CRC32 (lane segments joined
// over GF(2)).  Failures set bit 0 of *flags.
template <int kMinCtas>
__global__ void __launch_bounds__(kInflateWarps * 32, kMinCtas) k_inflate(const uint8_t *__restrict__ comp,
                                                               const DevBlk *__restrict__ blk,
                                                               int nb, uint8_t *__restrict__ out,
                                                               uint32_t *__restrict__ flags) {
  __shared__ uint32_t crc_t[256];
  __shared__ inflate::Tables tabs[kInflateWarps];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    uint32_t c = (uint32_t)i;
    for (int k = 0; k < 8; ++k) c = (c & 1) ? inflate::kCrcPoly ^ (c >> 1) : c >> 1;
    crc_t[i] = c;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5;
  const inflate::WarpLanes L{(int)(threadIdx.x & 31)};
  for (int i = blockIdx.x * kInflateWarps + w; i < nb; i += gridDim.x * kInflateWarps) {
    const DevBlk b = blk[i];
    int st = inflate::inflate_block(comp + b.cofs, b.clen, out + b.uofs, b.isize, tabs[w], L);
    __syncwarp();
    if (st == inflate::kOk && inflate::crc32(crc_t, out + b.uofs, b.isize, L) != b.crc) st = 9;
    if (st != inflate::kOk && L.leader()) atomicOr(flags, 1u);
    __syncwarp();
  }
}

// Record chain of each block, assuming every block starts on a record (as
// htslib writes BGZF: a record that would not fit starts the next block):
// from the block's start (or the header's end) records are followed to the
// block's end.  A record that does not fit the chunk, or a chain that does not
// end exactly at the block's end, sets bit 1 of *flags (the file then goes
// through the host walk).  Pass 0 counts, pass 1 writes the records' offsets
// at the block's place in the scan.
__global__ void k_walk(const uint8_t *__restrict__ out, const uint64_t *__restrict__ ubound, int nb,
                       uint64_t hdr_end, uint32_t *__restrict__ counts,
                       const uint32_t *__restrict__ scan, uint32_t *__restrict__ offs,
                       uint32_t *__restrict__ flags, int pass) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const uint64_t end = ubound[nb];
  uint64_t p = ubound[i] < hdr_end ? hdr_end : ubound[i];
  const uint64_t hi = ubound[i + 1];
  uint32_t n = 0, base = pass ? scan[i] : 0;
  bool bad = false;
  while (p < hi) {
    const uint32_t rb = depth::record_bytes(out + p, end - p);
    if (!rb) {
      bad = true;
      break;
    }
    if (pass) offs[base + n] = (uint32_t)p;
    ++n;
    p += rb;
  }
  if (!pass) {
    counts[i] = n;
    const uint64_t start = ubound[i] < hdr_end ? hdr_end : ubound[i];
    if (bad || (start < hi && p != hi)) atomicOr(flags, 2u);
  }
}

// Exclusive scan of the per-block counts (one CTA); scan[nb] = total, also
// added to the file's record count.
__global__ void __launch_bounds__(1024) k_scan_counts(const uint32_t *__restrict__ counts, int nb,
                                                      uint32_t *__restrict__ scan,
                                                      unsigned long long *__restrict__ rec_total) {
  __shared__ uint32_t part[1024];
  const int per = (nb + blockDim.x - 1) / blockDim.x;
  const int a = threadIdx.x * per, b = min(nb, a + per);
  uint32_t s = 0;
  for (int i = a; i < b; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int d = 1; d < (int)blockDim.x; d <<= 1) {
    const uint32_t v = threadIdx.x >= (unsigned)d ? part[threadIdx.x - d] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
  for (int i = a; i < b; ++i) {
    scan[i] = run;
    run += counts[i];
  }
  if (threadIdx.x == blockDim.x - 1) {
    scan[nb] = part[threadIdx.x];
    atomicAdd(rec_total, (unsigned long long)part[threadIdx.x]);
  }
}

// The per-record rule over the chunk's walked records (count on the device);
// nothing is added when the chunk's chain did not hold.
__global__ void __launch_bounds__(256) k_depth_reads_dev(const uint8_t *__restrict__ buf,
                                                         const uint32_t *__restrict__ rec_off,
                                                         const uint32_t *__restrict__ nrec_p,
                                                         const uint32_t *__restrict__ flags,
                                                         const uint32_t *__restrict__ target_len,
                                                         depth::Params P,
                                                         unsigned long long *__restrict__ sum,
                                                         unsigned long long *__restrict__ sum_u) {
  if (*flags & 3u) return;
  const uint32_t nrec = *nrec_p;
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < nrec; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    depth::Outcome o{-1, 0u, false, false};
    if (i < nrec) {
      const uint8_t *rec = buf + rec_off[i];
      o = depth::depth_of_record(rec, depth::ld_u32(rec) + 4u, target_len, P);
    }
    const unsigned active = __ballot_sync(0xffffffffu, o.add);
    if (!o.add) continue;
    const unsigned grp = __match_any_sync(active, o.tid);
    const int lane = threadIdx.x & 31;
    const bool leader = (__ffs(grp) - 1) == lane;
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

void launch_depth_device(const uint8_t *comp, const DevBlk *blk, int nb, const uint64_t *ubound,
                         uint64_t hdr_end, uint8_t *out, uint32_t *counts, uint32_t *scan,
                         uint32_t *offs, uint32_t *flags, unsigned long long *rec_total,
                         const uint32_t *target_len, const depth::Params &P,
                         unsigned long long *sum, unsigned long long *sum_u, int sms,
                         cudaStream_t s) {
  if (nb <= 0) return;
  // four CTAs per SM (64 registers, a few spilled: 40 ms against 46 ms for the
  // 80-register build on the 5.6 M-read benchmark BAM); RBG_INFLATE_CTAS=3
  // takes the 80-register build
  static const int per_sm = [] {
    const char *e = getenv("RBG_INFLATE_CTAS");
    return (e && atoi(e) == 3) ? 3 : 4;
  }();
  const int ctas = std::min((nb + kInflateWarps - 1) / kInflateWarps, sms * per_sm);
  if (per_sm == 4)
    k_inflate<4><<<ctas, kInflateWarps * 32, 0, s>>>(comp, blk, nb, out, flags);
  else
    k_inflate<3><<<ctas, kInflateWarps * 32, 0, s>>>(comp, blk, nb, out, flags);
  const unsigned g = (unsigned)((nb + 127) / 128);
  k_walk<<<g, 128, 0, s>>>(out, ubound, nb, hdr_end, counts, scan, offs, flags, 0);
  k_scan_counts<<<1, 1024, 0, s>>>(counts, nb, scan, rec_total);
  k_walk<<<g, 128, 0, s>>>(out, ubound, nb, hdr_end, counts, scan, offs, flags, 1);
  k_depth_reads_dev<<<(unsigned)(sms * 8), 256, 0, s>>>(out, offs, scan + nb, flags, target_len, P,
                                                        sum, sum_u);
}

}  // namespace rbg
