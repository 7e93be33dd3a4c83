// Reference harness for the BAM -> depth summariser (test infrastructure only).
//
// Compiles the reference's own per-read depth code, cut out of the reference
// tree at build time into oracle/_ref/frag/ (nothing of it is committed):
//   src/BamUtils.h:275-318          BamNameTrackingChooser, warnMalformedBamRead,
//                                   expectMalformedBamInvariant
//   src/CheckRead.hpp:20-276        CheckRead (checkEnd, fixEndClip)
//   src/rabbit_depth.h:48-66        ThreadBlocker
//   src/rabbit_depth.h:70-162       DepthCounts
//   src/rabbit_depth.h:181-376      ReadStatistics
//   src/rabbit_depth.h:601-887      calcMismatches, caldepth
//   src/rabbit_depth_fuse.h:65-68   DepthColumn
//   src/rabbit_depth.cpp:1615-1685  depth_accumulate_sample
// against oracle/htslib_shim.h in place of htslib.  ref_depth_accumulate()
// decodes raw BAM records (block_size, fixed fields, variable part) into
// bam1_t the way htslib lays them out and runs depth_accumulate_sample on them.
#include <unistd.h>

#include "htslib_shim.h"

typedef uint64_t CountType;
typedef uint32_t ContigIdxType;

#include "frag_bam_chooser.inc"
#include "frag_checkread.inc"
#include "frag_thread_blocker.inc"
ThreadBlocker tb;
#include "frag_depth_counts.inc"
#include "frag_read_stats.inc"
#include "frag_caldepth.inc"
#include "frag_depth_column.inc"
#include "frag_depth_accumulate.inc"

extern "C" int ref_depth_accumulate(const uint8_t *recs, int64_t nbytes, const uint32_t *tlen,
                                    int32_t nt, float pctid, int max_edge, int include_edge,
                                    int min_mapq, int threads, uint64_t *depth_out,
                                    int32_t *avg_read) {
  std::vector<bam1_t *> v;
  int64_t o = 0;
  while (nbytes - o >= 36) {
    int32_t bs;
    memcpy(&bs, recs + o, 4);
    if (bs < 32 || o + 4 + bs > nbytes) return -1;
    const uint8_t *r = recs + o + 4;
    bam1_t *b = (bam1_t *)calloc(1, sizeof(bam1_t));
    int32_t i32;
    memcpy(&i32, r + 0, 4); b->core.tid = i32;
    memcpy(&i32, r + 4, 4); b->core.pos = i32;
    const uint8_t l_rn = r[8];
    b->core.qual = r[9];
    uint16_t u16;
    memcpy(&u16, r + 10, 2); b->core.bin = u16;
    memcpy(&u16, r + 12, 2); b->core.n_cigar = u16;
    memcpy(&u16, r + 14, 2); b->core.flag = u16;
    memcpy(&i32, r + 16, 4); b->core.l_qseq = i32;
    memcpy(&i32, r + 20, 4); b->core.mtid = i32;
    memcpy(&i32, r + 24, 4); b->core.mpos = i32;
    memcpy(&i32, r + 28, 4); b->core.isize = i32;
    const int extranul = (4 - (l_rn & 3)) & 3;
    b->core.l_extranul = (uint8_t)extranul;
    b->core.l_qname = (uint16_t)(l_rn + extranul);
    b->l_data = bs - 32 + extranul;
    b->m_data = (uint32_t)b->l_data + 8;
    b->data = (uint8_t *)calloc(b->m_data, 1);
    memcpy(b->data, r + 32, l_rn);
    memcpy(b->data + l_rn + extranul, r + 32 + l_rn, (size_t)(bs - 32 - l_rn));
    v.push_back(b);
    o += 4 + bs;
  }
  if (o != nbytes) {
    for (bam1_t *b : v) { free(b->data); free(b); }
    return -1;
  }
  std::vector<uint32_t> tl(tlen, tlen + nt);
  std::vector<std::string> nm(nt);
  std::vector<char *> np(nt);
  for (int32_t t = 0; t < nt; ++t) {
    nm[t] = "t" + std::to_string(t);
    np[t] = (char *)nm[t].c_str();
  }
  sam_hdr_t h;
  memset(&h, 0, sizeof h);
  h.n_targets = nt;
  h.target_len = tl.data();
  h.target_name = np.data();
  if (threads > 0) omp_set_num_threads(threads);
  // the reference writes a warning line per clipped or malformed read to
  // std::cerr; the harness keeps them out of the test log
  std::streambuf *keep = std::cerr.rdbuf(nullptr);
  DepthColumn col = depth_accumulate_sample(v, &h, pctid, max_edge, include_edge != 0, min_mapq);
  std::cerr.rdbuf(keep);
  std::cerr.clear();
  for (int32_t t = 0; t < nt; ++t) depth_out[t] = col.depth[t];
  *avg_read = col.avgRead;
  // fixEndClip rewrites records in place and returns the same record
  for (bam1_t *b : v) { free(b->data); free(b); }
  return 0;
}
