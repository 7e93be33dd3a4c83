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
//   src/rabbit_depth.h:164-176      VarianceType
//   src/rabbit_depth.cpp:114-123    get_basename
//   src/rabbit_depth.cpp:125-313    printDepthTableHeader, ContigDepth, printDepthTable
// against oracle/htslib_shim.h in place of htslib.  ref_depth_accumulate()
// decodes raw BAM records (block_size, fixed fields, variable part) into
// bam1_t the way htslib lays them out and runs depth_accumulate_sample on them.
#include <climits>
#include <unistd.h>

#include <charconv>

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
#include "frag_variance_type.inc"
typedef vector<std::shared_ptr<CountType[]>> CountTypeMatrix;
#include "frag_depth_basename.inc"
#include "frag_depth_table.inc"

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

// The depth table of compute_depth_tsv_inmem's TSV output
// (src/rabbit_depth.cpp:1474-1486 for the variance means, :1589-1593 for the
// call) from per-BAM sums and read lengths.  names / bam_names: NUL-separated.
extern "C" int ref_depth_tsv(const uint64_t *sums, const int32_t *avg, int32_t nb,
                             const uint32_t *tlen, const char *names, int32_t nt,
                             const char *bam_names, int variance, int include_edge, int max_edge,
                             int min_contig_len, float min_contig_depth, char **out,
                             int64_t *out_len) {
  std::vector<std::string> tn(nt), bn(nb);
  for (int32_t t = 0; t < nt; ++t) {
    tn[t] = names;
    names += tn[t].size() + 1;
  }
  for (int32_t b = 0; b < nb; ++b) {
    bn[b] = bam_names;
    bam_names += bn[b].size() + 1;
  }
  std::vector<char *> np(nt);
  for (int32_t t = 0; t < nt; ++t) np[t] = (char *)tn[t].c_str();
  std::vector<uint32_t> tl(tlen, tlen + nt);
  sam_hdr_t h;
  memset(&h, 0, sizeof h);
  h.n_targets = nt;
  h.target_len = tl.data();
  h.target_name = np.data();
  CountTypeMatrix depths(nb);
  VarianceTypeMatrix vars(nb);
  std::vector<int> avgv(nb);
  int minAvgRead = INT_MAX;
  for (int32_t b = 0; b < nb; ++b) {
    depths[b].reset(new CountType[nt > 0 ? nt : 1]());
    for (int32_t t = 0; t < nt; ++t) depths[b][t] = sums[(size_t)b * nt + t];
    avgv[b] = avg[b];
    if (minAvgRead > avgv[b]) minAvgRead = avgv[b];
    if (variance) {
      vars[b].assign(nt, VarianceType());
      const int edge = include_edge ? 0 : std::min(max_edge, avgv[b] / 3);
      for (int32_t t = 0; t < nt; ++t) {
        int32_t cl = tl[t];
        int32_t adj = (cl > 2 * edge + 1) ? (cl - 2 * edge) : cl;
        vars[b][t].mean = (adj > 2) ? (float)((double)depths[b][t] / adj) : 0.0f;
        vars[b][t].variance = 0.0f;
      }
    }
  }
  BoolVector lenPass(nt, false), depthPass(nt, true);
  for (int32_t t = 0; t < nt; ++t) lenPass[t] = ((int)tl[t] >= min_contig_len);
  std::ostringstream o;
  std::streambuf *keep = std::cerr.rdbuf(nullptr);
  printDepthTable(o, bn, variance != 0, depths, avgv, 0.97f, vars, &h, lenPass, depthPass,
                  min_contig_depth, include_edge != 0, std::min(max_edge, minAvgRead / 3));
  std::cerr.rdbuf(keep);
  std::cerr.clear();
  const std::string r = o.str();
  *out = (char *)malloc(r.size() + 1);
  memcpy(*out, r.c_str(), r.size() + 1);
  *out_len = (int64_t)r.size();
  return 0;
}

extern "C" void ref_free(void *p) { free(p); }
