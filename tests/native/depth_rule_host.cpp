// Test harness: the library's per-record depth rule (rabbitbin_b200/csrc/
// depth_record.cuh, the code the device kernel runs) compiled for the host,
// so the CPU test suite can compare it with the reference's own code without a
// GPU.  Not part of the library.
#include <cstdint>
#include <cstring>

#include "../../rabbitbin_b200/csrc/depth_record.cuh"

extern "C" int host_depth_rule(const uint8_t *recs, int64_t nbytes, const uint32_t *tlen,
                               int32_t nt, float pctid, int max_edge, int include_edge,
                               int min_mapq, int dual_q, uint64_t *sum, uint64_t *sum_u,
                               int32_t *avg_read) {
  using namespace rbg::depth;
  int64_t srs = 0, src = 0;
  for (int64_t o = 0; o < nbytes && src < 4000;) {
    const uint32_t rb = record_bytes(recs + o, (uint64_t)(nbytes - o));
    if (!rb) return -1;
    if (!(ld_u16(recs + o + 18) & kUnmap)) {
      srs += ld_i32(recs + o + 20);
      ++src;
    }
    o += rb;
  }
  *avg_read = src ? (int32_t)(srs / src) : 0;
  Params P{pctid, include_edge ? 0 : (max_edge < *avg_read / 3 ? max_edge : *avg_read / 3),
           min_mapq, dual_q, nt};
  std::memset(sum, 0, sizeof(uint64_t) * (size_t)nt);
  std::memset(sum_u, 0, sizeof(uint64_t) * (size_t)nt);
  for (int64_t o = 0; o < nbytes;) {
    const uint32_t rb = record_bytes(recs + o, (uint64_t)(nbytes - o));
    if (!rb) return -1;
    const Outcome r = depth_of_record(recs + o, rb, tlen, P);
    if (r.add) {
      sum[r.tid] += r.bases;
      if (r.uniq) sum_u[r.tid] += r.bases;
    }
    o += rb;
  }
  return 0;
}
