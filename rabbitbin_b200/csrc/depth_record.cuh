// Per-record depth rule of the BAM -> depth summariser (host and device).
//
// One BAM record (as stored in the decompressed stream: block_size, the 32-byte
// fixed part, read name, CIGAR, sequence, qualities, aux fields) is turned into
// the number of bases it adds to its contig's depth sum, or rejected.  The rule
// is the reference's per-read path of the fused depth pass:
//
//   filters            src/rabbit_depth.cpp:1656-1667 (depth_accumulate_sample)
//                      and :679-693 (process_depth_shard); BAM_FSECONDARY |
//                      BAM_FQCFAIL | BAM_FDUP from src/BamUtils.h:281-283
//   end check / clip   src/CheckRead.hpp:82-99 (checkEnd), :101-135 and
//                      :138-265 (fixEndClip)
//   covered bases      src/rabbit_depth.h:618-887 (caldepth, ref == NULL, no
//                      per-base buffer, edge trimming)
//   read statistics    src/rabbit_depth.h:193-316 (ReadStatistics and
//                      calculateAlignment), :342-346 (getPctId)
//
// fixEndClip rewrites the record (CIGAR cut after the op that crosses the
// contig end, that op turned into a soft clip); here the rewrite is kept as a
// view: the first `n_eff` ops, op n_eff-1 replaced by `last_op`.  The integer
// types follow the reference's (uint32 counters, int lengths, wrap-around where
// it mixes them) so that malformed records are judged as it judges them.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define RBG_HD __host__ __device__ __forceinline__
#else
#define RBG_HD inline
#endif

namespace rbg {
namespace depth {

// SAM flag bits and CIGAR operations (SAM/BAM format specification).
constexpr uint32_t kPaired = 0x1, kUnmap = 0x4, kMUnmap = 0x8, kSecondary = 0x100,
                   kQcFail = 0x200, kDup = 0x400;
enum : uint32_t { kM = 0, kI = 1, kD = 2, kN = 3, kS = 4, kH = 5, kP = 6, kEq = 7, kX = 8 };

// bit 0: the op consumes query bases, bit 1: reference bases (ops 0..9; the
// rest consume neither), as the format specification's table gives them.
RBG_HD uint32_t cigar_type(uint32_t op) { return (0x3C1A7u >> (op << 1)) & 3u; }

RBG_HD uint32_t ld_u8(const uint8_t *p) { return p[0]; }
RBG_HD uint32_t ld_u16(const uint8_t *p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
RBG_HD uint32_t ld_u32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
RBG_HD int32_t ld_i32(const uint8_t *p) { return (int32_t)ld_u32(p); }

struct Params {
  float pctid;        // minimum percent identity as a fraction (97 -> 0.97f)
  int32_t edge;       // bases ignored at each contig end (0 with edges included)
  int32_t min_mapq;   // reads below this MAPQ are skipped
  int32_t dual_q;     // > 0: a second sum of reads with MAPQ >= dual_q
  int32_t n_targets;
};

// The CIGAR as the depth rule sees it: the record's ops, or the clipped view.
struct Cigar {
  const uint8_t *ops;   // little-endian uint32 ops
  uint32_t n;           // ops in the view
  uint32_t last_op;     // replaces op n-1 when `clipped`
  bool clipped;
  RBG_HD uint32_t at(uint32_t i) const {
    return (clipped && i + 1 == n) ? last_op : ld_u32(ops + 4 * (size_t)i);
  }
};

// bam_endpos of a mapped read: pos + reference length of the CIGAR (1 when it
// has none), as htslib defines it.
RBG_HD int64_t end_pos(int64_t pos, const Cigar &c) {
  int64_t rlen = 0;
  for (uint32_t i = 0; i < c.n; ++i) {
    const uint32_t v = c.at(i);
    if (cigar_type(v & 0xf) & 2) rlen += v >> 4;
  }
  if (rlen == 0) rlen = 1;
  return pos + rlen;
}

// Value of the integer aux field "NM", found by walking the aux fields between
// `a` and `end` (htslib's bam_aux_get / bam_aux2i).  Returns false when the tag
// is absent or the fields cannot be walked; a non-integer NM reads as 0.
RBG_HD bool aux_nm(const uint8_t *a, const uint8_t *end, int32_t &nm) {
  while (end - a >= 3) {
    const uint8_t t0 = a[0], t1 = a[1], ty = a[2];
    const uint8_t *v = a + 3;
    if (t0 == 'N' && t1 == 'M') {
      int64_t x = 0;
      switch (ty) {
        case 'c': if (end - v < 1) return false; x = (int8_t)v[0]; break;
        case 'C': if (end - v < 1) return false; x = v[0]; break;
        case 's': if (end - v < 2) return false; x = (int16_t)ld_u16(v); break;
        case 'S': if (end - v < 2) return false; x = ld_u16(v); break;
        case 'i': if (end - v < 4) return false; x = ld_i32(v); break;
        case 'I': if (end - v < 4) return false; x = ld_u32(v); break;
        default: x = 0; break;
      }
      nm = (int32_t)x;
      return true;
    }
    int64_t sz;
    switch (ty) {
      case 'A': case 'c': case 'C': sz = 1; break;
      case 's': case 'S': sz = 2; break;
      case 'i': case 'I': case 'f': sz = 4; break;
      case 'd': sz = 8; break;
      case 'Z': case 'H': {
        const uint8_t *q = v;
        while (q < end && *q) ++q;
        if (q >= end) return false;
        sz = (q - v) + 1;
        break;
      }
      case 'B': {
        if (end - v < 5) return false;
        const uint8_t sub = v[0];
        const int64_t cnt = ld_u32(v + 1);
        int64_t es;
        switch (sub) {
          case 'c': case 'C': es = 1; break;
          case 's': case 'S': es = 2; break;
          case 'i': case 'I': case 'f': es = 4; break;
          default: return false;
        }
        sz = 5 + cnt * es;
        break;
      }
      default: return false;
    }
    if (end - v < sz) return false;
    a = v + sz;
  }
  return false;
}

// Result of one record.
struct Outcome {
  int32_t tid;        // contig (valid when `add`)
  uint32_t bases;     // covered bases after edge trimming and substitutions
  bool add;           // the read passes every filter and the percent identity
  bool uniq;          // and has MAPQ >= dual_q (dual sums only)
};

// `rec` points at the record's block_size field; `rec_bytes` = 4 + block_size
// (checked by the caller to lie inside the stream and to hold the fixed part,
// the read name, the CIGAR and the sequence and quality bytes).
RBG_HD Outcome depth_of_record(const uint8_t *rec, uint32_t rec_bytes, const uint32_t *target_len,
                               const Params &P) {
  Outcome o{-1, 0, false, false};
  const int32_t tid = ld_i32(rec + 4);
  const int64_t pos = ld_i32(rec + 8);
  const uint32_t l_qname = ld_u8(rec + 12);
  const uint32_t mapq = ld_u8(rec + 13);
  const uint32_t n_cigar = ld_u16(rec + 16);
  const uint32_t flag = ld_u16(rec + 18);
  const int32_t l_qseq = ld_i32(rec + 20);
  const int32_t mtid = ld_i32(rec + 24);
  const uint8_t *data = rec + 36;                   // read name first
  const uint8_t *rec_end = rec + rec_bytes;
  // the unmapped tail of a sorted file (and any tid < 0) adds nothing
  if (tid < 0) return o;
  if ((flag & kUnmap) == 0 && (tid >= P.n_targets || pos < 0)) return o;
  if ((flag & (kPaired | kMUnmap)) == kPaired && (mtid < 0 || mtid >= P.n_targets)) return o;
  if (flag & (kSecondary | kQcFail | kDup)) return o;
  if ((flag & kUnmap) || (int32_t)mapq < P.min_mapq) return o;
  const uint32_t refLen = target_len[tid];
  Cigar cg{data + l_qname, n_cigar, 0u, false};
  const uint32_t seq_bytes = (uint32_t)((l_qseq + 1) / 2), qual_bytes = (uint32_t)l_qseq;
  const uint8_t *aux = cg.ops + 4 * (size_t)n_cigar + seq_bytes + qual_bytes;

  // checkEnd, then fixEndClip and checkEnd again (CheckRead.hpp:82-265)
  if (refLen > 0 && (uint32_t)end_pos(pos, cg) > refLen) {
    if ((uint32_t)pos >= refLen || pos < 0) return o;     // left as is: fails again
    uint32_t seqpos = 0, refpos = (uint32_t)pos;
    bool cut = false;
    for (uint32_t i = 0; i < n_cigar; ++i) {
      const uint32_t v = cg.at(i), op = v & 0xf, oplen = v >> 4, ty = cigar_type(op);
      if (ty & 1) seqpos += oplen;
      if (ty & 2) refpos += oplen;
      if (refpos > refLen) {
        // remainder after the CIGAR must be non-empty, and the CIGAR must shrink
        const int64_t remainder = (int64_t)rec_bytes - 36 - l_qname - 4 * (int64_t)n_cigar;
        if (remainder <= 0 || i + 1 == n_cigar) return o;
        const uint32_t pre = (ty & 1) ? seqpos - oplen : seqpos;
        if (pre > (uint32_t)l_qseq) return o;    // ops cut, this op kept: still past the end
        cg.n = i + 1;
        cg.clipped = true;
        cg.last_op = (((uint32_t)l_qseq - pre) << 4) | kS;
        cut = true;
        break;
      }
    }
    if (!cut) return o;
    if ((uint32_t)end_pos(pos, cg) > refLen) return o;
  }

  // caldepth (rabbit_depth.h:618-887), ref == NULL, ignoreEdges = P.edge
  const int32_t refLenI = (int32_t)refLen;
  uint32_t refpos = (uint32_t)pos;
  if (refpos >= (uint32_t)refLenI && refLenI > 0) return o;
  int32_t len = 0;
  uint32_t ins = 0, del = 0, seqpos = 0, mism = 0, exact = 0, soft = 0, hard = 0, skip = 0;
  uint32_t cmatches = 0;
  bool isCEQUAL = false;
  const int32_t E = P.edge;
  for (uint32_t i = 0; i < cg.n; ++i) {
    const uint32_t v = cg.at(i), op = v & 0xf, ty = cigar_type(op);
    const int32_t oplen = (int32_t)(v >> 4);
    int32_t mmOp = 0;
    if (op == kM || op == kX || op == kEq) {
      if (op == kM) cmatches += oplen;
      if (op == kX) {
        isCEQUAL = true;
        mmOp = oplen;
        mism += oplen;
      }
      if (op == kEq) isCEQUAL = true;
      exact += oplen - mmOp;
      len += oplen;
      if (E > 0 && refLenI > 2 * E) {
        if ((int32_t)refpos < E) {
          const int32_t d = (int32_t)((uint32_t)E - refpos);
          len -= d < oplen ? d : oplen;
        }
        if (refLenI > 0 && (refpos + (uint32_t)oplen) > ((uint32_t)refLenI - (uint32_t)E)) {
          if (refpos + (uint32_t)oplen > (uint32_t)refLenI) return o;
          const int32_t d = (int32_t)(refpos + (uint32_t)oplen) - (refLenI - E);
          len -= d < oplen ? d : oplen;
        }
      }
    } else if (op == kI) {
      ins += oplen;
    } else if (op == kD) {
      del += oplen;
    } else if (op == kN) {
      skip += oplen;
    } else if (op == kS) {
      soft += oplen;
    } else if (op == kH) {
      hard += oplen;
    }
    if (ty & 1) seqpos += oplen;
    if (ty & 2) refpos += oplen;
  }
  (void)hard;
  (void)seqpos;
  int32_t nm_tag = 0;
  uint32_t nm;                            // the statistics' NM (uint32 as they hold it)
  if (aux_nm(aux, rec_end, nm_tag)) {
    int32_t nmv = nm_tag;
    if (nmv < (int32_t)(ins + del)) nmv = (int32_t)(ins + del + mism);
    if (isCEQUAL) {
      if (cmatches > 0 && nmv != (int32_t)(ins + del + mism)) {
        if (nmv == (int32_t)(ins + del + mism + cmatches)) {
          mism += cmatches;
          exact -= cmatches;
        } else {
          const int32_t newmm = (int32_t)((uint32_t)nmv - (ins + del));
          int64_t adj = (int64_t)exact - ((int64_t)newmm - (int64_t)mism);
          if (adj < 0) adj = 0;
          exact = (uint32_t)adj;
          mism = (uint32_t)newmm;
        }
      }
    } else {
      const int32_t newmm = (int32_t)((uint32_t)nmv - (ins + del));
      int64_t adj = (int64_t)exact - ((int64_t)newmm - (int64_t)mism);
      if (adj < 0) adj = 0;
      exact = (uint32_t)adj;
      mism = (uint32_t)newmm;
    }
    if (nmv != (int32_t)(ins + del + mism)) nmv = (int32_t)(ins + del + mism);
    const int32_t subs = (int32_t)((uint32_t)nmv - (ins + del));
    if (subs != (int32_t)mism) mism = (uint32_t)subs;
    if (subs > len) len = 0;
    else if (subs > 0) len -= subs;
    nm = (uint32_t)nmv;
  } else {
    nm = mism + ins + del;
  }

  // ReadStatistics: calculateAlignment and the consistency checks
  const uint32_t seqlen = (uint32_t)l_qseq;
  uint32_t astart = 0, aend = 0, sstart = 0, send = 0, alen = 0;
  if (cg.n > 0) {
    astart = (uint32_t)pos;
    aend = (uint32_t)end_pos(pos, cg);
    send = (uint32_t)l_qseq;
    const uint32_t v0 = cg.at(0), op0 = v0 & 0xf, len0 = v0 >> 4, ty0 = cigar_type(op0);
    if (!(ty0 & 1) && (ty0 & 2) && ((op0 & kD) != kD)) astart += len0;
    if ((ty0 & 1) && !(ty0 & 2) && ((op0 & kI) != kI)) sstart += len0;
    bool ok = true;
    if (cg.n > 1) {
      const uint32_t vl = cg.at(cg.n - 1), lenl = vl >> 4, tyl = cigar_type(vl & 0xf);
      if ((tyl & 1) && !(tyl & 2)) {
        if (lenl > send) ok = false;
        else send -= lenl;
      }
    }
    if (ok) {
      alen = aend - astart;
      if (alen != 0 && !((send == 0 && sstart == 0) || send > sstart)) alen = 0;
    }
  }
  bool valid = true;
  if (nm != mism + ins + del) valid = false;
  if (seqlen != 0 && seqlen != exact + mism + ins + soft) valid = false;
  if (alen != aend - astart) valid = false;
  if (alen - skip != exact + mism + del) valid = false;
  if (seqlen != 0 && ins - del + soft != seqlen - (alen - skip)) valid = false;
  if (seqlen != 0 && seqlen < send - sstart) valid = false;
  if (alen == 0) valid = false;                      // the read is mapped here
  if (!valid) return o;
  const uint32_t denom = exact + mism + ins + del;
  const float pid = denom > 0 ? (float)exact / (float)denom : 0.0f;
  if (!(pid >= P.pctid)) return o;
  o.tid = tid;
  o.bases = len < 0 ? 0u : (uint32_t)len;
  o.add = true;
  o.uniq = P.dual_q > 0 && (int32_t)mapq >= P.dual_q;
  return o;
}

// Checks a record's sizes against the stream: the record must hold its fixed
// part, read name (>= 1 byte), CIGAR, sequence and qualities.  Returns the
// record's length (4 + block_size) or 0 when it does not fit or is malformed.
RBG_HD uint32_t record_bytes(const uint8_t *rec, uint64_t avail) {
  if (avail < 36) return 0;
  const int32_t bs = ld_i32(rec);
  if (bs < 32 || (uint64_t)bs + 4 > avail) return 0;
  const uint32_t l_qname = ld_u8(rec + 12), n_cigar = ld_u16(rec + 16);
  const int32_t l_qseq = ld_i32(rec + 20);
  if (l_qname < 1 || l_qseq < 0) return 0;
  const uint64_t need = 32ull + l_qname + 4ull * n_cigar + (uint64_t)((l_qseq + 1) / 2) +
                        (uint64_t)l_qseq;
  if (need > (uint64_t)bs) return 0;
  return (uint32_t)bs + 4;
}

}  // namespace depth
}  // namespace rbg
