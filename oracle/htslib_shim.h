// Minimal stand-in for the htslib declarations the reference's depth code
// uses (test infrastructure: lets oracle/ref_depth_shim.cpp compile the
// reference's own caldepth, ReadStatistics, CheckRead and
// depth_accumulate_sample without htslib, which is not in this image).
//
// The record layout and the helpers follow the SAM/BAM format specification
// and htslib's documented API: bam1_core_t / bam1_t as htslib lays a decoded
// record out in memory (read name padded with NULs to a 4-byte boundary, then
// CIGAR, 4-bit sequence, qualities, aux fields), CIGAR op codes and their
// query/reference consumption, bam_endpos (pos + reference length of the
// CIGAR, 1 when it has none), and the aux lookup of integer tags.
#pragma once
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cassert>
#include <cstdio>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

using namespace std;

typedef int64_t hts_pos_t;

typedef struct bam1_core_t {
  hts_pos_t pos;
  int32_t tid;
  uint16_t bin;
  uint8_t qual;
  uint8_t l_extranul;
  uint16_t flag;
  uint16_t l_qname;
  uint32_t n_cigar;
  int32_t l_qseq;
  int32_t mtid;
  hts_pos_t mpos;
  hts_pos_t isize;
} bam1_core_t;

typedef struct bam1_t {
  bam1_core_t core;
  uint64_t id;
  uint8_t *data;
  int l_data;
  uint32_t m_data;
  uint32_t mempolicy : 2, : 30;
} bam1_t;

typedef struct sam_hdr_t {
  int32_t n_targets, ignore_sam_err;
  size_t l_text;
  uint32_t *target_len;
  const int8_t *cigar_tab;
  char **target_name;
  char *text;
  void *sdict;
  void *hrecs;
  uint32_t ref_count;
} sam_hdr_t;
typedef sam_hdr_t bam_hdr_t;
typedef bam_hdr_t bam_header_t;
typedef shared_ptr<bam_header_t> BamHeaderT;

enum {
  BAM_FPAIRED = 1, BAM_FPROPER_PAIR = 2, BAM_FUNMAP = 4, BAM_FMUNMAP = 8, BAM_FREVERSE = 16,
  BAM_FMREVERSE = 32, BAM_FREAD1 = 64, BAM_FREAD2 = 128, BAM_FSECONDARY = 256, BAM_FQCFAIL = 512,
  BAM_FDUP = 1024, BAM_FSUPPLEMENTARY = 2048
};
enum {
  BAM_CMATCH = 0, BAM_CINS = 1, BAM_CDEL = 2, BAM_CREF_SKIP = 3, BAM_CSOFT_CLIP = 4,
  BAM_CHARD_CLIP = 5, BAM_CPAD = 6, BAM_CEQUAL = 7, BAM_CDIFF = 8, BAM_CBACK = 9
};

// bits per op (two each, ops 0..9): query-consuming, reference-consuming
static inline int shim_cigar_type(uint32_t op) { return (0x3C1A7 >> (op << 1)) & 3; }
#define bam_cigar_op(c) ((c) & 0xf)
#define bam_cigar_oplen(c) ((c) >> 4)
#define bam_cigar_type(o) shim_cigar_type((uint32_t)(o))
#define bam_cigar_gen(l, o) ((uint32_t)(l) << 4 | (uint32_t)(o))
#define bam_cigar_opchr(o) ("MIDNSHP=XB??????"[(o) & 0xf])
#define bam_get_qname(b) ((char *)(b)->data)
#define bam_get_cigar(b) ((uint32_t *)((b)->data + (b)->core.l_qname))
#define bam_get_seq(b) ((b)->data + ((b)->core.n_cigar << 2) + (b)->core.l_qname)
#define bam_get_qual(b) (bam_get_seq(b) + (((b)->core.l_qseq + 1) >> 1))
#define bam_get_aux(b) (bam_get_qual(b) + (b)->core.l_qseq)
#define bam_get_l_aux(b) ((b)->l_data - (int)(bam_get_aux(b) - (b)->data))
#define bam_seqi(s, i) ((s)[(i) >> 1] >> ((~(i) & 1) << 2) & 0xf)
#define bam1_qname(b) bam_get_qname(b)
#define bam1_cigar(b) bam_get_cigar(b)
#define bam1_seq(b) bam_get_seq(b)
#define bam1_seqi(s, i) bam_seqi(s, i)
static const char bam_nt16_rev_table[] = "=ACMGRSVTWYHKDBN";

static inline hts_pos_t bam_cigar2rlen(int n, const uint32_t *c) {
  hts_pos_t l = 0;
  for (int k = 0; k < n; ++k)
    if (bam_cigar_type(bam_cigar_op(c[k])) & 2) l += bam_cigar_oplen(c[k]);
  return l;
}
static inline hts_pos_t bam_cigar2qlen(int n, const uint32_t *c) {
  hts_pos_t l = 0;
  for (int k = 0; k < n; ++k)
    if (bam_cigar_type(bam_cigar_op(c[k])) & 1) l += bam_cigar_oplen(c[k]);
  return l;
}
#define bam1_cigar2qlen(b, c) bam_cigar2qlen((b)->core.n_cigar, (c))

static inline hts_pos_t bam_endpos(const bam1_t *b) {
  hts_pos_t rlen = (b->core.flag & BAM_FUNMAP) ? 0 : bam_cigar2rlen(b->core.n_cigar, bam_get_cigar(b));
  if (rlen == 0) rlen = 1;
  return b->core.pos + rlen;
}

// aux fields: two-character tag, type, value
static inline uint8_t *shim_aux_skip(uint8_t *s, uint8_t *end) {
  const uint8_t ty = *s++;
  switch (ty) {
    case 'A': case 'c': case 'C': return end - s >= 1 ? s + 1 : NULL;
    case 's': case 'S': return end - s >= 2 ? s + 2 : NULL;
    case 'i': case 'I': case 'f': return end - s >= 4 ? s + 4 : NULL;
    case 'd': return end - s >= 8 ? s + 8 : NULL;
    case 'Z': case 'H': {
      while (s < end && *s) ++s;
      return s < end ? s + 1 : NULL;
    }
    case 'B': {
      if (end - s < 5) return NULL;
      const uint8_t sub = *s++;
      uint32_t n;
      memcpy(&n, s, 4);
      s += 4;
      int sz = (sub == 'c' || sub == 'C') ? 1 : (sub == 's' || sub == 'S') ? 2
             : (sub == 'i' || sub == 'I' || sub == 'f') ? 4 : 0;
      if (!sz || (uint64_t)(end - s) < (uint64_t)n * sz) return NULL;
      return s + (size_t)n * sz;
    }
    default: return NULL;
  }
}
static inline uint8_t *bam_aux_get(const bam1_t *b, const char tag[2]) {
  uint8_t *s = bam_get_aux(b), *end = b->data + b->l_data;
  while (s && end - s >= 3) {
    if (s[0] == tag[0] && s[1] == tag[1]) return s + 2;
    s = shim_aux_skip(s + 2, end);
  }
  return NULL;
}
static inline int64_t bam_aux2i(const uint8_t *s) {
  const uint8_t ty = *s++;
  switch (ty) {
    case 'c': return (int8_t)s[0];
    case 'C': return s[0];
    case 's': { int16_t v; memcpy(&v, s, 2); return v; }
    case 'S': { uint16_t v; memcpy(&v, s, 2); return v; }
    case 'i': { int32_t v; memcpy(&v, s, 4); return v; }
    case 'I': { uint32_t v; memcpy(&v, s, 4); return v; }
    default: return 0;
  }
}
