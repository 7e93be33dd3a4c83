/* Seeded synthetic BAM files for the depth summariser's tests and benchmark.
 *
 * Reads are drawn per contig (count from the contig's mean depth, positions
 * uniform and sorted, so the file is coordinate-sorted), with the variety the
 * depth rule has to judge: soft clips, insertions and deletions, '='/'X' and
 * mixed 'M'/'=' CIGARs, NM tags of every integer type (or none), mismatch
 * rates around the 97% identity cut, reads that run past the contig end,
 * secondary / duplicate / QC-fail / unmapped reads, mates on unknown contigs,
 * low MAPQ, extra aux fields before NM, and a tail of unplaced reads.  The
 * stream is cut into BGZF blocks the way htslib writes them (a record starts a
 * new block when it would not fit) or, with `straddle`, at fixed sizes so
 * records cross block boundaries; blocks are deflated in parallel. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

typedef struct synth_bam_opts {
  uint64_t seed;
  int32_t read_len;
  int32_t level;          /* deflate level */
  int32_t straddle;       /* 1: fixed 65280-byte payloads, records cross blocks */
  int32_t n_unmapped_tail;
  double p_indel, p_soft, p_overhang, p_secondary, p_dup, p_qcfail, p_unmapped, p_badmate;
  double p_nonm, p_lowq, p_eqx, p_mixed, p_nm_off, err_mean;
} synth_bam_opts;

static inline uint64_t sm64(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static inline double u01(uint64_t *s) { return (double)(sm64(s) >> 11) * (1.0 / 9007199254740992.0); }
static inline uint32_t below(uint64_t *s, uint32_t n) { return n ? (uint32_t)(sm64(s) % n) : 0; }

typedef struct {
  uint8_t *p;
  size_t n, cap;
} buf_t;

static void put(buf_t *b, const void *src, size_t n) {
  if (b->n + n > b->cap) {
    size_t c = b->cap ? b->cap * 2 : 4096;
    while (c < b->n + n) c *= 2;
    b->p = (uint8_t *)realloc(b->p, c);
    b->cap = c;
  }
  memcpy(b->p + b->n, src, n);
  b->n += n;
}
static void put32(buf_t *b, uint32_t v) { put(b, &v, 4); }
static void put16(buf_t *b, uint16_t v) { put(b, &v, 2); }
static void put8(buf_t *b, uint8_t v) { put(b, &v, 1); }

static int cmp_i32(const void *a, const void *b) {
  const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

static const uint8_t nt16[256] = {
    ['A'] = 1, ['C'] = 2, ['G'] = 4, ['T'] = 8, ['a'] = 1, ['c'] = 2, ['g'] = 4, ['t'] = 8};

/* One record: fixed fields, name, CIGAR, sequence, qualities, aux. */
static void emit(buf_t *b, int32_t tid, int32_t pos, uint8_t mapq, uint16_t flag, int32_t mtid,
                 int32_t mpos, int64_t rid, const uint32_t *cig, int ncig, int32_t lseq,
                 const char *ref, int64_t reflen, uint64_t *s, int nm, int nm_type, int extra_aux) {
  char name[32];
  const int ln = snprintf(name, sizeof name, "r%lld", (long long)rid) + 1;
  const size_t at = b->n;
  put32(b, 0); /* block_size, set below */
  put32(b, (uint32_t)tid);
  put32(b, (uint32_t)pos);
  put8(b, (uint8_t)ln);
  put8(b, mapq);
  put16(b, 4680);
  put16(b, (uint16_t)ncig);
  put16(b, flag);
  put32(b, (uint32_t)lseq);
  put32(b, (uint32_t)mtid);
  put32(b, (uint32_t)mpos);
  put32(b, 0);
  put(b, name, (size_t)ln);
  for (int i = 0; i < ncig; ++i) put32(b, cig[i]);
  for (int i = 0; i < (lseq + 1) / 2; ++i) {
    uint8_t hi = 15, lo = 15;
    const int64_t r0 = (int64_t)pos + 2 * i, r1 = r0 + 1;
    if (ref && r0 >= 0 && r0 < reflen) hi = nt16[(uint8_t)ref[r0]] ? nt16[(uint8_t)ref[r0]] : 15;
    else hi = (uint8_t)(1u << below(s, 4));
    if (2 * i + 1 < lseq) {
      if (ref && r1 >= 0 && r1 < reflen) lo = nt16[(uint8_t)ref[r1]] ? nt16[(uint8_t)ref[r1]] : 15;
      else lo = (uint8_t)(1u << below(s, 4));
    } else {
      lo = 0;
    }
    put8(b, (uint8_t)(hi << 4 | lo));
  }
  for (int i = 0; i < lseq;) {
    const uint32_t r = below(s, 100);
    const uint8_t q = r < 85 ? 37 : (r < 93 ? 23 : (r < 98 ? 12 : 2));
    int run = 1 + (int)below(s, 24);
    for (; run > 0 && i < lseq; --run, ++i) put8(b, q);
  }
  if (extra_aux & 1) { /* AS:C */
    put(b, "ASC", 3);
    put8(b, (uint8_t)below(s, 200));
  }
  if (extra_aux & 2) { /* XB:B:C,3 values and RG:Z */
    put(b, "XBBC", 4);
    put32(b, 3);
    put8(b, 1), put8(b, 2), put8(b, 3);
    put(b, "RGZgrp1", 7);
    put8(b, 0);
  }
  if (nm >= 0) {
    switch (nm_type) {
      case 0: put(b, "NMC", 3); put8(b, (uint8_t)(nm > 255 ? 255 : nm)); break;
      case 1: put(b, "NMc", 3); put8(b, (uint8_t)(int8_t)(nm > 127 ? 127 : nm)); break;
      case 2: put(b, "NMs", 3); put16(b, (uint16_t)nm); break;
      case 3: put(b, "NMS", 3); put16(b, (uint16_t)nm); break;
      case 4: put(b, "NMI", 3); put32(b, (uint32_t)nm); break;
      default: put(b, "NMi", 3); put32(b, (uint32_t)nm); break;
    }
  }
  if (extra_aux & 4) { /* XS:i after NM */
    put(b, "XSi", 3);
    put32(b, 7);
  }
  const uint32_t bs = (uint32_t)(b->n - at - 4);
  memcpy(b->p + at, &bs, 4);
}

/* Reads of one contig appended to b. */
static void contig_reads(const synth_bam_opts *o, int32_t tid, int32_t n_targets, uint32_t len,
                         float depth, const char *ref, uint64_t seed, int64_t *rid, buf_t *b) {
  uint64_t s = seed;
  const int L = o->read_len;
  const double lam = (double)depth * (double)len / (double)L;
  int64_t n = (int64_t)(lam + (u01(&s) - 0.5) * 2.0 * (lam > 4 ? 2.0 * __builtin_sqrt(lam) : 1.0));
  if (n < 0) n = 0;
  if (len == 0) n = 0;
  int32_t *pos = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t span = len > (uint32_t)L ? len - (uint32_t)L + 1 : 1;
    uint32_t p = below(&s, span);
    if (u01(&s) < o->p_overhang && len > 2) p = len - 1 - below(&s, (uint32_t)(L < (int)len ? L : (int)len - 1));
    pos[i] = (int32_t)p;
  }
  qsort(pos, (size_t)n, sizeof(int32_t), cmp_i32);
  for (int64_t i = 0; i < n; ++i) {
    uint32_t cig[16];
    int nc = 0;
    int q = L, ins = 0, del = 0, mm = 0;
    const int soft = u01(&s) < o->p_soft ? 1 + (int)below(&s, 20) : 0;
    const int soft_end = u01(&s) < o->p_soft * 0.5 ? 1 + (int)below(&s, 10) : 0;
    if (soft) cig[nc++] = (uint32_t)soft << 4 | 4;
    q -= soft + soft_end;
    const double e = -o->err_mean * __builtin_log(1.0 - u01(&s) + 1e-300);
    mm = (int)(e * q + 0.5);
    if (mm > q / 2) mm = q / 2;
    const int eqx = u01(&s) < o->p_eqx, mixed = !eqx && u01(&s) < o->p_mixed;
    int a = q, c = 0, k = 0, kind = 0; /* a M, kind I/D k, c M */
    if (u01(&s) < o->p_indel && q > 20) {
      kind = 1 + (int)below(&s, 2);
      k = 1 + (int)below(&s, 6);
      a = 5 + (int)below(&s, (uint32_t)(q - 15));
      c = kind == 1 ? q - a - k : q - a;
      if (c < 1) c = 1, a = q - k - 1;
      if (kind == 1) ins = k;
      else del = k;
    }
    if (eqx) {
      /* a bases as '=' runs with the mismatches as one 'X' run in the middle */
      int x = mm < a - 2 ? mm : 0;
      int left = (a - x) / 2, right = a - x - left;
      if (left) cig[nc++] = (uint32_t)left << 4 | 7;
      if (x) cig[nc++] = (uint32_t)x << 4 | 8;
      if (right) cig[nc++] = (uint32_t)right << 4 | 7;
      mm = x;
    } else if (mixed) {
      const int h = a / 2;
      cig[nc++] = (uint32_t)h << 4 | 0;
      cig[nc++] = (uint32_t)(a - h) << 4 | 7;
    } else {
      cig[nc++] = (uint32_t)a << 4 | 0;
    }
    if (kind) {
      cig[nc++] = (uint32_t)k << 4 | (kind == 1 ? 1 : 2);
      cig[nc++] = (uint32_t)c << 4 | (eqx ? 7 : 0);
    }
    if (soft_end) cig[nc++] = (uint32_t)soft_end << 4 | 4;
    int nm = mm + ins + del;
    if (u01(&s) < o->p_nm_off) nm += 1 + (int)below(&s, 3);
    if (u01(&s) < o->p_nonm) nm = -1;
    uint16_t flag = 0x1 | ((i & 1) ? 0x80 : 0x40) | (u01(&s) < 0.5 ? 0x10 : 0);
    int32_t mtid = tid, mpos = pos[i] + 200;
    if (u01(&s) < o->p_badmate) {
      const uint32_t r = below(&s, 3);
      if (r == 0) mtid = n_targets;
      else if (r == 1) mtid = -1;
      else flag |= 0x8;
    }
    if (u01(&s) < o->p_secondary) flag |= 0x100;
    if (u01(&s) < o->p_dup) flag |= 0x400;
    if (u01(&s) < o->p_qcfail) flag |= 0x200;
    uint8_t mapq = u01(&s) < o->p_lowq ? (uint8_t)below(&s, 30) : 60;
    const int unm = u01(&s) < o->p_unmapped;
    if (unm) {
      flag |= 0x4;
      nc = 0;
      mapq = 0;
    }
    const int nm_type = (int)below(&s, 6);
    const int extra = (int)below(&s, 8);
    emit(b, tid, pos[i], mapq, flag, mtid, mpos, (*rid)++, cig, nc, L, ref, (int64_t)len, &s, unm ? -1 : nm,
         nm_type, extra);
  }
  free(pos);
}

static void bgzf_block(const uint8_t *src, uint32_t n, int level, buf_t *out) {
  uLongf cap = compressBound(n) + 64;
  uint8_t *tmp = (uint8_t *)malloc(cap + 26);
  z_stream z;
  memset(&z, 0, sizeof z);
  deflateInit2(&z, level, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY);
  z.next_in = (Bytef *)src;
  z.avail_in = n;
  z.next_out = tmp + 18;
  z.avail_out = (uInt)cap;
  deflate(&z, Z_FINISH);
  const uint32_t clen = (uint32_t)z.total_out;
  deflateEnd(&z);
  const uint32_t bsize = 18 + clen + 8;
  static const uint8_t hdr[16] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 'B', 'C', 2, 0};
  memcpy(tmp, hdr, 16);
  const uint16_t bs1 = (uint16_t)(bsize - 1);
  memcpy(tmp + 16, &bs1, 2);
  const uint32_t crc = (uint32_t)crc32(0L, src, n);
  memcpy(tmp + 18 + clen, &crc, 4);
  memcpy(tmp + 22 + clen, &n, 4);
  out->p = tmp;
  out->n = bsize;
}

/* Writes a BAM; returns its size and sets *out (free with synth_bam_free).
 * names: the contigs' names back to back, NUL-terminated; depth: mean depth
 * per contig; seq / seq_off (may be null): the contigs' bases for the reads. */
int64_t synth_bam(const synth_bam_opts *o, int32_t n_targets, const uint32_t *tlen, const char *names,
                  const float *depth, const char *seq, const int64_t *seq_off, uint8_t **out) {
  buf_t *per = (buf_t *)calloc((size_t)(n_targets ? n_targets : 1), sizeof(buf_t));
  int64_t *base_rid = (int64_t *)calloc((size_t)n_targets + 1, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 8)
  for (int32_t t = 0; t < n_targets; ++t) {
    int64_t rid = (int64_t)t << 24;
    uint64_t sd = o->seed ^ (0x632BE59BD9B4E019ULL * (uint64_t)(t + 1));
    contig_reads(o, t, n_targets, tlen[t], depth[t], seq ? seq + seq_off[t] : NULL, sd, &rid, &per[t]);
  }
  buf_t st = {0};
  put(&st, "BAM\1", 4);
  static const char text[] = "@HD\tVN:1.6\tSO:coordinate\n";
  put32(&st, (uint32_t)(sizeof text - 1));
  put(&st, text, sizeof text - 1);
  put32(&st, (uint32_t)n_targets);
  const char *nm = names;
  for (int32_t t = 0; t < n_targets; ++t) {
    const size_t l = strlen(nm) + 1;
    put32(&st, (uint32_t)l);
    put(&st, nm, l);
    put32(&st, tlen[t]);
    nm += l;
  }
  const size_t hdr_len = st.n;
  /* record boundaries for the htslib-style cut */
  size_t nrec_cap = 1024, nrec = 0;
  size_t *rstart = (size_t *)malloc(nrec_cap * sizeof(size_t));
  for (int32_t t = 0; t < n_targets; ++t) {
    size_t q = 0;
    while (q < per[t].n) {
      if (nrec == nrec_cap) rstart = (size_t *)realloc(rstart, (nrec_cap *= 2) * sizeof(size_t));
      rstart[nrec++] = st.n + q;
      uint32_t bs;
      memcpy(&bs, per[t].p + q, 4);
      q += 4 + bs;
    }
    put(&st, per[t].p, per[t].n);
    free(per[t].p);
  }
  free(per);
  free(base_rid);
  uint64_t s = o->seed ^ 0xA5A5A5A5ULL;
  for (int32_t i = 0; i < o->n_unmapped_tail; ++i) {
    if (nrec == nrec_cap) rstart = (size_t *)realloc(rstart, (nrec_cap *= 2) * sizeof(size_t));
    rstart[nrec++] = st.n;
    emit(&st, -1, -1, 0, 0x1 | 0x4 | 0x8, -1, -1, ((int64_t)1 << 40) + i, NULL, 0, o->read_len, NULL, 0,
         &s, -1, 0, 0);
  }
  /* block cuts: the header alone first, then records */
  const size_t MAXP = 65280;
  size_t ncut = 0, cut_cap = 1024;
  size_t *cut = (size_t *)malloc(cut_cap * sizeof(size_t));
#define ADDCUT(x)                                                                      \
  do {                                                                                 \
    if (ncut == cut_cap) cut = (size_t *)realloc(cut, (cut_cap *= 2) * sizeof(size_t)); \
    cut[ncut++] = (x);                                                                 \
  } while (0)
  ADDCUT(0);
  for (size_t a = MAXP; a < hdr_len; a += MAXP) ADDCUT(a);
  ADDCUT(hdr_len);
  if (o->straddle) {
    for (size_t a = hdr_len + MAXP; a < st.n; a += MAXP) ADDCUT(a);
  } else {
    size_t blk = hdr_len;
    for (size_t r = 0; r < nrec; ++r) {
      const size_t end = r + 1 < nrec ? rstart[r + 1] : st.n;
      if (end - blk > MAXP && rstart[r] > blk) {
        ADDCUT(rstart[r]);
        blk = rstart[r];
      }
      while (end - blk > MAXP) { /* a record longer than a block */
        blk += MAXP;
        ADDCUT(blk);
      }
    }
  }
  if (cut[ncut - 1] != st.n) ADDCUT(st.n);
  free(rstart);
  const size_t nb = ncut - 1;
  buf_t *blocks = (buf_t *)calloc(nb ? nb : 1, sizeof(buf_t));
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t i = 0; i < nb; ++i)
    bgzf_block(st.p + cut[i], (uint32_t)(cut[i + 1] - cut[i]), o->level, &blocks[i]);
  static const uint8_t eof[28] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67,
                                  2,  0,   27, 0, 3, 0, 0, 0, 0, 0, 0,   0, 0, 0};
  size_t tot = 28;
  for (size_t i = 0; i < nb; ++i) tot += blocks[i].n;
  uint8_t *res = (uint8_t *)malloc(tot);
  size_t w = 0;
  for (size_t i = 0; i < nb; ++i) {
    memcpy(res + w, blocks[i].p, blocks[i].n);
    w += blocks[i].n;
    free(blocks[i].p);
  }
  memcpy(res + w, eof, 28);
  free(blocks);
  free(cut);
  free(st.p);
  *out = res;
  return (int64_t)tot;
}

void synth_bam_free(uint8_t *p) { free(p); }
