// RBCACHE1 version 3: the on-disk state of a built graph (rbg_write_cache /
// rbg_read_cache).
//
// RabbitBin writes this file after the expensive stages (FASTA parse, sketch,
// depth load and rank transform, the O(N^2) graph) so that a later run goes
// straight to the cheap tail (edge weights, incidence, label propagation,
// recruitment, split, output) under other parameters
// (rb_write_cache / rb_load_cache, src/impl/rb_cache.cpp:103-319).  The
// serving form uses it for warm restarts: a finished request's graph and the
// per-contig state it was built from can be stored and read back by either
// program.
//
// Layout (little endian, as the reference writes it with fwrite on x86-64):
//   "RBCACHE1", u32 version (3), u32 sizeof(float) (4), u32 sizeof(size_t) (8),
//   u64 n_large, u64 n_small, u64 samples, u64 seed, u64 total_size,
//   u64 total_size_small, f64 sim_cutoff, f64 b0, u64 min_contig,
//   u64 min_small_contig, u8 has_depth,
//   names of the large contigs, of the small ones (u64 count, then u32 length
//   + bytes each), lengths of the large and the small contigs (u64 count +
//   u64 each), the ranked depth matrix and the raw small-contig depth matrix
//   (u64 rows, u64 cols, rows * cols f32), the large contigs' raw means, the
//   raw depths (u64 count + f32 each), the per-sample norms (u64 count + f64
//   each), the graph's from, to (u64 count + u32 each) and sComp (u64 count +
//   f32 each), u8 has_snv and, when set, the SNV pi (f32), SNV counts and
//   covered sites (u32) arrays.
// Reading accepts versions 1 and 2 too (endpoints stored as u64, no SNV block
// in version 1), with the reference's range checks on the endpoints.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "engine_internal.h"

namespace {

const char kMagic[8] = {'R', 'B', 'C', 'A', 'C', 'H', 'E', '1'};
constexpr uint32_t kVersion = 3;

struct Writer {
  FILE *f;
  template <class T> void pod(const T &v) { fwrite(&v, sizeof(T), 1, f); }
  template <class T> void vec(const T *p, uint64_t n) {
    pod(n);
    if (n) fwrite(p, sizeof(T), n, f);
  }
  void strvec(const char *bytes, const int64_t *off, uint64_t n) {
    pod(n);
    for (uint64_t i = 0; i < n; ++i) {
      const uint32_t len = (uint32_t)(off[i + 1] - off[i]);
      pod(len);
      if (len) fwrite(bytes + off[i], 1, len, f);
    }
  }
  void mat(const float *p, uint64_t r, uint64_t c) {
    pod(r);
    pod(c);
    if (r && c) fwrite(p, sizeof(float), r * c, f);
  }
};

struct Reader {
  FILE *f;
  bool ok = true;
  template <class T> void pod(T &v) { ok = ok && fread(&v, sizeof(T), 1, f) == 1; }
  // u64 count + elements into a malloc'd array (null when empty)
  template <class T> T *vec(uint64_t &n) {
    n = 0;
    pod(n);
    if (!ok || n == 0) return nullptr;
    if (n > ((uint64_t)1 << 40) / sizeof(T)) { ok = false; return nullptr; }
    T *p = (T *)malloc(n * sizeof(T));
    if (!p || fread(p, sizeof(T), n, f) != n) { ok = false; free(p); return nullptr; }
    return p;
  }
  void strvec(char *&bytes, int64_t *&off, uint64_t &n) {
    n = 0;
    pod(n);
    bytes = nullptr;
    off = nullptr;
    if (!ok) return;
    if (n > ((uint64_t)1 << 34)) { ok = false; return; }
    off = (int64_t *)malloc((n + 1) * sizeof(int64_t));
    if (!off) { ok = false; return; }
    off[0] = 0;
    std::string all;
    for (uint64_t i = 0; i < n && ok; ++i) {
      uint32_t len = 0;
      pod(len);
      if (!ok) break;
      const size_t at = all.size();
      all.resize(at + len);
      if (len && fread(&all[at], 1, len, f) != len) ok = false;
      off[i + 1] = (int64_t)all.size();
    }
    bytes = (char *)malloc(all.size() + 1);
    if (!bytes) { ok = false; return; }
    if (!all.empty()) std::memcpy(bytes, all.data(), all.size());
    bytes[all.size()] = 0;
  }
  float *mat(uint64_t &r, uint64_t &c) {
    r = c = 0;
    pod(r);
    pod(c);
    if (!ok || r == 0 || c == 0) return nullptr;
    if (r > ((uint64_t)1 << 40) / c) { ok = false; return nullptr; }
    float *p = (float *)malloc(r * c * sizeof(float));
    if (!p || fread(p, sizeof(float), r * c, f) != r * c) { ok = false; free(p); return nullptr; }
    return p;
  }
};

}  // namespace

extern "C" {

int rbg_write_cache(const char *path, const rbg_cache *st) {
  if (!path || !st || st->n_large < 0 || st->n_small < 0 || st->n_edges < 0) return RBG_ERR_ARG;
  FILE *f = fopen(path, "wb");
  if (!f) return RBG_ERR_ARG;
  Writer w{f};
  fwrite(kMagic, 1, 8, f);
  w.pod(kVersion);
  w.pod((uint32_t)sizeof(float));
  w.pod((uint32_t)8);
  w.pod((uint64_t)st->n_large);
  w.pod((uint64_t)st->n_small);
  w.pod((uint64_t)st->samples);
  w.pod((uint64_t)st->seed);
  w.pod((uint64_t)st->total_size);
  w.pod((uint64_t)st->total_size_small);
  w.pod(st->sim_cutoff);
  w.pod(st->b0);
  w.pod((uint64_t)st->min_contig);
  w.pod((uint64_t)st->min_small_contig);
  w.pod((uint8_t)(st->has_depth ? 1 : 0));
  w.strvec(st->large_names, st->large_name_off, (uint64_t)(st->large_names ? st->n_large : 0));
  w.strvec(st->small_names, st->small_name_off, (uint64_t)(st->small_names ? st->n_small : 0));
  w.vec(st->large_len, st->large_len ? (uint64_t)st->n_large : 0);
  w.vec(st->small_len, st->small_len ? (uint64_t)st->n_small : 0);
  w.mat(st->depth_ranked, (uint64_t)st->depth_rows, (uint64_t)st->depth_cols);
  w.mat(st->small_depth, (uint64_t)st->small_depth_rows, (uint64_t)st->small_depth_cols);
  w.vec(st->large_means, (uint64_t)st->n_large_means);
  w.vec(st->depth_raw, (uint64_t)st->n_depth_raw);
  w.vec(st->colnorm, (uint64_t)st->n_colnorm);
  w.vec(st->from, (uint64_t)st->n_edges);
  w.vec(st->to, (uint64_t)st->n_edges);
  w.vec(st->scomp, (uint64_t)st->n_edges);
  const uint8_t hs = (st->has_snv && st->n_snv > 0) ? 1 : 0;
  w.pod(hs);
  if (hs) {
    w.vec(st->snv_pi, (uint64_t)st->n_snv);
    w.vec(st->snv_nsnv, (uint64_t)st->n_snv);
    w.vec(st->snv_cov, (uint64_t)st->n_snv);
  }
  const bool ok = ferror(f) == 0;
  return (fclose(f) == 0 && ok) ? RBG_OK : RBG_ERR_ARG;
}

int rbg_read_cache(const char *path, rbg_cache *out) {
  if (!path || !out) return RBG_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  FILE *f = fopen(path, "rb");
  if (!f) return RBG_ERR_ARG;
  Reader r{f};
  char magic[8];
  uint32_t ver = 0, sz_sd = 0, sz_st = 0;
  if (fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kMagic, 8) != 0) {
    fclose(f);
    return RBG_ERR_ARG;
  }
  r.pod(ver);
  r.pod(sz_sd);
  r.pod(sz_st);
  if (!r.ok || ver < 1 || ver > kVersion || sz_sd != 4 || sz_st != 8) {
    fclose(f);
    return RBG_ERR_UNSUPPORTED;
  }
  uint64_t nl = 0, ns = 0, S = 0, seed = 0, ts = 0, ts1 = 0, mc = 0, msc = 0;
  double sim = 0.0, b0 = 0.0;
  uint8_t hd = 0;
  r.pod(nl); r.pod(ns); r.pod(S); r.pod(seed); r.pod(ts); r.pod(ts1);
  r.pod(sim); r.pod(b0); r.pod(mc); r.pod(msc); r.pod(hd);
  if (!r.ok || nl > 0xFFFFFFFFull) {          // endpoints are 32-bit node ids
    fclose(f);
    return RBG_ERR_ARG;
  }
  out->n_large = (int64_t)nl;
  out->n_small = (int64_t)ns;
  out->samples = (int64_t)S;
  out->seed = seed;
  out->total_size = ts;
  out->total_size_small = ts1;
  out->sim_cutoff = sim;
  out->b0 = b0;
  out->min_contig = mc;
  out->min_small_contig = msc;
  out->has_depth = hd != 0;
  uint64_t cnt = 0, r0 = 0, c0 = 0;
  char *nb = nullptr;
  int64_t *no = nullptr;
  r.strvec(nb, no, cnt);
  out->large_names = nb;
  out->large_name_off = no;
  out->n_large_names = (int64_t)cnt;
  r.strvec(nb, no, cnt);
  out->small_names = nb;
  out->small_name_off = no;
  out->n_small_names = (int64_t)cnt;
  out->large_len = r.vec<uint64_t>(cnt);
  out->n_large_len = (int64_t)cnt;
  out->small_len = r.vec<uint64_t>(cnt);
  out->n_small_len = (int64_t)cnt;
  out->depth_ranked = r.mat(r0, c0);
  out->depth_rows = (int64_t)r0;
  out->depth_cols = (int64_t)c0;
  out->small_depth = r.mat(r0, c0);
  out->small_depth_rows = (int64_t)r0;
  out->small_depth_cols = (int64_t)c0;
  out->large_means = r.vec<float>(cnt);
  out->n_large_means = (int64_t)cnt;
  out->depth_raw = r.vec<float>(cnt);
  out->n_depth_raw = (int64_t)cnt;
  out->colnorm = r.vec<double>(cnt);
  out->n_colnorm = (int64_t)cnt;
  uint64_t nf = 0, nt = 0, nsc = 0;
  if (ver >= 3) {
    out->from = r.vec<uint32_t>(nf);
    out->to = r.vec<uint32_t>(nt);
  } else {                                     // versions 1, 2: size_t endpoints
    uint64_t *lf = r.vec<uint64_t>(nf), *lt = r.vec<uint64_t>(nt);
    if (r.ok && nf) out->from = (uint32_t *)malloc(nf * 4);
    if (r.ok && nt) out->to = (uint32_t *)malloc(nt * 4);
    for (uint64_t e = 0; r.ok && e < nf; ++e) {
      if (lf[e] > 0xFFFFFFFFull) r.ok = false;
      else out->from[e] = (uint32_t)lf[e];
    }
    for (uint64_t e = 0; r.ok && e < nt; ++e) {
      if (lt[e] > 0xFFFFFFFFull) r.ok = false;
      else out->to[e] = (uint32_t)lt[e];
    }
    free(lf);
    free(lt);
  }
  out->scomp = r.vec<float>(nsc);
  if (r.ok && (nf != nt || nf != nsc)) r.ok = false;
  for (uint64_t e = 0; r.ok && e < nf; ++e)
    if (out->from[e] >= nl || out->to[e] >= nl) r.ok = false;
  out->n_edges = (int64_t)nf;
  if (r.ok && ver >= 2) {
    uint8_t hs = 0;
    r.pod(hs);
    if (r.ok && hs) {
      uint64_t a = 0, b = 0, c = 0;
      out->snv_pi = r.vec<float>(a);
      out->snv_nsnv = r.vec<uint32_t>(b);
      out->snv_cov = r.vec<uint32_t>(c);
      out->n_snv = (int64_t)a;
      out->has_snv = r.ok ? 1 : 0;
    }
  }
  out->version = (int32_t)ver;
  fclose(f);
  if (!r.ok) {
    rbg_free_cache(out);
    return RBG_ERR_ARG;
  }
  return RBG_OK;
}

int rbg_free_cache(rbg_cache *c) {
  if (!c) return RBG_ERR_ARG;
  void *ps[] = {(void *)c->large_names, (void *)c->large_name_off, (void *)c->small_names,
                (void *)c->small_name_off, (void *)c->large_len, (void *)c->small_len,
                (void *)c->depth_ranked, (void *)c->small_depth, (void *)c->large_means,
                (void *)c->depth_raw, (void *)c->colnorm, (void *)c->from, (void *)c->to,
                (void *)c->scomp, (void *)c->snv_pi, (void *)c->snv_nsnv, (void *)c->snv_cov};
  for (void *p : ps) free(p);
  std::memset(c, 0, sizeof(*c));
  return RBG_OK;
}

}  // extern "C"
