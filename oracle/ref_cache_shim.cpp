// Reference harness, second translation unit: RabbitBin's own RBCACHE1
// writer and reader (src/impl/rb_cache.cpp:26-319, cut out verbatim into
// oracle/_ref/frag/frag_cache.inc at build time and #included below).
//
// TEST INFRASTRUCTURE ONLY (see ref_shim.cpp).  What this file adds are the
// rb_cmd_bin globals the two functions read and write, with the reference's
// names and types (src/rabbitbin.h:121-222, src/rabbitbin.cpp:155-341), a
// row-major float matrix standing in for the ublas matrix (size1, size2,
// data, resize: the members rb_cache.cpp uses), and C entry points that copy
// a flat state into those globals and out of them.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

using std::cerr;
typedef float StoredDistance;
typedef double Similarity;
using GraphNodeId = uint32_t;

struct Matrix {
  std::vector<StoredDistance> v;
  size_t r = 0, c = 0;
  size_t size1() const { return r; }
  size_t size2() const { return c; }
  std::vector<StoredDistance> &data() { return v; }
  const std::vector<StoredDistance> &data() const { return v; }
  void resize(size_t rr, size_t cc, bool) { r = rr; c = cc; v.resize(rr * cc); }
};

struct Graph {
  std::vector<GraphNodeId> from, to;
  std::vector<StoredDistance> sComp;
};

static size_t nobs = 0, nobs1 = 0, num_depth_samples = 0;
static unsigned long long seed = 0, totalSize = 0, totalSize1 = 0;
static Similarity simCutoff = 0;
static double g_pmh_baseline = 0.0;
static size_t minContig = 2500, min_small_contig = 1000;
static std::vector<std::string> contig_names, small_contig_names;
static std::vector<size_t> seq_lens, small_seq_lens;
static Matrix depth_matrix, small_depth_matrix;
static std::vector<float> g_large_means, g_depth_raw;
static std::vector<double> g_depth_colnorm;
static bool g_strain_scan = false;
static std::vector<float> g_snv_pi;
static std::vector<uint32_t> g_snv_nsnv, g_snv_cov;
static unsigned long long g_cache_seed = 0;
static bool g_cache_has_depth = false, g_cache_has_snv = false;
static std::vector<GraphNodeId> g_cache_from, g_cache_to;
static std::vector<StoredDistance> g_cache_scomp;

#include "frag_cache.inc"            // src/impl/rb_cache.cpp:26-319

extern "C" {

// The flat state both programs agree on (the fields of rbg_cache that the
// reference stores), names as bytes + offsets.
struct RefCacheState {
  int64_t n_large, n_small, samples;
  uint64_t seed, total_size, total_size_small;
  double sim_cutoff, b0;
  uint64_t min_contig, min_small_contig;
  int32_t has_depth, has_snv;
  const char *large_names; const int64_t *large_name_off; int64_t n_large_names;
  const char *small_names; const int64_t *small_name_off; int64_t n_small_names;
  const uint64_t *large_len; int64_t n_large_len;
  const uint64_t *small_len; int64_t n_small_len;
  const float *depth_ranked; int64_t depth_rows, depth_cols;
  const float *small_depth; int64_t small_depth_rows, small_depth_cols;
  const float *large_means; int64_t n_large_means;
  const float *depth_raw; int64_t n_depth_raw;
  const double *colnorm; int64_t n_colnorm;
  const uint32_t *from, *to; const float *scomp; int64_t n_edges;
  const float *snv_pi; const uint32_t *snv_nsnv, *snv_cov; int64_t n_snv;
};

static std::vector<std::string> names_of(const char *b, const int64_t *off, int64_t n) {
  std::vector<std::string> v;
  for (int64_t i = 0; b && i < n; ++i) v.emplace_back(b + off[i], (size_t)(off[i + 1] - off[i]));
  return v;
}

int ref_cache_write(const char *path, const RefCacheState *s) {
  nobs = (size_t)s->n_large;
  nobs1 = (size_t)s->n_small;
  num_depth_samples = (size_t)s->samples;
  seed = s->seed;
  totalSize = s->total_size;
  totalSize1 = s->total_size_small;
  simCutoff = s->sim_cutoff;
  g_pmh_baseline = s->b0;
  minContig = (size_t)s->min_contig;
  min_small_contig = (size_t)s->min_small_contig;
  contig_names = names_of(s->large_names, s->large_name_off, s->n_large_names);
  small_contig_names = names_of(s->small_names, s->small_name_off, s->n_small_names);
  seq_lens.assign(s->large_len, s->large_len + (s->large_len ? s->n_large_len : 0));
  small_seq_lens.assign(s->small_len, s->small_len + (s->small_len ? s->n_small_len : 0));
  depth_matrix.resize((size_t)s->depth_rows, (size_t)s->depth_cols, false);
  if (s->depth_rows * s->depth_cols)
    std::memcpy(depth_matrix.v.data(), s->depth_ranked, depth_matrix.v.size() * 4);
  small_depth_matrix.resize((size_t)s->small_depth_rows, (size_t)s->small_depth_cols, false);
  if (s->small_depth_rows * s->small_depth_cols)
    std::memcpy(small_depth_matrix.v.data(), s->small_depth, small_depth_matrix.v.size() * 4);
  g_large_means.assign(s->large_means, s->large_means + s->n_large_means);
  g_depth_raw.assign(s->depth_raw, s->depth_raw + s->n_depth_raw);
  g_depth_colnorm.assign(s->colnorm, s->colnorm + s->n_colnorm);
  Graph g;
  g.from.assign(s->from, s->from + s->n_edges);
  g.to.assign(s->to, s->to + s->n_edges);
  g.sComp.assign(s->scomp, s->scomp + s->n_edges);
  g_strain_scan = s->has_snv != 0;
  g_snv_pi.assign(s->snv_pi, s->snv_pi + (s->has_snv ? s->n_snv : 0));
  g_snv_nsnv.assign(s->snv_nsnv, s->snv_nsnv + (s->has_snv ? s->n_snv : 0));
  g_snv_cov.assign(s->snv_cov, s->snv_cov + (s->has_snv ? s->n_snv : 0));
  return rb_write_cache(path, g, s->has_depth != 0) ? 0 : -1;
}

// rb_load_cache, then the restored globals: scalars into *s (pointers not
// touched) and the arrays into caller buffers sized from ref_cache_read's
// first call (counts in *s).  Returns 0 / -1 as the reference's bool.
int ref_cache_read(const char *path, RefCacheState *s, char *lnames, int64_t *lnoff,
                   char *snames, int64_t *snoff, uint64_t *llen, uint64_t *slen, float *dr,
                   float *sd, float *lm, float *raw, double *cn, uint32_t *fr, uint32_t *to,
                   float *sc, float *pi, uint32_t *nsnv, uint32_t *cov) {
  if (!rb_load_cache(path)) return -1;
  s->n_large = (int64_t)nobs;
  s->n_small = (int64_t)nobs1;
  s->samples = (int64_t)num_depth_samples;
  s->seed = g_cache_seed;
  s->total_size = totalSize;
  s->total_size_small = totalSize1;
  s->sim_cutoff = simCutoff;
  s->b0 = g_pmh_baseline;
  s->has_depth = g_cache_has_depth;
  s->has_snv = g_cache_has_snv;
  s->n_large_names = (int64_t)contig_names.size();
  s->n_small_names = (int64_t)small_contig_names.size();
  s->n_large_len = (int64_t)seq_lens.size();
  s->n_small_len = (int64_t)small_seq_lens.size();
  s->depth_rows = (int64_t)depth_matrix.r;
  s->depth_cols = (int64_t)depth_matrix.c;
  s->small_depth_rows = (int64_t)small_depth_matrix.r;
  s->small_depth_cols = (int64_t)small_depth_matrix.c;
  s->n_large_means = (int64_t)g_large_means.size();
  s->n_depth_raw = (int64_t)g_depth_raw.size();
  s->n_colnorm = (int64_t)g_depth_colnorm.size();
  s->n_edges = (int64_t)g_cache_from.size();
  s->n_snv = g_cache_has_snv ? (int64_t)g_snv_pi.size() : 0;
  if (!lnames) return 0;                       // counts only
  auto put_names = [](const std::vector<std::string> &v, char *b, int64_t *off) {
    off[0] = 0;
    for (size_t i = 0; i < v.size(); ++i) {
      std::memcpy(b + off[i], v[i].data(), v[i].size());
      off[i + 1] = off[i] + (int64_t)v[i].size();
    }
  };
  put_names(contig_names, lnames, lnoff);
  put_names(small_contig_names, snames, snoff);
  std::copy(seq_lens.begin(), seq_lens.end(), llen);
  std::copy(small_seq_lens.begin(), small_seq_lens.end(), slen);
  std::copy(depth_matrix.v.begin(), depth_matrix.v.end(), dr);
  std::copy(small_depth_matrix.v.begin(), small_depth_matrix.v.end(), sd);
  std::copy(g_large_means.begin(), g_large_means.end(), lm);
  std::copy(g_depth_raw.begin(), g_depth_raw.end(), raw);
  std::copy(g_depth_colnorm.begin(), g_depth_colnorm.end(), cn);
  std::copy(g_cache_from.begin(), g_cache_from.end(), fr);
  std::copy(g_cache_to.begin(), g_cache_to.end(), to);
  std::copy(g_cache_scomp.begin(), g_cache_scomp.end(), sc);
  if (g_cache_has_snv) {
    std::copy(g_snv_pi.begin(), g_snv_pi.end(), pi);
    std::copy(g_snv_nsnv.begin(), g_snv_nsnv.end(), nsnv);
    std::copy(g_snv_cov.begin(), g_snv_cov.end(), cov);
  }
  return 0;
}

}  // extern "C"
