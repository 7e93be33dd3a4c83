// Reference harness: runs RabbitBin's own hot-path code on the host.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit is the checker, never the
// product: only tests/, the smoke check and bench.py's CPU-baseline leg load
// the library it builds (oracle/_ref/librbref.so).
//
// The full `rabbitbin` binary cannot be built here (it needs Boost >= 1.66
// headers and libdeflate).  oracle/build.py therefore compiles the hot-path
// functions where they lie in the reference tree:
//   * src/probmh.cpp (whole file, unchanged) + src/probmh.h, src/hash_int.h,
//     src/rabbit_sketch.h, src/ranker.h, src/tile.h (headers, unchanged);
//   * line ranges of src/rabbitbin.cpp, src/rabbitbin.h, src/impl/rb_graph.cpp
//     and src/impl/rb_abundance.cpp, cut out verbatim into oracle/_ref/frag/
//     at build time (never committed) and #included below.
// What this file adds is only the surrounding declarations those functions
// read (globals with the reference's names and defaults, a row-major stand-in
// for the ublas depth matrix, logging stubs) and the glue that the reference
// keeps inline in rb_cmd_bin (the winner pack loop src/rabbitbin.cpp:4934-4952,
// b0 setup :4958-4965, colnorm :4792-4809, rank loop :4867-4874, unit rows
// :4972-4988, graph dispatch :5035-5054, edge-weight loop :5482-5509).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <immintrin.h>
#include <limits>
#include <memory>
#include <numeric>
#include <queue>
#include <random>
#include <string>
#include <unordered_set>
#include <utility>
#include <vector>
#include <omp.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "probmh.h"
#include "rabbit_invidx.h"
#include "rabbit_sketch.h"
#include "ranker.h"
#include "tile.h"
#include "ProgressTracker.h"

// ── typedefs the fragments use (src/rabbitbin.h:71-102, :207, :213, :261-262) ──
typedef double Distance;
typedef double Similarity;
typedef float StoredDistance;
typedef std::pair<size_t, StoredDistance> Edge;
typedef std::unordered_set<size_t> ContigSet;
using GraphNodeId = uint32_t;
using GraphEdgeId = uint32_t;

// Data contract of the reference graph (src/rabbitbin.h:264-301), reduced to
// the members the hot path touches.
struct Graph {
  size_t n;
  std::vector<GraphNodeId> from, to;
  std::vector<StoredDistance> sComp, edgeScore;
  explicit Graph(size_t num_nodes) : n(num_nodes) {}
  size_t getEdgeCount() { return from.size(); }
};

// Row-major float matrix standing in for boost::numeric::ublas::matrix<float>.
struct RowMajorMatrix {
  std::vector<float> v;
  size_t cols = 0;
  float &operator()(size_t r, size_t c) { return v[r * cols + c]; }
  float operator()(size_t r, size_t c) const { return v[r * cols + c]; }
};

// ── globals read by the fragments, reference names and defaults ─────────────
static bool verbose = false;
static std::string depth_file;               // non-empty <=> depth input given
static size_t numThreads = 1;
static Similarity min_edge_weight = 0.70;
static Distance minCV = 1.0;
static size_t maxEdges = 200;
static size_t nobs = 0;
static size_t num_depth_samples = 0;
static uint32_t sketch_size = 500;
static uint32_t sketch_bits = 1;
static RowMajorMatrix depth_matrix;
static const size_t RB_SIM_FLOOR = 50;

static int g_depth_sim = 2;
static int g_depth_fuse = 1;
static double g_depth_wjac_cut = 0.0;
static bool g_depth_wjac_gate = false;
static std::vector<float> g_depth_raw;
static std::vector<double> g_depth_colnorm;
static std::vector<float> g_depth_unit;
static std::vector<float> g_snv_traj;
static std::vector<char> g_snv_traj_have;
static bool g_snv_edge = false;
static double g_snv_edge_lo = 0.10;
static bool g_dual_conj = false;
static std::vector<float> g_depth_unit_blk;

static std::vector<uint64_t> g_sig_flat;
static uint32_t g_sig_nw = 0, g_sig_np = 0, g_sig_m = 0;
static bool g_pmh_mode = true;
static uint32_t g_pmh_m = 0;
static std::vector<uint32_t> g_win_flat;
static std::vector<uint64_t> g_win64_flat;
static std::vector<uint16_t> g_win16;
static int g_win_bits = 32;
static bool g_pmh_base_on = true;
static double g_pmh_baseline = 0.0;
static double g_inv_pmh_m = 0.0;
static double g_inv_one_minus_b0 = 1.0;
static double g_w_comp = 0.5;
static bool g_mutual_knn = true;
static double g_neg_depth_thr = -0.3;
static int g_gc_norm = 1;
static double g_gc_norm_cap = 20.0;
static bool g_exact_cos_cmp = false;
static std::vector<float> g_k4cosine_flat;
static std::vector<uint8_t> g_anynz;

static void verbose_message(const char *, ...) {}
static double getUsedPhysMem() { return 0.0; }
static double getTotalPhysMem() { return 0.0; }
static inline void numa_interleave_buffer(void *, size_t) {}
static const char *rb_getenv(const char *key) {
  const char *e = getenv(key);
  return (e && e[0]) ? e : nullptr;
}
// Unused branch of the fragments (Welford correlation).
double cal_depth_corr(size_t, size_t, bool = false, bool = false) { abort(); }

#pragma omp declare reduction (merge_graphnode : std::vector<GraphNodeId> : omp_out.insert(omp_out.end(), omp_in.begin(), omp_in.end()) )
#pragma omp declare reduction (merge_storeddist : std::vector<StoredDistance> : omp_out.insert(omp_out.end(), omp_in.begin(), omp_in.end()) )

// ── reference code, verbatim line ranges (see oracle/build.py) ───────────────
#include "frag_random_unique.inc"   // src/rabbitbin.h:330-341
#include "frag_compare_edge.inc"    // src/rabbitbin.h:418-429
#include "frag_fold16.inc"          // src/rabbitbin.cpp:249-253
#include "frag_depth_terms.inc"     // src/rabbitbin.cpp:685-970
#include "frag_jaccard_raw.inc"     // src/rabbitbin.cpp:1031-1135
#include "frag_pmh_sim.inc"         // src/rabbitbin.cpp:1194-1426
#include "frag_build_winners.inc"   // src/rabbitbin.cpp:1436-1589
// globals and helpers the FASTA parser reads (src/rabbitbin.h:198-199 and the
// rb_cmd_bin state); the TNF branch is never taken here (collect_tnf = false)
static const char *g_fasta_mmap = nullptr;
static size_t g_fasta_mmap_len = 0;
static std::vector<std::string> g_seq_arenas;
static bool g_idf_norm = false;
static inline void rb_phase(const char *) {}
static inline void rb_fill_tnf(const char *, size_t, float *) { abort(); }
#include "frag_contig_rec.inc"      // src/rabbitbin.cpp:1876-1888
#include "frag_parse_fasta.inc"     // src/rabbitbin.cpp:1890-2248
#include "frag_anynz.inc"           // src/impl/rb_abundance.cpp:94-114
#include "frag_graph_allpairs.inc"  // src/impl/rb_graph.cpp:7-72
// state of the inverted-index graph build (src/rabbitbin.cpp:209, :1593)
static std::vector<rabbit_sketch::KmerSketch *> g_sketches;
static std::unique_ptr<rabbit_invidx::InvertedIndex> g_inv_idx;
#include "frag_graph_index.inc"     // src/impl/rb_graph.cpp:199-383
#include "frag_calib_converge.inc"  // src/impl/rb_graph.cpp:390-415
#include "frag_fused_graph.inc"     // src/impl/rb_graph.cpp:480-1356
#include "frag_calibrate.inc"       // src/impl/rb_graph.cpp:1362-1384
#include "frag_calibrate_fused.inc" // src/impl/rb_graph.cpp:1386-1438

// ═════════════════════════════════════════════════════════════════════════════
// C entry points used by the tests and the CPU baseline.
// ═════════════════════════════════════════════════════════════════════════════
extern "C" {

// Winner rows for n contigs (concatenated ASCII, offsets[n+1]), the parallel
// sketch loop of src/rabbitbin.cpp:4849-4865 (one thread-local scratch each).
void ref_build_winners(const char *seqcat, const int64_t *offsets, int64_t n,
                       int k, uint32_t m, uint64_t seed, int gc_norm,
                       double gc_cap, uint32_t *out32, int nthreads) {
  g_gc_norm = gc_norm;
  g_gc_norm_cap = gc_cap;
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
  {
    std::vector<uint64_t> scratch;
#pragma omp for schedule(dynamic, 8)
    for (int64_t r = 0; r < n; ++r)
      build_pmh_winners(seqcat + offsets[r], (size_t)(offsets[r + 1] - offsets[r]),
                        k, m, seed, out32 + (size_t)r * m, scratch);
  }
}

void ref_fold16(const uint32_t *in, uint16_t *out, int64_t n) {
  for (int64_t t = 0; t < n; ++t) out[t] = fold_win16(in[t]);
}

// Parameters of one graph + edge-weight run (the rb_cmd_bin globals).
struct RefParams {
  int64_t n;            // large contigs
  int32_t m;            // --sketch-m
  int32_t S;            // depth samples (0 = no depth file)
  int32_t win_bits;     // 16 (default) or 32
  int32_t max_edges;    // --max-edges
  int32_t mutual;       // RABBIT_MUTUAL_KNN
  int32_t base_on;      // RABBIT_PMH_BASE
  int32_t nthreads;
  uint32_t seed;        // --seed (srand)
  int32_t force_path;   // 0 auto, 1 small-N, 2 fused large-N
  double coverage;      // --max-posterior / 100
  double min_edge;      // --min-edge-score / 100
  double w_comp;        // < 0: auto_w_comp(S)
  double min_cv;        // --min-coverage
  double neg_thr;       // RABBIT_NEG_DEPTH
  int32_t depth_sim;    // RABBIT_DEPTH_SIM
  int32_t depth_fuse;   // RABBIT_DEPTH_FUSE
  int32_t wjac_norm;    // RABBIT_DEPTH_WJAC_NORM
  int32_t no_abdfirst;  // RABBIT_NO_ABDFIRST set
  int32_t oph_k;        // 0: PMH metric; > 0: RABBIT_PMH=0 with sketch_kmer_size = oph_k
  int32_t oph_bits;     // sketch_bits
  int32_t graph_index;  // RABBIT_GRAPH_INDEX=1 (small path: inverted-index candidates)
  int32_t min_common;   // RABBIT_MINCOMMON (0: unset)
  int32_t index_k;      // sketch_kmer_size of the index's one-permutation sketches
};

struct RefOut {
  double b0;
  double sim_cutoff;    // simCutoff (x1000 units, as returned by the reference)
  int64_t n_edges;
  uint32_t *from, *to;  // malloc'd, caller frees with ref_free
  float *scomp, *score;
};

void ref_free(void *p) { free(p); }

// parse_fasta_mmap_parallel (src/rabbitbin.cpp:1890-2248) on a file, as
// rb_cmd_bin calls it for binning (full headers off, no streamed sketches, no
// tiny or TNF collection).  Large then small contigs, each in file order:
// names joined in `names` (offsets name_off[n+1]), sequences in `seqcat`
// (offsets seq_off[n+1]); arrays malloc'd, free each with ref_free.
struct RefFasta {
  int64_t num_seqs, n_large, n_small;
  char *names;
  int64_t *name_off;
  char *seqcat;
  int64_t *seq_off;
};

int ref_parse_fasta(const char *path, int nthreads, int64_t min_contig, int64_t min_small,
                    RefFasta *out) {
  std::vector<ContigRec> large, small;
  std::vector<std::pair<std::string, std::string>> tiny;
  size_t nseq = 0;
  if (!parse_fasta_mmap_parallel(path, nthreads, (size_t)min_contig, (size_t)min_small,
                                 false, false, false, false, false, 500, 4, large, small,
                                 tiny, nseq))
    return -1;
  std::vector<const ContigRec *> recs;
  for (auto &r : large) recs.push_back(&r);
  for (auto &r : small) recs.push_back(&r);
  const size_t n = recs.size();
  size_t nb = 0, sb = 0;
  for (auto *r : recs) { nb += r->name.size(); sb += r->len; }
  out->num_seqs = (int64_t)nseq;
  out->n_large = (int64_t)large.size();
  out->n_small = (int64_t)small.size();
  out->names = (char *)malloc(nb + 1);
  out->name_off = (int64_t *)malloc((n + 1) * sizeof(int64_t));
  out->seqcat = (char *)malloc(sb + 1);
  out->seq_off = (int64_t *)malloc((n + 1) * sizeof(int64_t));
  size_t a = 0, b = 0;
  out->name_off[0] = 0;
  out->seq_off[0] = 0;
  for (size_t i = 0; i < n; ++i) {
    const ContigRec &r = *recs[i];
    memcpy(out->names + a, r.name.data(), r.name.size());
    a += r.name.size();
    const char *s = r.seq_view_ptr ? r.seq_view_ptr : g_seq_arenas[r.arena_tid].data() + r.arena_off;
    memcpy(out->seqcat + b, s, r.len);
    b += r.len;
    out->name_off[i + 1] = (int64_t)a;
    out->seq_off[i + 1] = (int64_t)b;
  }
  if (g_fasta_mmap) munmap((void *)g_fasta_mmap, g_fasta_mmap_len);
  g_fasta_mmap = nullptr;
  g_fasta_mmap_len = 0;
  g_seq_arenas.clear();
  return 0;
}

// One-permutation MinHash signatures of n contigs, the sketch loop of
// src/rabbitbin.cpp:4819-4841 (KmerSketch(m, K, bits), update, getSignature):
// rows of nw * bits words (plane p at [p * nw]) into sig_out.
static void oph_signatures(const char *seqcat, const int64_t *offsets, int64_t n, uint32_t m,
                           int K, uint32_t bits, int nthreads, uint64_t *sig_out) {
  const uint32_t nw = (m + 63) / 64;
  const size_t stride = (size_t)nw * bits;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 16)
  for (int64_t r = 0; r < n; ++r) {
    rabbit_sketch::KmerSketch sk(m, K, bits);
    sk.update(seqcat + offsets[r], (uint64_t)(offsets[r + 1] - offsets[r]));
    const uint64_t *sig = sk.getSignature();
    std::memcpy(sig_out + (size_t)r * stride, sig, stride * sizeof(uint64_t));
  }
}

static int run_graph_body(const RefParams *p, const uint32_t *winners32,
                          const float *depth_raw, float *unit_out, RefOut *out);

// Bucket values of the one-permutation signatures: bit p of values[r][b] =
// bit b of plane p.
void ref_oph_values(const char *seqcat, const int64_t *offsets, int64_t n, uint32_t m, int K,
                    uint32_t bits, uint8_t *values) {
  const uint32_t nw = (m + 63) / 64;
  const size_t stride = (size_t)nw * bits;
  std::vector<uint64_t> sig((size_t)n * stride);
  oph_signatures(seqcat, offsets, n, m, K, bits, omp_get_max_threads(), sig.data());
  for (int64_t r = 0; r < n; ++r)
    for (uint32_t b = 0; b < m; ++b) {
      uint32_t v = 0;
      for (uint32_t q = 0; q < bits; ++q)
        v |= (uint32_t)((sig[(size_t)r * stride + (size_t)q * nw + (b >> 6)] >> (b & 63)) & 1u) << q;
      values[(size_t)r * m + b] = (uint8_t)v;
    }
}

// The same run with RABBIT_PMH=0: the graph similarity is jaccard_raw over
// the one-permutation signatures (graph_sim, src/rabbitbin.cpp:1403-1426) and
// no baseline is estimated (:4958).
int ref_run_graph_oph(const RefParams *p, const char *seqcat, const int64_t *offsets,
                      const float *depth_raw, float *unit_out, RefOut *out) {
  const uint32_t m = (uint32_t)p->m, bits = (uint32_t)p->oph_bits;
  g_sig_m = m;
  g_sig_nw = (m + 63) / 64;
  g_sig_np = bits;
  g_sig_flat.assign((size_t)p->n * g_sig_nw * g_sig_np, 0ull);
  oph_signatures(seqcat, offsets, p->n, m, p->oph_k, bits, p->nthreads > 0 ? p->nthreads : 1,
                 g_sig_flat.data());
  g_pmh_mode = false;
  const int rc = run_graph_body(p, nullptr, depth_raw, unit_out, out);
  g_pmh_mode = true;
  std::vector<uint64_t>().swap(g_sig_flat);
  return rc;
}

static bool g_use_index = false;

// The same run with RABBIT_GRAPH_INDEX=1: the one-permutation sketches of
// every contig (KmerSketch(sketch_size, index_k, sketch_bits), update) and
// the inverted index of their keys, built as the sketch loop of rb_cmd_bin
// builds them (src/rabbitbin.cpp:4737-4741, :4819-4830, :4885-4891) but with
// one insertion thread, so every posting list holds its contigs in ascending
// order; the small path's graph then comes from build_similarity_graph
// (src/impl/rb_graph.cpp:199-383).
int ref_run_graph_index(const RefParams *p, const char *seqcat, const int64_t *offsets,
                        const uint32_t *winners32, const float *depth_raw, float *unit_out,
                        RefOut *out) {
  const int64_t n = p->n;
  const uint32_t bits = (uint32_t)(p->oph_bits > 0 ? p->oph_bits : 2);
  g_sketches.assign((size_t)n, nullptr);
  rabbit_invidx::InvertedIndexBuilder builder(1);
  std::vector<uint64_t> ks;
  for (int64_t r = 0; r < n; ++r) {
    g_sketches[r] = new rabbit_sketch::KmerSketch((uint32_t)p->m, p->index_k > 0 ? p->index_k : 8,
                                                  bits);
    g_sketches[r]->update(seqcat + offsets[r], (uint64_t)(offsets[r + 1] - offsets[r]));
    g_sketches[r]->getKeys(ks);
    for (uint64_t k : ks) builder.insert(0, k, (uint32_t)r);
  }
  g_inv_idx = std::make_unique<rabbit_invidx::InvertedIndex>(builder.build(1));
  setenv("RABBIT_GRAPH_INDEX", "1", 1);
  if (p->min_common > 0) setenv("RABBIT_MINCOMMON", std::to_string(p->min_common).c_str(), 1);
  g_pmh_mode = true;
  g_use_index = true;
  const int rc = run_graph_body(p, winners32, depth_raw, unit_out, out);
  g_use_index = false;
  unsetenv("RABBIT_GRAPH_INDEX");
  unsetenv("RABBIT_MINCOMMON");
  for (auto *sk : g_sketches) delete sk;
  g_sketches.clear();
  g_inv_idx.reset();
  return rc;
}

// Runs pack -> b0 -> ranks/unit rows -> graph -> edge weights exactly as
// rb_cmd_bin does for a PMH run; winners32 holds the build_pmh_winners rows.
// unit_out (n*S floats, may be null) receives g_depth_unit.
int ref_run_graph(const RefParams *p, const uint32_t *winners32,
                  const float *depth_raw, float *unit_out, RefOut *out) {
  g_pmh_mode = true;
  return run_graph_body(p, winners32, depth_raw, unit_out, out);
}

}  // extern "C"

static int run_graph_body(const RefParams *p, const uint32_t *winners32,
                          const float *depth_raw, float *unit_out, RefOut *out) {
  nobs = (size_t)p->n;
  g_pmh_m = (uint32_t)p->m;
  sketch_size = g_pmh_m;
  g_inv_pmh_m = (g_pmh_m > 0) ? (1.0 / (double)g_pmh_m) : 0.0;
  num_depth_samples = (size_t)(p->S > 0 ? p->S : 0);
  depth_file = p->S > 0 ? "depth.tsv" : "";
  maxEdges = (size_t)p->max_edges;
  g_mutual_knn = p->mutual != 0;
  g_pmh_base_on = p->base_on != 0;
  numThreads = (size_t)(p->nthreads > 0 ? p->nthreads : 1);
  min_edge_weight = p->min_edge;
  minCV = p->min_cv;
  g_neg_depth_thr = p->neg_thr;
  g_depth_sim = p->depth_sim;
  g_depth_fuse = p->depth_fuse;
  // src/rabbitbin.cpp:4670-4673 (auto_w_comp: S<=2 -> 1, else 0)
  g_w_comp = (p->w_comp < 0.0) ? (num_depth_samples <= 2 ? 1.0 : 0.0) : p->w_comp;
  const size_t S = num_depth_samples;

  // depth_matrix rows in FASTA order; raw snapshot + column norm
  // (src/rabbitbin.cpp:4792-4809).
  depth_matrix.cols = S;
  depth_matrix.v.assign(depth_raw, depth_raw + nobs * S);
  g_depth_raw.clear();
  g_depth_colnorm.clear();
  if (g_depth_sim >= 1 && S > 1) {
    g_depth_raw.assign(depth_raw, depth_raw + nobs * S);
    if (p->wjac_norm) {
      g_depth_colnorm.assign(S, 1.0);
      for (size_t i = 0; i < S; ++i) {
        double s = 0.0;
        for (size_t r = 0; r < nobs; ++r) s += g_depth_raw[r * S + i];
        double mean = s / std::max<size_t>(nobs, 1);
        g_depth_colnorm[i] = (mean > 1e-12) ? 1.0 / mean : 0.0;
      }
    }
  }
  // In-place Spearman rank per row (src/rabbitbin.cpp:4867-4874).
  if (S > 1) {
    std::vector<float> rowMat(S);
    for (size_t r = 0; r < nobs; ++r) {
      for (size_t k = 0; k < S; ++k) rowMat[k] = depth_matrix(r, k);
      rank(rowMat, rowMat);
      for (size_t k = 0; k < S; ++k) depth_matrix(r, k) = rowMat[k];
    }
  }
  g_anynz.clear();
  build_anynz_cache();

  // 16-bit pack (src/rabbitbin.cpp:4934-4952).
  g_win_flat.clear();
  if (g_pmh_mode) g_win_flat.assign(winners32, winners32 + nobs * g_pmh_m);
  g_win16.clear();
  g_win_bits = 32;
  if (p->win_bits == 16 && !g_win_flat.empty()) {
    g_win16.resize(g_win_flat.size());
    for (size_t t = 0; t < g_win_flat.size(); ++t) g_win16[t] = fold_win16(g_win_flat[t]);
    g_win_bits = 16;
    std::vector<uint32_t>().swap(g_win_flat);
  }
  // b0 (src/rabbitbin.cpp:4958-4965).
  g_pmh_baseline = 0.0;
  g_inv_one_minus_b0 = 1.0;
  if (g_pmh_mode && g_pmh_base_on) {
    g_pmh_baseline = estimate_pmh_baseline(nobs);
    g_inv_one_minus_b0 = (g_pmh_baseline < 1.0) ? (1.0 / (1.0 - g_pmh_baseline)) : 1.0;
  }
  // Unit rank rows (src/rabbitbin.cpp:4972-4988).
  g_depth_unit.clear();
  if (S > 1) {
    g_depth_unit.assign(nobs * S, 0.0f);
    for (size_t r = 0; r < nobs; ++r) {
      double mean = 0.0;
      for (size_t k = 0; k < S; ++k) mean += depth_matrix(r, k);
      mean /= (double)S;
      double ss = 0.0;
      for (size_t k = 0; k < S; ++k) { double d = (double)depth_matrix(r, k) - mean; ss += d * d; }
      if (ss > 0.0) {
        const double inv = 1.0 / std::sqrt(ss);
        float *u = g_depth_unit.data() + r * S;
        for (size_t k = 0; k < S; ++k)
          u[k] = (float)(((double)depth_matrix(r, k) - mean) * inv);
      }
    }
    if (unit_out) std::copy(g_depth_unit.begin(), g_depth_unit.end(), unit_out);
  }

  // Graph (src/rabbitbin.cpp:5035-5054).
  if (p->no_abdfirst) setenv("RABBIT_NO_ABDFIRST", "1", 1);
  else unsetenv("RABBIT_NO_ABDFIRST");
  srand(p->seed);
  Graph g(nobs);
  double simCutoff = 0.0;
  const bool fused = (p->force_path == 2) || (p->force_path == 0 && nobs > 25000);
  if (fused && g_pmh_mode) {
    simCutoff = gen_fused_calib_graph(g, p->coverage);
  } else {
    // small N, or the one-permutation metric at large N (calibration on ten
    // 2500-contig samples, then the same all-pairs build), :5035-5054
    simCutoff = fused ? (double)calibrate_sim_cutoff_fused(p->coverage)
                      : (double)calibrate_sim_cutoff(p->coverage, true);
    if (g_use_index) build_similarity_graph(g, simCutoff / 1000.);
    else build_graph_allpairs(g, simCutoff / 1000.);
  }

  // Edge weights, default fixed-cutoff branch (src/rabbitbin.cpp:5482-5509
  // and the no-depth branch :5532-5536).  The GFA sentinel never occurs here.
  const size_t ne = g.getEdgeCount();
  g.edgeScore.assign(ne, 0.0f);
  if (S > 0) {
    for (size_t e = 0; e < ne; ++e) {
      size_t i = g.from[e], j = g.to[e];
      if (S <= 1) {
        g.edgeScore[e] = (StoredDistance)(double)g.sComp[e];
      } else {
        bool depth_ok;
        double dterm = depth_edge_term(i, j, depth_ok);
        if (!depth_ok) { g.edgeScore[e] = 0.0f; continue; }
        double sComp_v = g.sComp[e];
        double min_edge_weight_v = min_edge_weight;
        double w = g_w_comp * sComp_v + (1.0 - g_w_comp) * dterm;
        if (!std::isfinite(w) || w < min_edge_weight_v) w = 0.0;
        g.edgeScore[e] = (StoredDistance)w;
      }
    }
  } else {
    for (size_t e = 0; e < ne; ++e) {
      float s = g.sComp[e];
      if (s < min_edge_weight) s = 0.0f;
      g.edgeScore[e] = s;
    }
  }

  out->b0 = g_pmh_baseline;
  out->sim_cutoff = simCutoff;
  out->n_edges = (int64_t)ne;
  out->from = (uint32_t *)malloc(sizeof(uint32_t) * (ne + 1));
  out->to = (uint32_t *)malloc(sizeof(uint32_t) * (ne + 1));
  out->scomp = (float *)malloc(sizeof(float) * (ne + 1));
  out->score = (float *)malloc(sizeof(float) * (ne + 1));
  for (size_t e = 0; e < ne; ++e) {
    out->from[e] = g.from[e];
    out->to[e] = g.to[e];
    out->scomp[e] = g.sComp[e];
    out->score[e] = g.edgeScore[e];
  }
  return 0;
}

extern "C" {

// Float dot of two unit rows exactly as the abundance-first prune computes it.
float ref_unit_dot_f(const float *a, const float *b, uint32_t S) {
  return unit_dot_f(a, b, S);
}

// Full ProbMinHash4 state for one weighted element list (addHash order), for
// kernel-level parity of registers and winners.
// jaccard_weighted, jaccard, distance, ani of sketch A against sketch B (each
// built by addHash over its elements), through ProbMinHash4's own methods.
void ref_pmh_metrics(const uint64_t *ka, const double *wa, int64_t na, const uint64_t *kb,
                     const double *wb, int64_t nb, uint32_t m, uint64_t seed, int kmer,
                     double *out4) {
  Sketch::ProbMinHash4 a(m, kmer, seed), b(m, kmer, seed);
  for (int64_t t = 0; t < na; ++t) a.addHash(ka[t], wa[t]);
  for (int64_t t = 0; t < nb; ++t) b.addHash(kb[t], wb[t]);
  out4[0] = a.jaccard_weighted(b);
  out4[1] = a.jaccard(b);
  out4[2] = a.distance(b);
  out4[3] = a.ani(b);
}

void ref_pmh_elements(const uint64_t *keys, const double *weights, int64_t ne,
                      uint32_t m, uint64_t seed, double *regs_out,
                      uint64_t *winners_out) {
  Sketch::ProbMinHash4 pmh(m, 4, seed);
  for (int64_t t = 0; t < ne; ++t) pmh.addHash(keys[t], weights[t]);
  const double *r = pmh.getRegisters();
  const uint64_t *w = pmh.getWinners();
  for (uint32_t t = 0; t < m; ++t) { regs_out[t] = r[t]; winners_out[t] = w[t]; }
}

}  // extern "C"
