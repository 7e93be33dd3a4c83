/*
 * rabbitbin_b200 — C ABI of the B200 graph-construction hot path of RabbitBin.
 *
 * The reference has no plugin or FFI layer: its seams are C++ functions inside
 * one translation unit.  Each entry point below replaces one of them, keeps its
 * argument meaning, and adds only what a device boundary needs (a context that
 * owns the CUDA stream and device buffers, batching over contigs, an int status).
 *
 *   rbg_build_pmh_winners  ← build_pmh_winners            src/rabbitbin.cpp:1436-1589
 *                            (called per contig at :2164, :4375, :4854-4863)
 *   rbg_pack_win16         ← fold_win16 + pack loop       src/rabbitbin.cpp:249-253, :4934-4952
 *   rbg_estimate_pmh_baseline ← estimate_pmh_baseline     src/rabbitbin.cpp:1340-1369, :4958-4965
 *   rbg_build_graph        ← calibrate_sim_cutoff + build_similarity_graph (N <= 25000)
 *                            src/impl/rb_graph.cpp:1362-1384, :199-220, :7-72
 *                            gen_fused_calib_graph (N > 25000)  src/impl/rb_graph.cpp:501-1356
 *                            dispatched as at src/rabbitbin.cpp:5035-5054, followed by
 *                            the edge-weight loop src/rabbitbin.cpp:5482-5509
 *                            (depth_edge_term :930-970) on the same device state
 *   rbg_bin_graph          ← the whole hot path of rb_cmd_bin (sketch loop :4817-4882,
 *                            pack, b0, unit rows :4972-4988, graph, edge weights)
 *                            from sequences + coverage, without host round trips
 *
 * Conventions: all buffers are caller-owned host memory unless a name says
 * "device"; sizes are element counts; every function returns RBG_OK (0) or a
 * negative status and never throws.  rbg_last_error(ctx) describes the last
 * failure on that context.  Calls on one context are serialised; different
 * contexts may be used from different host threads.
 */
#ifndef RABBITBIN_B200_H
#define RABBITBIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  RBG_OK = 0,
  RBG_ERR_ARG = -1,        /* bad argument (reference: cerr + return 1)          */
  RBG_ERR_NOMEM = -2,      /* device or host allocation failed / over budget     */
  RBG_ERR_CUDA = -3,       /* CUDA runtime error                                 */
  RBG_ERR_UNSUPPORTED = -4,/* option value this build does not implement         */
  RBG_ERR_TIMEOUT = -5,    /* a bounded device wait gave up                      */
  RBG_ERR_COMM = -6        /* the caller's collective reported a failure         */
};

/* Options of `rabbitbin bin` and the hot-path RABBIT_* variables, with the
 * reference defaults (src/rabbitbin.cpp:3339-3445, :4660-4705). */
typedef struct rbg_params {
  int32_t k;              /* RABBIT_PMHK (4); 1..4 supported                       */
  int32_t m;              /* --sketch-m (500); 2..4096                             */
  uint64_t pmh_seed;      /* g_pmh_seed (42)                                       */
  int32_t gc_norm;        /* RABBIT_GC_NORM (1); 0, 1 and 2                        */
  int32_t win_bits;       /* RABBIT_WIN_BITS (16) or 32                            */
  double gc_norm_cap;     /* RABBIT_GC_NORM_CAP (20)                               */
  int32_t max_edges;      /* --max-edges (200)                                     */
  int32_t mutual;         /* RABBIT_MUTUAL_KNN (1)                                 */
  int32_t base_on;        /* RABBIT_PMH_BASE (1)                                   */
  uint32_t seed;          /* --seed, the srand() seed of the calibration (1)       */
  int32_t force_path;     /* 0: N > 25000 -> fused path as the reference; 1 small; 2 fused */
  int32_t abdfirst;       /* 1 unless RABBIT_NO_ABDFIRST is set                    */
  double coverage;        /* --max-posterior / 100 (0.95)                          */
  double min_edge;        /* --min-edge-score / 100 (0.70)                         */
  double w_comp;          /* RABBIT_W_COMP, < 0 = auto (S <= 2 -> 1, else 0)       */
  double min_cv;          /* --min-coverage (1.0)                                  */
  double neg_thr;         /* RABBIT_NEG_DEPTH (-0.3)                               */
  int32_t depth_sim;      /* RABBIT_DEPTH_SIM: 0 corr, 1 wjac, 2 fuse (2)          */
  int32_t depth_fuse;     /* RABBIT_DEPTH_FUSE: 0 geo-mean, 1 min, 2 product (1)   */
  int32_t wjac_norm;      /* RABBIT_DEPTH_WJAC_NORM (1)                            */
  int32_t fp_contract;    /* 1: arithmetic of the reference's release build, where
                             GCC contracts a*b+c into FMA; 0: -ffp-contract=off   */
  double wjac_cut;        /* RABBIT_DEPTH_WJAC_CUT (0)                             */
  int32_t wjac_gate;      /* RABBIT_DEPTH_WJAC_GATE (0)                            */
  int32_t oph_k;          /* 0: ProbMinHash composition similarity (RABBIT_PMH, the
                             default); > 0: RABBIT_PMH=0, the one-permutation
                             MinHash metric of rabbit_sketch.h with k-mers of this
                             size (sketch_kmer_size, 8; 1..32) and m buckets     */
  int32_t oph_bits;       /* sketch_bits: bit-planes per OPH bucket (2; 1..7)      */
  int32_t graph_index;    /* RABBIT_GRAPH_INDEX (0): 1 restricts the small path's
                             neighbours to contigs sharing >= min_common
                             one-permutation sketch keys (build_similarity_graph,
                             src/impl/rb_graph.cpp:199-383); rbg_bin_graph, or
                             rbg_bin_batch through the single-assembly path */
  int32_t index_k;        /* sketch_kmer_size of the index's sketches (8; 1..32;
                             oph_k when the one-permutation metric is on)      */
  int32_t min_common;     /* RABBIT_MINCOMMON (0: floor(cutoff * m * 0.7), >= 1)  */
  int32_t reserved;
} rbg_params;

/* Graph + edge weights (the reference Graph's from/to/sComp/edgeScore,
 * src/rabbitbin.h:264-301), sorted by (from, to).  Arrays are allocated by the
 * library; release them with rbg_free_graph. */
typedef struct rbg_graph {
  int64_t n_edges;
  uint32_t *from;
  uint32_t *to;
  float *scomp;           /* composition similarity sComp                          */
  float *score;           /* edgeScore                                             */
  double b0;              /* g_pmh_baseline                                        */
  double sim_cutoff;      /* simCutoff as the reference returns it (x1000 units)   */
  int32_t path;           /* 1 small-N path, 2 fused large-N path                  */
  int32_t reserved;
} rbg_graph;

/* Per-stage device time of the last rbg_bin_graph / rbg_run_resident call. */
typedef struct rbg_timing {
  float pack_ms, count_ms, sketch_ms, unit_ms, b0_ms, allpairs_ms, finalize_ms,
        emit_ms, weight_ms, total_ms;
  int64_t pairs_prefiltered;   /* ordered pairs through the abundance test      */
  int64_t pairs_compared;      /* ordered pairs through the register compare    */
  int32_t kernel_launches;     /* kernels launched by the call                  */
  int32_t reserved;
} rbg_timing;

typedef struct rbg_ctx rbg_ctx;

/* Fill *p with the reference defaults. */
int rbg_default_params(rbg_params *p);

/* Create a context on CUDA device `device` (owns a stream and device buffers). */
int rbg_create(int device, rbg_ctx **out);
int rbg_destroy(rbg_ctx *ctx);
const char *rbg_last_error(rbg_ctx *ctx);
/* cudaStream_t of the context, as void*, for callers that time or order work. */
void *rbg_stream(rbg_ctx *ctx);

/* build_pmh_winners for n contigs.  seqcat holds the ASCII sequences back to
 * back, contig r = seqcat[offsets[r], offsets[r+1]).  out_winners32 (n*m) gets
 * the 64->32-bit folded winner rows (src/rabbitbin.cpp:1582-1588). */
int rbg_build_pmh_winners(rbg_ctx *ctx, const rbg_params *p, const char *seqcat,
                          const int64_t *offsets, int64_t n,
                          uint32_t *out_winners32);

/* ── ProbMinHash4 sketches and queries (src/probmh.h:103-283) ────────────
 * rbg_build_pmh_sketches: the ProbMinHash4(m, k, pmh_seed) sketch that
 * build_pmh_winners builds per contig (src/rabbitbin.cpp:1436-1589), as
 * ProbMinHash4::getWinners() (out_winners64 [n][m]: RNG state of the element
 * that won each register, 0 unset; the out64 argument of build_pmh_winners)
 * and ProbMinHash4::getRegisters() (out_registers [n][m]: register values,
 * +inf unset).  Either output may be NULL.  The ProbMinHash metric only. */
int rbg_build_pmh_sketches(rbg_ctx *ctx, const rbg_params *p, const char *seqcat,
                           const int64_t *offsets, int64_t n, uint64_t *out_winners64,
                           double *out_registers);

/* Many-vs-many sketch comparison: out[i * nb + j] = metric(A_i, B_j) for row
 * sets A [na][m] and B [nb][m], exactly as the ProbMinHash4 method of sketch
 * A_i called on B_j:
 *   RBG_PMH_JACCARD_WEIGHTED  jaccard_weighted (src/probmh.cpp:1364-1376):
 *                             rows are winners (uint64_t), equal and nonzero
 *   RBG_PMH_JACCARD           jaccard (:1325-1362): rows are register values
 *                             (double), equal and finite
 *   RBG_PMH_DISTANCE          distance (:1378-1385) = -ln(2J/(1+J)) / kmer_size
 *   RBG_PMH_ANI               ani (:1404-1410) = (2J/(1+J))^(1/kmer_size)
 * (J = jaccard for the last two; kmer_size is the sketch's k, 4 for the
 * winners build_pmh_winners makes). */
enum {
  RBG_PMH_JACCARD_WEIGHTED = 0,
  RBG_PMH_JACCARD = 1,
  RBG_PMH_DISTANCE = 2,
  RBG_PMH_ANI = 3
};
int rbg_pmh_compare(rbg_ctx *ctx, int32_t metric, int32_t m, int32_t kmer_size, const void *A,
                    int64_t na, const void *B, int64_t nb, double *out);

/* ProbMinHash4::merge (src/probmh.cpp:1416-1440) of n pairs of register rows:
 * out[i][r] = min(A[i][r], B[i][r]) (the merged sketch's getRegisters()). */
int rbg_pmh_merge_registers(rbg_ctx *ctx, const double *A, const double *B, int64_t n,
                            int32_t m, double *out);

/* One-permutation MinHash signatures (the RABBIT_PMH=0 metric): replaces
 * rabbit_sketch::KmerSketch(m, oph_k, oph_bits).update(seq, len) followed by
 * getSignature() (src/rabbit_sketch.h:197-285) for n contigs.  out[n][m]
 * receives each bucket's value: bit p of out[i][r] is bit r of bit-plane p of
 * contig i's signature (a densified bucket's borrowed value; 0 for every
 * bucket of a contig with no valid k-mer).  Requires p->oph_k in 1..32. */
int rbg_build_oph_signature(rbg_ctx *ctx, const rbg_params *params, const char *seqcat,
                            const int64_t *offsets, int64_t n, uint8_t *out);

/* fold_win16 over `count` folded winners (src/rabbitbin.cpp:249-253). */
int rbg_pack_win16(rbg_ctx *ctx, const uint32_t *in, int64_t count, uint16_t *out);

/* estimate_pmh_baseline over n winner rows of width p->m; `winners` is
 * uint16_t[n*m] when win_bits == 16, else uint32_t[n*m]. */
int rbg_estimate_pmh_baseline(rbg_ctx *ctx, const rbg_params *p,
                              const void *winners, int32_t win_bits, int64_t n,
                              double *out_b0);

/* Graph + edge weights from folded 32-bit winner rows (n*m) and the raw
 * coverage means depth (n*S floats, S = 0 for no depth file). */
int rbg_build_graph(rbg_ctx *ctx, const rbg_params *p, const uint32_t *winners32,
                    int64_t n, const float *depth, int32_t S, rbg_graph *out);

/* The whole hot path: sequences + coverage -> graph with edge weights. */
int rbg_bin_graph(rbg_ctx *ctx, const rbg_params *p, const char *seqcat,
                  const int64_t *offsets, int64_t n, const float *depth,
                  int32_t S, rbg_graph *out);

/* ── FASTA ingest on the device ───────────────────────────────────────────
 * parse_fasta_mmap_parallel (src/rabbitbin.cpp:1890-2248) as rb_cmd_bin calls
 * it for binning: records start at the first '>' of a line, names end at the
 * first byte <= ' ', multi-line bodies lose their newlines and one '\r' per
 * line, records of length >= min_contig are large, >= min_small_contig small,
 * shorter ones dropped; num_seqs counts every record with a header line.
 * Large and small contigs come back in file order, sequences back to back
 * (offsets n + 1), names as byte ranges of the input.  Free with
 * rbg_free_fasta. */
typedef struct rbg_fasta {
  int64_t num_seqs, n_large, n_small;
  char *large_seq;  int64_t *large_off;  int64_t *large_name_start;  int32_t *large_name_len;
  char *small_seq;  int64_t *small_off;  int64_t *small_name_start;  int32_t *small_name_len;
} rbg_fasta;

int rbg_parse_fasta(rbg_ctx *ctx, const char *fasta, int64_t nbytes, int64_t min_contig,
                    int64_t min_small_contig, rbg_fasta *out);
int rbg_free_fasta(rbg_fasta *f);

/* The whole hot path from a FASTA file's bytes: the device parse, then the
 * large contigs (>= min_contig) go straight into rbg_bin_graph's pipeline
 * without a host round trip of the sequences.  depth: n_large x S coverage
 * means of the large contigs in file order. */
int rbg_bin_fasta(rbg_ctx *ctx, const rbg_params *p, const char *fasta, int64_t nbytes,
                  int64_t min_contig, const float *depth, int32_t S, rbg_graph *out);

/* ── one assembly over several GPUs ────────────────────────────────────────
 * No counterpart in the reference (one process on one host).  The caller
 * supplies the collective: gather `bytes` from every rank into recv, rank r's
 * block at recv + r * bytes, complete when the function returns; return 0 on
 * success.  With device_buffers set, send and recv are memory of the
 * context's device (NCCL over NVLink/NVSwitch); otherwise pinned host memory
 * (gloo, MPI, sockets). */
typedef int (*rbg_allgather_fn)(const void *send, void *recv, size_t bytes, void *user);

typedef struct rbg_shard {
  int32_t rank, world;
  int32_t device_buffers;
  int32_t reserved;
  rbg_allgather_fn allgather;
  void *user;
} rbg_shard;

/* rbg_bin_graph for one assembly split into contiguous row ranges: rank r
 * passes its n_local contigs (ranks in contig order) and their coverage rows.
 * It sketches them; the ranks gather the register codes and coverage rows.
 * In the abundance-pruned regime (the fused path with S > 1) each rank runs
 * its share of the symmetric pass (every unordered pair scored by one rank),
 * the ranks gather their admitted pairs and partial row maxima, and every
 * rank selects every row's top-K from the whole list; otherwise each rank
 * scores the full rows of its contigs and the ranks gather the row maxima and
 * the neighbour lists.  The rank returns the edges whose `from` is one of its
 * contigs, with global contig ids and weights; the ranks' edges concatenated
 * in rank order are rbg_bin_graph's graph of the whole assembly.  Every rank
 * calls with the same params and S; the collective is called five times per
 * call (two more for each rerun after a pair list overflowed on some rank),
 * in the same order on every rank. */
int rbg_bin_graph_sharded(rbg_ctx *ctx, const rbg_params *p, const rbg_shard *sh,
                          const char *seqcat, const int64_t *offsets, int64_t n_local,
                          const float *depth, int32_t S, rbg_graph *out);

/* ── batching: many assemblies per launch ─────────────────────────────────
 * No counterpart in the reference, which bins one assembly per process
 * (rb_cmd_bin, src/rabbitbin.cpp:4660-5622).  Each assembly's graph equals
 * rbg_bin_graph on that assembly alone (same edges, same weights). */
typedef struct rbg_assembly {
  const char *seqcat;          /* host ASCII contigs back to back              */
  const int64_t *offsets;      /* n + 1 offsets into seqcat, offsets[0] == 0   */
  int64_t n;                   /* contigs                                      */
  const float *depth;          /* n x S coverage means (NULL when S == 0)      */
  int32_t S;                   /* coverage samples                             */
  int32_t reserved;
  const rbg_params *params;    /* NULL: the call's default parameters          */
} rbg_assembly;

typedef struct rbg_batch_stats {
  float stage_ms;              /* input copies with, behind them, each run of
                                  assemblies' sketch, depth rows, b0, all-pairs
                                  and dense GEMMs (device)                      */
  float graph_ms;              /* row top-K of the symmetric pass, and the
                                  resident rerun if its pair list overflowed    */
  float calib_ms;              /* cutoff calibration of every assembly (host)   */
  float emit_ms;               /* edges + weights + copies back (device)        */
  float total_ms;              /* the whole call (host clock)                   */
  int32_t n_assemblies;
  int32_t kernel_launches;     /* kernels in the call's launch sequence          */
  int32_t graph_launches;      /* CUDA graph launches (0 with RBG_NO_GRAPHS set) */
  int32_t tuned_keys;          /* (variant, m, log2 n) keys whose all-pairs tile
                                  shape the autotuner chose in this call: the
                                  first call that meets a key times 3 shapes
                                  (RBG_NO_AUTOTUNE set: none, the fixed rule)   */
  int64_t rows;                /* contigs over all assemblies                   */
  int64_t pairs;               /* contig pairs scored, sum of n (n - 1) / 2     */
  int64_t items;               /* all-pairs work items (32 rows x 4 slices)     */
  int64_t edges;
} rbg_batch_stats;

/* Sketch and graph n_asm assemblies together: one pass of every kernel over
 * all of them (persistent all-pairs kernels pull (assembly, row block)
 * items from a device queue; each stage's launches form one CUDA graph) and
 * one host round trip for all calibrations.  out[i] (n_asm entries) receives
 * assembly i's graph; free each with rbg_free_graph.  `stats` may be NULL and
 * covers the batched assemblies.  Assemblies on the one-permutation metric
 * (oph_k > 0) or the inverted-index graph (graph_index) have no batch kernels:
 * they run one after the other through rbg_bin_graph's path in the same call. */
int rbg_bin_batch(rbg_ctx *ctx, const rbg_params *defaults, const rbg_assembly *asms,
                  int32_t n_asm, rbg_graph *out, rbg_batch_stats *stats);

/* ── serving: a request loop over a stream of assemblies ──────────────────
 * No counterpart in the reference.  Requests are queued on submit in two size
 * classes (small: at most small_pairs contig pairs).  Each lane is a worker
 * thread with its own device context: lane 0 serves large requests first and
 * small ones when no large one waits, the other lanes serve small requests
 * only.  A lane that becomes free folds every queued request of its class
 * that fits into the HBM budget the running batches leave (a batch's share is
 * released when it finishes) into one batch: small requests through one
 * rbg_bin_batch call, large ones through rbg_bin_graph each.  Requests that
 * arrive while others are on the GPU are therefore admitted as soon as a lane
 * of their class and the memory are free, small requests never wait behind a
 * large batch, and the lanes' batches overlap on the device.  Each result
 * equals rbg_bin_graph on that assembly alone. */
typedef struct rbg_server rbg_server;

typedef struct rbg_server_config {
  int32_t device;              /* CUDA device                                   */
  int32_t workers;             /* lanes (contexts, concurrent batches); 0 -> 2  */
  int64_t hbm_budget;          /* bytes of device memory for request state;
                                  0 -> 150 GB, capped at the free memory        */
  int32_t max_batch;           /* assemblies folded into one launch; 0 -> 64    */
  int32_t plain;               /* 1: one rbg_bin_graph call per request, one
                                  worker (the unbatched comparison path)        */
  int64_t max_batch_pairs;     /* fold requests while the batch's contig pairs
                                  stay below this (a larger request runs alone);
                                  0 -> 2e9                                      */
  int64_t small_pairs;         /* requests with at most this many contig pairs
                                  are small; 0 -> 2e8 (about 20,000 contigs)    */
} rbg_server_config;

typedef struct rbg_request_stats {
  double queue_ms;             /* submit -> start of its batch                  */
  double service_ms;           /* start of its batch -> result                  */
  double latency_ms;           /* submit -> result                              */
  int32_t batch_size;          /* assemblies in the batch it ran in             */
  int32_t worker;
  int64_t est_bytes;           /* device bytes reserved for it at admission     */
  double submit_s;             /* submit time, seconds since rbg_server_create  */
  double done_s;               /* result time, seconds since rbg_server_create  */
} rbg_request_stats;

int rbg_server_create(const rbg_server_config *cfg, const rbg_params *defaults,
                      rbg_server **out);
/* Queue one assembly.  The arrays a->seqcat, a->offsets and a->depth must stay
 * valid until rbg_server_wait returns for this request; a->params (if set) is
 * copied.  Validation errors are returned here. */
int rbg_server_submit(rbg_server *srv, const rbg_assembly *a, int64_t *request_id);
/* Wait up to timeout_s seconds (< 0: forever) for a request's graph.  Returns
 * RBG_ERR_TIMEOUT if it is not done yet (it stays queued), else the request's
 * status; on RBG_OK *out owns the edges (free with rbg_free_graph).  A request
 * can be waited for once after it completes.  `stats` may be NULL. */
int rbg_server_wait(rbg_server *srv, int64_t request_id, double timeout_s, rbg_graph *out,
                    rbg_request_stats *stats);
/* Last error message of the server (submit-time validation, device errors). */
const char *rbg_server_last_error(rbg_server *srv);
/* Stops accepting work, finishes queued requests, frees the contexts. */
int rbg_server_destroy(rbg_server *srv);

/* ── RBCACHE1 v3: the on-disk state of a built graph ──────────────────────
 * rb_write_cache / rb_load_cache (src/impl/rb_cache.cpp:103-319): the state
 * RabbitBin keeps after the expensive stages so that a later run (or a
 * restarted server) goes straight to the cheap tail.  The file is byte for
 * byte the one the reference writes for the same state and is readable by
 * either program; reading also accepts versions 1 and 2.  Names are bytes
 * back to back with n + 1 offsets; matrices are row-major floats (the ranked
 * depth matrix of the large contigs, the raw one of the small contigs).
 * rbg_read_cache allocates every array (free with rbg_free_cache). */
typedef struct rbg_cache {
  int64_t n_large, n_small, samples;            /* nobs, nobs1, num_depth_samples */
  uint64_t seed, total_size, total_size_small;  /* --seed, totalSize, totalSize1  */
  double sim_cutoff, b0;                        /* simCutoff, g_pmh_baseline      */
  uint64_t min_contig, min_small_contig;
  int32_t has_depth, has_snv;
  char *large_names;   int64_t *large_name_off;   int64_t n_large_names;
  char *small_names;   int64_t *small_name_off;   int64_t n_small_names;
  uint64_t *large_len; int64_t n_large_len;      /* seq_lens                       */
  uint64_t *small_len; int64_t n_small_len;      /* small_seq_lens                 */
  float *depth_ranked; int64_t depth_rows, depth_cols;              /* depth_matrix */
  float *small_depth;  int64_t small_depth_rows, small_depth_cols;  /* small_depth_matrix */
  float *large_means;  int64_t n_large_means;    /* g_large_means                  */
  float *depth_raw;    int64_t n_depth_raw;      /* g_depth_raw                    */
  double *colnorm;     int64_t n_colnorm;        /* g_depth_colnorm                */
  uint32_t *from, *to; float *scomp; int64_t n_edges;   /* the graph              */
  float *snv_pi; uint32_t *snv_nsnv, *snv_cov; int64_t n_snv;   /* --strain block */
  int32_t version;                               /* read: the file's version       */
  int32_t reserved;
} rbg_cache;

/* Write the state (names, lengths and vectors with a null pointer are written
 * as empty; the SNV block only with has_snv and n_snv > 0). */
int rbg_write_cache(const char *path, const rbg_cache *state);
/* Read a cache written by either program (RBG_ERR_ARG: missing, truncated or
 * corrupt file; RBG_ERR_UNSUPPORTED: other version or ABI). */
int rbg_read_cache(const char *path, rbg_cache *out);
int rbg_free_cache(rbg_cache *c);

/* Device-resident form used by batching, serving and the benchmark: stage the
 * inputs once (host -> device), run the hot path on them any number of times,
 * then fetch the graph (device -> host). */
int rbg_stage(rbg_ctx *ctx, const char *seqcat, const int64_t *offsets,
              int64_t n, const float *depth, int32_t S);
int rbg_run_resident(rbg_ctx *ctx, const rbg_params *p, rbg_timing *timing);
int rbg_fetch_graph(rbg_ctx *ctx, rbg_graph *out);

int rbg_free_graph(rbg_graph *g);

/* rbg_build_pmh_winners for callers that cannot allocate device memory (a host
 * framework that owns the device heap through its own pool, a plugin inside
 * another process's CUDA context with a fixed budget, a caller that must not
 * synchronise on an allocation).  No counterpart in the reference: it is the
 * same sketch, but inputs and outputs are caller-owned DEVICE buffers and every
 * intermediate lives in one static 24 MiB device array that the library
 * reserves on each GPU that loads it (held until exit).  seq_device is the
 * concatenated ASCII (16-byte aligned, readable up to a multiple of 16 bytes),
 * offsets_device the n+1 base offsets, which must start at 0, end at nbases
 * and never decrease (checked on the device: RBG_ERR_ARG otherwise, before any
 * sketch work), winners_device n*m folded 32-bit winner rows.  Parameters as
 * rbg_build_pmh_winners: k 1..4, m 2..4096, gc_norm 0..2, the ProbMinHash
 * metric only (oph_k = 0).  Requests needing more scratch than the array
 * holds (roughly > 4,000 contigs or > 40 Mbp per call at m = 500) return
 * RBG_ERR_ARG (message in errbuf) before any device work.  The first call on
 * a device looks up the array's address.  Every call reads a check flag back
 * and synchronises `stream`, so it must never be called while that stream is
 * being captured.  Calls share the array; calls that overlap on the GPU race.
 * `stream` is a cudaStream_t (null: the default stream); the call returns
 * after the work has finished on it. */
int rbg_build_pmh_winners_noalloc(const rbg_params *p, const char *seq_device,
                                  const int64_t *offsets_device, int64_t n, int64_t nbases,
                                  uint32_t *winners_device, void *stream, char *errbuf,
                                  size_t errlen);

/* Introspection (host only, no device needed): the ProbMinHash element streams
 * the sketch kernel reduces over for one configuration.  For every canonical
 * k-mer e (ascending code canon_codes[e]) and register r, U[e*m + r] is the
 * weight-free value e offers to r (the offer is (1/w) * U) and W32[e*m + r]
 * the folded winner it leaves there.  Call with null arrays to read *n_elems.
 * Replaces nothing in the reference: ProbMinHash4 (src/probmh.cpp:634-686)
 * draws these values inline for each element of each contig. */
int rbg_pmh_stream_tables(int32_t k, int32_t m, uint64_t pmh_seed, int32_t fp_contract,
                          int32_t *n_elems, int32_t *canon_codes, double *U, uint32_t *W32);

/* ── Fisher label propagation: the step after the graph ───────────────────
 *   rbg_label_propagation ← the incidence build src/rabbitbin.cpp:5597-5622
 *                           (edges with edgeScore > 0, clamped to 1 - 1e-6f,
 *                           lists ordered by neighbour id), the node order
 *                           :5643-5645 (std::shuffle of 0..n-1 with
 *                           std::default_random_engine(seed)) and
 *                           cluster_by_propagation src/impl/rb_cluster.cpp:376-740
 * Score rules of RABBIT_LPA_SCORE (rb_cluster.cpp:40-70); RABBIT_PAR_LPA
 * selects the synchronous sweep (:490-594), otherwise the sequential
 * (Gauss-Seidel) sweep in node order (:596-714), both until a round changes no
 * label.  membership[v] is v's label (a node id), identity for nodes without
 * edges; with no edges at all every node keeps its own label (the reference
 * returns early there, :381-385).  Status: RBG_ERR_ARG for a negative score
 * ("edgeScore must be non-negative", :441-444) or an endpoint >= n_nodes.
 * The Louvain, fused and multilevel variants of RABBIT_CLUSTER and the seed
 * ensemble are not built. */
enum {
  RBG_LPA_FISHER = 0,   /* chi2 CDF of -2 sum log(1 - w) (default)               */
  RBG_LPA_TAIL = 1,     /* minus the chi2 upper tail                              */
  RBG_LPA_LOGSUM = 2,   /* sum of -log(1 - w)                                     */
  RBG_LPA_SUM = 3,      /* sum of w                                               */
  RBG_LPA_MEAN = 4,     /* sum of w / count                                       */
  RBG_LPA_MAX = 5       /* max w                                                  */
};

typedef struct rbg_lpa_params {
  uint64_t seed;                /* --seed: the node order                            */
  const uint32_t *node_order;   /* or an explicit order (a permutation of 0..n-1)    */
  int32_t score_rule;           /* RBG_LPA_* (RABBIT_LPA_SCORE)                      */
  int32_t synchronous;          /* RABBIT_PAR_LPA                                    */
  int32_t max_rounds;           /* 0: until converged (the reference has no limit)   */
  int32_t reserved;
} rbg_lpa_params;

typedef struct rbg_lpa_stats {
  int32_t rounds;               /* sweeps run, the last one without a change         */
  int32_t reserved;
  int64_t changes;              /* label changes over all rounds                     */
  int64_t frozen;               /* nodes frozen by the cycle guard                   */
  int64_t arcs;                 /* incidence entries (2 x edges with a score > 0)    */
  float incidence_ms;           /* device time: incidence lists                      */
  float sweep_ms;               /* device time: all rounds                           */
} rbg_lpa_stats;

/* Reference defaults: seed 1 (the bin command's default), the rule and the
 * sweep from RABBIT_LPA_SCORE / RABBIT_PAR_LPA as the reference reads them. */
int rbg_default_lpa_params(rbg_lpa_params *lp);
/* On a host edge list (n_edges entries each of from, to, edge_score). */
int rbg_label_propagation(rbg_ctx *ctx, const rbg_lpa_params *lp, int64_t n_nodes,
                          int64_t n_edges, const uint32_t *from, const uint32_t *to,
                          const float *edge_score, uint32_t *membership, rbg_lpa_stats *stats);
/* On the graph of the context's last rbg_bin_graph / rbg_run_resident call,
 * still on the device (no edge copy); n_nodes is that call's contig count. */
int rbg_label_propagation_resident(rbg_ctx *ctx, const rbg_lpa_params *lp, uint32_t *membership,
                                   rbg_lpa_stats *stats);

/* ── BAM -> depth: the step before the path when the bin command gets BAMs ──
 *   rbg_bam_depth ← compute_depth_tsv_inmem with a DepthMatrixOut
 *                   (src/rabbit_depth_fuse.h:114-123, src/rabbit_depth.cpp:1096-1535),
 *                   as the bin command calls it (src/rabbitbin.cpp:3806-3811):
 *                   means only (intraDepthVariance = false), edges excluded
 *   rbg_depth_accumulate ← depth_accumulate_sample (src/rabbit_depth_fuse.h:72-75,
 *                   src/rabbit_depth.cpp:1615-1685) on records already in memory
 * Per read: the filters of src/rabbit_depth.cpp:1656-1667 (mapped, mate on a
 * known contig when paired, not secondary / QC-fail / duplicate, MAPQ >=
 * min_map_qual), the end check and clip of src/CheckRead.hpp:82-265, the
 * covered bases of caldepth (src/rabbit_depth.h:618-887: aligned M/=/X bases
 * minus the edge bases and the NM-derived substitutions) and the percent
 * identity of ReadStatistics (:193-346), kept when >= percent_identity.
 * edge = include_edge_bases ? 0 : min(max_edge_bases, avg_read / 3), avg_read
 * being the integer mean query length of the first 4,000 mapped records of
 * that BAM (:787-834).  Mean of (contig, BAM) = sum / (len - 2 edge) for
 * contigs longer than 2 edge + 1 (else sum / len), 0 for len <= 2, values above
 * 1e6 set to 0 (:1515-1534).  Rows: the contigs of the first BAM's header with
 * length >= min_contig_length, in header order; columns: one per BAM, then
 * with dual_map_qual > 0 a second block of the reads with MAPQ >= dual_map_qual.
 * Every BAM must carry the same contigs.  Records must be complete and
 * consistent (block_size, name, CIGAR, sequence and qualities inside the
 * record): a malformed record or BGZF block returns RBG_ERR_ARG (the reference
 * stops reading that file there).  CIGARs of more than 65,535 ops (the CG tag)
 * are taken as stored. */
typedef struct rbg_depth_params {
  float percent_identity;       /* --percent-identity / 100 (0.97)                   */
  int32_t min_contig_length;    /* rows: contigs at least this long (1)              */
  int32_t max_edge_bases;       /* 75                                                */
  int32_t include_edge_bases;   /* 0                                                 */
  int32_t min_map_qual;         /* 0                                                 */
  int32_t dual_map_qual;        /* 0: off                                            */
  int32_t threads;              /* host threads (0: all)                             */
  int32_t chunk_mb;             /* host route: decompressed MiB per hand-over (64)   */
  int32_t device_inflate;       /* 1: BGZF blocks inflated on the device (default);
                                   0: on the host threads                          */
  int32_t device_chunk_mb;      /* device route: decompressed MiB per chunk (1024)   */
} rbg_depth_params;

typedef struct rbg_depth_matrix {
  int64_t n_rows;               /* kept contigs                                      */
  int32_t n_cols;               /* BAMs (x 2 with dual_map_qual)                     */
  int32_t n_targets;            /* contigs in the header                             */
  int32_t *tid;                 /* [n_rows] header index of each row                 */
  int32_t *lens;                /* [n_rows]                                          */
  float *means;                 /* [n_rows][n_cols] row-major                        */
  char *names;                  /* the rows' names, each NUL-terminated              */
  int64_t *name_off;            /* [n_rows] offset of each name in `names`           */
  int32_t *avg_read;            /* [n_bams]                                          */
  uint64_t *sums;               /* [n_cols][n_targets] depth sums (CountType)        */
  int64_t records;              /* records read over all BAMs                        */
  int64_t compressed_bytes;     /* BGZF bytes read                                   */
  int64_t decompressed_bytes;   /* bytes after inflation                             */
  float inflate_ms;             /* host time inflating and walking records           */
  float total_ms;               /* host time of the whole call                       */
  float kernel_ms;              /* device time of the launches (inflate, walk, sums) */
  int32_t device_bams;          /* BAMs that took the device route                   */
} rbg_depth_matrix;

int rbg_default_depth_params(rbg_depth_params *p);
/* BAM files by path. */
int rbg_bam_depth(rbg_ctx *ctx, const char *const *bam_paths, int32_t n_bams,
                  const rbg_depth_params *p, rbg_depth_matrix *out);
/* BAM files already in host memory (whole files, BGZF as on disk). */
int rbg_bam_depth_mem(rbg_ctx *ctx, const uint8_t *const *bam_bytes, const int64_t *bam_sizes,
                      int32_t n_bams, const rbg_depth_params *p, rbg_depth_matrix *out);
int rbg_free_depth_matrix(rbg_depth_matrix *m);
/* The MetaBAT / JGI depth table of a matrix from rbg_bam_depth*: the TSV that
 * compute_depth_tsv_inmem returns without a DepthMatrixOut (printDepthTable,
 * src/rabbit_depth.cpp:125-313, called at :1589-1593), byte for byte.  Header
 * "contigName contigLen totalAvgDepth" and each BAM's base name (with a "-var"
 * column when intra_depth_variance); one row per matrix row: the name up to
 * its first blank, the length, the corrected-length-weighted total depth and
 * each BAM's mean, printed as "%g" of the float value.  Without the variance
 * columns each mean is the integer quotient sum / corrected length, corrected
 * length = len - 2 min(min(max_edge_bases, min avg_read / 3), avg_read / 3)
 * (len when edges are included or that reaches the whole contig); with them,
 * the matrix's mean and a variance of 0, as the reference computes them.
 * Means above 1e6 print as 0.  bam_names: the n_bams file names for the
 * header; the unique-read block of a dual matrix is not part of the table.
 * Host only; free *tsv with rbg_free_tsv. */
int rbg_depth_tsv(const rbg_depth_matrix *m, const char *const *bam_names, int32_t n_bams,
                  const rbg_depth_params *p, int32_t intra_depth_variance, char **tsv,
                  int64_t *tsv_len);
int rbg_free_tsv(char *tsv);
/* One sample's sums from decompressed records (each: block_size, then the
 * record, back to back) on host memory; depth_out[n_targets] receives the
 * sums of the reads with MAPQ >= min_map_qual, depth_u_out (may be null) those
 * with MAPQ >= dual_map_qual; *avg_read the sampled read length. */
int rbg_depth_accumulate(rbg_ctx *ctx, const uint8_t *records, int64_t n_bytes,
                         const uint32_t *target_len, int32_t n_targets,
                         const rbg_depth_params *p, uint64_t *depth_out, uint64_t *depth_u_out,
                         int32_t *avg_read);

#ifdef __cplusplus
}
#endif

#endif /* RABBITBIN_B200_H */
