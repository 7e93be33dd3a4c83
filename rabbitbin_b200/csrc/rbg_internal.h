// Internal declarations shared by the host engine and the CUDA kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rabbitbin_b200.h"

namespace rbg {

// Largest element universe handled with 8-bit register codes: the canonical
// k-mers of k <= 4 (136 for k = 4).
constexpr int kMaxElems = 136;
constexpr int kMaxM = 4096;
constexpr int kMaxS = 64;          // coverage samples held in registers
constexpr int kRowsPerCta = 32;    // rows of one all-pairs CTA (one per lane)

// ── PMH element streams (host, pmh_streams.cpp) ─────────────────────────────
// For one sketch configuration (k, m, seed, arithmetic mode) every canonical
// k-mer e has a fixed ProbMinHash stream: the register it visits at each step
// and the weight-independent part U of the value it offers there
// (hv = (1/w) * U).  Tables are indexed [e][register].
// One entry of a register's visiting order: the elements of register r sorted
// by ascending U[e][r], ties by ascending e (16 bytes, one vector load).
struct RegOrder {
  double u;
  uint32_t e;
  uint32_t pad;
};

struct PmhTables {
  int k = 0, m = 0, n_elems = 0, contract = 1;
  uint64_t seed = 0;
  std::vector<int> canon_codes;        // ascending canonical codes, size n_elems
  std::vector<int> rank_of_code;       // 4^k -> element index or -1
  std::vector<double> U;               // [n_elems][m]
  std::vector<RegOrder> order;         // [m][n_elems] visiting order per register
  std::vector<double> UT;              // [m][n_elems] U by register, then element
  std::vector<uint64_t> W64;           // [n_elems][m] winner (RNG state)
  std::vector<uint32_t> W32;           // folded h ^ (h >> 32)
  std::vector<uint16_t> W16;           // fold_win16(W32)
  std::vector<uint8_t> code16;         // 8-bit code of W16 per column (0 = unset)
  std::vector<uint8_t> code32;         // 8-bit code of W32 per column (0 = unset)
};

// Builds (or returns the cached) tables for (k, m, seed, contract).
std::shared_ptr<const PmhTables> pmh_tables(int k, int m, uint64_t seed, int contract);

// The reference's similarity of a winner-match count, as a float and its
// double (pmh_sv_from_count, src/rabbitbin.cpp:1297-1305).
// Similarity by equal-bucket count of the one-permutation metric: c / m.
void oph_sv_table(int m, std::vector<double> &sv_d, std::vector<float> &sv_f);
void sv_table(int m, bool base_on, double b0, std::vector<double> &sv_d,
              std::vector<float> &sv_f);

// One BGZF block of a device chunk: its deflate data (offset in the chunk's
// compressed bytes), inflated size, CRC32 and place in the chunk's output.
struct DevBlk {
  uint32_t cofs, clen, isize, crc;
  uint64_t uofs;
};
constexpr int kInflateWarps = 8;        // BGZF blocks in flight per CTA of the inflate kernel

// ── kernel launchers (kernels_*.cu) ─────────────────────────────────────────
struct SketchArgs {
  // input: 2-bit packed bases (16 per word, first base in the top bits) and
  // invalid-base mask (1 bit per base), covering the concatenated contigs
  const uint32_t *packed = nullptr;
  const uint32_t *nmask = nullptr;
  const int64_t *offsets = nullptr;    // [n+1] base offsets
  int64_t n = 0;
  int k = 4, m = 500, gc_norm = 1, n_elems = 136;
  double gc_cap = 20.0;
  const int16_t *rank_of_code = nullptr;  // [4^k]
  // per-contig element weights: 1/w of canonical k-mer e, +inf when absent
  double *elem_winv = nullptr;         // [n][n_elems]
  int32_t *elem_cnt = nullptr;         // [n] number of present elements
  // tables
  const RegOrder *order = nullptr;     // [m][E] elements by ascending U per register
  const double *UT = nullptr;          // [m][E] U by register, then element
  const uint8_t *codeA = nullptr;      // [E][m]
  const uint32_t *W32 = nullptr;       // [E][m]
  // outputs
  uint8_t *codesA = nullptr;           // [n][mpad]  (0 = unset)
  uint8_t *codesB = nullptr;           // [n][mpad]  (0xFF = unset)
  uint32_t *winners32 = nullptr;       // [n][m], optional
  uint8_t *win_elem = nullptr;         // [n][m], optional: winning element (0xFF unset)
  // one-permutation sketch keys instead of codes (launch_oph): [n][m], 0 = empty bucket
  uint64_t *oph_keys = nullptr;
  int mpad = 512;                      // row stride of the code arrays (bytes)
  // optional: a counter, zero at the launch, from which the count kernel's
  // warps take their contigs (null: a fixed stride)
  unsigned *work = nullptr;
};

void launch_pack(const char *ascii, int64_t nbases, uint32_t *packed, uint32_t *nmask,
                 cudaStream_t s);
// Words [w_begin, w_end) only (w_begin even): the packing of one chunk of a
// copy that is still arriving.
void launch_pack_range(const char *ascii, int64_t nbases, int64_t w_begin, int64_t w_end,
                       uint32_t *packed, uint32_t *nmask, cudaStream_t s);
void launch_count(const SketchArgs &a, cudaStream_t s);
void launch_minreduce(const SketchArgs &a, cudaStream_t s);
// codesB from codesA over `bytes` (a multiple of 16): equal codes, 0xFF for unset.
void launch_codes_b(const uint8_t *codesA, uint8_t *codesB, int64_t bytes, cudaStream_t s);
// One-permutation MinHash codes of contigs [0, a.n) (a.packed, a.nmask,
// a.offsets, a.m buckets, a.mpad) into a.codesA / a.codesB: each bucket's low
// `bits` bits + 1, padding 0 / 0xFF.  K: k-mer size (1..32).
void launch_oph(const SketchArgs &a, int K, int bits, uint64_t seed, cudaStream_t s);
// Bucket values (code - 1) of n OPH code rows into out[n][m].
void launch_oph_values(const uint8_t *codes, int64_t n, int m, int mpad, uint8_t *out,
                       cudaStream_t s);
// Seed of rabbit_sketch::KmerSketch as rb_cmd_bin constructs it (default, 42).
constexpr uint64_t kOphSeed = 42;

struct GraphArgs {
  int64_t n = 0;
  int m = 500, mpad = 512, S = 0, K = 200;
  int Su = 4;                          // row stride of `unit` (S rounded up to 4)
  const uint8_t *codesA = nullptr, *codesB = nullptr;
  const float *depth_raw = nullptr;    // [n][S]
  float *unit = nullptr;               // [n][Su] centred + L2-normalised ranks, 0-padded
  uint16_t *unit16 = nullptr;          // [n][Kp] the same rows rounded to FP16 (tensor-core prefilter)
  int Kp = 16;                         // row stride of unit16 (S rounded up to 16)
  uint8_t *anynz = nullptr;            // [n]
  double *colnorm = nullptr;           // [S]
  float min_cv = 1.0f;
  double min_cv_d = 1.0;
  int has_depth = 0;
  int wjac_norm = 1;
  // all-pairs
  int small_path = 0;                  // N <= 25000 path: maxima over all j != i
  int prefilter = 0;                   // abundance-first prune on
  float prefilter_eps = 0.f;           // (float)(abd_corr_min - 1e-4)
  const uint32_t *sv_bits = nullptr;   // [m+1] float bits of the similarity
  uint64_t *topk = nullptr;            // [n][K] keys, descending
  int32_t *topk_cnt = nullptr;         // [n]
  uint32_t *maxcnt_cand = nullptr;     // [n] over candidates
  uint32_t *maxcnt_all = nullptr;      // [n] over all j != i
  unsigned long long *stats = nullptr; // [2] prefiltered, compared
  // Keys at or below key_floor are never admitted to a row's candidates
  // (admission_floor()).
  uint64_t key_floor = 0;
  // rows scored by the per-ordered-pair kernels (launch_allpairs): [row_lo,
  // row_hi) against every column; row_hi < 0 means n (a sharded assembly
  // scores its own rows)
  int64_t row_lo = 0, row_hi = -1;
};

// The lowest key worth keeping: similarity 0.039 with the largest id bits.
// The calibrated cutoff a graph is cut at is at least 0.040 (the small path's
// walk stops at p <= RB_SIM_FLOOR = 50 after a step of at most 11,
// src/impl/rb_graph.cpp:395-415; the fused path clamps each round to >= 50,
// :1248-1252), and only keys with similarity above the cutoff become edges.  The top-K of the keys above the floor, cut at the cutoff, is the
// same set as the top-K of all keys cut at the cutoff, so rows skip every
// pair that could not be an edge.  The row maxima the calibration reads are
// taken before admission.
inline uint64_t admission_floor() {
  const float f = 0.039f;
  uint32_t bits;
  std::memcpy(&bits, &f, sizeof(bits));
  return ((uint64_t)bits << 32) | 0xFFFFFFFFull;
}

void launch_unit_rows(const GraphArgs &g, cudaStream_t s);
void launch_colnorm(const GraphArgs &g, double *acc, cudaStream_t s);
// b0 from the np sample counts on the device (median by histogram) into
// *b0_out (float, as stored) and the similarity table sv_out[m+1]; one CTA.
void launch_b0(const uint32_t *counts, int np, int m, float *b0_out, uint32_t *sv_out,
               cudaStream_t s);
void launch_pair_counts(const uint8_t *codesA, const uint8_t *codesB, int mpad, int m,
                        const int64_t *pairs, int npairs, uint32_t *out, cudaStream_t s);
void launch_allpairs(const GraphArgs &g, uint64_t *gbuf, int32_t *gcnt, cudaStream_t s);
// Warp per row of [g.row_lo, row_hi): its top-K from P partial lists of up to
// cap keys (list of row r, part s at ((r/32 * P + s) * 32 + r%32) * cap).
// ProbMinHash4 rows of n contigs from their winning elements (win_elem [n][m])
// and 1/w rows (elem_winv [n][E]): winners_ (W64 [E][m]; 0 unset) and the
// register values (1/w_e) * U_e(r) (U [E][m]; +inf unset).  Either output may be null.
void launch_pmh_rows(const uint8_t *win_elem, const double *elem_winv, int64_t n, int m, int E,
                     const uint64_t *W64, const double *U, uint64_t *w64_out, double *reg_out,
                     cudaStream_t s);
// out[i * nb + j] = table[count(A_i, B_j)], count = registers with equal values
// that are set (winners != 0 with regs == false; register values != +inf with
// regs == true); A [na][m], B [nb][m] 64-bit words.
void launch_pmh_compare(const uint64_t *A, int64_t na, const uint64_t *B, int64_t nb, int m,
                        bool regs, const double *table, double *out, cudaStream_t s);
// out[i][r] = std::min(a[i][r], b[i][r]) over n x m register values.
void launch_pmh_merge(const double *a, const double *b, int64_t count, double *out, cudaStream_t s);
// Inverted-index candidate graph (kernels_index.cu).
size_t index_rows_smem(int64_t n, int K);
size_t index_build_bytes(int64_t total);
int launch_index_build(const uint64_t *row_keys, int64_t n, int m, uint64_t *keys_sorted,
                       uint32_t *contig_in, uint32_t *post, uint64_t *ukeys, int32_t *ucount,
                       int64_t *uoff, int32_t *nruns_dev, void *scratch, size_t scratch_bytes,
                       cudaStream_t s);
void launch_index_rows(const GraphArgs &g, const uint64_t *row_keys, const uint64_t *ukeys,
                       const int32_t *ucount, const int64_t *uoff, const uint32_t *post,
                       const int32_t *nk, int64_t pl_cap, int min_common, double cutoff, int sms,
                       cudaStream_t s);
void launch_merge_topk(const GraphArgs &g, const uint64_t *gbuf, const int32_t *gcnt, int cap,
                       int P, cudaStream_t s);
// Dense regime on tcgen05 (kernels_onehot_mma.cu): counts of the rows
// [g.row_lo, g.row_lo + rows) against every contig as the int8 product of
// one-hot rows X [n][ldx] (ldx a multiple of 128), consumed in the kernel into
// per-(row, column group, tile half) lists of 32-bit keys (2 GC lists of cap
// keys per row) and the row maxima, then merged into g.topk / g.topk_cnt; tab [2m + 4]
// is scratch for the similarity-rank tables; *err != 0 after it ran when a
// bounded wait gave up.  Needs onehot_mma_fits(n, m) and 1 <= K <= 448.
bool onehot_mma_fits(int64_t n, int m);
int onehot_mma_cap(int64_t n, int GC, int K, int cap_max);
void onehot_mma_grid(int RB, int NT, int sms, int *GR, int *GC);
int launch_onehot_mma(const GraphArgs &g, const int8_t *X, int64_t ldx, int64_t rows,
                      uint32_t *cand, int cap, int32_t *cand_cnt, uint32_t *tab, int *err, int GR,
                      int GC, cudaStream_t s, const char **why);

// Output of the symmetric all-pairs pass (each unordered pair scored once): the
// admitted pairs and, per row, how many admitted keys it holds (both ends).
struct SymOut {
  uint4 *pairs = nullptr;               // {i, j, similarity bits, r0}: rows i < j of the
                                        // row space, r0 the first row of their assembly
  unsigned long long *npairs = nullptr; // admitted pairs found (may exceed cap)
  uint64_t cap = 0;                     // pairs written: min(npairs, cap)
  int32_t *rowcnt = nullptr;            // [n], zero before the pass
  // Deferred admission (the similarity table is not known yet): every survivor
  // with a nonzero match count is kept, with the count in place of the
  // similarity bits; launch_rows_topk converts it.  The top-K of all keys cut
  // at the calibrated cutoff equals the top-K of the admitted keys cut there.
  int defer = 0;
};
// Symmetric pass of the abundance-pruned (tensor-core) regime: row maxima into
// g.maxcnt_cand, admitted pairs into o.  Requires allpairs_variant(g) != 0.
void launch_allpairs_sym(const GraphArgs &g, const SymOut &o, cudaStream_t s, int x0 = 0,
                         int xs = 1);

// Symmetric pass in two kernels (kernels_sym_tc5.cu, kernels_allpairs.cu) over
// the pairs i < j with j in [cb, ce): the tcgen05 abundance prefilter writes
// each 32-row block's candidates (entries r << 27 | j at cand + coff[b],
// capacity coff[b + 1] - coff[b], the count in ccnt[b] even past it; *overflow
// set then), k_sym_check decides and counts them into o (blocks below
// ceil(ce / 32)).  The item table [RB + 1] comes from launch_tc5_items (its
// total from sym_tc5_items); u16p: the unit16 rows padded to 64 halves by
// launch_pad_unit16, a row copy and a column copy carrying the threshold lo16
// in the last half (2 x n x 128 bytes, 16-byte aligned).  Needs g.S < 64 and
// n < 2^27.  The offsets and item tables are made on the device, so nothing
// crosses PCIe while input chunks stream in; tc5_capacity is the total of the
// frac-based capacities of launch_tc5_coff (caps null).
int sym_tc5_items(int64_t cb, int64_t ce, int *RB, int *NT);
int64_t tc5_capacity(int64_t n, double frac);
void launch_tc5_coff(int64_t n, double frac, const int64_t *caps, int64_t *coff, cudaStream_t s);
void launch_tc5_items(int64_t cb, int64_t ce, int32_t *item0, cudaStream_t s);
void launch_pad_unit16(const GraphArgs &g, float lo16, uint16_t *u16p, cudaStream_t s);
int launch_sym_prefilter(const GraphArgs &g, const uint16_t *u16p, int64_t cb, int64_t ce,
                         const int32_t *item0, int RB, int NT, int items, uint32_t *cand,
                         const int64_t *coff, int32_t *ccnt, int *overflow, int *err, int sms,
                         cudaStream_t s, const char **why);
void launch_sym_check(const GraphArgs &g, const SymOut &o, const uint32_t *cand,
                      const int64_t *coff, const int32_t *ccnt, int64_t blocks, cudaStream_t s);
float prefilter_lo16(int S, float eps);

// A pair list gathered from several ranks: its per-row key counts (rowcnt
// zeroed by the caller), and the elementwise maximum of W blocks of partial
// row maxima.
void launch_pair_rowcounts(const uint4 *pairs, unsigned long long np, int32_t *rowcnt,
                           cudaStream_t s);
void launch_max_blocks(const uint32_t *blocks, int W, int64_t stride, int64_t n, uint32_t *out,
                       cudaStream_t s);
// The same pass over the pairs (i, j), i < j, whose column j lies in [cb, ce):
// rows [0, ce) against those columns.  Windows that tile [0, n) score every
// pair once; rows at or past ce are not read as candidates.
void launch_allpairs_sym_window(const GraphArgs &g, const SymOut &o, int64_t cb, int64_t ce,
                                cudaStream_t s);
// Per-row top-K of the admitted pairs (both keys of each pair) into g.topk /
// g.topk_cnt.  rowoff [n+1] and keys [2 * cap] are scratch; o.rowcnt ends zero.
void launch_rows_topk(const GraphArgs &g, const SymOut &o, int64_t *rowoff, uint64_t *keys,
                      cudaStream_t s);
// Pass with deferred admission: o.pairs hold match counts; svtab [m+1] maps a
// count to its similarity bits.
void launch_rows_topk_counts(const GraphArgs &g, const SymOut &o, const uint32_t *svtab,
                             int64_t *rowoff, uint64_t *keys, cudaStream_t s);
int allpairs_slices(int64_t n, int K);
// Column slices for `rows` rows against n columns (launch_allpairs on a row range).
int allpairs_slices_rows(int64_t rows, int64_t n, int K);
int allpairs_cap(int K);

struct EmitArgs {
  int64_t n = 0;
  int K = 200, mutual = 1, small_path = 0;
  const uint64_t *topk = nullptr;
  const int32_t *topk_cnt = nullptr;
  double cutoff = 0.0;
  uint32_t *nbr_sorted = nullptr;      // [n][K] ids of kept neighbours, ascending
  float *nbr_sv = nullptr;             // [n][K]
  int32_t *nbr_cnt = nullptr;          // [n]
  int32_t *row_edges = nullptr;        // [n+1] edges per row, then exclusive scan
  uint32_t *from = nullptr, *to = nullptr;
  float *scomp = nullptr;
  // optional [n][ceil(K/32)] bit masks: the edge count records which of a
  // row's neighbours it kept, and the edge write reads them (null: the write
  // tests each neighbour again)
  uint32_t *kept = nullptr;
  // rows whose neighbour lists and edges the plain launchers produce:
  // [row_lo, row_hi), row_hi < 0 means n; row_edges is scanned over that range
  int64_t row_lo = 0, row_hi = -1;
};

void launch_sort_rows(const EmitArgs &e, cudaStream_t s);
void launch_count_edges(const EmitArgs &e, cudaStream_t s);
void launch_write_edges(const EmitArgs &e, cudaStream_t s);

struct WeightArgs {
  int64_t n_edges = 0;
  int S = 0;
  const uint32_t *from = nullptr, *to = nullptr;
  const float *scomp = nullptr;
  float *score = nullptr;
  const float *unit = nullptr;         // [n][Su]
  int Su = 4;
  const float *depth_raw = nullptr;
  const double *colnorm = nullptr;     // null = no column normalisation
  double w_comp = 0.0, min_edge = 0.7, neg_thr = -0.3, wjac_cut = 0.0;
  int depth_sim = 2, depth_fuse = 1, wjac_gate = 0, contract = 1;
};

void launch_edge_weights(const WeightArgs &w, cudaStream_t s);

// ── batches of assemblies (kernels over many assemblies in one launch) ─────
// One assembly of a batch, held in device memory.  Every pointer in g, e and
// w addresses that assembly's own rows (local ids 0..n-1); the edge arrays
// e.from/to/scomp and w.from/to/scomp/score are the batch's global ones and
// e.row_edges points at the assembly's first row of the batch-wide scan.
struct BatchAsm {
  GraphArgs g;
  EmitArgs e;
  WeightArgs w;
  int64_t row0 = 0;                    // first row in the batch's row space
  // all-pairs
  uint64_t *gbuf = nullptr;            // candidate buffers [ceil(n/32)][P][32][cap]
  int32_t *gcnt = nullptr;             // [ceil(n/32)][P][32]
  int cap = 0, P = 0, variant = 0;     // variant: 0 dense (ALU), -1 dense (one-hot GEMM),
                                       // 1/2/4 tensor-core KS
  float lo = 0.f, hi = 0.f, lo16 = 0.f;
  // column norms
  int colnorm_on = 0;
  double *colacc = nullptr;            // [3 S]
  // b0: register-match counts of this assembly's sampled pairs
  int base_on = 0, np = 0;
  int64_t pair0 = 0;                   // first pair in the batch's pair list
  float *b0 = nullptr;                 // out: b0 of the assembly (float, as stored)
  uint32_t *sv_out = nullptr;          // out: [m+1] similarity float bits (== g.sv_bits)
};

// Raise a kernel's dynamic shared-memory cap once per device to the opt-in
// maximum; every launch then passes its own size.  Setting the cap to each
// launch's size instead races when host threads (serving workers, contexts on
// other threads) launch the kernel with different sizes.
void smem_cap_max(const void *func);

// Index helper arrays ("starts") are ascending int64 with starts[nb] = total;
// a batch kernel maps a global index x to the last assembly a with
// starts[a] <= x.  Row-range launchers cover batch rows [r_begin, rows).
void launch_unit_rows_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                            cudaStream_t s, int64_t r_begin = 0);
// Column norms of the assemblies B[0..nb) (pass B + first for a range).
void launch_colnorm_batch(const BatchAsm *B, int nb, int max_s, cudaStream_t s);
void launch_b0_batch(const BatchAsm *B, const int64_t *pair0s, int nb, int64_t npairs,
                     const int32_t *pairs, uint32_t *counts, int max_m, cudaStream_t s);
// b0 and similarity tables of assemblies [b_begin, b_end), whose sampled
// pairs are [p_begin, p_end).
void launch_b0_batch_range(const BatchAsm *B, const int64_t *pair0s, int nb, int64_t p_begin,
                           int64_t p_end, const int32_t *pairs, uint32_t *counts, int max_m,
                           int b_begin, int b_end, cudaStream_t s);
// Persistent all-pairs over the assemblies list[0..nv) of one variant: work
// item x of assembly list[k] is x - item0s[k] (row block, slice group); CTAs
// pull items from *next (zeroed by the caller).
// The tensor-core variants run the symmetric pass into o (row space of the
// batch); the dense one fills the assemblies' candidate buffers.
void launch_allpairs_batch(const BatchAsm *B, int variant, const int32_t *list,
                           const int64_t *item0s, int nv, int64_t items, size_t smem,
                           unsigned long long *next, const SymOut &o, cudaStream_t s);
// Top-K of the dense assemblies' candidate buffers (others skipped).
void launch_merge_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                        cudaStream_t s, int64_t r_begin = 0);
// Top-K of the tensor-core assemblies from the symmetric pass's pairs (dense
// ones skipped); rowoff [rows+1] and keys [2 * o.cap] are scratch.
void launch_rows_topk_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                            const SymOut &o, int64_t *rowoff, uint64_t *keys, cudaStream_t s);
void launch_emit_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows, int max_k,
                       int32_t *row_edges, int64_t *edge0s, cudaStream_t s);
void launch_write_edges_batch(const BatchAsm *B, const int64_t *row0s, int nb, int64_t rows,
                              cudaStream_t s);
void launch_edge_weights_batch(const BatchAsm *B, const int64_t *edge0s, int nb, int64_t edges,
                               cudaStream_t s);
// ── dense regime on the tensor cores (kernels_onehot.cu) ───────────────────
// Codes occurring per register column of rows [0, n): pres[m][8] (256 bits).
void launch_code_presence(const uint8_t *codesA, int64_t n, int m, int mpad, uint32_t *pres,
                          cudaStream_t s);
// One-hot column of (register, code): map[r * 256 + code] (-1 absent);
// koff[m + 1], koff[m] = K the one-hot width.
void launch_onehot_map(const uint32_t *pres, int m, int32_t *map, int32_t *koff, cudaStream_t s);
// X [n][ldx] int8: 1 at (i, map[r][code_i(r)]) for every set register, else 0.
void launch_onehot_fill(const uint8_t *codesA, int64_t n, int m, int mpad, const int32_t *map,
                        int8_t *X, int64_t ldx, cudaStream_t s);
// Rows [r0, r0 + nr) from their counts D[(i - r0) * ldd + j]: per-row top-K
// keys, row maxima and compared pairs, as the dense all-pairs kernel gives.
void launch_dense_select(const GraphArgs &g, const int32_t *D, int64_t ldd, int64_t r0, int64_t nr,
                         cudaStream_t s);

// ── FASTA ingest (kernels_fasta.cu) ────────────────────────────────────────
// One record of a FASTA file on the device: its name range in the input, its
// body [b0, b1) with body newlines nl_pos[nl0..nl1), its length after newline
// removal, single-line flag and class (0 tiny, 1 small, 2 large, 3 no header
// newline: dropped and not counted).
struct FastaRec {
  int64_t name_start, b0, b1, nl0, nl1, len;
  int32_t name_len;
  int8_t cls, single;
};
// Tile counts of '\n' and '>' and their exclusive scans (totals at [tiles]).
void launch_fasta_positions(const uint8_t *in, int64_t F, int *tile_nl, int *tile_gt,
                            int64_t *nl_base, int64_t *gt_base, cudaStream_t s);
void launch_fasta_scatter(const uint8_t *in, int64_t F, const int64_t *nl_base,
                          const int64_t *gt_base, int64_t *nl_pos, int64_t *gt_pos,
                          cudaStream_t s);
// flag[0..ngt] becomes the exclusive scan of record-start flags; rs the starts.
void launch_fasta_starts(const int64_t *gt_pos, int64_t ngt, const int64_t *nl_pos, int64_t nnl,
                         int64_t *flag, int64_t *rs, cudaStream_t s);
void launch_fasta_records(const uint8_t *in, int64_t F, const int64_t *rs, int64_t nrs,
                          const int64_t *nl_pos, int64_t nnl, int64_t min_contig,
                          int64_t min_small, FastaRec *rec, cudaStream_t s);
// Exclusive scans of class-c membership (output index) and length (byte
// offset) over the records, totals at [nrs].
void launch_fasta_class(const FastaRec *rec, int64_t nrs, int c, int64_t *flag, int64_t *bytes,
                        cudaStream_t s);
void launch_fasta_copy(const uint8_t *in, const FastaRec *rec, int64_t nrs, const int64_t *nl_pos,
                       int c, const int64_t *idx, const int64_t *off, uint8_t *out,
                       int64_t *out_off, int64_t *name_start, int32_t *name_len, cudaStream_t s);

// Work items of the all-pairs kernels for one assembly.
int64_t allpairs_items(int64_t n, int P);
size_t allpairs_batch_smem(int variant, int mpad, int Su);
// 0 (dense) or the tensor-core prefilter's k-steps KS (1, 2, 4).
int allpairs_variant(const GraphArgs &g);
// lo/hi: band of the exact-safe FP32 chain; lo16: the tensor-core prune bound.
void prefilter_bands(int S, float eps, float *lo, float *hi, float *lo16);

// Label propagation (kernels_lpa.cu).  Incidence: per-edge quantities q and
// endpoint degrees (err: 1 negative score, 2 endpoint out of range), offsets
// (n + 1) and the largest degree, arc keys scattered per node, keys sorted per
// node into neighbour and quantity arrays.
int lpa_raw_rule(int rule);
void launch_lpa_edges(const uint32_t *from, const uint32_t *to, const float *score, int64_t E,
                      int64_t n, int rule, float *q, uint32_t *deg, int *err, cudaStream_t s);
void launch_lpa_offsets(const uint32_t *deg, int64_t n, int64_t *off, int64_t *maxdeg,
                        cudaStream_t s);
void launch_lpa_scatter(const uint32_t *from, const uint32_t *to, const float *score, int64_t E,
                        int64_t n, const int64_t *off, uint32_t *fill, uint64_t *key,
                        cudaStream_t s);
void launch_lpa_sort(const int64_t *off, int64_t n, uint64_t *key, const float *q, uint32_t *nbr,
                     float *w, cudaStream_t s);
void launch_lpa_init(const uint32_t *order, int64_t n, uint32_t *pos, uint32_t *label,
                     uint8_t *active, uint8_t *next_active, uint8_t *frozen, uint32_t *done,
                     uint32_t *vcnt, uint32_t *vnext, cudaStream_t s);
// State of the sweeps (see kernels_lpa.cu); vlab holds lpa_visit_block()
// labels per visited-set block, blocks 0..n-1 owned by the nodes, vpool_cap
// spill blocks after them; gtab: gtab_slots x 20 bytes per sweep warp when the
// largest degree exceeds lpa_table_max_deg() (slots >= 4/3 of it, a power of 2).
struct LpaSweepArgs {
  int64_t n = 0;
  const int64_t *off = nullptr;
  const uint32_t *nbr = nullptr;
  const float *w = nullptr;
  const uint32_t *order = nullptr, *pos = nullptr;
  const uint8_t *early = nullptr;         // per arc: neighbour earlier in the order
  const uint4 *rec = nullptr;             // per position: node, degree, first arc
  uint32_t *label = nullptr;
  uint8_t *active = nullptr, *next_active = nullptr, *frozen = nullptr;
  uint32_t *done = nullptr, *prop = nullptr;
  uint32_t *vlab = nullptr, *vcnt = nullptr, *vnext = nullptr, *vpool_used = nullptr;
  uint32_t vpool_cap = 0;
  uint32_t *claim = nullptr;
  unsigned long long *counts = nullptr;   // [0] changes, [1] freezes of the round
  uint32_t *gtab = nullptr;
  int gtab_slots = 0;
  int rule = 0;
  uint32_t round = 0;
  int *err = nullptr;
};
// Per arc: the neighbour precedes the node in the order; per position: node,
// degree, first arc (low, high word).
void launch_lpa_early(const int64_t *off, const uint32_t *nbr, const uint32_t *pos, int64_t n,
                      uint8_t *early, uint4 *rec, cudaStream_t s);
// Warps of one sweep launch (a multiple of the CTA's 8).
int lpa_sweep_warps(int sms);
int lpa_table_max_deg();
int lpa_visit_block();
void launch_lpa_round(const LpaSweepArgs &a, int sync, int warps, cudaStream_t s);

}  // namespace rbg
