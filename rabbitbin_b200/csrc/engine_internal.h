// Host-side internals shared by the single-assembly engine (engine.cpp) and
// the batch engine (batch.cpp): errors, device and pinned buffers, the
// per-configuration table cache, the context, and the host steps of the
// calibration.
#pragma once
#include <cstdlib>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "rbg_internal.h"

struct rbg_ctx;

namespace rbg {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                     \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess)                                                        \
      throw ::rbg::Error(e_ == cudaErrorMemoryAllocation ? RBG_ERR_NOMEM : RBG_ERR_CUDA, \
                         std::string(#x) + ": " + cudaGetErrorString(e_));        \
  } while (0)

// A growable device allocation.  It grows by at least half its size, so a
// stream of growing requests reallocates (cudaFree synchronises the device)
// only a logarithmic number of times.
struct DBuf {
  void *p = nullptr;
  size_t cap = 0;
  template <typename T> T *as() const { return (T *)p; }
  void ensure(size_t bytes) {
    if (bytes <= cap) return;
    const size_t grown = cap + cap / 2;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    if (grown > want) {
      // fall back to the exact size when the grown one does not fit
      if (cudaMalloc(&p, grown) == cudaSuccess) {
        cap = grown;
        return;
      }
      cudaGetLastError();
      p = nullptr;
    }
    CK(cudaMalloc(&p, want));
    cap = want;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Pinned host staging buffer.
struct HBuf {
  void *p = nullptr;
  size_t cap = 0;
  template <typename T> T *as() const { return (T *)p; }
  void ensure(size_t bytes) {
    if (bytes <= cap) return;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t want = bytes < 256 ? 256 : bytes;
    CK(cudaMallocHost(&p, want));
    cap = want;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

inline int mpad_of(int m) { return (m + 15) & ~15; }

// Chunks of the host-to-device copy that rbg_bin_graph overlaps with the sketch.
constexpr int kChunks = 8;

// Row stride (halves) of the FP16 unit rows: 16, 32 or 64, the k extent of the
// tensor-core prefilter variant that reads them.
inline int unit16_stride(int S) { return S <= 16 ? 16 : (S <= 32 ? 32 : 64); }

inline bool need_colnorm(const rbg_params *p, int S) {
  return p->depth_sim >= 1 && S > 1 && p->wjac_norm;
}

// Device copy of one sketch configuration's tables.
struct Tables {
  std::shared_ptr<const PmhTables> t;
  int win_bits = 16;
  DBuf order, UT, codeA, W32, rank;
  DBuf dict_vals, dict_codes, dict_n;   // per-column sorted dictionaries
  bool dict_ready = false;
  DBuf W64, U;                          // winner states and U by element (sketch rows)
  bool rows_ready = false;
  void release() {
    order.release(); UT.release(); codeA.release(); W32.release(); rank.release();
    dict_vals.release(); dict_codes.release(); dict_n.release();
    W64.release(); U.release();
  }
};

// Uploads (k, m, seed, contract, win_bits) tables to the device on `s`
// (synchronised before returning).
std::unique_ptr<Tables> make_tables(const rbg_params *p, cudaStream_t s);

// Dense regime (no abundance prune) of rows [g.row_lo, row_hi): the one-hot
// int8 product of the register codes on the tensor cores (k_onehot_mma) and
// the merge of its candidate lists; writes g.topk, g.topk_cnt, g.maxcnt_all,
// g.maxcnt_cand (which the caller zeroed) and g.stats[1].  Synchronises
// c->stream once (the one-hot width); call check_onehot_status after the
// caller's next synchronisation of c->stream.
void dense_allpairs_onehot(rbg_ctx *c, const GraphArgs &g);
void check_onehot_status(rbg_ctx *c);

// Symmetric pass on the tcgen05 prefilter (engine.cpp): whether it takes the
// assembly; per-assembly setup (list capacities, padded FP16 rows, cleared
// flags; `slots` item tables for passes in flight); one pass over the pairs
// i < j with j in [cb, ce); the flags and block counts read back on the stream;
// after the sync, false when a list overflowed (the caller reruns).
bool sym_tc5_fits(const GraphArgs &g);
void sym_tc5_setup(rbg_ctx *c, const GraphArgs &g, int slots);
void sym_tc5_pass(rbg_ctx *c, const GraphArgs &g, const SymOut &o, int64_t cb, int64_t ce,
                  int slot);
void sym_tc5_readback(rbg_ctx *c, int64_t n);
bool sym_tc5_settle(rbg_ctx *c, int64_t n);
// The dense regime runs on the one-hot tensor-core kernel unless RBG_DENSE_ALU
// is set (then the integer-ALU register compare, kept for the measured
// comparison).
inline bool dense_on_gemm() { return getenv("RBG_DENSE_ALU") == nullptr; }

// 2-bit packing on the host (host_pack.cpp): words [w0, w1) of the packed
// bases (w0 even; rounded up to whole word pairs: 2 * ceil((w1 - w0) / 2)
// words) and their ceil((w1 - w0) / 2) mask words, in k_pack's layout.
void host_pack_words(const char *ascii, int64_t nbases, int64_t w0, int64_t w1,
                     uint32_t *packed, uint32_t *mask);
int host_pack_threads();
// The end-to-end call copies the ASCII and packs on the device unless
// RBG_HOST_PACK is set (then the host packs and the copies carry 3/8 of a byte
// per base; it pays only where the host packs faster than the link copies
// ASCII) and the host has at least four threads.
inline bool pack_on_host() {
  return getenv("RBG_HOST_PACK") != nullptr && host_pack_threads() >= 4;
}

// Pinned result blocks (pooled).  pinned_take: a block of `bytes` or null;
// pinned_share: the block now backs graphs whose first edge arrays are
// `firsts` (distinct), and returns to the pool when rbg_free_graph has been
// called on each of them.
void *pinned_take(size_t bytes);
void pinned_share(void *blk, const std::vector<void *> &firsts);

// Buffers of the batch engine (many assemblies per launch).
struct BatchBufs {
  DBuf ascii, offsets, depth, packed, nmask, winv, ecnt, codesA, codesB;
  DBuf unit, unit16, anynz, colnorm, colacc, svbits, topk, topk_cnt, maxc_cand, maxc_all, stats;
  DBuf gbuf, gcnt, pairs, pair_cnt, b0;
  DBuf nbr, nbr_sv, nbr_cnt, row_edges, edge0s;
  DBuf e_from, e_to, e_scomp, e_score;
  DBuf desc, row0s, lists, item0s, queues, pair0s;
  // symmetric all-pairs pass of the tensor-core assemblies (row space of the batch)
  DBuf sym_pairs, sym_np, sym_rowcnt, sym_rowoff, sym_keys;
  uint64_t sym_cap = 0;
  // autotuner: multiplier of the pairs-per-item target (the all-pairs tile
  // shape) chosen per (variant, m, log2 n), and events timing each variant's
  // persistent launch
  std::map<std::tuple<int, int, int>, double> tune;
  cudaEvent_t tev[8] = {};
  HBuf hstage, hout, hedge, hdepth;     // hdepth: depth rows staged pinned for async copies
  std::map<std::tuple<int, int, uint64_t, int, int>, std::unique_ptr<Tables>> tables;
  void release() {
    DBuf *all[] = {&ascii, &offsets, &depth, &packed, &nmask, &winv, &ecnt, &codesA, &codesB,
                   &unit, &unit16, &anynz, &colnorm, &colacc, &svbits, &topk, &topk_cnt,
                   &maxc_cand, &maxc_all, &stats, &gbuf, &gcnt, &pairs, &pair_cnt, &b0, &nbr,
                   &nbr_sv, &nbr_cnt, &row_edges, &edge0s, &e_from, &e_to, &e_scomp, &e_score,
                   &desc, &row0s, &lists, &item0s, &queues, &pair0s, &sym_pairs, &sym_np,
                   &sym_rowcnt, &sym_rowoff, &sym_keys};
    for (DBuf *b : all) b->release();
    hstage.release();
    hout.release();
    hedge.release();
    hdepth.release();
    sym_cap = 0;
    tune.clear();
    for (auto &e : tev)
      if (e) cudaEventDestroy(e);
    for (auto &e : tev) e = nullptr;
    for (auto &kv : tables) kv.second->release();
    tables.clear();
  }
};

// Buffers of the device FASTA parser.
struct FastaBufs {
  DBuf in, tile_nl, tile_gt, nl_base, gt_base, nl_pos, gt_pos, flag, rs, rec;
  DBuf idx[2], off[2], seq[2], seq_off[2], name_start[2], name_len[2];
  void release() {
    DBuf *all[] = {&in, &tile_nl, &tile_gt, &nl_base, &gt_base, &nl_pos, &gt_pos, &flag, &rs,
                   &rec, &idx[0], &idx[1], &off[0], &off[1], &seq[0], &seq[1], &seq_off[0],
                   &seq_off[1], &name_start[0], &name_start[1], &name_len[0], &name_len[1]};
    for (DBuf *b : all) b->release();
  }
};

// Buffers of label propagation (lpa.cpp): the edge list as copied in, the
// incidence lists and the sweep state.
struct LpaBufs {
  DBuf from, to, score, q, deg, off, fill, key, nbr, w, early, rec, order, pos, label, act0,
      act1, frozen, done, prop, vlab, vcnt, vnext, misc, gtab;
  HBuf pin, order_pin;
  void release() {
    DBuf *all[] = {&from, &to, &score, &q, &deg, &off, &fill, &key, &nbr, &w, &early, &rec, &order, &pos,
                   &label, &act0, &act1, &frozen, &done, &prop, &vlab, &vcnt, &vnext, &misc,
                   &gtab};
    for (DBuf *b : all) b->release();
    pin.release();
    order_pin.release();
  }
};

// BAM -> depth: two hand-over slots (decompressed records and one offset per
// record, pinned on the host and on the device), the sums, the header's
// lengths, the kept rows, each column's edge and the means.
struct DepthBufs {
  DBuf buf[2], off[2], sums, tlen, kept, edge, means;
  HBuf slot[2], offp[2];
  // device route: compressed chunk, block table, inflated chunk, counts and
  // scan, record offsets; the route's flags and record count
  DBuf cdev[2], tdev[2], outd[2], cntd[2], offd[2], flags;
  HBuf cpin[2], tpin[2], hflag;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaEvent_t k0[2] = {nullptr, nullptr}, k1[2] = {nullptr, nullptr};   // per-record launch times
  cudaEvent_t evc[2] = {nullptr, nullptr};                             // device route: chunk copied
  void release() {
    DBuf *all[] = {&buf[0], &buf[1], &off[0], &off[1], &sums, &tlen, &kept, &edge, &means,
                   &cdev[0], &cdev[1], &tdev[0], &tdev[1], &outd[0], &outd[1], &cntd[0],
                   &cntd[1], &offd[0], &offd[1], &flags};
    for (DBuf *b : all) b->release();
    hflag.release();
    for (int i = 0; i < 2; ++i) {
      slot[i].release();
      offp[i].release();
      cpin[i].release();
      tpin[i].release();
      if (ev[i]) cudaEventDestroy(ev[i]);
      if (k0[i]) cudaEventDestroy(k0[i]);
      if (k1[i]) cudaEventDestroy(k1[i]);
      if (evc[i]) cudaEventDestroy(evc[i]);
      ev[i] = k0[i] = k1[i] = evc[i] = nullptr;
    }
  }
};

// Counts of one parse; the outputs are in FastaBufs: slot 0 large, 1 small
// (seq: sequences back to back, seq_off: n+1 offsets, name_start / name_len:
// name ranges in the input).
struct FastaCounts {
  int64_t num_seqs = 0, n[2] = {0, 0}, bytes[2] = {0, 0};
};

// glibc's rand() sequence of one seed (srand(seed); rand(); ...) on private
// state, so concurrent calibrations do not share the process-wide generator.
struct CRand {
  random_data rd;
  char state[128];
  explicit CRand(unsigned seed) {
    std::memset(&rd, 0, sizeof(rd));
    std::memset(state, 0, sizeof(state));
    initstate_r(seed, state, sizeof(state), &rd);
  }
  int operator()() {
    int32_t r = 0;
    random_r(&rd, &r);
    return (int)r;
  }
};

// Calibration of the similarity cutoff:
//   all          calibrate_sim_cutoff over every contig (src/impl/rb_graph.cpp:1362-1384),
//                the small path; maxc over all j != i
//   fused        the sampling rounds of gen_fused_calib_graph (:505-522, per-round
//                converge and mean); maxc over the candidates
//   samples_all  calibrate_sim_cutoff_fused (:1386-1431), the large-N route of the
//                one-permutation metric: ten 2500-contig samples, each sampled
//                contig's maximum over all j != i
enum class CalibMode { all, fused, samples_all };

// The calibrated similarity cutoff (x1000) of one assembly from its per-row
// maximum register-match counts and its similarity tables.
double calibrate_cutoff(const uint32_t *maxc, int64_t n, CalibMode mode, int m,
                        const std::vector<double> &sv_d, const std::vector<float> &sv_f,
                        double coverage, unsigned seed);

// b0 sampling pairs of an assembly of n contigs (estimate_pmh_baseline,
// src/rabbitbin.cpp:1340-1369: mt19937_64 draws, i == j skipped), as local ids.
std::shared_ptr<const std::vector<int32_t>> b0_pairs(int64_t n);

void validate_params(const rbg_params *p);

// Parses `F` bytes of FASTA (host memory) on the context's device.
FastaCounts fasta_parse(rbg_ctx *c, const char *data, int64_t F, int64_t min_contig,
                        int64_t min_small);

// Frees the CUDA graphs the batch engine keeps for a context.
void release_batch_graphs(rbg_ctx *c);

// Device bytes the batch engine needs for one assembly (its share of every
// batch buffer; a bound on the edge arrays).
int64_t batch_request_bytes(const rbg_params *p, int64_t n, int64_t nbases, int S);

// Validation of one assembly's arguments (the checks rbg_bin_batch makes).
void validate_assembly(const rbg_assembly &x, const rbg_params *p, const std::string &who);
void bin_graph_one(rbg_ctx *c, const rbg_params *p, const rbg_assembly &x, rbg_graph *out);

}  // namespace rbg

struct rbg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::mutex mu;
  // staged inputs
  int64_t n = 0, nbases = 0;
  int S = 0;
  std::vector<int64_t> h_offsets;
  rbg::DBuf ascii, offsets, depth;
  // sketch state
  rbg::DBuf packed, nmask, elem_idx, elem_winv, elem_cnt, codesA, codesB, winners32;
  // graph state
  rbg::DBuf unit, unit16, anynz, colnorm, svbits, topk, topk_cnt, maxc_cand, maxc_all, stats;
  rbg::DBuf pairs, pair_out, nbr, nbr_sv, nbr_cnt, row_edges, cand_buf, cand_cnt;
  rbg::DBuf e_from, e_to, e_scomp, e_score, badflag, tmp, colacc;
  rbg::DBuf kept;                        // kept-neighbour masks of the edge count
  rbg::DBuf b0dev;                       // b0 as made on the device (float)
  rbg::HBuf b0pin;                       // and its pinned host copy
  int64_t pairs_n = -1;                  // contig count whose b0 sample `pairs` holds
  // symmetric all-pairs pass: admitted pairs, per-row counts, offsets and keys
  rbg::DBuf sym_pairs, sym_np, sym_rowcnt, sym_rowoff, sym_keys;
  uint64_t sym_cap = 0;                  // pair-list capacity (grows when a pass overflows)
  rbg::DBuf shard_send, shard_recv;      // exchange blocks of rbg_bin_graph_sharded
  // dense regime on the tensor cores: code presence, one-hot map and offsets,
  // the one-hot matrix, the candidate lists and their counts, the kernel's
  // wait status (and its pinned copy, valid after the next synchronisation)
  rbg::DBuf oh_pres, oh_map, oh_koff, oh_X, oh_cand, oh_cnt, oh_tab, oh_err;
  rbg::DBuf count_work;                 // contig counter of the k-mer count kernel
  // symmetric pass on the tensor-core prefilter: candidate lists per 32-row
  // block (capacities tc5_cap, sized from the kept fraction tc5_frac)
  rbg::DBuf tc5_u16p, tc5_cand, tc5_cnt, tc5_items, tc5_coff, tc5_caps, tc5_flags;
  rbg::HBuf tc5_pin, tc5_host;
  std::vector<int64_t> tc5_cap;
  int64_t tc5_n = -1;
  double tc5_frac = 0.03;
  bool tc5_exact = false;               // tc5_cap holds exact capacities for the next setup
  int64_t tc5_rbmax = 0;                // item-table slot length - 1
  bool streamed_tc5 = false;            // the pairs behind the copy went through that pass
  rbg::HBuf oh_errpin;
  bool oh_pending = false;
  // ProbMinHash4 queries: operand blocks, output block, metric table
  rbg::DBuf qa, qb, qo, qt;
  // inverted-index graph: sketch keys, sorted pairs, unique keys, list
  // lengths and offsets, their count, sort scratch
  rbg::DBuf ix_keys, ix_sorted, ix_contig, ix_post, ix_ukeys, ix_count, ix_off, ix_nk, ix_scratch;
  rbg::HBuf shard_host;                  // their host staging for host-memory collectives
  bool streamed = false;                 // rbg_bin_graph scored the pairs behind the copy
  uint64_t no_stream_S = 0;              // bit S: survivors outgrew the list when streamed
  rbg::HBuf pin;                         // row maxima and pair count read back for calibration
  int64_t n_edges = 0;
  double b0 = 0.0, sim_cutoff = 0.0;
  int path = 0;
  bool graph_ready = false;
  // tables (one configuration cached)
  // sketch tables by (k, m, seed, contract, win_bits), most recently used first
  std::list<std::pair<std::tuple<int, int, uint64_t, int, int>, std::unique_ptr<rbg::Tables>>>
      tab_cache;
  cudaEvent_t ev[12];
  cudaStream_t aux = nullptr;            // depth preparation, overlapped with the sketch
  cudaEvent_t ev_in = nullptr, ev_aux = nullptr, ev_a0 = nullptr, ev_a1 = nullptr;
  bool prep_done = false;
  int launches = 0;
  // chunked input copy behind the sketch (rbg_bin_graph)
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_cin = nullptr, ev_chunk[rbg::kChunks] = {};
  // chunks packed on the host (2-bit words, then mask words), two slots, and
  // the events of their copies
  rbg::HBuf pack_pin[2];
  cudaEvent_t ev_slot[2] = {};
  // batch engine
  std::unique_ptr<rbg::BatchBufs> batch;
  // FASTA ingest
  std::unique_ptr<rbg::FastaBufs> fasta;
  // label propagation
  std::unique_ptr<rbg::LpaBufs> lpa;
  // BAM -> depth
  std::unique_ptr<rbg::DepthBufs> depthb;
};

namespace rbg {

// Runs f under the context's lock with the context's device current and maps
// exceptions onto status codes and the context's error string.
template <typename F>
int guarded(rbg_ctx *c, F &&f) {
  if (!c) return RBG_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  try {
    CK(cudaSetDevice(c->device));
    f();
    c->err.clear();
    return RBG_OK;
  } catch (const Error &e) {
    c->err = e.what();
    return e.code;
  } catch (const std::bad_alloc &) {
    c->err = "host allocation failed";
    return RBG_ERR_NOMEM;
  } catch (const std::exception &e) {
    c->err = e.what();
    return RBG_ERR_CUDA;
  }
}

}  // namespace rbg
