// Batch engine: many assemblies sketched and graphed together.
//
// The assemblies of a call share one set of device buffers (rows of all
// assemblies laid end to end).  In runs of batch positions of about equal
// bases, each run behind its input copy on a second stream:
//   pack -> count (per k / GC-norm group) -> register minimum (per sketch-table
//   group) -> unit rows + column norms -> b0 and similarity tables (on the
//   device) -> persistent all-pairs kernels pulling (assembly, row block,
//   slice group) items from a device counter, one per variant (dense /
//   tensor-core KS) -> dense assemblies' one-hot GEMMs
// then the row top-K of the symmetric pass over the whole batch, one host
// round trip for the rand()-driven calibration of every assembly (the maxima
// and b0 come back together), then neighbour lists, edge counts and the
// batch-wide scan, one more round trip for the edge total, and edge emission
// + weights.  The device part of each of the three segments after the runs
// is captured into a CUDA graph; an instantiated graph is updated in place
// when the next batch has the same launch topology.
//
// Each assembly's result equals rbg_bin_graph on that assembly alone: the
// kernels are the single-assembly kernels behind a descriptor lookup, and
// the host steps are the same functions with private rand() state.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <tuple>
#include <thread>

#include "engine_internal.h"

namespace rbg {
namespace {

constexpr int kVariants[4] = {0, 1, 2, 4};

inline int vslot(int v) { return v == 0 ? 0 : (v == 1 ? 1 : (v == 2 ? 2 : 3)); }

struct AsmPlan {
  int orig = 0;
  const rbg_params *p = nullptr;
  const rbg_assembly *in = nullptr;
  int64_t n = 0, nbases = 0;
  int S = 0, Su = 4, Kp = 16, m = 500, mpad = 512, K = 200, E = 136;
  bool fused = false, abdfirst = false;
  bool gemm = false;                   // dense regime on the one-hot GEMM (not in the queue)
  double w_comp = 0.0;
  int variant = 0, P = 4, cap = 288;
  // offsets into the batch buffers (elements of each buffer's type)
  int64_t row0 = 0, base0 = 0, dep0 = 0, code0 = 0, unit0 = 0, u16_0 = 0, col0 = 0, acc0 = 0;
  int64_t sv0 = 0, topk0 = 0, gbuf0 = 0, gcnt0 = 0, pair0 = 0, winv0 = 0;
  int np = 0;
  std::shared_ptr<const std::vector<int32_t>> pairs;
};

// Slices per row block for an assembly of the batch: the batch's row blocks
// already give the GPU its parallelism, so slices only bound the size of one
// work item (32 rows x n*4/P columns), which bounds the tail of the
// persistent kernel.  `mult` scales the pairs-per-item target (the autotuner's
// choice for the assembly's (variant, m, log2 n)).
int batch_slices(int64_t n, int K, int variant, double mult = 1.0) {
  const double target = (variant == 0 ? 4.0e5 : 3.0e6) * mult;   // pairs per work item
  int64_t P = (int64_t)std::ceil(4.0 * 32.0 * (double)n / target);
  const int pmax = std::max(4, std::min(32, (6400 / std::max(K, 1)) / 4 * 4));
  P = std::min<int64_t>(std::max<int64_t>(P, 4), pmax);
  P = std::min<int64_t>(P, std::max<int64_t>(4, (n / 64) / 4 * 4));
  return (int)((P + 3) / 4 * 4);
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// A captured stream segment, instantiated once and updated in place while the
// launch topology stays the same.
struct GraphSlot {
  cudaGraphExec_t exec = nullptr;
  void run(cudaStream_t s, cudaGraph_t g, int &launches) {
    if (exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(exec, g, &info) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphExecDestroy(exec);
        exec = nullptr;
      }
    }
    if (!exec) {
      const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        exec = nullptr;
        CK(e);
      }
    }
    cudaGraphDestroy(g);
    CK(cudaGraphLaunch(exec, s));
    ++launches;
  }
};

struct GraphCache {
  GraphSlot seg[3];
};

std::mutex g_graph_mu;
std::map<rbg_ctx *, std::unique_ptr<GraphCache>> g_graphs;

GraphCache &graphs_of(rbg_ctx *c) {
  std::lock_guard<std::mutex> lk(g_graph_mu);
  auto &p = g_graphs[c];
  if (!p) p = std::make_unique<GraphCache>();
  return *p;
}

// Runs `body` (stream work on c->stream) directly or as a captured graph.
template <typename F>
void captured(rbg_ctx *c, int seg, bool use_graph, int &graph_launches, F &&body) {
  if (!use_graph) {
    body();
    CK(cudaGetLastError());
    return;
  }
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
  try {
    body();
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(c->stream, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamEndCapture(c->stream, &g));
  graphs_of(c).seg[seg].run(c->stream, g, graph_launches);
}

template <typename T>
T *dptr(DBuf &b, int64_t off) { return b.as<T>() + off; }

inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

void validate_assembly(const rbg_assembly &x, const rbg_params *p, const std::string &who) {
  validate_params(p);
  if (x.n < 0 || (x.n > 0 && (!x.offsets || !x.seqcat)))
    throw Error(RBG_ERR_ARG, who + "bad sequence arguments");
  if (x.S < 0 || x.S > kMaxS) throw Error(RBG_ERR_UNSUPPORTED, who + "S must be in 0..64");
  if (x.S > 0 && x.n > 0 && !x.depth) throw Error(RBG_ERR_ARG, who + "depth is null");
  if (x.n >= (1 << 27)) throw Error(RBG_ERR_UNSUPPORTED, who + "at most 2^27 - 1 contigs");
  if (x.n > 0 && x.offsets[0] != 0) throw Error(RBG_ERR_ARG, who + "offsets[0] must be 0");
  for (int64_t q = 0; q < x.n; ++q)
    if (x.offsets[q + 1] < x.offsets[q])
      throw Error(RBG_ERR_ARG, who + "offsets must be non-decreasing");
  const bool fused = (p->force_path == 2) || (p->force_path == 0 && x.n > 25000);
  if (fused && x.n <= 2500)
    throw Error(RBG_ERR_ARG, who + "the fused path samples 2500 contigs; need n > 2500");
}

int64_t batch_request_bytes(const rbg_params *p, int64_t n, int64_t nbases, int S) {
  const int m = p->m, mpad = mpad_of(m), K = p->max_edges;
  const int Su = (std::max(S, 1) + 3) & ~3, Kp = unit16_stride(S);
  const int E = p->k == 4 ? 136 : (p->k == 3 ? 32 : (p->k == 2 ? 10 : 2));
  const double w_comp = (p->w_comp < 0.0) ? (S <= 2 ? 1.0 : 0.0) : p->w_comp;
  const bool fused = (p->force_path == 2) || (p->force_path == 0 && n > 25000);
  const bool abd = fused && p->abdfirst && S > 1 && w_comp < 1.0 && w_comp < p->min_edge;
  const int P = batch_slices(n, K, abd ? Kp / 16 : 0);
  const int64_t cap = allpairs_cap(K);
  int64_t b = nbases + nbases / 4 + nbases / 8 + 64;             // ASCII, 2-bit words, mask
  b += n * (int64_t)(S * 4 + 8 + E * 8 + 4 + 2 * mpad + Su * 4 + Kp * 2 + 1);
  b += n * (int64_t)K * (8 + 4 + 4) + n * 32;                    // top-K, neighbour lists
  if (abd)
    b += n * 256 * (16 + 2 * 8) + n * 12;                        // admitted pairs, keys, rows
  else if (dense_on_gemm() && onehot_mma_fits(n, m)) {           // one-hot rows, candidate lists
    int GR = 1, GC = 1;
    onehot_mma_grid((int)((n + 255) / 256), (int)((n + 255) / 256), 148, &GR, &GC);
    b += n * (int64_t)std::max(128, 136 * m / 8) +
         ((n + 31) / 32) * 32 * 2 * GC * ((int64_t)onehot_mma_cap(n, GC, K, 0) * 4 + 4);
  }
  else
    b += ((n + 31) / 32) * P * 32 * (cap * 8 + 4);               // slice candidate buffers
  b += n * (int64_t)K / 2 * 16;                                   // edge arrays (bound)
  b += 30000 * 12 + (m + 1) * 4 + 4096;                          // b0 pairs, tables of sv
  return b;
}

void release_batch_graphs(rbg_ctx *c) {
  std::lock_guard<std::mutex> lk(g_graph_mu);
  auto it = g_graphs.find(c);
  if (it == g_graphs.end()) return;
  for (auto &s : it->second->seg)
    if (s.exec) cudaGraphExecDestroy(s.exec);
  g_graphs.erase(it);
}

namespace {

// Layout of one batch: per-assembly plans in batch order (grouped by sketch
// configuration) and the sizes of the shared buffers.
struct BatchPlan {
  std::vector<AsmPlan> P;              // caller order
  std::vector<int> ord;                // batch position -> caller index
  int64_t rows = 0, bases = 0, dep = 0, code = 0, unit = 0, u16 = 0, col = 0, acc = 0, sv = 0;
  int64_t topk = 0, gbuf = 0, gcnt = 0, npairs = 0, winv = 0, pairs_scored = 0;
  int64_t sym_rows = 0;                // rows of the tensor-core (symmetric pass) assemblies
  int max_m = 2, max_k = 1, max_s = 0;
  const AsmPlan &at(int b) const { return P[ord[b]]; }
};

using TuneKey = std::tuple<int, int, int>;

TuneKey tune_key(const AsmPlan &a) {
  int lg = 0;
  while (lg < 62 && ((int64_t)1 << (lg + 1)) <= std::max<int64_t>(a.n, 1)) ++lg;
  return TuneKey(a.variant, a.m, lg);
}

// tune: the autotuner's choices (null: none); untuned: the multiplier for keys
// it has no choice for yet.
void plan_batch(const rbg_params *defaults, const rbg_assembly *asms, int nb, BatchPlan &L,
                const std::map<TuneKey, double> *tune = nullptr, double untuned = 1.0) {
  L.P.assign(nb, AsmPlan());
  for (int i = 0; i < nb; ++i) {
    AsmPlan &a = L.P[i];
    const rbg_assembly &x = asms[i];
    a.orig = i;
    a.in = &x;
    a.p = x.params ? x.params : defaults;
    validate_assembly(x, a.p, "assembly " + std::to_string(i) + ": ");
    // (assemblies on the one-permutation metric or the inverted index are
    // routed to the single-assembly path by rbg_bin_batch)
    if (a.p->oph_k > 0 || a.p->graph_index)
      throw Error(RBG_ERR_ARG, "assembly " + std::to_string(i) + ": not a batch-kernel assembly");
    a.n = x.n;
    a.nbases = x.n > 0 ? x.offsets[x.n] : 0;
    a.S = x.S;
    a.Su = (std::max(a.S, 1) + 3) & ~3;
    a.Kp = unit16_stride(a.S);
    a.m = a.p->m;
    a.mpad = mpad_of(a.m);
    a.K = a.p->max_edges;
    a.E = a.p->k == 4 ? 136 : (a.p->k == 3 ? 32 : (a.p->k == 2 ? 10 : 2));
    a.w_comp = (a.p->w_comp < 0.0) ? (a.S <= 2 ? 1.0 : 0.0) : a.p->w_comp;
    a.fused = (a.p->force_path == 2) || (a.p->force_path == 0 && a.n > 25000);
    a.abdfirst = a.fused && a.p->abdfirst && a.S > 1 && a.w_comp < 1.0 && a.w_comp < a.p->min_edge;
    a.variant = a.abdfirst ? a.Kp / 16 : 0;
    a.gemm = !a.abdfirst && dense_on_gemm() && onehot_mma_fits(a.n, a.m);
    double mult = untuned;
    if (tune) {
      const auto it = tune->find(tune_key(a));
      if (it != tune->end()) mult = it->second;
    }
    a.P = batch_slices(a.n, a.K, a.variant, mult);
    a.cap = allpairs_cap(a.K);
  }
  // group order: equal count configuration, then equal sketch tables
  L.ord.resize(nb);
  std::iota(L.ord.begin(), L.ord.end(), 0);
  auto key = [&](int i) {
    const rbg_params *p = L.P[i].p;
    return std::make_tuple(p->k, p->gc_norm, p->gc_norm_cap, p->m, p->pmh_seed,
                           p->fp_contract != 0, p->win_bits);
  };
  std::stable_sort(L.ord.begin(), L.ord.end(), [&](int x, int y) { return key(x) < key(y); });
  for (int b = 0; b < nb; ++b) {
    AsmPlan &a = L.P[L.ord[b]];
    a.row0 = L.rows; L.rows += a.n;
    a.base0 = L.bases; L.bases += a.nbases;
    a.dep0 = L.dep; L.dep += a.n * a.S;
    a.code0 = L.code; L.code += a.n * a.mpad;
    a.unit0 = L.unit; L.unit += a.n * a.Su;
    a.u16_0 = L.u16; L.u16 += a.n * a.Kp;
    a.col0 = L.col; L.col += std::max(a.S, 1);
    a.acc0 = L.acc; L.acc += 3 * std::max(a.S, 1);
    a.sv0 = L.sv; L.sv += a.m + 1;
    a.topk0 = L.topk; L.topk += a.n * a.K;
    const int64_t nbk = (a.n + 31) / 32;
    a.gbuf0 = L.gbuf;
    a.gcnt0 = L.gcnt;
    if (a.variant != 0) {
      L.sym_rows += a.n;
    } else if (!a.gemm) {
      L.gbuf += nbk * a.P * 32 * a.cap;
      L.gcnt += nbk * a.P * 32;
    }
    a.winv0 = L.winv; L.winv += a.n * a.E;
    if (a.p->base_on) {
      a.pairs = b0_pairs(a.n);
      a.np = (int)(a.pairs->size() / 2);
    }
    a.pair0 = L.npairs; L.npairs += a.np;
    L.max_m = std::max(L.max_m, a.m);
    L.max_k = std::max(L.max_k, a.K);
    L.max_s = std::max(L.max_s, a.S);
    L.pairs_scored += a.n * (a.n - 1) / 2;
  }
  if ((double)L.rows * L.max_k >= 2147483647.0)
    throw Error(RBG_ERR_UNSUPPORTED, "batch too large: rows x max_edges must stay below 2^31");
}

void ensure_buffers(BatchBufs &B, const BatchPlan &L, int nb) {
  const int64_t rows1 = std::max<int64_t>(L.rows, 1);
  const int64_t nwords = (L.bases + 15) / 16 + 1;
  B.ascii.ensure((size_t)((L.bases + 15) / 16) * 16 + 16);
  B.offsets.ensure((L.rows + 1) * sizeof(int64_t));
  B.depth.ensure(std::max<int64_t>(L.dep, 1) * sizeof(float));
  B.packed.ensure(nwords * 4);
  B.nmask.ensure((nwords / 2 + 2) * 4);
  B.winv.ensure(std::max<int64_t>(L.winv, 1) * sizeof(double));
  B.ecnt.ensure(rows1 * sizeof(int32_t));
  B.codesA.ensure(std::max<int64_t>(L.code, 16));
  B.codesB.ensure(std::max<int64_t>(L.code, 16));
  B.unit.ensure(std::max<int64_t>(L.unit, 4) * sizeof(float));
  B.unit16.ensure(std::max<int64_t>(L.u16, 16) * sizeof(uint16_t));
  B.anynz.ensure(rows1);
  B.colnorm.ensure(L.col * sizeof(double));
  B.colacc.ensure(L.acc * sizeof(double));
  B.svbits.ensure(L.sv * sizeof(uint32_t));
  B.topk.ensure(std::max<int64_t>(L.topk, 1) * sizeof(uint64_t));
  B.topk_cnt.ensure(rows1 * sizeof(int32_t));
  B.maxc_cand.ensure(rows1 * sizeof(uint32_t));
  B.maxc_all.ensure(rows1 * sizeof(uint32_t));
  B.stats.ensure(2 * sizeof(unsigned long long));
  B.gbuf.ensure(std::max<int64_t>(L.gbuf, 1) * sizeof(uint64_t));
  B.gcnt.ensure(std::max<int64_t>(L.gcnt, 1) * sizeof(int32_t));
  B.pairs.ensure(std::max<int64_t>(L.npairs, 1) * 2 * sizeof(int32_t));
  B.pair_cnt.ensure(std::max<int64_t>(L.npairs, 1) * sizeof(uint32_t));
  B.b0.ensure(nb * sizeof(float));
  B.nbr.ensure(std::max<int64_t>(L.topk, 1) * sizeof(uint32_t));
  B.nbr_sv.ensure(std::max<int64_t>(L.topk, 1) * sizeof(float));
  B.nbr_cnt.ensure(rows1 * sizeof(int32_t));
  B.row_edges.ensure((L.rows + 1) * sizeof(int32_t));
  B.edge0s.ensure((nb + 1) * sizeof(int64_t));
  B.desc.ensure(nb * sizeof(BatchAsm));
  B.row0s.ensure((nb + 1) * sizeof(int64_t));
  B.pair0s.ensure((nb + 1) * sizeof(int64_t));
  // work lists and queue counters: the whole batch, then one set per run
  B.lists.ensure((1 + kChunks) * 4 * (nb + 1) * sizeof(int32_t));
  B.item0s.ensure((1 + kChunks) * 4 * (nb + 1) * sizeof(int64_t));
  B.queues.ensure((1 + kChunks) * 4 * sizeof(unsigned long long));
  B.e_from.ensure(4); B.e_to.ensure(4); B.e_scomp.ensure(4); B.e_score.ensure(4);
  if (L.sym_rows > 0) {
    // RBG_PAIR_CAP: a small first list, to exercise the overflow path
    const char *pc = getenv("RBG_PAIR_CAP");
    if (pc && B.sym_cap == 0) B.sym_cap = std::max<uint64_t>(1024, strtoull(pc, nullptr, 10));
    else
      B.sym_cap = std::max<uint64_t>(B.sym_cap,
                                     std::max<uint64_t>(1u << 16, (uint64_t)L.sym_rows * 256));
    B.sym_pairs.ensure(B.sym_cap * sizeof(uint4));
    B.sym_keys.ensure(2 * B.sym_cap * sizeof(uint64_t));
    B.sym_rowcnt.ensure(rows1 * sizeof(int32_t));
    B.sym_rowoff.ensure((rows1 + 1) * sizeof(int64_t));
    B.sym_np.ensure(sizeof(unsigned long long));
  }
}

SymOut sym_out(BatchBufs &B) {
  SymOut o;
  o.pairs = B.sym_pairs.as<uint4>();
  o.npairs = B.sym_np.as<unsigned long long>();
  o.cap = B.sym_cap;
  o.rowcnt = B.sym_rowcnt.as<int32_t>();
  return o;
}

// The device descriptor of the assembly at batch position b (edge arrays are
// filled in once the edge total is known).
BatchAsm describe(BatchBufs &B, const AsmPlan &a, int b) {
  const rbg_params *p = a.p;
  BatchAsm d;
  GraphArgs &g = d.g;
  g.n = a.n; g.m = a.m; g.mpad = a.mpad; g.S = a.S; g.K = a.K; g.Su = a.Su; g.Kp = a.Kp;
  g.codesA = dptr<uint8_t>(B.codesA, a.code0);
  g.codesB = dptr<uint8_t>(B.codesB, a.code0);
  g.depth_raw = dptr<float>(B.depth, a.dep0);
  g.unit = dptr<float>(B.unit, a.unit0);
  g.unit16 = dptr<uint16_t>(B.unit16, a.u16_0);
  g.anynz = dptr<uint8_t>(B.anynz, a.row0);
  g.colnorm = dptr<double>(B.colnorm, a.col0);
  g.min_cv = (float)p->min_cv;
  g.min_cv_d = p->min_cv;
  g.has_depth = a.S > 0;
  g.wjac_norm = p->wjac_norm;
  g.small_path = a.fused ? 0 : 1;
  g.prefilter = a.abdfirst ? 1 : 0;
  const double abd_corr_min = a.abdfirst ? (p->min_edge - a.w_comp) / (1.0 - a.w_comp) : -2.0;
  g.prefilter_eps = (float)(abd_corr_min - 1e-4);
  g.sv_bits = dptr<uint32_t>(B.svbits, a.sv0);
  g.topk = dptr<uint64_t>(B.topk, a.topk0);
  g.topk_cnt = dptr<int32_t>(B.topk_cnt, a.row0);
  g.maxcnt_cand = dptr<uint32_t>(B.maxc_cand, a.row0);
  g.maxcnt_all = dptr<uint32_t>(B.maxc_all, a.row0);
  g.stats = B.stats.as<unsigned long long>();
  g.key_floor = admission_floor();
  d.row0 = a.row0;
  d.gbuf = dptr<uint64_t>(B.gbuf, a.gbuf0);
  d.gcnt = dptr<int32_t>(B.gcnt, a.gcnt0);
  d.cap = a.cap;
  d.P = a.P;
  d.variant = a.gemm ? -1 : a.variant;   // -1: neither the merge nor the pair-list selection
  prefilter_bands(a.S, g.prefilter_eps, &d.lo, &d.hi, &d.lo16);
  d.colnorm_on = need_colnorm(p, a.S) ? 1 : 0;
  d.colacc = dptr<double>(B.colacc, a.acc0);
  d.base_on = p->base_on ? 1 : 0;
  d.np = a.np;
  d.pair0 = a.pair0;
  d.b0 = dptr<float>(B.b0, b);
  d.sv_out = dptr<uint32_t>(B.svbits, a.sv0);
  EmitArgs &e = d.e;
  e.n = a.n; e.K = a.K; e.mutual = p->mutual; e.small_path = a.fused ? 0 : 1;
  e.topk = g.topk; e.topk_cnt = g.topk_cnt;
  e.nbr_sorted = dptr<uint32_t>(B.nbr, a.topk0);
  e.nbr_sv = dptr<float>(B.nbr_sv, a.topk0);
  e.nbr_cnt = dptr<int32_t>(B.nbr_cnt, a.row0);
  e.row_edges = dptr<int32_t>(B.row_edges, a.row0);
  WeightArgs &w = d.w;
  w.S = a.S;
  w.unit = g.unit;
  w.Su = a.Su;
  w.depth_raw = g.depth_raw;
  w.colnorm = d.colnorm_on ? g.colnorm : nullptr;
  w.w_comp = a.w_comp;
  w.min_edge = p->min_edge;
  w.neg_thr = p->neg_thr;
  w.wjac_cut = p->wjac_cut;
  w.depth_sim = p->depth_sim;
  w.depth_fuse = p->depth_fuse;
  w.wjac_gate = p->wjac_gate;
  w.contract = p->fp_contract;
  return d;
}

// Work lists of the persistent all-pairs kernels, one per variant slot.
struct Lists {
  std::vector<int32_t> list[4];
  std::vector<int64_t> item0[4];
  size_t smem[4] = {0, 0, 0, 0};
};

// Sketch of the batch positions [bb, be): pack of the words holding their
// bases, count (one launch per k / GC-norm run), register minimum (one per
// sketch-table run); returns the number of kernel launches.  A word shared
// with the next range is packed again by that range's call (same stream,
// complete bytes by then); this range's contigs read only their own bases.
int launch_sketch_groups(rbg_ctx *c, BatchBufs &B, const BatchPlan &L,
                         const std::vector<Tables *> &tab, int bb, int be) {
  int launches = 0;
  if (bb >= be) return 0;
  const int64_t base_lo = L.at(bb).base0, base_hi = L.at(be - 1).base0 + L.at(be - 1).nbases;
  if (base_hi > base_lo) {
    launch_pack_range(B.ascii.as<char>(), L.bases, (base_lo / 16) & ~(int64_t)1,
                      (base_hi + 15) / 16, B.packed.as<uint32_t>(), B.nmask.as<uint32_t>(),
                      c->stream);
    ++launches;
  }
  for (int b0 = bb; b0 < be;) {
    const rbg_params *p = L.at(b0).p;
    int b1 = b0;
    while (b1 < be && L.at(b1).p->k == p->k && L.at(b1).p->gc_norm == p->gc_norm &&
           L.at(b1).p->gc_norm_cap == p->gc_norm_cap)
      ++b1;
    const AsmPlan &f = L.at(b0);
    const AsmPlan &l = L.at(b1 - 1);
    SketchArgs a;
    a.packed = B.packed.as<uint32_t>();
    a.nmask = B.nmask.as<uint32_t>();
    a.offsets = B.offsets.as<int64_t>() + f.row0;
    a.n = l.row0 + l.n - f.row0;
    a.k = p->k;
    a.gc_norm = p->gc_norm;
    a.gc_cap = p->gc_norm_cap;
    a.n_elems = tab[b0]->t->n_elems;
    a.rank_of_code = tab[b0]->rank.as<int16_t>();
    a.elem_winv = B.winv.as<double>() + f.winv0;
    a.elem_cnt = B.ecnt.as<int32_t>() + f.row0;
    launch_count(a, c->stream);
    launches += a.n ? 1 : 0;
    for (int t0 = b0; t0 < b1;) {
      int t1 = t0;
      while (t1 < b1 && tab[t1] == tab[t0]) ++t1;
      const AsmPlan &tf = L.at(t0);
      const AsmPlan &tl = L.at(t1 - 1);
      SketchArgs r = a;
      r.offsets = B.offsets.as<int64_t>() + tf.row0;
      r.n = tl.row0 + tl.n - tf.row0;
      r.m = tf.m;
      r.mpad = tf.mpad;
      r.elem_winv = B.winv.as<double>() + tf.winv0;
      r.elem_cnt = B.ecnt.as<int32_t>() + tf.row0;
      r.order = tab[t0]->order.as<RegOrder>();
      r.UT = tab[t0]->UT.as<double>();
      r.codeA = tab[t0]->codeA.as<uint8_t>();
      r.W32 = tab[t0]->W32.as<uint32_t>();
      r.codesA = B.codesA.as<uint8_t>() + tf.code0;
      r.codesB = B.codesB.as<uint8_t>() + tf.code0;
      r.winners32 = nullptr;
      launch_minreduce(r, c->stream);
      launches += r.n ? 1 : 0;
      t0 = t1;
    }
    b0 = b1;
  }
  return launches;
}

// Depth rows, b0, all-pairs and merge for the whole batch.
int launch_graph_stage(rbg_ctx *c, BatchBufs &B, const BatchPlan &L, const Lists &W, int nb,
                       bool timed = false) {
  const BatchAsm *dD = B.desc.as<BatchAsm>();
  const int64_t rows1 = std::max<int64_t>(L.rows, 1);
  int launches = 0;
  launch_unit_rows_batch(dD, B.row0s.as<int64_t>(), nb, L.rows, c->stream);
  CK(cudaMemsetAsync(B.colacc.p, 0, L.acc * sizeof(double), c->stream));
  launch_colnorm_batch(dD, nb, L.max_s, c->stream);
  launch_b0_batch(dD, B.pair0s.as<int64_t>(), nb, L.npairs, B.pairs.as<int32_t>(),
                  B.pair_cnt.as<uint32_t>(), L.max_m, c->stream);
  launches += (L.rows ? 1 : 0) + (L.max_s > 1 ? 2 : 0) + (L.npairs ? 2 : 1);
  CK(cudaMemsetAsync(B.maxc_cand.p, 0, rows1 * sizeof(uint32_t), c->stream));
  CK(cudaMemsetAsync(B.maxc_all.p, 0, rows1 * sizeof(uint32_t), c->stream));
  CK(cudaMemsetAsync(B.stats.p, 0, 2 * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(B.queues.p, 0, 4 * sizeof(unsigned long long), c->stream));
  const SymOut o = L.sym_rows > 0 ? sym_out(B) : SymOut{};
  if (L.sym_rows > 0) {
    CK(cudaMemsetAsync(B.sym_rowcnt.p, 0, rows1 * sizeof(int32_t), c->stream));
    CK(cudaMemsetAsync(B.sym_np.p, 0, sizeof(unsigned long long), c->stream));
  }
  for (int v = 0; v < 4; ++v) {
    if (W.list[v].empty()) continue;
    if (timed) CK(cudaEventRecord(B.tev[2 * v], c->stream));
    launch_allpairs_batch(dD, kVariants[v], B.lists.as<int32_t>() + v * (nb + 1),
                          B.item0s.as<int64_t>() + v * (nb + 1), (int)W.list[v].size(),
                          W.item0[v].back(), W.smem[v], B.queues.as<unsigned long long>() + v,
                          o, c->stream);
    if (timed) CK(cudaEventRecord(B.tev[2 * v + 1], c->stream));
    ++launches;
  }
  if (!W.list[0].empty()) {
    launch_merge_batch(dD, B.row0s.as<int64_t>(), nb, L.rows, c->stream);
    ++launches;
  }
  if (L.sym_rows > 0) {
    launch_rows_topk_batch(dD, B.row0s.as<int64_t>(), nb, L.rows, o, B.sym_rowoff.as<int64_t>(),
                           B.sym_keys.as<uint64_t>(), c->stream);
    launches += 3;
  }
  return launches;
}

// Graph stage of the batch positions [bb, be) (rows [r0, r1), sampled pairs
// [p0, p1)) on work lists Wr whose device copies start at `lists` / `item0s`,
// with queue counters `next` (zeroed by the caller): depth rows, column norms,
// b0, the all-pairs passes and the dense merge.  The row top-K of the
// symmetric pass follows once every run is in.
int launch_graph_run(rbg_ctx *c, BatchBufs &B, const BatchPlan &L, const Lists &Wr, int nb,
                     int bb, int be, const int32_t *lists, const int64_t *item0s,
                     unsigned long long *next) {
  const BatchAsm *dD = B.desc.as<BatchAsm>();
  if (bb >= be) return 0;
  const AsmPlan &f = L.at(bb), &l = L.at(be - 1);
  const int64_t r0 = f.row0, r1 = l.row0 + l.n, p0 = f.pair0, p1 = l.pair0 + l.np;
  int launches = 0;
  launch_unit_rows_batch(dD, B.row0s.as<int64_t>(), nb, r1, c->stream, r0);
  launch_colnorm_batch(dD + bb, be - bb, L.max_s, c->stream);
  launch_b0_batch_range(dD, B.pair0s.as<int64_t>(), nb, p0, p1, B.pairs.as<int32_t>(),
                        B.pair_cnt.as<uint32_t>(), L.max_m, bb, be, c->stream);
  launches += (r1 > r0 ? 1 : 0) + (L.max_s > 1 ? 2 : 0) + (p1 > p0 ? 2 : 1);
  const SymOut o = L.sym_rows > 0 ? sym_out(B) : SymOut{};
  for (int v = 0; v < 4; ++v) {
    if (Wr.list[v].empty()) continue;
    launch_allpairs_batch(dD, kVariants[v], lists + v * (nb + 1), item0s + v * (nb + 1),
                          (int)Wr.list[v].size(), Wr.item0[v].back(), Wr.smem[v], next + v, o,
                          c->stream);
    ++launches;
  }
  if (!Wr.list[0].empty()) {
    launch_merge_batch(dD, B.row0s.as<int64_t>(), nb, r1, c->stream, r0);
    ++launches;
  }
  return launches;
}

// The work lists of batch positions [bb, be) only.
Lists sub_lists(const Lists &W, int bb, int be) {
  Lists R;
  for (int v = 0; v < 4; ++v) {
    R.smem[v] = W.smem[v];
    for (size_t k = 0; k < W.list[v].size(); ++k) {
      const int b = W.list[v][k];
      if (b < bb || b >= be) continue;
      if (R.item0[v].empty()) R.item0[v].push_back(0);
      R.list[v].push_back(b);
      R.item0[v].push_back(R.item0[v].back() + (W.item0[v][k + 1] - W.item0[v][k]));
    }
  }
  return R;
}

// Device descriptors of the batch positions and the per-variant work lists.
void build_items(BatchBufs &B, const BatchPlan &L, int nb, std::vector<BatchAsm> &D, Lists &W) {
  D.assign(nb, BatchAsm());
  W = Lists();
  for (int b = 0; b < nb; ++b) {
    const AsmPlan &a = L.at(b);
    D[b] = describe(B, a, b);
    if (a.n > 0 && !a.gemm) {
      const int vs = vslot(a.variant);
      if (W.item0[vs].empty()) W.item0[vs].push_back(0);
      W.list[vs].push_back(b);
      W.item0[vs].push_back(W.item0[vs].back() + allpairs_items(a.n, a.P));
      W.smem[vs] = std::max(W.smem[vs], allpairs_batch_smem(a.variant, a.mpad, a.Su));
    }
  }
}

// Autotuner.  For keys (variant, m, log2 n) of this batch it has no choice for,
// the graph stage runs again with the pairs-per-item target at 1x, 1/4 and 4x
// the rule's (outside the CUDA graphs), each variant's persistent launch timed
// by events; the fastest multiplier per variant becomes the choice for
// the batch's untuned keys of that variant.  The runs recompute the same
// values (top-K sets and maxima do not depend on the tiling).
int autotune_batch(rbg_ctx *c, BatchBufs &B, const rbg_params *defaults,
                   const rbg_assembly *asms, int nb, const BatchPlan &L0) {
  std::vector<TuneKey> fresh;
  for (int b = 0; b < nb; ++b) {
    const AsmPlan &a = L0.at(b);
    if (a.n == 0 || a.gemm) continue;
    const TuneKey k = tune_key(a);
    if (B.tune.count(k)) continue;
    if (std::find(fresh.begin(), fresh.end(), k) == fresh.end()) fresh.push_back(k);
  }
  if (fresh.empty()) return 0;
  const double mults[3] = {1.0, 0.25, 4.0};
  float t[3][4];
  for (auto &e : B.tev)
    if (!e) CK(cudaEventCreate(&e));
  for (int ci = 0; ci < 3; ++ci) {
    BatchPlan L;
    plan_batch(defaults, asms, nb, L, &B.tune, mults[ci]);
    ensure_buffers(B, L, nb);
    std::vector<BatchAsm> D;
    Lists W;
    build_items(B, L, nb, D, W);
    std::vector<int32_t> lists(4 * (nb + 1), 0);
    std::vector<int64_t> item0s(4 * (nb + 1), 0);
    for (int v = 0; v < 4; ++v) {
      std::copy(W.list[v].begin(), W.list[v].end(), lists.begin() + v * (nb + 1));
      std::copy(W.item0[v].begin(), W.item0[v].end(), item0s.begin() + v * (nb + 1));
    }
    CK(cudaMemcpyAsync(B.desc.p, D.data(), (size_t)nb * sizeof(BatchAsm), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(B.lists.p, lists.data(), lists.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(B.item0s.p, item0s.data(), item0s.size() * sizeof(int64_t),
                       cudaMemcpyHostToDevice, c->stream));
    launch_graph_stage(c, B, L, W, nb, true);
    CK(cudaStreamSynchronize(c->stream));
    for (int v = 0; v < 4; ++v) {
      t[ci][v] = 0.f;
      if (!W.list[v].empty()) CK(cudaEventElapsedTime(&t[ci][v], B.tev[2 * v], B.tev[2 * v + 1]));
    }
  }
  double best[4];
  for (int v = 0; v < 4; ++v) {
    int bi = 0;
    for (int ci = 1; ci < 3; ++ci)
      if (t[ci][v] < t[bi][v]) bi = ci;
    best[v] = mults[bi];
  }
  for (const TuneKey &k : fresh) B.tune[k] = best[vslot(std::get<0>(k))];
  return (int)fresh.size();
}

}  // namespace

void run_batch(rbg_ctx *c, const rbg_params *defaults, const rbg_assembly *asms, int nb,
               rbg_graph *out, rbg_batch_stats *st) {
  const auto t_start = std::chrono::steady_clock::now();
  if (nb < 0 || (nb > 0 && (!asms || !out))) throw Error(RBG_ERR_ARG, "bad batch arguments");
  for (int i = 0; i < nb; ++i) std::memset(&out[i], 0, sizeof(out[i]));
  rbg_batch_stats stats;
  std::memset(&stats, 0, sizeof(stats));
  stats.n_assemblies = nb;
  if (nb == 0) {
    if (st) *st = stats;
    return;
  }
  if (!c->batch) c->batch = std::make_unique<BatchBufs>();
  BatchBufs &B = *c->batch;
  const bool use_graph = getenv("RBG_NO_GRAPHS") == nullptr;

  BatchPlan L;
  plan_batch(defaults, asms, nb, L, &B.tune, 1.0);
  const int64_t rows = L.rows, rows1 = std::max<int64_t>(rows, 1);
  stats.rows = rows;
  stats.pairs = L.pairs_scored;
  ensure_buffers(B, L, nb);
  std::vector<Tables *> tab(nb);
  for (int b = 0; b < nb; ++b) {
    const rbg_params *p = L.at(b).p;
    auto k = std::make_tuple(p->k, p->m, p->pmh_seed, (int)(p->fp_contract != 0), p->win_bits);
    auto &slot = B.tables[k];
    if (!slot) slot = make_tables(p, c->stream);
    tab[b] = slot.get();
  }
  std::vector<BatchAsm> D;
  Lists W;
  build_items(B, L, nb, D, W);
  const bool autotune = getenv("RBG_NO_AUTOTUNE") == nullptr;
  for (int v = 0; v < 4; ++v) stats.items += W.item0[v].empty() ? 0 : W.item0[v].back();

  // Batch positions in up to kChunks runs of about equal bases: the copy
  // stream brings in run r's sequences and depths while the main stream
  // sketches and graphs run r - 1.
  std::vector<int> runcut{0};
  {
    const int64_t per = std::max<int64_t>(L.bases / kChunks, 1);
    for (int b = 0; b < nb; ++b) {
      const AsmPlan &a = L.at(b);
      if (b + 1 < nb && (int)runcut.size() < kChunks && a.base0 + a.nbases >= per * (int64_t)runcut.size())
        runcut.push_back(b + 1);
    }
    runcut.push_back(nb);
  }
  const int nruns = (int)runcut.size() - 1;
  std::vector<Lists> Wr(nruns);
  for (int r = 0; r < nruns; ++r) Wr[r] = sub_lists(W, runcut[r], runcut[r + 1]);

  // pinned staging: global offsets, b0 pairs, descriptors, index arrays (the
  // work lists of the whole batch, then of each run)
  const size_t off_bytes = (rows + 1) * sizeof(int64_t);
  const size_t pair_bytes = (size_t)L.npairs * 2 * sizeof(int32_t);
  const size_t desc_bytes = (size_t)nb * sizeof(BatchAsm);
  const size_t nlist = (size_t)(1 + nruns) * 4 * (nb + 1);
  const size_t idx_bytes = 2 * (nb + 1) * sizeof(int64_t) + nlist * (sizeof(int32_t) + sizeof(int64_t));
  B.hstage.ensure(up256(off_bytes) + up256(pair_bytes) + up256(desc_bytes) + up256(idx_bytes));
  char *hs = B.hstage.as<char>();
  int64_t *h_off = (int64_t *)hs;
  int32_t *h_pairs = (int32_t *)(hs + up256(off_bytes));
  BatchAsm *h_desc = (BatchAsm *)(hs + up256(off_bytes) + up256(pair_bytes));
  int64_t *h_row0s = (int64_t *)(hs + up256(off_bytes) + up256(pair_bytes) + up256(desc_bytes));
  int64_t *h_pair0s = h_row0s + (nb + 1);
  int32_t *h_lists = (int32_t *)(h_pair0s + (nb + 1));
  int64_t *h_item0s = (int64_t *)(h_lists + nlist);
  for (int b = 0; b < nb; ++b) {
    const AsmPlan &a = L.at(b);
    for (int64_t q = 0; q < a.n; ++q) h_off[a.row0 + q] = a.base0 + a.in->offsets[q];
    if (a.np) std::memcpy(h_pairs + 2 * a.pair0, a.pairs->data(), (size_t)a.np * 2 * sizeof(int32_t));
    h_row0s[b] = a.row0;
    h_pair0s[b] = a.pair0;
  }
  h_off[rows] = L.bases;
  h_row0s[nb] = rows;
  h_pair0s[nb] = L.npairs;
  std::memcpy(h_desc, D.data(), desc_bytes);
  std::fill(h_lists, h_lists + nlist, 0);
  std::fill(h_item0s, h_item0s + nlist, 0);
  for (int r = -1; r < nruns; ++r) {
    const Lists &X = r < 0 ? W : Wr[r];
    const size_t base = (size_t)(r + 1) * 4 * (nb + 1);
    for (int v = 0; v < 4; ++v) {
      std::copy(X.list[v].begin(), X.list[v].end(), h_lists + base + v * (nb + 1));
      std::copy(X.item0[v].begin(), X.item0[v].end(), h_item0s + base + v * (nb + 1));
    }
  }

  // ── inputs to the device, sketched behind the copies ────────────────────
  cudaEvent_t ev0 = c->ev[0], ev1 = c->ev[1], ev2 = c->ev[2], ev3 = c->ev[3], ev4 = c->ev[4];
  CK(cudaEventRecord(ev0, c->stream));
  CK(cudaMemcpyAsync(B.offsets.p, h_off, off_bytes, cudaMemcpyHostToDevice, c->stream));
  if (pair_bytes) CK(cudaMemcpyAsync(B.pairs.p, h_pairs, pair_bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(B.desc.p, h_desc, desc_bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(B.row0s.p, h_row0s, (nb + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(B.pair0s.p, h_pair0s, (nb + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(B.lists.p, h_lists, nlist * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(B.item0s.p, h_item0s, nlist * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  // graph-stage accumulators, zeroed once for all runs
  CK(cudaMemsetAsync(B.colacc.p, 0, L.acc * sizeof(double), c->stream));
  CK(cudaMemsetAsync(B.maxc_cand.p, 0, rows1 * sizeof(uint32_t), c->stream));
  CK(cudaMemsetAsync(B.maxc_all.p, 0, rows1 * sizeof(uint32_t), c->stream));
  CK(cudaMemsetAsync(B.stats.p, 0, 2 * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(B.queues.p, 0, (size_t)(1 + nruns) * 4 * sizeof(unsigned long long),
                     c->stream));
  if (L.sym_rows > 0) {
    CK(cudaMemsetAsync(B.sym_rowcnt.p, 0, rows1 * sizeof(int32_t), c->stream));
    CK(cudaMemsetAsync(B.sym_np.p, 0, sizeof(unsigned long long), c->stream));
  }
  int launches = 0;
  {
    CK(cudaEventRecord(c->ev_cin, c->stream));             // earlier work on the buffers is done
    CK(cudaStreamWaitEvent(c->copy, c->ev_cin, 0));
    const size_t abytes = (size_t)((L.bases + 15) / 16) * 16 + 16;
    // Every copy is queued first: the host waits inside the dense GEMMs below,
    // and the copies must not wait for it.  The depth rows go through pinned
    // staging, since a copy from pageable memory would hold the host until the
    // copies queued before it are done.
    B.hdepth.ensure(std::max<int64_t>(L.dep, 1) * sizeof(float));
    for (size_t r = 0; r + 1 < runcut.size(); ++r) {
      for (int b = runcut[r]; b < runcut[r + 1]; ++b) {
        const AsmPlan &a = L.at(b);
        if (a.nbases)
          CK(cudaMemcpyAsync(B.ascii.as<char>() + a.base0, a.in->seqcat, (size_t)a.nbases,
                             cudaMemcpyHostToDevice, c->copy));
        if (a.n && a.S) {
          float *hd = B.hdepth.as<float>() + a.dep0;
          std::memcpy(hd, a.in->depth, (size_t)a.n * a.S * sizeof(float));
          CK(cudaMemcpyAsync(B.depth.as<float>() + a.dep0, hd, (size_t)a.n * a.S * sizeof(float),
                             cudaMemcpyHostToDevice, c->copy));
        }
      }
      if (r + 2 == runcut.size())
        CK(cudaMemsetAsync(B.ascii.as<char>() + L.bases, 0, abytes - (size_t)L.bases, c->copy));
      CK(cudaEventRecord(c->ev_chunk[r], c->copy));
    }
    for (size_t r = 0; r + 1 < runcut.size(); ++r) {
      CK(cudaStreamWaitEvent(c->stream, c->ev_chunk[r], 0));
      launches += launch_sketch_groups(c, B, L, tab, runcut[r], runcut[r + 1]);
      const size_t base = (size_t)(r + 1) * 4 * (nb + 1);
      launches += launch_graph_run(c, B, L, Wr[r], nb, runcut[r], runcut[r + 1],
                                   B.lists.as<int32_t>() + base, B.item0s.as<int64_t>() + base,
                                   B.queues.as<unsigned long long>() + (size_t)(r + 1) * 4);
      // dense assemblies of the run: one-hot GEMM and row scan each, on the
      // b0 and similarity tables just computed
      for (int b = runcut[r]; b < runcut[r + 1]; ++b)
        if (L.at(b).gemm && L.at(b).n > 0) {
          dense_allpairs_onehot(c, D[b].g);
          launches += 6;
        }
    }
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(ev1, c->stream));

  // ── segment 1: row top-K of the symmetric pass, maxima and b0 to the host ──
  const size_t mx_bytes = up256(2 * rows1 * sizeof(uint32_t));
  const size_t e0_bytes = up256((nb + 1) * sizeof(int64_t));
  B.hout.ensure(mx_bytes + up256(nb * sizeof(float)) + e0_bytes + sizeof(unsigned long long));
  uint32_t *h_maxc = B.hout.as<uint32_t>();
  float *h_b0 = (float *)(B.hout.as<char>() + mx_bytes);
  int64_t *h_edge0s = (int64_t *)(B.hout.as<char>() + mx_bytes + up256(nb * sizeof(float)));
  unsigned long long *h_np =
      (unsigned long long *)(B.hout.as<char>() + mx_bytes + up256(nb * sizeof(float)) + e0_bytes);
  // The symmetric pass reports how many pairs it admitted; a pass whose pairs
  // did not fit the list runs again, resident, with a larger one.
  bool reran = false;
  for (bool first = true;; first = false) {
    reran = !first;
    captured(c, 0, use_graph && first, stats.graph_launches, [&] {
      if (!first) {
        launches += launch_graph_stage(c, B, L, W, nb);
      } else if (L.sym_rows > 0) {
        launch_rows_topk_batch(B.desc.as<BatchAsm>(), B.row0s.as<int64_t>(), nb, rows, sym_out(B),
                               B.sym_rowoff.as<int64_t>(), B.sym_keys.as<uint64_t>(), c->stream);
        launches += 3;
      }
      if (rows) {
        CK(cudaMemcpyAsync(h_maxc, B.maxc_cand.p, rows * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaMemcpyAsync(h_maxc + rows1, B.maxc_all.p, rows * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, c->stream));
      }
      CK(cudaMemcpyAsync(h_b0, B.b0.p, nb * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      if (L.sym_rows > 0)
        CK(cudaMemcpyAsync(h_np, B.sym_np.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           c->stream));
    });
    CK(cudaEventRecord(ev2, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    check_onehot_status(c);
    if (L.sym_rows == 0 || *h_np <= B.sym_cap) break;
    B.sym_cap = *h_np + *h_np / 4;
    B.sym_pairs.ensure(B.sym_cap * sizeof(uint4));
    B.sym_keys.ensure(2 * B.sym_cap * sizeof(uint64_t));
  }
  // a resident rerun cleared every row's maxima: the dense assemblies run
  // their GEMMs again, then the maxima are read again
  if (reran) {
    bool any = false;
    for (int b = 0; b < nb; ++b)
      if (L.at(b).gemm && L.at(b).n > 0) {
        dense_allpairs_onehot(c, D[b].g);
        launches += 6;
        any = true;
      }
    if (any && rows) {
      CK(cudaMemcpyAsync(h_maxc, B.maxc_cand.p, rows * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaMemcpyAsync(h_maxc + rows1, B.maxc_all.p, rows * sizeof(uint32_t),
                         cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      check_onehot_status(c);
    }
  }
  if (autotune) {
    stats.tuned_keys = autotune_batch(c, B, defaults, asms, nb, L);
    // the later segments read this call's descriptors again
    CK(cudaMemcpyAsync(B.desc.p, h_desc, desc_bytes, cudaMemcpyHostToDevice, c->stream));
  }

  // ── host calibration of every assembly ─────────────────────────────────
  const auto t_cal = std::chrono::steady_clock::now();
  std::vector<double> cut(nb, 0.0);
  std::vector<float> b0f(h_b0, h_b0 + nb);
  auto calibrate = [&](int b) {
    const AsmPlan &a = L.at(b);
    std::vector<double> sv_d;
    std::vector<float> sv_f;
    sv_table(a.m, a.p->base_on != 0, a.p->base_on ? (double)b0f[b] : 0.0, sv_d, sv_f);
    const uint32_t *mc = (a.fused ? h_maxc : h_maxc + rows1) + a.row0;
    cut[b] = calibrate_cutoff(mc, a.n, a.fused ? CalibMode::fused : CalibMode::all, a.m, sv_d,
                              sv_f, a.p->coverage, a.p->seed);
  };
  {
    const int nt = std::max(1, std::min<int>(nb, (int)std::thread::hardware_concurrency()));
    if (nt <= 1 || nb < 4) {
      for (int b = 0; b < nb; ++b) calibrate(b);
    } else {
      std::vector<std::thread> th;
      std::atomic<int> next{0};
      for (int t = 0; t < nt; ++t)
        th.emplace_back([&] {
          for (int b; (b = next.fetch_add(1)) < nb;) calibrate(b);
        });
      for (auto &t : th) t.join();
    }
  }
  stats.calib_ms = (float)ms_since(t_cal);
  for (int b = 0; b < nb; ++b) h_desc[b].e.cutoff = cut[b] / 1000.;

  // ── segment 2: neighbour lists, edge counts, batch-wide scan ───────────
  const BatchAsm *dD = B.desc.as<BatchAsm>();
  captured(c, 1, use_graph, stats.graph_launches, [&] {
    CK(cudaMemcpyAsync(B.desc.p, h_desc, desc_bytes, cudaMemcpyHostToDevice, c->stream));
    launch_emit_batch(dD, B.row0s.as<int64_t>(), nb, rows, L.max_k, B.row_edges.as<int32_t>(),
                      B.edge0s.as<int64_t>(), c->stream);
    launches += (rows ? 2 : 0) + 2;
    CK(cudaMemcpyAsync(h_edge0s, B.edge0s.p, (nb + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                       c->stream));
  });
  CK(cudaEventRecord(ev3, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<int64_t> edge0v(h_edge0s, h_edge0s + nb + 1);
  const int64_t E = edge0v[nb];
  stats.edges = E;

  // ── segment 3: edges and weights, then the copies back ─────────────────
  const size_t E1 = (size_t)std::max<int64_t>(E, 1);
  B.e_from.ensure(E1 * 4); B.e_to.ensure(E1 * 4); B.e_scomp.ensure(E1 * 4); B.e_score.ensure(E1 * 4);
  for (int b = 0; b < nb; ++b) {
    EmitArgs &e = h_desc[b].e;
    e.from = B.e_from.as<uint32_t>(); e.to = B.e_to.as<uint32_t>(); e.scomp = B.e_scomp.as<float>();
    WeightArgs &w = h_desc[b].w;
    w.from = e.from; w.to = e.to; w.scomp = e.scomp; w.score = B.e_score.as<float>();
    w.n_edges = edge0v[b + 1] - edge0v[b];
  }
  // the edge arrays land in one pinned block that the graphs share (no host
  // copy per graph); the staging buffer and copies are the fallback
  const size_t eb = up256(E1 * 4);
  char *shared = (char *)pinned_take(4 * eb);
  struct Back {                         // an error before the graphs own it: back to the pool
    void *p;
    ~Back() { if (p) pinned_share(p, {}); }
  } back{shared};
  if (!shared) B.hedge.ensure(4 * eb);
  char *hb = shared ? shared : B.hedge.as<char>();
  uint32_t *h_from = (uint32_t *)hb;
  uint32_t *h_to = (uint32_t *)(hb + eb);
  float *h_scomp = (float *)(hb + 2 * eb);
  float *h_score = (float *)(hb + 3 * eb);
  captured(c, 2, use_graph, stats.graph_launches, [&] {
    CK(cudaMemcpyAsync(B.desc.p, h_desc, desc_bytes, cudaMemcpyHostToDevice, c->stream));
    launch_write_edges_batch(dD, B.row0s.as<int64_t>(), nb, rows, c->stream);
    launch_edge_weights_batch(dD, B.edge0s.as<int64_t>(), nb, E, c->stream);
    launches += (rows ? 1 : 0) + (E ? 1 : 0);
    if (E) {
      CK(cudaMemcpyAsync(h_from, B.e_from.p, E * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(h_to, B.e_to.p, E * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(h_scomp, B.e_scomp.p, E * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(h_score, B.e_score.p, E * 4, cudaMemcpyDeviceToHost, c->stream));
    }
  });
  CK(cudaEventRecord(ev4, c->stream));
  CK(cudaStreamSynchronize(c->stream));

  // ── results in the caller's order ──────────────────────────────────────
  std::vector<void *> firsts;
  bool nomem = false;
  for (int b = 0; b < nb; ++b) {
    const AsmPlan &a = L.at(b);
    rbg_graph &g = out[a.orig];
    const int64_t e0 = edge0v[b], ne = edge0v[b + 1] - e0;
    g.n_edges = ne;
    g.b0 = a.p->base_on ? (double)b0f[b] : 0.0;
    g.sim_cutoff = cut[b];
    g.path = a.fused ? 2 : 1;
    if (shared && ne > 0) {
      g.from = h_from + e0;
      g.to = h_to + e0;
      g.scomp = h_scomp + e0;
      g.score = h_score + e0;
      firsts.push_back(g.from);
      continue;
    }
    const size_t bytes = (size_t)std::max<int64_t>(ne, 1) * 4;
    g.from = (uint32_t *)malloc(bytes);
    g.to = (uint32_t *)malloc(bytes);
    g.scomp = (float *)malloc(bytes);
    g.score = (float *)malloc(bytes);
    if (!g.from || !g.to || !g.scomp || !g.score) {
      nomem = true;
      break;
    }
    if (ne) {
      std::memcpy(g.from, h_from + e0, ne * 4);
      std::memcpy(g.to, h_to + e0, ne * 4);
      std::memcpy(g.scomp, h_scomp + e0, ne * 4);
      std::memcpy(g.score, h_score + e0, ne * 4);
    }
  }
  back.p = nullptr;
  if (shared) pinned_share(shared, firsts);
  if (nomem) {
    for (int q = 0; q < nb; ++q) rbg_free_graph(&out[q]);
    throw Error(RBG_ERR_NOMEM, "host allocation of the edge arrays failed");
  }
  float t01 = 0, t12 = 0, t34 = 0;
  cudaEventElapsedTime(&t01, ev0, ev1);
  cudaEventElapsedTime(&t12, ev1, ev2);
  cudaEventElapsedTime(&t34, ev3, ev4);
  stats.stage_ms = t01;
  stats.graph_ms = t12;
  stats.emit_ms = t34;
  stats.kernel_launches = launches;
  stats.total_ms = (float)ms_since(t_start);
  if (st) *st = stats;
}

}  // namespace rbg

extern "C" int rbg_bin_batch(rbg_ctx *c, const rbg_params *defaults, const rbg_assembly *asms,
                             int32_t n_asm, rbg_graph *out, rbg_batch_stats *stats) {
  return rbg::guarded(c, [&] {
    if (n_asm > 0 && (!asms || !out || !defaults)) throw rbg::Error(RBG_ERR_ARG, "null argument");
    // Assemblies on the one-permutation metric or the inverted-index graph
    // have no batch kernels: they run one after the other through the
    // single-assembly path on this context, after the batch of the others.
    std::vector<int> one, many;
    for (int i = 0; i < n_asm; ++i) {
      const rbg_params *p = asms[i].params ? asms[i].params : defaults;
      (p->oph_k > 0 || p->graph_index ? one : many).push_back(i);
    }
    if (one.empty()) {
      rbg::run_batch(c, defaults, asms, n_asm, out, stats);
      return;
    }
    std::vector<rbg_assembly> sub;
    for (int i : many) sub.push_back(asms[i]);
    std::vector<rbg_graph> got(sub.size());
    if (!sub.empty()) rbg::run_batch(c, defaults, sub.data(), (int)sub.size(), got.data(), stats);
    else if (stats) std::memset(stats, 0, sizeof(*stats));
    for (size_t k = 0; k < many.size(); ++k) out[many[k]] = got[k];
    for (int i : one) {
      const rbg_params *p = asms[i].params ? asms[i].params : defaults;
      try {
        rbg::validate_assembly(asms[i], p, "assembly " + std::to_string(i) + ": ");
        rbg::bin_graph_one(c, p, asms[i], &out[i]);
      } catch (...) {
        for (int j : many) rbg_free_graph(&out[j]);
        throw;
      }
    }
  });
}
