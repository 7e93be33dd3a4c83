// Host engine: device buffers, the orchestration of the hot path, the host
// steps that stay sequential by definition (b0 sampling with mt19937_64, the
// rand()-driven cutoff calibration), and the C ABI of include/rabbitbin_b200.h.
#include <algorithm>
#include <deque>
#include <limits>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <map>
#include <mutex>
#include <numeric>
#include <random>
#include <stdexcept>
#include <unordered_map>
#include <string>
#include <vector>


#include "engine_internal.h"

namespace rbg {
void launch_fold16(const uint32_t *in, int64_t n, uint16_t *out, cudaStream_t s);
void launch_raw_pair_counts(const void *win, int bits, int m, const int64_t *pairs, int np,
                            uint32_t *out, cudaStream_t s);
void launch_codes_from_winners(const uint32_t *w32, int64_t n, int m, int mpad, int use16,
                               const uint32_t *vals, const uint8_t *codes, const int32_t *nvals,
                               uint8_t *A, uint8_t *B, int *bad, cudaStream_t s);
}  // namespace rbg

namespace {

using namespace rbg;

void validate(const rbg_params *p) { validate_params(p); }

// The device tables of the last few (k, m, seed, contract, win_bits)
// configurations stay resident (about 10 MB each at m = 1000): a stream of
// assemblies with different sketch sizes reuses them instead of freeing and
// re-uploading a set per call (cudaFree waits for the device).
Tables &tables_for(rbg_ctx *c, const rbg_params *p) {
  const auto key = std::make_tuple(p->k, p->m, p->pmh_seed, p->fp_contract != 0 ? 1 : 0,
                                   p->win_bits);
  for (auto it = c->tab_cache.begin(); it != c->tab_cache.end(); ++it)
    if (it->first == key) {
      if (it != c->tab_cache.begin())            // most recently used first
        c->tab_cache.splice(c->tab_cache.begin(), c->tab_cache, it);
      return *c->tab_cache.front().second;
    }
  constexpr size_t kKeep = 6;
  if (c->tab_cache.size() >= kKeep) {
    c->tab_cache.back().second->release();
    c->tab_cache.pop_back();
  }
  c->tab_cache.emplace_front(key, make_tables(p, c->stream));
  return *c->tab_cache.front().second;
}

// Checks, sizes, offsets and coverage to the device; the ASCII bases are
// copied by the caller (whole, or in chunks behind the sketch).
void stage_meta(rbg_ctx *c, const char *seqcat, const int64_t *offsets, int64_t n,
                const float *depth, int S) {
  if (n < 0 || (n > 0 && (!offsets || !seqcat))) throw Error(RBG_ERR_ARG, "bad sequence arguments");
  if (S < 0 || S > kMaxS) throw Error(RBG_ERR_UNSUPPORTED, "S must be in 0..64");
  if (S > 0 && n > 0 && !depth) throw Error(RBG_ERR_ARG, "depth is null");
  if (n > 0 && offsets[0] != 0) throw Error(RBG_ERR_ARG, "offsets[0] must be 0");
  if (n >= (1 << 27)) throw Error(RBG_ERR_UNSUPPORTED, "at most 2^27 - 1 contigs per assembly");
  for (int64_t i = 0; i < n; ++i)
    if (offsets[i + 1] < offsets[i]) throw Error(RBG_ERR_ARG, "offsets must be non-decreasing");
  c->streamed = false;
  c->n = n;
  c->S = S;
  c->nbases = n > 0 ? offsets[n] : 0;
  c->h_offsets.assign(offsets, offsets + n + 1);
  c->graph_ready = false;
  const size_t abytes = (size_t)((c->nbases + 15) / 16) * 16 + 16;
  c->ascii.ensure(abytes);
  c->offsets.ensure((n + 1) * sizeof(int64_t));
  c->depth.ensure(std::max<size_t>(1, (size_t)n * S) * sizeof(float));
  (void)abytes;
  CK(cudaMemcpyAsync(c->offsets.p, offsets, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  if (S > 0 && n > 0)
    CK(cudaMemcpyAsync(c->depth.p, depth, (size_t)n * S * sizeof(float), cudaMemcpyHostToDevice, c->stream));
}

void stage(rbg_ctx *c, const char *seqcat, const int64_t *offsets, int64_t n,
           const float *depth, int S) {
  stage_meta(c, seqcat, offsets, n, depth, S);
  const size_t abytes = (size_t)((c->nbases + 15) / 16) * 16 + 16;
  CK(cudaMemsetAsync(c->ascii.p, 0, abytes, c->stream));
  if (c->nbases)
    CK(cudaMemcpyAsync(c->ascii.p, seqcat, (size_t)c->nbases, cudaMemcpyHostToDevice, c->stream));
}

// Inputs already on the device (the FASTA parser's output): sequences and
// offsets are copied device to device, the coverage table from the host.
void stage_device(rbg_ctx *c, const char *dseq, const int64_t *doffsets, int64_t n,
                  int64_t nbases, const float *depth, int S) {
  if (S < 0 || S > kMaxS) throw Error(RBG_ERR_UNSUPPORTED, "S must be in 0..64");
  if (S > 0 && n > 0 && !depth) throw Error(RBG_ERR_ARG, "depth is null");
  if (n >= (1 << 27)) throw Error(RBG_ERR_UNSUPPORTED, "at most 2^27 - 1 contigs per assembly");
  c->streamed = false;
  c->n = n;
  c->S = S;
  c->nbases = nbases;
  c->h_offsets.clear();
  c->graph_ready = false;
  const size_t abytes = (size_t)((nbases + 15) / 16) * 16 + 16;
  c->ascii.ensure(abytes);
  c->offsets.ensure((n + 1) * sizeof(int64_t));
  c->depth.ensure(std::max<size_t>(1, (size_t)n * S) * sizeof(float));
  CK(cudaMemsetAsync(c->ascii.p, 0, abytes, c->stream));
  if (nbases)
    CK(cudaMemcpyAsync(c->ascii.p, dseq, (size_t)nbases, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->offsets.p, doffsets, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                     c->stream));
  if (S > 0 && n > 0)
    CK(cudaMemcpyAsync(c->depth.p, depth, (size_t)n * S * sizeof(float), cudaMemcpyHostToDevice,
                       c->stream));
}

// Unit rank rows, anynz and column norms on the auxiliary stream: they depend
// only on the coverage table, so they overlap the sketch kernels.
void prep_depth(rbg_ctx *c, const rbg_params *p) {
  const int64_t n = c->n, n1 = std::max<int64_t>(n, 1);
  const int S = c->S;
  const int Su = (std::max(S, 1) + 3) & ~3;
  const int Kp = unit16_stride(S);
  c->unit.ensure(n1 * Su * sizeof(float));
  c->unit16.ensure(n1 * Kp * sizeof(uint16_t));
  c->anynz.ensure(n1);
  c->colnorm.ensure(std::max(S, 1) * sizeof(double));
  GraphArgs g;
  g.n = n; g.S = S; g.Su = Su; g.Kp = Kp;
  g.unit16 = c->unit16.as<uint16_t>();
  g.depth_raw = c->depth.as<float>();
  g.unit = c->unit.as<float>();
  g.anynz = c->anynz.as<uint8_t>();
  g.colnorm = c->colnorm.as<double>();
  g.min_cv = (float)p->min_cv;
  g.min_cv_d = p->min_cv;
  g.has_depth = S > 0;
  g.wjac_norm = p->wjac_norm;
  CK(cudaEventRecord(c->ev_in, c->stream));
  CK(cudaStreamWaitEvent(c->aux, c->ev_in, 0));
  CK(cudaEventRecord(c->ev_a0, c->aux));
  launch_unit_rows(g, c->aux);
  c->launches += n ? 1 : 0;
  if (need_colnorm(p, S)) {
    c->colacc.ensure(3 * sizeof(double) * std::max(S, 1));
    launch_colnorm(g, c->colacc.as<double>(), c->aux);
    c->launches += 2;
  }
  CK(cudaEventRecord(c->ev_a1, c->aux));
  CK(cudaEventRecord(c->ev_aux, c->aux));
  c->prep_done = true;
}

// Sketch stage: pack, count + weights, register minimum.
// Sketch buffers and the kernel arguments over all contigs.
SketchArgs sketch_setup(rbg_ctx *c, const rbg_params *p, bool want_winners) {
  const bool oph = p->oph_k > 0;          // one-permutation MinHash: no PMH tables
  if (want_winners && oph)
    throw Error(RBG_ERR_ARG, "winner rows exist only for the ProbMinHash metric (oph_k = 0)");
  Tables *T = oph ? nullptr : &tables_for(c, p);
  const int64_t n = c->n;
  const int m = p->m, mpad = mpad_of(p->m);
  const int64_t nwords = (c->nbases + 15) / 16 + 1;
  c->packed.ensure(nwords * 4);
  c->nmask.ensure((nwords / 2 + 2) * 4);
  c->codesA.ensure(std::max<int64_t>(n, 1) * mpad);
  c->codesB.ensure(std::max<int64_t>(n, 1) * mpad);
  SketchArgs a;
  a.packed = c->packed.as<uint32_t>();
  a.nmask = c->nmask.as<uint32_t>();
  a.offsets = c->offsets.as<int64_t>();
  a.n = n;
  a.k = p->k;
  a.m = m;
  a.mpad = mpad;
  a.gc_norm = p->gc_norm;
  a.gc_cap = p->gc_norm_cap;
  a.codesA = c->codesA.as<uint8_t>();
  a.codesB = c->codesB.as<uint8_t>();
  if (!oph) {
    c->elem_winv.ensure(std::max<int64_t>(n, 1) * T->t->n_elems * sizeof(double));
    c->elem_cnt.ensure(std::max<int64_t>(n, 1) * sizeof(int32_t));
    if (want_winners) c->winners32.ensure(std::max<int64_t>(n, 1) * m * sizeof(uint32_t));
    a.n_elems = T->t->n_elems;
    a.rank_of_code = T->rank.as<int16_t>();
    a.elem_winv = c->elem_winv.as<double>();
    a.elem_cnt = c->elem_cnt.as<int32_t>();
    a.order = T->order.as<RegOrder>();
    a.UT = T->UT.as<double>();
    a.codeA = T->codeA.as<uint8_t>();
    a.W32 = T->W32.as<uint32_t>();
    a.winners32 = want_winners ? c->winners32.as<uint32_t>() : nullptr;
  }
  return a;
}

// Sketch of contigs [a.offsets - first, + a.n): k-mer counts and the register
// minimum (ProbMinHash), or the one-permutation MinHash buckets; `mid` is
// recorded between the two ProbMinHash kernels (null: none).
void sketch_contigs(rbg_ctx *c, const rbg_params *p, const SketchArgs &a, cudaEvent_t mid) {
  if (p->oph_k > 0) {
    if (mid) CK(cudaEventRecord(mid, c->stream));
    launch_oph(a, p->oph_k, p->oph_bits, kOphSeed, c->stream);
    c->launches += a.n ? 1 : 0;
    return;
  }
  c->count_work.ensure(sizeof(unsigned));
  CK(cudaMemsetAsync(c->count_work.p, 0, sizeof(unsigned), c->stream));
  SketchArgs ac = a;
  ac.work = c->count_work.as<unsigned>();
  launch_count(ac, c->stream);
  if (mid) CK(cudaEventRecord(mid, c->stream));
  launch_minreduce(a, c->stream);
  c->launches += a.n ? 2 : 0;
}

// The host-input path of rbg_bin_graph: the ASCII copy runs in chunks on the
// copy stream; each chunk's words are packed as it lands, and the contigs
// whose words are all packed (e <= 16 * packed words) are counted and reduced
// while the next chunks copy.
bool sym_regime(const rbg_params *p, int64_t n, int S);
GraphArgs graph_args(rbg_ctx *c, const rbg_params *p);
SymOut sym_buffers(rbg_ctx *c, int64_t n1);
void sym_clear(rbg_ctx *c, int64_t n1);

// In the tensor-core regime the all-pairs pass runs behind the copy too: once
// chunk g's contigs [c0, c1) are sketched, the pairs whose later member lies
// in [c0, c1) are scored (rows [0, c1)), with admission deferred until b0 is
// known (run_graph finishes the selection).
void stage_sketch_chunked(rbg_ctx *c, const rbg_params *p, const char *seqcat,
                          const int64_t *offsets, int64_t n, const float *depth, int S) {
  stage_meta(c, seqcat, offsets, n, depth, S);
  const SketchArgs all = sketch_setup(c, p, false);
  const int64_t nb = c->nbases, nwords = (nb + 15) / 16;
  const int E = all.n_elems, mpad = all.mpad;
  CK(cudaEventRecord(c->ev[0], c->stream));
  prep_depth(c, p);
  CK(cudaEventRecord(c->ev_cin, c->stream));             // the buffers are free to overwrite
  CK(cudaStreamWaitEvent(c->copy, c->ev_cin, 0));
  const int G = nwords >= ((int64_t)kChunks << 16) ? kChunks : 1;
  // Streaming keeps every survivor of the prune until b0 is known; with few
  // samples the prune passes a large share of the pairs, so it streams from
  // S >= 10, and never again at an S whose survivors outgrew the list.
  const bool stream_pairs = G > 1 && S >= 10 && sym_regime(p, n, S) &&
                            !((c->no_stream_S >> (S & 63)) & 1u);
  GraphArgs ga;
  SymOut o;
  bool tc5 = false;
  if (stream_pairs) {
    ga = graph_args(c, p);
    o = sym_buffers(c, std::max<int64_t>(n, 1));
    o.defer = 1;
    sym_clear(c, std::max<int64_t>(n, 1));
    CK(cudaStreamWaitEvent(c->stream, c->ev_aux, 0));   // unit rows, anynz
    tc5 = sym_tc5_fits(ga);
    if (tc5) sym_tc5_setup(c, ga, G);
  }
  // Packing on the host sends 3/8 of a byte per base instead of the ASCII
  // byte: while chunk g's words copy, the host packs chunk g + 1 into the
  // other pinned slot.
  const bool hpack = pack_on_host();
  int64_t c0 = 0;
  for (int g = 0; g < G; ++g) {
    const int64_t w0 = (int64_t)g * nwords / G & ~(int64_t)1;
    const int64_t w1 = g + 1 == G ? nwords : ((int64_t)(g + 1) * nwords / G & ~(int64_t)1);
    const int64_t b0 = 16 * w0, b1 = std::min<int64_t>(16 * w1, nb);
    if (hpack) {
      const int sl = g & 1;
      const int64_t pairs = (w1 - w0 + 1) / 2;
      if (pairs > 0) {
        if (g >= 2) CK(cudaEventSynchronize(c->ev_slot[sl]));   // its previous copy is done
        const size_t wbytes = (size_t)pairs * 8, mbytes = (size_t)pairs * 4;
        c->pack_pin[sl].ensure(wbytes + mbytes);
        uint32_t *hw = c->pack_pin[sl].as<uint32_t>(), *hm = hw + 2 * pairs;
        host_pack_words(seqcat, nb, w0, w1, hw, hm);
        CK(cudaMemcpyAsync(c->packed.as<uint32_t>() + w0, hw, wbytes, cudaMemcpyHostToDevice,
                           c->copy));
        CK(cudaMemcpyAsync(c->nmask.as<uint32_t>() + w0 / 2, hm, mbytes, cudaMemcpyHostToDevice,
                           c->copy));
        CK(cudaEventRecord(c->ev_slot[sl], c->copy));
      }
      CK(cudaEventRecord(c->ev_chunk[g], c->copy));
      CK(cudaStreamWaitEvent(c->stream, c->ev_chunk[g], 0));
    } else {
      if (b1 > b0)
        CK(cudaMemcpyAsync(c->ascii.as<char>() + b0, seqcat + b0, (size_t)(b1 - b0),
                           cudaMemcpyHostToDevice, c->copy));
      CK(cudaEventRecord(c->ev_chunk[g], c->copy));
      CK(cudaStreamWaitEvent(c->stream, c->ev_chunk[g], 0));
      launch_pack_range(c->ascii.as<char>(), nb, w0, w1, c->packed.as<uint32_t>(),
                        c->nmask.as<uint32_t>(), c->stream);
    }
    const int64_t c1 = g + 1 == G ? n
                     : (int64_t)(std::upper_bound(offsets + 1, offsets + n + 1, 16 * w1) -
                                 (offsets + 1));
    if (c1 > c0) {
      SketchArgs a = all;
      a.offsets += c0;
      a.n = c1 - c0;
      if (a.elem_winv) a.elem_winv += c0 * E;
      if (a.elem_cnt) a.elem_cnt += c0;
      a.codesA += c0 * mpad;
      a.codesB += c0 * mpad;
      sketch_contigs(c, p, a, nullptr);
      if (stream_pairs) {
        if (tc5) {
          sym_tc5_pass(c, ga, o, c0, c1, g);
        } else {
          launch_allpairs_sym_window(ga, o, c0, c1, c->stream);
          c->launches += 1;
        }
      }
    }
    c0 = c1;
  }
  c->streamed = stream_pairs;
  c->streamed_tc5 = stream_pairs && tc5;
  c->launches += hpack ? 0 : G;
  CK(cudaEventRecord(c->ev[1], c->stream));
  CK(cudaEventRecord(c->ev[2], c->stream));
  CK(cudaEventRecord(c->ev[3], c->stream));
  CK(cudaGetLastError());
}

void run_sketch(rbg_ctx *c, const rbg_params *p, bool want_winners, uint8_t *win_elem = nullptr) {
  SketchArgs a = sketch_setup(c, p, want_winners);
  a.win_elem = win_elem;
  CK(cudaEventRecord(c->ev[0], c->stream));
  prep_depth(c, p);
  launch_pack(c->ascii.as<char>(), c->nbases, c->packed.as<uint32_t>(), c->nmask.as<uint32_t>(),
              c->stream);
  c->launches += c->nbases ? 1 : 0;
  CK(cudaEventRecord(c->ev[1], c->stream));
  sketch_contigs(c, p, a, c->ev[2]);
  CK(cudaEventRecord(c->ev[3], c->stream));
  CK(cudaGetLastError());
}

// b0: median raw match fraction over 30000 mt19937_64 draws
// (estimate_pmh_baseline, src/rabbitbin.cpp:1340-1369).
double estimate_b0(rbg_ctx *c, int64_t n, int m, const std::function<void(const int64_t *, int, uint32_t *)> &count) {
  (void)c;
  const auto prs = b0_pairs(n);
  const int np = (int)(prs->size() / 2);
  if (np == 0) return 0.0;
  std::vector<int64_t> pr(prs->begin(), prs->end());
  std::vector<uint32_t> cnt(np);
  count(pr.data(), np, cnt.data());
  const double inv_m = 1.0 / (double)m;
  std::vector<float> vals(np);
  for (int q = 0; q < np; ++q) vals[q] = (float)((double)cnt[q] * inv_m);
  std::nth_element(vals.begin(), vals.begin() + vals.size() / 2, vals.end());
  return (double)vals[vals.size() / 2];
}

void count_pairs_codes(rbg_ctx *c, int mpad, int m, const int64_t *pr, int np, uint32_t *out) {
  c->pairs.ensure((size_t)np * 2 * sizeof(int64_t));
  c->pair_out.ensure((size_t)np * sizeof(uint32_t));
  c->pairs_n = -1;                       // no longer the run_graph sample
  CK(cudaMemcpyAsync(c->pairs.p, pr, (size_t)np * 2 * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  launch_pair_counts(c->codesA.as<uint8_t>(), c->codesB.as<uint8_t>(), mpad, m,
                     c->pairs.as<int64_t>(), np, c->pair_out.as<uint32_t>(), c->stream);
  c->launches++;
  CK(cudaMemcpyAsync(out, c->pair_out.p, (size_t)np * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

// The abundance-pruned regime of the fused path, whose all-pairs pass is the
// symmetric tensor-core pass (src/rabbitbin.cpp:5035-5054 picks the fused
// path; the prune applies when S > 1 and the depth term can decide an edge).
bool sym_regime(const rbg_params *p, int64_t n, int S) {
  const double w_comp = (p->w_comp < 0.0) ? (S <= 2 ? 1.0 : 0.0) : p->w_comp;
  const bool fused = (p->force_path == 2) || (p->force_path == 0 && n > 25000);
  return n > 0 && fused && p->oph_k == 0 && p->abdfirst && S > 1 && w_comp < 1.0 &&
         w_comp < p->min_edge;
}

// Graph-stage buffers and kernel arguments of the staged assembly (the
// similarity table's contents come once b0 is known).
GraphArgs graph_args(rbg_ctx *c, const rbg_params *p) {
  const int64_t n = c->n;
  const int m = p->m, mpad = mpad_of(m), S = c->S, K = p->max_edges;
  const int64_t n1 = std::max<int64_t>(n, 1);
  const int Su = (std::max(S, 1) + 3) & ~3;
  c->svbits.ensure((m + 1) * sizeof(uint32_t));
  c->topk.ensure(n1 * K * sizeof(uint64_t));
  c->topk_cnt.ensure(n1 * sizeof(int32_t));
  c->maxc_cand.ensure(n1 * sizeof(uint32_t));
  c->maxc_all.ensure(n1 * sizeof(uint32_t));
  c->stats.ensure(2 * sizeof(unsigned long long));
  const double w_comp = (p->w_comp < 0.0) ? (S <= 2 ? 1.0 : 0.0) : p->w_comp;
  // the one-permutation metric has no fused path: its large-N route builds the
  // small path's graph (only its calibration differs)
  const bool fused = p->oph_k == 0 && ((p->force_path == 2) || (p->force_path == 0 && n > 25000));
  GraphArgs g;
  g.n = n; g.m = m; g.mpad = mpad; g.S = S; g.K = K; g.Su = Su;
  g.codesA = c->codesA.as<uint8_t>();
  g.codesB = c->codesB.as<uint8_t>();
  g.depth_raw = c->depth.as<float>();
  g.unit = c->unit.as<float>();
  g.unit16 = c->unit16.as<uint16_t>();
  g.Kp = unit16_stride(S);
  g.anynz = c->anynz.as<uint8_t>();
  g.colnorm = c->colnorm.as<double>();
  g.has_depth = S > 0;
  g.wjac_norm = p->wjac_norm;
  g.small_path = fused ? 0 : 1;
  const bool abdfirst = sym_regime(p, n, S);
  const double abd_corr_min = abdfirst ? (p->min_edge - w_comp) / (1.0 - w_comp) : -2.0;
  g.prefilter = abdfirst ? 1 : 0;
  g.prefilter_eps = (float)(abd_corr_min - 1e-4);
  g.sv_bits = c->svbits.as<uint32_t>();
  g.topk = c->topk.as<uint64_t>();
  g.topk_cnt = c->topk_cnt.as<int32_t>();
  g.maxcnt_cand = c->maxc_cand.as<uint32_t>();
  g.maxcnt_all = c->maxc_all.as<uint32_t>();
  g.stats = c->stats.as<unsigned long long>();
  g.key_floor = admission_floor();
  return g;
}

// Pair-list buffers of the symmetric pass (capacity c->sym_cap pairs).
SymOut sym_buffers(rbg_ctx *c, int64_t n1) {
  if (c->sym_cap == 0) {
    // RBG_PAIR_CAP: a smaller first list, to exercise the overflow path
    const char *e = getenv("RBG_PAIR_CAP");
    c->sym_cap = e ? std::max<uint64_t>(1024, strtoull(e, nullptr, 10))
                   : std::max<uint64_t>(1u << 20, (uint64_t)n1 * 256);
  }
  c->sym_pairs.ensure(c->sym_cap * sizeof(uint4));
  c->sym_keys.ensure(2 * c->sym_cap * sizeof(uint64_t));
  c->sym_rowcnt.ensure(n1 * sizeof(int32_t));
  c->sym_rowoff.ensure((n1 + 1) * sizeof(int64_t));
  c->sym_np.ensure(sizeof(unsigned long long));
  SymOut o;
  o.pairs = c->sym_pairs.as<uint4>();
  o.npairs = c->sym_np.as<unsigned long long>();
  o.cap = c->sym_cap;
  o.rowcnt = c->sym_rowcnt.as<int32_t>();
  return o;
}

// Zeroes what a symmetric pass accumulates into.
void sym_clear(rbg_ctx *c, int64_t n1) {
  CK(cudaMemsetAsync(c->stats.p, 0, 2 * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(c->maxc_cand.p, 0, n1 * sizeof(uint32_t), c->stream));
  CK(cudaMemsetAsync(c->sym_rowcnt.p, 0, n1 * sizeof(int32_t), c->stream));
  CK(cudaMemsetAsync(c->sym_np.p, 0, sizeof(unsigned long long), c->stream));
}

// One assembly over several ranks (rbg_bin_graph_sharded): this rank scores
// rows [row_lo, row_hi); row0[r] is rank r's first row (row0[world] = n) and
// nmax the most rows a rank holds.  gather(dsend, drecv, bytes) exchanges
// equal-size device blocks, rank r's block at drecv + r * bytes.
struct ShardCtx {
  int rank = 0, world = 1;
  int64_t row_lo = 0, row_hi = 0, nmax = 0;
  std::vector<int64_t> row0;
  std::function<void(const void *, void *, size_t)> gather;
};

// Every rank's rows [row0[r], row0[r+1]) of `elem`-byte items: rank r's items
// from the block exchange (blocks of nmax * elem bytes) into dst.
void scatter_blocks(rbg_ctx *c, const ShardCtx &sc, const void *recv, void *dst, size_t elem) {
  const size_t blk = (size_t)sc.nmax * elem;
  for (int r = 0; r < sc.world; ++r) {
    const size_t bytes = (size_t)(sc.row0[r + 1] - sc.row0[r]) * elem;
    if (bytes)
      CK(cudaMemcpyAsync((char *)dst + (size_t)sc.row0[r] * elem, (const char *)recv + r * blk,
                         bytes, cudaMemcpyDeviceToDevice, c->stream));
  }
}

// This rank's rows [row_lo, row_hi) of `elem`-byte items from src, gathered
// from every rank into dst (the whole row range).
void share_rows(rbg_ctx *c, const ShardCtx &sc, const void *src, void *dst, size_t elem) {
  const size_t blk = (size_t)sc.nmax * elem, mine = (size_t)(sc.row_hi - sc.row_lo) * elem;
  c->shard_send.ensure(std::max<size_t>(blk, 16));
  c->shard_recv.ensure(std::max<size_t>(blk * sc.world, 16));
  CK(cudaMemsetAsync(c->shard_send.p, 0, blk, c->stream));
  if (mine)
    CK(cudaMemcpyAsync(c->shard_send.p, (const char *)src + (size_t)sc.row_lo * elem, mine,
                       cudaMemcpyDeviceToDevice, c->stream));
  sc.gather(c->shard_send.p, c->shard_recv.p, blk);
  scatter_blocks(c, sc, c->shard_recv.p, dst, elem);
}

// The inverted-index candidate graph of the small path: one-permutation
// sketch keys of every contig (KmerSketch(m, index_k, bits), getKeys), the
// index of those keys, and each row's neighbours from its candidates, written
// over the row's top-K keys.  minCommon and the posting-list cap as
// build_similarity_graph computes them (src/impl/rb_graph.cpp:228-246, :287).
void index_graph(rbg_ctx *c, const rbg_params *p, const GraphArgs &g, double cutoff) {
  const int64_t n = c->n;
  if (n == 0) return;
  const int m = p->m, K = p->max_edges;
  if (index_rows_smem(n, K) > (size_t)227 * 1024)
    throw Error(RBG_ERR_UNSUPPORTED, "graph_index: at most about 37,000 contigs");
  const double Md = (double)m;
  size_t min_common = (size_t)std::floor(cutoff * Md * 0.7);
  if (min_common < 1) min_common = 1;
  if (p->min_common >= 1) min_common = (size_t)p->min_common;
  const int64_t pl_cap = (int64_t)(uint32_t)std::max((size_t)256, (size_t)n / 8);
  const int64_t total = n * (int64_t)m;
  c->ix_keys.ensure((size_t)total * 8);
  c->ix_sorted.ensure((size_t)total * 8);
  c->ix_contig.ensure((size_t)total * 4);
  c->ix_post.ensure((size_t)total * 4);
  c->ix_ukeys.ensure((size_t)total * 8);
  c->ix_count.ensure((size_t)total * 4);
  c->ix_off.ensure((size_t)total * 8);
  c->ix_nk.ensure(16);
  const size_t sb = index_build_bytes(total);
  c->ix_scratch.ensure(sb);
  // keys of the one-permutation sketches (the packed bases are still staged)
  SketchArgs a;
  a.packed = c->packed.as<uint32_t>();
  a.nmask = c->nmask.as<uint32_t>();
  a.offsets = c->offsets.as<int64_t>();
  a.n = n;
  a.m = m;
  a.mpad = mpad_of(m);
  a.oph_keys = c->ix_keys.as<uint64_t>();
  launch_oph(a, p->oph_k > 0 ? p->oph_k : p->index_k, 1, kOphSeed, c->stream);
  if (launch_index_build(c->ix_keys.as<uint64_t>(), n, m, c->ix_sorted.as<uint64_t>(),
                         c->ix_contig.as<uint32_t>(), c->ix_post.as<uint32_t>(),
                         c->ix_ukeys.as<uint64_t>(), c->ix_count.as<int32_t>(),
                         c->ix_off.as<int64_t>(), c->ix_nk.as<int32_t>(), c->ix_scratch.p, sb,
                         c->stream) != 0)
    throw Error(RBG_ERR_CUDA, "graph_index: index build failed");
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  launch_index_rows(g, c->ix_keys.as<uint64_t>(), c->ix_ukeys.as<uint64_t>(),
                    c->ix_count.as<int32_t>(), c->ix_off.as<int64_t>(), c->ix_post.as<uint32_t>(),
                    c->ix_nk.as<int32_t>(), pl_cap, (int)min_common, cutoff, sms, c->stream);
  CK(cudaGetLastError());
  c->launches += 6;
}

// Dense regime (no abundance prune): the counts of rows [g.row_lo, row_hi)
// against every contig as the product of one-hot int8 rows on the tensor
// cores (k_onehot_mma, int32 accumulation in TMEM: exact), consumed in the
// kernel into per-(row, column group) candidate lists, the row maxima and the
// compared-pair count; k_merge_topk then gives each row its top-K keys.
}  // namespace

namespace rbg {

void dense_allpairs_onehot(rbg_ctx *c, const GraphArgs &g) {
  const int64_t n = g.n, lo = g.row_lo, hi = g.row_hi < 0 ? n : g.row_hi, rows = hi - lo;
  if (n == 0 || rows <= 0) return;
  const int m = g.m, mpad = g.mpad;
  cudaStream_t s = c->stream;
  c->oh_pres.ensure((size_t)m * 8 * sizeof(uint32_t));
  c->oh_map.ensure((size_t)m * 256 * sizeof(int32_t));
  c->oh_koff.ensure((size_t)(m + 1) * sizeof(int32_t));
  launch_code_presence(g.codesA, n, m, mpad, c->oh_pres.as<uint32_t>(), s);
  launch_onehot_map(c->oh_pres.as<uint32_t>(), m, c->oh_map.as<int32_t>(), c->oh_koff.as<int32_t>(),
                    s);
  int32_t K1 = 0;
  CK(cudaMemcpyAsync(&K1, c->oh_koff.as<int32_t>() + m, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  // one-hot rows zero-padded to whole 128-byte chunks of the contraction
  const int64_t ldx = std::max<int64_t>(128, ((int64_t)K1 + 127) / 128 * 128);
  c->oh_X.ensure((size_t)n * ldx);
  launch_onehot_fill(g.codesA, n, m, mpad, c->oh_map.as<int32_t>(), c->oh_X.as<int8_t>(), ldx, s);
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int GR = 1, GC = 1;
  onehot_mma_grid((int)((rows + 255) / 256), (int)((n + 255) / 256), sms, &GR, &GC);
  // RBG_ONEHOT_CAP: shorter lists, to exercise the cut inside the kernel
  const char *cap_env = getenv("RBG_ONEHOT_CAP");
  const int cap = onehot_mma_cap(n, GC, g.K, cap_env ? atoi(cap_env) : 0);
  const size_t lists = (size_t)((rows + 31) / 32) * 32 * 2 * GC;
  c->oh_cand.ensure(lists * cap * sizeof(uint32_t));
  c->oh_cnt.ensure(lists * sizeof(int32_t));
  c->oh_tab.ensure((size_t)(2 * m + 4) * sizeof(uint32_t));
  c->oh_err.ensure(sizeof(int));
  c->oh_errpin.ensure(sizeof(int));
  // the status accumulates over the calls before the caller's next check
  if (!c->oh_pending) CK(cudaMemsetAsync(c->oh_err.p, 0, sizeof(int), s));
  const char *why = "";
  const int rc = launch_onehot_mma(g, c->oh_X.as<int8_t>(), ldx, rows, c->oh_cand.as<uint32_t>(),
                                   cap, c->oh_cnt.as<int32_t>(), c->oh_tab.as<uint32_t>(),
                                   c->oh_err.as<int>(), GR, GC, s, &why);
  if (rc != RBG_OK) throw Error(rc, std::string("one-hot tensor-core pass: ") + why);
  // the kernel's wait status comes back with the caller's next synchronisation
  CK(cudaMemcpyAsync(c->oh_errpin.p, c->oh_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  c->oh_pending = true;
  c->launches += 6;
}

// Symmetric pass as the tcgen05 prefilter and the per-block check
// (kernels_sym_tc5.cu): candidate lists per 32-row block, with capacities
// from the fraction of pairs the last passes kept (or exact ones after a pass
// whose lists overflowed).  RBG_SYM_SINGLE=1: the single-kernel pass
// (mma.sync prefilter) instead.
bool sym_tc5_on() { return getenv("RBG_SYM_SINGLE") == nullptr; }

bool sym_tc5_fits(const GraphArgs &g) {
  // S < 64 leaves the last of the 64 padded halves for the threshold column
  return sym_tc5_on() && g.S < 64 && g.Kp <= 64 && g.n > 0 && g.n < ((int64_t)1 << 27);
}

// Buffers, list capacities (for the whole assembly), the padded FP16 rows and
// cleared flags for the passes over one assembly; `slots` item tables (one per
// pass in flight).  The capacities come from the kept fraction, or exact ones
// right after a pass whose lists overflowed (the one host copy here, on a
// rerun only); offsets and item tables are made on the device, so nothing is
// copied in while input chunks stream in.
void sym_tc5_setup(rbg_ctx *c, const GraphArgs &g, int slots) {
  const int64_t n = g.n, B32 = (n + 31) / 32, RBmax = (n + 127) / 128;
  cudaStream_t s = c->stream;
  int64_t total = 0;
  c->tc5_coff.ensure((size_t)(B32 + 1) * sizeof(int64_t));
  if (c->tc5_exact && c->tc5_n == n && c->tc5_cap.size() == (size_t)B32) {
    for (int64_t b = 0; b < B32; ++b) total += c->tc5_cap[b];
    c->tc5_pin.ensure((size_t)B32 * sizeof(int64_t));
    std::memcpy(c->tc5_pin.p, c->tc5_cap.data(), (size_t)B32 * sizeof(int64_t));
    c->tc5_caps.ensure((size_t)B32 * sizeof(int64_t));
    CK(cudaMemcpyAsync(c->tc5_caps.p, c->tc5_pin.p, (size_t)B32 * sizeof(int64_t),
                       cudaMemcpyHostToDevice, s));
    launch_tc5_coff(n, 0.0, c->tc5_caps.as<int64_t>(), c->tc5_coff.as<int64_t>(), s);
  } else {
    total = tc5_capacity(n, c->tc5_frac);
    launch_tc5_coff(n, c->tc5_frac, nullptr, c->tc5_coff.as<int64_t>(), s);
  }
  c->tc5_exact = false;
  c->tc5_n = n;
  c->tc5_rbmax = RBmax;
  c->tc5_items.ensure((size_t)slots * (RBmax + 1) * sizeof(int32_t));
  c->tc5_cand.ensure((size_t)std::max<int64_t>(total, 1) * sizeof(uint32_t));
  c->tc5_cnt.ensure((size_t)B32 * sizeof(int32_t));
  c->tc5_u16p.ensure((size_t)n * 256);         // row and column copies
  c->tc5_flags.ensure(2 * sizeof(int));
  CK(cudaMemsetAsync(c->tc5_flags.p, 0, 2 * sizeof(int), s));
  launch_pad_unit16(g, prefilter_lo16(g.S, g.prefilter_eps), c->tc5_u16p.as<uint16_t>(), s);
  c->launches += 2;
}

// The pass over the pairs i < j with j in [cb, ce) (item table in `slot`).
void sym_tc5_pass(rbg_ctx *c, const GraphArgs &g, const SymOut &o, int64_t cb, int64_t ce,
                  int slot) {
  int RB = 0, NT = 0;
  const int items = sym_tc5_items(cb, ce, &RB, &NT);
  if (items == 0) return;
  const int64_t blocks = (ce + 31) / 32;
  int32_t *di0 = c->tc5_items.as<int32_t>() + (size_t)slot * (c->tc5_rbmax + 1);
  cudaStream_t s = c->stream;
  launch_tc5_items(cb, ce, di0, s);
  CK(cudaMemsetAsync(c->tc5_cnt.p, 0, (size_t)blocks * sizeof(int32_t), s));
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const char *why = "";
  const int rc = launch_sym_prefilter(
      g, c->tc5_u16p.as<uint16_t>(), cb, ce, di0, RB, NT, items, c->tc5_cand.as<uint32_t>(), c->tc5_coff.as<int64_t>(), c->tc5_cnt.as<int32_t>(),
      c->tc5_flags.as<int>(), c->tc5_flags.as<int>() + 1, sms, s, &why);
  if (rc != RBG_OK) throw Error(rc, std::string("tensor-core prefilter: ") + why);
  launch_sym_check(g, o, c->tc5_cand.as<uint32_t>(), c->tc5_coff.as<int64_t>(),
                   c->tc5_cnt.as<int32_t>(), blocks, s);
  c->launches += 3;
}

// After the pass's synchronisation (the flags and counts read back into
// c->tc5_host): false when a list overflowed (capacities now exact: rerun).
bool sym_tc5_settle(rbg_ctx *c, int64_t n) {
  const int64_t B32 = (n + 31) / 32;
  const int *fl = c->tc5_host.as<int>();
  const int32_t *cnt = fl + 4;
  if (fl[1] != 0)
    throw Error(RBG_ERR_TIMEOUT, "tensor-core prefilter: a bounded device wait gave up (stage " +
                                     std::to_string(fl[1]) + ")");
  double frac = 0.0;
  for (int64_t b = 0; b < B32; ++b) {
    const double pairs = 32.0 * (double)std::max<int64_t>(n - 32 * b, 0);
    if (pairs > 0) frac = std::max(frac, cnt[b] / pairs);
  }
  if (fl[0] != 0) {                          // rerun with room for every block's count
    c->tc5_cap.assign((size_t)B32, 0);
    for (int64_t b = 0; b < B32; ++b) {
      const double pairs = 32.0 * (double)std::max<int64_t>(n - 32 * b, 0);
      const int64_t fc = ((int64_t)(pairs * c->tc5_frac) + 256 + 31) & ~(int64_t)31;
      c->tc5_cap[b] = std::max<int64_t>(fc, ((int64_t)cnt[b] + 256 + 31) & ~(int64_t)31);
    }
    c->tc5_exact = true;
    c->tc5_frac = std::max(c->tc5_frac, frac * 1.25);
    return false;
  }
  if (frac * 1.25 > c->tc5_frac) c->tc5_frac = frac * 1.25;   // room to spare next time
  return true;
}

// The flags and per-block counts to the host on the stream (read after its sync).
void sym_tc5_readback(rbg_ctx *c, int64_t n) {
  const int64_t B32 = (n + 31) / 32;
  c->tc5_host.ensure((size_t)(4 + B32) * sizeof(int32_t));
  CK(cudaMemcpyAsync(c->tc5_host.p, c->tc5_flags.p, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaMemcpyAsync(c->tc5_host.as<int32_t>() + 4, c->tc5_cnt.p, (size_t)B32 * sizeof(int32_t),
                     cudaMemcpyDeviceToHost, c->stream));
}

void check_onehot_status(rbg_ctx *c) {
  if (!c->oh_pending) return;
  c->oh_pending = false;
  const int e = *c->oh_errpin.as<int>();
  if (e != 0)
    throw Error(RBG_ERR_TIMEOUT, "one-hot tensor-core pass: a bounded device wait gave up (stage " +
                                     std::to_string(e) + ")");
}

}  // namespace rbg

namespace {

// Graph + edge weights on the codes already in c->codesA/B and the staged depth.
// With sc, the rows of one rank of a sharded assembly (full rows scored, row
// maxima and neighbour lists exchanged).
void run_graph(rbg_ctx *c, const rbg_params *p, const ShardCtx *sc = nullptr) {
  const bool streamed_in = c->streamed;     // pairs scored behind the copy (this call only)
  c->streamed = false;
  const int64_t n = c->n;
  const int m = p->m, mpad = mpad_of(m), S = c->S, K = p->max_edges;
  const int64_t n1 = std::max<int64_t>(n, 1);
  const int Su = (std::max(S, 1) + 3) & ~3;
  const double w_comp = (p->w_comp < 0.0) ? (S <= 2 ? 1.0 : 0.0) : p->w_comp;
  if (!c->prep_done) prep_depth(c, p);
  GraphArgs g = graph_args(c, p);
  const bool use_colnorm = need_colnorm(p, S);
  CK(cudaEventRecord(c->ev[4], c->stream));

  // b0 on the codes (equal codes <=> equal winners of the chosen width); the
  // one-permutation metric has no baseline (src/rabbitbin.cpp:4958)
  // With the baseline on, b0 and the similarity table are made on the device
  // (sample counts, median by histogram) and b0 comes back with the row maxima.
  const bool oph = p->oph_k > 0;
  const bool dev_b0 = p->base_on && !oph;
  c->b0 = 0.0;
  std::vector<double> sv_d;
  std::vector<float> sv_f;
  if (dev_b0) {
    const auto prs = b0_pairs(n);
    const int np = (int)(prs->size() / 2);
    c->pairs.ensure(std::max<size_t>((size_t)np, 1) * 2 * sizeof(int64_t));
    c->pair_out.ensure(std::max<size_t>((size_t)np, 1) * sizeof(uint32_t) + 16);
    if (np) {
      if (c->pairs_n != n) {              // the sample depends on n only: uploaded once per n
        std::vector<int64_t> pr(prs->begin(), prs->end());
        CK(cudaMemcpyAsync(c->pairs.p, pr.data(), pr.size() * sizeof(int64_t),
                           cudaMemcpyHostToDevice, c->stream));
        c->pairs_n = n;
      }
      launch_pair_counts(c->codesA.as<uint8_t>(), c->codesB.as<uint8_t>(), mpad, m,
                         c->pairs.as<int64_t>(), np, c->pair_out.as<uint32_t>(), c->stream);
      c->launches++;
    }
    c->b0dev.ensure(sizeof(float));
    launch_b0(c->pair_out.as<uint32_t>(), np, m, c->b0dev.as<float>(), c->svbits.as<uint32_t>(),
              c->stream);
    c->launches++;
    // comes back with the row maxima (their read synchronises the stream)
    c->b0pin.ensure(sizeof(float));
    CK(cudaMemcpyAsync(c->b0pin.p, c->b0dev.p, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  } else {
    if (oph) oph_sv_table(m, sv_d, sv_f);
    else sv_table(m, false, 0.0, sv_d, sv_f);
    std::vector<uint32_t> sv_bits(m + 1);
    std::memcpy(sv_bits.data(), sv_f.data(), (m + 1) * sizeof(uint32_t));
    CK(cudaMemcpyAsync(c->svbits.p, sv_bits.data(), (m + 1) * sizeof(uint32_t),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));               // sv_bits is a stack vector
  }
  CK(cudaEventRecord(c->ev[5], c->stream));

  // N > 25000 (or force_path 2): the fused path of the ProbMinHash metric; the
  // one-permutation metric keeps the small path's graph and calibrates on ten
  // 2500-contig samples (calibrate_sim_cutoff_fused, src/impl/rb_graph.cpp:1386-1431)
  const bool large = (p->force_path == 2) || (p->force_path == 0 && n > 25000);
  const bool fused = large && !oph;
  if (large && n <= 2500) throw Error(RBG_ERR_ARG, "the large-N path samples 2500 contigs; need n > 2500");
  const CalibMode cmode = !large ? CalibMode::all : (oph ? CalibMode::samples_all : CalibMode::fused);
  c->path = fused ? 2 : 1;
  CK(cudaStreamWaitEvent(c->stream, c->ev_aux, 0));   // unit rows, anynz, column norms
  c->prep_done = false;
  std::vector<uint32_t> maxc;
  const uint32_t *maxc_host = nullptr;
  const bool sym_shard = sc && g.prefilter && n > 0;
  if (sym_shard) {
    // Sharded assembly, tensor-core regime: this rank runs its share of the
    // symmetric pass (every unordered pair is scored by exactly one rank), then
    // the ranks exchange their admitted pairs and partial row maxima, and every
    // rank selects every row's top-K from the whole pair list (so no neighbour
    // lists need exchanging for the mutual filter).  A list that overflowed on
    // any rank is rerun everywhere with a larger one: every rank sees the same
    // gathered counts, so all take the same collective steps.
    const int W = sc->world;
    const size_t nm4 = (size_t)((n1 + 3) & ~3);
    c->pin.ensure(nm4 * sizeof(uint32_t) + sizeof(unsigned long long));
    uint32_t *hmax = c->pin.as<uint32_t>();
    for (;;) {
      SymOut o = sym_buffers(c, n1);
      sym_clear(c, n1);
      launch_allpairs_sym(g, o, c->stream, sc->rank, W);
      c->launches += 1;
      CK(cudaGetLastError());
      CK(cudaEventRecord(c->ev[6], c->stream));
      c->shard_send.ensure(16);
      c->shard_recv.ensure(16 * (size_t)W);
      CK(cudaMemcpyAsync(c->shard_send.p, c->sym_np.p, sizeof(unsigned long long),
                         cudaMemcpyDeviceToDevice, c->stream));
      sc->gather(c->shard_send.p, c->shard_recv.p, sizeof(unsigned long long));
      std::vector<unsigned long long> np(W);
      CK(cudaMemcpy(np.data(), c->shard_recv.p, W * sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost));
      unsigned long long npmax = 0, total = 0;
      for (int r = 0; r < W; ++r) {
        npmax = std::max(npmax, np[r]);
        total += np[r];
      }
      if (npmax > c->sym_cap) {
        c->sym_cap = npmax + npmax / 4;
        continue;
      }
      const size_t blk = (size_t)std::max<unsigned long long>(npmax, 1) * sizeof(uint4);
      c->shard_send.ensure(blk);
      c->shard_recv.ensure(blk * W);
      if (np[sc->rank])
        CK(cudaMemcpyAsync(c->shard_send.p, c->sym_pairs.p, np[sc->rank] * sizeof(uint4),
                           cudaMemcpyDeviceToDevice, c->stream));
      sc->gather(c->shard_send.p, c->shard_recv.p, blk);
      if (total > c->sym_cap) c->sym_cap = total;
      o = sym_buffers(c, n1);
      unsigned long long at = 0;
      for (int r = 0; r < W; ++r) {
        if (np[r])
          CK(cudaMemcpyAsync(o.pairs + at, c->shard_recv.as<char>() + r * blk,
                             np[r] * sizeof(uint4), cudaMemcpyDeviceToDevice, c->stream));
        at += np[r];
      }
      CK(cudaMemcpyAsync(o.npairs, &total, sizeof(total), cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemsetAsync(o.rowcnt, 0, n1 * sizeof(int32_t), c->stream));
      launch_pair_rowcounts(o.pairs, total, o.rowcnt, c->stream);
      // row maxima: the largest of every rank's partial maxima
      const size_t mb = ((size_t)n1 * sizeof(uint32_t) + 15) & ~(size_t)15;
      c->shard_send.ensure(mb);
      c->shard_recv.ensure(mb * W);
      CK(cudaMemcpyAsync(c->shard_send.p, c->maxc_cand.p, n * sizeof(uint32_t),
                         cudaMemcpyDeviceToDevice, c->stream));
      sc->gather(c->shard_send.p, c->shard_recv.p, mb);
      launch_max_blocks(c->shard_recv.as<uint32_t>(), W, (int64_t)(mb / sizeof(uint32_t)), n,
                        c->maxc_cand.as<uint32_t>(), c->stream);
      CK(cudaMemcpyAsync(hmax, c->maxc_cand.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                         c->stream));
      launch_rows_topk(g, o, c->sym_rowoff.as<int64_t>(), c->sym_keys.as<uint64_t>(), c->stream);
      CK(cudaGetLastError());
      c->launches += 5;
      CK(cudaStreamSynchronize(c->stream));          // `total` and the maxima on the host
      break;
    }
    maxc_host = hmax;
  } else if (g.prefilter && n > 0 && !sc) {
    // Tensor-core regime: every unordered pair scored once, admitted pairs
    // listed, then each row's top-K selected from its keys.  The row maxima and
    // the pair count come back while the selection runs; a pass whose pairs did
    // not fit the list is run again with a larger one.  When rbg_bin_graph
    // already scored the pairs behind the input copy (admission deferred), the
    // selection converts the stored counts; if those did not fit, this
    // configuration is scored here from then on.
    const size_t nm4 = (size_t)((n1 + 3) & ~3);
    c->pin.ensure(nm4 * sizeof(uint32_t) + sizeof(unsigned long long));
    uint32_t *hmax = c->pin.as<uint32_t>();
    unsigned long long *hnp = (unsigned long long *)(hmax + nm4);
    bool streamed = streamed_in;
    for (;;) {
      SymOut o = sym_buffers(c, n1);
      const bool tc5 = !streamed && sym_tc5_fits(g);
      if (streamed) {
        o.defer = 1;
        if (c->streamed_tc5) sym_tc5_readback(c, n);
      } else {
        sym_clear(c, n1);
        if (tc5) {
          sym_tc5_setup(c, g, 1);
          sym_tc5_pass(c, g, o, 0, n, 0);
          sym_tc5_readback(c, n);
        } else {
          launch_allpairs_sym(g, o, c->stream);
          c->launches += 1;
        }
      }
      CK(cudaGetLastError());
      CK(cudaEventRecord(c->ev[6], c->stream));
      CK(cudaMemcpyAsync(hmax, c->maxc_cand.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaMemcpyAsync(hnp, c->sym_np.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaEventRecord(c->ev[10], c->stream));
      if (streamed)
        launch_rows_topk_counts(g, o, g.sv_bits, c->sym_rowoff.as<int64_t>(),
                                c->sym_keys.as<uint64_t>(), c->stream);
      else
        launch_rows_topk(g, o, c->sym_rowoff.as<int64_t>(), c->sym_keys.as<uint64_t>(), c->stream);
      CK(cudaGetLastError());
      c->launches += 3;
      CK(cudaEventSynchronize(c->ev[10]));
      if (streamed && c->streamed_tc5) {
        const int *fl = c->tc5_host.as<int>();
        if (fl[1] != 0)
          throw Error(RBG_ERR_TIMEOUT, "tensor-core prefilter: a bounded device wait gave up "
                                       "(stage " + std::to_string(fl[1]) + ")");
        if (fl[0] != 0) {                            // a window's list overflowed: rescore
          CK(cudaStreamSynchronize(c->stream));
          c->tc5_frac *= 2.0;
          streamed = false;
          continue;
        }
      }
      if (tc5 && !sym_tc5_settle(c, n)) {           // a candidate list overflowed: rerun
        CK(cudaStreamSynchronize(c->stream));
        continue;
      }
      if (*hnp <= c->sym_cap) break;
      CK(cudaStreamSynchronize(c->stream));
      if (streamed) {
        c->no_stream_S |= 1ull << (S & 63);  // survivors outgrow the list at this S
        streamed = false;
      } else {
        c->sym_cap = *hnp + *hnp / 4;
      }
    }
    maxc_host = hmax;
  } else {
    CK(cudaMemsetAsync(c->stats.p, 0, 2 * sizeof(unsigned long long), c->stream));
    if (sc) {
      g.row_lo = sc->row_lo;
      g.row_hi = sc->row_hi;
    }
    const int64_t rows = sc ? sc->row_hi - sc->row_lo : n;
    CK(cudaMemsetAsync(c->maxc_cand.p, 0, n1 * sizeof(uint32_t), c->stream));
    CK(cudaMemsetAsync(c->maxc_all.p, 0, n1 * sizeof(uint32_t), c->stream));
    if (!g.prefilter && dense_on_gemm() && onehot_mma_fits(n, m)) {
      dense_allpairs_onehot(c, g);                      // tensor cores, exact counts
    } else {
      const size_t slots = (size_t)((rows + 31) / 32) * allpairs_slices_rows(rows, n, K) * 32;
      c->cand_buf.ensure(std::max<size_t>(slots, 1) * allpairs_cap(K) * sizeof(uint64_t));
      c->cand_cnt.ensure(std::max<size_t>(slots, 1) * sizeof(int32_t));
      launch_allpairs(g, c->cand_buf.as<uint64_t>(), c->cand_cnt.as<int32_t>(), c->stream);
      c->launches += rows ? 2 : 0;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev[6], c->stream));
    uint32_t *dmax = fused ? c->maxc_cand.as<uint32_t>() : c->maxc_all.as<uint32_t>();
    if (sc) share_rows(c, *sc, dmax, dmax, sizeof(uint32_t));     // every rank's maxima
    maxc.assign(n1, 0);
    CK(cudaMemcpyAsync(maxc.data(), dmax, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    check_onehot_status(c);
    maxc_host = maxc.data();
  }

  if (dev_b0) {
    // b0 as the device stored it (float; its copy completed with the maxima
    // read), and the same tables on the host
    c->b0 = (double)*c->b0pin.as<float>();
    sv_table(m, true, c->b0, sv_d, sv_f);
  }
  // calibration on the host (rand() sequence of the reference)
  const double simCutoff = calibrate_cutoff(maxc_host, n, cmode, m, sv_d, sv_f, p->coverage, p->seed);
  c->sim_cutoff = simCutoff;
  CK(cudaEventRecord(c->ev[7], c->stream));

  // RABBIT_GRAPH_INDEX=1 on the small path: each row's neighbours again, from
  // the candidates of the inverted index (src/impl/rb_graph.cpp:199-383)
  if (!fused && p->graph_index) {
    if (sc) throw Error(RBG_ERR_UNSUPPORTED, "graph_index is not available for sharded assemblies");
    index_graph(c, p, g, simCutoff / 1000.);
  }

  // neighbour lists, edges
  c->nbr.ensure(n1 * K * sizeof(uint32_t));
  c->nbr_sv.ensure(n1 * K * sizeof(float));
  c->nbr_cnt.ensure(n1 * sizeof(int32_t));
  c->row_edges.ensure((n1 + 1) * sizeof(int32_t));
  EmitArgs e;
  e.n = n; e.K = K; e.mutual = p->mutual; e.small_path = fused ? 0 : 1;
  e.topk = g.topk; e.topk_cnt = g.topk_cnt;
  e.cutoff = simCutoff / 1000.;
  e.nbr_sorted = c->nbr.as<uint32_t>();
  e.nbr_sv = c->nbr_sv.as<float>();
  e.nbr_cnt = c->nbr_cnt.as<int32_t>();
  e.row_edges = c->row_edges.as<int32_t>();
  c->kept.ensure(n1 * ((K + 31) / 32) * sizeof(uint32_t));
  e.kept = c->kept.as<uint32_t>();
  if (sc && !sym_shard) {
    e.row_lo = sc->row_lo;
    e.row_hi = sc->row_hi;
  }
  const int64_t e_hi = sc ? sc->row_hi : n;
  launch_sort_rows(e, c->stream);
  if (sc && !sym_shard) {
    // the mutual filter reads the partners' lists: every rank's rows
    share_rows(c, *sc, e.nbr_sorted, e.nbr_sorted, (size_t)K * sizeof(uint32_t));
    share_rows(c, *sc, e.nbr_cnt, e.nbr_cnt, sizeof(int32_t));
  }
  if (sym_shard) {                      // every row's list is here; the edges of this rank's rows
    e.row_lo = sc->row_lo;
    e.row_hi = sc->row_hi;
  }
  launch_count_edges(e, c->stream);
  c->launches += n ? 3 : 0;
  int32_t ne = 0;
  if (n > 0 && e_hi > e.row_lo) {
    CK(cudaMemcpyAsync(&ne, c->row_edges.as<int32_t>() + e_hi, sizeof(int32_t),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  c->n_edges = ne;
  const size_t ne1 = std::max<int64_t>(ne, 1);
  c->e_from.ensure(ne1 * 4);
  c->e_to.ensure(ne1 * 4);
  c->e_scomp.ensure(ne1 * 4);
  c->e_score.ensure(ne1 * 4);
  e.from = c->e_from.as<uint32_t>();
  e.to = c->e_to.as<uint32_t>();
  e.scomp = c->e_scomp.as<float>();
  launch_write_edges(e, c->stream);
  c->launches += n ? 1 : 0;
  CK(cudaEventRecord(c->ev[8], c->stream));

  WeightArgs w;
  w.n_edges = ne;
  w.S = S;
  w.from = e.from; w.to = e.to; w.scomp = e.scomp;
  w.score = c->e_score.as<float>();
  w.unit = c->unit.as<float>();
  w.Su = Su;
  w.depth_raw = c->depth.as<float>();
  w.colnorm = use_colnorm ? c->colnorm.as<double>() : nullptr;
  w.w_comp = w_comp;
  w.min_edge = p->min_edge;
  w.neg_thr = p->neg_thr;
  w.wjac_cut = p->wjac_cut;
  w.depth_sim = p->depth_sim;
  w.depth_fuse = p->depth_fuse;
  w.wjac_gate = p->wjac_gate;
  w.contract = p->fp_contract;
  launch_edge_weights(w, c->stream);
  c->launches += ne ? 1 : 0;
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[9], c->stream));
  c->graph_ready = true;
}

// Pinned host blocks for graph results: the four edge arrays of one graph
// share one block, which the device writes at DMA speed (pageable destinations
// are slow and page-fault on first touch).  rbg_free_graph returns a block to
// the pool.  Blocks come in sizes 2^k and 1.5 x 2^k from 1 MB, so a stream of
// graphs of varying sizes reuses a few blocks instead of pinning and unpinning
// memory per call (each costs milliseconds); up to 16 idle blocks and 4 GB are
// kept, the longest idle freed first.  A batch's graphs share one block (each
// graph's arrays are ranges of the batch-wide arrays): it returns to the pool
// when the last of them is freed.
struct PinnedPool {
  struct Shared {
    void *blk;
    int refs;
  };
  std::mutex mu;
  std::unordered_map<void *, size_t> live;
  std::unordered_map<void *, Shared *> part;   // a graph's first array -> its shared block
  std::deque<std::pair<size_t, void *>> idle;  // oldest first
  size_t idle_bytes = 0;

  // 1, 1.5, 2, 3, 4, 6, ... MB: at most a third of a block unused
  static size_t size_class(size_t bytes) {
    size_t c = (size_t)1 << 20;
    while (c < bytes) c = (c & (c - 1)) == 0 ? c / 2 * 3 : c / 3 * 4;
    return c;
  }

  void *take(size_t bytes) {
    const size_t cls = size_class(bytes);
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = idle.rbegin(); it != idle.rend(); ++it)
      if (it->first == cls) {
        void *p = it->second;
        idle_bytes -= cls;
        idle.erase(std::next(it).base());
        live[p] = cls;
        return p;
      }
    void *p = nullptr;
    if (cudaHostAlloc(&p, cls, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    live[p] = cls;
    return p;
  }

  // Hand a block taken with take() to graphs whose first arrays are `firsts`
  // (distinct pointers inside the block); none: the block goes back at once.
  void share(void *blk, const std::vector<void *> &firsts) {
    if (firsts.empty()) {
      give(blk);
      return;
    }
    std::lock_guard<std::mutex> lk(mu);
    Shared *sh = new Shared{blk, (int)firsts.size()};
    for (void *f : firsts) part[f] = sh;
  }

  bool give(void *p) {
    std::lock_guard<std::mutex> lk(mu);
    auto sp = part.find(p);
    if (sp != part.end()) {
      Shared *sh = sp->second;
      part.erase(sp);
      if (--sh->refs > 0) return true;
      p = sh->blk;
      delete sh;
    }
    auto it = live.find(p);
    if (it == live.end()) return false;
    idle.emplace_back(it->second, p);
    idle_bytes += it->second;
    live.erase(it);
    while (idle.size() > 16 || idle_bytes > ((size_t)4 << 30)) {
      idle_bytes -= idle.front().first;
      cudaFreeHost(idle.front().second);
      idle.pop_front();
    }
    return true;
  }
};

PinnedPool &pinned_pool() {
  static PinnedPool *pool = new PinnedPool();     // outlives every context
  return *pool;
}

}  // namespace

namespace rbg {

void *pinned_take(size_t bytes) { return pinned_pool().take(bytes); }
void pinned_share(void *blk, const std::vector<void *> &firsts) {
  pinned_pool().share(blk, firsts);
}

}  // namespace rbg

namespace {

void fetch(rbg_ctx *c, rbg_graph *out) {
  if (!out) throw Error(RBG_ERR_ARG, "null graph");
  if (!c->graph_ready) throw Error(RBG_ERR_ARG, "no graph has been built on this context");
  std::memset(out, 0, sizeof(*out));
  const size_t ne = (size_t)c->n_edges;
  out->n_edges = (int64_t)ne;
  out->b0 = c->b0;
  out->sim_cutoff = c->sim_cutoff;
  out->path = c->path;
  const size_t n1 = std::max<size_t>(ne, 1);
  const size_t nb = n1 * 4;
  if (void *blk = pinned_pool().take(4 * nb)) {
    out->from = (uint32_t *)blk;
    out->to = out->from + n1;
    out->scomp = (float *)(out->to + n1);
    out->score = out->scomp + n1;
  } else {
    out->from = (uint32_t *)malloc(nb);
    out->to = (uint32_t *)malloc(nb);
    out->scomp = (float *)malloc(nb);
    out->score = (float *)malloc(nb);
  }
  if (!out->from || !out->to || !out->scomp || !out->score) {
    rbg_free_graph(out);
    throw Error(RBG_ERR_NOMEM, "host allocation of the edge arrays failed");
  }
  if (ne) {
    // from, to and sComp are final once the edges are written (event 8): they
    // come back on the copy stream while the edge weights are computed
    CK(cudaStreamWaitEvent(c->copy, c->ev[8], 0));
    CK(cudaMemcpyAsync(out->from, c->e_from.p, ne * 4, cudaMemcpyDeviceToHost, c->copy));
    CK(cudaMemcpyAsync(out->to, c->e_to.p, ne * 4, cudaMemcpyDeviceToHost, c->copy));
    CK(cudaMemcpyAsync(out->scomp, c->e_scomp.p, ne * 4, cudaMemcpyDeviceToHost, c->copy));
    CK(cudaMemcpyAsync(out->score, c->e_score.p, ne * 4, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->copy));
  CK(cudaStreamSynchronize(c->stream));
}

// One rank of rbg_bin_graph_sharded.
void bin_graph_sharded(rbg_ctx *c, const rbg_params *p, const rbg_shard *sh, const char *seqcat,
                       const int64_t *offsets, int64_t n_local, const float *depth, int S,
                       rbg_graph *out) {
  if (!sh || !sh->allgather || sh->world < 1 || sh->rank < 0 || sh->rank >= sh->world)
    throw Error(RBG_ERR_ARG, "bad shard description");
  if (n_local < 0) throw Error(RBG_ERR_ARG, "n_local < 0");
  if (p->oph_k > 0)
    throw Error(RBG_ERR_UNSUPPORTED, "sharded assemblies use the ProbMinHash metric (oph_k = 0)");
  const int W = sh->world;
  const int m = p->m, mpad = mpad_of(m);
  ShardCtx sc;
  sc.rank = sh->rank;
  sc.world = W;
  sc.gather = [c, sh, W](const void *dsend, void *drecv, size_t bytes) {
    CK(cudaStreamSynchronize(c->stream));
    int rc;
    if (sh->device_buffers) {
      rc = sh->allgather(dsend, drecv, bytes, sh->user);
    } else {
      c->shard_host.ensure(bytes * (W + 1));
      char *h = c->shard_host.as<char>();
      CK(cudaMemcpy(h, dsend, bytes, cudaMemcpyDeviceToHost));
      rc = sh->allgather(h, h + bytes, bytes, sh->user);
      if (rc == 0) CK(cudaMemcpy(drecv, h + bytes, bytes * W, cudaMemcpyHostToDevice));
    }
    if (rc != 0) throw Error(RBG_ERR_COMM, "the caller's allgather failed");
  };
  // 1. how many rows each rank holds (and the same S everywhere)
  {
    c->shard_send.ensure(16);
    c->shard_recv.ensure(16 * W);
    const int64_t mine[2] = {n_local, S};
    CK(cudaMemcpyAsync(c->shard_send.p, mine, sizeof(mine), cudaMemcpyHostToDevice, c->stream));
    sc.gather(c->shard_send.p, c->shard_recv.p, sizeof(mine));
    std::vector<int64_t> all(2 * W);
    CK(cudaMemcpy(all.data(), c->shard_recv.p, all.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
    sc.row0.assign(W + 1, 0);
    for (int r = 0; r < W; ++r) {
      if (all[2 * r + 1] != S) throw Error(RBG_ERR_ARG, "ranks disagree on S");
      if (all[2 * r] < 0) throw Error(RBG_ERR_ARG, "a rank passed n_local < 0");
      sc.row0[r + 1] = sc.row0[r] + all[2 * r];
      sc.nmax = std::max(sc.nmax, all[2 * r]);
    }
  }
  const int64_t n = sc.row0[W];
  if (n >= (1 << 27)) throw Error(RBG_ERR_UNSUPPORTED, "at most 2^27 - 1 contigs per assembly");
  sc.row_lo = sc.row0[sc.rank];
  sc.row_hi = sc.row0[sc.rank + 1];
  // 2. this rank's contigs: stage and sketch
  stage(c, seqcat, offsets, n_local, depth, S);
  run_sketch(c, p, false);
  // 3. every rank's register codes and coverage rows
  const size_t code_b = (size_t)sc.nmax * mpad, dep_b = (size_t)sc.nmax * S * sizeof(float);
  const size_t blk = code_b + ((dep_b + 15) & ~(size_t)15);
  c->shard_send.ensure(std::max<size_t>(blk, 16));
  c->shard_recv.ensure(std::max<size_t>(blk * W, 16));
  CK(cudaMemsetAsync(c->shard_send.p, 0, blk, c->stream));
  if (n_local) {
    CK(cudaMemcpyAsync(c->shard_send.p, c->codesA.p, (size_t)n_local * mpad, cudaMemcpyDeviceToDevice,
                       c->stream));
    if (S)
      CK(cudaMemcpyAsync(c->shard_send.as<char>() + code_b, c->depth.p,
                         (size_t)n_local * S * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
  }
  sc.gather(c->shard_send.p, c->shard_recv.p, blk);
  const int64_t n1 = std::max<int64_t>(n, 1);
  c->n = n;
  c->codesA.ensure(n1 * mpad);
  c->codesB.ensure(n1 * mpad);
  c->depth.ensure(std::max<size_t>(1, (size_t)n * S) * sizeof(float));
  const char *rb = c->shard_recv.as<char>();
  for (int r = 0; r < W; ++r) {
    const int64_t nr = sc.row0[r + 1] - sc.row0[r];
    if (!nr) continue;
    CK(cudaMemcpyAsync(c->codesA.as<char>() + sc.row0[r] * mpad, rb + r * blk, (size_t)nr * mpad,
                       cudaMemcpyDeviceToDevice, c->stream));
    if (S)
      CK(cudaMemcpyAsync(c->depth.as<float>() + sc.row0[r] * S, rb + r * blk + code_b,
                         (size_t)nr * S * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
  }
  launch_codes_b(c->codesA.as<uint8_t>(), c->codesB.as<uint8_t>(), n * mpad, c->stream);
  c->launches += n ? 1 : 0;
  c->prep_done = false;                // coverage rows of the whole assembly
  // 4. full rows of this rank's contigs; maxima and neighbour lists exchanged
  run_graph(c, p, &sc);
  fetch(c, out);
}

// Map externally produced 32-bit winner rows onto register codes.
void codes_from_winners(rbg_ctx *c, const rbg_params *p, const uint32_t *w32, int64_t n) {
  Tables &T = tables_for(c, p);
  const PmhTables &t = *T.t;
  const int m = p->m, mpad = mpad_of(m);
  if (!T.dict_ready) {
    std::vector<uint32_t> vals((size_t)m * kMaxElems, 0);
    std::vector<uint8_t> codes((size_t)m * kMaxElems, 0);
    std::vector<int32_t> nv(m, 0);
    const std::vector<uint8_t> &cd = p->win_bits == 16 ? t.code16 : t.code32;
    for (int r = 0; r < m; ++r) {
      std::vector<std::pair<uint32_t, uint8_t>> col;
      for (int e = 0; e < t.n_elems; ++e) {
        const size_t q = (size_t)e * m + r;
        const uint32_t v = p->win_bits == 16 ? (uint32_t)t.W16[q] : t.W32[q];
        if (v) col.emplace_back(v, cd[q]);
      }
      std::sort(col.begin(), col.end());
      col.erase(std::unique(col.begin(), col.end()), col.end());
      nv[r] = (int32_t)col.size();
      for (size_t q = 0; q < col.size(); ++q) {
        vals[(size_t)r * kMaxElems + q] = col[q].first;
        codes[(size_t)r * kMaxElems + q] = col[q].second;
      }
    }
    T.dict_vals.ensure(vals.size() * 4);
    T.dict_codes.ensure(codes.size());
    T.dict_n.ensure(nv.size() * 4);
    CK(cudaMemcpyAsync(T.dict_vals.p, vals.data(), vals.size() * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.dict_codes.p, codes.data(), codes.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.dict_n.p, nv.data(), nv.size() * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    T.dict_ready = true;
  }
  const int64_t n1 = std::max<int64_t>(n, 1);
  c->winners32.ensure(n1 * m * 4);
  c->codesA.ensure(n1 * mpad);
  c->codesB.ensure(n1 * mpad);
  c->badflag.ensure(sizeof(int));
  CK(cudaMemsetAsync(c->badflag.p, 0, sizeof(int), c->stream));
  if (n) CK(cudaMemcpyAsync(c->winners32.p, w32, (size_t)n * m * 4, cudaMemcpyHostToDevice, c->stream));
  launch_codes_from_winners(c->winners32.as<uint32_t>(), n, m, mpad, p->win_bits == 16,
                            T.dict_vals.as<uint32_t>(), T.dict_codes.as<uint8_t>(),
                            T.dict_n.as<int32_t>(), c->codesA.as<uint8_t>(), c->codesB.as<uint8_t>(),
                            c->badflag.as<int>(), c->stream);
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, c->badflag.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (bad) throw Error(RBG_ERR_ARG, "winner rows do not come from this sketch configuration (k, m, seed)");
}

}  // namespace

namespace rbg {
// One assembly through the single-assembly path (sketch behind the chunked
// copy, graph, fetch) under a lock the caller already holds.
void bin_graph_one(rbg_ctx *c, const rbg_params *p, const rbg_assembly &x, rbg_graph *out) {
  validate(p);
  stage_sketch_chunked(c, p, x.seqcat, x.offsets, x.n, x.depth, x.S);
  run_graph(c, p);
  fetch(c, out);
}
}  // namespace rbg

extern "C" {

int rbg_default_params(rbg_params *p) {
  if (!p) return RBG_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->k = 4;
  p->m = 500;
  p->pmh_seed = 42;
  p->gc_norm = 1;
  p->win_bits = 16;
  p->gc_norm_cap = 20.0;
  p->max_edges = 200;
  p->mutual = 1;
  p->base_on = 1;
  p->seed = 1;
  p->force_path = 0;
  p->abdfirst = 1;
  p->coverage = 0.95;
  p->min_edge = 0.70;
  p->w_comp = -1.0;
  p->min_cv = 1.0;
  p->neg_thr = -0.3;
  p->depth_sim = 2;
  p->depth_fuse = 1;
  p->wjac_norm = 1;
  p->fp_contract = 1;
  p->wjac_cut = 0.0;
  p->wjac_gate = 0;
  p->oph_k = 0;
  p->oph_bits = 2;
  p->graph_index = 0;
  p->index_k = 8;
  p->min_common = 0;
  return RBG_OK;
}

int rbg_create(int device, rbg_ctx **out) {
  if (!out) return RBG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RBG_ERR_CUDA;
  if (device < 0 || device >= ndev) return RBG_ERR_ARG;
  auto *c = new (std::nothrow) rbg_ctx();
  if (!c) return RBG_ERR_NOMEM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return RBG_ERR_CUDA;
  }
  for (auto &e : c->ev) cudaEventCreate(&e);
  if (cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return RBG_ERR_CUDA;
  }
  cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&c->ev_aux, cudaEventDisableTiming);
  cudaEventCreate(&c->ev_a0);
  cudaEventCreate(&c->ev_a1);
  if (cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess) {
    cudaStreamDestroy(c->aux);
    cudaStreamDestroy(c->stream);
    delete c;
    return RBG_ERR_CUDA;
  }
  cudaEventCreateWithFlags(&c->ev_cin, cudaEventDisableTiming);
  for (auto &e : c->ev_chunk) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (auto &e : c->ev_slot) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  *out = c;
  return RBG_OK;
}

int rbg_destroy(rbg_ctx *c) {
  if (!c) return RBG_ERR_ARG;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  DBuf *bufs[] = {&c->ascii, &c->offsets, &c->depth, &c->packed, &c->nmask, &c->elem_idx,
                  &c->elem_winv, &c->elem_cnt, &c->codesA, &c->codesB, &c->winners32, &c->unit,
                  &c->anynz, &c->colnorm, &c->svbits, &c->topk, &c->topk_cnt, &c->maxc_cand,
                  &c->maxc_all, &c->stats, &c->pairs, &c->pair_out, &c->nbr, &c->nbr_sv,
                  &c->nbr_cnt, &c->row_edges, &c->e_from, &c->e_to, &c->e_scomp, &c->e_score,
                  &c->badflag, &c->tmp, &c->cand_buf, &c->cand_cnt, &c->colacc, &c->unit16,
                  &c->sym_pairs, &c->sym_np, &c->sym_rowcnt, &c->sym_rowoff, &c->sym_keys,
                  &c->shard_send, &c->shard_recv, &c->oh_pres, &c->oh_map, &c->oh_koff,
                  &c->oh_X, &c->oh_cand, &c->oh_cnt, &c->oh_tab, &c->oh_err, &c->kept, &c->b0dev,
                  &c->count_work, &c->tc5_u16p, &c->tc5_cand, &c->tc5_cnt, &c->tc5_items,
                  &c->tc5_coff, &c->tc5_caps, &c->tc5_flags,
                  &c->qa, &c->qb, &c->qo, &c->qt, &c->ix_keys, &c->ix_sorted,
                  &c->ix_contig, &c->ix_post, &c->ix_ukeys, &c->ix_count, &c->ix_off,
                  &c->ix_nk, &c->ix_scratch};
  for (DBuf *b : bufs) b->release();
  for (auto &t : c->tab_cache) t.second->release();
  release_batch_graphs(c);
  if (c->batch) c->batch->release();
  if (c->fasta) c->fasta->release();
  if (c->lpa) c->lpa->release();
  if (c->depthb) c->depthb->release();
  c->pin.release();
  c->b0pin.release();
  c->shard_host.release();
  for (auto &e : c->ev) cudaEventDestroy(e);
  cudaStreamSynchronize(c->aux);
  cudaStreamSynchronize(c->copy);
  for (cudaEvent_t e : {c->ev_in, c->ev_aux, c->ev_a0, c->ev_a1, c->ev_cin}) cudaEventDestroy(e);
  for (auto &e : c->ev_chunk) cudaEventDestroy(e);
  for (auto &e : c->ev_slot) cudaEventDestroy(e);
  c->pack_pin[0].release();
  c->pack_pin[1].release();
  c->tc5_pin.release();
  c->tc5_host.release();
  cudaStreamDestroy(c->copy);
  cudaStreamDestroy(c->aux);
  cudaStreamDestroy(c->stream);
  delete c;
  return RBG_OK;
}

const char *rbg_last_error(rbg_ctx *c) { return c ? c->err.c_str() : "null context"; }

void *rbg_stream(rbg_ctx *c) { return c ? (void *)c->stream : nullptr; }

int rbg_build_pmh_winners(rbg_ctx *c, const rbg_params *p, const char *seqcat,
                          const int64_t *offsets, int64_t n, uint32_t *out) {
  return guarded(c, [&] {
    validate(p);
    if (!out && n > 0) throw Error(RBG_ERR_ARG, "null output");
    stage(c, seqcat, offsets, n, nullptr, 0);
    run_sketch(c, p, true);
    c->prep_done = false;
    if (n) CK(cudaMemcpyAsync(out, c->winners32.p, (size_t)n * p->m * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int rbg_build_oph_signature(rbg_ctx *c, const rbg_params *p, const char *seqcat,
                            const int64_t *offsets, int64_t n, uint8_t *out) {
  return guarded(c, [&] {
    validate(p);
    if (p->oph_k < 1) throw Error(RBG_ERR_ARG, "oph_k must be set (1..32)");
    if (!out && n > 0) throw Error(RBG_ERR_ARG, "null output");
    stage(c, seqcat, offsets, n, nullptr, 0);
    run_sketch(c, p, false);
    c->prep_done = false;
    const int m = p->m, mpad = mpad_of(m);
    if (n) {
      c->tmp.ensure((size_t)n * m);
      launch_oph_values(c->codesA.as<uint8_t>(), n, m, mpad, c->tmp.as<uint8_t>(), c->stream);
      CK(cudaMemcpyAsync(out, c->tmp.p, (size_t)n * m, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
  });
}

int rbg_pack_win16(rbg_ctx *c, const uint32_t *in, int64_t count, uint16_t *out) {
  return guarded(c, [&] {
    if (count < 0 || (count > 0 && (!in || !out))) throw Error(RBG_ERR_ARG, "bad arguments");
    if (count == 0) return;
    c->winners32.ensure(count * 4);
    c->tmp.ensure(count * 2);
    CK(cudaMemcpyAsync(c->winners32.p, in, count * 4, cudaMemcpyHostToDevice, c->stream));
    launch_fold16(c->winners32.as<uint32_t>(), count, c->tmp.as<uint16_t>(), c->stream);
    CK(cudaMemcpyAsync(out, c->tmp.p, count * 2, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int rbg_estimate_pmh_baseline(rbg_ctx *c, const rbg_params *p, const void *winners,
                              int32_t win_bits, int64_t n, double *b0) {
  return guarded(c, [&] {
    validate(p);
    if (!b0 || (n > 0 && !winners) || (win_bits != 16 && win_bits != 32))
      throw Error(RBG_ERR_ARG, "bad arguments");
    const int m = p->m;
    const size_t bytes = (size_t)n * m * (win_bits / 8);
    c->tmp.ensure(std::max<size_t>(bytes, 4));
    if (bytes) CK(cudaMemcpyAsync(c->tmp.p, winners, bytes, cudaMemcpyHostToDevice, c->stream));
    *b0 = estimate_b0(c, n, m, [&](const int64_t *pr, int np, uint32_t *o) {
      c->pairs.ensure((size_t)np * 16);
      c->pairs_n = -1;                   // no longer the run_graph sample
      c->pair_out.ensure((size_t)np * 4);
      CK(cudaMemcpyAsync(c->pairs.p, pr, (size_t)np * 16, cudaMemcpyHostToDevice, c->stream));
      launch_raw_pair_counts(c->tmp.p, win_bits, m, c->pairs.as<int64_t>(), np,
                             c->pair_out.as<uint32_t>(), c->stream);
      CK(cudaMemcpyAsync(o, c->pair_out.p, (size_t)np * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    });
  });
}

int rbg_build_graph(rbg_ctx *c, const rbg_params *p, const uint32_t *winners32, int64_t n,
                    const float *depth, int32_t S, rbg_graph *out) {
  return guarded(c, [&] {
    validate(p);
    if (n < 0 || (n > 0 && !winners32) || !out) throw Error(RBG_ERR_ARG, "bad arguments");
    if (p->oph_k > 0)
      throw Error(RBG_ERR_ARG, "winner rows are ProbMinHash sketches; the one-permutation "
                               "metric starts from sequences (rbg_bin_graph)");
    if (S < 0 || S > kMaxS) throw Error(RBG_ERR_UNSUPPORTED, "S must be in 0..64");
    c->streamed = false;
    c->n = n;
    c->S = S;
    c->depth.ensure(std::max<size_t>(1, (size_t)n * S) * sizeof(float));
    if (S > 0 && n > 0) {
      if (!depth) throw Error(RBG_ERR_ARG, "depth is null");
      CK(cudaMemcpyAsync(c->depth.p, depth, (size_t)n * S * 4, cudaMemcpyHostToDevice, c->stream));
    }
    codes_from_winners(c, p, winners32, n);
    c->prep_done = false;                    // coverage changed: prepare it again
    run_graph(c, p);
    fetch(c, out);
  });
}

int rbg_bin_fasta(rbg_ctx *c, const rbg_params *p, const char *fasta, int64_t nbytes,
                  int64_t min_contig, const float *depth, int32_t S, rbg_graph *out) {
  return guarded(c, [&] {
    validate(p);
    // small contigs are not needed here: a small threshold equal to the large
    // one leaves that class empty
    const FastaCounts k = fasta_parse(c, fasta, nbytes, min_contig, min_contig);
    stage_device(c, c->fasta->seq[0].as<char>(), c->fasta->seq_off[0].as<int64_t>(), k.n[0],
                 k.bytes[0], depth, S);
    run_sketch(c, p, false);
    run_graph(c, p);
    fetch(c, out);
  });
}

int rbg_bin_graph(rbg_ctx *c, const rbg_params *p, const char *seqcat, const int64_t *offsets,
                  int64_t n, const float *depth, int32_t S, rbg_graph *out) {
  return guarded(c, [&] {
    validate(p);
    stage_sketch_chunked(c, p, seqcat, offsets, n, depth, S);
    run_graph(c, p);
    fetch(c, out);
  });
}

int rbg_bin_graph_sharded(rbg_ctx *c, const rbg_params *p, const rbg_shard *sh,
                          const char *seqcat, const int64_t *offsets, int64_t n_local,
                          const float *depth, int32_t S, rbg_graph *out) {
  return guarded(c, [&] {
    validate(p);
    if (!out) throw Error(RBG_ERR_ARG, "out is null");
    bin_graph_sharded(c, p, sh, seqcat, offsets, n_local, depth, S, out);
  });
}

int rbg_stage(rbg_ctx *c, const char *seqcat, const int64_t *offsets, int64_t n,
              const float *depth, int32_t S) {
  return guarded(c, [&] {
    stage(c, seqcat, offsets, n, depth, S);
    CK(cudaStreamSynchronize(c->stream));
  });
}

int rbg_run_resident(rbg_ctx *c, const rbg_params *p, rbg_timing *t) {
  return guarded(c, [&] {
    validate(p);
    c->launches = 0;
    run_sketch(c, p, false);
    run_graph(c, p);
    CK(cudaStreamSynchronize(c->stream));
    if (t) {
      std::memset(t, 0, sizeof(*t));
      auto el = [&](int a, int b) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]);
        return ms;
      };
      t->pack_ms = el(0, 1);
      t->count_ms = el(1, 2);
      t->sketch_ms = el(2, 3);
      {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev_a0, c->ev_a1);
        t->unit_ms = ms;
      }
      t->b0_ms = el(4, 5);
      t->allpairs_ms = el(5, 6);
      t->finalize_ms = el(6, 7);
      t->emit_ms = el(7, 8);
      t->weight_ms = el(8, 9);
      t->total_ms = el(0, 9);
      unsigned long long st[2] = {0, 0};
      CK(cudaMemcpy(st, c->stats.p, sizeof(st), cudaMemcpyDeviceToHost));
      t->pairs_prefiltered = (int64_t)st[0];
      t->pairs_compared = (int64_t)st[1];
      t->kernel_launches = c->launches;
    }
  });
}

int rbg_fetch_graph(rbg_ctx *c, rbg_graph *out) {
  return guarded(c, [&] { fetch(c, out); });
}

int rbg_pmh_stream_tables(int32_t k, int32_t m, uint64_t seed, int32_t contract, int32_t *n_elems,
                          int32_t *codes, double *U, uint32_t *W32) {
  if (k < 1 || k > 4 || m < 2 || m > kMaxM || !n_elems) return RBG_ERR_ARG;
  try {
    auto t = pmh_tables(k, m, seed, contract != 0);
    *n_elems = t->n_elems;
    if (codes) std::copy(t->canon_codes.begin(), t->canon_codes.end(), codes);
    if (U) std::copy(t->U.begin(), t->U.end(), U);
    if (W32) std::copy(t->W32.begin(), t->W32.end(), W32);
    return RBG_OK;
  } catch (...) {
    return RBG_ERR_NOMEM;
  }
}

// ── ProbMinHash4 rows and queries ──────────────────────────────────────────
// getWinners() / getRegisters() of the sketch build_pmh_winners makes per
// contig (src/rabbitbin.cpp:1436-1589: ProbMinHash4(m, k, seed) with one
// addHash per canonical k-mer), for n contigs.
int rbg_build_pmh_sketches(rbg_ctx *c, const rbg_params *p, const char *seqcat,
                           const int64_t *offsets, int64_t n, uint64_t *out_winners64,
                           double *out_registers) {
  return guarded(c, [&] {
    validate(p);
    if (p->oph_k > 0) throw Error(RBG_ERR_ARG, "ProbMinHash sketches need oph_k = 0");
    if (n > 0 && !out_winners64 && !out_registers) throw Error(RBG_ERR_ARG, "null outputs");
    stage(c, seqcat, offsets, n, nullptr, 0);
    const int m = p->m;
    c->tmp.ensure(std::max<size_t>((size_t)n * m, 16));
    run_sketch(c, p, false, c->tmp.as<uint8_t>());
    c->prep_done = false;
    Tables &T = tables_for(c, p);
    if (!T.rows_ready) {                 // winner states and U by element, once per table
      const PmhTables &t = *T.t;
      const size_t EM = (size_t)t.n_elems * t.m;
      T.W64.ensure(EM * sizeof(uint64_t));
      T.U.ensure(EM * sizeof(double));
      CK(cudaMemcpyAsync(T.W64.p, t.W64.data(), EM * sizeof(uint64_t), cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaMemcpyAsync(T.U.p, t.U.data(), EM * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      T.rows_ready = true;
    }
    if (n) {
      const size_t cells = (size_t)n * m;
      c->qa.ensure(cells * sizeof(uint64_t) * (out_winners64 && out_registers ? 2 : 1));
      uint64_t *dw = out_winners64 ? c->qa.as<uint64_t>() : nullptr;
      double *dr = out_registers ? (double *)(c->qa.as<uint64_t>() + (dw ? cells : 0)) : nullptr;
      launch_pmh_rows(c->tmp.as<uint8_t>(), c->elem_winv.as<double>(), n, m, T.t->n_elems,
                      T.W64.as<uint64_t>(), T.U.as<double>(), dw, dr, c->stream);
      CK(cudaGetLastError());
      if (dw) CK(cudaMemcpyAsync(out_winners64, dw, cells * 8, cudaMemcpyDeviceToHost, c->stream));
      if (dr) CK(cudaMemcpyAsync(out_registers, dr, cells * 8, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
  });
}

// Value of a comparison for every register-match count 0..m, with the
// reference's formulas (src/probmh.cpp:1325-1414) on the host's libm.
static std::vector<double> pmh_metric_table(int metric, int m, int kmer_size) {
  std::vector<double> t((size_t)m + 1);
  for (int c = 0; c <= m; ++c) {
    const double j = static_cast<double>(c) / static_cast<double>(m);
    double v = j;
    if (metric == RBG_PMH_DISTANCE) {
      if (j <= 0.0) v = std::numeric_limits<double>::infinity();
      else if (j >= 1.0) v = 0.0;
      else v = -std::log(2.0 * j / (1.0 + j)) / static_cast<double>(kmer_size);
    } else if (metric == RBG_PMH_ANI) {
      if (j <= 0.0) v = 0.0;
      else if (j >= 1.0) v = 1.0;
      else v = std::pow(2.0 * j / (1.0 + j), 1.0 / static_cast<double>(kmer_size));
    }
    t[c] = v;
  }
  return t;
}

int rbg_pmh_compare(rbg_ctx *c, int32_t metric, int32_t m, int32_t kmer_size, const void *A,
                    int64_t na, const void *B, int64_t nb, double *out) {
  return guarded(c, [&] {
    if (metric < RBG_PMH_JACCARD_WEIGHTED || metric > RBG_PMH_ANI)
      throw Error(RBG_ERR_ARG, "unknown ProbMinHash metric");
    if (m < 2 || m > kMaxM || na < 0 || nb < 0 || kmer_size < 1)
      throw Error(RBG_ERR_ARG, "m, row counts or k-mer size out of range");
    if (na == 0 || nb == 0) return;
    if (!A || !B || !out) throw Error(RBG_ERR_ARG, "null argument");
    const std::vector<double> tab = pmh_metric_table(metric, m, kmer_size);
    c->qt.ensure(tab.size() * sizeof(double));
    CK(cudaMemcpyAsync(c->qt.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    const size_t rowb = (size_t)m * 8;
    c->qb.ensure((size_t)nb * rowb);
    CK(cudaMemcpyAsync(c->qb.p, B, (size_t)nb * rowb, cudaMemcpyHostToDevice, c->stream));
    // A in blocks of rows whose outputs stay within 1 GiB (and the grid's y limit)
    int64_t blk = std::max<int64_t>(32, std::min<int64_t>(((int64_t)1 << 27) / nb, 65535 * 32));
    blk = std::min(blk, na);
    c->qa.ensure((size_t)blk * rowb);
    c->qo.ensure((size_t)blk * nb * sizeof(double));
    const bool regs = metric != RBG_PMH_JACCARD_WEIGHTED;
    for (int64_t a0 = 0; a0 < na; a0 += blk) {
      const int64_t ra = std::min(blk, na - a0);
      CK(cudaMemcpyAsync(c->qa.p, (const char *)A + (size_t)a0 * rowb, (size_t)ra * rowb,
                         cudaMemcpyHostToDevice, c->stream));
      launch_pmh_compare(c->qa.as<uint64_t>(), ra, c->qb.as<uint64_t>(), nb, m, regs,
                         c->qt.as<double>(), c->qo.as<double>(), c->stream);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(out + (size_t)a0 * nb, c->qo.p, (size_t)ra * nb * sizeof(double),
                         cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
  });
}

int rbg_pmh_merge_registers(rbg_ctx *c, const double *A, const double *B, int64_t n, int32_t m,
                            double *out) {
  return guarded(c, [&] {
    if (n < 0 || m < 2 || m > kMaxM) throw Error(RBG_ERR_ARG, "row count or m out of range");
    if (n == 0) return;
    if (!A || !B || !out) throw Error(RBG_ERR_ARG, "null argument");
    const size_t bytes = (size_t)n * m * sizeof(double);
    c->qa.ensure(bytes);
    c->qb.ensure(bytes);
    c->qo.ensure(bytes);
    CK(cudaMemcpyAsync(c->qa.p, A, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->qb.p, B, bytes, cudaMemcpyHostToDevice, c->stream));
    launch_pmh_merge(c->qa.as<double>(), c->qb.as<double>(), (int64_t)n * m, c->qo.as<double>(),
                     c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, c->qo.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int rbg_free_graph(rbg_graph *g) {
  if (!g) return RBG_ERR_ARG;
  if (!(g->from && pinned_pool().give(g->from))) {     // one pinned block, or four mallocs
    free(g->from);
    free(g->to);
    free(g->scomp);
    free(g->score);
  }
  g->from = g->to = nullptr;
  g->scomp = g->score = nullptr;
  g->n_edges = 0;
  return RBG_OK;
}

}  // extern "C"
