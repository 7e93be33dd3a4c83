// Label propagation: host side of rbg_label_propagation and
// rbg_label_propagation_resident (the kernels are in kernels_lpa.cu).
//
// The call builds the incidence lists on the device, takes the node order from
// the reference's generator (std::shuffle of 0..n-1 with
// std::default_random_engine(seed), src/rabbitbin.cpp:5643-5645, the same
// libstdc++ code on the host), and runs one sweep launch per round until a
// round changes no label (src/impl/rb_cluster.cpp:584-590, :711-714).  A round
// reads back two counters; nothing else crosses PCIe until the labels do.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "engine_internal.h"

using namespace rbg;

namespace {

// RABBIT_LPA_SCORE as the reference parses it (rb_cluster.cpp:41-50).
int rule_from_env() {
  const char *e = getenv("RABBIT_LPA_SCORE");
  if (!e || !*e) return RBG_LPA_FISHER;
  if (!std::strcmp(e, "sum")) return RBG_LPA_SUM;
  if (!std::strcmp(e, "mean")) return RBG_LPA_MEAN;
  if (!std::strcmp(e, "max")) return RBG_LPA_MAX;
  if (!std::strcmp(e, "logsum")) return RBG_LPA_LOGSUM;
  if (!std::strcmp(e, "tail")) return RBG_LPA_TAIL;
  return RBG_LPA_FISHER;
}

// Device-resident edge list the propagation runs on.
struct EdgeView {
  const uint32_t *from, *to;
  const float *score;
  int64_t E;
};

// Node order: the caller's permutation (checked) or the reference's shuffle.
void node_order(const rbg_lpa_params *lp, int64_t n, uint32_t *out) {
  if (lp->node_order) {
    std::vector<uint8_t> seen((size_t)n, 0);
    for (int64_t i = 0; i < n; ++i) {
      const uint32_t v = lp->node_order[i];
      if ((int64_t)v >= n || seen[v]) throw Error(RBG_ERR_ARG, "node_order is not a permutation of 0..n-1");
      seen[v] = 1;
      out[i] = v;
    }
    return;
  }
  // the reference shuffles a std::vector<size_t> (the element type does not
  // change the draws, but keep it identical)
  std::vector<size_t> ord((size_t)n);
  std::iota(ord.begin(), ord.end(), (size_t)0);
  std::shuffle(ord.begin(), ord.end(), std::default_random_engine((unsigned long long)lp->seed));
  for (int64_t i = 0; i < n; ++i) out[i] = (uint32_t)ord[(size_t)i];
}

void check_rule(const rbg_lpa_params *lp) {
  if (lp->score_rule < RBG_LPA_FISHER || lp->score_rule > RBG_LPA_MAX)
    throw Error(RBG_ERR_ARG, "score_rule out of range");
}

// Runs the propagation on a device edge list; labels into membership (host).
void propagate(rbg_ctx *c, const rbg_lpa_params *lp, int64_t n, const EdgeView &ev,
               uint32_t *membership, rbg_lpa_stats *stats) {
  cudaStream_t s = c->stream;
  if (!c->lpa) c->lpa.reset(new LpaBufs());
  LpaBufs &B = *c->lpa;
  const int64_t E = ev.E;
  rbg_lpa_stats st;
  std::memset(&st, 0, sizeof(st));

  // misc: [0] edge error, [1] sweep error, [2..3] max degree (int64), [4] claim,
  // [5] spill blocks used, [8..11] counts (two u64)
  B.misc.ensure(64);
  int *misc = B.misc.as<int>();
  B.pin.ensure(64);
  volatile int *pin = B.pin.as<int>();
  CK(cudaMemsetAsync(B.misc.p, 0, 64, s));

  cudaEvent_t e0 = c->ev[0], e1 = c->ev[1], e2 = c->ev[2];
  CK(cudaEventRecord(e0, s));
  // ── incidence lists ──
  B.deg.ensure((size_t)std::max<int64_t>(n, 1) * 4);
  B.off.ensure((size_t)(n + 1) * 8);
  B.q.ensure((size_t)std::max<int64_t>(E, 1) * 4);
  CK(cudaMemsetAsync(B.deg.p, 0, (size_t)n * 4, s));
  launch_lpa_edges(ev.from, ev.to, ev.score, E, n, lp->score_rule, B.q.as<float>(),
                   B.deg.as<uint32_t>(), misc, s);
  launch_lpa_offsets(B.deg.as<uint32_t>(), n, B.off.as<int64_t>(), (int64_t *)(misc + 2), s);
  CK(cudaMemcpyAsync((void *)pin, misc, 16, cudaMemcpyDeviceToHost, s));
  int64_t arcs = 0;
  CK(cudaMemcpyAsync(B.pin.as<char>() + 16, B.off.as<int64_t>() + n, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (pin[0] == 1) throw Error(RBG_ERR_ARG, "edgeScore must be non-negative");
  if (pin[0] == 2) throw Error(RBG_ERR_ARG, "an edge endpoint is not below n_nodes");
  int64_t maxdeg = 0;
  std::memcpy(&maxdeg, (const char *)pin + 8, 8);
  std::memcpy(&arcs, (const char *)pin + 16, 8);
  st.arcs = arcs;

  const size_t a1 = (size_t)std::max<int64_t>(arcs, 1);
  B.key.ensure(a1 * 8);
  B.nbr.ensure(a1 * 4);
  B.w.ensure(a1 * 4);
  B.fill.ensure((size_t)std::max<int64_t>(n, 1) * 4);
  CK(cudaMemsetAsync(B.fill.p, 0, (size_t)n * 4, s));
  launch_lpa_scatter(ev.from, ev.to, ev.score, E, n, B.off.as<int64_t>(), B.fill.as<uint32_t>(),
                     B.key.as<uint64_t>(), s);
  launch_lpa_sort(B.off.as<int64_t>(), n, B.key.as<uint64_t>(), B.q.as<float>(),
                  B.nbr.as<uint32_t>(), B.w.as<float>(), s);
  CK(cudaEventRecord(e1, s));

  // ── sweep state ──
  const size_t n1 = (size_t)std::max<int64_t>(n, 1);
  B.order_pin.ensure(n1 * 4);
  node_order(lp, n, B.order_pin.as<uint32_t>());
  B.order.ensure(n1 * 4);
  CK(cudaMemcpyAsync(B.order.p, B.order_pin.p, (size_t)n * 4, cudaMemcpyHostToDevice, s));
  B.pos.ensure(n1 * 4);
  B.label.ensure(n1 * 4);
  B.act0.ensure(n1);
  B.act1.ensure(n1);
  B.frozen.ensure(n1);
  B.done.ensure(n1 * 4);
  B.prop.ensure(n1 * 4);
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int warps = lpa_sweep_warps(sms);
  int gslots = 0;
  if (maxdeg > lpa_table_max_deg()) {
    gslots = 1024;
    while ((int64_t)gslots * 3 < maxdeg * 4) gslots <<= 1;
    // keep the per-warp tables within 4 GiB (fewer sweep warps otherwise)
    const int64_t per = (int64_t)gslots * 20;
    const int64_t cap = ((int64_t)4 << 30) / per;
    if (cap < warps) warps = (int)std::max<int64_t>(8, cap / 8 * 8);
    B.gtab.ensure((size_t)warps * (size_t)per);
  }
  const int vb = lpa_visit_block();
  uint32_t vcap = (uint32_t)std::max<int64_t>(n / 4, 1024);

  LpaSweepArgs a;
  a.n = n;
  a.off = B.off.as<int64_t>();
  a.nbr = B.nbr.as<uint32_t>();
  a.w = B.w.as<float>();
  a.order = B.order.as<uint32_t>();
  a.pos = B.pos.as<uint32_t>();
  a.label = B.label.as<uint32_t>();
  a.frozen = B.frozen.as<uint8_t>();
  a.done = B.done.as<uint32_t>();
  a.prop = B.prop.as<uint32_t>();
  a.vpool_used = (uint32_t *)(misc + 5);
  a.claim = (uint32_t *)(misc + 4);
  a.counts = (unsigned long long *)(misc + 8);
  a.gtab = gslots ? B.gtab.as<uint32_t>() : nullptr;
  a.gtab_slots = gslots;
  a.rule = lp->score_rule;
  a.err = misc + 1;

  float sweep_ms = 0.f;
  for (int attempt = 0;; ++attempt) {         // reruns only when the visited-set pool ran out
    B.vlab.ensure(((size_t)n + vcap) * (size_t)vb * 4);
    B.vcnt.ensure(((size_t)n + vcap) * 4);
    B.vnext.ensure(((size_t)n + vcap) * 4);
    a.vlab = B.vlab.as<uint32_t>();
    a.vcnt = B.vcnt.as<uint32_t>();
    a.vnext = B.vnext.as<uint32_t>();
    a.vpool_cap = vcap;
    uint8_t *act = B.act0.as<uint8_t>(), *nxt = B.act1.as<uint8_t>();
    CK(cudaMemsetAsync(misc + 1, 0, 4, s));
    CK(cudaMemsetAsync(misc + 5, 0, 4, s));
    launch_lpa_init(a.order, n, B.pos.as<uint32_t>(), a.label, act, nxt, a.frozen, a.done, a.vcnt,
                    a.vnext, s);
    if (attempt == 0) {
      B.early.ensure(a1);
      B.rec.ensure(n1 * 16);
      launch_lpa_early(a.off, a.nbr, a.pos, n, B.early.as<uint8_t>(), B.rec.as<uint4>(), s);
      a.early = B.early.as<uint8_t>();
      a.rec = B.rec.as<uint4>();
    }
    st.rounds = 0;
    st.changes = 0;
    st.frozen = 0;
    bool pool_out = false;
    const bool trace = getenv("RB_LPA_TRACE") != nullptr;
    auto tr0 = std::chrono::steady_clock::now();
    for (uint32_t round = 1;; ++round) {
      if (lp->max_rounds > 0 && (int)round > lp->max_rounds)
        throw Error(RBG_ERR_TIMEOUT, "label propagation did not converge within max_rounds");
      a.round = round;
      a.active = act;
      a.next_active = nxt;
      CK(cudaMemsetAsync(misc + 4, 0, 4, s));
      CK(cudaMemsetAsync(misc + 8, 0, 16, s));
      CK(cudaMemsetAsync(nxt, 0, (size_t)n, s));            // marks for the next round
      launch_lpa_round(a, lp->synchronous, warps, s);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync((void *)pin, misc, 64, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      st.rounds = (int)round;
      unsigned long long cnt[2];
      std::memcpy(cnt, (const char *)pin + 32, 16);
      if (trace) {                                   // RB_LPA_TRACE, rb_cluster.cpp:711-713
        const auto t1 = std::chrono::steady_clock::now();
        fprintf(stderr, "[LPA] round=%u changed=%llu frozen=%llu ms=%.3f\n", round, cnt[0], cnt[1],
                std::chrono::duration<double, std::milli>(t1 - tr0).count());
        tr0 = t1;
      }
      st.changes += (int64_t)cnt[0];
      st.frozen += (int64_t)cnt[1];
      const int err = pin[1];
      if (err == RBG_ERR_NOMEM) {
        pool_out = true;
        break;
      }
      if (err == RBG_ERR_TIMEOUT)
        throw Error(RBG_ERR_TIMEOUT, "label propagation: a bounded wait for an earlier node ran out");
      if (err != 0) throw Error(RBG_ERR_CUDA, "label propagation: device error");
      if (cnt[0] == 0) break;
      std::swap(act, nxt);
    }
    if (!pool_out) break;
    if (attempt >= 4) throw Error(RBG_ERR_NOMEM, "label propagation: visited sets outgrew their pool");
    vcap *= 4;
  }
  CK(cudaEventRecord(e2, s));
  CK(cudaMemcpyAsync(membership, a.label, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float inc_ms = 0.f;
  cudaEventElapsedTime(&inc_ms, e0, e1);
  cudaEventElapsedTime(&sweep_ms, e1, e2);
  st.incidence_ms = inc_ms;
  st.sweep_ms = sweep_ms;
  if (stats) *stats = st;
}

}  // namespace

extern "C" {

int rbg_default_lpa_params(rbg_lpa_params *lp) {
  if (!lp) return RBG_ERR_ARG;
  std::memset(lp, 0, sizeof(*lp));
  lp->seed = 1;
  lp->score_rule = rule_from_env();
  lp->synchronous = getenv("RABBIT_PAR_LPA") != nullptr;   // rb_cluster.cpp:490
  return RBG_OK;
}

int rbg_label_propagation(rbg_ctx *c, const rbg_lpa_params *lp, int64_t n, int64_t E,
                          const uint32_t *from, const uint32_t *to, const float *score,
                          uint32_t *membership, rbg_lpa_stats *stats) {
  return guarded(c, [&] {
    if (!lp || n < 0 || E < 0 || (n > 0 && !membership) || (E > 0 && (!from || !to || !score)))
      throw Error(RBG_ERR_ARG, "null or negative argument");
    if (n >= (int64_t)0xFFFFFFFF || E >= (int64_t)0xFFFFFFFF)
      throw Error(RBG_ERR_ARG, "node or edge count beyond the 32-bit ids of the reference graph");
    check_rule(lp);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    for (int64_t i = 0; i < n; ++i) membership[i] = (uint32_t)i;
    if (n == 0 || E == 0) return;                       // rb_cluster.cpp:381-385
    if (!c->lpa) c->lpa.reset(new LpaBufs());
    LpaBufs &B = *c->lpa;
    cudaStream_t s = c->stream;
    B.from.ensure((size_t)E * 4);
    B.to.ensure((size_t)E * 4);
    B.score.ensure((size_t)E * 4);
    CK(cudaMemcpyAsync(B.from.p, from, (size_t)E * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.to.p, to, (size_t)E * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.score.p, score, (size_t)E * 4, cudaMemcpyHostToDevice, s));
    propagate(c, lp, n, EdgeView{B.from.as<uint32_t>(), B.to.as<uint32_t>(), B.score.as<float>(), E},
              membership, stats);
  });
}

int rbg_label_propagation_resident(rbg_ctx *c, const rbg_lpa_params *lp, uint32_t *membership,
                                   rbg_lpa_stats *stats) {
  return guarded(c, [&] {
    if (!lp) throw Error(RBG_ERR_ARG, "null parameters");
    if (!c->graph_ready) throw Error(RBG_ERR_ARG, "no graph has been built on this context");
    check_rule(lp);
    const int64_t n = c->n, E = c->n_edges;
    if (n > 0 && !membership) throw Error(RBG_ERR_ARG, "null membership");
    if (stats) std::memset(stats, 0, sizeof(*stats));
    for (int64_t i = 0; i < n; ++i) membership[i] = (uint32_t)i;
    if (n == 0 || E == 0) return;
    propagate(c, lp, n, EdgeView{c->e_from.as<uint32_t>(), c->e_to.as<uint32_t>(),
                                 c->e_score.as<float>(), E},
              membership, stats);
  });
}

}  // extern "C"
