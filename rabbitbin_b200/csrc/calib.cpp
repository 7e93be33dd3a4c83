// Host steps of the graph stage that are sequential by definition: the
// rand()-driven cutoff calibration and the mt19937_64 draws of the b0 pairs;
// plus parameter validation and the device upload of the sketch tables.
#include <algorithm>
#include <cstring>
#include <list>
#include <random>

#include "engine_internal.h"

namespace rbg {

namespace {

// calib_converge (src/impl/rb_graph.cpp:390-415): walk the cutoff p (x1000)
// down in rand()-sized steps until the connected fraction reaches coverage.
// Every value is val[c] for a key c in 0..m with val non-decreasing in c, so
// the number of values >= cutoff is a suffix sum of the key histogram (the
// same counts a sorted copy gives, and the same rand() calls).
size_t converge_hist(const std::vector<int64_t> &hist, const std::vector<double> &val,
                     int64_t n, double coverage, CRand &rnd) {
  const size_t K = val.size();
  std::vector<int64_t> suffix(K + 1, 0);
  for (size_t c = K; c-- > 0;) suffix[c] = suffix[c + 1] + hist[c];
  size_t p = 999, pp = 1000;
  double cov = 0, pcov = 0;
  for (; p > 50;) {
    const double cutoff = (double)p / 1000.;
    const size_t c0 = (size_t)(std::lower_bound(val.begin(), val.end(), cutoff) - val.begin());
    const int64_t on = suffix[c0];
    cov = (double)on / (double)n;
    if (cov >= coverage) {
      if (cov - coverage > coverage - pcov) { p = pp; cov = pcov; }
      break;
    }
    pp = p;
    pcov = cov;
    if (p > 990) p -= rnd() % 3 + 1;
    else if (p > 900) p -= rnd() % 3 + 3;
    else p -= rnd() % 3 + 9;
  }
  return p;
}

// random_unique (src/rabbitbin.h:330-341), a partial Fisher-Yates driven by
// rand(): the first `count` entries it leaves in iota(n), without
// materialising the n-entry vector (positions touched are tracked lazily).
// `val`/`stamp` are scratch of n entries reused across calls (stamp marks the
// positions this call has written).
void rand_prefix_of_iota(size_t n, size_t count, std::vector<size_t> &val,
                         std::vector<uint32_t> &stamp, uint32_t cur, CRand &rnd,
                         std::vector<size_t> &out) {
  auto at = [&](size_t i) { return stamp[i] == cur ? val[i] : i; };
  auto put = [&](size_t i, size_t v) { val[i] = v; stamp[i] = cur; };
  out.resize(count);
  size_t left = n;
  for (size_t b = 0; b < count; ++b, --left) {
    const size_t r = b + (size_t)rnd() % left;
    const size_t vb = at(b), vr = at(r);
    put(r, vb);
    put(b, vr);
    out[b] = vr;
  }
}

}  // namespace

double calibrate_cutoff(const uint32_t *maxc, int64_t n, CalibMode mode, int m,
                        const std::vector<double> &sv_d, const std::vector<float> &sv_f,
                        double coverage, unsigned seed) {
  CRand rnd(seed);
  if (mode == CalibMode::all) {
    // random_unique over all n contigs: only its rand() calls matter here,
    // the maxima are counted, not ordered
    for (int64_t left = n; left > 0; --left) (void)(rnd() % left);
    std::vector<int64_t> hist(m + 1, 0);
    for (int64_t i = 0; i < n; ++i) ++hist[maxc[i]];
    return (double)converge_hist(hist, sv_d, n, coverage, rnd);
  }
  const size_t NR = 10, SAMP = 2500;
  std::vector<std::vector<size_t>> idxs(NR);
  std::vector<size_t> val((size_t)n);
  std::vector<uint32_t> stamp((size_t)n, 0);
  for (size_t r = 0; r < NR; ++r)
    rand_prefix_of_iota((size_t)n, SAMP, val, stamp, (uint32_t)(r + 1), rnd, idxs[r]);
  if (mode == CalibMode::samples_all) {
    // every (round, slot) holds its contig's maximum over all others, as a
    // double similarity (Similarity); each round converges on its own
    std::vector<int64_t> hist(m + 1);
    double sum_p = 0;
    for (size_t r = 0; r < NR; ++r) {
      std::fill(hist.begin(), hist.end(), 0);
      for (size_t li = 0; li < SAMP; ++li) ++hist[maxc[idxs[r][li]]];
      double mp = (double)converge_hist(hist, sv_d, (int64_t)SAMP, coverage, rnd);
      if (mp < 51.0) mp = 50.0;
      sum_p += mp;
      if (r == 1 && sum_p / 2 < 51.0) return 50.0;
    }
    return sum_p / (double)NR;
  }
  // each sampled contig feeds the slot of the first round that drew it; a
  // slot holds sv_f of its maximum count (sv_f is non-decreasing, sv_f[0] = 0)
  std::vector<int8_t> sround((size_t)n, -1);
  std::vector<uint32_t> slocal((size_t)n, 0);
  for (int r = (int)NR - 1; r >= 0; --r)
    for (size_t li = 0; li < SAMP; ++li) {
      sround[idxs[r][li]] = (int8_t)r;
      slocal[idxs[r][li]] = (uint32_t)li;
    }
  std::vector<std::vector<uint32_t>> key(NR, std::vector<uint32_t>(SAMP, 0));
  for (int64_t ci = 0; ci < n; ++ci)
    if (sround[ci] >= 0) {
      uint32_t &slot = key[sround[ci]][slocal[ci]];
      slot = std::max(slot, maxc[ci]);
    }
  std::vector<double> valf(m + 1);
  for (int c = 0; c <= m; ++c) valf[c] = (double)sv_f[c];
  double sum_p = 0;
  std::vector<int64_t> hist(m + 1);
  for (size_t r = 0; r < NR; ++r) {
    std::fill(hist.begin(), hist.end(), 0);
    for (size_t li = 0; li < SAMP; ++li) ++hist[key[r][li]];
    double mp = (double)converge_hist(hist, valf, (int64_t)SAMP, coverage, rnd);
    if (mp < 51.0) mp = 50.0;
    sum_p += mp;
    if (r == 1 && sum_p / 2 < 51.0) { sum_p = 500.0; break; }
  }
  return sum_p / (double)NR;
}

std::shared_ptr<const std::vector<int32_t>> b0_pairs(int64_t n) {
  // a small cache: batches see the same contig counts repeatedly
  static std::mutex mu;
  static std::list<std::pair<int64_t, std::shared_ptr<const std::vector<int32_t>>>> lru;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = lru.begin(); it != lru.end(); ++it)
      if (it->first == n) {
        lru.splice(lru.begin(), lru, it);
        return lru.front().second;
      }
  }
  auto pr = std::make_shared<std::vector<int32_t>>();
  if (n >= 4) {
    const size_t NP = 30000;
    std::mt19937_64 rng(0x9E3779B97F4A7C15ULL);
    std::uniform_int_distribution<size_t> uni(0, (size_t)n - 1);
    pr->reserve(2 * NP);
    for (size_t s = 0; s < NP; ++s) {
      const size_t i = uni(rng), j = uni(rng);
      if (i == j) continue;
      pr->push_back((int32_t)i);
      pr->push_back((int32_t)j);
    }
  }
  std::lock_guard<std::mutex> lk(mu);
  lru.emplace_front(n, pr);
  if (lru.size() > 256) lru.pop_back();
  return pr;
}

void validate_params(const rbg_params *p) {
  if (!p) throw Error(RBG_ERR_ARG, "null params");
  if (p->k < 1 || p->k > 4) throw Error(RBG_ERR_UNSUPPORTED, "k must be in 1..4");
  if (p->m < 2 || p->m > kMaxM) throw Error(RBG_ERR_ARG, "m must be in 2..4096");
  if (p->win_bits != 16 && p->win_bits != 32) throw Error(RBG_ERR_ARG, "win_bits must be 16 or 32");
  if (p->gc_norm < 0 || p->gc_norm > 2) throw Error(RBG_ERR_UNSUPPORTED, "gc_norm must be 0, 1 or 2");
  if (p->max_edges < 1 || p->max_edges > 448) throw Error(RBG_ERR_UNSUPPORTED, "max_edges must be in 1..448");
  if (!(p->coverage > 0.0 && p->coverage < 1.0)) throw Error(RBG_ERR_ARG, "coverage must be in (0,1)");
  if (p->oph_k < 0 || p->oph_k > 32) throw Error(RBG_ERR_ARG, "oph_k must be in 0..32");
  if (p->oph_k > 0 && (p->oph_bits < 1 || p->oph_bits > 7))
    throw Error(RBG_ERR_UNSUPPORTED, "oph_bits must be in 1..7");
  if (p->graph_index < 0 || p->graph_index > 1) throw Error(RBG_ERR_ARG, "graph_index must be 0 or 1");
  if (p->graph_index && (p->index_k < 1 || p->index_k > 32))
    throw Error(RBG_ERR_ARG, "index_k must be in 1..32");
  if (p->min_common < 0) throw Error(RBG_ERR_ARG, "min_common must be >= 0");
}

std::unique_ptr<Tables> make_tables(const rbg_params *p, cudaStream_t s) {
  auto T = std::make_unique<Tables>();
  T->t = pmh_tables(p->k, p->m, p->pmh_seed, p->fp_contract != 0);
  T->win_bits = p->win_bits;
  const PmhTables &t = *T->t;
  const size_t EM = (size_t)t.n_elems * t.m;
  T->order.ensure(EM * sizeof(RegOrder));
  T->UT.ensure(EM * sizeof(double));
  T->codeA.ensure(EM);
  T->W32.ensure(EM * sizeof(uint32_t));
  std::vector<int16_t> rk(t.rank_of_code.begin(), t.rank_of_code.end());
  T->rank.ensure(rk.size() * sizeof(int16_t));
  CK(cudaMemcpyAsync(T->order.p, t.order.data(), EM * sizeof(RegOrder), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(T->UT.p, t.UT.data(), EM * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(T->codeA.p, p->win_bits == 16 ? t.code16.data() : t.code32.data(), EM,
                     cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(T->W32.p, t.W32.data(), EM * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(T->rank.p, rk.data(), rk.size() * sizeof(int16_t), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return T;
}

}  // namespace rbg
