// CPU restatement of RabbitBin's graph-construction hot path.
//
// TEST INFRASTRUCTURE ONLY: tests/, the smoke check and bench.py's CPU-baseline
// leg load this library as the checker; the product never calls it.
//
// It restates, in plain sequential code, what the reference computes:
//   sketch      build_pmh_winners            src/rabbitbin.cpp:1436-1589
//               ProbMinHash4::addHashFromRng src/probmh.cpp:634-686 (+ :60-87,
//               :319-357, :410-479, :506-572)
//   pack        fold_win16 + pack loop       src/rabbitbin.cpp:249-253, :4934-4952
//   b0          estimate_pmh_baseline        src/rabbitbin.cpp:1340-1369
//   similarity  pmh_match_count16 / pmh_sv_from_count  src/rabbitbin.cpp:1261-1305
//   ranks/unit  src/ranker.h:55-66, src/rabbitbin.cpp:4867-4874, :4972-4988
//   anynz       src/impl/rb_abundance.cpp:94-114
//   small N     calibrate_sim_cutoff + build_graph_allpairs src/impl/rb_graph.cpp:1362-1384, :7-72
//   large N     gen_fused_calib_graph        src/impl/rb_graph.cpp:501-1356
//   calibration calib_converge               src/impl/rb_graph.cpp:390-415
//   weights     depth_edge_term etc.         src/rabbitbin.cpp:685-970, :5482-5509
//   OPH metric  KmerSketch update/densify/buildSig  src/rabbit_sketch.h:197-281
//               (RABBIT_PMH=0; similarity jaccard_raw src/rabbitbin.cpp:1031-1135)
// Floating point follows the reference's release build on an AVX-512 host:
// compiled with -ffp-contract=off, with std::fma written where that build
// fuses (AVX-512 FMA intrinsics and GCC-contracted expressions).  The third
// party routines it relies on are the same as the reference's: glibc rand()/
// srand(), libm exp/log1p/expm1/sqrt and libstdc++ mt19937_64 +
// uniform_int_distribution + nth_element (GCC 13.3 / glibc 2.39 of this image).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <string>
#include <vector>
#include <omp.h>

namespace {

#include "../rabbitbin_b200/csrc/zig_tables.inc"

// ── RNG (wyrand) and hash ────────────────────────────────────────────────────
uint64_t fmix64(uint64_t x, uint64_t seed) {
  x ^= seed;
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}
uint64_t rng_next(uint64_t &s) {
  s += 0xa0761d6478bd642fULL;
  const unsigned __int128 p = (unsigned __int128)s * (s ^ 0xe7037ed1a0b428dbULL);
  return (uint64_t)(p >> 64) ^ (uint64_t)p;
}
double rng_unit(uint64_t &s) { return (double)(rng_next(s) >> 11) * (1.0 / 9007199254740992.0); }
uint32_t rng_below(uint32_t n, uint64_t &s) {
  for (;;) {
    const uint64_t x = rng_next(s) >> 32;
    const uint64_t mm = x * (uint64_t)n;
    const uint32_t lo = (uint32_t)mm;
    if (lo >= n || lo >= (uint32_t)(0u - n) % n) return (uint32_t)(mm >> 32);
  }
}

struct TedP { double b, gap, c1, c2, c3; };

void build_ted(int m, std::vector<TedP> &t, double &finv) {
  t.assign(m - 1, TedP{});
  const double f = std::log1p(1.0 / (double)(m - 1));
  finv = 1.0 / f;
  auto cst = [](double r, TedP &p) {
    p.c1 = (r != 0.0) ? std::expm1(r) / r : 1.0;
    p.c2 = (r != 0.0) ? -std::log1p(std::expm1(-r) * 0.5) / r : 0.5;
    p.c3 = (r != 0.0) ? -std::expm1(-r) / r : 1.0;
  };
  t[0].b = 1.0;
  t[0].gap = 1.0;
  cst(f, t[0]);
  double prev = f;
  for (int i = 1; i < m - 1; ++i) {
    const double b = std::log1p((double)(i + 1) / (double)(m - i - 1));
    t[i].b = b / f;
    t[i].gap = t[i].b - t[i - 1].b;
    cst(b - prev, t[i]);
    prev = b;
  }
}

double ted_sample(const TedP &p, uint64_t &s) {
  double x = rng_unit(s) * p.c1;
  if (x < 1.0) return x;
  for (;;) {
    x = rng_unit(s);
    if (x <= p.c2) return x;
    double y = rng_unit(s) * 0.5;
    if (y > 1.0 - x) { x = 1.0 - x; y = 1.0 - y; }
    if (x <= p.c3 * (1.0 - y)) return x;
    if (p.c1 * y <= 1.0 - x) return x;
  }
}

double zig_exp(uint64_t &s) {
  double shift = 0.0;
  for (;;) {
    const uint64_t bits = rng_next(s);
    const int i = (int)(bits & 0xFF);
    const double x = (double)(bits >> 11) * (1.0 / 9007199254740992.0) * kZigX[i];
    if (x < kZigX[i + 1]) return shift + x;
    if (i == 0) { shift += kZigX[1]; continue; }
    const double y01 = rng_unit(s);
    const double y = std::fma(y01, kZigY[i + 1] - kZigY[i], kZigY[i]);
    const double ub = std::fma(kZigX[i] - kZigX[i + 1], y01, -(kZigX[i] - x));
    const double lb = y - std::fma(kZigX[i + 1] - x, kZigY[i + 1], kZigY[i + 1]);
    if (ub < 0 && (lb < 0 || y < std::exp(-x))) return x + shift;
  }
}

// ── weighted ProbMinHash with a max tree over the registers ─────────────────
struct Sketch {
  int m;
  std::vector<TedP> ted;
  double finv;
  int leaves;
  std::vector<double> tree;     // max tree, registers at the leaves
  std::vector<uint64_t> win;
  std::vector<uint32_t> pval, pver;
  uint32_t ver = 0;

  explicit Sketch(int m_) : m(m_) {
    build_ted(m, ted, finv);
    leaves = 1;
    while (leaves < m) leaves <<= 1;
    pval.assign(m, 0);
    pver.assign(m, 0);
    clear();
  }
  void clear() {
    tree.assign(2 * leaves, -std::numeric_limits<double>::infinity());
    for (int r = 0; r < m; ++r) tree[leaves + r] = std::numeric_limits<double>::infinity();
    for (int q = leaves - 1; q >= 1; --q) tree[q] = std::max(tree[2 * q], tree[2 * q + 1]);
    win.assign(m, 0);
  }
  double top() const { return tree[1]; }
  void put(int r, double v) {
    int q = leaves + r;
    tree[q] = v;
    for (q >>= 1; q >= 1; q >>= 1) tree[q] = std::max(tree[2 * q], tree[2 * q + 1]);
  }
  uint32_t perm_next(uint32_t idx, uint64_t &s) {
    const uint32_t kk = idx + rng_below((uint32_t)m - idx, s);
    const uint32_t res = (pver[kk] == ver) ? pval[kk] : kk;
    const uint32_t mv = (pver[idx] == ver) ? pval[idx] : idx;
    pval[kk] = mv;
    pver[kk] = ver;
    return res;
  }
  void offer(int reg, double hv, uint64_t s) {
    if (hv < tree[leaves + reg]) { put(reg, hv); win[reg] = s; }
  }
  void add(uint64_t key, double w, uint64_t seed) {
    if (!(w > 0.0)) return;
    uint64_t s = fmix64(key, seed);
    const double winv = 1.0 / w;
    double h = (double)(s >> 11) * (1.0 / 9007199254740992.0) * ted[0].c1;
    if (!(h < 1.0)) h = ted_sample(ted[0], s);
    double hv = winv * h;
    if (!(hv < top())) return;
    ++ver;
    uint32_t steps = 0;
    for (int i = 1; hv < top(); ++i) {
      {
        const int reg = (int)perm_next(steps, s);   // advances s: the winner is the post-draw state
        offer(reg, hv, s);
      }
      if (++steps >= (uint32_t)m) break;
      if (!(winv * ted[i - 1].b < top())) break;
      if (i < m - 1) {
        const TedP &p = ted[i];
        hv = winv * std::fma(p.gap, ted_sample(p, s), ted[i - 1].b);
      } else {
        hv = winv * std::fma(finv, zig_exp(s), ted[m - 2].b);
        if (steps < (uint32_t)m && hv < top()) {
          const int reg = (int)perm_next(steps, s);
          offer(reg, hv, s);
        }
        break;
      }
    }
  }
};

// Canonical k-mer histogram + GC-normalised weights of one contig, then the
// sketch; writes folded 32-bit winners.
void contig_winners(const char *seq, size_t len, int k, int m, uint64_t seed, int gc_norm,
                    double cap, Sketch &sk, std::vector<uint64_t> &hist, uint32_t *out) {
  sk.clear();
  if (len >= (size_t)k && k >= 1 && k <= 8) {
    const size_t nb = (size_t)1 << (2 * k);
    hist.assign(nb, 0);
    const uint64_t mask = nb - 1;
    uint64_t f = 0, r = 0, bc[4] = {0, 0, 0, 0};
    uint64_t dn[4][4] = {};           // consecutive valid bases (prev, next), mode 2
    int run = 0, prevb = -1;
    size_t total = 0;
    for (size_t i = 0; i < len; ++i) {
      int b;
      switch (seq[i] | 0x20) {
        case 'a': b = 0; break;
        case 'c': b = 1; break;
        case 'g': b = 2; break;
        case 't': b = 3; break;
        default: b = -1;
      }
      if (b < 0) { run = 0; f = r = 0; prevb = -1; continue; }
      bc[b]++;
      if (prevb >= 0) dn[prevb][b]++;
      prevb = b;
      f = ((f << 2) | (uint64_t)b) & mask;
      r = (r >> 2) | ((uint64_t)(3 - b) << (2 * (k - 1)));
      if (++run >= k) { hist[f <= r ? f : r]++; total++; }
    }
    if (total) {
      const double inv = 1.0 / (double)total;
      const uint64_t vb = bc[0] + bc[1] + bc[2] + bc[3];
      double p[4];
      for (int b = 0; b < 4; ++b) p[b] = vb > 0 ? (double)bc[b] / (double)vb : 0.25;
      for (uint64_t v = 0; v < nb; ++v) {
        if (!hist[v]) continue;
        double w;
        if (gc_norm == 0) {
          w = (double)hist[v] * inv;
        } else if (gc_norm == 2) {
          // first-order Markov model (src/rabbitbin.cpp:1517-1554): base
          // frequencies with pseudocount 1, P(next | prev) with Laplace
          // pseudocount 1; bases[i] = (v >> 2i) & 3
          double pm[4], pc[4][4];
          for (int b = 0; b < 4; ++b)
            pm[b] = vb > 0 ? ((double)bc[b] + 1.0) / ((double)vb + 4.0) : 0.25;
          for (int x = 0; x < 4; ++x) {
            double rs = 4.0;
            for (int y = 0; y < 4; ++y) rs += (double)dn[x][y];
            for (int y = 0; y < 4; ++y) pc[x][y] = ((double)dn[x][y] + 1.0) / rs;
          }
          int bs[8];
          for (int q = 0; q < k; ++q) bs[q] = (int)((v >> (2 * q)) & 3);
          double pf = pm[bs[0]];
          for (int q = 1; q < k; ++q) pf *= pc[bs[q - 1]][bs[q]];
          double pr = pm[3 - bs[k - 1]];
          for (int q = 1; q < k; ++q) pr *= pc[3 - bs[k - q]][3 - bs[k - 1 - q]];
          const double ex = pf + pr;
          const double obs = (double)hist[v] * inv;
          w = (ex > 1e-16) ? std::min(obs / ex, cap) : 0.0;
        } else {
          double pf = 1.0, pr = 1.0;
          uint64_t code = v;
          for (int q = 0; q < k; ++q) {
            pf *= p[code & 3];
            pr *= p[3 - (code & 3)];
            code >>= 2;
          }
          const double ex = pf + pr;
          const double obs = (double)hist[v] * inv;
          w = (ex > 1e-14) ? std::min(obs / ex, cap) : 0.0;
        }
        if (w > 0.0) sk.add(v, w, seed);
      }
    }
  }
  for (int q = 0; q < m; ++q) out[q] = (uint32_t)(sk.win[q] ^ (sk.win[q] >> 32));
}

uint16_t fold16(uint32_t w) {
  if (!w) return 0;
  const uint16_t h = (uint16_t)(w ^ (w >> 16));
  return h ? h : 1;
}

// ── float orders of the AVX-512 build ────────────────────────────────────────
float reduce16(const float *v0) {
  float v[16];
  for (int l = 0; l < 16; ++l) v[l] = v0[l];
  for (int l = 0; l < 8; ++l) v[l] = v[l] + v[l + 8];
  for (int l = 0; l < 4; ++l) v[l] = v[l] + v[l + 4];
  return (v[0] + v[2]) + (v[1] + v[3]);
}

// unit_dot_f: 16-lane FMA accumulators, masked tail into acc0, tree reduce.
float unit_dot(const float *a, const float *b, int S) {
  float acc0[16] = {0}, acc1[16] = {0};
  int k = 0;
  for (; k + 32 <= S; k += 32)
    for (int l = 0; l < 16; ++l) {
      acc0[l] = std::fmaf(a[k + l], b[k + l], acc0[l]);
      acc1[l] = std::fmaf(a[k + 16 + l], b[k + 16 + l], acc1[l]);
    }
  for (; k + 16 <= S; k += 16)
    for (int l = 0; l < 16; ++l) acc0[l] = std::fmaf(a[k + l], b[k + l], acc0[l]);
  if (k < S)
    for (int l = 0; l < S - k; ++l) acc0[l] = std::fmaf(a[k + l], b[k + l], acc0[l]);
  if (S == 0) return 0.0f;
  float v[16];
  for (int l = 0; l < 16; ++l) v[l] = acc0[l] + acc1[l];
  return reduce16(v);
}

// depth_corr_fast: float blocks of 16, double tail.
double depth_corr(const float *a, const float *b, int S) {
  float acc0[16] = {0}, acc1[16] = {0};
  int k = 0;
  for (; k + 32 <= S; k += 32)
    for (int l = 0; l < 16; ++l) {
      acc0[l] = std::fmaf(a[k + l], b[k + l], acc0[l]);
      acc1[l] = std::fmaf(a[k + 16 + l], b[k + 16 + l], acc1[l]);
    }
  for (; k + 16 <= S; k += 16)
    for (int l = 0; l < 16; ++l) acc0[l] = std::fmaf(a[k + l], b[k + l], acc0[l]);
  double s = 0.0;
  if (k > 0) {
    float v[16];
    for (int l = 0; l < 16; ++l) v[l] = acc0[l] + acc1[l];
    s = (double)reduce16(v);
  }
  for (; k < S; ++k) s += (double)a[k] * (double)b[k];
  return s;
}

double depth_wjac(const float *a, const float *b, int S, const double *cn) {
  double mn = 0.0, mx = 0.0;
  for (int i = 0; i < S; ++i) {
    double x = a[i], y = b[i];
    if (cn) { x *= cn[i]; y *= cn[i]; }
    if (x < y) { mn += x; mx += y; } else { mn += y; mx += x; }
  }
  return mx <= 0.0 ? 0.0 : mn / mx;
}

void avg_ranks(const float *x, int S, float *out) {
  std::vector<int> o(S);
  std::iota(o.begin(), o.end(), 0);
  std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return x[a] < x[b]; });
  for (int c = 0; c < S;) {
    int reps = 1;
    while (c + reps < S && x[o[c]] == x[o[c + reps]]) ++reps;
    for (int q = 0; q < reps; ++q) out[o[c + q]] = (float)(2 * c + reps - 1) / 2 + 1;
    c += reps;
  }
}

size_t converge(const std::vector<double> &ms, double coverage) {
  size_t p = 999, pp = 1000;
  double pcov = 0.0;
  while (p > 50) {
    const double cut = (double)p / 1000.;
    size_t on = 0;
    for (double v : ms) on += (v >= cut);
    const double cov = (double)on / (double)ms.size();
    if (cov >= coverage) {
      if (cov - coverage > coverage - pcov) p = pp;
      break;
    }
    pp = p;
    pcov = cov;
    const int step = rand() % 3;
    p -= (p > 990) ? step + 1 : (p > 900) ? step + 3 : step + 9;
  }
  return p;
}

void pick_prefix(std::vector<size_t> &v, size_t cnt) {
  size_t left = v.size();
  for (size_t b = 0; b < cnt; ++b, --left) std::swap(v[b], v[b + (size_t)rand() % left]);
}

}  // namespace

extern "C" {

void orc_build_winners(const char *seqcat, const int64_t *offsets, int64_t n, int k,
                       uint32_t m, uint64_t seed, int gc_norm, double gc_cap, uint32_t *out32,
                       int nthreads) {
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    Sketch sk((int)m);
    std::vector<uint64_t> hist;
#pragma omp for schedule(dynamic, 4)
    for (int64_t r = 0; r < n; ++r)
      contig_winners(seqcat + offsets[r], (size_t)(offsets[r + 1] - offsets[r]), k, (int)m, seed,
                     gc_norm, gc_cap, sk, hist, out32 + (size_t)r * m);
  }
}

struct OrcParams {
  int64_t n;
  int32_t m, S, win_bits, max_edges, mutual, base_on, nthreads;
  uint32_t seed;
  int32_t force_path;
  double coverage, min_edge, w_comp, min_cv, neg_thr;
  int32_t depth_sim, depth_fuse, wjac_norm, no_abdfirst;
};

struct OrcOut {
  double b0, sim_cutoff;
  int64_t n_edges;
  uint32_t *from, *to;
  float *scomp, *score;
};

void orc_free(void *p) { free(p); }

int orc_run_graph(const OrcParams *P, const uint32_t *w32, const float *depth, float *unit_out,
                  OrcOut *out) {
  const int64_t n = P->n;
  const int m = P->m, S = P->S, K = P->max_edges;
  const int nth = P->nthreads > 0 ? P->nthreads : 1;
  // winner rows at the compared width
  std::vector<uint32_t> W((size_t)n * m);
  for (size_t q = 0; q < W.size(); ++q) W[q] = P->win_bits == 16 ? fold16(w32[q]) : w32[q];
  auto count = [&](int64_t i, int64_t j) {
    const uint32_t *a = &W[(size_t)i * m], *b = &W[(size_t)j * m];
    uint32_t c = 0;
    for (int q = 0; q < m; ++q) c += (a[q] != 0 && a[q] == b[q]);
    return c;
  };
  const double inv_m = 1.0 / (double)m;
  // b0
  double b0 = 0.0;
  if (P->base_on && n >= 4) {
    std::mt19937_64 g(0x9E3779B97F4A7C15ULL);
    std::uniform_int_distribution<size_t> u(0, (size_t)n - 1);
    std::vector<float> vals;
    for (int s = 0; s < 30000; ++s) {
      const size_t i = u(g), j = u(g);
      if (i == j) continue;
      vals.push_back((float)((double)count(i, j) * inv_m));
    }
    if (!vals.empty()) {
      std::nth_element(vals.begin(), vals.begin() + vals.size() / 2, vals.end());
      b0 = (double)vals[vals.size() / 2];
    }
  }
  const double i1mb0 = b0 < 1.0 ? 1.0 / (1.0 - b0) : 1.0;
  auto sim = [&](uint32_t c) {
    double j = (double)c * inv_m;
    if (P->base_on && b0 > 0.0 && b0 < 1.0) {
      j = (j - b0) * i1mb0;
      if (j < 0.0) j = 0.0;
    }
    if (j > 1.0 - 1e-6) j = 1.0 - 1e-6;
    return j;
  };
  // ranks, anynz, unit rows, column norms
  std::vector<float> rk((size_t)n * std::max(S, 1)), U((size_t)n * std::max(S, 1), 0.f);
  std::vector<uint8_t> nz(n, 1);
  for (int64_t r = 0; r < n; ++r) {
    const float *x = depth + (size_t)r * S;
    if (S > 1) avg_ranks(x, S, &rk[(size_t)r * S]);
    else if (S == 1) rk[r] = x[0];
    if (S > 0) {
      nz[r] = 0;
      for (int k = 0; k < S; ++k) if (rk[(size_t)r * S + k] > P->min_cv) nz[r] = 1;
    }
    if (S > 1) {
      double mean = 0;
      for (int k = 0; k < S; ++k) mean += rk[(size_t)r * S + k];
      mean /= (double)S;
      double ss = 0;
      for (int k = 0; k < S; ++k) { const double d = rk[(size_t)r * S + k] - mean; ss += d * d; }
      if (ss > 0.0) {
        const double inv = 1.0 / std::sqrt(ss);
        for (int k = 0; k < S; ++k) U[(size_t)r * S + k] = (float)((rk[(size_t)r * S + k] - mean) * inv);
      }
    }
  }
  if (unit_out && S > 1) std::copy(U.begin(), U.end(), unit_out);
  std::vector<double> cn;
  if (P->depth_sim >= 1 && S > 1 && P->wjac_norm) {
    cn.assign(S, 0.0);
    for (int i = 0; i < S; ++i) {
      double s = 0.0;
      for (int64_t r = 0; r < n; ++r) s += depth[(size_t)r * S + i];
      const double mean = s / (double)std::max<int64_t>(n, 1);
      cn[i] = mean > 1e-12 ? 1.0 / mean : 0.0;
    }
  }
  const double wc = P->w_comp < 0 ? (S <= 2 ? 1.0 : 0.0) : P->w_comp;
  const bool fused = P->force_path == 2 || (P->force_path == 0 && n > 25000);
  // per-row candidates (sv, id) and maxima
  std::vector<std::vector<std::pair<float, uint32_t>>> top(n);
  std::vector<uint32_t> maxc_all(n, 0), maxc_cand(n, 0);
  const bool abd = fused && !P->no_abdfirst && S > 1 && wc < 1.0 && wc < P->min_edge;
  const float abd_eps = (float)((abd ? (P->min_edge - wc) / (1.0 - wc) : -2.0) - 1e-4);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
  for (int64_t i = 0; i < n; ++i) {
    std::vector<std::pair<float, uint32_t>> c;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const bool isnz = nz[i] || nz[j];
      if (!fused) {
        const uint32_t cnt = count(i, j);
        maxc_all[i] = std::max(maxc_all[i], cnt);
        if (isnz) c.emplace_back((float)sim(cnt), (uint32_t)j);
      } else {
        if (!isnz) continue;
        if (abd && unit_dot(&U[(size_t)std::min(i, j) * S], &U[(size_t)std::max(i, j) * S], S) < abd_eps)
          continue;
        const uint32_t cnt = count(i, j);
        maxc_cand[i] = std::max(maxc_cand[i], cnt);
        c.emplace_back((float)sim(cnt), (uint32_t)j);
      }
    }
    auto better = [](const std::pair<float, uint32_t> &a, const std::pair<float, uint32_t> &b) {
      return a.first != b.first ? a.first > b.first : a.second < b.second;
    };
    const size_t keep = std::min<size_t>(c.size(), (size_t)K);
    std::partial_sort(c.begin(), c.begin() + keep, c.end(), better);
    c.resize(keep);
    top[i] = std::move(c);
  }
  // calibration
  srand(P->seed);
  double simCutoff;
  if (!fused) {
    std::vector<size_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    pick_prefix(idx, (size_t)n);
    std::vector<double> ms(n);
    for (int64_t i = 0; i < n; ++i) ms[i] = sim(maxc_all[idx[i]]);
    simCutoff = (double)converge(ms, P->coverage);
  } else {
    const int NR = 10, SP = 2500;
    std::vector<std::vector<size_t>> idx(NR, std::vector<size_t>(n));
    for (int r = 0; r < NR; ++r) {
      std::iota(idx[r].begin(), idx[r].end(), 0);
      pick_prefix(idx[r], SP);
    }
    std::vector<int> rr(n, -1);
    std::vector<int> ll(n, 0);
    for (int r = NR - 1; r >= 0; --r)
      for (int li = 0; li < SP; ++li) { rr[idx[r][li]] = r; ll[idx[r][li]] = li; }
    std::vector<std::vector<double>> ms(NR, std::vector<double>(SP, 0.0));
    for (int64_t c = 0; c < n; ++c)
      if (rr[c] >= 0) ms[rr[c]][ll[c]] = (double)(float)sim(maxc_cand[c]);
    double sp = 0;
    for (int r = 0; r < NR; ++r) {
      double p = (double)converge(ms[r], P->coverage);
      if (p < 51.0) p = 50.0;
      sp += p;
      if (r == 1 && sp / 2 < 51.0) { sp = 500.0; break; }
    }
    simCutoff = sp / NR;
  }
  const double cutoff = simCutoff / 1000.;
  // edges
  std::vector<std::vector<uint32_t>> kept(n);
  for (int64_t i = 0; i < n; ++i) {
    for (auto &e : top[i]) if ((double)e.first > cutoff) kept[i].push_back(e.second);
    std::sort(kept[i].begin(), kept[i].end());
  }
  std::vector<uint32_t> F, T;
  std::vector<float> SC, SW;
  for (int64_t i = 0; i < n; ++i) {
    std::vector<std::pair<uint32_t, float>> row;
    for (auto &e : top[i])
      if ((double)e.first > cutoff && e.second > (uint32_t)i) row.emplace_back(e.second, e.first);
    std::sort(row.begin(), row.end());
    for (auto &e : row) {
      if (fused && P->mutual &&
          !std::binary_search(kept[e.first].begin(), kept[e.first].end(), (uint32_t)i))
        continue;
      F.push_back((uint32_t)i);
      T.push_back(e.first);
      SC.push_back(e.second);
    }
  }
  // weights
  const size_t ne = F.size();
  SW.assign(ne, 0.f);
  for (size_t e = 0; e < ne; ++e) {
    const float sc = SC[e];
    if (S <= 0) { SW[e] = sc < P->min_edge ? 0.f : sc; continue; }
    if (S == 1) { SW[e] = sc; continue; }
    const size_t i = F[e], j = T[e];
    const double *cnp = cn.empty() ? nullptr : cn.data();
    bool ok = true;
    double dterm = 0.0;
    if (P->depth_sim == 1) {
      const double wj = depth_wjac(depth + i * S, depth + j * S, S, cnp);
      if (!std::isfinite(wj)) ok = false;
      else dterm = wj < 0 ? 0 : (wj > 1 ? 1 : wj);
    } else {
      const double corr = depth_corr(&U[i * S], &U[j * S], S);
      if (!std::isfinite(corr) || (P->neg_thr > -0.99 && corr < P->neg_thr)) ok = false;
      else {
        const double cp = corr < 0.0 ? 0.0 : corr;
        dterm = cp;
        if (P->depth_sim == 2) {
          double wj = depth_wjac(depth + i * S, depth + j * S, S, cnp);
          if (!std::isfinite(wj)) wj = 0.0;
          wj = wj < 0 ? 0 : (wj > 1 ? 1 : wj);
          dterm = P->depth_fuse == 1 ? std::min(cp, wj)
                : P->depth_fuse == 2 ? cp * wj : std::sqrt(cp * wj);
        }
      }
    }
    if (!ok) { SW[e] = 0.f; continue; }
    double w = std::fma(wc, (double)sc, (1.0 - wc) * dterm);
    if (!std::isfinite(w) || w < P->min_edge) w = 0.0;
    SW[e] = (float)w;
  }
  out->b0 = b0;
  out->sim_cutoff = simCutoff;
  out->n_edges = (int64_t)ne;
  out->from = (uint32_t *)malloc(4 * (ne + 1));
  out->to = (uint32_t *)malloc(4 * (ne + 1));
  out->scomp = (float *)malloc(4 * (ne + 1));
  out->score = (float *)malloc(4 * (ne + 1));
  std::copy(F.begin(), F.end(), out->from);
  std::copy(T.begin(), T.end(), out->to);
  std::copy(SC.begin(), SC.end(), out->scomp);
  std::copy(SW.begin(), SW.end(), out->score);
  return 0;
}

float orc_unit_dot_f(const float *a, const float *b, uint32_t S) { return unit_dot(a, b, (int)S); }

void orc_pmh_elements(const uint64_t *keys, const double *w, int64_t ne, uint32_t m, uint64_t seed,
                      double *regs, uint64_t *win) {
  Sketch sk((int)m);
  for (int64_t t = 0; t < ne; ++t) sk.add(keys[t], w[t], seed);
  for (uint32_t r = 0; r < m; ++r) { regs[r] = sk.tree[sk.leaves + r]; win[r] = sk.win[r]; }
}

// ── FASTA ingest (parse_fasta_mmap_parallel, src/rabbitbin.cpp:1998-2196) ──
// Sequential restatement over an in-memory file.  A record starts at the first
// '>' of a line; its name is the run of bytes > ' ' after it; the header ends at
// the next '\n' (a record without one is dropped, :2037-2038); the body runs to
// the next record start.  A body whose bytes after its first '\n' are all '\n'
// or '\r' is single-line: its first line minus one trailing '\r' (:2084-2096).
// Otherwise every '\n'-separated segment minus one trailing '\r' is kept
// (:2097-2117).  Records of length >= min_contig are large, >= min_small small,
// the rest dropped (:2131-2136); num_seqs counts every record with a header line.
// Output: large then small records, each in file order; name_start/name_len
// index the input; sequences back to back in `seq` with offsets seq_off.
struct OrcFasta {
  int64_t num_seqs, n_large, n_small;
  int64_t *name_start;
  int32_t *name_len;
  char *seq;
  int64_t *seq_off;
};

int orc_parse_fasta(const char *buf, int64_t n, int64_t min_contig, int64_t min_small,
                    OrcFasta *out) {
  struct Rec { int64_t ns; int32_t nl; std::string s; };
  std::vector<Rec> large, small;
  int64_t nseq = 0, p = 0;
  auto find = [&](int64_t from, char c) -> int64_t {
    for (int64_t q = from; q < n; ++q) if (buf[q] == c) return q;
    return -1;
  };
  while (p < n) {
    const int64_t gt = find(p, '>');
    if (gt < 0) break;
    int64_t q = gt + 1;
    const int64_t ns = q;
    while (q < n && (uint8_t)buf[q] > ' ') ++q;
    const int32_t nl_len = (int32_t)(q - ns);
    const int64_t hnl = find(q, '\n');
    if (hnl < 0) break;
    const int64_t b0 = hnl + 1;
    int64_t b1 = find(b0, '>');
    if (b1 < 0) b1 = n;
    std::string s;
    int64_t first_nl = -1;
    for (int64_t t = b0; t < b1; ++t) if (buf[t] == '\n') { first_nl = t; break; }
    bool single = true;
    if (first_nl >= 0)
      for (int64_t t = first_nl + 1; t < b1; ++t)
        if (buf[t] != '\n' && buf[t] != '\r') { single = false; break; }
    if (single) {
      int64_t e = first_nl >= 0 ? first_nl : b1;
      if (e > b0 && buf[e - 1] == '\r') --e;
      s.assign(buf + b0, buf + e);
    } else {
      int64_t seg = b0;
      while (seg < b1) {
        int64_t e = seg;
        while (e < b1 && buf[e] != '\n') ++e;
        int64_t l = e - seg;
        if (l > 0 && buf[seg + l - 1] == '\r') --l;
        s.append(buf + seg, buf + seg + l);
        if (e >= b1) break;
        seg = e + 1;
      }
    }
    ++nseq;
    const int64_t L = (int64_t)s.size();
    if (L >= min_contig) large.push_back({ns, nl_len, std::move(s)});
    else if (L >= min_small) small.push_back({ns, nl_len, std::move(s)});
    p = b1;
  }
  const size_t cnt = large.size() + small.size();
  size_t tot = 0;
  for (auto &r : large) tot += r.s.size();
  for (auto &r : small) tot += r.s.size();
  out->num_seqs = nseq;
  out->n_large = (int64_t)large.size();
  out->n_small = (int64_t)small.size();
  out->name_start = (int64_t *)malloc((cnt + 1) * sizeof(int64_t));
  out->name_len = (int32_t *)malloc((cnt + 1) * sizeof(int32_t));
  out->seq = (char *)malloc(tot + 1);
  out->seq_off = (int64_t *)malloc((cnt + 1) * sizeof(int64_t));
  size_t k = 0, o = 0;
  out->seq_off[0] = 0;
  for (auto *v : {&large, &small})
    for (auto &r : *v) {
      out->name_start[k] = r.ns;
      out->name_len[k] = r.nl;
      memcpy(out->seq + o, r.s.data(), r.s.size());
      o += r.s.size();
      out->seq_off[++k] = (int64_t)o;
    }
  return 0;
}

// One-permutation MinHash bucket values (RABBIT_PMH=0 sketch) of n contigs:
// out[r][b] = the low `bits` bits of bucket b after densification, i.e. the
// bit-planes of KmerSketch::getSignature read per bucket.
//   update  src/rabbit_sketch.h:199-238 (2-bit lex codes, windows of K valid
//           bases, canonical = min(forward, reverse complement),
//           h = murmur3_fmix(canonical, 42), bucket (h>>32)*m>>32, keep min (uint32)h)
//   densify src/rabbit_sketch.h:245-259 (probe base/step from murmur3_fmix of the
//           bucket index, value ^ (uint32)murmur3_fmix(hop, 0x9E3779B97F4A7C15))
//   buildSig src/rabbit_sketch.h:264-281 (no k-mer at all: every bucket 0)
void orc_oph_values(const char *seqcat, const int64_t *offsets, int64_t n, uint32_t m, int K,
                   uint32_t bits, uint8_t *out) {
  auto fmix = [](uint64_t x, uint64_t seed) {
    x ^= seed;
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
  };
  auto reduce = [](uint64_t h, uint32_t mm) { return (uint32_t)(((h >> 32) * (uint64_t)mm) >> 32); };
  auto code = [](char ch) -> int {
    switch (ch) {
      case 'A': case 'a': return 0;
      case 'C': case 'c': return 1;
      case 'G': case 'g': return 2;
      case 'T': case 't': return 3;
      default: return -1;
    }
  };
  const uint64_t seed = 42;
  const uint32_t empty = 0xFFFFFFFFu;
  std::vector<uint32_t> reg(m);
  for (int64_t r = 0; r < n; ++r) {
    std::fill(reg.begin(), reg.end(), empty);
    const char *sq = seqcat + offsets[r];
    const int64_t L = offsets[r + 1] - offsets[r];
    uint32_t nonempty = 0;
    for (int64_t i = 0; i + K <= L; ++i) {
      uint64_t fwd = 0, rc = 0;
      bool ok = true;
      for (int q = 0; q < K && ok; ++q) {
        const int c = code(sq[i + q]);
        if (c < 0) ok = false;
        fwd = (fwd << 2) | (uint64_t)c;
        rc |= (uint64_t)(3 - c) << (2 * q);          // base q lands at position K-1-q
      }
      if (!ok) continue;
      const uint64_t h = fmix(fwd < rc ? fwd : rc, seed);
      const uint32_t b = reduce(h, m), v = (uint32_t)h;
      if (v < reg[b]) {
        if (reg[b] == empty) ++nonempty;
        reg[b] = v;
      }
    }
    const uint32_t mask = (1u << bits) - 1u;
    for (uint32_t b = 0; b < m; ++b) {
      uint32_t v = reg[b];
      if (nonempty == 0) {
        v = 0;
      } else if (v == empty) {
        const uint64_t base = fmix(b, seed ^ 0xA5A5A5A5DEADBEEFull);
        const uint64_t step = fmix(b, seed ^ 0x123456789ABCDEF0ull) | 1ull;
        uint64_t cur = base;
        v = 0;
        for (uint32_t t = 1; t <= m; ++t) {
          cur += step;
          const uint32_t x = reg[reduce(cur, m)];
          if (x != empty) {
            v = x ^ (uint32_t)fmix(t, 0x9E3779B97F4A7C15ull);
            break;
          }
        }
      }
      out[(size_t)r * m + b] = (uint8_t)(v & mask);
    }
  }
}

}  // extern "C"
