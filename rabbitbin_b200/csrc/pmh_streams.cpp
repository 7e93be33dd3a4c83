// ProbMinHash element streams and the similarity table (host side).
//
// Weighted ProbMinHash (Ertl, "ProbMinHash – A Class of Locality-Sensitive
// Hash Algorithms for the (Probability) Jaccard Similarity", TKDE 2020) as
// RabbitBin runs it (src/probmh.cpp:628-686): an element with hash h and
// weight w draws, from an RNG seeded by murmur3_fmix(h, seed), a random
// permutation of the m registers and an increasing sequence of values
// U_1 <= U_2 <= ... (truncated-exponential samples on a fixed grid of
// boundaries); it offers hv_s = (1/w) * U_s to register perm(s).
//
// Every random draw of that process depends only on the RNG state, never on
// w: the weight enters only through the multiplication by 1/w and through the
// early exits, which never change the final registers (each exit is taken only
// when no later offer can be smaller than the current largest register).  The
// sketch is therefore the order-respecting minimum
//     reg[r] = min over elements e, in insertion order, of (1/w_e) * U_e(r)
// (first-inserted wins ties, like the tracker's strict <), and the winner of
// register r is the RNG state e held when it visited r.  This file builds, once
// per (k, m, seed), the full stream of every canonical k-mer: U_e(r) and the
// winner state W_e(r).  The per-contig work on the GPU is then the min above.
//
// Floating-point operations follow the reference's release build exactly:
// -ffp-contract=off here, with std::fma written where GCC contracts the
// reference's expressions (the TED step, the exponential tail and the
// ziggurat's rejection test); contract = 0 reproduces a -ffp-contract=off
// build of the reference instead.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <unordered_map>

#include "rbg_internal.h"

namespace rbg {
namespace {

#include "zig_tables.inc"

// murmur3 64-bit finaliser with seed xor (src/hash_int.h:77-86).
inline uint64_t fmix64(uint64_t x, uint64_t seed) {
  x ^= seed;
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

// wyrand step and its derived draws (src/probmh.cpp:60-87).
inline uint64_t wy_next(uint64_t &st) {
  st += 0xa0761d6478bd642fULL;
  unsigned __int128 r = (unsigned __int128)st * (st ^ 0xe7037ed1a0b428dbULL);
  return (uint64_t)(r >> 64) ^ (uint64_t)r;
}
inline double wy_unit(uint64_t &st) {
  return (double)(wy_next(st) >> 11) * (1.0 / (double)(1ULL << 53));
}
// Lemire's bounded integer in [0, n) with rejection.
inline uint32_t wy_below(uint32_t n, uint64_t &st) {
  uint64_t x = wy_next(st) >> 32;
  uint64_t mm = x * (uint64_t)n;
  uint32_t lo = (uint32_t)mm;
  if (lo < n) {
    const uint32_t t = (uint32_t)(0u - n) % n;
    while (lo < t) {
      x = wy_next(st) >> 32;
      mm = x * (uint64_t)n;
      lo = (uint32_t)mm;
    }
  }
  return (uint32_t)(mm >> 32);
}

struct Ted { double boundary, gap, c1, c2, c3; };

// Truncated-exponential grid for m registers (src/probmh.cpp:506-572).
void ted_grid(int m, std::vector<Ted> &t, double &first_inv) {
  t.assign(m - 1, Ted{});
  const double fb = std::log1p(1.0 / (double)(m - 1));
  first_inv = 1.0 / fb;
  auto consts = [](double rate, Ted &p) {
    p.c1 = (rate != 0.0) ? std::expm1(rate) / rate : 1.0;
    p.c2 = (rate != 0.0) ? -std::log1p(std::expm1(-rate) * 0.5) / rate : 0.5;
    p.c3 = (rate != 0.0) ? -std::expm1(-rate) / rate : 1.0;
  };
  t[0].boundary = 1.0;
  t[0].gap = 1.0;
  consts(fb, t[0]);
  double prev = fb;
  for (int i = 1; i < m - 1; ++i) {
    const double b = std::log1p((double)(i + 1) / (double)(m - i - 1));
    const double bn = b / fb;
    t[i].boundary = bn;
    t[i].gap = bn - t[i - 1].boundary;
    consts(b - prev, t[i]);
    prev = b;
  }
}

// Truncated-exponential sample on [0, 1) (rejection with squeeze).
double ted_draw(const Ted &p, uint64_t &st) {
  double x = wy_unit(st) * p.c1;
  if (x < 1.0) return x;
  for (;;) {
    x = wy_unit(st);
    if (x <= p.c2) return x;
    double y = wy_unit(st) * 0.5;
    if (y > 1.0 - x) { x = 1.0 - x; y = 1.0 - y; }
    if (x <= p.c3 * (1.0 - y)) return x;
    if (p.c1 * y <= 1.0 - x) return x;
  }
}

// Exp(1) by the 256-layer ziggurat; the rejection test evaluates e^-x with the
// host libm, the same function the reference calls.
double zig_exp(uint64_t &st, bool fused) {
  double shift = 0.0;
  for (;;) {
    const uint64_t bits = wy_next(st);
    const int i = (int)(bits & 0xFF);
    const double u = (double)(bits >> 11) * (1.0 / (double)(1ULL << 53));
    const double x = u * kZigX[i];
    if (x < kZigX[i + 1]) return shift + x;
    if (i == 0) { shift += kZigX[1]; continue; }
    const double y01 = wy_unit(st);
    double y, ub, lb;
    if (fused) {
      y = std::fma(y01, kZigY[i + 1] - kZigY[i], kZigY[i]);
      ub = std::fma(kZigX[i] - kZigX[i + 1], y01, -(kZigX[i] - x));
      lb = y - std::fma(kZigX[i + 1] - x, kZigY[i + 1], kZigY[i + 1]);
    } else {
      y = kZigY[i] + y01 * (kZigY[i + 1] - kZigY[i]);
      ub = (kZigX[i] - kZigX[i + 1]) * y01 - (kZigX[i] - x);
      lb = y - (kZigY[i + 1] + (kZigX[i + 1] - x) * kZigY[i + 1]);
    }
    if (ub < 0 && (lb < 0 || y < std::exp(-x))) return x + shift;
  }
}

inline uint16_t fold16(uint32_t w) {
  if (w == 0) return 0;
  const uint16_t h = (uint16_t)(w ^ (w >> 16));
  return h ? h : (uint16_t)1;
}

int revcomp_code(int v, int k) {
  int r = 0;
  for (int i = 0; i < k; ++i) { r = (r << 2) | (3 - (v & 3)); v >>= 2; }
  return r;
}

// Full m-step stream of one element: U and winner per register.
void element_stream(uint64_t rng, int m, const std::vector<Ted> &ted, double first_inv,
                    bool fused, double *U, uint64_t *W, std::vector<uint32_t> &perm) {
  // initial offer (src/probmh.cpp:643-649)
  const double u0 = (double)(rng >> 11) * (1.0 / (double)(1ULL << 53));
  const double h0 = u0 * ted[0].c1;
  double cur = (h0 < 1.0) ? h0 : ted_draw(ted[0], rng);
  // fresh lazy Fisher-Yates permutation (src/probmh.cpp:460-479)
  perm.resize(m);
  for (int i = 0; i < m; ++i) perm[i] = (uint32_t)i;
  for (int s = 0; s < m; ++s) {
    const uint32_t kk = (uint32_t)s + wy_below((uint32_t)(m - s), rng);
    const uint32_t reg = perm[kk];
    perm[kk] = perm[s];
    U[reg] = cur;
    W[reg] = rng;
    if (s + 1 >= m) break;
    if (s + 1 < m - 1) {          // loop index i = s + 1 < m - 1: TED step
      const Ted &tp = ted[s + 1];
      const double t = ted_draw(tp, rng);
      cur = fused ? std::fma(tp.gap, t, ted[s].boundary) : ted[s].boundary + tp.gap * t;
    } else {                      // i = m - 1: exponential tail
      const double z = zig_exp(rng, fused);
      cur = fused ? std::fma(first_inv, z, ted[m - 2].boundary)
                  : ted[m - 2].boundary + first_inv * z;
    }
  }
}

}  // namespace

std::shared_ptr<const PmhTables> pmh_tables(int k, int m, uint64_t seed, int contract) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, uint64_t, int>, std::shared_ptr<const PmhTables>> cache;
  const auto key = std::make_tuple(k, m, seed, contract);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  auto t = std::make_shared<PmhTables>();
  t->k = k; t->m = m; t->seed = seed; t->contract = contract;
  const int nb = 1 << (2 * k);
  t->rank_of_code.assign(nb, -1);
  for (int v = 0; v < nb; ++v)
    if (v <= revcomp_code(v, k)) {
      t->rank_of_code[v] = (int)t->canon_codes.size();
      t->canon_codes.push_back(v);
    }
  const int E = (int)t->canon_codes.size();
  t->n_elems = E;
  std::vector<Ted> ted;
  double first_inv = 0.0;
  ted_grid(m, ted, first_inv);
  t->U.resize((size_t)E * m);
  t->W64.resize((size_t)E * m);
  std::vector<uint32_t> perm;
  for (int e = 0; e < E; ++e)
    element_stream(fmix64((uint64_t)t->canon_codes[e], seed), m, ted, first_inv,
                   contract != 0, &t->U[(size_t)e * m], &t->W64[(size_t)e * m], perm);
  t->order.resize((size_t)m * E);
  t->UT.resize((size_t)m * E);
  for (int r = 0; r < m; ++r) {
    for (int e = 0; e < E; ++e) t->UT[(size_t)r * E + e] = t->U[(size_t)e * m + r];
    RegOrder *o = &t->order[(size_t)r * E];
    for (int e = 0; e < E; ++e) o[e] = RegOrder{t->U[(size_t)e * m + r], (uint32_t)e, 0u};
    std::stable_sort(o, o + E, [](const RegOrder &x, const RegOrder &y) { return x.u < y.u; });
  }
  t->W32.resize((size_t)E * m);
  t->W16.resize((size_t)E * m);
  for (size_t q = 0; q < t->W64.size(); ++q) {
    const uint64_t h = t->W64[q];
    t->W32[q] = (uint32_t)(h ^ (h >> 32));
    t->W16[q] = fold16(t->W32[q]);
  }
  // Per-column dictionaries: equal folded winners share a code, 0 stays 0.
  t->code16.assign((size_t)E * m, 0);
  t->code32.assign((size_t)E * m, 0);
  for (int r = 0; r < m; ++r) {
    std::unordered_map<uint32_t, int> d16, d32;
    for (int e = 0; e < E; ++e) {
      const size_t q = (size_t)e * m + r;
      if (t->W16[q]) {
        auto it = d16.emplace(t->W16[q], (int)d16.size() + 1).first;
        t->code16[q] = (uint8_t)it->second;
      }
      if (t->W32[q]) {
        auto it = d32.emplace(t->W32[q], (int)d32.size() + 1).first;
        t->code32[q] = (uint8_t)it->second;
      }
    }
  }
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.emplace(key, t).first;
  return it->second;
}

// Similarity of c equal buckets of m under the one-permutation metric:
// jaccard_raw's matches / m (src/rabbitbin.cpp:1035-1130), as graph_sim returns
// it (:1423-1425; no baseline, no clamp).
void oph_sv_table(int m, std::vector<double> &sv_d, std::vector<float> &sv_f) {
  sv_d.resize(m + 1);
  sv_f.resize(m + 1);
  for (int c = 0; c <= m; ++c) {
    sv_d[c] = (double)(uint64_t)c / (double)(uint32_t)m;
    sv_f[c] = (float)sv_d[c];
  }
}

void sv_table(int m, bool base_on, double b0, std::vector<double> &sv_d,
              std::vector<float> &sv_f) {
  const double inv_m = 1.0 / (double)m;
  const double inv1mb0 = (b0 < 1.0) ? 1.0 / (1.0 - b0) : 1.0;
  sv_d.resize(m + 1);
  sv_f.resize(m + 1);
  for (int c = 0; c <= m; ++c) {
    double j = (double)(uint32_t)c * inv_m;
    if (base_on && b0 > 0.0 && b0 < 1.0) {
      j = (j - b0) * inv1mb0;
      if (j < 0.0) j = 0.0;
    }
    if (j > 1.0 - 1e-6) j = 1.0 - 1e-6;
    sv_d[c] = j;
    sv_f[c] = (float)j;
  }
}

}  // namespace rbg
