// Correctly rounded double exp and log from double-double arithmetic, for the
// label-propagation scores, which the reference evaluates with the C library's
// exp and log (src/impl/rb_cluster.cpp:12-22, :453).  Both are written here
// from the mathematics, not taken from any library:
//
//   exp(x): Cody-Waite reduction x = k ln2 + r with ln2 split in three parts
//           (the first has 41 significant bits, so k ln2_1 is exact for
//           |k| < 2^12), s = r / 64, expm1(s) by its Taylor series (terms
//           through s^12, the first five with double-double coefficients),
//           six squarings E <- 2E + E^2 (expm1 of the doubled argument), then
//           (1 + E) 2^k rounded once, subnormal results included.
//   log(x): one Newton step on exp from y0 = log(x) (any approximation within
//           a few ulps): y = y0 + log1p(d), d = x e^-y0 - 1 in double-double.
//
// The double-double values carry about 100 correct bits, so the rounding to
// double is the correctly rounded one unless the exact value lies within about
// 2^-100 relative of a rounding boundary.  The C library's exp and log are not
// correctly rounded in every case (they differ from the exact rounding on
// about 1e-3 and 2e-4 of random arguments); the label decisions depend on
// these values only through comparisons, which a difference of one ulp
// changes only when two scores agree to about 1e-16.
//
// Every operation is an explicit round-to-nearest primitive, so the code gives
// the same bits on the host (compiled with -ffp-contract=off) and the device.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define RBG_DD __host__ __device__ __forceinline__
#else
#define RBG_DD inline
#endif

namespace rbg {
namespace dd {

RBG_DD double add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
RBG_DD double sub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
RBG_DD double mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
RBG_DD double fma_(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
RBG_DD double ldexp_(double x, int e) {   // exact while the result stays normal
#if defined(__CUDA_ARCH__)
  return ::ldexp(x, e);
#else
  return std::ldexp(x, e);
#endif
}
RBG_DD double rint_(double x) {
#if defined(__CUDA_ARCH__)
  return ::rint(x);
#else
  return std::nearbyint(x);
#endif
}

struct D2 {
  double hi, lo;
};

RBG_DD D2 two_sum(double a, double b) {
  const double s = add(a, b);
  const double bb = sub(s, a);
  const double e = add(sub(a, sub(s, bb)), sub(b, bb));
  return {s, e};
}
RBG_DD D2 fast_two_sum(double a, double b) {   // |a| >= |b|
  const double s = add(a, b);
  return {s, sub(b, sub(s, a))};
}
RBG_DD D2 two_prod(double a, double b) {
  const double p = mul(a, b);
  return {p, fma_(a, b, -p)};
}
RBG_DD D2 dadd(D2 a, D2 b) {
  const D2 s = two_sum(a.hi, b.hi);
  const D2 t = two_sum(a.lo, b.lo);
  D2 r = fast_two_sum(s.hi, add(s.lo, t.hi));
  return fast_two_sum(r.hi, add(r.lo, t.lo));
}
RBG_DD D2 dadd_d(D2 a, double b) {
  const D2 s = two_sum(a.hi, b);
  return fast_two_sum(s.hi, add(s.lo, a.lo));
}
RBG_DD D2 dmul(D2 a, D2 b) {
  const D2 p = two_prod(a.hi, b.hi);
  const double c = fma_(a.hi, b.lo, mul(a.lo, b.hi));
  return fast_two_sum(p.hi, add(p.lo, c));
}
RBG_DD D2 dmul_d(D2 a, double b) {
  const D2 p = two_prod(a.hi, b);
  return fast_two_sum(p.hi, fma_(a.lo, b, p.lo));
}

// ln 2 = L1 + L2 + L3 (L1: 41 significant bits); 1/ln 2 rounded.
constexpr double kL1 = 0x1.62e42fefa4000p-1;
constexpr double kL2 = -0x1.8432a1b0e2634p-43;
constexpr double kL3 = 0x1.f97b57a079a19p-103;
constexpr double kInvLn2 = 0x1.71547652b82fep+0;

// exp(x) = (1 + E) 2^k as a double-double E and k, |x| <= 746.
RBG_DD void exp_parts(double x, D2 *E, int *k_out) {
  const double k = rint_(mul(x, kInvLn2));
  // r = x - k ln2: x - k L1 is exact (k L1 fits 53 bits, Sterbenz for k != 0)
  const double t1 = sub(x, mul(k, kL1));
  const D2 kl2 = two_prod(k, kL2);
  D2 r = dadd(D2{t1, 0.0}, D2{-kl2.hi, -kl2.lo});
  r = dadd_d(r, -mul(k, kL3));
  const D2 s{ldexp_(r.hi, -6), ldexp_(r.lo, -6)};   // |s| <= 0.0055
  // expm1(s) = s (1 + s (1/2 + s (1/6 + s (1/24 + s (1/120 + s q(s))))))
  double q = 0x1.1eed8eff8d898p-29;                 // 1/12!
  q = fma_(q, s.hi, 0x1.ae64567f544e4p-26);         // 1/11!
  q = fma_(q, s.hi, 0x1.27e4fb7789f5cp-22);         // 1/10!
  q = fma_(q, s.hi, 0x1.71de3a556c734p-19);         // 1/9!
  q = fma_(q, s.hi, 0x1.a01a01a01a01ap-16);         // 1/8!
  q = fma_(q, s.hi, 0x1.a01a01a01a01ap-13);         // 1/7!
  q = fma_(q, s.hi, 0x1.6c16c16c16c17p-10);         // 1/6!
  D2 p = dadd(D2{0x1.1111111111111p-7, 0x1.1111111111111p-63}, dmul_d(s, q));   // 1/120
  p = dadd(D2{0x1.5555555555555p-5, 0x1.5555555555555p-59}, dmul(s, p));        // 1/24
  p = dadd(D2{0x1.5555555555555p-3, 0x1.5555555555555p-57}, dmul(s, p));        // 1/6
  p = dadd_d(dmul(s, p), 0.5);
  p = dadd_d(dmul(s, p), 1.0);
  D2 e = dmul(s, p);
  for (int i = 0; i < 6; ++i)                       // expm1(2s) = 2 expm1(s) + expm1(s)^2
    e = dadd(D2{ldexp_(e.hi, 1), ldexp_(e.lo, 1)}, dmul(e, e));
  *E = e;
  *k_out = (int)k;
}

// (hi + lo) 2^k rounded to nearest even, for a normalised hi + lo in
// [0.7, 1.42] (the range of 1 + expm1(r)); subnormal and zero results included.
RBG_DD double scale_round(D2 v, int k) {
  if (k > -1022 || (k == -1022 && v.hi >= 1.0)) {  // a normal result: hi = RN(v), scaled exactly
    if (k > 1000) return mul(ldexp_(v.hi, k - 1000), 0x1p1000);
    return ldexp_(v.hi, k);
  }
  // Subnormal range: the value in units of 2^-1074 is a + b (a = hi 2^sh has
  // an ulp of at most 1/2, |b| <= ulp(a) / 2), rounded to an integer count.
  const int sh = k + 1074;
  if (sh < -2) return 0.0;                          // below half the least subnormal
  const double a = ldexp_(v.hi, sh), b = ldexp_(v.lo, sh);
  double f = rint_(a);                              // nearest, ties to even
  const double d = sub(a, f);                       // exact
  // only an exact half-way a can be moved by b
  if (d == 0.5 && b > 0.0) f = add(f, 1.0);
  else if (d == -0.5 && b < 0.0) f = sub(f, 1.0);
  return mul(f, 0x1p-1074);
}

// Correctly rounded exp (see the header for the accuracy statement).
RBG_DD double exp_cr(double x) {
  if (x != x) return x;
  if (x > 709.8) return INFINITY;
  if (x < -746.0) return 0.0;
  D2 E;
  int k;
  exp_parts(x, &E, &k);
  return scale_round(dadd_d(E, 1.0), k);
}

// Correctly rounded log for x > 0 normal, from any approximation y0.
RBG_DD double log_cr_from(double x, double y0) {
  if (x == 1.0) return 0.0;
  D2 E;
  int k;
  exp_parts(-y0, &E, &k);
  // d = x (1 + E) 2^k - 1
  D2 v = dadd_d(dmul_d(E, x), x);                   // x (1 + E)
  v.hi = ldexp_(v.hi, k);
  v.lo = ldexp_(v.lo, k);
  const D2 d = dadd_d(v, -1.0);
  // log(x) = y0 + log1p(d) = y0 + d - d^2/2 (|d| ~ 1e-16)
  const double d2 = mul(mul(d.hi, d.hi), -0.5);
  const D2 y = dadd(D2{y0, 0.0}, dadd_d(d, d2));
  return add(y.hi, y.lo);
}

RBG_DD double log_cr(double x) {
#if defined(__CUDA_ARCH__)
  return log_cr_from(x, ::log(x));
#else
  return log_cr_from(x, std::log(x));
#endif
}

}  // namespace dd
}  // namespace rbg
