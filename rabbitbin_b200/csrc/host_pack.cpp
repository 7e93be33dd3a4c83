// 2-bit packing on the host for the end-to-end call (rbg_bin_graph).
//
// The end-to-end call receives the contigs as host ASCII and used to copy the
// bytes to the device and pack them there (k_pack).  Packing on the host first
// sends 3/8 of a byte per base instead of one: the 2-bit codes (16 bases per
// 32-bit word, first base in the top bits, 0 for an invalid base) and the
// invalid-base mask (one bit per base; mask word w/2 holds words w and w+1,
// base t of the pair at bit 31 - t).  The layout is exactly the one k_pack
// writes, so the device kernels that follow cannot tell the difference.
//
// Encoding (RB_BASE_ENC_LUT, src/rabbit_sketch.h:56-75): A/a 0, C/c 1, G/g 2,
// T/t 3, anything else invalid.  32 bases at a time with AVX2 where the host
// has it (l = byte | 0x20; ((l >> 1) ^ (l >> 2)) & 3 is the code of a, c, g,
// t; the letter rebuilt from the code equals l exactly for the eight valid
// letters), a byte table otherwise.  A chunk is split over a small pool of
// host threads that lives as long as the library.
#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "engine_internal.h"

namespace rbg {
namespace {

uint32_t reverse_bits(uint32_t x) {
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
  x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
  return (x >> 16) | (x << 16);
}

// 32 bases -> two packed words and one mask word (scalar table).
void pack32_scalar(const unsigned char *s, uint32_t *w2, uint32_t *mask) {
  uint32_t a = 0, b = 0, bad = 0;
  for (int t = 0; t < 32; ++t) {
    const unsigned l = s[t] | 0x20u;
    uint32_t code = 0;
    bool ok = true;
    switch (l) {
      case 'a': code = 0; break;
      case 'c': code = 1; break;
      case 'g': code = 2; break;
      case 't': code = 3; break;
      default: ok = false;
    }
    if (!ok) bad |= 1u << (31 - t);
    if (t < 16) a |= code << (30 - 2 * t);
    else b |= code << (30 - 2 * (t - 16));
  }
  w2[0] = a;
  w2[1] = b;
  *mask = bad;
}

__attribute__((target("avx2"))) void pack32_avx2(const unsigned char *s, uint32_t *w2,
                                                 uint32_t *mask) {
  const __m256i v = _mm256_loadu_si256((const __m256i *)s);
  const __m256i l = _mm256_or_si256(v, _mm256_set1_epi8(0x20));
  const __m256i three = _mm256_set1_epi8(3);
  __m256i code = _mm256_and_si256(
      _mm256_xor_si256(_mm256_srli_epi16(l, 1), _mm256_srli_epi16(l, 2)), three);
  const __m256i letters = _mm256_setr_epi8('a', 'c', 'g', 't', 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                           'a', 'c', 'g', 't', 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0);
  const __m256i valid = _mm256_cmpeq_epi8(_mm256_shuffle_epi8(letters, code), l);
  code = _mm256_and_si256(code, valid);
  // 4 * c0 + c1 per byte pair, then 16 * (4 c0 + c1) + (4 c2 + c3) per 4 bases
  const __m256i p16 = _mm256_maddubs_epi16(code, _mm256_set1_epi16(0x0104));
  const __m256i p32 = _mm256_madd_epi16(p16, _mm256_set1_epi32(0x00010010));
  // low bytes of the four 32-bit lanes of each half, last group first
  const __m256i sel = _mm256_setr_epi8(12, 8, 4, 0, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                                       12, 8, 4, 0, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1);
  const __m256i g = _mm256_shuffle_epi8(p32, sel);
  w2[0] = (uint32_t)_mm256_extract_epi32(g, 0);
  w2[1] = (uint32_t)_mm256_extract_epi32(g, 4);
  *mask = reverse_bits(~(uint32_t)_mm256_movemask_epi8(valid));
}

bool have_avx2() {
  static const bool yes = __builtin_cpu_supports("avx2");
  return yes;
}

// Persistent worker pool: run(fn, parts) calls fn(0..parts-1) across the
// workers and the caller, and returns when all have finished.
class Pool {
 public:
  Pool() {
    const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
    nthreads_ = (int)std::min(hc, 32u);
    for (int t = 1; t < nthreads_; ++t) threads_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : threads_) t.join();
  }
  int size() const { return nthreads_; }
  void run(const std::function<void(int)> &fn, int parts) {
    std::lock_guard<std::mutex> one(run_mu_);         // one job at a time
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      parts_ = parts;
      next_.store(0);
      done_ = 0;
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return done_ == parts_; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      const int i = next_.fetch_add(1);
      if (i >= parts_) return;
      (*fn_)(i);
      std::lock_guard<std::mutex> lk(mu_);
      if (++done_ == parts_) done_cv_.notify_all();
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
    }
  }
  int nthreads_ = 1;
  std::vector<std::thread> threads_;
  std::mutex mu_, run_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)> *fn_ = nullptr;
  int parts_ = 0, done_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
  std::atomic<int> next_{0};
};

Pool &pool() {
  static Pool p;
  return p;
}

}  // namespace

int host_pack_threads() { return pool().size(); }

void host_pack_words(const char *ascii, int64_t nbases, int64_t w0, int64_t w1,
                     uint32_t *packed, uint32_t *mask) {
  // word pairs [w0, w1) rounded up to an even count; w0 is even
  const int64_t pairs = (w1 - w0 + 1) / 2;
  if (pairs <= 0) return;
  const bool avx2 = have_avx2();
  const int parts = (int)std::min<int64_t>(pool().size() * 4, std::max<int64_t>(1, pairs / 4096));
  pool().run(
      [&](int part) {
        const int64_t p0 = pairs * part / parts, p1 = pairs * (part + 1) / parts;
        for (int64_t p = p0; p < p1; ++p) {
          const int64_t b = 16 * (w0 + 2 * p);               // first base of the pair
          uint32_t *wp = packed + 2 * p, *mp = mask + p;
          if (b + 32 <= nbases) {
            if (avx2) pack32_avx2((const unsigned char *)ascii + b, wp, mp);
            else pack32_scalar((const unsigned char *)ascii + b, wp, mp);
          } else {
            unsigned char tail[32] = {0};                    // bases past nbases: invalid
            if (nbases > b) std::memcpy(tail, ascii + b, (size_t)(nbases - b));
            pack32_scalar(tail, wp, mp);
          }
        }
      },
      parts);
}

}  // namespace rbg
