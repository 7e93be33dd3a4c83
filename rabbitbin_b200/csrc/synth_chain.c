/* Order-3 DNA Markov chains for the seeded synthetic assemblies (synth.py).
 * One independent chain per contig, each from its own splitmix64 stream. */
#include <stdint.h>

static inline uint64_t splitmix64(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* cum: [G][64][3] cumulative transition probabilities; out: ASCII, contig r
 * written at out[offsets[r] .. offsets[r+1]). */
void synth_chains(const double *cum, const int32_t *genome, const int64_t *offsets,
                  const uint64_t *seeds, int64_t n, char *out) {
  static const char acgt[4] = {'A', 'C', 'G', 'T'};
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t r = 0; r < n; ++r) {
    uint64_t s = seeds[r];
    const double *c = cum + (int64_t)genome[r] * 64 * 3;
    unsigned ctx = (unsigned)(splitmix64(&s) & 63u);
    for (int64_t t = offsets[r]; t < offsets[r + 1]; ++t) {
      const double u = (double)(splitmix64(&s) >> 11) * (1.0 / 9007199254740992.0);
      const double *p = c + ctx * 3;
      const unsigned b = (u > p[0]) + (u > p[1]) + (u > p[2]);
      out[t] = acgt[b];
      ctx = ((ctx << 2) | b) & 63u;
    }
  }
}
