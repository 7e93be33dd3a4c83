// Small kernels behind the single-function entry points: fold_win16, the
// winner-match count of sampled pairs on raw 16/32-bit winners, and the
// mapping of externally produced winner rows to register codes.
#include <cstdint>

#include "rbg_internal.h"

namespace rbg {
namespace {

// fold_win16 (src/rabbitbin.cpp:249-253)
__global__ void k_fold16(const uint32_t *__restrict__ in, int64_t n, uint16_t *__restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t w = in[t];
  uint16_t h = 0;
  if (w) {
    h = (uint16_t)(w ^ (w >> 16));
    if (!h) h = 1;
  }
  out[t] = h;
}

// pmh_match_count16 / pmh_match_count (src/rabbitbin.cpp:1194-1293):
// registers with a == b and a != 0.
template <typename T>
__global__ void k_raw_pair_counts(const T *__restrict__ win, int m, const int64_t *__restrict__ pairs,
                                  int np, uint32_t *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const T *a = win + pairs[2 * p] * (int64_t)m;
  const T *b = win + pairs[2 * p + 1] * (int64_t)m;
  uint32_t c = 0;
  for (int k = 0; k < m; ++k) {
    const T x = a[k];
    c += (x != 0 && x == b[k]);
  }
  out[p] = c;
}

// Winner value -> register code through per-column sorted dictionaries
// (vals[r][0..E) ascending, codes alongside).  Unknown values raise *bad.
__global__ void k_codes_from_winners(const uint32_t *__restrict__ w32, int64_t n, int m, int mpad,
                                     int use16, const uint32_t *__restrict__ vals,
                                     const uint8_t *__restrict__ codes, const int32_t *__restrict__ nvals,
                                     uint8_t *__restrict__ A, uint8_t *__restrict__ B,
                                     int *__restrict__ bad) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * (int64_t)mpad) return;
  const int64_t row = t / mpad;
  const int r = (int)(t - row * mpad);
  uint8_t code = 0;
  if (r < m) {
    uint32_t v = w32[row * m + r];
    if (use16 && v) {
      uint32_t h = (v ^ (v >> 16)) & 0xFFFFu;
      v = h ? h : 1u;
    }
    if (v) {
      const uint32_t *col = vals + (int64_t)r * kMaxElems;
      int lo = 0, hi = nvals[r];
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (col[mid] < v) lo = mid + 1; else hi = mid;
      }
      if (lo < nvals[r] && col[lo] == v) code = codes[(int64_t)r * kMaxElems + lo];
      else atomicExch(bad, 1);
    }
  }
  A[t] = code;
  B[t] = code ? code : (uint8_t)0xFF;
}

}  // namespace

void launch_fold16(const uint32_t *in, int64_t n, uint16_t *out, cudaStream_t s) {
  if (n == 0) return;
  k_fold16<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, n, out);
}

void launch_raw_pair_counts(const void *win, int bits, int m, const int64_t *pairs, int np,
                            uint32_t *out, cudaStream_t s) {
  if (np == 0) return;
  if (bits == 16)
    k_raw_pair_counts<uint16_t><<<(np + 127) / 128, 128, 0, s>>>((const uint16_t *)win, m, pairs, np, out);
  else
    k_raw_pair_counts<uint32_t><<<(np + 127) / 128, 128, 0, s>>>((const uint32_t *)win, m, pairs, np, out);
}

void launch_codes_from_winners(const uint32_t *w32, int64_t n, int m, int mpad, int use16,
                               const uint32_t *vals, const uint8_t *codes, const int32_t *nvals,
                               uint8_t *A, uint8_t *B, int *bad, cudaStream_t s) {
  const int64_t tot = n * (int64_t)mpad;
  if (tot == 0) return;
  k_codes_from_winners<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(w32, n, m, mpad, use16, vals,
                                                                    codes, nvals, A, B, bad);
}

}  // namespace rbg
