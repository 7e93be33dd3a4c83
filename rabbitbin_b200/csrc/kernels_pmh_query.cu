// ProbMinHash4 sketch rows and sketch-vs-sketch queries on the device: the
// batch counterparts of ProbMinHash4::getWinners / getRegisters,
// jaccard_weighted, jaccard, distance, ani and merge (src/probmh.h:103-283,
// src/probmh.cpp:1325-1440).
//
// A sketch row is m 64-bit words: the winners (RNG state of the element that
// won each register, 0 when unset) or the register values (doubles, +inf when
// unset).  A comparison counts the registers whose words are equal and set --
// jaccard_weighted on winners (:1364-1376), jaccard on register values
// (:1325-1362, exact double equality) -- and maps the count through a table of
// m + 1 doubles the host made with the reference's own formulas (count / m,
// and the distance / ANI transforms of it with the host's libm), so every
// value equals the reference's bit for bit.
#include <algorithm>
#include <cstdint>

#include "rbg_internal.h"

namespace rbg {
namespace {

__global__ void k_pmh_rows(const uint8_t *__restrict__ win_elem,
                           const double *__restrict__ elem_winv, int64_t n, int m, int E,
                           const uint64_t *__restrict__ W64, const double *__restrict__ U,
                           uint64_t *__restrict__ w64_out, double *__restrict__ reg_out) {
  const int64_t total = n * (int64_t)m;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = q / m;
    const int r = (int)(q - c * m);
    const uint32_t e = win_elem[q];
    uint64_t w = 0;
    double v = __longlong_as_double(0x7ff0000000000000ll);     // +inf
    if (e != 0xFFu) {
      w = __ldg(W64 + (size_t)e * m + r);
      // the same rounded product the register minimum compared
      v = __dmul_rn(__ldg(elem_winv + c * E + e), __ldg(U + (size_t)e * m + r));
    }
    if (w64_out) w64_out[q] = w;
    if (reg_out) reg_out[q] = v;
  }
}

constexpr int kQT = 32;       // rows of A and of B per CTA
constexpr int kQC = 32;       // registers per staged chunk

// CTA: a 32 x 32 tile of (A row, B row) pairs; thread (tx, ty) owns the pairs
// (ty + 8 u, tx), u = 0..3.  Register chunks of A and B rows are staged in
// shared memory (padded rows: no bank conflicts on the column reads).
template <bool REGS>
__global__ void __launch_bounds__(256)
k_pmh_compare(const uint64_t *__restrict__ A, int64_t na, const uint64_t *__restrict__ B,
              int64_t nb, int m, const double *__restrict__ table, double *__restrict__ out) {
  __shared__ uint64_t sa[kQT][kQC + 1], sb[kQT][kQC + 1];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t a0 = (int64_t)blockIdx.y * kQT, b0 = (int64_t)blockIdx.x * kQT;
  int cnt[4] = {0, 0, 0, 0};
  const uint64_t unset = REGS ? 0x7ff0000000000000ull : 0ull;
  for (int k0 = 0; k0 < m; k0 += kQC) {
    for (int t = threadIdx.x; t < kQT * kQC; t += 256) {
      const int row = t / kQC, col = t - row * kQC;
      const bool in = k0 + col < m;
      sa[row][col] = (in && a0 + row < na) ? __ldg(A + (a0 + row) * m + k0 + col) : unset;
      sb[row][col] = (in && b0 + row < nb) ? __ldg(B + (b0 + row) * m + k0 + col) : unset;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kQC; ++k) {
      const uint64_t bv = sb[tx][k];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint64_t av = sa[ty + 8 * u][k];
        if (REGS) {
          const double x = __longlong_as_double((long long)av), y = __longlong_as_double((long long)bv);
          cnt[u] += (x == y && x != __longlong_as_double(0x7ff0000000000000ll)) ? 1 : 0;
        } else {
          cnt[u] += (av != 0ull && av == bv) ? 1 : 0;
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int64_t i = a0 + ty + 8 * u, j = b0 + tx;
    if (i < na && j < nb) out[i * nb + j] = __ldg(table + cnt[u]);
  }
}

__global__ void k_pmh_merge(const double *__restrict__ a, const double *__restrict__ b,
                            int64_t count, double *__restrict__ out) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < count;
       q += (int64_t)gridDim.x * blockDim.x) {
    const double x = a[q], y = b[q];
    out[q] = (y < x) ? y : x;                 // std::min(x, y)
  }
}

}  // namespace

void launch_pmh_rows(const uint8_t *win_elem, const double *elem_winv, int64_t n, int m, int E,
                     const uint64_t *W64, const double *U, uint64_t *w64_out, double *reg_out,
                     cudaStream_t s) {
  const int64_t total = n * (int64_t)m;
  if (total == 0) return;
  const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 16);
  k_pmh_rows<<<(unsigned)blocks, 256, 0, s>>>(win_elem, elem_winv, n, m, E, W64, U, w64_out,
                                              reg_out);
}

void launch_pmh_compare(const uint64_t *A, int64_t na, const uint64_t *B, int64_t nb, int m,
                        bool regs, const double *table, double *out, cudaStream_t s) {
  if (na == 0 || nb == 0) return;
  const dim3 grid((unsigned)((nb + kQT - 1) / kQT), (unsigned)((na + kQT - 1) / kQT));
  if (regs) k_pmh_compare<true><<<grid, 256, 0, s>>>(A, na, B, nb, m, table, out);
  else k_pmh_compare<false><<<grid, 256, 0, s>>>(A, na, B, nb, m, table, out);
}

void launch_pmh_merge(const double *a, const double *b, int64_t count, double *out,
                      cudaStream_t s) {
  if (count == 0) return;
  const int64_t blocks = std::min<int64_t>((count + 255) / 256, 148 * 16);
  k_pmh_merge<<<(unsigned)blocks, 256, 0, s>>>(a, b, count, out);
}

}  // namespace rbg
