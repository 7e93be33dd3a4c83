// Sketch stage kernels: 2-bit packing, canonical k-mer counting with GC-norm
// weights, and the ProbMinHash register minimum.
//
// Compiled with -fmad=false: every double operation below rounds exactly like
// the reference's (which has no contracted expression in build_pmh_winners).
#include <cstdint>

#include "rbg_internal.h"

namespace rbg {
namespace {

// A/a->0, C/c->1, G/g->2, T/t->3, anything else invalid
// (RB_BASE_ENC_LUT, src/rabbit_sketch.h:56-75).
__device__ __forceinline__ uint32_t enc_base(uint32_t c, uint32_t &bad) {
  const uint32_t l = c | 0x20u;
  uint32_t code = 0;
  bad = 0;
  if (l == 'a') code = 0;
  else if (l == 'c') code = 1;
  else if (l == 'g') code = 2;
  else if (l == 't') code = 3;
  else bad = 1;
  return code;
}

// One thread per 16 bases: a 128-bit load of ASCII, one packed word out
// (first base in the top two bits) and 16 bits of the invalid mask; lane pairs
// merge their halves into one 32-bit mask word.
__global__ void k_pack(const uint4 *__restrict__ ascii, int64_t nbases, int64_t nwords,
                       uint32_t *__restrict__ packed, uint32_t *__restrict__ nmask) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t word = 0, bad16 = 0;
  if (w < nwords) {
    const uint4 v = ascii[w];
    const uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const uint32_t c = (q[t >> 2] >> (8 * (t & 3))) & 0xFFu;
      uint32_t bad;
      uint32_t code = enc_base(c, bad);
      if (w * 16 + t >= nbases) bad = 1;
      if (bad) code = 0;
      word |= code << (30 - 2 * t);
      bad16 |= bad << (15 - t);
    }
    packed[w] = word;
  }
  const uint32_t other = __shfl_xor_sync(0xffffffffu, bad16, 1);
  if (w < nwords && (threadIdx.x & 1) == 0) {
    const uint32_t m = (bad16 << 16) | ((w + 1 < nwords) ? other : 0xFFFFu);
    nmask[w >> 1] = m;
  }
}

// Invalid bits of the 16 bases of packed word wi, restricted to [s, e).
__device__ __forceinline__ uint32_t invalid16(const uint32_t *__restrict__ nmask, int64_t wi,
                                              int64_t s, int64_t e) {
  if (wi < 0) return 0xFFFFu;
  const uint32_t mw = __ldg(nmask + (wi >> 1));
  uint32_t b = (wi & 1) ? (mw & 0xFFFFu) : (mw >> 16);
  const int64_t g0 = wi * 16;
  if (g0 < s || g0 + 16 > e) {
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int64_t g = g0 + t;
      if (g < s || g >= e) b |= 1u << (15 - t);
    }
  }
  return b;
}

// Warp per contig: histogram of canonical k-mers (k <= 4) and base counts over
// the packed sequence, then the GC-normalised weights of build_pmh_winners
// (src/rabbitbin.cpp:1459-1516) and the ascending element list (rank, 1/w).
__global__ void k_count(SketchArgs a) {
  extern __shared__ uint32_t sh_hist[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  const int nb = 1 << (2 * a.k);
  uint32_t *hist = sh_hist + wib * 256;
  for (int v = lane; v < 256; v += 32) hist[v] = 0;
  __syncwarp();
  if (c >= a.n) return;
  const int64_t s = a.offsets[c], e = a.offsets[c + 1];
  const int k = a.k;
  const uint32_t kmask = (uint32_t)nb - 1u;
  uint32_t bc0 = 0, bc1 = 0, bc2 = 0, bc3 = 0;
  if (e - s >= k) {
    const int64_t w0 = s >> 4, w1 = (e + 15) >> 4;
    uint32_t carry_word = 0, carry_bad = 0xFFFFu;     // word before w0: all invalid
    for (int64_t base = w0; base < w1; base += 32) {
      const int64_t wi = base + lane;
      uint32_t cur = 0, bad = 0xFFFFu;
      if (wi < w1) {
        cur = __ldg(a.packed + wi);
        bad = invalid16(a.nmask, wi, s, e);
      }
      uint32_t prev = __shfl_up_sync(0xffffffffu, cur, 1);
      uint32_t prevbad = __shfl_up_sync(0xffffffffu, bad, 1);
      if (lane == 0) { prev = carry_word; prevbad = carry_bad; }
      carry_word = __shfl_sync(0xffffffffu, cur, 31);
      carry_bad = __shfl_sync(0xffffffffu, bad, 31);
      if (wi < w1) {
        const uint64_t win = ((uint64_t)prev << 32) | cur;
        const uint32_t winbad = (prevbad << 16) | bad;
#pragma unroll 4
        for (int t = 0; t < 16; ++t) {
          if ((bad >> (15 - t)) & 1u) continue;
          const uint32_t b = (cur >> (30 - 2 * t)) & 3u;
          bc0 += (b == 0); bc1 += (b == 1); bc2 += (b == 2); bc3 += (b == 3);
          // k-mer ending here: bases t-k+1 .. t of the window all valid
          const uint32_t need = (1u << k) - 1u;
          if (((winbad >> (15 - t)) & need) != 0) continue;
          const uint32_t fwd = (uint32_t)(win >> (2 * (15 - t))) & kmask;
          uint32_t rev = 0, x = fwd;
          for (int q = 0; q < k; ++q) { rev = (rev << 2) | (3u - (x & 3u)); x >>= 2; }
          atomicAdd(&hist[fwd <= rev ? fwd : rev], 1u);
        }
      }
    }
  }
  __syncwarp();
  // totals
  uint32_t tot = 0;
  for (int v = lane; v < nb; v += 32) tot += hist[v];
  tot = __reduce_add_sync(0xffffffffu, tot);
  bc0 = __reduce_add_sync(0xffffffffu, bc0);
  bc1 = __reduce_add_sync(0xffffffffu, bc1);
  bc2 = __reduce_add_sync(0xffffffffu, bc2);
  bc3 = __reduce_add_sync(0xffffffffu, bc3);
  int pos = 0;
  uint8_t *eidx = a.elem_idx + c * kMaxElems;
  double *ewinv = a.elem_winv + c * kMaxElems;
  if (tot > 0) {
    const uint64_t vb = (uint64_t)bc0 + bc1 + bc2 + bc3;
    double p[4];
    p[0] = vb > 0 ? (double)bc0 / (double)vb : 0.25;
    p[1] = vb > 0 ? (double)bc1 / (double)vb : 0.25;
    p[2] = vb > 0 ? (double)bc2 / (double)vb : 0.25;
    p[3] = vb > 0 ? (double)bc3 / (double)vb : 0.25;
    const double inv = 1.0 / (double)tot;
    for (int v0 = 0; v0 < nb; v0 += 32) {
      const int v = v0 + lane;
      double w = 0.0;
      if (v < nb) {
        const uint32_t cnt = hist[v];
        if (cnt) {
          if (a.gc_norm == 0) {
            w = (double)cnt * inv;
          } else {
            double pf = 1.0, pr = 1.0;
            uint32_t code = (uint32_t)v;
            for (int q = 0; q < k; ++q) {
              const uint32_t b = code & 3u;
              pf = __dmul_rn(pf, p[b]);
              pr = __dmul_rn(pr, p[3u - b]);
              code >>= 2;
            }
            const double obs = (double)cnt * inv;
            const double ex = __dadd_rn(pf, pr);
            if (ex > 1e-14) {
              const double r = obs / ex;
              w = (a.gc_cap < r) ? a.gc_cap : r;
            }
          }
        }
      }
      const bool take = w > 0.0;
      const uint32_t bal = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int q = pos + __popc(bal & ((1u << lane) - 1u));
        eidx[q] = (uint8_t)a.rank_of_code[v];
        ewinv[q] = 1.0 / w;
      }
      pos += __popc(bal);
    }
  }
  if (lane == 0) a.elem_cnt[c] = pos;
}

// CTA per contig: register r gets the first-inserted element with the smallest
// offer (1/w_e) * U_e(r); its code and folded winner are written out.
__global__ void k_minreduce(SketchArgs a) {
  __shared__ uint8_t s_idx[kMaxElems];
  __shared__ double s_winv[kMaxElems];
  const int64_t c = blockIdx.x;
  const int cnt = a.elem_cnt[c];
  for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
    s_idx[q] = a.elem_idx[c * kMaxElems + q];
    s_winv[q] = a.elem_winv[c * kMaxElems + q];
  }
  __syncthreads();
  const int m = a.m;
  uint8_t *rowA = a.codesA + c * a.mpad;
  uint8_t *rowB = a.codesB + c * a.mpad;
  for (int r = threadIdx.x; r < a.mpad; r += blockDim.x) {
    if (r >= m) { rowA[r] = 0; rowB[r] = 0xFF; continue; }
    double best = __longlong_as_double(0x7FF0000000000000LL);   // +inf
    int win = -1;
    for (int q = 0; q < cnt; ++q) {
      const int e = s_idx[q];
      const double hv = __dmul_rn(s_winv[q], __ldg(a.U + (size_t)e * m + r));
      if (hv < best) { best = hv; win = e; }
    }
    uint8_t code = 0;
    uint32_t w32 = 0;
    if (win >= 0) {
      code = __ldg(a.codeA + (size_t)win * m + r);
      w32 = __ldg(a.W32 + (size_t)win * m + r);
    }
    rowA[r] = code;
    rowB[r] = code ? code : (uint8_t)0xFF;
    if (a.winners32) a.winners32[c * m + r] = w32;
  }
}

}  // namespace

void launch_pack(const char *ascii, int64_t nbases, uint32_t *packed, uint32_t *nmask,
                 cudaStream_t s) {
  const int64_t nwords = (nbases + 15) / 16;
  if (nwords == 0) return;
  const int tb = 256;
  const int64_t grid = (nwords + tb - 1) / tb;
  k_pack<<<(unsigned)grid, tb, 0, s>>>((const uint4 *)ascii, nbases, nwords, packed, nmask);
}

void launch_count(const SketchArgs &a, cudaStream_t s) {
  if (a.n == 0) return;
  const int warps = 8;
  const int64_t grid = (a.n + warps - 1) / warps;
  k_count<<<(unsigned)grid, warps * 32, warps * 256 * sizeof(uint32_t), s>>>(a);
}

void launch_minreduce(const SketchArgs &a, cudaStream_t s) {
  if (a.n == 0) return;
  k_minreduce<<<(unsigned)a.n, 128, 0, s>>>(a);
}

}  // namespace rbg
