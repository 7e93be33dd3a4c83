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
                       int64_t w_begin, int64_t w_end, uint32_t *__restrict__ packed,
                       uint32_t *__restrict__ nmask) {
  // w_begin is even, so lane pairs (2i, 2i+1) hold the word pairs of one mask word
  const int64_t w = w_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t word = 0, bad16 = 0;
  if (w < w_end) {
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
  if (w < w_end && (threadIdx.x & 1) == 0) {
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

// Spread the 16 bits of x to the even bit positions of a 32-bit word.
__device__ __forceinline__ uint32_t spread16(uint32_t x) {
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// Warp per contig: histogram of canonical k-mers (k <= 4) and base counts over
// the packed sequence, then the GC-normalised weights of build_pmh_winners
// (src/rabbitbin.cpp:1459-1516) and the ascending element list (rank, 1/w).
// A lane takes one packed word (16 bases) per step, the 3 bases before it come
// from the previous lane; base counts use popcounts over the 2-bit fields and a
// shared table maps each k-mer code to its canonical code.
__global__ void k_count(SketchArgs a) {
  extern __shared__ uint32_t sh_hist[];
  __shared__ uint8_t canon[256];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  const int nb = 1 << (2 * a.k);
  const int k = a.k;
  for (int v = threadIdx.x; v < nb; v += blockDim.x) {
    uint32_t rev = 0, x = (uint32_t)v;
    for (int q = 0; q < k; ++q) { rev = (rev << 2) | (3u - (x & 3u)); x >>= 2; }
    canon[v] = (uint8_t)((uint32_t)v <= rev ? (uint32_t)v : rev);
  }
  uint32_t *hist = sh_hist + wib * 256;
  for (int v = lane; v < 256; v += 32) hist[v] = 0;
  __syncthreads();
  if (c >= a.n) return;
  const int64_t s = a.offsets[c], e = a.offsets[c + 1];
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
        // base counts of the valid bases (base t occupies bits 31-2t .. 30-2t)
        const uint32_t vs = spread16(~bad & 0xFFFFu);
        const uint32_t hi = (cur >> 1) & 0x55555555u, lo = cur & 0x55555555u;
        bc3 += __popc(hi & lo & vs);
        bc2 += __popc(hi & ~lo & vs);
        bc1 += __popc(~hi & lo & vs);
        bc0 += __popc(~hi & ~lo & vs);
        // k-mers ending at base t: window bases t-k+1 .. t all valid
        const uint32_t winbad = (prevbad << 16) | bad;
        uint32_t any = winbad;
        for (int q = 1; q < k; ++q) any |= winbad >> q;
        uint32_t kv = ~any & 0xFFFFu;                   // bit 15-t: k-mer ending at t
        const uint64_t win = ((uint64_t)prev << 32) | cur;
        while (kv) {
          const int bp = __ffs(kv) - 1;                 // = 15 - t
          kv &= kv - 1;
          const uint32_t fwd = (uint32_t)(win >> (2 * bp)) & kmask;
          atomicAdd(&hist[canon[fwd]], 1u);
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
  double *ewinv = a.elem_winv + c * a.n_elems;
  const double inf = __longlong_as_double(0x7FF0000000000000LL);
  const uint64_t vb = (uint64_t)bc0 + bc1 + bc2 + bc3;
  double p[4];
  p[0] = vb > 0 ? (double)bc0 / (double)vb : 0.25;
  p[1] = vb > 0 ? (double)bc1 / (double)vb : 0.25;
  p[2] = vb > 0 ? (double)bc2 / (double)vb : 0.25;
  p[3] = vb > 0 ? (double)bc3 / (double)vb : 0.25;
  const double inv = tot > 0 ? 1.0 / (double)tot : 0.0;
  for (int v0 = 0; v0 < nb; v0 += 32) {
    const int v = v0 + lane;
    double w = 0.0;
    if (v < nb && tot > 0) {
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
    pos += __popc(__ballot_sync(0xffffffffu, take));
    const int e = v < nb ? a.rank_of_code[v] : -1;
    if (e >= 0) ewinv[e] = take ? 1.0 / w : inf;
  }
  if (lane == 0) a.elem_cnt[c] = pos;
}

// Register minimum, tiled for reuse of the stream table: a CTA owns a slice of
// 32 registers (lane = register) and walks batches of 32 contigs (warp w holds
// contigs 8w .. 8w+7 of the batch).  The slice U[:, r0:r0+32] and the batch's
// dense 1/w table (+inf for absent elements, which then never win: inf*U is
// inf or NaN, neither is < best) live in shared memory.  Elements are visited
// in ascending order with a strict <, so ties keep the first-inserted element.
constexpr int kMRegs = 32;      // registers per CTA
constexpr int kMCon = 32;       // contigs per batch
constexpr int kMBatches = 4;    // batches per CTA

__global__ void __launch_bounds__(128) k_minreduce(SketchArgs a) {
  extern __shared__ __align__(16) double msh[];
  const int E = a.n_elems, m = a.m;
  double *sU = msh;                               // [E][kMRegs]
  double *sW = msh + (size_t)E * kMRegs;          // [kMCon][E]   1/w, +inf = absent
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = blockIdx.x * kMRegs;
  const int r = r0 + lane;
  for (int i = threadIdx.x; i < E * kMRegs; i += blockDim.x) {
    const int e = i / kMRegs, rr = r0 + (i - e * kMRegs);
    sU[i] = rr < m ? __ldg(a.U + (size_t)e * m + rr) : 0.0;
  }
  const double inf = __longlong_as_double(0x7FF0000000000000LL);
  for (int b = 0; b < kMBatches; ++b) {
    const int64_t c0 = ((int64_t)blockIdx.y * kMBatches + b) * kMCon;
    if (c0 >= a.n) break;
    __syncthreads();
    for (int i = threadIdx.x; i < kMCon * E; i += blockDim.x) {
      const int cl = i / E;
      sW[i] = (c0 + cl < a.n) ? __ldg(a.elem_winv + c0 * E + i) : inf;
    }
    __syncthreads();
    double best[8];
    int win[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) { best[t] = inf; win[t] = -1; }
    const double *wrow = sW + (size_t)warp * 8 * E;     // [8 contigs][E]
    for (int e = 0; e < E; ++e) {
      const double u = sU[e * kMRegs + lane];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const double h = __dmul_rn(wrow[t * E + e], u);
        if (h < best[t]) { best[t] = h; win[t] = e; }
      }
    }
    if (r < m) {
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int64_t c = c0 + warp * 8 + t;
        if (c >= a.n) break;
        uint8_t code = 0;
        uint32_t w32 = 0;
        if (win[t] >= 0) {
          code = __ldg(a.codeA + (size_t)win[t] * m + r);
          w32 = __ldg(a.W32 + (size_t)win[t] * m + r);
        }
        a.codesA[c * a.mpad + r] = code;
        a.codesB[c * a.mpad + r] = code ? code : (uint8_t)0xFF;
        if (a.winners32) a.winners32[c * m + r] = w32;
      }
    }
  }
}

}  // namespace

void launch_pack(const char *ascii, int64_t nbases, uint32_t *packed, uint32_t *nmask,
                 cudaStream_t s) {
  launch_pack_range(ascii, nbases, 0, (nbases + 15) / 16, packed, nmask, s);
}

void launch_pack_range(const char *ascii, int64_t nbases, int64_t w_begin, int64_t w_end,
                       uint32_t *packed, uint32_t *nmask, cudaStream_t s) {
  const int64_t nwords = (nbases + 15) / 16;
  if (w_end > nwords) w_end = nwords;
  if (w_end <= w_begin) return;
  const int tb = 256;
  const int64_t grid = (w_end - w_begin + tb - 1) / tb;
  k_pack<<<(unsigned)grid, tb, 0, s>>>((const uint4 *)ascii, nbases, nwords, w_begin, w_end,
                                      packed, nmask);
}

void launch_count(const SketchArgs &a, cudaStream_t s) {
  if (a.n == 0) return;
  const int warps = 8;
  const int64_t grid = (a.n + warps - 1) / warps;
  k_count<<<(unsigned)grid, warps * 32, warps * 256 * sizeof(uint32_t), s>>>(a);  // + 256 B static
}

void launch_minreduce(const SketchArgs &a, cudaStream_t s) {
  if (a.n == 0) return;
  // padding registers [m, mpad): A = 0, B = 0xFF (never equal)
  cudaMemsetAsync(a.codesA, 0, (size_t)a.n * a.mpad, s);
  cudaMemsetAsync(a.codesB, 0xFF, (size_t)a.n * a.mpad, s);
  const size_t smem = (size_t)a.n_elems * (kMRegs + kMCon) * sizeof(double);
  cudaFuncSetAttribute(k_minreduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const dim3 grid((unsigned)((a.m + kMRegs - 1) / kMRegs),
                  (unsigned)((a.n + kMCon * kMBatches - 1) / (kMCon * kMBatches)));
  k_minreduce<<<grid, 128, smem, s>>>(a);
}

}  // namespace rbg
