// Sketch stage kernels: 2-bit packing, canonical k-mer counting with GC-norm
// weights, and the ProbMinHash register minimum.
//
// Compiled with -fmad=false: every double operation below rounds exactly like
// the reference's (which has no contracted expression in build_pmh_winners).
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <set>
#include <utility>

#include "rbg_internal.h"

namespace rbg {
namespace {

// Base encoding: A/a->0, C/c->1, G/g->2, T/t->3, anything else invalid
// (RB_BASE_ENC_LUT, src/rabbit_sketch.h:56-75).
// One thread per 32 bases: two 128-bit loads of ASCII, two packed words out
// (first base in the top two bits) and the mask word of the pair (16 invalid
// bits per word, the first word in the high half).  Four bases per 32-bit
// step: with l = byte | 0x20, ((l >> 1) ^ (l >> 2)) & 3 is 0, 1, 2, 3 for a,
// c, g, t; the letter rebuilt from that code (a byte permute of "acgt") equals
// l exactly for the eight valid letters, which a zero-byte test of the
// difference marks.  Two multiplies gather the four codes and the four invalid
// bits, first base highest.  Bases past nbases are invalid.
__device__ __forceinline__ void pack16(const uint4 v, int64_t w, int64_t nbases, uint32_t &word,
                                       uint32_t &bad16) {
  word = 0;
  bad16 = 0;
  const uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t l = q[k] | 0x20202020u;
    uint32_t cw = ((l >> 1) ^ (l >> 2)) & 0x03030303u;
    const uint32_t sel = (cw & 0x3u) | ((cw >> 4) & 0x30u) | ((cw >> 8) & 0x300u) |
                         ((cw >> 12) & 0x3000u);
    const uint32_t y = __byte_perm(0x74676361u, 0u, sel) ^ l;
    const uint32_t ok = ~(((y & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | y) & 0x80808080u;
    const uint32_t b = (ok ^ 0x80808080u) >> 7;          // 0x01 in each invalid byte
    cw &= ~(b * 3u);
    const uint32_t c8 = (uint32_t)(((uint64_t)cw * 0x40100401ull) >> 24) & 0xFFu;
    const uint32_t b4 = (uint32_t)(((uint64_t)b * 0x08040201ull) >> 24) & 0xFu;
    word |= c8 << (24 - 8 * k);
    bad16 |= b4 << (12 - 4 * k);
  }
  const int64_t lim = nbases - w * 16;
  if (lim < 16) {
    const int keep = lim > 0 ? (int)lim : 0;
    bad16 |= 0xFFFFu >> keep;
    word &= ~(0xFFFFFFFFu >> (2 * keep));
  }
}

// Words [w_begin, w_end) (w_begin even): thread t packs words w_begin + 2t, + 1.
__global__ void k_pack(const uint4 *__restrict__ ascii, int64_t nbases, int64_t nwords,
                       int64_t w_begin, int64_t w_end, uint32_t *__restrict__ packed,
                       uint32_t *__restrict__ nmask) {
  const int64_t w = w_begin + 2 * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x);
  if (w >= w_end) return;
  const bool two = w + 1 < w_end;
  const uint4 v0 = ascii[w];
  const uint4 v1 = two ? ascii[w + 1] : make_uint4(0u, 0u, 0u, 0u);
  uint32_t p0, b0, p1, b1;
  pack16(v0, w, nbases, p0, b0);
  pack16(v1, w + 1, nbases, p1, b1);
  if (two) {
    *reinterpret_cast<uint2 *>(packed + w) = make_uint2(p0, p1);   // w even: 8-byte aligned
  } else {
    packed[w] = p0;
  }
  nmask[w >> 1] = (b0 << 16) | ((w + 1 < nwords) ? b1 : 0xFFFFu);
}

// Invalid bits of the 16 bases of packed word wi, restricted to [s, e)
// (base t of the word at bit 15 - t; bases before s or from e on are invalid).
__device__ __forceinline__ uint32_t invalid16(const uint32_t *__restrict__ nmask, int64_t wi,
                                              int64_t s, int64_t e) {
  if (wi < 0) return 0xFFFFu;
  const uint32_t mw = __ldg(nmask + (wi >> 1));
  uint32_t b = (wi & 1) ? (mw & 0xFFFFu) : (mw >> 16);
  const int64_t g0 = wi * 16;
  const int64_t dl = s - g0, dh = e - g0;             // first valid, first invalid offset
  if (dl > 0) b |= dl >= 16 ? 0xFFFFu : (0xFFFFu << (16 - (int)dl)) & 0xFFFFu;
  if (dh < 16) b |= dh <= 0 ? 0xFFFFu : 0xFFFFu >> (int)dh;
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
template <bool GC2>                    // GC-norm mode 2 (dinucleotide model)
__global__ void k_count(SketchArgs a) {
  extern __shared__ uint32_t sh_hist[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nb = 1 << (2 * a.k);
  const int k = a.k;
  uint32_t *hist = sh_hist + wib * 256;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  // Each warp takes its next contig from a.work (a counter zeroed before the
  // launch) when the caller gives one, else every warps-th contig: contig
  // lengths vary by an order of magnitude, and the counter keeps every warp
  // busy until the last contigs.
  auto next_contig = [&](int64_t cur) -> int64_t {
    if (a.work == nullptr) return cur + warps;
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(a.work, 1u);
    return (int64_t)__shfl_sync(0xffffffffu, t, 0);
  };
  const int64_t c_first = a.work ? next_contig(0)
                                 : (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  for (int64_t c = c_first; c < a.n; c = next_contig(c)) {
  for (int v = lane; v < 256; v += 32) hist[v] = 0;
  __syncwarp();
  const int64_t s = a.offsets[c], e = a.offsets[c + 1];
  const uint32_t kmask = (uint32_t)nb - 1u;
  uint32_t bc0 = 0, bc1 = 0, bc2 = 0, bc3 = 0;
  uint32_t dn[GC2 ? 16 : 1] = {};      // mode 2: dinucleotides (prev, next) = dn[4 prev + next]
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
        if constexpr (GC2) {
          // consecutive valid bases (t-1, t); base -1 is the previous word's last
          const uint32_t vprev = ((((~prevbad & 0xFFFFu) << 16) | (~bad & 0xFFFFu)) >> 1) & 0xFFFFu;
          const uint32_t vp = spread16(~bad & vprev & 0xFFFFu);
          const uint32_t q = (uint32_t)((((uint64_t)prev << 32) | cur) >> 2);
          const uint32_t qh = (q >> 1) & 0x55555555u, ql = q & 0x55555555u;
          const uint32_t mb[4] = {~hi & ~lo & vp, ~hi & lo & vp, hi & ~lo & vp, hi & lo & vp};
          const uint32_t ma[4] = {~qh & ~ql, ~qh & ql, qh & ~ql, qh & ql};
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) dn[4 * x + y] += __popc(ma[x] & mb[y]);
        }
        // k-mers ending at base t: window bases t-k+1 .. t all valid; forward
        // codes are counted and folded onto canonical codes per contig
        const uint32_t winbad = (prevbad << 16) | bad;
        uint32_t any = winbad;
        for (int q = 1; q < k; ++q) any |= winbad >> q;
        uint32_t kv = ~any & 0xFFFFu;                   // bit 15-t: k-mer ending at t
        const uint64_t win = ((uint64_t)prev << 32) | cur;
        if (kv == 0xFFFFu && k == 4) {
          // the 16 codes are the bytes of the window shifted by 0, 2, 4 and 6 bits
          const uint32_t sw[4] = {cur, __funnelshift_r(cur, prev, 2),
                                  __funnelshift_r(cur, prev, 4), __funnelshift_r(cur, prev, 6)};
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) atomicAdd(&hist[__byte_perm(sw[x], 0u, 0x4440u + y)], 1u);
        } else if (kv == 0xFFFFu) {
#pragma unroll
          for (int bp = 15; bp >= 0; --bp)
            atomicAdd(&hist[(uint32_t)(win >> (2 * bp)) & kmask], 1u);
        } else {
          while (kv) {
            const int bp = __ffs(kv) - 1;               // = 15 - t
            kv &= kv - 1;
            atomicAdd(&hist[(uint32_t)(win >> (2 * bp)) & kmask], 1u);
          }
        }
      }
    }
  }
  __syncwarp();
  // fold each reverse-complement code onto its canonical (the smaller) code
  for (int v = lane; v < nb; v += 32) {
    uint32_t rev = 0, x = (uint32_t)v;
    for (int q = 0; q < k; ++q) { rev = (rev << 2) | (3u - (x & 3u)); x >>= 2; }
    if ((uint32_t)v < rev) {
      hist[v] += hist[rev];
      hist[rev] = 0;
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
  // mode 2 (src/rabbitbin.cpp:1517-1554): base frequencies with pseudocount 1,
  // P(next | prev) with Laplace pseudocount 1
  double pm[4], pc[GC2 ? 16 : 1];
  if constexpr (GC2) {
#pragma unroll
    for (int x = 0; x < 16; ++x) dn[x] = __reduce_add_sync(0xffffffffu, dn[x]);
    const uint32_t bcs[4] = {bc0, bc1, bc2, bc3};
#pragma unroll
    for (int b = 0; b < 4; ++b)
      pm[b] = vb > 0 ? ((double)bcs[b] + 1.0) / ((double)vb + 4.0) : 0.25;
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      double rs = 4.0;
#pragma unroll
      for (int y = 0; y < 4; ++y) rs += (double)dn[4 * x + y];
#pragma unroll
      for (int y = 0; y < 4; ++y) pc[4 * x + y] = ((double)dn[4 * x + y] + 1.0) / rs;
    }
  }
  for (int v0 = 0; v0 < nb; v0 += 32) {
    const int v = v0 + lane;
    double w = 0.0;
    if (v < nb && tot > 0) {
      const uint32_t cnt = hist[v];
      if (cnt) {
        if (a.gc_norm == 0) {
          w = (double)cnt * inv;
        } else if constexpr (GC2) {
          // bases[i] = (v >> 2i) & 3; forward and reverse-complement chains
          uint32_t bs[4];
          for (int q = 0; q < k; ++q) bs[q] = ((uint32_t)v >> (2 * q)) & 3u;
          double pf = pm[bs[0]];
          for (int q = 1; q < k; ++q) pf = __dmul_rn(pf, pc[4 * bs[q - 1] + bs[q]]);
          double pr = pm[3u - bs[k - 1]];
          for (int q = 1; q < k; ++q) pr = __dmul_rn(pr, pc[4 * (3u - bs[k - q]) + (3u - bs[k - 1 - q])]);
          const double obs = (double)cnt * inv;
          const double ex = __dadd_rn(pf, pr);
          if (ex > 1e-16) {
            const double r = obs / ex;
            w = (a.gc_cap < r) ? a.gc_cap : r;
          }
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
  __syncwarp();                        // the next contig clears the histogram
  }
}

// Register minimum with an exact early exit.  The winner of register r for a
// contig is the element e with the smallest rounded product h = (1/w_e) * U[e][r],
// ties to the smallest e (the reference inserts elements in ascending order with
// a strict <), so the result is the lexicographic minimum of (h, e).
//
// Per contig, the kMHeavy elements with the smallest 1/w are evaluated directly;
// the others are bounded below by wb, the next smallest 1/w.  The elements of
// register r are then visited in ascending U (table `order`, ties by e): once
// round(wb * U_next) > best, no element left can reach best, since each remaining
// element is either already evaluated or has 1/w >= wb and U >= U_next, and a
// rounded product is monotonic in both factors.  Elements met again on the walk
// change nothing.  Absent elements (1/w = +inf) give inf or NaN, never below or
// equal to a finite best.
//
// A CTA holds 32 contigs (lane = contig) with their 1/w rows transposed in shared
// memory ([E][32]: the per-step gather is conflict-free).  Each warp takes one
// register at a time: the first 32 entries of its visiting order and its U row
// (by element, table UT) are loaded into registers one register ahead, stored in
// the warp's shared slot, and walked in lock step until every lane's bound has
// passed (entries past 32 come straight from the table).  Winners go to a shared
// tile and leave as 4-byte code words, padding columns included.
constexpr int kMC = 32;          // contigs per CTA, one per lane
constexpr int kMThreads = 256;
constexpr int kMWarps = kMThreads / 32;
constexpr int kMHeavy = 8;       // smallest-1/w elements evaluated directly
constexpr int kMChunk = 256;     // registers per pass; a multiple of 16
constexpr int kMWinStride = kMChunk + 4;
constexpr int kMRec = 32;        // visiting-order entries staged per register (one per lane)
constexpr int kMUcPerLane = (kMaxElems / 2 + 31) / 32;   // 16-byte chunks of a U row per lane
static_assert(kMaxElems % 2 == 0 && kMaxElems <= 5 * 32, "U rows in 16-byte chunks, 5 values per lane");

__host__ __device__ constexpr size_t minreduce_smem(int E) {
  return (size_t)E * kMC * sizeof(double)            // sW   [E][kMC]
         + (size_t)kMHeavy * kMC * sizeof(double)     // sHw  [kMHeavy][kMC]
         + (size_t)kMC * sizeof(double)               // sWb  [kMC]
         + (size_t)kMWarps * kMRec * 16               // sRec [kMWarps][kMRec]
         + (size_t)kMWarps * E * sizeof(double)       // sUc  [kMWarps][E]
         + (size_t)kMHeavy * kMC                      // sHe  [kMHeavy][kMC]
         + (size_t)kMC * kMWinStride;                 // sWin [kMC][kMWinStride]
}

__device__ __forceinline__ void lex_min(double h, int e, double &best, int &win) {
  if (h < best || (h == best && e < win)) {
    best = h;
    win = e;
  }
}

__device__ __forceinline__ void cswap(uint64_t &a, int &ia, uint64_t &b, int &ib) {
  if (b < a) {
    const uint64_t t = a; a = b; b = t;
    const int u = ia; ia = ib; ib = u;
  }
}

// One register's staging data, loaded a register ahead: entry `lane` of the
// visiting order and the lane's 16-byte chunks of the U row.
struct MinStage {
  double2 rec;
  double2 uc[kMUcPerLane];
};

__device__ __forceinline__ void min_fetch(MinStage &st, const double2 *ord, const double2 *ut,
                                          int r, int E, int lane) {
  const int half = E >> 1;
  st.rec = lane < E ? __ldg(ord + (size_t)r * E + lane) : make_double2(0.0, 0.0);
#pragma unroll
  for (int q = 0; q < kMUcPerLane; ++q) {
    const int ch = lane + 32 * q;
    st.uc[q] = ch < half ? __ldg(ut + (size_t)r * half + ch) : make_double2(0.0, 0.0);
  }
}

__global__ void __launch_bounds__(kMThreads, 3) k_minreduce(SketchArgs a) {
  extern __shared__ __align__(16) unsigned char msh[];
  const int E = a.n_elems, m = a.m, mpad = a.mpad;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *sW = reinterpret_cast<double *>(msh);
  double *sHw = sW + (size_t)E * kMC;
  double *sWb = sHw + kMHeavy * kMC;
  double2 *sRec = reinterpret_cast<double2 *>(sWb + kMC);
  double *sUc = reinterpret_cast<double *>(sRec + kMWarps * kMRec);
  uint8_t *sHe = reinterpret_cast<uint8_t *>(sUc + (size_t)kMWarps * E);
  uint8_t *sWin = sHe + kMHeavy * kMC;
  double2 *myRec = sRec + warp * kMRec;
  double *myUc = sUc + (size_t)warp * E;
  const int64_t c0 = (int64_t)blockIdx.x * kMC;
  const int nc = (int)(a.n - c0 < kMC ? a.n - c0 : kMC);
  const double inf = __longlong_as_double(0x7FF0000000000000LL);
  const uint64_t kNone = ~0ull;                      // key of a slot that is no element
  for (int i = threadIdx.x; i < kMC * E; i += kMThreads) {
    const int c = i / E, e = i - c * E;
    sW[e * kMC + c] = c < nc ? __ldg(a.elem_winv + c0 * E + i) : inf;
  }
  // Heavy sets.  A non-negative double orders as its bit pattern, so 1/w values
  // are compared as 64-bit keys.  Each lane sorts its (up to 5) values; kMHeavy + 1
  // rounds of a warp minimum over the lanes' heads take one element each (the
  // lowest lane on ties), the last round giving the bound.
  for (int c = warp; c < kMC; c += kMWarps) {
    uint64_t v[5];
    int id[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const int e = lane + 32 * j;
      id[j] = e;
      v[j] = (c < nc && e < E) ? (uint64_t)__double_as_longlong(__ldg(a.elem_winv + (c0 + c) * E + e))
                                : kNone;
    }
    cswap(v[0], id[0], v[1], id[1]); cswap(v[3], id[3], v[4], id[4]);
    cswap(v[2], id[2], v[4], id[4]); cswap(v[2], id[2], v[3], id[3]);
    cswap(v[0], id[0], v[3], id[3]); cswap(v[0], id[0], v[2], id[2]);
    cswap(v[1], id[1], v[4], id[4]); cswap(v[1], id[1], v[3], id[3]);
    cswap(v[1], id[1], v[2], id[2]);
    for (int i = 0; i <= kMHeavy; ++i) {
      uint64_t mn = v[0];
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        const uint64_t ov = __shfl_xor_sync(0xffffffffu, mn, o);
        mn = ov < mn ? ov : mn;
      }
      const int src = __ffs(__ballot_sync(0xffffffffu, v[0] == mn)) - 1;
      const int ej = __shfl_sync(0xffffffffu, id[0], src);
      if (i < kMHeavy) {
        if (lane == src) {
#pragma unroll
          for (int j = 0; j < 4; ++j) { v[j] = v[j + 1]; id[j] = id[j + 1]; }
          v[4] = kNone;
        }
        if (lane == 0) {
          const bool real = mn != kNone;
          sHe[i * kMC + c] = real ? (uint8_t)ej : (uint8_t)0;
          sHw[i * kMC + c] = real ? __longlong_as_double((long long)mn) : inf;
        }
      } else if (lane == 0) {
        sWb[c] = mn != kNone ? __longlong_as_double((long long)mn) : inf;
      }
    }
  }
  __syncthreads();
  int he[kMHeavy];
  double hw[kMHeavy];
#pragma unroll
  for (int i = 0; i < kMHeavy; ++i) {
    he[i] = sHe[i * kMC + lane];
    hw[i] = sHw[i * kMC + lane];
  }
  const double wb = sWb[lane];
  const bool empty = lane >= nc || !(hw[0] < inf);
  const double2 *ord = reinterpret_cast<const double2 *>(a.order);
  const double2 *ut = reinterpret_cast<const double2 *>(a.UT);
  const int half = E >> 1;
  for (int rb = 0; rb < mpad; rb += kMChunk) {
    const int rn = (m - rb < kMChunk) ? m - rb : kMChunk;
    MinStage st;
    if (warp < rn) min_fetch(st, ord, ut, rb + warp, E, lane);
    for (int rl = warp; rl < rn; rl += kMWarps) {
      const int r = rb + rl;
      myRec[lane] = st.rec;
#pragma unroll
      for (int q = 0; q < kMUcPerLane; ++q) {
        const int ch = lane + 32 * q;
        if (ch < half) reinterpret_cast<double2 *>(myUc)[ch] = st.uc[q];
      }
      __syncwarp();
      if (rl + kMWarps < rn) min_fetch(st, ord, ut, r + kMWarps, E, lane);
      double best = inf;
      int win = -1;
      bool done = empty;
      if (!done) {
#pragma unroll
        for (int i = 0; i < kMHeavy; ++i) lex_min(__dmul_rn(hw[i], myUc[he[i]]), he[i], best, win);
      }
      for (int k = 0; k < E; ++k) {
        if (__all_sync(0xffffffffu, done)) break;
        const double2 v = k < kMRec ? myRec[k] : __ldg(ord + (size_t)r * E + k);
        if (!done) {
          if (__dmul_rn(wb, v.x) > best) {
            done = true;
          } else {
            const int e = (int)__double_as_longlong(v.y);
            lex_min(__dmul_rn(sW[e * kMC + lane], v.x), e, best, win);
          }
        }
      }
      if (lane < nc) sWin[lane * kMWinStride + rl] = win < 0 ? (uint8_t)0xFF : (uint8_t)win;
      __syncwarp();
    }
    __syncthreads();
    // code words: columns [rb, rend) of the nc rows; padding columns A = 0, B = 0xFF
    const int rend = (rb + kMChunk < mpad) ? rb + kMChunk : mpad;
    const int q4 = (rend - rb) >> 2;
    for (int i = threadIdx.x; i < nc * q4; i += kMThreads) {
      const int cc = i / q4, rl = (i - cc * q4) * 4, r4 = rb + rl;
      const uint32_t wins = *reinterpret_cast<const uint32_t *>(sWin + cc * kMWinStride + rl);
      uint32_t va = 0, vb = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int rr = r4 + b;
        uint32_t code = 0;
        if (rr < m) {
          const uint32_t wi = (wins >> (8 * b)) & 0xFFu;
          uint32_t w32 = 0;
          if (wi != 0xFFu) {
            code = __ldg(a.codeA + (size_t)wi * m + rr);
            w32 = __ldg(a.W32 + (size_t)wi * m + rr);
          }
          if (a.winners32) a.winners32[(c0 + cc) * m + rr] = w32;
          if (a.win_elem) a.win_elem[(c0 + cc) * m + rr] = (uint8_t)wi;
        }
        va |= code << (8 * b);
        vb |= (code ? code : 0xFFu) << (8 * b);
      }
      *reinterpret_cast<uint32_t *>(a.codesA + (c0 + cc) * mpad + r4) = va;
      *reinterpret_cast<uint32_t *>(a.codesB + (c0 + cc) * mpad + r4) = vb;
    }
    __syncthreads();
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
  const int64_t pairs = (w_end - w_begin + 1) / 2;
  const int64_t grid = (pairs + tb - 1) / tb;
  k_pack<<<(unsigned)grid, tb, 0, s>>>((const uint4 *)ascii, nbases, nwords, w_begin, w_end,
                                      packed, nmask);
}

namespace {

// Column-side codes from row-side ones: B = A, with 0xFF where A is 0 (unset).
__global__ void k_codes_b(const uint4 *__restrict__ A, uint4 *__restrict__ B, int64_t n16) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n16) return;
  const uint4 a = A[i];
  uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    // 0x80 in each zero byte (the add cannot carry out of a byte)
    const uint32_t z = ~(((w[q] & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | w[q]) & 0x80808080u;
    w[q] |= (z >> 7) * 0xFFu;
  }
  B[i] = make_uint4(w[0], w[1], w[2], w[3]);
}

}  // namespace

void launch_codes_b(const uint8_t *codesA, uint8_t *codesB, int64_t bytes, cudaStream_t s) {
  const int64_t n16 = bytes / 16;
  if (n16 == 0) return;
  k_codes_b<<<(unsigned)((n16 + 255) / 256), 256, 0, s>>>((const uint4 *)codesA, (uint4 *)codesB,
                                                          n16);
}

void launch_count(const SketchArgs &a, cudaStream_t s) {
  if (a.n == 0) return;
  const int warps = 8;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // with the contig counter, as many warps as fit (five blocks of 48-register
  // threads per SM); without it, about eight contigs per warp to even out the
  // contig lengths
  const int64_t blocks = (a.n + warps - 1) / warps;
  const int64_t grid =
      std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)sms * (a.work ? 5 : 4)));
  if (a.gc_norm == 2)
    k_count<true><<<(unsigned)grid, warps * 32, warps * 256 * sizeof(uint32_t), s>>>(a);
  else
    k_count<false><<<(unsigned)grid, warps * 32, warps * 256 * sizeof(uint32_t), s>>>(a);
}

void smem_cap_max(const void *func) {
  static std::mutex mu;
  static std::set<std::pair<int, const void *>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (!done.insert({dev, func}).second) return;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, func) != cudaSuccess) return;   // the launch reports it
  cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       optin - (int)fa.sharedSizeBytes);
}

void launch_minreduce(const SketchArgs &a, cudaStream_t s) {
  if (a.n == 0) return;
  const size_t smem = minreduce_smem(a.n_elems);
  smem_cap_max((const void *)k_minreduce);
  const int64_t grid = (a.n + kMC - 1) / kMC;
  k_minreduce<<<(unsigned)grid, kMThreads, smem, s>>>(a);
}

namespace {

// ── One-permutation MinHash (the RABBIT_PMH=0 metric, src/rabbit_sketch.h) ──
// KmerSketch::update (src/rabbit_sketch.h:199-238): every window of K bases
// that are all A/C/G/T offers h = murmur3_fmix(min(forward, reverse
// complement), seed) to bucket ((h >> 32) * m) >> 32 with value (uint32_t)h,
// kept if smaller.  buildSig (:264-281) gives an empty bucket the value that
// densify (:245-259) borrows along its probe sequence, and keeps `bits` low
// bits of every bucket (bit-planes); a sketch with no k-mer at all has an
// all-zero signature.  Here a bucket's kept bits + 1 are its 8-bit code (A
// side; the B side is the same), so equal codes are exactly the buckets whose
// bit-planes all agree (jaccard_raw, src/rabbitbin.cpp:1035-1130).

__device__ __forceinline__ uint64_t oph_fmix(uint64_t x, uint64_t seed) {
  x ^= seed;
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

__device__ __forceinline__ uint32_t oph_bucket(uint64_t h, uint32_t m) {
  return (uint32_t)(((h >> 32) * (uint64_t)m) >> 32);
}

// Reverse complement of a K-base word (2 bits a base, first base highest).
__device__ __forceinline__ uint64_t oph_revcomp(uint64_t x, int K) {
  x = __brevll(~x);                        // complement, then every bit reversed
  x = ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
  return x >> (64 - 2 * K);                // the base pairs back in order
}

constexpr int kOphWarps = 4;

// Warp per contig (warps stride over the contigs); the warp's m registers in
// shared memory; a lane takes one 16-base word per step and the windows that
// end in it.
__global__ void __launch_bounds__(kOphWarps * 32)
k_oph(SketchArgs a, int K, int bits, uint64_t seed) {
  extern __shared__ uint32_t sh_oph[];
  constexpr uint32_t kEmpty = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t m = (uint32_t)a.m;
  uint32_t *reg = sh_oph + (size_t)wib * m;
  const uint64_t kmask = K >= 32 ? ~0ull : ((1ull << (2 * K)) - 1ull);
  const uint32_t vmask = (1u << bits) - 1u;
  const int64_t warps = (int64_t)gridDim.x * kOphWarps;
  for (int64_t c = (int64_t)blockIdx.x * kOphWarps + wib; c < a.n; c += warps) {
    for (uint32_t r = lane; r < m; r += 32) reg[r] = kEmpty;
    __syncwarp();
    const int64_t s = a.offsets[c], e = a.offsets[c + 1];
    if (e - s >= K) {
      const int64_t w0 = s >> 4, w1 = (e + 15) >> 4;
      uint32_t c1 = 0, c2 = 0, b1 = 0xFFFFu, b2 = 0xFFFFu;   // the two words before w0
      for (int64_t base = w0; base < w1; base += 32) {
        const int64_t wi = base + lane;
        uint32_t cur = 0, bad = 0xFFFFu;
        if (wi < w1) {
          cur = __ldg(a.packed + wi);
          bad = invalid16(a.nmask, wi, s, e);
        }
        uint32_t p1 = __shfl_up_sync(0xffffffffu, cur, 1), q1 = __shfl_up_sync(0xffffffffu, bad, 1);
        uint32_t p2 = __shfl_up_sync(0xffffffffu, cur, 2), q2 = __shfl_up_sync(0xffffffffu, bad, 2);
        if (lane == 0) { p1 = c1; q1 = b1; p2 = c2; q2 = b2; }
        if (lane == 1) { p2 = c1; q2 = b1; }
        c2 = __shfl_sync(0xffffffffu, cur, 30);
        b2 = __shfl_sync(0xffffffffu, bad, 30);
        c1 = __shfl_sync(0xffffffffu, cur, 31);
        b1 = __shfl_sync(0xffffffffu, bad, 31);
        if (wi >= w1) continue;
        // bit 15 - p: base p of the word (p < 0: the words before); a window
        // ending at base t is valid when bits 15-t .. 15-t+K-1 are all clear
        const uint64_t wbad = ((uint64_t)q2 << 32) | ((uint64_t)q1 << 16) | bad;
        uint64_t any = wbad;
        for (int q = 1; q < K; ++q) any |= wbad >> q;
        uint32_t kv = ~(uint32_t)any & 0xFFFFu;
        const uint64_t lo = ((uint64_t)p1 << 32) | cur;
        while (kv) {
          const int bp = __ffs(kv) - 1;                // = 15 - t
          kv &= kv - 1;
          const int sh = 2 * bp;
          const uint64_t fwd = (sh ? (lo >> sh) | ((uint64_t)p2 << (64 - sh)) : lo) & kmask;
          const uint64_t rc = oph_revcomp(fwd, K);
          const uint64_t h = oph_fmix(fwd < rc ? fwd : rc, seed);
          atomicMin(&reg[oph_bucket(h, m)], (uint32_t)h);
        }
      }
    }
    __syncwarp();
    if (a.oph_keys) {
      // KmerSketch::getKeys (src/rabbit_sketch.h:166-175): one key per
      // non-empty bucket, murmur3_fmix((bucket << 32) | register, seed ^
      // 0x51A3C2B7); 0 marks an empty bucket here (no key)
      for (uint32_t r = lane; r < m; r += 32) {
        const uint32_t v = reg[r];
        a.oph_keys[c * m + r] =
            v == kEmpty ? 0ull : oph_fmix(((uint64_t)r << 32) | v, seed ^ 0x51A3C2B7ull);
      }
      __syncwarp();
      continue;
    }
    uint32_t ne = 0;
    for (uint32_t r = lane; r < m; r += 32) ne += reg[r] != kEmpty;
    ne = __reduce_add_sync(0xffffffffu, ne);
    uint8_t *ca = a.codesA + c * a.mpad, *cb = a.codesB + c * a.mpad;
    for (uint32_t r = lane; r < (uint32_t)a.mpad; r += 32) {
      if (r >= m) {                                    // padding never matches
        ca[r] = 0;
        cb[r] = 0xFF;
        continue;
      }
      uint32_t v = reg[r];
      if (ne == 0) {
        v = 0;
      } else if (v == kEmpty) {
        // densify: the shared probe sequence of bucket r
        const uint64_t pb = oph_fmix((uint64_t)r, seed ^ 0xA5A5A5A5DEADBEEFull);
        const uint64_t step = oph_fmix((uint64_t)r, seed ^ 0x123456789ABCDEF0ull) | 1ull;
        uint64_t cur = pb;
        v = 0;
        for (uint32_t t = 1; t <= m; ++t) {
          cur += step;
          const uint32_t x = reg[oph_bucket(cur, m)];
          if (x != kEmpty) {
            v = x ^ (uint32_t)oph_fmix((uint64_t)t, 0x9E3779B97F4A7C15ull);
            break;
          }
        }
      }
      const uint8_t code = (uint8_t)((v & vmask) + 1u);
      ca[r] = code;
      cb[r] = code;
    }
    __syncwarp();
  }
}

}  // namespace

namespace {
// Bucket values (code - 1) of n code rows, m per row, packed.
__global__ void k_oph_values(const uint8_t *__restrict__ codes, int64_t n, int m, int mpad,
                             uint8_t *__restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * m) return;
  const int64_t i = t / m, r = t - i * m;
  out[t] = (uint8_t)(codes[i * mpad + r] - 1u);
}
}  // namespace

void launch_oph_values(const uint8_t *codes, int64_t n, int m, int mpad, uint8_t *out,
                       cudaStream_t s) {
  if (n <= 0) return;
  const int64_t tot = n * m;
  k_oph_values<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(codes, n, m, mpad, out);
}

void launch_oph(const SketchArgs &a, int K, int bits, uint64_t seed, cudaStream_t s) {
  if (a.n == 0) return;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = (size_t)kOphWarps * a.m * sizeof(uint32_t);
  smem_cap_max((const void *)k_oph);
  const int64_t blocks = (a.n + kOphWarps - 1) / kOphWarps;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)sms * 8));
  k_oph<<<(unsigned)grid, kOphWarps * 32, smem, s>>>(a, K, bits, seed);
}

}  // namespace rbg
