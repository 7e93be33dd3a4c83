// Fisher label propagation on the device: the step after the graph
// (cluster_by_propagation, src/impl/rb_cluster.cpp:376-740), on the incidence
// lists of src/rabbitbin.cpp:5597-5622.
//
// Incidence.  Edges with a score above 0 enter both endpoints' lists, the
// score clamped to 1 - 1e-6 (as a float); each list is ordered by neighbour id
// (ties, i.e. parallel edges, by edge id) and carries, per arc, the per-edge
// quantity the rule accumulates: (float)log(1 - score) for the fisher, tail and
// logsum rules, the score itself for sum, mean and max (rb_cluster.cpp:449-454).
// The log is the correctly rounded one (ddmath.cuh).
//
// Gauss-Seidel sweep (the default).  The reference visits the nodes one after
// the other in node_order; a node sees the labels its earlier neighbours were
// given in the same round.  Here every warp claims the next position of the
// order (one atomic counter, so positions are claimed in order by running
// warps), waits until each neighbour that comes earlier in the order has been
// visited in this round (a per-node round stamp, published with release
// semantics after the node's writes), and then decides exactly as the
// sequential loop would: the labels of earlier neighbours are final for the
// round, those of later neighbours still hold the previous round's value
// (a later neighbour waits for this node before it writes).  Waiting only on
// positions that were claimed before cannot deadlock: the earliest unfinished
// claim has nothing left to wait for.  Every wait is bounded (5 s of
// %globaltimer, or at once after another warp gave up); a wait that runs out
// records RBG_ERR_TIMEOUT for the host and the kernel winds down.
//
// Per node the warp streams its arcs 32 at a time: each lane reads one
// neighbour's label, lanes holding the same label are grouped (match.any) and
// the group's lowest lane adds the group's quantities to that label's running
// score one by one in arc order, so every label's score is the reference's
// left-to-right double sum.  Labels live in a per-warp hash table (shared
// memory up to 256 arcs, a per-warp global table above), and the labels in
// order of first appearance in a list, which gives the reference's first-max
// tie-break.  The decision (keep the current label when it is within 1e-12 of
// the best), the cycle guard (a node that returns to a label it had is frozen)
// and the re-activation of the neighbours of a node that changed follow the
// reference line by line.
//
// Synchronous sweep (RABBIT_PAR_LPA, rb_cluster.cpp:490-594): every active
// node proposes from the round's snapshot, then the proposals are committed.
// The reference commits in node_order, but a commit writes only the node's own
// label, visited set and freeze flag (plus idempotent activation marks), so
// committing all nodes at once gives the same state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "ddmath.cuh"
#include "rbg_internal.h"

namespace rbg {
namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kLpaWarps = 8;                  // warps per CTA of the sweep kernels
constexpr int kTabSlots = 512;                // shared hash slots per warp
constexpr int kTabMaxDeg = 256;               // arcs above which a node takes the general path
// per-warp shared region: scores, keys, counts, first-appearance list, then the
// arc stage (neighbour / label and quantity per arc, later the label score
// intervals), then a 32-float exchange buffer of the general path
constexpr int kWarpSmem = kTabSlots * 16 + kTabMaxDeg * 4 + kTabMaxDeg * 16 + 32 * 4;
constexpr int kVisitPer = 14;                 // labels per visited-set block
constexpr uint64_t kWaitNs = 5000000000ull;   // bound of one wait

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// State that other launches wrote (labels, flags, visited sets, proposals) is
// read at the L2, never from a line an SM's L1 may still hold from an earlier
// round: ld.global.cg.
__device__ __forceinline__ uint32_t ld_cg(const uint32_t *p) { return __ldcg(p); }
__device__ __forceinline__ uint32_t ld_cg8(const uint8_t *p) {
  uint16_t v;
  asm volatile("ld.global.cg.u8 %0, [%1];" : "=h"(v) : "l"(p));
  return v;
}

// ── the score rules (rb_cluster.cpp:3-22, :40-76) ──────────────────────────
// chi-squared upper tail with 2 m degrees of freedom at x: e^-u sum_{i<m} u^i/i!
__device__ double chi2_sf(int m, double x) {
  const double u = dd::mul(0.5, x);
  double p = dd::exp_cr(-u);
  double Q = p;
  for (int i = 1; i < m; ++i) {
    p = dd::mul(p, __ddiv_rn(u, (double)i));
    Q = dd::add(Q, p);
  }
  return Q;
}
__device__ double lpa_combine(int rule, int m, double acc) {
  switch (rule) {
    case RBG_LPA_FISHER: {
      const double v = dd::sub(1.0, chi2_sf(m, dd::mul(-2.0, acc)));
      return v < 0.0 ? 0.0 : v;
    }
    case RBG_LPA_TAIL: return -chi2_sf(m, dd::mul(-2.0, acc));
    case RBG_LPA_LOGSUM: return -acc;
    case RBG_LPA_MEAN: return m > 0 ? __ddiv_rn(acc, (double)m) : 0.0;
    default: return acc;                                  // sum, max
  }
}
__device__ __forceinline__ void lpa_accumulate(int rule, double &dst, float x) {
  if (rule == RBG_LPA_MAX) {
    if ((double)x > dst) dst = (double)x;
  } else {
    dst = dd::add(dst, (double)x);
  }
}

// An interval [lo, hi] that holds lpa_combine(rule, m, acc) without its cost
// (lo == hi: the value itself).  The fisher and tail rules repeat the tail sum
// with the library exp (within 1 ulp) and u * (1/i) (inv[i] = RN(1/i)) in place
// of the correctly rounded exp and u / i.  Against the exact evaluation the
// start differs by at most 1.5 ulp and every step of the product chain adds at
// most 5 units of 2^-53 of relative drift (two operand roundings, two product
// roundings, the quotient), the m roundings of each sum another 2^-53 Q each,
// so |Q' - Q| <= (7m + 3) 2^-53 Q' (+ m 2^-1074 for subnormal terms); the bound
// used, (8m + 16) 2^-52 Q' + m 2^-1070, holds it twice over.  The value then
// lies in RN(1 - [Q' - E, Q' + E]) (fisher, monotone) or -[Q' - E, Q' + E]
// (tail).  Below acc = -700 the start is near the subnormal range: there the
// fisher value is exactly 1 when the whole tail sum is below 2^-60 (then the
// computed one is below 2^-54 and 1 - Q rounds to 1), which the largest term
// bounds (u > m - 1, so the terms rise: Q <= m e^-u u^(m-1) / (m-1)!, tested
// with one unit of slack in the log); anything else is evaluated exactly.
__device__ void lpa_interval(int rule, int m, double acc, const double *inv, double *lo,
                             double *hi) {
  if (rule != RBG_LPA_FISHER && rule != RBG_LPA_TAIL) {
    *lo = *hi = lpa_combine(rule, m, acc);              // no exp: exact and cheap
    return;
  }
  const double u = dd::mul(0.5, dd::mul(-2.0, acc));
  if (-u >= -700.0) {
    double p = ::exp(-u);
    double Q = p;
    for (int i = 1; i < m; ++i) {
      p = dd::mul(p, dd::mul(u, inv[i]));
      Q = dd::add(Q, p);
    }
    const double E = __dadd_ru(__dmul_ru(__dmul_ru(8.0 * m + 16.0, 0x1p-52), Q),
                               __dmul_ru((double)m, 0x1p-1070));
    const double tlo = fmax(0.0, __dsub_rd(Q, E)), thi = __dadd_ru(Q, E);
    if (rule == RBG_LPA_FISHER) {
      const double a = dd::sub(1.0, thi), b = dd::sub(1.0, tlo);
      *lo = a < 0.0 ? 0.0 : a;
      *hi = b < 0.0 ? 0.0 : b;
    } else {
      *lo = -thi;
      *hi = -tlo;
    }
    return;
  }
  if (rule == RBG_LPA_FISHER && u > (double)(m - 1)) {
    const double lq = ::log((double)m) - u + (double)(m - 1) * ::log(u) - ::lgamma((double)m);
    if (lq < -60.0 * 0.6931471805599453 - 1.0) {
      *lo = *hi = 1.0;
      return;
    }
  }
  *lo = *hi = lpa_combine(rule, m, acc);
}

// ── incidence ──────────────────────────────────────────────────────────────
// Per edge: validation, the clamp, the accumulated quantity, endpoint degrees.
__global__ void k_lpa_edges(const uint32_t *__restrict__ from, const uint32_t *__restrict__ to,
                            const float *__restrict__ score, int64_t E, int64_t n, int raw,
                            float *__restrict__ q, uint32_t *__restrict__ deg,
                            int *__restrict__ err) {
  const float kMax = 1.0f - 1e-6f;                         // SSCR_MAX, rabbitbin.cpp:5600
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {
    float s = score[e];
    if (s < 0.0f) atomicCAS(err, 0, 1);                   // "edgeScore must be non-negative"
    const bool keep = s > 0.0f;
    if (keep) {
      if (s > kMax) s = kMax;
      const uint32_t a = from[e], b = to[e];
      if ((int64_t)a >= n || (int64_t)b >= n) {
        atomicCAS(err, 0, 2);
        continue;
      }
      atomicAdd(deg + a, 1u);
      atomicAdd(deg + b, 1u);
    }
    q[e] = !keep ? 0.0f : (raw ? s : (float)dd::log_cr(dd::sub(1.0, (double)s)));
  }
}

// Exclusive scan of the degrees into n + 1 offsets, and the largest degree
// (one CTA of 1024).
__global__ void k_lpa_offsets(const uint32_t *__restrict__ deg, int64_t n, int64_t *__restrict__ off,
                              int64_t *__restrict__ maxdeg) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t per = (n + 1023) / 1024;
  const int64_t a = min(n, t * per), b = min(n, a + per);
  int64_t sum = 0;
  uint32_t mx = 0;
  for (int64_t k = a; k < b; ++k) {
    sum += deg[k];
    mx = max(mx, deg[k]);
  }
  mx = __reduce_max_sync(0xFFFFFFFFu, mx);
  if ((t & 31) == 0) atomicMax((unsigned long long *)maxdeg, (unsigned long long)mx);
  part[t] = sum;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int64_t add = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += add;
    __syncthreads();
  }
  int64_t run = t ? part[t - 1] : 0;
  for (int64_t k = a; k < b; ++k) {
    off[k] = run;
    run += deg[k];
  }
  if (t == 1023) off[n] = part[1023];
}

// Arc keys (neighbour << 32 | edge id) into each endpoint's range.
__global__ void k_lpa_scatter(const uint32_t *__restrict__ from, const uint32_t *__restrict__ to,
                             const float *__restrict__ score, int64_t E, int64_t n,
                             const int64_t *__restrict__ off, uint32_t *__restrict__ fill,
                             uint64_t *__restrict__ key) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (!(score[e] > 0.0f)) continue;
    const uint32_t a = from[e], b = to[e];
    if ((int64_t)a >= n || (int64_t)b >= n) continue;
    const uint32_t sa = atomicAdd(fill + a, 1u), sb = atomicAdd(fill + b, 1u);
    key[off[a] + sa] = ((uint64_t)b << 32) | (uint64_t)e;
    key[off[b] + sb] = ((uint64_t)a << 32) | (uint64_t)e;
  }
}

// Ascending sort of len keys at v by a bitonic network whose comparators all
// point the same way (each merge stage starts by comparing mirror positions),
// so positions at or past len act as +infinity and their comparators are
// skipped.  Called by all threads of the CTA.
__device__ void bitonic_sort_keys(uint64_t *v, int64_t len) {
  int64_t N = 1;
  while (N < len) N <<= 1;
  for (int64_t size = 2; size <= N; size <<= 1) {
    for (int64_t t = threadIdx.x; t < N / 2; t += blockDim.x) {
      const int64_t blk = t / (size / 2), r = t - blk * (size / 2);
      const int64_t i = blk * size + r, j = blk * size + size - 1 - r;
      if (j < len && v[j] < v[i]) {
        const uint64_t x = v[i];
        v[i] = v[j];
        v[j] = x;
      }
    }
    __syncthreads();
    for (int64_t stride = size / 4; stride > 0; stride >>= 1) {
      for (int64_t t = threadIdx.x; t < N / 2; t += blockDim.x) {
        const int64_t blk = t / stride, r = t - blk * stride;
        const int64_t i = blk * 2 * stride + r, j = i + stride;
        if (j < len && v[j] < v[i]) {
          const uint64_t x = v[i];
          v[i] = v[j];
          v[j] = x;
        }
      }
      __syncthreads();
    }
  }
}

constexpr int kSortSmem = 4096;                // keys sorted in shared memory

// One CTA per node: its arc keys sorted (shared memory up to 4096 arcs, in
// place in global memory above), then split into neighbour and quantity.
__global__ void __launch_bounds__(256) k_lpa_sort(const int64_t *__restrict__ off, uint64_t *key,
                                                  const float *__restrict__ q,
                                                  uint32_t *__restrict__ nbr,
                                                  float *__restrict__ w) {
  __shared__ uint64_t sk[kSortSmem];
  const int64_t v = blockIdx.x;
  const int64_t a0 = off[v], len = off[v + 1] - a0;
  if (len <= 0) return;
  uint64_t *k = key + a0;
  if (len > 1) {
    if (len <= kSortSmem) {
      for (int64_t i = threadIdx.x; i < len; i += blockDim.x) sk[i] = k[i];
      __syncthreads();
      bitonic_sort_keys(sk, len);
      for (int64_t i = threadIdx.x; i < len; i += blockDim.x) k[i] = sk[i];
    } else {
      bitonic_sort_keys(k, len);
    }
    __syncthreads();
  }
  for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
    const uint64_t x = k[i];
    nbr[a0 + i] = (uint32_t)(x >> 32);
    w[a0 + i] = q[x & 0xFFFFFFFFull];
  }
}

__global__ void k_lpa_init(const uint32_t *__restrict__ order, int64_t n, uint32_t *__restrict__ pos,
                           uint32_t *__restrict__ label, uint8_t *__restrict__ active,
                           uint8_t *__restrict__ next_active, uint8_t *__restrict__ frozen,
                           uint32_t *__restrict__ done, uint32_t *__restrict__ vcnt,
                           uint32_t *__restrict__ vnext) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    pos[order[p]] = (uint32_t)p;
    label[p] = (uint32_t)p;
    active[p] = 1;
    next_active[p] = 0;
    frozen[p] = 0;
    done[p] = 0;
    vcnt[p] = 0;
    vnext[p] = kEmpty;
  }
}

// Per arc: does the neighbour come earlier in the node order than the node?
// Per position: the node there, its degree and first arc.
__global__ void k_lpa_early(const int64_t *__restrict__ off, const uint32_t *__restrict__ nbr,
                            const uint32_t *__restrict__ pos, int64_t n,
                            uint8_t *__restrict__ early, uint4 *__restrict__ rec) {
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int lane = threadIdx.x & 31;
  for (int64_t v = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); v < n; v += nw) {
    const uint32_t pv = pos[v];
    const int64_t a0 = off[v], a1 = off[v + 1];
    for (int64_t a = a0 + lane; a < a1; a += 32) early[a] = pos[nbr[a]] < pv;
    if (lane == 0)
      rec[pv] = make_uint4((uint32_t)v, (uint32_t)(a1 - a0), (uint32_t)a0, (uint32_t)(a0 >> 32));
  }
}

// ── the sweeps ──────────────────────────────────────────────────────────────
struct Sweep {
  int64_t n;
  const int64_t *off;
  const uint32_t *nbr;
  const float *w;
  const uint32_t *order, *pos;
  const uint8_t *early;           // per arc: the neighbour comes earlier in the order
  const uint4 *rec;               // per position: node, degree, first arc (low, high)
  uint32_t *label;
  uint8_t *active, *next_active, *frozen;
  uint32_t *done;                 // round of a node's last visit (Gauss-Seidel)
  uint32_t *prop;                 // proposals (synchronous)
  // visited sets: block v belongs to node v; vcnt[v] labels, spill blocks
  // chained from vnext[v] (kEmpty: none) out of the pool above n
  uint32_t *vlab, *vcnt, *vnext, *vpool_used;
  uint32_t vpool_cap;
  uint32_t *claim;
  unsigned long long *counts;     // [0] changed, [1] frozen this round
  uint32_t *gtab;                 // global tables, gtab_slots per warp
  int gtab_slots;
  int rule;
  uint32_t round;
  int *err;
};

struct Table {                    // per-warp label table
  uint32_t *key;
  int32_t *cnt;
  double *score;
  uint32_t *list;                 // slots in order of first appearance
  int slots;
};

__device__ __forceinline__ uint32_t hslot(uint32_t L, int slots) {
  return (L * 0x9E3779B1u) & (uint32_t)(slots - 1);
}

// Slot of label L (inserted, with a zero score, when absent; *fresh set then).
__device__ __forceinline__ int table_find(Table &T, uint32_t L, bool *fresh) {
  uint32_t h = hslot(L, T.slots);
  for (;;) {
    const uint32_t k = T.key[h];
    if (k == L) {
      *fresh = false;
      return (int)h;
    }
    if (k == kEmpty) {
      const uint32_t old = atomicCAS(T.key + h, kEmpty, L);
      if (old == kEmpty) {
        T.cnt[h] = 0;
        T.score[h] = 0.0;
        *fresh = true;
        return (int)h;
      }
      if (old == L) {
        *fresh = false;
        return (int)h;
      }
    }
    h = (h + 1) & (uint32_t)(T.slots - 1);
  }
}

// Label scores of v's arcs [a0, a1) and the decision of rb_cluster.cpp:532-553:
// returns the chosen label (cur when the list is empty, *touched false then).
__device__ uint32_t decide(const Sweep &S, Table &T, float *wb, uint32_t v, int64_t a0,
                           int64_t a1, uint32_t cur, bool *touched) {
  const int lane = threadIdx.x & 31;
  int nlist = 0;
  for (int64_t c = a0; c < a1; c += 32) {
    const int64_t a = c + lane;
    const bool valid = a < a1;
    uint32_t L = kEmpty;
    if (valid) {
      L = ld_relaxed(S.label + __ldg(S.nbr + a));
      wb[lane] = __ldg(S.w + a);
    }
    __syncwarp();
    const uint32_t grp = __match_any_sync(FULL, L);
    const bool lead = valid && lane == __ffs(grp) - 1;
    bool fresh = false;
    int slot = 0;
    if (lead) {
      slot = table_find(T, L, &fresh);
      double s = T.score[slot];
      for (uint32_t g = grp; g; g &= g - 1) lpa_accumulate(S.rule, s, wb[__ffs(g) - 1]);
      T.score[slot] = s;
      T.cnt[slot] += __popc(grp);
    }
    const uint32_t nb = __ballot_sync(FULL, fresh);
    if (fresh) T.list[nlist + __popc(nb & ((1u << lane) - 1u))] = (uint32_t)slot;
    nlist += __popc(nb);
    __syncwarp();
  }
  *touched = nlist > 0;
  if (nlist == 0) return cur;
  double bv = -INFINITY, cv = -INFINITY;
  int bi = 0x7FFFFFFF;
  uint32_t bk = kEmpty;
  bool cp = false;
  for (int i = lane; i < nlist; i += 32) {
    const int s = (int)T.list[i];
    const uint32_t k = T.key[s];
    const double val = lpa_combine(S.rule, T.cnt[s], T.score[s]);
    if (val > bv || (val == bv && i < bi)) {
      bv = val;
      bi = i;
      bk = k;
    }
    if (k == cur) {
      cp = true;
      cv = val;
    }
    T.key[s] = kEmpty;                                    // reset for the next node
  }
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    const double ov = __shfl_xor_sync(FULL, bv, d);
    const int oi = __shfl_xor_sync(FULL, bi, d);
    const uint32_t ok = __shfl_xor_sync(FULL, bk, d);
    if (ov > bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
      bk = ok;
    }
  }
  const uint32_t cpm = __ballot_sync(FULL, cp);
  __syncwarp();
  if (cpm) {
    cv = __shfl_sync(FULL, cv, __ffs(cpm) - 1);
    if (cv >= dd::sub(bv, 1e-12)) bk = cur;               // LPA_SCORE_EPS
  }
  return bk;
}

// Applies a change of v from kprev to best (rb_cluster.cpp:565-582 and
// :685-708): label, counters, neighbours' activation marks, visited set and
// freeze.  Called by the whole warp.
// Marks go to next_active, which no one reads before the next round: in the
// synchronous sweep every neighbour, in the sequential one only the neighbours
// already visited in this round (and the node itself on a self-loop) -- the
// later ones learn of the change from the stamp within this round.
__device__ void commit(const Sweep &S, uint32_t v, uint32_t kprev, uint32_t best, int64_t a0,
                       int64_t a1, bool sequential) {
  const int lane = threadIdx.x & 31;
  for (int64_t a = a0 + lane; a < a1; a += 32) {
    const uint32_t u = __ldg(S.nbr + a);
    if (!sequential || __ldg(S.early + a) || u == v) S.next_active[u] = 1;
  }
  if (lane == 0) {
    st_relaxed(S.label + v, best);
    atomicAdd(S.counts, 1ull);
    // visited set: {kprev} on the first change, then best; a label seen before freezes v
    uint32_t *blk = S.vlab + (size_t)v * kVisitPer;
    uint32_t *cntp = S.vcnt + v, *nextp = S.vnext + v;
    if (ld_cg(S.vcnt + v) == 0) {
      blk[0] = kprev;
      S.vcnt[v] = 1;
    }
    bool seen = false;
    uint32_t c = 0;
    for (;;) {
      c = ld_cg(cntp);
      for (uint32_t i = 0; i < c && !seen; ++i) seen = ld_cg(blk + i) == best;
      const uint32_t b = ld_cg(nextp);
      if (seen || b == kEmpty) break;
      blk = S.vlab + (size_t)b * kVisitPer;
      cntp = S.vcnt + b;
      nextp = S.vnext + b;
    }
    if (seen) {
      S.frozen[v] = 1;
      atomicAdd(S.counts + 1, 1ull);
    } else if (c < (uint32_t)kVisitPer) {
      blk[c] = best;
      *cntp = c + 1;
    } else {
      const uint32_t b = atomicAdd(S.vpool_used, 1u);
      if (b >= S.vpool_cap) {
        atomicCAS(S.err, 0, RBG_ERR_NOMEM);               // pool too small: the host reruns bigger
      } else {
        const uint32_t id = (uint32_t)S.n + b;
        S.vlab[(size_t)id * kVisitPer] = best;
        S.vcnt[id] = 1;
        S.vnext[id] = kEmpty;
        *nextp = id;
      }
    }
  }
}

// Per-warp shared region (kWarpSmem bytes): table, then the arc stage.
__device__ __forceinline__ unsigned char *warp_region(unsigned char *smem) {
  return smem + (size_t)(threadIdx.x >> 5) * kWarpSmem;
}
__device__ __forceinline__ uint32_t *warp_stage_u(unsigned char *smem) {
  return (uint32_t *)(warp_region(smem) + kTabSlots * 16 + kTabMaxDeg * 4);
}
__device__ __forceinline__ float *warp_stage_w(unsigned char *smem) {
  return (float *)(warp_stage_u(smem) + kTabMaxDeg);
}
__device__ __forceinline__ double *warp_stage_d(unsigned char *smem) {   // lo, hi intervals
  return (double *)warp_stage_u(smem);
}
__device__ __forceinline__ float *warp_wbuf(unsigned char *smem) {
  return (float *)(warp_region(smem) + kTabSlots * 16 + kTabMaxDeg * 20);
}
// 1/i rounded, i < kTabMaxDeg, after the warps' regions
__device__ __forceinline__ double *cta_inv(unsigned char *smem) {
  return (double *)(smem + (size_t)kLpaWarps * kWarpSmem);
}

__device__ __forceinline__ Table warp_table(const Sweep &S, unsigned char *smem, int64_t deg,
                                            int gwarp) {
  Table T;
  if (deg <= kTabMaxDeg) {
    unsigned char *b = warp_region(smem);
    T.score = (double *)b;
    T.key = (uint32_t *)(b + kTabSlots * 8);
    T.cnt = (int32_t *)(b + kTabSlots * 12);
    T.list = (uint32_t *)(b + kTabSlots * 16);
    T.slots = kTabSlots;
  } else {
    const size_t G = (size_t)S.gtab_slots;
    uint32_t *b = S.gtab + (size_t)gwarp * G * 5;        // score (2 words), key, cnt, list
    T.score = (double *)b;
    T.key = b + 2 * G;
    T.cnt = (int32_t *)(b + 3 * G);
    T.list = b + 4 * G;
    T.slots = S.gtab_slots;
  }
  return T;
}

size_t sweep_smem() { return (size_t)kLpaWarps * kWarpSmem + kTabMaxDeg * 8; }

// Tables start empty: keys of every shared and global table set to kEmpty;
// the reciprocal table of the CTA filled.  Called by all threads of the CTA.
__device__ void clear_tables(const Sweep &S, unsigned char *smem, int gwarp) {
  const int lane = threadIdx.x & 31;
  uint32_t *k = (uint32_t *)(warp_region(smem) + kTabSlots * 8);
  for (int i = lane; i < kTabSlots; i += 32) k[i] = kEmpty;
  if (S.gtab) {
    const size_t G = (size_t)S.gtab_slots;
    uint32_t *gk = S.gtab + (size_t)gwarp * G * 5 + 2 * G;
    for (size_t i = lane; i < G; i += 32) gk[i] = kEmpty;
  }
  double *inv = cta_inv(smem);
  for (int i = threadIdx.x; i < kTabMaxDeg; i += blockDim.x)
    inv[i] = i ? __drcp_rn((double)i) : 0.0;
  __syncthreads();
}

// Visit stamps: a node visited in round r holds 2r + 1 when its label
// changed, 2r otherwise, published after its writes.  Bounded wait (relaxed
// polls; the caller fences before it reads what the node wrote) until u was
// visited in this round; returns its stamp, or 0 after giving up.
__device__ __forceinline__ uint32_t wait_visited(const Sweep &S, uint32_t u) {
  const uint32_t want = 2u * S.round;
  uint32_t st = ld_relaxed(S.done + u);
  if (st >= want) return st;
  const uint64_t t0 = now_ns();
  for (int it = 1;; ++it) {
    __nanosleep(it < 16 ? 20 : 200);
    st = ld_relaxed(S.done + u);
    if (st >= want) return st;
    if ((it & 15) == 0) {
      if (*(volatile int *)S.err != 0) return 0;
      if (now_ns() - t0 > kWaitNs) {
        atomicCAS(S.err, 0, RBG_ERR_TIMEOUT);
        return 0;
      }
    }
  }
}

// Fast path of a node with d <= kTabMaxDeg arcs whose labels are staged in su
// (and quantities in sw): the table accumulation of decide(), then label
// scores as intervals (lpa_interval), exact evaluation only where intervals
// leave the choice open (rb_cluster.cpp:532-553): the labels that can still be
// the best (upper end at or above the largest lower end) when more than one
// can, and the current label against the best when the 1e-12 rule is not
// settled by the intervals.  Same result as decide().
__device__ uint32_t decide_staged(const Sweep &S, Table &T, const uint32_t *su, const float *sw,
                                  double *dlo, const double *inv, int d, uint32_t cur,
                                  bool *touched) {
  const int lane = threadIdx.x & 31;
  int nlist = 0;
  for (int c = 0; c < d; c += 32) {
    const int i = c + lane;
    const bool valid = i < d;
    const uint32_t L = valid ? su[i] : kEmpty;
    const uint32_t grp = __match_any_sync(FULL, L);
    const bool lead = valid && lane == __ffs(grp) - 1;
    bool fresh = false;
    int slot = 0;
    if (lead) {
      slot = table_find(T, L, &fresh);
      double s = T.score[slot];
      for (uint32_t g = grp; g; g &= g - 1) lpa_accumulate(S.rule, s, sw[c + __ffs(g) - 1]);
      T.score[slot] = s;
      T.cnt[slot] += __popc(grp);
    }
    const uint32_t nb = __ballot_sync(FULL, fresh);
    if (fresh) T.list[nlist + __popc(nb & ((1u << lane) - 1u))] = (uint32_t)slot;
    nlist += __popc(nb);
    __syncwarp();
  }
  *touched = nlist > 0;
  if (nlist == 0) return cur;
  double *dhi = dlo + kTabMaxDeg;                         // the stage, now free
  double M = -INFINITY;
  int ci = -1;
  for (int i = lane; i < nlist; i += 32) {
    const int s = (int)T.list[i];
    double l, h;
    lpa_interval(S.rule, T.cnt[s], T.score[s], inv, &l, &h);
    dlo[i] = l;
    dhi[i] = h;
    M = fmax(M, l);
    if (T.key[s] == cur) ci = i;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) M = fmax(M, __shfl_xor_sync(FULL, M, o));
  ci = __reduce_max_sync(FULL, (unsigned)(ci + 1)) - 1;   // list index of the current label
  __syncwarp();
  int nc = 0, first = 0x7FFFFFFF;
  for (int i = lane; i < nlist; i += 32)
    if (dhi[i] >= M) {
      ++nc;
      first = min(first, i);
    }
  nc = (int)__reduce_add_sync(FULL, (unsigned)nc);
  int bi;
  if (nc == 1) {
    bi = (int)__reduce_min_sync(FULL, (unsigned)first);
  } else {
    double bv = -INFINITY;
    int b = 0x7FFFFFFF;
    for (int i = lane; i < nlist; i += 32) {
      if (!(dhi[i] >= M)) continue;
      double v = dlo[i];
      if (v != dhi[i]) {
        const int s = (int)T.list[i];
        v = lpa_combine(S.rule, T.cnt[s], T.score[s]);
        dlo[i] = dhi[i] = v;
      }
      if (v > bv || (v == bv && i < b)) {
        bv = v;
        b = i;
      }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const double ov = __shfl_xor_sync(FULL, bv, o);
      const int ob = __shfl_xor_sync(FULL, b, o);
      if (ov > bv || (ov == bv && ob < b)) {
        bv = ov;
        b = ob;
      }
    }
    bi = b;
  }
  __syncwarp();
  uint32_t bk = T.key[T.list[bi]];
  if (ci >= 0 && bk != cur) {
    // keep cur when cv >= RN(bv - 1e-12); decided by the intervals when they allow
    double blo = dlo[bi], bhi = dhi[bi], clo = dlo[ci], chi = dhi[ci];
    bool keep;
    if (clo >= dd::sub(bhi, 1e-12)) {
      keep = true;
    } else if (chi < dd::sub(blo, 1e-12)) {
      keep = false;
    } else {
      if (blo != bhi) blo = lpa_combine(S.rule, T.cnt[T.list[bi]], T.score[T.list[bi]]);
      if (clo != chi) clo = lpa_combine(S.rule, T.cnt[T.list[ci]], T.score[T.list[ci]]);
      keep = clo >= dd::sub(blo, 1e-12);
    }
    if (keep) bk = cur;
  }
  __syncwarp();
  for (int i = lane; i < nlist; i += 32) T.key[T.list[i]] = kEmpty;   // reset for the next node
  __syncwarp();
  return bk;
}

// Stages v's arcs (neighbour ids into su, quantities into sw) and, in the
// Gauss-Seidel sweep, waits (bounded) until every earlier neighbour has been
// visited in this round, polling all their stamps at once.  *chg: some earlier
// neighbour of this lane's arcs changed its label in this round.  Returns
// false after a wait gave up.  The caller fences before reading labels.
__device__ bool stage_and_wait(const Sweep &S, uint32_t *su, float *sw, int64_t a0, int d,
                               bool wait, bool *chg) {
  const int lane = threadIdx.x & 31;
  const uint32_t want = 2u * S.round;
  uint32_t pend = 0;
  *chg = false;
#pragma unroll
  for (int j = 0; j < kTabMaxDeg / 32; ++j) {
    const int i = lane + 32 * j;
    if (i < d) {
      const uint32_t u = __ldg(S.nbr + a0 + i);
      su[i] = u;
      sw[i] = __ldg(S.w + a0 + i);
      if (wait && __ldg(S.early + a0 + i)) pend |= 1u << j;
    }
  }
  if (!wait || __reduce_or_sync(FULL, pend) == 0) return true;
  uint64_t t0 = 0;
  bool changed = false;
  for (int it = 0; pend; ++it) {
#pragma unroll
    for (int j = 0; j < kTabMaxDeg / 32; ++j)
      if ((pend >> j) & 1u) {
        const uint32_t st = ld_relaxed(S.done + su[lane + 32 * j]);
        if (st >= want) {
          pend &= ~(1u << j);
          changed |= st == want + 1u;
        }
      }
    if (!pend) break;
    if (it == 0) t0 = now_ns();
    __nanosleep(it < 16 ? 20 : 200);
    if ((it & 15) == 15) {
      if (*(volatile int *)S.err != 0) return false;
      if (now_ns() - t0 > kWaitNs) {
        atomicCAS(S.err, 0, RBG_ERR_TIMEOUT);
        return false;
      }
    }
  }
  *chg = changed;
  return true;
}

// One Gauss-Seidel round (rb_cluster.cpp:611-714).
//
// Activity.  In the reference a node is active when a neighbour changed since
// its last visit.  Here that is split by when the change happened: changes of
// later neighbours in the previous round (after this node's visit there) are
// marks in `active`, written during the previous round into what is now read,
// and changes of earlier neighbours in this round are the change bits of their
// stamps.  No flag is written while it can be read, so nothing races.
// An inactive node writes nothing; it only publishes its stamp.
__global__ void __launch_bounds__(kLpaWarps * 32) k_lpa_gs_round(const Sweep S) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * kLpaWarps + (threadIdx.x >> 5);
  clear_tables(S, smem, gwarp);
  float *wb = warp_wbuf(smem);
  uint32_t *su = warp_stage_u(smem);
  float *sw = warp_stage_w(smem);
  double *sd = warp_stage_d(smem);
  const double *inv = cta_inv(smem);
  const uint32_t want = 2u * S.round;
  constexpr int J = kTabMaxDeg / 32;
  for (;;) {
    uint32_t p = 0;
    if (lane == 0) p = atomicAdd(S.claim, 1u);
    p = __shfl_sync(FULL, p, 0);
    if ((int64_t)p >= S.n) break;
    const uint4 r = __ldg(S.rec + p);
    const uint32_t v = r.x;
    const int64_t d = r.y, a0 = (int64_t)r.z | ((int64_t)r.w << 32), a1 = a0 + d;
    const bool marked = ld_cg8(S.active + v) != 0;          // written in the previous round
    bool ok = true, chg = false, changed = false;
    const uint32_t cur = ld_cg(S.label + v);
    if (d <= kTabMaxDeg) {
      // stage the arcs and poll the earlier neighbours once
      uint32_t uid[J];
      uint32_t pend = 0;
#pragma unroll
      for (int j = 0; j < J; ++j) {
        const int i = lane + 32 * j;
        uid[j] = 0;
        if (i < d) {
          uid[j] = __ldg(S.nbr + a0 + i);
          sw[i] = __ldg(S.w + a0 + i);
          if (__ldg(S.early + a0 + i)) pend |= 1u << j;
        }
      }
#pragma unroll
      for (int j = 0; j < J; ++j) {
        const int i = lane + 32 * j;
        if ((pend >> j) & 1u) {
          const uint32_t st = ld_relaxed(S.done + uid[j]);
          if (st >= want) {
            pend &= ~(1u << j);
            chg |= st == want + 1u;
          }
        }
      }
      bool touched = false;
      uint32_t best = cur;
      Table T = warp_table(S, smem, d, gwarp);
      // the remaining waits (bounded)
      uint64_t t0 = 0;
      for (int it = 0; pend && ok; ++it) {
        if (it == 0) t0 = now_ns();
        __nanosleep(it < 16 ? 20 : 200);
#pragma unroll
        for (int j = 0; j < J; ++j)
          if ((pend >> j) & 1u) {
            const uint32_t st = ld_relaxed(S.done + uid[j]);
            if (st >= want) {
              pend &= ~(1u << j);
              chg |= st == want + 1u;
            }
          }
        if (pend && (it & 15) == 15) {
          if (*(volatile int *)S.err != 0) ok = false;
          else if (now_ns() - t0 > kWaitNs) {
            atomicCAS(S.err, 0, RBG_ERR_TIMEOUT);
            ok = false;
          }
        }
      }
      if (!__all_sync(FULL, ok)) {
        if (lane == 0) st_release(S.done + v, want);
        break;
      }
      const bool anychg = __any_sync(FULL, chg);
      if ((marked || anychg) && d > 0) {
        // the labels after the waits: an earlier neighbour that changed wrote its
        // label before its stamp (acquired by the fence); the others did not move
        if (anychg) fence_acq_rel();
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const int i = lane + 32 * j;
          if (i < d) su[i] = ld_relaxed(S.label + uid[j]);
        }
        __syncwarp();
        best = decide_staged(S, T, su, sw, sd, inv, (int)d, cur, &touched);
        if (touched && best != cur && !ld_cg8(S.frozen + v)) {
          commit(S, v, cur, best, a0, a1, true);
          changed = true;
        }
      }
      __syncwarp();
      if (lane == 0) {
        if (marked || anychg) st_release(S.done + v, want + (changed ? 1u : 0u));
        else st_relaxed(S.done + v, want);
      }
      continue;
    }
    // general path (more arcs than the stage holds): wait, then decide
    for (int64_t a = a0 + lane; a < a1 && ok; a += 32)
      if (__ldg(S.early + a)) {
        const uint32_t st = wait_visited(S, __ldg(S.nbr + a));
        ok = st != 0;
        chg |= st == want + 1u;
      }
    if (!__all_sync(FULL, ok)) {
      if (lane == 0) st_release(S.done + v, want);
      break;
    }
    const bool act = __any_sync(FULL, marked || chg);
    if (act) {
      fence_acq_rel();
      Table T = warp_table(S, smem, d, gwarp);
      bool touched = false;
      const uint32_t best = decide(S, T, wb, v, a0, a1, cur, &touched);
      if (touched && best != cur && !ld_cg8(S.frozen + v)) {
        commit(S, v, cur, best, a0, a1, true);
        changed = true;
      }
    }
    __syncwarp();
    if (lane == 0) {
      if (act) st_release(S.done + v, want + (changed ? 1u : 0u));
      else st_relaxed(S.done + v, want);
    }
  }
}

// Synchronous round, part 1: proposals from the round's snapshot.
__global__ void __launch_bounds__(kLpaWarps * 32) k_lpa_sync_propose(const Sweep S) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * kLpaWarps + (threadIdx.x >> 5);
  clear_tables(S, smem, gwarp);
  float *wb = warp_wbuf(smem);
  uint32_t *su = warp_stage_u(smem);
  float *sw = warp_stage_w(smem);
  const double *inv = cta_inv(smem);
  const int64_t nw = (int64_t)gridDim.x * kLpaWarps;
  for (int64_t v = gwarp; v < S.n; v += nw) {
    uint32_t prop = kEmpty;
    const int64_t a0 = __ldg(S.off + v), a1 = __ldg(S.off + v + 1);
    if (ld_cg8(S.active + v) && a1 > a0) {
      Table T = warp_table(S, smem, a1 - a0, gwarp);
      bool touched = false;
      const uint32_t cur = ld_cg(S.label + v);
      uint32_t best;
      if (a1 - a0 <= kTabMaxDeg) {
        const int d = (int)(a1 - a0);
        bool chg = false;
        stage_and_wait(S, su, sw, a0, d, false, &chg);
#pragma unroll
        for (int j = 0; j < kTabMaxDeg / 32; ++j) {
          const int i = lane + 32 * j;
          if (i < d) su[i] = ld_cg(S.label + su[i]);
        }
        __syncwarp();
        best = decide_staged(S, T, su, sw, warp_stage_d(smem), inv, d, cur, &touched);
      } else {
        best = decide(S, T, wb, (uint32_t)v, a0, a1, cur, &touched);
      }
      if (touched) prop = best;
    }
    if (lane == 0) S.prop[v] = prop;
  }
}

// Synchronous round, part 2: the commits (marks into next_active).
__global__ void __launch_bounds__(kLpaWarps * 32) k_lpa_sync_commit(const Sweep S) {
  const int gwarp = blockIdx.x * kLpaWarps + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * kLpaWarps;
  for (int64_t v = gwarp; v < S.n; v += nw) {
    const uint32_t best = ld_cg(S.prop + v);
    if (best == kEmpty) continue;
    const uint32_t kprev = ld_cg(S.label + v);
    if (kprev != best && !ld_cg8(S.frozen + v))
      commit(S, (uint32_t)v, kprev, best, __ldg(S.off + v), __ldg(S.off + v + 1), false);
  }
}

}  // namespace

int lpa_raw_rule(int rule) {
  return rule == RBG_LPA_SUM || rule == RBG_LPA_MEAN || rule == RBG_LPA_MAX;
}

void launch_lpa_edges(const uint32_t *from, const uint32_t *to, const float *score, int64_t E,
                      int64_t n, int rule, float *q, uint32_t *deg, int *err, cudaStream_t s) {
  if (E == 0) return;
  const int64_t blocks = std::min<int64_t>((E + 255) / 256, 148 * 16);
  k_lpa_edges<<<(unsigned)blocks, 256, 0, s>>>(from, to, score, E, n, lpa_raw_rule(rule), q, deg,
                                               err);
}

void launch_lpa_offsets(const uint32_t *deg, int64_t n, int64_t *off, int64_t *maxdeg,
                        cudaStream_t s) {
  k_lpa_offsets<<<1, 1024, 0, s>>>(deg, n, off, maxdeg);
}

void launch_lpa_scatter(const uint32_t *from, const uint32_t *to, const float *score, int64_t E,
                        int64_t n, const int64_t *off, uint32_t *fill, uint64_t *key,
                        cudaStream_t s) {
  if (E == 0) return;
  const int64_t blocks = std::min<int64_t>((E + 255) / 256, 148 * 16);
  k_lpa_scatter<<<(unsigned)blocks, 256, 0, s>>>(from, to, score, E, n, off, fill, key);
}

void launch_lpa_sort(const int64_t *off, int64_t n, uint64_t *key, const float *q, uint32_t *nbr,
                     float *w, cudaStream_t s) {
  if (n == 0) return;
  k_lpa_sort<<<(unsigned)n, 256, 0, s>>>(off, key, q, nbr, w);
}

void launch_lpa_init(const uint32_t *order, int64_t n, uint32_t *pos, uint32_t *label,
                     uint8_t *active, uint8_t *next_active, uint8_t *frozen, uint32_t *done,
                     uint32_t *vcnt, uint32_t *vnext, cudaStream_t s) {
  if (n == 0) return;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_lpa_init<<<(unsigned)blocks, 256, 0, s>>>(order, n, pos, label, active, next_active, frozen,
                                              done, vcnt, vnext);
}

void launch_lpa_early(const int64_t *off, const uint32_t *nbr, const uint32_t *pos, int64_t n,
                      uint8_t *early, uint4 *rec, cudaStream_t s) {
  if (n == 0) return;
  const int64_t blocks = std::min<int64_t>((n + 7) / 8, 148 * 16);
  k_lpa_early<<<(unsigned)blocks, 256, 0, s>>>(off, nbr, pos, n, early, rec);
}

int lpa_sweep_warps(int sms) {
  static const int occ = [] {                         // once per process (thread-safe init)
    cudaFuncSetAttribute((const void *)k_lpa_gs_round, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sweep_smem());
    cudaFuncSetAttribute((const void *)k_lpa_sync_propose,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem());
    int o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, (const void *)k_lpa_gs_round,
                                                  kLpaWarps * 32, sweep_smem());
    return o < 1 ? 1 : o;
  }();
  return sms * occ * kLpaWarps;
}

int lpa_table_max_deg() { return kTabMaxDeg; }
int lpa_visit_block() { return kVisitPer; }

void launch_lpa_round(const LpaSweepArgs &a, int sync, int warps, cudaStream_t s) {
  Sweep S;
  S.n = a.n;
  S.off = a.off;
  S.nbr = a.nbr;
  S.w = a.w;
  S.order = a.order;
  S.pos = a.pos;
  S.early = a.early;
  S.rec = a.rec;
  S.label = a.label;
  S.active = a.active;
  S.next_active = a.next_active;
  S.frozen = a.frozen;
  S.done = a.done;
  S.prop = a.prop;
  S.vlab = a.vlab;
  S.vcnt = a.vcnt;
  S.vnext = a.vnext;
  S.vpool_used = a.vpool_used;
  S.vpool_cap = a.vpool_cap;
  S.claim = a.claim;
  S.counts = a.counts;
  S.gtab = a.gtab;
  S.gtab_slots = a.gtab_slots;
  S.rule = a.rule;
  S.round = a.round;
  S.err = a.err;
  const unsigned blocks = (unsigned)(warps / kLpaWarps);
  if (!sync) {
    k_lpa_gs_round<<<blocks, kLpaWarps * 32, sweep_smem(), s>>>(S);
  } else {
    k_lpa_sync_propose<<<blocks, kLpaWarps * 32, sweep_smem(), s>>>(S);
    k_lpa_sync_commit<<<blocks, kLpaWarps * 32, 0, s>>>(S);
  }
}

}  // namespace rbg
