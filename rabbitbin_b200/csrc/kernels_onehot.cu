// Dense regime (no abundance prune) on the tensor cores.  A register column r
// holds at most 136 distinct codes over an assembly, and far fewer in practice
// (a few tens: the elements of smallest U win most contigs), so a contig's
// codes are a short binary one-hot row X_i over the (register, code) pairs
// that occur in the assembly.  The register-match count of contigs i and j
// (src/rabbitbin.cpp:1261-1293: equal nonzero codes) is the exact integer dot
// product X_i . X_j, so all counts are one int8 GEMM with int32 accumulation
// (cuBLASLt, a plain library GEMM).  A warp per row then scans its counts and
// produces what the dense all-pairs kernel produces: the per-row top-K keys
// above the admission floor, the row maxima and the compared-pair count.
#include <cstdint>

#include "rbg_internal.h"
#include "select_topk.cuh"

namespace rbg {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kPresCols = 512;          // register columns per presence block (16 KB)

// Which codes occur in each register column: 256 bits per column.  A block
// takes rows_per_block rows and 512 register columns; a thread reads 4
// columns of a row at a time (mpad is a multiple of 16, so the 4-byte loads
// are aligned) and the block's two row streams run side by side.
__global__ void k_code_presence(const uint8_t *__restrict__ codesA, int64_t n, int m, int mpad,
                                int64_t rows_per_block, uint32_t *__restrict__ pres) {
  __shared__ uint32_t sp[kPresCols * 8];
  const int c0 = blockIdx.y * kPresCols;
  const int nc = (m - c0 < kPresCols) ? m - c0 : kPresCols;
  for (int i = threadIdx.x; i < kPresCols * 8; i += blockDim.x) sp[i] = 0;
  __syncthreads();
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
  const int64_t r1 = (r0 + rows_per_block < n) ? r0 + rows_per_block : n;
  const int cq = (threadIdx.x & 127) * 4;               // blockDim.x == 256
  if (cq < nc) {
    for (int64_t i = r0 + (threadIdx.x >> 7); i < r1; i += 2) {
      const uint32_t w4 = __ldg(reinterpret_cast<const uint32_t *>(codesA + i * mpad + c0 + cq));
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t code = (w4 >> (8 * u)) & 0xFFu;
        const int r = cq + u;
        // a column holds a few distinct codes: test before the (contended) atomic
        if (code && r < nc && !(sp[r * 8 + (code >> 5)] & (1u << (code & 31))))
          atomicOr(&sp[r * 8 + (code >> 5)], 1u << (code & 31));
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nc * 8; i += blockDim.x)
    if (sp[i]) atomicOr(&pres[(int64_t)c0 * 8 + i], sp[i]);
}

// One block: koff[r] = one-hot columns before register r (koff[m] = K), and
// map[r][code] = koff[r] + rank of code among the column's codes (-1 absent).
__global__ void k_onehot_map(const uint32_t *__restrict__ pres, int m, int32_t *__restrict__ map,
                             int32_t *__restrict__ koff) {
  __shared__ int32_t part[1024];
  const int t = threadIdx.x;
  const int per = (m + 1023) / 1024;
  const int a = t * per, b = (a + per < m) ? a + per : m;
  int s = 0;
  for (int r = a; r < b; ++r)
    for (int w = 0; w < 8; ++w) s += __popc(pres[r * 8 + w]);
  part[t] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int add = (t >= d) ? part[t - d] : 0;
    __syncthreads();
    part[t] += add;
    __syncthreads();
  }
  int run = (t > 0) ? part[t - 1] : 0;
  for (int r = a; r < b; ++r) {
    koff[r] = run;
    for (int w = 0; w < 8; ++w) run += __popc(pres[r * 8 + w]);
  }
  if (t == 1023) koff[m] = part[1023];
  __syncthreads();
  for (int64_t e = t; e < (int64_t)m * 256; e += 1024) {
    const int r = (int)(e >> 8), code = (int)(e & 255);
    const uint32_t *p = pres + r * 8;
    int32_t v = -1;
    if ((p[code >> 5] >> (code & 31)) & 1u) {
      int rank = __popc(p[code >> 5] & ((1u << (code & 31)) - 1u));
      for (int w = 0; w < (code >> 5); ++w) rank += __popc(p[w]);
      v = koff[r] + rank;
    }
    map[e] = v;
  }
}

// X[i][map[r][code_i(r)]] = 1 (X zeroed by the caller; row stride ldx bytes).
__global__ void k_onehot_fill(const uint8_t *__restrict__ codesA, int64_t n, int m, int mpad,
                              const int32_t *__restrict__ map, int8_t *__restrict__ X,
                              int64_t ldx) {
  const int64_t i = blockIdx.x;                     // one row per block
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const uint32_t code = codesA[i * mpad + r];
    if (code) X[i * ldx + __ldg(map + r * 256 + code)] = 1;
  }
}

// Warp per row i of [r0, r0 + nr): its counts against every contig j are
// D[(i - r0) * ldd + j].  Same outputs as the dense all-pairs kernel for the
// row: top-K keys (similarity bits << 32 | ~j) of the candidates above the
// admission floor, kept through a 512-key shared buffer and the register radix
// select; maxima over all other j and over the candidates (anynz); the number
// of pairs compared.  A step whose counts are all below the current threshold
// (the common case) takes one vote, not four.
constexpr int kSelWarps = 8;
constexpr int kSelBuf = 32 * kCapW;   // 512 keys per warp

__global__ void __launch_bounds__(kSelWarps * 32, 4)
k_dense_select(GraphArgs g, const int32_t *__restrict__ D, int64_t ldd, int64_t r0, int64_t nr) {
  __shared__ uint64_t sbuf[kSelWarps][kSelBuf];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t q = (int64_t)blockIdx.x * kSelWarps + wib;
  if (q >= nr) return;
  const int64_t i = r0 + q, n = g.n;
  const int K = g.K;
  const int32_t *row = D + q * ldd;
  uint64_t *buf = sbuf[wib];
  const uint8_t nz_i = g.anynz[i];
  // Keys are ranked as (count << 32 | ~j): among admitted keys the similarity
  // strictly increases with the count, so the order is the order of the
  // similarity keys, which replace the counts at the end.  Admission (similarity
  // above the floor) is a count threshold c_adm >= 1 (similarity 0 never passes).
  const uint32_t fbits = (uint32_t)(g.key_floor >> 32);
  int c_adm = g.m + 1;
  for (int c0 = 0; c0 <= g.m; c0 += 32) {
    const int cc = c0 + lane;
    const unsigned hit = __ballot_sync(FULL, cc <= g.m && __ldg(g.sv_bits + cc) > fbits);
    if (hit) {
      c_adm = c0 + __ffs(hit) - 1;
      break;
    }
  }
  uint64_t thr = ((uint64_t)c_adm << 32) - 1u;
  // anynz of a batch assembly starts at its first row: 4-byte loads only when aligned
  const bool nz_words = (((uintptr_t)g.anynz) & 3u) == 0;
  uint32_t mx_a = 0, mx_c = 0;
  int fill = 0;
  // lane takes 4 consecutive contigs per step (16-byte count loads; ldd and the
  // row starts are multiples of 4 counts); the next step's loads are issued
  // before this step's keys are ranked
  auto load = [&](int64_t jb, int4 &c4, uint32_t &nz4) {
    c4 = make_int4(0, 0, 0, 0);
    nz4 = 0;
    if (jb < n) {
      c4 = __ldcs(reinterpret_cast<const int4 *>(row + jb));   // read once: stream past L1/L2
      if (jb + 4 <= n && nz_words) {
        nz4 = __ldg(reinterpret_cast<const uint32_t *>(g.anynz + jb));
      } else {
        for (int t = 0; t < 4 && jb + t < n; ++t) nz4 |= (uint32_t)g.anynz[jb + t] << (8 * t);
      }
    }
  };
  int4 nxt_c;
  uint32_t nxt_nz;
  load(4 * lane, nxt_c, nxt_nz);
  for (int64_t j0 = 0; j0 < n; j0 += 128) {
    const int64_t jb = j0 + 4 * lane;
    const int4 c4 = nxt_c;
    const uint32_t nz4 = nxt_nz;
    load(jb + 128, nxt_c, nxt_nz);
    uint32_t cv[4] = {(uint32_t)c4.x, (uint32_t)c4.y, (uint32_t)c4.z, (uint32_t)c4.w};
    // the diagonal and the padding past n count as 0 (counts are >= 0, so the
    // maxima are those over the other contigs) and are no candidates
    unsigned cm = 0;
    bool may = false;
    const uint32_t thc = (uint32_t)(thr >> 32);   // a key passes only from this count on
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int64_t j = jb + t;
      if (j >= n || j == i) cv[t] = 0;
      const bool cand = j < n && j != i && (nz_i | ((nz4 >> (8 * t)) & 0xFFu));
      cm |= (unsigned)cand << t;
      mx_a = cv[t] > mx_a ? cv[t] : mx_a;
      if (cand && cv[t] > mx_c) mx_c = cv[t];
      may |= cand && cv[t] >= thc;
    }
    if (!__any_sync(FULL, may)) continue;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const uint64_t key = ((uint64_t)cv[t] << 32) | (uint64_t)(~(uint32_t)(jb + t));
      const bool adm = ((cm >> t) & 1u) && key > thr;
      const unsigned mk = __ballot_sync(FULL, adm);
      if (mk) {
        if (adm) buf[fill + __popc(mk & ((1u << lane) - 1u))] = key;
        fill += __popc(mk);
        __syncwarp();
        if (fill > kSelBuf - 32) {
          thr = select_topk(buf, fill, K);
          fill = K;
        }
      }
    }
  }
  if (fill > K) {
    select_topk(buf, fill, K);
    fill = K;
  }
  for (int t = lane; t < fill; t += 32) {
    const uint64_t ck = buf[t];
    g.topk[i * K + t] = ((uint64_t)__ldg(g.sv_bits + (ck >> 32)) << 32) | (ck & 0xFFFFFFFFull);
  }
  mx_a = __reduce_max_sync(FULL, mx_a);
  mx_c = __reduce_max_sync(FULL, mx_c);
  if (lane == 0) {
    g.topk_cnt[i] = fill;
    g.maxcnt_all[i] = mx_a;
    g.maxcnt_cand[i] = mx_c;
    if (g.stats) atomicAdd(g.stats + 1, (unsigned long long)(n - 1));   // every other contig
  }
}

}  // namespace

void launch_code_presence(const uint8_t *codesA, int64_t n, int m, int mpad, uint32_t *pres,
                          cudaStream_t s) {
  cudaMemsetAsync(pres, 0, (size_t)m * 8 * sizeof(uint32_t), s);
  if (n == 0) return;
  const int64_t rows_per_block = 64;
  const dim3 grid((unsigned)((n + rows_per_block - 1) / rows_per_block),
                  (unsigned)((m + kPresCols - 1) / kPresCols));
  k_code_presence<<<grid, 256, 0, s>>>(codesA, n, m, mpad, rows_per_block, pres);
}

void launch_onehot_map(const uint32_t *pres, int m, int32_t *map, int32_t *koff, cudaStream_t s) {
  k_onehot_map<<<1, 1024, 0, s>>>(pres, m, map, koff);
}

void launch_onehot_fill(const uint8_t *codesA, int64_t n, int m, int mpad, const int32_t *map,
                        int8_t *X, int64_t ldx, cudaStream_t s) {
  cudaMemsetAsync(X, 0, (size_t)n * ldx, s);
  if (n == 0 || m == 0) return;
  k_onehot_fill<<<(unsigned)n, 256, 0, s>>>(codesA, n, m, mpad, map, X, ldx);
}

void launch_dense_select(const GraphArgs &g, const int32_t *D, int64_t ldd, int64_t r0, int64_t nr,
                         cudaStream_t s) {
  if (nr <= 0) return;
  k_dense_select<<<(unsigned)((nr + kSelWarps - 1) / kSelWarps), kSelWarps * 32, 0, s>>>(
      g, D, ldd, r0, nr);
}

}  // namespace rbg
