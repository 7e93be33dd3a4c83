// Warp-cooperative selection of the K largest of up to 512 unique 64-bit
// keys, shared by the all-pairs kernels and the dense-regime row scan.
#pragma once
#include <cstdint>

namespace rbg {

constexpr int kCapW = 16;         // keys per lane: buffers hold up to 32 * kCapW keys

// Warp-cooperative: keep the K largest of the cnt unique keys in buf (global),
// in place; returns the K-th largest key (the new admission threshold).
// EARLY: stop the bit search once exactly K keys are >= the prefix (fewer
// steps, a few more registers: the candidate-buffer compaction inside the
// all-pairs kernels keeps the full search).
template <bool EARLY = true>
__device__ inline uint64_t select_topk(uint64_t *buf, int cnt, int K) {
  const int lane = threadIdx.x & 31;
  uint64_t v[kCapW];
#pragma unroll
  for (int t = 0; t < kCapW; ++t) {
    const int i = t * 32 + lane;
    v[t] = i < cnt ? buf[i] : 0ull;
  }
  // Bit-by-bit search for the K-th largest key, stopped as soon as exactly K
  // keys are >= the prefix found so far (the lower bits cannot change the set).
  uint64_t P = 0;
  bool exact = true;                   // P is the K-th largest key itself
  for (int bit = 63; bit >= 0; --bit) {
    const uint64_t c = P | (1ull << bit);
    int k = 0;
#pragma unroll
    for (int t = 0; t < kCapW; ++t) k += v[t] >= c;
    const int tot = (int)__reduce_add_sync(0xffffffffu, (unsigned)k);
    if (tot >= K) {
      P = c;
      if (EARLY && tot == K) {         // the lower bits cannot change the set
        exact = bit == 0;
        break;
      }
    }
  }
  __syncwarp();
  int out = 0;
  uint64_t kmin = ~0ull;
#pragma unroll
  for (int t = 0; t < kCapW; ++t) {
    const bool keep = v[t] >= P && v[t] != 0ull;
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      buf[out + __popc(m & ((1u << lane) - 1u))] = v[t];
      kmin = v[t] < kmin ? v[t] : kmin;
    }
    out += __popc(m);
  }
  __syncwarp();
  if (!exact) {                        // the smallest kept key
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      const uint64_t a = __shfl_xor_sync(0xffffffffu, kmin, d);
      kmin = a < kmin ? a : kmin;
    }
    P = kmin;
  }
  return P;
}

}  // namespace rbg

namespace rbg {

// The same selection over up to 32 * CAPW unique nonzero 32-bit keys (global
// or shared buffer), with the early stop; returns the K-th largest key.
template <int CAPW>
__device__ inline uint32_t select_topk32(uint32_t *buf, int cnt, int K) {
  const int lane = threadIdx.x & 31;
  uint32_t v[CAPW];
#pragma unroll
  for (int t = 0; t < CAPW; ++t) {
    const int i = t * 32 + lane;
    v[t] = i < cnt ? buf[i] : 0u;
  }
  uint32_t P = 0;
  bool exact = true;
  for (int bit = 31; bit >= 0; --bit) {
    const uint32_t c = P | (1u << bit);
    int k = 0;
#pragma unroll
    for (int t = 0; t < CAPW; ++t) k += v[t] >= c;
    const int tot = (int)__reduce_add_sync(0xffffffffu, (unsigned)k);
    if (tot >= K) {
      P = c;
      if (tot == K) {
        exact = bit == 0;
        break;
      }
    }
  }
  __syncwarp();
  int out = 0;
  uint32_t kmin = ~0u;
#pragma unroll
  for (int t = 0; t < CAPW; ++t) {
    const bool keep = v[t] >= P && v[t] != 0u;
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      buf[out + __popc(m & ((1u << lane) - 1u))] = v[t];
      kmin = v[t] < kmin ? v[t] : kmin;
    }
    out += __popc(m);
  }
  __syncwarp();
  if (!exact) P = __reduce_min_sync(0xffffffffu, kmin);
  return P;
}

}  // namespace rbg
