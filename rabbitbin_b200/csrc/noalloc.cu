// Sketch without device allocation: rbg_build_pmh_winners_noalloc.
//
// Some callers cannot call cudaMalloc: code that runs while a host framework
// owns the whole device heap through its own pool, plugins loaded into another
// process's CUDA context with a fixed memory budget, or callers that must not
// synchronise on an allocation while their streams are busy.  This entry point
// serves them: the caller passes the ASCII sequences, the offsets and the
// output winner rows as device buffers, and every intermediate buffer (2-bit
// packed bases, invalid-base mask, 1/w table, register codes, the ProbMinHash
// stream tables, the offsets check flag) lives in one file-scope array
// reserved when the library is loaded.  The array is kRbgNoAllocScratchBytes
// (24 MiB) on every GPU that loads the library, kept until the process exits;
// requests that need more are rejected with RBG_ERR_ARG before anything runs
// on the device.
//
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress, once per device, with that device current).  Every
// call reads a check flag back and synchronises the caller's stream, so no
// call may be made while that stream is being captured into a CUDA graph.
// All calls share the array and it keeps the previous call's contents; every
// part a call reads is written by the same call first (the check kernel writes
// its flag unconditionally, the register-minimum kernel writes the code
// padding too), but two calls that overlap on the GPU race on it.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "rbg_internal.h"

namespace rbg {

constexpr size_t kRbgNoAllocScratchBytes = 24u << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kRbgNoAllocScratchBytes];

namespace {

std::mutex g_setup_mu;
void *g_scratch_ptr[64] = {nullptr};     // device address per device ordinal

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

void put_err(char *buf, size_t len, const char *msg) {
  if (buf && len) {
    std::strncpy(buf, msg, len - 1);
    buf[len - 1] = 0;
  }
}

// Offsets check, one block: flag = 1 unless offsets[0] == 0, offsets[n] ==
// nbases and 0 <= offsets[i] <= offsets[i+1] <= nbases for every i.  The
// flag is written whatever the outcome, so nothing needs clearing first.
__global__ void k_check_offsets(const int64_t *__restrict__ off, int64_t n, int64_t nbases,
                                int32_t *__restrict__ flag) {
  int bad = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int64_t a = off[i], b = off[i + 1];
    bad |= (a < 0) | (a > b) | (b > nbases);
  }
  if (threadIdx.x == 0) bad |= (off[0] != 0) | (off[n] != nbases);
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) *flag = bad;
}

}  // namespace
}  // namespace rbg

extern "C" int rbg_build_pmh_winners_noalloc(const rbg_params *p, const char *seq_device,
                                             const int64_t *offsets_device, int64_t n,
                                             int64_t nbases, uint32_t *winners_device,
                                             void *stream, char *errbuf, size_t errlen) {
  using namespace rbg;
  if (!p || n < 0 || nbases < 0 || (n > 0 && (!seq_device || !offsets_device || !winners_device))) {
    put_err(errbuf, errlen, "null or negative argument");
    return RBG_ERR_ARG;
  }
  if (p->oph_k > 0) {
    put_err(errbuf, errlen, "winner rows exist only for the ProbMinHash metric (oph_k = 0)");
    return RBG_ERR_ARG;
  }
  if (p->k < 1 || p->k > 4 || p->m < 2 || p->m > 4096 || p->gc_norm < 0 || p->gc_norm > 2 ||
      (p->win_bits != 16 && p->win_bits != 32)) {
    put_err(errbuf, errlen, "unsupported parameters (k 1..4, m 2..4096, gc_norm 0..2)");
    return RBG_ERR_UNSUPPORTED;
  }
  if (((uintptr_t)seq_device & 15u) != 0) {
    put_err(errbuf, errlen, "seq_device must be 16-byte aligned (and readable to a 16-byte multiple)");
    return RBG_ERR_ARG;
  }
  if (n == 0) return RBG_OK;
  // scratch plan
  const int m = p->m, mpad = (m + 15) & ~15;
  const int E = p->k == 4 ? 136 : (p->k == 3 ? 32 : (p->k == 2 ? 10 : 2));
  const int64_t nwords = (nbases + 15) / 16 + 1;
  size_t off = 0;
  const size_t oOrd = off;     off += up256((size_t)E * m * sizeof(RegOrder));
  const size_t oUT = off;      off += up256((size_t)E * m * sizeof(double));
  const size_t oCode = off;    off += up256((size_t)E * m);
  const size_t oW = off;       off += up256((size_t)E * m * sizeof(uint32_t));
  const size_t oRank = off;    off += up256(256 * sizeof(int16_t));
  const size_t oPacked = off;  off += up256((size_t)nwords * 4);
  const size_t oMask = off;    off += up256((size_t)(nwords / 2 + 2) * 4);
  const size_t oWinv = off;    off += up256((size_t)n * E * sizeof(double));
  const size_t oCnt = off;     off += up256((size_t)n * sizeof(int32_t));
  const size_t oA = off;       off += up256((size_t)n * mpad);
  const size_t oB = off;       off += up256((size_t)n * mpad);
  const size_t oFlag = off;    off += 256;
  if (off > kRbgNoAllocScratchBytes) {
    char msg[200];
    std::snprintf(msg, sizeof(msg),
                  "request needs %zu bytes of scratch, more than the %zu-byte static array "
                  "(fewer contigs or bases per call)", off, kRbgNoAllocScratchBytes);
    put_err(errbuf, errlen, msg);
    return RBG_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    put_err(errbuf, errlen, "no current CUDA device");
    return RBG_ERR_CUDA;
  }
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      void *ptr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr) {
        put_err(errbuf, errlen, cudaGetErrorString(e));
        return RBG_ERR_CUDA;
      }
      g_scratch_ptr[dev] = ptr;
    }
    base = g_scratch_ptr[dev];
  }
  unsigned char *S = (unsigned char *)base;
  cudaStream_t s = (cudaStream_t)stream;
  // offsets check on the device; its flag comes back before any sketch work
  int32_t bad = 1;
  k_check_offsets<<<1, 1024, 0, s>>>(offsets_device, n, nbases, (int32_t *)(S + oFlag));
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    put_err(errbuf, errlen, cudaGetErrorString(e));
    return RBG_ERR_CUDA;
  }
  if ((e = cudaMemcpyAsync(&bad, S + oFlag, sizeof(bad), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    put_err(errbuf, errlen, cudaGetErrorString(e));
    return RBG_ERR_CUDA;
  }
  if (bad) {
    put_err(errbuf, errlen, "offsets_device must start at 0, end at nbases and never decrease");
    return RBG_ERR_ARG;
  }
  std::shared_ptr<const PmhTables> t;
  try {
    t = pmh_tables(p->k, m, p->pmh_seed, p->fp_contract != 0);
  } catch (...) {
    put_err(errbuf, errlen, "host table construction failed");
    return RBG_ERR_NOMEM;
  }
  int16_t rank[256];
  for (int v = 0; v < 256; ++v) rank[v] = v < (int)t->rank_of_code.size() ? (int16_t)t->rank_of_code[v] : -1;
  const size_t EM = (size_t)E * m;
  if (cudaMemcpyAsync(S + oOrd, t->order.data(), EM * sizeof(RegOrder), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S + oUT, t->UT.data(), EM * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S + oCode, p->win_bits == 16 ? t->code16.data() : t->code32.data(), EM,
                      cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S + oW, t->W32.data(), EM * sizeof(uint32_t), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S + oRank, rank, sizeof(rank), cudaMemcpyHostToDevice, s) != cudaSuccess) {
    put_err(errbuf, errlen, "table upload failed");
    return RBG_ERR_CUDA;
  }
  launch_pack(seq_device, nbases, (uint32_t *)(S + oPacked), (uint32_t *)(S + oMask), s);
  SketchArgs a;
  a.packed = (const uint32_t *)(S + oPacked);
  a.nmask = (const uint32_t *)(S + oMask);
  a.offsets = offsets_device;
  a.n = n;
  a.k = p->k;
  a.m = m;
  a.gc_norm = p->gc_norm;
  a.gc_cap = p->gc_norm_cap;
  a.n_elems = E;
  a.rank_of_code = (const int16_t *)(S + oRank);
  a.elem_winv = (double *)(S + oWinv);
  a.elem_cnt = (int32_t *)(S + oCnt);
  a.order = (const RegOrder *)(S + oOrd);
  a.UT = (const double *)(S + oUT);
  a.codeA = (const uint8_t *)(S + oCode);
  a.W32 = (const uint32_t *)(S + oW);
  a.codesA = S + oA;
  a.codesB = S + oB;
  a.winners32 = winners_device;
  a.mpad = mpad;
  launch_count(a, s);
  launch_minreduce(a, s);
  // a failed launch is reported by its own code; the sync's code separately
  if ((e = cudaPeekAtLastError()) != cudaSuccess) {
    cudaStreamSynchronize(s);              // the host tables must outlive the copies
    put_err(errbuf, errlen, cudaGetErrorString(e));
    return RBG_ERR_CUDA;
  }
  // the host tables must outlive the asynchronous copies
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
    put_err(errbuf, errlen, cudaGetErrorString(e));
    return RBG_ERR_CUDA;
  }
  return RBG_OK;
}
