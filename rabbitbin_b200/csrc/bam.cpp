// BAM -> depth summariser, host side: BGZF blocks, the header, the record walk
// and the hand-over to the device (kernels in kernels_depth.cu).
//
// Reference: compute_depth_tsv_inmem with a DepthMatrixOut
// (src/rabbit_depth.cpp:1096-1535) as the bin command calls it
// (src/rabbitbin.cpp:3806-3811), and depth_accumulate_sample
// (src/rabbit_depth.cpp:1615-1685).  The reference splits each BAM into shards
// that htslib threads decompress and one thread per shard parses; here the
// per-read work runs on the device, one thread per record, and the host keeps
// only what is inherently sequential or byte-serial:
//
//   * the block index: every BGZF member's compressed range and inflated size
//     (its ISIZE field) are read first, so each block's place in the
//     decompressed stream is known before any block is inflated;
//   * inflation: a pool of host threads inflates the blocks of a chunk
//     (64 MiB of decompressed bytes by default) straight into their places in
//     a pinned slot, checking each block's length and CRC32;
//   * the record walk: records are found by following block_size from one to
//     the next; each record's sizes are checked against the stream, its offset
//     goes into a pinned list, and the first 4,000 mapped records give the
//     sample's mean read length (src/rabbit_depth.cpp:787-834);
//   * a record cut by the chunk's end moves to the front of the next slot.
//
// Two slots alternate: while the device copies and scores chunk c, the host
// inflates chunk c + 1 into the other slot.  Nothing but the sums stays on the
// device between chunks; the means matrix is made on the device at the end.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "depth_record.cuh"
#include "engine_internal.h"

namespace rbg {

void launch_depth_reads(const uint8_t *buf, const uint32_t *rec_off, int64_t nrec,
                        const uint32_t *target_len, const depth::Params &P, unsigned long long *sum,
                        unsigned long long *sum_u, cudaStream_t s);
void launch_depth_means(const unsigned long long *sums, int64_t n_targets, const int32_t *kept_tid,
                        int64_t n_kept, const uint32_t *target_len, const int32_t *edge_of_col,
                        int ncols, float *out, cudaStream_t s);
void launch_depth_device(const uint8_t *comp, const DevBlk *blk, int nb, const uint64_t *ubound,
                         uint64_t hdr_end, uint8_t *out, uint32_t *counts, uint32_t *scan,
                         uint32_t *offs, uint32_t *flags, unsigned long long *rec_total,
                         const uint32_t *target_len, const depth::Params &P,
                         unsigned long long *sum, unsigned long long *sum_u, int sms,
                         cudaStream_t s);

namespace {

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

uint32_t le16(const uint8_t *p) { return depth::ld_u16(p); }
uint32_t le32(const uint8_t *p) { return depth::ld_u32(p); }

// One BGZF member: its deflate data, inflated size and CRC32.
struct Blk {
  uint64_t start, cdata;     // the member's first byte, its deflate data
  uint32_t clen, isize, crc;
};

// Block index of one file (SAM/BAM format specification, BGZF): gzip members
// with the FEXTRA flag and a 'BC' subfield holding the member's size - 1.
void index_blocks(const uint8_t *f, uint64_t n, std::vector<Blk> &out) {
  uint64_t o = 0;
  while (o < n) {
    if (n - o < 26) throw Error(RBG_ERR_ARG, "truncated BGZF block");
    if (f[o] != 31 || f[o + 1] != 139 || f[o + 2] != 8 || !(f[o + 3] & 4))
      throw Error(RBG_ERR_ARG, "not a BGZF stream (gzip member without the extra field)");
    const uint32_t xlen = le16(f + o + 10);
    if (n - o < 12ull + xlen) throw Error(RBG_ERR_ARG, "truncated BGZF header");
    uint32_t bsize = 0;
    for (uint32_t x = 0; x + 4 <= xlen;) {
      const uint8_t *sf = f + o + 12 + x;
      const uint32_t slen = le16(sf + 2);
      if (sf[0] == 'B' && sf[1] == 'C' && slen == 2 && x + 6 <= xlen) bsize = le16(sf + 4) + 1;
      x += 4 + slen;
    }
    if (!bsize) throw Error(RBG_ERR_ARG, "BGZF block without its BC size field");
    if (bsize < 12 + xlen + 8 || bsize > n - o) throw Error(RBG_ERR_ARG, "BGZF block size out of range");
    Blk b;
    b.start = o;
    b.cdata = o + 12 + xlen;
    b.clen = bsize - 12 - xlen - 8;
    b.crc = le32(f + o + bsize - 8);
    b.isize = le32(f + o + bsize - 4);
    if (b.isize > 65536) throw Error(RBG_ERR_ARG, "BGZF block inflates beyond 64 KiB");
    out.push_back(b);
    o += bsize;
  }
}

int host_threads(const rbg_depth_params *p) {
  int t = p->threads > 0 ? p->threads : (int)std::thread::hardware_concurrency();
  return std::max(1, std::min(t, 256));
}

// Inflates blocks [b0, b1) into dst (block i at dst + uoff[i] - uoff[b0]).
void inflate_blocks(const uint8_t *f, const std::vector<Blk> &B, const std::vector<uint64_t> &uoff,
                    size_t b0, size_t b1, uint8_t *dst, int threads) {
  if (b1 <= b0) return;
  std::atomic<size_t> next{b0};
  std::atomic<int> bad{0};
  auto work = [&] {
    z_stream z;
    std::memset(&z, 0, sizeof z);
    if (inflateInit2(&z, -15) != Z_OK) {
      bad = 3;
      return;
    }
    uint8_t dummy[1];
    for (;;) {
      const size_t i = next.fetch_add(1, std::memory_order_relaxed);
      if (i >= b1 || bad.load(std::memory_order_relaxed)) break;
      const Blk &b = B[i];
      uint8_t *out = b.isize ? dst + (uoff[i] - uoff[b0]) : dummy;
      inflateReset(&z);
      z.next_in = (Bytef *)(f + b.cdata);
      z.avail_in = b.clen;
      z.next_out = out;
      z.avail_out = b.isize ? b.isize : 1;
      const int r = inflate(&z, Z_FINISH);
      if (r != Z_STREAM_END || z.total_out != b.isize) {
        bad = 1;
        break;
      }
      if ((uint32_t)crc32(0L, out, b.isize) != b.crc) {
        bad = 2;
        break;
      }
    }
    inflateEnd(&z);
  };
  const int nt = (int)std::min<size_t>((size_t)threads, b1 - b0);
  if (nt <= 1) {
    work();
  } else {
    std::vector<std::thread> pool;
    pool.reserve(nt);
    for (int t = 0; t < nt; ++t) pool.emplace_back(work);
    for (auto &t : pool) t.join();
  }
  if (bad == 1) throw Error(RBG_ERR_ARG, "BGZF block does not inflate to its stated size");
  if (bad == 2) throw Error(RBG_ERR_ARG, "BGZF block fails its CRC32");
  if (bad == 3) throw Error(RBG_ERR_NOMEM, "zlib initialisation failed");
}

struct Header {
  std::vector<uint32_t> tlen;
  std::vector<std::string> names;
};

// Parses the BAM header at the start of the decompressed stream: returns its
// length (the offset of the first record), or 0 when more bytes are needed.
int64_t parse_header(const uint8_t *p, int64_t n, Header &h) {
  h.tlen.clear();
  h.names.clear();
  if (n < 4) return 0;
  if (std::memcmp(p, "BAM\1", 4) != 0) throw Error(RBG_ERR_ARG, "not a BAM stream (magic)");
  if (n < 12) return 0;
  const int32_t l_text = depth::ld_i32(p + 4);
  if (l_text < 0) throw Error(RBG_ERR_ARG, "BAM header text length is negative");
  int64_t o = 8 + (int64_t)l_text;
  if (n < o + 4) return 0;
  const int32_t n_ref = depth::ld_i32(p + o);
  if (n_ref < 0) throw Error(RBG_ERR_ARG, "BAM header contig count is negative");
  o += 4;
  for (int32_t i = 0; i < n_ref; ++i) {
    if (n < o + 4) return 0;
    const int32_t l_name = depth::ld_i32(p + o);
    if (l_name < 1) throw Error(RBG_ERR_ARG, "BAM header contig name is empty");
    if (n < o + 8 + l_name) return 0;
    const char *nm = (const char *)(p + o + 4);
    h.names.emplace_back(nm, strnlen(nm, (size_t)l_name));
    const int32_t l_ref = depth::ld_i32(p + o + 4 + l_name);
    if (l_ref < 0) throw Error(RBG_ERR_ARG, "BAM header contig length is negative");
    h.tlen.push_back((uint32_t)l_ref);
    o += 8 + l_name;
  }
  return o;
}

// A decompressed byte stream handed over in pieces of whole blocks.
struct Source {
  virtual ~Source() {}
  virtual bool done() const = 0;
  // bytes of the next piece: whole units (blocks) adding up to at most
  // `budget`, at least one unit
  virtual uint64_t plan(uint64_t budget) = 0;
  virtual void produce(uint8_t *dst) = 0;   // writes the planned piece
};

struct BgzfSource : Source {
  const uint8_t *f;
  const std::vector<Blk> &B;
  const std::vector<uint64_t> &uoff;
  size_t bi, be = 0;
  int threads;
  BgzfSource(const uint8_t *f_, const std::vector<Blk> &B_, const std::vector<uint64_t> &u, size_t b0,
             int t)
      : f(f_), B(B_), uoff(u), bi(b0), threads(t) {}
  bool done() const override { return bi >= B.size(); }
  uint64_t plan(uint64_t budget) override {
    be = bi;
    uint64_t bytes = 0;
    while (be < B.size() && (be == bi || bytes + B[be].isize <= budget)) bytes += B[be++].isize;
    return bytes;
  }
  void produce(uint8_t *dst) override {
    inflate_blocks(f, B, uoff, bi, be, dst, threads);
    bi = be;
  }
};

struct MemSource : Source {
  const uint8_t *p;
  uint64_t n, o = 0, take = 0;
  MemSource(const uint8_t *p_, uint64_t n_) : p(p_), n(n_) {}
  bool done() const override { return o >= n; }
  uint64_t plan(uint64_t budget) override {
    take = std::min<uint64_t>(std::max<uint64_t>(budget, 1), n - o);
    return take;
  }
  void produce(uint8_t *dst) override {
    std::memcpy(dst, p + o, take);
    o += take;
  }
};

struct SampleOut {
  int32_t avg_read = 0;
  int64_t records = 0;
  double kernel_ms = 0;     // device time of the per-record launches
};

// Streams one sample's records through the device: sums into sum / sum_u
// (device, n_targets each).  `carry` holds the bytes before the first piece
// (the end of the header's last block).
SampleOut run_sample(rbg_ctx *c, Source &src, std::vector<uint8_t> carry, const rbg_depth_params *p,
                     const uint32_t *d_tlen, int32_t n_targets, unsigned long long *sum,
                     unsigned long long *sum_u, double &walk_ms) {
  DepthBufs &D = *c->depthb;
  cudaStream_t s = c->stream;
  for (int i = 0; i < 2; ++i) {
    if (!D.ev[i]) CK(cudaEventCreateWithFlags(&D.ev[i], cudaEventDisableTiming));
    if (!D.k0[i]) CK(cudaEventCreate(&D.k0[i]));
    if (!D.k1[i]) CK(cudaEventCreate(&D.k1[i]));
  }
  bool timed[2] = {false, false};
  const uint64_t budget = (uint64_t)std::max(1, std::min(p->chunk_mb, 4095)) << 20;
  SampleOut so;
  bool avg_final = false;
  int64_t srs = 0, src_n = 0;
  int slot = 0;
  depth::Params P{p->percent_identity, 0, p->min_map_qual, p->dual_map_qual, n_targets};
  bool edge_set = false;
  while (!src.done() || !carry.empty()) {
    const bool more = !src.done();
    const uint64_t piece = more ? src.plan(budget) : 0;
    const uint64_t bytes = carry.size() + piece;
    // the slot's last copies (of this or an earlier call) have finished; an
    // event never recorded returns at once
    CK(cudaEventSynchronize(D.ev[slot]));
    if (timed[slot]) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, D.k0[slot], D.k1[slot]));
      so.kernel_ms += ms;
      timed[slot] = false;
    }
    D.slot[slot].ensure(bytes + 16);
    uint8_t *h = D.slot[slot].as<uint8_t>();
    if (!carry.empty()) std::memcpy(h, carry.data(), carry.size());
    const auto t0 = Clock::now();
    if (more) src.produce(h + carry.size());
    // walk the records
    D.offp[slot].ensure((bytes / 36 + 2) * sizeof(uint32_t));
    uint32_t *offs = D.offp[slot].as<uint32_t>();
    if (bytes > 0xFFFFFFFFull) throw Error(RBG_ERR_ARG, "chunk too large (chunk_mb)");
    uint64_t q = 0;
    int64_t nrec = 0;
    if (!avg_final) srs = src_n = 0;         // the walk starts at the sample's first record
    while (bytes - q >= 4) {
      const int32_t bs = depth::ld_i32(h + q);
      if (bs < 32) throw Error(RBG_ERR_ARG, "malformed BAM record (block_size)");
      if (q + 4 + (uint64_t)bs > bytes) break;                    // cut by the piece's end
      if (!depth::record_bytes(h + q, bytes - q))
        throw Error(RBG_ERR_ARG, "malformed BAM record (sizes beyond block_size)");
      offs[nrec++] = (uint32_t)q;
      if (!avg_final && !(depth::ld_u16(h + q + 18) & depth::kUnmap)) {
        srs += depth::ld_i32(h + q + 20);
        if (++src_n >= 4000) avg_final = true;
      }
      q += 4 + (uint64_t)bs;
    }
    walk_ms += ms_since(t0);
    if (!more && q < bytes) throw Error(RBG_ERR_ARG, "truncated BAM record at the end of the stream");
    if (!avg_final && !src.done()) {
      // the read-length sample needs records beyond this piece: keep all bytes
      carry.assign(h, h + bytes);
      continue;
    }
    if (!edge_set) {
      if (!avg_final) avg_final = true;
      so.avg_read = src_n ? (int32_t)(srs / src_n) : 0;
      P.edge = p->include_edge_bases ? 0 : std::min(p->max_edge_bases, so.avg_read / 3);
      edge_set = true;
    }
    carry.assign(h + q, h + bytes);
    if (nrec > 0) {
      D.buf[slot].ensure(q + 16);
      D.off[slot].ensure((size_t)nrec * sizeof(uint32_t));
      CK(cudaMemcpyAsync(D.buf[slot].p, h, q, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(D.off[slot].p, offs, (size_t)nrec * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
      CK(cudaEventRecord(D.k0[slot], s));
      launch_depth_reads(D.buf[slot].as<uint8_t>(), D.off[slot].as<uint32_t>(), nrec, d_tlen, P, sum,
                         p->dual_map_qual > 0 ? sum_u : nullptr, s);
      CK(cudaGetLastError());
      CK(cudaEventRecord(D.k1[slot], s));
      timed[slot] = true;
      CK(cudaEventRecord(D.ev[slot], s));
      ++c->launches;
      so.records += nrec;
    }
    slot ^= 1;
  }
  if (!edge_set) so.avg_read = 0;
  for (int i = 0; i < 2; ++i)
    if (timed[i]) {
      CK(cudaEventSynchronize(D.k1[i]));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, D.k0[i], D.k1[i]));
      so.kernel_ms += ms;
    }
  return so;
}

struct FileView {
  const uint8_t *p = nullptr;
  uint64_t n = 0;
};

// memcpy on `threads` host threads (the copy into a pinned slot)
void par_copy(uint8_t *dst, const uint8_t *src, size_t n, int threads) {
  const size_t per = std::max<size_t>(n / (size_t)std::max(1, threads) + 1, 1 << 20);
  if (n <= per) {
    std::memcpy(dst, src, n);
    return;
  }
  std::vector<std::thread> pool;
  for (size_t a = 0; a < n; a += per)
    pool.emplace_back([=] { std::memcpy(dst + a, src + a, std::min(per, n - a)); });
  for (auto &t : pool) t.join();
}

// The header and the read-length sample of one BAM, from its first blocks
// inflated on the host (groups of `threads` blocks until 4,000 mapped records
// have been seen or the file ends).
struct Prefix {
  Header h;
  int64_t hdr_end = 0;
  int32_t avg = 0;
};

Prefix host_prefix(const FileView &f, const std::vector<Blk> &B, const std::vector<uint64_t> &uoff,
                   int threads) {
  Prefix r;
  std::vector<uint8_t> buf;
  size_t done_blocks = 0;
  uint64_t q = 0;
  int64_t srs = 0, src = 0;
  bool have_hdr = false, full = false;
  while (!full && done_blocks < B.size()) {
    const size_t take = std::min(B.size() - done_blocks, (size_t)std::max(1, threads));
    buf.resize(uoff[done_blocks + take]);
    inflate_blocks(f.p, B, uoff, done_blocks, done_blocks + take, buf.data() + uoff[done_blocks],
                   threads);
    done_blocks += take;
    if (!have_hdr) {
      r.hdr_end = parse_header(buf.data(), (int64_t)buf.size(), r.h);
      if (!r.hdr_end) continue;
      have_hdr = true;
      q = (uint64_t)r.hdr_end;
    }
    while (buf.size() - q >= 36) {
      const uint32_t rb = depth::record_bytes(buf.data() + q, buf.size() - q);
      if (!rb) break;                 // cut by the inflated prefix, or malformed
      if (!(depth::ld_u16(buf.data() + q + 18) & depth::kUnmap)) {
        srs += depth::ld_i32(buf.data() + q + 20);
        if (++src >= 4000) {
          full = true;
          break;
        }
      }
      q += rb;
    }
  }
  if (!have_hdr) throw Error(RBG_ERR_ARG, "truncated BAM header");
  r.avg = src ? (int32_t)(srs / src) : 0;
  return r;
}

// One BAM through the device route: chunks of compressed blocks are copied in
// and inflated, walked and summed on the device.  Returns false when a block
// did not start on a record (a writer that lets records cross blocks): the
// caller then clears the sums and takes the host route.
// The BAM's status goes to its 16-byte slot on the device (flags, then the
// record count; zeroed by the caller): bit 0 a block that does not inflate or
// fails its CRC32, bit 1 a block that does not start on a record.  Nothing
// waits for the device here, so the next BAM's host work overlaps this one's
// kernels; `timed` (per slot: its launch times are not read yet) and
// `kernel_ms` carry over from BAM to BAM.
void run_sample_device(rbg_ctx *c, const FileView &f, const std::vector<Blk> &B,
                       const std::vector<uint64_t> &uoff, int64_t hdr_end, const depth::Params &P,
                       const rbg_depth_params *p, const uint32_t *d_tlen, unsigned long long *sum,
                       unsigned long long *sum_u, int threads, uint8_t *slot_dev, bool timed[2],
                       double &kernel_ms) {
  DepthBufs &D = *c->depthb;
  cudaStream_t s = c->stream;
  for (int i = 0; i < 2; ++i) {
    if (!D.ev[i]) CK(cudaEventCreateWithFlags(&D.ev[i], cudaEventDisableTiming));
    if (!D.evc[i]) CK(cudaEventCreateWithFlags(&D.evc[i], cudaEventDisableTiming));
    if (!D.k0[i]) CK(cudaEventCreate(&D.k0[i]));
    if (!D.k1[i]) CK(cudaEventCreate(&D.k1[i]));
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const uint64_t budget = (uint64_t)std::max(1, std::min(p->device_chunk_mb, 3072)) << 20;
  uint32_t *flags = (uint32_t *)slot_dev;
  unsigned long long *rec_total = (unsigned long long *)(slot_dev + 8);
  size_t b0 = 0;
  int slot = 0;
  while (b0 < B.size()) {
    size_t b1 = b0;
    uint64_t bytes = 0;
    while (b1 < B.size() && (b1 == b0 || bytes + B[b1].isize <= budget)) bytes += B[b1++].isize;
    const int nb = (int)(b1 - b0);
    const uint64_t cstart = B[b0].start;
    const uint64_t cend = B[b1 - 1].cdata + B[b1 - 1].clen + 8;
    const size_t cbytes = (size_t)(cend - cstart);
    if (cbytes > 0xFFFFFFFFull) throw Error(RBG_ERR_ARG, "device chunk too large");
    CK(cudaEventSynchronize(D.ev[slot]));
    if (timed[slot]) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, D.k0[slot], D.k1[slot]));
      kernel_ms += ms;
      timed[slot] = false;
    }
    D.cpin[slot].ensure(cbytes + 16);
    const size_t tab_bytes = (size_t)nb * sizeof(DevBlk) + (size_t)(nb + 1) * 8;
    D.tpin[slot].ensure(tab_bytes);
    par_copy(D.cpin[slot].as<uint8_t>(), f.p + cstart, cbytes, threads);
    DevBlk *tb = D.tpin[slot].as<DevBlk>();
    uint64_t *ub = (uint64_t *)(D.tpin[slot].as<uint8_t>() + (size_t)nb * sizeof(DevBlk));
    for (int i = 0; i < nb; ++i) {
      const Blk &x = B[b0 + i];
      tb[i].cofs = (uint32_t)(x.cdata - cstart);
      tb[i].clen = x.clen;
      tb[i].isize = x.isize;
      tb[i].crc = x.crc;
      tb[i].uofs = uoff[b0 + i] - uoff[b0];
      ub[i] = tb[i].uofs;
    }
    ub[nb] = bytes;
    D.cdev[slot].ensure(cbytes + 16);
    D.tdev[slot].ensure(tab_bytes);
    D.outd[slot].ensure(bytes + 64);
    D.cntd[slot].ensure((size_t)(2 * nb + 2) * 4);
    D.offd[slot].ensure((size_t)(bytes / 36 + nb + 16) * 4);
    // copies on the context's copy stream, so that chunk c + 1 arrives while
    // chunk c is inflated
    CK(cudaStreamWaitEvent(c->copy, D.ev[slot], 0));
    CK(cudaMemcpyAsync(D.cdev[slot].p, D.cpin[slot].p, cbytes, cudaMemcpyHostToDevice, c->copy));
    CK(cudaMemcpyAsync(D.tdev[slot].p, D.tpin[slot].p, tab_bytes, cudaMemcpyHostToDevice, c->copy));
    CK(cudaEventRecord(D.evc[slot], c->copy));
    CK(cudaStreamWaitEvent(s, D.evc[slot], 0));
    const int64_t he = hdr_end - (int64_t)uoff[b0];
    const uint64_t hdr_chunk = he <= 0 ? 0 : std::min<uint64_t>((uint64_t)he, bytes);
    uint32_t *cnt = D.cntd[slot].as<uint32_t>();
    CK(cudaEventRecord(D.k0[slot], s));
    launch_depth_device(D.cdev[slot].as<uint8_t>(), D.tdev[slot].as<DevBlk>(), nb,
                        (const uint64_t *)(D.tdev[slot].as<uint8_t>() + (size_t)nb * sizeof(DevBlk)),
                        hdr_chunk, D.outd[slot].as<uint8_t>(), cnt, cnt + nb + 1,
                        D.offd[slot].as<uint32_t>(), flags, rec_total, d_tlen, P, sum,
                        p->dual_map_qual > 0 ? sum_u : nullptr, sms, s);
    CK(cudaGetLastError());
    CK(cudaEventRecord(D.k1[slot], s));
    CK(cudaEventRecord(D.ev[slot], s));
    timed[slot] = true;
    c->launches += 5;
    b0 = b1;
    slot ^= 1;
  }
}

void bam_depth(rbg_ctx *c, const std::vector<FileView> &files, const rbg_depth_params *p,
               rbg_depth_matrix *out) {
  const auto t_all = Clock::now();
  if (!p || !out || files.empty()) throw Error(RBG_ERR_ARG, "null argument or no BAM");
  if (p->max_edge_bases < 0 || p->chunk_mb < 0) throw Error(RBG_ERR_ARG, "negative parameter");
  std::memset(out, 0, sizeof(*out));
  if (!c->depthb) c->depthb.reset(new DepthBufs());
  DepthBufs &D = *c->depthb;
  cudaStream_t s = c->stream;
  const int threads = host_threads(p);
  const int nb = (int)files.size();
  const bool dual = p->dual_map_qual > 0;
  const int ncols = dual ? 2 * nb : nb;
  Header h0;
  std::vector<int32_t> avg(nb, 0), edge_col(ncols, 0);
  double walk_ms = 0, kernel_ms = 0;
  int64_t records = 0, cbytes = 0, ubytes = 0;
  int32_t device_bams = 0;
  bool have_h0 = false;
  auto set_h0 = [&](const Header &h) {
    h0 = h;
    have_h0 = true;
    const int32_t nt = (int32_t)h0.tlen.size();
    D.tlen.ensure(std::max<size_t>(1, (size_t)nt) * 4);
    if (nt) CK(cudaMemcpyAsync(D.tlen.p, h0.tlen.data(), (size_t)nt * 4, cudaMemcpyHostToDevice, s));
    D.sums.ensure(std::max<size_t>(1, (size_t)ncols * nt) * 8);
    CK(cudaMemsetAsync(D.sums.p, 0, std::max<size_t>(1, (size_t)ncols * nt) * 8, s));
  };
  auto index_file = [&](int b, std::vector<Blk> &B, std::vector<uint64_t> &uoff) {
    index_blocks(files[b].p, files[b].n, B);
    uoff.assign(B.size() + 1, 0);
    for (size_t i = 0; i < B.size(); ++i) uoff[i + 1] = uoff[i] + B[i].isize;
  };
  auto set_edge = [&](int b, int32_t a) {
    avg[b] = a;
    edge_col[b] = p->include_edge_bases ? 0 : std::min(p->max_edge_bases, a / 3);
    if (dual) edge_col[nb + b] = edge_col[b];
  };
  std::vector<int> host_route;
  if (p->device_inflate) {
    // every BAM through the device route without waiting in between, then one
    // read-back of all their status slots
    D.flags.ensure((size_t)16 * nb);
    CK(cudaMemsetAsync(D.flags.p, 0, (size_t)16 * nb, s));
    bool timed[2] = {false, false};
    std::vector<int32_t> pre_avg(nb, 0);
    for (int b = 0; b < nb; ++b) {
      std::vector<Blk> B;
      std::vector<uint64_t> uoff;
      index_file(b, B, uoff);
      cbytes += (int64_t)files[b].n;
      ubytes += (int64_t)uoff.back();
      const auto t0 = Clock::now();
      Prefix pre = host_prefix(files[b], B, uoff, threads);
      walk_ms += ms_since(t0);
      if (!have_h0) set_h0(pre.h);
      else if (pre.h.tlen != h0.tlen) throw Error(RBG_ERR_ARG, "BAM files carry different contigs");
      const int32_t nt = (int32_t)h0.tlen.size();
      unsigned long long *sums_all = D.sums.as<unsigned long long>();
      depth::Params P{p->percent_identity,
                      p->include_edge_bases ? 0 : std::min(p->max_edge_bases, pre.avg / 3),
                      p->min_map_qual, p->dual_map_qual, nt};
      run_sample_device(c, files[b], B, uoff, pre.hdr_end, P, p, D.tlen.as<uint32_t>(),
                        sums_all + (size_t)b * nt, sums_all + (size_t)(nb + b) * nt, threads,
                        D.flags.as<uint8_t>() + (size_t)16 * b, timed, kernel_ms);
      pre_avg[b] = pre.avg;
    }
    D.hflag.ensure((size_t)16 * nb);
    CK(cudaMemcpyAsync(D.hflag.p, D.flags.p, (size_t)16 * nb, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int i = 0; i < 2; ++i)
      if (timed[i]) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, D.k0[i], D.k1[i]));
        kernel_ms += ms;
      }
    const int32_t nt = (int32_t)h0.tlen.size();
    unsigned long long *sums_all = D.sums.as<unsigned long long>();
    for (int b = 0; b < nb; ++b) {
      const uint8_t *slot = D.hflag.as<uint8_t>() + (size_t)16 * b;
      uint32_t fl;
      uint64_t recs;
      std::memcpy(&fl, slot, 4);
      std::memcpy(&recs, slot + 8, 8);
      if (fl & 1u)
        throw Error(RBG_ERR_ARG, "BGZF block does not inflate to its stated size or fails its CRC32");
      if (fl & 2u) {
        // a block did not start on a record: this BAM takes the host route
        CK(cudaMemsetAsync(sums_all + (size_t)b * nt, 0, (size_t)nt * 8, s));
        if (dual) CK(cudaMemsetAsync(sums_all + (size_t)(nb + b) * nt, 0, (size_t)nt * 8, s));
        host_route.push_back(b);
        continue;
      }
      set_edge(b, pre_avg[b]);
      records += (int64_t)recs;
      ++device_bams;
    }
  } else {
    for (int b = 0; b < nb; ++b) host_route.push_back(b);
  }
  for (int b : host_route) {
    std::vector<Blk> B;
    std::vector<uint64_t> uoff;
    index_file(b, B, uoff);
    if (!p->device_inflate) {
      cbytes += (int64_t)files[b].n;
      ubytes += (int64_t)uoff.back();
    }
    // header: inflate blocks one by one until it is complete
    std::vector<uint8_t> hb;
    Header h;
    int64_t hlen = 0;
    size_t hblk = 0;
    while ((hlen = parse_header(hb.data(), (int64_t)hb.size(), h)) == 0) {
      if (hblk == B.size()) throw Error(RBG_ERR_ARG, "truncated BAM header");
      hb.resize(uoff[hblk + 1]);
      inflate_blocks(files[b].p, B, uoff, hblk, hblk + 1, hb.data() + uoff[hblk], 1);
      ++hblk;
    }
    if (!have_h0) set_h0(h);
    else if (h.tlen != h0.tlen) throw Error(RBG_ERR_ARG, "BAM files carry different contigs");
    const int32_t nt = (int32_t)h0.tlen.size();
    std::vector<uint8_t> carry(hb.begin() + hlen, hb.end());
    BgzfSource src(files[b].p, B, uoff, hblk, threads);
    unsigned long long *sums = D.sums.as<unsigned long long>();
    const SampleOut so = run_sample(c, src, std::move(carry), p, D.tlen.as<uint32_t>(), nt,
                                    sums + (size_t)b * nt, sums + (size_t)(nb + b) * nt, walk_ms);
    set_edge(b, so.avg_read);
    records += so.records;
    kernel_ms += so.kernel_ms;
  }
  const int32_t nt = (int32_t)h0.tlen.size();
  std::vector<int32_t> kept;
  for (int32_t t = 0; t < nt; ++t)
    if ((int32_t)h0.tlen[t] >= p->min_contig_length) kept.push_back(t);
  const int64_t nk = (int64_t)kept.size();
  D.kept.ensure(std::max<size_t>(1, (size_t)nk) * 4);
  D.edge.ensure((size_t)ncols * 4);
  D.means.ensure(std::max<size_t>(1, (size_t)nk * ncols) * 4);
  if (nk) CK(cudaMemcpyAsync(D.kept.p, kept.data(), (size_t)nk * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(D.edge.p, edge_col.data(), (size_t)ncols * 4, cudaMemcpyHostToDevice, s));
  launch_depth_means(D.sums.as<unsigned long long>(), nt, D.kept.as<int32_t>(), nk,
                     D.tlen.as<uint32_t>(), D.edge.as<int32_t>(), ncols, D.means.as<float>(), s);
  CK(cudaGetLastError());
  ++c->launches;
  // results
  size_t name_bytes = 0;
  for (int32_t t : kept) name_bytes += h0.names[t].size() + 1;
  out->n_rows = nk;
  out->n_cols = ncols;
  out->n_targets = nt;
  out->tid = (int32_t *)malloc(std::max<size_t>(1, nk) * 4);
  out->lens = (int32_t *)malloc(std::max<size_t>(1, nk) * 4);
  out->means = (float *)malloc(std::max<size_t>(1, (size_t)nk * ncols) * 4);
  out->names = (char *)malloc(std::max<size_t>(1, name_bytes));
  out->name_off = (int64_t *)malloc(std::max<size_t>(1, nk) * 8);
  out->avg_read = (int32_t *)malloc((size_t)nb * 4);
  out->sums = (uint64_t *)malloc(std::max<size_t>(1, (size_t)ncols * nt) * 8);
  if (!out->tid || !out->lens || !out->means || !out->names || !out->name_off || !out->avg_read ||
      !out->sums) {
    rbg_free_depth_matrix(out);
    throw Error(RBG_ERR_NOMEM, "host allocation failed");
  }
  if (nk * ncols)
    CK(cudaMemcpyAsync(out->means, D.means.p, (size_t)nk * ncols * 4, cudaMemcpyDeviceToHost, s));
  if ((size_t)ncols * nt)
    CK(cudaMemcpyAsync(out->sums, D.sums.p, (size_t)ncols * nt * 8, cudaMemcpyDeviceToHost, s));
  size_t o = 0;
  for (int64_t r = 0; r < nk; ++r) {
    const int32_t t = kept[r];
    out->tid[r] = t;
    out->lens[r] = (int32_t)h0.tlen[t];
    out->name_off[r] = (int64_t)o;
    std::memcpy(out->names + o, h0.names[t].c_str(), h0.names[t].size() + 1);
    o += h0.names[t].size() + 1;
  }
  std::memcpy(out->avg_read, avg.data(), (size_t)nb * 4);
  CK(cudaStreamSynchronize(s));
  out->records = records;
  out->compressed_bytes = cbytes;
  out->decompressed_bytes = ubytes;
  out->inflate_ms = (float)walk_ms;
  out->total_ms = (float)ms_since(t_all);
  out->kernel_ms = (float)kernel_ms;
  out->device_bams = device_bams;
}

}  // namespace
}  // namespace rbg

using namespace rbg;

extern "C" {

int rbg_default_depth_params(rbg_depth_params *p) {
  if (!p) return RBG_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->percent_identity = 97.0f / 100.0f;   // src/rabbitbin.cpp:3428, :3749
  p->min_contig_length = 1;               // src/rabbitbin.cpp:6383
  p->max_edge_bases = 75;
  p->include_edge_bases = 0;
  p->min_map_qual = 0;
  p->dual_map_qual = 0;
  p->threads = 0;
  p->chunk_mb = 64;
  p->device_inflate = 1;
  p->device_chunk_mb = 1024;
  return RBG_OK;
}

int rbg_free_depth_matrix(rbg_depth_matrix *m) {
  if (!m) return RBG_ERR_ARG;
  free(m->tid);
  free(m->lens);
  free(m->means);
  free(m->names);
  free(m->name_off);
  free(m->avg_read);
  free(m->sums);
  std::memset(m, 0, sizeof(*m));
  return RBG_OK;
}

int rbg_bam_depth_mem(rbg_ctx *c, const uint8_t *const *bam_bytes, const int64_t *bam_sizes,
                      int32_t n_bams, const rbg_depth_params *p, rbg_depth_matrix *out) {
  return guarded(c, [&] {
    if (!bam_bytes || !bam_sizes || n_bams < 1) throw Error(RBG_ERR_ARG, "null argument or no BAM");
    std::vector<FileView> files((size_t)n_bams);
    for (int32_t b = 0; b < n_bams; ++b) {
      if (!bam_bytes[b] || bam_sizes[b] < 0) throw Error(RBG_ERR_ARG, "null or negative BAM buffer");
      files[b].p = bam_bytes[b];
      files[b].n = (uint64_t)bam_sizes[b];
    }
    bam_depth(c, files, p, out);
  });
}

int rbg_bam_depth(rbg_ctx *c, const char *const *paths, int32_t n_bams, const rbg_depth_params *p,
                  rbg_depth_matrix *out) {
  return guarded(c, [&] {
    if (!paths || n_bams < 1) throw Error(RBG_ERR_ARG, "null argument or no BAM");
    // the files are mapped read-only, not read into memory: BAMs can be far
    // larger than the host's memory, and every byte is touched once
    struct Mapped {
      void *p = MAP_FAILED;
      size_t n = 0;
      ~Mapped() {
        if (p != MAP_FAILED && n) munmap(p, n);
      }
    };
    std::vector<Mapped> maps((size_t)n_bams);
    std::vector<FileView> files((size_t)n_bams);
    for (int32_t b = 0; b < n_bams; ++b) {
      if (!paths[b]) throw Error(RBG_ERR_ARG, "null BAM path");
      const int fd = open(paths[b], O_RDONLY);
      if (fd < 0) throw Error(RBG_ERR_ARG, std::string("cannot open ") + paths[b]);
      struct stat st;
      if (fstat(fd, &st) != 0) {
        close(fd);
        throw Error(RBG_ERR_ARG, std::string("cannot size ") + paths[b]);
      }
      maps[b].n = (size_t)st.st_size;
      if (maps[b].n) {
        maps[b].p = mmap(nullptr, maps[b].n, PROT_READ, MAP_PRIVATE, fd, 0);
        if (maps[b].p == MAP_FAILED) {
          close(fd);
          throw Error(RBG_ERR_ARG, std::string("cannot map ") + paths[b]);
        }
        madvise(maps[b].p, maps[b].n, MADV_SEQUENTIAL);
      }
      close(fd);
      static const uint8_t none = 0;
      files[b].p = maps[b].n ? (const uint8_t *)maps[b].p : &none;
      files[b].n = (uint64_t)maps[b].n;
    }
    bam_depth(c, files, p, out);
  });
}

int rbg_depth_tsv(const rbg_depth_matrix *m, const char *const *bam_names, int32_t n_bams,
                  const rbg_depth_params *p, int32_t intra_depth_variance, char **tsv,
                  int64_t *tsv_len) {
  if (!m || !bam_names || n_bams < 1 || !p || !tsv || !tsv_len) return RBG_ERR_ARG;
  if ((m->n_cols != n_bams && m->n_cols != 2 * n_bams) || !m->avg_read ||
      (m->n_rows > 0 && (!m->tid || !m->lens || !m->names || !m->name_off || !m->sums)))
    return RBG_ERR_ARG;
  for (int32_t b = 0; b < n_bams; ++b)
    if (!bam_names[b]) return RBG_ERR_ARG;
  try {
    const int nb = n_bams;
    const int64_t nt = m->n_targets;
    int min_avg = INT32_MAX;
    for (int b = 0; b < nb; ++b) min_avg = std::min(min_avg, (int)m->avg_read[b]);
    const int edge_all = std::min(p->max_edge_bases, min_avg / 3);
    std::string out;
    out.reserve((size_t)(m->n_rows + 1) * (24 + 12 * (size_t)nb));
    out += "contigName\tcontigLen\ttotalAvgDepth";
    for (int b = 0; b < nb; ++b) {
      // the file's base name: no directories, no extension
      std::string n(bam_names[b]);
      const size_t sl = n.find_last_of('/');
      if (sl != std::string::npos) n = n.substr(sl + 1);
      const size_t dot = n.find_last_of('.');
      if (dot != std::string::npos) n = n.substr(0, dot);
      out += "\t" + n;
      if (intra_depth_variance) out += "\t" + n + "-var";
    }
    out += "\n";
    // rows [r0, r1) into `dst`
    auto rows = [&](int64_t r0, int64_t r1, std::string &dst) {
      auto put_float = [&](double v) {
        char b[64];
        const int k = std::snprintf(b, sizeof b, "%g", (double)(float)v);
        dst.append(b, (size_t)k);
      };
      std::vector<double> mv((size_t)nb);
      for (int64_t r = r0; r < r1; ++r) {
        const int32_t t = m->tid[r], cl = m->lens[r];
        double weighted = 0.0;
        uint64_t total_len = 0;
        for (int b = 0; b < nb; ++b) {
          // corrected length: 2 min(edge, avg_read / 3) bases fewer, unless that
          // is the whole contig or edges are included
          const int x = 2 * std::min(edge_all, (int)m->avg_read[b] / 3);
          const int corr = (p->include_edge_bases || x >= cl) ? cl : cl - x;
          const uint64_t sum = m->sums[(size_t)b * (size_t)nt + (size_t)t];
          double mean;
          if (intra_depth_variance) {
            const int e = p->include_edge_bases ? 0 : std::min(p->max_edge_bases, (int)m->avg_read[b] / 3);
            const int32_t adj = (cl > 2 * e + 1) ? (cl - 2 * e) : cl;
            mean = (double)(adj > 2 ? (float)((double)sum / (double)adj) : 0.0f);
          } else {
            mean = corr > 0 ? (double)(sum / (uint64_t)corr) : 0.0;   // integer quotient
          }
          if (mean > 1000000) mean = 0;
          total_len += (uint64_t)(int64_t)corr;
          // with the variance columns the mean is a float and its product with
          // the corrected length is a float product, as the reference forms it
          weighted += intra_depth_variance ? (double)((float)mean * (float)corr) : mean * corr;
          mv[b] = mean;
        }
        double total = total_len > 0 ? weighted / (double)total_len : 0.0;
        total *= nb;
        const char *name = m->names + m->name_off[r];
        dst.append(name, std::strcspn(name, " \t"));
        dst += '\t';
        dst += std::to_string(cl);
        dst += '\t';
        put_float(total);
        for (int b = 0; b < nb; ++b) {
          dst += '\t';
          put_float(mv[b]);
          if (intra_depth_variance) {
            dst += '\t';
            put_float(0.0);
          }
        }
        dst += '\n';
      }
    };
    // contiguous row ranges formatted on host threads, joined in row order
    const int64_t cells = m->n_rows * (int64_t)(nb + 1);
    const int nth = (int)std::max<int64_t>(1, std::min<int64_t>(host_threads(p), cells / 20000));
    if (nth <= 1) {
      rows(0, m->n_rows, out);
    } else {
      std::vector<std::string> part((size_t)nth);
      std::vector<std::thread> pool;
      std::atomic<int> nomem{0};
      for (int i = 0; i < nth; ++i)
        pool.emplace_back([&, i] {
          try {
            rows(m->n_rows * i / nth, m->n_rows * (i + 1) / nth, part[(size_t)i]);
          } catch (const std::bad_alloc &) {
            nomem = 1;
          }
        });
      for (auto &th : pool) th.join();
      if (nomem) return RBG_ERR_NOMEM;
      for (auto &x : part) out += x;
    }
    char *buf = (char *)malloc(out.size() + 1);
    if (!buf) return RBG_ERR_NOMEM;
    std::memcpy(buf, out.c_str(), out.size() + 1);
    *tsv = buf;
    *tsv_len = (int64_t)out.size();
    return RBG_OK;
  } catch (const std::bad_alloc &) {
    return RBG_ERR_NOMEM;
  }
}

int rbg_free_tsv(char *tsv) {
  free(tsv);
  return RBG_OK;
}

int rbg_depth_accumulate(rbg_ctx *c, const uint8_t *records, int64_t n_bytes,
                         const uint32_t *target_len, int32_t n_targets, const rbg_depth_params *p,
                         uint64_t *depth_out, uint64_t *depth_u_out, int32_t *avg_read) {
  return guarded(c, [&] {
    if (!p || n_bytes < 0 || n_targets < 0 || (n_bytes > 0 && !records) ||
        (n_targets > 0 && (!target_len || !depth_out)))
      throw Error(RBG_ERR_ARG, "null or negative argument");
    if (!c->depthb) c->depthb.reset(new DepthBufs());
    DepthBufs &D = *c->depthb;
    cudaStream_t s = c->stream;
    const size_t nt = (size_t)n_targets;
    D.tlen.ensure(std::max<size_t>(1, nt) * 4);
    D.sums.ensure(std::max<size_t>(1, 2 * nt) * 8);
    if (nt) CK(cudaMemcpyAsync(D.tlen.p, target_len, nt * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(D.sums.p, 0, std::max<size_t>(1, 2 * nt) * 8, s));
    MemSource src(records, (uint64_t)n_bytes);
    double walk_ms = 0;
    unsigned long long *sums = D.sums.as<unsigned long long>();
    const SampleOut so = run_sample(c, src, {}, p, D.tlen.as<uint32_t>(), n_targets, sums,
                                    sums + nt, walk_ms);
    if (nt) CK(cudaMemcpyAsync(depth_out, D.sums.p, nt * 8, cudaMemcpyDeviceToHost, s));
    if (nt && depth_u_out)
      CK(cudaMemcpyAsync(depth_u_out, sums + nt, nt * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (avg_read) *avg_read = so.avg_read;
  });
}

}  // extern "C"
