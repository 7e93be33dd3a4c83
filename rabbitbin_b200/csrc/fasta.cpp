// FASTA ingest on the device: the host side of kernels_fasta.cu and the C ABI
// entry points rbg_parse_fasta / rbg_free_fasta.  rbg_bin_fasta (engine.cpp)
// feeds the parsed large contigs straight into the hot path without a host
// round trip of the sequences.
#include <cstdlib>
#include <cstring>

#include "engine_internal.h"

namespace rbg {

FastaCounts fasta_parse(rbg_ctx *c, const char *data, int64_t F, int64_t min_contig,
                        int64_t min_small) {
  if (F < 0 || (F > 0 && !data)) throw Error(RBG_ERR_ARG, "bad FASTA buffer");
  if (min_contig < 1 || min_small < 1) throw Error(RBG_ERR_ARG, "minimum lengths must be >= 1");
  if (!c->fasta) c->fasta = std::make_unique<FastaBufs>();
  FastaBufs &B = *c->fasta;
  cudaStream_t s = c->stream;
  FastaCounts out;
  const int64_t words = (F + 15) / 16;
  const int64_t tiles = (words + 255) / 256;
  B.in.ensure((size_t)words * 16 + 16);
  CK(cudaMemsetAsync(B.in.p, 0, (size_t)words * 16 + 16, s));
  if (F) CK(cudaMemcpyAsync(B.in.p, data, (size_t)F, cudaMemcpyHostToDevice, s));
  const uint8_t *in = B.in.as<uint8_t>();
  B.tile_nl.ensure(std::max<int64_t>(tiles, 1) * sizeof(int));
  B.tile_gt.ensure(std::max<int64_t>(tiles, 1) * sizeof(int));
  B.nl_base.ensure((tiles + 1) * sizeof(int64_t));
  B.gt_base.ensure((tiles + 1) * sizeof(int64_t));
  CK(cudaMemsetAsync(B.nl_base.p, 0, (tiles + 1) * sizeof(int64_t), s));
  CK(cudaMemsetAsync(B.gt_base.p, 0, (tiles + 1) * sizeof(int64_t), s));
  launch_fasta_positions(in, F, B.tile_nl.as<int>(), B.tile_gt.as<int>(), B.nl_base.as<int64_t>(),
                         B.gt_base.as<int64_t>(), s);
  int64_t nnl = 0, ngt = 0;
  CK(cudaMemcpyAsync(&nnl, B.nl_base.as<int64_t>() + tiles, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&ngt, B.gt_base.as<int64_t>() + tiles, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  B.nl_pos.ensure(std::max<int64_t>(nnl, 1) * sizeof(int64_t));
  B.gt_pos.ensure(std::max<int64_t>(ngt, 1) * sizeof(int64_t));
  launch_fasta_scatter(in, F, B.nl_base.as<int64_t>(), B.gt_base.as<int64_t>(),
                       B.nl_pos.as<int64_t>(), B.gt_pos.as<int64_t>(), s);
  B.flag.ensure((ngt + 1) * sizeof(int64_t));
  B.rs.ensure(std::max<int64_t>(ngt, 1) * sizeof(int64_t));
  CK(cudaMemsetAsync(B.flag.p, 0, (ngt + 1) * sizeof(int64_t), s));
  launch_fasta_starts(B.gt_pos.as<int64_t>(), ngt, B.nl_pos.as<int64_t>(), nnl,
                      B.flag.as<int64_t>(), B.rs.as<int64_t>(), s);
  int64_t nrs = 0;
  CK(cudaMemcpyAsync(&nrs, B.flag.as<int64_t>() + ngt, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  B.rec.ensure(std::max<int64_t>(nrs, 1) * sizeof(FastaRec));
  launch_fasta_records(in, F, B.rs.as<int64_t>(), nrs, B.nl_pos.as<int64_t>(), nnl, min_contig,
                       min_small, B.rec.as<FastaRec>(), s);
  // records without a header newline (a suffix of the records) are not counted
  int64_t dropped = 0;
  {
    B.idx[0].ensure((nrs + 1) * sizeof(int64_t));
    B.off[0].ensure((nrs + 1) * sizeof(int64_t));
    CK(cudaMemsetAsync(B.idx[0].p, 0, (nrs + 1) * sizeof(int64_t), s));
    launch_fasta_class(B.rec.as<FastaRec>(), nrs, 3, B.idx[0].as<int64_t>(), B.off[0].as<int64_t>(), s);
    CK(cudaMemcpyAsync(&dropped, B.idx[0].as<int64_t>() + nrs, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }
  out.num_seqs = nrs - dropped;
  for (int slot = 0; slot < 2; ++slot) {
    const int cls = slot == 0 ? 2 : 1;
    B.idx[slot].ensure((nrs + 1) * sizeof(int64_t));
    B.off[slot].ensure((nrs + 1) * sizeof(int64_t));
    CK(cudaMemsetAsync(B.idx[slot].p, 0, (nrs + 1) * sizeof(int64_t), s));
    CK(cudaMemsetAsync(B.off[slot].p, 0, (nrs + 1) * sizeof(int64_t), s));
    launch_fasta_class(B.rec.as<FastaRec>(), nrs, cls, B.idx[slot].as<int64_t>(),
                       B.off[slot].as<int64_t>(), s);
    int64_t cnt[2] = {0, 0};
    CK(cudaMemcpyAsync(&cnt[0], B.idx[slot].as<int64_t>() + nrs, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&cnt[1], B.off[slot].as<int64_t>() + nrs, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    out.n[slot] = cnt[0];
    out.bytes[slot] = cnt[1];
    const size_t sb = (size_t)((cnt[1] + 15) / 16) * 16 + 16;
    B.seq[slot].ensure(sb);
    B.seq_off[slot].ensure((cnt[0] + 1) * sizeof(int64_t));
    B.name_start[slot].ensure(std::max<int64_t>(cnt[0], 1) * sizeof(int64_t));
    B.name_len[slot].ensure(std::max<int64_t>(cnt[0], 1) * sizeof(int32_t));
    CK(cudaMemsetAsync(B.seq[slot].p, 0, sb, s));
    CK(cudaMemsetAsync(B.seq_off[slot].p, 0, (cnt[0] + 1) * sizeof(int64_t), s));
    launch_fasta_copy(in, B.rec.as<FastaRec>(), nrs, B.nl_pos.as<int64_t>(), cls,
                      B.idx[slot].as<int64_t>(), B.off[slot].as<int64_t>(),
                      B.seq[slot].as<uint8_t>(), B.seq_off[slot].as<int64_t>(),
                      B.name_start[slot].as<int64_t>(), B.name_len[slot].as<int32_t>(), s);
  }
  CK(cudaGetLastError());
  return out;
}

}  // namespace rbg

extern "C" {

int rbg_parse_fasta(rbg_ctx *c, const char *fasta, int64_t nbytes, int64_t min_contig,
                    int64_t min_small_contig, rbg_fasta *out) {
  if (!out) return RBG_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  return rbg::guarded(c, [&] {
    const rbg::FastaCounts k = rbg::fasta_parse(c, fasta, nbytes, min_contig, min_small_contig);
    rbg::FastaBufs &B = *c->fasta;
    out->num_seqs = k.num_seqs;
    out->n_large = k.n[0];
    out->n_small = k.n[1];
    char **seq[2] = {&out->large_seq, &out->small_seq};
    int64_t **off[2] = {&out->large_off, &out->small_off};
    int64_t **ns[2] = {&out->large_name_start, &out->small_name_start};
    int32_t **nl[2] = {&out->large_name_len, &out->small_name_len};
    for (int slot = 0; slot < 2; ++slot) {
      const int64_t n = k.n[slot];
      *seq[slot] = (char *)malloc((size_t)k.bytes[slot] + 1);
      *off[slot] = (int64_t *)malloc((size_t)(n + 1) * sizeof(int64_t));
      *ns[slot] = (int64_t *)malloc((size_t)std::max<int64_t>(n, 1) * sizeof(int64_t));
      *nl[slot] = (int32_t *)malloc((size_t)std::max<int64_t>(n, 1) * sizeof(int32_t));
      if (!*seq[slot] || !*off[slot] || !*ns[slot] || !*nl[slot]) {
        rbg_free_fasta(out);
        throw rbg::Error(RBG_ERR_NOMEM, "host allocation of the parsed contigs failed");
      }
      if (k.bytes[slot])
        CK(cudaMemcpyAsync(*seq[slot], B.seq[slot].p, (size_t)k.bytes[slot], cudaMemcpyDeviceToHost,
                           c->stream));
      CK(cudaMemcpyAsync(*off[slot], B.seq_off[slot].p, (size_t)(n + 1) * sizeof(int64_t),
                         cudaMemcpyDeviceToHost, c->stream));
      if (n) {
        CK(cudaMemcpyAsync(*ns[slot], B.name_start[slot].p, (size_t)n * sizeof(int64_t),
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(*nl[slot], B.name_len[slot].p, (size_t)n * sizeof(int32_t),
                           cudaMemcpyDeviceToHost, c->stream));
      }
    }
    CK(cudaStreamSynchronize(c->stream));
  });
}

int rbg_free_fasta(rbg_fasta *f) {
  if (!f) return RBG_ERR_ARG;
  void *ps[] = {f->large_seq, f->large_off, f->large_name_start, f->large_name_len,
                f->small_seq, f->small_off, f->small_name_start, f->small_name_len};
  for (void *p : ps) free(p);
  std::memset(f, 0, sizeof(*f));
  return RBG_OK;
}

}  // extern "C"
