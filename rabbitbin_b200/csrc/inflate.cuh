// DEFLATE decoder (RFC 1951) for one BGZF block, host and device.
//
// A BGZF member holds at most 64 KiB of output, and its deflate stream refers
// only to bytes of the same member, so every block decodes on its own: the
// device runs one warp per block.  All lanes of the warp decode the same
// symbols in lockstep (same bits, same tables: no divergence, broadcast loads);
// the leader lane stores literals, and the lanes copy matches and stored
// blocks together, in rounds no longer than the match distance so that every
// byte read was written in an earlier round.  The same code runs on the host
// with one lane (the CPU tests).  Symbols are decoded with a 9-bit (literal /
// length) and 8-bit (distance) lookup table of 32-bit entries that carry each
// symbol's meaning (literal byte, length or distance base, extra bits), with
// the canonical code walk for longer codes.  Every read stays inside [in, in + inlen),
// every write inside [out, out + outlen), and every match must point into
// bytes already written: a stream that breaks a rule ends with a status, never
// with an access out of bounds.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define RBG_IHD __host__ __device__ __forceinline__
#else
#define RBG_IHD inline
#endif

namespace rbg {
namespace inflate {

enum Status : int32_t {
  kOk = 0,
  kErrInput = 1,        // the stream ends early
  kErrBlockType = 2,    // reserved block type 3
  kErrStored = 3,       // stored block length and its complement disagree
  kErrCodes = 4,        // over-subscribed or empty code lengths, bad repeat
  kErrSymbol = 5,       // a code that is not in the table, or symbol 286/287, 30/31
  kErrDistance = 6,     // a match reaching before the start of the output
  kErrOutput = 7,       // more output than the block's ISIZE
  kErrShort = 8         // less output than the block's ISIZE
};

constexpr int kLitBits = 9, kDistBits = 8;

// The lanes that decode one block: one host thread, or one device warp.
struct SerialLanes {
  RBG_IHD int lane() const { return 0; }
  RBG_IHD int width() const { return 1; }
  RBG_IHD bool leader() const { return true; }
  RBG_IHD void sync() const {}
};
#ifdef __CUDACC__
struct WarpLanes {
  int l;
  __device__ __forceinline__ int lane() const { return l; }
  __device__ __forceinline__ int width() const { return 32; }
  __device__ __forceinline__ bool leader() const { return l == 0; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
};
#endif

// One Huffman code: lookup table for codes up to kBits bits and the canonical
// tables for the rest.  A table entry carries what the symbol means, so the
// decode loop needs no per-symbol arithmetic:
//   bits 0-3   code length (0: longer code, or no code)
//   bits 4-5   kind: 0 literal / distance / code-length symbol, 1 length,
//              2 end of block, 3 invalid symbol
//   bits 6-9   extra bits that follow the code
//   bits 16-31 value: the literal byte, the length or distance base, or the
//              code-length symbol
template <int kBits, int kSyms>
struct Code {
  uint32_t lut[1 << kBits];
  uint16_t count[16];
  uint16_t sym[kSyms];
};
constexpr uint32_t kEndOfInput = 0xFFFFFFFFu, kNoCode = 0xFFFFFFFEu;

struct Tables {
  Code<kLitBits, 288> lit;
  Code<kDistBits, 32> dist;
  uint8_t lens[320];          // code lengths being read (litlen then distance)
};

struct Bits {
  const uint8_t *p;
  uint32_t n, pos;
  uint64_t buf;
  int cnt;
  RBG_IHD void refill() {
#ifdef __CUDA_ARCH__
    // two aligned 8-byte loads and a funnel shift; the device buffers hold the
    // input from a 256-byte aligned start with 16 bytes of slack after its end,
    // and bytes past the stream's end are masked off
    if (pos >= n || cnt > 56) return;
    const uintptr_t a = (uintptr_t)(p + pos);
    const uint64_t *q = (const uint64_t *)(a & ~(uintptr_t)7);
    const uint32_t sh = (uint32_t)(a & 7) * 8;
    uint64_t w = __ldg(q) >> sh;
    if (sh) w |= __ldg(q + 1) << (64 - sh);
    uint32_t take = (uint32_t)(63 - cnt) >> 3;
    if (take > n - pos) take = n - pos;
    w &= take >= 8 ? ~0ull : ((1ull << (8 * take)) - 1);
    buf |= w << cnt;
    pos += take;
    cnt += 8 * (int)take;
#else
    while (cnt <= 56 && pos < n) {
      buf |= (uint64_t)p[pos++] << cnt;
      cnt += 8;
    }
#endif
  }
  RBG_IHD bool need(int k) {
    if (cnt < k) refill();
    return cnt >= k;
  }
  RBG_IHD uint32_t peek(int k) const { return (uint32_t)(buf & ((1ull << k) - 1)); }
  RBG_IHD void drop(int k) {
    buf >>= k;
    cnt -= k;
  }
  RBG_IHD bool get(int k, uint32_t &v) {
    if (!need(k)) return false;
    v = peek(k);
    drop(k);
    return true;
  }
};

RBG_IHD uint32_t reverse_bits(uint32_t v, int n) {
  uint32_t r = 0;
  for (int i = 0; i < n; ++i) {
    r = (r << 1) | (v & 1);
    v >>= 1;
  }
  return r;
}

// Length symbols 257 + i: i < 8 give 3 + i with no extra bits; then groups of
// four with e = (i - 4) / 4 extra bits starting at ((4 + (i & 3)) << e) + 3;
// i = 28 (symbol 285) is 258.  Distance symbols d < 4 give d + 1; then pairs
// with e = (d - 2) / 2 extra bits starting at ((2 + (d & 1)) << e) + 1.
RBG_IHD int len_extra(int i) { return (i < 8 || i == 28) ? 0 : (i - 4) / 4; }
RBG_IHD uint32_t len_base(int i) {
  return i < 8 ? 3u + i : (i == 28 ? 258u : ((4u + (i & 3)) << len_extra(i)) + 3u);
}
RBG_IHD int dist_extra(int d) { return d < 4 ? 0 : (d - 2) / 2; }
RBG_IHD uint32_t dist_base(int d) { return d < 4 ? 1u + d : ((2u + (d & 1)) << dist_extra(d)) + 1u; }


// Table entries of the three codes.
struct LitEntry {
  RBG_IHD static uint32_t make(int s, int l) {
    if (s < 256) return (uint32_t)s << 16 | (uint32_t)l;
    if (s == 256) return 2u << 4 | (uint32_t)l;
    const int i = s - 257;
    if (i >= 29) return 3u << 4 | (uint32_t)l;
    return len_base(i) << 16 | (uint32_t)len_extra(i) << 6 | 1u << 4 | (uint32_t)l;
  }
};
struct DistEntry {
  RBG_IHD static uint32_t make(int s, int l) {
    if (s >= 30) return 3u << 4 | (uint32_t)l;
    return dist_base(s) << 16 | (uint32_t)dist_extra(s) << 6 | (uint32_t)l;
  }
};
struct PlainEntry {
  RBG_IHD static uint32_t make(int s, int l) { return (uint32_t)s << 16 | (uint32_t)l; }
};

// Builds a code from `n` code lengths.  Incomplete codes are accepted (a code
// of one distance symbol is legal); over-subscribed ones are not.
template <class Entry, int kBits, int kSyms>
RBG_IHD int build(Code<kBits, kSyms> &c, const uint8_t *len, int n) {
  for (int i = 0; i < 16; ++i) c.count[i] = 0;
  for (int s = 0; s < n; ++s) c.count[len[s]]++;
  c.count[0] = 0;
  int left = 1;
  for (int l = 1; l < 16; ++l) {
    left <<= 1;
    left -= c.count[l];
    if (left < 0) return kErrCodes;
  }
  uint16_t offs[16];
  offs[1] = 0;
  for (int l = 1; l < 15; ++l) offs[l + 1] = (uint16_t)(offs[l] + c.count[l]);
  for (int s = 0; s < n; ++s)
    if (len[s]) c.sym[offs[len[s]]++] = (uint16_t)s;
  for (int i = 0; i < (1 << kBits); ++i) c.lut[i] = 0;
  // canonical codes in symbol order, entered bit-reversed into the table
  uint32_t code = 0, next[16];
  for (int l = 1; l < 16; ++l) {
    code = (code + c.count[l - 1]) << 1;
    next[l] = code;
  }
  for (int s = 0; s < n; ++s) {
    const int l = len[s];
    if (!l) continue;
    const uint32_t cd = next[l]++;
    if (l > kBits) continue;
    const uint32_t r = reverse_bits(cd, l);
    const uint32_t e = Entry::make(s, l);
    for (uint32_t f = r; f < (1u << kBits); f += (1u << l)) c.lut[f] = e;
  }
  return kOk;
}

// Decodes one symbol and returns its table entry; kEndOfInput when the stream
// ends, kNoCode for a code that is not in the table.
template <class Entry, int kBits, int kSyms>
RBG_IHD uint32_t decode(const Code<kBits, kSyms> &c, Bits &b) {
  if (b.cnt < 15) b.refill();
  // bits above cnt are zero, so the table index is defined near the end too;
  // an entry counts only when its whole code is in the buffer
  const uint32_t e = c.lut[b.peek(kBits)];
  if (e && (int)(e & 15) <= b.cnt) {
    b.drop(e & 15);
    return e;
  }
  // canonical walk, one bit at a time (codes longer than the table)
  int code = 0, first = 0, index = 0;
  for (int l = 1; l < 16; ++l) {
    if (!b.need(1)) return kEndOfInput;
    code |= (int)b.peek(1);
    b.drop(1);
    const int cnt = c.count[l];
    if (code - cnt < first) return Entry::make(c.sym[index + (code - first)], l);
    index += cnt;
    first += cnt;
    first <<= 1;
    code <<= 1;
  }
  return kNoCode;
}

// Inflates one raw deflate stream into out[0, outlen).  Returns kOk when the
// final block ends with exactly outlen bytes written.
template <class Lanes>
RBG_IHD int inflate_block(const uint8_t *in, uint32_t inlen, uint8_t *out, uint32_t outlen,
                          Tables &T, const Lanes &L) {
  const int lane = L.lane(), W = L.width();
  Bits b{in, inlen, 0, 0, 0};
  uint32_t o = 0;
  for (;;) {
    uint32_t hdr;
    if (!b.get(3, hdr)) return kErrInput;
    const uint32_t final = hdr & 1, type = hdr >> 1;
    if (type == 0) {
      // stored: skip to a byte boundary, LEN, NLEN, bytes
      b.drop(b.cnt & 7);
      uint32_t len, nlen;
      if (!b.get(16, len) || !b.get(16, nlen)) return kErrInput;
      if ((len ^ 0xffffu) != nlen) return kErrStored;
      // bytes still held in the bit buffer come first
      while (len && b.cnt >= 8) {
        if (o >= outlen) return kErrOutput;
        if (L.leader()) out[o] = (uint8_t)b.peek(8);
        ++o;
        b.drop(8);
        --len;
      }
      if (len > b.n - b.pos) return kErrInput;
      if (len > outlen - o) return kErrOutput;
      for (uint32_t i = lane; i < len; i += W) out[o + i] = b.p[b.pos + i];
      o += len;
      b.pos += len;
    } else if (type == 1 || type == 2) {
      // no lane may still read the previous block's tables
      L.sync();
      int nlen = 288, ndist = 30;
      if (type == 1) {
        for (int s = 0; s < 144; ++s) T.lens[s] = 8;
        for (int s = 144; s < 256; ++s) T.lens[s] = 9;
        for (int s = 256; s < 280; ++s) T.lens[s] = 7;
        for (int s = 280; s < 288; ++s) T.lens[s] = 8;
        for (int s = 0; s < 30; ++s) T.lens[288 + s] = 5;
      } else {
        uint32_t hlit, hdist, hclen;
        if (!b.get(5, hlit) || !b.get(5, hdist) || !b.get(4, hclen)) return kErrInput;
        nlen = (int)hlit + 257;
        ndist = (int)hdist + 1;
        if (nlen > 286 || ndist > 30) return kErrCodes;
        // code-length code: lengths in the fixed permuted order
        const uint8_t ord[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
        uint8_t cl[19];
        for (int i = 0; i < 19; ++i) cl[i] = 0;
        for (uint32_t i = 0; i < hclen + 4; ++i) {
          uint32_t v;
          if (!b.get(3, v)) return kErrInput;
          cl[ord[i]] = (uint8_t)v;
        }
        // the code-length code decodes through the distance table's storage
        // (it has 19 symbols and codes of at most 7 bits)
        Code<kDistBits, 32> &cc = T.dist;
        if (build<PlainEntry>(cc, cl, 19) != kOk) return kErrCodes;
        L.sync();
        int i = 0;
        while (i < nlen + ndist) {
          const uint32_t ce = decode<PlainEntry>(cc, b);
          if (ce >= kNoCode) return ce == kEndOfInput ? kErrInput : kErrSymbol;
          const int sym = (int)(ce >> 16);
          if (sym < 16) {
            T.lens[i < nlen ? i : 288 + (i - nlen)] = (uint8_t)sym;
            ++i;
            continue;
          }
          uint32_t rep;
          uint8_t val = 0;
          if (sym == 16) {
            if (i == 0) return kErrCodes;
            const int prev = i - 1;
            val = T.lens[prev < nlen ? prev : 288 + (prev - nlen)];
            if (!b.get(2, rep)) return kErrInput;
            rep += 3;
          } else if (sym == 17) {
            if (!b.get(3, rep)) return kErrInput;
            rep += 3;
          } else {
            if (!b.get(7, rep)) return kErrInput;
            rep += 11;
          }
          if ((int)(i + rep) > nlen + ndist) return kErrCodes;
          for (uint32_t r = 0; r < rep; ++r, ++i) T.lens[i < nlen ? i : 288 + (i - nlen)] = val;
        }
        if (T.lens[256] == 0) return kErrCodes;       // no end-of-block code
      }
      L.sync();
      if (build<LitEntry>(T.lit, T.lens, nlen) != kOk) return kErrCodes;
      if (build<DistEntry>(T.dist, T.lens + 288, ndist) != kOk) return kErrCodes;
      L.sync();
      for (;;) {
        const uint32_t e = decode<LitEntry>(T.lit, b);
        if (e >= kNoCode) return e == kEndOfInput ? kErrInput : kErrSymbol;
        const uint32_t kind = (e >> 4) & 3;
        if (kind == 0) {
          if (o >= outlen) return kErrOutput;
          if (L.leader()) out[o] = (uint8_t)(e >> 16);
          ++o;
          continue;
        }
        if (kind == 2) break;
        if (kind == 3) return kErrSymbol;
        uint32_t len = e >> 16, ex;
        const int le = (int)((e >> 6) & 15);
        if (le) {
          if (!b.get(le, ex)) return kErrInput;
          len += ex;
        }
        const uint32_t d = decode<DistEntry>(T.dist, b);
        if (d >= kNoCode) return d == kEndOfInput ? kErrInput : kErrSymbol;
        if (((d >> 4) & 3) == 3) return kErrSymbol;
        uint32_t dist = d >> 16;
        const int de = (int)((d >> 6) & 15);
        if (de) {
          if (!b.get(de, ex)) return kErrInput;
          dist += ex;
        }
        if (dist > o) return kErrDistance;
        if (len > outlen - o) return kErrOutput;
        // rounds of at most `dist` bytes: each round reads only bytes written
        // before it (the leader's literals included, after the barrier)
        L.sync();
        const uint8_t *src = out + (o - dist);
        uint8_t *dst = out + o;
        for (uint32_t base = 0; base < len; base += dist) {
          const uint32_t step = len - base < dist ? len - base : dist;
          for (uint32_t k = lane; k < step; k += W) dst[base + k] = src[base + k];
          if (base + step < len) L.sync();
        }
        o += len;
      }
    } else {
      return kErrBlockType;
    }
    if (final) break;
  }
  return o == outlen ? kOk : kErrShort;
}

// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320) with a 256-entry table.
// The lanes each take one segment of the block and run the table CRC from 0;
// the segments are joined with the CRC's linearity: crc(A || B) = crc(A) * x^(8|B|)
// + crc(B) over GF(2) modulo the polynomial, and the standard pre- and post-
// inversion is applied to the whole: crc = raw(data) + 0xffffffff * x^(8n) +
// 0xffffffff.  In the reflected representation bit 31 holds x^0.
constexpr uint32_t kCrcPoly = 0xEDB88320u;

RBG_IHD void crc32_table(uint32_t *t) {
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t c = i;
    for (int k = 0; k < 8; ++k) c = (c & 1) ? kCrcPoly ^ (c >> 1) : c >> 1;
    t[i] = c;
  }
}
RBG_IHD uint32_t crc_raw(const uint32_t *t, uint32_t c, const uint8_t *p, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i) c = t[(c ^ p[i]) & 0xff] ^ (c >> 8);
  return c;
}
// a * b modulo the polynomial (shift-and-add; b is multiplied by x each step)
RBG_IHD uint32_t gf2_mul(uint32_t a, uint32_t b) {
  uint32_t r = 0;
  for (uint32_t m = 1u << 31; m; m >>= 1) {
    if (a & m) r ^= b;
    b = (b & 1) ? (b >> 1) ^ kCrcPoly : b >> 1;
  }
  return r;
}
// x^(8 n) modulo the polynomial, by squaring
RBG_IHD uint32_t x_pow8(uint32_t n) {
  uint32_t r = 1u << 31, sq = 1u << (31 - 8);      // x^0, x^8
  while (n) {
    if (n & 1) r = gf2_mul(r, sq);
    sq = gf2_mul(sq, sq);
    n >>= 1;
  }
  return r;
}
template <class Lanes>
RBG_IHD uint32_t crc32(const uint32_t *t, const uint8_t *p, uint32_t n, const Lanes &L) {
  const uint32_t W = (uint32_t)L.width();
  const uint32_t seg = (n + W - 1) / W;
  uint32_t acc = 0;
#ifdef __CUDA_ARCH__
  if (W > 1) {
    const uint32_t a = (uint32_t)L.lane() * seg;
    const uint32_t e = a + seg < n ? a + seg : n;
    const uint32_t c = a < n ? crc_raw(t, 0u, p + a, e - a) : 0u;
    const uint32_t xs = x_pow8(seg);
    // Horner over the lanes: acc = acc * x^(8 len_i) + c_i
    for (uint32_t i = 0; i < W; ++i) {
      const uint32_t ci = __shfl_sync(0xffffffffu, c, (int)i);
      const uint32_t ai = i * seg;
      const uint32_t li = ai >= n ? 0u : (ai + seg < n ? seg : n - ai);
      if (li == seg) acc = gf2_mul(acc, xs) ^ ci;
      else if (li) acc = gf2_mul(acc, x_pow8(li)) ^ ci;
    }
  } else
#endif
  {
    // one lane: the same joining, over W = 32 virtual segments
    const uint32_t vs = (n + 31) / 32;
    const uint32_t xs = x_pow8(vs);
    for (uint32_t a = 0; a < n; a += vs) {
      const uint32_t li = a + vs < n ? vs : n - a;
      const uint32_t ci = crc_raw(t, 0u, p + a, li);
      acc = gf2_mul(acc, li == vs ? xs : x_pow8(li)) ^ ci;
    }
  }
  return acc ^ gf2_mul(0xffffffffu, x_pow8(n)) ^ 0xffffffffu;
}

}  // namespace inflate
}  // namespace rbg
