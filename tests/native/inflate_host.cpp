// Test harness: the library's DEFLATE decoder (rabbitbin_b200/csrc/inflate.cuh,
// the code the device kernel runs) compiled for the host, so the CPU test suite
// can compare it with zlib.  Not part of the library.
#include <cstdint>
#include <memory>

#include "../../rabbitbin_b200/csrc/inflate.cuh"

extern "C" int host_inflate(const uint8_t *in, uint32_t inlen, uint8_t *out, uint32_t outlen) {
  std::unique_ptr<rbg::inflate::Tables> t(new rbg::inflate::Tables());
  return rbg::inflate::inflate_block(in, inlen, out, outlen, *t, rbg::inflate::SerialLanes{});
}

extern "C" uint32_t host_crc32(const uint8_t *p, uint32_t n) {
  uint32_t t[256];
  rbg::inflate::crc32_table(t);
  return rbg::inflate::crc32(t, p, n, rbg::inflate::SerialLanes{});
}
