// Test harness: runs the library's DEFLATE decoder over a file of damaged
// streams (records of u32 input length, u32 output length, input bytes), built
// with AddressSanitizer by tests/test_inflate_cpu.py so that any read or write
// out of bounds ends the process with an error.  Not part of the library.
#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

#include "../../rabbitbin_b200/csrc/inflate.cuh"

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  std::unique_ptr<rbg::inflate::Tables> t(new rbg::inflate::Tables());
  long runs = 0, ok = 0;
  for (;;) {
    uint32_t hdr[2];
    if (std::fread(hdr, 4, 2, f) != 2) break;
    std::vector<uint8_t> in(hdr[0]);
    if (hdr[0] && std::fread(in.data(), 1, hdr[0], f) != hdr[0]) return 3;
    // exact-size heap buffers, so that the sanitizer sees any overrun
    uint8_t *ib = new uint8_t[hdr[0] ? hdr[0] : 1];
    for (uint32_t i = 0; i < hdr[0]; ++i) ib[i] = in[i];
    uint8_t *ob = new uint8_t[hdr[1] ? hdr[1] : 1];
    ok += rbg::inflate::inflate_block(ib, hdr[0], ob, hdr[1], *t, rbg::inflate::SerialLanes{}) == 0;
    delete[] ib;
    delete[] ob;
    ++runs;
  }
  std::fclose(f);
  std::printf("%ld %ld\n", runs, ok);
  return 0;
}
