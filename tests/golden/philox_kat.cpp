// philox_kat.cpp -- prints Philox4x32-10 blocks from PyTorch's open-source
// engine (ATen/core/PhiloxRNGEngine.h), an implementation independent of
// this repository's, for the known-answer fixture philox_kat.json.
// Built and run by make_golden.py; reads "k0 k1 c0 c1 c2 c3" lines on stdin.
#include <ATen/core/PhiloxRNGEngine.h>
#include <cstdio>

int main() {
  unsigned k0, k1, c0, c1, c2, c3;
  while (scanf("%x %x %x %x %x %x", &k0, &k1, &c0, &c1, &c2, &c3) == 6) {
    uint64_t seed = ((uint64_t)k1 << 32) | k0;
    uint64_t subseq = ((uint64_t)c3 << 32) | c2;
    uint64_t offset = ((uint64_t)c1 << 32) | c0;
    at::Philox4_32 eng(seed, subseq, offset);
    unsigned o0 = eng(), o1 = eng(), o2 = eng(), o3 = eng();
    printf("%08x %08x %08x %08x\n", o0, o1, o2, o3);
  }
  return 0;
}
