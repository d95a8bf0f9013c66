/* Hashes the reference's correctly rounded sinf / cosf / tanf (oracle/_ref/librsprobe.so) over chunks of 2^24
 * consecutive input bit patterns: hash = wrapping sum of mix64((x << 32) | f(x)), NaN results canonical (0x7FC00000).
 * usage: oracle_libm_hash <probe.so> <fn 0|1|2> <first_chunk> <nchunks>  -> one line per chunk: "<chunk> <hash hex>" */
#include <dlfcn.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
static uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
int main(int argc, char** argv) {
  if (argc < 5) return 2;
  void* L = dlopen(argv[1], RTLD_NOW);
  if (!L) { fprintf(stderr, "%s\n", dlerror()); return 1; }
  const char* names[3] = {"rsref_sinf", "rsref_cosf", "rsref_tanf"};
  int fn = atoi(argv[2]);
  float (*f)(float) = (float (*)(float))dlsym(L, names[fn]);
  unsigned first = (unsigned)atoi(argv[3]), nch = (unsigned)atoi(argv[4]);
  for (unsigned c = first; c < first + nch; ++c) {
    uint64_t h = 0;
    for (uint32_t i = 0; i < (1u << 24); ++i) {
      uint32_t xb = (c << 24) | i, yb;
      float x, y;
      memcpy(&x, &xb, 4);
      y = f(x);
      memcpy(&yb, &y, 4);
      if ((yb & 0x7FFFFFFFu) > 0x7F800000u) yb = 0x7FC00000u;
      h += mix64(((uint64_t)xb << 32) | yb);
    }
    printf("%u %016llx\n", c, (unsigned long long)h);
    fflush(stdout);
  }
  return 0;
}
