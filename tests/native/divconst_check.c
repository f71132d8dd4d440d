/* Exhaustive check of the division by a constant used in the CUDA smoothstep:
 * for each divisor c given on the command line (as a float in hex, e.g.
 * 0x1.1eb852p-1), with r = RN(1/c), q0 = RN(x * r), e = fma(-q0, c, x) and
 * q = fma(e, r, q0), checks q == RN(x / c) for every float x with
 * 2^-100 <= |x| <= 2^100 (the sequence is odd in x, so positive x suffice).
 * Prints one line per divisor: "<c> <mismatches> <first bad x or 0>".
 * Build: gcc -O2 -mfma -fopenmp -ffp-contract=off divconst_check.c -o divconst_check -lm */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static float from_bits(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}
static uint32_t to_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

int main(int argc, char** argv) {
  const uint32_t lo = to_bits(0x1p-100f), hi = to_bits(0x1p100f);
  for (int a = 1; a < argc; ++a) {
    const float c = strtof(argv[a], NULL);
    const volatile float one = 1.0f;
    const float r = one / c;
    long long bad = 0;
    uint32_t first = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
    for (long long u = lo; u <= (long long)hi; ++u) {
      const float x = from_bits((uint32_t)u);
      const float q0 = x * r;
      const float q = fmaf(fmaf(-q0, c, x), r, q0);
      const float want = x / c;
      if (to_bits(q) != to_bits(want)) {
        ++bad;
#pragma omp critical
        if (!first || (uint32_t)u < first) first = (uint32_t)u;
      }
    }
    printf("%a %lld %a\n", c, bad, first ? from_bits(first) : 0.0f);
  }
  return 0;
}
