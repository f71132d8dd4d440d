/* Check of a division by a shared reciprocal: for floats x and y (y normal),
 * q = RN32(RN64(x * r)) with r = RN64(1/y), or r one f64 ulp away from it on
 * either side (a reciprocal refined to within one ulp), against the IEEE
 * quotient RN32(x / y).
 * Where the exact quotient has magnitude at least 2^-126 they must agree: the
 * f64 product's relative error is below 2^-51, while a quotient of two floats in
 * the normal range is never a midpoint of two floats and lies at least 2^-48
 * (relative) from one. Below 2^-126 an exact quotient can sit on a midpoint of
 * the subnormal grid (x / y = 2^-150, or (2^24 - 1) * 2^-150 rounding up to
 * 2^-126), where the product's error can decide the rounding: a division by a
 * shared reciprocal must take the IEEE division there (|x| < 2^-126 |y|).
 * Cases: zeros, subnormal and normal x against powers of two and other y,
 * pairs with few significant bits, and `n` seeded random pairs over all finite
 * floats (x) and normal floats (y), both signs.
 * Prints "<checked> <mismatches> <mismatches with |x / y| >= 2^-126> <a bad x> <its y>";
 * the third number must be 0.
 * Build: gcc -O2 -fopenmp -ffp-contract=off recip_division_check.c -o recip_division_check -lm */
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

/* 0 when every variant of the reciprocal gives the IEEE quotient. */
static int check(float x, float y) {
  const float want = x / y;
  const volatile double one = 1.0;
  const double r = one / (double)y;
  const double rs[3] = {r, nextafter(r, 0.0), nextafter(r, r > 0 ? INFINITY : -INFINITY)};
  for (int k = 0; k < 3; ++k) {
    const float q = (float)((double)x * rs[k]);
    if (isnan(want) ? !isnan(q) : to_bits(q) != to_bits(want)) return 1;
  }
  return 0;
}

static uint64_t mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int main(int argc, char** argv) {
  const long long n = argc > 1 ? atoll(argv[1]) : (1ll << 24);
  long long bad = 0, checked = 0, bad_normal = 0;
  float bx = 0.0f, by = 0.0f;
  /* structured: x from a spread of exponents and significands, y from powers of
     two and small-significand values, both signs */
  static const float ys[] = {1.0f, 2.0f, 0.5f, 3.0f, 6.0f, 7.0f, 10.0f, 0.0001f, 1.0e-30f, 1.0e30f, 1.5f, 1.25f, 1.75f, 9.0f, 11.0f,
                             0x1.fffffep-1f, 0x1.000002p0f, 0x1p-126f, 0x1.fffffep127f, 3.4e38f, 1.17549435e-38f, 12345.0f, 0.1f, 0.3f};
  const int nys = (int)(sizeof ys / sizeof ys[0]);
#pragma omp parallel for reduction(+ : bad, checked, bad_normal) schedule(dynamic, 64)
  for (long long e = 0; e < 256 * 64; ++e) {
    const uint32_t expo = (uint32_t)(e / 64), sig = (uint32_t)mix((uint64_t)e) & 0x7FFFFFu;
    const uint32_t sigs[4] = {sig, 0u, sig & 0x7FF000u, 0x7FFFFFu};
    for (int s = 0; s < 4; ++s) {
      const float x = from_bits((expo << 23) | sigs[s]);
      if (!isfinite(x)) continue;
      for (int k = 0; k < nys; ++k)
        for (int sg = 0; sg < 4; ++sg) {
          const float xs = (sg & 1) ? -x : x, yv = (sg & 2) ? -ys[k] : ys[k];
          ++checked;
          if (check(xs, yv)) {
            ++bad;
            if (fabs((double)xs / (double)yv) >= 0x1p-126) ++bad_normal;
#pragma omp critical
            {
              bx = xs;
              by = yv;
            }
          }
        }
    }
  }
  /* random pairs */
#pragma omp parallel for reduction(+ : bad, checked, bad_normal) schedule(static)
  for (long long i = 0; i < n; ++i) {
    const uint64_t h = mix((uint64_t)i * 2 + 1);
    float x = from_bits((uint32_t)h);
    float y = from_bits((uint32_t)(h >> 32));
    if (!isfinite(x)) x = from_bits((uint32_t)h & 0x807FFFFFu);          /* exponent 0: subnormal or zero */
    if (!isnormal(y)) y = from_bits(((uint32_t)(h >> 32) & 0x807FFFFFu) | 0x3F800000u);
    ++checked;
    if (check(x, y)) {
      ++bad;
      if (fabs((double)x / (double)y) >= 0x1p-126) ++bad_normal;
#pragma omp critical
      {
        bx = x;
        by = y;
      }
    }
  }
  printf("%lld %lld %lld %a %a\n", checked, bad, bad_normal, bx, by);
  return 0;
}
