/* The exact division by six of the pressure stencils (plume_b200/csrc/poisson.cuh, div6), restated with the same
 * float operations, checked against IEEE x / 6: every significand at several exponents of both signs, every
 * float within a factor of 4 of the 2^-120 guard, subnormals, zeros, infinities and NaN. Prints the number of
 * mismatches (bit patterns that differ) and the number of values checked. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static float div6(float x) {
  if (fabsf(x) >= 0x1p-120f && fabsf(x) <= 0x1p+127f) {
    const float z = 0x1.555556p-3f;
    const float q0 = x * z;
    return fmaf(fmaf(-q0, 6.0f, x), z, q0);
  }
  return x / 6.0f;
}

static uint64_t bad = 0, checked = 0;

static void check(uint32_t bits) {
  float x, want, got;
  memcpy(&x, &bits, 4);
  volatile float six = 6.0f;
  want = x / six;
  got = div6(x);
  uint32_t a, b;
  memcpy(&a, &want, 4);
  memcpy(&b, &got, 4);
  if (a != b && !(isnan(want) && isnan(got))) bad++;
  checked++;
}

int main(void) {
  const int exponents[] = {1, 7, 60, 127, 180, 250, 253, 254};  /* biased exponents */
  for (uint32_t sign = 0; sign < 2; ++sign) {
    for (size_t e = 0; e < sizeof exponents / sizeof exponents[0]; ++e)
      for (uint32_t m = 0; m < (1u << 23); ++m) check(sign << 31 | (uint32_t)exponents[e] << 23 | m);
    for (uint32_t bits = 0; bits < (1u << 23); ++bits) check(sign << 31 | bits);  /* zero and subnormals */
    for (uint32_t bits = 5u << 23; bits < 9u << 23; ++bits) check(sign << 31 | bits);  /* 2^-122 .. 2^-118 */
    check(sign << 31 | 0x7f800000u);  /* infinity */
    check(sign << 31 | 0x7fc00000u);  /* NaN */
  }
  printf("%llu %llu\n", (unsigned long long)bad, (unsigned long long)checked);
  return 0;
}
