/* Exhaustive check of the single-precision division by 12 used by the
 * reference-arithmetic kernels (coffee_b200/csrc/ez_refarith.cuh,
 * xa::div12_fast): q = t * (1/12), e = fma(-q, 12, t), q' = fma(e, 1/12, q)
 * with the sign of t.  For every finite float t it compares q' with the
 * IEEE quotient t / 12, bit for bit, and counts the mismatches inside and
 * outside the range 0 < |t| < 2^-124 that the kernels send to the IEEE
 * division.  Prints "outside <n> inside <m>"; the claim holds when the
 * first count is 0.  Built with -ffp-contract=off so that every operation
 * is the one written. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

int main(void) {
  const float r12 = 1.0f / 12.0f;
  unsigned long long outside = 0, inside = 0;
#pragma omp parallel for reduction(+ : outside, inside) schedule(static)
  for (long long u = 0; u < (1LL << 32); ++u) {
    const uint32_t b = (uint32_t)u;
    float t;
    memcpy(&t, &b, 4);
    if (!isfinite(t)) continue;
    const float ref = t / 12.0f;
    float q = t * r12;
    const float e = fmaf(-q, 12.0f, t);
    q = copysignf(fmaf(e, r12, q), t);
    uint32_t a1, a2;
    memcpy(&a1, &ref, 4);
    memcpy(&a2, &q, 4);
    if (a1 != a2) {
      if (fabsf(t) < 0x1p-124f && t != 0.0f) ++inside;
      else ++outside;
    }
  }
  printf("outside %llu inside %llu\n", outside, inside);
  return 0;
}
