/* Exhaustive check of the single-precision division by 12 used by the
 * reference-arithmetic kernels (coffee_b200/csrc/ez_refarith.cuh,
 * xa::div12_fast): q = t * (1/12), e = fma(q, 12, -t) (the exact residual
 * 12 q - t), q' = fma(e, -1/12, q).  For every finite float t it compares
 * q' with the IEEE quotient t / 12, bit for bit, and counts the mismatches
 * inside and outside the range 0 < |t| < 2^-124 that the kernels send to
 * the IEEE division.  It also checks the kernels' integer test of that
 * range, key(t) = 2 bits(t) - 1 (mod 2^32) < 0x02FFFFFE, against the
 * floating-point one for every bit pattern.  Prints
 * "outside <n> inside <m> key <k>"; the claims hold when n and k are 0.
 * Built with -ffp-contract=off so that every operation is the one
 * written. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

int main(void) {
  const float r12 = 1.0f / 12.0f;
  unsigned long long outside = 0, inside = 0, key = 0;
#pragma omp parallel for reduction(+ : outside, inside, key) schedule(static)
  for (long long u = 0; u < (1LL << 32); ++u) {
    const uint32_t b = (uint32_t)u;
    float t;
    memcpy(&t, &b, 4);
    const int in_range = fabsf(t) < 0x1p-124f && t != 0.0f;
    const int key_says = (uint32_t)(b + b - 1u) < 0x02FFFFFEu;
    if (in_range != key_says) ++key;
    if (!isfinite(t)) continue;
    const float ref = t / 12.0f;
    float q = t * r12;
    const float e = fmaf(q, 12.0f, -t);
    q = fmaf(e, -r12, q);
    uint32_t a1, a2;
    memcpy(&a1, &ref, 4);
    memcpy(&a2, &q, 4);
    if (a1 != a2) {
      if (in_range) ++inside;
      else ++outside;
    }
  }
  printf("outside %llu inside %llu key %llu\n", outside, inside, key);
  return 0;
}
