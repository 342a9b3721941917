/* ffe_oracle.c -- instantiates the oracle restatement (ffe_oracle_impl.h) in
 * float and double.  Test infrastructure only; see ffe_oracle.h. */
#define _GNU_SOURCE
#include "ffe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#include <stdint.h>

/* Single-precision tanh of the reference's vector library (Agner Fog's
 * vectorclass 1.40, vendored at deps/vectorclass): tanh_f,
 * vectormath_hyp.h:302-340, and the exp_f it calls for |x| > 5/8,
 * vectormath_exp.h:377-460 (BA = 0, M1 = 0), restated lane by lane from the
 * published source: a degree-4 polynomial in x^2 for |x| <= 5/8, else
 * 1 - 2 / (exp(2|x|) + 1) with exp(y) = 2^r (1 + y' + y'^2 P(y')),
 * r = round(y log2 e), y' = y - r ln2 in two parts; 1 for |x| > 44.4; the sign
 * of x.  The multiply-adds are single-rounding fmaf where the library calls
 * mul_add / nmul_add, and where the reference build's compiler (g++ -O3,
 * x86-64-v4, default -ffp-contract=fast) contracts the polynomial's x^8 term
 * (polynomial_4's last product-plus-sum). */
static float vcl_expf(float x0) {
  const float r = rintf(x0 * 1.44269502162933349609375f); /* round(x * VM_LOG2E) */
  float x = fmaf(-r, 0.693359375f, x0);                   /* x -= r * ln2f_hi */
  x = fmaf(-r, -2.12194440e-4f, x);                       /* x -= r * ln2f_lo */
  const float x2 = x * x, x4 = x2 * x2;
  /* polynomial_5(x, 1/2, 1/6, 1/24, 1/120, 1/720, 1/5040), then x + x^2 z */
  float z = fmaf(fmaf(1.f / 5040.f, x, 1.f / 720.f), x4, fmaf(1.f / 6.f, x, 1.f / 2.f));
  z = fmaf(fmaf(1.f / 120.f, x, 1.f / 24.f), x2, z);
  z = fmaf(z, x2, x);
  /* vm_pow2n: 2^r from the bits of r + (127 + 2^23) moved into the exponent */
  float t = r + 8388735.0f;
  uint32_t b;
  memcpy(&b, &t, 4);
  b <<= 23;
  float n2;
  memcpy(&n2, &b, 4);
  z = (z + 1.0f) * n2;
  if (!(fabsf(x0) < 87.3f)) z = isnan(x0) ? x0 : (signbit(x0) ? 0.0f : INFINITY);
  return z;
}

static float vcl_tanhf(float x0) {
  const float x = fabsf(x0);
  float y;
  if (x <= 0.625f) {
    const float x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
    /* polynomial_4(x2, r0..r4), then y = x + (x2 x) y */
    float p = fmaf(x8, -5.70498872745E-3f, fmaf(1.33314422036E-1f, x2, -3.33332819422E-1f));
    p = fmaf(fmaf(2.06390887954E-2f, x2, -5.37397155531E-2f), x4, p);
    y = fmaf(p, x * x2, x);
  } else {
    const float e = vcl_expf(x + x);
    y = 1.0f - 2.0f / (e + 1.0f);
  }
  if (x > 44.4f) y = 1.0f;
  return copysignf(y, x0); /* sign_combine(y, x0), y >= 0 */
}

/* TINY of the reference (src/data/typedefs.h:6-12) */
#define REAL float
#define SFX _f32
#define TINYR ((float)(1e-7))
#define TANHR tanhf
#define TANHX vcl_tanhf
#define FMAR fmaf
#define SQRTR sqrtf
#include "ffe_oracle_impl.h"
#undef REAL
#undef SFX
#undef TINYR
#undef TANHR
#undef TANHX
#undef FMAR
#undef SQRTR

/* The double build's taper calls the library's double tanh (tanh_d), which
 * agrees with libm's to rounding: the FP64 restatement is the double build
 * to rounding where the taper acts, bit for bit elsewhere. */
#define REAL double
#define SFX _f64
#define TINYR 1e-11
#define TANHR tanh
#define TANHX tanh
#define FMAR fma
#define SQRTR sqrt
#include "ffe_oracle_impl.h"
#undef REAL
#undef SFX
#undef TINYR
#undef TANHR
#undef TANHX
#undef FMAR
#undef SQRTR
