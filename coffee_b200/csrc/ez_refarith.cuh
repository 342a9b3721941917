// The reference CPU build's arithmetic, operation for operation.
//
// The reference's CPU build (src/algorithms/field_solver_EZ.cpp with the
// vectorclass library) is compiled by g++ -O3 for x86-64-v4, whose default
// floating-point contraction fuses a product into the add or subtract that
// consumes it.  The functions here make every one of those fused
// multiply-adds an explicit single-rounding FMA and every other operation a
// single correctly rounded IEEE operation (the __f*_rn / __d*_rn intrinsics,
// which the CUDA compiler never contracts or reassociates), in the
// reference's order.  With them the FP32 stage and KO kernels of the CPU
// semantics compute the float build's results bit for bit.
//
// Which products the reference build fuses follows one rule, read from the
// compiler's own record of its FMA formation pass on field_solver_EZ.cpp:
// in a left-to-right sum a*b + c*d + e*f the first product is rounded and
// each later one is fused into the running sum; a product subtracted from a
// rounded value is a fused negative multiply-add.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ez_common.cuh"

namespace coffee {
namespace xa {

__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }

// t / 12, correctly rounded.  FP32: q = t (1/12), then one Newton
// correction with the exact residual e = 12 q - t (an FMA): q - e/12 as
// fma(e, -1/12, q), which also keeps the sign of a zero t.  An exhaustive
// check over every finite float (on the CPU, with the same IEEE operations)
// shows that this is the IEEE quotient for every t except
// 0 < |t| < 2^-124, whose quotient is subnormal.  Those are found by an
// integer key, 2 bits(t) - 1 (mod 2^32): it drops the sign, sends zero to
// the largest value, and is below kTinyKey exactly for that range (the same
// check covers all 2^32 patterns).  The caller keeps the running minimum of
// the keys in `kmin` and recomputes with div12_exact when it is below
// kTinyKey.
constexpr uint32_t kTinyKey = 0x02FFFFFEu;
__device__ __forceinline__ float div12_fast(float t, uint32_t& kmin) {
  constexpr float r12 = 1.0f / 12.0f;
  const float q = __fmul_rn(t, r12);
  const float e = __fmaf_rn(q, 12.0f, -t);
  const uint32_t b = __float_as_uint(t);
  kmin = min(kmin, b + b - 1u);
  return __fmaf_rn(e, -r12, q);
}
__device__ __forceinline__ double div12_fast(double t, uint32_t&) { return __ddiv_rn(t, 12.0); }
__device__ __forceinline__ float div12_exact(float t) {
  uint32_t k = 0xFFFFFFFFu;
  const float q = div12_fast(t, k);
  return k < kTinyKey ? __fdiv_rn(t, 12.0f) : q;
}
__device__ __forceinline__ double div12_exact(double t) { return __ddiv_rn(t, 12.0); }

// diff1_4 of the reference (finite_diff_simd.h:15-25) before its inv_delta
// factor: (((f-2 - 8 f-1) + 8 f+1) - f+2) / 12, the two products by 8 fused
// (they are exact, so fused or not gives the same value).  EXACT = false
// folds into `kmin` the key of the quotient's input (div12_fast).
template <bool EXACT, typename T>
__device__ __forceinline__ T dq(T m2, T m1, T p1, T p2, uint32_t& kmin) {
  T t = fma(m1, (T)-8, m2);
  t = fma(p1, (T)8, t);
  t = sub(t, p2);
  if constexpr (EXACT) return div12_exact(t);
  else return div12_fast(t, kmin);
}

// diff6_2 of the reference (finite_diff_simd.h:41-58): each weighted term
// fused into the running sum, f+3 added last.
template <typename T>
__device__ __forceinline__ T d6(T m3, T m2, T m1, T c, T p1, T p2, T p3) {
  T t = fma(m2, (T)-6, m3);
  t = fma(m1, (T)15, t);
  t = fma(c, (T)-20, t);
  t = fma(p1, (T)15, t);
  t = fma(p2, (T)-6, t);
  return add(p3, t);
}

// ax*bx + ay*by + az*bz in the reference's rounding: the first product
// rounded, the other two fused
template <typename T>
__device__ __forceinline__ T dot3(T ax, T bx, T ay, T by, T az, T bz) {
  return fma(az, bz, fma(ay, by, mul(ax, bx)));
}

// vectorclass max(B2, TINY) (x86 maxps: TINY unless B2 is greater)
template <typename T>
__device__ __forceinline__ T floor_tiny(T b2) {
  return b2 > Tiny<T>::v ? b2 : Tiny<T>::v;
}

// ---- tanh of the reference's vector library, single precision ----------
// Agner Fog's vectorclass 1.40 (vendored in the reference at
// deps/vectorclass): tanh_f (vectormath_hyp.h:302-340) and the exp_f it
// calls for |x| > 5/8 (vectormath_exp.h:377-460, BA = 0, M1 = 0), restated
// per lane from the published source: a degree-4 polynomial in x^2 for
// |x| <= 5/8, else 1 - 2 / (exp(2|x|) + 1), with exp(y) = 2^r (1 + y' +
// y'^2 P5(y')), r = round(y log2 e), y' = y - r ln2 in two parts; 1 for
// |x| > 44.4; the sign of x.  mul_add / nmul_add of the library are FMAs,
// and so is the x^8 term of the polynomial, which the reference build's
// compiler contracts.
__device__ __forceinline__ float vcl_expf(float x0) {
  const float r = rintf(__fmul_rn(x0, 1.44269502162933349609375f));  // round(x log2 e)
  float x = __fmaf_rn(-r, 0.693359375f, x0);                         // x -= r ln2_hi
  x = __fmaf_rn(-r, -2.12194440e-4f, x);                             // x -= r ln2_lo
  const float x2 = __fmul_rn(x, x), x4 = __fmul_rn(x2, x2);
  // polynomial_5(x, 1/2, 1/6, 1/24, 1/120, 1/720, 1/5040), then x + x^2 z
  float z = __fmaf_rn(__fmaf_rn(1.f / 5040.f, x, 1.f / 720.f), x4,
                      __fmaf_rn(1.f / 6.f, x, 1.f / 2.f));
  z = __fmaf_rn(__fmaf_rn(1.f / 120.f, x, 1.f / 24.f), x2, z);
  z = __fmaf_rn(z, x2, x);
  // vm_pow2n: 2^r from the bits of r + (127 + 2^23) moved into the exponent
  const float n2 = __int_as_float(__float_as_int(__fadd_rn(r, 8388735.0f)) << 23);
  z = __fmul_rn(__fadd_rn(z, 1.0f), n2);
  if (!(fabsf(x0) < 87.3f))
    z = isnan(x0) ? x0 : (signbit(x0) ? 0.0f : __int_as_float(0x7f800000));
  return z;
}

__device__ __forceinline__ float vcl_tanhf(float x0) {
  const float x = fabsf(x0);
  float y;
  if (x <= 0.625f) {
    const float x2 = __fmul_rn(x, x), x4 = __fmul_rn(x2, x2), x8 = __fmul_rn(x4, x4);
    float p = __fmaf_rn(x8, -5.70498872745E-3f,
                        __fmaf_rn(1.33314422036E-1f, x2, -3.33332819422E-1f));
    p = __fmaf_rn(__fmaf_rn(2.06390887954E-2f, x2, -5.37397155531E-2f), x4, p);
    y = __fmaf_rn(p, __fmul_rn(x, x2), x);
  } else {
    const float e = vcl_expf(__fadd_rn(x, x));
    y = __fsub_rn(1.0f, __fdiv_rn(2.0f, __fadd_rn(e, 1.0f)));
  }
  if (x > 44.4f) y = 1.0f;
  return copysignf(y, x0);
}

// The P-gradient taper of the CPU build's rk_step (field_solver_EZ.cpp:
// 222-230), s = (1 - tanh((r - 3) / 0.5)) / 2, the division by 0.5 being a
// multiplication by 2 (exact).  FP64: CUDA's tanh (the reference's double
// build uses its library's double tanh; the two agree to rounding).
__device__ __forceinline__ float taper_of_r(float r) {
  return __fmul_rn(__fsub_rn(1.0f, vcl_tanhf(__fmul_rn(__fadd_rn(r, -3.0f), 2.0f))), 0.5f);
}
__device__ __forceinline__ double taper_of_r(double r) {
  return __dmul_rn(__dsub_rn(1.0, ::tanh(__dmul_rn(__dadd_rn(r, -3.0), 2.0))), 0.5);
}

// Grid::pos(axis, n, 1) = lower + delta (n - guard + 0) as the reference
// build computes it (one FMA), shifted by `lane` points (another FMA): the
// taper's coordinates, each offset by the SIMD lane of point i.
template <typename T>
__device__ __forceinline__ T lane_pos(T delta, T lower, int n_minus_guard, T lane) {
  return fma(delta, lane, fma(delta, (T)n_minus_guard, lower));
}

}  // namespace xa
}  // namespace coffee
