// Shared device-side definitions of the flat-Cartesian EZ kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace coffee {

// TINY of the reference (src/data/typedefs.h:6-12)
template <typename T> struct Tiny;
template <> struct Tiny<float> { static constexpr float v = 1e-7f; };
template <> struct Tiny<double> { static constexpr double v = 1e-11; };

enum Semantics { SEM_CPU_REF = 0, SEM_GPU_REF = 1 };

// Grid geometry of one rank, in points (guards included).
struct GridGeom {
  int dims[3];
  int guard[3];
  int N[3];        // interior points per axis
  int lo[3], hi[3];// update box [lo, hi): guard - shift_ghost .. dims - guard + shift_ghost
  int periodic[3];
  long long sy, sz;// strides of j and k
};

// Everything a flat EZ kernel needs besides pointers, in field precision.
// Passed by value as a kernel parameter (no __constant__ state, so several
// solvers can run side by side).
template <typename T>
struct EzConst {
  GridGeom g;
  T delta[3], inv_delta[3], lower[3];
  T dt, ch2, tau, inv_tau;
  T ko_c;           // -KOeps * KO_const, KO_const = -1/64
  T gam_dt;         // damp_gamma / dt
  int use_edotb, divB_clean, clean_ep, check_egb;
  int semantics;
  int taper_lanes;  // CPU-build SIMD width for the P-gradient taper
  int problem;      // 0 periodic box, 1 pulsar, 2 Alfven wave from pulsar
  int absorbing;    // absorbing layer present
  T pml_lo[3], pml_hi[3], pml_scale[3], sigpml;
  T radius, omega, b0;
  T p1, p2, p3, q11, q12, q13, q22, q23, qox, qoy, qoz;
  T tp_start, tp_end, rpert1, rpert2, dw0, nT, ph1, ph2, dph, theta0, drpert;
  T tp_start1, tp_end1, rpert11, rpert21, dw1, nT1, ph11, ph21, dph1;
  int pert_type;
};

template <typename T> struct F7 { T* p[7]; };
// Seven values of one point, passed by value to the out-of-line boundary
// functions so that the caller's registers never need an address.
template <typename T> struct V7 { T v[7]; };
template <typename T> struct F5 { T* p[5]; };
// The CPU build's energy-change arrays (sim_data.h:15-16), in this order:
// dU_EgtB, dU_Epar, dU_KO, dU_EgtB_cum, dU_Epar_cum, dU_KO_cum.
template <typename T> struct F6 { T* p[6]; };

// ---- cp.async helpers (sm_80+ asynchronous global->shared copies) --------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void* src) {
  static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async size");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(src),
               "n"(BYTES));
}
// the same with a compile-time offset OFF added to the shared address
template <int BYTES, int OFF>
__device__ __forceinline__ void cp_async_off(uint32_t dst, const void* src) {
  static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async size");
  static_assert(OFF >= 0, "offsets are measured from the slot base");
  asm volatile("cp.async.ca.shared.global [%0+%3], [%1], %2;\n" ::"r"(dst), "l"(src),
               "n"(BYTES), "n"(OFF));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---- shared-memory loads at a 32-bit address plus a compile-time offset --
// (one instruction per operand: no address arithmetic in the stencil loop)
template <typename T, int OFF>
__device__ __forceinline__ T lds(uint32_t a) {
  static_assert(OFF >= 0, "offsets are measured from the tile corner");
  T v;
  if constexpr (sizeof(T) == 4)
    asm volatile("ld.shared.f32 %0, [%1+%2];\n" : "=f"(v) : "r"(a), "n"(OFF));
  else
    asm volatile("ld.shared.f64 %0, [%1+%2];\n" : "=d"(v) : "r"(a), "n"(OFF));
  return v;
}

// static_for<N>(fn) calls fn(std::integral_constant<int, 0..N-1>) in order,
// so the index can feed template arguments (compile-time offsets).
template <int I, int N>
struct StaticFor {
  template <class Fn>
  __device__ __forceinline__ static void run(Fn& fn) {
    fn(std::integral_constant<int, I>{});
    StaticFor<I + 1, N>::run(fn);
  }
};
template <int N>
struct StaticFor<N, N> {
  template <class Fn>
  __device__ __forceinline__ static void run(Fn&) {}
};
template <int N, class Fn>
__device__ __forceinline__ void static_for(Fn&& fn) {
  StaticFor<0, N>::run(fn);
}

// ---- field-precision arithmetic helpers ---------------------------------
// FP32: hardware reciprocal-based division (max 2 ulp for the operand
// ranges here: divisors are floored at TINY); FP64: IEEE division.
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }

}  // namespace coffee
