// Device code of the staggered (Yee) RK3 solver in Cartesian Kerr-Schild
// coordinates, the reference's field_solver_gr
// (src/algorithms/field_solver_gr.cu).  sim_data's E holds the densitised
// D; the curl acts on E = alpha D_i + sqrt(gamma) (beta x B)_i at the E
// positions and H = alpha B_i - sqrt(gamma) (beta x D)_i at the B positions.
//
// A substep is: gyee_eh_kernel (E, H and the lowered B over [1, dims - 1),
// the reference's compute_E_gr / compute_H_gr), gyee_rho_kernel (the
// sqrt(gamma)-weighted div D), gyee_update_kernel (push and RK update in one
// pass), [gyee_clean_kernel], gyee_clamp_kernel (the |E| <= |B| rescale and,
// in the last substep, the absorbing layers, storing D and B).  One point per
// thread: the metric is evaluated analytically at each staggered position
// (Cks), and the stencil loads go through the read-only cache.
#pragma once

#include "gr_kernels.cuh"
#include "yee_kernels.cuh"

// Resident CTAs of 256 threads per SM for the metric-heavy E, H and
// cleaning passes, FP32: 3 (at most 85 registers) instead of the 2 that 86
// registers allow.  Measured on the Wald field 256^3: the step 10.2 -> 9.1 ms,
// bitwise the same fields; the rescale pass is faster without the cap.
#ifndef COFFEE_GYEE_MIN_BLOCKS
#define COFFEE_GYEE_MIN_BLOCKS 3
#endif

namespace coffee {

template <typename T>
struct GYeeArgs {
  YeeArgs<T> y;              // geometry, state (D in E), D*, B', Dn, Bn, outer layer
  T spin;
  int calc_current, clean_ep, check_egb;
  T r1, r2, dd;              // inner layer: 0.8 r_H, 0.01 r_H, 0.2 r_H (field_solver_gr.cu:666-669)
  T half[3];                 // delta / 2 (:671-673)
  T upper[3];                // lower + size
  T* Ed[3];                  // E at the E positions
  T* Hd[3];                  // H at the B positions
  T* Bd[3];                  // lowered B at the B positions (the reference keeps it in B0)
  T* rho;                    // sqrt(gamma)-weighted div D at the vertices (the reference's divE)
  T* Dc[3];                  // D after the E_par cleaning (last substep)
};

template <typename T>
__device__ __forceinline__ void gyee_pos(const YeeArgs<T>& a, int st, int i, int j, int k, T p[3]) {
  p[0] = vpos(a, 0, i, st & 1);
  p[1] = vpos(a, 1, j, (st >> 1) & 1);
  p[2] = vpos(a, 2, k, (st >> 2) & 1);
}

// Component C of an E-type (IN = kStE[C]) or B-type (kStB[C]) field at a
// point of stagger OUT.
template <int C, int OUT, typename T>
__device__ __forceinline__ T e_at(T* const f[3], uint32_t o, int sy, int sz) {
  return interp_at<kStE[C], OUT>(f[C], o, sy, sz);
}
template <int C, int OUT, typename T>
__device__ __forceinline__ T b_at(T* const f[3], uint32_t o, int sy, int sz) {
  return interp_at<kStB[C], OUT>(f[C], o, sy, sz);
}
template <int C, int OUT, typename T>
__device__ __forceinline__ T e_at(const T* const f[3], uint32_t o, int sy, int sz) {
  return interp_at<kStE[C], OUT>(f[C], o, sy, sz);
}
template <int C, int OUT, typename T>
__device__ __forceinline__ T b_at(const T* const f[3], uint32_t o, int sy, int sz) {
  return interp_at<kStB[C], OUT>(f[C], o, sy, sz);
}

// ------------------------------------------------------------- E, H pass

template <int A, typename T>
__device__ __forceinline__ void gyee_e(const GYeeArgs<T>& g, int i, int j, int k, uint32_t o,
                                       int sy, int sz) {
  constexpr int st = kStE[A], b = (A + 1) % 3, c = (A + 2) % 3;
  const YeeArgs<T>& a = g.y;
  T p[3];
  gyee_pos(a, st, i, j, k, p);
  const Cks<T> m(g.spin, p[0], p[1], p[2]);
  const T iD[3] = {e_at<0, st>(a.E, o, sy, sz), e_at<1, st>(a.E, o, sy, sz),
                   e_at<2, st>(a.E, o, sy, sz)};
  T iB[3];
  iB[b] = b_at<b, st>(a.B, o, sy, sz);
  iB[c] = b_at<c, st>(a.B, o, sy, sz);
  T dl[3];
  m.lower(iD, dl);
  // kernel_compute_E_gr_thread (field_solver_gr.cu:99-149)
  g.Ed[A][o] = m.alpha * dl[A] + m.sg * (m.bu[b] * iB[c] - m.bu[c] * iB[b]);
}

template <int A, typename T>
__device__ __forceinline__ void gyee_h(const GYeeArgs<T>& g, int i, int j, int k, uint32_t o,
                                       int sy, int sz) {
  constexpr int st = kStB[A], b = (A + 1) % 3, c = (A + 2) % 3;
  const YeeArgs<T>& a = g.y;
  T p[3];
  gyee_pos(a, st, i, j, k, p);
  const Cks<T> m(g.spin, p[0], p[1], p[2]);
  const T iB[3] = {b_at<0, st>(a.B, o, sy, sz), b_at<1, st>(a.B, o, sy, sz),
                   b_at<2, st>(a.B, o, sy, sz)};
  T iD[3];
  iD[b] = e_at<b, st>(a.E, o, sy, sz);
  iD[c] = e_at<c, st>(a.E, o, sy, sz);
  T bl[3];
  m.lower(iB, bl);
  // kernel_compute_H_gr_thread (field_solver_gr.cu:152-225)
  g.Hd[A][o] = m.alpha * bl[A] - m.sg * (m.bu[b] * iD[c] - m.bu[c] * iD[b]);
  g.Bd[A][o] = bl[A];
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? COFFEE_GYEE_MIN_BLOCKS : 1)
gyee_eh_kernel(const GYeeArgs<T> g) {
  const YeeArgs<T>& a = g.y;
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = 1 + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i >= a.g.dims[0] - 1 || j >= a.g.dims[1] - 1 || k >= a.g.dims[2] - 1) return;
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  const uint32_t o = (uint32_t)k * (uint32_t)sz + (uint32_t)j * (uint32_t)sy + (uint32_t)i;
  gyee_e<0>(g, i, j, k, o, sy, sz);
  gyee_e<1>(g, i, j, k, o, sy, sz);
  gyee_e<2>(g, i, j, k, o, sy, sz);
  gyee_h<0>(g, i, j, k, o, sy, sz);
  gyee_h<1>(g, i, j, k, o, sy, sz);
  gyee_h<2>(g, i, j, k, o, sy, sz);
}

// rho = div(sqrt(gamma) D) / sqrt(gamma) at the vertex, backward differences
// (kernel_compute_rho_gr_thread, field_solver_gr.cu:29-53)
template <typename T>
__global__ void __launch_bounds__(256) gyee_rho_kernel(const GYeeArgs<T> g) {
  const YeeArgs<T>& a = g.y;
  const int i = a.g.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.g.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = a.g.lo[2] + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i >= a.g.hi[0] || j >= a.g.hi[1] || k >= a.g.hi[2]) return;
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  const uint32_t o = (uint32_t)k * (uint32_t)sz + (uint32_t)j * (uint32_t)sy + (uint32_t)i;
  const T x = vpos(a, 0, i, 1), y = vpos(a, 1, j, 1), z = vpos(a, 2, k, 1);
  const T s = g.spin;
  const T* D0 = a.E[0];
  const T* D1 = a.E[1];
  const T* D2 = a.E[2];
  g.rho[o] = (a.inv[0] * (D0[o] * cks_sqrt_gamma(s, x + g.half[0], y, z) -
                          D0[o - 1] * cks_sqrt_gamma(s, x - g.half[0], y, z)) +
              a.inv[1] * (D1[o] * cks_sqrt_gamma(s, x, y + g.half[1], z) -
                          D1[o - (uint32_t)sy] * cks_sqrt_gamma(s, x, y - g.half[1], z)) +
              a.inv[2] * (D2[o] * cks_sqrt_gamma(s, x, y, z + g.half[2]) -
                          D2[o - (uint32_t)sz] * cks_sqrt_gamma(s, x, y, z - g.half[2]))) /
             cks_sqrt_gamma(s, x, y, z);
}

// ----------------------------------------------------------- update pass

template <typename T>
__device__ __forceinline__ T gyee_sg(const GYeeArgs<T>& g, int st, int i, int j, int k) {
  T p[3];
  gyee_pos(g.y, st, i, j, k, p);
  return cks_sqrt_gamma(g.spin, p[0], p[1], p[2]);
}

// dt times the current at E position A (field_solver_gr.cu:292-373):
// dt rho (E x B_lower)_A / sqrt(gamma) / (B . B_lower + TINY)
template <int A, typename T>
__device__ __forceinline__ T gyee_current(const GYeeArgs<T>& g, uint32_t o, int sy, int sz,
                                          T sg) {
  constexpr int out = kStE[A], b = (A + 1) % 3, c = (A + 2) % 3;
  const YeeArgs<T>& a = g.y;
  const T* Ed[3] = {g.Ed[0], g.Ed[1], g.Ed[2]};
  const T* Bd[3] = {g.Bd[0], g.Bd[1], g.Bd[2]};
  const T ir = interp_at<kStRho, out>(g.rho, o, sy, sz);
  const T ie[3] = {e_at<0, out>(Ed, o, sy, sz), e_at<1, out>(Ed, o, sy, sz),
                   e_at<2, out>(Ed, o, sy, sz)};
  const T ib[3] = {b_at<0, out>(a.B, o, sy, sz), b_at<1, out>(a.B, o, sy, sz),
                   b_at<2, out>(a.B, o, sy, sz)};
  const T ibd[3] = {b_at<0, out>(Bd, o, sy, sz), b_at<1, out>(Bd, o, sy, sz),
                    b_at<2, out>(Bd, o, sy, sz)};
  const T den = ib[0] * ibd[0] + ib[1] * ibd[1] + ib[2] * ibd[2] + Tiny<T>::v;
  return a.dt * ir * (ie[b] * ibd[c] - ibd[b] * ie[c]) / sg / den;
}

template <typename T, bool FIRST>
__global__ void __launch_bounds__(256) gyee_update_kernel(const GYeeArgs<T> g, const T c1,
                                                          const T c2, const T c3) {
  const YeeArgs<T>& a = g.y;
  const int i = a.g.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.g.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = a.g.lo[2] + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i >= a.g.hi[0] || j >= a.g.hi[1] || k >= a.g.hi[2]) return;
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  const uint32_t o = (uint32_t)k * (uint32_t)sz + (uint32_t)j * (uint32_t)sy + (uint32_t)i;
  const uint32_t ox = 1, oy = (uint32_t)sy, oz = (uint32_t)sz;
  const T CCx = a.cc[0], CCy = a.cc[1], CCz = a.cc[2];
  const T *ex = g.Ed[0], *ey = g.Ed[1], *ez = g.Ed[2];
  const T *hx = g.Hd[0], *hy = g.Hd[1], *hz = g.Hd[2];
  // dB = -curl E dt / sqrt(gamma), dD = curl H dt / sqrt(gamma) (:258-283)
  const T dbx = (CCz * (ey[o + oz] - ey[o]) - CCy * (ez[o + oy] - ez[o])) /
                gyee_sg(g, kStB[0], i, j, k);
  const T dby = (CCx * (ez[o + ox] - ez[o]) - CCz * (ex[o + oz] - ex[o])) /
                gyee_sg(g, kStB[1], i, j, k);
  const T dbz = (CCy * (ex[o + oy] - ex[o]) - CCx * (ey[o + ox] - ey[o])) /
                gyee_sg(g, kStB[2], i, j, k);
  const T sgx = gyee_sg(g, kStE[0], i, j, k), sgy = gyee_sg(g, kStE[1], i, j, k),
          sgz = gyee_sg(g, kStE[2], i, j, k);
  T ddx = (CCz * (hy[o - oz] - hy[o]) - CCy * (hz[o - oy] - hz[o])) / sgx;
  T ddy = (CCx * (hz[o - ox] - hz[o]) - CCz * (hx[o - oz] - hx[o])) / sgy;
  T ddz = (CCy * (hx[o - oy] - hx[o]) - CCx * (hy[o - ox] - hy[o])) / sgz;
  if (g.calc_current) {
    ddx = ddx - gyee_current<0>(g, o, sy, sz, sgx);
    ddy = ddy - gyee_current<1>(g, o, sy, sz, sgy);
    ddz = ddz - gyee_current<2>(g, o, sy, sz, sgz);
  }
  // D = c1 Dn + c2 D + c3 dD, B likewise (kernel_rk_update_gr_thread, :382-414)
  const T d[3] = {a.E[0][o], a.E[1][o], a.E[2][o]};
  const T b[3] = {a.B[0][o], a.B[1][o], a.B[2][o]};
  T dn[3], bn[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if constexpr (FIRST) {
      dn[q] = d[q];
      bn[q] = b[q];
      a.En[q][o] = d[q];
      a.Bn[q][o] = b[q];
    } else {
      dn[q] = a.En[q][o];
      bn[q] = a.Bn[q][o];
    }
  }
  a.Es[0][o] = c1 * dn[0] + c2 * d[0] + c3 * ddx;
  a.Es[1][o] = c1 * dn[1] + c2 * d[1] + c3 * ddy;
  a.Es[2][o] = c1 * dn[2] + c2 * d[2] + c3 * ddz;
  a.Bs[0][o] = c1 * bn[0] + c2 * b[0] + c3 * dbx;
  a.Bs[1][o] = c1 * bn[1] + c2 * b[1] + c3 * dby;
  a.Bs[2][o] = c1 * bn[2] + c2 * b[2] + c3 * dbz;
}

// ------------------------------------------------------------ clean, clamp

// E_par cleaning at E position A (kernel_clean_epar_gr_thread, :416-517):
// D - (D . B_lower) B_A / (B . B_lower + TINY), D and B interpolated there.
template <int A, typename T>
__device__ __forceinline__ T gyee_clean_comp(const GYeeArgs<T>& g, int i, int j, int k,
                                             uint32_t o, int sy, int sz) {
  constexpr int st = kStE[A];
  const YeeArgs<T>& a = g.y;
  T p[3];
  gyee_pos(a, st, i, j, k, p);
  const Cks<T> m(g.spin, p[0], p[1], p[2]);
  const T* Ds[3] = {a.Es[0], a.Es[1], a.Es[2]};
  const T* Bs[3] = {a.Bs[0], a.Bs[1], a.Bs[2]};
  const T iD[3] = {e_at<0, st>(Ds, o, sy, sz), e_at<1, st>(Ds, o, sy, sz),
                   e_at<2, st>(Ds, o, sy, sz)};
  const T iB[3] = {b_at<0, st>(Bs, o, sy, sz), b_at<1, st>(Bs, o, sy, sz),
                   b_at<2, st>(Bs, o, sy, sz)};
  T bl[3];
  m.lower(iB, bl);
  return iD[A] - (iD[0] * bl[0] + iD[1] * bl[1] + iD[2] * bl[2]) * iB[A] /
                     (iB[0] * bl[0] + iB[1] * bl[1] + iB[2] * bl[2] + Tiny<T>::v);
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? COFFEE_GYEE_MIN_BLOCKS : 1)
gyee_clean_kernel(const GYeeArgs<T> g) {
  const YeeArgs<T>& a = g.y;
  const int i = a.g.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.g.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = a.g.lo[2] + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i >= a.g.hi[0] || j >= a.g.hi[1] || k >= a.g.hi[2]) return;
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  const uint32_t o = (uint32_t)k * (uint32_t)sz + (uint32_t)j * (uint32_t)sy + (uint32_t)i;
  g.Dc[0][o] = gyee_clean_comp<0>(g, i, j, k, o, sy, sz);
  g.Dc[1][o] = gyee_clean_comp<1>(g, i, j, k, o, sy, sz);
  g.Dc[2][o] = gyee_clean_comp<2>(g, i, j, k, o, sy, sz);
}

// |D| <= |B| in the metric at E position A (kernel_check_eGTb_gr_thread,
// :519-647): reads the D of before the pass (src) and B', so it is free of
// the flat solver's race.
template <int A, typename T>
__device__ __forceinline__ T gyee_check_comp(const GYeeArgs<T>& g, const T* const src[3], int i,
                                             int j, int k, uint32_t o, int sy, int sz) {
  constexpr int st = kStE[A];
  const YeeArgs<T>& a = g.y;
  T p[3];
  gyee_pos(a, st, i, j, k, p);
  const Cks<T> m(g.spin, p[0], p[1], p[2]);
  const T* Bs[3] = {a.Bs[0], a.Bs[1], a.Bs[2]};
  const T iD[3] = {e_at<0, st>(src, o, sy, sz), e_at<1, st>(src, o, sy, sz),
                   e_at<2, st>(src, o, sy, sz)};
  T dl[3];
  m.lower(iD, dl);
  const T emag = iD[0] * dl[0] + iD[1] * dl[1] + iD[2] * dl[2] + Tiny<T>::v;
  const T iB[3] = {b_at<0, st>(Bs, o, sy, sz), b_at<1, st>(Bs, o, sy, sz),
                   b_at<2, st>(Bs, o, sy, sz)};
  T bl[3];
  m.lower(iB, bl);
  const T bmag = iB[0] * bl[0] + iB[1] * bl[1] + iB[2] * bl[2] + Tiny<T>::v;
  const T temp = emag > bmag ? sqrt(bmag / emag) : (T)1;
  return temp * src[A][o];
}

// pmlsigma_gr (:657-661): sig0 (distance / scale)^3 through pow in double
template <typename T>
__device__ __forceinline__ T gyee_pml(T v, T lo, T hi, T scale, T sig0) {
  if (v > hi) return (T)((double)sig0 * pow((double)((v - hi) / scale), 3.0));
  if (v < lo) return (T)((double)sig0 * pow((double)((lo - v) / scale), 3.0));
  return (T)0;
}

// The absorbing layers of the last substep at vertex (i, j, k)
// (kernel_absorbing_boundary_gr_thread, :663-775)
template <typename T>
__device__ __forceinline__ void gyee_absorb(const GYeeArgs<T>& g, int i, int j, int k,
                                            uint32_t o, T u[6]) {
  const YeeArgs<T>& a = g.y;
  const T x = vpos(a, 0, i, 1), y = vpos(a, 1, j, 1), z = vpos(a, 2, k, 1);
  T un[6];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    un[c] = a.En[c][o];
    un[3 + c] = a.Bn[c][o];
  }
  const T r = cks_r(g.spin, x, y, z);
  if (r < g.r1) {
    // each component damped at its own position: sig0 cube((r1 - r) / dd) dt
    const T hx = g.half[0], hy = g.half[1], hz = g.half[2];
    const T px[6] = {x + hx, x, x, x, x + hx, x + hx};
    const T py[6] = {y, y + hy, y, y + hy, y, y + hy};
    const T pz[6] = {z, z, z + hz, z + hz, z + hz, z};
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const T q = (g.r1 - cks_r(g.spin, px[c], py[c], pz[c])) / g.dd;
      const T sig = a.sigpml * (q * q * q) * a.dt;
      if (sig > Tiny<T>::v) u[c] = absorb(sig, u[c], un[c]);
    }
  }
  if (r < g.r2) {
#pragma unroll
    for (int c = 0; c < 6; ++c) u[c] = (T)0;
  }
  if (x > a.pml_hi[0] || x < a.pml_lo[0] || y > a.pml_hi[1] || y < a.pml_lo[1] ||
      z > a.pml_hi[2] || z < a.pml_lo[2]) {
    const T sig = gyee_pml(x, a.pml_lo[0], a.pml_hi[0], a.pml_scale, a.sigpml) +
                  gyee_pml(y, a.pml_lo[1], a.pml_hi[1], a.pml_scale, a.sigpml) +
                  gyee_pml(z, a.pml_lo[2], a.pml_hi[2], a.pml_scale, a.sigpml);
    if (sig > Tiny<T>::v) {
#pragma unroll
      for (int c = 0; c < 6; ++c) u[c] = absorb(sig, u[c], un[c]);
    }
  }
  const T* lo = a.c.lower;
  if (x <= lo[0] || x >= g.upper[0] || y <= lo[1] || y >= g.upper[1] || z <= lo[2] ||
      z >= g.upper[2]) {
#pragma unroll
    for (int c = 0; c < 6; ++c) u[c] = un[c];
  }
}

template <typename T, bool LAST>
__global__ void __launch_bounds__(256) gyee_clamp_kernel(const GYeeArgs<T> g) {
  const YeeArgs<T>& a = g.y;
  const int i = a.g.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.g.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = a.g.lo[2] + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i >= a.g.hi[0] || j >= a.g.hi[1] || k >= a.g.hi[2]) return;
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  const uint32_t o = (uint32_t)k * (uint32_t)sz + (uint32_t)j * (uint32_t)sy + (uint32_t)i;
  T u[6];
  if (g.check_egb) {
    // the rescale reads the cleaned D in the last substep; without the
    // rescale the cleaned D is never stored (the reference cleans into dD and
    // only the rescale writes D from it)
    const bool cleaned = LAST && g.clean_ep;
    const T* src[3] = {cleaned ? g.Dc[0] : a.Es[0], cleaned ? g.Dc[1] : a.Es[1],
                       cleaned ? g.Dc[2] : a.Es[2]};
    u[0] = gyee_check_comp<0>(g, src, i, j, k, o, sy, sz);
    u[1] = gyee_check_comp<1>(g, src, i, j, k, o, sy, sz);
    u[2] = gyee_check_comp<2>(g, src, i, j, k, o, sy, sz);
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = a.Es[c][o];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) u[3 + c] = a.Bs[c][o];
  if (LAST) gyee_absorb(g, i, j, k, o, u);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    a.Eo[c][o] = u[c];
    a.Bo[c][o] = u[3 + c];
  }
}

}  // namespace coffee
