// Kernels of the GR force-free solver in Cartesian Kerr-Schild coordinates
// (reference src/algorithms/field_solver_gr_EZ.cu, metric
// src/algorithms/metric_cks_impl.hpp).
//
// sim_data's E holds the densitised displacement D; the curl acts on the
// constitutive fields E = alpha D_i + sqrt(gamma) (beta x B)_i and
// H = alpha B_i - sqrt(gamma) (beta x D)_i.  A stage is two launches: one
// writes E and H over the whole grid (the reference's get_Ed / get_Hd), the
// other does the LSRK update, the clamps and, in the last stage, both
// absorbing layers in one pass over the update box, reading the current
// buffer and writing the other one.  Near the horizon the metric comes from
// a table evaluated once per solver in FP64 (gr_metric_kernel); elsewhere it
// is evaluated per point in field precision, as the reference does, but
// once per point and launch (the reference calls get_r inside every metric
// component, about forty times per point).
#pragma once

#include "axisym_kernels.cuh"
#include "ez_common.cuh"

namespace coffee {

template <typename T>
struct GrConst {
  int d[3];                 // dims
  int lo[3], hi[3];         // update box
  int g[3];                 // guards
  T lower[3], delta[3], inv_delta[3];
  T a, dt, tau, ko_c;
  int calc_current, divB_clean, clean_ep, check_egb;
  int absorbing;
  T xl[3], xh[3];           // outer layer edges (boundary.cu:43-54)
  T pmlscale, sigpml;
  T r1, r2, dd;             // inner layer: 0.7 r_H, 0.01 r_H, 0.2 r_H (:617-621)
  int nb_lo[3], nb_n[3];    // the near-horizon box of the metric table (grid indices)
};

// r of the Kerr-Schild coordinates (metric_cks_impl.hpp:17-24)
template <typename T>
__device__ __forceinline__ T cks_r(T a, T x, T y, T z) {
  const T R2 = x * x + y * y + z * z;
  const T q = R2 - a * a;
  T s = q * q + T(4) * (a * z) * (a * z);
  if (s < Tiny<T>::v) s = Tiny<T>::v;
  return sqrt((q + sqrt(s)) * T(0.5));
}

// sqrt(gamma) = sqrt(1 + 2 r^3 / (r^4 + a^2 z^2)) (:77-83)
template <typename T>
__device__ __forceinline__ T cks_sqrt_gamma(T a, T x, T y, T z) {
  const T r = cks_r(a, x, y, z);
  T den = r * r * r * r + a * a * z * z;
  if (den < Tiny<T>::v) den = Tiny<T>::v;
  return sqrt(T(1) + T(2) * r * r * r / den);
}

// All metric functions at one point (metric_cks_impl.hpp:13-181), in
// precision T with the TINY floors of the field precision TF.
template <typename T, typename TF = T>
struct Cks {
  T r, alpha, sg;
  T bu[3];
  T gd11, gd12, gd13, gd22, gd23, gd33;
  T gu11, gu12, gu13, gu22, gu23, gu33;

  Cks() = default;
  __device__ __forceinline__ Cks(T a, T x, T y, T z) {
    constexpr T tiny = (T)Tiny<TF>::v;
    {
      const T R2 = x * x + y * y + z * z;
      const T q = R2 - a * a;
      T s = q * q + T(4) * (a * z) * (a * z);
      if (s < tiny) s = tiny;
      r = sqrt((q + sqrt(s)) * T(0.5));
    }
    const T r2 = r * r, r3 = r2 * r, r4 = r2 * r2;
    const T aa = a * a, azz = aa * z * z;
    T den = r4 + azz;
    if (den < tiny) den = tiny;
    T denu = T(2) * r3 + r4 + azz;
    if (denu < tiny) denu = tiny;
    T ar = aa + r2;
    T ar2 = ar * ar;
    if (ar < tiny) ar = tiny;
    if (ar2 < tiny) ar2 = tiny;
    const T lx = r * x + a * y, ly = -a * x + r * y;
    const T iden = T(1) / den, idenu = T(1) / denu, iar = T(1) / ar, iar2 = T(1) / ar2;
    const T gam = T(1) + T(2) * r3 * iden;
    sg = sqrt(gam);
    alpha = sqrt(T(1) / gam);
    bu[0] = T(2) * r3 * lx * iar * idenu;
    bu[1] = T(2) * r3 * ly * iar * idenu;
    bu[2] = T(2) * r2 * z * idenu;
    const T hd = T(2) * r3 * iar2 * iden, hu = T(2) * r3 * iar2 * idenu;
    const T kd = T(2) * r2 * iar * iden, ku = T(2) * r2 * iar * idenu;
    gd11 = T(1) + hd * lx * lx;
    gd12 = hd * lx * ly;
    gd13 = kd * lx * z;
    gd22 = T(1) + hd * ly * ly;
    gd23 = kd * ly * z;
    gd33 = T(1) + T(2) * r * z * z * iden;
    gu11 = T(1) - hu * lx * lx;
    gu12 = -hu * lx * ly;
    gu13 = -ku * lx * z;
    gu22 = T(1) - hu * ly * ly;
    gu23 = -ku * ly * z;
    gu33 = T(1) - T(2) * r * z * z * idenu;
  }
  __device__ __forceinline__ void lower(const T* v, T* o) const {
    o[0] = gd11 * v[0] + gd12 * v[1] + gd13 * v[2];
    o[1] = gd12 * v[0] + gd22 * v[1] + gd23 * v[2];
    o[2] = gd13 * v[0] + gd23 * v[1] + gd33 * v[2];
  }
  __device__ __forceinline__ void raise(const T* v, T* o) const {
    o[0] = gu11 * v[0] + gu12 * v[1] + gu13 * v[2];
    o[1] = gu12 * v[0] + gu22 * v[1] + gu23 * v[2];
    o[2] = gu13 * v[0] + gu23 * v[1] + gu33 * v[2];
  }
};

template <typename T>
__device__ __forceinline__ T gr_pos(const GrConst<T>& c, int a, int n) {
  return c.lower[a] + c.delta[a] * (T)(n - c.g[a]);
}

// The near-horizon metric table.  Within a box of half-width kNearRH r_H
// around the hole the metric is evaluated once per solver in FP64 (at the
// grid's coordinates in the field precision, where the reference evaluates
// it) and rounded to the field precision: there the field-precision formula
// loses digits (r from sqrt((q + sqrt(q^2 + 4 a^2 z^2)) / 2) with
// q = R^2 - a^2 cancels inside the horizon, giving FP32 errors of 1e-5 in r
// and the shift against 1e-7 outside 1.5 r_H).  Elsewhere it is evaluated in
// the field precision per point, as the reference does.  kMetricComps
// components, component q of table point t at m[q * nt + t]: r, alpha,
// sqrt(gamma), beta^1..3, gamma_11, _12, _13, _22, _23, _33, gamma^11, ^12,
// ^13, ^22, ^23, ^33.
constexpr int kMetricComps = 18;
constexpr double kNearRH = 3.0;

template <typename T>
__device__ __forceinline__ long long near_index(const GrConst<T>& c, int i, int j, int k) {
  const int a = i - c.nb_lo[0], b = j - c.nb_lo[1], e = k - c.nb_lo[2];
  if ((unsigned)a >= (unsigned)c.nb_n[0] || (unsigned)b >= (unsigned)c.nb_n[1] ||
      (unsigned)e >= (unsigned)c.nb_n[2])
    return -1;
  return a + (long long)c.nb_n[0] * (b + (long long)c.nb_n[1] * e);
}

template <typename T>
__global__ void gr_metric_kernel(const __grid_constant__ GrConst<T> c, T* __restrict__ m,
                                 T* __restrict__ sg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= c.d[0] || j >= c.d[1] || k >= c.d[2]) return;
  const long long o = i + (long long)c.d[0] * (j + (long long)c.d[1] * k);
  const Cks<double, T> q((double)c.a, (double)gr_pos(c, 0, i), (double)gr_pos(c, 1, j),
                         (double)gr_pos(c, 2, k));
  // sqrt(gamma) of every point: the divergence stencil (div4,
  // field_solver_gr_EZ.cu:44-86) weights each neighbour by it
  sg[o] = (T)q.sg;
  const long long t = near_index(c, i, j, k);
  if (t < 0) return;
  const long long nt = (long long)c.nb_n[0] * c.nb_n[1] * c.nb_n[2];
  const double v[kMetricComps] = {q.r,    q.alpha, q.sg,   q.bu[0], q.bu[1], q.bu[2],
                                  q.gd11, q.gd12,  q.gd13, q.gd22,  q.gd23,  q.gd33,
                                  q.gu11, q.gu12,  q.gu13, q.gu22,  q.gu23,  q.gu33};
#pragma unroll
  for (int a = 0; a < kMetricComps; ++a) m[a * nt + t] = (T)v[a];
}

// The metric at grid point (i, j, k) with coordinates (x, y, z): from the
// table inside the near-horizon box, else evaluated here.
template <typename T>
__device__ __forceinline__ Cks<T> metric_at(const GrConst<T>& c, const T* __restrict__ m,
                                            int i, int j, int k, T x, T y, T z) {
  const long long t = near_index(c, i, j, k);
  if (t < 0) return Cks<T>(c.a, x, y, z);
  const long long nt = (long long)c.nb_n[0] * c.nb_n[1] * c.nb_n[2];
  Cks<T> q;
  q.r = __ldg(m + t);
  q.alpha = __ldg(m + nt + t);
  q.sg = __ldg(m + 2 * nt + t);
#pragma unroll
  for (int a = 0; a < 3; ++a) q.bu[a] = __ldg(m + (3 + a) * nt + t);
  q.gd11 = __ldg(m + 6 * nt + t);
  q.gd12 = __ldg(m + 7 * nt + t);
  q.gd13 = __ldg(m + 8 * nt + t);
  q.gd22 = __ldg(m + 9 * nt + t);
  q.gd23 = __ldg(m + 10 * nt + t);
  q.gd33 = __ldg(m + 11 * nt + t);
  q.gu11 = __ldg(m + 12 * nt + t);
  q.gu12 = __ldg(m + 13 * nt + t);
  q.gu13 = __ldg(m + 14 * nt + t);
  q.gu22 = __ldg(m + 15 * nt + t);
  q.gu23 = __ldg(m + 16 * nt + t);
  q.gu33 = __ldg(m + 17 * nt + t);
  return q;
}

// E = alpha D + sqrt(gamma) beta x B and H = alpha B - sqrt(gamma) beta x D
// (lowered D, B) at one point, stored at offset o of eh[0..5]
// (kernel_compute_E_gr / kernel_compute_H_gr, field_solver_gr_EZ.cu:88-186).
// Every kernel that writes D and B at a point also writes E and H there
// through this function, so they are computed the same way everywhere.
template <typename T>
__device__ __forceinline__ void gr_eh_store(const Cks<T>& m, const T* D, const T* B,
                                            const F7<T>& eh, long long o) {
  T Dd[3], Bd[3];
  m.lower(D, Dd);
  m.lower(B, Bd);
  eh.p[0][o] = m.alpha * Dd[0] + m.sg * (m.bu[1] * B[2] - m.bu[2] * B[1]);
  eh.p[1][o] = m.alpha * Dd[1] + m.sg * (m.bu[2] * B[0] - m.bu[0] * B[2]);
  eh.p[2][o] = m.alpha * Dd[2] + m.sg * (m.bu[0] * B[1] - m.bu[1] * B[0]);
  eh.p[3][o] = m.alpha * Bd[0] - m.sg * (m.bu[1] * D[2] - m.bu[2] * D[1]);
  eh.p[4][o] = m.alpha * Bd[1] - m.sg * (m.bu[2] * D[0] - m.bu[0] * D[2]);
  eh.p[5][o] = m.alpha * Bd[2] - m.sg * (m.bu[0] * D[1] - m.bu[1] * D[0]);
}

// E and H over the whole grid (guards included): once per call of the
// solver, for both field buffers; afterwards every stage and KO pass writes
// E and H of the points it updates (ehout), so the next kernel finds those
// of its input.  eh[0..2] = E, eh[3..5] = H.
template <typename T>
__global__ void __launch_bounds__(256) gr_eh_kernel(const __grid_constant__ GrConst<T> c,
                                                    const F7<T> u, const F7<T> eh,
                                                    const T* __restrict__ mt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= c.d[0] || j >= c.d[1] || k >= c.d[2]) return;
  const long long o = i + (long long)c.d[0] * (j + (long long)c.d[1] * k);
  const Cks<T> m =
      metric_at(c, mt, i, j, k, gr_pos(c, 0, i), gr_pos(c, 1, j), gr_pos(c, 2, k));
  const T D[3] = {__ldg(u.p[0] + o), __ldg(u.p[1] + o), __ldg(u.p[2] + o)};
  const T B[3] = {__ldg(u.p[3] + o), __ldg(u.p[4] + o), __ldg(u.p[5] + o)};
  gr_eh_store(m, D, B, eh, o);
}

// clean_epar / check_eGTb with the 3-metric (kernel_clean_epar_gr,
// kernel_check_eGTb_gr, field_solver_gr_EZ.cu:422-521)
template <typename T>
__device__ __forceinline__ void gr_clamps(const GrConst<T>& c, const Cks<T>& m, T* v) {
  if (c.clean_ep) {
    T Bd[3];
    m.lower(v + 3, Bd);
    T B2 = v[3] * Bd[0] + v[4] * Bd[1] + v[5] * Bd[2];
    if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
    const T q = fdiv(v[0] * Bd[0] + v[1] * Bd[1] + v[2] * Bd[2], B2);
    v[0] -= q * v[3];
    v[1] -= q * v[4];
    v[2] -= q * v[5];
  }
  if (c.check_egb) {
    T Dd[3], Bd[3];
    m.lower(v, Dd);
    m.lower(v + 3, Bd);
    T D2 = v[0] * Dd[0] + v[1] * Dd[1] + v[2] * Dd[2];
    if (D2 < Tiny<T>::v) D2 = Tiny<T>::v;
    const T B2 = v[3] * Bd[0] + v[4] * Bd[1] + v[5] * Bd[2];
    if (D2 > B2) {
      const T s = sqrt(fdiv(B2, D2));
      v[0] *= s;
      v[1] *= s;
      v[2] *= s;
    }
  }
}

// Outer layer at the six faces (kernel_boundary_absorbing_thread,
// src/algorithms/boundary.cu:17-79), then the inner layer inside 0.7 r_H and
// the zeroed core inside 0.01 r_H (kernel_absorbing_inner,
// field_solver_gr_EZ.cu:610-701); both blend towards the start-of-step
// values n.
template <typename T>
__device__ __noinline__ V7<T> gr_absorb(const GrConst<T>& c, V7<T> v, V7<T> n, T x, T y, T z,
                                        T r) {
  const T pos[3] = {x, y, z};
  bool outside = false;
  T sig = T(0);
  for (int a = 0; a < 3; ++a) {
    outside = outside || pos[a] > c.xh[a] || pos[a] < c.xl[a];
    sig += cyl_pmlsigma(pos[a], c.xl[a], c.xh[a], c.pmlscale, c.sigpml);
  }
  if (outside && sig > Tiny<T>::v) {
    const T e = exp(-sig);
    const T f = (T(1) - e) / sig;
    for (int a = 0; a < 6; ++a) v.v[a] = e * n.v[a] + f * (v.v[a] - n.v[a]);
  }
  if (r < c.r1) {
    const T q = (c.r1 - r) / c.dd;
    const T s = c.sigpml * q * q * q * c.dt;
    if (s > Tiny<T>::v) {
      const T e = exp(-s);
      const T f = (T(1) - e) / s;
      for (int a = 0; a < 6; ++a) v.v[a] = e * n.v[a] + f * (v.v[a] - n.v[a]);
    }
  }
  if (r < c.r2)
    for (int a = 0; a < 6; ++a) v.v[a] = T(0);
  return v;
}

// One LSRK stage of the GR solver (kernel_rk_step1_gr + kernel_rk_step2_gr,
// field_solver_gr_EZ.cu:188-420, then the clamps and, in the last stage,
// the absorbing layers: order of :876-893).  u: D, B, P of the current
// buffer; eh: E, H of the same buffer.
// Minimum resident 256-thread CTAs per SM of the stage kernel: the kernel is
// bound by the latency of its stencil loads, and 6 CTAs (40 registers, a
// little spilling) hide it best (1.31 -> 1.19 ms per launch at 256^3; 7 or 8
// CTAs spill too much).
#ifndef COFFEE_GR_STAGE_MIN_BLOCKS
#define COFFEE_GR_STAGE_MIN_BLOCKS 6
#endif
// The stage at one point, given its stencil values through fetch(q, ax,
// n): array q (0-2 E, 3-5 H, 6-8 D, 9-11 B, 12 P, 13 sqrt(gamma)) at offset
// n = -2, -1, 1, 2 along axis ax from the point, and own(q), array q at the
// point (read where the values are first needed, which keeps them out of
// the registers of the stencil sums).  Both stage kernels (global stencil
// loads, shared-memory tiles) run this code, so their arithmetic is the
// same.
template <typename T, bool FIRST, typename Metric, typename Fetch, typename Own>
__device__ __forceinline__ void gr_stage_point(const GrConst<T>& c, Metric&& metric, const T x,
                                               const T y, const T z, const long long o,
                                               Fetch&& f, Own&& own,
                                               const F7<T>& out, const F7<T>& du,
                                               const F7<T>& un, const F5<T>& aux, const T As,
                                               const T Bs, const int flags,
                                               const F7<T>& ehout) {
  auto d1 = [&](auto qc, auto ac) {
    constexpr int ax = decltype(ac)::value;
    return d1_4w(f(qc, ac, -2), f(qc, ac, -1), f(qc, ac, 1), f(qc, ac, 2)) * c.inv_delta[ax];
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  // the curls and divergences before their 1 / sqrt(gamma) factor: the
  // metric is evaluated after the stencil sums, so that its values do not
  // take registers while those are formed (the same operations either way)
  T rotH[3] = {d1(std::integral_constant<int, 5>{}, I1{}) -
                   d1(std::integral_constant<int, 4>{}, I2{}),
               d1(std::integral_constant<int, 3>{}, I2{}) -
                   d1(std::integral_constant<int, 5>{}, I0{}),
               d1(std::integral_constant<int, 4>{}, I0{}) -
                   d1(std::integral_constant<int, 3>{}, I1{})};
  T rotE[3] = {d1(std::integral_constant<int, 2>{}, I1{}) -
                   d1(std::integral_constant<int, 1>{}, I2{}),
               d1(std::integral_constant<int, 0>{}, I2{}) -
                   d1(std::integral_constant<int, 2>{}, I0{}),
               d1(std::integral_constant<int, 1>{}, I0{}) -
                   d1(std::integral_constant<int, 0>{}, I1{})};
  // div4 (:44-86): each neighbour weighted by sqrt(gamma) there (the
  // per-solver table; the reference evaluates it at the shifted coordinates)
  T divD = T(0), divB = T(0);
  static_for<3>([&](auto ac) {
    constexpr int ax = decltype(ac)::value;
    using QS = std::integral_constant<int, 13>;
    using QD = std::integral_constant<int, 6 + ax>;
    using QB = std::integral_constant<int, 9 + ax>;
    const T w[4] = {f(QS{}, ac, -2), f(QS{}, ac, -1), f(QS{}, ac, 1), f(QS{}, ac, 2)};
    divD += d1_4w(f(QD{}, ac, -2) * w[0], f(QD{}, ac, -1) * w[1], f(QD{}, ac, 1) * w[2],
                  f(QD{}, ac, 2) * w[3]) * c.inv_delta[ax];
    divB += d1_4w(f(QB{}, ac, -2) * w[0], f(QB{}, ac, -1) * w[1], f(QB{}, ac, 1) * w[2],
                  f(QB{}, ac, 2) * w[3]) * c.inv_delta[ax];
  });
  const Cks<T> m = metric();
  const T igms = T(1) / m.sg;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    rotH[a] *= igms;
    rotE[a] *= igms;
  }
  divD *= igms;
  divB *= igms;
  T v[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) v[a] = own(6 + a);
  T Bd[3], Dd[3];
  m.lower(v + 3, Bd);
  m.lower(v, Dd);
  T J[3] = {T(0), T(0), T(0)};
  if (c.calc_current) {
    T B2 = v[3] * Bd[0] + v[4] * Bd[1] + v[5] * Bd[2];
    if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
    const T Jp = (Bd[0] * rotH[0] + Bd[1] * rotH[1] + Bd[2] * rotH[2]) -
                 (Dd[0] * rotE[0] + Dd[1] * rotE[1] + Dd[2] * rotE[2]);
    const T e0 = own(0), e1 = own(1), e2 = own(2);
    const T iB2 = fdiv(T(1), B2);
    J[0] = (divD * (e1 * Bd[2] - e2 * Bd[1]) * igms + Jp * v[3]) * iB2;
    J[1] = (divD * (e2 * Bd[0] - e0 * Bd[2]) * igms + Jp * v[4]) * iB2;
    J[2] = (divD * (e0 * Bd[1] - e1 * Bd[0]) * igms + Jp * v[5]) * iB2;
  }
  using QP = std::integral_constant<int, 12>;
  const T Pd[3] = {d1(QP{}, I0{}), d1(QP{}, I1{}), d1(QP{}, I2{})};
  T Pu[3];
  m.raise(Pd, Pu);
  const T shape = T(0.5) * (T(1) - tanh((m.r - T(5)) / T(1)));  // r0 = 5, del = 1 (:276-278)
  const T dt = c.dt;
  T rhs[7];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    rhs[a] = dt * (rotH[a] - J[a]);
    rhs[3 + a] = c.divB_clean ? dt * (-rotE[a] + (-m.alpha * Pu[a] + m.bu[a] * divB) * shape)
                              : -dt * rotE[a];
  }
  rhs[6] = dt * (-m.alpha * divB + m.bu[0] * Pd[0] + m.bu[1] * Pd[1] + m.bu[2] * Pd[2]) -
           m.alpha * v[6] / c.tau;
  if (flags & AX_WRITE_UN) {
#pragma unroll
    for (int a = 0; a < 6; ++a) un.p[a][o] = v[a];
  }
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const T dd = FIRST ? rhs[a] : As * du.p[a][o] + rhs[a];
    du.p[a][o] = dd;
    v[a] += Bs * dd;
  }
  if (flags & AX_AUX) {
    aux.p[0][o] = J[0];
    aux.p[1][o] = J[1];
    aux.p[2][o] = J[2];
    aux.p[3][o] = divD;
    aux.p[4][o] = divB;
  }
  gr_clamps(c, m, v);
  V7<T> w;
#pragma unroll
  for (int a = 0; a < 7; ++a) w.v[a] = v[a];
  const bool in_layer = x > c.xh[0] || x < c.xl[0] || y > c.xh[1] || y < c.xl[1] ||
                        z > c.xh[2] || z < c.xl[2] || m.r < c.r1;
  if ((flags & AX_LAST) && c.absorbing && in_layer) {
    V7<T> n;
#pragma unroll
    for (int a = 0; a < 6; ++a) n.v[a] = un.p[a][o];
    n.v[6] = T(0);
    w = gr_absorb(c, w, n, x, y, z, m.r);
  }
#pragma unroll
  for (int a = 0; a < 7; ++a) out.p[a][o] = w.v[a];
  if (ehout.p[0]) gr_eh_store(m, w.v, w.v + 3, ehout, o);
}

template <typename T, bool FIRST>
__global__ void __launch_bounds__(256, COFFEE_GR_STAGE_MIN_BLOCKS) gr_stage_kernel(const __grid_constant__ GrConst<T> c,
                                                       const F7<T> u, const F7<T> eh,
                                                       const F7<T> out, const F7<T> du,
                                                       const F7<T> un, const F5<T> aux,
                                                       const T* __restrict__ mt,
                                                       const T* __restrict__ sgt, const T As,
                                                       const T Bs, const int flags,
                                                       const F7<T> ehout) {
  const int i = c.lo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = c.lo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = c.lo[2] + blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= c.hi[0] || j >= c.hi[1] || k >= c.hi[2]) return;
  const long long sx = 1, sy = c.d[0], sz = (long long)c.d[0] * c.d[1];
  const long long o = i + sy * j + sz * k;
  const long long st[3] = {sx, sy, sz};
  const T x = gr_pos(c, 0, i), y = gr_pos(c, 1, j), z = gr_pos(c, 2, k);
  auto metric = [&]() { return metric_at(c, mt, i, j, k, x, y, z); };
  // the array pointers straight from the kernel parameters (a local array
  // of them would take registers this kernel does not have)
  auto fetch = [&](auto qc, auto ac, int n) {
    constexpr int q = decltype(qc)::value;
    const T* p;
    if constexpr (q < 6) p = eh.p[q];
    else if constexpr (q < 13) p = u.p[q - 6];
    else p = sgt;
    return __ldg(p + o + n * st[decltype(ac)::value]);
  };
  auto own = [&](int q) { return __ldg((q < 6 ? eh.p[q] : u.p[q - 6]) + o); };
  gr_stage_point<T, FIRST>(c, metric, x, y, z, o, fetch, own, out, du, un, aux, As, Bs, flags,
                           ehout);
}

// The same stage streamed along z through shared memory (FP32; opt-in with
// COFFEE_GR_TILED=1).  A CTA owns a 32 x 8 column of points and a chunk of
// z planes; each plane of the 14 stencil arrays (E, H, D, B, P,
// sqrt(gamma)) with its 2-point x / y halo is copied by cp.async into a ring
// of kGrRing planes ahead of the one computed, and the z neighbours of the
// point's own column of the 8 arrays that are differentiated along z (E_x,
// E_y, H_x, H_y, D_z, B_z, P, sqrt(gamma)) are kept in a register window of
// planes k-2 .. k+2.  The per-point global stencil loads of gr_stage_kernel
// become one coalesced copy per array and plane, but the metric, the
// near-horizon table and the per-point reads and writes of dU, the
// start-of-step copy, J and E, H keep the kernel latency-bound, and the
// registers and shared memory of the tiles leave too few warps to hide it.
// Measured at 256^3 (the Wald run): 5 slots and one CTA per SM 2.50 ms per
// stage, 4 slots and two CTAs per SM 1.61 ms, the per-point gr_stage_kernel
// 1.09 ms, which stays the default.
#ifndef COFFEE_GR_TILE_RING
#define COFFEE_GR_TILE_RING 4
#endif
#ifndef COFFEE_GR_TILE_MINB
#define COFFEE_GR_TILE_MINB 2
#endif
// ring slots: planes k .. k+2, PF = kGrRing - 4 planes in flight, the spare
constexpr int kGrTX = 32, kGrTY = 8, kGrRing = COFFEE_GR_TILE_RING, kGrArrays = 14;
constexpr int kGrPF = kGrRing - 4;
static_assert(kGrPF == 0 || kGrPF == 1, "a ring of 4 or 5 planes");
constexpr int kGrSX = kGrTX + 4, kGrSP = kGrSX * (kGrTY + 4);
#ifndef COFFEE_GR_KCHUNK
#define COFFEE_GR_KCHUNK 64
#endif

__host__ __device__ constexpr size_t gr_tile_smem_bytes() {
  return (size_t)kGrRing * kGrArrays * kGrSP * sizeof(float);
}

// window slot of array q (only the 8 arrays differentiated along z)
template <int Q>
__device__ __forceinline__ constexpr int gr_wslot() {
  return Q == 0 ? 0 : Q == 1 ? 1 : Q == 3 ? 2 : Q == 4 ? 3 : Q == 8 ? 4 : Q == 11 ? 5 : Q == 12 ? 6 : 7;
}

template <bool FIRST>
__global__ void __launch_bounds__(kGrTX * kGrTY, COFFEE_GR_TILE_MINB) gr_stage_tile_kernel(
    const __grid_constant__ GrConst<float> c, const F7<float> u, const F7<float> eh,
    const F7<float> out, const F7<float> du, const F7<float> un, const F5<float> aux,
    const float* __restrict__ mt, const float* __restrict__ sgt, const float As, const float Bs,
    const int flags, const F7<float> ehout, const int kchunk) {
  constexpr int NT = kGrTX * kGrTY, NLOAD = (kGrSP + NT - 1) / NT;
  constexpr int WQ[8] = {0, 1, 3, 4, 8, 11, 12, 13};  // the window's arrays
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* ring = reinterpret_cast<float*>(smem_raw);  // [kGrRing][kGrArrays][kGrSP]
  const uint32_t rbase = smem_u32(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kGrTX + tx;
  const int i = c.lo[0] + blockIdx.x * kGrTX + tx;
  const int j = c.lo[1] + blockIdx.y * kGrTY + ty;
  const int k0 = c.lo[2] + blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, c.hi[2]);
  const bool active = i < c.hi[0] && j < c.hi[1];
  const long long sy = c.d[0], sz = (long long)c.d[0] * c.d[1];
  const float* arr[kGrArrays] = {eh.p[0], eh.p[1], eh.p[2], eh.p[3], eh.p[4],
                                 eh.p[5], u.p[0],  u.p[1],  u.p[2],  u.p[3],
                                 u.p[4],  u.p[5],  u.p[6],  sgt};
  // this thread's copies of a plane: tile point e -> shared slot, global offset
  const int gx0 = c.lo[0] + (int)blockIdx.x * kGrTX - 2, gy0 = c.lo[1] + (int)blockIdx.y * kGrTY - 2;
  int soff[NLOAD];
  long long goff[NLOAD];
  bool lv[NLOAD];
#pragma unroll
  for (int m = 0; m < NLOAD; ++m) {
    const int e = tid + m * NT, r = e / kGrSX, cl = e - r * kGrSX;
    lv[m] = e < kGrSP && gx0 + cl < c.d[0] && gy0 + r < c.d[1];
    soff[m] = e;
    goff[m] = (long long)(gy0 + r) * sy + gx0 + cl;
  }
  const int kend = k1 + 2;  // planes [k0 - 2, k1 + 2) are read
  auto slot_of = [&](int kp) { return (kp - k0) % kGrRing; };
  auto issue = [&](int kp) {
    if (kp < kend) {
      const uint32_t sb = rbase + (uint32_t)(slot_of(kp) * kGrArrays * kGrSP) * 4u;
#pragma unroll
      for (int m = 0; m < NLOAD; ++m) {
        if (!lv[m]) continue;
        const long long g = (long long)kp * sz + goff[m];
#pragma unroll
        for (int q = 0; q < kGrArrays; ++q)
          cp_async<4>(sb + (uint32_t)(q * kGrSP + soff[m]) * 4u, arr[q] + g);
      }
    }
    cp_async_commit();
  };
#pragma unroll 1
  for (int p = 0; p < 3 + kGrPF; ++p) issue(k0 + p);

  const int own = (ty + 2) * kGrSX + tx + 2;
  const long long ocol = (long long)j * sy + i;
  // window: w[s][q'] = array WQ[q'] at (i, j, k - 2 + s)
  float w[5][8];
  if (active) {
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2)
#pragma unroll
      for (int q = 0; q < 8; ++q) w[s2][q] = arr[WQ[q]][(long long)(k0 - 2 + s2) * sz + ocol];
  }
#pragma unroll 1
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<kGrPF>();  // planes up to k + 2 have landed
    __syncthreads();
    issue(k + 3 + kGrPF);    // into the slot of plane k - 1
    if (active) {
      const float* cs = ring + slot_of(k) * kGrArrays * kGrSP;
      const float* c2 = ring + slot_of(k + 2) * kGrArrays * kGrSP;
#pragma unroll
      for (int q = 0; q < 8; ++q) w[4][q] = c2[WQ[q] * kGrSP + own];
      auto fetch = [&](auto qc, auto ac, int n) -> float {
        constexpr int q = decltype(qc)::value, ax = decltype(ac)::value;
        if constexpr (ax == 2) return w[2 + n][gr_wslot<q>()];
        else if constexpr (ax == 0) return cs[q * kGrSP + own + n];
        else return cs[q * kGrSP + own + n * kGrSX];
      };
      auto ownv = [&](int q) { return cs[q * kGrSP + own]; };
      const float x = gr_pos(c, 0, i), y = gr_pos(c, 1, j), z = gr_pos(c, 2, k);
      auto metric = [&]() { return metric_at(c, mt, i, j, k, x, y, z); };
      gr_stage_point<float, FIRST>(c, metric, x, y, z, (long long)k * sz + ocol, fetch, ownv, out,
                                   du, un, aux, As, Bs, flags, ehout);
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2)
#pragma unroll
        for (int q = 0; q < 8; ++q) w[s2][q] = w[s2 + 1][q];
    }
  }
  cp_async_wait<0>();
}

// Kreiss-Oliger pass (kernel_KO_step1_gr / _step2_gr, :523-608, with the
// 3D 6th difference of finite_diff.h:84-92), then the clamps (:895-900).
template <typename T>
__global__ void __launch_bounds__(256) gr_ko_kernel(const __grid_constant__ GrConst<T> c,
                                                    const F7<T> u, const F7<T> out,
                                                    const T* __restrict__ mt,
                                                    const F7<T> ehout) {
  const int i = c.lo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = c.lo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = c.lo[2] + blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= c.hi[0] || j >= c.hi[1] || k >= c.hi[2]) return;
  const long long sy = c.d[0], sz = (long long)c.d[0] * c.d[1];
  const long long o = i + sy * j + sz * k;
  constexpr T K6[7] = {T(1), T(-6), T(15), T(-20), T(15), T(-6), T(1)};
  T v[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const T* f = u.p[a];
    T tx = T(0), ty = T(0), tz = T(0);
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      tx += K6[q] * __ldg(f + o + (q - 3));
      ty += K6[q] * __ldg(f + o + (q - 3) * sy);
      tz += K6[q] * __ldg(f + o + (q - 3) * sz);
    }
    v[a] = __ldg(f + o) + c.ko_c * (tx + ty + tz);
  }
  const Cks<T> m =
      metric_at(c, mt, i, j, k, gr_pos(c, 0, i), gr_pos(c, 1, j), gr_pos(c, 2, k));
  gr_clamps(c, m, v);
#pragma unroll
  for (int a = 0; a < 7; ++a) out.p[a][o] = v[a];
  if (ehout.p[0]) gr_eh_store(m, v, v + 3, ehout, o);
}

}  // namespace coffee
