// Kernels of the two 2D axisymmetric EZ solvers: log-spherical (x = ln r,
// y = theta; reference src/algorithms/field_solver_EZ_spherical.cu) and
// cylindrical (x = R, y = z; src/algorithms/field_solver_EZ_cylindrical.cu).
//
// Both run on one plane of (d0 x d1) points stored as the flat solver's
// arrays (i fastest).  A stage is one launch over the update box
// [guard - shift, dims - guard + shift) of axes 0 and 1 that reads the
// current buffer and writes the other one (the reference's rk_step1 ->
// rk_step2 -> clamps -> point boundaries, with no intermediate arrays), plus
// a small launch for the non-local axis boundary of the log-spherical
// solver.  These grids are small enough (a few million points) that the
// stencil neighbours of a warp are served from L1/L2; the kernels read
// global memory directly.
#pragma once

#include "coffee_b200.h"
#include "ez_common.cuh"

namespace coffee {

enum AxiFlags { AX_LAST = 1, AX_AUX = 2, AX_WRITE_UN = 4 };

// CTAs of 256 threads kept resident per SM (bounds the registers per thread;
// the kernels are latency-bound on their stencil loads, so more warps help,
// until spilling costs more).  Measured on 2048 x 1024 / 1024 x 2048 grids:
// the log-spherical kernels are fastest with 8 (32 registers), the
// cylindrical stage with 6 (40), the cylindrical KO with 4 (64); the
// batched log-spherical kernels (64 runs) with 4.
#ifndef COFFEE_SPH_MIN_BLOCKS
#define COFFEE_SPH_MIN_BLOCKS 8
#endif
#ifndef COFFEE_SPH_BATCH_MIN_BLOCKS
#define COFFEE_SPH_BATCH_MIN_BLOCKS 4
#endif
#ifndef COFFEE_CYL_STAGE_MIN_BLOCKS
#define COFFEE_CYL_STAGE_MIN_BLOCKS 6
#endif
#ifndef COFFEE_CYL_KO_MIN_BLOCKS
#define COFFEE_CYL_KO_MIN_BLOCKS 4
#endif
constexpr int kSphMinBlocks = COFFEE_SPH_MIN_BLOCKS;
constexpr int kSphBatchMinBlocks = COFFEE_SPH_BATCH_MIN_BLOCKS;
constexpr int kCylStageMinBlocks = COFFEE_CYL_STAGE_MIN_BLOCKS;
constexpr int kCylKoMinBlocks = COFFEE_CYL_KO_MIN_BLOCKS;

// Load of a field value.  NC: through the read-only data path (__ldg), for
// kernels in which nothing writes the array; otherwise a plain load, as the
// persistent batch kernel needs: it reads in one phase what other CTAs wrote
// in an earlier phase of the same launch, which the read-only path does not
// promise to see.
template <bool NC, typename T>
__device__ __forceinline__ T ldf(const T* p) {
  if constexpr (NC) return __ldg(p);
  else return *p;
}

// ---- parameter block of the log-spherical solver ------------------------
template <typename T>
struct SphConst {
  int d0, d1;
  int lo0, hi0, lo1, hi1;  // update box
  int axis_lo, axis_hi;    // theta = 0 / theta = pi rows, -1 if not on the grid
  int g0, g1;              // guards: x_i = x0 + dx * (i - g0), y_j = y0 + dy * (j - g1)
  T dx, dy, inv_dx, inv_dy, x0, y0;
  T dt, ch2, tau, gam_dt, ko_c;
  int calc_current, edotb, divB_clean, clean_ep, check_egb, ko_geometry;
  T radius, b0, omega;
  T tp_start, tp_end, dw0, nT, thp1, thp2;
  T tp_start1, tp_end1, dw1, nT1, thp11, thp21;
  int absorbing;
  T xh, rh, pmllen, sigpml;
  const T* rt;  // r_i = exp(x_i), i in [0, d0)
  const T* st;  // sin(theta_j), j in [0, d1)
  const T* ct;  // cos(theta_j)
};

// ---- parameter block of the cylindrical solver --------------------------
template <typename T>
struct CylConst {
  int d0, d1;
  int lo0, hi0, lo1, hi1;
  int axis_col;  // the R = 0 column, -1 if not on the grid
  int g0, g1;    // guards: R_i = R0 + dR * (i - g0), z_j = z0 + dz * (j - g1)
  T dR, dz, inv_dR, inv_dz, R0, z0;
  T dt, ch2, tau, ko_c;
  int clean_ep, check_egb;
  T radius, b0, omega;
  T tp_start, tp_end, dw0, th1, th2;  // wpert window in theta (precomputed)
  int absorbing;
  T xh, xl, yh, yl, pmlscale, sigpml;
};

template <typename T>
__device__ __forceinline__ T d1_4w(T a0, T a1, T a3, T a4) {
  // diff1_4 (src/algorithms/finite_diff.h:14-19)
  return (a0 - T(8) * a1 + T(8) * a3 - a4) * T(1.0 / 12.0);
}

// ---- log-spherical helpers ----------------------------------------------
// wpert_sph_angle (field_solver_EZ_spherical.cu:576-595)
template <typename T>
__device__ __noinline__ T sph_wpert_angle(T t, T th, T tp_start, T tp_end, T dw0, T nT, T thp1,
                                          T thp2) {
  if (thp1 > thp2) {
    const T tmp = thp1;
    thp1 = thp2;
    thp2 = tmp;
  }
  const T mu = (thp1 + thp2) * T(0.5);
  if (t >= tp_start && t <= tp_end && th >= thp1 && th <= thp2) {
    const double a = cos((double)(th - mu) * M_PI / (double)(thp2 - thp1));
    const double b = sin((double)(t - tp_start) * M_PI / (double)(tp_end - tp_start));
    const double c = sin((double)(t - tp_start) * 2.0 * M_PI * (double)nT /
                         (double)(tp_end - tp_start));
    return (T)((double)dw0 * (a * a) * (b * b) * c);
  }
  return T(0);
}

// Star surface and interior of the log-spherical run
// (kernel_boundary_pulsar_sph, field_solver_EZ_spherical.cu:617-688).
template <typename T>
__device__ __noinline__ V7<T> sph_pulsar(const SphConst<T>& c, V7<T> v, T r, T sn, T cs, T th,
                                         T t) {
  if (!(r < c.radius + c.dx)) return v;
  const T w = c.omega +
              sph_wpert_angle(t, th, c.tp_start, c.tp_end, c.dw0, c.nT, c.thp1, c.thp2) +
              sph_wpert_angle(t, th, c.tp_start1, c.tp_end1, c.dw1, c.nT1, c.thp11, c.thp21);
  const T r3 = r * r * r;
  const T bxn = c.b0 * (T(2) * cs / r3);
  const T byn = c.b0 * (sn / r3);
  const T v3n = w * r * sn;
  const T exn = v3n * byn;
  const T eyn = -v3n * bxn;
  const T g11s = r;  // sqrt(r^2)
  const T g22s = r;
  if (fabs(r - c.radius) < c.dx * T(0.5)) {
    v.v[3] = fdiv(bxn, g11s);
    v.v[1] = fdiv(eyn, g22s);
    v.v[2] = T(0);
  } else if (r < c.radius - Tiny<T>::v) {
    v.v[3] = fdiv(bxn, g11s);
    v.v[4] = fdiv(byn, g22s);
    v.v[5] = T(0);  // bzn / g33 with bzn = 0
    v.v[0] = fdiv(exn, g11s);
    v.v[1] = fdiv(eyn, g22s);
    v.v[2] = T(0);
  }
  return v;
}

// E.B = 0 and |E| <= |B| with the diagonal metric
// (kernel_Epar_sph / kernel_EgtB_sph, field_solver_EZ_spherical.cu:361-442).
template <typename T>
__device__ __forceinline__ void sph_clamps(const SphConst<T>& c, T* v, T g11, T g33) {
  if (c.clean_ep) {
    T B2 = g11 * v[3] * v[3] + g11 * v[4] * v[4] + g33 * v[5] * v[5];
    if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
    const T EB = g11 * v[0] * v[3] + g11 * v[1] * v[4] + g33 * v[2] * v[5];
    const T q = fdiv(EB, B2);
    v[0] -= q * v[3];
    v[1] -= q * v[4];
    v[2] -= q * v[5];
  }
  if (c.check_egb) {
    T B2 = g11 * v[3] * v[3] + g11 * v[4] * v[4] + g33 * v[5] * v[5];
    if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
    const T E2 = g11 * v[0] * v[0] + g11 * v[1] * v[1] + g33 * v[2] * v[2];
    if (E2 > B2) {
      const T s = sqrt(fdiv(B2, E2));
      v[0] *= s;
      v[1] *= s;
      v[2] *= s;
    }
  }
}

// Absorbing layer in r (kernel_boundary_absorbing_sph,
// field_solver_EZ_spherical.cu:758-802): blend towards the start-of-step
// values where x > xh.
template <typename T>
__device__ __noinline__ V7<T> sph_absorb(const SphConst<T>& c, V7<T> v, V7<T> n, T x, T r) {
  if (!(x > c.xh)) return v;
  T sig = T(0);
  if (r > c.rh) {
    const T q = (r - c.rh) / c.pmllen;
    sig = c.sigpml * q * q * q;
  }
  if (sig > Tiny<T>::v) {
    const T e = exp(-sig);
    const T f = (T(1) - e) / sig;
    for (int a = 0; a < 6; ++a) v.v[a] = e * n.v[a] + f * (v.v[a] - n.v[a]);
  }
  return v;
}

// One LSRK stage of the log-spherical solver at point (i, j):
// kernel_compute_ElBl + kernel_rk_step1_sph + kernel_rk_step2_sph, then
// kernel_Epar_sph, kernel_EgtB_sph, kernel_boundary_pulsar_sph and, in the
// last stage, kernel_boundary_absorbing_sph (field_solver_EZ_spherical.cu:
// 175-802, order of :967-990).  FIRST: As = 0, dU is not read.  NC: field
// loads through the read-only path (ldf).
template <typename T, bool FIRST, bool NC = true>
__device__ __forceinline__ void sph_stage_point(const SphConst<T>& c, const int i, const int j,
                                                const F7<T>& u, const F7<T>& out,
                                                const F7<T>& du, const F7<T>& un,
                                                const F5<T>& aux, const T As, const T Bs,
                                                const T tst, const int flags) {
  const long long d0 = c.d0;
  const long long o = i + j * d0;
  T r[5], sn[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    r[k] = __ldg(c.rt + i - 2 + k);
    sn[k] = __ldg(c.st + j - 2 + k);
  }
  const T rc = r[2], sc = sn[2];
  const T g11 = rc * rc;
  const T g33 = (rc * sc) * (rc * sc);
  T gms = rc * rc * rc * fabs(sc);
  if (gms < Tiny<T>::v) gms = Tiny<T>::v;
  const T igms = T(1) / gms;

  const T* Ex = u.p[0];
  const T* Ey = u.p[1];
  const T* Ez = u.p[2];
  const T* Bx = u.p[3];
  const T* By = u.p[4];
  const T* Bz = u.p[5];
  const T* P = u.p[6];
  auto X = [&](const T* f, int k) { return ldf<NC>(f + o + (k - 2)); };
  auto Y = [&](const T* f, int k) { return ldf<NC>(f + o + (k - 2) * d0); };

  // lowered fields at the stencil points: El_x = r^2 E_x, El_y = r^2 E_y,
  // El_z = (r sin th)^2 E_z (metric_sph.h:90-122)
  auto g33x = [&](int k) { return (r[k] * sc) * (r[k] * sc); };
  auto g33y = [&](int k) { return (rc * sn[k]) * (rc * sn[k]); };
  const T idx12 = c.inv_dx, idy12 = c.inv_dy;
  auto dX = [&](auto fn) { return d1_4w(fn(0), fn(1), fn(3), fn(4)) * idx12; };
  auto dY = [&](auto fn) { return d1_4w(fn(0), fn(1), fn(3), fn(4)) * idy12; };

  const T rotBx = dY([&](int k) { return g33y(k) * Y(Bz, k); }) * igms;
  const T rotEx = dY([&](int k) { return g33y(k) * Y(Ez, k); }) * igms;
  const T rotBy = -dX([&](int k) { return g33x(k) * X(Bz, k); }) * igms;
  const T rotEy = -dX([&](int k) { return g33x(k) * X(Ez, k); }) * igms;
  const T rotBz = (dX([&](int k) { return r[k] * r[k] * X(By, k); }) -
                   dY([&](int k) { return g11 * Y(Bx, k); })) * igms;
  const T rotEz = (dX([&](int k) { return r[k] * r[k] * X(Ey, k); }) -
                   dY([&](int k) { return g11 * Y(Ex, k); })) * igms;
  // div4_sph (field_solver_EZ_spherical.cu:99-124): sqrt(gamma) = r^3 |sin th|
  const T asc = fabs(sc);
  auto sgx = [&](int k) { return r[k] * r[k] * r[k] * asc; };
  auto sgy = [&](int k) { return rc * rc * rc * fabs(sn[k]); };
  const T divE = (dX([&](int k) { return X(Ex, k) * sgx(k); }) +
                  dY([&](int k) { return Y(Ey, k) * sgy(k); })) * igms;
  const T divB = (dX([&](int k) { return X(Bx, k) * sgx(k); }) +
                  dY([&](int k) { return Y(By, k) * sgy(k); })) * igms;

  T v[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) v[a] = ldf<NC>(u.p[a] + o);
  const T el[3] = {g11 * v[0], g11 * v[1], g33 * v[2]};
  const T bl[3] = {g11 * v[3], g11 * v[4], g33 * v[5]};
  T B2 = v[3] * bl[0] + v[4] * bl[1] + v[5] * bl[2];
  if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
  T J[3] = {T(0), T(0), T(0)};
  if (c.calc_current) {
    T Jp = (bl[0] * rotBx + bl[1] * rotBy + bl[2] * rotBz) -
           (el[0] * rotEx + el[1] * rotEy + el[2] * rotEz);
    const T cx = el[1] * bl[2] - el[2] * bl[1];
    const T cy = el[2] * bl[0] - el[0] * bl[2];
    const T cz = el[0] * bl[1] - el[1] * bl[0];
    if (c.edotb) {
      const T E2 = v[0] * el[0] + v[1] * el[1] + v[2] * el[2];
      const T chi2 = B2 - E2;
      const T EdotB = v[0] * bl[0] + v[1] * bl[1] + v[2] * bl[2];
      const T E02 = T(0.5) * (sqrt(chi2 * chi2 + T(4) * EdotB * EdotB) - chi2);
      Jp += c.gam_dt * EdotB;
      const T a = fdiv(divE * igms, E02 + B2);
      const T q = fdiv(Jp, B2);
      J[0] = a * cx + q * v[3];
      J[1] = a * cy + q * v[4];
      J[2] = a * cz + q * v[5];
    } else {
      const T iB2 = fdiv(T(1), B2);
      J[0] = (divE * cx * igms + Jp * v[3]) * iB2;
      J[1] = (divE * cy * igms + Jp * v[4]) * iB2;
      J[2] = (divE * cz * igms + Jp * v[5]) * iB2;
    }
  }
  T Px = T(0), Py = T(0);
  if (c.divB_clean) {
    Px = fdiv(dX([&](int k) { return X(P, k); }), g11);
    Py = fdiv(dY([&](int k) { return Y(P, k); }), g11);
    // Pz = dfdz(P) / gamma_33 with dfdz = 0; the reference's 0/0 on the
    // theta = 0 row only reaches dB_z of that row, which the axis
    // boundary overwrites.
  }
  const T dt = c.dt;
  T rhs[7];
  rhs[0] = dt * (rotBx - J[0]);
  rhs[1] = dt * (rotBy - J[1]);
  rhs[2] = dt * (rotBz - J[2]);
  rhs[3] = -dt * (rotEx + Px);
  rhs[4] = -dt * (rotEy + Py);
  rhs[5] = -dt * rotEz;
  rhs[6] = -dt * c.ch2 * divB - v[6] / c.tau;

  if (flags & AX_WRITE_UN) {
#pragma unroll
    for (int a = 0; a < 6; ++a) un.p[a][o] = v[a];
  }
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const T d = FIRST ? rhs[a] : As * du.p[a][o] + rhs[a];
    du.p[a][o] = d;
    v[a] += Bs * d;
  }
  if (flags & AX_AUX) {
    aux.p[0][o] = J[0];
    aux.p[1][o] = J[1];
    aux.p[2][o] = J[2];
    aux.p[3][o] = divE;
    aux.p[4][o] = divB;
  }
  sph_clamps(c, v, g11, g33);
  V7<T> w;
#pragma unroll
  for (int a = 0; a < 7; ++a) w.v[a] = v[a];
  // the out-of-line boundary code is entered only where it can act
  if (rc < c.radius + c.dx) {
    const T th = c.y0 + c.dy * (T)(j - c.g1);
    w = sph_pulsar(c, w, rc, sc, __ldg(c.ct + j), th, tst);
  }
  const T xi = c.x0 + c.dx * (T)(i - c.g0);
  if ((flags & AX_LAST) && c.absorbing && xi > c.xh) {
    V7<T> n;
#pragma unroll
    for (int a = 0; a < 6; ++a) n.v[a] = un.p[a][o];
    n.v[6] = T(0);
    w = sph_absorb(c, w, n, xi, rc);
  }
#pragma unroll
  for (int a = 0; a < 7; ++a) out.p[a][o] = w.v[a];
}

template <typename T, bool FIRST>
__global__ void __launch_bounds__(256, kSphMinBlocks) sph_stage_kernel(const __grid_constant__ SphConst<T> c,
                                                        const F7<T> u, const F7<T> out,
                                                        const F7<T> du, const F7<T> un,
                                                        const F5<T> aux, const T As,
                                                        const T Bs, const T tst,
                                                        const int flags) {
  const int i = c.lo0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = c.lo1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= c.hi0 || j >= c.hi1) return;
  sph_stage_point<T, FIRST>(c, i, j, u, out, du, un, aux, As, Bs, tst, flags);
}

// Kreiss-Oliger pass of the log-spherical solver at point (i, j):
// kernel_KO_step1_sph + kernel_KO_step2_sph, then kernel_Epar_sph,
// kernel_EgtB_sph and kernel_boundary_pulsar_sph at t + dt
// (field_solver_EZ_spherical.cu:444-555, order of :996-1004).  KO_geometry
// weights the 6th differences by sqrt(gamma) (KO_2d6, :150-173), otherwise
// they are plain (KO_2d0, :142-148).  NC as for sph_stage_point.
template <typename T, bool NC = true>
__device__ __forceinline__ void sph_ko_point(const SphConst<T>& c, const int i, const int j,
                                             const F7<T>& u, const F7<T>& out, const T tend) {
  const long long d0 = c.d0;
  const long long o = i + j * d0;
  constexpr T K6[7] = {T(1), T(-6), T(15), T(-20), T(15), T(-6), T(1)};
  T wx[7], wy[7];
  const T rc = __ldg(c.rt + i), sc = __ldg(c.st + j);
  T gms = rc * rc * rc * fabs(sc);
  if (gms < Tiny<T>::v) gms = Tiny<T>::v;
  if (c.ko_geometry) {  // sqrt(gamma) at the stencil points
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const T rk = __ldg(c.rt + i - 3 + k);
      wx[k] = K6[k] * (rk * rk * rk * fabs(sc));
      wy[k] = K6[k] * (rc * rc * rc * fabs(__ldg(c.st + j - 3 + k)));
    }
  } else {
#pragma unroll
    for (int k = 0; k < 7; ++k) wx[k] = wy[k] = K6[k];
  }
  T v[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const T* f = u.p[a];
    T tx = T(0), ty = T(0);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      tx += wx[k] * ldf<NC>(f + o + (k - 3));
      ty += wy[k] * ldf<NC>(f + o + (k - 3) * d0);
    }
    T t = tx + ty;
    if (c.ko_geometry) t = t / gms;
    v[a] = ldf<NC>(f + o) + c.ko_c * t;
  }
  sph_clamps(c, v, rc * rc, (rc * sc) * (rc * sc));
  V7<T> w;
#pragma unroll
  for (int a = 0; a < 7; ++a) w.v[a] = v[a];
  if (rc < c.radius + c.dx)
    w = sph_pulsar(c, w, rc, sc, __ldg(c.ct + j), c.y0 + c.dy * (T)(j - c.g1), tend);
#pragma unroll
  for (int a = 0; a < 7; ++a) out.p[a][o] = w.v[a];
}

template <typename T>
__global__ void __launch_bounds__(256, kSphMinBlocks) sph_ko_kernel(const __grid_constant__ SphConst<T> c,
                                                     const F7<T> u, const F7<T> out,
                                                     const T tend) {
  const int i = c.lo0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = c.lo1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= c.hi0 || j >= c.hi1) return;
  sph_ko_point(c, i, j, u, out, tend);
}

// Axis boundary of the log-spherical solver at column i
// (kernel_boundary_axis_sph, field_solver_EZ_spherical.cu:690-748): on the
// theta = 0 row E_r, B_r, P take the next row's values and the other
// components vanish; the three rows beyond the axis mirror the rows inside
// with the parity of each component.  The theta = pi row (the first guard
// row) likewise.
template <typename T>
__device__ __forceinline__ void sph_axis_column(const SphConst<T>& c, const int i,
                                                const F7<T>& u) {
  const long long d0 = c.d0;
  constexpr T par[6] = {T(1), T(-1), T(-1), T(1), T(-1), T(-1)};
  for (int side = 0; side < 2; ++side) {
    const int j = side == 0 ? c.axis_lo : c.axis_hi;
    if (j < 0) continue;
    const int in = side == 0 ? 1 : -1;  // direction of the rows inside
    const long long o = i + j * d0;
    u.p[0][o] = u.p[0][o + in * d0];
    u.p[1][o] = T(0);
    u.p[2][o] = T(0);
    u.p[3][o] = u.p[3][o + in * d0];
    u.p[4][o] = T(0);
    u.p[5][o] = T(0);
    u.p[6][o] = u.p[6][o + in * d0];
    for (int l = 1; l <= 3; ++l)
#pragma unroll
      for (int a = 0; a < 6; ++a) u.p[a][o - in * l * d0] = par[a] * u.p[a][o + in * l * d0];
  }
}

template <typename T>
__global__ void sph_axis_kernel(const __grid_constant__ SphConst<T> c, const F7<T> u) {
  const int i = c.lo0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.hi0) return;
  sph_axis_column(c, i, u);
}

// ---- batches of independent log-spherical runs ---------------------------
// One launch per phase covers every run of a batch: block b belongs to the
// run whose first block index is the largest one <= b.  The run's table
// entry (parameters and array pointers) is copied to shared memory, then the
// threads proceed exactly as the single-run kernels do.
constexpr int kSphBatchMax = 128;

template <typename T>
struct SphBatchEntry {
  SphConst<T> c;
  F7<T> A, B, dU, Un;
  F5<T> aux;
  int tile0;    // first stage/KO block of this run
  int tiles_x;  // blocks along i
  int axis0;    // first axis block of this run
  int want_aux;
  int index;    // position in the batch
};

// Times of the runs of a batch live in device memory (the current step's
// start time t and the time step dt of each run), so that one captured step
// serves every step.  A stage at t + cs dt evaluates that time exactly as the
// host loop of a single run does, in field precision with one rounding per
// operation (no fused multiply-add).
__device__ __forceinline__ float batch_time(float t, float cs, float dt) {
  return __fadd_rn(t, __fmul_rn(cs, dt));
}
__device__ __forceinline__ double batch_time(double t, double cs, double dt) {
  return __dadd_rn(t, __dmul_rn(cs, dt));
}

template <typename T>
__device__ __forceinline__ const SphBatchEntry<T>& sph_batch_entry(
    const SphBatchEntry<T>* __restrict__ tab, int n, int b, bool axis, unsigned char* buf) {
  __shared__ int m_s;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nt = blockDim.x * blockDim.y;
  if (tid == 0) {
    int lo = 0, hi = n - 1;  // largest m with start(m) <= b
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      const int st = axis ? tab[mid].axis0 : tab[mid].tile0;
      if (st <= b) lo = mid;
      else hi = mid - 1;
    }
    m_s = lo;
  }
  __syncthreads();
  const int* src = reinterpret_cast<const int*>(tab + m_s);
  int* dst = reinterpret_cast<int*>(buf);
  for (int q = tid; q < (int)(sizeof(SphBatchEntry<T>) / 4); q += nt) dst[q] = src[q];
  __syncthreads();
  return *reinterpret_cast<const SphBatchEntry<T>*>(buf);
}

template <typename T, bool FIRST>
__global__ void __launch_bounds__(256, kSphBatchMinBlocks) sph_stage_batch_kernel(
    const SphBatchEntry<T>* __restrict__ tab, const int n, const int to_b,
    const T* __restrict__ tnow, const T* __restrict__ tdt, const T cs, const T As, const T Bs,
    const int last) {
  __shared__ __align__(16) unsigned char buf[sizeof(SphBatchEntry<T>)];
  const SphBatchEntry<T>& e = sph_batch_entry(tab, n, (int)blockIdx.x, false, buf);
  const int lt = (int)blockIdx.x - e.tile0;
  const int i = e.c.lo0 + (lt % e.tiles_x) * blockDim.x + threadIdx.x;
  const int j = e.c.lo1 + (lt / e.tiles_x) * blockDim.y + threadIdx.y;
  if (i >= e.c.hi0 || j >= e.c.hi1) return;
  int flags = 0;
  if (last) flags |= AX_LAST | (e.want_aux ? AX_AUX : 0);
  if (FIRST && e.c.absorbing) flags |= AX_WRITE_UN;
  const T tst = batch_time(tnow[e.index], cs, tdt[e.index]);
  sph_stage_point<T, FIRST>(e.c, i, j, to_b ? e.A : e.B, to_b ? e.B : e.A, e.dU, e.Un, e.aux,
                            As, Bs, tst, flags);
}

template <typename T>
__global__ void __launch_bounds__(256, kSphBatchMinBlocks) sph_ko_batch_kernel(
    const SphBatchEntry<T>* __restrict__ tab, const int n, const T* __restrict__ tnow,
    const T* __restrict__ tdt) {
  __shared__ __align__(16) unsigned char buf[sizeof(SphBatchEntry<T>)];
  const SphBatchEntry<T>& e = sph_batch_entry(tab, n, (int)blockIdx.x, false, buf);
  const int lt = (int)blockIdx.x - e.tile0;
  const int i = e.c.lo0 + (lt % e.tiles_x) * blockDim.x + threadIdx.x;
  const int j = e.c.lo1 + (lt / e.tiles_x) * blockDim.y + threadIdx.y;
  if (i >= e.c.hi0 || j >= e.c.hi1) return;
  sph_ko_point(e.c, i, j, e.B, e.A, batch_time(tnow[e.index], T(1), tdt[e.index]));
}

// end of a step: t += dt for every run, in field precision
template <typename T>
__global__ void sph_batch_advance_kernel(T* __restrict__ tnow, const T* __restrict__ tdt,
                                         const int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) tnow[m] = batch_time(tnow[m], T(1), tdt[m]);
}

// axis boundary of every run; `on_b`: the buffer that was just written
template <typename T>
__global__ void sph_axis_batch_kernel(const SphBatchEntry<T>* __restrict__ tab, const int n,
                                      const int on_b) {
  __shared__ __align__(16) unsigned char buf[sizeof(SphBatchEntry<T>)];
  const SphBatchEntry<T>& e = sph_batch_entry(tab, n, (int)blockIdx.x, true, buf);
  if (e.c.axis_lo < 0 && e.c.axis_hi < 0) return;
  const int i = e.c.lo0 + ((int)blockIdx.x - e.axis0) * blockDim.x + threadIdx.x;
  if (i >= e.c.hi0) return;
  sph_axis_column(e.c, i, on_b ? e.B : e.A);
}

// ---- the whole batch step in one persistent launch ----------------------
// One cooperative launch (every CTA resident) runs nsteps steps of every run
// of a batch: the phases of the per-phase launches (5 x (stage, axis), KO,
// axis), each over all runs, separated by grid-wide barriers.  In a stage or
// KO phase the CTAs take kTicketTiles tiles at a time from a ticket counter
// (the tiles differ in cost: star and absorbing-layer points), asking for
// the next ticket before working on the current one; the axis phases are
// split evenly.  On each tile a CTA runs the single-run per-point code, so
// the results are bitwise those of the per-phase launches.  The run times alternate between two
// rows of `tbuf`: during step s the stages read row s & 1 and CTA 0 writes
// t + dt into the other row, which the next step reads after the
// barriers between.
//
// Every barrier wait is bounded, by `limit_ns` of %globaltimer and by an
// iteration cap: a CTA that gives up records COFFEE_E_TIMEOUT, the barrier
// and its block in GridSync and returns, and the CTAs still waiting see the
// status and return as well, so the launch always ends.
struct GridSync {
  unsigned int count;  // arrivals so far (barrier q completes at (q + 1) * gridDim.x)
  int status;          // 0, or COFFEE_E_TIMEOUT once a wait has run out
  int where;           // index of the barrier that ran out
  int block;           // the CTA whose wait ran out first
  unsigned int tickets[2];  // tile tickets of the stage / KO phases (alternating)
};
// Tiles a CTA takes per ticket in the stage and KO phases.
constexpr int kTicketTiles = 4;
// Phase coefficients of the LSRK stages.
template <typename T>
struct LsrkCoef {
  T As[5], Bs[5], Cs[5];
};

__device__ __forceinline__ long long globaltimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier number q (0, 1, ...).  `arrive` = false leaves this
// CTA's arrival out (the stalled-CTA test of the wait limit).  Returns
// false when the barrier gave up.
__device__ __forceinline__ bool grid_barrier(GridSync* gs, unsigned q, long long limit_ns,
                                             bool arrive) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    int ok = 1;
    if (arrive) {
      __threadfence();  // this CTA's writes, seen by thread 0 through the barrier above
      atomicAdd(&gs->count, 1u);
    }
    const unsigned target = (q + 1u) * gridDim.x;
    const long long t0 = globaltimer_ns();
    const long long cap = limit_ns / 32 + 4096;  // iterations, should the timer stall
    for (long long it = 0;; ++it) {
      unsigned c;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(&gs->count) : "memory");
      if (c >= target) break;
      if (*(volatile int*)&gs->status != 0) {
        ok = 0;
        break;
      }
      if (it >= cap || globaltimer_ns() - t0 > limit_ns) {
        if (atomicCAS(&gs->status, 0, (int)COFFEE_E_TIMEOUT) == 0) {
          gs->where = (int)q;
          gs->block = (int)blockIdx.x;
        }
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

template <typename T>
__global__ void __launch_bounds__(256, kSphBatchMinBlocks) sph_batch_persistent_kernel(
    const SphBatchEntry<T>* __restrict__ tab, const int n, const int nblocks, const int naxis,
    T* __restrict__ tbuf, const T* __restrict__ tdt, const LsrkCoef<T> k, const int nsteps,
    GridSync* __restrict__ gs, const long long limit_ns, const int stall_block) {
  __shared__ __align__(16) unsigned char buf[sizeof(SphBatchEntry<T>)];
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nt = blockDim.x * blockDim.y;
  unsigned q = 0;  // barriers passed
  auto barrier = [&]() {
    const bool arrive = !(q == 0 && (int)blockIdx.x == stall_block);
    return grid_barrier(gs, q++, limit_ns, arrive);
  };
  // one stage (s = 0..4) or, for s = 5, the KO pass, over every tile
  __shared__ unsigned base_s;
  unsigned tp = 0;  // tile phases begun
  auto tiles = [&](const int s, const T* tcur) {
    // tile phase tp takes its tickets from counter tp & 1; the other
    // counter, last used by the tile phase before (finished at a barrier
    // before this one began), is cleared for the next
    unsigned* ctr = &gs->tickets[tp & 1];
    if (blockIdx.x == 0 && tid == 0) gs->tickets[(tp + 1) & 1] = 0u;
    ++tp;
    if (tid == 0) base_s = atomicAdd(ctr, (unsigned)kTicketTiles);
    __syncthreads();
    unsigned base = base_s;
    while (base < (unsigned)nblocks) {
      unsigned pending = 0;
      if (tid == 0) pending = atomicAdd(ctr, (unsigned)kTicketTiles);  // used after the tiles
      const int bend = min((int)base + kTicketTiles, nblocks);
      for (int b = (int)base; b < bend; ++b) {
        const SphBatchEntry<T>& e = sph_batch_entry(tab, n, b, false, buf);
        const int lt = b - e.tile0;
        const int i = e.c.lo0 + (lt % e.tiles_x) * blockDim.x + threadIdx.x;
        const int j = e.c.lo1 + (lt / e.tiles_x) * blockDim.y + threadIdx.y;
        if (i < e.c.hi0 && j < e.c.hi1) {
          if (s == 5) {
            sph_ko_point<T, false>(e.c, i, j, e.B, e.A,
                                   batch_time(tcur[e.index], T(1), tdt[e.index]));
          } else {
            const int to_b = (s % 2 == 0) ? 1 : 0;
            int flags = 0;
            if (s == 4) flags |= AX_LAST | (e.want_aux ? AX_AUX : 0);
            if (s == 0 && e.c.absorbing) flags |= AX_WRITE_UN;
            const T tst = batch_time(tcur[e.index], k.Cs[s], tdt[e.index]);
            if (s == 0)
              sph_stage_point<T, true, false>(e.c, i, j, e.A, e.B, e.dU, e.Un, e.aux, k.As[0],
                                              k.Bs[0], tst, flags);
            else
              sph_stage_point<T, false, false>(e.c, i, j, to_b ? e.A : e.B, to_b ? e.B : e.A,
                                               e.dU, e.Un, e.aux, k.As[s], k.Bs[s], tst, flags);
          }
        }
        __syncthreads();  // buf is refilled for the next tile
      }
      if (tid == 0) base_s = pending;
      __syncthreads();
      base = base_s;
    }
  };
  // the axis boundary of every run on buffer B (on_b) or A, 128 columns a tile
  auto axis = [&](const int on_b) {
    for (int b = blockIdx.x; b < naxis; b += gridDim.x) {
      const SphBatchEntry<T>& e = sph_batch_entry(tab, n, b, true, buf);
      if ((e.c.axis_lo >= 0 || e.c.axis_hi >= 0) && tid < 128) {
        const int i = e.c.lo0 + (b - e.axis0) * 128 + tid;
        if (i < e.c.hi0) sph_axis_column(e.c, i, on_b ? e.B : e.A);
      }
      __syncthreads();
    }
  };
  for (int step = 0; step < nsteps; ++step) {
    const T* tcur = tbuf + (step & 1) * n;
    if (blockIdx.x == 0)
      for (int m = tid; m < n; m += nt)
        tbuf[((step + 1) & 1) * n + m] = batch_time(tcur[m], T(1), tdt[m]);
    for (int s = 0; s < 5; ++s) {
      tiles(s, tcur);
      if (!barrier()) return;
      axis((s % 2 == 0) ? 1 : 0);
      if (!barrier()) return;
    }
    tiles(5, tcur);
    if (!barrier()) return;
    axis(0);
    if (!barrier()) return;
  }
}

// ---- cylindrical helpers ------------------------------------------------
// shape (src/algorithms/pulsar_impl.hpp:52-55)
template <typename T>
__device__ __forceinline__ T cyl_shape(T r, T r0, T del) {
  return T(0.5) * (T(1) - tanh((r - r0) / del));
}

// wpert of the cylindrical run (field_solver_EZ_cylindrical.cu:413-443); the
// angular window [th1, th2] = acos(sqrt(1 - 1/rpert)) is precomputed.
template <typename T>
__device__ __noinline__ T cyl_wpert(const CylConst<T>& c, T t, T R, T z) {
  const T r = sqrt(R * R + z * z);
  const T th = acos(z / r);  // NaN at the origin: no perturbation there
  const T mu = (c.th1 + c.th2) * T(0.5);
  const T s = (mu - c.th1) / T(3);
  if (t >= c.tp_start && t <= c.tp_end && th >= c.th1 && th <= c.th2) {
    const T q = (th - mu) / s;
    return c.dw0 * exp(T(-0.5) * q * q) *
           (T)sin((double)(t - c.tp_start) * 2.0 * M_PI / (double)(c.tp_end - c.tp_start)) *
           T(0.5) * (T(1) + tanh((r - T(0.5) * c.radius) / (T(0.05) * c.radius)));
  }
  return T(0);
}

// Rotating dipole star blended in over r < 2 R (kernel_boundary_pulsar_thread,
// field_solver_EZ_cylindrical.cu:445-530).  Components: 0 E_R, 1 E_z,
// 2 E_phi, 3 B_R, 4 B_z, 5 B_phi.
template <typename T>
__device__ __noinline__ V7<T> cyl_pulsar(const CylConst<T>& c, V7<T> v, T R, T z, T t) {
  T r2 = R * R + z * z;
  if (r2 < Tiny<T>::v) r2 = Tiny<T>::v;
  const T r = sqrt(r2);
  if (!(r < T(2) * c.radius)) return v;
  const T ri = T(0.5) * c.radius;
  const T sEpar = T(0.5) * c.dR, sEperp = T(0.25) * c.dR;
  const T sB = sEpar;
  const T d1 = T(4) * c.dR;
  // dipole_x / dipole_z (pulsar_impl.hpp:10-50) with alpha = phase = 0
  T rr = sqrt(R * R + z * z);
  if (fabs(rr) < Tiny<T>::v) rr = Tiny<T>::v;
  const T xn = R / rr, zn = z / rr;
  const T rr3 = rr * rr * rr + Tiny<T>::v;
  const T m3 = c.b0 * c.radius * c.radius * c.radius;
  const T bRn = m3 * ((T(3) * xn * zn) / rr3);
  const T bzn = m3 * ((T(3) * zn * zn - T(1)) / rr3);
  const T bfn = T(0);
  const T BR = v.v[3], Bz = v.v[4], Bf = v.v[5];
  const T ER = v.v[0], Ez = v.v[1], Ef = v.v[2];
  const T bnp = bRn * R + bzn * z, bp = BR * R + Bz * z;
  T s = cyl_shape(r, c.radius - d1, sB);
  T BRn = bnp * R / r2 * s + bp * R / r2 * (T(1) - s);
  T Bzn = bnp * z / r2 * s + bp * z / r2 * (T(1) - s);
  BRn += (bRn - bnp * R / r2) * s + (BR - bp * R / r2) * (T(1) - s);
  Bzn += (bzn - bnp * z / r2) * s + (Bz - bp * z / r2) * (T(1) - s);
  const T Bfn = bfn * s + Bf * (T(1) - s);
  const T w = c.omega + cyl_wpert(c, t, R, z);
  const T eRn = -w * R * Bz;
  const T ezn = w * R * BR;
  const T efn = T(0);
  const T enp = eRn * R + ezn * z, ep = ER * R + Ez * z;
  s = cyl_shape(r, c.radius, sEperp);
  T ERn = enp * R / r2 * s + ep * R / r2 * (T(1) - s);
  T Ezn = enp * z / (r * r) * s + ep * z / r2 * (T(1) - s);
  s = cyl_shape(r, c.radius, sEpar);
  ERn += (eRn - enp * R / r2) * s + (ER - ep * R / r2) * (T(1) - s);
  Ezn += (ezn - enp * z / r2) * s + (Ez - ep * z / r2) * (T(1) - s);
  const T Efn = efn * s + Ef * (T(1) - s);
  if (r < ri) {
    v.v[3] = bRn; v.v[4] = bzn; v.v[5] = bfn;
    v.v[0] = eRn; v.v[1] = ezn; v.v[2] = efn;
  } else {
    v.v[3] = BRn; v.v[4] = Bzn; v.v[5] = Bfn;
    v.v[0] = ERn; v.v[1] = Ezn; v.v[2] = Efn;
  }
  return v;
}

// pmlsigma (src/algorithms/boundary.cu:7-15)
template <typename T>
__device__ __forceinline__ T cyl_pmlsigma(T x, T xl, T xh, T scale, T sig0) {
  if (x > xh) {
    const T q = (x - xh) / scale;
    return sig0 * q * q * q;
  }
  if (x < xl) {
    const T q = (xl - x) / scale;
    return sig0 * q * q * q;
  }
  return T(0);
}

// Absorbing layer at large R and both z ends
// (kernel_boundary_absorbing_cylindrical, field_solver_EZ_cylindrical.cu:532-591).
template <typename T>
__device__ __noinline__ V7<T> cyl_absorb(const CylConst<T>& c, V7<T> v, V7<T> n, T R, T z) {
  if (!(R > c.xh || z < c.yl || z > c.yh)) return v;
  const T sig = cyl_pmlsigma(R, c.xl, c.xh, c.pmlscale, c.sigpml) +
                cyl_pmlsigma(z, c.yl, c.yh, c.pmlscale, c.sigpml);
  if (sig > Tiny<T>::v) {
    const T e = exp(-sig);
    const T f = (T(1) - e) / sig;
    for (int a = 0; a < 6; ++a) v.v[a] = e * n.v[a] + f * (v.v[a] - n.v[a]);
  }
  return v;
}

// kernel_Epar_thread / kernel_EgtB_thread (field_solver_EZ_cylindrical.cu:236-294)
template <typename T>
__device__ __forceinline__ void cyl_clamps(const CylConst<T>& c, T* v) {
  if (c.clean_ep) {
    T B2 = v[3] * v[3] + v[4] * v[4] + v[5] * v[5];
    if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
    const T q = fdiv(v[0] * v[3] + v[1] * v[4] + v[2] * v[5], B2);
    v[0] -= q * v[3];
    v[1] -= q * v[4];
    v[2] -= q * v[5];
  }
  if (c.check_egb) {
    T B2 = v[3] * v[3] + v[4] * v[4] + v[5] * v[5];
    if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
    const T E2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (E2 > B2) {
      const T s = sqrt(fdiv(B2, E2));
      v[0] *= s;
      v[1] *= s;
      v[2] *= s;
    }
  }
}

// The point boundaries that follow the clamps in a cylindrical stage, in the
// reference's order (field_solver_EZ_cylindrical.cu:688-700): the axis
// boundary (kernel_boundary_axis_thread, :371-411), the star at time t and,
// in the last stage, the absorbing layer.  v holds this point's values after
// the clamps.  The axis boundary copies values of the three columns next to
// the axis before the star is applied to them, so the threads of those
// columns write the mirror columns (and the one next to the axis also the
// axis column, which it then passes through the star and the layer); the
// thread of the axis column itself writes nothing.
template <typename T>
__device__ __forceinline__ void cyl_finish(const CylConst<T>& c, int i, int j, long long o,
                                          const T* v, const F7<T>& out, const F7<T>& un,
                                          T t, bool last) {
  const T z = c.z0 + c.dz * (T)(j - c.g1);
  auto bc = [&](V7<T> w, long long p, T R) {
    // the out-of-line boundary code is entered only where it can act
    if (R * R + z * z < T(4) * c.radius * c.radius + Tiny<T>::v) w = cyl_pulsar(c, w, R, z, t);
    if (last && c.absorbing && (R > c.xh || z < c.yl || z > c.yh)) {
      V7<T> n;
      for (int a = 0; a < 6; ++a) n.v[a] = un.p[a][p];
      n.v[6] = T(0);
      w = cyl_absorb(c, w, n, R, z);
    }
    for (int a = 0; a < 7; ++a) out.p[a][p] = w.v[a];
  };
  const int da = c.axis_col >= 0 ? i - c.axis_col : -1;
  if (da == 0) return;
  if (da >= 1 && da <= 3) {
    // mirror column axis - da: E_z, B_z, P even, the rest odd
    constexpr T par[7] = {T(-1), T(1), T(-1), T(-1), T(1), T(-1), T(1)};
    const long long m = o - 2 * da;
    for (int a = 0; a < 7; ++a) out.p[a][m] = par[a] * v[a];
    if (da == 1) {
      V7<T> w;
      w.v[0] = T(0); w.v[1] = v[1]; w.v[2] = T(0);
      w.v[3] = T(0); w.v[4] = v[4]; w.v[5] = T(0);
      w.v[6] = v[6];
      bc(w, o - 1, c.R0 + c.dR * (T)(c.axis_col - c.g0));
    }
  }
  V7<T> w;
  for (int a = 0; a < 7; ++a) w.v[a] = v[a];
  bc(w, o, c.R0 + c.dR * (T)(i - c.g0));
}

// One LSRK stage of the cylindrical solver: kernel_rk_step1_thread +
// kernel_rk_step2_thread, the clamps, then cyl_finish
// (field_solver_EZ_cylindrical.cu:143-234, 674-703).  The reference's
// cylindrical stage writes no J / divE / divB.
template <typename T, bool FIRST>
__global__ void __launch_bounds__(256, kCylStageMinBlocks) cyl_stage_kernel(const __grid_constant__ CylConst<T> c,
                                                        const F7<T> u, const F7<T> out,
                                                        const F7<T> du, const F7<T> un,
                                                        const T As, const T Bs, const T tst,
                                                        const int flags) {
  const int i = c.lo0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = c.lo1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= c.hi0 || j >= c.hi1) return;
  const long long d0 = c.d0;
  const long long o = i + j * d0;
  T R = c.R0 + c.dR * (T)(i - c.g0);
  if (fabs(R) < Tiny<T>::v) R = Tiny<T>::v;
  auto X = [&](const T* f, int k) { return __ldg(f + o + (k - 2)); };
  auto Y = [&](const T* f, int k) { return __ldg(f + o + (k - 2) * d0); };
  auto dR = [&](const T* f) { return d1_4w(X(f, 0), X(f, 1), X(f, 3), X(f, 4)) * c.inv_dR; };
  auto dz = [&](const T* f) { return d1_4w(Y(f, 0), Y(f, 1), Y(f, 3), Y(f, 4)) * c.inv_dz; };
  // dfRdRR (:110-113): (R f)_R / R, 2 f_R on the axis
  const bool on_axis = fabs(R) < c.dR * T(0.25);
  auto dRR = [&](const T* f) {
    if (on_axis) return T(2) * dR(f);
    const T h = c.dR;
    return d1_4w(X(f, 0) * (R - T(2) * h), X(f, 1) * (R - h), X(f, 3) * (R + h),
                 X(f, 4) * (R + T(2) * h)) * c.inv_dR / R;
  };
  const T *ER = u.p[0], *Ez = u.p[1], *Ef = u.p[2], *BR = u.p[3], *Bz = u.p[4], *Bf = u.p[5];
  const T rotBR = -dz(Bf), rotBz = dRR(Bf), rotBf = dz(BR) - dR(Bz);
  const T rotER = -dz(Ef), rotEz = dRR(Ef), rotEf = dz(ER) - dR(Ez);
  const T divE = dRR(ER) + dz(Ez);
  const T divB = dRR(BR) + dz(Bz);
  T v[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) v[a] = __ldg(u.p[a] + o);
  T B2 = v[3] * v[3] + v[4] * v[4] + v[5] * v[5];
  if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
  const T Jp = (v[3] * rotBR + v[4] * rotBz + v[5] * rotBf) -
               (v[0] * rotER + v[1] * rotEz + v[2] * rotEf);
  const T iB2 = fdiv(T(1), B2);
  const T JR = (divE * (v[2] * v[4] - v[1] * v[5]) + Jp * v[3]) * iB2;
  const T Jf = (divE * (v[1] * v[3] - v[0] * v[4]) + Jp * v[5]) * iB2;
  const T Jz = (divE * (v[0] * v[5] - v[2] * v[3]) + Jp * v[4]) * iB2;
  const T dt = c.dt;
  T rhs[7];
  rhs[0] = dt * (rotBR - JR);
  rhs[1] = dt * (rotBz - Jz);
  rhs[2] = dt * (rotBf - Jf);
  rhs[3] = -dt * (rotER + dR(u.p[6]));
  rhs[4] = -dt * (rotEz + dz(u.p[6]));
  rhs[5] = -dt * rotEf;
  rhs[6] = -dt * c.ch2 * divB - v[6] / c.tau;
  if (flags & AX_WRITE_UN) {
#pragma unroll
    for (int a = 0; a < 6; ++a) un.p[a][o] = v[a];
  }
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const T d = FIRST ? rhs[a] : As * du.p[a][o] + rhs[a];
    du.p[a][o] = d;
    v[a] += Bs * d;
  }
  cyl_clamps(c, v);
  cyl_finish(c, i, j, o, v, out, un, tst, (flags & AX_LAST) != 0);
}

// Kreiss-Oliger pass of the cylindrical solver (kernel_KO_step1_thread +
// _step2_thread, field_solver_EZ_cylindrical.cu:297-369; order of :705-712):
// plain 6th differences in R and z, the clamps, then cyl_finish at t + dt.
template <typename T>
__global__ void __launch_bounds__(256, kCylKoMinBlocks) cyl_ko_kernel(const __grid_constant__ CylConst<T> c,
                                                     const F7<T> u, const F7<T> out,
                                                     const F7<T> un, const T tend) {
  const int i = c.lo0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = c.lo1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= c.hi0 || j >= c.hi1) return;
  const long long d0 = c.d0;
  const long long o = i + j * d0;
  constexpr T K6[7] = {T(1), T(-6), T(15), T(-20), T(15), T(-6), T(1)};
  T v[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const T* f = u.p[a];
    T tx = T(0), ty = T(0);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      tx += K6[k] * __ldg(f + o + (k - 3));
      ty += K6[k] * __ldg(f + o + (k - 3) * d0);
    }
    v[a] = __ldg(f + o) + c.ko_c * (tx + ty);
  }
  cyl_clamps(c, v);
  cyl_finish(c, i, j, o, v, out, un, tend, false);
}

}  // namespace coffee
