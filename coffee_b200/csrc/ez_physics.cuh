// Pointwise physics of the flat EZ update, shared by the stage and KO
// kernels: the force-free current and RHS, the E.B = 0 / |E| <= |B| clamps,
// the rotating-star boundaries and the absorbing layer.  Every function acts
// on one grid point held in registers.
#pragma once

#include "ez_common.cuh"
#include "ez_refarith.cuh"

namespace coffee {

// Grid::pos(axis, n, 1) = lower + delta * (n - guard)  (src/data/grid.h:116-134)
template <typename T>
__device__ __forceinline__ T grid_pos(const EzConst<T>& c, int axis, int n) {
  return c.lower[axis] + c.delta[axis] * (T)(n - c.g.guard[axis]);
}

// ---------------------------------------------------------------- clamps
// CPU build: clean_epar_check_eGTb, unconditional
// (src/algorithms/field_solver_EZ.cpp:552-634).  GPU build: kernel_Epar if
// clean_ep, then kernel_EgtB if check_egb (field_solver_EZ.cu:213-270).
template <typename T>
__device__ __forceinline__ void apply_clamps(const EzConst<T>& c, T& ex, T& ey, T& ez, T bx,
                                             T by, T bz) {
  const bool cpu = c.semantics == SEM_CPU_REF;
  T B2 = bx * bx + by * by + bz * bz;
  if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
  if (cpu || c.clean_ep) {
    // E -= (E.B / B^2) B, one division shared by the three components
    const T q = fdiv(bx * ex + by * ey + bz * ez, B2);
    ex = ex - q * bx;
    ey = ey - q * by;
    ez = ez - q * bz;
  }
  if (cpu || c.check_egb) {
    const T E2 = ex * ex + ey * ey + ez * ez;
    if (E2 > B2) {
      const T s = sqrt(B2 / E2);
      ex *= s;
      ey *= s;
      ez *= s;
    }
  }
}

// The CPU build's clean_epar_check_eGTb in that build's own arithmetic
// (field_solver_EZ.cpp:552-634; the rounding and fusing rules are those of
// ez_refarith.cuh): E -= ((E.B) B_a) / B^2 per component, then, where
// |E|^2 > B^2, E *= sqrt(B^2 / |E|^2).
template <typename T>
__device__ __forceinline__ void apply_clamps_xa(T& ex, T& ey, T& ez, T bx, T by, T bz) {
  const T B2 = xa::floor_tiny(xa::dot3(bx, bx, by, by, bz, bz));
  const T EB = xa::dot3(bx, ex, by, ey, bz, ez);
  ex = xa::sub(ex, xa::div(xa::mul(EB, bx), B2));
  ey = xa::sub(ey, xa::div(xa::mul(EB, by), B2));
  ez = xa::sub(ez, xa::div(xa::mul(EB, bz), B2));
  const T E2 = xa::dot3(ex, ex, ey, ey, ez, ez);
  if (E2 > B2) {
    const T s = xa::sqrt(xa::div(B2, E2));
    ex = xa::mul(ex, s);
    ey = xa::mul(ey, s);
    ez = xa::mul(ez, s);
  }
}

// The same clamps, adding the energy changes they make at point o to the
// CPU build's diagnostics (clean_epar_check_eGTb, field_solver_EZ.cpp:
// 578-624): |E|^2 after the cleaning minus before it to dU_Epar and
// dU_Epar_cum, |E|^2 after both clamps minus before the cleaning to dU_EgtB
// and dU_EgtB_cum.  FIRST: the step's first accumulation into dU_Epar and
// dU_EgtB, which evolve_fields zeroes at its start (:1019-1021).
template <bool FIRST, typename T>
__device__ __forceinline__ void apply_clamps_xa_dg(T& ex, T& ey, T& ez, T bx, T by, T bz,
                                                   const F6<T>& dg, uint32_t o) {
  const T B2 = xa::floor_tiny(xa::dot3(bx, bx, by, by, bz, bz));
  const T EB = xa::dot3(bx, ex, by, ey, bz, ez);
  const T u0 = xa::dot3(ex, ex, ey, ey, ez, ez);
  ex = xa::sub(ex, xa::div(xa::mul(EB, bx), B2));
  ey = xa::sub(ey, xa::div(xa::mul(EB, by), B2));
  ez = xa::sub(ez, xa::div(xa::mul(EB, bz), B2));
  const T E2 = xa::dot3(ex, ex, ey, ey, ez, ez);
  T u1g = E2;
  if (E2 > B2) {
    const T s = xa::sqrt(xa::div(B2, E2));
    ex = xa::mul(ex, s);
    ey = xa::mul(ey, s);
    ez = xa::mul(ez, s);
    u1g = xa::dot3(ex, ex, ey, ey, ez, ez);
  }
  const T dp = xa::sub(E2, u0), dgt = xa::sub(u1g, u0);
  dg.p[4][o] = xa::add(dp, dg.p[4][o]);
  dg.p[1][o] = xa::add(FIRST ? (T)0 : dg.p[1][o], dp);
  dg.p[3][o] = xa::add(dgt, dg.p[3][o]);
  dg.p[0][o] = xa::add(FIRST ? (T)0 : dg.p[0][o], dgt);
}

// ------------------------------------------------------- star field models
// dipole2 / quadrupole / quadru_dipole (src/algorithms/pulsar_impl.hpp:57-129),
// evaluated in double (the reference promotes through its double literals)
// and returned in field precision.
__device__ inline void dipole2_d(double x, double y, double z, double p1, double p2,
                                 double p3, double phase, double tiny, double out[3]) {
  const double cph = cos(phase), sph = sin(phase);
  const double p1t = p1 * cph - p2 * sph, p2t = p1 * sph + p2 * cph, p3t = p3;
  const double r2 = x * x + y * y + z * z;
  const double pr = p1t * x + p2t * y + p3t * z;
  const double den = sqrt(r2 * r2 * r2) + tiny;
  out[0] = (3.0 * x * pr / (r2 + tiny) - p1t) / den;
  out[1] = (3.0 * y * pr / (r2 + tiny) - p2t) / den;
  out[2] = (3.0 * z * pr / (r2 + tiny) - p3t) / den;
}

template <typename T>
__device__ inline void quadrupole_d(const EzConst<T>& c, double x, double y, double z,
                                    double phase, double tiny, double out[3]) {
  const double cph = cos(phase), sph = sin(phase);
  const double q11 = c.q11, q12 = c.q12, q13 = c.q13, q22 = c.q22, q23 = c.q23;
  const double q11t = q11 * cph * cph - 2.0 * q12 * cph * sph + q22 * sph * sph;
  const double q12t = q12 * cos(2.0 * phase) + (q11 - q22) * cph * sph;
  const double q22t = q22 * cph * cph + q11 * sph * sph + 2.0 * q12 * cph * sph;
  const double q13t = q13 * cph - q23 * sph;
  const double q23t = q23 * cph + q13 * sph;
  const double q33t = -q11 - q22;
  const double ox = (double)c.qox * cph - (double)c.qoy * sph;
  const double oy = (double)c.qox * sph + (double)c.qoy * cph;
  const double x1 = x - ox, y1 = y - oy, z1 = z - (double)c.qoz;
  const double r2 = x1 * x1 + y1 * y1 + z1 * z1;
  const double r7 = r2 * r2 * r2 * sqrt(r2);
  const double xqx = q11t * x1 * x1 + 2.0 * q12t * x1 * y1 + q22t * y1 * y1 +
                     2.0 * (q13t * x1 + q23t * y1) * z1 + q33t * z1 * z1;
  out[0] = (-2.0 * (q11t * x1 + q12t * y1 + q13t * z1) * r2 + 5.0 * x1 * xqx) / (r7 + tiny);
  out[1] = (-2.0 * (q12t * x1 + q22t * y1 + q23t * z1) * r2 + 5.0 * y1 * xqx) / (r7 + tiny);
  out[2] = (-2.0 * (q13t * x1 + q23t * y1 + q33t * z1) * r2 + 5.0 * z1 * xqx) / (r7 + tiny);
}

// b0 * quadru_dipole(x, y, z, ..., phase) as three field-precision values.
template <typename T>
__device__ inline void star_field(const EzConst<T>& c, T x, T y, T z, T phase, T out[3]) {
  const double tiny = (double)Tiny<T>::v;
  double d[3], q[3];
  dipole2_d(x, y, z, c.p1, c.p2, c.p3, phase, tiny, d);
  quadrupole_d(c, x, y, z, phase, tiny, q);
  for (int a = 0; a < 3; ++a) out[a] = c.b0 * ((T)d[a] + (T)q[a]);
}

// shape(r, r0, del) = 0.5 (1 - tanh((r - r0) / del))  (pulsar_impl.hpp:52-55)
template <typename T>
__device__ __forceinline__ T shape_fn(T r, T r0, T del) {
  return (T)(0.5 * (1.0 - tanh((double)((r - r0) / del))));
}

// Alfven-wave perturbations of the CPU build's boundary_alfven:
// wpert, wpert3d, twistv (src/algorithms/field_solver_EZ.cpp:644-709).
template <typename T>
__device__ inline T wpert_dev(T t, T th, T tp_start, T tp_end, T dw0, T nT, T rp1, T rp2) {
  T th1 = (T)acos(sqrt(1.0 - 1.0 / (double)rp1));
  T th2 = (T)acos(sqrt(1.0 - 1.0 / (double)rp2));
  if (th1 > th2) { T tmp = th1; th1 = th2; th2 = tmp; }
  const T mu = (T)((double)(th1 + th2) / 2.0);
  const T s = (T)((double)(mu - th1) / 3.0);
  if (t >= tp_start && t <= tp_end && th >= th1 && th <= th2) {
    const T q = (th - mu) / s;
    return (T)((double)dw0 * exp(-0.5 * (double)(q * q)) *
               sin((double)(t - tp_start) * 2.0 * M_PI * (double)nT / (double)(tp_end - tp_start)));
  }
  return 0;
}

template <typename T>
__device__ inline T wpert3d_dev(T t, T th, T ph, T tp_start, T tp_end, T dw0, T nT, T rp1,
                                T rp2, T ph1, T ph2, T dph) {
  T th1 = (T)acos(sqrt(1.0 - 1.0 / (double)rp1));
  T th2 = (T)acos(sqrt(1.0 - 1.0 / (double)rp2));
  if (th1 > th2) { T tmp = th1; th1 = th2; th2 = tmp; }
  const T mu = (T)((double)(th1 + th2) / 2.0);
  const T s = (T)((double)(mu - th1) / 3.0);
  if (t >= tp_start && t <= tp_end && th >= th1 && th <= th2) {
    const T q = (th - mu) / s;
    const double v =
        (double)dw0 * exp(-0.5 * (double)(q * q)) *
        sin((double)(t - tp_start) * 2.0 * M_PI * (double)nT / (double)(tp_end - tp_start)) *
        (double)shape_fn<T>(ph, (T)((double)ph2 * M_PI), (T)((double)dph * M_PI)) *
        (1.0 - (double)shape_fn<T>(ph, (T)((double)ph1 * M_PI), (T)((double)dph * M_PI)));
    return (T)v;
  }
  return 0;
}

template <typename T>
__device__ inline void twistv_dev(const EzConst<T>& c, T t, T x, T y, T z, T ri, T v[3]) {
  const T costh0 = (T)cos((double)c.theta0), sinth0 = (T)sin((double)c.theta0);
  const T x1 = -x * costh0 + z * sinth0, y1 = y, z1 = x * sinth0 + z * costh0;
  const T r = sqrt(x * x + y * y + z * z);
  const T R1 = sqrt(x1 * x1 + y1 * y1);
  const T costh = x1 / (R1 + Tiny<T>::v), sinth = y1 / (R1 + Tiny<T>::v);
  T dw = 0;
  if (r > ri && z1 >= 0 && R1 <= c.drpert && t >= c.tp_start && t <= c.tp_end) {
    const double cc = cos((double)(R1 / c.drpert) * M_PI / 2.0);
    const double ss = sin((double)(t - c.tp_start) * M_PI / (double)(c.tp_end - c.tp_start));
    dw = (T)((double)c.dw0 * cc * cc *
             sin((double)(t - c.tp_start) * 2.0 * M_PI * (double)c.nT /
                 (double)(c.tp_end - c.tp_start)) *
             ss * ss);
  }
  v[0] = dw * R1 * sinth * costh0;
  v[1] = dw * R1 * costh;
  v[2] = -dw * R1 * sinth * sinth0;
}

// ------------------------------------------------------------ star boundary
// boundary_pulsar (CPU field_solver_EZ.cpp:711-839 with rl = 1.5 R; GPU
// field_solver_EZ.cu:394-528 with rl = 2 R) and, for problem 2 in the CPU
// build, boundary_alfven (field_solver_EZ.cpp:841-1005).  Blends the radial
// and tangential parts of B and E toward the corotating star inside rl and
// imposes them inside R/2.
// The blend itself, kept out of line: only points near the star reach it,
// so its registers do not weigh on the streaming loop.
template <typename T>
__device__ __noinline__ V7<T> star_blend(const EzConst<T>& c, T x, T y, T z, T r2, T r, T t,
                                         V7<T> u) {
  const bool cpu = c.semantics == SEM_CPU_REF;
  const bool alfven = (c.problem == 2);
  T ex = u.v[0], ey = u.v[1], ez = u.v[2], bx = u.v[3], by = u.v[4], bz = u.v[5];
  const T R = c.radius;
  const T ri = (T)(0.5 * (double)R);
  const T scaleEpar = (T)(0.5 * (double)c.delta[0]);
  const T scaleEperp = (T)(0.25 * (double)c.delta[0]);
  const T scaleB = scaleEpar;
  const T d1 = (T)(4.0 * (double)c.delta[0]);
  const T phase = c.omega * t;
  T vx, vy, vz, bn[3];
  if (alfven) {
    const T th = (T)acos((double)(z / r));
    const T ph = (T)atan2((double)y, (double)x);
    if (c.pert_type == 2) {
      T v[3];
      twistv_dev(c, t, x, y, z, ri, v);
      vx = v[0]; vy = v[1]; vz = v[2];
    } else {
      T w0, w1;
      if (c.pert_type == 0) {
        w0 = wpert_dev(t, th, c.tp_start, c.tp_end, c.dw0, c.nT, c.rpert1, c.rpert2);
        w1 = wpert_dev(t, th, c.tp_start1, c.tp_end1, c.dw1, c.nT1, c.rpert11, c.rpert21);
      } else {
        w0 = wpert3d_dev(t, th, ph, c.tp_start, c.tp_end, c.dw0, c.nT, c.rpert1, c.rpert2,
                         c.ph1, c.ph2, c.dph);
        w1 = wpert3d_dev(t, th, ph, c.tp_start1, c.tp_end1, c.dw1, c.nT1, c.rpert11,
                         c.rpert21, c.ph11, c.ph21, c.dph1);
      }
      const T w = c.omega + w0 + w1;
      vx = -w * y; vy = w * x; vz = 0;
    }
    double d[3];
    dipole2_d(x, y, z, c.p1, c.p2, c.p3, phase, (double)Tiny<T>::v, d);
    for (int a = 0; a < 3; ++a) bn[a] = c.b0 * (T)d[a];
  } else {
    vx = -c.omega * y; vy = c.omega * x; vz = 0;
    star_field(c, x, y, z, phase, bn);
  }
  T s = shape_fn(r, R - d1, scaleB);
  const T bn_r = bn[0] * x + bn[1] * y + bn[2] * z;
  const T B_r = bx * x + by * y + bz * z;
  T nbx = bn_r * x / r2 * s + B_r * x / r2 * (1 - s);
  T nby = bn_r * y / r2 * s + B_r * y / r2 * (1 - s);
  T nbz = bn_r * z / r2 * s + B_r * z / r2 * (1 - s);
  nbx += (bn[0] - bn_r * x / r2) * s + (bx - B_r * x / r2) * (1 - s);
  nby += (bn[1] - bn_r * y / r2) * s + (by - B_r * y / r2) * (1 - s);
  nbz += (bn[2] - bn_r * z / r2) * s + (bz - B_r * z / r2) * (1 - s);
  bx = nbx; by = nby; bz = nbz;
  const T exn = -vy * bz + vz * by;
  const T eyn = vx * bz - vz * bx;
  const T ezn = -vx * by + vy * bx;
  const T en_r = exn * x + eyn * y + ezn * z;
  const T E_r = ex * x + ey * y + ez * z;
  s = shape_fn(r, R, scaleEperp);
  T nex = en_r * x / r2 * s + E_r * x / r2 * (1 - s);
  T ney = en_r * y / r2 * s + E_r * y / r2 * (1 - s);
  T nez = en_r * z / r2 * s + E_r * z / r2 * (1 - s);
  s = shape_fn(r, R, scaleEpar);
  nex += (exn - en_r * x / r2) * s + (ex - E_r * x / r2) * (1 - s);
  ney += (eyn - en_r * y / r2) * s + (ey - E_r * y / r2) * (1 - s);
  nez += (ezn - en_r * z / r2) * s + (ez - E_r * z / r2) * (1 - s);
  ex = nex; ey = ney; ez = nez;
  if (r < ri) {
    bx = bn[0]; by = bn[1]; bz = bn[2];
    ex = exn; ey = eyn; ez = ezn;
  }
  u.v[0] = ex; u.v[1] = ey; u.v[2] = ez; u.v[3] = bx; u.v[4] = by; u.v[5] = bz;
  return u;
}

template <typename T>
__device__ __forceinline__ void star_boundary(const EzConst<T>& c, int i, int j, int k, T t,
                                              T u[7]) {
  const bool cpu = c.semantics == SEM_CPU_REF;
  if (c.problem != 1 && !(c.problem == 2 && cpu)) return;
  const T x = grid_pos(c, 0, i), y = grid_pos(c, 1, j), z = grid_pos(c, 2, k);
  T r2 = x * x + y * y + z * z;
  if (r2 < Tiny<T>::v) r2 = Tiny<T>::v;
  const T r = sqrt(r2);
  const T rl = cpu ? (T)(1.5 * (double)c.radius) : (T)(2.0 * (double)c.radius);
  if (r < rl) {
    V7<T> in;
#pragma unroll
    for (int f = 0; f < 7; ++f) in.v[f] = u[f];
    const V7<T> out = star_blend(c, x, y, z, r2, r, t, in);
#pragma unroll
    for (int f = 0; f < 6; ++f) u[f] = out.v[f];
  }
}

// ---------------------------------------------------------- absorbing layer
// pmlsigma (src/algorithms/damping_boundary.h:14-22)
template <typename T>
__device__ __forceinline__ T pml_sigma(T x, T xl, T xh, T scale, T sig0) {
  if (x > xh) { const T q = (x - xh) / scale; return sig0 * (q * q * q); }
  if (x < xl) { const T q = (xl - x) / scale; return sig0 * (q * q * q); }
  return 0;
}

// Conductivity of the absorbing layer at point (i, j, k): the sum over axes
// of pmlsigma outside [pml_lo, pml_hi] (damping_boundary.cpp:32-62,
// boundary.cu:105-125), or 0 where the reference leaves the point alone
// (inside the box, or sigma <= TINY).
template <typename T>
__device__ __forceinline__ T absorbing_sigma(const EzConst<T>& c, int i, int j, int k) {
  const T x = grid_pos(c, 0, i), y = grid_pos(c, 1, j), z = grid_pos(c, 2, k);
  if (!(x > c.pml_hi[0] || x < c.pml_lo[0] || y > c.pml_hi[1] || y < c.pml_lo[1] ||
        z > c.pml_hi[2] || z < c.pml_lo[2]))
    return 0;
  const T sig = pml_sigma(x, c.pml_lo[0], c.pml_hi[0], c.pml_scale[0], c.sigpml) +
                pml_sigma(y, c.pml_lo[1], c.pml_hi[1], c.pml_scale[1], c.sigpml) +
                pml_sigma(z, c.pml_lo[2], c.pml_hi[2], c.pml_scale[2], c.sigpml);
  return (sig > Tiny<T>::v) ? sig : (T)0;
}

// Relaxation toward the start-of-step state un[7] at the last stage, for a
// point with absorbing_sigma() = sig > 0.  CPU build
// (damping_boundary.cpp:63-78): B relaxes toward the background dipole,
// P is left alone, the length scale uses each axis' delta.  GPU build
// (boundary.cu:127-142): B toward zero, P toward Pn, delta[0] on every axis.
template <typename T>
__device__ __noinline__ V7<T> absorbing_apply(const EzConst<T>& c, int i, int j, int k, T sig,
                                              V7<T> u, const V7<T> un) {
  const double ed = exp(-(double)sig);
  const double fd = (1.0 - ed) / (double)sig;
  for (int a = 0; a < 3; ++a)
    u.v[a] = (T)(ed * (double)un.v[a] + fd * (double)(u.v[a] - un.v[a]));
  if (c.semantics == SEM_CPU_REF) {
    T bg[3];
    star_field(c, grid_pos(c, 0, i), grid_pos(c, 1, j), grid_pos(c, 2, k), (T)0, bg);
    for (int a = 0; a < 3; ++a)
      u.v[3 + a] = (T)((double)bg[a] + ed * (double)(un.v[3 + a] - bg[a]) +
                       fd * (double)(u.v[3 + a] - un.v[3 + a]));
  } else {
    for (int a = 3; a < 7; ++a)
      u.v[a] = (T)(ed * (double)un.v[a] + fd * (double)(u.v[a] - un.v[a]));
  }
  return u;
}

// Per-thread constants of a column (i, j) of a z-streaming kernel: its
// indices and the parts of the P-gradient taper that do not depend on k.
template <typename T>
struct ColumnCtx {
  int i, j;
  bool xy_simple;  // the point writes only itself along x and y (no guard image)
  T taper_x, taper_y, taper_dz;  // (reference arithmetic: taper_dz holds the lane)
};

// The P-gradient taper of the CPU build's rk_step
// (field_solver_EZ.cpp:222-230): s = (1 - tanh((r - 3)/0.5)) / 2 with x, y
// and z each offset by lane*delta, lane = position of i within the
// reference's SIMD vector.  x and y are fixed per column (ColumnCtx).
// In FP32 the taper is evaluated as 1 / (1 + exp(4 (r - 3))), the same
// function written with one exponential and one reciprocal.
__device__ __forceinline__ float taper_fn(float r) {
  return __fdividef(1.0f, 1.0f + __expf(4.0f * (r - 3.0f)));
}
__device__ __forceinline__ double taper_fn(double r) { return 0.5 * (1.0 - tanh((r - 3.0) / 0.5)); }

template <typename T>
__device__ __forceinline__ T p_taper(const EzConst<T>& c, const ColumnCtx<T>& col, int k) {
  const T z = col.taper_dz + grid_pos(c, 2, k);
  const T r = sqrt(col.taper_x * col.taper_x + col.taper_y * col.taper_y + z * z);
  return taper_fn(r);
}

// Index lists of the points that hold the value computed at (i, j, k):
// itself (unless it is a periodic guard, which its image overwrites) and, in
// each periodic direction, the guard image of a point within `guard` of the
// face.  Composing the three directions reproduces the x -> y -> z order of
// the reference's exchange, corners included.
__device__ __forceinline__ int periodic_targets(const GridGeom& g, int axis, int i, int out[2]) {
  const int gd = g.guard[axis], d = g.dims[axis], N = g.N[axis];
  out[0] = i;
  out[1] = i;
  if (!g.periodic[axis]) return 1;
  // at most two of: the point itself (interior), i + N, i - N
  const bool self = (i >= gd && i < d - gd);
  const bool up = (i >= gd && i < 2 * gd);
  const bool down = (i >= d - 2 * gd && i < d - gd);
  int n = 0;
  if (self) { out[0] = i; n = 1; }
  if (up) { if (n == 0) out[0] = i + N; else out[1] = i + N; ++n; }
  if (down) { if (n == 0) out[0] = i - N; else out[1] = i - N; ++n; }
  return n;
}

// True when index i along `axis` has no periodic guard image and is not a
// periodic guard itself, i.e. the value computed there is stored only there.
__device__ __forceinline__ bool only_self(const GridGeom& g, int axis, int i) {
  if (!g.periodic[axis]) return true;
  const int gd = g.guard[axis];
  return i >= 2 * gd && i < g.dims[axis] - 2 * gd;
}

// The same taper in the CPU build's own arithmetic (ez_refarith.cuh):
// coordinates by two FMAs each, r = sqrt(x x + y y + z z) with the last two
// products fused, and the vectorclass tanh.
template <typename T>
__device__ __forceinline__ T p_taper_xa(const EzConst<T>& c, const ColumnCtx<T>& col, int k) {
  const T z = xa::lane_pos(c.delta[2], c.lower[2], k - c.g.guard[2], col.taper_dz);
  const T r = xa::sqrt(xa::dot3(col.taper_x, col.taper_x, col.taper_y, col.taper_y, z, z));
  return xa::taper_of_r(r);
}

template <bool XA, typename T>
__device__ __forceinline__ ColumnCtx<T> make_column(const EzConst<T>& c, int i, int j) {
  ColumnCtx<T> col;
  col.i = i;
  col.j = j;
  col.xy_simple = only_self(c.g, 0, i) && only_self(c.g, 1, j);
  const int lane = (i - c.g.lo[0]) % c.taper_lanes;
  const T fl = (T)lane;
  if constexpr (XA) {
    col.taper_x = xa::lane_pos(c.delta[0], c.lower[0], i - lane - c.g.guard[0], fl);
    col.taper_y = xa::lane_pos(c.delta[1], c.lower[1], j - c.g.guard[1], fl);
    col.taper_dz = fl;
  } else {
    col.taper_x = fl * c.delta[0] + grid_pos(c, 0, i - lane);
    col.taper_y = fl * c.delta[1] + grid_pos(c, 1, j);
    col.taper_dz = fl * c.delta[2];
  }
  return col;
}

}  // namespace coffee
