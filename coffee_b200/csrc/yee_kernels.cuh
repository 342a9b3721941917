// Device code of the staggered (Yee) RK3 solver, the reference's
// field_solver (src/algorithms/field_solver.cu), for the flat Cartesian grid.
//
// Layout (src/data/sim_data.cpp:19-25): E_x at (i+1/2, j, k), E_y at
// (i, j+1/2, k), E_z at (i, j, k+1/2); B_x at (i, j+1/2, k+1/2), B_y at
// (i+1/2, j, k+1/2), B_z at (i+1/2, j+1/2, k); the charge density at the
// vertex (i, j, k).  A stagger bit set means "on the vertex along that axis".
//
// One substep of the reference is seven kernels over the whole grid (rho,
// push, update, [clean], check, [two pulsar passes], absorbing) plus the
// guard exchange.  Here it is two streaming passes:
//   update: rho = div E, dB = -curl E, dE = curl (B - B0) - J, then
//           E* = c1 En + c2 E + c3 dE, B' = c1 Bn + c2 B + c3 dB
//           (kernel_compute_rho_thread, kernel_rk_push_thread and
//           kernel_rk_update_thread, field_solver.cu:22-184), written to
//           scratch because the neighbours still need the old E and B;
//   clamp:  [E_par cleaning,] the |E| <= |B| rescale, [absorbing layer],
//           and the store of E and B with their periodic guard images
//           (kernel_clean_epar_thread, kernel_check_eGTb_thread,
//           boundary.cu:18-78, field_solver.cu:186-342).
// The rotating-star boundary (problem 1) adds three small passes over the
// box around the star and a guard pass.
//
// Every thread owns one (i, j) column of a z range and walks it plane by
// plane.  The values a point reads live in a 3 x 3 x 3 register window per
// array (Win): moving to the next plane shifts the window down in z and
// loads only the entries that were not already in it.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ez_common.cuh"
#include "ez_physics.cuh"

// Resident CTAs of 256 threads per SM that the register allocation of the
// streaming passes must allow (FP32; FP64 builds ask for 1).  The passes are
// latency bound: 3 CTAs (80 registers) beat 2 (116) by 20% and 4 (64, with
// spills); the first substep's update, which also writes the start-of-step
// copies, keeps 2.
#ifndef COFFEE_YEE_UPDATE_MIN_BLOCKS
#define COFFEE_YEE_UPDATE_MIN_BLOCKS 3
#endif
#ifndef COFFEE_YEE_FIRST_MIN_BLOCKS
#define COFFEE_YEE_FIRST_MIN_BLOCKS 2
#endif
#ifndef COFFEE_YEE_CLAMP_MIN_BLOCKS
#define COFFEE_YEE_CLAMP_MIN_BLOCKS 3
#endif

namespace coffee {

constexpr int kStE[3] = {0b110, 0b101, 0b011};
constexpr int kStB[3] = {0b001, 0b010, 0b100};
constexpr int kStRho = 0b111;

__host__ __device__ constexpr int widx(int dx, int dy, int dz) {
  return (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
}
__host__ __device__ constexpr uint32_t wbit(int dx, int dy, int dz) {
  return 1u << widx(dx, dy, dz);
}
// Entries (dx, dy, dz) of box {x0..x1} x {y0..y1} x {z0..z1}.
__host__ __device__ constexpr uint32_t wbox(int x0, int x1, int y0, int y1, int z0, int z1) {
  uint32_t m = 0;
  for (int z = z0; z <= z1; ++z)
    for (int y = y0; y <= y1; ++y)
      for (int x = x0; x <= x1; ++x) m |= wbit(x, y, z);
  return m;
}

// Offsets along each axis of the points `interpolate` averages for a value
// of stagger IN at a point of stagger OUT (src/algorithms/interpolation.h:9-17):
// none where the staggers agree, else {-out, 1 - out}.
__host__ __device__ constexpr int ilo(int in, int out, int a) {
  return ((in >> a) & 1) == ((out >> a) & 1) ? 0 : -((out >> a) & 1);
}
__host__ __device__ constexpr int ihi(int in, int out, int a) {
  return ((in >> a) & 1) == ((out >> a) & 1) ? 0 : 1 - ((out >> a) & 1);
}
__host__ __device__ constexpr uint32_t interp_mask(int in, int out) {
  return wbox(ilo(in, out, 0), ihi(in, out, 0), ilo(in, out, 1), ihi(in, out, 1),
              ilo(in, out, 2), ihi(in, out, 2));
}
// Register window of one array around the current point.
template <uint32_t M, typename T>
struct Win {
  T v[27];
  template <int DX, int DY, int DZ>
  __device__ __forceinline__ T at() const {
    static_assert((M >> widx(DX, DY, DZ)) & 1u, "window entry is not loaded");
    return v[widx(DX, DY, DZ)];
  }
  // every entry, at the first point of a column
  __device__ __forceinline__ void load(const T* __restrict__ f, uint32_t o, int sy, int sz) {
#pragma unroll
    for (int q = 0; q < 27; ++q)
      if ((M >> q) & 1u) v[q] = __ldg(f + (o + (uint32_t)((q % 3 - 1) + (q / 3 % 3 - 1) * sy +
                                                          (q / 9 - 1) * sz)));
  }
  // one plane up: entries whose z + 1 neighbour is in the window take its
  // value (ascending q reads each source before it is overwritten), the
  // rest are loaded at the new point o
  __device__ __forceinline__ void advance(const T* __restrict__ f, uint32_t o, int sy, int sz) {
#pragma unroll
    for (int q = 0; q < 27; ++q) {
      if (!((M >> q) & 1u)) continue;
      if (q < 18 && ((M >> (q + 9)) & 1u))
        v[q] = v[q + 9];
      else
        v[q] = __ldg(f + (o + (uint32_t)((q % 3 - 1) + (q / 3 % 3 - 1) * sy +
                                         (q / 9 - 1) * sz)));
    }
  }
};

// interpolate(f, ijk, IN, OUT) of the reference: pairs summed along z, then
// y, then x, each halved (interpolation.h:18-33; the 0.5 literal is exact in
// both precisions).
template <int IN, int OUT, uint32_t M, typename T>
__device__ __forceinline__ T interp(const Win<M, T>& w) {
  constexpr int im = ilo(IN, OUT, 0), ip = ihi(IN, OUT, 0);
  constexpr int jm = ilo(IN, OUT, 1), jp = ihi(IN, OUT, 1);
  constexpr int km = ilo(IN, OUT, 2), kp = ihi(IN, OUT, 2);
  const T h = (T)0.5;
  const T f11 = h * (w.template at<ip, jp, km>() + w.template at<ip, jp, kp>());
  const T f10 = h * (w.template at<ip, jm, km>() + w.template at<ip, jm, kp>());
  const T f01 = h * (w.template at<im, jp, km>() + w.template at<im, jp, kp>());
  const T f00 = h * (w.template at<im, jm, km>() + w.template at<im, jm, kp>());
  const T f1 = h * (f11 + f10);
  const T f0 = h * (f01 + f00);
  return h * (f1 + f0);
}

// Window masks.  The update pass reads, around the point: E for rho at the
// point and at +x, +y, +z, for -curl E and for the interpolations to the
// three E positions; B for curl B and the interpolations; B0 for its curl.
constexpr uint32_t kUpEx = wbit(0, 0, 0) | wbit(0, 0, 1) | wbit(-1, 0, 0) | wbit(-1, 0, 1) |
                           wbit(1, 0, 0) | wbit(0, 1, 0) | wbit(-1, 1, 0);
constexpr uint32_t kUpEy = wbit(0, 0, 0) | wbit(0, 0, 1) | wbit(0, -1, 0) | wbit(0, -1, 1) |
                           wbit(1, 0, 0) | wbit(1, -1, 0) | wbit(0, 1, 0);
constexpr uint32_t kUpEz = wbit(0, 0, -1) | wbit(0, 0, 0) | wbit(0, 0, 1) | wbit(1, 0, -1) |
                           wbit(1, 0, 0) | wbit(0, 1, -1) | wbit(0, 1, 0);
constexpr uint32_t kWinBx = wbox(0, 1, -1, 0, -1, 0);
constexpr uint32_t kWinBy = wbox(-1, 0, 0, 1, -1, 0);
constexpr uint32_t kWinBz = wbox(-1, 0, -1, 0, 0, 1);
constexpr uint32_t kUpB0x = wbit(0, 0, -1) | wbit(0, 0, 0) | wbit(0, -1, 0);
constexpr uint32_t kUpB0y = wbit(0, 0, -1) | wbit(0, 0, 0) | wbit(-1, 0, 0);
constexpr uint32_t kUpB0z = wbit(0, 0, 0) | wbit(0, -1, 0) | wbit(-1, 0, 0);
constexpr uint32_t kRhoWin = wbit(0, 0, 0) | wbit(1, 0, 0) | wbit(0, 1, 0) | wbit(0, 0, 1);
// The clamp pass interpolates E* and B' to the three E positions.
constexpr uint32_t kClEx = interp_mask(0b110, 0b110) | interp_mask(0b110, 0b101) |
                           interp_mask(0b110, 0b011);
constexpr uint32_t kClEy = interp_mask(0b101, 0b110) | interp_mask(0b101, 0b101) |
                           interp_mask(0b101, 0b011);
constexpr uint32_t kClEz = interp_mask(0b011, 0b110) | interp_mask(0b011, 0b101) |
                           interp_mask(0b011, 0b011);
static_assert((kClEx & kUpEx) == kClEx && (kClEy & kUpEy) == kClEy && (kClEz & kUpEz) == kClEz,
              "the update windows hold every E value the interpolations read");
static_assert((interp_mask(0b001, 0b110) | interp_mask(0b001, 0b101) |
               interp_mask(0b001, 0b011)) == kWinBx,
              "B_x window");
static_assert((interp_mask(0b010, 0b110) | interp_mask(0b010, 0b101) |
               interp_mask(0b010, 0b011)) == kWinBy,
              "B_y window");
static_assert((interp_mask(0b100, 0b110) | interp_mask(0b100, 0b101) |
               interp_mask(0b100, 0b011)) == kWinBz,
              "B_z window");

// Everything the staggered passes need besides the substep coefficients.
template <typename T>
struct YeeArgs {
  GridGeom g;          // box [lo, hi) = the interior (shift_ghost 0)
  T inv[3];            // inv_delta
  T cc[3];             // dt * inv_delta
  T dt;
  const T* E[3];       // state (read by the update pass)
  const T* B[3];
  const T* B0[3];      // background field, or null
  T* Eo[3];            // state (written by the clamp and boundary passes)
  T* Bo[3];
  T* Es[3];            // E* of the update pass (and its guard shell)
  T* Bs[3];            // B' of the update pass (and its guard shell)
  T* En[3];            // start-of-step copies (written in the first substep)
  T* Bn[3];
  T* Et[3];            // scratch of the star boundary
  T* Bt[3];
  int kchunk;          // planes per thread
  // absorbing layer (kernel_boundary_absorbing_thread, boundary.cu:38-62)
  int absorbing;
  T pml_lo[3], pml_hi[3], pml_scale, sigpml;
  // star boundary: the box of vertices within 2 radius of the origin, and
  // the same box grown by one point (the absorbing layer of its points is
  // applied by the star passes, after them)
  int star;
  int plo[3], phi[3];  // star box, inside the interior
  int hlo[3], hhi[3];  // star box + 1, inside the interior
  EzConst<T> c;        // star parameters (b0, moments, radius, omega)
};

template <typename T>
__device__ __forceinline__ T vpos(const YeeArgs<T>& a, int axis, int n, int stagger) {
  // Grid::pos(axis, n, stagger): lower + delta * (n - guard + (stagger ? 0 : 0.5))
  // (src/data/grid.h:116-134)
  return a.c.lower[axis] +
         a.c.delta[axis] * ((T)(n - a.g.guard[axis]) + (stagger ? (T)0 : (T)0.5));
}

__device__ __forceinline__ bool in_box(const int lo[3], const int hi[3], int i, int j, int k) {
  return i >= lo[0] && i < hi[0] && j >= lo[1] && j < hi[1] && k >= lo[2] && k < hi[2];
}

// rho = div E at one vertex, from the backward differences of the three
// components there (kernel_compute_rho_thread, field_solver.cu:35-39).
template <typename T>
__device__ __forceinline__ T rho_of(const YeeArgs<T>& a, T dex, T dey, T dez) {
  return a.inv[0] * dex + a.inv[1] * dey + a.inv[2] * dez;
}

// Current density times dt along component A at its E position
// (field_solver.cu:94-145): dt rho (E x B)_A / (B^2 + TINY).
template <int A, typename T, uint32_t MX, uint32_t MY, uint32_t MZ>
__device__ __forceinline__ T current(const YeeArgs<T>& a, const Win<kRhoWin, T>& r,
                                     const Win<MX, T>& ex, const Win<MY, T>& ey,
                                     const Win<MZ, T>& ez, const Win<kWinBx, T>& bx,
                                     const Win<kWinBy, T>& by, const Win<kWinBz, T>& bz) {
  constexpr int out = kStE[A];
  const T ir = interp<kStRho, out>(r);
  const T iex = interp<0b110, out>(ex), iey = interp<0b101, out>(ey), iez = interp<0b011, out>(ez);
  const T ibx = interp<0b001, out>(bx), iby = interp<0b010, out>(by), ibz = interp<0b100, out>(bz);
  const T b2 = ibx * ibx + iby * iby + ibz * ibz + Tiny<T>::v;
  if constexpr (A == 0) return a.dt * ir * (iey * ibz - iby * iez) / b2;
  else if constexpr (A == 1) return a.dt * ir * (iez * ibx - iex * ibz) / b2;
  else return a.dt * ir * (iex * iby - ibx * iey) / b2;
}

// ---------------------------------------------------------------- update

template <typename T, bool FIRST, bool HAS_B0>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? (FIRST ? COFFEE_YEE_FIRST_MIN_BLOCKS
                                                         : COFFEE_YEE_UPDATE_MIN_BLOCKS)
                                      : 1)
yee_update_kernel(const YeeArgs<T> a, const T c1, const T c2, const T c3) {
  const int i = a.g.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.g.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (i >= a.g.hi[0] || j >= a.g.hi[1]) return;
  const int k0 = a.g.lo[2] + (int)blockIdx.z * a.kchunk;
  const int k1 = min(k0 + a.kchunk, a.g.hi[2]);
  if (k0 >= k1) return;
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  uint32_t o = (uint32_t)k0 * (uint32_t)sz + (uint32_t)j * (uint32_t)sy + (uint32_t)i;
  Win<kUpEx, T> ex;
  Win<kUpEy, T> ey;
  Win<kUpEz, T> ez;
  Win<kWinBx, T> bx;
  Win<kWinBy, T> by;
  Win<kWinBz, T> bz;
  Win<kUpB0x, T> b0x;
  Win<kUpB0y, T> b0y;
  Win<kUpB0z, T> b0z;
  Win<kRhoWin, T> r;
  ex.load(a.E[0], o, sy, sz);
  ey.load(a.E[1], o, sy, sz);
  ez.load(a.E[2], o, sy, sz);
  bx.load(a.B[0], o, sy, sz);
  by.load(a.B[1], o, sy, sz);
  bz.load(a.B[2], o, sy, sz);
  if constexpr (HAS_B0) {
    b0x.load(a.B0[0], o, sy, sz);
    b0y.load(a.B0[1], o, sy, sz);
    b0z.load(a.B0[2], o, sy, sz);
  }
  // rho vanishes outside the box: the reference's rho array is written only there
  const bool xin = i + 1 < a.g.hi[0], yin = j + 1 < a.g.hi[1];
  r.v[widx(0, 0, 0)] = rho_of(a, ex.template at<0, 0, 0>() - ex.template at<-1, 0, 0>(),
                              ey.template at<0, 0, 0>() - ey.template at<0, -1, 0>(),
                              ez.template at<0, 0, 0>() - ez.template at<0, 0, -1>());
  const T zero = (T)0;
  for (int k = k0;;) {
    r.v[widx(1, 0, 0)] = xin ? rho_of(a, ex.template at<1, 0, 0>() - ex.template at<0, 0, 0>(),
                                      ey.template at<1, 0, 0>() - ey.template at<1, -1, 0>(),
                                      ez.template at<1, 0, 0>() - ez.template at<1, 0, -1>())
                             : zero;
    r.v[widx(0, 1, 0)] = yin ? rho_of(a, ex.template at<0, 1, 0>() - ex.template at<-1, 1, 0>(),
                                      ey.template at<0, 1, 0>() - ey.template at<0, 0, 0>(),
                                      ez.template at<0, 1, 0>() - ez.template at<0, 1, -1>())
                             : zero;
    r.v[widx(0, 0, 1)] = (k + 1 < a.g.hi[2])
                             ? rho_of(a, ex.template at<0, 0, 1>() - ex.template at<-1, 0, 1>(),
                                      ey.template at<0, 0, 1>() - ey.template at<0, -1, 1>(),
                                      ez.template at<0, 0, 1>() - ez.template at<0, 0, 0>())
                             : zero;
    const T CCx = a.cc[0], CCy = a.cc[1], CCz = a.cc[2];
    // dB = -curl E dt (field_solver.cu:78-84)
    const T dbx = CCz * (ey.template at<0, 0, 1>() - ey.template at<0, 0, 0>()) -
                  CCy * (ez.template at<0, 1, 0>() - ez.template at<0, 0, 0>());
    const T dby = CCx * (ez.template at<1, 0, 0>() - ez.template at<0, 0, 0>()) -
                  CCz * (ex.template at<0, 0, 1>() - ex.template at<0, 0, 0>());
    const T dbz = CCy * (ex.template at<0, 1, 0>() - ex.template at<0, 0, 0>()) -
                  CCx * (ey.template at<1, 0, 0>() - ey.template at<0, 0, 0>());
    // dE = (curl B - curl B0) dt - J dt (field_solver.cu:86-95, 147-149)
    T dex = CCz * (by.template at<0, 0, -1>() - by.template at<0, 0, 0>()) -
            CCy * (bz.template at<0, -1, 0>() - bz.template at<0, 0, 0>());
    T dey = CCx * (bz.template at<-1, 0, 0>() - bz.template at<0, 0, 0>()) -
            CCz * (bx.template at<0, 0, -1>() - bx.template at<0, 0, 0>());
    T dez = CCy * (bx.template at<0, -1, 0>() - bx.template at<0, 0, 0>()) -
            CCx * (by.template at<-1, 0, 0>() - by.template at<0, 0, 0>());
    if constexpr (HAS_B0) {
      dex = dex - (CCz * (b0y.template at<0, 0, -1>() - b0y.template at<0, 0, 0>()) -
                   CCy * (b0z.template at<0, -1, 0>() - b0z.template at<0, 0, 0>()));
      dey = dey - (CCx * (b0z.template at<-1, 0, 0>() - b0z.template at<0, 0, 0>()) -
                   CCz * (b0x.template at<0, 0, -1>() - b0x.template at<0, 0, 0>()));
      dez = dez - (CCy * (b0x.template at<0, -1, 0>() - b0x.template at<0, 0, 0>()) -
                   CCx * (b0y.template at<-1, 0, 0>() - b0y.template at<0, 0, 0>()));
    }
    dex = dex - current<0>(a, r, ex, ey, ez, bx, by, bz);
    dey = dey - current<1>(a, r, ex, ey, ez, bx, by, bz);
    dez = dez - current<2>(a, r, ex, ey, ez, bx, by, bz);
    // E = c1 En + c2 E + c3 dE, B likewise (field_solver.cu:170-183)
    const T e0 = ex.template at<0, 0, 0>(), e1 = ey.template at<0, 0, 0>(),
            e2 = ez.template at<0, 0, 0>();
    const T b0 = bx.template at<0, 0, 0>(), b1 = by.template at<0, 0, 0>(),
            b2 = bz.template at<0, 0, 0>();
    T en0, en1, en2, bn0, bn1, bn2;
    if constexpr (FIRST) {
      // En, Bn are copies of E, B taken at the start of the step
      en0 = e0; en1 = e1; en2 = e2; bn0 = b0; bn1 = b1; bn2 = b2;
      a.En[0][o] = e0; a.En[1][o] = e1; a.En[2][o] = e2;
      a.Bn[0][o] = b0; a.Bn[1][o] = b1; a.Bn[2][o] = b2;
    } else {
      en0 = __ldg(a.En[0] + o); en1 = __ldg(a.En[1] + o); en2 = __ldg(a.En[2] + o);
      bn0 = __ldg(a.Bn[0] + o); bn1 = __ldg(a.Bn[1] + o); bn2 = __ldg(a.Bn[2] + o);
    }
    a.Es[0][o] = c1 * en0 + c2 * e0 + c3 * dex;
    a.Es[1][o] = c1 * en1 + c2 * e1 + c3 * dey;
    a.Es[2][o] = c1 * en2 + c2 * e2 + c3 * dez;
    a.Bs[0][o] = c1 * bn0 + c2 * b0 + c3 * dbx;
    a.Bs[1][o] = c1 * bn1 + c2 * b1 + c3 * dby;
    a.Bs[2][o] = c1 * bn2 + c2 * b2 + c3 * dbz;
    if (++k >= k1) break;
    o += (uint32_t)sz;
    r.v[widx(0, 0, 0)] = r.v[widx(0, 0, 1)];
    ex.advance(a.E[0], o, sy, sz);
    ey.advance(a.E[1], o, sy, sz);
    ez.advance(a.E[2], o, sy, sz);
    bx.advance(a.B[0], o, sy, sz);
    by.advance(a.B[1], o, sy, sz);
    bz.advance(a.B[2], o, sy, sz);
    if constexpr (HAS_B0) {
      b0x.advance(a.B0[0], o, sy, sz);
      b0y.advance(a.B0[1], o, sy, sz);
      b0z.advance(a.B0[2], o, sy, sz);
    }
  }
}

// The clamp pass reads E* and B' one point beyond the box, where the
// reference reads the state's guard values of before the exchange; this pass
// copies them into the scratch arrays (with e_state 0 the E* shell is 0
// instead: what the Kerr-Schild solver's rescale reads there, its dD being
// zero outside the box).  blockIdx.z picks one of the six faces of the box
// grown by one point (the z faces whole, the y faces between them, the x
// faces between those); (x, y) threads cover the face.
template <typename T>
__global__ void yee_shell_kernel(const YeeArgs<T> a, const int e_state) {
  const int u = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int v = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int face = (int)blockIdx.z;
  const int* lo = a.g.lo;
  const int* hi = a.g.hi;
  const int nx = hi[0] - lo[0], ny = hi[1] - lo[1], nz = hi[2] - lo[2];
  int i, j, k;
  if (face < 2) {         // z = lo - 1 or hi, the whole grown face
    if (u >= nx + 2 || v >= ny + 2) return;
    i = lo[0] - 1 + u; j = lo[1] - 1 + v; k = face == 0 ? lo[2] - 1 : hi[2];
  } else if (face < 4) {  // y = lo - 1 or hi, between the z faces
    if (u >= nx + 2 || v >= nz) return;
    i = lo[0] - 1 + u; j = face == 2 ? lo[1] - 1 : hi[1]; k = lo[2] + v;
  } else {                // x = lo - 1 or hi, between the y faces
    if (u >= ny || v >= nz) return;
    i = face == 4 ? lo[0] - 1 : hi[0]; j = lo[1] + u; k = lo[2] + v;
  }
  const uint32_t o = (uint32_t)k * (uint32_t)a.g.sz + (uint32_t)j * (uint32_t)a.g.sy + (uint32_t)i;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    a.Es[c][o] = e_state ? a.E[c][o] : (T)0;
    a.Bs[c][o] = a.B[c][o];
  }
}

// ----------------------------------------------------------------- clamp

// Absorbing layer at vertex (i, j, k) (kernel_boundary_absorbing_thread,
// boundary.cu:38-62): the conductivity, or 0 where the point is left alone.
template <typename T>
__device__ __forceinline__ T yee_sigma(const YeeArgs<T>& a, int i, int j, int k) {
  const T x = vpos(a, 0, i, 1), y = vpos(a, 1, j, 1), z = vpos(a, 2, k, 1);
  if (!(x > a.pml_hi[0] || x < a.pml_lo[0] || y > a.pml_hi[1] || y < a.pml_lo[1] ||
        z > a.pml_hi[2] || z < a.pml_lo[2]))
    return 0;
  // pmlsigma (boundary.cu:7-15): sig0 * cube(distance / scale)
  auto sig1 = [&](T v, T lo, T hi) -> T {
    if (v > hi) { const T q = (v - hi) / a.pml_scale; return a.sigpml * (q * q * q); }
    if (v < lo) { const T q = (lo - v) / a.pml_scale; return a.sigpml * (q * q * q); }
    return (T)0;
  };
  const T sig = sig1(x, a.pml_lo[0], a.pml_hi[0]) + sig1(y, a.pml_lo[1], a.pml_hi[1]) +
                sig1(z, a.pml_lo[2], a.pml_hi[2]);
  return sig > Tiny<T>::v ? sig : (T)0;
}

// u relaxed toward its start-of-step value un: exp(-sig) un +
// (1 - exp(-sig)) / sig (u - un) with the reference's promotions (the
// exponential in Scalar, the rest through its double literal).
template <typename T>
__device__ __forceinline__ T absorb(T sig, T u, T un) {
  const T ed = exp(-sig);
  const double f = (1.0 - (double)ed) / (double)sig;
  return (T)((double)(ed * un) + f * (double)(u - un));
}

// One E component after [clean_epar and] check_eGTb: E* and B' are
// interpolated to the component's position; the cleaned value
// E* - (E*.B') B'_A / (B'^2 + TINY) (last substep) is scaled by
// sqrt(B^2 / E^2) where E^2 > B^2, E^2 taken from E* before cleaning.
template <int A, bool LAST, typename T>
__device__ __forceinline__ T clamp_component(const Win<kClEx, T>& ex, const Win<kClEy, T>& ey,
                                             const Win<kClEz, T>& ez, const Win<kWinBx, T>& bx,
                                             const Win<kWinBy, T>& by, const Win<kWinBz, T>& bz) {
  constexpr int out = kStE[A];
  const T iex = interp<0b110, out>(ex), iey = interp<0b101, out>(ey), iez = interp<0b011, out>(ez);
  const T ibx = interp<0b001, out>(bx), iby = interp<0b010, out>(by), ibz = interp<0b100, out>(bz);
  const T emag = iex * iex + iey * iey + iez * iez + Tiny<T>::v;
  const T bmag = ibx * ibx + iby * iby + ibz * ibz + Tiny<T>::v;
  T e;
  if constexpr (A == 0) e = ex.template at<0, 0, 0>();
  else if constexpr (A == 1) e = ey.template at<0, 0, 0>();
  else e = ez.template at<0, 0, 0>();
  if constexpr (LAST) {
    const T ib = A == 0 ? ibx : (A == 1 ? iby : ibz);
    e = e - (iex * ibx + iey * iby + iez * ibz) * ib / bmag;
  }
  const T temp = emag > bmag ? sqrt(bmag / emag) : (T)1;
  return temp * e;
}

template <typename T, bool LAST, bool IMAGES>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? COFFEE_YEE_CLAMP_MIN_BLOCKS : 1)
yee_clamp_kernel(const YeeArgs<T> a) {
  const int i = a.g.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.g.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (i >= a.g.hi[0] || j >= a.g.hi[1]) return;
  const int k0 = a.g.lo[2] + (int)blockIdx.z * a.kchunk;
  const int k1 = min(k0 + a.kchunk, a.g.hi[2]);
  if (k0 >= k1) return;
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  uint32_t o = (uint32_t)k0 * (uint32_t)sz + (uint32_t)j * (uint32_t)sy + (uint32_t)i;
  Win<kClEx, T> ex;
  Win<kClEy, T> ey;
  Win<kClEz, T> ez;
  Win<kWinBx, T> bx;
  Win<kWinBy, T> by;
  Win<kWinBz, T> bz;
  ex.load(a.Es[0], o, sy, sz);
  ey.load(a.Es[1], o, sy, sz);
  ez.load(a.Es[2], o, sy, sz);
  bx.load(a.Bs[0], o, sy, sz);
  by.load(a.Bs[1], o, sy, sz);
  bz.load(a.Bs[2], o, sy, sz);
  int xs[2], ys[2], zs[2];
  const int nx = IMAGES ? periodic_targets(a.g, 0, i, xs) : 1;
  const int ny = IMAGES ? periodic_targets(a.g, 1, j, ys) : 1;
  if (!IMAGES) { xs[0] = i; ys[0] = j; }
  for (int k = k0;;) {
    T u[6];
    u[0] = clamp_component<0, LAST>(ex, ey, ez, bx, by, bz);
    u[1] = clamp_component<1, LAST>(ex, ey, ez, bx, by, bz);
    u[2] = clamp_component<2, LAST>(ex, ey, ez, bx, by, bz);
    u[3] = bx.template at<0, 0, 0>();
    u[4] = by.template at<0, 0, 0>();
    u[5] = bz.template at<0, 0, 0>();
    if (LAST && a.absorbing && !(a.star && in_box(a.hlo, a.hhi, i, j, k))) {
      const T sig = yee_sigma(a, i, j, k);
      if (sig > (T)0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          u[c] = absorb(sig, u[c], __ldg(a.En[c] + o));
          u[3 + c] = absorb(sig, u[3 + c], __ldg(a.Bn[c] + o));
        }
      }
    }
    if (!IMAGES || (nx == 1 && ny == 1 && only_self(a.g, 2, k))) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        a.Eo[c][o] = u[c];
        a.Bo[c][o] = u[3 + c];
      }
    } else {
      const int nz = periodic_targets(a.g, 2, k, zs);
      for (int cz = 0; cz < nz; ++cz)
        for (int cy = 0; cy < ny; ++cy)
          for (int cx = 0; cx < nx; ++cx) {
            const uint32_t q = (uint32_t)zs[cz] * (uint32_t)sz + (uint32_t)ys[cy] * (uint32_t)sy +
                               (uint32_t)xs[cx];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              a.Eo[c][q] = u[c];
              a.Bo[c][q] = u[3 + c];
            }
          }
    }
    if (++k >= k1) break;
    o += (uint32_t)sz;
    ex.advance(a.Es[0], o, sy, sz);
    ey.advance(a.Es[1], o, sy, sz);
    ez.advance(a.Es[2], o, sy, sz);
    bx.advance(a.Bs[0], o, sy, sz);
    by.advance(a.Bs[1], o, sy, sz);
    bz.advance(a.Bs[2], o, sy, sz);
  }
}

// ------------------------------------------------------ rotating star
// kernel_boundary_pulsar_{B,E}_thread (field_solver.cu:344-638): inside
// r < 2 radius (measured at the vertex), each component is blended from the
// star's value (the rotating dipole for B, -v x B for E) and its own, the
// radial and the tangential parts with their own tanh profiles.

// shape(r, r0, del) with tanh in Scalar, as the GPU build evaluates it
// (src/algorithms/pulsar_impl.hpp:52-55)
template <typename T>
__device__ __forceinline__ T yee_shape(T r, T r0, T del) {
  return (T)(0.5 * (1.0 - (double)tanh((r - r0) / del)));
}

template <int A, typename T>
__device__ __forceinline__ T star_blend(const T st[3], const T in[3], const T p[3], T r2, T s_perp,
                                        T s_par) {
  const T rs = (st[0] * p[0] + st[1] * p[1] + st[2] * p[2]) * p[A] / r2;
  const T ri = (in[0] * p[0] + in[1] * p[1] + in[2] * p[2]) * p[A] / r2;
  T v = rs * s_perp + ri * (1 - s_perp);
  v += (st[A] - rs) * s_par + (in[A] - ri) * (1 - s_par);
  return v;
}

template <typename T>
__device__ __forceinline__ T point_at(const T* f, uint32_t o, int dx, int dy, int dz, int sy,
                                      int sz) {
  return f[o + (uint32_t)(dx + dy * sy + dz * sz)];
}

// interpolate() at a single point with runtime strides (the star passes
// touch a few thousand points; no windows)
template <int IN, int OUT, typename T>
__device__ __forceinline__ T interp_at(const T* f, uint32_t o, int sy, int sz) {
  constexpr int im = ilo(IN, OUT, 0), ip = ihi(IN, OUT, 0);
  constexpr int jm = ilo(IN, OUT, 1), jp = ihi(IN, OUT, 1);
  constexpr int km = ilo(IN, OUT, 2), kp = ihi(IN, OUT, 2);
  const T h = (T)0.5;
  const T f11 = h * (point_at(f, o, ip, jp, km, sy, sz) + point_at(f, o, ip, jp, kp, sy, sz));
  const T f10 = h * (point_at(f, o, ip, jm, km, sy, sz) + point_at(f, o, ip, jm, kp, sy, sz));
  const T f01 = h * (point_at(f, o, im, jp, km, sy, sz) + point_at(f, o, im, jp, kp, sy, sz));
  const T f00 = h * (point_at(f, o, im, jm, km, sy, sz) + point_at(f, o, im, jm, kp, sy, sz));
  return h * (h * (f11 + f10) + h * (f01 + f00));
}

template <typename T>
__device__ __forceinline__ bool star_point(const YeeArgs<T>& a, int i, int j, int k) {
  const T x0 = vpos(a, 0, i, 1), y0 = vpos(a, 1, j, 1), z0 = vpos(a, 2, k, 1);
  const T rl = (T)(2.0 * (double)a.c.radius);
  return x0 * x0 + y0 * y0 + z0 * z0 < rl * rl;
}

template <int A, typename T>
__device__ __forceinline__ T star_b_component(const YeeArgs<T>& a, int i, int j, int k, uint32_t o,
                                              T phase) {
  constexpr int st = kStB[A];
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  const T p[3] = {vpos(a, 0, i, st & 1), vpos(a, 1, j, (st >> 1) & 1),
                  vpos(a, 2, k, (st >> 2) & 1)};
  const T r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  const T r = sqrt(r2);
  T bs[3];
  star_field(a.c, p[0], p[1], p[2], phase, bs);
  T in[3];
  in[0] = A == 0 ? a.Bo[0][o] : interp_at<0b001, st>(a.Bo[0], o, sy, sz);
  in[1] = A == 1 ? a.Bo[1][o] : interp_at<0b010, st>(a.Bo[1], o, sy, sz);
  in[2] = A == 2 ? a.Bo[2][o] : interp_at<0b100, st>(a.Bo[2], o, sy, sz);
  const T d1 = (T)4 * a.c.delta[0];
  const T s = yee_shape(r, a.c.radius - d1, (T)1.0 * a.c.delta[0]);
  return star_blend<A>(bs, in, p, r2, s, s);
}

template <int A, typename T>
__device__ __forceinline__ T star_e_component(const YeeArgs<T>& a, int i, int j, int k,
                                              uint32_t o) {
  constexpr int st = kStE[A];
  const int sy = (int)a.g.sy, sz = (int)a.g.sz;
  const T p[3] = {vpos(a, 0, i, st & 1), vpos(a, 1, j, (st >> 1) & 1),
                  vpos(a, 2, k, (st >> 2) & 1)};
  const T r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  const T r = sqrt(r2);
  const T w = a.c.omega;
  const T vx = -w * p[1], vy = w * p[0];
  const T in[3] = {interp_at<0b110, st>(a.Eo[0], o, sy, sz), interp_at<0b101, st>(a.Eo[1], o, sy, sz),
                   interp_at<0b011, st>(a.Eo[2], o, sy, sz)};
  const T ibx = interp_at<0b001, st>(a.Bt[0], o, sy, sz);
  const T iby = interp_at<0b010, st>(a.Bt[1], o, sy, sz);
  const T ibz = interp_at<0b100, st>(a.Bt[2], o, sy, sz);
  const T es[3] = {-vy * ibz, vx * ibz, -vx * iby + vy * ibx};
  const T r0 = a.c.radius - (T)0;
  const T s_perp = yee_shape(r, r0, (T)0.5 * a.c.delta[0]);
  const T s_par = yee_shape(r, r0, (T)1.0 * a.c.delta[0]);
  return star_blend<A>(es, in, p, r2, s_perp, s_par);
}

// B of the star box grown by one point into Bt: the blended value inside
// r < 2 radius, the state's value elsewhere in the interior, 0 outside it
// (the reference copies its whole scratch array back, whose guards are 0).
template <typename T>
__global__ void yee_star_b_kernel(const YeeArgs<T> a, const T t) {
  const int i = a.plo[0] - 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.plo[1] - 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = a.plo[2] - 1 + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i > a.phi[0] || j > a.phi[1] || k > a.phi[2]) return;
  const uint32_t o = (uint32_t)k * (uint32_t)a.g.sz + (uint32_t)j * (uint32_t)a.g.sy + (uint32_t)i;
  T v[3];
  if (!in_box(a.g.lo, a.g.hi, i, j, k)) {
    v[0] = v[1] = v[2] = (T)0;
  } else if (in_box(a.plo, a.phi, i, j, k) && star_point(a, i, j, k)) {
    const T phase = a.c.omega * t;
    v[0] = star_b_component<0>(a, i, j, k, o, phase);
    v[1] = star_b_component<1>(a, i, j, k, o, phase);
    v[2] = star_b_component<2>(a, i, j, k, o, phase);
  } else {
    v[0] = a.Bo[0][o]; v[1] = a.Bo[1][o]; v[2] = a.Bo[2][o];
  }
  a.Bt[0][o] = v[0]; a.Bt[1][o] = v[1]; a.Bt[2][o] = v[2];
}

// E of the star box into Et, from the state's E and the new B in Bt.
template <typename T>
__global__ void yee_star_e_kernel(const YeeArgs<T> a) {
  const int i = a.plo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.plo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = a.plo[2] + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i >= a.phi[0] || j >= a.phi[1] || k >= a.phi[2]) return;
  const uint32_t o = (uint32_t)k * (uint32_t)a.g.sz + (uint32_t)j * (uint32_t)a.g.sy + (uint32_t)i;
  T v[3];
  if (star_point(a, i, j, k)) {
    v[0] = star_e_component<0>(a, i, j, k, o);
    v[1] = star_e_component<1>(a, i, j, k, o);
    v[2] = star_e_component<2>(a, i, j, k, o);
  } else {
    v[0] = a.Eo[0][o]; v[1] = a.Eo[1][o]; v[2] = a.Eo[2][o];
  }
  a.Et[0][o] = v[0]; a.Et[1][o] = v[1]; a.Et[2][o] = v[2];
}

// Star box back into the state, then (last substep) the absorbing layer of
// the grown box, whose points the clamp pass left alone.
template <typename T, bool LAST>
__global__ void yee_star_store_kernel(const YeeArgs<T> a) {
  const int i = a.hlo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = a.hlo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = a.hlo[2] + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i >= a.hhi[0] || j >= a.hhi[1] || k >= a.hhi[2]) return;
  const uint32_t o = (uint32_t)k * (uint32_t)a.g.sz + (uint32_t)j * (uint32_t)a.g.sy + (uint32_t)i;
  T u[6];
  const bool star = in_box(a.plo, a.phi, i, j, k);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    u[c] = star ? a.Et[c][o] : a.Eo[c][o];
    u[3 + c] = star ? a.Bt[c][o] : a.Bo[c][o];
  }
  if (LAST && a.absorbing) {
    const T sig = yee_sigma(a, i, j, k);
    if (sig > (T)0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        u[c] = absorb(sig, u[c], a.En[c][o]);
        u[3 + c] = absorb(sig, u[3 + c], a.Bn[c][o]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    a.Eo[c][o] = u[c];
    a.Bo[c][o] = u[3 + c];
  }
}

// ------------------------------------------------------------ guard pass
// The single-rank guard exchange of E and B after a substep: every guard
// point along a periodic axis takes the value of the point with its
// periodic coordinates wrapped into the interior (the x -> y -> z plane
// copies of the exchange compose to exactly that).  With ZERO (star
// boundary), a point outside the interior along a non-periodic axis holds 0,
// as the reference's copy_from of its scratch arrays leaves it.  One thread
// per (i, j) column; interior columns visit only their guard planes.
template <typename T, bool ZERO>
__global__ void yee_guard_kernel(const YeeArgs<T> a) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const GridGeom& g = a.g;
  if (i >= g.dims[0] || j >= g.dims[1]) return;
  const bool xi = i >= g.lo[0] && i < g.hi[0], yi = j >= g.lo[1] && j < g.hi[1];
  auto wrap = [&](int axis, int n) {
    if (!g.periodic[axis]) return n;
    if (n < g.lo[axis]) return n + g.N[axis];
    if (n >= g.hi[axis]) return n - g.N[axis];
    return n;
  };
  for (int k = 0; k < g.dims[2]; ++k) {
    const bool zi = k >= g.lo[2] && k < g.hi[2];
    if (xi && yi && zi) {  // skip the interior of the column
      k = g.hi[2] - 1;
      continue;
    }
    const bool np_out = (!xi && !g.periodic[0]) || (!yi && !g.periodic[1]) ||
                        (!zi && !g.periodic[2]);
    const bool p_out = (!xi && g.periodic[0]) || (!yi && g.periodic[1]) || (!zi && g.periodic[2]);
    const uint32_t o = (uint32_t)k * (uint32_t)g.sz + (uint32_t)j * (uint32_t)g.sy + (uint32_t)i;
    if (ZERO && np_out) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        a.Eo[c][o] = (T)0;
        a.Bo[c][o] = (T)0;
      }
      continue;
    }
    if (!p_out) continue;  // a non-periodic guard point: left as it is
    // the source has every periodic coordinate inside, so this pass never
    // writes it
    const uint32_t q = (uint32_t)wrap(2, k) * (uint32_t)g.sz + (uint32_t)wrap(1, j) * (uint32_t)g.sy +
                       (uint32_t)wrap(0, i);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      a.Eo[c][o] = a.Eo[c][q];
      a.Bo[c][o] = a.Bo[c][q];
    }
  }
}

}  // namespace coffee
