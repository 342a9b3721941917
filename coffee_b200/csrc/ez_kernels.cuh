// Flat-Cartesian EZ kernels: one fused LSRK stage, and the Kreiss-Oliger
// pass that closes a step.
//
// Both kernels stream along z.  A CTA owns a TX x TY column of points and a
// chunk of z planes.  Each z plane of the 7 fields (E, B, P), with a halo of
// H points in x and y, is copied global -> shared memory by cp.async into a
// ring of 2H+1+PF planes, PF planes ahead of the plane being computed, so the
// HBM reads of the next planes overlap the arithmetic of this one.  Every
// stencil operand (x, y and z neighbours) is then read from shared memory.
// The LSRK accumulators dU are read in the same copy groups (no halo) and
// written back in place; the new E, B, P go to a second buffer (stencil
// reads of other points still need the old values), together with their
// periodic guard images, so no separate halo-exchange pass is needed.
#pragma once

#include "ez_physics.cuh"

namespace coffee {

template <typename T, int TX, int TY, int H, int PF, bool WITH_DU>
struct TileCfg {
  static constexpr int R = 2 * H + 1 + PF;  // ring depth in planes
  static constexpr int SX = TX + 2 * H;     // shared row pitch
  static constexpr int SY = TY + 2 * H;
  static constexpr int PLANE = SX * SY;     // one field, one plane
  static constexpr int NT = TX * TY;
  static constexpr int NLOAD = (PLANE + NT - 1) / NT;
  static constexpr int DU_SLOTS = WITH_DU ? PF + 1 : 0;
  static constexpr size_t smem_bytes =
      ((size_t)R * 7 * PLANE + (size_t)DU_SLOTS * 7 * NT) * sizeof(T);
};

// Flags of the stage kernel.
enum StageFlags { ST_LAST = 1, ST_AUX = 2, ST_WRITE_UN = 4 };

// 4th-order first derivative (reference diff1_4, finite_diff.h:13-18):
// ((f-2 - f+2) + 8 (f+1 - f-1)) * inv_delta / 12.
template <typename T>
__device__ __forceinline__ T d1_4(T m2, T m1, T p1, T p2, T s) {
  return ((m2 - p2) + (T)8 * (p1 - m1)) * s;
}

// 6th-order, 2nd-difference KO operator along one axis (reference diff6_2,
// finite_diff.h:25-30): f-3 - 6 f-2 + 15 f-1 - 20 f0 + 15 f+1 - 6 f+2 + f+3.
template <typename T>
__device__ __forceinline__ T d6_2(T m3, T m2, T m1, T c, T p1, T p2, T p3) {
  return ((m3 + p3) - (T)6 * (m2 + p2)) + ((T)15 * (m1 + p1) - (T)20 * c);
}

// Write the 7 new values of point (i, j, k) to `out` at the point and at
// its periodic guard images.
template <typename T>
__device__ __forceinline__ void store_with_images(const GridGeom& g, const F7<T>& out, int i,
                                                  int j, int k, const T u[7]) {
  int xs[2], ys[2], zs[2];
  const int nx = periodic_targets(g, 0, i, xs);
  const int ny = periodic_targets(g, 1, j, ys);
  const int nz = periodic_targets(g, 2, k, zs);
  for (int c = 0; c < nz; ++c)
    for (int b = 0; b < ny; ++b)
      for (int a = 0; a < nx; ++a) {
        const long long o = (long long)zs[c] * g.sz + (long long)ys[b] * g.sy + xs[a];
#pragma unroll
        for (int f = 0; f < 7; ++f) out.p[f][o] = u[f];
      }
}

// Everything a stage does at one point once its derivatives are known:
// the current J, the new accumulators dU (from dold unless FIRST), the new
// fields U + Bs dU, the clamps, the star boundary, the absorbing layer
// (ST_LAST) and the stores of dU, J/divE/divB (ST_AUX), Un (ST_WRITE_UN) and
// of U' with its guard images.  d{x,y,z}[f] are the inv_delta-scaled
// 4th-order derivatives of field f at the point, u[f] its values.
template <typename T, bool FIRST>
__device__ __forceinline__ void stage_point(const EzConst<T>& c, const T u[7], const T dx[7],
                                            const T dy[7], const T dz[7], const T dold[7],
                                            const T As, const T Bs, const T tst,
                                            const int flags, const int i, const int j,
                                            const int k, const long long o, const F7<T>& du,
                                            const F7<T>& un, const F5<T>& aux,
                                            const F7<T>& uout) {
  const bool cpu = c.semantics == SEM_CPU_REF;
  const T ex = u[0], ey = u[1], ez = u[2], bx = u[3], by = u[4], bz = u[5], P = u[6];
  const T rotBx = dy[5] - dz[4], rotBy = dz[3] - dx[5], rotBz = dx[4] - dy[3];
  const T rotEx = dy[2] - dz[1], rotEy = dz[0] - dx[2], rotEz = dx[1] - dy[0];
  const T divE = dx[0] + dy[1] + dz[2];
  const T divB = dx[3] + dy[4] + dz[5];
  T B2 = bx * bx + by * by + bz * bz;
  if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
  const T BrotB = bx * rotBx + by * rotBy + bz * rotBz;
  const T ErotE = ex * rotEx + ey * rotEy + ez * rotEz;
  const T cx = ey * bz - ez * by, cy = ez * bx - ex * bz, cz = ex * by - ey * bx;
  T Jx, Jy, Jz;
  if (c.use_edotb) {
    // J with E.B damping (field_solver_EZ.cpp:170-186, .cu:72-91)
    const T E2 = ex * ex + ey * ey + ez * ez;
    const T chi2 = B2 - E2;
    const T EdotB = ex * bx + ey * by + ez * bz;
    const T E02 = (T)0.5 * (sqrt(chi2 * chi2 + (T)4 * EdotB * EdotB) - chi2) + B2;
    const T Jp = BrotB - ErotE + EdotB * c.gam_dt;
    const T a = divE / E02, b = Jp / B2;
    Jx = a * cx + b * bx;
    Jy = a * cy + b * by;
    Jz = a * cz + b * bz;
  } else {
    const T Jp = BrotB - ErotE;
    const T rB2 = (T)1 / B2;
    Jx = (divE * cx + Jp * bx) * rB2;
    Jy = (divE * cy + Jp * by) * rB2;
    Jz = (divE * cz + Jp * bz) * rB2;
  }
  T Px = 0, Py = 0, Pz = 0;
  if (c.divB_clean) {
    Px = dx[6];
    Py = dy[6];
    Pz = dz[6];
    if (cpu) {
      const T s = p_taper(c, i, j, k);
      Px *= s;
      Py *= s;
      Pz *= s;
    }
  }
  // new accumulators
  T d[7];
  const T dt = c.dt;
  d[0] = (rotBx - Jx) * dt;
  d[1] = (rotBy - Jy) * dt;
  d[2] = (rotBz - Jz) * dt;
  d[3] = -(rotEx + Px) * dt;
  d[4] = -(rotEy + Py) * dt;
  d[5] = -(rotEz + Pz) * dt;
  d[6] = -P / c.tau - divB * c.ch2 * dt;
  if constexpr (!FIRST) {
#pragma unroll
    for (int f = 0; f < 7; ++f) d[f] = fma(dold[f], As, d[f]);
  }
  // the start-of-step copy is only read inside the absorbing layer
  const T sig = c.absorbing ? absorbing_sigma(c, i, j, k) : (T)0;
  if ((flags & ST_WRITE_UN) != 0 && sig > (T)0) {
#pragma unroll
    for (int f = 0; f < 7; ++f) un.p[f][o] = u[f];
  }
#pragma unroll
  for (int f = 0; f < 7; ++f) du.p[f][o] = d[f];
  if ((flags & ST_AUX) != 0) {
    aux.p[0][o] = Jx;
    aux.p[1][o] = Jy;
    aux.p[2][o] = Jz;
    aux.p[3][o] = divE;
    aux.p[4][o] = divB;
  }
  T nu[7];
#pragma unroll
  for (int f = 0; f < 7; ++f) nu[f] = fma(d[f], Bs, u[f]);
  apply_clamps(c, nu[0], nu[1], nu[2], nu[3], nu[4], nu[5]);
  star_boundary(c, i, j, k, tst, nu);
  if ((flags & ST_LAST) != 0 && sig > (T)0) {
    V7<T> uv, unv;
#pragma unroll
    for (int f = 0; f < 7; ++f) {
      uv.v[f] = nu[f];
      unv.v[f] = un.p[f][o];
    }
    uv = absorbing_apply(c, i, j, k, sig, uv, unv);
#pragma unroll
    for (int f = 0; f < 7; ++f) nu[f] = uv.v[f];
  }
  store_with_images(c.g, uout, i, j, k, nu);
}

// ---------------------------------------------------------------------------
// One LSRK stage (reference rk_step + clamps + star boundary + absorbing
// layer + send_guard_cells, src/algorithms/field_solver_EZ.cpp:1024-1055,
// .cu:669-694):
//   dU  <- As dU + dt RHS(U)        (FIRST: As = 0, so dU is not read)
//   U'  <- U + Bs dU
//   U'  <- clamps, star boundary at tst, absorbing layer (ST_LAST)
// reading U from `uin` and writing U' (with guard images) to `uout`.
// ---------------------------------------------------------------------------
template <typename T, int TX, int TY, int PF, bool FIRST>
__global__ void __launch_bounds__(TX * TY, (sizeof(T) == 4) ? (512 / (TX * TY) > 0 ? 512 / (TX * TY) : 1) : 1)
    ez_stage_kernel(const __grid_constant__ EzConst<T> c, const F7<const T> uin, const F7<T> uout,
                    const F7<T> du, const F7<T> un, const F5<T> aux, const T As, const T Bs,
                    const T tst, const int kchunk, const int flags) {
  using C = TileCfg<T, TX, TY, 2, PF, !FIRST>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sU = reinterpret_cast<T*>(smem_raw);
  T* sD = sU + (size_t)C::R * 7 * C::PLANE;

  const GridGeom& g = c.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = g.lo[0] + blockIdx.x * TX + tx;
  const int j = g.lo[1] + blockIdx.y * TY + ty;
  const int k0 = g.lo[2] + blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.hi[2]);
  const bool active = (i < g.hi[0]) && (j < g.hi[1]);
  const int gx0 = g.lo[0] + blockIdx.x * TX - 2;
  const int gy0 = g.lo[1] + blockIdx.y * TY - 2;
  const long long own = (long long)j * g.sy + i;

  int soff[C::NLOAD];
  long long goff[C::NLOAD];
  bool lv[C::NLOAD];
#pragma unroll
  for (int m = 0; m < C::NLOAD; ++m) {
    const int e = tid + m * C::NT;
    const int r = e / C::SX, col = e - r * C::SX;
    const int gx = gx0 + col, gy = gy0 + r;
    lv[m] = (e < C::PLANE) && gx < g.dims[0] && gy < g.dims[1];
    soff[m] = e;
    goff[m] = (long long)gy * g.sy + gx;
  }
  const int kend = k1 + 2;  // planes [k0-2, k1+2) are read

  auto issue = [&](int kp) {
    if (kp < kend) {
      const int slot = kp % C::R;
#pragma unroll
      for (int f = 0; f < 7; ++f) {
        T* base = sU + (size_t)(slot * 7 + f) * C::PLANE;
        const T* gb = uin.p[f] + (long long)kp * g.sz;
#pragma unroll
        for (int m = 0; m < C::NLOAD; ++m)
          if (lv[m]) cp_async<sizeof(T)>(smem_u32(base + soff[m]), gb + goff[m]);
      }
    }
    if constexpr (!FIRST) {
      const int kd = kp - 2;
      if (kd >= k0 && kd < k1 && active) {
        const int slot = kd % (PF + 1);
#pragma unroll
        for (int f = 0; f < 7; ++f)
          cp_async<sizeof(T)>(smem_u32(sD + (size_t)(slot * 7 + f) * C::NT + tid),
                              du.p[f] + (long long)kd * g.sz + own);
      }
    }
    cp_async_commit();
  };

#pragma unroll 1
  for (int p = 0; p < C::R; ++p) issue(k0 - 2 + p);

  const T six = c.inv_delta[0] / (T)12, siy = c.inv_delta[1] / (T)12,
          siz = c.inv_delta[2] / (T)12;

#pragma unroll 1
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<PF>();
    __syncthreads();
    if (active) {
      const int sl[5] = {(k - 2) % C::R, (k - 1) % C::R, k % C::R, (k + 1) % C::R,
                         (k + 2) % C::R};
      const int rc = (ty + 2) * C::SX + tx + 2;  // own point within a plane
      T u[7], dx[7], dy[7], dz[7];
#pragma unroll
      for (int f = 0; f < 7; ++f) {
        const T* pc = sU + (size_t)(sl[2] * 7 + f) * C::PLANE + rc;
        u[f] = pc[0];
        dx[f] = d1_4(pc[-2], pc[-1], pc[1], pc[2], six);
        dy[f] = d1_4(pc[-2 * C::SX], pc[-C::SX], pc[C::SX], pc[2 * C::SX], siy);
        const T zm2 = sU[(size_t)(sl[0] * 7 + f) * C::PLANE + rc];
        const T zm1 = sU[(size_t)(sl[1] * 7 + f) * C::PLANE + rc];
        const T zp1 = sU[(size_t)(sl[3] * 7 + f) * C::PLANE + rc];
        const T zp2 = sU[(size_t)(sl[4] * 7 + f) * C::PLANE + rc];
        dz[f] = d1_4(zm2, zm1, zp1, zp2, siz);
      }
      T dold[7];
      if constexpr (!FIRST) {
        const int sd = k % (PF + 1);
#pragma unroll
        for (int f = 0; f < 7; ++f) dold[f] = sD[(size_t)(sd * 7 + f) * C::NT + tid];
      }
      stage_point<T, FIRST>(c, u, dx, dy, dz, dold, As, Bs, tst, flags, i, j, k,
                            (long long)k * g.sz + own, du, un, aux, uout);
    }
    __syncthreads();
    issue(k + 3 + PF);
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// The same LSRK stage with the z stencil in registers.  Each thread keeps,
// for its own column, the values of planes k-2..k+2 of the 7 fields in a
// sliding register window; shared memory holds only the planes still needed
// for x/y neighbours (k) or arriving (k+1..k+2+PF), so the ring is 3 + PF
// planes deep and a point costs 9 shared loads per field instead of 13.
// The accumulators dU of plane k+1 are loaded straight into registers while
// plane k is computed (they have no stencil), which takes them off the
// shared-memory path entirely.  Results are bit-identical to
// ez_stage_kernel: only where the operands are fetched from changes.
// ---------------------------------------------------------------------------
template <typename T, int TX, int TY, int PF, bool FIRST>
__global__ void __launch_bounds__(TX * TY, (sizeof(T) == 4) ? (512 / (TX * TY) > 0 ? 512 / (TX * TY) : 1) : 1)
    ez_stage_rw_kernel(const __grid_constant__ EzConst<T> c, const F7<const T> uin, const F7<T> uout,
                       const F7<T> du, const F7<T> un, const F5<T> aux, const T As,
                       const T Bs, const T tst, const int kchunk, const int flags) {
  constexpr int R = 3 + PF;  // planes k .. k+2+PF
  constexpr int SX = TX + 4, SY = TY + 4, PLANE = SX * SY, NT = TX * TY;
  constexpr int NLOAD = (PLANE + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sU = reinterpret_cast<T*>(smem_raw);

  const GridGeom& g = c.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = g.lo[0] + blockIdx.x * TX + tx;
  const int j = g.lo[1] + blockIdx.y * TY + ty;
  const int k0 = g.lo[2] + blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.hi[2]);
  const bool active = (i < g.hi[0]) && (j < g.hi[1]);
  const int gx0 = g.lo[0] + blockIdx.x * TX - 2;
  const int gy0 = g.lo[1] + blockIdx.y * TY - 2;
  const long long own = (long long)j * g.sy + i;

  int soff[NLOAD];
  long long goff[NLOAD];
  bool lv[NLOAD];
#pragma unroll
  for (int m = 0; m < NLOAD; ++m) {
    const int e = tid + m * NT;
    const int r = e / SX, col = e - r * SX;
    const int gx = gx0 + col, gy = gy0 + r;
    lv[m] = (e < PLANE) && gx < g.dims[0] && gy < g.dims[1];
    soff[m] = e;
    goff[m] = (long long)gy * g.sy + gx;
  }
  const int kend = k1 + 2;  // planes [k0, k1+2) pass through shared memory
  auto issue = [&](int kp) {
    if (kp < kend) {
      const int slot = kp % R;
#pragma unroll
      for (int f = 0; f < 7; ++f) {
        T* base = sU + (size_t)(slot * 7 + f) * PLANE;
        const T* gb = uin.p[f] + (long long)kp * g.sz;
#pragma unroll
        for (int m = 0; m < NLOAD; ++m)
          if (lv[m]) cp_async<sizeof(T)>(smem_u32(base + soff[m]), gb + goff[m]);
      }
    }
    cp_async_commit();
  };
#pragma unroll 1
  for (int p = 0; p < R; ++p) issue(k0 + p);

  // register window: w[q][f] = U_f at (i, j, k - 2 + q), q = 0..3 held
  // across iterations (plane k+2 is read each iteration)
  T w0[7], w1[7], w2[7], w3[7], dn[7];
  if (active) {
#pragma unroll
    for (int f = 0; f < 7; ++f) {
      const T* col = uin.p[f] + own;
      w0[f] = col[(long long)(k0 - 2) * g.sz];
      w1[f] = col[(long long)(k0 - 1) * g.sz];
      w2[f] = col[(long long)k0 * g.sz];
      w3[f] = col[(long long)(k0 + 1) * g.sz];
      if constexpr (!FIRST) dn[f] = du.p[f][(long long)k0 * g.sz + own];
      else dn[f] = (T)0;
    }
  }
  const T six = c.inv_delta[0] / (T)12, siy = c.inv_delta[1] / (T)12,
          siz = c.inv_delta[2] / (T)12;
  const int rc = (ty + 2) * SX + tx + 2;

#pragma unroll 1
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<PF>();  // plane k+2 has landed
    __syncthreads();
    if (active) {
      T dcur[7];
#pragma unroll
      for (int f = 0; f < 7; ++f) dcur[f] = dn[f];
      if constexpr (!FIRST) {
        if (k + 1 < k1) {
#pragma unroll
          for (int f = 0; f < 7; ++f) dn[f] = du.p[f][(long long)(k + 1) * g.sz + own];
        }
      }
      const int sc = k % R, s2 = (k + 2) % R;
      T u[7], dx[7], dy[7], dz[7], w4[7];
#pragma unroll
      for (int f = 0; f < 7; ++f) {
        const T* pc = sU + (size_t)(sc * 7 + f) * PLANE + rc;
        w4[f] = sU[(size_t)(s2 * 7 + f) * PLANE + rc];
        u[f] = w2[f];
        dx[f] = d1_4(pc[-2], pc[-1], pc[1], pc[2], six);
        dy[f] = d1_4(pc[-2 * SX], pc[-SX], pc[SX], pc[2 * SX], siy);
        dz[f] = d1_4(w0[f], w1[f], w3[f], w4[f], siz);
      }
      stage_point<T, FIRST>(c, u, dx, dy, dz, dcur, As, Bs, tst, flags, i, j, k,
                            (long long)k * g.sz + own, du, un, aux, uout);
#pragma unroll
      for (int f = 0; f < 7; ++f) {
        w0[f] = w1[f];
        w1[f] = w2[f];
        w2[f] = w3[f];
        w3[f] = w4[f];
      }
    }
    __syncthreads();
    issue(k + R);
  }
  cp_async_wait<0>();
}

template <typename T, int TX, int TY, int PF>
constexpr size_t stage_rw_smem_bytes() {
  return (size_t)(3 + PF) * 7 * (TX + 4) * (TY + 4) * sizeof(T);
}

// ---------------------------------------------------------------------------
// Kreiss-Oliger dissipation + clamps + star boundary at t + dt + guard fill
// (reference Kreiss_Oliger and the tail of evolve_fields,
// field_solver_EZ.cpp:324-457, 1057-1072; .cu:272-392, 696-706):
//   f' = f + (-KOeps * KO_const) * sum_axes diff6_2(f)
// for E and B (CPU build) or E, B and P (GPU build).
// ---------------------------------------------------------------------------
template <typename T, int TX, int TY, int PF>
__global__ void __launch_bounds__(TX * TY, (sizeof(T) == 4) ? (512 / (TX * TY) > 0 ? 512 / (TX * TY) : 1) : 1)
    ez_ko_kernel(const __grid_constant__ EzConst<T> c, const F7<const T> uin, const F7<T> uout, const T tko,
                 const int kchunk) {
  using C = TileCfg<T, TX, TY, 3, PF, false>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sU = reinterpret_cast<T*>(smem_raw);

  const GridGeom& g = c.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = g.lo[0] + blockIdx.x * TX + tx;
  const int j = g.lo[1] + blockIdx.y * TY + ty;
  const int k0 = g.lo[2] + blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.hi[2]);
  const bool active = (i < g.hi[0]) && (j < g.hi[1]);
  const int gx0 = g.lo[0] + blockIdx.x * TX - 3;
  const int gy0 = g.lo[1] + blockIdx.y * TY - 3;

  int soff[C::NLOAD];
  long long goff[C::NLOAD];
  bool lv[C::NLOAD];
#pragma unroll
  for (int m = 0; m < C::NLOAD; ++m) {
    const int e = tid + m * C::NT;
    const int r = e / C::SX, col = e - r * C::SX;
    const int gx = gx0 + col, gy = gy0 + r;
    lv[m] = (e < C::PLANE) && gx < g.dims[0] && gy < g.dims[1];
    soff[m] = e;
    goff[m] = (long long)gy * g.sy + gx;
  }
  const int kend = k1 + 3;
  auto issue = [&](int kp) {
    if (kp < kend) {
      const int slot = kp % C::R;
#pragma unroll
      for (int f = 0; f < 7; ++f) {
        T* base = sU + (size_t)(slot * 7 + f) * C::PLANE;
        const T* gb = uin.p[f] + (long long)kp * g.sz;
#pragma unroll
        for (int m = 0; m < C::NLOAD; ++m)
          if (lv[m]) cp_async<sizeof(T)>(smem_u32(base + soff[m]), gb + goff[m]);
      }
    }
    cp_async_commit();
  };
#pragma unroll 1
  for (int p = 0; p < C::R; ++p) issue(k0 - 3 + p);

  const int nko = (c.semantics == SEM_CPU_REF) ? 6 : 7;
#pragma unroll 1
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<PF>();
    __syncthreads();
    if (active) {
      int sl[7];
#pragma unroll
      for (int q = 0; q < 7; ++q) sl[q] = (k - 3 + q) % C::R;
      const int rc = (ty + 3) * C::SX + tx + 3;
      T nu[7];
#pragma unroll
      for (int f = 0; f < 7; ++f) {
        const T* pc = sU + (size_t)(sl[3] * 7 + f) * C::PLANE + rc;
        const T cv = pc[0];
        if (f < nko) {
          const T kx = d6_2(pc[-3], pc[-2], pc[-1], cv, pc[1], pc[2], pc[3]);
          const T ky = d6_2(pc[-3 * C::SX], pc[-2 * C::SX], pc[-C::SX], cv, pc[C::SX],
                            pc[2 * C::SX], pc[3 * C::SX]);
          T zv[7];
#pragma unroll
          for (int q = 0; q < 7; ++q) zv[q] = sU[(size_t)(sl[q] * 7 + f) * C::PLANE + rc];
          const T kz = d6_2(zv[0], zv[1], zv[2], cv, zv[4], zv[5], zv[6]);
          nu[f] = fma(kx + ky + kz, c.ko_c, cv);
        } else {
          nu[f] = cv;
        }
      }
      apply_clamps(c, nu[0], nu[1], nu[2], nu[3], nu[4], nu[5]);
      star_boundary(c, i, j, k, tko, nu);
      store_with_images(g, uout, i, j, k, nu);
    }
    __syncthreads();
    issue(k + 4 + PF);
  }
  cp_async_wait<0>();
}

}  // namespace coffee
