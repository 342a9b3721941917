// Flat-Cartesian EZ kernels: one fused LSRK stage, and the Kreiss-Oliger
// pass that closes a step.
//
// Both kernels stream along z.  A CTA owns a TX x TY column of points and a
// chunk of z planes.  Each z plane of the 7 fields (E, B, P), with a halo of
// H points in x and y, is copied global -> shared memory by cp.async into a
// ring of planes, PF planes ahead of the plane being computed, so the HBM
// reads of the next planes overlap the arithmetic of this one.  The new
// E, B, P go to a second buffer (stencil reads of other points still need
// the old values), together with their periodic guard images, so no separate
// halo-exchange pass is needed.
//
// The kernels are bound by instruction issue more than by anything else, so
// the stencil loops are written to cost one instruction per operand: shared
// memory is addressed by 32-bit addresses with the field / neighbour offsets
// as compile-time immediates (lds<T, OFF>), loops over the 7 fields are
// unrolled at compile time (static_for), and the guard-image bookkeeping is
// skipped for points that have no image.  Global element offsets are 32-bit
// (an array has fewer than 2^31 points: flat_plan checks it), so that every
// global address is one wide multiply-add of an offset onto an array base.
#pragma once

#include "ez_physics.cuh"

namespace coffee {

// Flags of the stage kernel.
enum StageFlags { ST_LAST = 1, ST_AUX = 2, ST_WRITE_UN = 4 };

// Minimum resident CTAs for __launch_bounds__: two 256-thread CTAs (or the
// equivalent) per SM in FP32, which caps registers at 128 per thread.
#ifndef COFFEE_F32_THREADS_PER_SM
#define COFFEE_F32_THREADS_PER_SM 512
#endif
template <typename T, int NT>
constexpr int min_blocks() {
  return (sizeof(T) == 4)
             ? ((COFFEE_F32_THREADS_PER_SM / NT) > 0 ? COFFEE_F32_THREADS_PER_SM / NT : 1)
             : 1;
}

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

// Write the 7 new values of point (i, j, k) (linear index o) to `out` at the
// point and at its periodic guard images.
template <typename T>
__device__ __forceinline__ void store_with_images(const GridGeom& g, const ColumnCtx<T>& col,
                                                  const F7<T>& out, int k, uint32_t o,
                                                  const T u[7]) {
  if (col.xy_simple && only_self(g, 2, k)) {
#pragma unroll
    for (int f = 0; f < 7; ++f) out.p[f][o] = u[f];
    return;
  }
  int xs[2], ys[2], zs[2];
  const int nx = periodic_targets(g, 0, col.i, xs);
  const int ny = periodic_targets(g, 1, col.j, ys);
  const int nz = periodic_targets(g, 2, k, zs);
#pragma unroll
  for (int cz = 0; cz < 2; ++cz) {
    if (cz >= nz) break;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if (b >= ny) break;
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        if (a >= nx) break;
        const uint32_t q = (uint32_t)zs[cz] * (uint32_t)g.sz + (uint32_t)ys[b] * (uint32_t)g.sy +
                           (uint32_t)xs[a];
#pragma unroll
        for (int f = 0; f < 7; ++f) out.p[f][q] = u[f];
      }
    }
  }
}

// Everything a stage does at one point once its derivatives are known:
// the current J, the new accumulators dU (from dold unless FIRST), the new
// fields U + Bs dU, the clamps, the star boundary, the absorbing layer
// (ST_LAST) and the stores of dU, J/divE/divB (ST_AUX), Un (ST_WRITE_UN) and
// of U' with its guard images.  d{x,y,z}[f] are the inv_delta-scaled
// 4th-order derivatives of field f at the point, u[f] its values.
// Curl, divergence and gradient of the fields at one point, as the stage
// needs them (all inv_delta-scaled 4th-order differences).
template <typename T>
struct Derivs {
  T rotE[3], rotB[3], divE, divB, gradP[3];
};

// XA selects the CPU build's own arithmetic (ez_refarith.cuh) for the
// current, the taper, the accumulators, the update and the clamps; the
// derivatives then come in already combined in that arithmetic (Derivs).
template <typename T, bool FIRST, bool BC, bool XA, bool DG>
__device__ __forceinline__ void stage_point(const EzConst<T>& c, const T u[7],
                                            const Derivs<T>& dv, const T dold[7],
                                            const T As, const T Bs, const T tst,
                                            const int flags, const ColumnCtx<T>& col,
                                            const int k, const uint32_t o, const F7<T>& du,
                                            const F7<T>& un, const F5<T>& aux,
                                            const F7<T>& uout, const F6<T>& dg) {
  const bool cpu = c.semantics == SEM_CPU_REF;
  const T ex = u[0], ey = u[1], ez = u[2], bx = u[3], by = u[4], bz = u[5], P = u[6];
  const T rotBx = dv.rotB[0], rotBy = dv.rotB[1], rotBz = dv.rotB[2];
  const T rotEx = dv.rotE[0], rotEy = dv.rotE[1], rotEz = dv.rotE[2];
  const T divE = dv.divE;
  const T divB = dv.divB;
  T d[7];
  T Jx, Jy, Jz;
  if constexpr (XA) {
    // rk_step of the CPU build (field_solver_EZ.cpp:143-259) operation for
    // operation
    const T B2 = xa::floor_tiny(xa::dot3(bx, bx, by, by, bz, bz));
    const T BrotB = xa::dot3(bx, rotBx, by, rotBy, bz, rotBz);
    const T ErotE = xa::dot3(ex, rotEx, ey, rotEy, ez, rotEz);
    const T cx = xa::fma(-by, ez, xa::mul(bz, ey));
    const T cy = xa::fma(-bz, ex, xa::mul(bx, ez));
    const T cz = xa::fma(-bx, ey, xa::mul(by, ex));
    if (c.use_edotb) {
      const T E2 = xa::dot3(ex, ex, ey, ey, ez, ez);
      const T chi2 = xa::sub(B2, E2);
      const T EdotB = xa::dot3(bx, ex, by, ey, bz, ez);
      const T E02 = xa::fma(
          xa::sub(xa::sqrt(xa::fma(xa::mul(EdotB, (T)4), EdotB, xa::mul(chi2, chi2))), chi2),
          (T)0.5, B2);
      const T Jp = xa::fma(EdotB, c.gam_dt, xa::sub(BrotB, ErotE));
      Jx = xa::add(xa::div(xa::mul(divE, cx), E02), xa::div(xa::mul(bx, Jp), B2));
      Jy = xa::add(xa::div(xa::mul(divE, cy), E02), xa::div(xa::mul(by, Jp), B2));
      Jz = xa::add(xa::div(xa::mul(divE, cz), E02), xa::div(xa::mul(bz, Jp), B2));
    } else {
      const T Jp = xa::sub(BrotB, ErotE);
      Jx = xa::div(xa::fma(bx, Jp, xa::mul(divE, cx)), B2);
      Jy = xa::div(xa::fma(by, Jp, xa::mul(divE, cy)), B2);
      Jz = xa::div(xa::fma(bz, Jp, xa::mul(divE, cz)), B2);
    }
    T Px = 0, Py = 0, Pz = 0;
    if (c.divB_clean) {
      Px = dv.gradP[0];
      Py = dv.gradP[1];
      Pz = dv.gradP[2];
    }
    const T s = p_taper_xa(c, col, k);
    const T dt = c.dt;
    // dU As (As = 0 on the first stage, where the old dU is not read)
    T da[7];
#pragma unroll
    for (int f = 0; f < 7; ++f) {
      if constexpr (FIRST) da[f] = (T)0;
      else da[f] = xa::mul(dold[f], As);
    }
    d[0] = xa::fma(dt, xa::sub(rotBx, Jx), da[0]);
    d[1] = xa::fma(dt, xa::sub(rotBy, Jy), da[1]);
    d[2] = xa::fma(dt, xa::sub(rotBz, Jz), da[2]);
    d[3] = xa::fma(-dt, xa::fma(Px, s, rotEx), da[3]);
    d[4] = xa::fma(-dt, xa::fma(Py, s, rotEy), da[4]);
    d[5] = xa::fma(-dt, xa::fma(Pz, s, rotEz), da[5]);
    // dP As - P / tau with the product fused, minus dt (divB ch2)
    if constexpr (FIRST)
      d[6] = xa::fma(-dt, xa::mul(divB, c.ch2), -xa::div(P, c.tau));
    else
      d[6] = xa::fma(-dt, xa::mul(divB, c.ch2), xa::fma(dold[6], As, -xa::div(P, c.tau)));
  } else {
    T B2 = bx * bx + by * by + bz * bz;
    if (B2 < Tiny<T>::v) B2 = Tiny<T>::v;
    const T BrotB = bx * rotBx + by * rotBy + bz * rotBz;
    const T ErotE = ex * rotEx + ey * rotEy + ez * rotEz;
    const T cx = ey * bz - ez * by, cy = ez * bx - ex * bz, cz = ex * by - ey * bx;
    if (c.use_edotb) {
      // J with E.B damping (field_solver_EZ.cpp:170-186, .cu:72-91)
      const T E2 = ex * ex + ey * ey + ez * ez;
      const T chi2 = B2 - E2;
      const T EdotB = ex * bx + ey * by + ez * bz;
      const T E02 = (T)0.5 * (sqrt(chi2 * chi2 + (T)4 * EdotB * EdotB) - chi2) + B2;
      const T Jp = BrotB - ErotE + EdotB * c.gam_dt;
      const T a = fdiv(divE, E02), b = fdiv(Jp, B2);
      Jx = a * cx + b * bx;
      Jy = a * cy + b * by;
      Jz = a * cz + b * bz;
    } else {
      const T Jp = BrotB - ErotE;
      const T rB2 = fdiv((T)1, B2);
      Jx = (divE * cx + Jp * bx) * rB2;
      Jy = (divE * cy + Jp * by) * rB2;
      Jz = (divE * cz + Jp * bz) * rB2;
    }
    T Px = 0, Py = 0, Pz = 0;
    if (c.divB_clean) {
      Px = dv.gradP[0];
      Py = dv.gradP[1];
      Pz = dv.gradP[2];
      if (cpu) {
        const T s = p_taper(c, col, k);
        Px *= s;
        Py *= s;
        Pz *= s;
      }
    }
    // new accumulators
    const T dt = c.dt;
    d[0] = (rotBx - Jx) * dt;
    d[1] = (rotBy - Jy) * dt;
    d[2] = (rotBz - Jz) * dt;
    d[3] = -(rotEx + Px) * dt;
    d[4] = -(rotEy + Py) * dt;
    d[5] = -(rotEz + Pz) * dt;
    d[6] = -P * c.inv_tau - divB * c.ch2 * dt;
    if constexpr (!FIRST) {
#pragma unroll
      for (int f = 0; f < 7; ++f) d[f] = fma(dold[f], As, d[f]);
    }
  }
  // the start-of-step copy is only read inside the absorbing layer
  T sig = (T)0;
  if constexpr (BC) sig = c.absorbing ? absorbing_sigma(c, col.i, col.j, k) : (T)0;
  if (BC && (flags & ST_WRITE_UN) != 0 && sig > (T)0) {
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
  if constexpr (XA) {
    // mul_add(dU, Bs, U), then clean_epar_check_eGTb
#pragma unroll
    for (int f = 0; f < 7; ++f) nu[f] = xa::fma(d[f], Bs, u[f]);
    if constexpr (DG)
      apply_clamps_xa_dg<FIRST>(nu[0], nu[1], nu[2], nu[3], nu[4], nu[5], dg, o);
    else
      apply_clamps_xa(nu[0], nu[1], nu[2], nu[3], nu[4], nu[5]);
  } else {
#pragma unroll
    for (int f = 0; f < 7; ++f) nu[f] = fma(d[f], Bs, u[f]);
    apply_clamps(c, nu[0], nu[1], nu[2], nu[3], nu[4], nu[5]);
  }
  if constexpr (BC) star_boundary(c, col.i, col.j, k, tst, nu);
  if (BC && (flags & ST_LAST) != 0 && sig > (T)0) {
    V7<T> uv, unv;
#pragma unroll
    for (int f = 0; f < 7; ++f) {
      uv.v[f] = nu[f];
      unv.v[f] = un.p[f][o];
    }
    uv = absorbing_apply(c, col.i, col.j, k, sig, uv, unv);
#pragma unroll
    for (int f = 0; f < 7; ++f) nu[f] = uv.v[f];
  }
  store_with_images(c.g, col, uout, k, o, nu);
}

// Per-thread table of the shared-memory slots and global offsets that a
// CTA's threads copy for one (TX + 2H) x (TY + 2H) tile of one field plane.
// V = 1 copies one element per cp.async; V = 2 copies aligned pairs (8 bytes
// in FP32), which needs an even row length d0: the copied row then starts at
// the even column at or left of the tile's first column, `xoff` (0 or 1)
// columns before it, and a row holds TX + 2H + 2 elements.
template <typename T, int TX, int TY, int H, int V = 1>
struct TileLoader {
  static_assert(V == 1 || V == 2, "one element or an aligned pair per copy");
  static constexpr int SX = TX + 2 * H + (V == 2 ? 2 : 0);  // shared row stride (elements)
  static constexpr int SY = TY + 2 * H, NT = TX * TY;
  static constexpr int PER_ROW = SX / V;                    // copies per row
  static constexpr int NCOPY = PER_ROW * SY;
  static constexpr int NLOAD = (NCOPY + NT - 1) / NT;
  static constexpr int FB = SX * SY * (int)sizeof(T);       // bytes of one field plane
  uint32_t sadd[NLOAD];  // shared byte address within slot 0, field 0
  uint32_t eoff[NLOAD];  // element offset within a global plane
  bool lv[NLOAD];
  int xoff;               // shared column of the tile's first column

  __device__ __forceinline__ TileLoader(const GridGeom& g, uint32_t sbase, int tid, int gx0,
                                        int gy0) {
    xoff = (V == 2) ? (gx0 & 1) : 0;
    const int xs = gx0 - xoff;
#pragma unroll
    for (int m = 0; m < NLOAD; ++m) {
      const int e = tid + m * NT;
      const int r = e / PER_ROW, cl = (e - r * PER_ROW) * V;
      const int gx = xs + cl, gy = gy0 + r;
      lv[m] = (e < NCOPY) && gx + (V - 1) < g.dims[0] && gy < g.dims[1];
      sadd[m] = sbase + (uint32_t)((r * SX + cl) * (int)sizeof(T));
      eoff[m] = (uint32_t)gy * (uint32_t)g.sy + (uint32_t)gx;
    }
  }

  // Copy one plane (element offset pe into each field array) of the 7
  // fields into the ring slot at byte offset `slot`.
  __device__ __forceinline__ void copy(const F7<const T>& uin, uint32_t pe,
                                       uint32_t slot) const {
#pragma unroll
    for (int m = 0; m < NLOAD; ++m) {
      if (!lv[m]) continue;
      const uint32_t e = pe + eoff[m], d = sadd[m] + slot;
      static_for<7>([&](auto fc) {
        constexpr int f = decltype(fc)::value;
        cp_async_off<sizeof(T) * V, f * FB>(d, uin.p[f] + e);
      });
    }
  }
};

// ---------------------------------------------------------------------------
// One LSRK stage (reference rk_step + clamps + star boundary + absorbing
// layer + send_guard_cells, src/algorithms/field_solver_EZ.cpp:1024-1055,
// .cu:669-694).  BC = false compiles the kernel without the star and
// absorbing-layer code, for runs that have neither (their out-of-line calls
// cost registers even when not taken):
//   dU  <- As dU + dt RHS(U)        (FIRST: As = 0, so dU is not read)
//   U'  <- U + Bs dU
//   U'  <- clamps, star boundary at tst, absorbing layer (ST_LAST)
// reading U from `uin` and writing U' (with guard images) to `uout`.
// Shared memory: a ring of 3 + PF + kRingSpare planes (k .. k+2, the
// prefetch, the spare) of the 7 fields with a 2-point x/y halo, then
// PF + 1 + kRingSpare planes of dU.  The z
// neighbours of a thread's own column are kept in a register window of
// planes k-2 .. k+2: each plane is read from shared memory once, as the
// window's leading plane.
// ---------------------------------------------------------------------------
// z-loop unroll of the stage kernel: 5 (the window length, no register
// moves) or 1 (one plane per iteration, window shifted by moves), chosen
// separately for the instances without and with the boundary code (BC):
// the five copies of the out-of-line boundary calls make the BC instance
// spill, and it runs faster plane by plane.
#ifndef COFFEE_STAGE_ZUNROLL
#define COFFEE_STAGE_ZUNROLL 5
#endif
#ifndef COFFEE_STAGE_ZUNROLL_BC
#define COFFEE_STAGE_ZUNROLL_BC 1
#endif
template <bool BC>
__host__ __device__ constexpr int stage_zunroll() {
  return BC ? COFFEE_STAGE_ZUNROLL_BC : COFFEE_STAGE_ZUNROLL;
}
static_assert((stage_zunroll<false>() == 1 || stage_zunroll<false>() == 5) &&
                  (stage_zunroll<true>() == 1 || stage_zunroll<true>() == 5),
              "stage z unroll is 1 or 5");

// Spare ring slots (0 or 1) of the stage and KO kernels.  With a spare slot
// the copies of a new plane are issued right after the one barrier at the
// top of an iteration, into the slot of the plane the previous iteration
// finished with; without it they wait for a second barrier after the
// iteration's arithmetic.  Measured at 512^3: the stage kernel is faster with
// the spare slot, the KO kernel (two CTAs per SM) without.
#ifndef COFFEE_STAGE_RING_SPARE
#define COFFEE_STAGE_RING_SPARE 1
#endif
#ifndef COFFEE_KO_RING_SPARE
#define COFFEE_KO_RING_SPARE 0
#endif
constexpr int kRingSpare = COFFEE_STAGE_RING_SPARE;
constexpr int kKoRingSpare = COFFEE_KO_RING_SPARE;
static_assert((kRingSpare == 0 || kRingSpare == 1) && (kKoRingSpare == 0 || kKoRingSpare == 1),
              "0 or 1 spare ring slot");

// Ring slots of the stage kernel.  Plane k lives in slot (k - lo[2]) % R of
// the field ring and its dU in slot (k - lo[2]) % DR of the dU ring.  With
// PF = 1 and the spare slot the field ring has 5 slots, the z unroll length:
// every chunk then starts a multiple of 5 planes from lo[2] (the host picks
// such chunks) and the field slot of every plane an unrolled iteration
// touches is a compile-time constant.  (Rings grown to make the dU slots
// constant too measured slower: shared memory taken from the L1 cache.)
template <bool BC, int PF>
__host__ __device__ constexpr int stage_ring() {
  return 3 + PF + kRingSpare;
}
template <bool BC, int PF>
__host__ __device__ constexpr int stage_dring() {
  return PF + 1 + kRingSpare;
}

template <typename T, int TX, int TY, int PF, int V, bool BC>
constexpr size_t stage_smem_bytes(bool first) {
  return (size_t)stage_ring<BC, PF>() * 7 * TileLoader<T, TX, TY, 2, V>::FB +
         (first ? 0 : (size_t)stage_dring<BC, PF>() * 7 * TX * TY * sizeof(T));
}

// DG (with XA only): also accumulate the CPU build's energy-change
// diagnostics of the clamps into dg.
template <typename T, int TX, int TY, int PF, bool FIRST, bool BC, int V, bool XA, bool DG>
__global__ void __launch_bounds__(TX * TY, min_blocks<T, TX * TY>())
    ez_stage_kernel(const __grid_constant__ EzConst<T> c, const F7<const T> uin,
                    const F7<T> uout, const F7<T> du, const F7<T> un, const F5<T> aux,
                    const F6<T> dg, const T As, const T Bs, const T tst, const int kchunk,
                    const int flags) {
  static_assert(XA || !DG, "the energy diagnostics need the reference arithmetic");
  using L = TileLoader<T, TX, TY, 2, V>;
  constexpr int R = stage_ring<BC, PF>();    // field ring slots
  constexpr int DR = stage_dring<BC, PF>();  // dU ring slots
  constexpr int ZU = stage_zunroll<BC>();

  constexpr int ES = (int)sizeof(T);
  constexpr int SX = L::SX, FB = L::FB, SB = 7 * FB;
  constexpr int NT = TX * TY, DFB = NT * ES, DSB = 7 * DFB;
  constexpr int CEN = (2 * SX + 2) * ES;  // own point, from the corner of its 5x5 patch
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t sbase = smem_u32(smem_raw);
  const uint32_t dbase = sbase + (uint32_t)(R * SB);

  const GridGeom& g = c.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = g.lo[0] + blockIdx.x * TX + tx;
  const int j = g.lo[1] + blockIdx.y * TY + ty;
  const int k0 = g.lo[2] + blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.hi[2]);
  const bool active = (i < g.hi[0]) && (j < g.hi[1]);
  // lanes of this warp that compute points: the fences between the field
  // groups below are executed by these lanes only (a tile that overhangs
  // the grid has idle lanes, which must not be named in the mask)
  const unsigned amask = __ballot_sync(0xffffffffu, active);
  const uint32_t sz = (uint32_t)g.sz;
  const uint32_t own = (uint32_t)j * (uint32_t)g.sy + (uint32_t)i;
  const ColumnCtx<T> col = make_column<XA>(c, i, j);
  const L loader(g, sbase, tid, g.lo[0] + (int)blockIdx.x * TX - 2,
                 g.lo[1] + (int)blockIdx.y * TY - 2);
  const uint32_t dme = dbase + (uint32_t)(tid * ES);
  const int kend = k1 + 2;  // planes [k0-2, k1+2) are read
  const int lo2 = g.lo[2];
  // byte offsets of the ring slots of plane k + OFF in window phase S:
  // compile-time constants in the unrolled loop
  auto fslot = [&](auto sc, auto oc, int k) -> uint32_t {
    constexpr int S = decltype(sc)::value, OFF = decltype(oc)::value;
    if constexpr (ZU == R) return (uint32_t)(((S + OFF) % R) * SB);
    else return (uint32_t)(((k + OFF - lo2) % R) * SB);
  };
  auto dslot = [&](auto sc, auto oc, int k) -> uint32_t {
    constexpr int S = decltype(sc)::value, OFF = decltype(oc)::value;
    if constexpr (ZU == DR) return (uint32_t)(((S + OFF) % DR) * DSB);
    else return (uint32_t)(((k + OFF - lo2) % DR) * DSB);
  };

  // copy plane kp into field slot fs and the dU of plane kp - 2 into dU
  // slot ds
  auto issue = [&](int kp, uint32_t fs, uint32_t dsl) {
    if (kp < kend) loader.copy(uin, (uint32_t)kp * sz, fs);
    if constexpr (!FIRST) {
      const int kd = kp - 2;
      if (kd >= k0 && kd < k1 && active) {
        const uint32_t ds = dme + dsl;
        const uint32_t e = (uint32_t)kd * sz + own;
        static_for<7>([&](auto fc) {
          constexpr int f = decltype(fc)::value;
          cp_async_off<sizeof(T), f * DFB>(ds, du.p[f] + e);
        });
      }
    }
    cp_async_commit();
  };
#pragma unroll 1
  for (int p = 0; p < 3 + PF; ++p)
    issue(k0 + p, (uint32_t)(((k0 + p - lo2) % R) * SB),
          (uint32_t)((((k0 + p - 2 - lo2) % DR + DR) % DR) * DSB));

  const T six = c.inv_delta[0] / (T)12, siy = c.inv_delta[1] / (T)12,
          siz = c.inv_delta[2] / (T)12;
  const T ix = c.inv_delta[0], iy = c.inv_delta[1], iz = c.inv_delta[2];
  const uint32_t corner = sbase + (uint32_t)((ty * SX + tx + loader.xoff) * ES);
  // Register window: in window phase S, w[(S + q) % 5][f] = field f at
  // (i, j, k - 2 + q).  Planes k-2 .. k+1 are carried from the previous
  // plane and k+2 is read from the ring into the slot of the dead plane k-3,
  // so advancing the window moves no registers when the z loop is unrolled
  // by the window length (ZU = 5).
  T w[5][7];
  if (active) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int f = 0; f < 7; ++f) w[q][f] = uin.p[f][(uint32_t)(k0 - 2 + q) * sz + own];
  }

  auto plane = [&](auto sc, const int k) {
    constexpr int S = decltype(sc)::value;
    cp_async_wait<PF>();  // planes up to k+2 (and the dU of k) have landed
    __syncthreads();
    using Z = std::integral_constant<int, 0>;
    using P2 = std::integral_constant<int, 2>;
    using PN = std::integral_constant<int, 3 + PF>;   // the plane issued now
    using PD = std::integral_constant<int, 1 + PF>;   // and its dU plane
    if constexpr (kRingSpare == 1)  // into the slot of plane k-1
      issue(k + 3 + PF, fslot(sc, PN{}, k), dslot(sc, PD{}, k));
    if (active && k < k1) {
      const uint32_t a0 = corner + fslot(sc, Z{}, k);
      const uint32_t ap2 = corner + fslot(sc, P2{}, k);
      // The stencil is consumed field group by field group (B, then E, then
      // P); the warp-level fence between groups keeps the shared loads of the
      // next group from being hoisted, which bounds the live registers.
      T u[7], dold[7];
      Derivs<T> dv;
      // dxyz[a]: the derivative of field f along axis a, inv_delta-scaled;
      // in the reference arithmetic (XA) the unscaled quotient of diff1_4,
      // which curl_div scales and combines as the CPU build does.  EX
      // selects the exact division for the rare quotients the fast one
      // flags through the key minimum `kmin` (xa::div12_fast).
      uint32_t kmin = 0xFFFFFFFFu;
      auto d1 = [&](auto fc, auto ex, T* dxyz) {
        constexpr int f = decltype(fc)::value;
        constexpr bool EX = decltype(ex)::value;
        constexpr int o = f * FB;
        if constexpr (XA) {
          dxyz[0] = xa::dq<EX>(lds<T, o + CEN - 2 * ES>(a0), lds<T, o + CEN - ES>(a0),
                               lds<T, o + CEN + ES>(a0), lds<T, o + CEN + 2 * ES>(a0), kmin);
          dxyz[1] = xa::dq<EX>(lds<T, o + 2 * ES>(a0), lds<T, o + (SX + 2) * ES>(a0),
                               lds<T, o + (3 * SX + 2) * ES>(a0),
                               lds<T, o + (4 * SX + 2) * ES>(a0), kmin);
        } else {
          dxyz[0] = d1_4(lds<T, o + CEN - 2 * ES>(a0), lds<T, o + CEN - ES>(a0),
                         lds<T, o + CEN + ES>(a0), lds<T, o + CEN + 2 * ES>(a0), six);
          dxyz[1] = d1_4(lds<T, o + 2 * ES>(a0), lds<T, o + (SX + 2) * ES>(a0),
                         lds<T, o + (3 * SX + 2) * ES>(a0), lds<T, o + (4 * SX + 2) * ES>(a0), siy);
        }
        w[(S + 4) % 5][f] = lds<T, o + CEN>(ap2);
        u[f] = w[(S + 2) % 5][f];
        if constexpr (XA)
          dxyz[2] = xa::dq<EX>(w[S % 5][f], w[(S + 1) % 5][f], w[(S + 3) % 5][f],
                               w[(S + 4) % 5][f], kmin);
        else
          dxyz[2] = d1_4(w[S % 5][f], w[(S + 1) % 5][f], w[(S + 3) % 5][f], w[(S + 4) % 5][f],
                         siz);
      };
      // curl and divergence of one vector field from its derivatives; in the
      // reference arithmetic the curl's first product is rounded and its
      // second fused (rk_step, field_solver_EZ.cpp:143-150)
      auto curl_div = [&](const T* xd, const T* yd, const T* zd, T* rot, T& dvg) {
        if constexpr (XA) {
          rot[0] = xa::fma(-iz, yd[2], xa::mul(iy, zd[1]));
          rot[1] = xa::fma(-ix, zd[0], xa::mul(iz, xd[2]));
          rot[2] = xa::fma(-iy, xd[1], xa::mul(ix, yd[0]));
          dvg = xa::fma(iz, zd[2], xa::fma(iy, yd[1], xa::mul(ix, xd[0])));
        } else {
          rot[0] = zd[1] - yd[2];
          rot[1] = xd[2] - zd[0];
          rot[2] = yd[0] - xd[1];
          dvg = xd[0] + yd[1] + zd[2];
        }
      };
      auto derivatives = [&](auto ex) {
        {
          T bxd[3], byd[3], bzd[3];
          d1(std::integral_constant<int, 3>{}, ex, bxd);
          d1(std::integral_constant<int, 4>{}, ex, byd);
          d1(std::integral_constant<int, 5>{}, ex, bzd);
          curl_div(bxd, byd, bzd, dv.rotB, dv.divB);
        }
        __syncwarp(amask);
        {
          T exd[3], eyd[3], ezd[3];
          d1(std::integral_constant<int, 0>{}, ex, exd);
          d1(std::integral_constant<int, 1>{}, ex, eyd);
          d1(std::integral_constant<int, 2>{}, ex, ezd);
          curl_div(exd, eyd, ezd, dv.rotE, dv.divE);
        }
        __syncwarp(amask);
        d1(std::integral_constant<int, 6>{}, ex, dv.gradP);
      };
      derivatives(std::false_type{});
      // a quotient in the subnormal range (|t| < 2^-124, t != 0): the whole
      // warp recomputes its derivatives with the exact division (the same
      // operands are still in shared memory and the window)
      if constexpr (XA)
        if (__any_sync(amask, kmin < xa::kTinyKey)) derivatives(std::true_type{});
      if constexpr (XA) {
        dv.gradP[0] = xa::mul(ix, dv.gradP[0]);
        dv.gradP[1] = xa::mul(iy, dv.gradP[1]);
        dv.gradP[2] = xa::mul(iz, dv.gradP[2]);
      }
      if constexpr (!FIRST) {
        const uint32_t ad = dme + dslot(sc, Z{}, k);
        static_for<7>([&](auto fc) {
          constexpr int f = decltype(fc)::value;
          dold[f] = lds<T, f * DFB>(ad);
        });
      }
      stage_point<T, FIRST, BC, XA, DG>(c, u, dv, dold, As, Bs, tst, flags, col, k,
                                        (uint32_t)k * sz + own, du, un, aux, uout, dg);
      if constexpr (ZU == 1) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int f = 0; f < 7; ++f) w[q][f] = w[q + 1][f];
      }
    }
    if constexpr (kRingSpare == 0) {
      __syncthreads();
      issue(k + 3 + PF, fslot(sc, PN{}, k), dslot(sc, PD{}, k));  // into the slot of plane k
    }
  };
  if constexpr (ZU == 5) {
    // planes past k1 in the last group only wait, synchronise and commit
    // empty copy groups (issue() copies nothing past kend), so the ring's
    // group accounting stays the same as plane-by-plane
#pragma unroll 1
    for (int k = k0; k < k1; k += 5) {
      plane(std::integral_constant<int, 0>{}, k);
      plane(std::integral_constant<int, 1>{}, k + 1);
      plane(std::integral_constant<int, 2>{}, k + 2);
      plane(std::integral_constant<int, 3>{}, k + 3);
      plane(std::integral_constant<int, 4>{}, k + 4);
    }
  } else {
#pragma unroll 1
    for (int k = k0; k < k1; ++k) plane(std::integral_constant<int, 0>{}, k);
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Kreiss-Oliger dissipation + clamps + star boundary at t + dt + guard fill
// (reference Kreiss_Oliger and the tail of evolve_fields,
// field_solver_EZ.cpp:324-457, 1057-1072; .cu:272-392, 696-706):
//   f' = f + (-KOeps * KO_const) * sum_axes diff6_2(f)
// for E and B (CPU build) or E, B and P (GPU build).  The operator has 18
// neighbours per field, so the z direction is held in a register window of
// planes k-3..k+3 per thread; shared memory keeps plane k (x/y neighbours)
// and the arriving planes k+1..k+3+PF.
// ---------------------------------------------------------------------------
// z-loop unroll of the KO kernel: 7 (the window length, no register moves)
// or 1 (one plane per iteration, window shifted by moves), per instance
// (with and without the boundary code); both are faster unrolled.
#ifndef COFFEE_KO_ZUNROLL
#define COFFEE_KO_ZUNROLL 7
#endif
#ifndef COFFEE_KO_ZUNROLL_BC
#define COFFEE_KO_ZUNROLL_BC 7
#endif
template <bool BC>
__host__ __device__ constexpr int ko_zunroll() {
  return BC ? COFFEE_KO_ZUNROLL_BC : COFFEE_KO_ZUNROLL;
}
static_assert((ko_zunroll<false>() == 1 || ko_zunroll<false>() == 7) &&
                  (ko_zunroll<true>() == 1 || ko_zunroll<true>() == 7),
              "KO z unroll is 1 or 7");

// Ring slots of the KO kernel (plane k in slot (k - lo[2]) % R).  A 7-slot
// ring, matching the z unroll, would make the slots compile-time constants
// but measured far slower (its shared memory leaves the two resident CTAs
// little L1 cache).
template <bool BC, int PF>
__host__ __device__ constexpr int ko_ring() {
  return 4 + PF + kKoRingSpare;
}

template <typename T, int TX, int TY, int PF, int V, bool BC>
constexpr size_t ko_smem_bytes() {
  return (size_t)ko_ring<BC, PF>() * 7 * TileLoader<T, TX, TY, 3, V>::FB;
}

template <typename T, int TX, int TY, int PF, bool BC, int V, bool XA, bool DG>
__global__ void __launch_bounds__(TX * TY, min_blocks<T, TX * TY>())
    ez_ko_kernel(const __grid_constant__ EzConst<T> c, const F7<const T> uin,
                 const F7<T> uout, const F6<T> dg, const T tko, const int kchunk) {
  static_assert(XA || !DG, "the energy diagnostics need the reference arithmetic");
  using L = TileLoader<T, TX, TY, 3, V>;
  constexpr int R = ko_ring<BC, PF>();
  constexpr int ZU = ko_zunroll<BC>();

  constexpr int ES = (int)sizeof(T);
  constexpr int SX = L::SX, FB = L::FB, SB = 7 * FB;
  constexpr int CEN = (3 * SX + 3) * ES;  // own point, from the corner of its 7x7 patch
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t sbase = smem_u32(smem_raw);

  const GridGeom& g = c.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = g.lo[0] + blockIdx.x * TX + tx;
  const int j = g.lo[1] + blockIdx.y * TY + ty;
  const int k0 = g.lo[2] + blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.hi[2]);
  const bool active = (i < g.hi[0]) && (j < g.hi[1]);
  const uint32_t sz = (uint32_t)g.sz;
  const uint32_t own = (uint32_t)j * (uint32_t)g.sy + (uint32_t)i;
  const ColumnCtx<T> col = make_column<XA>(c, i, j);
  const L loader(g, sbase, tid, g.lo[0] + (int)blockIdx.x * TX - 3,
                 g.lo[1] + (int)blockIdx.y * TY - 3);
  const int kend = k1 + 3;  // planes [k0, k1+3) pass through shared memory
  const int lo2 = g.lo[2];
  // byte offset of the ring slot of plane k + OFF in window phase S
  auto fslot = [&](auto sc, auto oc, int k) -> uint32_t {
    constexpr int S = decltype(sc)::value, OFF = decltype(oc)::value;
    if constexpr (ZU == R) return (uint32_t)(((S + OFF) % R) * SB);
    else return (uint32_t)(((k + OFF - lo2) % R) * SB);
  };
  auto issue = [&](int kp, uint32_t fs) {
    if (kp < kend) loader.copy(uin, (uint32_t)kp * sz, fs);
    cp_async_commit();
  };
#pragma unroll 1
  for (int p = 0; p < 4 + PF; ++p) issue(k0 + p, (uint32_t)(((k0 + p - lo2) % R) * SB));

  // Register window: in window phase S, w[(S + q) % 7][f] = field f at
  // (i, j, k - 3 + q); planes k-3 .. k+2 are carried, k+3 is read from the
  // ring into the slot of the dead plane k-4 (no register moves when the z
  // loop is unrolled by the window length, ZU = 7).
  T w[7][7];
  if (active) {
#pragma unroll
    for (int f = 0; f < 7; ++f)
#pragma unroll
      for (int q = 0; q < 6; ++q) w[q][f] = uin.p[f][(uint32_t)(k0 - 3 + q) * sz + own];
  }
  const bool ko_p = (c.semantics != SEM_CPU_REF);
  const uint32_t corner = sbase + (uint32_t)((ty * SX + tx + loader.xoff) * ES);
  auto plane = [&](auto sc, const int k) {
    constexpr int S = decltype(sc)::value;
    cp_async_wait<PF>();  // plane k+3 has landed
    __syncthreads();
    using PN = std::integral_constant<int, 4 + PF>;  // the plane issued now
    if constexpr (kKoRingSpare == 1) issue(k + 4 + PF, fslot(sc, PN{}, k));  // slot of plane k-1
    if (active && k < k1) {
      const uint32_t a0 = corner + fslot(sc, std::integral_constant<int, 0>{}, k);
      const uint32_t a3 = corner + fslot(sc, std::integral_constant<int, 3>{}, k);
      T nu[7];
      static_for<7>([&](auto fc) {
        constexpr int f = decltype(fc)::value;
        constexpr int o = f * FB;
        w[(S + 6) % 7][f] = lds<T, o + CEN>(a3);
        const T cv = w[(S + 3) % 7][f];
        if (f < 6 || ko_p) {
          auto d6 = [](T m3, T m2, T m1, T c0, T p1, T p2, T p3) {
            if constexpr (XA) return xa::d6(m3, m2, m1, c0, p1, p2, p3);
            else return d6_2(m3, m2, m1, c0, p1, p2, p3);
          };
          const T kx = d6(lds<T, o + CEN - 3 * ES>(a0), lds<T, o + CEN - 2 * ES>(a0),
                          lds<T, o + CEN - ES>(a0), cv, lds<T, o + CEN + ES>(a0),
                          lds<T, o + CEN + 2 * ES>(a0), lds<T, o + CEN + 3 * ES>(a0));
          const T ky = d6(lds<T, o + 3 * ES>(a0), lds<T, o + (SX + 3) * ES>(a0),
                          lds<T, o + (2 * SX + 3) * ES>(a0), cv,
                          lds<T, o + (4 * SX + 3) * ES>(a0), lds<T, o + (5 * SX + 3) * ES>(a0),
                          lds<T, o + (6 * SX + 3) * ES>(a0));
          const T kz = d6(w[S % 7][f], w[(S + 1) % 7][f], w[(S + 2) % 7][f], cv,
                          w[(S + 4) % 7][f], w[(S + 5) % 7][f], w[(S + 6) % 7][f]);
          // the reference arithmetic sums the axes x, y, z left to right and
          // fuses f + KO (-KOeps KO_const) (field_solver_EZ.cpp:350-420)
          if constexpr (XA) nu[f] = xa::fma(c.ko_c, xa::add(xa::add(kx, ky), kz), cv);
          else nu[f] = fma(kx + ky + kz, c.ko_c, cv);
        } else {
          nu[f] = cv;
        }
      });
      const uint32_t o = (uint32_t)k * sz + own;
      if constexpr (DG) {
        // dU_KO = (|B|^2 + |E|^2) after the pass minus before it, and
        // dU_KO_cum += it (field_solver_EZ.cpp:398-455)
        constexpr int C3 = (S + 3) % 7;  // the window slot of plane k
        const T u0 = xa::add(xa::dot3(w[C3][3], w[C3][3], w[C3][4], w[C3][4], w[C3][5], w[C3][5]),
                             xa::dot3(w[C3][0], w[C3][0], w[C3][1], w[C3][1], w[C3][2], w[C3][2]));
        const T u1 = xa::add(xa::dot3(nu[3], nu[3], nu[4], nu[4], nu[5], nu[5]),
                             xa::dot3(nu[0], nu[0], nu[1], nu[1], nu[2], nu[2]));
        const T dko = xa::sub(u1, u0);
        dg.p[5][o] = xa::add(dko, dg.p[5][o]);
        dg.p[2][o] = dko;
        apply_clamps_xa_dg<false>(nu[0], nu[1], nu[2], nu[3], nu[4], nu[5], dg, o);
      } else if constexpr (XA) {
        apply_clamps_xa(nu[0], nu[1], nu[2], nu[3], nu[4], nu[5]);
      } else {
        apply_clamps(c, nu[0], nu[1], nu[2], nu[3], nu[4], nu[5]);
      }
      if constexpr (BC) star_boundary(c, i, j, k, tko, nu);
      store_with_images(g, col, uout, k, o, nu);
      if constexpr (ZU == 1) {
#pragma unroll
        for (int q = 0; q < 6; ++q)
#pragma unroll
          for (int f = 0; f < 7; ++f) w[q][f] = w[q + 1][f];
      }
    }
    if constexpr (kKoRingSpare == 0) {
      __syncthreads();
      issue(k + 4 + PF, fslot(sc, PN{}, k));  // into the slot of plane k (or k-2 of 7)
    }
  };
  if constexpr (ZU == 7) {
    // planes past k1 in the last group only wait, synchronise and commit
    // empty copy groups (issue() copies nothing past kend)
#pragma unroll 1
    for (int k = k0; k < k1; k += 7) {
      plane(std::integral_constant<int, 0>{}, k);
      plane(std::integral_constant<int, 1>{}, k + 1);
      plane(std::integral_constant<int, 2>{}, k + 2);
      plane(std::integral_constant<int, 3>{}, k + 3);
      plane(std::integral_constant<int, 4>{}, k + 4);
      plane(std::integral_constant<int, 5>{}, k + 5);
      plane(std::integral_constant<int, 6>{}, k + 6);
    }
  } else {
#pragma unroll 1
    for (int k = k0; k < k1; ++k) plane(std::integral_constant<int, 0>{}, k);
  }
  cp_async_wait<0>();
}

}  // namespace coffee
