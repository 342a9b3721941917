// Host-side helpers shared by the translation units that launch the flat
// EZ kernels: the environment record, tile shapes and their shared-memory
// sizes, the LSRK coefficients, the z-chunk choice and the construction of
// the kernels' parameter block from the simulation parameters.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

#include "coffee_b200.h"
#include "coffee_internal.h"
#include "ez_kernels.cuh"

// sim_environment of one rank on one GPU
struct coffee_env {
  coffee_params p;
  coffee_grid grid;
  int device;
  // fields and solvers created on this environment keep it alive: it is
  // deleted when it has been destroyed and the last of them is gone, in
  // whatever order the host releases them
  std::atomic<int> users{0};
  std::atomic<bool> released{false};
};

namespace coffee {


template <typename T> struct Shape;
// FP32 tile shapes; the defaults are the tuned values, the macros exist so
// that a build can be made with other shapes to measure them.
#ifndef COFFEE_F32_STY
#define COFFEE_F32_STY 16
#endif
#ifndef COFFEE_F32_SPF
#define COFFEE_F32_SPF 1
#endif
#ifndef COFFEE_F32_KTY
#define COFFEE_F32_KTY 8
#endif
#ifndef COFFEE_F32_KPF
#define COFFEE_F32_KPF 1
#endif
template <> struct Shape<float> {
  static constexpr int STX = 32, STY = COFFEE_F32_STY, SPF = COFFEE_F32_SPF;  // stage tile, prefetch
  static constexpr int KTX = 32, KTY = COFFEE_F32_KTY, KPF = COFFEE_F32_KPF;  // KO tile, prefetch
};
template <> struct Shape<double> {
  static constexpr int STX = 32, STY = 4, SPF = 1;
  static constexpr int KTX = 32, KTY = 4, KPF = 1;
};

template <typename T, int V, bool BC>
size_t stage_smem(bool first) {
  using S = Shape<T>;
  return stage_smem_bytes<T, S::STX, S::STY, S::SPF, V, BC>(first);
}
template <typename T, int V, bool BC>
size_t ko_smem() {
  using S = Shape<T>;
  return ko_smem_bytes<T, S::KTX, S::KTY, S::KPF, V, BC>();
}

// LSRK(5,4) coefficients of the reference (field_solver_EZ.cpp:1009-1014)
constexpr double kAs[5] = {0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257};
constexpr double kBs[5] = {0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488,
                       0.1530572479681};
constexpr double kCs[5] = {0, 0.1496590219993, 0.3704009573644, 0.6222557631345, 0.9582821306784};

// Choose the z chunk of a CTA: enough CTAs to fill the GPU in whole waves,
// while the 2H halo planes each chunk re-reads stay a small fraction.  The
// chunk is a multiple of `mult` (the kernel's z unroll, whose ring slots are
// then compile-time constants), except that it may be all nz planes.
inline int pick_kchunk(int nz, int nxy_tiles, int slots, int halo, int mult) {
  int best = nz;
  double best_cost = 1e300;
  const int step = mult > 1 ? mult : 4;
  for (int kc = step; kc <= nz + step - 1; kc += step) {
    const int kk = std::min(kc, nz);
    const long long ctas = (long long)nxy_tiles * ((nz + kk - 1) / kk);
    const double waves = std::ceil((double)ctas / (double)slots);
    const double cost = waves * (kk + 0.5 * halo);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = kk;
    }
    if (kk == nz) break;
  }
  return best;
}

template <typename T>
void build_const(const coffee_env* env, int semantics, EzConst<T>* c) {
  const coffee_params& p = env->p;
  const coffee_grid& gr = env->grid;
  std::memset(c, 0, sizeof(*c));
  GridGeom& g = c->g;
  for (int a = 0; a < 3; ++a) {
    g.dims[a] = gr.dims[a];
    g.guard[a] = gr.guard[a];
    g.N[a] = gr.dims[a] - 2 * gr.guard[a];
    g.lo[a] = gr.guard[a] - p.shift_ghost;
    g.hi[a] = gr.dims[a] - gr.guard[a] + p.shift_ghost;
    g.periodic[a] = p.periodic_boundary[a] ? 1 : 0;
    c->delta[a] = (T)(T(p.size[a]) / (T)p.N[a]);
    c->inv_delta[a] = (T)(1.0 / (double)c->delta[a]);
    c->lower[a] = (T)p.lower[a];
  }
  g.sy = gr.dims[0];
  g.sz = (long long)gr.dims[0] * gr.dims[1];
  c->dt = (T)p.dt;
  c->ch2 = (T)p.ch2;
  c->tau = (T)p.tau;
  c->inv_tau = (T)(1.0 / (double)c->tau);
  // -KOeps * KO_const with KO_const = -1/64 (FFE_DISSIPATION_ORDER 6)
  c->ko_c = -(T)p.KOeps * (T)(-1.0 / 64.0);
  c->gam_dt = (T)p.damp_gamma / (T)p.dt;
  c->use_edotb = p.use_edotb_damping;
  c->divB_clean = p.divB_clean;
  c->clean_ep = p.clean_ep;
  c->check_egb = p.check_egb;
  c->semantics = semantics;
  c->taper_lanes = (sizeof(T) == 4) ? 16 : 8;  // AVX-512 width of the reference CPU build
  c->problem = p.problem;
  bool abs_any = p.shift_ghost > 0;
  for (int a = 0; a < 3; ++a) {
    const T pm = (T)p.pml[a] * c->delta[a];
    c->pml_hi[a] = (T)p.lower[a] + (T)p.size[a] - pm;
    c->pml_lo[a] = (T)p.lower[a] + pm;
    c->pml_scale[a] = (T)p.pmllen * (semantics == SEM_CPU_REF ? c->delta[a] : c->delta[0]);
    if (p.pml[a] > 0) abs_any = true;
  }
  c->absorbing = abs_any ? 1 : 0;
  c->sigpml = (T)p.sigpml;
  c->radius = (T)p.radius;
  c->omega = (T)p.omega;
  c->b0 = (T)p.b0;
  c->p1 = (T)p.p1; c->p2 = (T)p.p2; c->p3 = (T)p.p3;
  c->q11 = (T)p.q11; c->q12 = (T)p.q12; c->q13 = (T)p.q13; c->q22 = (T)p.q22;
  c->q23 = (T)p.q23;
  c->qox = (T)p.q_offset_x; c->qoy = (T)p.q_offset_y; c->qoz = (T)p.q_offset_z;
  c->tp_start = (T)p.tp_start; c->tp_end = (T)p.tp_end; c->rpert1 = (T)p.rpert1;
  c->rpert2 = (T)p.rpert2; c->dw0 = (T)p.dw0; c->nT = (T)p.nT; c->ph1 = (T)p.ph1;
  c->ph2 = (T)p.ph2; c->dph = (T)p.dph; c->theta0 = (T)p.theta0; c->drpert = (T)p.drpert;
  c->tp_start1 = (T)p.tp_start1; c->tp_end1 = (T)p.tp_end1; c->rpert11 = (T)p.rpert11;
  c->rpert21 = (T)p.rpert21; c->dw1 = (T)p.dw1; c->nT1 = (T)p.nT1; c->ph11 = (T)p.ph11;
  c->ph21 = (T)p.ph21; c->dph1 = (T)p.dph1;
  c->pert_type = p.pert_type;
}

template <typename T>
inline F7<T> f7(void* const* a) {
  F7<T> r;
  for (int f = 0; f < 7; ++f) r.p[f] = static_cast<T*>(a[f]);
  return r;
}
template <typename T>
inline F7<const T> f7c(void* const* a) {
  F7<const T> r;
  for (int f = 0; f < 7; ++f) r.p[f] = static_cast<const T*>(a[f]);
  return r;
}

inline int num_sms(int device) {
  int n = 148;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  return n;
}

// Whether a run needs the star / absorbing-layer code in its kernels (the
// kernels are compiled with and without it, see ez_stage_kernel).
inline bool flat_needs_bc(const coffee_params& p, int semantics) {
  if (p.problem == 1 || (p.problem == 2 && semantics == SEM_CPU_REF)) return true;
  if (p.shift_ghost > 0) return true;
  for (int a = 0; a < 3; ++a)
    if (p.pml[a] > 0) return true;
  return false;
}

// Launch geometry of the flat kernels for one grid.
struct FlatLaunch {
  bool bc;   // star / absorbing-layer code compiled in
  bool vec;  // planes copied as aligned element pairs (even row length d0)
  bool xa;   // the CPU build's own arithmetic (CPU semantics, ez_refarith.cuh)
  bool dg;   // and its energy-change diagnostics (xa only)
  int kchunk_stage, kchunk_ko;
  dim3 grid_stage, grid_ko;
};

template <typename T, bool BC, int V, bool XA, bool DG = false>
struct FlatKernels {
  using S = Shape<T>;
  static constexpr auto first = ez_stage_kernel<T, S::STX, S::STY, S::SPF, true, BC, V, XA, DG>;
  static constexpr auto rest = ez_stage_kernel<T, S::STX, S::STY, S::SPF, false, BC, V, XA, DG>;
  static constexpr auto ko = ez_ko_kernel<T, S::KTX, S::KTY, S::KPF, BC, V, XA, DG>;

  static cudaError_t set_attributes() {
    cudaError_t e = cudaFuncSetAttribute(first, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)stage_smem<T, V, BC>(true));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(rest, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)stage_smem<T, V, BC>(false));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ko, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ko_smem<T, V, BC>());
    return e;
  }
  static cudaError_t occupancy(int* stage, int* kop) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(stage, rest, S::STX * S::STY,
                                                                  stage_smem<T, V, BC>(false));
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(kop, ko, S::KTX * S::KTY,
                                                        ko_smem<T, V, BC>());
    return e;
  }
  static void stage(bool is_first, const FlatLaunch& L, cudaStream_t st, const EzConst<T>& c,
                    const F7<const T>& src, const F7<T>& dst, const F7<T>& du, const F7<T>& un,
                    const F5<T>& aux, const F6<T>& dg, T As, T Bs, T tst, int flags) {
    const dim3 bs(S::STX, S::STY);
    if (is_first)
      first<<<L.grid_stage, bs, stage_smem<T, V, BC>(true), st>>>(
          c, src, dst, du, un, aux, dg, As, Bs, tst, L.kchunk_stage, flags);
    else
      rest<<<L.grid_stage, bs, stage_smem<T, V, BC>(false), st>>>(
          c, src, dst, du, un, aux, dg, As, Bs, tst, L.kchunk_stage, flags);
  }
  static void ko_pass(const FlatLaunch& L, cudaStream_t st, const EzConst<T>& c,
                      const F7<const T>& src, const F7<T>& dst, const F6<T>& dg, T tko) {
    ko<<<L.grid_ko, dim3(S::KTX, S::KTY), ko_smem<T, V, BC>(), st>>>(c, src, dst, dg, tko,
                                                                     L.kchunk_ko);
  }
};

// Calls fn(FlatKernels<T, BC, V, XA, DG>{}) for the kernel set L selects.
template <typename T, bool XA, bool DG, class Fn>
inline void with_flat_kernels_xa(const FlatLaunch& L, Fn&& fn) {
  if (L.bc) {
    if (L.vec) fn(FlatKernels<T, true, 2, XA, DG>{});
    else fn(FlatKernels<T, true, 1, XA, DG>{});
  } else {
    if (L.vec) fn(FlatKernels<T, false, 2, XA, DG>{});
    else fn(FlatKernels<T, false, 1, XA, DG>{});
  }
}
template <typename T, class Fn>
inline void with_flat_kernels(const FlatLaunch& L, Fn&& fn) {
  if (L.xa && L.dg) with_flat_kernels_xa<T, true, true>(L, fn);
  else if (L.xa) with_flat_kernels_xa<T, true, false>(L, fn);
  else with_flat_kernels_xa<T, false, false>(L, fn);
}

// Set the shared-memory limits of every flat kernel of precision T on the
// current device and plan the launch geometry of `env`'s grid.
// reference_arith: the CPU semantics run in the CPU build's own arithmetic
// (the default); false selects the regrouped, faster arithmetic.
// energy_diag: with the reference arithmetic, also accumulate the CPU
// build's energy-change diagnostics.
template <typename T>
inline int flat_plan(const coffee_env* env, int semantics, FlatLaunch* L,
                     bool reference_arith = true, bool energy_diag = false) {
  using S = Shape<T>;
  L->bc = flat_needs_bc(env->p, semantics);
  L->vec = env->grid.dims[0] % 2 == 0;
  L->xa = reference_arith && semantics == SEM_CPU_REF;
  L->dg = L->xa && energy_diag;
  // the shared-memory limits of the four kernel sets of this arithmetic (a
  // caller may still switch the pair copies off, as coffee_noalloc.cu does)
  if (L->dg) {
    COFFEE_CUDA_TRY((FlatKernels<T, true, 1, true, true>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, false, 1, true, true>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, true, 2, true, true>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, false, 2, true, true>::set_attributes()));
  } else if (L->xa) {
    COFFEE_CUDA_TRY((FlatKernels<T, true, 1, true>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, false, 1, true>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, true, 2, true>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, false, 2, true>::set_attributes()));
  } else {
    COFFEE_CUDA_TRY((FlatKernels<T, true, 1, false>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, false, 1, false>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, true, 2, false>::set_attributes()));
    COFFEE_CUDA_TRY((FlatKernels<T, false, 2, false>::set_attributes()));
  }
  // the flat kernels index an array with 32-bit element offsets (an FP32
  // array of 2^31 points alone would take a twentieth of the GPU's memory,
  // and a run holds at least 21 of them)
  const long long npts =
      (long long)env->grid.dims[0] * env->grid.dims[1] * (long long)env->grid.dims[2];
  if (npts >= (1LL << 31))
    return fail(COFFEE_E_CONFIG, "%lld points per array: the flat solver takes fewer than 2^31",
                npts);
  int per_sm_stage = 1, per_sm_ko = 1;
  cudaError_t occ = cudaSuccess;
  with_flat_kernels<T>(*L, [&](auto K) { occ = decltype(K)::occupancy(&per_sm_stage, &per_sm_ko); });
  COFFEE_CUDA_TRY(occ);
  if (per_sm_stage < 1 || per_sm_ko < 1)
    return fail(COFFEE_E_CUDA, "stage/KO kernels cannot be resident (occupancy 0)");
  const int sms = num_sms(env->device);
  const coffee_params& p = env->p;
  int box[3];
  for (int a = 0; a < 3; ++a) box[a] = p.N[a] + 2 * p.shift_ghost;
  const int sx = (box[0] + S::STX - 1) / S::STX, sy = (box[1] + S::STY - 1) / S::STY;
  // a kernel whose ring length equals its z unroll needs chunks of a
  // multiple of it (its ring slots are then compile-time constants)
  auto chunk_mult = [](int unroll, int ring) { return unroll == ring ? unroll : 1; };
  L->kchunk_stage = pick_kchunk(
      box[2], sx * sy, sms * per_sm_stage, 4,
      L->bc ? chunk_mult(stage_zunroll<true>(), stage_ring<true, S::SPF>())
            : chunk_mult(stage_zunroll<false>(), stage_ring<false, S::SPF>()));
  L->grid_stage = dim3(sx, sy, (box[2] + L->kchunk_stage - 1) / L->kchunk_stage);
  const int kx = (box[0] + S::KTX - 1) / S::KTX, ky = (box[1] + S::KTY - 1) / S::KTY;
  L->kchunk_ko = pick_kchunk(box[2], kx * ky, sms * per_sm_ko, 6,
                             L->bc ? chunk_mult(ko_zunroll<true>(), ko_ring<true, S::KPF>())
                                   : chunk_mult(ko_zunroll<false>(), ko_ring<false, S::KPF>()));
  L->grid_ko = dim3(kx, ky, (box[2] + L->kchunk_ko - 1) / L->kchunk_ko);
  return COFFEE_OK;
}

// Optional callbacks around every launch of flat_steps (timing).
struct LaunchHook {
  virtual int before(int kind) = 0;  // kind: COFFEE_KERNEL_*
  virtual int after(int kind) = 0;
  virtual ~LaunchHook() {}
};

// nsteps evolve_fields calls from `time` (reference field_solver_EZ.cpp:1007-1073):
// 5 stages A -> B -> A -> B -> A -> B, then the KO pass B -> A, advancing
// time by dt in field precision after each step (src/main-alfven3d.cpp:61,119).
template <typename T>
inline int flat_steps(const EzConst<T>& c, const FlatLaunch& L, const F7<T>& A, const F7<T>& Bb,
                      const F7<T>& dU, const F7<T>& Un, const F5<T>& aux, bool want_aux,
                      double time, int nsteps, cudaStream_t st, LaunchHook* hook,
                      const F6<T>* dg = nullptr) {
  F6<T> dgv;
  for (int a = 0; a < 6; ++a) dgv.p[a] = dg ? dg->p[a] : nullptr;
  if (L.dg && !dg) return fail(COFFEE_E_INVALID, "energy diagnostics planned without arrays");
  const T dt = c.dt;
  T t = (T)time;
  for (int step = 0; step < nsteps; ++step) {
    for (int i = 0; i < 5; ++i) {
      const F7<T>& src = (i % 2 == 0) ? A : Bb;
      const F7<T>& dst = (i % 2 == 0) ? Bb : A;
      F7<const T> srcc;
      for (int a = 0; a < 7; ++a) srcc.p[a] = src.p[a];
      int flags = 0;
      if (i == 4) flags |= ST_LAST;
      if (i == 4 && want_aux) flags |= ST_AUX;
      if (i == 0 && c.absorbing) flags |= ST_WRITE_UN;
      const T tst = t + (T)kCs[i] * dt;
      const int kind = (i == 0) ? COFFEE_KERNEL_STAGE_FIRST : COFFEE_KERNEL_STAGE;
      if (hook) {
        int rc = hook->before(kind);
        if (rc) return rc;
      }
      with_flat_kernels<T>(L, [&](auto K) {
        decltype(K)::stage(i == 0, L, st, c, srcc, dst, dU, Un, aux, dgv, (T)kAs[i], (T)kBs[i],
                           tst, flags);
      });
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook) {
        int rc = hook->after(kind);
        if (rc) return rc;
      }
    }
    F7<const T> srcc;
    for (int a = 0; a < 7; ++a) srcc.p[a] = Bb.p[a];
    if (hook) {
      int rc = hook->before(COFFEE_KERNEL_KO);
      if (rc) return rc;
    }
    with_flat_kernels<T>(L, [&](auto K) { decltype(K)::ko_pass(L, st, c, srcc, A, dgv, t + dt); });
    COFFEE_CUDA_TRY(cudaGetLastError());
    if (hook) {
      int rc = hook->after(COFFEE_KERNEL_KO);
      if (rc) return rc;
    }
    t = t + dt;
  }
  return COFFEE_OK;
}

}  // namespace coffee
