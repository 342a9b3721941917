// Host side of the GR (Kerr-Schild) solver: configuration checks, scratch
// for the constitutive fields E and H, and the step loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "coffee_b200.h"
#include "coffee_internal.h"
#include "ez_launch.cuh"
#include "gr_kernels.cuh"
#include "variants.h"

namespace coffee {

namespace {

// 32 x 4 x 2 blocks: measured twice as fast as 32 x 8 x 1 or 32 x 2 x 4 for
// the stage kernel's stencil loads.
const dim3 kBlock(32, 4, 2);

template <typename T>
void fill_gr_const(const coffee_env* env, GrConst<T>* c) {
  const coffee_params& p = env->p;
  const coffee_grid& g = env->grid;
  const int s = p.shift_ghost;
  for (int a = 0; a < 3; ++a) {
    c->d[a] = g.dims[a];
    c->g[a] = g.guard[a];
    c->lo[a] = g.guard[a] - s;
    c->hi[a] = g.dims[a] - g.guard[a] + s;
    c->lower[a] = (T)g.lower[a];
    c->delta[a] = (T)g.delta[a];
    c->inv_delta[a] = (T)(1.0 / (double)c->delta[a]);
    // kernel_boundary_absorbing_thread (src/algorithms/boundary.cu:43-54)
    c->xh[a] = (T)((T)p.lower[a] + (T)p.size[a] - (T)p.pml[a] * c->delta[a]);
    c->xl[a] = (T)((T)p.lower[a] + (T)p.pml[a] * c->delta[a]);
  }
  c->a = (T)p.a;
  c->dt = (T)p.dt;
  c->tau = (T)p.tau;
  c->ko_c = (T)(p.KOeps / 64.0);
  c->calc_current = p.calc_current;
  c->divB_clean = p.divB_clean;
  c->clean_ep = p.clean_ep;
  c->check_egb = p.check_egb;
  c->pmlscale = (T)((T)p.pmllen * c->delta[0]);
  c->sigpml = (T)p.sigpml;
  // kernel_absorbing_inner (field_solver_gr_EZ.cu:617-621)
  const double rH = 1.0 + std::sqrt(1.0 - (double)c->a * (double)c->a);
  c->r1 = (T)(0.7 * rH);
  c->r2 = (T)(0.01 * rH);
  c->dd = (T)(0.2 * rH);
  c->absorbing = 1;  // the inner layer always acts in the last stage
  // the near-horizon box of the FP64 metric table: grid points within
  // kNearRH r_H of the hole along every axis (possibly empty)
  for (int a = 0; a < 3; ++a) {
    const double lo = -kNearRH * rH, hi = kNearRH * rH;
    int i0 = (int)std::ceil((lo - (double)g.lower[a]) / (double)g.delta[a]) + g.guard[a];
    int i1 = (int)std::floor((hi - (double)g.lower[a]) / (double)g.delta[a]) + g.guard[a] + 1;
    i0 = std::max(0, std::min(i0, g.dims[a]));
    i1 = std::max(i0, std::min(i1, g.dims[a]));
    c->nb_lo[a] = i0;
    c->nb_n[a] = i1 - i0;
  }
}

// points of the near-horizon metric table of env's grid
template <typename T>
size_t near_points(const coffee_env* env) {
  GrConst<T> c;
  fill_gr_const<T>(env, &c);
  return (size_t)c.nb_n[0] * c.nb_n[1] * c.nb_n[2];
}

template <typename T>
F7<T> as_f7(void* const a[7]) {
  F7<T> f;
  for (int k = 0; k < 7; ++k) f.p[k] = static_cast<T*>(a[k]);
  return f;
}

dim3 grid_over(int n0, int n1, int n2) {
  return dim3((unsigned)((n0 + kBlock.x - 1) / kBlock.x), (unsigned)((n1 + kBlock.y - 1) / kBlock.y),
              (unsigned)((n2 + kBlock.z - 1) / kBlock.z));
}

template <typename T>
int gr_steps_t(const coffee_env* env, void* ehbuf, void* const A_[7], void* const B_[7],
               void* const dU_[7], void* const Un_[7], void* const aux_[5], int nsteps,
               cudaStream_t st, LaunchHook* hook) {
  GrConst<T> c;
  fill_gr_const<T>(env, &c);
  const F7<T> A = as_f7<T>(A_), Bb = as_f7<T>(B_), dU = as_f7<T>(dU_), Un = as_f7<T>(Un_);
  F5<T> aux;
  for (int k = 0; k < 5; ++k) aux.p[k] = aux_ ? static_cast<T*>(aux_[k]) : nullptr;
  const size_t n = (size_t)c.d[0] * c.d[1] * c.d[2];
  // E and H of each field buffer: ehA of A, ehB of B
  F7<T> ehA, ehB, none;
  for (int k = 0; k < 6; ++k) {
    ehA.p[k] = static_cast<T*>(ehbuf) + k * n;
    ehB.p[k] = static_cast<T*>(ehbuf) + (6 + k) * n;
  }
  ehA.p[6] = ehB.p[6] = nullptr;
  for (int k = 0; k < 7; ++k) none.p[k] = nullptr;
  const T* sgt = static_cast<const T*>(ehbuf) + 12 * n;  // sqrt(gamma), set up by gr_setup
  const T* mt = sgt + n;                                  // the near-horizon metric table
  const dim3 gfull = grid_over(c.d[0], c.d[1], c.d[2]);
  const dim3 gbox = grid_over(c.hi[0] - c.lo[0], c.hi[1] - c.lo[1], c.hi[2] - c.lo[2]);
  // COFFEE_GR_EH_PER_STAGE=1: the E, H pass before every stage instead
  // (the same values; for comparisons)
  const char* ev = std::getenv("COFFEE_GR_EH_PER_STAGE");
  const bool per_stage = ev != nullptr && ev[0] == '1';
  // COFFEE_GR_TILED=1: FP32 stages stream through shared-memory tiles
  // (gr_stage_tile_kernel, the same arithmetic as gr_stage_kernel)
  const char* et = std::getenv("COFFEE_GR_TILED");
  const bool tiled = std::is_same<T, float>::value && et != nullptr && et[0] == '1';
  const int kchunk = COFFEE_GR_KCHUNK;
  const dim3 tblock(kGrTX, kGrTY, 1);
  const dim3 gtile((unsigned)((c.hi[0] - c.lo[0] + kGrTX - 1) / kGrTX),
                   (unsigned)((c.hi[1] - c.lo[1] + kGrTY - 1) / kGrTY),
                   (unsigned)((c.hi[2] - c.lo[2] + kchunk - 1) / kchunk));
  if (tiled && nsteps > 0) {
    static bool attr_set[2] = {false, false};
    for (int f = 0; f < 2; ++f) {
      if (attr_set[f]) continue;
      const void* fn = f ? (const void*)gr_stage_tile_kernel<true> : (const void*)gr_stage_tile_kernel<false>;
      COFFEE_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)gr_tile_smem_bytes()));
      attr_set[f] = true;
    }
  }
  if (nsteps > 0 && !per_stage) {
    // the fields may have changed since the last call (upload, pointer
    // access): E and H of both buffers, guards included; B's interior is
    // rewritten by the first stage
    gr_eh_kernel<T><<<gfull, kBlock, 0, st>>>(c, A, ehA, mt);
    COFFEE_CUDA_TRY(cudaGetLastError());
    gr_eh_kernel<T><<<gfull, kBlock, 0, st>>>(c, Bb, ehB, mt);
    COFFEE_CUDA_TRY(cudaGetLastError());
  }
  for (int step = 0; step < nsteps; ++step) {
    for (int s = 0; s < 5; ++s) {
      const F7<T>& src = (s % 2 == 0) ? A : Bb;
      const F7<T>& dst = (s % 2 == 0) ? Bb : A;
      const F7<T>& ehs = (s % 2 == 0) ? ehA : ehB;
      const F7<T>& ehd = per_stage ? none : ((s % 2 == 0) ? ehB : ehA);
      int flags = 0;
      if (s == 4) flags |= AX_LAST | (aux_ ? AX_AUX : 0);
      if (s == 0) flags |= AX_WRITE_UN;
      if (per_stage) {
        gr_eh_kernel<T><<<gfull, kBlock, 0, st>>>(c, src, ehs, mt);
        COFFEE_CUDA_TRY(cudaGetLastError());
      }
      const int kind = s == 0 ? COFFEE_KERNEL_STAGE_FIRST : COFFEE_KERNEL_STAGE;
      int rc = hook ? hook->before(kind) : COFFEE_OK;
      if (rc) return rc;
      if (tiled) {
        if constexpr (std::is_same<T, float>::value) {
          if (s == 0)
            gr_stage_tile_kernel<true><<<gtile, tblock, gr_tile_smem_bytes(), st>>>(
                c, src, ehs, dst, dU, Un, aux, mt, sgt, (T)kAs[s], (T)kBs[s], flags, ehd, kchunk);
          else
            gr_stage_tile_kernel<false><<<gtile, tblock, gr_tile_smem_bytes(), st>>>(
                c, src, ehs, dst, dU, Un, aux, mt, sgt, (T)kAs[s], (T)kBs[s], flags, ehd, kchunk);
        }
      } else if (s == 0) {
        gr_stage_kernel<T, true><<<gbox, kBlock, 0, st>>>(c, src, ehs, dst, dU, Un, aux, mt, sgt,
                                                          (T)kAs[s], (T)kBs[s], flags, ehd);
      } else {
        gr_stage_kernel<T, false><<<gbox, kBlock, 0, st>>>(c, src, ehs, dst, dU, Un, aux, mt, sgt,
                                                           (T)kAs[s], (T)kBs[s], flags, ehd);
      }
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook && (rc = hook->after(kind))) return rc;
    }
    int rc = hook ? hook->before(COFFEE_KERNEL_KO) : COFFEE_OK;
    if (rc) return rc;
    gr_ko_kernel<T><<<gbox, kBlock, 0, st>>>(c, Bb, A, mt, per_stage ? none : ehA);
    COFFEE_CUDA_TRY(cudaGetLastError());
    if (hook && (rc = hook->after(COFFEE_KERNEL_KO))) return rc;
  }
  return COFFEE_OK;
}

}  // namespace

int gr_check(const coffee_env* env) {
  const coffee_params& p = env->p;
  for (int a = 0; a < 3; ++a) {
    if (p.periodic_boundary[a])
      return fail(COFFEE_E_CONFIG, "the GR solver has no periodic axis (axis %d)", a);
    if (p.guard[a] < p.shift_ghost + 3)
      return fail(COFFEE_E_CONFIG, "the GR solver needs guard[%d] >= shift_ghost + 3", a);
  }
  if (!(std::fabs(p.a) < 1.0)) return fail(COFFEE_E_CONFIG, "the spin a must satisfy |a| < 1");
  return COFFEE_OK;
}

namespace {
template <typename T>
int gr_fill_metric(const coffee_env* env, void* ehbuf) {
  GrConst<T> c;
  fill_gr_const<T>(env, &c);
  const size_t n = (size_t)c.d[0] * c.d[1] * c.d[2];
  T* sg = static_cast<T*>(ehbuf) + 12 * n;
  gr_metric_kernel<T><<<grid_over(c.d[0], c.d[1], c.d[2]), kBlock>>>(c, sg + n, sg);
  COFFEE_CUDA_TRY(cudaGetLastError());
  COFFEE_CUDA_TRY(cudaDeviceSynchronize());
  return COFFEE_OK;
}
}  // namespace

// Scratch of the GR solver: E and H of each field buffer (2 x 6 arrays),
// sqrt(gamma) of every point and the near-horizon metric table
// (kMetricComps arrays over the box), the last two evaluated in FP64.
int gr_setup(const coffee_env* env, int elem, void** ehbuf) {
  const coffee_grid& g = env->grid;
  const size_t n = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
  const size_t nt = elem == 4 ? near_points<float>(env) : near_points<double>(env);
  *ehbuf = nullptr;
  cudaError_t err = cudaMalloc(ehbuf, (13 * n + kMetricComps * nt + 1) * (size_t)elem);
  if (err != cudaSuccess) {
    *ehbuf = nullptr;
    return fail(COFFEE_E_NOMEM, "GR scratch (E, H, metric table) allocation failed: %s",
                cudaGetErrorString(err));
  }
  const int rc = elem == 4 ? gr_fill_metric<float>(env, *ehbuf)
                           : gr_fill_metric<double>(env, *ehbuf);
  if (rc) {
    cudaFree(*ehbuf);
    *ehbuf = nullptr;
  }
  return rc;
}

int gr_steps(const coffee_env* env, int elem, void* ehbuf, void* const A[7], void* const B[7],
             void* const dU[7], void* const Un[7], void* const aux[5], int nsteps,
             cudaStream_t st, LaunchHook* hook) {
  return elem == 4 ? gr_steps_t<float>(env, ehbuf, A, B, dU, Un, aux, nsteps, st, hook)
                   : gr_steps_t<double>(env, ehbuf, A, B, dU, Un, aux, nsteps, st, hook);
}

}  // namespace coffee
