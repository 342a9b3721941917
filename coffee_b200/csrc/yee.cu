// Host side of the staggered (Yee) RK3 solvers: configuration checks, the
// launch geometry and the step loops of field_solver::evolve_fields
// (COFFEE_VARIANT_YEE, src/algorithms/field_solver.cu:690-726) and
// field_solver_gr::evolve_fields_gr (COFFEE_VARIANT_GRYEE,
// src/algorithms/field_solver_gr.cu:810-861).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "coffee_b200.h"
#include "coffee_internal.h"
#include "ez_launch.cuh"
#include "variants.h"
#include "gryee_kernels.cuh"
#include "yee_kernels.cuh"

namespace coffee {

namespace {

#ifndef COFFEE_YEE_BX
#define COFFEE_YEE_BX 32
#endif
#ifndef COFFEE_YEE_BY
#define COFFEE_YEE_BY 8
#endif
// streaming passes: one (i, j) column per thread; at 512^3, 32 x 8 and
// 64 x 4 take the same time, 32 x 4 is 9% slower
const dim3 kColBlock(COFFEE_YEE_BX, COFFEE_YEE_BY, 1);
const dim3 kStarBlock(32, 4, 2);  // star passes: one point per thread

// SSP-RK3 as E = c1 En + c2 E + c3 dE, and the time of the star boundary
// after each substep (field_solver.cu:694-718)
const double kC[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};

template <typename T>
T* tp(void* p) { return static_cast<T*>(p); }

// The interior points of one axis whose vertex coordinate lies within rl of
// 0, grown by one point on each side and clipped to [lo, hi): a box that
// holds every point of r < rl.
void star_range(double lower, double delta, int guard, int lo, int hi, double rl, int* a, int* b) {
  const double n0 = std::floor((-rl - lower) / delta) + guard - 1;
  const double n1 = std::ceil((rl - lower) / delta) + guard + 2;
  *a = (int)std::max<double>(lo, n0);
  *b = (int)std::min<double>(hi, n1);
  if (*b < *a) *b = *a;
}

template <typename T>
void fill_args(const coffee_env* env, void* const A[7], void* const B0[3], void* const Es[7],
               void* const Un[7], void* const Tb[7], YeeArgs<T>* a) {
  const coffee_params& p = env->p;
  const coffee_grid& gr = env->grid;
  build_const<T>(env, SEM_GPU_REF, &a->c);
  a->g = a->c.g;
  for (int d = 0; d < 3; ++d) {
    a->inv[d] = a->c.inv_delta[d];
    a->cc[d] = (T)p.dt * a->c.inv_delta[d];  // dev_params.dt * dev_grid.inv_delta
  }
  a->dt = (T)p.dt;
  for (int c = 0; c < 3; ++c) {
    a->E[c] = tp<T>(A[c]);
    a->B[c] = tp<T>(A[3 + c]);
    a->Eo[c] = tp<T>(A[c]);
    a->Bo[c] = tp<T>(A[3 + c]);
    a->B0[c] = B0 ? tp<T>(B0[c]) : nullptr;
    a->Es[c] = tp<T>(Es[c]);
    a->Bs[c] = tp<T>(Es[3 + c]);
    a->En[c] = tp<T>(Un[c]);
    a->Bn[c] = tp<T>(Un[3 + c]);
    a->Et[c] = tp<T>(Tb[c]);
    a->Bt[c] = tp<T>(Tb[3 + c]);
  }
  // kernel_boundary_absorbing_thread (boundary.cu:41-60): the box edges use
  // each axis' delta, the length scale delta[0].  The reference applies it
  // in every last substep whatever pml is (with pml 0 no vertex is outside).
  for (int d = 0; d < 3; ++d) {
    const T dl = a->c.delta[d];
    a->pml_hi[d] = (T)((T)p.lower[d] + (T)p.size[d] - (T)p.pml[d] * dl);
    a->pml_lo[d] = (T)((T)p.lower[d] + (T)p.pml[d] * dl);
  }
  a->pml_scale = (T)p.pmllen * a->c.delta[0];
  a->sigpml = (T)p.sigpml;
  a->absorbing = 1;
  a->star = p.problem == 1 ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    a->plo[d] = a->phi[d] = a->hlo[d] = a->hhi[d] = a->g.lo[d];
  }
  if (a->star) {
    const double rl = 2.0 * (double)(T)p.radius;
    for (int d = 0; d < 3; ++d) {
      star_range((double)a->c.lower[d], (double)a->c.delta[d], gr.guard[d], a->g.lo[d],
                 a->g.hi[d], rl, &a->plo[d], &a->phi[d]);
      a->hlo[d] = std::max(a->g.lo[d], a->plo[d] - 1);
      a->hhi[d] = std::min(a->g.hi[d], a->phi[d] + 1);
    }
    if (a->plo[0] >= a->phi[0] || a->plo[1] >= a->phi[1] || a->plo[2] >= a->phi[2]) a->star = 0;
  }
}

// z range per thread: enough (i, j, k-chunk) blocks for four waves of CTAs
int kchunk_for(const coffee_env* env, int nx, int ny, int nz) {
  int dev = env->device, sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long cols = (long long)((nx + kColBlock.x - 1) / kColBlock.x) *
                         ((ny + kColBlock.y - 1) / kColBlock.y);
  const long long want = 4LL * sms * 2;  // 2 CTAs per SM, 4 waves
  long long chunks = (want + cols - 1) / cols;
  chunks = std::max<long long>(1, std::min<long long>(chunks, nz));
  const int kc = (int)((nz + chunks - 1) / chunks);
  return std::max(kc, 8 < nz ? 8 : nz);
}

dim3 grid3(dim3 blk, int n0, int n1, int n2) {
  return dim3((unsigned)((n0 + blk.x - 1) / blk.x), (unsigned)((n1 + blk.y - 1) / blk.y),
              (unsigned)((n2 + blk.z - 1) / blk.z));
}

template <typename T>
int yee_steps_t(const coffee_env* env, void* const A[7], void* const B0[3], void* const Es[7],
                void* const Un[7], void* const Tb[7], double time, int nsteps, cudaStream_t st,
                LaunchHook* hook) {
  YeeArgs<T> a;
  fill_args<T>(env, A, B0, Es, Un, Tb, &a);
  const int nx = a.g.hi[0] - a.g.lo[0], ny = a.g.hi[1] - a.g.lo[1], nz = a.g.hi[2] - a.g.lo[2];
  a.kchunk = kchunk_for(env, nx, ny, nz);
  const dim3 gcol((unsigned)((nx + kColBlock.x - 1) / kColBlock.x),
                  (unsigned)((ny + kColBlock.y - 1) / kColBlock.y),
                  (unsigned)((nz + a.kchunk - 1) / a.kchunk));
  // the six faces of the shell: (x, y) threads over the largest face extent
  const dim3 gface = grid3(kColBlock, std::max(nx + 2, ny), std::max(ny + 2, nz), 1);
  const dim3 gshell(gface.x, gface.y, 6);
  const dim3 gguard = grid3(kColBlock, a.g.dims[0], a.g.dims[1], 1);
  const dim3 gstar_b = grid3(kStarBlock, a.phi[0] - a.plo[0] + 2, a.phi[1] - a.plo[1] + 2,
                             a.phi[2] - a.plo[2] + 2);
  const dim3 gstar_e = grid3(kStarBlock, a.phi[0] - a.plo[0], a.phi[1] - a.plo[1],
                             a.phi[2] - a.plo[2]);
  const dim3 gstar_s = grid3(kStarBlock, a.hhi[0] - a.hlo[0], a.hhi[1] - a.hlo[1],
                             a.hhi[2] - a.hlo[2]);
  const bool has_b0 = B0 != nullptr;
  const bool star_pb = env->p.problem == 1;
  const T dt = (T)env->p.dt;
  T t = (T)time;
  bool guards_synced = false;
  for (int step = 0; step < nsteps; ++step) {
    for (int sub = 0; sub < 3; ++sub) {
      const bool last = sub == 2;
      const T c1 = (T)kC[sub][0], c2 = (T)kC[sub][1], c3 = (T)kC[sub][2];
      yee_shell_kernel<T><<<gshell, kColBlock, 0, st>>>(a, 1);
      COFFEE_CUDA_TRY(cudaGetLastError());
      const int kind = sub == 0 ? COFFEE_KERNEL_STAGE_FIRST : COFFEE_KERNEL_STAGE;
      int rc = hook ? hook->before(kind) : COFFEE_OK;
      if (rc) return rc;
      if (sub == 0) {
        if (has_b0) yee_update_kernel<T, true, true><<<gcol, kColBlock, 0, st>>>(a, c1, c2, c3);
        else yee_update_kernel<T, true, false><<<gcol, kColBlock, 0, st>>>(a, c1, c2, c3);
      } else {
        if (has_b0) yee_update_kernel<T, false, true><<<gcol, kColBlock, 0, st>>>(a, c1, c2, c3);
        else yee_update_kernel<T, false, false><<<gcol, kColBlock, 0, st>>>(a, c1, c2, c3);
      }
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook && (rc = hook->after(kind))) return rc;
      if ((rc = hook ? hook->before(COFFEE_KERNEL_KO) : COFFEE_OK)) return rc;
      if (star_pb) {
        if (last) yee_clamp_kernel<T, true, false><<<gcol, kColBlock, 0, st>>>(a);
        else yee_clamp_kernel<T, false, false><<<gcol, kColBlock, 0, st>>>(a);
      } else {
        if (last) yee_clamp_kernel<T, true, true><<<gcol, kColBlock, 0, st>>>(a);
        else yee_clamp_kernel<T, false, true><<<gcol, kColBlock, 0, st>>>(a);
      }
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook && (rc = hook->after(COFFEE_KERNEL_KO))) return rc;
      if (star_pb) {
        // t + dt in Scalar, or t + 0.5 dt through double (field_solver.cu:697, 707, 717)
        const T ts = sub == 1 ? (T)((double)t + 0.5 * (double)dt) : (T)(t + dt);
        if (a.star) {
          yee_star_b_kernel<T><<<gstar_b, kStarBlock, 0, st>>>(a, ts);
          yee_star_e_kernel<T><<<gstar_e, kStarBlock, 0, st>>>(a);
          if (last) yee_star_store_kernel<T, true><<<gstar_s, kStarBlock, 0, st>>>(a);
          else yee_star_store_kernel<T, false><<<gstar_s, kStarBlock, 0, st>>>(a);
          COFFEE_CUDA_TRY(cudaGetLastError());
        }
        yee_guard_kernel<T, true><<<gguard, kColBlock, 0, st>>>(a);
        COFFEE_CUDA_TRY(cudaGetLastError());
      } else if (!guards_synced) {
        // the clamp pass wrote the images of the interior; this pass also
        // brings the guard points whose source is a non-periodic guard point
        // (corners of a mixed box) in line, after which they never change
        yee_guard_kernel<T, false><<<gguard, kColBlock, 0, st>>>(a);
        COFFEE_CUDA_TRY(cudaGetLastError());
        guards_synced = true;
      }
    }
    t = (T)(t + dt);
  }
  return COFFEE_OK;
}

}  // namespace

int yee_check(const coffee_env* env) {
  const coffee_params& p = env->p;
  if (p.shift_ghost != 0)
    return fail(COFFEE_E_CONFIG, "the staggered solver updates the interior only (shift_ghost 0)");
  const coffee_grid& g = env->grid;
  for (int a = 0; a < 3; ++a) {
    if (g.guard[a] < 1) return fail(COFFEE_E_CONFIG, "the staggered solver needs guard[%d] >= 1", a);
    if (p.periodic_boundary[a] && p.N[a] < g.guard[a])
      return fail(COFFEE_E_CONFIG, "periodic axis %d needs N >= guard", a);
  }
  const double n = (double)g.dims[0] * g.dims[1] * g.dims[2];
  if (n >= 2147483648.0)
    return fail(COFFEE_E_CONFIG, "the staggered solver indexes a rank's arrays in 32 bits");
  return COFFEE_OK;
}

int yee_steps(const coffee_env* env, int elem, void* const A[7], void* const B0[3],
              void* const Es[7], void* const Un[7], void* const Tb[7], double time, int nsteps,
              cudaStream_t st, LaunchHook* hook) {
  return elem == 4 ? yee_steps_t<float>(env, A, B0, Es, Un, Tb, time, nsteps, st, hook)
                   : yee_steps_t<double>(env, A, B0, Es, Un, Tb, time, nsteps, st, hook);
}

// ------------------------------------------------------ Kerr-Schild

namespace {

const dim3 kPointBlock(32, 4, 2);  // one point per thread

template <typename T>
int gryee_steps_t(const coffee_env* env, void* const A[7], void* const Es[7], void* const Un[7],
                  void* scratch, int nsteps, cudaStream_t st, LaunchHook* hook) {
  const coffee_params& p = env->p;
  GYeeArgs<T> g;
  fill_args<T>(env, A, nullptr, Es, Un, Es, &g.y);
  g.y.star = 0;
  g.spin = (T)p.a;
  g.calc_current = p.calc_current;
  g.clean_ep = p.clean_ep;
  g.check_egb = p.check_egb;
  // rH = 1 + sqrt(1 - a^2) through double, then 0.8, 0.01, 0.2 rH (field_solver_gr.cu:666-669)
  const T rH = (T)(1.0 + std::sqrt(1.0 - (double)(g.spin * g.spin)));
  g.r1 = (T)(0.8 * (double)rH);
  g.r2 = (T)(0.01 * (double)rH);
  g.dd = (T)(0.2 * (double)rH);
  for (int d = 0; d < 3; ++d) {
    g.half[d] = (T)((double)g.y.c.delta[d] / 2.0);
    g.upper[d] = (T)((T)p.lower[d] + (T)p.size[d]);
  }
  const size_t n = (size_t)g.y.g.dims[0] * g.y.g.dims[1] * g.y.g.dims[2];
  T* s = static_cast<T*>(scratch);
  for (int c = 0; c < 3; ++c) {
    g.Ed[c] = s + (0 + c) * n;
    g.Hd[c] = s + (3 + c) * n;
    g.Bd[c] = s + (6 + c) * n;
    g.Dc[c] = s + (10 + c) * n;
  }
  g.rho = s + 9 * n;
  const YeeArgs<T>& a = g.y;
  const int nx = a.g.hi[0] - a.g.lo[0], ny = a.g.hi[1] - a.g.lo[1], nz = a.g.hi[2] - a.g.lo[2];
  const dim3 geh = grid3(kPointBlock, a.g.dims[0] - 2, a.g.dims[1] - 2, a.g.dims[2] - 2);
  const dim3 gbox = grid3(kPointBlock, nx, ny, nz);
  const dim3 gface = grid3(kColBlock, std::max(nx + 2, ny), std::max(ny + 2, nz), 1);
  const dim3 gshell(gface.x, gface.y, 6);
  for (int step = 0; step < nsteps; ++step) {
    for (int sub = 0; sub < 3; ++sub) {
      const bool last = sub == 2;
      const bool clean = last && g.clean_ep;
      const T c1 = (T)kC[sub][0], c2 = (T)kC[sub][1], c3 = (T)kC[sub][2];
      gyee_eh_kernel<T><<<geh, kPointBlock, 0, st>>>(g);
      gyee_rho_kernel<T><<<gbox, kPointBlock, 0, st>>>(g);
      // the cleaning reads D* beyond the box where the state's D is; the
      // rescale reads zeros there (its dD is zero outside the box)
      yee_shell_kernel<T><<<gshell, kColBlock, 0, st>>>(a, clean ? 1 : 0);
      COFFEE_CUDA_TRY(cudaGetLastError());
      const int kind = sub == 0 ? COFFEE_KERNEL_STAGE_FIRST : COFFEE_KERNEL_STAGE;
      int rc = hook ? hook->before(kind) : COFFEE_OK;
      if (rc) return rc;
      if (sub == 0) gyee_update_kernel<T, true><<<gbox, kPointBlock, 0, st>>>(g, c1, c2, c3);
      else gyee_update_kernel<T, false><<<gbox, kPointBlock, 0, st>>>(g, c1, c2, c3);
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook && (rc = hook->after(kind))) return rc;
      if (clean) gyee_clean_kernel<T><<<gbox, kPointBlock, 0, st>>>(g);
      if ((rc = hook ? hook->before(COFFEE_KERNEL_KO) : COFFEE_OK)) return rc;
      if (last) gyee_clamp_kernel<T, true><<<gbox, kPointBlock, 0, st>>>(g);
      else gyee_clamp_kernel<T, false><<<gbox, kPointBlock, 0, st>>>(g);
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook && (rc = hook->after(COFFEE_KERNEL_KO))) return rc;
    }
  }
  return COFFEE_OK;
}

}  // namespace

int gryee_check(const coffee_env* env) {
  const coffee_params& p = env->p;
  if (p.shift_ghost != 0)
    return fail(COFFEE_E_CONFIG, "the staggered solver updates the interior only (shift_ghost 0)");
  for (int a = 0; a < 3; ++a) {
    if (p.periodic_boundary[a])
      return fail(COFFEE_E_CONFIG, "the Kerr-Schild solvers have no periodic axis (axis %d)", a);
    if (env->grid.guard[a] < 1)
      return fail(COFFEE_E_CONFIG, "the staggered solver needs guard[%d] >= 1", a);
  }
  if (!(std::fabs(p.a) < 1.0)) return fail(COFFEE_E_CONFIG, "the spin a must satisfy |a| < 1");
  const coffee_grid& g = env->grid;
  const double n = (double)g.dims[0] * g.dims[1] * g.dims[2];
  if (n >= 2147483648.0)
    return fail(COFFEE_E_CONFIG, "the staggered solver indexes a rank's arrays in 32 bits");
  return COFFEE_OK;
}

// E, H, the lowered B, rho and the cleaned D: 13 arrays, zero outside what
// the passes write (what the reference's arrays hold there)
int gryee_setup(const coffee_env* env, int elem, void** scratch) {
  const coffee_grid& g = env->grid;
  const size_t bytes = (size_t)g.dims[0] * g.dims[1] * g.dims[2] * (size_t)elem * 13;
  *scratch = nullptr;
  cudaError_t err = cudaMalloc(scratch, bytes);
  if (err == cudaSuccess) err = cudaMemset(*scratch, 0, bytes);
  if (err != cudaSuccess) {
    if (*scratch) cudaFree(*scratch);
    *scratch = nullptr;
    return fail(COFFEE_E_NOMEM, "staggered Kerr-Schild scratch allocation failed: %s",
                cudaGetErrorString(err));
  }
  return COFFEE_OK;
}

int gryee_steps(const coffee_env* env, int elem, void* const A[7], void* const Es[7],
                void* const Un[7], void* scratch, int nsteps, cudaStream_t st, LaunchHook* hook) {
  return elem == 4 ? gryee_steps_t<float>(env, A, Es, Un, scratch, nsteps, st, hook)
                   : gryee_steps_t<double>(env, A, Es, Un, scratch, nsteps, st, hook);
}

}  // namespace coffee
