// Host side of the 2D axisymmetric solvers (log-spherical and cylindrical):
// checks of the configuration, the per-solver tables, the step loop and the
// batched step loop of many log-spherical runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "axisym_kernels.cuh"
#include "coffee_b200.h"
#include "coffee_internal.h"
#include "ez_launch.cuh"
#include "variants.h"

namespace coffee {

namespace {

constexpr int kTX = 32, kTY = 8;
// stage times of the cylindrical solver, shifted by one stage
// (field_solver_EZ_cylindrical.cu:684-685)
constexpr double kCsCyl[5] = {0.1496590219993, 0.3704009573644, 0.6222557631345,
                              0.9582821306784, 1.0};

struct Box {
  int lo0, hi0, lo1, hi1;
};

Box update_box(const coffee_env* env) {
  const int s = env->p.shift_ghost;
  const coffee_grid& g = env->grid;
  return {g.guard[0] - s, g.dims[0] - g.guard[0] + s, g.guard[1] - s, g.dims[1] - g.guard[1] + s};
}

// Reference coordinate of point n of axis a with stagger bit 1
// (src/data/grid.h:116-134), in field precision.
template <typename T>
T grid_pos(const coffee_env* env, int a, int n) {
  return (T)env->grid.lower[a] + (T)env->grid.delta[a] * (T)(n - env->grid.guard[a]);
}

template <typename T>
void fill_sph_const(const coffee_env* env, const void* tab, SphConst<T>* c) {
  const coffee_params& p = env->p;
  const coffee_grid& g = env->grid;
  const Box b = update_box(env);
  c->d0 = g.dims[0];
  c->d1 = g.dims[1];
  c->lo0 = b.lo0;
  c->hi0 = b.hi0;
  c->lo1 = b.lo1;
  c->hi1 = b.hi1;
  c->g0 = g.guard[0];
  c->g1 = g.guard[1];
  c->dx = (T)g.delta[0];
  c->dy = (T)g.delta[1];
  c->inv_dx = (T)(1.0 / (double)c->dx);
  c->inv_dy = (T)(1.0 / (double)c->dy);
  c->x0 = (T)g.lower[0];
  c->y0 = (T)g.lower[1];
  // kernel_boundary_axis_sph checks rows guard and dims - guard
  // (field_solver_EZ_spherical.cu:698-745)
  const T th_lo = grid_pos<T>(env, 1, g.guard[1]);
  const T th_hi = grid_pos<T>(env, 1, g.dims[1] - g.guard[1]);
  c->axis_lo = std::fabs((double)th_lo) < (double)c->dy / 2.0 ? g.guard[1] : -1;
  c->axis_hi =
      std::fabs((double)th_hi - M_PI) < (double)c->dy / 2.0 ? g.dims[1] - g.guard[1] : -1;
  c->dt = (T)p.dt;
  c->ch2 = (T)p.ch2;
  c->tau = (T)p.tau;
  c->gam_dt = (T)((T)p.damp_gamma / (T)p.dt);
  c->ko_c = (T)(p.KOeps / 64.0);
  c->calc_current = p.calc_current;
  c->edotb = p.use_edotb_damping;
  c->divB_clean = p.divB_clean;
  c->clean_ep = p.clean_ep;
  c->check_egb = p.check_egb;
  c->ko_geometry = p.KO_geometry;
  c->radius = (T)p.radius;
  c->b0 = (T)p.b0;
  c->omega = (T)p.omega;
  c->tp_start = (T)p.tp_start;
  c->tp_end = (T)p.tp_end;
  c->dw0 = (T)p.dw0;
  c->nT = (T)p.nT;
  c->thp1 = (T)p.thp1;
  c->thp2 = (T)p.thp2;
  c->tp_start1 = (T)p.tp_start1;
  c->tp_end1 = (T)p.tp_end1;
  c->dw1 = (T)p.dw1;
  c->nT1 = (T)p.nT1;
  c->thp11 = (T)p.thp11;
  c->thp21 = (T)p.thp21;
  // kernel_boundary_absorbing_sph (:771-775)
  c->xh = (T)((T)p.lower[0] + (T)p.size[0] - (T)p.pml[0] * c->dx);
  c->rh = (T)std::exp((double)c->xh);
  c->pmllen = (T)p.pmllen;
  c->sigpml = (T)p.sigpml;
  c->absorbing = p.pml[0] > 0 || p.shift_ghost > 0 ? 1 : 0;
  const T* t = static_cast<const T*>(tab);
  c->rt = t;
  c->st = t ? t + g.dims[0] : nullptr;
  c->ct = t ? t + g.dims[0] + g.dims[1] : nullptr;
}

template <typename T>
void fill_cyl_const(const coffee_env* env, CylConst<T>* c) {
  const coffee_params& p = env->p;
  const coffee_grid& g = env->grid;
  const Box b = update_box(env);
  c->d0 = g.dims[0];
  c->d1 = g.dims[1];
  c->lo0 = b.lo0;
  c->hi0 = b.hi0;
  c->lo1 = b.lo1;
  c->hi1 = b.hi1;
  c->g0 = g.guard[0];
  c->g1 = g.guard[1];
  c->dR = (T)g.delta[0];
  c->dz = (T)g.delta[1];
  c->inv_dR = (T)(1.0 / (double)c->dR);
  c->inv_dz = (T)(1.0 / (double)c->dz);
  c->R0 = (T)g.lower[0];
  c->z0 = (T)g.lower[1];
  c->axis_col = -1;
  for (int i = b.lo0; i < b.hi0; ++i)
    if (std::fabs((double)grid_pos<T>(env, 0, i)) < (double)c->dR / 4.0) c->axis_col = i;
  c->dt = (T)p.dt;
  c->ch2 = (T)p.ch2;
  c->tau = (T)p.tau;
  c->ko_c = (T)(p.KOeps / 64.0);
  c->clean_ep = p.clean_ep;
  c->check_egb = p.check_egb;
  c->radius = (T)p.radius;
  c->b0 = (T)p.b0;
  c->omega = (T)p.omega;
  c->tp_start = (T)p.tp_start;
  c->tp_end = (T)p.tp_end;
  c->dw0 = (T)p.dw0;
  // wpert window (field_solver_EZ_cylindrical.cu:419-426)
  double th1 = std::acos(std::sqrt(1.0 - 1.0 / (double)(T)p.rpert1));
  double th2 = std::acos(std::sqrt(1.0 - 1.0 / (double)(T)p.rpert2));
  if (th1 > th2) std::swap(th1, th2);
  c->th1 = (T)th1;
  c->th2 = (T)th2;
  // kernel_boundary_absorbing_cylindrical (:553-561)
  c->xh = (T)((T)p.lower[0] + (T)p.size[0] - (T)p.pml[0] * c->dR);
  c->xl = -c->xh;
  c->yh = (T)((T)p.lower[1] + (T)p.size[1] - (T)p.pml[1] * c->dz);
  c->yl = (T)((T)p.lower[1] + (T)p.pml[1] * c->dz);
  c->pmlscale = (T)((T)p.pmllen * c->dR);
  c->sigpml = (T)p.sigpml;
  c->absorbing = p.pml[0] > 0 || p.pml[1] > 0 || p.shift_ghost > 0 ? 1 : 0;
}

template <typename T>
F7<T> as_f7(void* const a[7]) {
  F7<T> f;
  for (int k = 0; k < 7; ++k) f.p[k] = static_cast<T*>(a[k]);
  return f;
}

dim3 box_grid(const Box& b) {
  return dim3((unsigned)((b.hi0 - b.lo0 + kTX - 1) / kTX),
              (unsigned)((b.hi1 - b.lo1 + kTY - 1) / kTY), 1);
}

template <typename T>
int sph_steps(const coffee_env* env, const void* tab, void* const A_[7], void* const B_[7],
              void* const dU_[7], void* const Un_[7], void* const aux_[5], double time, int nsteps,
              cudaStream_t st, LaunchHook* hook) {
  SphConst<T> c;
  fill_sph_const<T>(env, tab, &c);
  const F7<T> A = as_f7<T>(A_), Bb = as_f7<T>(B_), dU = as_f7<T>(dU_);
  F7<T> Un;
  for (int k = 0; k < 7; ++k) Un.p[k] = c.absorbing ? static_cast<T*>(Un_[k]) : nullptr;
  F5<T> aux;
  for (int k = 0; k < 5; ++k) aux.p[k] = aux_ ? static_cast<T*>(aux_[k]) : nullptr;
  const Box b = update_box(env);
  const dim3 grid = box_grid(b), block(kTX, kTY, 1);
  const unsigned axis_blocks = (unsigned)((b.hi0 - b.lo0 + 127) / 128);
  const bool has_axis = c.axis_lo >= 0 || c.axis_hi >= 0;
  const T dt = c.dt;
  T t = (T)time;
  // boundary_axis() at the start of evolve_fields (:966); idempotent after
  // the first step, so once per call
  if (has_axis && nsteps > 0) {
    sph_axis_kernel<T><<<axis_blocks, 128, 0, st>>>(c, A);
    COFFEE_CUDA_TRY(cudaGetLastError());
  }
  for (int step = 0; step < nsteps; ++step) {
    for (int s = 0; s < 5; ++s) {
      const F7<T>& src = (s % 2 == 0) ? A : Bb;
      const F7<T>& dst = (s % 2 == 0) ? Bb : A;
      int flags = 0;
      if (s == 4) flags |= AX_LAST | (aux_ ? AX_AUX : 0);
      if (s == 0 && c.absorbing) flags |= AX_WRITE_UN;
      const T tst = (T)(t + (T)kCs[s] * dt);
      const int kind = s == 0 ? COFFEE_KERNEL_STAGE_FIRST : COFFEE_KERNEL_STAGE;
      int rc = hook ? hook->before(kind) : COFFEE_OK;
      if (rc) return rc;
      if (s == 0)
        sph_stage_kernel<T, true><<<grid, block, 0, st>>>(c, src, dst, dU, Un, aux, (T)kAs[s],
                                                          (T)kBs[s], tst, flags);
      else
        sph_stage_kernel<T, false><<<grid, block, 0, st>>>(c, src, dst, dU, Un, aux, (T)kAs[s],
                                                           (T)kBs[s], tst, flags);
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook && (rc = hook->after(kind))) return rc;
      if (has_axis) {
        sph_axis_kernel<T><<<axis_blocks, 128, 0, st>>>(c, dst);
        COFFEE_CUDA_TRY(cudaGetLastError());
      }
    }
    int rc = hook ? hook->before(COFFEE_KERNEL_KO) : COFFEE_OK;
    if (rc) return rc;
    sph_ko_kernel<T><<<grid, block, 0, st>>>(c, Bb, A, (T)(t + dt));
    COFFEE_CUDA_TRY(cudaGetLastError());
    if (hook && (rc = hook->after(COFFEE_KERNEL_KO))) return rc;
    if (has_axis) {
      sph_axis_kernel<T><<<axis_blocks, 128, 0, st>>>(c, A);
      COFFEE_CUDA_TRY(cudaGetLastError());
    }
    t = (T)(t + dt);
  }
  return COFFEE_OK;
}

template <typename T>
int cyl_steps(const coffee_env* env, void* const A_[7], void* const B_[7], void* const dU_[7],
              void* const Un_[7], double time, int nsteps, cudaStream_t st, LaunchHook* hook) {
  CylConst<T> c;
  fill_cyl_const<T>(env, &c);
  const F7<T> A = as_f7<T>(A_), Bb = as_f7<T>(B_), dU = as_f7<T>(dU_);
  F7<T> Un;
  for (int k = 0; k < 7; ++k) Un.p[k] = c.absorbing ? static_cast<T*>(Un_[k]) : nullptr;
  const Box b = update_box(env);
  const dim3 grid = box_grid(b), block(kTX, kTY, 1);
  const T dt = c.dt;
  T t = (T)time;
  for (int step = 0; step < nsteps; ++step) {
    for (int s = 0; s < 5; ++s) {
      const F7<T>& src = (s % 2 == 0) ? A : Bb;
      const F7<T>& dst = (s % 2 == 0) ? Bb : A;
      int flags = 0;
      if (s == 4) flags |= AX_LAST;
      if (s == 0 && c.absorbing) flags |= AX_WRITE_UN;
      const T tst = (T)(t + (T)kCsCyl[s] * dt);
      const int kind = s == 0 ? COFFEE_KERNEL_STAGE_FIRST : COFFEE_KERNEL_STAGE;
      int rc = hook ? hook->before(kind) : COFFEE_OK;
      if (rc) return rc;
      if (s == 0)
        cyl_stage_kernel<T, true><<<grid, block, 0, st>>>(c, src, dst, dU, Un, (T)kAs[s],
                                                          (T)kBs[s], tst, flags);
      else
        cyl_stage_kernel<T, false><<<grid, block, 0, st>>>(c, src, dst, dU, Un, (T)kAs[s],
                                                           (T)kBs[s], tst, flags);
      COFFEE_CUDA_TRY(cudaGetLastError());
      if (hook && (rc = hook->after(kind))) return rc;
    }
    int rc = hook ? hook->before(COFFEE_KERNEL_KO) : COFFEE_OK;
    if (rc) return rc;
    cyl_ko_kernel<T><<<grid, block, 0, st>>>(c, Bb, A, Un, (T)(t + dt));
    COFFEE_CUDA_TRY(cudaGetLastError());
    if (hook && (rc = hook->after(COFFEE_KERNEL_KO))) return rc;
    t = (T)(t + dt);
  }
  return COFFEE_OK;
}

template <typename T>
int make_sph_table(const coffee_env* env, void** tab) {
  const coffee_grid& g = env->grid;
  const int n = g.dims[0] + 2 * g.dims[1];
  std::vector<T> h(n);
  // r = exp(x), sin / cos of theta at the grid coordinates, evaluated in
  // FP64 from the field-precision coordinates (metric_sph.h:90-122)
  for (int i = 0; i < g.dims[0]; ++i) h[i] = (T)std::exp((double)grid_pos<T>(env, 0, i));
  for (int j = 0; j < g.dims[1]; ++j) {
    const double th = (double)grid_pos<T>(env, 1, j);
    h[g.dims[0] + j] = (T)std::sin(th);
    h[g.dims[0] + g.dims[1] + j] = (T)std::cos(th);
  }
  *tab = nullptr;
  cudaError_t err = cudaMalloc(tab, sizeof(T) * n);
  if (err == cudaSuccess) err = cudaMemcpy(*tab, h.data(), sizeof(T) * n, cudaMemcpyHostToDevice);
  if (err != cudaSuccess) {
    if (*tab) cudaFree(*tab);
    *tab = nullptr;
    return fail(COFFEE_E_NOMEM, "log-spherical table: %s", cudaGetErrorString(err));
  }
  return COFFEE_OK;
}

// Run table for tile shape tx x ty (tx * ty = 256) with the runs in `order`
// (indices into runs); e.index keeps each run's position in the batch.
template <typename T>
int sph_batch_table_t(const SphRun* runs, const std::vector<int>& order, int tx, int ty,
                      void** dev_table, int* nblocks, int* naxis_blocks) {
  const int n = (int)order.size();
  std::vector<SphBatchEntry<T>> h(n);
  int tiles = 0, axis = 0;
  for (int q = 0; q < n; ++q) {
    const int m = order[q];
    SphBatchEntry<T>& e = h[q];
    std::memset(&e, 0, sizeof(e));
    fill_sph_const<T>(runs[m].env, runs[m].tab, &e.c);
    e.A = as_f7<T>(runs[m].A);
    e.B = as_f7<T>(runs[m].B);
    e.dU = as_f7<T>(runs[m].dU);
    for (int k = 0; k < 7; ++k)
      e.Un.p[k] = e.c.absorbing ? static_cast<T*>(runs[m].Un[k]) : nullptr;
    for (int k = 0; k < 5; ++k)
      e.aux.p[k] = runs[m].want_aux ? static_cast<T*>(runs[m].aux[k]) : nullptr;
    e.want_aux = runs[m].want_aux;
    e.index = m;
    const Box b = update_box(runs[m].env);
    const int gx = (b.hi0 - b.lo0 + tx - 1) / tx, gy = (b.hi1 - b.lo1 + ty - 1) / ty;
    e.tile0 = tiles;
    e.tiles_x = gx;
    tiles += gx * gy;
    e.axis0 = axis;
    axis += (b.hi0 - b.lo0 + 127) / 128;
  }
  *dev_table = nullptr;
  cudaError_t err = cudaMalloc(dev_table, sizeof(SphBatchEntry<T>) * n);
  if (err == cudaSuccess)
    err = cudaMemcpy(*dev_table, h.data(), sizeof(SphBatchEntry<T>) * n, cudaMemcpyHostToDevice);
  if (err != cudaSuccess) {
    if (*dev_table) cudaFree(*dev_table);
    *dev_table = nullptr;
    return fail(COFFEE_E_NOMEM, "batch table: %s", cudaGetErrorString(err));
  }
  *nblocks = tiles;
  *naxis_blocks = axis;
  return COFFEE_OK;
}

// Tile shapes the autotuner tries (256 threads each: the kernels' launch
// bounds) and the run orders.
constexpr int kTuneShapes[][2] = {{32, 8}, {64, 4}, {128, 2}, {16, 16}};

template <typename T>
int sph_batch_plan_t(const SphRun* runs, int n, bool tune, cudaStream_t st, SphBatchPlan* pl) {
  pl->elem = (int)sizeof(T);
  pl->n = n;
  std::vector<int> given(n), largest(n);
  for (int m = 0; m < n; ++m) given[m] = largest[m] = m;
  auto points = [&](int m) {
    const Box b = update_box(runs[m].env);
    return (long long)(b.hi0 - b.lo0) * (b.hi1 - b.lo1);
  };
  std::stable_sort(largest.begin(), largest.end(),
                   [&](int a, int b) { return points(a) > points(b); });
  int best_shape = 0, best_order = 0;
  double best_ms = 0;
  if (tune) {
    cudaEvent_t e0, e1;
    COFFEE_CUDA_TRY(cudaEventCreate(&e0));
    COFFEE_CUDA_TRY(cudaEventCreate(&e1));
    // every run at its own time: the first stage only evaluates the star
    std::vector<T> h0(n, T(0)), hdt(n);
    for (int m = 0; m < n; ++m) hdt[m] = (T)runs[m].env->p.dt;
    void *t0 = nullptr, *tdt = nullptr;
    cudaError_t err = cudaMalloc(&t0, sizeof(T) * n);
    if (err == cudaSuccess) err = cudaMalloc(&tdt, sizeof(T) * n);
    if (err == cudaSuccess) err = cudaMemcpy(t0, h0.data(), sizeof(T) * n, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(tdt, hdt.data(), sizeof(T) * n, cudaMemcpyHostToDevice);
    int rc = err == cudaSuccess ? COFFEE_OK
                                : fail(COFFEE_E_NOMEM, "batch tuning: %s", cudaGetErrorString(err));
    for (int o = 0; o < 2 && rc == COFFEE_OK; ++o) {
      for (int sh = 0; sh < 4 && rc == COFFEE_OK; ++sh) {
        const int tx = kTuneShapes[sh][0], ty = kTuneShapes[sh][1];
        void* tab = nullptr;
        int nb = 0, na = 0;
        rc = sph_batch_table_t<T>(runs, o ? largest : given, tx, ty, &tab, &nb, &na);
        if (rc) break;
        const auto* tt = static_cast<const SphBatchEntry<T>*>(tab);
        float best = 1e30f;
        for (int rep = 0; rep < 4 && rc == COFFEE_OK; ++rep) {
          cudaEventRecord(e0, st);
          sph_stage_batch_kernel<T, true><<<nb, dim3(tx, ty, 1), 0, st>>>(
              tt, n, 1, static_cast<const T*>(t0), static_cast<const T*>(tdt), T(0), (T)kAs[0],
              (T)kBs[0], 0);
          cudaEventRecord(e1, st);
          err = cudaEventSynchronize(e1);
          if (err == cudaSuccess) err = cudaGetLastError();
          float ms = 0;
          if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
          if (err != cudaSuccess) {
            rc = fail(COFFEE_E_CUDA, "batch tuning launch: %s", cudaGetErrorString(err));
            break;
          }
          if (rep > 0) best = std::min(best, ms);  // the first launch warms up
        }
        cudaFree(tab);
        if (rc == COFFEE_OK && (best_ms == 0 || best < best_ms)) {
          best_ms = best;
          best_shape = sh;
          best_order = o;
        }
      }
    }
    cudaFree(t0);
    cudaFree(tdt);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
  }
  pl->tx = kTuneShapes[best_shape][0];
  pl->ty = kTuneShapes[best_shape][1];
  pl->order = best_order;
  pl->tuned_ms = best_ms;
  int rc = sph_batch_table_t<T>(runs, best_order ? largest : given, pl->tx, pl->ty, &pl->table,
                                &pl->nblocks, &pl->naxis);
  if (rc) return rc;
  std::vector<T> hdt(n);
  for (int m = 0; m < n; ++m) hdt[m] = (T)runs[m].env->p.dt;
  cudaError_t err = cudaMalloc(&pl->tnow, 2 * sizeof(T) * n);
  if (err == cudaSuccess) err = cudaMalloc(&pl->tdt, sizeof(T) * n);
  if (err == cudaSuccess)
    err = cudaMemcpy(pl->tdt, hdt.data(), sizeof(T) * n, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&pl->cap, cudaStreamNonBlocking);
  if (err != cudaSuccess) return fail(COFFEE_E_NOMEM, "batch plan: %s", cudaGetErrorString(err));
  return COFFEE_OK;
}

// The launches of one step of every run: 5 x (stage + axis), KO + axis,
// then t += dt.  The times come from plan->tnow / tdt.
template <typename T>
int sph_batch_step_launches(const SphBatchPlan* pl, cudaStream_t st) {
  const auto* tab = static_cast<const SphBatchEntry<T>*>(pl->table);
  const T* tnow = static_cast<const T*>(pl->tnow);
  const T* tdt = static_cast<const T*>(pl->tdt);
  const int n = pl->n;
  const dim3 block(pl->tx, pl->ty, 1);
  for (int s = 0; s < 5; ++s) {
    const int to_b = (s % 2 == 0) ? 1 : 0;
    if (s == 0)
      sph_stage_batch_kernel<T, true><<<pl->nblocks, block, 0, st>>>(
          tab, n, to_b, tnow, tdt, (T)kCs[s], (T)kAs[s], (T)kBs[s], 0);
    else
      sph_stage_batch_kernel<T, false><<<pl->nblocks, block, 0, st>>>(
          tab, n, to_b, tnow, tdt, (T)kCs[s], (T)kAs[s], (T)kBs[s], s == 4);
    COFFEE_CUDA_TRY(cudaGetLastError());
    sph_axis_batch_kernel<T><<<pl->naxis, 128, 0, st>>>(tab, n, to_b);
    COFFEE_CUDA_TRY(cudaGetLastError());
  }
  sph_ko_batch_kernel<T><<<pl->nblocks, block, 0, st>>>(tab, n, tnow, tdt);
  COFFEE_CUDA_TRY(cudaGetLastError());
  sph_axis_batch_kernel<T><<<pl->naxis, 128, 0, st>>>(tab, n, 0);
  COFFEE_CUDA_TRY(cudaGetLastError());
  sph_batch_advance_kernel<T><<<(n + 127) / 128, 128, 0, st>>>(static_cast<T*>(pl->tnow), tdt, n);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

template <typename T>
int sph_batch_capture(SphBatchPlan* pl) {
  COFFEE_CUDA_TRY(cudaStreamBeginCapture(pl->cap, cudaStreamCaptureModeThreadLocal));
  const int rc = sph_batch_step_launches<T>(pl, pl->cap);
  cudaGraph_t g = nullptr;
  const cudaError_t err = cudaStreamEndCapture(pl->cap, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (err != cudaSuccess) return fail(COFFEE_E_CUDA, "batch step capture: %s", cudaGetErrorString(err));
  const cudaError_t e2 = cudaGraphInstantiate(&pl->step, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) {
    pl->step = nullptr;
    return fail(COFFEE_E_CUDA, "batch step graph: %s", cudaGetErrorString(e2));
  }
  return COFFEE_OK;
}

// Barriers per step of the persistent kernel: 5 x (stage, axis), KO, axis.
constexpr int kBarriersPerStep = 12;

// nsteps steps of the batch as cooperative launches of the persistent
// kernel (as many steps per launch as the 32-bit arrival count allows),
// then a read of the barrier status: COFFEE_E_TIMEOUT if a wait ran out.
// Synchronises the stream.
template <typename T>
int sph_batch_persistent_t(SphBatchPlan* pl, int nsteps, cudaStream_t st) {
  const long long per_step = (long long)kBarriersPerStep * pl->coop_grid;
  const int max_steps = (int)std::min<long long>(nsteps, 0xFFFFFFFFLL / per_step - 1);
  LsrkCoef<T> k;
  for (int s = 0; s < 5; ++s) {
    k.As[s] = (T)kAs[s];
    k.Bs[s] = (T)kBs[s];
    k.Cs[s] = (T)kCs[s];
  }
  const auto* tab = static_cast<const SphBatchEntry<T>*>(pl->table);
  T* tbuf = static_cast<T*>(pl->tnow);
  const T* tdt = static_cast<const T*>(pl->tdt);
  GridSync* gs = static_cast<GridSync*>(pl->sync);
  int n = pl->n, nb = pl->nblocks, na = pl->naxis;
  for (int done = 0; done < nsteps;) {
    int steps = std::min(max_steps, nsteps - done);
    // an even count leaves the current times in row 0 for the next launch
    // (the host sets row 0 again at the start of every call)
    if (steps < nsteps - done && (steps & 1)) --steps;
    COFFEE_CUDA_TRY(cudaMemsetAsync(gs, 0, sizeof(GridSync), st));
    long long lim = pl->wait_ns;
    int stall = pl->stall_block;
    void* args[] = {(void*)&tab, (void*)&n,     (void*)&nb,  (void*)&na,  (void*)&tbuf,
                    (void*)&tdt, (void*)&k,     (void*)&steps, (void*)&gs, (void*)&lim,
                    (void*)&stall};
    COFFEE_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)sph_batch_persistent_kernel<T>,
                                                dim3(pl->coop_grid), dim3(pl->tx, pl->ty, 1),
                                                args, 0, st));
    GridSync h{};
    COFFEE_CUDA_TRY(cudaMemcpyAsync(&h, gs, sizeof(GridSync), cudaMemcpyDeviceToHost, st));
    COFFEE_CUDA_TRY(cudaStreamSynchronize(st));
    if (h.status != 0)
      return fail(COFFEE_E_TIMEOUT,
                  "persistent batch step: grid barrier %d gave up after %lld ns (block %d)",
                  h.where, pl->wait_ns, h.block);
    done += steps;
  }
  return COFFEE_OK;
}

// nsteps evolve_fields calls of every run of the batch, each from its own
// time (advanced in field precision by its own dt): the stage / axis / KO
// sequence of sph_steps with one launch per phase for the whole batch.
template <typename T>
int sph_batch_run_t(SphBatchPlan* pl, const SphRun* runs, double* times, int nsteps,
                    bool use_graph, cudaStream_t st) {
  const int n = pl->n;
  if (nsteps <= 0) return COFFEE_OK;
  std::vector<T> t(n), dt(n);
  for (int m = 0; m < n; ++m) {
    t[m] = (T)times[m];
    dt[m] = (T)runs[m].env->p.dt;
  }
  // pageable source: staged at once, so the vector may go out of scope
  COFFEE_CUDA_TRY(cudaMemcpyAsync(pl->tnow, t.data(), sizeof(T) * n, cudaMemcpyHostToDevice, st));
  sph_axis_batch_kernel<T><<<pl->naxis, 128, 0, st>>>(
      static_cast<const SphBatchEntry<T>*>(pl->table), n, 0);
  COFFEE_CUDA_TRY(cudaGetLastError());
  if (pl->persistent) {
    int rc = sph_batch_persistent_t<T>(pl, nsteps, st);
    if (rc) return rc;
  } else if (use_graph && !pl->step) {
    int rc = sph_batch_capture<T>(pl);
    if (rc) return rc;
  }
  for (int step = 0; step < nsteps && !pl->persistent; ++step) {
    if (use_graph) {
      COFFEE_CUDA_TRY(cudaGraphLaunch(pl->step, st));
    } else {
      int rc = sph_batch_step_launches<T>(pl, st);
      if (rc) return rc;
    }
  }
  // the same field-precision arithmetic as the device's t += dt
  for (int step = 0; step < nsteps; ++step)
    for (int m = 0; m < n; ++m) t[m] = (T)(t[m] + dt[m]);
  for (int m = 0; m < n; ++m) times[m] = (double)t[m];
  return COFFEE_OK;
}

}  // namespace

int sph_batch_plan(const SphRun* runs, int n, int elem, bool tune, cudaStream_t st,
                   SphBatchPlan* plan) {
  return elem == 4 ? sph_batch_plan_t<float>(runs, n, tune, st, plan)
                   : sph_batch_plan_t<double>(runs, n, tune, st, plan);
}

int sph_batch_run(SphBatchPlan* plan, const SphRun* runs, double* times, int nsteps,
                  bool use_graph, cudaStream_t st) {
  return plan->elem == 4 ? sph_batch_run_t<float>(plan, runs, times, nsteps, use_graph, st)
                         : sph_batch_run_t<double>(plan, runs, times, nsteps, use_graph, st);
}

int sph_batch_set_persistent(SphBatchPlan* pl, bool on) {
  if (on && !pl->sync) {
    int per_sm = 0, dev = 0, sms = 0, coop = 0;
    const void* fn = pl->elem == 4 ? (const void*)sph_batch_persistent_kernel<float>
                                   : (const void*)sph_batch_persistent_kernel<double>;
    COFFEE_CUDA_TRY(cudaGetDevice(&dev));
    COFFEE_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return fail(COFFEE_E_CUDA, "the device has no cooperative launch");
    COFFEE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    COFFEE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, pl->tx * pl->ty, 0));
    if (per_sm < 1) return fail(COFFEE_E_CUDA, "the persistent batch kernel does not fit an SM");
    // no more CTAs than the largest phase has tiles
    pl->coop_grid = std::max(1, std::min(per_sm * sms, std::max(pl->nblocks, pl->naxis)));
    cudaError_t err = cudaMalloc(&pl->sync, sizeof(GridSync));
    if (err != cudaSuccess) {
      pl->sync = nullptr;
      return fail(COFFEE_E_NOMEM, "persistent batch: %s", cudaGetErrorString(err));
    }
  }
  pl->persistent = on;
  return COFFEE_OK;
}

void sph_batch_free(SphBatchPlan* plan) {
  if (plan->sync) cudaFree(plan->sync);
  if (plan->step) cudaGraphExecDestroy(plan->step);
  if (plan->cap) cudaStreamDestroy(plan->cap);
  if (plan->table) cudaFree(plan->table);
  if (plan->tnow) cudaFree(plan->tnow);
  if (plan->tdt) cudaFree(plan->tdt);
  *plan = SphBatchPlan();
}

int axisym_check(const coffee_env* env, int variant) {
  const coffee_params& p = env->p;
  const coffee_grid& g = env->grid;
  const char* name = variant == COFFEE_VARIANT_LOGSPH ? "log-spherical" : "cylindrical";
  if (p.N[2] != 1 || p.guard[2] != 0)
    return fail(COFFEE_E_CONFIG, "the %s solver is 2D: it needs N[2] = 1 and guard[2] = 0", name);
  for (int a = 0; a < 2; ++a) {
    if (p.periodic_boundary[a])
      return fail(COFFEE_E_CONFIG, "the %s solver has no periodic axis (axis %d)", name, a);
    if (p.N[a] < 4) return fail(COFFEE_E_CONFIG, "N[%d] must be >= 4", a);
    if (p.guard[a] < p.shift_ghost + 3)
      return fail(COFFEE_E_CONFIG, "the %s solver needs guard[%d] >= shift_ghost + 3", name, a);
  }
  if (variant == COFFEE_VARIANT_LOGSPH) {
    SphConst<float> c;
    fill_sph_const<float>(env, nullptr, &c);
    // the reference writes rows dims - guard + 1 .. + 3 at theta = pi
    // (field_solver_EZ_spherical.cu:734-744): one past the array when
    // guard[1] = 3
    if (c.axis_hi >= 0 && g.guard[1] < 4)
      return fail(COFFEE_E_CONFIG,
                  "theta reaches pi: the axis boundary writes 3 rows past theta = pi, so "
                  "guard[1] must be >= 4 (it is %d)",
                  g.guard[1]);
  } else {
    CylConst<float> c;
    fill_cyl_const<float>(env, &c);
    const Box b = update_box(env);
    if (c.axis_col >= 0 && c.axis_col != b.lo0)
      return fail(COFFEE_E_CONFIG,
                  "the R = 0 axis must be the first column of the update box (column %d, box "
                  "starts at %d)",
                  c.axis_col, b.lo0);
    if (c.axis_col >= 0 && c.axis_col < 3)
      return fail(COFFEE_E_CONFIG, "the axis boundary needs 3 columns below R = 0");
  }
  return COFFEE_OK;
}

int axisym_setup(const coffee_env* env, int variant, int elem, void** tab) {
  *tab = nullptr;
  if (variant != COFFEE_VARIANT_LOGSPH) return COFFEE_OK;
  return elem == 4 ? make_sph_table<float>(env, tab) : make_sph_table<double>(env, tab);
}

int axisym_steps(const coffee_env* env, int variant, int elem, const void* tab,
                 void* const A[7], void* const B[7], void* const dU[7], void* const Un[7],
                 void* const aux[5], double time, int nsteps, cudaStream_t st, LaunchHook* hook) {
  if (variant == COFFEE_VARIANT_LOGSPH)
    return elem == 4 ? sph_steps<float>(env, tab, A, B, dU, Un, aux, time, nsteps, st, hook)
                     : sph_steps<double>(env, tab, A, B, dU, Un, aux, time, nsteps, st, hook);
  return elem == 4 ? cyl_steps<float>(env, A, B, dU, Un, time, nsteps, st, hook)
                   : cyl_steps<double>(env, A, B, dU, Un, time, nsteps, st, hook);
}

}  // namespace coffee
