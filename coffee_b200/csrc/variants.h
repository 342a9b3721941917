// Entry points of the non-Cartesian solvers, called by the C ABI.
#pragma once

#include <cuda_runtime.h>

#include "coffee_b200.h"

struct coffee_env;

namespace coffee {

struct LaunchHook;

// 2D axisymmetric solvers (COFFEE_VARIANT_LOGSPH, COFFEE_VARIANT_CYL).
int axisym_check(const coffee_env* env, int variant);
int axisym_setup(const coffee_env* env, int variant, int elem, void** tab);
int axisym_steps(const coffee_env* env, int variant, int elem, const void* tab,
                 void* const A[7], void* const B[7], void* const dU[7], void* const Un[7],
                 void* const aux[5], double time, int nsteps, cudaStream_t st, LaunchHook* hook);

// Batches of log-spherical runs advanced by one launch per phase.
struct SphRun {
  const coffee_env* env;
  const void* tab;  // the run's r / sin / cos table
  void* A[7];
  void* B[7];
  void* dU[7];
  void* Un[7];
  void* aux[5];
  int want_aux;
};
constexpr int kMaxBatch = 128;

// A batch ready to step: its run table (laid out for the chosen tile shape
// and run order), the runs' times in device memory, and the captured step.
struct SphBatchPlan {
  int elem = 4, n = 0;
  void* table = nullptr;  // SphBatchEntry<T>[n]
  int nblocks = 0, naxis = 0;
  int tx = 32, ty = 8;    // tile shape of the stage / KO launches (autotuned)
  int order = 0;          // 0: runs in the given order, 1: largest first
  double tuned_ms = 0;    // first-stage time of the chosen layout
  void* tnow = nullptr;   // field-precision start time of the current step, per run
                          // (2 rows of n: the persistent kernel alternates them)
  void* tdt = nullptr;    // field-precision dt, per run
  cudaStream_t cap = nullptr;          // stream the step is captured on
  cudaGraphExec_t step = nullptr;      // one captured step (made on first use)
  // the persistent mode: one cooperative launch for all steps of a call
  bool persistent = false;
  int coop_grid = 0;                   // its CTAs (all resident)
  void* sync = nullptr;                // GridSync of its barriers
  long long wait_ns = 2000000000LL;    // limit of one barrier wait
  int stall_block = -1;                // test: this CTA skips its first arrival
};
// Build the plan; with `tune`, time the first stage for every candidate tile
// shape and run order (the first stage writes only scratch: the second field
// buffer and dU) and keep the fastest.
int sph_batch_plan(const SphRun* runs, int n, int elem, bool tune, cudaStream_t st,
                   SphBatchPlan* plan);
// nsteps steps of every run from times[m] (updated on return); with
// use_graph the step is the captured graph, replayed nsteps times.
int sph_batch_run(SphBatchPlan* plan, const SphRun* runs, double* times, int nsteps,
                  bool use_graph, cudaStream_t st);
void sph_batch_free(SphBatchPlan* plan);
// Switch the persistent mode on or off (sizes its cooperative grid).
int sph_batch_set_persistent(SphBatchPlan* plan, bool on);

// GR force-free solver in Kerr-Schild coordinates (COFFEE_VARIANT_GR).
int gr_check(const coffee_env* env);
int gr_setup(const coffee_env* env, int elem, void** ehbuf);
int gr_steps(const coffee_env* env, int elem, void* ehbuf, void* const A[7], void* const B[7],
             void* const dU[7], void* const Un[7], void* const aux[5], int nsteps,
             cudaStream_t st, LaunchHook* hook);

// Staggered (Yee) RK3 solver (COFFEE_VARIANT_YEE).  A: state E, B (and P,
// untouched); B0: background field or null; Es: E*, B' scratch; Un: the
// start-of-step copies; Tb: scratch of the star boundary.
int yee_check(const coffee_env* env);
int yee_steps(const coffee_env* env, int elem, void* const A[7], void* const B0[3],
              void* const Es[7], void* const Un[7], void* const Tb[7], double time, int nsteps,
              cudaStream_t st, LaunchHook* hook);

// Staggered RK3 solver in Kerr-Schild coordinates (COFFEE_VARIANT_GRYEE):
// A holds D (in E) and B; scratch from gryee_setup.
int gryee_check(const coffee_env* env);
int gryee_setup(const coffee_env* env, int elem, void** scratch);
int gryee_steps(const coffee_env* env, int elem, void* const A[7], void* const Es[7],
                void* const Un[7], void* scratch, int nsteps, cudaStream_t st, LaunchHook* hook);

}  // namespace coffee
