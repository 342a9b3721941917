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
int sph_batch_create(const SphRun* runs, int n, int elem, void** dev_table, int* nblocks,
                     int* naxis_blocks);
int sph_batch_steps(const void* dev_table, int n, int elem, const SphRun* runs, double* times,
                    int nsteps, int nblocks, int naxis_blocks, cudaStream_t st);

// GR force-free solver in Kerr-Schild coordinates (COFFEE_VARIANT_GR).
int gr_check(const coffee_env* env);
int gr_setup(const coffee_env* env, int elem, void** ehbuf);
int gr_steps(const coffee_env* env, int elem, void* ehbuf, void* const A[7], void* const B[7],
             void* const dU[7], void* const Un[7], void* const aux[5], int nsteps,
             cudaStream_t st, LaunchHook* hook);

}  // namespace coffee
