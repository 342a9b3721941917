// coffee_evolve_noalloc: the flat step loop without any device allocation.
//
// Some callers cannot let a library allocate device memory: hosts whose
// device memory is all handed out by their own allocator or pool, and hosts
// that cannot take the device-wide synchronisation that cudaMalloc/cudaFree
// can cause in the middle of their own pipeline.  This entry point advances
// the caller's own arrays with the same kernels as coffee_solver_step and
// takes its scratch -- the second field buffer, the LSRK accumulators and
// the start-of-step copy of the absorbing layer -- from the file-scope array
// below.  Every GPU that loads the library holds that array until the
// process exits.  All calls share it, so calls that overlap on the GPU race.
// Each call first copies the caller's fields into the second buffer; nothing
// else in the array has to start at zero (the first stage does not read the
// accumulators, and the start-of-step copy is written before it is read).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "coffee_b200.h"
#include "coffee_internal.h"
#include "ez_launch.cuh"

using namespace coffee;

#define COFFEE_NOALLOC_SCRATCH_BYTES (32u << 20)  // 32 MiB
#define COFFEE_NOALLOC_ARRAYS 21                  // 7 second buffer + 7 dU + 7 Un

static __device__ __align__(256) float g_noalloc_scratch[COFFEE_NOALLOC_SCRATCH_BYTES / 4];

namespace {

struct NoallocDevice {
  bool ready;
  float* scratch;  // device address of g_noalloc_scratch on this device
};
NoallocDevice g_noalloc_dev[64];
std::mutex g_noalloc_mutex;

// Once per device, with that device current: look up the device address of
// the static array (a host-side name of a __device__ variable is not a
// device address).  The address is cached for the life of the process; it
// belongs to the device's primary context and goes stale if the caller
// resets the device (cudaDeviceReset), which the header documents.
int noalloc_setup(int device, float** scratch) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (device < 0 || device >= 64) return fail(COFFEE_E_INVALID, "device %d out of range", device);
  NoallocDevice& d = g_noalloc_dev[device];
  if (!d.ready) {
    void* ptr = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (err != cudaSuccess)
      return fail(COFFEE_E_CUDA, "cudaGetSymbolAddress of the static scratch failed: %s",
                  cudaGetErrorString(err));
    d.scratch = static_cast<float*>(ptr);
    d.ready = true;
  }
  *scratch = d.scratch;
  return COFFEE_OK;
}

}  // namespace

extern "C" int coffee_evolve_noalloc(const coffee_params* p, int semantics,
                                     float* const fields[7], double time, int nsteps,
                                     void* stream) {
  clear_error();
  if (!p || !fields) return fail(COFFEE_E_INVALID, "coffee_evolve_noalloc: null argument");
  for (int f = 0; f < 7; ++f)
    if (!fields[f]) return fail(COFFEE_E_INVALID, "coffee_evolve_noalloc: field %d is null", f);
  if (nsteps < 0) return fail(COFFEE_E_INVALID, "nsteps must be >= 0");
  if (semantics != COFFEE_SEM_CPU_REF && semantics != COFFEE_SEM_GPU_REF)
    return fail(COFFEE_E_INVALID, "unknown semantics %d", semantics);
  if (p->problem < 0 || p->problem > 2)
    return fail(COFFEE_E_CONFIG, "problem %d is not supported by the flat EZ solver", p->problem);
  for (int a = 0; a < 3; ++a) {
    if (p->N[a] < 1) return fail(COFFEE_E_CONFIG, "N[%d] = %d must be >= 1", a, p->N[a]);
    if (p->guard[a] < p->shift_ghost + 3)
      return fail(COFFEE_E_CONFIG, "guard[%d] = %d: needs guard >= shift_ghost + 3", a,
                  p->guard[a]);
    if (p->periodic_boundary[a] && p->N[a] < p->guard[a])
      return fail(COFFEE_E_CONFIG, "periodic axis %d needs N >= guard", a);
    if (!(p->size[a] > 0)) return fail(COFFEE_E_CONFIG, "size[%d] must be > 0", a);
  }
  if (p->shift_ghost < 0 || !(p->dt > 0) || p->tau == 0)
    return fail(COFFEE_E_CONFIG, "shift_ghost >= 0, dt > 0 and tau != 0 are required");
  const size_t n = (size_t)(p->N[0] + 2 * p->guard[0]) * (size_t)(p->N[1] + 2 * p->guard[1]) *
                   (size_t)(p->N[2] + 2 * p->guard[2]);
  const size_t max_points = (COFFEE_NOALLOC_SCRATCH_BYTES / 4) / COFFEE_NOALLOC_ARRAYS;
  if (n > max_points)
    return fail(COFFEE_E_INVALID,
                "coffee_evolve_noalloc: %zu points per array exceed its static scratch "
                "(at most %zu points per array, e.g. a 64^3 interior with 3 guards)",
                n, max_points);
  int device = 0;
  COFFEE_CUDA_TRY(cudaGetDevice(&device));
  float* scratch = nullptr;
  int rc = noalloc_setup(device, &scratch);
  if (rc) return rc;

  // one rank's environment on the stack, built as coffee_env_create builds it
  coffee_env env;
  env.p = *p;
  env.device = device;
  for (int a = 0; a < 3; ++a) {
    env.grid.guard[a] = p->guard[a];
    env.grid.sizes[a] = (float)p->size[a];
    env.grid.lower[a] = p->lower[a];
    env.grid.dims[a] = p->N[a] + 2 * p->guard[a];
    env.grid.delta[a] = p->size[a] / p->N[a];
    env.grid.inv_delta[a] = 1.0 / env.grid.delta[a];
    env.grid.offset[a] = 0;
  }
  FlatLaunch launch;
  rc = flat_plan<float>(&env, semantics, &launch);
  if (rc) return rc;
  // pair copies read 8-byte aligned element pairs: the caller's arrays must
  // allow it (the scratch offsets are multiples of n, which is even then)
  for (int f = 0; f < 7; ++f)
    if (reinterpret_cast<uintptr_t>(fields[f]) % 8 != 0) launch.vec = false;
  EzConst<float> c;
  build_const<float>(&env, semantics, &c);

  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  F7<float> A, Bb, dU, Un;
  for (int f = 0; f < 7; ++f) {
    A.p[f] = fields[f];
    Bb.p[f] = scratch + (size_t)f * n;
    dU.p[f] = scratch + (size_t)(7 + f) * n;
    Un.p[f] = scratch + (size_t)(14 + f) * n;
  }
  F5<float> aux;
  for (int a = 0; a < 5; ++a) aux.p[a] = nullptr;
  // the second buffer carries the caller's guard values (the kernels never
  // write guards of non-periodic axes)
  for (int f = 0; f < 7; ++f)
    COFFEE_CUDA_TRY(cudaMemcpyAsync(Bb.p[f], A.p[f], n * sizeof(float), cudaMemcpyDeviceToDevice,
                                    st));
  return flat_steps<float>(c, launch, A, Bb, dU, Un, aux, false, time, nsteps, st, nullptr);
}
