// C ABI of the B200 field-update library (declared in include/coffee_b200.h):
// environment, field storage, the flat EZ solver and its diagnostics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "coffee_b200.h"
#include "coffee_fld.h"
#include "coffee_internal.h"
#include "ez_launch.cuh"
#include "variants.h"
#include "yee_kernels.cuh"

#define COFFEE_VERSION_STRING "coffee_b200 0.1 (sm_100a)"

namespace coffee {

static thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }

}  // namespace coffee

using namespace coffee;

// ------------------------------------------------------------------ handles

// coffee_env is defined in ez_launch.cuh

struct coffee_fields {
  coffee_env* env;
  int elem;                          // 4 or 8
  size_t n;                          // points per array, guards included
  void* d[COFFEE_NUM_FIELDS];        // device arrays; J/divE/divB allocated on demand
  uint64_t generation;               // bumped whenever the host may have changed the fields
};

struct coffee_solver {
  coffee_env* env;
  coffee_fields* f;
  int variant;
  int semantics;
  cudaStream_t stream;
  void* B[7];   // second field buffer (stages alternate A -> B -> A ...)
  void* dU[7];  // LSRK accumulators dE, dB, dP
  void* Un[7];  // start-of-step copy, read by the absorbing layer
  bool absorbing;
  int aux;
  int timing;
  int arith;    // COFFEE_ARITH_* of the flat solver
  int taper_lanes;  // SIMD lanes of the CPU build's taper (0: by precision)
  int energy_diag;  // the CPU build's energy-change diagnostics kept
  uint64_t synced_generation;
  FlatLaunch launch;
  void* vtab;  // tables / scratch of a non-Cartesian variant (device), or null
  std::vector<cudaEvent_t> events;   // pairs around each launch (timing mode)
  std::vector<int> event_kind;       // COFFEE_KERNEL_* of each pair
  int events_used;
  cudaEvent_t ev_begin, ev_end;
  double* d_partials;
  int* d_count;
  int partial_blocks;
};

// ------------------------------------------------------------ kernel shapes

namespace {
// Periodic guard fill of all 7 arrays: every guard point of a periodic axis
// takes the value of the interior point at the wrapped coordinates.
template <typename T>
__global__ void fill_guards_kernel(const GridGeom g, const F7<T> u, const long long n) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % g.dims[0]);
    const int j = (int)((idx / g.dims[0]) % g.dims[1]);
    const int k = (int)(idx / g.sz);
    int c[3] = {i, j, k};
    bool moved = false;
    for (int a = 0; a < 3; ++a) {
      if (!g.periodic[a]) continue;
      if (c[a] < g.guard[a]) { c[a] += g.N[a]; moved = true; }
      else if (c[a] >= g.dims[a] - g.guard[a]) { c[a] -= g.N[a]; moved = true; }
    }
    if (!moved) continue;
    const long long src = (long long)c[2] * g.sz + (long long)c[1] * g.sy + c[0];
    for (int f = 0; f < 7; ++f) u.p[f][idx] = u.p[f][src];
  }
}

// ----------------------------------------------------------- diagnostics
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// One FP64 partial per block over the interior points.  what: see
// COFFEE_DIAG_*.  The energy region is that of total_energy
// (field_solver_EZ.cu:755-795): outside the star (problem 1) and strictly
// inside the absorbing layers.
// Staggered fields (COFFEE_VARIANT_YEE): each component is first
// interpolated to the vertex, as field_solver::total_energy does
// (field_solver.cu:829-866), and div B is the cell-centred forward
// difference that the staggered update keeps constant.
template <typename T>
__device__ __forceinline__ void vertex_values(const F7<const T>& u, uint32_t o, int sy, int sz,
                                              double e[3], double b[3]) {
  e[0] = interp_at<kStE[0], kStRho>(u.p[0], o, sy, sz);
  e[1] = interp_at<kStE[1], kStRho>(u.p[1], o, sy, sz);
  e[2] = interp_at<kStE[2], kStRho>(u.p[2], o, sy, sz);
  b[0] = interp_at<kStB[0], kStRho>(u.p[3], o, sy, sz);
  b[1] = interp_at<kStB[1], kStRho>(u.p[4], o, sy, sz);
  b[2] = interp_at<kStB[2], kStRho>(u.p[5], o, sy, sz);
}

template <typename T>
__global__ void diag_kernel(const EzConst<T> c, const F7<const T> u, const int what,
                            const T pml_xl0, const T pml_xl1, const T pml_xl2, const T pml_xh0,
                            const T pml_xh1, const T pml_xh2, const int stag, double* partials) {
  const GridGeom& g = c.g;
  const int n0 = g.N[0], n1 = g.N[1], n2 = g.N[2];
  const long long total = (long long)n0 * n1 * n2;
  const bool is_max = (what == COFFEE_DIAG_MAX_EDOTB || what == COFFEE_DIAG_MAX_EOVERB);
  double acc = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = g.guard[0] + (int)(q % n0);
    const int j = g.guard[1] + (int)((q / n0) % n1);
    const int k = g.guard[2] + (int)(q / ((long long)n0 * n1));
    const long long o = (long long)k * g.sz + (long long)j * g.sy + i;
    double v = 0.0;
    if (what == COFFEE_DIAG_ENERGY_E || what == COFFEE_DIAG_ENERGY_B) {
      const T x = grid_pos(c, 0, i), y = grid_pos(c, 1, j), z = grid_pos(c, 2, k);
      const T r = sqrt(x * x + y * y + z * z);
      const bool in_star = (c.problem == 1 && r < c.radius);
      if (!in_star && x < pml_xh0 && x > pml_xl0 && y < pml_xh1 && y > pml_xl1 &&
          z < pml_xh2 && z > pml_xl2) {
        const int b = (what == COFFEE_DIAG_ENERGY_E) ? 0 : 3;
        if (stag) {
          double e[3], bb[3];
          vertex_values(u, (uint32_t)o, (int)g.sy, (int)g.sz, e, bb);
          const double* f = b == 0 ? e : bb;
          v = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
        } else {
          for (int a = 0; a < 3; ++a) {
            const double f = (double)u.p[b + a][o];
            v += f * f;
          }
        }
      }
    } else if (what == COFFEE_DIAG_DIVB_L2 && stag) {
      const long long s[3] = {1, g.sy, g.sz};
      double d = 0.0;
      for (int a = 0; a < 3; ++a) {
        const T* f = u.p[3 + a];
        d += ((double)f[o + s[a]] - (double)f[o]) * (double)c.inv_delta[a];
      }
      v = d * d;
    } else if (what == COFFEE_DIAG_DIVB_L2) {
      double d = 0.0;
      const long long s[3] = {1, g.sy, g.sz};
      for (int a = 0; a < 3; ++a) {
        const T* f = u.p[3 + a];
        const double m2 = f[o - 2 * s[a]], m1 = f[o - s[a]], p1 = f[o + s[a]], p2 = f[o + 2 * s[a]];
        d += ((m2 - p2) + 8.0 * (p1 - m1)) / 12.0 * (double)c.inv_delta[a];
      }
      v = d * d;
    } else {
      double e[3] = {u.p[0][o], u.p[1][o], u.p[2][o]};
      double bb[3] = {u.p[3][o], u.p[4][o], u.p[5][o]};
      if (stag) vertex_values(u, (uint32_t)o, (int)g.sy, (int)g.sz, e, bb);
      const double ex = e[0], ey = e[1], ez = e[2];
      const double bx = bb[0], by = bb[1], bz = bb[2];
      const double B2 = fmax(bx * bx + by * by + bz * bz, (double)Tiny<T>::v);
      if (what == COFFEE_DIAG_MAX_EDOTB)
        v = fabs(ex * bx + ey * by + ez * bz) / B2;
      else
        v = sqrt((ex * ex + ey * ey + ez * ez) / B2);
    }
    acc = is_max ? fmax(acc, v) : acc + v;
  }
  __shared__ double red[32];
  acc = is_max ? warp_max(acc) : warp_sum(acc);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = acc;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    double v = lane < nw ? red[lane] : 0.0;
    v = is_max ? warp_max(v) : warp_sum(v);
    if (lane == 0) partials[blockIdx.x] = v;
  }
}

// Poynting luminosity through the sphere |x| = r (no reference counterpart):
// the flux of S = E x B, as the shell average
// L(r) = sum over interior points of (S . x/|x|) w(|x| - r) dV with the tent
// w(s) = max(0, 1 - |s|/h) / h (which integrates to 1 over s), h the largest
// grid spacing and dV = dx dy dz; coordinates and products in FP64.  The
// tent keeps the lattice-point noise of a thin shell well below 1%.
template <typename T>
__global__ void luminosity_kernel(const EzConst<T> c, const F7<const T> u, const double lx,
                                  const double ly, const double lz, const double dx,
                                  const double dy, const double dz, const double r,
                                  const double h, double* partials) {
  const GridGeom& g = c.g;
  const int n0 = g.N[0], n1 = g.N[1], n2 = g.N[2];
  const long long total = (long long)n0 * n1 * n2;
  const double ih = 1.0 / h;
  double acc = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int ii = (int)(q % n0), jj = (int)((q / n0) % n1), kk = (int)(q / ((long long)n0 * n1));
    const double x = lx + dx * ii, y = ly + dy * jj, z = lz + dz * kk;
    const double rr = sqrt(x * x + y * y + z * z);
    const double wt = 1.0 - fabs(rr - r) * ih;
    if (wt <= 0.0 || rr <= 0.0) continue;
    const long long o = (long long)(kk + g.guard[2]) * g.sz +
                        (long long)(jj + g.guard[1]) * g.sy + (ii + g.guard[0]);
    const double ex = u.p[0][o], ey = u.p[1][o], ez = u.p[2][o];
    const double bx = u.p[3][o], by = u.p[4][o], bz = u.p[5][o];
    const double sx = ey * bz - ez * by, sy = ez * bx - ex * bz, sz = ex * by - ey * bx;
    acc += (sx * x + sy * y + sz * z) / rr * wt;
  }
  __shared__ double red[32];
  acc = warp_sum(acc);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = acc;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    double v = lane < nw ? red[lane] : 0.0;
    v = warp_sum(v);
    if (lane == 0) partials[blockIdx.x] = v * (dx * dy * dz) * ih;
  }
}

template <typename T>
__global__ void count_nonfinite_kernel(const F7<const T> u, const long long n, int* count) {
  int local = 0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x)
    for (int f = 0; f < 7; ++f)
      if (!isfinite((double)u.p[f][idx])) ++local;
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}


}  // namespace

// ------------------------------------------------------------------ errors

extern "C" const char* coffee_last_error_string(void) { return g_last_error.c_str(); }
extern "C" const char* coffee_version(void) { return COFFEE_VERSION_STRING; }

// --------------------------------------------------------------- env

extern "C" int coffee_env_create(const coffee_params* p, int device, coffee_env** out) {
  clear_error();
  if (!p || !out) return fail(COFFEE_E_INVALID, "coffee_env_create: null argument");
  *out = nullptr;
  for (int a = 0; a < 3; ++a) {
    if (p->N[a] < 1) return fail(COFFEE_E_CONFIG, "N[%d] = %d must be >= 1", a, p->N[a]);
    // an axis of one point without guards is the third axis of a 2D run;
    // every solver reads at least one point beyond the update box (the EZ
    // solvers check their own three at solver creation)
    const bool plane_axis = p->N[a] == 1 && p->guard[a] == 0;
    if (!plane_axis && p->guard[a] < p->shift_ghost + 1)
      return fail(COFFEE_E_CONFIG, "guard[%d] = %d: needs guard >= shift_ghost + 1 = %d", a,
                  p->guard[a], p->shift_ghost + 1);
    if (p->periodic_boundary[a] && p->N[a] < p->guard[a])
      return fail(COFFEE_E_CONFIG, "periodic axis %d needs N >= guard (N=%d, guard=%d)", a,
                  p->N[a], p->guard[a]);
    if (!(p->size[a] > 0)) return fail(COFFEE_E_CONFIG, "size[%d] must be > 0", a);
  }
  if (p->shift_ghost < 0) return fail(COFFEE_E_CONFIG, "shift_ghost must be >= 0");
  if (!(p->dt > 0)) return fail(COFFEE_E_CONFIG, "dt must be > 0");
  if (p->tau == 0) return fail(COFFEE_E_CONFIG, "tau must be nonzero");
  const long long pts = (long long)(p->N[0] + 2 * p->guard[0]) * (p->N[1] + 2 * p->guard[1]) *
                        (p->N[2] + 2 * p->guard[2]);
  if (pts > (1LL << 40)) return fail(COFFEE_E_CONFIG, "grid too large");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(COFFEE_E_CUDA, "no CUDA device available");
  if (device < 0 || device >= ndev) return fail(COFFEE_E_INVALID, "device %d out of range", device);
  coffee_env* e = new (std::nothrow) coffee_env;
  if (!e) return fail(COFFEE_E_NOMEM, "out of host memory");
  e->p = *p;
  e->device = device;
  // sim_environment::sim_environment (src/sim_env_impl.hpp:52-60), one rank
  for (int a = 0; a < 3; ++a) {
    e->grid.guard[a] = p->guard[a];
    e->grid.sizes[a] = (float)p->size[a];
    e->grid.lower[a] = p->lower[a];
    e->grid.dims[a] = p->N[a] + 2 * p->guard[a];
    e->grid.delta[a] = p->size[a] / p->N[a];
    e->grid.inv_delta[a] = 1.0 / e->grid.delta[a];
    e->grid.offset[a] = 0;
  }
  *out = e;
  return COFFEE_OK;
}

extern "C" int coffee_env_destroy(coffee_env* env) {
  if (!env) return COFFEE_OK;
  env->released = true;
  if (env->users.load() == 0) delete env;
  return COFFEE_OK;
}

// A fields or solver object created on `env` is gone.
static void env_drop_user(coffee_env* env) {
  if (env->users.fetch_sub(1) == 1 && env->released.load()) delete env;
}

extern "C" int coffee_env_grid(const coffee_env* env, coffee_grid* grid) {
  if (!env || !grid) return fail(COFFEE_E_INVALID, "coffee_env_grid: null argument");
  *grid = env->grid;
  return COFFEE_OK;
}

extern "C" int coffee_env_params(const coffee_env* env, coffee_params* p) {
  if (!env || !p) return fail(COFFEE_E_INVALID, "coffee_env_params: null argument");
  *p = env->p;
  return COFFEE_OK;
}

// ------------------------------------------------------------------ fields

extern "C" int coffee_fields_create(coffee_env* env, int elem_size, coffee_fields** out) {
  clear_error();
  if (!env || !out) return fail(COFFEE_E_INVALID, "coffee_fields_create: null argument");
  if (elem_size != 4 && elem_size != 8)
    return fail(COFFEE_E_INVALID, "elem_size must be 4 or 8, got %d", elem_size);
  *out = nullptr;
  COFFEE_CUDA_TRY(cudaSetDevice(env->device));
  coffee_fields* f = new (std::nothrow) coffee_fields;
  if (!f) return fail(COFFEE_E_NOMEM, "out of host memory");
  std::memset(f, 0, sizeof(*f));
  f->env = env;
  f->elem = elem_size;
  f->n = (size_t)env->grid.dims[0] * env->grid.dims[1] * env->grid.dims[2];
  for (int a = 0; a < 7; ++a) {
    cudaError_t err = cudaMalloc(&f->d[a], f->n * elem_size);
    if (err == cudaSuccess) err = cudaMemset(f->d[a], 0, f->n * elem_size);
    if (err != cudaSuccess) {
      const size_t bytes = f->n * (size_t)elem_size;
      for (int b = 0; b <= a; ++b) cudaFree(f->d[b]);
      delete f;
      return fail(COFFEE_E_NOMEM, "cudaMalloc of field %d (%zu bytes) failed: %s", a, bytes,
                  cudaGetErrorString(err));
    }
  }
  f->generation = 1;
  env->users++;
  *out = f;
  return COFFEE_OK;
}

extern "C" int coffee_fields_destroy(coffee_fields* f) {
  if (!f) return COFFEE_OK;
  cudaSetDevice(f->env->device);
  for (int a = 0; a < COFFEE_NUM_FIELDS; ++a)
    if (f->d[a]) cudaFree(f->d[a]);
  (void)cudaGetLastError();  // leave no error of a release for the next call to find
  coffee_env* env = f->env;
  delete f;
  env_drop_user(env);
  return COFFEE_OK;
}

static int ensure_field(coffee_fields* f, int id) {
  if (id < 0 || id >= COFFEE_NUM_FIELDS) return fail(COFFEE_E_INVALID, "field id %d out of range", id);
  if (!f->d[id]) {
    COFFEE_CUDA_TRY(cudaSetDevice(f->env->device));
    COFFEE_CUDA_TRY(cudaMalloc(&f->d[id], f->n * f->elem));
    COFFEE_CUDA_TRY(cudaMemset(f->d[id], 0, f->n * f->elem));
  }
  return COFFEE_OK;
}

extern "C" int coffee_fields_ptr(coffee_fields* f, int id, void** dev_ptr) {
  clear_error();
  if (!f || !dev_ptr) return fail(COFFEE_E_INVALID, "coffee_fields_ptr: null argument");
  int rc = ensure_field(f, id);
  if (rc) return rc;
  *dev_ptr = f->d[id];
  if (id < 7) ++f->generation;  // the caller may write through it
  return COFFEE_OK;
}

extern "C" int coffee_fields_upload(coffee_fields* f, int id, const void* host) {
  clear_error();
  if (!f || !host) return fail(COFFEE_E_INVALID, "coffee_fields_upload: null argument");
  COFFEE_CUDA_TRY(cudaSetDevice(f->env->device));
  const size_t bytes = f->n * f->elem;
  if (id == -1) {
    for (int a = 0; a < 7; ++a)
      COFFEE_CUDA_TRY(cudaMemcpy(f->d[a], (const char*)host + a * bytes, bytes,
                                 cudaMemcpyHostToDevice));
  } else {
    int rc = ensure_field(f, id);
    if (rc) return rc;
    COFFEE_CUDA_TRY(cudaMemcpy(f->d[id], host, bytes, cudaMemcpyHostToDevice));
  }
  if (id < 7) ++f->generation;  // E, B, P: the solvers re-copy their second buffer
  return COFFEE_OK;
}

extern "C" int coffee_fields_download(coffee_fields* f, int id, void* host) {
  clear_error();
  if (!f || !host) return fail(COFFEE_E_INVALID, "coffee_fields_download: null argument");
  COFFEE_CUDA_TRY(cudaSetDevice(f->env->device));
  COFFEE_CUDA_TRY(cudaDeviceSynchronize());
  const size_t bytes = f->n * f->elem;
  if (id == -1) {
    for (int a = 0; a < 7; ++a)
      COFFEE_CUDA_TRY(
          cudaMemcpy((char*)host + a * bytes, f->d[a], bytes, cudaMemcpyDeviceToHost));
  } else {
    int rc = ensure_field(f, id);
    if (rc) return rc;
    COFFEE_CUDA_TRY(cudaMemcpy(host, f->d[id], bytes, cudaMemcpyDeviceToHost));
  }
  return COFFEE_OK;
}

template <typename T>
static int fill_guards_t(coffee_fields* f, cudaStream_t stream) {
  EzConst<T> c;
  build_const<T>(f->env, SEM_CPU_REF, &c);
  const int threads = 256;
  const long long n = (long long)f->n;
  const int blocks = (int)std::min<long long>((n + threads - 1) / threads, 148LL * 32);
  fill_guards_kernel<T><<<blocks, threads, 0, stream>>>(c.g, f7<T>(f->d), n);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

namespace {
struct FourierModes {
  int nb, nv;
  const double *kb, *bamp, *phib, *kv, *vamp, *phiv;  // device pointers
};

template <typename T>
__global__ void init_fourier_kernel(const EzConst<T> c, const F7<T> u, const long long n,
                                    const double b0x, const double b0y, const double b0z,
                                    const FourierModes m) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % c.g.dims[0]);
    const int j = (int)((idx / c.g.dims[0]) % c.g.dims[1]);
    const int k = (int)(idx / c.g.sz);
    // coordinates of the vertex, as the host generator computes them (FP64)
    const double x = (double)c.lower[0] + (double)c.delta[0] * (double)(i - c.g.guard[0]);
    const double y = (double)c.lower[1] + (double)c.delta[1] * (double)(j - c.g.guard[1]);
    const double z = (double)c.lower[2] + (double)c.delta[2] * (double)(k - c.g.guard[2]);
    double B[3] = {b0x, b0y, b0z}, v[3] = {0, 0, 0};
    for (int q = 0; q < m.nb; ++q) {
      const double s = sin(m.kb[3 * q] * x + m.kb[3 * q + 1] * y + m.kb[3 * q + 2] * z + m.phib[q]);
      for (int a = 0; a < 3; ++a) B[a] += m.bamp[3 * q + a] * s;
    }
    for (int q = 0; q < m.nv; ++q) {
      const double s = sin(m.kv[3 * q] * x + m.kv[3 * q + 1] * y + m.kv[3 * q + 2] * z + m.phiv[q]);
      for (int a = 0; a < 3; ++a) v[a] += m.vamp[3 * q + a] * s;
    }
    u.p[0][idx] = (T)(-(v[1] * B[2] - v[2] * B[1]));
    u.p[1][idx] = (T)(-(v[2] * B[0] - v[0] * B[2]));
    u.p[2][idx] = (T)(-(v[0] * B[1] - v[1] * B[0]));
    u.p[3][idx] = (T)B[0];
    u.p[4][idx] = (T)B[1];
    u.p[5][idx] = (T)B[2];
    u.p[6][idx] = (T)0;
  }
}
}  // namespace

extern "C" int coffee_fields_init_fourier(coffee_fields* f, const double b0[3], int nb,
                                          const double* kb, const double* bamp,
                                          const double* phib, int nv, const double* kv,
                                          const double* vamp, const double* phiv) {
  clear_error();
  if (!f || !b0 || nb < 0 || nv < 0 || (nb > 0 && (!kb || !bamp || !phib)) ||
      (nv > 0 && (!kv || !vamp || !phiv)))
    return fail(COFFEE_E_INVALID, "coffee_fields_init_fourier: bad argument");
  COFFEE_CUDA_TRY(cudaSetDevice(f->env->device));
  const size_t nd = (size_t)7 * (nb + nv) + 1;
  std::vector<double> h(nd, 0.0);
  double* p = h.data();
  std::memcpy(p, kb, sizeof(double) * 3 * nb);
  std::memcpy(p + 3 * nb, bamp, sizeof(double) * 3 * nb);
  std::memcpy(p + 6 * nb, phib, sizeof(double) * nb);
  double* q = p + 7 * nb;
  std::memcpy(q, kv, sizeof(double) * 3 * nv);
  std::memcpy(q + 3 * nv, vamp, sizeof(double) * 3 * nv);
  std::memcpy(q + 6 * nv, phiv, sizeof(double) * nv);
  double* d = nullptr;
  COFFEE_CUDA_TRY(cudaMalloc(&d, sizeof(double) * nd));
  cudaError_t err = cudaMemcpy(d, h.data(), sizeof(double) * nd, cudaMemcpyHostToDevice);
  if (err != cudaSuccess) {
    cudaFree(d);
    return fail(COFFEE_E_CUDA, "init_fourier upload: %s", cudaGetErrorString(err));
  }
  FourierModes m{nb, nv, d, d + 3 * nb, d + 6 * nb, d + 7 * nb, d + 7 * nb + 3 * nv,
                 d + 7 * nb + 6 * nv};
  const long long n = (long long)f->n;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 64);
  if (f->elem == 4) {
    EzConst<float> c;
    build_const<float>(f->env, SEM_CPU_REF, &c);
    init_fourier_kernel<float><<<blocks, 256>>>(c, f7<float>(f->d), n, b0[0], b0[1], b0[2], m);
  } else {
    EzConst<double> c;
    build_const<double>(f->env, SEM_CPU_REF, &c);
    init_fourier_kernel<double><<<blocks, 256>>>(c, f7<double>(f->d), n, b0[0], b0[1], b0[2], m);
  }
  err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaDeviceSynchronize();
  cudaFree(d);
  if (err != cudaSuccess) return fail(COFFEE_E_CUDA, "init_fourier: %s", cudaGetErrorString(err));
  ++f->generation;
  return COFFEE_OK;
}

extern "C" int coffee_fields_fill_guards(coffee_fields* f) {
  clear_error();
  if (!f) return fail(COFFEE_E_INVALID, "coffee_fields_fill_guards: null argument");
  COFFEE_CUDA_TRY(cudaSetDevice(f->env->device));
  int rc = (f->elem == 4) ? fill_guards_t<float>(f, 0) : fill_guards_t<double>(f, 0);
  if (rc) return rc;
  COFFEE_CUDA_TRY(cudaDeviceSynchronize());
  ++f->generation;
  return COFFEE_OK;
}

// ------------------------------------------------------------------ solver

template <typename T>
static int configure_solver(coffee_solver* s) {
  return flat_plan<T>(s->env, s->semantics, &s->launch, s->arith == COFFEE_ARITH_REFERENCE,
                      s->energy_diag != 0);
}

extern "C" int coffee_solver_create(coffee_env* env, coffee_fields* f, int variant,
                                    int semantics, void* stream, coffee_solver** out) {
  clear_error();
  if (!env || !f || !out) return fail(COFFEE_E_INVALID, "coffee_solver_create: null argument");
  *out = nullptr;
  if (f->env != env) return fail(COFFEE_E_INVALID, "fields belong to another environment");
  if (variant != COFFEE_VARIANT_FLAT && variant != COFFEE_VARIANT_LOGSPH &&
      variant != COFFEE_VARIANT_CYL && variant != COFFEE_VARIANT_GR &&
      variant != COFFEE_VARIANT_YEE && variant != COFFEE_VARIANT_GRYEE)
    return fail(COFFEE_E_INVALID, "solver variant %d is not available", variant);
  if (semantics != COFFEE_SEM_CPU_REF && semantics != COFFEE_SEM_GPU_REF)
    return fail(COFFEE_E_INVALID, "unknown semantics %d", semantics);
  if (variant == COFFEE_VARIANT_FLAT) {
    if (env->p.problem < 0 || env->p.problem > 2)
      return fail(COFFEE_E_CONFIG, "problem %d is not supported by the flat EZ solver",
                  env->p.problem);
    for (int a = 0; a < 3; ++a)
      if (env->p.guard[a] < env->p.shift_ghost + 3)
        return fail(COFFEE_E_CONFIG, "the flat EZ solver needs guard[%d] >= shift_ghost + 3",
                    a);
  } else {
    // the reference has these solvers only in its GPU build
    int rc = variant == COFFEE_VARIANT_GR      ? gr_check(env)
             : variant == COFFEE_VARIANT_YEE   ? yee_check(env)
             : variant == COFFEE_VARIANT_GRYEE ? gryee_check(env)
                                               : axisym_check(env, variant);
    if (rc) return rc;
  }
  COFFEE_CUDA_TRY(cudaSetDevice(env->device));
  coffee_solver* s = new (std::nothrow) coffee_solver();
  if (!s) return fail(COFFEE_E_NOMEM, "out of host memory");
  s->env = env;
  s->f = f;
  s->variant = variant;
  s->semantics = semantics;
  s->stream = static_cast<cudaStream_t>(stream);
  s->aux = 0;
  s->timing = 0;
  s->arith = COFFEE_ARITH_REFERENCE;
  s->taper_lanes = 0;
  s->energy_diag = 0;
  s->events_used = 0;
  s->synced_generation = 0;
  // the GR solver's inner absorbing region always needs the start-of-step
  // copy; the staggered solver's substeps read it
  bool abs_any = env->p.shift_ghost > 0 || variant == COFFEE_VARIANT_GR ||
                 variant == COFFEE_VARIANT_YEE || variant == COFFEE_VARIANT_GRYEE;
  for (int a = 0; a < 3; ++a) abs_any = abs_any || env->p.pml[a] > 0;
  s->absorbing = abs_any;
  const size_t bytes = f->n * f->elem;
  s->vtab = nullptr;
  auto cleanup = [&]() {
    for (int a = 0; a < 7; ++a) {
      if (s->B[a]) cudaFree(s->B[a]);
      if (s->dU[a]) cudaFree(s->dU[a]);
      if (s->Un[a]) cudaFree(s->Un[a]);
    }
    if (s->vtab) cudaFree(s->vtab);
    delete s;
  };
  for (int a = 0; a < 7; ++a) {
    cudaError_t err = cudaMalloc(&s->B[a], bytes);
    if (err == cudaSuccess) err = cudaMalloc(&s->dU[a], bytes);
    if (err == cudaSuccess) err = cudaMemset(s->dU[a], 0, bytes);
    if (err == cudaSuccess && abs_any) err = cudaMalloc(&s->Un[a], bytes);
    if (err == cudaSuccess && abs_any) err = cudaMemset(s->Un[a], 0, bytes);
    if (err != cudaSuccess) {
      cleanup();
      return fail(COFFEE_E_NOMEM, "solver scratch allocation failed: %s", cudaGetErrorString(err));
    }
  }
  int rc = variant == COFFEE_VARIANT_GR     ? gr_setup(env, f->elem, &s->vtab)
           : variant == COFFEE_VARIANT_YEE  ? COFFEE_OK
           : variant == COFFEE_VARIANT_GRYEE ? gryee_setup(env, f->elem, &s->vtab)
           : variant != COFFEE_VARIANT_FLAT ? axisym_setup(env, variant, f->elem, &s->vtab)
           : (f->elem == 4)               ? configure_solver<float>(s)
                                          : configure_solver<double>(s);
  if (rc) {
    cleanup();
    return rc;
  }
  s->partial_blocks = num_sms(env->device) * 4;
  cudaError_t err = cudaMalloc(&s->d_partials, sizeof(double) * s->partial_blocks);
  if (err == cudaSuccess) err = cudaMalloc(&s->d_count, sizeof(int));
  if (err == cudaSuccess) err = cudaEventCreate(&s->ev_begin);
  if (err == cudaSuccess) err = cudaEventCreate(&s->ev_end);
  if (err != cudaSuccess) {
    cleanup();
    return fail(COFFEE_E_NOMEM, "solver setup failed: %s", cudaGetErrorString(err));
  }
  env->users++;
  *out = s;
  return COFFEE_OK;
}

extern "C" int coffee_solver_destroy(coffee_solver* s) {
  if (!s) return COFFEE_OK;
  cudaSetDevice(s->env->device);
  cudaStreamSynchronize(s->stream);
  for (int a = 0; a < 7; ++a) {
    if (s->B[a]) cudaFree(s->B[a]);
    if (s->dU[a]) cudaFree(s->dU[a]);
    if (s->Un[a]) cudaFree(s->Un[a]);
  }
  if (s->vtab) cudaFree(s->vtab);
  for (auto e : s->events) cudaEventDestroy(e);
  cudaEventDestroy(s->ev_begin);
  cudaEventDestroy(s->ev_end);
  cudaFree(s->d_partials);
  cudaFree(s->d_count);
  (void)cudaGetLastError();  // leave no error of a release for the next call to find
  coffee_env* env = s->env;
  delete s;
  env_drop_user(env);
  return COFFEE_OK;
}

extern "C" int coffee_solver_set_aux(coffee_solver* s, int enable) {
  clear_error();
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_set_aux: null argument");
  if (enable && (s->variant == COFFEE_VARIANT_YEE || s->variant == COFFEE_VARIANT_GRYEE))
    return fail(COFFEE_E_INVALID, "the staggered solvers write no J, divE, divB");
  if (enable)
    for (int id = COFFEE_JX; id <= COFFEE_DIVB; ++id) {
      int rc = ensure_field(s->f, id);
      if (rc) return rc;
    }
  s->aux = enable ? 1 : 0;
  return COFFEE_OK;
}

extern "C" int coffee_solver_set_arithmetic(coffee_solver* s, int mode) {
  clear_error();
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_set_arithmetic: null argument");
  if (mode != COFFEE_ARITH_REFERENCE && mode != COFFEE_ARITH_FAST)
    return fail(COFFEE_E_INVALID, "unknown arithmetic mode %d", mode);
  if (s->variant != COFFEE_VARIANT_FLAT) {
    if (mode == COFFEE_ARITH_REFERENCE) return COFFEE_OK;
    return fail(COFFEE_E_INVALID, "only the flat EZ solver has a second arithmetic");
  }
  if (mode == s->arith) return COFFEE_OK;
  if (s->energy_diag && mode != COFFEE_ARITH_REFERENCE)
    return fail(COFFEE_E_INVALID, "the energy diagnostics need the reference arithmetic");
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  const int old = s->arith;
  s->arith = mode;
  const int rc = (s->f->elem == 4) ? configure_solver<float>(s) : configure_solver<double>(s);
  if (rc) {
    s->arith = old;  // keep the previous plan
    (void)((s->f->elem == 4) ? configure_solver<float>(s) : configure_solver<double>(s));
  }
  return rc;
}

extern "C" int coffee_solver_set_energy_diag(coffee_solver* s, int enable) {
  clear_error();
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_set_energy_diag: null argument");
  enable = enable ? 1 : 0;
  if (enable == s->energy_diag) return COFFEE_OK;
  if (enable && (s->variant != COFFEE_VARIANT_FLAT || s->semantics != COFFEE_SEM_CPU_REF ||
                 s->arith != COFFEE_ARITH_REFERENCE))
    return fail(COFFEE_E_INVALID,
                "the energy diagnostics are the CPU build's: flat solver, CPU semantics and "
                "the reference arithmetic only");
  if (enable)
    for (int id = COFFEE_DU_EGTB; id <= COFFEE_DU_KO_CUM; ++id) {
      int rc = ensure_field(s->f, id);
      if (rc) return rc;
    }
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  s->energy_diag = enable;
  const int rc = (s->f->elem == 4) ? configure_solver<float>(s) : configure_solver<double>(s);
  if (rc) {
    s->energy_diag = 1 - enable;
    (void)((s->f->elem == 4) ? configure_solver<float>(s) : configure_solver<double>(s));
  }
  return rc;
}

extern "C" int coffee_solver_set_taper_lanes(coffee_solver* s, int lanes) {
  clear_error();
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_set_taper_lanes: null argument");
  if (lanes < 0 || lanes > 64) return fail(COFFEE_E_INVALID, "taper lanes %d not in 0..64", lanes);
  if (s->variant != COFFEE_VARIANT_FLAT)
    return fail(COFFEE_E_INVALID, "only the flat EZ solver has the CPU build's taper");
  s->taper_lanes = lanes;
  return COFFEE_OK;
}

extern "C" int coffee_solver_set_timing(coffee_solver* s, int enable) {
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_set_timing: null argument");
  s->timing = enable ? 1 : 0;
  return COFFEE_OK;
}

extern "C" int coffee_solver_launches_per_step(coffee_solver* s) {
  if (s && s->variant == COFFEE_VARIANT_LOGSPH) return 12;  // + axis after each, + 1 per call
  if (s && s->variant == COFFEE_VARIANT_GR) return 6;       // + two E, H passes per call
  if (s && s->variant == COFFEE_VARIANT_YEE)
    // shell + update + clamp per substep; the star boundary adds its three
    // passes and the guard pass (the box problem: one guard pass per call)
    return s->env->p.problem == 1 ? 21 : 9;
  if (s && s->variant == COFFEE_VARIANT_GRYEE)
    // E, H + rho + shell + update + clamp per substep, and the cleaning
    return 15 + (s->env->p.clean_ep ? 1 : 0);
  return 6;  // 5 stage kernels + 1 KO kernel
}

static int next_event_pair(coffee_solver* s, int kind, cudaEvent_t* a, cudaEvent_t* b) {
  const size_t need = (size_t)(s->events_used + 1) * 2;
  while (s->events.size() < need) {
    cudaEvent_t e;
    COFFEE_CUDA_TRY(cudaEventCreate(&e));
    s->events.push_back(e);
  }
  if (s->event_kind.size() < (size_t)(s->events_used + 1)) s->event_kind.resize(s->events_used + 1);
  s->event_kind[s->events_used] = kind;
  *a = s->events[2 * s->events_used];
  *b = s->events[2 * s->events_used + 1];
  ++s->events_used;
  return COFFEE_OK;
}

// Timing mode: a pair of events around every launch.
struct EventHook : LaunchHook {
  coffee_solver* s;
  cudaEvent_t pending = nullptr;
  explicit EventHook(coffee_solver* sv) : s(sv) {}
  int before(int kind) override {
    cudaEvent_t a, b;
    int rc = next_event_pair(s, kind, &a, &b);
    if (rc) return rc;
    pending = b;
    COFFEE_CUDA_TRY(cudaEventRecord(a, s->stream));
    return COFFEE_OK;
  }
  int after(int) override {
    COFFEE_CUDA_TRY(cudaEventRecord(pending, s->stream));
    return COFFEE_OK;
  }
};

template <typename T>
static int run_steps(coffee_solver* s, double time, int nsteps) {
  EzConst<T> c;
  build_const<T>(s->env, s->semantics, &c);
  if (s->taper_lanes > 0) c.taper_lanes = s->taper_lanes;
  coffee_fields* f = s->f;
  cudaStream_t st = s->stream;
  const size_t bytes = f->n * f->elem;
  if (s->synced_generation != f->generation) {
    // the second buffer must carry the same guard values (non-periodic
    // guards are never written by the kernels)
    for (int a = 0; a < 7; ++a)
      COFFEE_CUDA_TRY(cudaMemcpyAsync(s->B[a], f->d[a], bytes, cudaMemcpyDeviceToDevice, st));
    s->synced_generation = f->generation;
  }
  F5<T> aux;
  for (int a = 0; a < 5; ++a) aux.p[a] = static_cast<T*>(f->d[COFFEE_JX + a]);
  s->events_used = 0;
  EventHook hook(s);
  if (s->timing) COFFEE_CUDA_TRY(cudaEventRecord(s->ev_begin, st));
  if (s->variant == COFFEE_VARIANT_GRYEE) {
    int rc = gryee_steps(s->env, f->elem, f->d, s->dU, s->Un, s->vtab, nsteps, st,
                         s->timing ? &hook : nullptr);
    if (rc) return rc;
    if (s->timing) COFFEE_CUDA_TRY(cudaEventRecord(s->ev_end, st));
    return COFFEE_OK;
  }
  if (s->variant == COFFEE_VARIANT_YEE) {
    void* b0[3] = {f->d[COFFEE_B0X], f->d[COFFEE_B0Y], f->d[COFFEE_B0Z]};
    const bool has_b0 = b0[0] && b0[1] && b0[2];
    int rc = yee_steps(s->env, f->elem, f->d, has_b0 ? b0 : nullptr, s->dU, s->Un, s->B, time,
                       nsteps, st, s->timing ? &hook : nullptr);
    if (rc) return rc;
    if (s->timing) COFFEE_CUDA_TRY(cudaEventRecord(s->ev_end, st));
    return COFFEE_OK;
  }
  if (s->variant != COFFEE_VARIANT_FLAT) {
    void* auxp[5];
    for (int a = 0; a < 5; ++a) auxp[a] = f->d[COFFEE_JX + a];
    LaunchHook* h = s->timing ? &hook : nullptr;
    int rc = s->variant == COFFEE_VARIANT_GR
                 ? gr_steps(s->env, f->elem, s->vtab, f->d, s->B, s->dU, s->Un,
                            s->aux ? auxp : nullptr, nsteps, st, h)
                 : axisym_steps(s->env, s->variant, f->elem, s->vtab, f->d, s->B, s->dU, s->Un,
                                s->aux ? auxp : nullptr, time, nsteps, st, h);
    if (rc) return rc;
    if (s->timing) COFFEE_CUDA_TRY(cudaEventRecord(s->ev_end, st));
    return COFFEE_OK;
  }
  F6<T> dg;
  for (int a = 0; a < 6; ++a) dg.p[a] = static_cast<T*>(f->d[COFFEE_DU_EGTB + a]);
  int rc = flat_steps<T>(c, s->launch, f7<T>(f->d), f7<T>(s->B), f7<T>(s->dU), f7<T>(s->Un), aux,
                         s->aux != 0, time, nsteps, st, s->timing ? &hook : nullptr,
                         s->energy_diag ? &dg : nullptr);
  if (rc) return rc;
  if (s->timing) COFFEE_CUDA_TRY(cudaEventRecord(s->ev_end, st));
  return COFFEE_OK;
}

extern "C" int coffee_solver_step(coffee_solver* s, double time, int nsteps) {
  clear_error();
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_step: null argument");
  if (nsteps < 0) return fail(COFFEE_E_INVALID, "nsteps must be >= 0");
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  return (s->f->elem == 4) ? run_steps<float>(s, time, nsteps) : run_steps<double>(s, time, nsteps);
}

// ------------------------------------------------------------------ batch

struct coffee_batch {
  std::vector<coffee_solver*> solvers;
  std::vector<SphRun> runs;
  SphBatchPlan plan;
  int elem;
  int device;
  cudaStream_t stream;
};

// COFFEE_BATCH_NO_TUNE=1 / COFFEE_BATCH_NO_GRAPH=1 in the environment keep
// the default tile shape / launch every kernel of every step (comparisons).
static bool env_flag(const char* name) {
  const char* v = std::getenv(name);
  return v != nullptr && v[0] == '1';
}

extern "C" int coffee_batch_create(coffee_solver* const* solvers, int n, void* stream,
                                   coffee_batch** out) {
  clear_error();
  if (!solvers || !out) return fail(COFFEE_E_INVALID, "coffee_batch_create: null argument");
  *out = nullptr;
  if (n < 1 || n > kMaxBatch)
    return fail(COFFEE_E_INVALID, "a batch holds 1 to %d runs (got %d)", kMaxBatch, n);
  for (int m = 0; m < n; ++m) {
    const coffee_solver* s = solvers[m];
    if (!s) return fail(COFFEE_E_INVALID, "solver %d is null", m);
    if (s->variant != COFFEE_VARIANT_LOGSPH)
      return fail(COFFEE_E_INVALID, "solver %d is not a log-spherical solver", m);
    if (s->f->elem != solvers[0]->f->elem || s->env->device != solvers[0]->env->device)
      return fail(COFFEE_E_INVALID, "solver %d differs in precision or device from solver 0", m);
  }
  COFFEE_CUDA_TRY(cudaSetDevice(solvers[0]->env->device));
  coffee_batch* b = new (std::nothrow) coffee_batch();
  if (!b) return fail(COFFEE_E_NOMEM, "out of host memory");
  b->solvers.assign(solvers, solvers + n);
  b->runs.resize(n);
  b->elem = solvers[0]->f->elem;
  b->device = solvers[0]->env->device;
  b->stream = static_cast<cudaStream_t>(stream);
  for (int m = 0; m < n; ++m) {
    coffee_solver* s = solvers[m];
    SphRun& r = b->runs[m];
    r.env = s->env;
    r.tab = s->vtab;
    for (int k = 0; k < 7; ++k) {
      r.A[k] = s->f->d[k];
      r.B[k] = s->B[k];
      r.dU[k] = s->dU[k];
      r.Un[k] = s->Un[k];
    }
    for (int k = 0; k < 5; ++k) r.aux[k] = s->f->d[COFFEE_JX + k];
    r.want_aux = s->aux;
  }
  int rc = sph_batch_plan(b->runs.data(), n, b->elem, !env_flag("COFFEE_BATCH_NO_TUNE"),
                          b->stream, &b->plan);
  if (rc) {
    sph_batch_free(&b->plan);
    delete b;
    return rc;
  }
  *out = b;
  return COFFEE_OK;
}

extern "C" int coffee_batch_info(coffee_batch* b, int* tile_x, int* tile_y, int* order,
                                 double* tuned_ms) {
  clear_error();
  if (!b) return fail(COFFEE_E_INVALID, "coffee_batch_info: null argument");
  if (tile_x) *tile_x = b->plan.tx;
  if (tile_y) *tile_y = b->plan.ty;
  if (order) *order = b->plan.order;
  if (tuned_ms) *tuned_ms = b->plan.tuned_ms;
  return COFFEE_OK;
}

extern "C" int coffee_batch_step(coffee_batch* b, double* times, int nsteps) {
  clear_error();
  if (!b || !times) return fail(COFFEE_E_INVALID, "coffee_batch_step: null argument");
  if (nsteps < 0) return fail(COFFEE_E_INVALID, "nsteps must be >= 0");
  COFFEE_CUDA_TRY(cudaSetDevice(b->device));
  for (coffee_solver* s : b->solvers) {
    coffee_fields* f = s->f;
    if (s->synced_generation != f->generation) {
      // the second buffer carries the same guard values
      for (int a = 0; a < 7; ++a)
        COFFEE_CUDA_TRY(cudaMemcpyAsync(s->B[a], f->d[a], f->n * f->elem,
                                        cudaMemcpyDeviceToDevice, b->stream));
      s->synced_generation = f->generation;
    }
  }
  return sph_batch_run(&b->plan, b->runs.data(), times, nsteps, !env_flag("COFFEE_BATCH_NO_GRAPH"),
                       b->stream);
}

extern "C" int coffee_batch_set_persistent(coffee_batch* b, int on) {
  clear_error();
  if (!b) return fail(COFFEE_E_INVALID, "coffee_batch_set_persistent: null argument");
  COFFEE_CUDA_TRY(cudaSetDevice(b->device));
  return sph_batch_set_persistent(&b->plan, on != 0);
}

extern "C" int coffee_batch_set_wait_limit(coffee_batch* b, long long limit_ns, int stall_block) {
  clear_error();
  if (!b) return fail(COFFEE_E_INVALID, "coffee_batch_set_wait_limit: null argument");
  if (limit_ns <= 0) return fail(COFFEE_E_INVALID, "the wait limit must be > 0 ns");
  if (stall_block < -1) return fail(COFFEE_E_INVALID, "stall_block must be >= -1");
  b->plan.wait_ns = limit_ns;
  b->plan.stall_block = stall_block;
  return COFFEE_OK;
}

extern "C" int coffee_batch_destroy(coffee_batch* b) {
  if (!b) return COFFEE_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  sph_batch_free(&b->plan);
  delete b;
  return COFFEE_OK;
}

extern "C" int coffee_solver_last_timing(coffee_solver* s, double ms[3], int launches[3],
                                         double* total_ms) {
  clear_error();
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_last_timing: null argument");
  if (!s->timing) return fail(COFFEE_E_INVALID, "timing is off (coffee_solver_set_timing)");
  COFFEE_CUDA_TRY(cudaEventSynchronize(s->ev_end));
  double sum[3] = {0, 0, 0};
  int cnt[3] = {0, 0, 0};
  for (int q = 0; q < s->events_used; ++q) {
    float t = 0;
    COFFEE_CUDA_TRY(cudaEventElapsedTime(&t, s->events[2 * q], s->events[2 * q + 1]));
    sum[s->event_kind[q]] += t;
    cnt[s->event_kind[q]] += 1;
  }
  float tot = 0;
  COFFEE_CUDA_TRY(cudaEventElapsedTime(&tot, s->ev_begin, s->ev_end));
  for (int k = 0; k < 3; ++k) {
    if (ms) ms[k] = sum[k];
    if (launches) launches[k] = cnt[k];
  }
  if (total_ms) *total_ms = tot;
  return COFFEE_OK;
}

template <typename T>
static int diag_t(coffee_solver* s, int what, double* out) {
  EzConst<T> c;
  build_const<T>(s->env, s->semantics, &c);
  const coffee_params& p = s->env->p;
  T xl[3], xh[3];
  for (int a = 0; a < 3; ++a) {
    // region of total_energy (field_solver_EZ.cu:759-770)
    xh[a] = (T)p.lower[a] + (T)p.size[a] - (T)p.pml[a] * c.delta[a];
    xl[a] = (T)p.lower[a] + (T)p.pml[a] * c.delta[a];
  }
  const int stag = (s->variant == COFFEE_VARIANT_YEE || s->variant == COFFEE_VARIANT_GRYEE) ? 1 : 0;
  diag_kernel<T><<<s->partial_blocks, 256, 0, s->stream>>>(c, f7c<T>(s->f->d), what, xl[0],
                                                           xl[1], xl[2], xh[0], xh[1], xh[2],
                                                           stag, s->d_partials);
  COFFEE_CUDA_TRY(cudaGetLastError());
  std::vector<double> h(s->partial_blocks);
  COFFEE_CUDA_TRY(cudaMemcpyAsync(h.data(), s->d_partials, sizeof(double) * h.size(),
                                  cudaMemcpyDeviceToHost, s->stream));
  COFFEE_CUDA_TRY(cudaStreamSynchronize(s->stream));
  const bool is_max = (what == COFFEE_DIAG_MAX_EDOTB || what == COFFEE_DIAG_MAX_EOVERB);
  double acc = 0;
  for (double v : h) acc = is_max ? std::max(acc, v) : acc + v;
  if (what == COFFEE_DIAG_DIVB_L2) acc = std::sqrt(acc);
  *out = acc;
  return COFFEE_OK;
}

extern "C" int coffee_diag_reduce(coffee_solver* s, int what, double* out) {
  clear_error();
  if (!s || !out) return fail(COFFEE_E_INVALID, "coffee_diag_reduce: null argument");
  if (what < COFFEE_DIAG_ENERGY_E || what > COFFEE_DIAG_MAX_EOVERB)
    return fail(COFFEE_E_INVALID, "unknown diagnostic %d", what);
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  return (s->f->elem == 4) ? diag_t<float>(s, what, out) : diag_t<double>(s, what, out);
}

template <typename T>
static int luminosity_t(coffee_solver* s, double r, double* out) {
  EzConst<T> c;
  build_const<T>(s->env, s->semantics, &c);
  const coffee_params& p = s->env->p;
  double lo[3], d[3];
  for (int a = 0; a < 3; ++a) {
    d[a] = p.size[a] / p.N[a];
    lo[a] = p.lower[a];  // coordinate of the first interior point (grid.h:116-134)
  }
  const double h = std::max(d[0], std::max(d[1], d[2]));
  luminosity_kernel<T><<<s->partial_blocks, 256, 0, s->stream>>>(
      c, f7c<T>(s->f->d), lo[0], lo[1], lo[2], d[0], d[1], d[2], r, h, s->d_partials);
  COFFEE_CUDA_TRY(cudaGetLastError());
  std::vector<double> hbuf(s->partial_blocks);
  COFFEE_CUDA_TRY(cudaMemcpyAsync(hbuf.data(), s->d_partials, sizeof(double) * hbuf.size(),
                                  cudaMemcpyDeviceToHost, s->stream));
  COFFEE_CUDA_TRY(cudaStreamSynchronize(s->stream));
  double acc = 0;
  for (double v : hbuf) acc += v;  // fixed order: deterministic
  *out = acc;
  return COFFEE_OK;
}

extern "C" int coffee_diag_luminosity(coffee_solver* s, double r, double* out) {
  clear_error();
  if (!s || !out) return fail(COFFEE_E_INVALID, "coffee_diag_luminosity: null argument");
  if (s->variant != COFFEE_VARIANT_FLAT)
    return fail(COFFEE_E_INVALID, "the Poynting luminosity is defined for the flat solver");
  if (!(r > 0)) return fail(COFFEE_E_INVALID, "the sphere radius must be > 0 (got %g)", r);
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  return (s->f->elem == 4) ? luminosity_t<float>(s, r, out) : luminosity_t<double>(s, r, out);
}

extern "C" int coffee_solver_check_finite(coffee_solver* s) {
  clear_error();
  if (!s) return fail(COFFEE_E_INVALID, "coffee_solver_check_finite: null argument");
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  COFFEE_CUDA_TRY(cudaMemsetAsync(s->d_count, 0, sizeof(int), s->stream));
  const long long n = (long long)s->f->n;
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)s->partial_blocks * 8);
  if (s->f->elem == 4)
    count_nonfinite_kernel<float><<<blocks, 256, 0, s->stream>>>(f7c<float>(s->f->d), n, s->d_count);
  else
    count_nonfinite_kernel<double><<<blocks, 256, 0, s->stream>>>(f7c<double>(s->f->d), n, s->d_count);
  COFFEE_CUDA_TRY(cudaGetLastError());
  int h = 0;
  COFFEE_CUDA_TRY(cudaMemcpyAsync(&h, s->d_count, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  COFFEE_CUDA_TRY(cudaStreamSynchronize(s->stream));
  if (h != 0) return fail(COFFEE_E_NONFINITE, "%d field values are NaN or Inf", h);
  return COFFEE_OK;
}

// ------------------------------------------------------------- snapshots

extern "C" int coffee_solver_save_snapshot(coffee_solver* s, const char* path, double time,
                                           int64_t step) {
  clear_error();
  if (!s || !path) return fail(COFFEE_E_INVALID, "coffee_solver_save_snapshot: null argument");
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  COFFEE_CUDA_TRY(cudaStreamSynchronize(s->stream));
  coffee_fields* f = s->f;
  const size_t bytes = f->n * f->elem;
  std::vector<char> host;
  try {
    host.resize(bytes * 7);
  } catch (...) {
    return fail(COFFEE_E_NOMEM, "snapshot: cannot allocate %zu host bytes", bytes * 7);
  }
  for (int a = 0; a < 7; ++a)
    COFFEE_CUDA_TRY(cudaMemcpy(host.data() + a * bytes, f->d[a], bytes, cudaMemcpyDeviceToHost));
  fld_header h;
  fld_header_init(&h, f->elem, 7, s->env->grid.dims, s->env->grid.guard);
  h.time = time;
  h.step = step;
  const void* arrays[7];
  for (int a = 0; a < 7; ++a) arrays[a] = host.data() + a * bytes;
  if (!fld_write(path, &h, arrays, f->n)) return fail(COFFEE_E_IO, "cannot write %s", path);
  return COFFEE_OK;
}

extern "C" int coffee_solver_load_snapshot(coffee_solver* s, const char* path, double* time,
                                           int64_t* step) {
  clear_error();
  if (!s || !path) return fail(COFFEE_E_INVALID, "coffee_solver_load_snapshot: null argument");
  fld_header h;
  std::vector<char> payload;
  if (!fld_read(path, &h, &payload)) return fail(COFFEE_E_IO, "cannot read %s", path);
  coffee_fields* f = s->f;
  for (int a = 0; a < 3; ++a)
    if (h.dims[a] != s->env->grid.dims[a])
      return fail(COFFEE_E_IO, "%s: dims do not match the grid", path);
  if (h.elem_size != f->elem || h.nfields < 7)
    return fail(COFFEE_E_IO, "%s: precision or field count does not match", path);
  const size_t bytes = f->n * f->elem;
  if (h.crc32 != 0) {
    uint32_t crc = fld_crc32_update(0, payload.data(), bytes * (size_t)h.nfields);
    if (crc != h.crc32) return fail(COFFEE_E_IO, "%s: CRC mismatch", path);
  }
  COFFEE_CUDA_TRY(cudaSetDevice(s->env->device));
  COFFEE_CUDA_TRY(cudaStreamSynchronize(s->stream));
  for (int a = 0; a < 7; ++a)
    COFFEE_CUDA_TRY(cudaMemcpy(f->d[a], payload.data() + a * bytes, bytes, cudaMemcpyHostToDevice));
  ++f->generation;
  if (time) *time = h.time;
  if (step) *step = h.step;
  return COFFEE_OK;
}
