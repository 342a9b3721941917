// Single-rank test double of Coffee::sim_environment for the reference's GPU
// solvers (test infrastructure only; see oracle/Makefile target gpuref).
//
// As the reference's GPU environment (src/cuda/sim_env.cpp:250-268) it copies
// the parameters and grid to the reference's __constant__ dev_params and
// dev_grid (src/cuda/constant_mem.cu).  The config is parsed with the
// reference's parse_config from $COFFEE_ORACLE_CONFIG (default
// ./config.toml), the grid laid out as src/sim_env_impl.hpp:52-60, and
// send_guard_cells is the single-rank periodic fill of E, B, P on the device
// in the x -> y -> z order of the reference's exchange; non-periodic axes are
// left alone.
#include <cstdlib>
#include <cstring>
#include <string>

#include "sim_env.h"
#include "data/sim_data.h"
#include "cuda/constant_mem_func.h"

int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op,
               int, MPI_Comm) {
  std::memcpy(recvbuf, sendbuf, (size_t)count * (type == 8 ? 8 : sizeof(Coffee::Scalar)));
  return 0;
}

namespace Coffee {

namespace {

// Periodic copy of the guard slabs along `dir` for one device array: index
// (p, q) runs over the two other axes, s over the guard depth.
__global__ void periodic_fill_kernel(Scalar* a, int d0, int d1, int d2, int dir, int g) {
  const int ext[3] = {d0, d1, d2};
  const long long stride[3] = {1, d0, (long long)d0 * d1};
  const int a1 = (dir == 0) ? 1 : 0, a2 = (dir == 2) ? 1 : 2;
  const int n = ext[dir] - 2 * g;
  const long long total = (long long)ext[a1] * ext[a2] * g;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t % g);
    const int p = (int)((t / g) % ext[a1]);
    const int q = (int)(t / ((long long)g * ext[a1]));
    const long long base = p * stride[a1] + q * stride[a2];
    a[base + (long long)(n + g + s) * stride[dir]] = a[base + (long long)(g + s) * stride[dir]];
    a[base + (long long)s * stride[dir]] = a[base + (long long)(n + s) * stride[dir]];
  }
}

void periodic_fill(Scalar* a, const Grid& grid, int dir) {
  const int g = grid.guard[dir];
  if (g == 0 || grid.dims[dir] - 2 * g <= 0) return;
  periodic_fill_kernel<<<256, 256>>>(a, grid.dims[0], grid.dims[1], grid.dims[2], dir, g);
}

}  // namespace

sim_environment::sim_environment(int* argc, char*** argv) {
  (void)argc;
  (void)argv;
  const char* cfg = std::getenv("COFFEE_ORACLE_CONFIG");
  m_params = parse_config(cfg ? std::string(cfg) : std::string("config.toml"));
  for (int i = 0; i < 3; i++) {
    m_grid.guard[i] = m_params.guard[i];
    m_grid.sizes[i] = m_params.size[i];
    m_grid.lower[i] = m_params.lower[i];
    m_grid.dims[i] = m_params.N[i] + 2 * m_params.guard[i];
    m_grid.delta[i] = m_params.size[i] / m_params.N[i];
    m_grid.inv_delta[i] = 1.0 / m_grid.delta[i];
    m_grid.offset[i] = 0;
    m_is_periodic[i] = m_params.periodic_boundary[i];
    m_mpi_dims[i] = 1;
    m_mpi_coord[i] = 0;
    m_neighbor_left[i] = m_is_periodic[i] ? 0 : NEIGHBOR_NULL;
    m_neighbor_right[i] = m_is_periodic[i] ? 0 : NEIGHBOR_NULL;
    m_is_boundary[2 * i] = !m_is_periodic[i];
    m_is_boundary[2 * i + 1] = !m_is_periodic[i];
  }
  m_size = 1;
  m_rank = 0;
  m_dev_id = 0;
  cudaSetDevice(0);
  init_dev_params(m_params);
  init_dev_grid(m_grid);
}

sim_environment::~sim_environment() {}

void sim_environment::send_guard_cells(sim_data& data) {
  Scalar* arrays[7] = {data.E.dev_ptr(0), data.E.dev_ptr(1), data.E.dev_ptr(2),
                       data.B.dev_ptr(0), data.B.dev_ptr(1), data.B.dev_ptr(2),
                       data.P.dev_ptr()};
  for (int dir = 0; dir < 3; ++dir) {
    if (!m_is_periodic[dir]) continue;
    for (auto* a : arrays) periodic_fill(a, m_grid, dir);
  }
  cudaDeviceSynchronize();
}

void sim_environment::send_guard_cell_array(multi_array<Scalar>& array) {
  for (int dir = 0; dir < 3; ++dir)
    if (m_is_periodic[dir]) periodic_fill(array.dev_ptr(), m_grid, dir);
  cudaDeviceSynchronize();
}

}  // namespace Coffee
