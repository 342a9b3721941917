// Single-rank test double for the reference's Coffee::sim_environment.
//
// Test infrastructure for the oracle only: it lets the reference's own CPU
// solver translation units (src/algorithms/field_solver_EZ.cpp and friends,
// compiled unmodified from the reference tree) run in one process without
// MPI.  It supplies the three members those units need at link time:
//
//  * the constructor.  Like src/sim_env_impl.hpp:12-86 it parses the TOML
//    config with the reference's own parse_config (src/sim_params.cpp:7-146)
//    and lays out the grid the same way (dims = N + 2*guard,
//    delta = size / N, inv_delta = 1 / delta; sim_env_impl.hpp:52-60).  The
//    config path is $COFFEE_ORACLE_CONFIG, default "config.toml" in the
//    working directory (the reference hard-codes the latter).
//  * the destructor (no MPI_Finalize: there is no MPI).
//  * send_guard_cells.  With one rank, the reference's halo exchange
//    (sim_env_impl.hpp:179-228, src/sim_env.cpp:42-115) reduces to a
//    periodic copy of the 3-deep faces of E, B and P in each periodic
//    direction, x first, then y (whole x extent, guards included), then z
//    (whole xy planes).  Non-periodic directions are left untouched.
#include <cstdlib>
#include <cstring>
#include <string>

#include "data/sim_data.h"
#include "sim_env.h"

namespace Coffee {

namespace {

// Copy the periodic images of the guard slabs of one array along `dir`.
// Destination [dims-g, dims) receives source [g, 2g); destination [0, g)
// receives source [dims-2g, dims-g).  Every other index runs over the full
// extent, so slabs copied along an earlier direction carry their guards.
void periodic_fill(Scalar* a, const Grid& grid, int dir) {
  const int d0 = grid.dims[0], d1 = grid.dims[1], d2 = grid.dims[2];
  const int g = grid.guard[dir];
  const int n = grid.dims[dir] - 2 * g;
  if (g == 0 || n <= 0) return;
  const size_t stride[3] = {1, (size_t)d0, (size_t)d0 * d1};
  const int ext[3] = {d0, d1, d2};
  // the two directions that are not `dir`
  const int a1 = (dir == 0) ? 1 : 0;
  const int a2 = (dir == 2) ? 1 : 2;
  for (int q = 0; q < ext[a2]; ++q)
    for (int p = 0; p < ext[a1]; ++p) {
      const size_t base = p * stride[a1] + q * stride[a2];
      for (int s = 0; s < g; ++s) {
        // upper guard from the first interior slab
        a[base + (size_t)(n + g + s) * stride[dir]] =
            a[base + (size_t)(g + s) * stride[dir]];
        // lower guard from the last interior slab
        a[base + (size_t)s * stride[dir]] =
            a[base + (size_t)(n + s) * stride[dir]];
      }
    }
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
}

sim_environment::~sim_environment() {}

void sim_environment::send_guard_cells(sim_data& data) {
  Scalar* arrays[7] = {data.E.host_ptr(0), data.E.host_ptr(1),
                       data.E.host_ptr(2), data.B.host_ptr(0),
                       data.B.host_ptr(1), data.B.host_ptr(2),
                       data.P.host_ptr()};
  for (int dir = 0; dir < 3; ++dir) {
    if (!m_is_periodic[dir]) continue;
    for (auto* a : arrays) periodic_fill(a, m_grid, dir);
  }
}

void sim_environment::send_guard_cell_array(multi_array<Scalar>& array) {
  for (int dir = 0; dir < 3; ++dir)
    if (m_is_periodic[dir]) periodic_fill(array.host_ptr(), m_grid, dir);
}

}  // namespace Coffee
