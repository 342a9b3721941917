// Driver for the reference's own GPU EZ solvers (test infrastructure only).
//
// Usage:  coffee_refgpu_{float,double} SOLVER IN.fld OUT.fld NSTEPS [--aux] [--warmup W]
//
//   SOLVER  ez   field_solver_EZ            (src/algorithms/field_solver_EZ.cu)
//           sph  field_solver_EZ_spherical  (src/algorithms/field_solver_EZ_spherical.cu)
//           cyl  field_solver_EZ_cylindrical(src/algorithms/field_solver_EZ_cylindrical.cu)
//           gr   field_solver_gr_EZ         (src/algorithms/field_solver_gr_EZ.cu)
//           yee  field_solver               (src/algorithms/field_solver.cu), the
//                staggered RK3 solver; keeps sim_data's Yee staggering
//                (src/data/sim_data.cpp:19-25) and, when IN.fld holds 10
//                arrays, loads arrays 7-9 as the background field B0
//           gryee field_solver_gr           (src/algorithms/field_solver_gr.cu), the
//                staggered solver in Kerr-Schild coordinates
//                (evolve_fields_gr(); Yee staggering; E holds D)
//
// The config is read by the reference's parse_config through the single-rank
// environment double (ref_gpu_env.cu), which also fills the reference's
// __constant__ dev_params / dev_grid.  IN.fld holds E, B, P with guard cells
// in the reference layout (i fastest).  The driver:
//   1. builds sim_data, sets the collocated stagger 0b111 as the reference's
//      user files do (src/user_pulsar_sph.hpp:6-9, src/user_wald2.hpp:7-11),
//      except for yee;
//   2. constructs the solver (before the data is loaded, as the reference's
//      drivers do: src/main-pulsar2d-spherical.cpp:25-27);
//   3. loads E, B, P to the host arrays and copies them to the device; the
//      cylindrical solver evolves its own P (field_solver_EZ_cylindrical.h:10),
//      so IN's P is copied there too;
//   4. calls evolve_fields NSTEPS times, advancing time by dt in Scalar as
//      src/main-pulsar2d-spherical.cpp:87-89;
//   5. writes E, B, P (the solver's own P for cyl; with --aux also the
//      B0 arrays, divE and divB of sim_data) to OUT.fld;
//   6. prints one JSON line with the time of step 4 (the reference synchronises
//      the device inside every evolve_fields call).
#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "algorithms/field_solver_EZ.h"
#include "algorithms/field_solver_EZ_cylindrical.h"
#include "algorithms/field_solver_EZ_spherical.h"
#include "algorithms/field_solver_gr_EZ.h"
#include "algorithms/field_solver.h"
#include "algorithms/field_solver_gr.h"
#include "coffee_fld.h"
#include "data/sim_data.h"
#include "sim_env.h"

using namespace Coffee;

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s ez|sph|cyl|gr|yee|gryee IN.fld OUT.fld NSTEPS [--aux] [--warmup W]\n",
                 argv[0]);
    return 2;
  }
  const std::string solver_name = argv[1], in_path = argv[2], out_path = argv[3];
  const long nsteps = std::atol(argv[4]);
  bool aux = false;
  long warmup = 0;
  for (int a = 5; a < argc; ++a) {
    const std::string opt = argv[a];
    if (opt == "--aux") aux = true;
    else if (opt == "--warmup" && a + 1 < argc) warmup = std::atol(argv[++a]);
    else {
      std::fprintf(stderr, "unknown option %s\n", opt.c_str());
      return 2;
    }
  }
  if (solver_name != "ez" && solver_name != "sph" && solver_name != "cyl" && solver_name != "gr" &&
      solver_name != "yee" && solver_name != "gryee") {
    std::fprintf(stderr, "unknown solver %s\n", solver_name.c_str());
    return 2;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    std::fprintf(stderr, "no CUDA device\n");
    return 6;
  }

  fld_header hin;
  std::vector<char> payload;
  if (!fld_read(in_path.c_str(), &hin, &payload)) {
    std::fprintf(stderr, "cannot read %s\n", in_path.c_str());
    return 3;
  }

  sim_environment env(nullptr, nullptr);
  const Grid& grid = env.grid();
  const size_t n = (size_t)grid.dims[0] * grid.dims[1] * grid.dims[2];
  if (hin.elem_size != (int)sizeof(Scalar) || hin.nfields < 7 ||
      hin.dims[0] != grid.dims[0] || hin.dims[1] != grid.dims[1] ||
      hin.dims[2] != grid.dims[2]) {
    std::fprintf(stderr,
                 "input mismatch: elem %d (want %d), dims %d %d %d (want %d %d %d)\n",
                 hin.elem_size, (int)sizeof(Scalar), hin.dims[0], hin.dims[1],
                 hin.dims[2], grid.dims[0], grid.dims[1], grid.dims[2]);
    return 4;
  }

  sim_data data(env);
  const bool staggered = solver_name == "yee" || solver_name == "gryee";
  if (!staggered) {
    Stagger st[3] = {Stagger(0b111), Stagger(0b111), Stagger(0b111)};
    data.E.set_stagger(st);
    data.B.set_stagger(st);
    data.B0.set_stagger(st);
  }

  // Silence the reference's own prints (block sizes, per-phase timers).
  std::fflush(stdout);
  const int saved_stdout = dup(1);
  const int devnull = open("/dev/null", O_WRONLY);
  dup2(devnull, 1);

  std::unique_ptr<field_solver_EZ> s_ez;
  std::unique_ptr<field_solver_EZ_spherical> s_sph;
  std::unique_ptr<field_solver_EZ_cylindrical> s_cyl;
  std::unique_ptr<field_solver_gr_EZ> s_gr;
  std::unique_ptr<field_solver> s_yee;
  std::unique_ptr<field_solver_gr> s_gryee;
  std::function<void(Scalar)> evolve;
  if (solver_name == "ez") {
    s_ez.reset(new field_solver_EZ(data, env));
    evolve = [&](Scalar t) { s_ez->evolve_fields(t); };
  } else if (solver_name == "sph") {
    s_sph.reset(new field_solver_EZ_spherical(data, env));
    evolve = [&](Scalar t) { s_sph->evolve_fields(t); };
  } else if (solver_name == "cyl") {
    s_cyl.reset(new field_solver_EZ_cylindrical(data, env));
    evolve = [&](Scalar t) { s_cyl->evolve_fields(t); };
  } else if (solver_name == "gr") {
    s_gr.reset(new field_solver_gr_EZ(data, env));
    evolve = [&](Scalar t) { s_gr->evolve_fields(t); };
  } else if (solver_name == "yee") {
    s_yee.reset(new field_solver(data, env));
    evolve = [&](Scalar t) { s_yee->evolve_fields(t); };
  } else {
    s_gryee.reset(new field_solver_gr(data, env));
    evolve = [&](Scalar) { s_gryee->evolve_fields_gr(); };
  }

  Scalar* dst[7] = {data.E.host_ptr(0), data.E.host_ptr(1), data.E.host_ptr(2),
                    data.B.host_ptr(0), data.B.host_ptr(1), data.B.host_ptr(2),
                    data.P.host_ptr()};
  for (int f = 0; f < 7; ++f)
    std::memcpy(dst[f], payload.data() + f * n * sizeof(Scalar), n * sizeof(Scalar));
  {
    // B0 as the user files leave it (data.B0.initialize(): zero), or
    // arrays 7-9 of IN.fld for the staggered solver
    Scalar* b0[3] = {data.B0.host_ptr(0), data.B0.host_ptr(1), data.B0.host_ptr(2)};
    for (int f = 0; f < 3; ++f) {
      if (solver_name == "yee" && hin.nfields >= 10)
        std::memcpy(b0[f], payload.data() + (7 + f) * n * sizeof(Scalar), n * sizeof(Scalar));
      else
        std::memset(b0[f], 0, n * sizeof(Scalar));
    }
    // divE holds the staggered GR solver's rho, which it writes only inside
    // the update box and reads one point beyond it: start it at zero
    std::memset(data.divE.host_ptr(), 0, n * sizeof(Scalar));
    std::memset(data.divB.host_ptr(), 0, n * sizeof(Scalar));
  }
  payload.clear();
  payload.shrink_to_fit();
  data.sync_to_device();
  multi_array<Scalar>* Pout = &data.P;
  if (s_cyl) {
    cudaMemcpy(s_cyl->P.dev_ptr(), data.P.dev_ptr(), n * sizeof(Scalar),
               cudaMemcpyDeviceToDevice);
    Pout = &s_cyl->P;
  }
  cudaDeviceSynchronize();

  Scalar time = (Scalar)hin.time;
  for (long s = 0; s < warmup; ++s) {
    evolve(time);
    time += env.params().dt;
  }
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  for (long s = 0; s < nsteps; ++s) {
    evolve(time);
    time += env.params().dt;
  }
  cudaDeviceSynchronize();
  const auto t1 = std::chrono::steady_clock::now();
  const cudaError_t err = cudaGetLastError();

  std::fflush(stdout);
  dup2(saved_stdout, 1);
  close(devnull);
  close(saved_stdout);
  if (err != cudaSuccess) {
    std::fprintf(stderr, "CUDA error after evolve_fields: %s\n", cudaGetErrorString(err));
    return 7;
  }

  data.E.sync_to_host();
  data.B.sync_to_host();
  Pout->sync_to_host();
  std::vector<const Scalar*> out = {
      data.E.host_ptr(0), data.E.host_ptr(1), data.E.host_ptr(2),
      data.B.host_ptr(0), data.B.host_ptr(1), data.B.host_ptr(2),
      Pout->host_ptr()};
  if (aux) {
    data.B0.sync_to_host();
    data.divE.sync_to_host();
    data.divB.sync_to_host();
    out.push_back(data.B0.host_ptr(0));
    out.push_back(data.B0.host_ptr(1));
    out.push_back(data.B0.host_ptr(2));
    out.push_back(data.divE.host_ptr());
    out.push_back(data.divB.host_ptr());
  }
  fld_header hout = hin;
  hout.nfields = (int)out.size();
  hout.time = time;
  hout.step = hin.step + warmup + nsteps;
  if (!fld_write(out_path.c_str(), &hout, (const void* const*)out.data(), n)) {
    std::fprintf(stderr, "cannot write %s\n", out_path.c_str());
    return 5;
  }
  const double secs = std::chrono::duration<double>(t1 - t0).count();
  long long interior = 1;
  for (int a = 0; a < 3; ++a) interior *= (long long)(grid.dims[a] - 2 * grid.guard[a]);
  std::printf(
      "{\"impl\": \"reference-gpu\", \"solver\": \"%s\", \"scalar_bytes\": %d, \"steps\": %ld, "
      "\"seconds\": %.6f, \"interior_cells\": %lld, \"cell_updates_per_s\": %.6e}\n",
      solver_name.c_str(), (int)sizeof(Scalar), nsteps, secs, interior,
      secs > 0 ? (double)interior * nsteps / secs : 0.0);
  return 0;
}
